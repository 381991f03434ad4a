// soup_common.cuh -- device-side types and pair physics shared by the soup kernels (sm_100a).
//
// Physics follows the reference's WGSL: engine/wgsl/forces.wgsl:17-37 (wca_dv, fene_dv, bend_dv,
// attr_dv), soup/wgsl/pair.wgsl:64-204 (mi3, pairB, class table, acidSoapScale, nonbondedSoup),
// soup/wgsl/electrostatics.wgsl:65-99 (screened Coulomb with the shifted-force constant).
//
// Two arithmetic paths:
//  * EXACT helpers (ex_*) use round-to-nearest intrinsics with no FMA contraction, in the
//    reference's operation order.  They decide set membership (Verlet/head lists, bond contact
//    tests) so that those sets are bit-identical to the CPU oracle's.
//  * FAST helpers evaluate the force with FMA, rsqrt and the SFU (accuracy bar: 1e-5 relative RMS
//    against FP64).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define SOUP_NONE_U32 0xFFFFFFFFu
#define SOUP_KMAX 8
#define SOUP_RMAX 4
#define SOUP_CAND_CAP 6   // soup/wgsl/bond-dispatch.wgsl:12 CANDIDATE_CAP

namespace soup {

// Per-system parameters (one entry per replica; a single system is a batch of one).
struct SysParams {
  float box[3], inv_box[3];
  float list_range;          // VL.x
  float es_A, es_kappa, es_rc, es_fc, es_split, es_list_range;
  float wall_r, wall_k;
  float kT, gamma, dt, hdt, gdt, sigma_v;
  float acid;                // AttrScale.pair.x
  float skin_half2;          // (skin/2)^2 for the drift trigger
  int dims[3];               // list-build grid
  uint32_t cell_off;         // first global cell of this system
  int walk;                  // list-build walk radius (cells)
  uint32_t slot_off, n;      // slot range of this system
  uint32_t head_off, nheads; // head range (ES heads)
  int hdims[3];              // head grid
  int hwalk;                 // head-grid walk radius (cells)
  uint32_t hcell_off;
  uint32_t list_cap, es_cap; // capacities (overflow threshold)
  uint32_t es_on;            // electrostatics enabled
  int32_t charged_kind;
  // FP64 host-style numbers for the constant-pH sweep
  double d_box[3], d_inv_box[3];
  double d_A, d_kappa, d_rc, d_shiftU, d_shiftF, d_pka, d_ph, d_kT, d_q;
  double d_acid, d_rcattr, d_wc, d_eps;
};

// Batch-wide constants (identical data/soup.json and data/params.json for every replica).
struct PairConst {
  float wcut2;   // (c6 * b)^2 for WCA
  float wcut;    // c6 * b
  float b2;      // b^2
  float attr;    // class-table depth
};
struct Shared {
  PairConst pair[SOUP_KMAX * SOUP_KMAX];
  float radius[SOUP_KMAX];
  uint32_t cls[SOUP_KMAX];
  float sigma, eps, b_tt, k_fene, r_inf, k_bend, r_bend, wc, c6;
  float rc_attr;             // c6 * b_tt (f32)
  float attr_k;              // pi / (2 wc) (fast path)
  float attr_amp;            // eps * pi / (2 wc) (fast path)
  float rmax2;               // max squared pair reach of any nonbonded term (fast path skip)
  // bond rules (soup/wgsl/bond-common.wgsl:54-80 BondParams)
  float kindA[SOUP_RMAX], kindB[SOUP_RMAX];
  float att_form[SOUP_RMAX], att_break[SOUP_RMAX], acc_form[SOUP_RMAX], acc_break[SOUP_RMAX];
  float req_cat[SOUP_RMAX], roleA[SOUP_RMAX], roleB[SOUP_RMAX];
  float cat_kind, head_terminal, head_cap, max_hold, interval;
  uint32_t n_kinds;
};

#ifdef __CUDACC__
// ---------------------------------------------------------------------------------------------
// RNG: soup/wgsl/step.wgsl:18-23 pcgSoup / uniform01Soup (== bond-common.wgsl bondPcg)
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t pcg_hash(uint32_t v) {
  uint32_t state = v * 747796405u + 2891336453u;
  uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
  return (word >> 22u) ^ word;
}
__device__ __forceinline__ float u01(uint32_t v) { return __fdiv_rn(__uint2float_rn(v), 4294967296.0f); }

// soup/src/electrostatics.ts:308-315 pcgNext (LCG state, hashed output, as double)
__device__ __forceinline__ double pcg_next(uint32_t& s) {
  uint32_t v = s * 747796405u + 2891336453u;
  s = v;
  v = ((v >> ((v >> 28u) + 4u)) ^ v) * 277803737u;
  v = (v >> 22u) ^ v;
  return (double)v / 4294967296.0;
}

// ---------------------------------------------------------------------------------------------
// Exact f32 helpers (no contraction)
// ---------------------------------------------------------------------------------------------
// soup/wgsl/pair.wgsl:64-66 mi3: d - round(d / box) * box, round = half to even
__device__ __forceinline__ float ex_mi(float d, float L) {
  return __fsub_rn(d, __fmul_rn(rintf(__fdiv_rn(d, L)), L));
}
__device__ __forceinline__ float ex_len(float x, float y, float z) {
  return __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), __fmul_rn(z, z)));
}
__device__ __forceinline__ float ex_dist(const float4& a, const float4& b, const float* box) {
  return ex_len(ex_mi(__fsub_rn(a.x, b.x), box[0]), ex_mi(__fsub_rn(a.y, b.y), box[1]),
                ex_mi(__fsub_rn(a.z, b.z), box[2]));
}
// soup/wgsl/bond-common.wgsl:123 bPairB and engine/wgsl/forces.wgsl:17 wca_cut, f32 in order
__device__ __forceinline__ float ex_pairB(const Shared& S, float ti, float tj) {
  return __fmul_rn(__fmul_rn(S.sigma, __fadd_rn(S.radius[(int)ti], S.radius[(int)tj])), 0.5f);
}
__device__ __forceinline__ float ex_wcut(const Shared& S, float b) { return __fmul_rn(S.c6, b); }

// engine/wgsl/forces.wgsl:215-219 cell_coord (f32 floor of (p/box)*n, clamped)
__device__ __forceinline__ int ex_cell_axis(float p, float L, int n) {
  float f = floorf(__fmul_rn(__fdiv_rn(p, L), (float)n));
  int c = (int)fmaxf(f, -1.0f);
  return min(max(c, 0), n - 1);
}

// ---------------------------------------------------------------------------------------------
// Fast force helpers
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ float fast_mi(float d, float L, float invL) { return fmaf(-rintf(d * invL), L, d); }

// The per-system numbers the pair loop needs, held in registers.
struct PairP {
  float box[3], inv_box[3];
  float es_A, es_kappa, es_rc, es_fc, es_split, acid;
  __device__ __forceinline__ static PairP of(const SysParams& P) {
    PairP q;
    for (int a = 0; a < 3; ++a) { q.box[a] = P.box[a]; q.inv_box[a] = P.inv_box[a]; }
    q.es_A = P.es_A; q.es_kappa = P.es_kappa; q.es_rc = P.es_rc; q.es_fc = P.es_fc; q.es_split = P.es_split;
    q.acid = P.acid;
    return q;
  }
};

// Scalar s such that the pair force on i is s * d (d = mi(xi - xj)), for every term the
// neighbour list carries: WCA, class attraction (+ acid-soap depth), near-half screened Coulomb.
// WCA and the attraction are evaluated unconditionally and selected (no divergent branches); the
// screened Coulomb term only exists between charged beads and stays a branch.
template <class PP>
__device__ __forceinline__ float pair_scalar(const Shared& S, const PP& P, const PairConst& pc,
                                             float r2, int ki, int kj, float qi, float qj) {
  const float rinv = rsqrtf(r2);
  const float r = r2 * rinv;
  const float rinv2 = rinv * rinv;
  const float s2 = pc.b2 * rinv2;                         // forces.wgsl:19-23: -wca_dv(r)/r
  const float s6 = s2 * s2 * s2;
  const float fw = 24.0f * S.eps * (2.0f * s6 * s6 - s6) * rinv2;
  float s = (r2 < pc.wcut2) ? fw : 0.f;
  float scale = pc.attr;                                  // pair.wgsl:188 class depth + acid-soap depth
  if (P.acid > 0.f && ((qi != 0.f) != (qj != 0.f)) && S.cls[ki] == 1u && S.cls[kj] == 1u) scale += P.acid;
  const float x = (r - S.rc_attr) * S.attr_k;            // forces.wgsl:32-37
  const float fa = scale * S.attr_amp * __sinf(2.0f * x) * rinv;
  s -= (r >= S.rc_attr && r <= S.rc_attr + S.wc) ? fa : 0.f;
  const float qq = qi * qj;                               // electrostatics.wgsl:65-83, near half
  if (qq != 0.f && r < P.es_split && r < P.es_rc && P.es_A != 0.f) {
    const float u = P.es_A * __expf(-P.es_kappa * r) * rinv;
    s += qq * (u * (rinv + P.es_kappa) - P.es_fc) * rinv;
  }
  return s;
}

// engine/wgsl/forces.wgsl:25-30 fene_dv / bend_dv, as a force scalar on d (r clamped at 1e-6)
__device__ __forceinline__ float bonded_scalar(const Shared& S, float r2, bool fene) {
  float r = fmaxf(sqrtf(r2), 1e-6f);
  float dv;
  if (fene) { float x = r / S.r_inf; dv = S.k_fene * r / (1.0f - x * x); }
  else dv = S.k_bend * (r - S.r_bend);
  return -dv / r;
}

#endif  // __CUDACC__

}  // namespace soup

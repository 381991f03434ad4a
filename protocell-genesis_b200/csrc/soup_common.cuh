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
// The list force's per-kind-pair numbers, premultiplied for the pair loop.
struct PairW {
  float b2;      // b^2
  float wcut2;   // (c6 * b)^2
  float amp;     // class-table depth * eps * pi / (2 wc)
  float polar;   // 1 when both kinds are of the polar class (the acid-soap depth applies), else 0
};
struct Shared {
  PairConst pair[SOUP_KMAX * SOUP_KMAX];
  PairW pw[SOUP_KMAX * SOUP_KMAX];
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

// The pair loop's constants of one replica, held in registers (batch-wide numbers from Shared, the
// replica's acid-soap depth and screened-Coulomb numbers from its SysParams).
struct PairLean {
  float c48, c24;         // 48 eps, 24 eps
  float k2, k2rc;         // sin argument 2 (r - rc) pi / (2 wc) = r k2 - k2rc
  float rc2, rcw2;        // the attraction window [rc, rc + wc], squared
  float acid_amp;         // acid-soap depth * eps * pi / (2 wc), 0 without it
  float es_A, es_kappa, es_fc, es_lim2;   // near screened Coulomb below min(split, rc)^2 (-1: none)
  __device__ __forceinline__ static PairLean of(const Shared& S, const SysParams& P) {
    PairLean L;
    L.c48 = 48.0f * S.eps;
    L.c24 = 24.0f * S.eps;
    L.k2 = 2.0f * S.attr_k;
    L.k2rc = L.k2 * S.rc_attr;
    L.rc2 = S.rc_attr * S.rc_attr;
    const float rcw = S.rc_attr + S.wc;
    L.rcw2 = rcw * rcw;
    L.acid_amp = P.acid > 0.f ? P.acid * S.attr_amp : 0.f;
    L.es_A = P.es_A; L.es_kappa = P.es_kappa; L.es_fc = P.es_fc;
    const float lim = fminf(P.es_split, P.es_rc);
    L.es_lim2 = P.es_A != 0.f ? lim * lim : -1.f;
    return L;
  }
};

// Scalar s such that the pair force on i is s * d (d = mi(xi - xj)), for every term the neighbour
// list carries (soup/wgsl/pair.wgsl:168-204 nonbondedSoup): WCA below c6 b (forces.wgsl:19-23,
// -wca_dv(r)/r = 24 eps (2 (b/r)^12 - (b/r)^6) / r^2), the class attraction on [rc, rc + wc] with the
// acid-soap depth added between two polar beads of which exactly one is charged (forces.wgsl:32-37,
// pair.wgsl:151-160, 188: -(A + acid) eps pi / (2 wc) sin(pi (r - rc) / wc) / r), and the near half of
// the screened Coulomb force between charged beads (electrostatics.wgsl:65-83).  WCA and the
// attraction are selected, not branched on; the windows are tested on r^2 (both forces vanish at
// their edges).  The screened Coulomb term only exists between charged beads and stays a branch.
// qi_nz: the owner's charge is nonzero.
__device__ __forceinline__ float pair_lean(const PairW& pc, const PairLean& L, float r2, bool qi_nz, float qi,
                                           float qj) {
  const float rinv = rsqrtf(r2);
  const float r = r2 * rinv;
  const float rinv2 = rinv * rinv;
  const float s2 = pc.b2 * rinv2;
  const float s6 = s2 * s2 * s2;
  float s = (r2 < pc.wcut2) ? (L.c48 * s6 - L.c24) * s6 * rinv2 : 0.f;
  const float amp = pc.amp + ((pc.polar != 0.f && (qi_nz != (qj != 0.f))) ? L.acid_amp : 0.f);
  const float sn = __sinf(fmaf(r, L.k2, -L.k2rc));
  s -= (r2 >= L.rc2 && r2 <= L.rcw2) ? amp * sn * rinv : 0.f;
  const float qq = qi * qj;
  if (qq != 0.f && r2 < L.es_lim2) {
    const float u = L.es_A * __expf(-L.es_kappa * r) * rinv;
    s += qq * (u * (rinv + L.es_kappa) - L.es_fc) * rinv;
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

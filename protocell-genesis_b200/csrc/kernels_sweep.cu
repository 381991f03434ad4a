// kernels_sweep.cu -- the constant-pH Monte Carlo sweep on the device.
//
// Reference: soup/src/electrostatics.ts:435-496 protonationSweep (CPU, sequential, FP64 JavaScript
// numbers), electrostatics.ts:277-281 esPairEnergy, soup/src/acid-soap.ts:147-198 (acidSoapWell,
// acidSoapSiteWork), electrostatics.ts:308-315 pcgNext.
//
// The attempt chain is inherently sequential (attempt a+1's site depends on how many draws attempt a
// used, which depends on its free energy).  What is not sequential is the energy: the reference
// recomputes, per attempt, E_s = kT ln10 (pKa - pH) + sum over neighbours of the screened Coulomb work
// + the acid-soap pair work, and E_s depends on the site's neighbours' charges only (not its own).
// So:
//   k_sweep_init   (all SMs) evaluates E_s for every head in FP64 from the head list.
//   k_sweep_walk   (one CTA per replica) keeps E in shared memory and walks the attempts.  Every
//                  thread walks the chain redundantly (same RNG, same shared reads), so a rejected
//                  attempt needs no barrier; an accepted flip of site s adds its exact change to
//                  E_t of every neighbour t (cooperatively), then one barrier.
// Arithmetic is FP64 with JavaScript rounding of the minimum image, as the reference's.  E is
// summed in a different order than the reference's cell walk, so it agrees to FP64 rounding (the
// decisions agree unless a draw lands within ~1e-15 of its threshold).
#include "soup_internal.h"

namespace soup {

namespace {

__device__ __forceinline__ double js_round(double x) {
  const double r = floor(x);
  return (x - r >= 0.5) ? r + 1.0 : r;
}
__device__ __forceinline__ double es_energy(const SysParams& P, double r, double qq) {
  if (P.d_A == 0.0 || qq == 0.0 || r >= P.d_rc || r <= 0.0) return 0.0;
  const double u1 = (P.d_A * exp(-P.d_kappa * r)) / r;
  return qq * (u1 - P.d_shiftU + P.d_shiftF * (r - P.d_rc));
}
__device__ __forceinline__ double acid_well(const SysParams& P, double r) {
  if (P.d_acid <= 0.0) return 0.0;
  if (r < P.d_rcattr) return -P.d_acid * P.d_eps;
  if (r > P.d_rcattr + P.d_wc) return 0.0;
  const double c = cos((3.141592653589793 * (r - P.d_rcattr)) / (2.0 * P.d_wc));
  return -P.d_acid * P.d_eps * c * c;
}
__device__ __forceinline__ double dist2(const SysParams& P, const float4& a, const float4& b) {
  double dx = (double)a.x - (double)b.x, dy = (double)a.y - (double)b.y, dz = (double)a.z - (double)b.z;
  dx -= js_round(dx / P.d_box[0]) * P.d_box[0];
  dy -= js_round(dy / P.d_box[1]) * P.d_box[1];
  dz -= js_round(dz / P.d_box[2]) * P.d_box[2];
  return dx * dx + dy * dy + dz * dz;
}
// the energy a neighbour of charge qj at squared distance r2 contributes to a site's E
__device__ __forceinline__ double site_term(const SysParams& P, double r2, float qj, double cut2, double reach2) {
  double e = 0.0;
  if (qj != 0.f && r2 < cut2) e += es_energy(P, sqrt(r2), P.d_q * (double)qj);
  if (P.d_acid > 0.0 && r2 < reach2 && r2 > 0.0) {
    const double v = acid_well(P, sqrt(r2));
    e += (qj == 0.f) ? v : -v;
  }
  return e;
}

// E_h = kT ln10 (pKa - pH) + uEs(h), a warp per head
__global__ void __launch_bounds__(256) k_sweep_init(const SysParams* __restrict__ sp, const uint32_t* __restrict__ head_sys,
                                                    const uint32_t* __restrict__ head_slot, uint32_t H,
                                                    const float4* __restrict__ pos, const float* __restrict__ charge,
                                                    const uint32_t* __restrict__ es_nl, const uint32_t* __restrict__ es_cnt,
                                                    uint32_t cap, double* __restrict__ E, uint32_t only) {
  const uint32_t h = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (h >= H) return;
  const uint32_t r = head_sys[h];
  if (only != SOUP_NONE_U32 && r != only) return;
  const SysParams& P = sp[r];
  if (!P.es_on) return;
  const double cut2 = P.d_rc * P.d_rc, reach = P.d_rcattr + P.d_wc, reach2 = reach * reach;
  const float4 xi = pos[head_slot[h]];
  double es = 0.0, w = 0.0;
  const uint32_t cnt = es_cnt[h];
  const uint32_t* row = es_nl + (size_t)h * cap;
  for (uint32_t s = lane; s < cnt; s += 32) {
    const uint32_t js = head_slot[row[s]];
    const float qj = charge[js];
    const double r2 = dist2(P, xi, pos[js]);
    if (qj != 0.f && r2 < cut2) es += es_energy(P, sqrt(r2), P.d_q * (double)qj);
    if (P.d_acid > 0.0 && r2 < reach2 && r2 > 0.0) {
      const double v = acid_well(P, sqrt(r2));
      w += (qj == 0.f) ? v : -v;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    es += __shfl_xor_sync(0xffffffffu, es, o);
    w += __shfl_xor_sync(0xffffffffu, w, o);
  }
  if (lane == 0) E[h] = P.d_kT * 2.302585092994046 * (P.d_pka - P.d_ph) + (es + w);
}

// exp(-dG/kT) > u  decided by an FP32 estimate when far from the threshold, else in FP64
__device__ __forceinline__ bool metropolis(double dG, double kT, double u) {
  const float x = (float)(-dG / kT);
  const double est = (double)__expf(x);
  if (u < est * (1.0 - 1e-5)) return true;
  if (u > est * (1.0 + 1e-5) + 1e-300) return false;
  return u < exp(-dG / kT);
}

constexpr int kWalkThreads = 512;

template <bool SMEM>
__global__ void __launch_bounds__(kWalkThreads) k_sweep_walk(const SysParams* __restrict__ sp,
                                                             const uint32_t* __restrict__ head_slot,
                                                             const float4* __restrict__ pos, float* __restrict__ charge,
                                                             const uint32_t* __restrict__ es_nl,
                                                             const uint32_t* __restrict__ es_cnt, uint32_t cap,
                                                             double* __restrict__ Eg, uint32_t* __restrict__ rng_io,
                                                             double* __restrict__ out, uint32_t only) {
  extern __shared__ __align__(16) unsigned char smem[];
  const uint32_t r = (only == SOUP_NONE_U32) ? blockIdx.x : only;
  const SysParams& P = sp[r];
  const uint32_t H = P.nheads;
  if (H == 0 || !P.es_on) return;
  const uint32_t off = P.head_off;
  double* E = SMEM ? reinterpret_cast<double*>(smem) : Eg + off;
  unsigned char* flag = SMEM ? smem + 8 * (size_t)H : nullptr;
  __shared__ double s_stats[2];
  __shared__ uint32_t s_acc;
  if (SMEM) {
    for (uint32_t h = threadIdx.x; h < H; h += kWalkThreads) {
      E[h] = Eg[off + h];
      flag[h] = charge[head_slot[off + h]] != 0.f ? 1 : 0;
    }
  }
  if (threadIdx.x == 0) { s_stats[0] = 0.0; s_stats[1] = 0.0; s_acc = 0; }
  __syncthreads();
  const double kT = P.d_kT;
  const double dGintr = kT * 2.302585092994046 * (P.d_pka - P.d_ph);
  const double cut2 = P.d_rc * P.d_rc, reach = P.d_rcattr + P.d_wc, reach2 = reach * reach;
  uint32_t rng = rng_io[r];
  for (uint32_t a = 0; a < H; ++a) {
    const double u = pcg_next(rng);
    const uint32_t s = (uint32_t)fmin((double)(H - 1), floor(u * (double)H));
    const double Es = E[s];
    const bool ch = SMEM ? flag[s] != 0 : charge[head_slot[off + s]] != 0.f;
    const double dG = ch ? -Es : Es;
    bool acc = dG <= 0.0;
    if (!acc) acc = metropolis(dG, kT, pcg_next(rng));
    if (!acc) continue;
    const uint32_t ks = head_slot[off + s];
    const float q_old = charge[ks];
    const float q_new = ch ? 0.f : (float)P.d_q;
    const float4 xi = pos[ks];
    const uint32_t cnt = es_cnt[off + s];
    const uint32_t* row = es_nl + (size_t)(off + s) * cap;
    for (uint32_t k = threadIdx.x; k < cnt; k += kWalkThreads) {
      const uint32_t t = row[k];
      const double r2 = dist2(P, xi, pos[head_slot[t]]);
      E[t - off] += site_term(P, r2, q_new, cut2, reach2) - site_term(P, r2, q_old, cut2, reach2);
    }
    __syncthreads();   // every thread has read charge[ks] and E[s] for this attempt
    if (threadIdx.x == 0) {
      charge[ks] = q_new;
      if (SMEM) flag[s] = ch ? 0 : 1;
      ++s_acc;
      if (!ch) { s_stats[0] += (Es - dGintr) / kT; s_stats[1] += 1.0; }
    }
    __syncthreads();
  }
  double dep = 0.0;
  for (uint32_t h = threadIdx.x; h < H; h += kWalkThreads) dep += charge[head_slot[off + h]] != 0.f ? 1.0 : 0.0;
  for (int o = 16; o > 0; o >>= 1) dep += __shfl_xor_sync(0xffffffffu, dep, o);
  __shared__ double s_dep[kWalkThreads / 32];
  if ((threadIdx.x & 31) == 0) s_dep[threadIdx.x >> 5] = dep;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kWalkThreads / 32; ++w) t += s_dep[w];
    rng_io[r] = rng;
    out[4 * r + 0] = (double)H;
    out[4 * r + 1] = (double)s_acc;
    out[4 * r + 2] = s_stats[1] > 0 ? s_stats[0] / s_stats[1] : 0.0;
    out[4 * r + 3] = t;
  }
}

}  // namespace

// replica == SOUP_NONE_U32: every replica, one CTA each
void launch_sweep(Batch& b, uint32_t replica) {
  if (b.H == 0) return;
  uint32_t hmax = 0;
  for (uint32_t r = 0; r < b.R; ++r)
    if (replica == SOUP_NONE_U32 || r == replica) hmax = std::max(hmax, b.hsp[r].nheads);
  b.launches += 2;
  prof_begin(b, SOUP_K_SWEEP);
  k_sweep_init<<<(unsigned)(((uint64_t)b.H * 32 + 255) / 256), 256, 0, b.stream>>>(
      b.sp, b.head_sys, b.head_slot, b.H, b.pos, b.charge, b.es_nl, b.es_cnt, b.es_cap, b.head_e, replica);
  const unsigned grid = replica == SOUP_NONE_U32 ? b.R : 1;
  const size_t smem = 9 * (size_t)hmax;
  if (smem <= 200 * 1024) {
    static bool attr = false;
    if (!attr) {
      SOUP_CUDA_TRY(cudaFuncSetAttribute(k_sweep_walk<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
      attr = true;
    }
    k_sweep_walk<true><<<grid, kWalkThreads, smem, b.stream>>>(b.sp, b.head_slot, b.pos, b.charge, b.es_nl, b.es_cnt,
                                                               b.es_cap, b.head_e, b.prot_rng_dev, b.sweep_out, replica);
  } else {
    k_sweep_walk<false><<<grid, kWalkThreads, 0, b.stream>>>(b.sp, b.head_slot, b.pos, b.charge, b.es_nl, b.es_cnt,
                                                             b.es_cap, b.head_e, b.prot_rng_dev, b.sweep_out, replica);
  }
  prof_end(b);
}

}  // namespace soup

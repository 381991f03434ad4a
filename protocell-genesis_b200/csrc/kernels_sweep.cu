// kernels_sweep.cu -- the constant-pH Monte Carlo sweep on the device.
//
// Reference: soup/src/electrostatics.ts:435-496 protonationSweep (CPU, sequential, FP64 JavaScript
// numbers), electrostatics.ts:277-281 esPairEnergy, soup/src/acid-soap.ts:147-198 (acidSoapWell,
// acidSoapSiteWork), electrostatics.ts:308-315 pcgNext.
//
// The sweep is inherently sequential: attempt a+1's site depends on how many draws attempt a used,
// which depends on its dG.  One CTA per replica walks the attempts in order; each attempt's
// neighbour energy is a block-wide FP64 reduction over the site's head list (the long-range list,
// built at rc_es + skin, holds every head within rc_es of the site while drift < skin/2).  The
// reference sums the same terms in its cell-walk order; the totals agree to FP64 rounding.
#include "soup_internal.h"

namespace soup {

namespace {

__device__ __forceinline__ double js_round(double x) {
  double r = floor(x);
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

template <int NT>
__device__ __forceinline__ void block_sum2(double& a, double& b, double* red) {
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) { red[2 * w] = a; red[2 * w + 1] = b; }
  __syncthreads();
  if (w == 0) {
    a = lane < NT / 32 ? red[2 * lane] : 0.0;
    b = lane < NT / 32 ? red[2 * lane + 1] : 0.0;
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_xor_sync(0xffffffffu, a, o);
      b += __shfl_xor_sync(0xffffffffu, b, o);
    }
  }
}

constexpr int kSweepThreads = 256;

__global__ void __launch_bounds__(kSweepThreads) k_sweep(const SysParams* __restrict__ sp, const uint32_t* __restrict__ heads,
                                                         const uint32_t* __restrict__ slot_of, const float4* __restrict__ pos,
                                                         float* __restrict__ charge, const uint32_t* __restrict__ es_nl,
                                                         const uint32_t* __restrict__ es_cnt, uint32_t cap,
                                                         uint32_t* __restrict__ rng_io, double* __restrict__ out,
                                                         uint32_t only) {
  const uint32_t r = (only == SOUP_NONE_U32) ? blockIdx.x : only;
  const SysParams& P = sp[r];
  __shared__ double red[2 * kSweepThreads / 32];
  __shared__ uint32_t s_site;
  const uint32_t H = P.nheads;
  if (H == 0 || !P.es_on) return;
  const uint32_t* hd = heads + P.head_off;
  const double dGintr = P.d_kT * 2.302585092994046 * (P.d_pka - P.d_ph);   // kT ln(10) (pKa - pH)
  const double q = P.d_q;
  const double cut2 = P.d_rc * P.d_rc;
  const double reach = P.d_rcattr + P.d_wc, reach2 = reach * reach;
  uint32_t rng = rng_io[r];
  uint32_t accepted = 0, dEsCount = 0;
  double dEsSum = 0.0;
  for (uint32_t a = 0; a < H; ++a) {
    if (threadIdx.x == 0) {
      double u = pcg_next(rng);
      uint32_t h = (uint32_t)fmin((double)(H - 1), floor(u * (double)H));
      s_site = h;
    }
    __syncthreads();
    const uint32_t h = s_site;
    const uint32_t ks = slot_of[hd[h]];
    const float4 xi = pos[ks];
    const uint32_t cnt = es_cnt[P.head_off + h];
    const uint32_t* row = es_nl + (size_t)(P.head_off + h) * cap;
    double ues = 0.0, uw = 0.0;
    for (uint32_t s = threadIdx.x; s < cnt; s += kSweepThreads) {
      const uint32_t js = row[s];
      const float4 xj = pos[js];
      const float qj = charge[js];
      double dx = (double)xi.x - (double)xj.x, dy = (double)xi.y - (double)xj.y, dz = (double)xi.z - (double)xj.z;
      dx -= js_round(dx / P.d_box[0]) * P.d_box[0];
      dy -= js_round(dy / P.d_box[1]) * P.d_box[1];
      dz -= js_round(dz / P.d_box[2]) * P.d_box[2];
      const double r2 = dx * dx + dy * dy + dz * dz;
      if (qj != 0.f && r2 < cut2) ues += es_energy(P, sqrt(r2), q * (double)qj);
      if (P.d_acid > 0.0 && r2 < reach2 && r2 > 0.0) {
        const double v = acid_well(P, sqrt(r2));
        uw += (qj == 0.f) ? v : -v;
      }
    }
    block_sum2<kSweepThreads>(ues, uw, red);
    if (threadIdx.x == 0) {
      const double uEs = ues + uw;
      const bool charged = charge[ks] != 0.f;
      const double dG = charged ? -(dGintr + uEs) : dGintr + uEs;
      bool acc = dG <= 0.0;
      if (!acc) acc = pcg_next(rng) < exp(-dG / P.d_kT);
      if (acc) {
        charge[ks] = charged ? 0.f : (float)q;
        ++accepted;
        if (!charged) { dEsSum += uEs / P.d_kT; ++dEsCount; }
      }
    }
    __syncthreads();
  }
  // deprotonated count
  double dep = 0.0, dummy = 0.0;
  for (uint32_t h = threadIdx.x; h < H; h += kSweepThreads) dep += charge[slot_of[hd[h]]] != 0.f ? 1.0 : 0.0;
  block_sum2<kSweepThreads>(dep, dummy, red);
  if (threadIdx.x == 0) {
    rng_io[r] = rng;
    out[4 * r + 0] = (double)H;
    out[4 * r + 1] = (double)accepted;
    out[4 * r + 2] = dEsCount > 0 ? dEsSum / dEsCount : 0.0;
    out[4 * r + 3] = dep;
  }
}

}  // namespace

// replica == SOUP_NONE_U32: every replica, one CTA each
void launch_sweep(Batch& b, uint32_t replica) {
  if (b.H == 0) return;
  unsigned grid = replica == SOUP_NONE_U32 ? b.R : 1;
  k_sweep<<<grid, kSweepThreads, 0, b.stream>>>(b.sp, b.heads, b.slot_of, b.pos, b.charge, b.es_nl, b.es_cnt, b.es_cap,
                                                 b.prot_rng_dev, b.sweep_out, replica);
}

}  // namespace soup

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
// squared minimum-image distance, FP64, JavaScript rounding of the image (Math.round(d / L)).  The
// image index is taken from d * (1/L): it can differ from d / L only within an ulp of a half-box
// offset, where every pair is beyond the (at most 0.45 L) cutoffs either way.
__device__ __forceinline__ double dist2(const SysParams& P, const float4& a, const float4& b) {
  double dx = (double)a.x - (double)b.x, dy = (double)a.y - (double)b.y, dz = (double)a.z - (double)b.z;
  dx -= js_round(dx * P.d_inv_box[0]) * P.d_box[0];
  dy -= js_round(dy * P.d_inv_box[1]) * P.d_box[1];
  dz -= js_round(dz * P.d_inv_box[2]) * P.d_box[2];
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

// the pcgNext LCG (state' = a state + c mod 2^32) advanced n steps at once
struct Lcg { uint32_t a, c; };
__device__ __forceinline__ Lcg lcg_pow(uint32_t n) {
  Lcg acc{1u, 0u}, b{747796405u, 2891336453u};
  while (n) {
    if (n & 1u) acc = Lcg{acc.a * b.a, acc.c * b.a + b.c};
    b = Lcg{b.a * b.a, b.c * b.a + b.c};
    n >>= 1;
  }
  return acc;
}
__device__ __forceinline__ double pcg_out(uint32_t v) {
  v = ((v >> ((v >> 28u) + 4u)) ^ v) * 277803737u;
  v = (v >> 22u) ^ v;
  return (double)v / 4294967296.0;
}

// Draws of the pcgNext stream, 32 at a time: lane l of every warp holds draw base+l; the walker
// takes them in order through a shuffle (the same values in every warp).
struct Stream {
  uint32_t st;       // state after draw base+lane
  double u;          // draw base+lane
  uint32_t base, p;  // first draw held, next draw to hand out
  Lcg jump32;
  __device__ void init(uint32_t s0, int lane) {
    const Lcg j = lcg_pow((uint32_t)lane + 1u);
    st = j.a * s0 + j.c;
    u = pcg_out(st);
    base = 0; p = 0;
    jump32 = lcg_pow(32u);
  }
  __device__ double next() {
    if (p - base == 32u) {
      st = jump32.a * st + jump32.c;
      u = pcg_out(st);
      base += 32u;
    }
    const int l = (int)(p - base);
    ++p;
    return __shfl_sync(0xffffffffu, u, l);
  }
};

constexpr int kWalkThreads = 1024;

// head positions for the flip updates: by head index (hpos) and in head-cell order with the head
// index in w (spos), so a flip scans contiguous, L2-resident candidate ranges
__global__ void k_gather_heads(const uint32_t* __restrict__ head_slot, uint32_t H, const float4* __restrict__ pos,
                               const uint32_t* __restrict__ hsorted, float4* __restrict__ hpos,
                               float4* __restrict__ spos) {
  const uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= H) return;
  hpos[h] = pos[head_slot[h]];
  const uint32_t g = hsorted[h];
  const float4 p = pos[head_slot[g]];
  spos[h] = make_float4(p.x, p.y, p.z, __uint_as_float(g));
}

template <bool SMEM>
__global__ void __launch_bounds__(kWalkThreads) k_sweep_walk(const SysParams* __restrict__ sp,
                                                             const uint32_t* __restrict__ head_slot,
                                                             const float4* __restrict__ hpos, float* __restrict__ charge,
                                                             const uint32_t* __restrict__ es_nl,
                                                             const uint32_t* __restrict__ es_cnt, uint32_t cap,
                                                             const uint32_t* __restrict__ hcell_of,
                                                             const uint32_t* __restrict__ hstart,
                                                             const float4* __restrict__ spos,
                                                             double* __restrict__ Eg, uint8_t* __restrict__ flag_g,
                                                             uint32_t* __restrict__ rng_io, double* __restrict__ out,
                                                             uint32_t only) {
  extern __shared__ __align__(16) unsigned char smem[];
  const uint32_t r = (only == SOUP_NONE_U32) ? blockIdx.x : only;
  const SysParams& P = sp[r];
  const uint32_t H = P.nheads;
  if (H == 0 || !P.es_on) return;
  const uint32_t off = P.head_off;
  double* E = SMEM ? reinterpret_cast<double*>(smem) : Eg + off;
  uint8_t* flag = SMEM ? smem + 8 * (size_t)H : flag_g + off;
  const float qd = (float)P.d_q;
  // flag: 0 neutral, 1 charged with the deprotonated charge, 2 charged with another value
  for (uint32_t h = threadIdx.x; h < H; h += kWalkThreads) {
    if (SMEM) E[h] = Eg[off + h];
    const float q = charge[head_slot[off + h]];
    flag[h] = q == 0.f ? 0 : (q == qd ? 1 : 2);
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const double kT = P.d_kT;
  const double dGintr = kT * 2.302585092994046 * (P.d_pka - P.d_ph);
  const double cut2 = P.d_rc * P.d_rc, reach = P.d_rcattr + P.d_wc, reach2 = reach * reach;
  const uint32_t s0 = rng_io[r];
  Stream rs;
  rs.init(s0, lane);
  uint32_t accepted = 0, dcount = 0;
  double dsum = 0.0;
  for (uint32_t a = 0; a < H; ++a) {
    const double u = rs.next();
    const uint32_t s = (uint32_t)fmin((double)(H - 1), floor(u * (double)H));
    const double Es = E[s];
    const uint8_t f = flag[s];
    const bool ch = f != 0;
    const double dG = ch ? -Es : Es;
    bool acc = dG <= 0.0;
    if (!acc) acc = metropolis(dG, kT, rs.next());
    if (!acc) continue;
    const float q_old = f == 0 ? 0.f : (f == 1 ? qd : charge[head_slot[off + s]]);
    const float q_new = ch ? 0.f : qd;
    const float4 xi = hpos[off + s];
    {
      // candidates: the +-hwalk head cells around the site's cell at the last rebuild (complete for
      // r < rc_es while every head has drifted less than skin/2), one row of cells per warp
      const uint32_t c = hcell_of[off + s] - P.hcell_off;
      const int nx = P.hdims[0], ny = P.hdims[1], nz = P.hdims[2], R = P.hwalk;
      const int qx = (int)(c % (uint32_t)nx), qy = (int)((c / (uint32_t)nx) % (uint32_t)ny),
                qz = (int)(c / ((uint32_t)nx * (uint32_t)ny));
      const int span = 2 * R + 1;
      const int nyv = span < ny ? span : ny, nzv = span < nz ? span : nz;
      int xlo[2], xhi[2], nxr;
      {
        const int lo = qx - R, hi = qx + R;
        if (hi - lo + 1 >= nx) { nxr = 1; xlo[0] = 0; xhi[0] = nx - 1; }
        else if (lo < 0) { nxr = 2; xlo[0] = lo + nx; xhi[0] = nx - 1; xlo[1] = 0; xhi[1] = hi; }
        else if (hi >= nx) { nxr = 2; xlo[0] = lo; xhi[0] = nx - 1; xlo[1] = 0; xhi[1] = hi - nx; }
        else { nxr = 1; xlo[0] = lo; xhi[0] = hi; }
      }
      const int w = threadIdx.x >> 5;
      for (int rowi = w; rowi < nyv * nzv; rowi += kWalkThreads / 32) {
        const int y = (span < ny) ? ((qy - R + rowi % nyv) % ny + ny) % ny : rowi % nyv;
        const int z = (span < nz) ? ((qz - R + rowi / nyv) % nz + nz) % nz : rowi / nyv;
        const uint32_t rb = P.hcell_off + (uint32_t)(nx * (y + ny * z));
        for (int xr = 0; xr < nxr; ++xr) {
          const uint32_t a0 = hstart[rb + xlo[xr]], e0 = hstart[rb + xhi[xr] + 1];
          for (uint32_t k = a0 + lane; k < e0; k += 32) {
            const float4 pj = spos[k];
            const uint32_t t = __float_as_uint(pj.w);
            if (t == off + s) continue;
            const double r2 = dist2(P, xi, pj);
            if (r2 < cut2 || r2 < reach2)
              E[t - off] += site_term(P, r2, q_new, cut2, reach2) - site_term(P, r2, q_old, cut2, reach2);
          }
        }
      }
    }
    __syncthreads();   // every update of this flip is in E; every thread has read this attempt's state
    flag[s] = ch ? 0 : 1;
    if (threadIdx.x == 0) {
      charge[head_slot[off + s]] = q_new;
      ++accepted;
      if (!ch) { dsum += (Es - dGintr) / kT; ++dcount; }
    }
  }
  __syncthreads();
  __shared__ uint32_t s_dep;
  if (threadIdx.x == 0) s_dep = 0;
  __syncthreads();
  uint32_t dep = 0;
  for (uint32_t h = threadIdx.x; h < H; h += kWalkThreads) dep += flag[h] != 0;
  for (int o = 16; o > 0; o >>= 1) dep += __shfl_xor_sync(0xffffffffu, dep, o);
  if (lane == 0) atomicAdd(&s_dep, dep);
  __syncthreads();
  if (threadIdx.x == 0) {
    const Lcg j = lcg_pow(rs.p);
    rng_io[r] = j.a * s0 + j.c;
    out[4 * r + 0] = (double)H;
    out[4 * r + 1] = (double)accepted;
    out[4 * r + 2] = dcount > 0 ? dsum / dcount : 0.0;
    out[4 * r + 3] = (double)s_dep;
  }
}

}  // namespace

// replica == SOUP_NONE_U32: every replica, one CTA each
void launch_sweep(Batch& b, uint32_t replica) {
  if (b.H == 0) return;
  uint32_t hmax = 0;
  for (uint32_t r = 0; r < b.R; ++r)
    if (replica == SOUP_NONE_U32 || r == replica) hmax = std::max(hmax, b.hsp[r].nheads);
  b.launches += 3;
  prof_begin(b, SOUP_K_SWEEP);
  k_gather_heads<<<(b.H + 255) / 256, 256, 0, b.stream>>>(b.head_slot, b.H, b.pos, b.hsorted, b.head_pos,
                                                           b.head_spos);
  k_sweep_init<<<(unsigned)(((uint64_t)b.H * 32 + 255) / 256), 256, 0, b.stream>>>(
      b.sp, b.head_sys, b.head_slot, b.H, b.pos, b.charge, b.es_nl, b.es_cnt, b.es_cap, b.head_e, replica);
  const unsigned grid = replica == SOUP_NONE_U32 ? b.R : 1;
  const size_t smem = 9 * (size_t)hmax;
  if (smem <= 200 * 1024) {
    k_sweep_walk<true><<<grid, kWalkThreads, smem, b.stream>>>(b.sp, b.head_slot, b.head_pos, b.charge, b.es_nl,
                                                               b.es_cnt, b.es_cap, b.hcell_of, b.hcell_start,
                                                               b.head_spos, b.head_e, b.head_flag,
                                                               b.prot_rng_dev, b.sweep_out, replica);
  } else {
    k_sweep_walk<false><<<grid, kWalkThreads, 0, b.stream>>>(b.sp, b.head_slot, b.head_pos, b.charge, b.es_nl,
                                                             b.es_cnt, b.es_cap, b.hcell_of, b.hcell_start,
                                                             b.head_spos, b.head_e, b.head_flag,
                                                             b.prot_rng_dev, b.sweep_out, replica);
  }
  prof_end(b);
}

void sweep_prepare(Batch& b) {
  SOUP_CUDA_TRY(cudaFuncSetAttribute(k_sweep_walk<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
}

}  // namespace soup

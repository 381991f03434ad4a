// kernels_sweep.cu -- the constant-pH Monte Carlo sweep on the device.
//
// Reference: soup/src/electrostatics.ts:435-496 protonationSweep (CPU, sequential, FP64 JavaScript
// numbers), electrostatics.ts:277-281 esPairEnergy, soup/src/acid-soap.ts:147-198 (acidSoapWell,
// acidSoapSiteWork), electrostatics.ts:308-315 pcgNext.
//
// The attempt chain is sequential: attempt a+1's site draw depends on whether attempt a took an
// acceptance draw, which depends on its free energy.  The energy itself is not sequential: the
// reference recomputes, per attempt, E_s = kT ln10 (pKa - pH) + the screened Coulomb work + the
// acid-soap pair work over the site's neighbours, and E_s depends on the neighbours' charges only.
// Positions are fixed during a sweep, so the change of E_t when neighbour s flips is a fixed number
// per pair.  So:
//   k_sweep_init  (all SMs, a warp per head) evaluates E_h in FP64 from the head list, and for every
//                 list entry t of h the change D_ht of E_t when h deprotonates (-D_ht when it
//                 protonates).
//   k_sweep_walk  (one CTA per replica) keeps E in shared memory and walks the chain in windows of
//                 32 draws.  Warp 0 holds the draws, their sites and those sites' positions in its
//                 lanes (prefetched a window ahead); it resolves the window's attempts one by one (the
//                 deciding lane, one shuffle), and when a flip is accepted every later lane adds the
//                 flip's change to its own site energy (exact, the formula of D).  Then all warps add
//                 the window's flips to E from the D rows, and the next window starts.
// E and D are fixed point (2^-40 kT, int64): integer adds commute, so E does not depend on the
// order the updates land in and every run is reproducible.  E_h is the FP64 sum rounded once, each
// D_ht is rounded once, so the energies agree with the reference's FP64 sums to about 1e-11 kT (the
// decisions agree unless a draw lands that close to its threshold).
// Arithmetic is FP64 with JavaScript rounding of the minimum image, as the reference's.
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

constexpr double kFix = 1099511627776.0;            // 2^40 fixed-point units per kT
constexpr double kUnfix = 1.0 / 1099511627776.0;
constexpr long long kSameSite = (long long)0x8000000000000000ull;   // M marker: both draws pick one site
__device__ __forceinline__ long long to_fix(double x) { return __double2ll_rn(x * kFix); }
// change of a neighbour's E when a site at squared distance r2 goes from charge qo to qn
// (round-to-nearest-even is odd-symmetric, so the reverse flip gives exactly the negative)
__device__ __forceinline__ long long flip_delta(const SysParams& P, double r2, float qo, float qn, double cut2,
                                                double reach2) {
  return to_fix(site_term(P, r2, qn, cut2, reach2) - site_term(P, r2, qo, cut2, reach2));
}
// flip_delta(r2, 0, qd) with one square root (the same operations in the same order, so the same
// bits); the value of every D entry and of every in-window correction
__device__ __forceinline__ long long std_delta(const SysParams& P, double r2, float qd, double cut2, double reach2) {
  double t1 = 0.0, t0 = 0.0;
  const bool es_in = qd != 0.f && r2 < cut2;
  const bool ac_in = P.d_acid > 0.0 && r2 < reach2 && r2 > 0.0;
  if (es_in || ac_in) {
    const double rr = sqrt(r2);
    if (es_in) t1 += es_energy(P, rr, P.d_q * (double)qd);
    if (ac_in) {
      const double v = acid_well(P, rr);
      t1 += -v;
      t0 += v;
    }
  }
  return to_fix(t1 - t0);
}

// E_h = kT ln10 (pKa - pH) + uEs(h) and the row D_h, a warp per head
__global__ void __launch_bounds__(256) k_sweep_init(const SysParams* __restrict__ sp, const uint32_t* __restrict__ head_sys,
                                                    const uint32_t* __restrict__ head_slot, uint32_t H,
                                                    const float4* __restrict__ pos, const float* __restrict__ charge,
                                                    const uint32_t* __restrict__ es_nl, const uint32_t* __restrict__ es_cnt,
                                                    uint32_t cap, long long* __restrict__ E, long long* __restrict__ D,
                                                    uint32_t only) {
  const uint32_t h = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (h >= H) return;
  const uint32_t r = head_sys[h];
  if (only != SOUP_NONE_U32 && r != only) return;
  const SysParams& P = sp[r];
  if (!P.es_on) return;
  const double cut2 = P.d_rc * P.d_rc, reach = P.d_rcattr + P.d_wc, reach2 = reach * reach;
  const float qd = (float)P.d_q;
  const float4 xi = pos[head_slot[h]];
  double es = 0.0, w = 0.0;
  const uint32_t cnt = es_cnt[h];
  const uint32_t* row = es_nl + (size_t)h * cap;
  long long* drow = D + (size_t)h * cap;
  for (uint32_t s = lane; s < cnt; s += 32) {
    const uint32_t js = head_slot[row[s]];
    const float qj = charge[js];
    const double r2 = dist2(P, xi, pos[js]);
    if (qj != 0.f && r2 < cut2) es += es_energy(P, sqrt(r2), P.d_q * (double)qj);
    if (P.d_acid > 0.0 && r2 < reach2 && r2 > 0.0) {
      const double v = acid_well(P, sqrt(r2));
      w += (qj == 0.f) ? v : -v;
    }
    drow[s] = std_delta(P, r2, qd, cut2, reach2);
  }
  for (int o = 16; o > 0; o >>= 1) {
    es += __shfl_xor_sync(0xffffffffu, es, o);
    w += __shfl_xor_sync(0xffffffffu, w, o);
  }
  if (lane == 0) E[h] = to_fix(P.d_kT * 2.302585092994046 * (P.d_pka - P.d_ph) + (es + w));
}

// u < exp(-dG/kT) for dG > 0.  For -dG/kT > -20 an FP32 estimate decides when u is more than 1e-5
// (relative) away from it: __expf's error there is below 2 + 1.16*20 ulp and the FP32 rounding of
// the exponent adds 1e-6, together under 5e-6.  Below -20 only u < 1e-8 can pass.  Otherwise, and
// near the threshold, FP64 decides.
__device__ __forceinline__ bool metropolis(double dG, double kT, double inv_kT, double u) {
  const double xd = -dG * inv_kT;
  if (xd > -20.0) {
    const double est = (double)__expf((float)xd);
    if (u < est * (1.0 - 1e-5)) return true;
    if (u > est * (1.0 + 1e-5)) return false;
  } else if (u >= 1e-8) {
    return false;                 // exp(-dG/kT) <= e^-20 (1 + 1e-15) < 2.1e-9
  }
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

constexpr int kWalkThreads = 512;
constexpr int kUpd = 8;
constexpr uint32_t kQueue = 512;

// one draw of the stream as a lane holds it: the LCG state that produced it, the draw, the site it
// selects when it is a site draw, that site's position and its head-list length
struct Draw {
  uint32_t st, site, cnt;
  double u;
  float x, y, z;
};
__device__ __forceinline__ void draw_from(Draw& d, uint32_t st, uint32_t H, uint32_t off,
                                          const float4* __restrict__ hpos, const uint32_t* __restrict__ es_cnt) {
  d.st = st;
  d.u = pcg_out(st);
  d.site = (uint32_t)fmin((double)(H - 1), floor(d.u * (double)H));
  const float4 p = hpos[off + d.site];
  d.x = p.x; d.y = p.y; d.z = p.z;
  d.cnt = es_cnt[off + d.site];
}
__device__ __forceinline__ Draw shfl_draw(const Draw& d, int src) {
  Draw o;
  o.st = __shfl_sync(0xffffffffu, d.st, src);
  o.site = __shfl_sync(0xffffffffu, d.site, src);
  o.cnt = __shfl_sync(0xffffffffu, d.cnt, src);
  o.u = __shfl_sync(0xffffffffu, d.u, src);
  o.x = __shfl_sync(0xffffffffu, d.x, src);
  o.y = __shfl_sync(0xffffffffu, d.y, src);
  o.z = __shfl_sync(0xffffffffu, d.z, src);
  return o;
}

// the flips one window accepted: the scatter into E that runs during the next window, and the
// corrections the next window's lanes take before E has them
struct Flips {
  uint32_t site[32];
  uint32_t start[33];    // prefix of the flipped heads' list lengths; ~0 above the last flip
  float qo[32], qn[32];
  float x[32], y[32], z[32];
  int sign[32];          // +1 deprotonated, -1 protonated, 0 the old charge was another value
  uint32_t n;
};
// the sites and positions of a window's 32 draws, the pair changes between them
// (M[k][q], k < q: D of draw k's site on draw q's site, the exact value its D row holds, or
// kSameSite when both draws select one site) and the previous window's flips summed per draw
struct Window {
  uint32_t site[32];
  float x[32], y[32], z[32];
  long long M[32][32];
  long long corr[32];
  uint16_t queue[kQueue];   // pairs within reach awaiting FP64: k*32+q (M), or 1024 + g*32+q (corr)
  uint32_t nq, done;
};

// window lane q's share of the previous window's flip g (the exact value g's D row holds for q)
__device__ __forceinline__ void corr_term(const SysParams& P, const Flips& Fp, Window& W, uint32_t g, uint32_t q,
                                          float qd, double cut2, double reach2) {
  const double r2 = dist2(P, make_float4(Fp.x[g], Fp.y[g], Fp.z[g], 0.f), make_float4(W.x[q], W.y[q], W.z[q], 0.f));
  const int sg = Fp.sign[g];
  long long d;
  if (sg != 0) {
    d = std_delta(P, r2, qd, cut2, reach2);
    if (sg < 0) d = -d;
  } else {
    d = flip_delta(P, r2, Fp.qo[g], Fp.qn[g], cut2, reach2);
  }
  if (d != 0) atomicAdd(reinterpret_cast<unsigned long long*>(&W.corr[q]), (unsigned long long)d);
}

// The site energies of one replica: in shared memory as two 32-bit halves (32-bit shared atomics are
// native, 64-bit ones are not; an add carries from the low half into the high half exactly, so the
// sum does not depend on the order of the adds), or in global memory as int64.
template <bool SMEM>
struct Energies {
  uint32_t* lo;
  int32_t* hi;
  long long* g;
  __device__ __forceinline__ long long get(uint32_t i) const {
    if (SMEM) return (long long)(((unsigned long long)(uint32_t)hi[i] << 32) | lo[i]);
    return g[i];
  }
  __device__ __forceinline__ void set(uint32_t i, long long v) const {
    if (SMEM) { lo[i] = (uint32_t)(unsigned long long)v; hi[i] = (int32_t)((unsigned long long)v >> 32); }
    else g[i] = v;
  }
  __device__ __forceinline__ void add(uint32_t i, long long d) const {
    if (SMEM) {
      const unsigned long long ud = (unsigned long long)d;
      const uint32_t dl = (uint32_t)ud;
      const int32_t dh = (int32_t)(ud >> 32);
      const uint32_t old = atomicAdd(lo + i, dl);
      const int32_t up = dh + ((uint32_t)(old + dl) < old ? 1 : 0);
      if (up != 0) atomicAdd(hi + i, up);
    } else {
      atomicAdd(reinterpret_cast<unsigned long long*>(g + i), (unsigned long long)d);
    }
  }
};

// one attempt's decision from its site energy: bit 1 accepted, bit 2 took an acceptance draw,
// bit 4 its acceptance draw is the next window's first (lane 31; decided there)
__device__ __forceinline__ int decide(long long e, uint32_t f, double u_acc, double kT, double inv_kT, int lane) {
  const double Es = (double)e * kUnfix;
  const double dG = f != 0 ? -Es : Es;
  if (dG <= 0.0) return 1;
  if (lane == 31) return 4;
  return (metropolis(dG, kT, inv_kT, u_acc) ? 1 : 0) | 2;
}

// add the flips of G to the energies of their neighbours: `t` of `nt` threads, kUpd items per
// thread per pass, every load of a pass in flight before the first add
template <bool SMEM>
__device__ __forceinline__ void scatter_flips(const Flips& G, const SysParams& P, uint32_t off, uint32_t cap,
                                              const uint32_t* __restrict__ es_nl, const long long* __restrict__ D,
                                              const float4* __restrict__ hpos, const Energies<SMEM>& E, double cut2,
                                              double reach2, uint32_t t, uint32_t nt) {
  const uint32_t total = G.start[G.n];
  for (uint32_t base = 0; base < total; base += nt * kUpd) {
    uint32_t tv[kUpd], fv[kUpd];
    long long dv[kUpd];
#pragma unroll
    for (int u = 0; u < kUpd; ++u) {
      const uint32_t it = base + (uint32_t)u * nt + t;
      uint32_t lo = 0;
#pragma unroll
      for (uint32_t step = 16; step > 0; step >>= 1)
        if (G.start[lo + step] <= it) lo += step;
      const bool ok = it < total;
      const size_t k = ok ? (size_t)(off + G.site[lo]) * cap + (it - G.start[lo]) : 0;
      tv[u] = es_nl[k];
      dv[u] = D[k];
      fv[u] = ok ? lo : 32u;
    }
#pragma unroll
    for (int u = 0; u < kUpd; ++u) {
      if (fv[u] == 32u) continue;
      const int sg = G.sign[fv[u]];
      long long d = sg > 0 ? dv[u] : -dv[u];
      if (sg == 0) {
        const uint32_t h = off + G.site[fv[u]];
        d = flip_delta(P, dist2(P, hpos[h], hpos[tv[u]]), G.qo[fv[u]], G.qn[fv[u]], cut2, reach2);
      }
      E.add(tv[u] - off, d);
    }
  }
}

// Per window w (two barriers):
//   X  all warps: M of window w and corr of window w from the flips of window w-1 (not yet in E);
//      warp 0 reads E and the charge states of its sites (E holds every flip before window w-1)
//   R  warp 0 resolves window w; warps 1.. scatter window w-1's flips into E meanwhile
template <bool SMEM>
__global__ void __launch_bounds__(kWalkThreads) k_sweep_walk(const SysParams* __restrict__ sp,
                                                             const uint32_t* __restrict__ head_slot,
                                                             const float4* __restrict__ hpos, float* __restrict__ charge,
                                                             const uint32_t* __restrict__ es_nl,
                                                             const uint32_t* __restrict__ es_cnt,
                                                             const long long* __restrict__ D, uint32_t cap,
                                                             long long* __restrict__ Eg, uint8_t* __restrict__ flag_g,
                                                             uint32_t* __restrict__ rng_io, double* __restrict__ out,
                                                             uint32_t only) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ Flips F[2];
  __shared__ Window W;
  __shared__ uint32_t s_dep;
  const uint32_t r = (only == SOUP_NONE_U32) ? blockIdx.x : only;
  const SysParams& P = sp[r];
  const uint32_t H = P.nheads;
  if (H == 0 || !P.es_on) return;
  const uint32_t off = P.head_off;
  const Energies<SMEM> E{reinterpret_cast<uint32_t*>(smem), reinterpret_cast<int32_t*>(smem + 4 * (size_t)H), Eg + off};
  uint8_t* flag = SMEM ? smem + 8 * (size_t)H : flag_g + off;
  const float qd = (float)P.d_q;
  // flag: 0 neutral, 1 charged with the deprotonated charge, 2 charged with another value
  for (uint32_t h = threadIdx.x; h < H; h += kWalkThreads) {
    if (SMEM) E.set(h, Eg[off + h]);
    const float q = charge[head_slot[off + h]];
    flag[h] = q == 0.f ? 0 : (q == qd ? 1 : 2);
  }
  const int lane = threadIdx.x & 31;
  const bool chain = threadIdx.x < 32;
  if (chain) {
    F[0].start[lane + 1] = 0xFFFFFFFFu;
    F[1].start[lane + 1] = 0xFFFFFFFFu;
    W.corr[lane] = 0;
    if (lane == 0) { F[0].n = F[1].n = 0; F[0].start[0] = F[1].start[0] = 0; W.done = 0; W.nq = 0; s_dep = 0; }
  }
  const double kT = P.d_kT, inv_kT = 1.0 / P.d_kT;
  const double dGintr = kT * 2.302585092994046 * (P.d_pka - P.d_ph);
  const double cut2 = P.d_rc * P.d_rc, reach = P.d_rcattr + P.d_wc, reach2 = reach * reach;
  // pairs beyond both cutoffs contribute exactly nothing; the FP32 screen keeps a wide margin
  const float nr = (float)(fmax(P.d_rc, reach) * 1.001 + 1e-3);
  const float near2 = nr * nr;
  const float bx = (float)P.d_box[0], by = (float)P.d_box[1], bz = (float)P.d_box[2];
  const float ibx = 1.f / bx, iby = 1.f / by, ibz = 1.f / bz;
  const uint32_t s0 = rng_io[r];

  // warp 0: lane l holds draw base+l (A) and base+32+l (B)
  Draw A{}, B{};
  uint32_t attempts = 0, consumed = 0, accepted = 0, dcount = 0;
  double dsum = 0.0;
  Lcg j32{1u, 0u};
  long long e = 0;
  uint32_t f = 0;
  if (chain) {
    const Lcg j = lcg_pow((uint32_t)lane + 1u);
    j32 = lcg_pow(32u);
    const uint32_t sa = j.a * s0 + j.c;
    draw_from(A, sa, H, off, hpos, es_cnt);
    draw_from(B, j32.a * sa + j32.c, H, off, hpos, es_cnt);
    W.site[lane] = A.site; W.x[lane] = A.x; W.y[lane] = A.y; W.z[lane] = A.z;
  }
  __syncthreads();

  for (uint32_t wnd = 0;; ++wnd) {
    Flips& Fc = F[wnd & 1];          // this window's flips
    const Flips& Fp = F[(wnd + 1) & 1];   // the previous window's
    // ---- X ----
    if (chain) {
      e = E.get(A.site);
      f = flag[A.site];
    }
    // pairs within reach are queued and then evaluated in FP64 one per thread, so no warp runs the
    // FP64 path more than once per pass
    for (uint32_t t = threadIdx.x; t < 1024u + 32u * Fp.n; t += kWalkThreads) {
      if (t < 1024u) {
        const int k = (int)(t >> 5), q = (int)(t & 31);
        if (k >= q) continue;
        long long m = kSameSite;
        if (W.site[k] != W.site[q]) {
          m = 0;
          float dx = W.x[q] - W.x[k], dy = W.y[q] - W.y[k], dz = W.z[q] - W.z[k];
          dx -= rintf(dx * ibx) * bx;
          dy -= rintf(dy * iby) * by;
          dz -= rintf(dz * ibz) * bz;
          if (dx * dx + dy * dy + dz * dz < near2) {
            const uint32_t slot = atomicAdd(&W.nq, 1u);
            if (slot < kQueue) W.queue[slot] = (uint16_t)t;
            else m = std_delta(P, dist2(P, make_float4(W.x[k], W.y[k], W.z[k], 0.f),
                                        make_float4(W.x[q], W.y[q], W.z[q], 0.f)), qd, cut2, reach2);
          }
        }
        W.M[k][q] = m;
      } else {
        const uint32_t g = (t - 1024u) >> 5, q = (t - 1024u) & 31u;
        if (Fp.site[g] == W.site[q]) continue;        // a site's own flip leaves its E alone
        float dx = W.x[q] - Fp.x[g], dy = W.y[q] - Fp.y[g], dz = W.z[q] - Fp.z[g];
        dx -= rintf(dx * ibx) * bx;
        dy -= rintf(dy * iby) * by;
        dz -= rintf(dz * ibz) * bz;
        if (dx * dx + dy * dy + dz * dz < near2) {
          const uint32_t slot = atomicAdd(&W.nq, 1u);
          if (slot < kQueue) W.queue[slot] = (uint16_t)t;
          else corr_term(P, Fp, W, g, q, qd, cut2, reach2);
        }
      }
    }
    __syncthreads();
    {
      const uint32_t nq = W.nq < kQueue ? W.nq : kQueue;
      for (uint32_t i = threadIdx.x; i < nq; i += kWalkThreads) {
        const uint32_t t = W.queue[i];
        if (t < 1024u) {
          const uint32_t k = t >> 5, q = t & 31u;
          W.M[k][q] = std_delta(P, dist2(P, make_float4(W.x[k], W.y[k], W.z[k], 0.f),
                                         make_float4(W.x[q], W.y[q], W.z[q], 0.f)), qd, cut2, reach2);
        } else {
          corr_term(P, Fp, W, (t - 1024u) >> 5, (t - 1024u) & 31u, qd, cut2, reach2);
        }
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) W.nq = 0;
    if (W.done) break;
    // ---- R ----
    if (chain) {
      e += W.corr[lane];
      const double u_acc = __shfl_down_sync(0xffffffffu, A.u, 1);   // lane l: draw base+l+1 (l < 31)
      int res = decide(e, f, u_acc, kT, inv_kT, lane);
      uint32_t acc_m = __ballot_sync(0xffffffffu, res & 1), need_m = __ballot_sync(0xffffffffu, res & 2);
      uint32_t nxt_m = __ballot_sync(0xffffffffu, res & 4);
      uint32_t chg_m = __ballot_sync(0xffffffffu, f != 0), f2_m = __ballot_sync(0xffffffffu, f == 2);
      uint32_t dirty = 0, flipped = 0;
      uint32_t p = 0, nf = 0, my_nf = 0, my_fo = 0;
      long long my_e = 0;
      bool done = false;
      while (p < 32) {
        if (attempts == H) { done = true; break; }
        const uint32_t bit = 1u << p;
        const long long mq = W.M[p][lane];            // used by the lanes after p when p flips
        if (dirty & bit) {
          if (lane == (int)p) res = decide(e, f, u_acc, kT, inv_kT, lane);
          acc_m = __ballot_sync(0xffffffffu, res & 1);
          need_m = __ballot_sync(0xffffffffu, res & 2);
          nxt_m = __ballot_sync(0xffffffffu, res & 4);
        }
        if (nxt_m & bit) break;
        ++attempts;
        if (acc_m & bit) {
          const uint32_t fo = (chg_m & bit) ? ((f2_m & bit) ? 2u : 1u) : 0u;
          if (lane == (int)p) {
            flag[A.site] = fo != 0 ? 0 : 1;
            my_nf = nf; my_fo = fo; my_e = e;
          }
          flipped |= bit;
          // every later lane takes the flip into its own site energy (or charge state)
          bool ch = false, dup = false;
          if (lane > (int)p) {
            if (mq == kSameSite) {
              f = fo != 0 ? 0 : 1;
              ch = dup = true;
            } else if (fo != 2) {
              if (mq != 0) { e += fo == 0 ? mq : -mq; ch = true; }
            } else {
              const float qo = charge[head_slot[off + W.site[p]]];
              const long long m = flip_delta(P, dist2(P, make_float4(W.x[p], W.y[p], W.z[p], 0.f),
                                                      make_float4(A.x, A.y, A.z, 0.f)), qo, 0.f, cut2, reach2);
              if (m != 0) { e += m; ch = true; }
            }
          }
          dirty |= __ballot_sync(0xffffffffu, ch);
          if (__ballot_sync(0xffffffffu, dup)) {
            chg_m = __ballot_sync(0xffffffffu, f != 0);
            f2_m = __ballot_sync(0xffffffffu, f == 2);
          }
          ++nf;
        }
        p += (need_m & bit) ? 2 : 1;
      }
      const uint32_t c = p;
      consumed += c;
      // ---- this window's flip records, in lane (= attempt) order ----
      const bool mine = (flipped >> lane) & 1u;
      if (mine) {
        Fc.site[my_nf] = A.site;
        Fc.qo[my_nf] = my_fo == 0 ? 0.f : (my_fo == 1 ? qd : charge[head_slot[off + A.site]]);
        Fc.qn[my_nf] = my_fo != 0 ? 0.f : qd;
        Fc.sign[my_nf] = my_fo == 0 ? 1 : (my_fo == 1 ? -1 : 0);
        Fc.x[my_nf] = A.x; Fc.y[my_nf] = A.y; Fc.z[my_nf] = A.z;
        ++accepted;
        if (my_fo == 0) { dsum += (double)my_e * kUnfix - dGintr; ++dcount; }
      }
      uint32_t v = mine ? A.cnt : 0u;
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += y;
      }
      if (mine) Fc.start[my_nf + 1] = v;
      if (lane >= (int)nf) Fc.start[lane + 1] = 0xFFFFFFFFu;
      if (lane == 0) { Fc.n = nf; W.done = done ? 1u : 0u; }
      // ---- slide the draws by the c this window consumed; publish the next window's sites ----
      const int src = lane + (int)c;
      const Draw a1 = shfl_draw(A, src & 31);
      const Draw b1 = shfl_draw(B, src & 31);
      if (src < 32) {
        A = a1;
        B = b1;
      } else {
        A = b1;
        draw_from(B, j32.a * b1.st + j32.c, H, off, hpos, es_cnt);
      }
      __syncwarp();
      W.site[lane] = A.site; W.x[lane] = A.x; W.y[lane] = A.y; W.z[lane] = A.z;
      W.corr[lane] = 0;
    } else {
      scatter_flips(Fp, P, off, cap, es_nl, D, hpos, E, cut2, reach2, threadIdx.x - 32u, kWalkThreads - 32u);
    }
    __syncthreads();
  }
  // the charges from the final states (a head still in state 2 keeps its own value)
  uint32_t dep = 0;
  for (uint32_t h = threadIdx.x; h < H; h += kWalkThreads) {
    const uint8_t fl = flag[h];
    if (fl != 2) charge[head_slot[off + h]] = fl == 0 ? 0.f : qd;
    dep += fl != 0;
  }
  for (int o = 16; o > 0; o >>= 1) dep += __shfl_xor_sync(0xffffffffu, dep, o);
  if (lane == 0) atomicAdd(&s_dep, dep);
  if (chain) {
    for (int o = 16; o > 0; o >>= 1) {
      accepted += __shfl_xor_sync(0xffffffffu, accepted, o);
      dcount += __shfl_xor_sync(0xffffffffu, dcount, o);
      dsum += __shfl_xor_sync(0xffffffffu, dsum, o);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const Lcg j = lcg_pow(consumed);
    rng_io[r] = j.a * s0 + j.c;
    out[4 * r + 0] = (double)H;
    out[4 * r + 1] = (double)accepted;
    out[4 * r + 2] = dcount > 0 ? dsum / kT / dcount : 0.0;
    out[4 * r + 3] = (double)s_dep;
  }
}

// head positions by head index for the sweep
__global__ void k_gather_heads(const uint32_t* __restrict__ head_slot, uint32_t H, const float4* __restrict__ pos,
                               float4* __restrict__ hpos) {
  const uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h < H) hpos[h] = pos[head_slot[h]];
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
  k_gather_heads<<<(b.H + 255) / 256, 256, 0, b.stream>>>(b.head_slot, b.H, b.pos, b.head_pos);
  k_sweep_init<<<(unsigned)(((uint64_t)b.H * 32 + 255) / 256), 256, 0, b.stream>>>(
      b.sp, b.head_sys, b.head_slot, b.H, b.pos, b.charge, b.es_nl, b.es_cnt, b.es_cap, b.head_e, b.head_d, replica);
  const unsigned grid = replica == SOUP_NONE_U32 ? b.R : 1;
  const size_t smem = 9 * (size_t)hmax;
  if (smem <= 200 * 1024) {
    k_sweep_walk<true><<<grid, kWalkThreads, smem, b.stream>>>(b.sp, b.head_slot, b.head_pos, b.charge, b.es_nl,
                                                               b.es_cnt, b.head_d, b.es_cap, b.head_e, b.head_flag,
                                                               b.prot_rng_dev, b.sweep_out, replica);
  } else {
    k_sweep_walk<false><<<grid, kWalkThreads, 0, b.stream>>>(b.sp, b.head_slot, b.head_pos, b.charge, b.es_nl,
                                                             b.es_cnt, b.head_d, b.es_cap, b.head_e, b.head_flag,
                                                             b.prot_rng_dev, b.sweep_out, replica);
  }
  prof_end(b);
}

void sweep_prepare(Batch& b) {
  SOUP_CUDA_TRY(cudaFuncSetAttribute(k_sweep_walk<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
}

}  // namespace soup

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
//   k_sweep_draws, k_sweep_band (all SMs) precompute every draw's site and, for every pair of draws
//                 up to 63 apart, the change of the later draw's site energy when the earlier flips.
//   k_sweep_walk  (one thread-block cluster per replica) walks the chain in windows of 32 draws on
//                 warp 0 of CTA 0, a draw per lane: every lane decides at once, the changes of the
//                 window's interacting flips are applied speculatively from the band, and the lanes
//                 decide again until nothing changes.  The other CTAs add each window's flips to E
//                 (global memory) from the D rows while warp 0 resolves the next window.  (Polling the
//                 handoff flags with relaxed loads and one acquire fence after them was measured
//                 slower: 0.583 against 0.442 ms per step.)
// E and D are fixed point (2^-40 kT, int64): integer adds commute, so E does not depend on the
// order the updates land in and every run is reproducible.  E_h is the FP64 sum rounded once, each
// D_ht is rounded once, so the energies agree with the reference's FP64 sums to about 1e-11 kT (the
// decisions agree unless a draw lands that close to its threshold).
// The energies are FP64 with JavaScript rounding of the minimum image, as the reference's.
#include "soup_internal.h"

#include <cooperative_groups.h>
namespace cg = cooperative_groups;

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

// u < exp(-dG/kT) for dG > 0, with dG = g 2^-40 (g the fixed-point energy, g > 0) and u = v 2^-32 (v the
// draw's 32 output bits).  The walk's chain takes this decision once per attempt and again whenever
// an earlier flip of its window changes the site's energy, so the common case runs in FP32 and
// integers: for -dG/kT > -20 an FP32 estimate decides when u is more than 2e-5 (relative) away from
// it.  The estimate's error is below 6.8e-6: the exponent -g * (2^-40 / kT) carries three FP32
// roundings (1.8e-7 relative, 3.6e-6 absolute at |x| < 20), __expf adds at most 2 + 1.173 |x| ulp
// (3.0e-6), the draw's and the margin's roundings 2e-7.  Below -20 only u < 1e-8 can pass (v < 43).
// Otherwise, and near the threshold, FP64 decides: exp(-dG / kT) with dG and u exactly as the
// reference forms them.
__device__ __forceinline__ bool metropolis(long long g, uint32_t v, float x_scale, double kT) {
  const float xf = -(float)g * x_scale;
  if (xf > -20.f) {
    const float est = __expf(xf);
    const float u = (float)v * 2.3283064365386963e-10f;
    if (u < est * (1.f - 2e-5f)) return true;
    if (u > est * (1.f + 2e-5f)) return false;
  } else if (v >= 43u) {
    return false;                 // u >= 1.0012e-8 > exp(-20 + 4e-6)
  }
  return (double)v * 2.3283064365386963e-10 < exp(-((double)g * kUnfix) / kT);
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
// pcgNext's output bits; the draw is u = bits / 2^32
__device__ __forceinline__ uint32_t pcg_bits(uint32_t v) {
  v = ((v >> ((v >> 28u) + 4u)) ^ v) * 277803737u;
  return (v >> 22u) ^ v;
}

constexpr int kWalkThreads = 512;
constexpr uint32_t kEndOfSweep = 0xFFFFFFFFu;   // s_cflag once the sweep is over
constexpr uint32_t kSpinLimit = 1u << 25;       // default polls of a handoff flag before the walk gives up

// cluster-scope release / acquire on 32-bit words in shared memory (own or a peer CTA's, by generic
// address): the handoffs between the walking warp and the CTAs that scatter its flips
__device__ __forceinline__ uint32_t ld_acquire_cluster(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.cluster.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ uint32_t ld_relaxed_cluster(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.cluster.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_cluster(uint32_t* p, uint32_t v) {
  asm volatile("st.release.cluster.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void red_add_release_cluster(uint32_t* p, uint32_t v) {
  asm volatile("red.release.cluster.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
constexpr int kUpd = 8;
constexpr uint32_t kBand = 64;    // a band row: one draw's changes on the sites of the next 63 draws
constexpr uint32_t kRing = 64;    // band rows the walk keeps in shared memory
constexpr int kWalkSmemMax = 224 * 1024;   // the ring, the energies and the charge states

// Replica r's band rows and draw sites start at these offsets: a sweep consumes at most 2 H draws
// (an attempt takes a site draw and at most one acceptance draw) and a window reads kBand rows ahead.
__device__ __forceinline__ size_t band_row0(const SysParams& P, uint32_t r) {
  return 2 * (size_t)P.head_off + (size_t)kBand * r;
}
__device__ __forceinline__ size_t draw_site0(const SysParams& P, uint32_t r) {
  return 2 * (size_t)P.head_off + 2 * (size_t)kBand * r;
}
// the reference's min(H - 1, floor(u H)) for u = bits / 2^32: u H = bits H / 2^32 is exact in FP64
// (bits H < 2^52), so its floor is the high word of the 64-bit product, always below H
__device__ __forceinline__ uint32_t site_of(uint32_t bits, uint32_t H) {
  return (uint32_t)(((uint64_t)bits * H) >> 32);
}

// the site every draw of the sweep's stream selects when it is a site draw (all SMs)
__global__ void k_sweep_draws(const SysParams* __restrict__ sp, const uint32_t* __restrict__ rng_io, uint32_t only,
                              uint32_t* __restrict__ draw_site) {
  const uint32_t r = only == SOUP_NONE_U32 ? blockIdx.y : only;
  const SysParams& P = sp[r];
  const uint32_t H = P.nheads;
  if (H == 0 || !P.es_on) return;
  const uint32_t d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= 2 * H + 2 * kBand) return;
  const Lcg j = lcg_pow(d + 1u);
  draw_site[draw_site0(P, r) + d] = site_of(pcg_bits(j.a * rng_io[r] + j.c), H);
}

// band[d][k] (k = 1..63): the change of draw d+k's site energy when draw d's site deprotonates
// (std_delta, the value the D rows hold), or kSameSite when both draws select one site; band[d][0]
// is the mask of the row's nonzero entries.  Positions are fixed during a sweep, so the whole band is
// known before the walk starts.  A warp per row.
__device__ __forceinline__ long long band_entry(const SysParams& P, const float4* __restrict__ hpos,
                                                const uint32_t* __restrict__ ds, uint32_t row, uint32_t k) {
  if (k == 0) return 0;
  const uint32_t a = ds[row], c = ds[row + k];
  if (a == c) return kSameSite;
  const float4 pa = hpos[P.head_off + a], pc = hpos[P.head_off + c];
  const double cut2 = P.d_rc * P.d_rc, reach = P.d_rcattr + P.d_wc, reach2 = reach * reach;
  // pairs beyond both cutoffs change nothing; the FP32 screen keeps a wide margin
  const float nr = (float)(fmax(P.d_rc, reach) * 1.001 + 1e-3);
  float dx = pc.x - pa.x, dy = pc.y - pa.y, dz = pc.z - pa.z;
  dx -= rintf(dx * P.inv_box[0]) * P.box[0];
  dy -= rintf(dy * P.inv_box[1]) * P.box[1];
  dz -= rintf(dz * P.inv_box[2]) * P.box[2];
  if (dx * dx + dy * dy + dz * dz >= nr * nr) return 0;
  return std_delta(P, dist2(P, pa, pc), (float)P.d_q, cut2, reach2);
}
__global__ void k_sweep_band(const SysParams* __restrict__ sp, const float4* __restrict__ hpos,
                             const uint32_t* __restrict__ draw_site, uint32_t only, long long* __restrict__ band) {
  const uint32_t r = only == SOUP_NONE_U32 ? blockIdx.y : only;
  const SysParams& P = sp[r];
  const uint32_t H = P.nheads;
  if (H == 0 || !P.es_on) return;
  const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  if (w >= 2 * (uint64_t)H + kBand) return;   // whole warps
  const uint32_t row = (uint32_t)w;
  const uint32_t* ds = draw_site + draw_site0(P, r);
  const long long m0 = band_entry(P, hpos, ds, row, lane), m1 = band_entry(P, hpos, ds, row, lane + 32u);
  const uint32_t b0 = __ballot_sync(0xffffffffu, m0 != 0), b1 = __ballot_sync(0xffffffffu, m1 != 0);
  long long* out = band + (band_row0(P, r) + row) * kBand;
  out[lane] = lane == 0 ? (long long)(((unsigned long long)b1 << 32) | b0) : m0;
  out[lane + 32u] = m1;
}

// one draw of the stream as a lane holds it: the LCG state that produced it, its output bits, the
// site it selects when it is a site draw and that site's head-list length
struct Draw {
  uint32_t st, v, site, cnt;
};
__device__ __forceinline__ void draw_from(Draw& d, uint32_t st, uint32_t H, uint32_t off,
                                          const uint32_t* __restrict__ es_cnt) {
  d.st = st;
  d.v = pcg_bits(st);
  d.site = site_of(d.v, H);
  d.cnt = es_cnt[off + d.site];
}
__device__ __forceinline__ Draw shfl_draw(const Draw& d, int src) {
  Draw o;
  o.st = __shfl_sync(0xffffffffu, d.st, src);
  o.v = __shfl_sync(0xffffffffu, d.v, src);
  o.site = __shfl_sync(0xffffffffu, d.site, src);
  o.cnt = __shfl_sync(0xffffffffu, d.cnt, src);
  return o;
}

// the flips one window accepted: the scatter into E that runs during the next window, and the
// corrections the next window's lanes take before E has them
struct Flips {
  uint32_t site[32];
  uint32_t draw[32];     // the flip's draw in the sweep's stream
  uint32_t start[33];    // prefix of the flipped heads' list lengths; ~0 above the last flip
  float qo[32], qn[32];
  int sign[32];          // +1 deprotonated, -1 protonated, 0 the old charge was another value
  uint32_t n;
};

// The attempt lanes of a window from lane p on: an attempt whose need bit is set takes the next
// draw as its acceptance draw, and the lane after that is an attempt again.  Every run of set need
// bits (restricted to lanes >= p) therefore starts at an attempt, its attempts are the run's even
// offsets, and each of them skips the following lane.  Even offsets are read off the prefix parity
// of the need bits against the parity just before the run (spread over the run by a carry).
__device__ __forceinline__ uint32_t attempt_mask(uint32_t need_m, uint32_t p) {
  const uint32_t range = 0xffffffffu << p;
  const uint32_t x = need_m & range;
  uint32_t px = x;                      // px bit i: parity of x's bits 0..i
  px ^= px << 1;
  px ^= px << 2;
  px ^= px << 4;
  px ^= px << 8;
  px ^= px << 16;
  const uint32_t starts = ((px & ~x) << 1) & x & ~(x << 1);   // runs whose preceding parity is 1
  const uint32_t fill = (x ^ (x + starts)) & x;                 // that parity spread over the run
  const uint32_t even = x & (px ^ fill);                        // the run's even offsets
  return range & ~(even << 1);
}

// one attempt's decision from its site energy: bit 1 accepted, bit 2 took an acceptance draw,
// bit 4 its acceptance draw is the next window's first (lane 31; decided there)
// (dG = E_s for a neutral site, -E_s for a charged one; its sign is the fixed-point value's)
__device__ __forceinline__ int decide(long long e, uint32_t f, uint32_t v_acc, float x_scale, double kT, int lane) {
  const long long g = f != 0 ? -e : e;
  if (g <= 0) return 1;
  if (lane == 31) return 4;
  return (metropolis(g, v_acc, x_scale, kT) ? 1 : 0) | 2;
}

// add the flips of G to the energies of their neighbours (global int64, reductions in L2): `t` of
// `nt` threads of whole warps across the cluster, kUpd items per thread per pass.  An item's flip is
// counted from the flips' list starts held one per lane; every load of a pass is in flight before
// the first add.
__device__ __forceinline__ void scatter_flips(const Flips& G, const SysParams& P, uint32_t off, uint32_t cap,
                                              const uint32_t* __restrict__ es_nl, const long long* __restrict__ D,
                                              const float4* __restrict__ hpos, long long* __restrict__ E, double cut2,
                                              double reach2, uint32_t t, uint32_t nt) {
  const uint32_t total = G.start[G.n], nfl = G.n;
  const uint32_t start_next = G.start[(threadIdx.x & 31u) + 1u];   // lane g: start of flip g + 1
  for (uint32_t base = 0; base < total; base += nt * kUpd) {
    uint32_t tv[kUpd], fv[kUpd];
    long long dv[kUpd];
#pragma unroll
    for (int u = 0; u < kUpd; ++u) fv[u] = 0;
    for (uint32_t g = 0; g < nfl; ++g) {
      const uint32_t sn = __shfl_sync(0xffffffffu, start_next, (int)g);
#pragma unroll
      for (int u = 0; u < kUpd; ++u) fv[u] += sn <= base + (uint32_t)u * nt + t ? 1u : 0u;
    }
#pragma unroll
    for (int u = 0; u < kUpd; ++u) {
      const uint32_t it = base + (uint32_t)u * nt + t;
      const bool ok = it < total;
      const uint32_t lo = fv[u];
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
      atomicAdd(reinterpret_cast<unsigned long long*>(E + (tv[u] - off)), (unsigned long long)d);
    }
  }
}

// band rows [row0, row0 + 32) into the ring, 16 bytes a thread at a time
__device__ __forceinline__ void fetch_rows(long long (*ring)[kBand], const long long* __restrict__ brow, uint32_t row0,
                                           uint32_t t, uint32_t nt) {
  constexpr uint32_t kPairs = kBand / 2;
  for (uint32_t i = t; i < 32u * kPairs; i += nt) {
    const uint32_t row = row0 + i / kPairs, c = i % kPairs;
    reinterpret_cast<longlong2*>(ring[row & (kRing - 1)])[c] =
        reinterpret_cast<const longlong2*>(brow + (size_t)row * kBand)[c];
  }
}

// The D and head-list rows the flips of the draws [d0, d0 + n) would scatter, into L2 (their flips
// are scattered a window or two later): `t` of `nt` threads.  Every prefetched address lies inside
// its row.
__device__ __forceinline__ void prefetch_rows(const SysParams& P, uint32_t r, uint32_t off, uint32_t cap,
                                              const uint32_t* __restrict__ draw_site,
                                              const uint32_t* __restrict__ es_cnt, const uint32_t* __restrict__ es_nl,
                                              const long long* __restrict__ D, uint32_t d0, uint32_t n, uint32_t t,
                                              uint32_t nt) {
  const uint32_t lstep = nt / n, j = t % n, l0 = t / n;
  if (l0 >= lstep) return;
  const uint32_t site = draw_site[draw_site0(P, r) + d0 + j];
  const uint32_t cnt = es_cnt[off + site];
  if (cnt == 0) return;
  const char* drow = reinterpret_cast<const char*>(D + (size_t)(off + site) * cap);
  const char* nrow = reinterpret_cast<const char*>(es_nl + (size_t)(off + site) * cap);
  const uint32_t db = cnt * 8u, nb = cnt * 4u;
  const uint32_t ld = (db + 127u) / 128u + 1u, ln = (nb + 127u) / 128u + 1u;
  for (uint32_t l = l0; l < ld + ln; l += lstep) {
    const char* a = l < ld ? drow + min(l * 128u, db - 1u) : nrow + min((l - ld) * 128u, nb - 1u);
    asm volatile("prefetch.global.L2 [%0];" ::"l"(a));
  }
}

// One cluster per replica.  CTA 0 walks the chain (warp 0) and keeps the charge states and the ring of
// band rows in shared memory; the site energies E live in global memory and every thread of the
// cluster but warp 0 of CTA 0 scatters flips into them.  Per window (two cluster barriers):
//   C  warp 0 reads E and the charge states of its sites (E holds every flip before window w-1)
//      and adds the flips of window w-1 from the band rows in the ring
//   R  warp 0 resolves window w; the rest scatter window w-1's flips into E, and CTA 0's other
//      warps fetch the band rows the next window can need
// Window w's draws are consumed+0..31; the ring holds band rows [consumed - 32, consumed + 32) at C
// (rows of window w-1's flips and of window w's draws) and the fetch during R adds rows
// consumed+32..63, which covers window w+1 (it starts at consumed + 31 or + 32).
__global__ void __launch_bounds__(kWalkThreads) k_sweep_walk(const SysParams* __restrict__ sp,
                                                             const uint32_t* __restrict__ head_slot,
                                                             const float4* __restrict__ hpos, float* __restrict__ charge,
                                                             const uint32_t* __restrict__ es_nl,
                                                             const uint32_t* __restrict__ es_cnt,
                                                             const long long* __restrict__ D, uint32_t cap,
                                                             long long* __restrict__ Eg,
                                                             const long long* __restrict__ band,
                                                             const uint32_t* __restrict__ draw_site,
                                                             uint32_t* __restrict__ rng_io, double* __restrict__ out,
                                                             uint32_t only, uint32_t spin_limit) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ Flips F[2];
  __shared__ Flips Fh;                 // a helper CTA's copy of the flips it scatters
  __shared__ uint32_t s_dep, s_done, s_base;
  __shared__ uint32_t s_cflag, s_scat, s_timeout;   // CTA 0: the handoffs with the helper CTAs
  __shared__ uint32_t s_hv;                         // a helper CTA: the signal its thread 0 read
  cg::cluster_group cluster = cg::this_cluster();
  const uint32_t crank = cluster.block_rank(), csize = cluster.num_blocks();
  const bool lead = crank == 0;
  const uint32_t r = (only == SOUP_NONE_U32) ? blockIdx.x / csize : only;
  const SysParams& P = sp[r];
  const uint32_t H = P.nheads;
  if (H == 0 || !P.es_on) return;     // the whole cluster leaves together
  const uint32_t off = P.head_off;
  long long (*ring)[kBand] = reinterpret_cast<long long (*)[kBand]>(smem);
  uint8_t* flag = smem + sizeof(long long) * kRing * kBand;
  long long* E = Eg + off;
  const long long* brow = band + band_row0(P, r) * kBand;
  const float qd = (float)P.d_q;
  const int lane = threadIdx.x & 31;
  const bool chain = lead && threadIdx.x < 32;
  if (lead) {
    // flag: 0 neutral, 1 charged with the deprotonated charge, 2 charged with another value
    for (uint32_t h = threadIdx.x; h < H; h += kWalkThreads) {
      const float q = charge[head_slot[off + h]];
      flag[h] = q == 0.f ? 0 : (q == qd ? 1 : 2);
    }
    fetch_rows(ring, brow, 0, threadIdx.x, kWalkThreads);
    if (threadIdx.x < 32) {
      F[0].start[lane + 1] = 0xFFFFFFFFu;
      F[1].start[lane + 1] = 0xFFFFFFFFu;
      if (lane == 0) {
        F[0].n = F[1].n = 0; F[0].start[0] = F[1].start[0] = 0; s_done = 0; s_base = 0; s_dep = 0;
        s_cflag = 0; s_scat = 0; s_timeout = 0;
      }
    }
  }
  // the lead CTA's window state, read by every CTA of the cluster
  const Flips* lead_F = cluster.map_shared_rank(&F[0], 0);
  uint32_t* lead_cflag = cluster.map_shared_rank(&s_cflag, 0);
  uint32_t* lead_scat = cluster.map_shared_rank(&s_scat, 0);
  uint32_t* lead_timeout = cluster.map_shared_rank(&s_timeout, 0);
  const uint32_t* lead_base = cluster.map_shared_rank(&s_base, 0);
  // scatter threads: every thread of the other CTAs, or CTA 0's warps 1.. when the cluster is one CTA
  // (then they also fetch the band rows, which is all they do otherwise)
  const bool lead_scatters = csize == 1u;
  const uint32_t nscat = lead_scatters ? kWalkThreads - 32u : (csize - 1u) * kWalkThreads;
  const uint32_t tscat = lead ? threadIdx.x - 32u : (crank - 1u) * kWalkThreads + threadIdx.x;
  const double kT = P.d_kT;
  const float x_scale = (float)(kUnfix / P.d_kT);   // -dG/kT per fixed-point unit of dG
  const double dGintr = kT * 2.302585092994046 * (P.d_pka - P.d_ph);
  const double cut2 = P.d_rc * P.d_rc, reach = P.d_rcattr + P.d_wc, reach2 = reach * reach;
  const uint32_t s0 = rng_io[r];

  // warp 0: lane l holds draw consumed+l (A) and consumed+32+l (B)
  Draw A{}, B{};
  uint32_t attempts = 0, consumed = 0, accepted = 0, dcount = 0;
  double dsum = 0.0;
  Lcg j32{1u, 0u};
  long long e = 0;
  uint32_t f = 0, inter_m = 0;
  long long corr = 0;          // the previous window's flips on this lane's site energy
  bool other_prev = false;     // the previous window flipped a head from a non-standard charge
  if (chain) {
    const Lcg j = lcg_pow((uint32_t)lane + 1u);
    j32 = lcg_pow(32u);
    const uint32_t sa = j.a * s0 + j.c;
    draw_from(A, sa, H, off, es_cnt);
    draw_from(B, j32.a * sa + j32.c, H, off, es_cnt);
  }
  cluster.sync();

  // ---- the chain's two phases of a window (warp 0 of CTA 0) ----
  // C: E and the charge states of this window's sites, with the previous window's flips added
  // sig != 0: the helpers' signal for this window, released as soon as the E loads are issued (the
  // release waits for them; the rest of C and the fence then overlap)
  auto chain_C = [&](const Flips& Fp, uint32_t sig) {
      e = (long long)__ldcg(reinterpret_cast<const unsigned long long*>(E + A.site));
      if (sig) {
        __syncwarp();
        if (lane == 0) st_release_cluster(&s_cflag, sig);
      }
      f = flag[A.site];
      // the previous window's flips, accumulated for this window's draws while they were taken; a
      // flip from a charge other than the standard one is rare and evaluated here.  A site's own
      // flip leaves its E alone.
      e += corr;
      if (other_prev)
        for (uint32_t g = 0; g < Fp.n; ++g)
          if (Fp.sign[g] == 0 && Fp.site[g] != A.site)
            e += flip_delta(P, dist2(P, hpos[off + Fp.site[g]], hpos[off + A.site]), Fp.qo[g], Fp.qn[g], cut2, reach2);
      // this lane's flip would change a later lane of the window: its band row's nonzero mask
      const unsigned long long nz = (unsigned long long)ring[(consumed + (uint32_t)lane) & (kRing - 1)][0];
      inter_m = __ballot_sync(0xffffffffu, ((nz >> 1) & ((1ull << (31 - lane)) - 1ull)) != 0);
  };
  // R: resolve the window, record its flips, slide the draws
  auto chain_R = [&](Flips& Fc) {
      const uint32_t v_acc = __shfl_down_sync(0xffffffffu, A.v, 1);   // lane l: draw consumed+l+1 (l < 31)
      int res = decide(e, f, v_acc, x_scale, kT, lane);
      uint32_t acc_m = __ballot_sync(0xffffffffu, res & 1), need_m = __ballot_sync(0xffffffffu, res & 2);
      uint32_t nxt_m = __ballot_sync(0xffffffffu, res & 4);
      uint32_t flipped = 0, p = 0, my_fo = 0;
      long long my_e = 0;
      bool done = false;
      // the next window's draws are consumed+31..63: lane l accumulates the flips' changes of draw
      // consumed+31+l (nc) and lane 31 also of draw consumed+63 (nc2), from the flips' band rows
      long long nc = 0, nc2 = 0;
      bool other = false;
      // the lanes of m flip; no later lane of this window depends on them
      auto commit = [&](uint32_t m) {
        if ((m >> lane) & 1u) {
          flag[A.site] = f != 0 ? 0 : 1;
          my_fo = f; my_e = e;
        }
        flipped |= m;
        for (uint32_t mm = m; mm; mm &= mm - 1u) {
          const uint32_t q = (uint32_t)(__ffs(mm) - 1);
          const uint32_t fq = __shfl_sync(0xffffffffu, f, (int)q);
          if (fq == 2u) { other = true; continue; }
          const long long* row = ring[(consumed + q) & (kRing - 1)];
          const long long v = row[(31u + (uint32_t)lane - q) & (kBand - 1)];
          const long long v2 = row[(63u - q) & (kBand - 1)];
          if (31u + (uint32_t)lane != q && v != kSameSite) nc += fq == 0 ? v : -v;
          if (lane == 31 && v2 != kSameSite) nc2 += fq == 0 ? v2 : -v2;
        }
      };
      // lane q flips and every later lane takes the flip into its own site energy (or charge
      // state), deciding again if that changed
      auto flip_at = [&](uint32_t q) {
        const uint32_t site_q = __shfl_sync(0xffffffffu, A.site, (int)q);
        const uint32_t fo = __shfl_sync(0xffffffffu, f, (int)q);
        commit(1u << q);
        bool ch = false;
        if (lane > (int)q) {
          const long long mq = ring[(consumed + q) & (kRing - 1)][(uint32_t)lane - q];
          if (mq == kSameSite) {
            f = fo != 0 ? 0 : 1;
            ch = true;
          } else if (fo != 2) {
            if (mq != 0) { e += fo == 0 ? mq : -mq; ch = true; }
          } else {
            const float qo = charge[head_slot[off + site_q]];
            const long long m = flip_delta(P, dist2(P, hpos[off + site_q], hpos[off + A.site]), qo, 0.f, cut2, reach2);
            if (m != 0) { e += m; ch = true; }
          }
        }
        if (ch) res = decide(e, f, v_acc, x_scale, kT, lane);
        if (__ballot_sync(0xffffffffu, ch)) {
          acc_m = __ballot_sync(0xffffffffu, res & 1);
          need_m = __ballot_sync(0xffffffffu, res & 2);
          nxt_m = __ballot_sync(0xffffffffu, res & 4);
        }
      };
      // the changes of the flips of lanes X (ascending) on every later lane's site energy or charge
      // state: E_, F_ as they stand before those flips (standard charges only)
      auto apply = [&](uint32_t X, long long& E_, uint32_t& F_) {
        for (uint32_t mm = X; mm; mm &= mm - 1u) {
          const uint32_t q = (uint32_t)(__ffs(mm) - 1);
          const uint32_t fq = __shfl_sync(0xffffffffu, F_, (int)q);
          if ((uint32_t)lane > q) {
            const long long mq = ring[(consumed + q) & (kRing - 1)][(uint32_t)lane - q];
            if (mq == kSameSite) F_ ^= 1u;
            else E_ += fq == 0 ? mq : -mq;
          }
        }
      };
      // the window's flips m, once e and f hold every lane's final energy and state: the charge
      // states (a site drawn twice takes the state its last flip left), the records' values and the
      // next window's corrections, kNcBatch flips' band entries in flight at a time
      auto commit_final = [&](uint32_t m) {
        const bool fl = (m >> lane) & 1u;
        const uint32_t same = __match_any_sync(0xffffffffu, fl ? A.site : (0x80000000u | (uint32_t)lane));
        if (fl) {
          my_fo = f; my_e = e;
          if ((same >> lane) == 1u) flag[A.site] = f != 0 ? 0 : 1;
        }
        flipped |= m;
        constexpr int kNcBatch = 4;
        for (uint32_t mm = m; mm;) {
          uint32_t q[kNcBatch], fq[kNcBatch];
          long long v1[kNcBatch], v2[kNcBatch];
#pragma unroll
          for (int t = 0; t < kNcBatch; ++t) {
            q[t] = mm ? (uint32_t)(__ffs(mm) - 1) : 32u;
            mm &= mm - 1u;
          }
#pragma unroll
          for (int t = 0; t < kNcBatch; ++t) {
            const uint32_t qq = q[t] & 31u;
            fq[t] = __shfl_sync(0xffffffffu, f, (int)qq);
            const long long* row = ring[(consumed + qq) & (kRing - 1)];
            v1[t] = row[(31u + (uint32_t)lane - qq) & (kBand - 1)];
            v2[t] = row[(63u - qq) & (kBand - 1)];
          }
#pragma unroll
          for (int t = 0; t < kNcBatch; ++t) {
            if (q[t] == 32u) continue;
            if (31u + (uint32_t)lane != q[t] && v1[t] != kSameSite) nc += fq[t] == 0 ? v1[t] : -v1[t];
            if (lane == 31 && v2[t] != kSameSite) nc2 += fq[t] == 0 ? v2[t] : -v2[t];
          }
        }
      };
      if (H - attempts > 32u && !__any_sync(0xffffffffu, f == 2u)) {
        // The attempt limit cannot fall inside this window and every charge is a standard one.  From
        // lane p the attempts run up to the first one that takes an acceptance draw, skip that draw,
        // and so on.  The changes of every flip that changes some later lane (inter_m) are applied
        // at once and the lanes decide again; if no lane's attempt, acceptance or deferral changed,
        // that is the window's resolution.  Otherwise every lane up to the first one that changed
        // has its final decision (the flips before it are the real ones), their flips' changes are
        // kept, and the scan goes on behind it.
        uint32_t att_fin = 0, flip_fin = 0;
        for (;;) {
          const uint32_t am = attempt_mask(need_m, p);
          const uint32_t stop = am & nxt_m;                  // lane 31 decides in the next window
          const uint32_t fm = am & acc_m & ~stop;
          const uint32_t hits = inter_m & fm;
          if (!hits) {
            att_fin |= am & ~stop;
            flip_fin |= fm;
            p = stop ? 31u : 32u;
            break;
          }
          long long es = e;
          uint32_t fs = f;
          apply(hits, es, fs);
          const int rs = decide(es, fs, v_acc, x_scale, kT, lane);
          const uint32_t acc2 = __ballot_sync(0xffffffffu, rs & 1), need2 = __ballot_sync(0xffffffffu, rs & 2);
          const uint32_t nxt2 = __ballot_sync(0xffffffffu, rs & 4);
          const uint32_t am2 = attempt_mask(need2, p);
          const uint32_t stop2 = am2 & nxt2, fm2 = am2 & acc2 & ~stop2;
          const uint32_t diff = (am ^ am2) | (fm ^ fm2) | (stop ^ stop2);
          if (!diff) {
            e = es;
            f = fs;
            att_fin |= am & ~stop;
            flip_fin |= fm;
            p = stop ? 31u : 32u;
            break;
          }
          const uint32_t k = (uint32_t)(__ffs(diff) - 1);
          const uint32_t upto = k == 31u ? 0xffffffffu : (2u << k) - 1u;
          att_fin |= am2 & ~stop2 & upto;
          flip_fin |= fm2 & upto;
          apply(inter_m & fm2 & upto, e, f);
          if ((stop2 >> k) & 1u) { p = 31u; break; }
          p = k + ((((am2 & need2) >> k) & 1u) ? 2u : 1u);
          if (p >= 32u) break;
          res = decide(e, f, v_acc, x_scale, kT, lane);
          acc_m = __ballot_sync(0xffffffffu, res & 1);
          need_m = __ballot_sync(0xffffffffu, res & 2);
          nxt_m = __ballot_sync(0xffffffffu, res & 4);
        }
        attempts += __popc(att_fin);
        commit_final(flip_fin);
      } else if (H - attempts > 32u) {
        // a non-standard charge in the window: every flip before the first flip that changes some
        // later lane (inter_m) resolves at once; that flip resolves alone, and the scan starts again
        // behind it.
        while (p < 32u) {
          const uint32_t am = attempt_mask(need_m, p);
          const uint32_t stop = am & nxt_m;                  // lane 31 decides in the next window
          const uint32_t fm = am & acc_m & ~stop;
          const uint32_t hit = inter_m & fm;
          const uint32_t qs = hit ? (uint32_t)(__ffs(hit) - 1) : 32u;
          if (qs == 32u) {
            attempts += __popc(am & ~stop);
            commit(fm);
            p = stop ? 31u : 32u;
            break;
          }
          const uint32_t below = (1u << qs) - 1u;
          attempts += __popc(am & below) + 1u;
          commit(fm & below);
          flip_at(qs);
          p = qs + (((need_m >> qs) & 1u) ? 2u : 1u);
        }
      } else {
        // the last attempts of the sweep: one lane at a time, stopping at the limit
        while (p < 32u) {
          if (attempts == H) { done = true; break; }
          const uint32_t bit = 1u << p;
          if (nxt_m & bit) break;
          ++attempts;
          if (acc_m & bit) flip_at(p);
          p += (need_m & bit) ? 2u : 1u;
        }
      }
      const uint32_t c = p;
      // ---- this window's flip records, in lane (= attempt) order ----
      const bool mine = (flipped >> lane) & 1u;
      const uint32_t nf = __popc(flipped), my_nf = __popc(flipped & ((1u << lane) - 1u));
      if (mine) {
        Fc.site[my_nf] = A.site;
        Fc.draw[my_nf] = consumed + (uint32_t)lane;
        Fc.qo[my_nf] = my_fo == 0 ? 0.f : (my_fo == 1 ? qd : charge[head_slot[off + A.site]]);
        Fc.qn[my_nf] = my_fo != 0 ? 0.f : qd;
        Fc.sign[my_nf] = my_fo == 0 ? 1 : (my_fo == 1 ? -1 : 0);
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
      consumed += c;
      if (lane == 0) { Fc.n = nf; s_done = done ? 1u : 0u; s_base = consumed; }
      // ---- slide the draws by the c this window consumed (31 or 32 unless the sweep is done) ----
      {
        const long long ncs = __shfl_sync(0xffffffffu, nc, (lane + (int)c - 31) & 31);
        const long long nc2s = __shfl_sync(0xffffffffu, nc2, 31);
        corr = (c == 32u && lane == 31) ? nc2s : ncs;
        other_prev = __any_sync(0xffffffffu, other);
      }
      const int src = lane + (int)c;
      const Draw a1 = shfl_draw(A, src & 31);
      const Draw b1 = shfl_draw(B, src & 31);
      if (src < 32) {
        A = a1;
        B = b1;
      } else {
        A = b1;
        draw_from(B, j32.a * b1.st + j32.c, H, off, es_cnt);
      }
  };

  if (csize == 1u) {
    // one CTA: its other warps scatter the previous window's flips and fetch band rows while warp 0
    // resolves, between two CTA barriers a window
    for (uint32_t wnd = 0;; ++wnd) {
      Flips& Fc = F[wnd & 1];
      const Flips& Fp = F[(wnd + 1) & 1];
      if (s_done) break;
      const uint32_t base = s_base;
      if (chain) chain_C(Fp, 0u);
      __syncthreads();
      if (chain) {
        chain_R(Fc);
      } else {
        scatter_flips(Fp, P, off, cap, es_nl, D, hpos, E, cut2, reach2, tscat, nscat);
        fetch_rows(ring, brow, base + 32u, threadIdx.x - 32u, kWalkThreads - 32u);
      }
      __syncthreads();
    }
  } else if (lead) {
    // CTA 0 of a cluster.  Warp 0 signals (s_cflag, a release at cluster scope) once its E reads of
    // window w are done, so the helper CTAs may add window w-1's flips to E, and before window w+1
    // reads E it waits (s_scat) until every helper has.  The other warps fetch the band rows.  No
    // cluster barrier inside the loop.  Measured and dropped: relaying the signal through another
    // warp (it took the release's fence, about 900 cycles, off the chain, but reached the helpers
    // later); E in CTA 0's shared memory (the scatter became remote atomics into one SM, twice as
    // slow as reductions spread over L2); each helper staging the rows of the draws it owns in its
    // shared memory by asynchronous copies (the copies' issue took longer than the L2 reads saved).
    for (uint32_t wnd = 0;; ++wnd) {
      Flips& Fc = F[wnd & 1];
      const Flips& Fp = F[(wnd + 1) & 1];
      if (s_done) {
        if (threadIdx.x == 0) st_release_cluster(&s_cflag, kEndOfSweep);
        break;
      }
      const uint32_t base = s_base;
      if (chain) {
        chain_C(Fp, wnd + 1u);
        __syncwarp();
        chain_R(Fc);
        if (lane == 0) {
          const uint32_t want = (csize - 1u) * (wnd + 1u);
          uint32_t spins = 0;
          while (ld_acquire_cluster(&s_scat) < want) {
            if (++spins > spin_limit) { s_timeout = 1u; s_done = 1u; break; }
          }
        }
        __syncwarp();
      } else {
        fetch_rows(ring, brow, base + 32u, threadIdx.x - 32u, kWalkThreads - 32u);
      }
      __syncthreads();
    }
  } else {
    // a helper CTA: wait for window w's signal, copy window w-1's flips from CTA 0, add them to E,
    // report
    for (uint32_t wnd = 0;; ++wnd) {
      if (threadIdx.x == 0) {
        uint32_t v, spins = 0;
        for (;;) {
          v = ld_acquire_cluster(lead_cflag);
          if (v == kEndOfSweep || v >= wnd + 1u) break;
          if (++spins > spin_limit) { v = kEndOfSweep; atomicExch(lead_timeout, 1u); break; }
        }
        s_hv = v;
      }
      __syncthreads();
      if (s_hv == kEndOfSweep) break;
      const uint32_t* src = reinterpret_cast<const uint32_t*>(lead_F + ((wnd + 1) & 1));
      for (uint32_t i = threadIdx.x; i < sizeof(Flips) / 4; i += kWalkThreads) reinterpret_cast<uint32_t*>(&Fh)[i] = src[i];
      __syncthreads();
      scatter_flips(Fh, P, off, cap, es_nl, D, hpos, E, cut2, reach2, tscat, nscat);
      __syncthreads();
      if (threadIdx.x == 0) red_add_release_cluster(lead_scat, 1u);
      // the rows of the window after the chain's current one (its draws start 31 or 32 later)
      prefetch_rows(P, r, off, cap, draw_site, es_cnt, es_nl, D, ld_relaxed_cluster(lead_base) + 31u, 33u, tscat,
                    nscat);
    }
  }
  if (!lead) {
    cluster.sync();                       // CTA 0's shared memory stays up until every helper is done
    return;
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
  cluster.sync();
  if (threadIdx.x == 0) {
    const Lcg j = lcg_pow(consumed);
    rng_io[r] = j.a * s0 + j.c;
    out[4 * r + 0] = s_timeout ? -1.0 : (double)H;   // -1: a handoff gave up (the host reports it)
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
  if (hmax == 0) return;
  b.launches += 5;
  prof_begin(b, SOUP_K_SWEEP);
  const unsigned ry = replica == SOUP_NONE_U32 ? b.R : 1;
  k_gather_heads<<<(b.H + 255) / 256, 256, 0, b.stream>>>(b.head_slot, b.H, b.pos, b.head_pos);
  k_sweep_init<<<(unsigned)(((uint64_t)b.H * 32 + 255) / 256), 256, 0, b.stream>>>(
      b.sp, b.head_sys, b.head_slot, b.H, b.pos, b.charge, b.es_nl, b.es_cnt, b.es_cap, b.head_e, b.head_d, replica);
  k_sweep_draws<<<dim3((2 * hmax + 2 * kBand + 255) / 256, ry), 256, 0, b.stream>>>(b.sp, b.prot_rng_dev, replica,
                                                                                   b.draw_site);
  k_sweep_band<<<dim3((unsigned)(((uint64_t)(2 * hmax + kBand) * 32 + 255) / 256), ry), 256, 0, b.stream>>>(
      b.sp, b.head_pos, b.draw_site, replica, b.sweep_band);
  // flags (a byte per head) after the ring; one cluster per replica, as wide as the SM count allows
  const size_t smem = sizeof(long long) * kRing * kBand + (((size_t)hmax + 15) & ~(size_t)15);
  const unsigned cs = ry <= 16 ? 8u : (ry <= 32 ? 4u : (ry <= 64 ? 2u : 1u));
  cudaLaunchConfig_t lc = {};
  lc.gridDim = dim3(ry * cs);
  lc.blockDim = dim3(kWalkThreads);
  lc.dynamicSmemBytes = smem;
  lc.stream = b.stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  lc.attrs = attr;
  lc.numAttrs = 1;
  SOUP_CUDA_TRY(cudaLaunchKernelEx(&lc, k_sweep_walk, (const SysParams*)b.sp, (const uint32_t*)b.head_slot,
                                   (const float4*)b.head_pos, b.charge, (const uint32_t*)b.es_nl,
                                   (const uint32_t*)b.es_cnt, (const long long*)b.head_d, b.es_cap, b.head_e,
                                   (const long long*)b.sweep_band, (const uint32_t*)b.draw_site, b.prot_rng_dev,
                                   b.sweep_out, replica,
                                   b.wait_limit ? b.wait_limit : kSpinLimit));
  prof_end(b);
}

uint32_t sweep_max_heads() { return (uint32_t)(kWalkSmemMax - sizeof(long long) * kRing * kBand - 16); }
size_t sweep_band_rows(const Batch& b) { return 2 * (size_t)b.H + (size_t)kBand * b.R; }
size_t sweep_draw_sites(const Batch& b) { return 2 * (size_t)b.H + 2 * (size_t)kBand * b.R; }

void sweep_prepare(Batch& b) {
  SOUP_CUDA_TRY(cudaFuncSetAttribute(k_sweep_walk, cudaFuncAttributeMaxDynamicSharedMemorySize, kWalkSmemMax));
}

}  // namespace soup

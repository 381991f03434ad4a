// kernels_force.cu -- the force: list pair force + bonded terms + wall, the far Debye-Hueckel half,
// and the O(N^2) brute-force twin.
//
// Reference: soup/wgsl/verlet.wgsl:132-149 soup_force_list_main (bondedForce + sum over the list of
// nonbondedSoup), soup/wgsl/step.wgsl:152-193 bondedForce, soup/wgsl/electrostatics-long.wgsl:63-103
// (far half, accumulated), soup/wgsl/wall.wgsl:42-56 (wall, accumulated), step.wgsl:277-292 brute.
//
// TPP threads cooperate on one particle: lane t takes list entries t, t+TPP, ... and bonded terms
// t, t+TPP, ...; the group reduces with shuffles and lane 0 writes the force.  No atomics: every
// particle's force is produced by exactly one group (full list, no Newton-3), so the sum order is
// fixed and the result is run-to-run deterministic.
#include "soup_internal.h"

// four 256-thread blocks per SM (64 registers): the force is latency-bound on its gathers, and the
// fourth block hides more of it than the registers it costs (a few bytes of spill)
#ifndef SOUP_FORCE_MINB
#define SOUP_FORCE_MINB 4
#endif

namespace soup {

namespace {

constexpr int kBlock = 256;
inline unsigned nblocks(uint64_t n, int b = kBlock) { return (unsigned)((n + b - 1) / b); }

// One bonded term of particle (slot k, original id gi), term index t in [0, 13):
//   t < 3         FENE to slot partner t
//   3 <= t < 12   bend to partner-of-partner ((t-3)/3, (t-3)%3), skipping i itself
//   t == 12       FENE tether to the adsorbing catalyst (centerLink)
__device__ __forceinline__ void bonded_term(const Shared& S, const SysParams& P, int t, uint32_t gi, const float4& xi,
                                            const uint32_t* __restrict__ sl, uint32_t owner,
                                            const uint32_t* __restrict__ slots, const uint32_t* __restrict__ slot_of,
                                            const float4* __restrict__ pos, float& fx, float& fy, float& fz) {
  uint32_t other;
  bool fene;
  if (t < 3) { other = sl[t]; fene = true; }
  else if (t < 12) {
    uint32_t m = sl[(t - 3) / 3];
    if (m == SOUP_NONE_U32) return;
    other = slots[3 * slot_of[m] + (t - 3) % 3];
    if (other == gi) return;
    fene = false;
  } else { other = owner; fene = true; }
  if (other == SOUP_NONE_U32) return;
  float4 xo = pos[slot_of[other]];
  float dx = fast_mi(xi.x - xo.x, P.box[0], P.inv_box[0]);
  float dy = fast_mi(xi.y - xo.y, P.box[1], P.inv_box[1]);
  float dz = fast_mi(xi.z - xo.z, P.box[2], P.inv_box[2]);
  float s = bonded_scalar(S, dx * dx + dy * dy + dz * dz, fene);
  fx += s * dx; fy += s * dy; fz += s * dz;
}

// The end of the part of particle k's row a force pass must read.  The row is grouped by build
// distance (k_group_rows): shell 0 within the force's reach r0 = sqrt(rmax2), shells 1..4 the rest of the
// list range in four widths w.  No bead has moved more than dm since the build (the replica's largest
// drift), so a pair of shell s is at least r0 + (s - 1) w - 2 dm apart now, and shell s can hold an
// in-range pair only if (s - 1) w < 2 dm (a margin of 1e-3 sigma covers rounding).  Skipped entries are
// beyond the reach, so the force is the same bits as over the whole row.
__device__ __forceinline__ uint32_t list_force_end(uint32_t k, const uint32_t* __restrict__ nl_cnt,
                                                   const uint4* __restrict__ nl_shell, float drift2, float rmax2,
                                                   float list_range) {
  const uint32_t cnt = nl_cnt[k];
  const float r0 = sqrtf(rmax2), w = (list_range - r0) * 0.25f;
  if (!nl_shell || !(drift2 >= 0.f && drift2 < 1e30f) || !(w > 0.f)) return cnt;
  const float x = (2.0f * sqrtf(drift2) + 1e-3f) / w;
  if (x >= 3.0f) return cnt;
  const uint4 e = nl_shell[k];
  return x < 1.0f ? e.y : (x < 2.0f ? e.z : e.w);
}

// SEL: the particles are the nsel slots sel[] (the heads, after a charge sweep) instead of all N
template <int TPP, bool SEL>
__global__ void __launch_bounds__(256, SOUP_FORCE_MINB) k_force(
    const Shared* __restrict__ Sg, const SysParams* __restrict__ sp, const uint8_t* __restrict__ sysid, uint32_t N,
    const float4* __restrict__ pos, const float* __restrict__ charge, const uint32_t* __restrict__ slots,
    const uint32_t* __restrict__ center, const uint32_t* __restrict__ id, const uint32_t* __restrict__ slot_of,
    const uint32_t* __restrict__ nl, const uint32_t* __restrict__ nl_cnt, const uint4* __restrict__ nl_shell,
    const uint32_t* __restrict__ drift_bits, uint32_t cap, float4* __restrict__ force,
    const uint32_t* __restrict__ sel, uint32_t nsel) {
  __shared__ Shared S;
  for (int w = threadIdx.x; w < (int)(sizeof(Shared) / 4); w += blockDim.x)
    reinterpret_cast<uint32_t*>(&S)[w] = reinterpret_cast<const uint32_t*>(Sg)[w];
  __syncthreads();
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t g = gtid / TPP;
  const int lane = (int)(gtid % TPP);
  const bool active = SEL ? g < nsel : g < N;
  const uint32_t k = SEL ? (active ? sel[g] : 0u) : g;
  float fx = 0.f, fy = 0.f, fz = 0.f;
  if (active) {
    const uint32_t rs = sysid[k];
    const SysParams& Pg = sp[rs];
    const PairP P = PairP::of(Pg);
    const PairLean L = PairLean::of(S, Pg);
    const float4 xi = pos[k];
    const int ki = (int)xi.w;
    const float qi = charge[k];
    const bool qi_nz = qi != 0.f;
    const bool needq = qi_nz || (S.cls[ki] == 1u && P.acid > 0.f);
    const float rmax2 = S.rmax2;
    const uint32_t cnt = list_force_end(k, nl_cnt, nl_shell, __uint_as_float(drift_bits[rs]), rmax2, Pg.list_range);
    const uint32_t* row = nl + (size_t)k * cap;
    const PairW* prow = &S.pw[ki * SOUP_KMAX];
    // a particle at least the interaction reach inside every face has its in-range neighbours at
    // their stored (wrapped) coordinates: the minimum image is the plain difference there (fast_mi
    // returns it unchanged), and an entry beyond the reach by the plain difference is beyond it by the
    // minimum image too.  Decided per warp, so that whole warps skip the image.
    const float reach = sqrtf(rmax2) + 1e-3f;
    const bool inside = __all_sync(__activemask(), xi.x >= reach && xi.x <= P.box[0] - reach && xi.y >= reach &&
                                                   xi.y <= P.box[1] - reach && xi.z >= reach && xi.z <= P.box[2] - reach);
    // lane takes entries [c*4*TPP + 4*lane, +4): one 16-byte load (rows are 32-byte aligned); the
    // next chunk's load is issued before the current chunk is evaluated
    constexpr uint32_t CH = 4 * TPP;
    uint32_t base = 4u * (uint32_t)lane;
    uint4 nxt = base < cnt ? __ldg(reinterpret_cast<const uint4*>(row + base)) : make_uint4(k, k, k, k);
    for (; base < cnt; base += CH) {
      const uint4 jj = nxt;
      if (base + CH < cnt) nxt = __ldg(reinterpret_cast<const uint4*>(row + base + CH));
      const uint32_t jv[4] = {jj.x, base + 1 < cnt ? jj.y : k, base + 2 < cnt ? jj.z : k, base + 3 < cnt ? jj.w : k};
      float4 xj[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) xj[e] = __ldg(pos + jv[e]);
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        float dx = xi.x - xj[e].x, dy = xi.y - xj[e].y, dz = xi.z - xj[e].z;
        if (!inside) {
          dx = fast_mi(dx, P.box[0], P.inv_box[0]);
          dy = fast_mi(dy, P.box[1], P.inv_box[1]);
          dz = fast_mi(dz, P.box[2], P.inv_box[2]);
        }
        const float r2 = dx * dx + dy * dy + dz * dz;
        if (r2 >= rmax2 || r2 < 1e-12f) continue;
        const int kj = (int)xj[e].w;
        const float qj = needq ? __ldg(charge + jv[e]) : 0.f;
        const float sc = pair_lean(prow[kj], L, r2, qi_nz, qi, qj);
        fx += sc * dx; fy += sc * dy; fz += sc * dz;
      }
    }
    // bonded terms (bondedForce), spread over the group
    uint32_t sl[3] = {slots[3 * k], slots[3 * k + 1], slots[3 * k + 2]};
    uint32_t owner = center[k];
    if ((sl[0] & sl[1] & sl[2] & owner) != SOUP_NONE_U32) {
      const uint32_t gi = id[k];
      for (int t = lane; t < 13; t += TPP) bonded_term(S, Pg, t, gi, xi, sl, owner, slots, slot_of, pos, fx, fy, fz);
    }
  }
#pragma unroll
  for (int o = TPP / 2; o > 0; o >>= 1) {
    fx += __shfl_xor_sync(0xffffffffu, fx, o);
    fy += __shfl_xor_sync(0xffffffffu, fy, o);
    fz += __shfl_xor_sync(0xffffffffu, fz, o);
  }
  if (active && lane == 0) {
    const SysParams& P = sp[sysid[k]];
    if (P.wall_r > 0.f) {   // wall.wgsl:42-56
      const float4 xi = pos[k];
      float d0 = xi.x - P.box[0] * 0.5f, d1 = xi.y - P.box[1] * 0.5f, d2 = xi.z - P.box[2] * 0.5f;
      float r = sqrtf(d0 * d0 + d1 * d1 + d2 * d2);
      if (r > P.wall_r) {
        float w = -P.wall_k * (r - P.wall_r) / fmaxf(r, 1e-6f);
        fx += w * d0; fy += w * d1; fz += w * d2;
      }
    }
    force[k] = make_float4(fx, fy, fz, 0.f);
  }
}

// The list force with the pair maths evaluated only on in-range entries, every lane busy.  In k_force
// a warp runs the pair maths whenever any of its lanes holds an in-range entry, which at the skins in
// use is nearly every entry, with about half the lanes idle.  Here each lane owns one particle (its
// list row) and works in rounds: it screens its next four entries (index, gather, minimum image,
// squared distance), the warp compacts the in-range ones owner-major (lane 0's first, each lane's in
// list order) into shared memory, every lane evaluates pairs lane, lane + 32, .. of the compacted
// set, and each owner then adds sc * d for its own pairs in list order with its own separations.  So
// every particle accumulates exactly the terms k_force<1>'s lane does, in the same order and with the
// same arithmetic, and the force is bit-identical to k_force<1>'s.
//
// A warp whose particles all lie at least the interaction reach inside every face of one replica's box
// skips the minimum image: for such a particle every neighbour within the reach has its stored
// (wrapped) coordinates within the reach too, and an entry whose direct separation is beyond the
// reach is beyond it under the minimum image as well.  Per-pair numbers that depend on the replica are
// the owner's: a warp whose particles span replicas evaluates each owner's pairs on the owner's lane.
constexpr int kWBlock = 128;
constexpr int kWRound = 4;                      // entries a lane screens per round
constexpr int kWPairs = 32 * kWRound;           // in-range pairs of one warp round, at most
struct WarpPairs {
  float r2[kWPairs];
  float qj[kWPairs];
  uint32_t ko[kWPairs];                         // neighbour kind | owner lane << 8
  float sc[kWPairs];
  float oq[32];                                 // owner charge
  uint32_t okind[32];                           // owner kind | owner charge nonzero << 8
};

// six 128-thread blocks per SM: 80 registers, no spills (64 registers spill the round's arrays)
#ifndef SOUP_FORCE_W_MINB
#define SOUP_FORCE_W_MINB 6
#endif
template <bool SEL>
__global__ void __launch_bounds__(kWBlock, SOUP_FORCE_W_MINB) k_force_w(
    const Shared* __restrict__ Sg, const SysParams* __restrict__ sp, const uint8_t* __restrict__ sysid, uint32_t N,
    const float4* __restrict__ pos, const float* __restrict__ charge, const uint32_t* __restrict__ slots,
    const uint32_t* __restrict__ center, const uint32_t* __restrict__ id, const uint32_t* __restrict__ slot_of,
    const uint32_t* __restrict__ nl, const uint32_t* __restrict__ nl_cnt, const uint4* __restrict__ nl_shell,
    const uint32_t* __restrict__ drift_bits, uint32_t cap, float4* __restrict__ force,
    const uint32_t* __restrict__ sel, uint32_t nsel) {
  __shared__ Shared S;
  __shared__ WarpPairs W[kWBlock / 32];
  for (int w = threadIdx.x; w < (int)(sizeof(Shared) / 4); w += blockDim.x)
    reinterpret_cast<uint32_t*>(&S)[w] = reinterpret_cast<const uint32_t*>(Sg)[w];
  __syncthreads();
  WarpPairs& wp = W[threadIdx.x >> 5];
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t lt = (1u << lane) - 1u;
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = SEL ? g < nsel : g < N;
  const uint32_t k = SEL ? (active ? sel[g] : 0u) : (active ? g : 0u);
  const uint32_t rs = sysid[k];
  const SysParams& Pg = sp[rs];
  const PairP P = PairP::of(Pg);
  const PairLean L = PairLean::of(S, Pg);
  const float4 xi = pos[k];
  const int ki = (int)xi.w;
  const float qi = charge[k];
  const bool qi_nz = qi != 0.f;
  const bool needq = qi_nz || (S.cls[ki] == 1u && P.acid > 0.f);
  const float rmax2 = S.rmax2;
  const uint32_t cnt =
      active ? list_force_end(k, nl_cnt, nl_shell, __uint_as_float(drift_bits[rs]), rmax2, Pg.list_range) : 0u;
  const uint32_t* row = nl + (size_t)k * cap;
  wp.oq[lane] = qi;
  wp.okind[lane] = (uint32_t)ki | (qi_nz ? 0x100u : 0u);
  const bool uni = __all_sync(0xffffffffu, rs == __shfl_sync(0xffffffffu, rs, 0));
  const float reach = sqrtf(rmax2) + 1e-3f;
  const bool inside = !active || (xi.x >= reach && xi.x <= P.box[0] - reach && xi.y >= reach &&
                                  xi.y <= P.box[1] - reach && xi.z >= reach && xi.z <= P.box[2] - reach);
  const bool direct = uni && __all_sync(0xffffffffu, inside);
  float fx = 0.f, fy = 0.f, fz = 0.f;
  uint4 nxt = cnt > 0 ? __ldg(reinterpret_cast<const uint4*>(row)) : make_uint4(k, k, k, k);
  for (uint32_t base = 0;; base += kWRound) {
    if (!__any_sync(0xffffffffu, base < cnt)) break;
    const uint4 jj = nxt;
    if (base + kWRound < cnt) nxt = __ldg(reinterpret_cast<const uint4*>(row + base + kWRound));
    const uint32_t jv[4] = {base < cnt ? jj.x : k, base + 1 < cnt ? jj.y : k, base + 2 < cnt ? jj.z : k,
                            base + 3 < cnt ? jj.w : k};
    float4 xj[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) xj[e] = __ldg(pos + jv[e]);
    float dx[4], dy[4], dz[4], r2[4];
    bool in[4];
    uint32_t c = 0;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      if (direct) {
        dx[e] = xi.x - xj[e].x; dy[e] = xi.y - xj[e].y; dz[e] = xi.z - xj[e].z;
      } else {
        dx[e] = fast_mi(xi.x - xj[e].x, P.box[0], P.inv_box[0]);
        dy[e] = fast_mi(xi.y - xj[e].y, P.box[1], P.inv_box[1]);
        dz[e] = fast_mi(xi.z - xj[e].z, P.box[2], P.inv_box[2]);
      }
      r2[e] = dx[e] * dx[e] + dy[e] * dy[e] + dz[e] * dz[e];
      in[e] = base + e < cnt && r2[e] < rmax2 && r2[e] >= 1e-12f;
      c += in[e] ? 1u : 0u;
    }
    // owner-major offsets of this round's in-range pairs
    uint32_t incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= (uint32_t)o) incl += t;
    }
    const uint32_t first = incl - c;
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    uint32_t p = first;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      if (in[e]) {
        wp.r2[p] = r2[e];
        wp.qj[p] = needq ? __ldg(charge + jv[e]) : 0.f;
        wp.ko[p] = (uint32_t)xj[e].w | (lane << 8);
        ++p;
      }
    }
    __syncwarp();
    if (uni) {
      for (uint32_t q = lane; q < total; q += 32u) {
        const uint32_t ko = wp.ko[q];
        const uint32_t o = ko >> 8, kj = ko & 0xffu;
        const uint32_t ok = wp.okind[o];
        const uint32_t kio = ok & 0xffu;
        wp.sc[q] = pair_lean(S.pw[kio * SOUP_KMAX + kj], L, wp.r2[q], (ok >> 8) != 0u, wp.oq[o], wp.qj[q]);
      }
    } else {
      const PairW* prow = &S.pw[ki * SOUP_KMAX];
      for (uint32_t q = first; q < incl; ++q)
        wp.sc[q] = pair_lean(prow[wp.ko[q] & 0xffu], L, wp.r2[q], qi_nz, qi, wp.qj[q]);
    }
    __syncwarp();
    p = first;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      if (in[e]) {
        const float sc = wp.sc[p++];
        fx += sc * dx[e]; fy += sc * dy[e]; fz += sc * dz[e];
      }
    }
    __syncwarp();
  }
  if (active) {
    // bonded terms (bondedForce), all on the particle's lane
    uint32_t sl[3] = {slots[3 * k], slots[3 * k + 1], slots[3 * k + 2]};
    uint32_t owner = center[k];
    if ((sl[0] & sl[1] & sl[2] & owner) != SOUP_NONE_U32) {
      const uint32_t gi = id[k];
      for (int t = 0; t < 13; ++t) bonded_term(S, Pg, t, gi, xi, sl, owner, slots, slot_of, pos, fx, fy, fz);
    }
    if (Pg.wall_r > 0.f) {   // wall.wgsl:42-56
      float d0 = xi.x - Pg.box[0] * 0.5f, d1 = xi.y - Pg.box[1] * 0.5f, d2 = xi.z - Pg.box[2] * 0.5f;
      float r = sqrtf(d0 * d0 + d1 * d1 + d2 * d2);
      if (r > Pg.wall_r) {
        float w = -Pg.wall_k * (r - Pg.wall_r) / fmaxf(r, 1e-6f);
        fx += w * d0; fy += w * d1; fz += w * d2;
      }
    }
    force[k] = make_float4(fx, fy, fz, 0.f);
  }
}

// soup/wgsl/electrostatics-long.wgsl:63-82 soup_es_force_far_main, a warp per head.
// positions and charges of the heads by head index (x, y, z, q): the far half reads one 16-byte
// record per list entry instead of a slot lookup followed by two gathers
__global__ void k_gather_xq(const uint32_t* __restrict__ head_slot, uint32_t H, const float4* __restrict__ pos,
                            const float* __restrict__ charge, float4* __restrict__ xq) {
  const uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= H) return;
  const uint32_t k = head_slot[h];
  const float4 p = pos[k];
  xq[h] = make_float4(p.x, p.y, p.z, charge[k]);
}

__global__ void __launch_bounds__(256) k_es_far(const SysParams* __restrict__ sp, const uint32_t* __restrict__ head_slot,
                                                const uint32_t* __restrict__ head_sys, uint32_t H,
                                                const float4* __restrict__ xq, const uint32_t* __restrict__ es_nl,
                                                const uint32_t* __restrict__ es_cnt, uint32_t cap,
                                                float4* __restrict__ force) {
  const uint32_t h = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (h >= H) return;   // warp-uniform
  const SysParams& P = sp[head_sys[h]];
  const float4 xi = xq[h];
  const float qi = xi.w;
  if (qi == 0.f || P.es_A == 0.f) return;
  float fx = 0.f, fy = 0.f, fz = 0.f;
  const uint32_t cnt = es_cnt[h];
  const uint32_t* row = es_nl + (size_t)h * cap;
  auto add = [&](const float4& xj) {
    const float qj = xj.w;
    if (qj == 0.f) return;
    const float dx = fast_mi(xi.x - xj.x, P.box[0], P.inv_box[0]);
    const float dy = fast_mi(xi.y - xj.y, P.box[1], P.inv_box[1]);
    const float dz = fast_mi(xi.z - xj.z, P.box[2], P.inv_box[2]);
    const float r2 = dx * dx + dy * dy + dz * dz;
    const float rinv = rsqrtf(r2);
    const float r = r2 * rinv;
    if (r < P.es_split || r >= P.es_rc) return;   // esForceFar (electrostatics.wgsl:87-90)
    const float u = P.es_A * __expf(-P.es_kappa * r) * rinv;
    const float sc = qi * qj * (u * (rinv + P.es_kappa) - P.es_fc) * rinv;
    fx += sc * dx; fy += sc * dy; fz += sc * dz;
  };
  for (uint32_t s = (uint32_t)lane; s < cnt; s += 32u) add(__ldg(xq + __ldg(row + s)));
  for (int o = 16; o > 0; o >>= 1) {
    fx += __shfl_xor_sync(0xffffffffu, fx, o);
    fy += __shfl_xor_sync(0xffffffffu, fy, o);
    fz += __shfl_xor_sync(0xffffffffu, fz, o);
  }
  if (lane == 0) {
    const uint32_t ks = head_slot[h];
    float4 f = force[ks];
    force[ks] = make_float4(f.x + fx, f.y + fy, f.z + fz, 0.f);
  }
}

// soup/wgsl/step.wgsl:277-292 + electrostatics-long.wgsl:88-103 + wall: every pair of the replica.
__global__ void __launch_bounds__(128) k_force_brute(
    const Shared* __restrict__ Sg, const SysParams* __restrict__ sp, const uint8_t* __restrict__ sysid, uint32_t N,
    const float4* __restrict__ pos, const float* __restrict__ charge, const uint32_t* __restrict__ slots,
    const uint32_t* __restrict__ center, const uint32_t* __restrict__ id, const uint32_t* __restrict__ slot_of,
    float4* __restrict__ force) {
  __shared__ Shared S;
  for (int w = threadIdx.x; w < (int)(sizeof(Shared) / 4); w += blockDim.x)
    reinterpret_cast<uint32_t*>(&S)[w] = reinterpret_cast<const uint32_t*>(Sg)[w];
  __syncthreads();
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  const SysParams& P = sp[sysid[k]];
  const PairLean L = PairLean::of(S, P);
  const float4 xi = pos[k];
  const int ki = (int)xi.w;
  const float qi = charge[k];
  float fx = 0.f, fy = 0.f, fz = 0.f;
  for (uint32_t j = P.slot_off; j < P.slot_off + P.n; ++j) {
    if (j == k) continue;
    const float4 xj = pos[j];
    const float dx = fast_mi(xi.x - xj.x, P.box[0], P.inv_box[0]);
    const float dy = fast_mi(xi.y - xj.y, P.box[1], P.inv_box[1]);
    const float dz = fast_mi(xi.z - xj.z, P.box[2], P.inv_box[2]);
    const float r2 = dx * dx + dy * dy + dz * dz;
    if (r2 < 1e-12f) continue;
    const int kj = (int)xj.w;
    const float qj = charge[j];
    if (r2 < S.rmax2) {
      const float sc = pair_lean(S.pw[ki * SOUP_KMAX + kj], L, r2, qi != 0.f, qi, qj);
      fx += sc * dx; fy += sc * dy; fz += sc * dz;
    }
    const float qq = qi * qj;
    if (qq != 0.f && P.es_A != 0.f) {
      const float r = sqrtf(r2);
      if (r >= P.es_split && r < P.es_rc) {
        const float u = P.es_A * __expf(-P.es_kappa * r) / r;
        const float s = qq * (u * (1.0f / r + P.es_kappa) - P.es_fc) / r;
        fx += s * dx; fy += s * dy; fz += s * dz;
      }
    }
  }
  uint32_t sl[3] = {slots[3 * k], slots[3 * k + 1], slots[3 * k + 2]};
  uint32_t owner = center[k];
  const uint32_t gi = id[k];
  for (int t = 0; t < 13; ++t) bonded_term(S, P, t, gi, xi, sl, owner, slots, slot_of, pos, fx, fy, fz);
  if (P.wall_r > 0.f) {
    float d0 = xi.x - P.box[0] * 0.5f, d1 = xi.y - P.box[1] * 0.5f, d2 = xi.z - P.box[2] * 0.5f;
    float r = sqrtf(d0 * d0 + d1 * d1 + d2 * d2);
    if (r > P.wall_r) {
      float w = -P.wall_k * (r - P.wall_r) / fmaxf(r, 1e-6f);
      fx += w * d0; fy += w * d1; fz += w * d2;
    }
  }
  force[k] = make_float4(fx, fy, fz, 0.f);
}

void launch_force_w(Batch& b, bool heads) {
  if (heads) {
    if (b.H == 0) return;
    k_force_w<true><<<nblocks(b.H, kWBlock), kWBlock, 0, b.stream>>>(
        b.shared, b.sp, b.sysid, b.N, b.pos, b.charge, b.slots, b.center, b.id, b.slot_of, b.nl, b.nl_cnt, b.prune ? b.nl_shell : nullptr, b.drift_bits, b.list_cap,
        b.force, b.head_slot, b.H);
    return;
  }
  k_force_w<false><<<nblocks(b.N, kWBlock), kWBlock, 0, b.stream>>>(
      b.shared, b.sp, b.sysid, b.N, b.pos, b.charge, b.slots, b.center, b.id, b.slot_of, b.nl, b.nl_cnt, b.prune ? b.nl_shell : nullptr, b.drift_bits, b.list_cap,
      b.force, nullptr, 0u);
}

template <int TPP>
void launch_force_tpp(Batch& b, bool heads) {
  if (heads) {
    if (b.H == 0) return;
    k_force<TPP, true><<<nblocks((uint64_t)b.H * TPP, 256), 256, 0, b.stream>>>(
        b.shared, b.sp, b.sysid, b.N, b.pos, b.charge, b.slots, b.center, b.id, b.slot_of, b.nl, b.nl_cnt, b.prune ? b.nl_shell : nullptr, b.drift_bits, b.list_cap,
        b.force, b.head_slot, b.H);
    return;
  }
  k_force<TPP, false><<<nblocks((uint64_t)b.N * TPP, 256), 256, 0, b.stream>>>(
      b.shared, b.sp, b.sysid, b.N, b.pos, b.charge, b.slots, b.center, b.id, b.slot_of, b.nl, b.nl_cnt, b.prune ? b.nl_shell : nullptr, b.drift_bits, b.list_cap,
      b.force, nullptr, 0u);
}

}  // namespace

void launch_force(Batch& b) {
  prof_begin(b, SOUP_K_FORCE);
  launch_force_list(b);
  prof_end(b);
  if (b.H > 0) {
    prof_begin(b, SOUP_K_ES_FAR);
    launch_es_far(b);
    prof_end(b);
  }
}

void launch_force_list(Batch& b, bool heads) {
  b.launches += 1;
  if (b.queued) {   // the warp-compacted kernel: one lane per particle whatever tpp says
    launch_force_w(b, heads);
    return;
  }
  switch (b.tpp) {
    case 1: launch_force_tpp<1>(b, heads); break;
    case 2: launch_force_tpp<2>(b, heads); break;
    case 16: launch_force_tpp<16>(b, heads); break;
    case 32: launch_force_tpp<32>(b, heads); break;
    case 8: launch_force_tpp<8>(b, heads); break;
    default: launch_force_tpp<4>(b, heads); break;
  }
}

// after a charge sweep: only the heads' forces depend on charges (when only heads are charged and
// the polar class is the heads' kind alone), so they alone are recomputed, with the same arithmetic;
// timed with the sweep it completes (the force group keeps whole passes only)
void launch_force_heads(Batch& b) {
  prof_begin(b, SOUP_K_SWEEP);
  launch_force_list(b, true);
  if (b.H > 0) launch_es_far(b);
  prof_end(b);
}

void launch_es_far(Batch& b) {
  if (b.H == 0) return;
  b.launches += 2;
  k_gather_xq<<<nblocks(b.H), kBlock, 0, b.stream>>>(b.head_slot, b.H, b.pos, b.charge, b.head_xq);
  k_es_far<<<nblocks((uint64_t)b.H * 32, 256), 256, 0, b.stream>>>(b.sp, b.head_slot, b.head_sys, b.H, b.head_xq,
                                                                   b.es_nl, b.es_cnt, b.es_cap, b.force);
}

void launch_force_brute(Batch& b) {
  b.launches += 1;
  k_force_brute<<<nblocks(b.N, 128), 128, 0, b.stream>>>(b.shared, b.sp, b.sysid, b.N, b.pos, b.charge, b.slots,
                                                         b.center, b.id, b.slot_of, b.force);
}

}  // namespace soup

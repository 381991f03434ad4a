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

// SEL: the particles are the nsel slots sel[] (the heads, after a charge sweep) instead of all N
template <int TPP, bool SEL>
__global__ void __launch_bounds__(256, SOUP_FORCE_MINB) k_force(
    const Shared* __restrict__ Sg, const SysParams* __restrict__ sp, const uint8_t* __restrict__ sysid, uint32_t N,
    const float4* __restrict__ pos, const float* __restrict__ charge, const uint32_t* __restrict__ slots,
    const uint32_t* __restrict__ center, const uint32_t* __restrict__ id, const uint32_t* __restrict__ slot_of,
    const uint32_t* __restrict__ nl, const uint32_t* __restrict__ nl_cnt, uint32_t cap, float4* __restrict__ force,
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
    const SysParams& Pg = sp[sysid[k]];
    const PairP P = PairP::of(Pg);
    const float4 xi = pos[k];
    const int ki = (int)xi.w;
    const float qi = charge[k];
    const bool needq = (qi != 0.f) || (S.cls[ki] == 1u && P.acid > 0.f);
    const float rmax2 = S.rmax2;
    const uint32_t cnt = nl_cnt[k];
    const uint32_t* row = nl + (size_t)k * cap;
    const PairConst* prow = &S.pair[ki * SOUP_KMAX];
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
        const float dx = fast_mi(xi.x - xj[e].x, P.box[0], P.inv_box[0]);
        const float dy = fast_mi(xi.y - xj[e].y, P.box[1], P.inv_box[1]);
        const float dz = fast_mi(xi.z - xj[e].z, P.box[2], P.inv_box[2]);
        const float r2 = dx * dx + dy * dy + dz * dz;
        if (r2 >= rmax2 || r2 < 1e-12f) continue;
        const int kj = (int)xj[e].w;
        const float qj = needq ? __ldg(charge + jv[e]) : 0.f;
        const float sc = pair_scalar(S, P, prow[kj], r2, ki, kj, qi, qj);
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

// The same list force with the pair maths taken off the screening path.  In k_force a warp runs the
// pair maths whenever any of its lanes holds an in-range entry, which at a skin of 0.8 is nearly
// every chunk, so the out-of-range half of the list pays for it too.  Here each lane screens its
// entries (index, gather, minimum image, squared distance) and pushes the in-range ones -- their
// separation, the neighbour's charge and kind -- onto its own ring in shared memory; the warp then
// evaluates the rings' heads together, every lane on a pair of its own particle.  A ring is first in,
// first out in list order, so every lane accumulates exactly the terms k_force's lane does, in the
// same order, and the force is bit-identical to k_force's.
//
// Ring layout: entry s of lane l at [s][l], 16 bytes (dx, dy, dz, qj) plus one byte (kj), so a row of
// the warp's pushes or pops touches each bank once.  After each chunk of 4 entries a lane holds at
// most kQD - 4 + 4 entries: the warp evaluates min(count) rounds with every lane busy, and more
// rounds (lanes with empty rings idle) only when some ring could not take the next chunk.
constexpr int kQD = 16;
constexpr int kQBlock = 256;
constexpr size_t kQSmem = (size_t)(kQBlock / 32) * kQD * 32 * (sizeof(float4) + 1);

template <int TPP, bool SEL>
__global__ void __launch_bounds__(kQBlock, 3) k_force_q(
    const Shared* __restrict__ Sg, const SysParams* __restrict__ sp, const uint8_t* __restrict__ sysid, uint32_t N,
    const float4* __restrict__ pos, const float* __restrict__ charge, const uint32_t* __restrict__ slots,
    const uint32_t* __restrict__ center, const uint32_t* __restrict__ id, const uint32_t* __restrict__ slot_of,
    const uint32_t* __restrict__ nl, const uint32_t* __restrict__ nl_cnt, uint32_t cap, float4* __restrict__ force,
    const uint32_t* __restrict__ sel, uint32_t nsel) {
  __shared__ Shared S;
  extern __shared__ float4 qbuf[];
  for (int w = threadIdx.x; w < (int)(sizeof(Shared) / 4); w += blockDim.x)
    reinterpret_cast<uint32_t*>(&S)[w] = reinterpret_cast<const uint32_t*>(Sg)[w];
  __syncthreads();
  const int wib = threadIdx.x >> 5, l32 = threadIdx.x & 31;
  float4* qv = qbuf + (size_t)wib * kQD * 32 + l32;
  uint8_t* qk = reinterpret_cast<uint8_t*>(qbuf + (size_t)(kQBlock / 32) * kQD * 32) + (size_t)wib * kQD * 32 + l32;
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t g = gtid / TPP;
  const int lane = (int)(gtid % TPP);
  const bool active = SEL ? g < nsel : g < N;
  const uint32_t k = SEL ? (active ? sel[g] : 0u) : (active ? g : 0u);
  const SysParams& Pg = sp[sysid[k]];
  const PairP P = PairP::of(Pg);
  const float4 xi = pos[k];
  const int ki = (int)xi.w;
  const float qi = charge[k];
  const bool needq = (qi != 0.f) || (S.cls[ki] == 1u && P.acid > 0.f);
  const float rmax2 = S.rmax2;
  const uint32_t cnt = active ? nl_cnt[k] : 0u;
  const uint32_t* row = nl + (size_t)k * cap;
  const PairConst* prow = &S.pair[ki * SOUP_KMAX];
  float fx = 0.f, fy = 0.f, fz = 0.f;
  uint32_t head = 0, tail = 0;
  auto pop = [&]() {
    const uint32_t s = head & (kQD - 1);
    const float4 e = qv[s * 32];
    const int kj = qk[s * 32];
    ++head;
    const float r2 = e.x * e.x + e.y * e.y + e.z * e.z;
    const float sc = pair_scalar(S, P, prow[kj], r2, ki, kj, qi, e.w);
    fx += sc * e.x; fy += sc * e.y; fz += sc * e.z;
  };
  constexpr uint32_t CH = 4 * TPP;
  uint32_t base = 4u * (uint32_t)lane;
  uint4 nxt = base < cnt ? __ldg(reinterpret_cast<const uint4*>(row + base)) : make_uint4(k, k, k, k);
  for (;; base += CH) {
    const bool more = base < cnt;
    if (!__any_sync(0xffffffffu, more)) break;
    if (more) {
      const uint4 jj = nxt;
      if (base + CH < cnt) nxt = __ldg(reinterpret_cast<const uint4*>(row + base + CH));
      const uint32_t jv[4] = {jj.x, base + 1 < cnt ? jj.y : k, base + 2 < cnt ? jj.z : k, base + 3 < cnt ? jj.w : k};
      float4 xj[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) xj[e] = __ldg(pos + jv[e]);
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const float dx = fast_mi(xi.x - xj[e].x, P.box[0], P.inv_box[0]);
        const float dy = fast_mi(xi.y - xj[e].y, P.box[1], P.inv_box[1]);
        const float dz = fast_mi(xi.z - xj[e].z, P.box[2], P.inv_box[2]);
        const float r2 = dx * dx + dy * dy + dz * dz;
        if (r2 < rmax2 && r2 >= 1e-12f) {
          const uint32_t s = tail & (kQD - 1);
          qv[s * 32] = make_float4(dx, dy, dz, needq ? __ldg(charge + jv[e]) : 0.f);
          qk[s * 32] = (uint8_t)xj[e].w;
          ++tail;
        }
      }
    }
    // every lane busy for min(count) rounds; more only when a ring could not take the next chunk
    const uint32_t c = tail - head;
    const uint32_t mn = __reduce_min_sync(0xffffffffu, c), mx = __reduce_max_sync(0xffffffffu, c);
    const uint32_t rounds = max(mn, mx > (uint32_t)(kQD - 4) ? mx - (uint32_t)(kQD - 4) : 0u);
    for (uint32_t t = 0; t < rounds; ++t)
      if (tail != head) pop();
  }
  while (__any_sync(0xffffffffu, tail != head))
    if (tail != head) pop();
  if (active) {
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
  for (uint32_t s = lane; s < cnt; s += 32) {
    const float4 xj = __ldg(xq + __ldg(row + s));
    const float qj = xj.w;
    if (qj == 0.f) continue;
    const float dx = fast_mi(xi.x - xj.x, P.box[0], P.inv_box[0]);
    const float dy = fast_mi(xi.y - xj.y, P.box[1], P.inv_box[1]);
    const float dz = fast_mi(xi.z - xj.z, P.box[2], P.inv_box[2]);
    const float r2 = dx * dx + dy * dy + dz * dz;
    const float rinv = rsqrtf(r2);
    const float r = r2 * rinv;
    if (r < P.es_split || r >= P.es_rc) continue;   // esForceFar (electrostatics.wgsl:87-90)
    const float u = P.es_A * __expf(-P.es_kappa * r) * rinv;
    const float sc = qi * qj * (u * (rinv + P.es_kappa) - P.es_fc) * rinv;
    fx += sc * dx; fy += sc * dy; fz += sc * dz;
  }
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
      const float sc = pair_scalar(S, P, S.pair[ki * SOUP_KMAX + kj], r2, ki, kj, qi, qj);
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

template <int TPP>
void launch_force_q(Batch& b, bool heads) {
  static bool attr = false;   // once per process: the rings are dynamic shared memory above 48 KB
  if (!attr) {
    SOUP_CUDA_TRY(cudaFuncSetAttribute(k_force_q<TPP, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kQSmem));
    SOUP_CUDA_TRY(cudaFuncSetAttribute(k_force_q<TPP, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kQSmem));
    attr = true;
  }
  if (heads) {
    if (b.H == 0) return;
    k_force_q<TPP, true><<<nblocks((uint64_t)b.H * TPP, kQBlock), kQBlock, kQSmem, b.stream>>>(
        b.shared, b.sp, b.sysid, b.N, b.pos, b.charge, b.slots, b.center, b.id, b.slot_of, b.nl, b.nl_cnt, b.list_cap,
        b.force, b.head_slot, b.H);
    return;
  }
  k_force_q<TPP, false><<<nblocks((uint64_t)b.N * TPP, kQBlock), kQBlock, kQSmem, b.stream>>>(
      b.shared, b.sp, b.sysid, b.N, b.pos, b.charge, b.slots, b.center, b.id, b.slot_of, b.nl, b.nl_cnt, b.list_cap,
      b.force, nullptr, 0u);
}

template <int TPP>
void launch_force_tpp(Batch& b, bool heads) {
  if (heads) {
    if (b.H == 0) return;
    k_force<TPP, true><<<nblocks((uint64_t)b.H * TPP, 256), 256, 0, b.stream>>>(
        b.shared, b.sp, b.sysid, b.N, b.pos, b.charge, b.slots, b.center, b.id, b.slot_of, b.nl, b.nl_cnt, b.list_cap,
        b.force, b.head_slot, b.H);
    return;
  }
  k_force<TPP, false><<<nblocks((uint64_t)b.N * TPP, 256), 256, 0, b.stream>>>(
      b.shared, b.sp, b.sysid, b.N, b.pos, b.charge, b.slots, b.center, b.id, b.slot_of, b.nl, b.nl_cnt, b.list_cap,
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
  if (b.queued) {
    switch (b.tpp) {
      case 1: launch_force_q<1>(b, heads); break;
      case 2: launch_force_q<2>(b, heads); break;
      default: launch_force_q<4>(b, heads); break;
    }
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

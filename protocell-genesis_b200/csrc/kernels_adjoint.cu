// kernels_adjoint.cu -- the reverse pass of the force + Langevin step.
//
// The forward step is the reference's (soup/wgsl/step.wgsl:89-142 kick-drift / kick-thermostat,
// verlet.wgsl:132-149 + step.wgsl:152-193 + pair.wgsl:168-204 + electrostatics.wgsl:65-99 +
// electrostatics-long.wgsl:63-82 + wall.wgsl:42-56 for the force).  Every force term is central:
// F_i = sum_j s(r_ij) d_ij with d_ij = mi(x_i - x_j).  Its Jacobian applied to a vector g is
//   (J g)_i = sum_j M_ij (g_i - g_j),   M_ij = s I + (s'(r) / r) d d^T,
// symmetric, so the same product serves J^T.  The parameters' partials are
//   d/dtheta (g . F) = sum_i sum_j (ds_ij/dtheta) (g_i . d_ij).
// Parameters (theta): the class-pair attraction depths A[a][b] (apolar, polar, solvent; a <= b),
// k_fene, k_bend, and the Debye screening kappa with the electrostatics cutoff held fixed.
// Cotangents are indexed by ORIGINAL particle index; the kernels read the device's slot order.
#include "soup_internal.h"

namespace soup {

namespace {

constexpr int kBlock = 256;
inline unsigned nblocks(uint64_t n, int b = kBlock) { return (unsigned)((n + b - 1) / b); }
constexpr int kTpp = 4;

// theta index of the class pair (a, b), -1 for the mineral class
__device__ __forceinline__ int depth_index(uint32_t a, uint32_t b) {
  if (a > 2u || b > 2u) return -1;
  if (a > b) { const uint32_t t = a; a = b; b = t; }
  return a == 0 ? (int)b : (a == 1 ? 2 + (int)b : 5);   // (0,0)0 (0,1)1 (0,2)2 (1,1)3 (1,2)4 (2,2)5
}

// M (gi - gj) for one central pair term, accumulated into j3
__device__ __forceinline__ void add_m(float s, float sp, float rinv, float dx, float dy, float dz, float ex, float ey,
                                      float ez, float& jx, float& jy, float& jz) {
  const float c = sp * rinv * (dx * ex + dy * ey + dz * ez);
  jx += s * ex + c * dx;
  jy += s * ey + c * dy;
  jz += s * ez + c * dz;
}

struct ThetaAcc {
  double v[SOUP_DIFF_NPARAM];
  __device__ void zero() {
    for (int p = 0; p < SOUP_DIFF_NPARAM; ++p) v[p] = 0.0;
  }
};

// the nonbonded pair terms of the list (pair_scalar's three terms): s, s' and the parameter partials
template <class PP>
__device__ __forceinline__ void pair_terms(const Shared& S, const PP& P, const PairConst& pc, float r2, int ki, int kj,
                                           float qi, float qj, float gd, float& s, float& sp, ThetaAcc& th) {
  const float rinv = rsqrtf(r2);
  const float r = r2 * rinv;
  const float rinv2 = rinv * rinv;
  s = 0.f;
  sp = 0.f;
  if (r2 < pc.wcut2) {   // WCA: s = 24 eps (2 (b/r)^12 - (b/r)^6) / r^2
    const float s2 = pc.b2 * rinv2;
    const float s6 = s2 * s2 * s2;
    s += 24.0f * S.eps * (2.0f * s6 * s6 - s6) * rinv2;
    sp += 24.0f * S.eps * (-28.0f * s6 * s6 + 8.0f * s6) * rinv2 * rinv;
  }
  if (r >= S.rc_attr && r <= S.rc_attr + S.wc) {   // attraction: s = -scale amp sin(2x) / r
    float scale = pc.attr;
    if (P.acid > 0.f && ((qi != 0.f) != (qj != 0.f)) && S.cls[ki] == 1u && S.cls[kj] == 1u) scale += P.acid;
    const float x = (r - S.rc_attr) * S.attr_k;
    float sn, cs;
    sincosf(2.0f * x, &sn, &cs);
    s -= scale * S.attr_amp * sn * rinv;
    sp -= scale * S.attr_amp * (2.0f * S.attr_k * cs * rinv - sn * rinv2);
    const int p = depth_index(S.cls[ki], S.cls[kj]);
    if (p >= 0) th.v[p] += (double)(-S.attr_amp * sn * rinv) * (double)gd;
  }
  const float qq = qi * qj;
  if (qq != 0.f && r < P.es_split && r < P.es_rc && P.es_A != 0.f) {   // near screened Coulomb
    const float ek = expf(-P.es_kappa * r);
    const float g = P.es_A * ek * (rinv2 + P.es_kappa * rinv) - P.es_fc;
    const float gp = -P.es_A * ek * (2.0f * rinv2 * rinv + 2.0f * P.es_kappa * rinv2 + P.es_kappa * P.es_kappa * rinv);
    s += qq * g * rinv;
    sp += qq * (gp * rinv - g * rinv2);
    const float ekc = expf(-P.es_kappa * P.es_rc);
    th.v[8] += (double)(qq * rinv * (-P.es_kappa * P.es_A * (ek - ekc))) * (double)gd;
  }
}

// the bonded term t of particle (slot k, original id gi) as in bondedForce (step.wgsl:152-193)
__device__ __forceinline__ void bonded_adj(const Shared& S, const SysParams& P, int t, uint32_t gi, const float4& xi,
                                           const uint32_t* sl, uint32_t owner, const uint32_t* __restrict__ slots,
                                           const uint32_t* __restrict__ slot_of, const float4* __restrict__ pos,
                                           const float4* __restrict__ g, const float4& gi4, float& jx, float& jy,
                                           float& jz, ThetaAcc& th) {
  uint32_t other;
  bool fene;
  if (t < 3) { other = sl[t]; fene = true; }
  else if (t < 12) {
    const uint32_t m = sl[(t - 3) / 3];
    if (m == SOUP_NONE_U32) return;
    other = slots[3 * slot_of[m] + (t - 3) % 3];
    if (other == gi) return;
    fene = false;
  } else { other = owner; fene = true; }
  if (other == SOUP_NONE_U32) return;
  const float4 xo = pos[slot_of[other]];
  const float dx = fast_mi(xi.x - xo.x, P.box[0], P.inv_box[0]);
  const float dy = fast_mi(xi.y - xo.y, P.box[1], P.inv_box[1]);
  const float dz = fast_mi(xi.z - xo.z, P.box[2], P.inv_box[2]);
  const float r = fmaxf(sqrtf(dx * dx + dy * dy + dz * dz), 1e-6f);
  const float rinv = 1.0f / r;
  float s, sp;
  if (fene) {
    const float x = r / S.r_inf;
    const float den = 1.0f - x * x;
    s = -S.k_fene / den;
    sp = -S.k_fene * (2.0f * r / (S.r_inf * S.r_inf)) / (den * den);
  } else {
    s = -S.k_bend * (r - S.r_bend) * rinv;
    sp = -S.k_bend * S.r_bend * rinv * rinv;
  }
  const float4 go = g[other];
  add_m(s, sp, rinv, dx, dy, dz, gi4.x - go.x, gi4.y - go.y, gi4.z - go.z, jx, jy, jz);
  const double gd = (double)(gi4.x * dx + gi4.y * dy + gi4.z * dz);
  if (fene) th.v[6] += (double)(s / S.k_fene) * gd;
  else th.v[7] += (double)(s / S.k_bend) * gd;
}

__device__ __forceinline__ void block_theta(const ThetaAcc& th, double* __restrict__ partial) {
  __shared__ double red[kBlock / 32][SOUP_DIFF_NPARAM];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int p = 0; p < SOUP_DIFF_NPARAM; ++p) {
    double v = th.v[p];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[w][p] = v;
  }
  __syncthreads();
  if (threadIdx.x < SOUP_DIFF_NPARAM) {
    double v = 0.0;
    for (int k = 0; k < (int)(blockDim.x / 32); ++k) v += red[k][threadIdx.x];
    partial[(size_t)blockIdx.x * SOUP_DIFF_NPARAM + threadIdx.x] += v;   // this block's running sum over steps
  }
}

// (J g) of the list force (nonbonded + bonded + wall) and the parameter partials, kTpp lanes per
// particle; jg is written (not accumulated), by original index
__global__ void __launch_bounds__(kBlock) k_hvp(const Shared* __restrict__ Sg, const SysParams* __restrict__ sp,
                                                const uint8_t* __restrict__ sysid, uint32_t N,
                                                const float4* __restrict__ pos, const float* __restrict__ charge,
                                                const uint32_t* __restrict__ slots, const uint32_t* __restrict__ center,
                                                const uint32_t* __restrict__ id, const uint32_t* __restrict__ slot_of,
                                                const uint32_t* __restrict__ nl, const uint32_t* __restrict__ nl_cnt,
                                                uint32_t cap, const float4* __restrict__ g, float4* __restrict__ jg,
                                                double* __restrict__ partial) {
  __shared__ Shared S;
  for (int w = threadIdx.x; w < (int)(sizeof(Shared) / 4); w += blockDim.x)
    reinterpret_cast<uint32_t*>(&S)[w] = reinterpret_cast<const uint32_t*>(Sg)[w];
  __syncthreads();
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t k = gtid / kTpp;
  const int lane = (int)(gtid % kTpp);
  ThetaAcc th;
  th.zero();
  float jx = 0.f, jy = 0.f, jz = 0.f;
  const bool active = k < N;
  if (active) {
    const SysParams& Pg = sp[sysid[k]];
    const PairP P = PairP::of(Pg);
    const float4 xi = pos[k];
    const int ki = (int)xi.w;
    const float qi = charge[k];
    const uint32_t gi = id[k];
    const float4 gi4 = g[gi];
    const uint32_t cnt = nl_cnt[k];
    const uint32_t* row = nl + (size_t)k * cap;
    const PairConst* prow = &S.pair[ki * SOUP_KMAX];
    for (uint32_t e = (uint32_t)lane; e < cnt; e += kTpp) {
      const uint32_t j = row[e];
      const float4 xj = pos[j];
      const float dx = fast_mi(xi.x - xj.x, P.box[0], P.inv_box[0]);
      const float dy = fast_mi(xi.y - xj.y, P.box[1], P.inv_box[1]);
      const float dz = fast_mi(xi.z - xj.z, P.box[2], P.inv_box[2]);
      const float r2 = dx * dx + dy * dy + dz * dz;
      if (r2 >= S.rmax2 || r2 < 1e-12f) continue;
      const int kj = (int)xj.w;
      const float qj = charge[j];
      const float gd = gi4.x * dx + gi4.y * dy + gi4.z * dz;
      float s, spr;
      pair_terms(S, P, prow[kj], r2, ki, kj, qi, qj, gd, s, spr, th);
      if (s == 0.f && spr == 0.f) continue;
      const float4 gj = g[id[j]];
      add_m(s, spr, rsqrtf(r2), dx, dy, dz, gi4.x - gj.x, gi4.y - gj.y, gi4.z - gj.z, jx, jy, jz);
    }
    uint32_t sl[3] = {slots[3 * k], slots[3 * k + 1], slots[3 * k + 2]};
    const uint32_t owner = center[k];
    if ((sl[0] & sl[1] & sl[2] & owner) != SOUP_NONE_U32)
      for (int t = lane; t < 13; t += kTpp)
        bonded_adj(S, Pg, t, gi, xi, sl, owner, slots, slot_of, pos, g, gi4, jx, jy, jz, th);
    if (lane == 0 && Pg.wall_r > 0.f) {   // wall: F = w d about the box centre
      const float d0 = xi.x - Pg.box[0] * 0.5f, d1 = xi.y - Pg.box[1] * 0.5f, d2 = xi.z - Pg.box[2] * 0.5f;
      const float r = sqrtf(d0 * d0 + d1 * d1 + d2 * d2);
      if (r > Pg.wall_r) {
        const float rr = fmaxf(r, 1e-6f);
        const float w = -Pg.wall_k * (r - Pg.wall_r) / rr;
        const float wp = -Pg.wall_k * Pg.wall_r / (rr * rr);
        add_m(w, wp, 1.0f / rr, d0, d1, d2, gi4.x, gi4.y, gi4.z, jx, jy, jz);
      }
    }
  }
  for (int o = kTpp / 2; o > 0; o >>= 1) {
    jx += __shfl_xor_sync(0xffffffffu, jx, o);
    jy += __shfl_xor_sync(0xffffffffu, jy, o);
    jz += __shfl_xor_sync(0xffffffffu, jz, o);
  }
  if (active && lane == 0) jg[id[k]] = make_float4(jx, jy, jz, 0.f);
  block_theta(th, partial);
}

// the far screened-Coulomb half (split <= r < rc_es) over the head lists, a warp per head; added
__global__ void __launch_bounds__(kBlock) k_hvp_far(const SysParams* __restrict__ sp, const uint32_t* __restrict__ head_slot,
                                                    const uint32_t* __restrict__ head_sys, uint32_t H,
                                                    const float4* __restrict__ pos, const float* __restrict__ charge,
                                                    const uint32_t* __restrict__ id, const uint32_t* __restrict__ es_nl,
                                                    const uint32_t* __restrict__ es_cnt, uint32_t cap,
                                                    const float4* __restrict__ g, float4* __restrict__ jg,
                                                    double* __restrict__ partial) {
  const uint32_t h = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  ThetaAcc th;
  th.zero();
  float jx = 0.f, jy = 0.f, jz = 0.f;
  uint32_t gi = 0;
  bool live = false;
  if (h < H) {
    const SysParams& P = sp[head_sys[h]];
    const uint32_t ks = head_slot[h];
    const float qi = charge[ks];
    if (qi != 0.f && P.es_A != 0.f) {
      live = true;
      const float4 xi = pos[ks];
      gi = id[ks];
      const float4 gi4 = g[gi];
      const uint32_t cnt = es_cnt[h];
      const uint32_t* row = es_nl + (size_t)h * cap;
      const float ekc = expf(-P.es_kappa * P.es_rc);
      for (uint32_t s = lane; s < cnt; s += 32) {
        const uint32_t j = head_slot[row[s]];
        const float qj = charge[j];
        if (qj == 0.f) continue;
        const float4 xj = pos[j];
        const float dx = fast_mi(xi.x - xj.x, P.box[0], P.inv_box[0]);
        const float dy = fast_mi(xi.y - xj.y, P.box[1], P.inv_box[1]);
        const float dz = fast_mi(xi.z - xj.z, P.box[2], P.inv_box[2]);
        const float r2 = dx * dx + dy * dy + dz * dz;
        const float rinv = rsqrtf(r2);
        const float r = r2 * rinv;
        if (r < P.es_split || r >= P.es_rc) continue;
        const float rinv2 = rinv * rinv;
        const float qq = qi * qj;
        const float ek = expf(-P.es_kappa * r);
        const float gg = P.es_A * ek * (rinv2 + P.es_kappa * rinv) - P.es_fc;
        const float gp = -P.es_A * ek * (2.0f * rinv2 * rinv + 2.0f * P.es_kappa * rinv2 + P.es_kappa * P.es_kappa * rinv);
        const float s_ = qq * gg * rinv;
        const float sp_ = qq * (gp * rinv - gg * rinv2);
        const float4 gj = g[id[j]];
        add_m(s_, sp_, rinv, dx, dy, dz, gi4.x - gj.x, gi4.y - gj.y, gi4.z - gj.z, jx, jy, jz);
        const double gd = (double)(gi4.x * dx + gi4.y * dy + gi4.z * dz);
        th.v[8] += (double)(qq * rinv * (-P.es_kappa * P.es_A * (ek - ekc))) * gd;
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    jx += __shfl_xor_sync(0xffffffffu, jx, o);
    jy += __shfl_xor_sync(0xffffffffu, jy, o);
    jz += __shfl_xor_sync(0xffffffffu, jz, o);
  }
  if (live && lane == 0) {
    float4 a = jg[gi];
    jg[gi] = make_float4(a.x + jx, a.y + jy, a.z + jz, 0.f);
  }
  block_theta(th, partial);
}

__global__ void k_unpermute(const float4* __restrict__ pos, const uint32_t* __restrict__ id, uint32_t N,
                            float4* __restrict__ dst) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < N) dst[id[k]] = pos[k];
}
__global__ void k_scatter_pos(const float4* __restrict__ src, const uint32_t* __restrict__ slot_of, uint32_t N,
                              float4* __restrict__ pos) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) pos[slot_of[i]] = src[i];
}

// one reverse step at time t (see the header of this file and soup_diff_backward):
//   X = A + Jg;  B <- a B + dt X;  A <- l'_{t-1} + X;  g <- coef B   (frozen: B = g = 0)
__global__ void k_adj_update(uint32_t n, float4* __restrict__ A, float4* __restrict__ B, const float4* __restrict__ jg,
                             const float4* __restrict__ ldx, const uint8_t* __restrict__ frozen_o, float a, float dt,
                             float coef, float4* __restrict__ g, float4* __restrict__ xout) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 aa = A[i], j = jg[i];
  const float4 X = make_float4(aa.x + j.x, aa.y + j.y, aa.z + j.z, 0.f);
  if (xout) xout[i] = X;
  float4 b = B[i];
  if (frozen_o[i]) b = make_float4(0.f, 0.f, 0.f, 0.f);
  else b = make_float4(a * b.x + dt * X.x, a * b.y + dt * X.y, a * b.z + dt * X.z, 0.f);
  B[i] = b;
  const float4 l = ldx ? ldx[i] : make_float4(0.f, 0.f, 0.f, 0.f);
  A[i] = make_float4(l.x + X.x, l.y + X.y, l.z + X.z, 0.f);
  g[i] = frozen_o[i] ? make_float4(0.f, 0.f, 0.f, 0.f) : make_float4(coef * b.x, coef * b.y, coef * b.z, 0.f);
}

}  // namespace

void adj_unpermute(Batch& b, float4* dst) {
  b.launches += 1;
  k_unpermute<<<nblocks(b.N), kBlock, 0, b.stream>>>(b.pos, b.id, b.N, dst);
}
void adj_scatter_pos(Batch& b, const float4* src) {
  b.launches += 1;
  k_scatter_pos<<<nblocks(b.N), kBlock, 0, b.stream>>>(src, b.slot_of, b.N, b.pos);
}

// (J g) at the device's current positions and lists, into jg (original order); the parameter
// partials are added to each block's running sums in partial_dev (zeroed by the caller before the
// first step, summed by adj_theta_sum after the last), so the reverse pass never waits on the host
void adj_hvp(Batch& b, const float4* g, float4* jg, double* partial_dev) {
  const unsigned g1 = nblocks((uint64_t)b.N * kTpp, kBlock);
  const unsigned g2 = b.H ? nblocks((uint64_t)b.H * 32, kBlock) : 0;
  b.launches += 1 + (g2 ? 1 : 0);
  k_hvp<<<g1, kBlock, 0, b.stream>>>(b.shared, b.sp, b.sysid, b.N, b.pos, b.charge, b.slots, b.center, b.id, b.slot_of,
                                     b.nl, b.nl_cnt, b.list_cap, g, jg, partial_dev);
  if (g2)
    k_hvp_far<<<g2, kBlock, 0, b.stream>>>(b.sp, b.head_slot, b.head_sys, b.H, b.pos, b.charge, b.id, b.es_nl,
                                           b.es_cnt, b.es_cap, g, jg, partial_dev + (size_t)g1 * SOUP_DIFF_NPARAM);
}
// theta += the blocks' sums, in block order (deterministic)
void adj_theta_sum(Batch& b, const double* partial_dev, double* theta) {
  const size_t np = adj_partial_count(b);
  std::vector<double> host(np);
  SOUP_CUDA_TRY(cudaMemcpyAsync(host.data(), partial_dev, 8 * np, cudaMemcpyDeviceToHost, b.stream));
  SOUP_CUDA_TRY(cudaStreamSynchronize(b.stream));
  for (size_t k = 0; k < np / SOUP_DIFF_NPARAM; ++k)
    for (int p = 0; p < SOUP_DIFF_NPARAM; ++p) theta[p] += host[k * SOUP_DIFF_NPARAM + p];
}
size_t adj_partial_count(const Batch& b) {
  return ((size_t)nblocks((uint64_t)b.N * kTpp, kBlock) + (b.H ? nblocks((uint64_t)b.H * 32, kBlock) : 0)) *
         SOUP_DIFF_NPARAM;
}

void adj_update(Batch& b, uint32_t n, float4* A, float4* B, const float4* jg, const float4* ldx, const uint8_t* frozen_o,
                float a, float dt, float coef, float4* g, float4* xout) {
  b.launches += 1;
  k_adj_update<<<nblocks(n), kBlock, 0, b.stream>>>(n, A, B, jg, ldx, frozen_o, a, dt, coef, g, xout);
}

}  // namespace soup

// kernels_observables.cu -- trajectory observables on the device.
//
// Reference:
//   engine/src/metrics.ts:21-47 densityProfileZ (+ 106-121 dropEscapedZ): bead z histogram split
//     into heads and tails (the soup profiles a copy whose w is 0 for polar kinds and 1 otherwise,
//     soup/src/aggregates.ts:95-109; here a kind mask says which kinds count as heads);
//   soup/src/electrostatics.ts:520-561 pairingStats: per head, the like/unlike contacts with every
//     other head within the contact radius and the charge of its nearest one.
// Both reduce to integer counts (atomics on integers), so the results do not depend on the order the
// threads finish in.  Distances for pairingStats are FP64 with JavaScript rounding of the minimum
// image (mi(d, L) = d - Math.round(d / L) * L), as the reference computes them.
#include <algorithm>
#include <cmath>
#include <vector>

#include "soup_internal.h"

namespace soup {

namespace {

constexpr int kBlock = 256;
inline unsigned nblocks(uint64_t n, int b = kBlock) { return (unsigned)((n + b - 1) / b); }

__device__ __forceinline__ double js_round(double x) {
  const double r = floor(x);
  return (x - r >= 0.5) ? r + 1.0 : r;
}
__device__ __forceinline__ double mi_js(double d, double L) { return d - js_round(d / L) * L; }

// counts[0..bins) heads, counts[bins..2 bins) tails, counts[2 bins] escaped
__global__ void k_profile_z(const float4* __restrict__ pos, uint32_t off, uint32_t n, double box_z, uint32_t bins,
                            uint32_t head_mask, uint32_t* __restrict__ counts) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 p = pos[off + i];
  const double z = (double)p.z;
  if (!(z >= 0.0 && z < box_z)) {
    atomicAdd(&counts[2 * bins], 1u);
    return;
  }
  const double dz = box_z / (double)bins;
  const uint32_t b = min(bins - 1u, (uint32_t)floor(z / dz));
  const uint32_t kind = (uint32_t)(int)p.w;
  const bool head = kind < 32u && ((head_mask >> kind) & 1u);
  atomicAdd(&counts[head ? b : bins + b], 1u);
}

// a warp per head of the replica, over its head list (complete for r < rc_es >= the contact radius)
// out: [0] heads with a neighbour, [1] unlike contacts, [2] like contacts, [3] paired, [4] charged
__global__ void k_pairing(const uint32_t* __restrict__ head_slot, uint32_t head_off, uint32_t nheads,
                          const float4* __restrict__ pos, const float* __restrict__ charge,
                          const uint32_t* __restrict__ es_nl, const uint32_t* __restrict__ es_cnt, uint32_t cap,
                          double bx, double by, double bz, double contact, uint32_t* __restrict__ out) {
  const uint32_t hl = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (hl >= nheads) return;   // warp-uniform
  const uint32_t h = head_off + hl;
  const uint32_t ki = head_slot[h];
  const float4 xi = pos[ki];
  const bool qi0 = charge[ki] == 0.f;
  uint32_t unlike = 0, like = 0;
  double best = INFINITY;
  uint32_t best_h = 0xFFFFFFFFu;
  bool best_unlike = false;
  const uint32_t cnt = es_cnt[h];
  const uint32_t* row = es_nl + (size_t)h * cap;
  for (uint32_t s = lane; s < cnt; s += 32) {
    const uint32_t g = row[s];
    const uint32_t kj = head_slot[g];
    const float4 xj = pos[kj];
    const double dx = mi_js((double)xi.x - (double)xj.x, bx);
    const double dy = mi_js((double)xi.y - (double)xj.y, by);
    const double dz = mi_js((double)xi.z - (double)xj.z, bz);
    const double r = sqrt(dx * dx + dy * dy + dz * dz);
    if (r > contact) continue;
    const bool un = qi0 != (charge[kj] == 0.f);
    if (un) ++unlike; else ++like;
    if (r < best || (r == best && g < best_h)) { best = r; best_h = g; best_unlike = un; }
  }
  // the nearest over the warp (ties: the smaller head index)
  for (int o = 16; o > 0; o >>= 1) {
    const double rb = __shfl_xor_sync(0xffffffffu, best, o);
    const uint32_t hb = __shfl_xor_sync(0xffffffffu, best_h, o);
    const bool ub = __shfl_xor_sync(0xffffffffu, (int)best_unlike, o) != 0;
    if (rb < best || (rb == best && hb < best_h)) { best = rb; best_h = hb; best_unlike = ub; }
    unlike += __shfl_xor_sync(0xffffffffu, unlike, o);
    like += __shfl_xor_sync(0xffffffffu, like, o);
  }
  if (lane == 0) {
    if (unlike + like > 0) atomicAdd(&out[0], 1u);
    atomicAdd(&out[1], unlike);
    atomicAdd(&out[2], like);
    if (best_h != 0xFFFFFFFFu && best_unlike) atomicAdd(&out[3], 1u);
    if (!qi0) atomicAdd(&out[4], 1u);
  }
}

}  // namespace

int run_profile_z(Batch& b, uint32_t r, uint32_t bins, uint32_t head_mask, uint32_t* head, uint32_t* tail,
                  uint32_t* escaped, std::string& err) {
  const SoupConfig& c = b.cfg[r];
  std::vector<uint32_t> h(2 * (size_t)bins + 1, 0);
  uint32_t* d = reinterpret_cast<uint32_t*>(analysis_scratch(b, 4 * h.size()));
  SOUP_CUDA_TRY(cudaMemsetAsync(d, 0, 4 * h.size(), b.stream));
  b.launches += 1;
  k_profile_z<<<nblocks(c.n), kBlock, 0, b.stream>>>(b.pos, b.hsp[r].slot_off, c.n, c.box[2], bins, head_mask, d);
  SOUP_CUDA_TRY(cudaGetLastError());
  SOUP_CUDA_TRY(cudaMemcpyAsync(h.data(), d, 4 * h.size(), cudaMemcpyDeviceToHost, b.stream));
  SOUP_CUDA_TRY(cudaStreamSynchronize(b.stream));
  const uint32_t esc = h[2 * (size_t)bins];
  if (esc && !escaped) {
    err = "densityProfileZ: " + std::to_string(esc) + " bead(s) outside [0, " + std::to_string(c.box[2]) +
          "): the z profile is undefined for escaped beads (z is not periodic), and clamping them into the "
          "edge bin is not allowed: it creates a false peak";
    return SOUP_E_ARG;
  }
  std::copy(h.begin(), h.begin() + bins, head);
  std::copy(h.begin() + bins, h.begin() + 2 * (size_t)bins, tail);
  if (escaped) *escaped = esc;
  return SOUP_OK;
}

int run_pairing(Batch& b, uint32_t r, double contact, uint32_t out5[5], std::string& err) {
  const SysParams& P = b.hsp[r];
  const SoupConfig& c = b.cfg[r];
  if (!c.es_enabled || P.nheads == 0) {
    for (int k = 0; k < 5; ++k) out5[k] = 0;
    return SOUP_OK;
  }
  if (!(contact < c.es_cutoff)) {
    err = "pairingStats: the contact radius must be below the electrostatics cutoff (the head list's reach)";
    return SOUP_E_ARG;
  }
  uint32_t* d = reinterpret_cast<uint32_t*>(analysis_scratch(b, 4 * 5));
  SOUP_CUDA_TRY(cudaMemsetAsync(d, 0, 4 * 5, b.stream));
  b.launches += 1;
  k_pairing<<<nblocks((uint64_t)P.nheads * 32, kBlock), kBlock, 0, b.stream>>>(
      b.head_slot, P.head_off, P.nheads, b.pos, b.charge, b.es_nl, b.es_cnt, b.es_cap, c.box[0], c.box[1], c.box[2],
      contact, d);
  SOUP_CUDA_TRY(cudaGetLastError());
  SOUP_CUDA_TRY(cudaMemcpyAsync(out5, d, 4 * 5, cudaMemcpyDeviceToHost, b.stream));
  SOUP_CUDA_TRY(cudaStreamSynchronize(b.stream));
  return SOUP_OK;
}

}  // namespace soup

namespace soup {

namespace {

// shapeOf over unwrapAggregate (engine/src/aggregate.ts:245-262, 308-346) for one component per
// block: members[start[c] .. start[c+1]) as original indices, the first one the reference member.
// Unwrapped coordinates are rounded to f32 as the reference stores them (a Float32Array), then
// summed in FP64 in two passes (centre, then the second moments about it), each a fixed-order block
// reduction.  out[c]: n, centre x y z, Sxx Syy Szz Sxy Sxz Syz (per member).
constexpr int kShapeThreads = 256;
__device__ __forceinline__ double block_sum(double v, double* sh) {
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int s = kShapeThreads / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  const double r = sh[0];
  __syncthreads();
  return r;
}
__global__ void __launch_bounds__(kShapeThreads) k_shape(const float4* __restrict__ pos, const uint32_t* __restrict__ slot_of,
                                                         uint32_t off, const uint32_t* __restrict__ members,
                                                         const uint32_t* __restrict__ start, double bx, double by,
                                                         double bz, double* __restrict__ out) {
  __shared__ double sh[kShapeThreads];
  const uint32_t c = blockIdx.x;
  const uint32_t a = start[c], e = start[c + 1];
  const float4 r0 = pos[slot_of[off + members[a]]];
  const double ref[3] = {(double)r0.x, (double)r0.y, (double)r0.z};
  const double L[3] = {bx, by, bz};
  auto unwrap = [&](uint32_t k, double u[3]) {
    const float4 p = pos[slot_of[off + members[k]]];
    const double v[3] = {(double)p.x, (double)p.y, (double)p.z};
    for (int ax = 0; ax < 3; ++ax) u[ax] = (double)(float)(ref[ax] + mi_js(v[ax] - ref[ax], L[ax]));
  };
  double s[3] = {0, 0, 0};
  for (uint32_t k = a + threadIdx.x; k < e; k += kShapeThreads) {
    double u[3];
    unwrap(k, u);
    s[0] += u[0]; s[1] += u[1]; s[2] += u[2];
  }
  const double n = (double)(e - a);
  double cen[3];
  for (int ax = 0; ax < 3; ++ax) cen[ax] = block_sum(s[ax], sh) / n;
  double m[6] = {0, 0, 0, 0, 0, 0};
  for (uint32_t k = a + threadIdx.x; k < e; k += kShapeThreads) {
    double u[3];
    unwrap(k, u);
    const double dx = u[0] - cen[0], dy = u[1] - cen[1], dz = u[2] - cen[2];
    m[0] += dx * dx; m[1] += dy * dy; m[2] += dz * dz; m[3] += dx * dy; m[4] += dx * dz; m[5] += dy * dz;
  }
  double tot[6];
  for (int q = 0; q < 6; ++q) tot[q] = block_sum(m[q], sh) / n;
  if (threadIdx.x == 0) {
    double* o = out + 10 * (size_t)c;
    o[0] = n;
    for (int ax = 0; ax < 3; ++ax) o[1 + ax] = cen[ax];
    for (int q = 0; q < 6; ++q) o[4 + q] = tot[q];
  }
}

}  // namespace

int run_shapes(Batch& b, uint32_t r, const uint32_t* members_csr, const uint32_t* start, uint32_t ncomp,
               double* out10, std::string& err) {
  const SoupConfig& c = b.cfg[r];
  if (ncomp == 0) return SOUP_OK;
  const uint32_t total = start[ncomp];
  for (uint32_t k = 0; k < total; ++k)
    if (members_csr[k] >= c.n) { err = "aggregate shapes: member index out of range"; return SOUP_E_ARG; }
  ScratchLayout L;
  const size_t o_m = L.add<uint32_t>(total), o_s = L.add<uint32_t>((size_t)ncomp + 1), o_out = L.add<double>(10 * (size_t)ncomp);
  char* base = analysis_scratch(b, L.used);
  uint32_t* dm = reinterpret_cast<uint32_t*>(base + o_m);
  uint32_t* ds = reinterpret_cast<uint32_t*>(base + o_s);
  double* dout = reinterpret_cast<double*>(base + o_out);
  SOUP_CUDA_TRY(cudaMemcpyAsync(dm, members_csr, 4 * (size_t)total, cudaMemcpyHostToDevice, b.stream));
  SOUP_CUDA_TRY(cudaMemcpyAsync(ds, start, 4 * ((size_t)ncomp + 1), cudaMemcpyHostToDevice, b.stream));
  b.launches += 1;
  k_shape<<<ncomp, kShapeThreads, 0, b.stream>>>(b.pos, b.slot_of, b.hsp[r].slot_off, dm, ds, c.box[0], c.box[1],
                                                 c.box[2], dout);
  SOUP_CUDA_TRY(cudaGetLastError());
  SOUP_CUDA_TRY(cudaMemcpyAsync(out10, dout, 80 * (size_t)ncomp, cudaMemcpyDeviceToHost, b.stream));
  SOUP_CUDA_TRY(cudaStreamSynchronize(b.stream));
  return SOUP_OK;
}

// ---- per-aggregate detail (soup/src/aggregates.ts:350-476 shapeOfAggregate) -------------------
namespace {

// JavaScript's d - Math.round(d / L) * L with every operation rounded on its own (no FMA contraction)
__device__ __forceinline__ double mi_rn(double d, double L) { return __dsub_rn(d, __dmul_rn(js_round(__ddiv_rn(d, L)), L)); }

// unwrapAggregate (engine/src/aggregate.ts:245-262) on all three axes about the first member, each
// coordinate rounded to f32 as the reference stores it; w = kind
__global__ void k_unwrap_members(const float4* __restrict__ pos, const uint32_t* __restrict__ slot_of, uint32_t off,
                                 const uint32_t* __restrict__ members, uint32_t m, double bx, double by, double bz,
                                 float4* __restrict__ out) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  const float4 r0 = pos[slot_of[off + members[0]]], p = pos[slot_of[off + members[k]]];
  const double ref[3] = {(double)r0.x, (double)r0.y, (double)r0.z}, v[3] = {(double)p.x, (double)p.y, (double)p.z};
  const double L[3] = {bx, by, bz};
  float u[3];
  for (int a = 0; a < 3; ++a) u[a] = __double2float_rn(__dadd_rn(ref[a], mi_rn(__dsub_rn(v[a], ref[a]), L[a])));
  out[k] = make_float4(u[0], u[1], u[2], p.w);
}

// occupancy (engine/src/closure.ts:67-107) of a local grid: x and y wrap, z is open
struct LGrid {
  int n[3];
  double box[3], cell;
};
__global__ void k_local_occupancy(const float4* __restrict__ p, uint32_t n, LGrid g, int reach, double r2,
                                  uint8_t* __restrict__ occ) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double px = (double)p[i].x, py = (double)p[i].y, pz = (double)p[i].z;
  const int cx = (int)floor(__ddiv_rn(px, g.cell)), cy = (int)floor(__ddiv_rn(py, g.cell)),
            cz = (int)floor(__ddiv_rn(pz, g.cell));
  for (int dz = -reach; dz <= reach; ++dz) {
    const int gz = cz + dz;
    if (gz < 0 || gz >= g.n[2]) continue;
    const double ddz = __dsub_rn(__dmul_rn(gz + 0.5, g.cell), pz);
    for (int dy = -reach; dy <= reach; ++dy) {
      const int gy = ((cy + dy) % g.n[1] + g.n[1]) % g.n[1];
      const double ddy = mi_rn(__dsub_rn(__dmul_rn(gy + 0.5, g.cell), py), g.box[1]);
      for (int dx = -reach; dx <= reach; ++dx) {
        const int gx = ((cx + dx) % g.n[0] + g.n[0]) % g.n[0];
        const double ddx = mi_rn(__dsub_rn(__dmul_rn(gx + 0.5, g.cell), px), g.box[0]);
        if (__dadd_rn(__dadd_rn(__dmul_rn(ddx, ddx), __dmul_rn(ddy, ddy)), __dmul_rn(ddz, ddz)) <= r2)
          occ[(size_t)gx + (size_t)g.n[0] * ((size_t)gy + (size_t)g.n[1] * gz)] = 1;
      }
    }
  }
}

// floodOutside (engine/src/closure.ts:108-150): every empty cell connected to a face of the grid
// through empty cells, 6-neighbour, open boundary.  One pass marks an empty cell whose neighbour
// is marked (or that lies on a face); passes repeat until one marks nothing.  The marked set is the
// reachable set whatever order the passes run in.
__global__ void k_local_flood(const uint8_t* __restrict__ occ, uint8_t* __restrict__ vis, LGrid g, uint64_t nc,
                              uint32_t* __restrict__ changed) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nc; i += (uint64_t)gridDim.x * blockDim.x) {
    if (occ[i] || vis[i]) continue;
    const int x = (int)(i % (uint64_t)g.n[0]);
    const int y = (int)((i / (uint64_t)g.n[0]) % (uint64_t)g.n[1]);
    const int z = (int)(i / ((uint64_t)g.n[0] * g.n[1]));
    bool reach = x == 0 || y == 0 || z == 0 || x == g.n[0] - 1 || y == g.n[1] - 1 || z == g.n[2] - 1;
    if (!reach) {
      const uint64_t sx = 1, sy = (uint64_t)g.n[0], sz = (uint64_t)g.n[0] * g.n[1];
      reach = vis[i - sx] || vis[i + sx] || vis[i - sy] || vis[i + sy] || vis[i - sz] || vis[i + sz];
    }
    if (reach) {
      vis[i] = 1;
      *changed = 1u;
    }
  }
}

__global__ void k_local_unreached(const uint8_t* __restrict__ occ, const uint8_t* __restrict__ vis, uint64_t nc,
                                  unsigned long long* __restrict__ count) {
  unsigned long long c = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nc; i += (uint64_t)gridDim.x * blockDim.x)
    c += (!occ[i] && !vis[i]) ? 1ull : 0ull;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

}  // namespace

int run_unwrap(Batch& b, uint32_t r, const uint32_t* members, uint32_t m, float* out, std::string& err) {
  const SoupConfig& c = b.cfg[r];
  for (uint32_t k = 0; k < m; ++k)
    if (members[k] >= c.n) { err = "unwrapAggregate: member index out of range"; return SOUP_E_ARG; }
  if (m == 0) return SOUP_OK;
  ScratchLayout L;
  const size_t o_m = L.add<uint32_t>(m), o_out = L.add<float4>(m);
  char* base = analysis_scratch(b, L.used);
  uint32_t* dm = reinterpret_cast<uint32_t*>(base + o_m);
  float4* dout = reinterpret_cast<float4*>(base + o_out);
  SOUP_CUDA_TRY(cudaMemcpyAsync(dm, members, 4 * (size_t)m, cudaMemcpyHostToDevice, b.stream));
  k_unwrap_members<<<nblocks(m), kBlock, 0, b.stream>>>(b.pos, b.slot_of, b.hsp[r].slot_off, dm, m, c.box[0], c.box[1],
                                                       c.box[2], dout);
  b.launches += 1;
  SOUP_CUDA_TRY(cudaGetLastError());
  SOUP_CUDA_TRY(cudaMemcpyAsync(out, dout, 16 * (size_t)m, cudaMemcpyDeviceToHost, b.stream));
  SOUP_CUDA_TRY(cudaStreamSynchronize(b.stream));
  return SOUP_OK;
}

// localCavityVolume (soup/src/aggregates.ts:350-385): the bounding region of the unwrapped beads,
// padded by 4 radii, shifted to start at the pad (f32 positions, as the reference's Float32Array),
// its occupancy and the empty cells the open-boundary flood does not reach, times cell^3
int run_local_cavity(Batch& b, const float* positions, uint32_t n, double cell, double radius, double* volume,
                     std::string& err, const double* frame_box) {
  const std::string who = frame_box ? "enclosedVolume: " : "localCavityVolume: ";
  *volume = 0.0;
  if (n == 0) return SOUP_OK;   // nothing occupied: every empty cell is reached
  if (!(cell > 0) || !(radius >= 0)) { err = who + "cell must be positive and radius non-negative"; return SOUP_E_ARG; }
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint32_t i = 0; i < n; ++i)
    for (int a = 0; a < 3; ++a) {
      const double v = positions[4 * (size_t)i + a];
      lo[a] = std::min(lo[a], v);
      hi[a] = std::max(hi[a], v);
    }
  const double pad = radius * 4;
  LGrid g{};
  g.cell = cell;
  uint64_t nc = 1;
  double shift[3];
  for (int a = 0; a < 3; ++a) {
    if (!std::isfinite(lo[a]) || !std::isfinite(hi[a])) { err = who + "non-finite position"; return SOUP_E_ARG; }
    if (frame_box) {   // closure.ts:51-57 dimsFor over the periodic box, no shift
      if (!(frame_box[a] > 0)) { err = who + "the box must be positive"; return SOUP_E_ARG; }
      shift[a] = 0.0;
      g.box[a] = frame_box[a];
    } else {
      shift[a] = pad - lo[a];
      g.box[a] = hi[a] - lo[a] + 2 * pad;
    }
    g.n[a] = std::max(1, (int)std::ceil(g.box[a] / cell));
    nc *= (uint64_t)g.n[a];
  }
  if (nc > (uint64_t)1 << 31) { err = who + "the grid is too large"; return SOUP_E_ARG; }
  std::vector<float> sh(4 * (size_t)n);
  for (uint32_t i = 0; i < n; ++i) {
    for (int a = 0; a < 3; ++a) sh[4 * (size_t)i + a] = (float)((double)positions[4 * (size_t)i + a] + shift[a]);
    sh[4 * (size_t)i + 3] = positions[4 * (size_t)i + 3];
  }
  ScratchLayout L;
  const size_t o_p = L.add<float4>(n), o_occ = L.add<uint8_t>(nc), o_vis = L.add<uint8_t>(nc),
               o_cnt = L.add<unsigned long long>(2);
  char* base = analysis_scratch(b, L.used);
  float4* dp = reinterpret_cast<float4*>(base + o_p);
  uint8_t* occ = reinterpret_cast<uint8_t*>(base + o_occ);
  uint8_t* vis = reinterpret_cast<uint8_t*>(base + o_vis);
  unsigned long long* cnt = reinterpret_cast<unsigned long long*>(base + o_cnt);
  uint32_t* changed = reinterpret_cast<uint32_t*>(cnt + 1);
  cudaStream_t st = b.stream;
  SOUP_CUDA_TRY(cudaMemcpyAsync(dp, sh.data(), 16 * (size_t)n, cudaMemcpyHostToDevice, st));
  SOUP_CUDA_TRY(cudaMemsetAsync(occ, 0, nc, st));
  SOUP_CUDA_TRY(cudaMemsetAsync(vis, 0, nc, st));
  SOUP_CUDA_TRY(cudaMemsetAsync(cnt, 0, 16, st));
  const int reach = std::max(1, (int)std::ceil(radius / cell));
  k_local_occupancy<<<nblocks(n), kBlock, 0, st>>>(dp, n, g, reach, radius * radius, occ);
  const unsigned fgrid = (unsigned)std::min<uint64_t>(nblocks(nc), 148ull * 16ull);
  uint32_t ch = 1;
  uint64_t passes = 0;
  while (ch) {
    if (++passes > nc + 1) { err = who + "the flood did not finish"; return SOUP_E_STATE; }
    SOUP_CUDA_TRY(cudaMemsetAsync(changed, 0, 4, st));
    k_local_flood<<<fgrid, kBlock, 0, st>>>(occ, vis, g, nc, changed);
    SOUP_CUDA_TRY(cudaMemcpyAsync(&ch, changed, 4, cudaMemcpyDeviceToHost, st));
    SOUP_CUDA_TRY(cudaStreamSynchronize(st));
  }
  k_local_unreached<<<fgrid, kBlock, 0, st>>>(occ, vis, nc, cnt);
  b.launches += 2 + passes;
  unsigned long long unreached = 0;
  SOUP_CUDA_TRY(cudaMemcpyAsync(&unreached, cnt, 8, cudaMemcpyDeviceToHost, st));
  SOUP_CUDA_TRY(cudaStreamSynchronize(st));
  SOUP_CUDA_TRY(cudaGetLastError());
  *volume = (double)unreached * cell * cell * cell;
  return SOUP_OK;
}

}  // namespace soup

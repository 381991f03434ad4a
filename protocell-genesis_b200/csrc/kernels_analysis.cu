// kernels_analysis.cu -- closure flood fill, amphiphile recognition and aggregate labels on the device.
//
// Reference: soup/src/water-closure.ts:109-363 (occupancyPeriodic, farthestEmptyCellSeed,
// floodOutsidePeriodic, encapsulatedWaterVolume), soup/src/amphiphile.ts:55-141 (findAmphiphiles),
// engine/src/aggregate.ts:65-130,201-212 (buildClusterUnionFind with periodic z, clusterComponents).
//
// The reference computes these on the CPU in JavaScript doubles.  Here every geometric test is FP64
// with explicit round-to-nearest operations (no FMA contraction) and JavaScript Math.round, so the
// occupancy grid, the seed cell, the reached set and the labels equal the oracle's bit for bit.
// Labels are canonical: an aggregate is named by the minimum original index among its members.
#include <cmath>
#include <vector>

#include "soup_internal.h"

namespace soup {

namespace {

constexpr int kBlock = 256;
inline unsigned nblocks(uint64_t n, int b = kBlock) { return (unsigned)((n + b - 1) / b); }
constexpr uint32_t NONE = SOUP_NONE_U32;

__device__ __forceinline__ double js_round(double x) {
  const double r = floor(x);
  return (__dsub_rn(x, r) >= 0.5) ? r + 1.0 : r;
}
__device__ __forceinline__ double wrap1(double v, double L) { return __dsub_rn(v, __dmul_rn(floor(__ddiv_rn(v, L)), L)); }
__device__ __forceinline__ double mi1(double d, double L) { return __dsub_rn(d, __dmul_rn(js_round(__ddiv_rn(d, L)), L)); }
__device__ __forceinline__ double sq3(double a, double b, double c) {
  return __dadd_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)), __dmul_rn(c, c));
}

struct Grid {
  int nx, ny, nz;
  double cell;
  double box[3];
};

// occupancyPeriodic (water-closure.ts:109-150): one thread per member
__global__ void k_occupancy(const float4* __restrict__ pos, const uint32_t* __restrict__ slot_of, uint32_t off,
                            const uint32_t* __restrict__ mem, uint32_t nm, Grid g, int reach, double r2,
                            uint8_t* __restrict__ occ) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nm) return;
  const float4 p = pos[slot_of[off + mem[k]]];
  const double px = wrap1((double)p.x, g.box[0]), py = wrap1((double)p.y, g.box[1]), pz = wrap1((double)p.z, g.box[2]);
  const int cx = (int)floor(__ddiv_rn(px, g.cell)), cy = (int)floor(__ddiv_rn(py, g.cell)), cz = (int)floor(__ddiv_rn(pz, g.cell));
  for (int dz = -reach; dz <= reach; ++dz) {
    const int gz = ((cz + dz) % g.nz + g.nz) % g.nz;
    const double ddz = mi1(__dsub_rn(__dmul_rn(gz + 0.5, g.cell), pz), g.box[2]);
    for (int dy = -reach; dy <= reach; ++dy) {
      const int gy = ((cy + dy) % g.ny + g.ny) % g.ny;
      const double ddy = mi1(__dsub_rn(__dmul_rn(gy + 0.5, g.cell), py), g.box[1]);
      for (int dx = -reach; dx <= reach; ++dx) {
        const int gx = ((cx + dx) % g.nx + g.nx) % g.nx;
        const double ddx = mi1(__dsub_rn(__dmul_rn(gx + 0.5, g.cell), px), g.box[0]);
        if (sq3(ddx, ddy, ddz) <= r2) occ[(size_t)gx + (size_t)g.nx * ((size_t)gy + (size_t)g.ny * gz)] = 1;
      }
    }
  }
}

// farthestEmptyCellSeed (water-closure.ts:195-225): max d^2, first cell in scan order among ties
__device__ __forceinline__ double seed_d2(Grid g, const double c[3], uint64_t i) {
  const int z = (int)(i / ((uint64_t)g.nx * g.ny));
  const uint64_t rem = i - (uint64_t)z * g.nx * g.ny;
  const int y = (int)(rem / g.nx), x = (int)(rem - (uint64_t)y * g.nx);
  const double dx = mi1(__dsub_rn(__dmul_rn(x + 0.5, g.cell), c[0]), g.box[0]);
  const double dy = mi1(__dsub_rn(__dmul_rn(y + 0.5, g.cell), c[1]), g.box[1]);
  const double dz = mi1(__dsub_rn(__dmul_rn(z + 0.5, g.cell), c[2]), g.box[2]);
  return sq3(dx, dy, dz);
}
__global__ void k_seed_max(const uint8_t* __restrict__ occ, uint64_t nc, Grid g, double c0, double c1, double c2,
                           unsigned long long* __restrict__ best) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long v = 0;
  if (i < nc && !occ[i]) {
    const double c[3] = {c0, c1, c2};
    v = (unsigned long long)__double_as_longlong(seed_d2(g, c, i)) + 1ull;   // +1: "none" stays 0
  }
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0 && v) atomicMax(best, v);
}
__global__ void k_seed_min_index(const uint8_t* __restrict__ occ, uint64_t nc, Grid g, double c0, double c1, double c2,
                                 const unsigned long long* __restrict__ best, unsigned long long* __restrict__ idx) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nc || occ[i] || *best == 0) return;
  const double c[3] = {c0, c1, c2};
  if ((unsigned long long)__double_as_longlong(seed_d2(g, c, i)) + 1ull == *best) atomicMin(idx, (unsigned long long)i);
}

// floodOutsidePeriodic (water-closure.ts:154-189), one BFS level per launch
__global__ void k_flood_level(const uint8_t* __restrict__ occ, uint32_t* __restrict__ vis, Grid g,
                              const uint32_t* __restrict__ front, const uint32_t* __restrict__ nfront,
                              uint32_t* __restrict__ next, uint32_t* __restrict__ nnext, uint32_t cap) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= *nfront) return;
  const uint32_t i = front[t];
  const int z = (int)(i / ((uint32_t)g.nx * g.ny));
  const uint32_t rem = i - (uint32_t)z * g.nx * g.ny;
  const int y = (int)(rem / g.nx), x = (int)(rem - (uint32_t)y * g.nx);
  const int nb[6][3] = {{(x + 1) % g.nx, y, z}, {(x - 1 + g.nx) % g.nx, y, z}, {x, (y + 1) % g.ny, z},
                        {x, (y - 1 + g.ny) % g.ny, z}, {x, y, (z + 1) % g.nz}, {x, y, (z - 1 + g.nz) % g.nz}};
  for (int q = 0; q < 6; ++q) {
    const uint32_t ni = (uint32_t)nb[q][0] + (uint32_t)g.nx * ((uint32_t)nb[q][1] + (uint32_t)g.ny * nb[q][2]);
    if (occ[ni]) continue;
    if (atomicCAS(&vis[ni], 0u, 1u) == 0u) {
      const uint32_t at = atomicAdd(nnext, 1u);
      if (at < cap) next[at] = ni;
    }
  }
}

// cell counts and water classification (water-closure.ts:297-327)
__global__ void k_cell_counts(const uint8_t* __restrict__ occ, const uint32_t* __restrict__ vis, uint64_t nc,
                              unsigned long long* __restrict__ out /* totalEmpty, unreached, reachedEmpty */) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t a = 0, b = 0, c = 0;
  if (i < nc && !occ[i]) { a = 1; if (!vis[i]) b = 1; else c = 1; }
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o); b += __shfl_xor_sync(0xffffffffu, b, o); c += __shfl_xor_sync(0xffffffffu, c, o);
  }
  if ((threadIdx.x & 31) == 0) { atomicAdd(&out[0], a); atomicAdd(&out[1], b); atomicAdd(&out[2], c); }
}
__global__ void k_water(const float4* __restrict__ pos, const uint32_t* __restrict__ slot_of, uint32_t off,
                        const uint32_t* __restrict__ wat, uint32_t nw, Grid g, const uint8_t* __restrict__ occ,
                        const uint32_t* __restrict__ vis, unsigned long long* __restrict__ out /* enc, reachedWater */) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nw) return;
  const float4 p = pos[slot_of[off + wat[k]]];
  const int gx = min(g.nx - 1, (int)floor(__ddiv_rn(wrap1((double)p.x, g.box[0]), g.cell)));
  const int gy = min(g.ny - 1, (int)floor(__ddiv_rn(wrap1((double)p.y, g.box[1]), g.cell)));
  const int gz = min(g.nz - 1, (int)floor(__ddiv_rn(wrap1((double)p.z, g.box[2]), g.cell)));
  const size_t c = (size_t)gx + (size_t)g.nx * ((size_t)gy + (size_t)g.ny * gz);
  if (occ[c]) return;
  atomicAdd(&out[vis[c] ? 1 : 0], 1ull);
}

// ---- union-find helpers (hook the larger root under the smaller: roots are component minima) ----
__device__ __forceinline__ uint32_t uf_find(uint32_t* parent, uint32_t x) {
  volatile uint32_t* vp = parent;
  uint32_t p = vp[x];
  while (p != x) { x = p; p = vp[x]; }
  return x;
}
__device__ __forceinline__ void uf_union(uint32_t* parent, uint32_t a, uint32_t b) {
  for (;;) {
    a = uf_find(parent, a);
    b = uf_find(parent, b);
    if (a == b) return;
    if (a > b) { const uint32_t t = a; a = b; b = t; }
    if (atomicCAS(&parent[b], b, a) == b) return;
  }
}

// findAmphiphiles (amphiphile.ts:55-141) on the bond graph, indices local to the replica
__global__ void k_amph_union(const uint32_t* __restrict__ slots, const uint32_t* __restrict__ id, uint32_t off,
                             uint32_t n, uint32_t* __restrict__ parent) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const uint32_t i = id[off + k] - off;
  for (int s = 0; s < 3; ++s) {
    const uint32_t j = slots[3 * (size_t)(off + k) + s];
    if (j != NONE && j - off > i) uf_union(parent, i, j - off);
  }
}
__global__ void k_amph_stats(const float4* __restrict__ pos, const uint32_t* __restrict__ slots,
                             const uint32_t* __restrict__ id, uint32_t off, uint32_t n, const uint32_t* __restrict__ polar,
                             uint32_t* __restrict__ parent, uint32_t* __restrict__ size, uint32_t* __restrict__ sumdeg,
                             uint32_t* __restrict__ npolar, uint32_t* __restrict__ polar_idx, uint32_t* __restrict__ bad) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const uint32_t i = id[off + k] - off;
  uint32_t deg = 0;
  for (int s = 0; s < 3; ++s) deg += slots[3 * (size_t)(off + k) + s] != NONE;
  const uint32_t r = uf_find(parent, i);
  atomicAdd(&size[r], 1u);
  atomicAdd(&sumdeg[r], deg);
  const int kind = (int)lrintf(pos[off + k].w);
  if (polar[kind]) {
    atomicAdd(&npolar[r], 1u);
    polar_idx[r] = i;
    if (deg < 1 || deg > 2) bad[r] = 1;
  } else if (deg > 2) {
    bad[r] = 1;
  }
}
__global__ void k_amph_label(uint32_t n, uint32_t* __restrict__ parent, const uint32_t* __restrict__ size,
                             const uint32_t* __restrict__ sumdeg, const uint32_t* __restrict__ npolar,
                             const uint32_t* __restrict__ polar_idx, const uint32_t* __restrict__ bad,
                             uint32_t* __restrict__ head_of, uint32_t* __restrict__ count) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t r = uf_find(parent, i);
  const bool ok = !bad[r] && npolar[r] == 1 && sumdeg[r] / 2 == size[r] - 1;
  head_of[i] = ok ? polar_idx[r] : NONE;
  if (ok && r == i) atomicAdd(count, 1u);
}

// buildClusterUnionFind (aggregate.ts:65-130), periodic on all three axes; one thread per member
__global__ void k_agg_bin(const float4* __restrict__ pos, const uint32_t* __restrict__ slot_of, uint32_t off,
                          const uint32_t* __restrict__ mem, uint32_t m, Grid g, double wx, double wy, double wz,
                          uint32_t* __restrict__ cell, uint32_t* __restrict__ count) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  const float4 p = pos[slot_of[off + mem[k]]];
  const int cx = min(g.nx - 1, (int)floor(__ddiv_rn(wrap1((double)p.x, g.box[0]), wx)));
  const int cy = min(g.ny - 1, (int)floor(__ddiv_rn(wrap1((double)p.y, g.box[1]), wy)));
  const int cz = min(g.nz - 1, (int)floor(__ddiv_rn(wrap1((double)p.z, g.box[2]), wz)));
  const uint32_t c = (uint32_t)cx + (uint32_t)g.nx * ((uint32_t)cy + (uint32_t)g.ny * cz);
  cell[k] = c;
  atomicAdd(&count[c], 1u);
}
__global__ void k_agg_scatter(const uint32_t* __restrict__ cell, uint32_t m, const uint32_t* __restrict__ start,
                              uint32_t* __restrict__ cursor, uint32_t* __restrict__ sorted) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  const uint32_t c = cell[k];
  sorted[start[c] + atomicAdd(&cursor[c], 1u)] = k;
}
__global__ void k_agg_union(const float4* __restrict__ pos, const uint32_t* __restrict__ slot_of, uint32_t off,
                            const uint32_t* __restrict__ mem, uint32_t m, Grid g, const uint32_t* __restrict__ cell,
                            const uint32_t* __restrict__ start, const uint32_t* __restrict__ sorted, double c2,
                            uint32_t* __restrict__ parent) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  const float4 pi = pos[slot_of[off + mem[k]]];
  const uint32_t c = cell[k];
  const int cz = (int)(c / ((uint32_t)g.nx * g.ny)), cy = (int)((c / g.nx) % g.ny), cx = (int)(c % g.nx);
  for (int dx = -1; dx <= 1; ++dx) {
    const int ax = ((cx + dx) % g.nx + g.nx) % g.nx;
    for (int dy = -1; dy <= 1; ++dy) {
      const int ay = ((cy + dy) % g.ny + g.ny) % g.ny;
      for (int dz = -1; dz <= 1; ++dz) {
        const int az = ((cz + dz) % g.nz + g.nz) % g.nz;
        const uint32_t nc = (uint32_t)ax + (uint32_t)g.nx * ((uint32_t)ay + (uint32_t)g.ny * az);
        for (uint32_t t = start[nc]; t < start[nc + 1]; ++t) {
          const uint32_t l = sorted[t];
          if (l <= k) continue;
          const float4 pj = pos[slot_of[off + mem[l]]];
          const double ddx = mi1(__dsub_rn((double)pi.x, (double)pj.x), g.box[0]);
          const double ddy = mi1(__dsub_rn((double)pi.y, (double)pj.y), g.box[1]);
          const double ddz = mi1(__dsub_rn((double)pi.z, (double)pj.z), g.box[2]);
          if (sq3(ddx, ddy, ddz) <= c2) uf_union(parent, k, l);
        }
      }
    }
  }
}
__global__ void k_agg_min(const uint32_t* __restrict__ mem, uint32_t m, uint32_t* __restrict__ parent,
                          uint32_t* __restrict__ minidx, uint32_t* __restrict__ ncomp) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  const uint32_t r = uf_find(parent, k);
  atomicMin(&minidx[r], mem[k]);
  if (r == k) atomicAdd(ncomp, 1u);
}
__global__ void k_agg_label(const uint32_t* __restrict__ mem, uint32_t m, uint32_t* __restrict__ parent,
                            const uint32_t* __restrict__ minidx, uint32_t* __restrict__ labels) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  labels[k] = minidx[uf_find(parent, k)];
}
__global__ void k_iota(uint32_t* __restrict__ a, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = i;
}
__global__ void k_fill(uint32_t* __restrict__ a, uint32_t n, uint32_t v) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = v;
}

// scratch that lives for one call of the aggregate labels (soup_aggregate_labels allocates and
// frees per call, as its declaration states; the other analysis calls use the batch's scratch)
struct Scratch {
  std::vector<void*> ptrs;
  ~Scratch() { for (void* p : ptrs) cudaFree(p); }
  template <class T> T* get(size_t n) {
    T* p = nullptr;
    SOUP_CUDA_TRY(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)));
    ptrs.push_back(p);
    return p;
  }
};

}  // namespace

void exclusive_scan(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* tmp, cudaStream_t st);

char* analysis_scratch(Batch& b, size_t bytes) {
  if (bytes > b.an_cap) {
    SOUP_CUDA_TRY(cudaStreamSynchronize(b.stream));
    if (b.an_buf) SOUP_CUDA_TRY(cudaFree(b.an_buf));
    b.an_buf = nullptr;
    b.an_cap = 0;
    const size_t want = (bytes + (size_t(1) << 20) - 1) & ~((size_t(1) << 20) - 1);
    SOUP_CUDA_TRY(cudaMalloc(&b.an_buf, want));
    b.an_cap = want;
  }
  return b.an_buf;
}

int run_closure(Batch& b, uint32_t r, const uint32_t* mem, uint32_t nm, const uint32_t* wat, uint32_t nw,
                const double centre[3], double cell, double radius, double vmin, SoupClosureResult* out,
                std::string& err) {
  const SoupConfig& c = b.cfg[r];
  const uint32_t n = c.n, off = b.hsp[r].slot_off;
  for (uint32_t k = 0; k < nm; ++k) if (mem[k] >= n) { err = "closure: member index out of range"; return SOUP_E_ARG; }
  for (uint32_t k = 0; k < nw; ++k) if (wat[k] >= n) { err = "closure: water index out of range"; return SOUP_E_ARG; }
  Grid g;
  g.cell = cell;
  for (int a = 0; a < 3; ++a) g.box[a] = c.box[a];
  g.nx = std::max(1, (int)std::ceil(c.box[0] / cell));
  g.ny = std::max(1, (int)std::ceil(c.box[1] / cell));
  g.nz = std::max(1, (int)std::ceil(c.box[2] / cell));
  const uint64_t nc = (uint64_t)g.nx * g.ny * g.nz;
  if (nc >= 0xFFFFFFF0ull) { err = "closure: grid too large"; return SOUP_E_ARG; }
  const int reach = std::max(1, (int)std::ceil(radius / cell));
  ScratchLayout L;
  const size_t o_occ = L.add<uint8_t>(nc), o_vis = L.add<uint32_t>(nc), o_mem = L.add<uint32_t>(nm),
               o_wat = L.add<uint32_t>(nw), o_fa = L.add<uint32_t>(nc), o_fb = L.add<uint32_t>(nc),
               o_cnt = L.add<uint32_t>(2), o_u64 = L.add<unsigned long long>(8);
  char* base = analysis_scratch(b, L.used);
  uint8_t* occ = reinterpret_cast<uint8_t*>(base + o_occ);
  uint32_t* vis = reinterpret_cast<uint32_t*>(base + o_vis);
  uint32_t* dmem = reinterpret_cast<uint32_t*>(base + o_mem);
  uint32_t* dwat = reinterpret_cast<uint32_t*>(base + o_wat);
  uint32_t* fa = reinterpret_cast<uint32_t*>(base + o_fa);
  uint32_t* fb = reinterpret_cast<uint32_t*>(base + o_fb);
  uint32_t* cnt = reinterpret_cast<uint32_t*>(base + o_cnt);
  unsigned long long* u64 = reinterpret_cast<unsigned long long*>(base + o_u64);
  cudaStream_t st = b.stream;
  SOUP_CUDA_TRY(cudaMemsetAsync(occ, 0, nc, st));
  SOUP_CUDA_TRY(cudaMemsetAsync(vis, 0, 4 * nc, st));
  SOUP_CUDA_TRY(cudaMemsetAsync(u64, 0, 64, st));
  if (nm) SOUP_CUDA_TRY(cudaMemcpyAsync(dmem, mem, 4 * (size_t)nm, cudaMemcpyHostToDevice, st));
  if (nw) SOUP_CUDA_TRY(cudaMemcpyAsync(dwat, wat, 4 * (size_t)nw, cudaMemcpyHostToDevice, st));
  b.launches += 8;
  if (nm) k_occupancy<<<nblocks(nm), kBlock, 0, st>>>(b.pos, b.slot_of, off, dmem, nm, g, reach, radius * radius, occ);
  k_seed_max<<<nblocks(nc), kBlock, 0, st>>>(occ, nc, g, centre[0], centre[1], centre[2], u64);
  const unsigned long long init_idx = ~0ull;
  SOUP_CUDA_TRY(cudaMemcpyAsync(u64 + 1, &init_idx, 8, cudaMemcpyHostToDevice, st));
  k_seed_min_index<<<nblocks(nc), kBlock, 0, st>>>(occ, nc, g, centre[0], centre[1], centre[2], u64, u64 + 1);
  unsigned long long best[2];
  SOUP_CUDA_TRY(cudaMemcpyAsync(best, u64, 16, cudaMemcpyDeviceToHost, st));
  SOUP_CUDA_TRY(cudaStreamSynchronize(st));
  if (best[0] == 0) { err = "farthestEmptyCellSeed: the grid is fully occupied -- there is no empty cell to seed the periodic flood fill"; return SOUP_E_STATE; }
  const uint32_t seed = (uint32_t)best[1];
  const uint32_t one = 1;
  SOUP_CUDA_TRY(cudaMemcpyAsync(vis + seed, &one, 4, cudaMemcpyHostToDevice, st));
  SOUP_CUDA_TRY(cudaMemcpyAsync(fa, &seed, 4, cudaMemcpyHostToDevice, st));
  SOUP_CUDA_TRY(cudaMemcpyAsync(cnt, &one, 4, cudaMemcpyHostToDevice, st));
  uint32_t* front = fa; uint32_t* next = fb;
  uint32_t* nfront = cnt; uint32_t* nnext = cnt + 1;
  uint32_t level_size = 1;
  while (level_size > 0) {
    SOUP_CUDA_TRY(cudaMemsetAsync(nnext, 0, 4, st));
    k_flood_level<<<nblocks(level_size), kBlock, 0, st>>>(occ, vis, g, front, nfront, next, nnext, (uint32_t)nc);
    b.launches += 1;
    SOUP_CUDA_TRY(cudaMemcpyAsync(&level_size, nnext, 4, cudaMemcpyDeviceToHost, st));
    SOUP_CUDA_TRY(cudaStreamSynchronize(st));
    std::swap(front, next);
    std::swap(nfront, nnext);
  }
  k_cell_counts<<<nblocks(nc), kBlock, 0, st>>>(occ, vis, nc, u64 + 2);
  if (nw) k_water<<<nblocks(nw), kBlock, 0, st>>>(b.pos, b.slot_of, off, dwat, nw, g, occ, vis, u64 + 5);
  unsigned long long res[8];
  SOUP_CUDA_TRY(cudaMemcpyAsync(res, u64, 64, cudaMemcpyDeviceToHost, st));
  SOUP_CUDA_TRY(cudaStreamSynchronize(st));
  const double reached_empty = (double)res[4];
  const double bulk = res[4] > 0 ? (double)res[6] / (reached_empty * cell * cell * cell) : 0.0;
  const double thr = bulk > 0 ? vmin * bulk : NAN;
  out->encapsulated_count = (uint32_t)res[5];
  out->total_water = nw;
  out->bulk_water_density = bulk;
  out->threshold_count = thr;
  out->closed = (std::isfinite(thr) && (double)res[5] > thr) ? 1u : 0u;
  out->total_empty_cells = (uint32_t)res[2];
  out->unreached_cells = (uint32_t)res[3];
  out->seed_cell = seed;
  {
    const int z = (int)(seed / ((uint64_t)g.nx * g.ny));
    const uint64_t rem = seed - (uint64_t)z * g.nx * g.ny;
    const int y = (int)(rem / g.nx), x = (int)(rem - (uint64_t)y * g.nx);
    auto jr = [](double v) { double q = std::floor(v); return (v - q >= 0.5) ? q + 1 : q; };
    auto m1 = [&](double d, double L) { return d - jr(d / L) * L; };
    const double dx = m1((x + 0.5) * cell - centre[0], c.box[0]), dy = m1((y + 0.5) * cell - centre[1], c.box[1]),
                 dz = m1((z + 0.5) * cell - centre[2], c.box[2]);
    out->seed_dist_from_centre = std::sqrt(dx * dx + dy * dy + dz * dz);
  }
  return SOUP_OK;
}

int run_amphiphiles(Batch& b, uint32_t r, uint32_t* head_of, uint32_t* n_out, std::string& err) {
  (void)err;
  const uint32_t n = b.cfg[r].n, off = b.hsp[r].slot_off;
  ScratchLayout L;
  const size_t o_parent = L.add<uint32_t>(n), o_acc = L.add<uint32_t>(5 * (size_t)n + 1), o_dh = L.add<uint32_t>(n),
               o_polar = L.add<uint32_t>(SOUP_KMAX);
  char* base = analysis_scratch(b, L.used);
  uint32_t* parent = reinterpret_cast<uint32_t*>(base + o_parent);
  uint32_t* acc = reinterpret_cast<uint32_t*>(base + o_acc);
  uint32_t* dh = reinterpret_cast<uint32_t*>(base + o_dh);
  uint32_t* polar = reinterpret_cast<uint32_t*>(base + o_polar);
  uint32_t hp[SOUP_KMAX];
  for (int k = 0; k < SOUP_KMAX; ++k) hp[k] = b.cfg[r].kind_class[k] == SOUP_CLASS_POLAR ? 1u : 0u;
  cudaStream_t st = b.stream;
  SOUP_CUDA_TRY(cudaMemcpyAsync(polar, hp, sizeof hp, cudaMemcpyHostToDevice, st));
  SOUP_CUDA_TRY(cudaMemsetAsync(acc, 0, 4 * (5 * (size_t)n + 1), st));
  b.launches += 4;
  k_iota<<<nblocks(n), kBlock, 0, st>>>(parent, n);
  k_amph_union<<<nblocks(n), kBlock, 0, st>>>(b.slots, b.id, off, n, parent);
  k_amph_stats<<<nblocks(n), kBlock, 0, st>>>(b.pos, b.slots, b.id, off, n, polar, parent, acc, acc + n, acc + 2 * n,
                                                acc + 3 * n, acc + 4 * n);
  k_amph_label<<<nblocks(n), kBlock, 0, st>>>(n, parent, acc, acc + n, acc + 2 * n, acc + 3 * n, acc + 4 * n, dh,
                                                acc + 5 * n);
  SOUP_CUDA_TRY(cudaMemcpyAsync(head_of, dh, 4 * (size_t)n, cudaMemcpyDeviceToHost, st));
  uint32_t cnt = 0;
  SOUP_CUDA_TRY(cudaMemcpyAsync(&cnt, acc + 5 * n, 4, cudaMemcpyDeviceToHost, st));
  SOUP_CUDA_TRY(cudaStreamSynchronize(st));
  if (n_out) *n_out = cnt;
  return SOUP_OK;
}

int run_aggregates(Batch& b, uint32_t r, const uint32_t* mem, uint32_t m, double cutoff, uint32_t* labels,
                   uint32_t* ncomp, std::string& err) {
  const SoupConfig& c = b.cfg[r];
  const uint32_t n = c.n, off = b.hsp[r].slot_off;
  for (uint32_t k = 0; k < m; ++k) if (mem[k] >= n) { err = "aggregates: member index out of range"; return SOUP_E_ARG; }
  if (m == 0) { if (ncomp) *ncomp = 0; return SOUP_OK; }
  Grid g;
  for (int a = 0; a < 3; ++a) g.box[a] = c.box[a];
  g.nx = std::max(1, (int)std::floor(c.box[0] / cutoff));
  g.ny = std::max(1, (int)std::floor(c.box[1] / cutoff));
  g.nz = std::max(1, (int)std::floor(c.box[2] / cutoff));
  g.cell = 0;
  const uint32_t nc = (uint32_t)((uint64_t)g.nx * g.ny * g.nz);
  Scratch S;
  uint32_t* dmem = S.get<uint32_t>(m);
  uint32_t* cell = S.get<uint32_t>(m);
  uint32_t* count = S.get<uint32_t>(nc + 1);
  uint32_t* start = S.get<uint32_t>(nc + 1);
  uint32_t* cursor = S.get<uint32_t>(nc + 1);
  uint32_t* sorted = S.get<uint32_t>(m);
  uint32_t* parent = S.get<uint32_t>(m);
  uint32_t* minidx = S.get<uint32_t>(m);
  uint32_t* dl = S.get<uint32_t>(m);
  uint32_t* cnt = S.get<uint32_t>(1);
  uint32_t* tmp = S.get<uint32_t>(4 * (nc / 4096 + 64) + 256);
  cudaStream_t st = b.stream;
  SOUP_CUDA_TRY(cudaMemcpyAsync(dmem, mem, 4 * (size_t)m, cudaMemcpyHostToDevice, st));
  SOUP_CUDA_TRY(cudaMemsetAsync(count, 0, 4 * ((size_t)nc + 1), st));
  SOUP_CUDA_TRY(cudaMemsetAsync(cursor, 0, 4 * ((size_t)nc + 1), st));
  SOUP_CUDA_TRY(cudaMemsetAsync(cnt, 0, 4, st));
  b.launches += 8;
  k_agg_bin<<<nblocks(m), kBlock, 0, st>>>(b.pos, b.slot_of, off, dmem, m, g, c.box[0] / g.nx, c.box[1] / g.ny,
                                           c.box[2] / g.nz, cell, count);
  exclusive_scan(count, start, nc, tmp, st);
  k_agg_scatter<<<nblocks(m), kBlock, 0, st>>>(cell, m, start, cursor, sorted);
  k_iota<<<nblocks(m), kBlock, 0, st>>>(parent, m);
  k_fill<<<nblocks(m), kBlock, 0, st>>>(minidx, m, NONE);
  k_agg_union<<<nblocks(m), kBlock, 0, st>>>(b.pos, b.slot_of, off, dmem, m, g, cell, start, sorted, cutoff * cutoff, parent);
  k_agg_min<<<nblocks(m), kBlock, 0, st>>>(dmem, m, parent, minidx, cnt);
  k_agg_label<<<nblocks(m), kBlock, 0, st>>>(dmem, m, parent, minidx, dl);
  SOUP_CUDA_TRY(cudaMemcpyAsync(labels, dl, 4 * (size_t)m, cudaMemcpyDeviceToHost, st));
  uint32_t nco = 0;
  SOUP_CUDA_TRY(cudaMemcpyAsync(&nco, cnt, 4, cudaMemcpyDeviceToHost, st));
  SOUP_CUDA_TRY(cudaStreamSynchronize(st));
  if (ncomp) *ncomp = nco;
  return SOUP_OK;
}

}  // namespace soup

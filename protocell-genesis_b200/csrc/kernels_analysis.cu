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
// reachedEmpty counts only cells whose centre lies in the parcel when pr2 >= 0 (water-closure.ts:323-337)
__global__ void k_cell_counts(const uint8_t* __restrict__ occ, const uint32_t* __restrict__ vis, uint64_t nc, Grid g,
                              double pcx, double pcy, double pcz, double pr2,
                              unsigned long long* __restrict__ out /* totalEmpty, unreached, reachedEmpty */) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t a = 0, b = 0, c = 0;
  if (i < nc && !occ[i]) {
    a = 1;
    if (!vis[i]) {
      b = 1;
    } else if (pr2 < 0.0) {
      c = 1;
    } else {
      const int cz = (int)(i / ((uint64_t)g.nx * g.ny));
      const uint64_t rem = i - (uint64_t)cz * g.nx * g.ny;
      const int cy = (int)(rem / (uint64_t)g.nx), cx = (int)(rem - (uint64_t)cy * g.nx);
      const double ex = __dsub_rn(__dmul_rn(cx + 0.5, g.cell), pcx), ey = __dsub_rn(__dmul_rn(cy + 0.5, g.cell), pcy),
                   ez = __dsub_rn(__dmul_rn(cz + 0.5, g.cell), pcz);
      c = sq3(ex, ey, ez) > pr2 ? 0u : 1u;
    }
  }
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

// buildClusterUnionFind (aggregate.ts:65-130); one thread per member.  With periodic_z = 0 the z
// separation is the raw difference (the reference's periodicZ = false).  The binning stays the
// wrapped periodic grid: cells are at least `cutoff` wide, so a pair within the cutoff in raw z lies
// in neighbouring wrapped cells, and the raw difference rejects the pairs the wrap brings together.
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
                            int periodic_z, uint32_t* __restrict__ parent) {
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
          const double rz = __dsub_rn((double)pi.z, (double)pj.z);
          const double ddz = periodic_z ? mi1(rz, g.box[2]) : rz;
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

uint64_t exclusive_scan(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* tmp, cudaStream_t st);

char* analysis_scratch(Batch& b, size_t bytes, int which) {
  if (bytes > b.an_cap[which]) {
    SOUP_CUDA_TRY(cudaStreamSynchronize(b.stream));
    if (b.an_buf[which]) SOUP_CUDA_TRY(cudaFree(b.an_buf[which]));
    b.an_buf[which] = nullptr;
    b.an_cap[which] = 0;
    const size_t want = (bytes + (size_t(1) << 20) - 1) & ~((size_t(1) << 20) - 1);
    SOUP_CUDA_TRY(cudaMalloc(&b.an_buf[which], want));
    b.an_cap[which] = want;
  }
  return b.an_buf[which];
}

int run_closure(Batch& b, uint32_t r, const uint32_t* mem, uint32_t nm, const uint32_t* wat, uint32_t nw,
                const double centre[3], double cell, double radius, double vmin, const double* parcel,
                SoupClosureResult* out, std::string& err) {
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
  k_cell_counts<<<nblocks(nc), kBlock, 0, st>>>(occ, vis, nc, g, parcel ? parcel[0] : 0.0, parcel ? parcel[1] : 0.0,
                                                parcel ? parcel[2] : 0.0, parcel ? parcel[3] * parcel[3] : -1.0, u64 + 2);
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
                   uint32_t* ncomp, std::string& err, bool periodic_z) {
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
  k_agg_union<<<nblocks(m), kBlock, 0, st>>>(b.pos, b.slot_of, off, dmem, m, g, cell, start, sorted, cutoff * cutoff,
                                             periodic_z ? 1 : 0, parent);
  k_agg_min<<<nblocks(m), kBlock, 0, st>>>(dmem, m, parent, minidx, cnt);
  k_agg_label<<<nblocks(m), kBlock, 0, st>>>(dmem, m, parent, minidx, dl);
  SOUP_CUDA_TRY(cudaMemcpyAsync(labels, dl, 4 * (size_t)m, cudaMemcpyDeviceToHost, st));
  uint32_t nco = 0;
  SOUP_CUDA_TRY(cudaMemcpyAsync(&nco, cnt, 4, cudaMemcpyDeviceToHost, st));
  SOUP_CUDA_TRY(cudaStreamSynchronize(st));
  if (ncomp) *ncomp = nco;
  return SOUP_OK;
}

// ---- box scale: scaleMoleculesRigid and proximityPairs (soup/src/soup-box-scale-math.ts:63-221) ----
//
// The rigid units are the connected components of the rigid edges (covalent bonds, plus proximity
// pairs when cohesion is asked for).  Each component is walked breadth first from its smallest index,
// one level per launch, each bead's offset accumulated from its parent's across one edge through mi1,
// exactly the reference's per-edge construction.  Where a bead can be reached from several beads of
// the previous level (a cycle), the smallest of them is its parent: on a component that does not
// wrap the box every path gives the same offset up to FP64 rounding.  The centre of mass is an exact
// integer sum (offsets in units of 2^-44 sigma, split in two 64-bit accumulators), so it does not
// depend on the order the atomics land in.
namespace {

constexpr uint32_t kUnset = 0xFFFFFFFFu;
constexpr double kOffScale = 17592186044416.0;        // 2^44
constexpr double kOffLimit = 262144.0;                // 2^18 sigma: |offset| * 2^44 stays below 2^62

struct PGrid {
  int n[3];
  double box[3], w[3];
};

__device__ __forceinline__ int pcell_axis(double x, const PGrid& g, int a) {
  return min(g.n[a] - 1, (int)floor(__ddiv_rn(wrap1(x, g.box[a]), g.w[a])));
}

// the distinct cells among c-1, c, c+1 (periodic) on an axis of n cells
__device__ __forceinline__ int near_cells(int c, int n, int out[3]) {
  int k = 0;
  for (int d = -1; d <= 1; ++d) {
    const int v = ((c + d) % n + n) % n;
    bool seen = false;
    for (int q = 0; q < k; ++q) seen |= out[q] == v;
    if (!seen) out[k++] = v;
  }
  return k;
}

__global__ void k_bs_bond_count(const uint32_t* __restrict__ slots, uint32_t n, uint32_t* __restrict__ cnt) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t c = 0;
  for (int e = 0; e < 3; ++e) {
    const uint32_t j = slots[3 * (size_t)i + e];
    c += (j != NONE && j > i && j < n) ? 1u : 0u;
  }
  cnt[i] = c;
}

__global__ void k_bs_bin(const float4* __restrict__ pos, const uint8_t* __restrict__ elig, uint32_t n, PGrid g,
                         uint32_t* __restrict__ cell, uint32_t* __restrict__ ccount) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (!elig[i]) { cell[i] = kUnset; return; }
  const float4 p = pos[i];
  const int cx = pcell_axis((double)p.x, g, 0), cy = pcell_axis((double)p.y, g, 1), cz = pcell_axis((double)p.z, g, 2);
  const uint32_t c = (uint32_t)(((size_t)cz * g.n[1] + cy) * g.n[0] + cx);
  cell[i] = c;
  atomicAdd(&ccount[c], 1u);
}

__global__ void k_bs_cell_scatter(const uint32_t* __restrict__ cell, uint32_t n, const uint32_t* __restrict__ cstart,
                                  uint32_t* __restrict__ ccursor, uint32_t* __restrict__ csorted) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || cell[i] == kUnset) return;
  csorted[cstart[cell[i]] + atomicAdd(&ccursor[cell[i]], 1u)] = i;
}

// proximity pairs (i, j > i) of bead i: counted when `edges` is NULL, written from edges[2 * at] on
template <bool FILL>
__global__ void k_bs_prox(const float4* __restrict__ pos, const uint32_t* __restrict__ cell, uint32_t n, PGrid g,
                          const uint32_t* __restrict__ cstart, const uint32_t* __restrict__ csorted, double c2,
                          uint32_t* __restrict__ cnt, const uint32_t* __restrict__ at, uint32_t* __restrict__ edges) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || cell[i] == kUnset) return;
  const uint32_t ci = cell[i];
  const int cx = (int)(ci % (uint32_t)g.n[0]), cy = (int)((ci / (uint32_t)g.n[0]) % (uint32_t)g.n[1]),
            cz = (int)(ci / ((uint32_t)g.n[0] * (uint32_t)g.n[1]));
  int xs[3], ys[3], zs[3];
  const int nxs = near_cells(cx, g.n[0], xs), nys = near_cells(cy, g.n[1], ys), nzs = near_cells(cz, g.n[2], zs);
  const float4 pi = pos[i];
  uint32_t k = FILL ? at[i] : 0u;
  for (int a = 0; a < nxs; ++a)
    for (int b2 = 0; b2 < nys; ++b2)
      for (int c = 0; c < nzs; ++c) {
        const uint32_t cc = (uint32_t)(((size_t)zs[c] * g.n[1] + ys[b2]) * g.n[0] + xs[a]);
        for (uint32_t q = cstart[cc]; q < cstart[cc + 1]; ++q) {
          const uint32_t j = csorted[q];
          if (j <= i) continue;
          const float4 pj = pos[j];
          const double dx = mi1(__dsub_rn((double)pi.x, (double)pj.x), g.box[0]);
          const double dy = mi1(__dsub_rn((double)pi.y, (double)pj.y), g.box[1]);
          const double dz = mi1(__dsub_rn((double)pi.z, (double)pj.z), g.box[2]);
          if (sq3(dx, dy, dz) <= c2) {
            if (FILL) { edges[2 * (size_t)k] = i; edges[2 * (size_t)k + 1] = j; }
            ++k;
          }
        }
      }
  if (!FILL) cnt[i] += k;
}

__global__ void k_bs_bond_fill(const uint32_t* __restrict__ slots, uint32_t n, const uint32_t* __restrict__ at,
                               uint32_t* __restrict__ next, uint32_t* __restrict__ edges) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t k = at[i];
  for (int e = 0; e < 3; ++e) {
    const uint32_t j = slots[3 * (size_t)i + e];
    if (j != NONE && j > i && j < n) { edges[2 * (size_t)k] = i; edges[2 * (size_t)k + 1] = j; ++k; }
  }
  next[i] = k;   // where this bead's proximity pairs start
}

__global__ void k_bs_degree(const uint32_t* __restrict__ edges, uint32_t ne, uint32_t n, uint32_t* __restrict__ deg,
                            uint32_t* __restrict__ bad) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ne) return;
  const uint32_t i = edges[2 * (size_t)k], j = edges[2 * (size_t)k + 1];
  if (i >= n || j >= n) { atomicExch(bad, 1u); return; }
  atomicAdd(&deg[i], 1u);
  atomicAdd(&deg[j], 1u);
}

__global__ void k_bs_adjacency(const uint32_t* __restrict__ edges, uint32_t ne, uint32_t n,
                               const uint32_t* __restrict__ astart, uint32_t* __restrict__ acursor,
                               uint32_t* __restrict__ adj) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ne) return;
  const uint32_t i = edges[2 * (size_t)k], j = edges[2 * (size_t)k + 1];
  if (i >= n || j >= n) return;
  adj[astart[i] + atomicAdd(&acursor[i], 1u)] = j;
  adj[astart[j] + atomicAdd(&acursor[j], 1u)] = i;
}

__global__ void k_bs_union(const uint32_t* __restrict__ edges, uint32_t ne, uint32_t n, uint32_t* __restrict__ parent) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ne) return;
  const uint32_t i = edges[2 * (size_t)k], j = edges[2 * (size_t)k + 1];
  if (i < n && j < n) uf_union(parent, i, j);
}

// roots (the smallest index of each component) start the walk at level 0 with a zero offset
__global__ void k_bs_roots(uint32_t* __restrict__ parent, uint32_t n, uint32_t* __restrict__ level,
                           uint32_t* __restrict__ cand, double* __restrict__ off, uint32_t* __restrict__ front,
                           uint32_t* __restrict__ nfront) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t r = uf_find(parent, i);
  cand[i] = kUnset;
  if (r == i) {
    level[i] = 0;
    off[3 * (size_t)i] = 0.0; off[3 * (size_t)i + 1] = 0.0; off[3 * (size_t)i + 2] = 0.0;
    front[atomicAdd(nfront, 1u)] = i;
  } else {
    level[i] = kUnset;
  }
}

__global__ void k_bs_root_store(uint32_t* __restrict__ parent, uint32_t n, uint32_t* __restrict__ root) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) root[i] = uf_find(parent, i);
}

// one level: every unreached neighbour of the frontier takes the smallest frontier bead as parent
__global__ void k_bs_claim(const uint32_t* __restrict__ front, const uint32_t* __restrict__ nfront,
                           const uint32_t* __restrict__ astart, const uint32_t* __restrict__ adj,
                           const uint32_t* __restrict__ level, uint32_t* __restrict__ cand, uint32_t* __restrict__ next,
                           uint32_t* __restrict__ nnext) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= *nfront) return;
  const uint32_t p = front[k];
  for (uint32_t q = astart[p]; q < astart[p + 1]; ++q) {
    const uint32_t c = adj[q];
    if (level[c] != kUnset) continue;
    if (atomicMin(&cand[c], p) == kUnset) next[atomicAdd(nnext, 1u)] = c;
  }
}

__global__ void k_bs_settle(const uint32_t* __restrict__ next, const uint32_t* __restrict__ nnext, uint32_t lev,
                            const float4* __restrict__ pos, const uint32_t* __restrict__ cand, Grid ob,
                            uint32_t* __restrict__ level, double* __restrict__ off) {
  const uint32_t m = *nnext;   // the size of the new level, known only on the device: grid-stride
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
    const uint32_t c = next[k], p = cand[c];
    const float4 pc = pos[c], pp = pos[p];
    level[c] = lev;
    off[3 * (size_t)c] = __dadd_rn(off[3 * (size_t)p], mi1(__dsub_rn((double)pc.x, (double)pp.x), ob.box[0]));
    off[3 * (size_t)c + 1] = __dadd_rn(off[3 * (size_t)p + 1], mi1(__dsub_rn((double)pc.y, (double)pp.y), ob.box[1]));
    off[3 * (size_t)c + 2] = __dadd_rn(off[3 * (size_t)p + 2], mi1(__dsub_rn((double)pc.z, (double)pp.z), ob.box[2]));
  }
}

// exact per-component sums of the offsets: value * 2^44 rounded, high part (>> 24) and low 24 bits
// accumulated separately so neither 64-bit sum can overflow
__global__ void k_bs_accumulate(const uint32_t* __restrict__ root, const double* __restrict__ off, uint32_t n,
                                unsigned long long* __restrict__ acc, uint32_t* __restrict__ cnt,
                                uint32_t* __restrict__ bad) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t r = root[i];
  for (int a = 0; a < 3; ++a) {
    const double o = off[3 * (size_t)i + a];
    if (!(fabs(o) < kOffLimit)) { atomicExch(bad, 2u); return; }
    const long long t = __double2ll_rn(__dmul_rn(o, kOffScale));
    const long long hi = t >> 24, lo = t & 0xFFFFFFll;
    atomicAdd(&acc[6 * (size_t)r + a], (unsigned long long)hi);
    atomicAdd(&acc[6 * (size_t)r + 3 + a], (unsigned long long)lo);
  }
  atomicAdd(&cnt[r], 1u);
}

// out = wrap1(wrap1(root + centre, old) * s + (offset - centre), new), the reference's expression order
__global__ void k_bs_place(const float4* __restrict__ pos, const uint32_t* __restrict__ root,
                           const double* __restrict__ off, const unsigned long long* __restrict__ acc,
                           const uint32_t* __restrict__ cnt, uint32_t n, Grid ob, Grid nb, double sx, double sy,
                           double sz, float4* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t r = root[i];
  const float4 pr = pos[r], pi = pos[i];
  const double s[3] = {sx, sy, sz};
  const double rp[3] = {(double)pr.x, (double)pr.y, (double)pr.z};
  float o3[3];
  for (int a = 0; a < 3; ++a) {
    const double hi = (double)(long long)acc[6 * (size_t)r + a], lo = (double)(long long)acc[6 * (size_t)r + 3 + a];
    const double sum = __dmul_rn(__dadd_rn(__dmul_rn(hi, 16777216.0), lo), 1.0 / kOffScale);
    const double cen = __ddiv_rn(sum, (double)cnt[r]);
    const double com = __dmul_rn(wrap1(__dadd_rn(rp[a], cen), ob.box[a]), s[a]);
    o3[a] = __double2float_rn(wrap1(__dadd_rn(com, __dsub_rn(off[3 * (size_t)i + a], cen)), nb.box[a]));
  }
  out[i] = make_float4(o3[0], o3[1], o3[2], pi.w);
}

__device__ __forceinline__ double mi3_distance(float4 a, float4 b, const Grid& g) {
  const double dx = mi1(__dsub_rn((double)a.x, (double)b.x), g.box[0]);
  const double dy = mi1(__dsub_rn((double)a.y, (double)b.y), g.box[1]);
  const double dz = mi1(__dsub_rn((double)a.z, (double)b.z), g.box[2]);
  return __dsqrt_rn(sq3(dx, dy, dz));
}

// applyBoxScaleOnce's self-check (soup/src/soup-box-scale.ts:117-128): the smallest edge index whose
// length moved by more than 1e-3
__global__ void k_bs_check(const uint32_t* __restrict__ edges, uint32_t ne, const float4* __restrict__ before,
                           const float4* __restrict__ after, Grid ob, Grid nb, uint32_t* __restrict__ first_bad) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ne) return;
  const uint32_t i = edges[2 * (size_t)k], j = edges[2 * (size_t)k + 1];
  const double d0 = mi3_distance(before[i], before[j], ob), d1 = mi3_distance(after[i], after[j], nb);
  if (fabs(d1 - d0) > 1e-3) atomicMin(first_bad, k);
}

}  // namespace

int run_rigid_map(Batch& b, const float4* pos_o, const uint32_t* slots_o, uint32_t n, const uint32_t* edges_host,
                  uint64_t n_edges_host, double cohesion, const uint8_t* eligible_host, const double old_box[3],
                  const double new_box[3], float4* out_o, bool check, std::string& err) {
  if (n == 0) return SOUP_OK;
  cudaStream_t st = b.stream;
  const bool prox = !edges_host && cohesion > 0;
  PGrid pg{};
  uint32_t ncell = 0;
  if (prox) {
    uint64_t nc = 1;
    for (int a = 0; a < 3; ++a) {
      pg.n[a] = std::max(1, (int)std::floor(old_box[a] / cohesion));
      pg.box[a] = old_box[a];
      pg.w[a] = old_box[a] / pg.n[a];
      nc *= (uint64_t)pg.n[a];
    }
    if (nc >= 0xFFFFFFF0ull) { err = "scaleBoxTo: the cohesion cutoff gives too many cells"; return SOUP_E_ARG; }
    ncell = (uint32_t)nc;
  }
  const uint32_t scan_words = std::max(4 * ((n + 1) / 4096 + 64) + 256, 4 * (ncell / 4096 + 64) + 256);
  // per-bead buffers, known before the edges are counted
  ScratchLayout L;
  const size_t o_elig = L.add<uint8_t>(n), o_cell = L.add<uint32_t>(n), o_ccount = L.add<uint32_t>(ncell + 1),
               o_cstart = L.add<uint32_t>(ncell + 1), o_ccur = L.add<uint32_t>(ncell + 1), o_csorted = L.add<uint32_t>(n),
               o_ecnt = L.add<uint32_t>(n + 1), o_estart = L.add<uint32_t>(n + 1), o_enext = L.add<uint32_t>(n),
               o_deg = L.add<uint32_t>(n + 1), o_astart = L.add<uint32_t>(n + 1), o_acur = L.add<uint32_t>(n),
               o_parent = L.add<uint32_t>(n), o_root = L.add<uint32_t>(n), o_level = L.add<uint32_t>(n),
               o_cand = L.add<uint32_t>(n), o_fa = L.add<uint32_t>(n), o_fb = L.add<uint32_t>(n),
               o_off = L.add<double>(3 * (size_t)n), o_acc = L.add<unsigned long long>(6 * (size_t)n),
               o_cnt = L.add<uint32_t>(n), o_misc = L.add<uint32_t>(8), o_tmp = L.add<uint32_t>(scan_words);
  char* base = analysis_scratch(b, L.used, 0);
  auto at = [base](size_t o) { return reinterpret_cast<uint32_t*>(base + o); };
  uint8_t* elig = reinterpret_cast<uint8_t*>(base + o_elig);
  uint32_t *cell = at(o_cell), *ccount = at(o_ccount), *cstart = at(o_cstart), *ccur = at(o_ccur), *csorted = at(o_csorted),
           *ecnt = at(o_ecnt), *estart = at(o_estart), *enext = at(o_enext), *deg = at(o_deg), *astart = at(o_astart),
           *acur = at(o_acur), *parent = at(o_parent), *root = at(o_root), *level = at(o_level), *cand = at(o_cand),
           *fa = at(o_fa), *fb = at(o_fb), *cnt = at(o_cnt), *misc = at(o_misc), *tmp = at(o_tmp);
  double* off = reinterpret_cast<double*>(base + o_off);
  unsigned long long* acc = reinterpret_cast<unsigned long long*>(base + o_acc);
  SOUP_CUDA_TRY(cudaMemsetAsync(misc, 0, 32, st));

  // ---- the rigid edges ----
  uint64_t ne64 = n_edges_host;
  uint32_t* edges = nullptr;
  if (edges_host) {
    if (ne64 >= 0x7FFFFFFFull) { err = "scaleMoleculesRigid: too many edges"; return SOUP_E_ARG; }
    edges = reinterpret_cast<uint32_t*>(analysis_scratch(b, 8 * std::max<uint64_t>(ne64, 1) * 2, 1));
    if (ne64) SOUP_CUDA_TRY(cudaMemcpyAsync(edges, edges_host, 8 * ne64, cudaMemcpyHostToDevice, st));
  } else {
    k_bs_bond_count<<<nblocks(n), kBlock, 0, st>>>(slots_o, n, ecnt);
    b.launches += 1;
    if (prox) {
      if (eligible_host) SOUP_CUDA_TRY(cudaMemcpyAsync(elig, eligible_host, n, cudaMemcpyHostToDevice, st));
      else SOUP_CUDA_TRY(cudaMemsetAsync(elig, 1, n, st));
      SOUP_CUDA_TRY(cudaMemsetAsync(ccount, 0, 4 * ((size_t)ncell + 1), st));
      SOUP_CUDA_TRY(cudaMemsetAsync(ccur, 0, 4 * ((size_t)ncell + 1), st));
      k_bs_bin<<<nblocks(n), kBlock, 0, st>>>(pos_o, elig, n, pg, cell, ccount);
      exclusive_scan(ccount, cstart, ncell, tmp, st);
      k_bs_cell_scatter<<<nblocks(n), kBlock, 0, st>>>(cell, n, cstart, ccur, csorted);
      k_bs_prox<false><<<nblocks(n), kBlock, 0, st>>>(pos_o, cell, n, pg, cstart, csorted, cohesion * cohesion, ecnt,
                                                      nullptr, nullptr);
      b.launches += 4;
    }
    exclusive_scan(ecnt, estart, n, tmp, st);
    uint32_t total = 0;
    SOUP_CUDA_TRY(cudaMemcpyAsync(&total, estart + n, 4, cudaMemcpyDeviceToHost, st));
    SOUP_CUDA_TRY(cudaStreamSynchronize(st));
    ne64 = total;
    edges = reinterpret_cast<uint32_t*>(analysis_scratch(b, 8 * std::max<uint64_t>(ne64, 1) * 2, 1));
    k_bs_bond_fill<<<nblocks(n), kBlock, 0, st>>>(slots_o, n, estart, enext, edges);
    b.launches += 1;
    if (prox) {
      k_bs_prox<true><<<nblocks(n), kBlock, 0, st>>>(pos_o, cell, n, pg, cstart, csorted, cohesion * cohesion, nullptr,
                                                     enext, edges);
      b.launches += 1;
    }
  }
  const uint32_t ne = (uint32_t)ne64;
  uint32_t* adj = edges + 2 * (size_t)std::max<uint32_t>(ne, 1);

  // ---- adjacency and components ----
  SOUP_CUDA_TRY(cudaMemsetAsync(deg, 0, 4 * ((size_t)n + 1), st));
  SOUP_CUDA_TRY(cudaMemsetAsync(acur, 0, 4 * (size_t)n, st));
  SOUP_CUDA_TRY(cudaMemsetAsync(acc, 0, 48 * (size_t)n, st));
  SOUP_CUDA_TRY(cudaMemsetAsync(cnt, 0, 4 * (size_t)n, st));
  k_iota<<<nblocks(n), kBlock, 0, st>>>(parent, n);
  b.launches += 1;
  if (ne) {
    k_bs_degree<<<nblocks(ne), kBlock, 0, st>>>(edges, ne, n, deg, misc + 4);
    exclusive_scan(deg, astart, n, tmp, st);
    k_bs_adjacency<<<nblocks(ne), kBlock, 0, st>>>(edges, ne, n, astart, acur, adj);
    k_bs_union<<<nblocks(ne), kBlock, 0, st>>>(edges, ne, n, parent);
    b.launches += 3;
  } else {
    SOUP_CUDA_TRY(cudaMemsetAsync(astart, 0, 4 * ((size_t)n + 1), st));
  }
  k_bs_roots<<<nblocks(n), kBlock, 0, st>>>(parent, n, level, cand, off, fa, misc);
  k_bs_root_store<<<nblocks(n), kBlock, 0, st>>>(parent, n, root);
  b.launches += 2;
  uint32_t h[2] = {0, 0};
  SOUP_CUDA_TRY(cudaMemcpyAsync(h, misc + 4, 4, cudaMemcpyDeviceToHost, st));
  SOUP_CUDA_TRY(cudaMemcpyAsync(h + 1, misc, 4, cudaMemcpyDeviceToHost, st));
  SOUP_CUDA_TRY(cudaStreamSynchronize(st));
  if (h[0]) { err = "scaleMoleculesRigid: an edge names a particle outside the system"; return SOUP_E_ARG; }

  // ---- breadth-first walk, one level per launch pair ----
  Grid ob{}, nb{};
  for (int a = 0; a < 3; ++a) { ob.box[a] = old_box[a]; nb.box[a] = new_box[a]; }
  uint32_t* front = fa; uint32_t* next = fb;
  uint32_t* nfront = misc; uint32_t* nnext = misc + 1;
  uint32_t level_size = h[1];
  for (uint32_t lev = 1; level_size > 0 && ne; ++lev) {
    if (lev > n) { err = "scaleMoleculesRigid: the walk did not finish"; return SOUP_E_STATE; }
    SOUP_CUDA_TRY(cudaMemsetAsync(nnext, 0, 4, st));
    k_bs_claim<<<nblocks(level_size), kBlock, 0, st>>>(front, nfront, astart, adj, level, cand, next, nnext);
    k_bs_settle<<<std::min(nblocks(n), 148u * 8u), kBlock, 0, st>>>(next, nnext, lev, pos_o, cand, ob, level, off);
    b.launches += 2;
    SOUP_CUDA_TRY(cudaMemcpyAsync(&level_size, nnext, 4, cudaMemcpyDeviceToHost, st));
    SOUP_CUDA_TRY(cudaStreamSynchronize(st));
    std::swap(front, next);
    std::swap(nfront, nnext);
  }

  // ---- centres, positions, self-check ----
  k_bs_accumulate<<<nblocks(n), kBlock, 0, st>>>(root, off, n, acc, cnt, misc + 4);
  k_bs_place<<<nblocks(n), kBlock, 0, st>>>(pos_o, root, off, acc, cnt, n, ob, nb, new_box[0] / old_box[0],
                                            new_box[1] / old_box[1], new_box[2] / old_box[2], out_o);
  const uint32_t none = kUnset;
  SOUP_CUDA_TRY(cudaMemcpyAsync(misc + 5, &none, 4, cudaMemcpyHostToDevice, st));
  b.launches += 2;
  if (ne && check) {
    k_bs_check<<<nblocks(ne), kBlock, 0, st>>>(edges, ne, pos_o, out_o, ob, nb, misc + 5);
    b.launches += 1;
  }
  uint32_t res[2];
  SOUP_CUDA_TRY(cudaMemcpyAsync(res, misc + 4, 8, cudaMemcpyDeviceToHost, st));
  SOUP_CUDA_TRY(cudaStreamSynchronize(st));
  SOUP_CUDA_TRY(cudaGetLastError());
  if (res[0] == 2) { err = "scaleMoleculesRigid: a rigid unit extends beyond 262144 sigma from its first bead"; return SOUP_E_STATE; }
  if (res[1] != kUnset) {
    uint32_t e[2];
    float4 p0[2], p1[2];
    SOUP_CUDA_TRY(cudaMemcpy(e, edges + 2 * (size_t)res[1], 8, cudaMemcpyDeviceToHost));
    for (int q = 0; q < 2; ++q) {
      SOUP_CUDA_TRY(cudaMemcpy(&p0[q], pos_o + e[q], 16, cudaMemcpyDeviceToHost));
      SOUP_CUDA_TRY(cudaMemcpy(&p1[q], out_o + e[q], 16, cudaMemcpyDeviceToHost));
    }
    auto dist = [](const float4& a, const float4& c, const double* L) {
      auto m = [](double d, double l) { double x = d / l, r = std::floor(x); r = (x - r >= 0.5) ? r + 1 : r; return d - r * l; };
      const double dx = m((double)a.x - c.x, L[0]), dy = m((double)a.y - c.y, L[1]), dz = m((double)a.z - c.z, L[2]);
      return std::sqrt(dx * dx + dy * dy + dz * dz);
    };
    char m[400];
    std::snprintf(m, sizeof m,
                  "applyBoxScale: an intramolecular distance changed (%.6f -> %.6f) for bond %u-%u at box [%g,%g,%g] -> "
                  "[%g,%g,%g] -- scaleMoleculesRigid is broken",
                  dist(p0[0], p0[1], old_box), dist(p1[0], p1[1], new_box), e[0], e[1], old_box[0], old_box[1],
                  old_box[2], new_box[0], new_box[1], new_box[2]);
    err = m;
    return SOUP_E_STATE;
  }
  return SOUP_OK;
}

}  // namespace soup

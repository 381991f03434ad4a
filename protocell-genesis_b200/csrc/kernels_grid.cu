// kernels_grid.cu -- cell binning, the deterministic re-sort, and the Verlet / head list builds.
//
// Reference: engine/wgsl/neighbor.wgsl:19-64 (clear/count/prefix/fill: an atomic counting sort with a
// one-thread prefix sum and an atomic, run-to-run varying fill order), soup/wgsl/verlet.wgsl:53-92
// (per-particle walk of (2R+1)^3 cells, keep |mi3(xi-xj)| < listRange), soup/wgsl/
// electrostatics-long.wgsl:15-56 (serial head compaction, O(N_h^2) head list).
//
// Here: a parallel counting sort whose order inside a cell is fixed (ascending original index), so
// every array is physically reordered into cell order at each rebuild (coalesced neighbour reads);
// list membership uses the exact f32 test of the reference, so the lists equal the oracle's sets.
// Walks are over x-rows of cells (contiguous slot ranges), a row at a time.
#include "soup_internal.h"

namespace soup {

namespace {

constexpr int kBlock = 256;
inline unsigned nblocks(uint64_t n, int b = kBlock) { return (unsigned)((n + b - 1) / b); }

__global__ void k_cell_index(const float4* __restrict__ pos, const uint8_t* __restrict__ sysid,
                             const SysParams* __restrict__ sp, uint32_t N, uint32_t* __restrict__ cell_of,
                             uint32_t* __restrict__ count) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  const SysParams& P = sp[sysid[k]];
  float4 p = pos[k];
  int cx = ex_cell_axis(p.x, P.box[0], P.dims[0]);
  int cy = ex_cell_axis(p.y, P.box[1], P.dims[1]);
  int cz = ex_cell_axis(p.z, P.box[2], P.dims[2]);
  uint32_t c = P.cell_off + (uint32_t)(cx + P.dims[0] * (cy + P.dims[1] * cz));
  cell_of[k] = c;
  atomicAdd(&count[c], 1u);
}

// Exclusive scan, 4 elements per thread, 1024 threads per block: block-local scan + block totals.
__global__ void k_scan_block(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, uint32_t n,
                             uint32_t* __restrict__ block_sums) {
  __shared__ uint32_t warp_tot[32];
  const uint32_t base = blockIdx.x * 4096u + threadIdx.x * 4u;
  uint32_t v[4];
  uint32_t t = 0;
  for (int e = 0; e < 4; ++e) { v[e] = (base + e < n) ? in[base + e] : 0u; t += v[e]; }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t incl = t;
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) warp_tot[w] = incl;
  __syncthreads();
  if (w == 0) {
    uint32_t x = warp_tot[lane];
    uint32_t xi = x;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, xi, o);
      if (lane >= o) xi += y;
    }
    warp_tot[lane] = xi - x;  // exclusive
    if (lane == 31 && block_sums) block_sums[blockIdx.x] = xi;
  }
  __syncthreads();
  uint32_t run = warp_tot[w] + incl - t;
  for (int e = 0; e < 4; ++e) {
    if (base + e < n) out[base + e] = run;
    run += v[e];
  }
}
__global__ void k_scan_add(uint32_t* __restrict__ out, uint32_t n, const uint32_t* __restrict__ block_offs) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] += block_offs[i / 4096u];
}
__global__ void k_set_total(uint32_t* __restrict__ start, const uint32_t* __restrict__ count, uint32_t n) {
  start[n] = start[n - 1] + count[n - 1];
}

}  // namespace

// exclusive scan of in[0..n) into out[0..n), out[n] = total; tmp must hold >= 2*ceil(n/4096)+2 words.
// Returns the kernels it launched (no shared counter: calls from several host threads do not race).
uint64_t exclusive_scan(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* tmp, cudaStream_t st) {
  if (n == 0) return 0;
  uint64_t launches = 2;
  uint32_t nb = (n + 4095) / 4096;
  if (nb == 1) {
    k_scan_block<<<1, 1024, 0, st>>>(in, out, n, nullptr);
  } else {
    uint32_t* sums = tmp;
    uint32_t* offs = tmp + nb + 1;
    k_scan_block<<<nb, 1024, 0, st>>>(in, out, n, sums);
    launches += exclusive_scan(sums, offs, nb, offs + nb + 1, st) + 1;
    k_scan_add<<<nblocks(n), kBlock, 0, st>>>(out, n, offs);
  }
  k_set_total<<<1, 1, 0, st>>>(out, in, n);
  return launches;
}

namespace {

__global__ void k_scatter(const uint32_t* __restrict__ cell_of, const uint32_t* __restrict__ start, uint32_t N,
                          uint32_t* __restrict__ cursor, uint32_t* __restrict__ perm) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  uint32_t c = cell_of[k];
  perm[start[c] + atomicAdd(&cursor[c], 1u)] = k;
}

// Inside each cell, order by original index: the atomic scatter order above varies run to run, this
// makes the slot order (and therefore every summation order) deterministic.
__global__ void k_sort_cells(const uint32_t* __restrict__ start, uint32_t ncells, const uint32_t* __restrict__ id,
                             uint32_t* __restrict__ perm) {
  uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncells) return;
  uint32_t a = start[c], e = start[c + 1];
  for (uint32_t x = a + 1; x < e; ++x) {
    uint32_t v = perm[x];
    uint32_t key = id[v];
    uint32_t y = x;
    while (y > a && id[perm[y - 1]] > key) { perm[y] = perm[y - 1]; --y; }
    perm[y] = v;
  }
}

__global__ void k_gather(uint32_t N, const uint32_t* __restrict__ perm,
                         const float4* __restrict__ pos, const float4* __restrict__ vel, const float4* __restrict__ force,
                         const float* __restrict__ charge, const uint32_t* __restrict__ slots,
                         const uint32_t* __restrict__ center, const uint32_t* __restrict__ held,
                         const uint32_t* __restrict__ brng, const uint32_t* __restrict__ trng,
                         const uint8_t* __restrict__ frozen, const uint32_t* __restrict__ id,
                         float4* __restrict__ pos2, float4* __restrict__ vel2, float4* __restrict__ force2,
                         float* __restrict__ charge2, uint32_t* __restrict__ slots2, uint32_t* __restrict__ center2,
                         uint32_t* __restrict__ held2, uint32_t* __restrict__ brng2, uint32_t* __restrict__ trng2,
                         uint8_t* __restrict__ frozen2, uint32_t* __restrict__ id2, uint32_t* __restrict__ slot_of,
                         float4* __restrict__ pos_ref) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  uint32_t o = perm[k];
  float4 p = pos[o];
  pos2[k] = p;
  pos_ref[k] = p;
  vel2[k] = vel[o];
  force2[k] = force[o];
  charge2[k] = charge[o];
  slots2[3 * k + 0] = slots[3 * o + 0];
  slots2[3 * k + 1] = slots[3 * o + 1];
  slots2[3 * k + 2] = slots[3 * o + 2];
  center2[k] = center[o];
  held2[k] = held[o];
  brng2[k] = brng[o];
  trng2[k] = trng[o];
  frozen2[k] = frozen[o];
  uint32_t g = id[o];
  id2[k] = g;
  slot_of[g] = k;
}

// the gathered arrays back into the primary buffers, so every array keeps its address across rebuilds
// (a captured step graph holds them as kernel arguments)
__global__ void k_copy_back(uint32_t N, const float4* __restrict__ pos2, const float4* __restrict__ vel2,
                            const float4* __restrict__ force2, const float* __restrict__ charge2,
                            const uint32_t* __restrict__ slots2, const uint32_t* __restrict__ center2,
                            const uint32_t* __restrict__ held2, const uint32_t* __restrict__ brng2,
                            const uint32_t* __restrict__ trng2, const uint8_t* __restrict__ frozen2,
                            const uint32_t* __restrict__ id2, float4* __restrict__ pos, float4* __restrict__ vel,
                            float4* __restrict__ force, float* __restrict__ charge, uint32_t* __restrict__ slots,
                            uint32_t* __restrict__ center, uint32_t* __restrict__ held, uint32_t* __restrict__ brng,
                            uint32_t* __restrict__ trng, uint8_t* __restrict__ frozen, uint32_t* __restrict__ id) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  pos[k] = pos2[k]; vel[k] = vel2[k]; force[k] = force2[k]; charge[k] = charge2[k];
  slots[3 * k] = slots2[3 * k]; slots[3 * k + 1] = slots2[3 * k + 1]; slots[3 * k + 2] = slots2[3 * k + 2];
  center[k] = center2[k]; held[k] = held2[k]; brng[k] = brng2[k]; trng[k] = trng2[k]; frozen[k] = frozen2[k];
  id[k] = id2[k];
}

// Distinct wrapped cell coordinates of a +-R walk along one axis, as at most two [lo,hi] intervals.
struct AxisRange { int lo[2], hi[2], n; };
__device__ __forceinline__ AxisRange axis_ranges(int q, int R, int dim) {
  AxisRange a;
  int lo = q - R, hi = q + R;
  if (hi - lo + 1 >= dim) { a.n = 1; a.lo[0] = 0; a.hi[0] = dim - 1; }
  else if (lo < 0) { a.n = 2; a.lo[0] = lo + dim; a.hi[0] = dim - 1; a.lo[1] = 0; a.hi[1] = hi; }
  else if (hi >= dim) { a.n = 2; a.lo[0] = lo; a.hi[0] = dim - 1; a.lo[1] = 0; a.hi[1] = hi - dim; }
  else { a.n = 1; a.lo[0] = lo; a.hi[0] = hi; }
  return a;
}

// The cells lo..hi (unwrapped, hi - lo + 1 < dim) as at most two wrapped [lo,hi] intervals, in the
// order axis_ranges gives them.
__device__ __forceinline__ AxisRange span_ranges(int lo, int hi, int dim) {
  AxisRange a;
  if (lo < 0) { a.n = 2; a.lo[0] = lo + dim; a.hi[0] = dim - 1; a.lo[1] = 0; a.hi[1] = hi; }
  else if (hi >= dim) { a.n = 2; a.lo[0] = lo; a.hi[0] = dim - 1; a.lo[1] = 0; a.hi[1] = hi - dim; }
  else { a.n = 1; a.lo[0] = lo; a.hi[0] = hi; }
  if (a.n == 2 && a.lo[1] > a.hi[1]) a.n = 1;
  if (a.n == 2 && a.lo[0] > a.hi[0]) { a.n = 1; a.lo[0] = a.lo[1]; a.hi[0] = a.hi[1]; }
  return a;
}
// distance from p to the cell interval [c cs, (c + 1) cs) along one axis (unwrapped c), less a
// margin for the rounding of the cell assignment
__device__ __forceinline__ float gap_to_cell(float p, int c, float cs) {
  const float lo = (float)c * cs - p, hi = (float)(c + 1) * cs - p;
  return fmaxf(0.f, fmaxf(lo, -hi) - 1e-4f);
}

// The build-distance shell of a list entry, carried in its top three bits until k_group_rows groups
// the row: 0 inside the force's reach (sqrt(rmax2)), 1..4 the rest of the list range in four equal
// widths.  A force pass needs shell k > 0 only once the largest displacement since the build can have
// closed (k - 1) widths (list_force_end).
struct Shells {
  float reach2, e1, e2, e3;
  __device__ __forceinline__ static Shells of(float rmax2, float list_range) {
    Shells s;
    const float r0 = sqrtf(rmax2), w = fmaxf(list_range - r0, 0.f) * 0.25f;
    s.reach2 = rmax2;
    s.e1 = (r0 + w) * (r0 + w); s.e2 = (r0 + 2.f * w) * (r0 + 2.f * w); s.e3 = (r0 + 3.f * w) * (r0 + 3.f * w);
    return s;
  }
  __device__ __forceinline__ uint32_t tag(float r2) const {
    const uint32_t k = r2 < reach2 ? 0u : 1u + (r2 >= e1) + (r2 >= e2) + (r2 >= e3);
    return k << 29;
  }
};

// soup/wgsl/verlet.wgsl:53-92, thread per particle, rows of cells as contiguous slot ranges.  When
// the walk does not wrap onto itself, each (y, z) row of cells is trimmed to the x cells that can
// reach the list sphere (with a margin) and rows wholly outside it are skipped; the accept test is
// unchanged, so the list is the same set.
__global__ void __launch_bounds__(128) k_build_list(
    const float4* __restrict__ pos, const uint8_t* __restrict__ sysid, const SysParams* __restrict__ sp,
    const uint32_t* __restrict__ cell_of, const uint32_t* __restrict__ start, uint32_t N, uint32_t cap,
    float rmax2, uint32_t* __restrict__ nl, uint32_t* __restrict__ nl_cnt, uint32_t* __restrict__ flags) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  const SysParams& P = sp[sysid[k]];
  const Shells sh = Shells::of(rmax2, P.list_range);
  const float4 xi = pos[k];
  const float box[3] = {P.box[0], P.box[1], P.box[2]};
  const float inv[3] = {P.inv_box[0], P.inv_box[1], P.inv_box[2]};
  const float lr = P.list_range;
  // fast squared distance decides unless it lies within 1e-5 of the range, where the exact
  // reference arithmetic decides (the minimum image cannot differ there: range < box/2)
  const float lr2_lo = lr * lr * (1.0f - 1e-5f), lr2_hi = lr * lr * (1.0f + 1e-5f);
  uint32_t c = cell_of[k] - P.cell_off;
  int qx = (int)(c % (uint32_t)P.dims[0]);
  int qy = (int)((c / (uint32_t)P.dims[0]) % (uint32_t)P.dims[1]);
  int qz = (int)(c / ((uint32_t)P.dims[0] * (uint32_t)P.dims[1]));
  const int R = P.walk;
  AxisRange ax = axis_ranges(qx, R, P.dims[0]);
  // distinct y and z coordinates in walk order
  int ys[16], zs[16], ny = 0, nz = 0;
  for (int d = -R; d <= R; ++d) {
    int y = ((qy + d) % P.dims[1] + P.dims[1]) % P.dims[1];
    bool dup = false;
    for (int t = 0; t < ny; ++t) dup |= ys[t] == y;
    if (!dup) ys[ny++] = y;
    int z = ((qz + d) % P.dims[2] + P.dims[2]) % P.dims[2];
    dup = false;
    for (int t = 0; t < nz; ++t) dup |= zs[t] == z;
    if (!dup) zs[nz++] = z;
  }
  uint32_t cnt = 0;
  uint32_t* row = nl + (size_t)k * cap;
  // a warp whose particles lie at least the list range inside every face screens with plain
  // differences: a candidate within the range sits at its stored coordinates (fast_mi would return the
  // same difference), and one beyond it by the plain difference is beyond it by the minimum image too
  const float rm = lr * (1.0f + 1e-5f) + 1e-3f;
  const bool direct = __all_sync(__activemask(), xi.x >= rm && xi.x <= box[0] - rm && xi.y >= rm &&
                                                   xi.y <= box[1] - rm && xi.z >= rm && xi.z <= box[2] - rm);
  auto take = [&](uint32_t a, uint32_t e) {
    for (uint32_t j = a; j < e; ++j) {
      if (j == k) continue;
      const float4 xj = pos[j];
      float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
      if (!direct) {
        dx = fast_mi(dx, box[0], inv[0]);
        dy = fast_mi(dy, box[1], inv[1]);
        dz = fast_mi(dz, box[2], inv[2]);
      }
      const float r2 = dx * dx + dy * dy + dz * dz;
      if (r2 > lr2_hi) continue;
      if (r2 >= lr2_lo && !(ex_dist(xi, xj, box) < lr)) continue;
      if (cnt < cap) row[cnt] = j | sh.tag(r2);
      ++cnt;
    }
  };
  if (P.dims[0] >= 2 * R + 1 && P.dims[1] >= 2 * R + 1 && P.dims[2] >= 2 * R + 1) {
    const float cs[3] = {box[0] / (float)P.dims[0], box[1] / (float)P.dims[1], box[2] / (float)P.dims[2]};
    const float lrm = lr * (1.0f + 1e-5f) + 1e-3f, lrm2 = lrm * lrm;
    for (int oz = -R; oz <= R; ++oz) {
      const float gz = gap_to_cell(xi.z, qz + oz, cs[2]);
      const int cz = (qz + oz + P.dims[2]) % P.dims[2];
      for (int oy = -R; oy <= R; ++oy) {
        const float gy = gap_to_cell(xi.y, qy + oy, cs[1]);
        const float g2 = gy * gy + gz * gz;
        if (g2 >= lrm2) continue;
        const float ext = sqrtf(lrm2 - g2);
        const int xlo = max(qx - R, (int)floorf((xi.x - ext) / cs[0]));
        const int xhi = min(qx + R, (int)floorf((xi.x + ext) / cs[0]));
        if (xlo > xhi) continue;
        const int cy = (qy + oy + P.dims[1]) % P.dims[1];
        const uint32_t rowbase = P.cell_off + (uint32_t)(P.dims[0] * (cy + P.dims[1] * cz));
        const AxisRange xr = span_ranges(xlo, xhi, P.dims[0]);
        for (int sgi = 0; sgi < xr.n; ++sgi) take(start[rowbase + xr.lo[sgi]], start[rowbase + xr.hi[sgi] + 1]);
      }
    }
    if (cnt > cap) { flags[0] = 1u; cnt = cap; }
    nl_cnt[k] = cnt;
    return;
  }
  for (int iz = 0; iz < nz; ++iz) {
    for (int iy = 0; iy < ny; ++iy) {
      uint32_t rowbase = P.cell_off + (uint32_t)(P.dims[0] * (ys[iy] + P.dims[1] * zs[iz]));
      for (int s = 0; s < ax.n; ++s) {
        uint32_t a = start[rowbase + ax.lo[s]], e = start[rowbase + ax.hi[s] + 1];
        for (uint32_t j = a; j < e; ++j) {
          if (j == k) continue;
          const float4 xj = pos[j];
          const float dx = fast_mi(xi.x - xj.x, box[0], inv[0]);
          const float dy = fast_mi(xi.y - xj.y, box[1], inv[1]);
          const float dz = fast_mi(xi.z - xj.z, box[2], inv[2]);
          const float r2 = dx * dx + dy * dy + dz * dz;
          if (r2 > lr2_hi) continue;
          if (r2 >= lr2_lo && !(ex_dist(xi, xj, box) < lr)) continue;
          if (cnt < cap) row[cnt] = j | sh.tag(r2);
          ++cnt;
        }
      }
    }
  }
  if (cnt > cap) { flags[0] = 1u; cnt = cap; }
  nl_cnt[k] = cnt;
}

// The same list build with the neighbour cells staged, for replicas whose walk does not wrap onto
// itself (every grid side at least 2 walk + 1 cells).  A group of 8 lanes takes one cell; its lanes
// hold up to 8 of the cell's particles at a time.  The group walks the cell's neighbour rows in
// k_build_list's order (z, then y, then the x cells of the row as at most two wrapped segments) and
// stages each segment 8 particles at a time in shared memory, shifted by the periodic image of the
// segment, so that the separation is a plain difference; every lane then tests the 8 staged beads
// against its particle.  A particle's accepted neighbours therefore come in k_build_list's order and
// pass its test (the fast squared distance away from the range, the exact reference arithmetic on
// the unshifted positions within 1e-5 of it), and the rows are the same lists.  Four groups in a warp
// take four consecutive cells of one x row, whose neighbour rows coincide.
constexpr int kGroup = 8;
constexpr int kGBlock = 128;
__global__ void __launch_bounds__(kGBlock) k_build_list_cells(
    const float4* __restrict__ pos, const SysParams* __restrict__ sp, const uint8_t* __restrict__ cell_sys,
    const uint32_t* __restrict__ start, uint32_t ncells, uint32_t cap, float rmax2, uint32_t* __restrict__ nl,
    uint32_t* __restrict__ nl_cnt, uint32_t* __restrict__ flags) {
  __shared__ float4 stage[kGBlock];
  // every loop below runs the same trip count on the whole warp (the maximum over its four groups,
  // with the shorter groups predicated off): groups that branched apart would run one after another
  const uint32_t cg = (blockIdx.x * blockDim.x + threadIdx.x) / kGroup;
  const bool have = cg < ncells;
  const uint32_t c = have ? cg : 0u;
  const uint32_t l8 = threadIdx.x & (kGroup - 1);
  float4* st = stage + (threadIdx.x & ~(kGroup - 1));
  const SysParams& P = sp[cell_sys[c]];
  const float bx = P.box[0], by = P.box[1], bz = P.box[2];
  const float lr = P.list_range;
  const float lr2_lo = lr * lr * (1.0f - 1e-5f), lr2_hi = lr * lr * (1.0f + 1e-5f);
  const Shells sh = Shells::of(rmax2, lr);
  const uint32_t cl = c - P.cell_off;
  const int dx = P.dims[0], dy = P.dims[1], dz = P.dims[2];
  const int qx = (int)(cl % (uint32_t)dx), qy = (int)((cl / (uint32_t)dx) % (uint32_t)dy),
            qz = (int)(cl / ((uint32_t)dx * (uint32_t)dy));
  const int R = P.walk;
  // the row's x cells as at most two wrapped segments, in axis_ranges' order (qx - R .. qx + R does
  // not wrap onto itself here), and the image shift of each: cells wrapped round a face sit one box
  // beyond it
  const bool wrap_lo = qx - R < 0, wrap_hi = qx + R >= dx;
  const int nseg = (wrap_lo || wrap_hi) ? 2 : 1;
  const int s0lo = wrap_lo ? qx - R + dx : qx - R, s0hi = (wrap_lo || wrap_hi) ? dx - 1 : qx + R;
  const int s1hi = wrap_lo ? qx + R : qx + R - dx;
  const float xs0 = wrap_lo ? -bx : 0.f;
  const float xs1 = wrap_hi ? bx : 0.f;
  const uint32_t a_i = have ? start[c] : 0u, e_i = have ? start[c + 1] : 0u;
  const uint32_t nib = __reduce_max_sync(0xffffffffu, (e_i - a_i + kGroup - 1) / kGroup);
  for (uint32_t ib = 0; ib < nib; ++ib) {
    const uint32_t k = a_i + ib * kGroup + l8;
    const bool mine = k < e_i;
    const float4 xi = mine ? pos[k] : make_float4(0.f, 0.f, 0.f, 0.f);
    uint32_t cnt = 0;
    uint32_t* row = nl + (size_t)(mine ? k : 0u) * cap;
    // R is the replica's walk; a warp spans one x row of one replica, so every bound is warp-uniform
    for (int oz = -R; oz <= R; ++oz) {
      const int z = qz + oz;
      const int cz = (z + dz) % dz;
      const float sz = z < 0 ? -bz : (z >= dz ? bz : 0.f);
      for (int oy = -R; oy <= R; ++oy) {
        const int y = qy + oy;
        const int cy = (y + dy) % dy;
        const float sy = y < 0 ? -by : (y >= dy ? by : 0.f);
        const uint32_t rowbase = P.cell_off + (uint32_t)(dx * (cy + dy * cz));
#pragma unroll
        for (int sgi = 0; sgi < 2; ++sgi) {
          uint32_t a = 0, len = 0;
          if (have && sgi < nseg) {
            a = start[rowbase + (sgi == 0 ? s0lo : 0)];
            len = start[rowbase + (sgi == 0 ? s0hi : s1hi) + 1] - a;
          }
          const float xs = sgi == 0 ? xs0 : xs1;
          const uint32_t mlen = __reduce_max_sync(0xffffffffu, len);
          for (uint32_t t0 = 0; t0 < mlen; t0 += kGroup) {
            if (t0 + l8 < len) {
              const uint32_t j = a + t0 + l8;
              const float4 p = pos[j];
              st[l8] = make_float4(p.x + xs, p.y + sy, p.z + sz, __uint_as_float(j));
            }
            __syncwarp();
#pragma unroll
            for (uint32_t u = 0; u < (uint32_t)kGroup; ++u) {
              const float4 q = st[u];
              const uint32_t jj = __float_as_uint(q.w);
              const float ddx = xi.x - q.x, ddy = xi.y - q.y, ddz = xi.z - q.z;
              const float r2 = ddx * ddx + ddy * ddy + ddz * ddz;
              if (!mine || t0 + u >= len || jj == k || r2 > lr2_hi) continue;
              if (r2 >= lr2_lo) {
                const float4 pj = pos[jj];
                const float ex = ex_len(ex_mi(__fsub_rn(xi.x, pj.x), bx), ex_mi(__fsub_rn(xi.y, pj.y), by),
                                        ex_mi(__fsub_rn(xi.z, pj.z), bz));
                if (!(ex < lr)) continue;
              }
              if (cnt < cap) row[cnt] = jj | sh.tag(r2);
              ++cnt;
            }
            __syncwarp();
          }
        }
      }
    }
    if (mine) {
      if (cnt > cap) { flags[0] = 1u; cnt = cap; }
      nl_cnt[k] = cnt;
    }
  }
}

// Group every row by build-distance shell, strip the tags, and record where shells 0..3 end.  A warp
// per row.  A row of up to 32 * kGRegs entries is read in one go into registers, lane l holding
// entries l, l + 32, ..; each lane counts its entries per shell (five 12-bit fields of one 64-bit word:
// a row holds fewer than 4096 entries), one warp scan of those words gives every lane the place of its
// entries, and each shell receives its entries lane by lane (lane 0's first, each lane's in row order),
// a deterministic order.  A longer row (dense aggregates) is grouped in shared memory, shell by shell
// with ballots, keeping the build's order inside a shell.
constexpr uint32_t kGRegs = 16;
__device__ __forceinline__ uint32_t field12(unsigned long long w, uint32_t t) {
  return (uint32_t)(w >> (12u * t)) & 0xFFFu;
}
__global__ void k_group_rows(uint32_t N, uint32_t cap, uint32_t* __restrict__ nl, const uint32_t* __restrict__ nl_cnt,
                             uint4* __restrict__ shell_end) {
  extern __shared__ uint32_t gbuf[];
  const uint32_t wib = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  const uint32_t k = blockIdx.x * (blockDim.x >> 5) + wib;
  if (k >= N) return;   // whole warps
  uint32_t* row = nl + (size_t)k * cap;
  const uint32_t cnt = min(nl_cnt[k], cap);
  uint32_t e[4];
  if (cnt <= 32u * kGRegs) {
    uint32_t v[kGRegs];
    unsigned long long mine = 0;
#pragma unroll
    for (uint32_t c = 0; c < kGRegs; ++c) {
      const uint32_t s = 32u * c + lane;
      v[c] = s < cnt ? row[s] : 0xFFFFFFFFu;
    }
#pragma unroll
    for (uint32_t c = 0; c < kGRegs; ++c)
      if (v[c] != 0xFFFFFFFFu) mine += 1ull << (12u * (v[c] >> 29));
    unsigned long long incl = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= (uint32_t)o) incl += y;
    }
    const unsigned long long tot = __shfl_sync(0xffffffffu, incl, 31);
    // the shells' first places, packed like the counts
    unsigned long long bases = 0;
    uint32_t run = 0;
#pragma unroll
    for (uint32_t t = 0; t < 5; ++t) {
      bases |= (unsigned long long)run << (12u * t);
      run += field12(tot, t);
      if (t < 4) e[t] = run;
    }
    unsigned long long at = bases + (incl - mine);   // this lane's first place in every shell
    __syncwarp();                                     // every lane has read its entries
#pragma unroll
    for (uint32_t c = 0; c < kGRegs; ++c) {
      if (v[c] == 0xFFFFFFFFu) continue;
      const uint32_t t = v[c] >> 29;
      row[field12(at, t)] = v[c] & 0x1FFFFFFFu;
      at += 1ull << (12u * t);
    }
  } else {
    uint32_t* sb = gbuf + (size_t)wib * cap;
    for (uint32_t s = lane; s < cnt; s += 32u) sb[s] = row[s];
    __syncwarp();
    const uint32_t lt = (1u << lane) - 1u;
    uint32_t out = 0;
#pragma unroll
    for (uint32_t b = 0; b < 5; ++b) {
      for (uint32_t s0 = 0; s0 < cnt; s0 += 32u) {
        const uint32_t s = s0 + lane;
        const uint32_t v = s < cnt ? sb[s] : 0xFFFFFFFFu;
        const bool hit = (v >> 29) == b;
        const uint32_t m = __ballot_sync(0xffffffffu, hit);
        if (hit) row[out + __popc(m & lt)] = v & 0x1FFFFFFFu;
        out += __popc(m);
      }
      if (b < 4) e[b] = out;
    }
  }
  if (lane == 0) shell_end[k] = make_uint4(e[0], e[1], e[2], e[3]);
}

// heads: bin into the coarse head grid (replica-local cells), deterministic order inside a cell
__global__ void k_head_index(const uint32_t* __restrict__ heads, const uint32_t* __restrict__ head_sys, uint32_t H,
                             const uint32_t* __restrict__ slot_of, const float4* __restrict__ pos,
                             const SysParams* __restrict__ sp, uint32_t* __restrict__ hcell_of,
                             uint32_t* __restrict__ hcount, uint32_t* __restrict__ head_slot) {
  uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= H) return;
  const SysParams& P = sp[head_sys[h]];
  const uint32_t ks = slot_of[heads[h]];
  head_slot[h] = ks;
  float4 p = pos[ks];
  int cx = ex_cell_axis(p.x, P.box[0], P.hdims[0]);
  int cy = ex_cell_axis(p.y, P.box[1], P.hdims[1]);
  int cz = ex_cell_axis(p.z, P.box[2], P.hdims[2]);
  uint32_t c = P.hcell_off + (uint32_t)(cx + P.hdims[0] * (cy + P.hdims[1] * cz));
  hcell_of[h] = c;
  atomicAdd(&hcount[c], 1u);
}
__global__ void k_head_scatter(const uint32_t* __restrict__ hcell_of, const uint32_t* __restrict__ hstart, uint32_t H,
                               uint32_t* __restrict__ hcursor, uint32_t* __restrict__ hsorted) {
  uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= H) return;
  uint32_t c = hcell_of[h];
  hsorted[hstart[c] + atomicAdd(&hcursor[c], 1u)] = h;
}
__global__ void k_head_sort_cells(const uint32_t* __restrict__ hstart, uint32_t ncells, uint32_t* __restrict__ hsorted) {
  uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncells) return;
  uint32_t a = hstart[c], e = hstart[c + 1];
  for (uint32_t x = a + 1; x < e; ++x) {
    uint32_t v = hsorted[x];
    uint32_t y = x;
    while (y > a && hsorted[y - 1] > v) { hsorted[y] = hsorted[y - 1]; --y; }
    hsorted[y] = v;
  }
}

// the heads in head-cell order with their positions: the list build reads one 16-byte record per
// candidate instead of the index, the head's slot and its position one after another
__global__ void k_head_gather_sorted(const uint32_t* __restrict__ hsorted, uint32_t H,
                                     const uint32_t* __restrict__ head_slot, const float4* __restrict__ pos,
                                     float4* __restrict__ xg) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= H) return;
  const uint32_t g = hsorted[t];
  const float4 p = pos[head_slot[g]];
  xg[t] = make_float4(p.x, p.y, p.z, __uint_as_float(g));
}

// soup/wgsl/electrostatics-long.wgsl:31-56 head list at rc_es + skin, via the head grid, a warp per
// head: lanes test 32 candidates at a time, hits are compacted with a ballot.  Entries are the
// neighbours' HEAD indices (head_slot maps them to slots); membership uses the exact test near the
// range, so the set equals the reference's.
__global__ void __launch_bounds__(256) k_build_es_list(const uint32_t* __restrict__ head_sys, uint32_t H,
                                                       const uint32_t* __restrict__ head_slot, const float4* __restrict__ pos,
                                                       const SysParams* __restrict__ sp, const uint32_t* __restrict__ hcell_of,
                                                       const uint32_t* __restrict__ hstart, const float4* __restrict__ hxg,
                                                       uint32_t cap, uint32_t* __restrict__ es_nl, uint32_t* __restrict__ es_cnt,
                                                       uint32_t* __restrict__ flags) {
  const uint32_t h = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (h >= H) return;   // warp-uniform
  const SysParams& P = sp[head_sys[h]];
  const float4 xi = pos[head_slot[h]];
  const float box[3] = {P.box[0], P.box[1], P.box[2]};
  const float inv[3] = {P.inv_box[0], P.inv_box[1], P.inv_box[2]};
  const float lr = P.es_list_range;
  const float lo = lr * lr * (1.0f - 1e-5f), hi = lr * lr * (1.0f + 1e-5f);
  const uint32_t c = hcell_of[h] - P.hcell_off;
  const int q[3] = {(int)(c % (uint32_t)P.hdims[0]), (int)((c / (uint32_t)P.hdims[0]) % (uint32_t)P.hdims[1]),
                    (int)(c / ((uint32_t)P.hdims[0] * (uint32_t)P.hdims[1]))};
  const int R = P.hwalk;
  int ax[3][8], na[3] = {0, 0, 0};
  for (int a = 0; a < 3; ++a)
    for (int d = -R; d <= R; ++d) {
      int v = ((q[a] + d) % P.hdims[a] + P.hdims[a]) % P.hdims[a];
      bool dup = false;
      for (int t = 0; t < na[a]; ++t) dup |= ax[a][t] == v;
      if (!dup) ax[a][na[a]++] = v;
    }
  uint32_t cnt = 0;
  uint32_t* row = es_nl + (size_t)h * cap;
  const uint32_t lt = (1u << lane) - 1u;
  auto scan_cell = [&](uint32_t cc) {
    const uint32_t a0 = hstart[cc], e0 = hstart[cc + 1];
    for (uint32_t b0 = a0; b0 < e0; b0 += 32) {
      const uint32_t t = b0 + lane;
      bool hit = false;
      uint32_t g = 0;
      if (t < e0) {
        const float4 xj = hxg[t];
        g = __float_as_uint(xj.w);
        if (g != h) {
          const float dx = fast_mi(xi.x - xj.x, box[0], inv[0]);
          const float dy = fast_mi(xi.y - xj.y, box[1], inv[1]);
          const float dz = fast_mi(xi.z - xj.z, box[2], inv[2]);
          const float r2 = dx * dx + dy * dy + dz * dz;
          hit = r2 < lo || (r2 <= hi && ex_dist(xi, xj, box) < lr);
        }
      }
      const uint32_t m = __ballot_sync(0xffffffffu, hit);
      if (hit) {
        const uint32_t at = cnt + __popc(m & lt);
        if (at < cap) row[at] = g;
      }
      cnt += __popc(m);
    }
  };
  if (P.hdims[0] >= 2 * R + 1 && P.hdims[1] >= 2 * R + 1 && P.hdims[2] >= 2 * R + 1) {
    // the walk does not wrap onto itself: cells wholly beyond the list sphere (with a margin) are
    // skipped, which leaves the list the same set
    const float cs[3] = {box[0] / (float)P.hdims[0], box[1] / (float)P.hdims[1], box[2] / (float)P.hdims[2]};
    const float lrm = lr * (1.0f + 1e-5f) + 1e-3f, lrm2 = lrm * lrm;
    for (int oz = -R; oz <= R; ++oz) {
      const float gz = gap_to_cell(xi.z, q[2] + oz, cs[2]);
      for (int oy = -R; oy <= R; ++oy) {
        const float gy = gap_to_cell(xi.y, q[1] + oy, cs[1]);
        for (int ox = -R; ox <= R; ++ox) {
          const float gx = gap_to_cell(xi.x, q[0] + ox, cs[0]);
          if (gx * gx + gy * gy + gz * gz >= lrm2) continue;
          const int cx = (q[0] + ox + P.hdims[0]) % P.hdims[0], cy = (q[1] + oy + P.hdims[1]) % P.hdims[1],
                    cz = (q[2] + oz + P.hdims[2]) % P.hdims[2];
          scan_cell(P.hcell_off + (uint32_t)(cx + P.hdims[0] * (cy + P.hdims[1] * cz)));
        }
      }
    }
  } else {
    for (int iz = 0; iz < na[2]; ++iz)
      for (int iy = 0; iy < na[1]; ++iy)
        for (int ix = 0; ix < na[0]; ++ix)
          scan_cell(P.hcell_off + (uint32_t)(ax[0][ix] + P.hdims[0] * (ax[1][iy] + P.hdims[1] * ax[2][iz])));
  }
  if (lane == 0) {
    if (cnt > cap) { flags[1] = 1u; cnt = cap; }
    es_cnt[h] = cnt;
  }
}

}  // namespace

void launch_cell_index(Batch& b) {
  b.launches += 1;
  prof_begin(b, SOUP_K_SORT);
  cudaMemsetAsync(b.cell_count, 0, sizeof(uint32_t) * (b.ncells + 1), b.stream);
  k_cell_index<<<nblocks(b.N), kBlock, 0, b.stream>>>(b.pos, b.sysid, b.sp, b.N, b.cell_of_slot, b.cell_count);
  prof_end(b);
}

void launch_sort_and_gather(Batch& b) {
  prof_begin(b, SOUP_K_SORT);
  const uint64_t scans = exclusive_scan(b.cell_count, b.cell_start, b.ncells, b.scan_tmp, b.stream);
  cudaMemsetAsync(b.cell_cursor, 0, sizeof(uint32_t) * b.ncells, b.stream);
  k_scatter<<<nblocks(b.N), kBlock, 0, b.stream>>>(b.cell_of_slot, b.cell_start, b.N, b.cell_cursor, b.perm);
  k_sort_cells<<<nblocks(b.ncells), kBlock, 0, b.stream>>>(b.cell_start, b.ncells, b.id, b.perm);
  k_gather<<<nblocks(b.N), kBlock, 0, b.stream>>>(b.N, b.perm, b.pos, b.vel, b.force, b.charge, b.slots, b.center,
                                                   b.held, b.brng, b.trng, b.frozen, b.id, b.pos2, b.vel2, b.force2,
                                                   b.charge2, b.slots2, b.center2, b.held2, b.brng2, b.trng2,
                                                   b.frozen2, b.id2, b.slot_of, b.pos_ref);
  k_copy_back<<<nblocks(b.N), kBlock, 0, b.stream>>>(b.N, b.pos2, b.vel2, b.force2, b.charge2, b.slots2, b.center2,
                                                      b.held2, b.brng2, b.trng2, b.frozen2, b.id2, b.pos, b.vel, b.force,
                                                      b.charge, b.slots, b.center, b.held, b.brng, b.trng, b.frozen,
                                                      b.id);
  // the cell of every new slot: cell_start is monotone, so recompute from the sorted positions
  cudaMemsetAsync(b.cell_count, 0, sizeof(uint32_t) * (b.ncells + 1), b.stream);
  k_cell_index<<<nblocks(b.N), kBlock, 0, b.stream>>>(b.pos, b.sysid, b.sp, b.N, b.cell_of_slot, b.cell_count);
  b.launches += 6 + scans;
  prof_end(b);
}

void launch_build_lists(Batch& b) {
  b.launches += 1;
  prof_begin(b, SOUP_K_LIST);
  if (b.list_by_cell && b.list_cells)
    k_build_list_cells<<<nblocks((uint64_t)b.ncells * kGroup, kGBlock), kGBlock, 0, b.stream>>>(
        b.pos, b.sp, b.cell_sys, b.cell_start, b.ncells, b.list_cap, b.hs.rmax2, b.nl, b.nl_cnt, b.flags);
  else
    k_build_list<<<nblocks(b.N, 128), 128, 0, b.stream>>>(b.pos, b.sysid, b.sp, b.cell_of_slot, b.cell_start, b.N,
                                                          b.list_cap, b.hs.rmax2, b.nl, b.nl_cnt, b.flags);
  // rows grouped by shell: four warps per block while four staged rows fit the shared memory
  const uint32_t wpb = 16u * b.list_cap <= 200u * 1024u ? 4u : 1u;
  const size_t smem = (size_t)wpb * b.list_cap * 4u;
  if (smem > 48u * 1024u && b.group_smem_set < smem) {
    SOUP_CUDA_TRY(cudaFuncSetAttribute(k_group_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    b.group_smem_set = smem;
  }
  k_group_rows<<<(unsigned)((b.N + wpb - 1) / wpb), 32u * wpb, smem, b.stream>>>(b.N, b.list_cap, b.nl, b.nl_cnt,
                                                                                b.nl_shell);
  b.launches += 1;
  prof_end(b);
}

void launch_build_es_lists(Batch& b) {
  if (b.H == 0) return;
  prof_begin(b, SOUP_K_LIST);
  cudaMemsetAsync(b.hcell_count, 0, sizeof(uint32_t) * (b.nhcells + 1), b.stream);
  k_head_index<<<nblocks(b.H), kBlock, 0, b.stream>>>(b.heads, b.head_sys, b.H, b.slot_of, b.pos, b.sp, b.hcell_of,
                                                       b.hcell_count, b.head_slot);
  const uint64_t scans = exclusive_scan(b.hcell_count, b.hcell_start, b.nhcells, b.scan_tmp, b.stream);
  cudaMemsetAsync(b.hcell_cursor, 0, sizeof(uint32_t) * b.nhcells, b.stream);
  k_head_scatter<<<nblocks(b.H), kBlock, 0, b.stream>>>(b.hcell_of, b.hcell_start, b.H, b.hcell_cursor, b.hsorted);
  k_head_sort_cells<<<nblocks(b.nhcells), kBlock, 0, b.stream>>>(b.hcell_start, b.nhcells, b.hsorted);
  k_head_gather_sorted<<<nblocks(b.H), kBlock, 0, b.stream>>>(b.hsorted, b.H, b.head_slot, b.pos, b.hsorted_xg);
  k_build_es_list<<<nblocks((uint64_t)b.H * 32, 256), 256, 0, b.stream>>>(b.head_sys, b.H, b.head_slot, b.pos, b.sp,
                                                                         b.hcell_of, b.hcell_start, b.hsorted_xg,
                                                                         b.es_cap, b.es_nl, b.es_cnt, b.flags);
  b.launches += 6 + scans;
  prof_end(b);
}

}  // namespace soup

// kernels_noalloc.cu -- aggregate labels without any device allocation.
//
// soup_aggregate_labels (kernels_analysis.cu) allocates its scratch (cell bins, union-find parents,
// component minima) with cudaMalloc on every call and frees it with cudaFree.  Some callers cannot
// do that: a host process whose GPU memory is already reserved by another allocator (a framework's
// caching allocator that holds the whole device) can see cudaMalloc fail with out-of-memory even
// though the job has room, and cudaFree synchronises the whole device, stalling the MD stream that
// shares the GPU.  This file gives them soup_aggregate_labels_noalloc: the same labels, computed
// with the scratch in one file-scope device array of fixed size.
//
// The array is linked into the library, so every GPU that loads the library holds it (about
// 9.4 MB) until the process exits.  Every call shares it and it keeps the last call's contents:
// whatever must start at zero is cleared at the start of each call, and calls that overlap on the
// GPU (two streams, two threads) race on it -- callers serialise them.
#include <cmath>
#include <mutex>

#include "soup_internal.h"

namespace soup {
uint64_t exclusive_scan(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* tmp, cudaStream_t st);
}

namespace {

constexpr uint32_t kMaxMembers = SOUP_NOALLOC_MAX_MEMBERS;
constexpr uint32_t kMaxCells = SOUP_NOALLOC_MAX_CELLS;
constexpr uint32_t kScanTmp = 4 * (kMaxCells / 4096 + 64) + 256;
// layout (u32 words): mem, cell, sorted, parent, minidx, labels [kMaxMembers each];
// count, start, cursor [kMaxCells + 1 each]; scan scratch; component counter
constexpr size_t kOffMem = 0;
constexpr size_t kOffCell = kOffMem + kMaxMembers;
constexpr size_t kOffSorted = kOffCell + kMaxMembers;
constexpr size_t kOffParent = kOffSorted + kMaxMembers;
constexpr size_t kOffMin = kOffParent + kMaxMembers;
constexpr size_t kOffLabels = kOffMin + kMaxMembers;
constexpr size_t kOffCount = kOffLabels + kMaxMembers;
constexpr size_t kOffStart = kOffCount + (kMaxCells + 1);
constexpr size_t kOffCursor = kOffStart + (kMaxCells + 1);
constexpr size_t kOffTmp = kOffCursor + (kMaxCells + 1);
constexpr size_t kOffCnt = kOffTmp + kScanTmp;
constexpr size_t kWords = kOffCnt + 64;

static __device__ __align__(256) uint32_t g_noalloc_scratch[kWords];

constexpr uint32_t NONE = SOUP_NONE_U32;
constexpr int kBlock = 256;
inline unsigned nblocks(uint64_t n) { return (unsigned)((n + kBlock - 1) / kBlock); }

__device__ __forceinline__ double js_round(double x) {
  const double r = floor(x);
  return (__dsub_rn(x, r) >= 0.5) ? r + 1.0 : r;
}
__device__ __forceinline__ double wrap1(double v, double L) { return __dsub_rn(v, __dmul_rn(floor(__ddiv_rn(v, L)), L)); }
__device__ __forceinline__ double mi1(double d, double L) { return __dsub_rn(d, __dmul_rn(js_round(__ddiv_rn(d, L)), L)); }

struct AggGrid {
  int nx, ny, nz;
  double box[3], w[3];
};

__device__ __forceinline__ uint32_t nf_find(uint32_t* parent, uint32_t x) {
  volatile uint32_t* vp = parent;
  uint32_t p = vp[x];
  while (p != x) { x = p; p = vp[x]; }
  return x;
}
__device__ __forceinline__ void nf_union(uint32_t* parent, uint32_t a, uint32_t b) {
  for (;;) {
    a = nf_find(parent, a);
    b = nf_find(parent, b);
    if (a == b) return;
    if (a > b) { const uint32_t t = a; a = b; b = t; }
    if (atomicCAS(&parent[b], b, a) == b) return;
  }
}

// engine/src/aggregate.ts:65-130 buildClusterUnionFind (periodic z), bins and union over the
// static scratch; one thread per member
__global__ void k_nf_bin(const float4* __restrict__ pos, const uint32_t* __restrict__ slot_of, uint32_t off, uint32_t m,
                         AggGrid g, uint32_t* __restrict__ s) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  const float4 p = pos[slot_of[off + s[kOffMem + k]]];
  const int cx = min(g.nx - 1, (int)floor(__ddiv_rn(wrap1((double)p.x, g.box[0]), g.w[0])));
  const int cy = min(g.ny - 1, (int)floor(__ddiv_rn(wrap1((double)p.y, g.box[1]), g.w[1])));
  const int cz = min(g.nz - 1, (int)floor(__ddiv_rn(wrap1((double)p.z, g.box[2]), g.w[2])));
  const uint32_t c = (uint32_t)cx + (uint32_t)g.nx * ((uint32_t)cy + (uint32_t)g.ny * cz);
  s[kOffCell + k] = c;
  s[kOffParent + k] = k;
  s[kOffMin + k] = NONE;
  atomicAdd(&s[kOffCount + c], 1u);
}
__global__ void k_nf_scatter(uint32_t m, uint32_t* __restrict__ s) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  const uint32_t c = s[kOffCell + k];
  s[kOffSorted + s[kOffStart + c] + atomicAdd(&s[kOffCursor + c], 1u)] = k;
}
__global__ void k_nf_union(const float4* __restrict__ pos, const uint32_t* __restrict__ slot_of, uint32_t off, uint32_t m,
                           AggGrid g, double c2, uint32_t* __restrict__ s) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  const float4 pi = pos[slot_of[off + s[kOffMem + k]]];
  const uint32_t c = s[kOffCell + k];
  const int cz = (int)(c / ((uint32_t)g.nx * g.ny)), cy = (int)((c / g.nx) % g.ny), cx = (int)(c % g.nx);
  for (int dx = -1; dx <= 1; ++dx) {
    const int ax = ((cx + dx) % g.nx + g.nx) % g.nx;
    for (int dy = -1; dy <= 1; ++dy) {
      const int ay = ((cy + dy) % g.ny + g.ny) % g.ny;
      for (int dz = -1; dz <= 1; ++dz) {
        const int az = ((cz + dz) % g.nz + g.nz) % g.nz;
        const uint32_t nc = (uint32_t)ax + (uint32_t)g.nx * ((uint32_t)ay + (uint32_t)g.ny * az);
        for (uint32_t t = s[kOffStart + nc]; t < s[kOffStart + nc + 1]; ++t) {
          const uint32_t l = s[kOffSorted + t];
          if (l <= k) continue;
          const float4 pj = pos[slot_of[off + s[kOffMem + l]]];
          const double ddx = mi1(__dsub_rn((double)pi.x, (double)pj.x), g.box[0]);
          const double ddy = mi1(__dsub_rn((double)pi.y, (double)pj.y), g.box[1]);
          const double ddz = mi1(__dsub_rn((double)pi.z, (double)pj.z), g.box[2]);
          const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(ddx, ddx), __dmul_rn(ddy, ddy)), __dmul_rn(ddz, ddz));
          if (r2 <= c2) nf_union(s + kOffParent, k, l);
        }
      }
    }
  }
}
__global__ void k_nf_min(uint32_t m, uint32_t* __restrict__ s) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  const uint32_t r = nf_find(s + kOffParent, k);
  atomicMin(&s[kOffMin + r], s[kOffMem + k]);
  if (r == k) atomicAdd(&s[kOffCnt], 1u);
}
__global__ void k_nf_label(uint32_t m, uint32_t* __restrict__ s) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  s[kOffLabels + k] = s[kOffMin + nf_find(s + kOffParent, k)];
}

// device address of the scratch array, looked up once per device (host code must not use the
// symbol itself: on the host it names a stand-in, not device memory)
std::mutex g_mu;
uint32_t* g_ptr[64] = {};

uint32_t* scratch_for(int dev, std::string& err) {
  if (dev < 0 || dev >= 64) { err = "device ordinal out of range"; return nullptr; }
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      err = std::string("cudaGetSymbolAddress failed: ") + cudaGetErrorString(e);
      return nullptr;
    }
    g_ptr[dev] = static_cast<uint32_t*>(p);
  }
  return g_ptr[dev];
}

}  // namespace

extern "C" int soup_aggregate_labels_noalloc(SoupHandle* h, const uint32_t* member_idx, uint32_t n_members,
                                             double cutoff, uint32_t* labels, uint32_t* n_components) {
  if (!h || !h->b) return SOUP_E_ARG;
  soup::Batch& b = *h->b;
  const SoupConfig& c = b.cfg[h->r];
  auto bad = [&](int code, const std::string& m) { h->err = m; return code; };
  if ((n_members && (!member_idx || !labels)) || !(cutoff > 0)) return bad(SOUP_E_ARG, "aggregate labels: bad argument");
  if (n_members > kMaxMembers)
    return bad(SOUP_E_ARG, "aggregate labels (no-alloc): " + std::to_string(n_members) + " members exceed the maximum of " +
                               std::to_string(kMaxMembers));
  for (uint32_t k = 0; k < n_members; ++k)
    if (member_idx[k] >= c.n) return bad(SOUP_E_ARG, "aggregate labels: member index out of range");
  AggGrid g;
  for (int a = 0; a < 3; ++a) g.box[a] = c.box[a];
  g.nx = std::max(1, (int)std::floor(c.box[0] / cutoff));
  g.ny = std::max(1, (int)std::floor(c.box[1] / cutoff));
  g.nz = std::max(1, (int)std::floor(c.box[2] / cutoff));
  g.w[0] = c.box[0] / g.nx; g.w[1] = c.box[1] / g.ny; g.w[2] = c.box[2] / g.nz;
  const uint64_t nc = (uint64_t)g.nx * g.ny * g.nz;
  if (nc > kMaxCells)
    return bad(SOUP_E_ARG, "aggregate labels (no-alloc): the grid of " + std::to_string(nc) + " cells exceeds the maximum of " +
                               std::to_string(kMaxCells) + " (box / cutoff too large)");
  // the calling thread's current device is put back on every return below
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
  struct Restore {
    int d;
    ~Restore() { if (d >= 0) cudaSetDevice(d); }
  } restore{prev};
  if (cudaSetDevice(b.device) != cudaSuccess) return bad(SOUP_E_CUDA, "cudaSetDevice failed");
  std::string err;
  uint32_t* s = scratch_for(b.device, err);
  if (!s) return bad(SOUP_E_CUDA, err);
  if (n_members == 0) { if (n_components) *n_components = 0; h->err.clear(); return SOUP_OK; }
  const uint32_t m = n_members;
  const uint32_t off = b.hsp[h->r].slot_off;
  cudaStream_t st = b.stream;
  cudaError_t e = cudaSuccess;
  auto ok = [&](cudaError_t x) { if (e == cudaSuccess) e = x; };
  ok(cudaMemcpyAsync(s + kOffMem, member_idx, 4 * (size_t)m, cudaMemcpyHostToDevice, st));
  ok(cudaMemsetAsync(s + kOffCount, 0, 4 * ((size_t)nc + 1), st));
  ok(cudaMemsetAsync(s + kOffCursor, 0, 4 * ((size_t)nc + 1), st));
  ok(cudaMemsetAsync(s + kOffCnt, 0, 4, st));
  k_nf_bin<<<nblocks(m), kBlock, 0, st>>>(b.pos, b.slot_of, off, m, g, s);
  const uint64_t scans = soup::exclusive_scan(s + kOffCount, s + kOffStart, (uint32_t)nc, s + kOffTmp, st);
  k_nf_scatter<<<nblocks(m), kBlock, 0, st>>>(m, s);
  k_nf_union<<<nblocks(m), kBlock, 0, st>>>(b.pos, b.slot_of, off, m, g, cutoff * cutoff, s);
  k_nf_min<<<nblocks(m), kBlock, 0, st>>>(m, s);
  k_nf_label<<<nblocks(m), kBlock, 0, st>>>(m, s);
  b.launches += 5 + scans;
  ok(cudaGetLastError());
  uint32_t ncomp = 0;
  ok(cudaMemcpyAsync(labels, s + kOffLabels, 4 * (size_t)m, cudaMemcpyDeviceToHost, st));
  ok(cudaMemcpyAsync(&ncomp, s + kOffCnt, 4, cudaMemcpyDeviceToHost, st));
  ok(cudaStreamSynchronize(st));
  if (e != cudaSuccess) return bad(SOUP_E_CUDA, std::string("CUDA: ") + cudaGetErrorString(e));
  if (n_components) *n_components = ncomp;
  h->err.clear();
  return SOUP_OK;
}

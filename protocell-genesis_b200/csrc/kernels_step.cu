// kernels_step.cu -- the Langevin integrator, drift and health scans, and the cold-start relax step.
//
// Reference: soup/wgsl/step.wgsl:89-142 (kick_drift_wrap_main, kick_thermostat_main, pcgSoup),
// soup/wgsl/verlet.wgsl:113-122 (soup_max_drift_main: atomicMax over the bits of drift^2),
// soup/wgsl/health.wgsl:52-68 (exponent-bits non-finite scan), soup/wgsl/relax.wgsl:50-72.
//
// The drift max is fused into the kick+drift kernel: both read the same post-drift positions the
// reference's max-drift pass reads after the force.
#include "soup_internal.h"

namespace soup {

namespace {

constexpr int kBlock = 256;
inline unsigned nblocks(uint64_t n, int b = kBlock) { return (unsigned)((n + b - 1) / b); }

__device__ __forceinline__ uint32_t warp_max(uint32_t v) {
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// step.wgsl:96-108 (+ verlet.wgsl:113-122 fused).  Positions follow the reference's f32 operation
// order exactly (x + dt*v, then x - floor(x/box)*box).
__global__ void __launch_bounds__(kBlock) k_kick_drift(const SysParams* __restrict__ sp, const uint8_t* __restrict__ sysid,
                                                       uint32_t N, float4* __restrict__ pos, float4* __restrict__ vel,
                                                       const float4* __restrict__ force, const uint8_t* __restrict__ frozen,
                                                       const float4* __restrict__ pos_ref, uint32_t* __restrict__ drift_bits) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t dbits = 0;
  uint32_t r = 0;
  if (k < N) {
    r = sysid[k];
    const SysParams& P = sp[r];
    float4 x = pos[k];
    if (frozen[k]) {
      vel[k] = make_float4(0.f, 0.f, 0.f, 0.f);
    } else {
      const float4 f = force[k];
      float4 v = vel[k];
      v.x = __fadd_rn(v.x, __fmul_rn(P.hdt, f.x));
      v.y = __fadd_rn(v.y, __fmul_rn(P.hdt, f.y));
      v.z = __fadd_rn(v.z, __fmul_rn(P.hdt, f.z));
      v.w = 0.f;
      vel[k] = v;
      float y;
      y = __fadd_rn(x.x, __fmul_rn(P.dt, v.x)); x.x = __fsub_rn(y, __fmul_rn(floorf(__fdiv_rn(y, P.box[0])), P.box[0]));
      y = __fadd_rn(x.y, __fmul_rn(P.dt, v.y)); x.y = __fsub_rn(y, __fmul_rn(floorf(__fdiv_rn(y, P.box[1])), P.box[1]));
      y = __fadd_rn(x.z, __fmul_rn(P.dt, v.z)); x.z = __fsub_rn(y, __fmul_rn(floorf(__fdiv_rn(y, P.box[2])), P.box[2]));
      pos[k] = x;
    }
    const float4 p0 = pos_ref[k];
    const float dx = ex_mi(__fsub_rn(x.x, p0.x), P.box[0]);
    const float dy = ex_mi(__fsub_rn(x.y, p0.y), P.box[1]);
    const float dz = ex_mi(__fsub_rn(x.z, p0.z), P.box[2]);
    const float d2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
    dbits = __float_as_uint(d2);
  }
  // one atomic per warp when the whole warp is in one replica (the common case)
  const uint32_t r0 = __shfl_sync(0xffffffffu, r, 0);
  if (__all_sync(0xffffffffu, r == r0)) {
    uint32_t m = warp_max(dbits);
    if ((threadIdx.x & 31) == 0 && k < N + 31) atomicMax(&drift_bits[r0], m);
  } else if (k < N) {
    atomicMax(&drift_bits[r], dbits);
  }
}

// step.wgsl:110-142 kick_thermostat_main
__global__ void __launch_bounds__(kBlock) k_kick_thermo(const SysParams* __restrict__ sp, const uint8_t* __restrict__ sysid,
                                                        uint32_t N, float4* __restrict__ vel, const float4* __restrict__ force,
                                                        const uint8_t* __restrict__ frozen, uint32_t* __restrict__ trng) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  if (frozen[k]) { vel[k] = make_float4(0.f, 0.f, 0.f, 0.f); return; }
  const SysParams& P = sp[sysid[k]];
  const float4 f = force[k];
  float4 v = vel[k];
  float w[3] = {__fadd_rn(v.x, __fmul_rn(P.hdt, f.x)), __fadd_rn(v.y, __fmul_rn(P.hdt, f.y)),
                __fadd_rn(v.z, __fmul_rn(P.hdt, f.z))};
  uint32_t s = trng[k];
  float noise[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    s = pcg_hash(s);
    const float u1 = fmaxf(u01(s), 1e-7f);
    s = pcg_hash(s);
    const float u2 = u01(s);
    noise[a] = __fmul_rn(sqrtf(__fmul_rn(-2.0f, logf(u1))), cosf(__fmul_rn(6.28318531f, u2)));
  }
  trng[k] = s;
  v.x = __fadd_rn(__fsub_rn(w[0], __fmul_rn(P.gdt, w[0])), __fmul_rn(P.sigma_v, noise[0]));
  v.y = __fadd_rn(__fsub_rn(w[1], __fmul_rn(P.gdt, w[1])), __fmul_rn(P.sigma_v, noise[1]));
  v.z = __fadd_rn(__fsub_rn(w[2], __fmul_rn(P.gdt, w[2])), __fmul_rn(P.sigma_v, noise[2]));
  v.w = 0.f;
  vel[k] = v;
}

// kick_thermostat_main of one step and kick_drift_wrap_main of the next in one pass, for the steps of a
// chunk (the force they both read is the same array: nothing between them changes it).  The operations
// are k_kick_thermo's and then k_kick_drift's, in order, so the results are the same bits.
__global__ void __launch_bounds__(kBlock) k_thermo_drift(const SysParams* __restrict__ sp, const uint8_t* __restrict__ sysid,
                                                         uint32_t N, float4* __restrict__ pos, float4* __restrict__ vel,
                                                         const float4* __restrict__ force, const uint8_t* __restrict__ frozen,
                                                         uint32_t* __restrict__ trng, const float4* __restrict__ pos_ref,
                                                         uint32_t* __restrict__ drift_bits) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t dbits = 0;
  uint32_t r = 0;
  if (k < N) {
    r = sysid[k];
    const SysParams& P = sp[r];
    float4 x = pos[k];
    if (frozen[k]) {
      vel[k] = make_float4(0.f, 0.f, 0.f, 0.f);
    } else {
      const float4 f = force[k];
      float4 v = vel[k];
      // step.wgsl:110-142
      float w[3] = {__fadd_rn(v.x, __fmul_rn(P.hdt, f.x)), __fadd_rn(v.y, __fmul_rn(P.hdt, f.y)),
                    __fadd_rn(v.z, __fmul_rn(P.hdt, f.z))};
      uint32_t s = trng[k];
      float noise[3];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        s = pcg_hash(s);
        const float u1 = fmaxf(u01(s), 1e-7f);
        s = pcg_hash(s);
        const float u2 = u01(s);
        noise[a] = __fmul_rn(sqrtf(__fmul_rn(-2.0f, logf(u1))), cosf(__fmul_rn(6.28318531f, u2)));
      }
      trng[k] = s;
      v.x = __fadd_rn(__fsub_rn(w[0], __fmul_rn(P.gdt, w[0])), __fmul_rn(P.sigma_v, noise[0]));
      v.y = __fadd_rn(__fsub_rn(w[1], __fmul_rn(P.gdt, w[1])), __fmul_rn(P.sigma_v, noise[1]));
      v.z = __fadd_rn(__fsub_rn(w[2], __fmul_rn(P.gdt, w[2])), __fmul_rn(P.sigma_v, noise[2]));
      // step.wgsl:96-108 of the next step
      v.x = __fadd_rn(v.x, __fmul_rn(P.hdt, f.x));
      v.y = __fadd_rn(v.y, __fmul_rn(P.hdt, f.y));
      v.z = __fadd_rn(v.z, __fmul_rn(P.hdt, f.z));
      v.w = 0.f;
      vel[k] = v;
      float y;
      y = __fadd_rn(x.x, __fmul_rn(P.dt, v.x)); x.x = __fsub_rn(y, __fmul_rn(floorf(__fdiv_rn(y, P.box[0])), P.box[0]));
      y = __fadd_rn(x.y, __fmul_rn(P.dt, v.y)); x.y = __fsub_rn(y, __fmul_rn(floorf(__fdiv_rn(y, P.box[1])), P.box[1]));
      y = __fadd_rn(x.z, __fmul_rn(P.dt, v.z)); x.z = __fsub_rn(y, __fmul_rn(floorf(__fdiv_rn(y, P.box[2])), P.box[2]));
      pos[k] = x;
    }
    const float4 p0 = pos_ref[k];
    const float dx = ex_mi(__fsub_rn(x.x, p0.x), P.box[0]);
    const float dy = ex_mi(__fsub_rn(x.y, p0.y), P.box[1]);
    const float dz = ex_mi(__fsub_rn(x.z, p0.z), P.box[2]);
    dbits = __float_as_uint(__fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz)));
  }
  const uint32_t r0 = __shfl_sync(0xffffffffu, r, 0);
  if (__all_sync(0xffffffffu, r == r0)) {
    uint32_t m = warp_max(dbits);
    if ((threadIdx.x & 31) == 0 && k < N + 31) atomicMax(&drift_bits[r0], m);
  } else if (k < N) {
    atomicMax(&drift_bits[r], dbits);
  }
}

// verlet.wgsl:113-122 as a standalone pass (used by the single-phase entry point)
__global__ void k_max_drift(const SysParams* __restrict__ sp, const uint8_t* __restrict__ sysid, uint32_t N,
                            const float4* __restrict__ pos, const float4* __restrict__ pos_ref,
                            uint32_t* __restrict__ drift_bits) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  const SysParams& P = sp[sysid[k]];
  const float4 x = pos[k], p0 = pos_ref[k];
  const float dx = ex_mi(__fsub_rn(x.x, p0.x), P.box[0]);
  const float dy = ex_mi(__fsub_rn(x.y, p0.y), P.box[1]);
  const float dz = ex_mi(__fsub_rn(x.z, p0.z), P.box[2]);
  atomicMax(&drift_bits[sysid[k]], __float_as_uint(__fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz))));
}

// health.wgsl:52-68: components whose exponent bits are all ones (Inf or NaN), per replica
__device__ __forceinline__ uint32_t nonfinite3(const float4& v) {
  return (((__float_as_uint(v.x) >> 23) & 0xFFu) == 0xFFu) + (((__float_as_uint(v.y) >> 23) & 0xFFu) == 0xFFu) +
         (((__float_as_uint(v.z) >> 23) & 0xFFu) == 0xFFu);
}
__global__ void k_nonfinite(const uint8_t* __restrict__ sysid, uint32_t N, const float4* __restrict__ pos,
                            const float4* __restrict__ vel, uint32_t* __restrict__ out /* [R][2] */) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  const uint32_t bp = nonfinite3(pos[k]), bv = nonfinite3(vel[k]);
  if (bp) atomicAdd(&out[2 * sysid[k]], bp);
  if (bv) atomicAdd(&out[2 * sysid[k] + 1], bv);
}

// relax.wgsl:50-72 soup_relax_step_main
__global__ void k_relax_step(const SysParams* __restrict__ sp, const uint8_t* __restrict__ sysid, uint32_t N,
                             float4* __restrict__ pos, const float4* __restrict__ force,
                             const uint8_t* __restrict__ frozen, float d) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N || frozen[k]) return;
  const SysParams& P = sp[sysid[k]];
  const float4 f = force[k];
  const float a = fmaxf(fmaxf(fabsf(f.x), fabsf(f.y)), fabsf(f.z));
  if (!(a > 0.f) || ((__float_as_uint(a) >> 23) & 0xFFu) == 0xFFu) return;
  const float g0 = __fdiv_rn(f.x, a), g1 = __fdiv_rn(f.y, a), g2 = __fdiv_rn(f.z, a);
  const float L = ex_len(g0, g1, g2);
  float4 x = pos[k];
  float y;
  y = __fadd_rn(x.x, __fmul_rn(__fdiv_rn(g0, L), d)); x.x = __fsub_rn(y, __fmul_rn(floorf(__fdiv_rn(y, P.box[0])), P.box[0]));
  y = __fadd_rn(x.y, __fmul_rn(__fdiv_rn(g1, L), d)); x.y = __fsub_rn(y, __fmul_rn(floorf(__fdiv_rn(y, P.box[1])), P.box[1]));
  y = __fadd_rn(x.z, __fmul_rn(__fdiv_rn(g2, L), d)); x.z = __fsub_rn(y, __fmul_rn(floorf(__fdiv_rn(y, P.box[2])), P.box[2]));
  pos[k] = x;
}

// the drift-triggered rebuild decision of a captured step: any replica whose largest drift since its
// last rebuild exceeds skin/2 (or is not a number) sets the graph's conditional node
__global__ void k_rebuild_decide(const SysParams* __restrict__ sp, const uint32_t* __restrict__ drift_bits, uint32_t R,
                                 cudaGraphConditionalHandle h, uint32_t* __restrict__ count) {
  bool any = false;
  for (uint32_t r = threadIdx.x; r < R; r += 32) any |= !(__uint_as_float(drift_bits[r]) <= sp[r].skin_half2);
  any = __any_sync(0xffffffffu, any);
  if (threadIdx.x == 0) {
    cudaGraphSetConditional(h, any ? 1u : 0u);
    if (any) *count += 1u;
  }
}

}  // namespace

void launch_rebuild_decide(Batch& b, cudaGraphConditionalHandle h) {
  b.launches += 1;
  k_rebuild_decide<<<1, 32, 0, b.stream>>>(b.sp, b.drift_bits, b.R, h, b.rebuild_count);
}

void launch_kick_drift(Batch& b) {
  b.launches += 1;
  prof_begin(b, SOUP_K_KICK_DRIFT);
  k_kick_drift<<<nblocks(b.N), kBlock, 0, b.stream>>>(b.sp, b.sysid, b.N, b.pos, b.vel, b.force, b.frozen, b.pos_ref,
                                                       b.drift_bits);
  prof_end(b);
}
void launch_kick_thermo(Batch& b) {
  b.launches += 1;
  prof_begin(b, SOUP_K_KICK_THERMO);
  k_kick_thermo<<<nblocks(b.N), kBlock, 0, b.stream>>>(b.sp, b.sysid, b.N, b.vel, b.force, b.frozen, b.trng);
  prof_end(b);
}
void launch_thermo_drift(Batch& b) {
  b.launches += 1;
  prof_begin(b, SOUP_K_KICK_THERMO);
  k_thermo_drift<<<nblocks(b.N), kBlock, 0, b.stream>>>(b.sp, b.sysid, b.N, b.pos, b.vel, b.force, b.frozen, b.trng,
                                                         b.pos_ref, b.drift_bits);
  prof_end(b);
}
void launch_max_drift(Batch& b) {
  b.launches += 1;
  k_max_drift<<<nblocks(b.N), kBlock, 0, b.stream>>>(b.sp, b.sysid, b.N, b.pos, b.pos_ref, b.drift_bits);
}
void launch_nonfinite(Batch& b) {
  b.launches += 1;
  cudaMemsetAsync(b.flags + kFlagWords, 0, sizeof(uint32_t) * 2 * b.R, b.stream);
  k_nonfinite<<<nblocks(b.N), kBlock, 0, b.stream>>>(b.sysid, b.N, b.pos, b.vel, b.flags + kFlagWords);
}
void launch_relax_step(Batch& b, float d) {
  b.launches += 1;
  k_relax_step<<<nblocks(b.N), kBlock, 0, b.stream>>>(b.sp, b.sysid, b.N, b.pos, b.force, b.frozen, d);
}

}  // namespace soup

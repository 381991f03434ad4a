// soup_capi.cu -- the C ABI (include/soup_b200.h): lifecycle, uploads/readbacks, the step schedule.
//
// Reference: soup/src/sim.ts:95-600 (createSoup and the SoupSystem surface), soup/src/soup-integrate.ts
// :83-175 (per-step dispatch order and the chunked stepper with its guards and the constant-pH sweep),
// soup/src/soup-grid-verlet.ts:236-313 (rebuild sequence and assertVerletSafety), soup/src/soup-health.ts
// (assertStateFinite), soup/src/soup-readback.ts (readbacks), soup/src/soup-relax.ts:87-185.
#include <algorithm>
#include <numeric>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include <cstdlib>

#include "soup_internal.h"

using namespace soup;

namespace {

thread_local std::string g_last_error;

constexpr uint32_t NONE = SOUP_NONE_U32;
constexpr uint32_t FLAG_WORDS = kFlagWords;

template <class T> T* dalloc(size_t n) {
  T* p = nullptr;
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc(&p, n * sizeof(T));
  if (e != cudaSuccess) throw CudaError(e, "cudaMalloc", __FILE__, __LINE__);
  return p;
}
template <class T> void dfree(T*& p) { if (p) cudaFree(p); p = nullptr; }

struct SoupException {
  int code;
  std::string msg;
};
[[noreturn]] void fail(int code, const std::string& m) { throw SoupException{code, m}; }

float sigma_v_f32(float gamma, float kT, float dt) {
  volatile float t = 2.0f * gamma;   // step.wgsl:130: sqrt(2.0 * P.gamma * P.kT * P.dt), f32, in order
  t = t * kT;
  t = t * dt;
  return std::sqrt((float)t);
}

// ---- parameters ----------------------------------------------------------------------------
void check_config(const SoupConfig& c) {
  if (c.abi_version != SOUP_ABI_VERSION) fail(SOUP_E_ARG, "SoupConfig.abi_version does not match this library");
  if (c.n == 0) fail(SOUP_E_ARG, "createSoup: the starting composition is empty");
  if (c.n_kinds == 0 || c.n_kinds > SOUP_MAX_KINDS) fail(SOUP_E_ARG, "n_kinds must be 1..8");
  uint64_t sum = 0;
  for (uint32_t k = 0; k < c.n_kinds; ++k) sum += c.counts[k];
  if (sum != c.n) fail(SOUP_E_ARG, "SoupConfig.n must equal the sum of counts");
  for (int a = 0; a < 3; ++a)
    if (!(c.box[a] > 0)) fail(SOUP_E_GEOMETRY, "box sides must be positive");
  if (!(c.list_range > 0) || c.list_capacity == 0) fail(SOUP_E_ARG, "list_range and list_capacity must be positive");
  if (c.n_rules > SOUP_MAX_RULES) fail(SOUP_E_ARG, "at most 4 bond rules");
  if (c.bond_interval == 0) fail(SOUP_E_ARG, "bond_interval must be >= 1");
  if (!c.rebuild_on_drift && c.rebuild_every == 0) fail(SOUP_E_ARG, "rebuild_every must be >= 1");
  if (c.es_enabled && (c.charged_kind < 0 || c.charged_kind >= (int)c.n_kinds)) fail(SOUP_E_ARG, "charged_kind out of range");
  if (c.es_enabled && c.es_list_capacity == 0) fail(SOUP_E_ARG, "es_list_capacity must be positive");
  if (c.es_enabled && c.sweep_every == 0) fail(SOUP_E_ARG, "sweep_every must be >= 1");
}

Shared make_shared(const SoupConfig& c) {
  Shared s{};
  s.n_kinds = c.n_kinds;
  s.sigma = (float)c.sigma; s.eps = (float)c.epsilon; s.b_tt = (float)c.b_tt; s.k_fene = (float)c.k_fene;
  s.r_inf = (float)c.r_inf; s.k_bend = (float)c.k_bend; s.r_bend = (float)c.r_bend; s.wc = (float)c.wc;
  s.c6 = (float)std::pow(2.0, (double)0.16666667f);
  { volatile float t = s.c6 * s.b_tt; s.rc_attr = t; }
  s.attr_k = 3.14159265f / (2.0f * s.wc);
  s.attr_amp = s.eps * 3.14159265f / (2.0f * s.wc);
  float rmax = s.rc_attr + s.wc;
  for (uint32_t k = 0; k < SOUP_KMAX; ++k) {
    s.radius[k] = (float)c.radius[k];
    s.cls[k] = c.kind_class[k] & 3u;
  }
  for (uint32_t i = 0; i < SOUP_KMAX; ++i)
    for (uint32_t j = 0; j < SOUP_KMAX; ++j) {
      volatile float b = s.sigma * (s.radius[i] + s.radius[j]);
      b = b * 0.5f;
      volatile float w = s.c6 * b;
      PairConst& p = s.pair[i * SOUP_KMAX + j];
      p.wcut = w; p.wcut2 = w * w; p.b2 = b * b;
      p.attr = (float)c.attr_scale[s.cls[i]][s.cls[j]];
      PairW& q = s.pw[i * SOUP_KMAX + j];
      q.b2 = p.b2; q.wcut2 = p.wcut2; q.amp = p.attr * s.attr_amp;
      q.polar = (s.cls[i] == 1u && s.cls[j] == 1u) ? 1.f : 0.f;
      if (i < c.n_kinds && j < c.n_kinds) rmax = std::max(rmax, (float)w);
    }
  if (c.es_enabled) rmax = std::max(rmax, (float)c.es_split_radius);
  s.rmax2 = rmax * rmax * 1.0001f;
  for (uint32_t r = 0; r < SOUP_RMAX; ++r) {
    const bool on = r < c.n_rules;
    s.kindA[r] = on ? (float)c.rule_kind_a[r] : -1.f; s.kindB[r] = on ? (float)c.rule_kind_b[r] : -1.f;
    s.att_form[r] = on ? (float)c.attempt_form[r] : 0.f; s.att_break[r] = on ? (float)c.attempt_break[r] : 0.f;
    s.acc_form[r] = on ? (float)c.accept_form[r] : 0.f; s.acc_break[r] = on ? (float)c.accept_break[r] : 0.f;
    s.req_cat[r] = on ? (float)c.requires_catalyst[r] : 0.f;
    s.roleA[r] = on ? (float)c.role_a[r] : 0.f; s.roleB[r] = on ? (float)c.role_b[r] : 0.f;
  }
  s.cat_kind = (float)c.catalyst_kind; s.head_terminal = (float)c.head_terminal_only;
  s.head_cap = (float)c.head_chain_capacity; s.max_hold = (float)c.max_hold_steps; s.interval = (float)c.bond_interval;
  return s;
}

void grid_of(const double box[3], double range, int walk, int dims[3]) {
  const double cell = range / walk;
  for (int a = 0; a < 3; ++a) dims[a] = std::max(1, (int)std::floor(box[a] / cell));
}

SysParams make_sys(const SoupConfig& c) {
  SysParams p{};
  for (int a = 0; a < 3; ++a) { p.box[a] = (float)c.box[a]; p.inv_box[a] = 1.0f / p.box[a]; p.d_box[a] = c.box[a]; p.d_inv_box[a] = 1.0 / c.box[a]; }
  p.list_range = (float)c.list_range;
  const bool es = c.es_enabled != 0;
  p.es_on = es ? 1u : 0u;
  p.es_A = es ? (float)c.es_coeff_a : 0.f;
  p.es_kappa = (float)c.es_kappa; p.es_rc = (float)c.es_cutoff; p.es_fc = (float)c.es_shift_f;
  p.es_split = (float)c.es_split_radius; p.es_list_range = (float)c.es_list_range;
  p.wall_r = (float)c.wall_radius; p.wall_k = (float)c.wall_k;
  p.kT = (float)c.kT; p.gamma = (float)c.gamma; p.dt = (float)c.dt;
  { volatile float t = 0.5f * p.dt; p.hdt = t; volatile float g = p.gamma * p.dt; p.gdt = g; }
  p.sigma_v = sigma_v_f32(p.gamma, p.kT, p.dt);
  p.acid = (float)c.acid_soap_scale;
  p.skin_half2 = (float)(0.25 * c.skin * c.skin);
  p.walk = 2;
  grid_of(c.box, c.list_range, p.walk, p.dims);
  p.hwalk = 2;
  grid_of(c.box, es ? c.es_list_range : c.list_range, p.hwalk, p.hdims);
  p.list_cap = c.list_capacity;
  p.es_cap = c.es_list_capacity;
  p.charged_kind = c.charged_kind;
  p.d_A = es ? c.es_coeff_a : 0.0; p.d_kappa = c.es_kappa; p.d_rc = c.es_cutoff; p.d_shiftU = c.es_shift_u;
  p.d_shiftF = c.es_shift_f; p.d_pka = c.pka_intrinsic; p.d_ph = c.ph; p.d_kT = c.kT; p.d_q = c.charge_deprotonated;
  p.d_acid = c.acid_soap_scale; p.d_rcattr = c.rc_attr; p.d_wc = c.wc; p.d_eps = c.epsilon;
  return p;
}

uint64_t cells_of(const int d[3]) { return (uint64_t)d[0] * d[1] * d[2]; }

}  // namespace

namespace soup {
void prof_begin(Batch& b, int k) {
  if (!b.prof) return;
  Batch::Mark m{};
  for (cudaEvent_t* e : {&m.a, &m.b}) {
    if (!b.event_pool.empty()) { *e = b.event_pool.back(); b.event_pool.pop_back(); }
    else SOUP_CUDA_TRY(cudaEventCreate(e));
  }
  m.k = k;
  SOUP_CUDA_TRY(cudaEventRecord(m.a, b.stream));
  b.marks.push_back(m);
}
void prof_end(Batch& b) {
  if (!b.prof || b.marks.empty()) return;
  SOUP_CUDA_TRY(cudaEventRecord(b.marks.back().b, b.stream));
}
void prof_flush(Batch& b) {
  if (b.marks.empty()) return;
  SOUP_CUDA_TRY(cudaStreamSynchronize(b.stream));
  for (const Batch::Mark& m : b.marks) {
    float ms = 0.f;
    SOUP_CUDA_TRY(cudaEventElapsedTime(&ms, m.a, m.b));
    b.kt_ms[m.k] += ms;
    b.kt_n[m.k] += 1;
    b.event_pool.push_back(m.a);
    b.event_pool.push_back(m.b);
  }
  b.marks.clear();
}
}  // namespace soup

namespace {

// ---- batch construction ----------------------------------------------------------------------
void alloc_grids(Batch& b) {
  dfree(b.cell_count); dfree(b.cell_start); dfree(b.cell_cursor); dfree(b.scan_tmp); dfree(b.cell_sys);
  dfree(b.hcell_count); dfree(b.hcell_start); dfree(b.hcell_cursor);
  uint64_t nc = 0, nh = 0;
  for (uint32_t r = 0; r < b.R; ++r) {
    b.hsp[r].cell_off = (uint32_t)nc;
    nc += cells_of(b.hsp[r].dims);
    b.hsp[r].hcell_off = (uint32_t)nh;
    nh += cells_of(b.hsp[r].hdims);
  }
  if (nc > 0x7fffffffull || nh > 0x7fffffffull) fail(SOUP_E_GEOMETRY, "neighbour grid too large");
  b.ncells = (uint32_t)nc;
  b.nhcells = (uint32_t)nh;
  b.cell_count = dalloc<uint32_t>(nc + 1);
  b.cell_start = dalloc<uint32_t>(nc + 1);
  b.cell_cursor = dalloc<uint32_t>(nc + 1);
  {
    std::vector<uint8_t> cs((size_t)nc);
    b.list_by_cell = true;
    for (uint32_t r = 0; r < b.R; ++r) {
      const SysParams& p = b.hsp[r];
      std::fill(cs.begin() + p.cell_off, cs.begin() + p.cell_off + cells_of(p.dims), (uint8_t)r);
      for (int a = 0; a < 3; ++a) b.list_by_cell = b.list_by_cell && p.dims[a] >= 2 * p.walk + 1;
    }
    b.cell_sys = dalloc<uint8_t>(nc);
    SOUP_CUDA_TRY(cudaMemcpy(b.cell_sys, cs.data(), nc, cudaMemcpyHostToDevice));
  }
  b.hcell_count = dalloc<uint32_t>(nh + 1);
  b.hcell_start = dalloc<uint32_t>(nh + 1);
  b.hcell_cursor = dalloc<uint32_t>(nh + 1);
  const uint64_t m = std::max(nc, nh);
  b.scan_tmp = dalloc<uint32_t>(4 * (m / 4096 + 64) + 256);
}

void upload_params(Batch& b) {
  SOUP_CUDA_TRY(cudaMemcpyAsync(b.sp, b.hsp.data(), sizeof(SysParams) * b.R, cudaMemcpyHostToDevice, b.stream));
  SOUP_CUDA_TRY(cudaMemcpyAsync(b.shared, &b.hs, sizeof(Shared), cudaMemcpyHostToDevice, b.stream));
}

void rebuild_launches(Batch& b) {
  launch_cell_index(b);
  launch_sort_and_gather(b);
  launch_build_lists(b);
  launch_build_es_lists(b);
  SOUP_CUDA_TRY(cudaMemsetAsync(b.drift_bits, 0, sizeof(uint32_t) * b.R, b.stream));
}
void rebuild(Batch& b) {
  rebuild_launches(b);
  b.rebuilds++;
}

void force_pass(Batch& b) {   // encodeVerletRebuild + encodeSoupForceList (the priming / recompute pass)
  rebuild(b);
  launch_force(b);
  b.force_fresh = true;
}

// Upload replica r's state from original-order host arrays (NULL members: fresh values).
void upload_replica(Batch& b, uint32_t r, const SoupInitState* init, bool fresh_allowed) {
  const SoupConfig& c = b.cfg[r];
  const uint32_t n = c.n, off = b.hsp[r].slot_off;
  std::vector<float> pos(4 * (size_t)n), vel(4 * (size_t)n), charge(n);
  std::vector<uint32_t> slots(3 * (size_t)n, NONE), center(n, NONE), held(n, 0), brng(n), trng(n), frozen32(n, 0);
  // the fresh lattice (a few tens of ms at 483k beads) only when the given state leaves one of its
  // arrays to it; its frozen flags are all zero in this build, as frozen32 already is
  const bool complete = init && init->positions && init->velocities && init->bond_rng && init->thermo_rng;
  if (fresh_allowed && !complete) host_fresh_state(c, pos.data(), vel.data(), frozen32.data(), brng.data(), trng.data());
  if (init) {
    if (init->positions) std::memcpy(pos.data(), init->positions, 16 * (size_t)n);
    if (init->velocities) std::memcpy(vel.data(), init->velocities, 16 * (size_t)n);
    if (init->bond_slots) std::memcpy(slots.data(), init->bond_slots, 12 * (size_t)n);
    if (init->center_link) std::memcpy(center.data(), init->center_link, 4 * (size_t)n);
    if (init->center_held) std::memcpy(held.data(), init->center_held, 4 * (size_t)n);
    if (init->bond_rng) std::memcpy(brng.data(), init->bond_rng, 4 * (size_t)n);
    if (init->thermo_rng) std::memcpy(trng.data(), init->thermo_rng, 4 * (size_t)n);
    if (init->frozen) std::memcpy(frozen32.data(), init->frozen, 4 * (size_t)n);
  }
  uint32_t prot = c.protonation_rng;
  if (init && init->charges) {
    std::memcpy(charge.data(), init->charges, 4 * (size_t)n);
  } else {
    uint32_t pr = 0;
    host_initial_charges(c, pos.data(), charge.data(), &pr);
    if (c.protonation_rng == 0) prot = pr;
  }
  b.prot_rng[r] = prot;
  for (uint32_t i = 0; i < n; ++i) {
    for (int a = 0; a < 3; ++a) {
      uint32_t& v = slots[3 * (size_t)i + a];
      if (v != NONE) { if (v >= n) fail(SOUP_E_ARG, "bond_slots names a particle outside the system"); v += off; }
    }
    if (center[i] != NONE) { if (center[i] >= n) fail(SOUP_E_ARG, "center_link names a particle outside the system"); center[i] += off; }
    const float kf = pos[4 * (size_t)i + 3];
    if (!(kf >= 0.f && kf < (float)c.n_kinds) || kf != std::floor(kf)) fail(SOUP_E_ARG, "positions[4i+3] must hold a kind index");
  }
  std::vector<uint8_t> frozen(n);
  std::vector<uint32_t> ids(n);
  for (uint32_t i = 0; i < n; ++i) { frozen[i] = frozen32[i] ? 1 : 0; ids[i] = off + i; }
  b.kinds[r].resize(n);
  b.off_head_charge[r] = 0;
  for (uint32_t i = 0; i < n; ++i) {
    b.kinds[r][i] = (uint8_t)pos[4 * (size_t)i + 3];
    if (charge[i] != 0.f && (int)b.kinds[r][i] != c.charged_kind) b.off_head_charge[r] = 1;
  }
  auto up = [&](void* dst, const void* src, size_t bytes) {
    SOUP_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, b.stream));
  };
  up(b.pos + off, pos.data(), 16 * (size_t)n);
  up(b.vel + off, vel.data(), 16 * (size_t)n);
  SOUP_CUDA_TRY(cudaMemsetAsync(b.force + off, 0, 16 * (size_t)n, b.stream));
  up(b.charge + off, charge.data(), 4 * (size_t)n);
  up(b.slots + 3 * (size_t)off, slots.data(), 12 * (size_t)n);
  up(b.center + off, center.data(), 4 * (size_t)n);
  up(b.held + off, held.data(), 4 * (size_t)n);
  up(b.brng + off, brng.data(), 4 * (size_t)n);
  up(b.trng + off, trng.data(), 4 * (size_t)n);
  up(b.frozen + off, frozen.data(), n);
  up(b.id + off, ids.data(), 4 * (size_t)n);
  up(b.slot_of + off, ids.data(), 4 * (size_t)n);
  if (init && init->events) up(b.events + 2 * SOUP_MAX_RULES * r, init->events, 8 * (size_t)c.n_rules);
  if (init && init->desorb_events) up(b.desorb + 2 * r, init->desorb_events, 8);
  up(b.prot_rng_dev + r, &b.prot_rng[r], 4);
  SOUP_CUDA_TRY(cudaStreamSynchronize(b.stream));   // host vectors go out of scope
}

Batch* make_batch(const SoupConfig* cfgs, const SoupInitState* inits, uint32_t R) {
  if (!cfgs || R == 0) fail(SOUP_E_ARG, "no configuration given");
  if (R > 255) fail(SOUP_E_ARG, "at most 255 replicas per batch");
  std::unique_ptr<Batch> bp(new Batch());
  Batch& b = *bp;
  b.R = R;
  b.cfg.assign(cfgs, cfgs + R);
  for (uint32_t r = 0; r < R; ++r) check_config(b.cfg[r]);
  b.kinds.resize(R);
  b.off_head_charge.assign(R, 1);
  b.polar_is_charged_kind = true;
  for (uint32_t r = 0; r < R; ++r)
    for (uint32_t k = 0; k < b.cfg[r].n_kinds; ++k)
      if ((b.cfg[r].kind_class[k] & 3u) == 1u && (int)k != b.cfg[r].charged_kind) b.polar_is_charged_kind = false;
  SOUP_CUDA_TRY(cudaGetDevice(&b.device));
  b.hs = make_shared(b.cfg[0]);
  for (uint32_t r = 1; r < R; ++r) {
    Shared o = make_shared(b.cfg[r]);
    o.rmax2 = b.hs.rmax2 = std::max(o.rmax2, b.hs.rmax2);
    if (std::memcmp(&o, &b.hs, sizeof(Shared)) != 0)
      fail(SOUP_E_ARG, "replicas of one batch must share the monomer table, force field and bond rules");
    if (b.cfg[r].global_step != b.cfg[0].global_step || b.cfg[r].bond_interval != b.cfg[0].bond_interval ||
        b.cfg[r].rebuild_on_drift != b.cfg[0].rebuild_on_drift || b.cfg[r].rebuild_every != b.cfg[0].rebuild_every ||
        (b.cfg[r].es_enabled && b.cfg[0].es_enabled && b.cfg[r].sweep_every != b.cfg[0].sweep_every) ||
        b.cfg[r].chunk_steps != b.cfg[0].chunk_steps)
      fail(SOUP_E_ARG, "replicas of one batch must share the step schedule");
  }
  uint64_t N = 0, H = 0;
  b.hsp.resize(R);
  b.list_cap = 0;
  b.es_cap = 0;
  std::vector<std::vector<uint32_t>> heads(R);
  for (uint32_t r = 0; r < R; ++r) {
    const SoupConfig& c = b.cfg[r];
    b.hsp[r] = make_sys(c);
    b.hsp[r].slot_off = (uint32_t)N;
    b.hsp[r].n = c.n;
    N += c.n;
    b.list_cap = std::max(b.list_cap, c.list_capacity);
    if (c.es_enabled) b.es_cap = std::max(b.es_cap, c.es_list_capacity);
  }
  if (N > 0xFFFFFFF0ull) fail(SOUP_E_ARG, "too many particles");
  b.N = (uint32_t)N;
  b.list_cap = (b.list_cap + 7u) & ~7u;
  b.prot_rng.assign(R, 0);
  for (uint32_t r = 0; r < R; ++r) {
    b.wall_r0.push_back(b.cfg[r].wall_radius);
    b.wall_box0.push_back(b.cfg[r].box[0]);
  }
  b.step.assign(R, 0);
  b.next_sweep.assign(R, UINT64_MAX);
  SOUP_CUDA_TRY(cudaStreamCreateWithFlags(&b.stream, cudaStreamNonBlocking));
  SOUP_CUDA_TRY(cudaStreamCreateWithFlags(&b.cap_stream, cudaStreamNonBlocking));
  // step chunks run as captured graphs; SOUP_NO_GRAPH=1 in the environment launches them one by one
  if (const char* e = std::getenv("SOUP_NO_GRAPH")) b.graphs_enabled = std::atoi(e) == 0;

  const size_t n = b.N;
  // a list entry carries its build-distance shell in its top three bits until the row is grouped
  if (n >= (1ull << 29)) fail(SOUP_E_ARG, "at most 2^29 - 1 particles per batch");
  b.pos = dalloc<float4>(n); b.vel = dalloc<float4>(n); b.force = dalloc<float4>(n); b.pos_ref = dalloc<float4>(n);
  b.charge = dalloc<float>(n); b.slots = dalloc<uint32_t>(3 * n); b.center = dalloc<uint32_t>(n);
  b.held = dalloc<uint32_t>(n); b.brng = dalloc<uint32_t>(n); b.trng = dalloc<uint32_t>(n); b.frozen = dalloc<uint8_t>(n);
  b.id = dalloc<uint32_t>(n); b.slot_of = dalloc<uint32_t>(n);
  b.pos2 = dalloc<float4>(n); b.vel2 = dalloc<float4>(n); b.force2 = dalloc<float4>(n); b.charge2 = dalloc<float>(n);
  b.slots2 = dalloc<uint32_t>(3 * n); b.center2 = dalloc<uint32_t>(n); b.held2 = dalloc<uint32_t>(n);
  b.brng2 = dalloc<uint32_t>(n); b.trng2 = dalloc<uint32_t>(n); b.frozen2 = dalloc<uint8_t>(n); b.id2 = dalloc<uint32_t>(n);
  b.cell_of_slot = dalloc<uint32_t>(n); b.perm = dalloc<uint32_t>(n);
  b.nl = dalloc<uint32_t>(n * (size_t)b.list_cap); b.nl_cnt = dalloc<uint32_t>(n); b.nl_shell = dalloc<uint4>(n);
  b.sysid = dalloc<uint8_t>(n);
  b.sp = dalloc<SysParams>(R); b.shared = dalloc<Shared>(1);
  b.flags = dalloc<uint32_t>(FLAG_WORDS + 2 * (size_t)R);
  b.events = dalloc<uint32_t>(2 * SOUP_MAX_RULES * (size_t)R);
  b.desorb = dalloc<uint32_t>(2 * (size_t)R);
  b.drift_bits = dalloc<uint32_t>(R);
  // [0] item count, [1] the walk's count, [2] the active beads (k_bond_select)
  b.bond_items = dalloc<uint32_t>(10 * n); b.bond_nitems = dalloc<uint32_t>(3); b.bond_sel = dalloc<uint32_t>(n);
  b.uf_parent = dalloc<uint32_t>(n); b.comp_min = dalloc<uint32_t>(n); b.item_done = dalloc<uint8_t>(n);
  b.has_item = dalloc<uint32_t>(n);
  b.prot_rng_dev = dalloc<uint32_t>(R);
  b.rebuild_count = dalloc<uint32_t>(1);
  SOUP_CUDA_TRY(cudaMemsetAsync(b.rebuild_count, 0, 4, b.stream));
  b.sweep_out = dalloc<double>(4 * (size_t)R);
  SOUP_CUDA_TRY(cudaMemsetAsync(b.flags, 0, sizeof(uint32_t) * (FLAG_WORDS + 2 * R), b.stream));
  SOUP_CUDA_TRY(cudaMemsetAsync(b.events, 0, sizeof(uint32_t) * 2 * SOUP_MAX_RULES * R, b.stream));
  SOUP_CUDA_TRY(cudaMemsetAsync(b.desorb, 0, sizeof(uint32_t) * 2 * R, b.stream));
  SOUP_CUDA_TRY(cudaMemsetAsync(b.drift_bits, 0, sizeof(uint32_t) * R, b.stream));
  {
    std::vector<uint8_t> sid(n);
    for (uint32_t r = 0; r < R; ++r)
      std::fill(sid.begin() + b.hsp[r].slot_off, sid.begin() + b.hsp[r].slot_off + b.cfg[r].n, (uint8_t)r);
    SOUP_CUDA_TRY(cudaMemcpyAsync(b.sysid, sid.data(), n, cudaMemcpyHostToDevice, b.stream));
    SOUP_CUDA_TRY(cudaStreamSynchronize(b.stream));
  }
  // state, per replica
  for (uint32_t r = 0; r < R; ++r) {
    upload_replica(b, r, inits ? &inits[r] : nullptr, true);
    b.step[r] = b.cfg[r].global_step;
    b.next_sweep[r] = b.cfg[r].es_enabled ? b.cfg[r].global_step + b.cfg[r].sweep_every : UINT64_MAX;
  }
  // heads: titratable beads in index order (static, electrostatics-long.wgsl:15-29)
  std::vector<uint32_t> hall, hsys;
  for (uint32_t r = 0; r < R; ++r) {
    const SoupConfig& c = b.cfg[r];
    b.hsp[r].head_off = (uint32_t)hall.size();
    if (c.es_enabled) {
      std::vector<float> pos(4 * (size_t)c.n);
      SOUP_CUDA_TRY(cudaMemcpy(pos.data(), b.pos + b.hsp[r].slot_off, 16 * (size_t)c.n, cudaMemcpyDeviceToHost));
      for (uint32_t i = 0; i < c.n; ++i)
        if (pos[4 * (size_t)i + 3] == (float)c.charged_kind) { hall.push_back(b.hsp[r].slot_off + i); hsys.push_back(r); }
    }
    b.hsp[r].nheads = (uint32_t)hall.size() - b.hsp[r].head_off;
    if (b.cfg[r].es_enabled && b.hsp[r].nheads > sweep_max_heads())
      fail(SOUP_E_ARG, "constant-pH sweep: " + std::to_string(b.hsp[r].nheads) + " heads in one replica exceed the " +
                           std::to_string(sweep_max_heads()) + " the device sweep holds");
  }
  b.H = (uint32_t)hall.size();
  b.heads = dalloc<uint32_t>(b.H); b.head_sys = dalloc<uint32_t>(b.H); b.head_slot = dalloc<uint32_t>(b.H);
  b.head_e = dalloc<long long>(b.H);
  b.head_pos = dalloc<float4>(b.H);
  b.head_xq = dalloc<float4>(b.H);
  b.head_flag = dalloc<uint8_t>(b.H);
  b.draw_site = dalloc<uint32_t>(std::max<size_t>(sweep_draw_sites(b), 1));
  b.sweep_band = dalloc<long long>(std::max<size_t>(sweep_band_rows(b) * 64, 1));
  sweep_prepare(b);
  b.es_nl = dalloc<uint32_t>((size_t)b.H * std::max<uint32_t>(b.es_cap, 1)); b.es_cnt = dalloc<uint32_t>(b.H);
  b.head_d = dalloc<long long>((size_t)b.H * std::max<uint32_t>(b.es_cap, 1));
  b.hcell_of = dalloc<uint32_t>(b.H); b.hsorted = dalloc<uint32_t>(b.H); b.hsorted_xg = dalloc<float4>(b.H);
  if (b.H) {
    SOUP_CUDA_TRY(cudaMemcpy(b.heads, hall.data(), 4 * (size_t)b.H, cudaMemcpyHostToDevice));
    SOUP_CUDA_TRY(cudaMemcpy(b.head_sys, hsys.data(), 4 * (size_t)b.H, cudaMemcpyHostToDevice));
  }
  alloc_grids(b);
  upload_params(b);
  // lanes per particle in the list force: 4 measured fastest at 483k beads (2: same, 8: +5%,
  // 16: +16%); SOUP_TPP in the environment overrides it for tuning (1, 2, 4, 8, 16 or 32)
  b.tpp = 4;
  if (const char* e = std::getenv("SOUP_TPP")) b.tpp = std::atoi(e);
  if (const char* e = std::getenv("SOUP_FORCE_QUEUED")) b.queued = std::atoi(e) != 0;
  if (const char* e = std::getenv("SOUP_LIST_BY_CELL")) b.list_cells = std::atoi(e) != 0;
  if (const char* e = std::getenv("SOUP_FULL_ROWS")) b.prune = std::atoi(e) == 0;
  force_pass(b);   // priming pass (soup/src/sim.ts:396-408)
  SOUP_CUDA_TRY(cudaStreamSynchronize(b.stream));
  SOUP_CUDA_TRY(cudaGetLastError());
  for (uint32_t r = 0; r < R; ++r) {
    SoupHandle* h = new SoupHandle();
    h->b = &b;
    h->r = r;
    b.views.push_back(h);
  }
  return bp.release();
}

void drop_graphs(Batch& b);

void destroy_batch(Batch* b) {
  if (!b) return;
  cudaStreamSynchronize(b->stream);
  drop_graphs(*b);
  if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
  void* ptrs[] = {b->rebuild_count, b->pos, b->vel, b->force, b->pos_ref, b->charge, b->slots, b->center, b->held, b->brng, b->trng,
                  b->frozen, b->id, b->slot_of, b->pos2, b->vel2, b->force2, b->charge2, b->slots2, b->center2,
                  b->held2, b->brng2, b->trng2, b->frozen2, b->id2, b->cell_of_slot, b->cell_count, b->cell_start, b->cell_sys,
                  b->cell_cursor, b->perm, b->scan_tmp, b->nl, b->nl_cnt, b->nl_shell, b->heads, b->head_sys, b->es_nl,
                  b->es_cnt, b->head_slot, b->head_e, b->head_pos, b->head_xq, b->head_d, b->head_flag, b->draw_site, b->sweep_band, b->hcell_count, b->hcell_start, b->hcell_cursor, b->hsorted, b->hsorted_xg, b->hcell_of, b->flags,
                  b->events, b->desorb, b->drift_bits, b->bond_items, b->bond_nitems, b->bond_sel, b->uf_parent, b->comp_min,
                  b->item_done, b->has_item, b->sweep_out, b->prot_rng_dev, b->sp, b->shared, b->sysid, b->an_buf[0],
                  b->an_buf[1]};
  for (void* p : ptrs) if (p) cudaFree(p);
  for (void* p : {(void*)b->diff.frames, (void*)b->diff.A, (void*)b->diff.B, (void*)b->diff.g, (void*)b->diff.jg,
                  (void*)b->diff.frozen_o, (void*)b->diff.partial, (void*)b->diff.all})
    if (p) cudaFree(p);
  for (const Batch::Mark& m : b->marks) { cudaEventDestroy(m.a); cudaEventDestroy(m.b); }
  for (cudaEvent_t e : b->event_pool) cudaEventDestroy(e);
  if (b->stream) cudaStreamDestroy(b->stream);
  for (SoupHandle* h : b->views) delete h;
  delete b;
}

// ---- guards (soup/src/soup-health.ts, soup/src/soup-grid-verlet.ts:266-313) ----------------
void guards(Batch& b, uint64_t chunk_start) {
  launch_nonfinite(b);
  std::vector<uint32_t> fl(FLAG_WORDS + 2 * b.R), drift(b.R);
  SOUP_CUDA_TRY(cudaMemcpyAsync(fl.data(), b.flags, 4 * fl.size(), cudaMemcpyDeviceToHost, b.stream));
  SOUP_CUDA_TRY(cudaMemcpyAsync(drift.data(), b.drift_bits, 4 * (size_t)b.R, cudaMemcpyDeviceToHost, b.stream));
  SOUP_CUDA_TRY(cudaStreamSynchronize(b.stream));
  SOUP_CUDA_TRY(cudaGetLastError());
  prof_flush(b);
  for (uint32_t r = 0; r < b.R; ++r) {
    const uint32_t np = fl[FLAG_WORDS + 2 * r], nv = fl[FLAG_WORDS + 2 * r + 1];
    if (np || nv) {
      char m[512];
      std::snprintf(m, sizeof m,
                    "non-finite state at step=%llu: non-finite components of positions=%u, velocities=%u of %u "
                    "(appeared in the step interval %llu..%llu) -- the computation diverged (Inf/NaN), any further "
                    "numbers from this run are meaningless",
                    (unsigned long long)b.step[r], np, nv, 3 * b.cfg[r].n, (unsigned long long)chunk_start,
                    (unsigned long long)b.step[r]);
      fail(SOUP_E_NONFINITE, m);
    }
  }
  if (fl[0]) {
    fail(SOUP_E_LIST_OVERFLOW, "Verlet list: verletList.listCapacity=" + std::to_string(b.list_cap) +
                                   " was insufficient -- at least one particle found more candidates than the list "
                                   "holds (data may have been silently dropped)");
  }
  if (fl[1]) {
    uint32_t r = 0;
    while (r + 1 < b.R && !b.cfg[r].es_enabled) ++r;
    char m[400];
    std::snprintf(m, sizeof m,
                  "long-range electrostatics list: longRangeListCapacity=%u or the headIdx size (%u) was insufficient "
                  "at rc_es=%.4f (heads found=%u) -- data may have been silently dropped",
                  b.cfg[r].es_list_capacity, b.hsp[r].nheads, b.cfg[r].es_cutoff, b.hsp[r].nheads);
    fail(SOUP_E_ES_OVERFLOW, m);
  }
  if (fl[6]) fail(SOUP_E_STATE, "bond pass: item buffer overflow");
  for (uint32_t r = 0; r < b.R; ++r) {
    float d2;
    std::memcpy(&d2, &drift[r], 4);
    const double d = std::sqrt(std::max(0.0, (double)d2));
    if (!std::isfinite(d))
      fail(SOUP_E_NONFINITE, "Verlet list: the measured drift is not a number (NaN) -- the state is already non-finite, "
                             "see soup/src/soup-health.ts's assertStateFinite");
    if (d > b.cfg[r].skin / 2 + 1e-6) {
      char m[320];
      std::snprintf(m, sizeof m,
                    "Verlet list: the measured drift %.4f exceeds skin/2=%.4f -- the analytic bound (verletList.basis) "
                    "did not hold for the real trajectory, the rebuild was not frequent enough",
                    d, b.cfg[r].skin / 2);
      fail(SOUP_E_DRIFT, m);
    }
  }
}

bool drift_exceeds(Batch& b) {
  std::vector<uint32_t> drift(b.R);
  SOUP_CUDA_TRY(cudaMemcpyAsync(drift.data(), b.drift_bits, 4 * (size_t)b.R, cudaMemcpyDeviceToHost, b.stream));
  SOUP_CUDA_TRY(cudaStreamSynchronize(b.stream));
  for (uint32_t r = 0; r < b.R; ++r) {
    float d2;
    std::memcpy(&d2, &drift[r], 4);
    if (!(d2 <= b.hsp[r].skin_half2)) return true;
  }
  return false;
}

void sweep_all(Batch& b, std::vector<SoupSweepResult>* out) {
  launch_sweep(b, SOUP_NONE_U32);
  std::vector<double> so(4 * (size_t)b.R);
  SOUP_CUDA_TRY(cudaMemcpyAsync(so.data(), b.sweep_out, 8 * so.size(), cudaMemcpyDeviceToHost, b.stream));
  SOUP_CUDA_TRY(cudaMemcpyAsync(b.prot_rng.data(), b.prot_rng_dev, 4 * (size_t)b.R, cudaMemcpyDeviceToHost, b.stream));
  // soup/src/soup-protonation.ts:62-73: F(x) is stale after the charges changed.  The reference
  // re-runs its rebuild+force pass; in drift-triggered mode only the force is recomputed (the lists
  // are sets that do not depend on charges, and the drift trigger keeps them complete).
  if (b.cfg[0].rebuild_on_drift) {
    // only head-head terms depend on charges when only heads carry charge and the polar class is
    // the heads' kind alone: the other particles' forces stand, bit for bit
    bool heads_only = b.polar_is_charged_kind && !std::getenv("SOUP_SWEEP_FORCE_ALL");
    for (uint32_t r = 0; r < b.R; ++r) heads_only = heads_only && !b.off_head_charge[r];
    if (heads_only) launch_force_heads(b);
    else launch_force(b);
    b.force_fresh = true;
  }
  else force_pass(b);
  SOUP_CUDA_TRY(cudaStreamSynchronize(b.stream));
  for (uint32_t r = 0; r < b.R; ++r)
    if (so[4 * r] < 0)
      fail(SOUP_E_TIMEOUT, "constant-pH sweep: a handoff between the cluster's CTAs did not arrive within its "
                           "poll limit; the charges of this sweep are not valid");
  b.sweeps++;
  if (out) {
    out->resize(b.R);
    for (uint32_t r = 0; r < b.R; ++r) {
      SoupSweepResult& s = (*out)[r];
      s.heads = (uint32_t)so[4 * r];
      s.attempts = s.heads;
      s.accepted = (uint32_t)so[4 * r + 1];
      s.d_es_mean_kt = so[4 * r + 2];
      s.deprotonated = (uint32_t)so[4 * r + 3];
      s.alpha = s.heads ? (double)s.deprotonated / s.heads : 0.0;
    }
  }
}

void drop_graphs(Batch& b) {
  for (auto& g : b.graphs) cudaGraphExecDestroy(g.exec);
  b.graphs.clear();
}

// Capture `chunk` steps starting at global step `start` (soup-integrate.ts's per-step schedule) as one
// graph.  With drift-triggered rebuilds each step holds a one-thread decision kernel and a
// conditional node whose body is the rebuild, so the graph never waits on the host.
Batch::ChunkGraph capture_chunk(Batch& b, uint64_t chunk, uint64_t start, uint64_t key) {
  const SoupConfig& c0 = b.cfg[0];
  const uint64_t l0 = b.launches;
  uint64_t fixed_rebuilds = 0;
  cudaStream_t main = b.stream;
  SOUP_CUDA_TRY(cudaStreamBeginCapture(main, cudaStreamCaptureModeThreadLocal));
  try {
    for (uint64_t k = 0; k < chunk; ++k) {
      const uint64_t g = start + k;
      if (k == 0) launch_kick_drift(b);   // later steps' kick and drift ride on the previous thermostat
      if (c0.rebuild_on_drift) {
        cudaStreamCaptureStatus st;
        cudaGraph_t cg = nullptr;
        const cudaGraphNode_t* deps = nullptr;
        size_t nd = 0;
        SOUP_CUDA_TRY(cudaStreamGetCaptureInfo(main, &st, nullptr, &cg, nullptr, nullptr));
        cudaGraphConditionalHandle h;
        SOUP_CUDA_TRY(cudaGraphConditionalHandleCreate(&h, cg, 0, 0));
        launch_rebuild_decide(b, h);
        SOUP_CUDA_TRY(cudaStreamGetCaptureInfo(main, &st, nullptr, &cg, &deps, &nd));
        cudaGraphNodeParams np = {};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = h;
        np.conditional.type = cudaGraphCondTypeIf;
        np.conditional.size = 1;
        cudaGraphNode_t node;
        SOUP_CUDA_TRY(cudaGraphAddNode(&node, cg, deps, nd, &np));
        const uint64_t lb = b.launches;
        b.stream = b.cap_stream;
        SOUP_CUDA_TRY(cudaStreamBeginCaptureToGraph(b.cap_stream, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                                    cudaStreamCaptureModeThreadLocal));
        rebuild_launches(b);
        cudaGraph_t body = nullptr;
        SOUP_CUDA_TRY(cudaStreamEndCapture(b.cap_stream, &body));
        b.stream = main;
        b.body_launches = b.launches - lb;
        b.launches = lb;
        SOUP_CUDA_TRY(cudaStreamUpdateCaptureDependencies(main, &node, 1, cudaStreamSetCaptureDependencies));
      } else if (g % c0.rebuild_every == 0) {
        rebuild_launches(b);
        ++fixed_rebuilds;
      }
      launch_force(b);
      if (g % c0.bond_interval == 0) launch_bonds(b);
      if (k + 1 < chunk) launch_thermo_drift(b);
      else launch_kick_thermo(b);
    }
  } catch (...) {
    b.stream = main;
    cudaGraph_t broken = nullptr;
    cudaStreamEndCapture(main, &broken);
    if (broken) cudaGraphDestroy(broken);
    b.launches = l0;
    throw;
  }
  cudaGraph_t graph = nullptr;
  SOUP_CUDA_TRY(cudaStreamEndCapture(main, &graph));
  Batch::ChunkGraph cgr{key, nullptr, b.launches - l0, fixed_rebuilds};
  b.launches = l0;
  const cudaError_t e = cudaGraphInstantiate(&cgr.exec, graph, 0);
  cudaGraphDestroy(graph);
  SOUP_CUDA_TRY(e);
  return cgr;
}

uint64_t chunk_key(const Batch& b, uint64_t chunk, uint64_t start) {
  const SoupConfig& c0 = b.cfg[0];
  return chunk | ((start % c0.bond_interval) << 20) | (c0.rebuild_on_drift ? 0ull : ((start % c0.rebuild_every) << 40));
}
const Batch::ChunkGraph* find_graph(const Batch& b, uint64_t key) {
  for (auto& x : b.graphs)
    if (x.key == key) return &x;
  return nullptr;
}
// capture (without running) the graphs of every schedule phase the chunks from `start` go through
void prepare_graphs(Batch& b, uint64_t chunk, uint64_t start) {
  const SoupConfig& c0 = b.cfg[0];
  const uint64_t period = c0.rebuild_on_drift ? c0.bond_interval : std::lcm<uint64_t>(c0.bond_interval, c0.rebuild_every);
  for (uint64_t s0 = start, k = 0; k < period; ++k, s0 += chunk) {
    const uint64_t key = chunk_key(b, chunk, s0);
    if (find_graph(b, key)) continue;
    if (b.graphs.size() >= 16) return;
    b.graphs.push_back(capture_chunk(b, chunk, s0, key));
    if (chunk_key(b, chunk, s0 + chunk) == chunk_key(b, chunk, start)) return;   // the phases repeat
  }
}

// one chunk from its cached graph (captured on first use); the host bookkeeping of the steps
void run_chunk_graph(Batch& b, uint64_t chunk, uint64_t start) {
  const uint64_t key = chunk_key(b, chunk, start);
  const Batch::ChunkGraph* g = find_graph(b, key);
  if (!g) {
    if (b.graphs.size() >= 16) drop_graphs(b);
    b.graphs.push_back(capture_chunk(b, chunk, start, key));
    g = &b.graphs.back();
  }
  SOUP_CUDA_TRY(cudaGraphLaunch(g->exec, b.stream));
  b.launches += g->launches;
  b.rebuilds += g->rebuilds_fixed;
  for (uint32_t r = 0; r < b.R; ++r) b.step[r] += chunk;
}

// the rebuilds the conditional nodes took since the last call (the stream is synchronised)
void count_graph_rebuilds(Batch& b) {
  uint32_t c = 0;
  SOUP_CUDA_TRY(cudaMemcpy(&c, b.rebuild_count, 4, cudaMemcpyDeviceToHost));
  const uint32_t d = c - b.rebuild_count_seen;
  b.rebuild_count_seen = c;
  b.rebuilds += d;
  b.launches += (uint64_t)d * b.body_launches;
}

// soup/src/soup-integrate.ts:136-175, for every replica in lockstep
void step_batch(Batch& b, uint64_t n) {
  const SoupConfig& c0 = b.cfg[0];
  const uint64_t chunk_max = c0.chunk_steps ? c0.chunk_steps : 1000;
  uint64_t done = 0;
  while (done < n) {
    const uint64_t chunk = std::min(chunk_max, n - done);
    const uint64_t chunk_start = b.step[0];
    const bool graph = b.graphs_enabled && !b.prof && chunk >= 4;
    if (graph) {
      run_chunk_graph(b, chunk, chunk_start);
    } else {
      for (uint64_t k = 0; k < chunk; ++k) {
        const uint64_t g = b.step[0];
        const bool bonds = g % c0.bond_interval == 0;
        if (k == 0) launch_kick_drift(b);
        bool reb;
        if (c0.rebuild_on_drift) reb = drift_exceeds(b);
        else reb = g % c0.rebuild_every == 0;
        if (reb) rebuild(b);
        launch_force(b);
        if (bonds) launch_bonds(b);
        if (k + 1 < chunk) launch_thermo_drift(b);
        else launch_kick_thermo(b);
        for (uint32_t r = 0; r < b.R; ++r) b.step[r]++;
      }
    }
    guards(b, chunk_start);
    if (graph) count_graph_rebuilds(b);
    bool any = false;
    for (uint32_t r = 0; r < b.R; ++r)
      if (b.cfg[r].es_enabled && b.step[r] >= b.next_sweep[r]) { any = true; b.next_sweep[r] = b.step[r] + b.cfg[r].sweep_every; }
    if (any) sweep_all(b, nullptr);
    done += chunk;
  }
}

// ---- readbacks -------------------------------------------------------------------------------
// Replica r's array in original order, gathered on the device into scratch (the gather's staging
// buffer, free outside a rebuild) and copied out in one piece; bond partners and centre links map
// from global slots back to replica indices.
template <class T>
__global__ void k_to_original(const T* __restrict__ src, const uint32_t* __restrict__ id, uint32_t off, uint32_t n,
                              uint32_t per, bool map_ids, T* __restrict__ dst) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const uint32_t i = id[off + k] - off;
  for (uint32_t e = 0; e < per; ++e) {
    T v = src[(size_t)(off + k) * per + e];
    if constexpr (std::is_same<T, uint32_t>::value) {
      if (map_ids && v != NONE) v -= off;
    }
    dst[(size_t)i * per + e] = v;
  }
}
template <class T>
void read_replica(Batch& b, uint32_t r, const T* dev, uint32_t per, T* dst, bool map_ids) {
  const uint32_t n = b.cfg[r].n, off = b.hsp[r].slot_off;
  static_assert(sizeof(T) <= 16, "scratch holds 16 bytes a particle");
  if (sizeof(T) * per > 16) fail(SOUP_E_ARG, "readback wider than the scratch");
  T* scratch = reinterpret_cast<T*>(b.pos2);
  if (n) k_to_original<T><<<(n + 255) / 256, 256, 0, b.stream>>>(dev, b.id, off, n, per, map_ids, scratch);
  SOUP_CUDA_TRY(cudaGetLastError());
  SOUP_CUDA_TRY(cudaMemcpyAsync(dst, scratch, sizeof(T) * (size_t)n * per, cudaMemcpyDeviceToHost, b.stream));
  SOUP_CUDA_TRY(cudaStreamSynchronize(b.stream));
}

void need(size_t bytes, size_t want) {
  if (bytes != want) fail(SOUP_E_ARG, "destination size " + std::to_string(bytes) + " does not match the array size " + std::to_string(want));
}

// ---- API plumbing ----------------------------------------------------------------------------
template <class F> int guarded(SoupHandle* h, F&& f) {
  try {
    if (!h || !h->b) fail(SOUP_E_ARG, "NULL handle");
    SOUP_CUDA_TRY(cudaSetDevice(h->b->device));
    f(*h->b, h->r);
    h->err.clear();
    return SOUP_OK;
  } catch (const SoupException& e) {
    if (h) h->err = e.msg;
    g_last_error = e.msg;
    return e.code;
  } catch (const CudaError& e) {
    std::string m = "CUDA: " + e.msg;
    if (h) h->err = m;
    g_last_error = m;
    return e.code == cudaErrorMemoryAllocation ? SOUP_E_OOM : SOUP_E_CUDA;
  } catch (const std::exception& e) {
    if (h) h->err = e.what();
    g_last_error = e.what();
    return SOUP_E_STATE;
  }
}

}  // namespace

// ---- differentiation ---------------------------------------------------------------------------
namespace {
// one step of the window: the plain step without bond Monte Carlo and without the sweep, every
// replica in lockstep
void diff_step(Batch& b) {
  const SoupConfig& c = b.cfg[0];
  launch_kick_drift(b);
  const bool reb = c.rebuild_on_drift ? drift_exceeds(b) : (b.step[0] % c.rebuild_every == 0);
  if (reb) rebuild(b);
  launch_force(b);
  launch_kick_thermo(b);
  for (uint32_t r = 0; r < b.R; ++r) b.step[r]++;
}
using ReplicaArrays = std::vector<std::vector<float>>;
using ReplicaWords = std::vector<std::vector<uint32_t>>;
void diff_read(Batch& b, ReplicaArrays& pos, ReplicaArrays& vel, ReplicaWords& trng) {
  pos.resize(b.R); vel.resize(b.R); trng.resize(b.R);
  for (uint32_t r = 0; r < b.R; ++r) {
    const uint32_t n = b.cfg[r].n;
    pos[r].resize(4 * (size_t)n); vel[r].resize(4 * (size_t)n); trng[r].resize(n);
    read_replica<float>(b, r, reinterpret_cast<const float*>(b.pos), 4, pos[r].data(), false);
    read_replica<float>(b, r, reinterpret_cast<const float*>(b.vel), 4, vel[r].data(), false);
    read_replica<uint32_t>(b, r, b.trng, 1, trng[r].data(), false);
  }
}
// the canonical state at a checkpoint: identity order, then the re-sort and force pass of a restore
void diff_restore(Batch& b, const ReplicaArrays& pos, const ReplicaArrays& vel, const ReplicaWords& trng) {
  DiffWindow& w = b.diff;
  for (uint32_t r = 0; r < b.R; ++r) {
    SoupInitState m{};
    m.positions = pos[r].data(); m.velocities = vel[r].data(); m.thermo_rng = trng[r].data();
    m.bond_slots = w.slots[r].data(); m.center_link = w.center[r].data(); m.center_held = w.held[r].data();
    m.bond_rng = w.brng[r].data(); m.charges = w.charge[r].data(); m.frozen = w.frozen[r].data();
    const uint32_t prot = b.prot_rng[r];
    upload_replica(b, r, &m, false);
    b.prot_rng[r] = prot;
  }
  force_pass(b);
}
// lists valid for the positions now in b.pos: kept while no particle has moved more than skin/2
// from where the lists were built (the forward step's own test), rebuilt otherwise
void refresh_lists(Batch& b) {
  SOUP_CUDA_TRY(cudaMemsetAsync(b.drift_bits, 0, sizeof(uint32_t) * b.R, b.stream));
  launch_max_drift(b);
  if (drift_exceeds(b)) rebuild(b);
}
// the device budget for keeping every frame of a window (SOUP_DIFF_FRAME_BUDGET_MB, default 8 GiB)
size_t frame_budget() {
  if (const char* e = std::getenv("SOUP_DIFF_FRAME_BUDGET_MB")) return (size_t)std::atoll(e) << 20;
  return (size_t)8 << 30;
}
template <class T> T* dgrow(T* p, size_t& cap, size_t want) {
  if (want <= cap) return p;
  if (p) cudaFree(p);
  T* q = nullptr;
  SOUP_CUDA_TRY(cudaMalloc(&q, sizeof(T) * want));
  cap = want;
  return q;
}
constexpr int kDepthPairs[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
}  // namespace

// ---- autotuning -------------------------------------------------------------------------------
namespace {
// Every replica's state in original order and the host schedule, to restore after trial steps.
struct TuneSnapshot {
  std::vector<std::vector<float>> pos, vel, q;
  std::vector<std::vector<uint32_t>> slots, center, held, brng, trng, frozen;
  std::vector<uint64_t> step, next_sweep;
  std::vector<uint32_t> prot_rng, events, desorb;
  uint64_t rebuilds = 0, sweeps = 0;
};
TuneSnapshot tune_snapshot(Batch& b) {
  TuneSnapshot t;
  const uint32_t R = b.R;
  t.pos.resize(R); t.vel.resize(R); t.q.resize(R); t.slots.resize(R); t.center.resize(R); t.held.resize(R);
  t.brng.resize(R); t.trng.resize(R); t.frozen.resize(R);
  for (uint32_t r = 0; r < R; ++r) {
    const uint32_t n = b.cfg[r].n;
    t.pos[r].resize(4 * (size_t)n); t.vel[r].resize(4 * (size_t)n); t.q[r].resize(n); t.slots[r].resize(3 * (size_t)n);
    t.center[r].resize(n); t.held[r].resize(n); t.brng[r].resize(n); t.trng[r].resize(n); t.frozen[r].resize(n);
    std::vector<uint8_t> fr(n);
    read_replica<float>(b, r, reinterpret_cast<const float*>(b.pos), 4, t.pos[r].data(), false);
    read_replica<float>(b, r, reinterpret_cast<const float*>(b.vel), 4, t.vel[r].data(), false);
    read_replica<float>(b, r, b.charge, 1, t.q[r].data(), false);
    read_replica<uint32_t>(b, r, b.slots, 3, t.slots[r].data(), true);
    read_replica<uint32_t>(b, r, b.center, 1, t.center[r].data(), true);
    read_replica<uint32_t>(b, r, b.held, 1, t.held[r].data(), false);
    read_replica<uint32_t>(b, r, b.brng, 1, t.brng[r].data(), false);
    read_replica<uint32_t>(b, r, b.trng, 1, t.trng[r].data(), false);
    read_replica<uint8_t>(b, r, b.frozen, 1, fr.data(), false);
    t.frozen[r].assign(fr.begin(), fr.end());
  }
  t.events.resize(2 * SOUP_MAX_RULES * (size_t)R);
  t.desorb.resize(2 * (size_t)R);
  SOUP_CUDA_TRY(cudaMemcpy(t.events.data(), b.events, 4 * t.events.size(), cudaMemcpyDeviceToHost));
  SOUP_CUDA_TRY(cudaMemcpy(t.desorb.data(), b.desorb, 4 * t.desorb.size(), cudaMemcpyDeviceToHost));
  t.step = b.step; t.next_sweep = b.next_sweep; t.prot_rng = b.prot_rng;
  t.rebuilds = b.rebuilds; t.sweeps = b.sweeps;
  return t;
}
void tune_restore(Batch& b, const TuneSnapshot& t) {
  for (uint32_t r = 0; r < b.R; ++r) {
    SoupInitState m{};
    m.positions = t.pos[r].data(); m.velocities = t.vel[r].data(); m.charges = t.q[r].data();
    m.bond_slots = t.slots[r].data(); m.center_link = t.center[r].data(); m.center_held = t.held[r].data();
    m.bond_rng = t.brng[r].data(); m.thermo_rng = t.trng[r].data(); m.frozen = t.frozen[r].data();
    upload_replica(b, r, &m, false);
  }
  SOUP_CUDA_TRY(cudaMemcpyAsync(b.events, t.events.data(), 4 * t.events.size(), cudaMemcpyHostToDevice, b.stream));
  SOUP_CUDA_TRY(cudaMemcpyAsync(b.desorb, t.desorb.data(), 4 * t.desorb.size(), cudaMemcpyHostToDevice, b.stream));
  b.step = t.step; b.next_sweep = t.next_sweep; b.prot_rng = t.prot_rng;
  for (uint32_t r = 0; r < b.R; ++r) SOUP_CUDA_TRY(cudaMemcpyAsync(b.prot_rng_dev + r, &b.prot_rng[r], 4, cudaMemcpyHostToDevice, b.stream));
  b.rebuilds = t.rebuilds; b.sweeps = t.sweeps;
  force_pass(b);
  SOUP_CUDA_TRY(cudaStreamSynchronize(b.stream));
}
// every replica's list geometry for a skin (scaled from the planned one) and a list-walk radius
// (the neighbour cell is list range / walk)
void tune_plan(Batch& b, const std::vector<double>& skin, int walk) {
  for (uint32_t r = 0; r < b.R; ++r) {
    SoupConfig& c = b.cfg[r];
    const double ds = skin[r] - c.skin;
    c.list_range += ds;
    if (c.es_enabled) c.es_list_range += ds;
    c.skin = skin[r];
    const SysParams old = b.hsp[r];
    SysParams p = make_sys(c);
    p.walk = walk;
    grid_of(c.box, c.list_range, walk, p.dims);
    p.slot_off = old.slot_off; p.n = old.n; p.head_off = old.head_off; p.nheads = old.nheads;
    b.hsp[r] = p;
  }
  drop_graphs(b);
  alloc_grids(b);
  upload_params(b);
}
template <class F> double tune_time(Batch& b, int reps, F&& f) {
  cudaEvent_t e0, e1;
  SOUP_CUDA_TRY(cudaEventCreate(&e0));
  SOUP_CUDA_TRY(cudaEventCreate(&e1));
  f();   // warm
  SOUP_CUDA_TRY(cudaEventRecord(e0, b.stream));
  for (int k = 0; k < reps; ++k) f();
  SOUP_CUDA_TRY(cudaEventRecord(e1, b.stream));
  SOUP_CUDA_TRY(cudaEventSynchronize(e1));
  float ms = 0.f;
  SOUP_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return ms / reps;
}
}  // namespace

extern "C" {

int soup_create(const SoupConfig* cfg, const SoupInitState* init, SoupHandle** out) {
  try {
    if (!out) fail(SOUP_E_ARG, "NULL output handle");
    *out = nullptr;
    Batch* b = make_batch(cfg, init, 1);
    SoupHandle* h = b->views[0];
    h->owns = true;
    *out = h;
    return SOUP_OK;
  } catch (const SoupException& e) {
    g_last_error = e.msg;
    return e.code;
  } catch (const CudaError& e) {
    g_last_error = "CUDA: " + e.msg;
    return e.code == cudaErrorMemoryAllocation ? SOUP_E_OOM : SOUP_E_CUDA;
  }
}

void soup_destroy(SoupHandle* h) {
  if (!h || !h->owns) return;
  destroy_batch(h->b);
}

const char* soup_last_error(const SoupHandle* h) { return h ? h->err.c_str() : g_last_error.c_str(); }

int soup_get_info(SoupHandle* h, SoupInfo* out) {
  return guarded(h, [&](Batch& b, uint32_t r) {
    if (!out) fail(SOUP_E_ARG, "NULL output");
    std::memset(out, 0, sizeof *out);
    out->n = b.cfg[r].n;
    out->global_step = b.step[r];
    out->list_capacity = b.cfg[r].list_capacity;
    out->es_list_capacity = b.cfg[r].es_enabled ? b.cfg[r].es_list_capacity : 0;
    out->heads = b.hsp[r].nheads;
    out->rebuilds = b.rebuilds;
    out->sweeps = b.sweeps;
    for (int a = 0; a < 3; ++a) out->box[a] = b.cfg[r].box[a];
    uint32_t bits = 0;
    SOUP_CUDA_TRY(cudaMemcpy(&bits, b.drift_bits + r, 4, cudaMemcpyDeviceToHost));
    float d2;
    std::memcpy(&d2, &bits, 4);
    out->max_drift = std::sqrt(std::max(0.0, (double)d2));
  });
}

int soup_fresh_state(const SoupConfig* cfg, float* positions, float* velocities, uint32_t* frozen, uint32_t* bond_rng,
                     uint32_t* thermo_rng) {
  if (!cfg) { g_last_error = "NULL config"; return SOUP_E_ARG; }
  host_fresh_state(*cfg, positions, velocities, frozen, bond_rng, thermo_rng);
  return SOUP_OK;
}
int soup_initial_charges(const SoupConfig* cfg, const float* positions, float* charges, uint32_t* prot) {
  if (!cfg || !positions || !charges) { g_last_error = "NULL argument"; return SOUP_E_ARG; }
  host_initial_charges(*cfg, positions, charges, prot);
  return SOUP_OK;
}

int soup_step(SoupHandle* h, uint64_t n) {
  return guarded(h, [&](Batch& b, uint32_t) {
    if (b.R != 1) fail(SOUP_E_STATE, "a replica of a batch is stepped with soup_batch_step");
    step_batch(b, n);
  });
}

int soup_relax_cold_start(SoupHandle* h, uint32_t iterations, double max_disp, double* out2) {
  return guarded(h, [&](Batch& b, uint32_t r) {
    if (iterations < 1) fail(SOUP_E_ARG, "relaxColdStart: iterations must be an integer >= 1");
    if (!(max_disp > 0)) fail(SOUP_E_ARG, "relaxColdStart: maxDisplacementSigma must be positive");
    if (b.step[r] != 0)
      fail(SOUP_E_STATE, "relaxColdStart: the system is already at step " + std::to_string(b.step[r]) +
                             " -- minimisation is allowed only before the first step");
    auto maxf = [&]() {
      force_pass(b);
      std::vector<float> f(4 * (size_t)b.N);
      SOUP_CUDA_TRY(cudaMemcpyAsync(f.data(), b.force, f.size() * 4, cudaMemcpyDeviceToHost, b.stream));
      SOUP_CUDA_TRY(cudaStreamSynchronize(b.stream));
      double m = 0;
      for (size_t i = 0; i < f.size(); ++i)
        if ((i & 3) != 3 && std::isfinite(f[i])) m = std::max(m, (double)std::fabs(f[i]));
      return m;
    };
    const double before = maxf();
    const double d0 = max_disp * b.cfg[r].sigma;
    for (uint32_t k = 0; k < iterations; ++k) {   // soup/src/soup-relax.ts:87-111
      const float d = (float)(d0 * (1.0 - (double)k / iterations));
      force_pass(b);
      launch_relax_step(b, d);
    }
    force_pass(b);
    guards(b, 0);
    const double after = maxf();
    if (out2) { out2[0] = before; out2[1] = after; }
  });
}

#define SOUP_READ(NAME, DEV, T, PER, MAP)                                                    \
  int NAME(SoupHandle* h, void* dst, size_t bytes) {                                           \
    return guarded(h, [&](Batch& b, uint32_t r) {                                              \
      if (!dst) fail(SOUP_E_ARG, "NULL destination");                                          \
      need(bytes, sizeof(T) * (PER) * (size_t)b.cfg[r].n);                                     \
      read_replica<T>(b, r, reinterpret_cast<const T*>(DEV), PER, static_cast<T*>(dst), MAP);  \
    });                                                                                        \
  }

SOUP_READ(soup_read_pos, b.pos, float, 4, false)
SOUP_READ(soup_read_vel, b.vel, float, 4, false)
SOUP_READ(soup_read_force, b.force, float, 4, false)
SOUP_READ(soup_read_slots, b.slots, uint32_t, 3, true)
SOUP_READ(soup_read_center_link, b.center, uint32_t, 1, true)
SOUP_READ(soup_read_center_held, b.held, uint32_t, 1, false)
SOUP_READ(soup_read_charges, b.charge, float, 1, false)
SOUP_READ(soup_read_rng_bond, b.brng, uint32_t, 1, false)
SOUP_READ(soup_read_rng_thermo, b.trng, uint32_t, 1, false)

int soup_read_frozen(SoupHandle* h, void* dst, size_t bytes) {
  return guarded(h, [&](Batch& b, uint32_t r) {
    if (!dst) fail(SOUP_E_ARG, "NULL destination");
    need(bytes, 4 * (size_t)b.cfg[r].n);
    std::vector<uint8_t> f(b.cfg[r].n);
    read_replica<uint8_t>(b, r, b.frozen, 1, f.data(), false);
    uint32_t* d = static_cast<uint32_t*>(dst);
    for (uint32_t i = 0; i < b.cfg[r].n; ++i) d[i] = f[i];
  });
}

int soup_forces(SoupHandle* h, void* dst, size_t bytes) {
  return guarded(h, [&](Batch& b, uint32_t r) {
    if (!dst) fail(SOUP_E_ARG, "NULL destination");
    need(bytes, 16 * (size_t)b.cfg[r].n);
    force_pass(b);
    read_replica<float>(b, r, reinterpret_cast<const float*>(b.force), 4, static_cast<float*>(dst), false);
  });
}
int soup_forces_brute(SoupHandle* h, void* dst, size_t bytes) {
  return guarded(h, [&](Batch& b, uint32_t r) {
    if (!dst) fail(SOUP_E_ARG, "NULL destination");
    need(bytes, 16 * (size_t)b.cfg[r].n);
    launch_force_brute(b);
    read_replica<float>(b, r, reinterpret_cast<const float*>(b.force), 4, static_cast<float*>(dst), false);
  });
}

int soup_read_events(SoupHandle* h, void* dst, size_t bytes) {
  return guarded(h, [&](Batch& b, uint32_t r) {
    need(bytes, 8 * (size_t)b.cfg[r].n_rules);
    SOUP_CUDA_TRY(cudaMemcpy(dst, b.events + 2 * SOUP_MAX_RULES * r, bytes, cudaMemcpyDeviceToHost));
  });
}
int soup_read_desorb(SoupHandle* h, void* dst, size_t bytes) {
  return guarded(h, [&](Batch& b, uint32_t r) {
    need(bytes, 8);
    SOUP_CUDA_TRY(cudaMemcpy(dst, b.desorb + 2 * r, 8, cudaMemcpyDeviceToHost));
  });
}
int soup_nonfinite_count(SoupHandle* h, uint32_t* out2) {
  return guarded(h, [&](Batch& b, uint32_t r) {
    launch_nonfinite(b);
    SOUP_CUDA_TRY(cudaMemcpyAsync(out2, b.flags + FLAG_WORDS + 2 * r, 8, cudaMemcpyDeviceToHost, b.stream));
    SOUP_CUDA_TRY(cudaStreamSynchronize(b.stream));
  });
}
int soup_read_protonation_rng(SoupHandle* h, uint32_t* out) {
  return guarded(h, [&](Batch& b, uint32_t r) { *out = b.prot_rng[r]; });
}

// ---- checkpoint payload (soup/src/checkpoint.ts:176-214) --------------------------------------
// One pass over replica r's slots un-permutes all eight arrays of a checkpoint into the re-sort
// gather's second buffers (free outside a rebuild); eight copies then land them back to back in the
// caller's buffer behind a single wait.
struct CkptArrays {
  const float4 *pos, *vel;
  const uint32_t *slots, *center, *held, *brng, *trng;
  const float* q;
  float4 *opos, *ovel;
  uint32_t *oslots, *ocenter, *oheld, *obrng, *otrng;
  float* oq;
};
__global__ void k_checkpoint_gather(CkptArrays a, const uint32_t* __restrict__ id, uint32_t off, uint32_t n) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const uint32_t s = off + k, i = id[s] - off;
  auto local = [off](uint32_t v) { return v == NONE ? v : v - off; };
  a.opos[i] = a.pos[s];
  a.ovel[i] = a.vel[s];
  for (int e = 0; e < 3; ++e) a.oslots[3 * (size_t)i + e] = local(a.slots[3 * (size_t)s + e]);
  a.ocenter[i] = local(a.center[s]);
  a.oheld[i] = a.held[s];
  a.obrng[i] = a.brng[s];
  a.otrng[i] = a.trng[s];
  a.oq[i] = a.q[s];
}

int soup_read_checkpoint(SoupHandle* h, void* dst, size_t bytes, SoupCheckpointScalars* scalars) {
  return guarded(h, [&](Batch& b, uint32_t r) {
    if (!dst) fail(SOUP_E_ARG, "NULL destination");
    const uint32_t n = b.cfg[r].n, off = b.hsp[r].slot_off;
    need(bytes, (size_t)SOUP_CHECKPOINT_BYTES_PER_PARTICLE * n);
    CkptArrays a{b.pos, b.vel, b.slots, b.center, b.held, b.brng, b.trng, b.charge,
                 b.pos2, b.vel2, b.slots2, b.center2, b.held2, b.brng2, b.trng2, b.charge2};
    if (n) k_checkpoint_gather<<<(n + 255) / 256, 256, 0, b.stream>>>(a, b.id, off, n);
    SOUP_CUDA_TRY(cudaGetLastError());
    char* o = static_cast<char*>(dst);
    const struct { const void* src; size_t per; } parts[] = {
        {b.pos2, 16}, {b.vel2, 16}, {b.slots2, 12}, {b.center2, 4}, {b.held2, 4}, {b.brng2, 4}, {b.trng2, 4}, {b.charge2, 4}};
    for (const auto& p : parts) {
      SOUP_CUDA_TRY(cudaMemcpyAsync(o, p.src, p.per * n, cudaMemcpyDeviceToHost, b.stream));
      o += p.per * n;
    }
    SoupCheckpointScalars s{};
    if (scalars) {
      s.global_step = b.step[r];
      s.n = n;
      s.n_rules = b.cfg[r].n_rules;
      s.protonation_rng = b.prot_rng[r];
      for (int a3 = 0; a3 < 3; ++a3) s.live_box[a3] = b.cfg[r].box[a3];
      SOUP_CUDA_TRY(cudaMemcpyAsync(s.desorb, b.desorb + 2 * r, 8, cudaMemcpyDeviceToHost, b.stream));
      SOUP_CUDA_TRY(cudaMemcpyAsync(s.events, b.events + 2 * SOUP_MAX_RULES * r, sizeof s.events,
                                    cudaMemcpyDeviceToHost, b.stream));
    }
    SOUP_CUDA_TRY(cudaStreamSynchronize(b.stream));
    if (scalars) *scalars = s;
  });
}

int soup_read_verlet(SoupHandle* h, uint32_t* counts, uint32_t* lists, size_t lists_cap) {
  return guarded(h, [&](Batch& b, uint32_t r) {
    const uint32_t n = b.cfg[r].n, off = b.hsp[r].slot_off;
    std::vector<uint32_t> cnt(n), ids(b.N), rows((size_t)n * b.list_cap);
    SOUP_CUDA_TRY(cudaMemcpyAsync(cnt.data(), b.nl_cnt + off, 4 * (size_t)n, cudaMemcpyDeviceToHost, b.stream));
    SOUP_CUDA_TRY(cudaMemcpyAsync(ids.data(), b.id, 4 * (size_t)b.N, cudaMemcpyDeviceToHost, b.stream));
    SOUP_CUDA_TRY(cudaMemcpyAsync(rows.data(), b.nl + (size_t)off * b.list_cap, 4 * rows.size(), cudaMemcpyDeviceToHost, b.stream));
    SOUP_CUDA_TRY(cudaStreamSynchronize(b.stream));
    std::vector<uint32_t> slot_of_local(n);
    for (uint32_t k = 0; k < n; ++k) slot_of_local[ids[off + k] - off] = k;
    uint64_t total = 0;
    for (uint32_t i = 0; i < n; ++i) { counts[i] = cnt[slot_of_local[i]]; total += counts[i]; }
    if (!lists) return;
    if (lists_cap < total) fail(SOUP_E_ARG, "lists buffer too small");
    uint64_t at = 0;
    for (uint32_t i = 0; i < n; ++i) {
      const uint32_t k = slot_of_local[i];
      uint32_t* o = lists + at;
      for (uint32_t s = 0; s < cnt[k]; ++s) o[s] = ids[rows[(size_t)k * b.list_cap + s]] - off;
      std::sort(o, o + cnt[k]);
      at += cnt[k];
    }
  });
}

int soup_read_es_list(SoupHandle* h, uint32_t* counts, uint32_t* lists, size_t lists_cap) {
  return guarded(h, [&](Batch& b, uint32_t r) {
    const SysParams& P = b.hsp[r];
    const uint32_t nh = P.nheads, hoff = P.head_off, off = P.slot_off;
    if (nh == 0) return;
    std::vector<uint32_t> cnt(nh), heads(b.H), rows((size_t)nh * b.es_cap);
    SOUP_CUDA_TRY(cudaMemcpyAsync(cnt.data(), b.es_cnt + hoff, 4 * (size_t)nh, cudaMemcpyDeviceToHost, b.stream));
    SOUP_CUDA_TRY(cudaMemcpyAsync(heads.data(), b.heads, 4 * (size_t)b.H, cudaMemcpyDeviceToHost, b.stream));
    SOUP_CUDA_TRY(cudaMemcpyAsync(rows.data(), b.es_nl + (size_t)hoff * b.es_cap, 4 * rows.size(), cudaMemcpyDeviceToHost,
                                  b.stream));
    SOUP_CUDA_TRY(cudaStreamSynchronize(b.stream));
    uint64_t total = 0;
    for (uint32_t h = 0; h < nh; ++h) { counts[h] = cnt[h]; total += cnt[h]; }
    if (!lists) return;
    if (lists_cap < total) fail(SOUP_E_ARG, "lists buffer too small");
    uint64_t at = 0;
    for (uint32_t h = 0; h < nh; ++h) {
      uint32_t* o = lists + at;
      for (uint32_t s = 0; s < cnt[h]; ++s) o[s] = heads[rows[(size_t)h * b.es_cap + s]] - off;
      std::sort(o, o + cnt[h]);
      at += cnt[h];
    }
  });
}

int soup_set_wait_limit(SoupHandle* h, uint32_t polls) {
  return guarded(h, [&](Batch& b, uint32_t) { b.wait_limit = polls; });
}

int soup_write_charges(SoupHandle* h, const float* src, size_t bytes) {
  return guarded(h, [&](Batch& b, uint32_t r) {
    const uint32_t n = b.cfg[r].n, off = b.hsp[r].slot_off;
    need(bytes, 4 * (size_t)n);
    std::vector<uint32_t> ids(n);
    SOUP_CUDA_TRY(cudaMemcpyAsync(ids.data(), b.id + off, 4 * (size_t)n, cudaMemcpyDeviceToHost, b.stream));
    SOUP_CUDA_TRY(cudaStreamSynchronize(b.stream));
    std::vector<float> q(n);
    for (uint32_t k = 0; k < n; ++k) q[k] = src[ids[k] - off];
    b.off_head_charge[r] = 0;
    for (uint32_t i = 0; i < n; ++i)
      if (src[i] != 0.f && (int)b.kinds[r][i] != b.cfg[r].charged_kind) b.off_head_charge[r] = 1;
    SOUP_CUDA_TRY(cudaMemcpyAsync(b.charge + off, q.data(), 4 * (size_t)n, cudaMemcpyHostToDevice, b.stream));
    force_pass(b);
    SOUP_CUDA_TRY(cudaStreamSynchronize(b.stream));
  });
}

int soup_write_state(SoupHandle* h, const SoupInitState* st) {
  return guarded(h, [&](Batch& b, uint32_t r) {
    if (!st) fail(SOUP_E_ARG, "NULL state");
    const uint32_t n = b.cfg[r].n, off = b.hsp[r].slot_off;
    // bring every current array of the replica to original order, overlay the given members
    std::vector<float> pos(4 * (size_t)n), vel(4 * (size_t)n), q(n);
    std::vector<uint32_t> slots(3 * (size_t)n), center(n), held(n), brng(n), trng(n);
    std::vector<uint8_t> fr(n);
    read_replica<float>(b, r, reinterpret_cast<const float*>(b.pos), 4, pos.data(), false);
    read_replica<float>(b, r, reinterpret_cast<const float*>(b.vel), 4, vel.data(), false);
    read_replica<float>(b, r, b.charge, 1, q.data(), false);
    read_replica<uint32_t>(b, r, b.slots, 3, slots.data(), true);
    read_replica<uint32_t>(b, r, b.center, 1, center.data(), true);
    read_replica<uint32_t>(b, r, b.held, 1, held.data(), false);
    read_replica<uint32_t>(b, r, b.brng, 1, brng.data(), false);
    read_replica<uint32_t>(b, r, b.trng, 1, trng.data(), false);
    read_replica<uint8_t>(b, r, b.frozen, 1, fr.data(), false);
    std::vector<uint32_t> fr32(fr.begin(), fr.end());
    SoupInitState m{};
    m.positions = st->positions ? st->positions : pos.data();
    m.velocities = st->velocities ? st->velocities : vel.data();
    m.bond_slots = st->bond_slots ? st->bond_slots : slots.data();
    m.center_link = st->center_link ? st->center_link : center.data();
    m.center_held = st->center_held ? st->center_held : held.data();
    m.bond_rng = st->bond_rng ? st->bond_rng : brng.data();
    m.thermo_rng = st->thermo_rng ? st->thermo_rng : trng.data();
    m.charges = st->charges ? st->charges : q.data();
    m.frozen = st->frozen ? st->frozen : fr32.data();
    m.events = st->events;
    m.desorb_events = st->desorb_events;
    // other replicas' slots stay where they are; this replica restarts from identity order
    upload_replica(b, r, &m, false);
    force_pass(b);
    SOUP_CUDA_TRY(cudaStreamSynchronize(b.stream));
  });
}

// resizeSoupGrid (soup/src/soup-buffers.ts:530-560): replica r's live box, its grid and the wall
// radius that follows it (liveRadius, soup/src/soup-confine.ts:76-78), then the rebuild and force pass
// planSoupGrid's refusal (soup/src/soup-plan.ts:133-146): the grid of cells of side
// interaction_range / cell_divisor needs 2 * ceil(list_range / cell) + 1 cells on every axis, and
// the box twice the bend rest length
void check_box(const SoupConfig& c, const double box[3]) {
  for (int a = 0; a < 3; ++a) if (!(box[a] > 0)) fail(SOUP_E_GEOMETRY, "box sides must be positive");
  const double cell = c.interaction_range / (c.cell_divisor ? c.cell_divisor : 1u);
  const int lwalk = (int)std::ceil(c.list_range / cell), min_cells = 2 * lwalk + 1;
  int dims[3];
  for (int a = 0; a < 3; ++a) dims[a] = std::max(1, (int)std::floor(box[a] / cell));
  const double half = std::min(box[0], std::min(box[1], box[2])) / 2;
  if (dims[0] < min_cells || dims[1] < min_cells || dims[2] < min_cells || !(half > c.r_bend)) {
    char m[400];
    std::snprintf(m, sizeof m,
                  "neighbour grid: box=[%g,%g,%g] gives cellSize=%.4f, dims=[%d,%d,%d] and min(box)/2=%.4f; it needs "
                  "dims>=%d (2*effectiveWalkRadius+1) on all three axes and min(box)/2 > bend.r0=%g",
                  box[0], box[1], box[2], cell, dims[0], dims[1], dims[2], half, min_cells, c.r_bend);
    fail(SOUP_E_GEOMETRY, m);
  }
}

void apply_box(Batch& b, uint32_t r, const double box[3]) {
  check_box(b.cfg[r], box);
  for (int a = 0; a < 3; ++a) b.cfg[r].box[a] = box[a];
  if (b.wall_r0[r] > 0) b.cfg[r].wall_radius = b.wall_r0[r] * (box[0] / b.wall_box0[r]);
  const SysParams old = b.hsp[r];
  SysParams p = make_sys(b.cfg[r]);
  p.slot_off = old.slot_off; p.n = old.n; p.head_off = old.head_off; p.nheads = old.nheads;
  b.hsp[r] = p;
  drop_graphs(b);
  alloc_grids(b);
  upload_params(b);
  force_pass(b);
  SOUP_CUDA_TRY(cudaStreamSynchronize(b.stream));
}

int soup_set_box(SoupHandle* h, const double box[3]) {
  return guarded(h, [&](Batch& b, uint32_t r) {
    if (!box) fail(SOUP_E_ARG, "NULL box");
    apply_box(b, r, box);
  });
}

__global__ void k_place_replica(const float4* __restrict__ src, const uint32_t* __restrict__ slot_of, uint32_t off,
                                uint32_t n, float4* __restrict__ pos) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) pos[slot_of[off + i]] = src[i];
}

int soup_scale_box(SoupHandle* h, const double target_box[3], double cohesion_cutoff, const uint32_t* cohesion_members,
                   uint32_t n_members) {
  return guarded(h, [&](Batch& b, uint32_t r) {
    if (!target_box) fail(SOUP_E_ARG, "NULL box");
    for (int a = 0; a < 3; ++a) if (!(target_box[a] > 0)) fail(SOUP_E_GEOMETRY, "box sides must be positive");
    if (!(cohesion_cutoff >= 0)) fail(SOUP_E_ARG, "scaleBoxTo: the cohesion cutoff must be a non-negative number");
    const uint32_t n = b.cfg[r].n, off = b.hsp[r].slot_off;
    std::vector<uint8_t> fr(n);
    if (n) SOUP_CUDA_TRY(cudaMemcpyAsync(fr.data(), b.frozen + off, n, cudaMemcpyDeviceToHost, b.stream));
    SOUP_CUDA_TRY(cudaStreamSynchronize(b.stream));
    size_t nfrozen = 0;
    for (uint8_t f : fr) nfrozen += f ? 1 : 0;
    if (nfrozen)
      fail(SOUP_E_STATE, "changing the box is impossible on a system with a mineral sheet: " + std::to_string(nfrozen) +
                             " immobile beads (areaMove/scaleBoxTo/dryWetCycle require CreateSoupOpts.clay=false, see "
                             "data/soup.json clay.basis §7)");
    std::vector<uint8_t> elig;
    if (cohesion_cutoff > 0 && cohesion_members) {
      elig.assign(n, 0);
      for (uint32_t k = 0; k < n_members; ++k) {
        if (cohesion_members[k] >= n) fail(SOUP_E_ARG, "scaleBoxTo: a cohesion member index is out of range");
        elig[cohesion_members[k]] = 1;
      }
    }
    // original-order positions and bond partners into the re-sort's second buffers (free outside a
    // rebuild); the new positions go to force2
    CkptArrays a{b.pos, b.vel, b.slots, b.center, b.held, b.brng, b.trng, b.charge,
                 b.pos2, b.vel2, b.slots2, b.center2, b.held2, b.brng2, b.trng2, b.charge2};
    if (n) k_checkpoint_gather<<<(n + 255) / 256, 256, 0, b.stream>>>(a, b.id, off, n);
    SOUP_CUDA_TRY(cudaGetLastError());
    const double* old_box = b.cfg[r].box;
    std::string err;
    const int st = run_rigid_map(b, b.pos2, b.slots2, n, nullptr, 0, cohesion_cutoff, elig.empty() ? nullptr : elig.data(),
                                 old_box, target_box, b.force2, true, err);
    if (st) fail(st, err);
    // planSoupGrid's refusal comes after the self-check, as in the reference (which throws it from
    // resizeSoupGrid), but before any position moves
    check_box(b.cfg[r], target_box);
    if (n) k_place_replica<<<(n + 255) / 256, 256, 0, b.stream>>>(b.force2, b.slot_of, off, n, b.pos);
    SOUP_CUDA_TRY(cudaGetLastError());
    b.launches += 2;
    const double nb[3] = {target_box[0], target_box[1], target_box[2]};
    apply_box(b, r, nb);
    guards(b, b.step[r]);
  });
}

int soup_scale_molecules_rigid(SoupHandle* h, const float* positions, uint32_t n, const uint32_t* edges,
                               uint32_t n_edges, const double old_box[3], const double new_box[3], float* out) {
  return guarded(h, [&](Batch& b, uint32_t) {
    if ((n && (!positions || !out)) || (n_edges && !edges) || !old_box || !new_box) fail(SOUP_E_ARG, "NULL argument");
    for (int a = 0; a < 3; ++a)
      if (!(old_box[a] > 0 && new_box[a] > 0)) fail(SOUP_E_GEOMETRY, "box sides must be positive");
    if (n == 0) return;
    float4 *dp = nullptr, *dout = nullptr;
    SOUP_CUDA_TRY(cudaMallocAsync(&dp, 16 * (size_t)n, b.stream));
    SOUP_CUDA_TRY(cudaMallocAsync(&dout, 16 * (size_t)n, b.stream));
    SOUP_CUDA_TRY(cudaMemcpyAsync(dp, positions, 16 * (size_t)n, cudaMemcpyHostToDevice, b.stream));
    std::string err;
    const int st = run_rigid_map(b, dp, nullptr, n, edges, n_edges, 0.0, nullptr, old_box, new_box, dout, false, err);
    if (st == SOUP_OK) SOUP_CUDA_TRY(cudaMemcpyAsync(out, dout, 16 * (size_t)n, cudaMemcpyDeviceToHost, b.stream));
    cudaFreeAsync(dp, b.stream);
    cudaFreeAsync(dout, b.stream);
    SOUP_CUDA_TRY(cudaStreamSynchronize(b.stream));
    if (st) fail(st, err);
  });
}

int soup_prepare_graphs(SoupHandle* h) {
  return guarded(h, [&](Batch& b, uint32_t) {
    const uint64_t chunk = b.cfg[0].chunk_steps ? b.cfg[0].chunk_steps : 1000;
    if (b.graphs_enabled && chunk >= 4) prepare_graphs(b, chunk, b.step[0]);
  });
}

int soup_autotune(SoupHandle* h, uint32_t steps, SoupTuneResult* out) {
  return guarded(h, [&](Batch& b, uint32_t) {
    if (steps != 0 && steps < 10) fail(SOUP_E_ARG, "autotune: at least 10 steps per candidate (0: shape only)");
    const TuneSnapshot snap = tune_snapshot(b);
    const bool prof = b.prof;
    b.prof = false;
    std::vector<double> planned(b.R);
    for (uint32_t r = 0; r < b.R; ++r) planned[r] = b.cfg[r].skin;
    const int walk0 = b.hsp[0].walk;
    const int tpp0 = b.tpp;
    auto steps_ms = [&]() { return tune_time(b, 1, [&] { step_batch(b, steps); }) / steps; };
    SoupTuneResult res{};
    if (steps) {
      res.ms_per_step_before = steps_ms();
      tune_restore(b, snap);
    }
    // block shape: lanes per particle of the list force, timed on the force alone
    const int tpps[4] = {1, 2, 4, 8};
    const bool queued0 = b.queued;
    double best = 1e30;
    for (int q = 0; q < 2; ++q)
      for (int t : tpps) {
        if (q && t != 1) continue;   // the compacted kernel is one lane per particle
        b.tpp = t;
        b.queued = q != 0;
        const double ms = tune_time(b, 5, [&] { launch_force_list(b); });
        if (ms < best) { best = ms; res.tpp = (uint32_t)t; res.queued = (uint32_t)q; }
      }
    b.tpp = (int)res.tpp;
    b.queued = res.queued != 0;
    drop_graphs(b);
    // cell size (the list-walk radius: cell = list range / walk) and the list build (a thread per
    // particle, or a group of lanes per cell), timed on the list build
    best = 1e30;
    bool cells_best = false;
    for (int w : {2, 3})
      for (int lc = 0; lc < 2; ++lc) {
        tune_plan(b, planned, w);
        if (lc && !b.list_by_cell) continue;
        b.list_cells = lc != 0;
        force_pass(b);
        // the walk sets the slot order the force gathers in: a rebuild and the ten force passes of a
        // typical rebuild interval
        const double ms = tune_time(b, 3, [&] {
          launch_cell_index(b);
          launch_build_lists(b);
          for (int f = 0; f < 10; ++f) launch_force_list(b);
        });
        if (ms < best) { best = ms; res.walk = (uint32_t)w; cells_best = lc != 0; }
      }
    b.list_cells = cells_best;
    res.list_cells = cells_best ? 1u : 0u;
    // skin (drift-triggered rebuilds only): at most the planned one, which sized the list capacity;
    // timed on whole steps, rebuilds and sweeps included
    res.skin_scale = 1.0;
    if (steps && b.cfg[0].rebuild_on_drift) {
      best = 1e30;
      for (double f : {0.6, 0.8, 1.0}) {
        std::vector<double> sk(b.R);
        for (uint32_t r = 0; r < b.R; ++r) sk[r] = planned[r] * f;
        tune_plan(b, sk, (int)res.walk);
        tune_restore(b, snap);
        const double ms = steps_ms();
        if (ms < best) { best = ms; res.skin_scale = f; }
      }
    }
    std::vector<double> sk(b.R);
    for (uint32_t r = 0; r < b.R; ++r) sk[r] = planned[r] * res.skin_scale;
    tune_plan(b, sk, (int)res.walk);
    tune_restore(b, snap);
    if (steps) {
      res.ms_per_step_after = steps_ms();
      tune_restore(b, snap);
    }
    b.prof = prof;
    res.tpp_before = (uint32_t)tpp0;
    res.queued_before = queued0 ? 1u : 0u;
    res.walk_before = (uint32_t)walk0;
    if (out) *out = res;
  });
}

int soup_apply_tuning(SoupHandle* h, const SoupTuneResult* t) {
  return guarded(h, [&](Batch& b, uint32_t) {
    if (!t) fail(SOUP_E_ARG, "NULL tuning");
    if (t->tpp != 1 && t->tpp != 2 && t->tpp != 4 && t->tpp != 8) fail(SOUP_E_ARG, "tuning: tpp must be 1, 2, 4 or 8");
    if (t->walk != 2 && t->walk != 3) fail(SOUP_E_ARG, "tuning: walk must be 2 or 3");
    if (!(t->skin_scale > 0.0 && t->skin_scale <= 1.0)) fail(SOUP_E_ARG, "tuning: skin_scale must be in (0, 1]");
    if (t->skin_scale != 1.0 && !b.cfg[0].rebuild_on_drift)
      fail(SOUP_E_ARG, "tuning: the skin can only be scaled with drift-triggered rebuilds");
    b.tpp = (int)t->tpp;
    b.queued = t->queued != 0;
    b.list_cells = t->list_cells != 0;
    std::vector<double> sk(b.R);
    for (uint32_t r = 0; r < b.R; ++r) sk[r] = b.cfg[r].skin * t->skin_scale;
    tune_plan(b, sk, (int)t->walk);
    force_pass(b);
    SOUP_CUDA_TRY(cudaStreamSynchronize(b.stream));
  });
}

int soup_protonation_sweep(SoupHandle* h, SoupSweepResult* out) {
  return guarded(h, [&](Batch& b, uint32_t r) {
    if (!b.cfg[r].es_enabled) fail(SOUP_E_STATE, "electrostatics is not enabled on this system");
    launch_sweep(b, r);
    std::vector<double> so(4);
    SOUP_CUDA_TRY(cudaMemcpyAsync(so.data(), b.sweep_out + 4 * r, 32, cudaMemcpyDeviceToHost, b.stream));
    SOUP_CUDA_TRY(cudaMemcpyAsync(&b.prot_rng[r], b.prot_rng_dev + r, 4, cudaMemcpyDeviceToHost, b.stream));
    force_pass(b);
    SOUP_CUDA_TRY(cudaStreamSynchronize(b.stream));
    if (so[0] < 0)
      fail(SOUP_E_TIMEOUT, "constant-pH sweep: a handoff between the cluster's CTAs did not arrive within its "
                           "poll limit; the charges of this sweep are not valid");
    b.sweeps++;
    b.next_sweep[r] = b.step[r] + b.cfg[r].sweep_every;
    if (out) {
      out->heads = (uint32_t)so[0]; out->attempts = out->heads; out->accepted = (uint32_t)so[1];
      out->d_es_mean_kt = so[2]; out->deprotonated = (uint32_t)so[3];
      out->alpha = out->heads ? (double)out->deprotonated / out->heads : 0.0;
    }
  });
}

int soup_debug_phase(SoupHandle* h, int phase) {
  return guarded(h, [&](Batch& b, uint32_t) {
    switch (phase) {
      case SOUP_PHASE_REBUILD: rebuild(b); break;
      case SOUP_PHASE_FORCE: launch_force(b); break;
      case SOUP_PHASE_KICK_DRIFT: launch_kick_drift(b); break;
      case SOUP_PHASE_KICK_THERMO: launch_kick_thermo(b); break;
      case SOUP_PHASE_BONDS: launch_bonds(b); break;
      case SOUP_PHASE_MAX_DRIFT: launch_max_drift(b); break;
      default: fail(SOUP_E_ARG, "unknown phase");
    }
    SOUP_CUDA_TRY(cudaStreamSynchronize(b.stream));
    SOUP_CUDA_TRY(cudaGetLastError());
  });
}

int soup_closure(SoupHandle* h, const uint32_t* member_idx, uint32_t n_members, const uint32_t* water_idx,
                 uint32_t n_water, const double centre[3], double cell, double radius, double vmin,
                 SoupClosureResult* out) {
  return guarded(h, [&](Batch& b, uint32_t r) {
    if (!out || !centre || (n_members && !member_idx) || (n_water && !water_idx)) fail(SOUP_E_ARG, "NULL argument");
    if (!(cell > 0) || !(radius > 0)) fail(SOUP_E_ARG, "cell and radius must be positive");
    std::string err;
    int st = run_closure(b, r, member_idx, n_members, water_idx, n_water, centre, cell, radius, vmin, nullptr, out, err);
    if (st) fail(st, err);
  });
}

int soup_closure_in_parcel(SoupHandle* h, const uint32_t* member_idx, uint32_t n_members, const uint32_t* water_idx,
                           uint32_t n_water, const double centre[3], double cell, double radius, double vmin,
                           const double parcel_centre[3], double parcel_radius, SoupClosureResult* out) {
  return guarded(h, [&](Batch& b, uint32_t r) {
    if (!out || !centre || !parcel_centre || (n_members && !member_idx) || (n_water && !water_idx))
      fail(SOUP_E_ARG, "NULL argument");
    if (!(cell > 0) || !(radius > 0)) fail(SOUP_E_ARG, "cell and radius must be positive");
    if (!(parcel_radius >= 0)) fail(SOUP_E_ARG, "the parcel radius must be a non-negative number");
    const double parcel[4] = {parcel_centre[0], parcel_centre[1], parcel_centre[2], parcel_radius};
    std::string err;
    int st = run_closure(b, r, member_idx, n_members, water_idx, n_water, centre, cell, radius, vmin, parcel, out, err);
    if (st) fail(st, err);
  });
}

int soup_amphiphile_labels(SoupHandle* h, uint32_t* head_of, uint32_t* n_out) {
  return guarded(h, [&](Batch& b, uint32_t r) {
    if (!head_of) fail(SOUP_E_ARG, "NULL argument");
    std::string err;
    int st = run_amphiphiles(b, r, head_of, n_out, err);
    if (st) fail(st, err);
  });
}


int soup_get_diff_params(SoupHandle* h, double* theta) {
  return guarded(h, [&](Batch& b, uint32_t r) {
    if (!theta) fail(SOUP_E_ARG, "NULL theta");
    const SoupConfig& c = b.cfg[r];
    for (int p = 0; p < 6; ++p) theta[p] = c.attr_scale[kDepthPairs[p][0]][kDepthPairs[p][1]];
    theta[6] = c.k_fene; theta[7] = c.k_bend; theta[8] = c.es_kappa;
  });
}

// the window's parameters are shared by the batch: every replica must agree on kappa (when its
// electrostatics is on), dt and gamma
void diff_check_batch(const Batch& b) {
  for (uint32_t r = 1; r < b.R; ++r) {
    if (b.cfg[r].dt != b.cfg[0].dt || b.cfg[r].gamma != b.cfg[0].gamma)
      fail(SOUP_E_STATE, "differentiation of a batch needs one dt and gamma for every replica");
    if (b.cfg[r].es_enabled && b.cfg[0].es_enabled && b.cfg[r].es_kappa != b.cfg[0].es_kappa)
      fail(SOUP_E_STATE, "differentiation of a batch needs one Debye kappa for every replica (equal ionic strength)");
  }
}

int soup_set_diff_params(SoupHandle* h, const double* theta) {
  return guarded(h, [&](Batch& b, uint32_t) {
    if (!theta) fail(SOUP_E_ARG, "NULL theta");
    diff_check_batch(b);
    for (int p = 0; p < SOUP_DIFF_NPARAM; ++p) if (!std::isfinite(theta[p])) fail(SOUP_E_ARG, "theta must be finite");
    if (!(theta[6] > 0) || !(theta[7] > 0) || !(theta[8] > 0)) fail(SOUP_E_ARG, "k_fene, k_bend and kappa must be positive");
    for (uint32_t r = 0; r < b.R; ++r) {
      SoupConfig& c = b.cfg[r];
      for (int p = 0; p < 6; ++p) {
        c.attr_scale[kDepthPairs[p][0]][kDepthPairs[p][1]] = theta[p];
        c.attr_scale[kDepthPairs[p][1]][kDepthPairs[p][0]] = theta[p];
      }
      c.k_fene = theta[6]; c.k_bend = theta[7]; c.es_kappa = theta[8];
      if (c.es_enabled) {
        c.es_shift_u = c.es_coeff_a * std::exp(-c.es_kappa * c.es_cutoff) / c.es_cutoff;
        c.es_shift_f = c.es_shift_u * (1 / c.es_cutoff + c.es_kappa);
      }
      SysParams& P = b.hsp[r];
      P.es_kappa = (float)c.es_kappa; P.es_fc = (float)c.es_shift_f;
      P.d_kappa = c.es_kappa; P.d_shiftU = c.es_shift_u; P.d_shiftF = c.es_shift_f;
    }
    b.hs = make_shared(b.cfg[0]);
    for (uint32_t r = 1; r < b.R; ++r) {
      const Shared o = make_shared(b.cfg[r]);
      b.hs.rmax2 = std::max(b.hs.rmax2, o.rmax2);
    }
    upload_params(b);
    launch_force(b);
    SOUP_CUDA_TRY(cudaStreamSynchronize(b.stream));
  });
}

int soup_diff_forward(SoupHandle* h, uint32_t steps, uint32_t checkpoint_every, float* traj_device) {
  return soup_diff_forward_strided(h, steps, checkpoint_every, 1, traj_device);
}

int soup_diff_forward_strided(SoupHandle* h, uint32_t steps, uint32_t checkpoint_every, uint32_t frame_stride,
                              float* traj_device) {
  return guarded(h, [&](Batch& b, uint32_t) {
    diff_check_batch(b);
    if (steps == 0 || checkpoint_every == 0) fail(SOUP_E_ARG, "steps and checkpoint_every must be positive");
    if (frame_stride == 0 || steps % frame_stride != 0)
      fail(SOUP_E_ARG, "frame_stride must be positive and divide steps");
    if (traj_device && (reinterpret_cast<uintptr_t>(traj_device) & 15u)) fail(SOUP_E_ARG, "traj_device must be 16-byte aligned");
    DiffWindow& w = b.diff;
    const uint32_t N = b.N, R = b.R;
    w.ready = false;
    w.charge.resize(R); w.slots.resize(R); w.center.resize(R); w.held.resize(R); w.brng.resize(R); w.frozen.resize(R);
    for (uint32_t r = 0; r < R; ++r) {
      const uint32_t n = b.cfg[r].n;
      w.charge[r].resize(n); w.slots[r].resize(3 * (size_t)n); w.center[r].resize(n); w.held[r].resize(n);
      w.brng[r].resize(n);
      std::vector<uint8_t> fr(n);
      read_replica<float>(b, r, b.charge, 1, w.charge[r].data(), false);
      read_replica<uint32_t>(b, r, b.slots, 3, w.slots[r].data(), true);
      read_replica<uint32_t>(b, r, b.center, 1, w.center[r].data(), true);
      read_replica<uint32_t>(b, r, b.held, 1, w.held[r].data(), false);
      read_replica<uint32_t>(b, r, b.brng, 1, w.brng[r].data(), false);
      read_replica<uint8_t>(b, r, b.frozen, 1, fr.data(), false);
      w.frozen[r].assign(fr.begin(), fr.end());
    }
    w.steps = steps; w.every = checkpoint_every; w.stride = frame_stride; w.step0 = b.step[0]; w.prot_rng = b.prot_rng;
    // the caller's frame of step t (t a multiple of the stride), or NULL
    auto out_frame = [&](uint32_t t) -> float4* {
      return (traj_device && t % frame_stride == 0) ? reinterpret_cast<float4*>(traj_device) + (size_t)(t / frame_stride) * N
                                                    : nullptr;
    };
    w.ck_pos.clear(); w.ck_vel.clear(); w.ck_trng.clear();
    const size_t frame_bytes = 16 * (size_t)N * (steps + 1);
    w.stored = frame_bytes <= frame_budget();
    if (w.stored) {   // keep every frame: the reverse pass reads them instead of replaying segments
      w.all = dgrow(w.all, w.all_cap, (size_t)N * (steps + 1));
      force_pass(b);
      adj_unpermute(b, w.all);
      for (uint32_t t = 0; t < steps; ++t) {
        diff_step(b);
        adj_unpermute(b, w.all + (size_t)(t + 1) * N);
      }
      for (uint32_t t = 0; t <= steps && traj_device; t += frame_stride)
        SOUP_CUDA_TRY(cudaMemcpyAsync(out_frame(t), w.all + (size_t)t * N, 16 * (size_t)N, cudaMemcpyDeviceToDevice,
                                      b.stream));
    }
    for (uint32_t t = 0; t < steps && !w.stored; ++t) {
      if (t % checkpoint_every == 0) {
        w.ck_pos.emplace_back(); w.ck_vel.emplace_back(); w.ck_trng.emplace_back();
        diff_read(b, w.ck_pos.back(), w.ck_vel.back(), w.ck_trng.back());
        diff_restore(b, w.ck_pos.back(), w.ck_vel.back(), w.ck_trng.back());
        if (t == 0 && traj_device) adj_unpermute(b, out_frame(0));
      }
      diff_step(b);
      if (float4* f = out_frame(t + 1)) adj_unpermute(b, f);
    }
    diff_read(b, w.end_pos, w.end_vel, w.end_trng);
    w.end_step = b.step[0];
    guards(b, w.step0);
    w.ready = true;
  });
}

int soup_diff_backward(SoupHandle* h, const float* dldx_device, double* theta_grad, float* dx0_device,
                       float* dv0_device) {
  return guarded(h, [&](Batch& b, uint32_t) {
    DiffWindow& w = b.diff;
    if (!w.ready) fail(SOUP_E_STATE, "no differentiable window: call soup_diff_forward first");
    if (!dldx_device || !theta_grad) fail(SOUP_E_ARG, "NULL argument");
    const uint32_t N = b.N, T = w.steps, K = w.every, S = w.stride;
    // dJ/dx_t: the caller gave it for the kept frames (every S-th step); the others are zero
    auto dldx_at = [&](uint32_t t) -> const float4* {
      return t % S == 0 ? reinterpret_cast<const float4*>(dldx_device) + (size_t)(t / S) * N : nullptr;
    };
    // scratch
    size_t cap1 = w.frames_cap;
    w.frames = dgrow(w.frames, cap1, (size_t)(K + 1) * N);
    w.frames_cap = cap1;
    if (!w.A) {
      SOUP_CUDA_TRY(cudaMalloc(&w.A, 16 * (size_t)N)); SOUP_CUDA_TRY(cudaMalloc(&w.B, 16 * (size_t)N));
      SOUP_CUDA_TRY(cudaMalloc(&w.g, 16 * (size_t)N)); SOUP_CUDA_TRY(cudaMalloc(&w.jg, 16 * (size_t)N));
      SOUP_CUDA_TRY(cudaMalloc(&w.frozen_o, (size_t)N));
    }
    size_t cap2 = w.partial_cap;
    w.partial = dgrow(w.partial, cap2, adj_partial_count(b));
    w.partial_cap = cap2;
    SOUP_CUDA_TRY(cudaMemsetAsync(w.partial, 0, 8 * adj_partial_count(b), b.stream));
    std::vector<uint8_t> fo(N, 0);   // by the batch's original index: replica r from its slot offset
    for (uint32_t r = 0; r < b.R; ++r)
      for (uint32_t i = 0; i < b.cfg[r].n; ++i) fo[b.hsp[r].slot_off + i] = (uint8_t)w.frozen[r][i];
    SOUP_CUDA_TRY(cudaMemcpyAsync(w.frozen_o, fo.data(), N, cudaMemcpyHostToDevice, b.stream));
    SOUP_CUDA_TRY(cudaMemcpyAsync(w.A, dldx_at(T), 16 * (size_t)N, cudaMemcpyDeviceToDevice, b.stream));
    SOUP_CUDA_TRY(cudaMemsetAsync(w.B, 0, 16 * (size_t)N, b.stream));
    SOUP_CUDA_TRY(cudaMemsetAsync(w.g, 0, 16 * (size_t)N, b.stream));
    const SysParams& P = b.hsp[0];
    const float a = 1.0f - P.gdt, hh = P.hdt, dt = P.dt;
    double theta[SOUP_DIFF_NPARAM] = {0};
    auto set_step = [&](uint64_t s0) { for (uint32_t r = 0; r < b.R; ++r) b.step[r] = s0; };
    if (w.stored) {
      for (uint32_t t = T; t > 0; --t) {
        adj_scatter_pos(b, w.all + (size_t)t * N);
        refresh_lists(b);
        adj_hvp(b, w.g, w.jg, w.partial);
        const float coef = (t - 1 == 0) ? hh : hh * (1.0f + a);
        adj_update(b, N, w.A, w.B, w.jg, dldx_at(t - 1), w.frozen_o, a, dt, coef, w.g, nullptr);
      }
      if (dv0_device) SOUP_CUDA_TRY(cudaMemcpyAsync(dv0_device, w.B, 16 * (size_t)N, cudaMemcpyDeviceToDevice, b.stream));
      adj_scatter_pos(b, w.all);
      refresh_lists(b);
      adj_hvp(b, w.g, w.jg, w.partial);
      adj_update(b, N, w.A, w.B, w.jg, nullptr, w.frozen_o, a, dt, 0.f, w.g, reinterpret_cast<float4*>(dx0_device));
    }
    const uint32_t nseg = w.stored ? 0 : (T + K - 1) / K;
    for (uint32_t seg = nseg; seg-- > 0;) {
      const uint32_t t0 = seg * K, t1 = std::min(t0 + K, T);
      set_step(w.step0 + t0);
      diff_restore(b, w.ck_pos[seg], w.ck_vel[seg], w.ck_trng[seg]);
      adj_unpermute(b, w.frames);
      for (uint32_t k = 0; k < t1 - t0; ++k) {
        diff_step(b);
        adj_unpermute(b, w.frames + (size_t)(k + 1) * N);
      }
      for (uint32_t t = t1; t > t0; --t) {
        adj_scatter_pos(b, w.frames + (size_t)(t - t0) * N);
        refresh_lists(b);
        adj_hvp(b, w.g, w.jg, w.partial);
        const float coef = (t - 1 == 0) ? hh : hh * (1.0f + a);
        adj_update(b, N, w.A, w.B, w.jg, dldx_at(t - 1), w.frozen_o, a, dt, coef, w.g, nullptr);
      }
      if (seg == 0) {   // time 0: the force at x_0 only feeds the first half kick
        if (dv0_device) SOUP_CUDA_TRY(cudaMemcpyAsync(dv0_device, w.B, 16 * (size_t)N, cudaMemcpyDeviceToDevice, b.stream));
        adj_scatter_pos(b, w.frames);
        refresh_lists(b);
        adj_hvp(b, w.g, w.jg, w.partial);
        adj_update(b, N, w.A, w.B, w.jg, nullptr, w.frozen_o, a, dt, 0.f, w.g, reinterpret_cast<float4*>(dx0_device));
      }
    }
    // back to the end of the window
    set_step(w.end_step);
    adj_theta_sum(b, w.partial, theta);
    diff_restore(b, w.end_pos, w.end_vel, w.end_trng);
    b.prot_rng = w.prot_rng;
    SOUP_CUDA_TRY(cudaStreamSynchronize(b.stream));
    for (int p = 0; p < SOUP_DIFF_NPARAM; ++p) theta_grad[p] = theta[p];
    // the sensitivity of a chaotic window grows exponentially with its length; once the FP32 adjoint
    // state overflows, the sum is no gradient
    for (int p = 0; p < SOUP_DIFF_NPARAM; ++p)
      if (!std::isfinite(theta[p]))
        fail(SOUP_E_NONFINITE, "adjoint: the parameter gradient is not finite (the window's sensitivity overflowed "
                               "the FP32 adjoint state); differentiate a shorter window");
  });
}

int soup_pairing_stats(SoupHandle* h, double contact_radius, SoupPairingStats* out) {
  return guarded(h, [&](Batch& b, uint32_t r) {
    if (!out || !(contact_radius > 0)) fail(SOUP_E_ARG, "pairingStats: bad argument");
    uint32_t c[5];
    std::string err;
    int st = run_pairing(b, r, contact_radius, c, err);
    if (st) fail(st, err);
    std::memset(out, 0, sizeof *out);
    out->heads = b.cfg[r].es_enabled ? b.hsp[r].nheads : 0;
    out->with_neighbour = c[0]; out->unlike_contacts = c[1]; out->like_contacts = c[2];
    out->paired = c[3]; out->charged = c[4];
    out->alpha = out->heads > 0 ? (double)c[4] / out->heads : 0.0;
    const uint32_t contacts = c[1] + c[2];
    out->unlike_fraction = contacts > 0 ? (double)c[1] / contacts : 0.0;
    out->unlike_fraction_random = 2 * out->alpha * (1 - out->alpha);
    out->paired_fraction = out->heads > 0 ? (double)c[3] / out->heads : 0.0;
    out->contact_radius = contact_radius;
  });
}

int soup_aggregate_shapes(SoupHandle* h, const uint32_t* member_idx, const uint32_t* labels, uint32_t n_members,
                          uint32_t max_shapes, SoupAggregateShape* out, uint32_t* n_components) {
  return guarded(h, [&](Batch& b, uint32_t r) {
    if (n_members && (!member_idx || !labels)) fail(SOUP_E_ARG, "aggregate shapes: bad argument");
    if (max_shapes && !out) fail(SOUP_E_ARG, "aggregate shapes: NULL output");
    // components by label, members ascending; largest first, then the smaller label
    std::vector<std::pair<uint32_t, uint32_t>> ml(n_members);
    for (uint32_t k = 0; k < n_members; ++k) ml[k] = {labels[k], member_idx[k]};
    std::sort(ml.begin(), ml.end());
    std::vector<std::pair<uint32_t, uint32_t>> comp;   // (begin in ml, size)
    for (uint32_t k = 0; k < n_members;) {
      uint32_t e = k;
      while (e < n_members && ml[e].first == ml[k].first) ++e;
      comp.push_back({k, e - k});
      k = e;
    }
    std::stable_sort(comp.begin(), comp.end(), [](const auto& x, const auto& y) { return x.second > y.second; });
    if (n_components) *n_components = (uint32_t)comp.size();
    const uint32_t ns = (uint32_t)std::min<size_t>(max_shapes, comp.size());
    if (ns == 0) return;
    std::vector<uint32_t> csr, start(1, 0);
    for (uint32_t c = 0; c < ns; ++c) {
      for (uint32_t k = 0; k < comp[c].second; ++k) csr.push_back(ml[comp[c].first + k].second);
      start.push_back((uint32_t)csr.size());
    }
    std::vector<double> o(10 * (size_t)ns);
    std::string err;
    int st = run_shapes(b, r, csr.data(), start.data(), ns, o.data(), err);
    if (st) fail(st, err);
    for (uint32_t c = 0; c < ns; ++c) {
      out[c].size = comp[c].second;
      out[c].label = ml[comp[c].first].first;
      for (int a = 0; a < 3; ++a) out[c].centre[a] = o[10 * c + 1 + a];
      for (int q = 0; q < 6; ++q) out[c].gyration[q] = o[10 * c + 4 + q];
    }
  });
}

int soup_aggregate_unwrap(SoupHandle* h, const uint32_t* members, uint32_t n_members, float* out) {
  return guarded(h, [&](Batch& b, uint32_t r) {
    if (n_members && (!members || !out)) fail(SOUP_E_ARG, "aggregate unwrap: NULL argument");
    std::string err;
    const int st = run_unwrap(b, r, members, n_members, out, err);
    if (st) fail(st, err);
  });
}

int soup_local_cavity_volume(SoupHandle* h, const float* positions, uint32_t n, double cell, double radius,
                             double* volume) {
  return guarded(h, [&](Batch& b, uint32_t) {
    if ((n && !positions) || !volume) fail(SOUP_E_ARG, "local cavity volume: NULL argument");
    std::string err;
    const int st = run_local_cavity(b, positions, n, cell, radius, volume, err);
    if (st) fail(st, err);
  });
}

int soup_box_cavity_volume(SoupHandle* h, const float* positions, uint32_t n, double cell, double radius,
                           double* volume) {
  return guarded(h, [&](Batch& b, uint32_t r) {
    if ((n && !positions) || !volume) fail(SOUP_E_ARG, "enclosedVolume: NULL argument");
    std::string err;
    const int st = run_local_cavity(b, positions, n, cell, radius, volume, err, b.cfg[r].box);
    if (st) fail(st, err);
  });
}

int soup_cluster_labels(SoupHandle* h, const uint32_t* member_idx, uint32_t n_members, double cutoff, int periodic_z,
                        uint32_t* labels, uint32_t* n_components) {
  return guarded(h, [&](Batch& b, uint32_t r) {
    if ((n_members && (!member_idx || !labels)) || !(cutoff > 0)) fail(SOUP_E_ARG, "bad argument");
    std::string err;
    int st = run_aggregates(b, r, member_idx, n_members, cutoff, labels, n_components, err, periodic_z != 0);
    if (st) fail(st, err);
  });
}

int soup_density_profile_z(SoupHandle* h, uint32_t bins, uint32_t head_kind_mask, uint32_t* head_counts,
                           uint32_t* tail_counts, uint32_t* escaped) {
  return guarded(h, [&](Batch& b, uint32_t r) {
    if (bins == 0 || bins > (1u << 24) || !head_counts || !tail_counts) fail(SOUP_E_ARG, "densityProfileZ: bad argument");
    std::string err;
    int st = run_profile_z(b, r, bins, head_kind_mask, head_counts, tail_counts, escaped, err);
    if (st) fail(st, err);
  });
}

int soup_aggregate_labels(SoupHandle* h, const uint32_t* member_idx, uint32_t n_members, double cutoff,
                          uint32_t* labels, uint32_t* n_components) {
  return guarded(h, [&](Batch& b, uint32_t r) {
    if ((n_members && (!member_idx || !labels)) || !(cutoff > 0)) fail(SOUP_E_ARG, "bad argument");
    std::string err;
    int st = run_aggregates(b, r, member_idx, n_members, cutoff, labels, n_components, err);
    if (st) fail(st, err);
  });
}

void* soup_stream(SoupHandle* h) { return (h && h->b) ? (void*)h->b->stream : nullptr; }

int soup_profile(SoupHandle* h, int enable) {
  return guarded(h, [&](Batch& b, uint32_t) {
    prof_flush(b);
    b.prof = enable != 0;
    for (int k = 0; k < SOUP_K_COUNT; ++k) { b.kt_ms[k] = 0; b.kt_n[k] = 0; }
  });
}

int soup_kernel_time(SoupHandle* h, int kernel, double* total_ms, uint64_t* launches) {
  return guarded(h, [&](Batch& b, uint32_t) {
    if (kernel < 0 || kernel >= SOUP_K_COUNT) fail(SOUP_E_ARG, "unknown kernel group");
    prof_flush(b);
    if (total_ms) *total_ms = b.kt_ms[kernel];
    if (launches) *launches = b.kt_n[kernel];
  });
}

uint64_t soup_launch_count(SoupHandle* h) { return (h && h->b) ? h->b->launches : 0; }

int soup_batch_create(const SoupConfig* cfgs, const SoupInitState* inits, uint32_t n_replicas, SoupBatch** out) {
  try {
    if (!out) fail(SOUP_E_ARG, "NULL output");
    *out = nullptr;
    Batch* b = make_batch(cfgs, inits, n_replicas);
    *out = new SoupBatch{b};
    return SOUP_OK;
  } catch (const SoupException& e) {
    g_last_error = e.msg;
    return e.code;
  } catch (const CudaError& e) {
    g_last_error = "CUDA: " + e.msg;
    return e.code == cudaErrorMemoryAllocation ? SOUP_E_OOM : SOUP_E_CUDA;
  }
}

int soup_batch_step(SoupBatch* sb, uint64_t n) {
  if (!sb || !sb->b) return SOUP_E_ARG;
  SoupHandle* h = sb->b->views[0];
  int st = guarded(h, [&](Batch& b, uint32_t) { step_batch(b, n); });
  if (st) sb->b->err = h->err;
  return st;
}
SoupHandle* soup_batch_replica(SoupBatch* sb, uint32_t r) {
  if (!sb || !sb->b || r >= sb->b->R) return nullptr;
  return sb->b->views[r];
}
const char* soup_batch_last_error(const SoupBatch* sb) { return sb && sb->b ? sb->b->err.c_str() : g_last_error.c_str(); }
void soup_batch_destroy(SoupBatch* sb) {
  if (!sb) return;
  destroy_batch(sb->b);
  delete sb;
}

}  // extern "C"

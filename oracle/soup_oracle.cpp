// soup_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A CPU restatement of the reference's soup MD step (nefayran/protocell-genesis), used as the
// parity checker for the CUDA library and as the timed CPU baseline.  Nothing in the product
// (protocell-genesis_b200/) links, loads or calls this file; only tests/, __graft_entry__.smoke()
// and bench.py's CPU legs do.
//
// Every function cites the reference file:line it restates.  Where the reference is racy
// (atomic list fill order, CAS arbitration in the bond kernels) this oracle defines the CANONICAL
// semantics the CUDA path must reproduce:
//   * Verlet and head lists are SETS, stored sorted by particle index;
//   * the bond-formation pass behaves as if one thread ran particle 0, 1, 2, ... to completion in
//     index order (a legal serialisation of the reference's concurrent dispatch);
//   * the constant-pH sweep keeps the reference's own candidate order (it is sequential there).
// Arithmetic: the per-pair f32 formulas are evaluated with no FMA contraction (built with
// -ffp-contract=off) in the reference's operation order; FP64 mode evaluates the same formulas in
// double for the force-accuracy reference; the pH sweep, closure and aggregate analyses use double
// with JavaScript Math.round semantics, as the reference's TypeScript does.
//
// Parity pinning: the reference cannot run in this environment (WebGPU in Chrome, TypeScript on
// Node; neither is available), so the oracle is pinned by the reference's own known-answer tests
// restated in tests/test_oracle_*.py (Henderson-Hasselbalch, exact two-head Boltzmann weights,
// F = -dU/dr, continuity at the cutoff, closure synthetics, list-vs-brute completeness).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <numeric>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/soup_b200.h"

namespace {

constexpr uint32_t NONE = 0xFFFFFFFFu;
constexpr uint32_t CANDIDATE_CAP = 6;  // soup/wgsl/bond-dispatch.wgsl:12

thread_local std::string g_err;

// ------------------------------------------------------------------------------------------------
// RNGs
// ------------------------------------------------------------------------------------------------

// soup/wgsl/step.wgsl:18-22 pcgSoup == soup/wgsl/bond-common.wgsl:132-136 bondPcg: a hash iterated
// on its own output (the state IS the last output).
inline uint32_t pcg_hash(uint32_t v) {
  uint32_t state = v * 747796405u + 2891336453u;
  uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
  return (word >> 22u) ^ word;
}
// soup/wgsl/step.wgsl:23 uniform01Soup: f32(v) / 2^32, f32 arithmetic (f32(v) rounds to nearest).
inline float u01f(uint32_t v) { return (float)v / 4294967296.0f; }

// soup/src/electrostatics.ts:308-315 pcgNext: an LCG state with the same output mix, as a double.
inline double pcg_next(uint32_t& s) {
  uint32_t v = s * 747796405u + 2891336453u;
  s = v;
  v = ((v >> ((v >> 28u) + 4u)) ^ v) * 277803737u;
  v = (v >> 22u) ^ v;
  return (double)v / 4294967296.0;
}

// soup/src/soup-init-state.ts:17-25 mulberry32.
struct Mulberry32 {
  uint32_t a;
  explicit Mulberry32(uint32_t seed) : a(seed) {}
  double operator()() {
    a = a + 0x6d2b79f5u;
    uint32_t t = (a ^ (a >> 15)) * (1u | a);
    t = (t + ((t ^ (t >> 7)) * (61u | t))) ^ t;
    return (double)(t ^ (t >> 14)) / 4294967296.0;
  }
};

// JavaScript Math.round: nearest integer, halves toward +infinity.
inline double js_round(double x) {
  double r = std::floor(x);
  return (x - r >= 0.5) ? r + 1.0 : r;
}
// JavaScript `%` on doubles is C fmod.
inline double js_mod(double a, double b) { return std::fmod(a, b); }

// ------------------------------------------------------------------------------------------------
// f32 uniforms, rounded the way the reference's Float32Array uploads round them
// ------------------------------------------------------------------------------------------------
struct U32f {
  float box[3];
  float sigma, eps, b_tt, k_fene, r_inf, k_bend, r_bend, wc, kT, gamma, dt;
  float radius[SOUP_MAX_KINDS];
  uint32_t cls[SOUP_MAX_KINDS];
  float attr[4][4];
  float acid;
  float c6;               // pow(2.0, 0.16666667) as a correctly rounded f32
  float list_range;       // VL.x
  float es_A, es_kappa, es_rc, es_fc, es_split, es_list_range, es_kind;
  float wall_r, wall_k;
  float kindA[SOUP_MAX_RULES], kindB[SOUP_MAX_RULES];
  float att_form[SOUP_MAX_RULES], att_break[SOUP_MAX_RULES];
  float acc_form[SOUP_MAX_RULES], acc_break[SOUP_MAX_RULES];
  float req_cat[SOUP_MAX_RULES], roleA[SOUP_MAX_RULES], roleB[SOUP_MAX_RULES];
  float cat_kind, head_terminal, head_cap, max_hold, interval;
};

U32f make_u32f(const SoupConfig& c) {
  U32f u{};
  for (int a = 0; a < 3; ++a) u.box[a] = (float)c.box[a];
  u.sigma = (float)c.sigma; u.eps = (float)c.epsilon; u.b_tt = (float)c.b_tt;
  u.k_fene = (float)c.k_fene; u.r_inf = (float)c.r_inf; u.k_bend = (float)c.k_bend;
  u.r_bend = (float)c.r_bend; u.wc = (float)c.wc; u.kT = (float)c.kT; u.gamma = (float)c.gamma;
  u.dt = (float)c.dt;
  for (int k = 0; k < SOUP_MAX_KINDS; ++k) { u.radius[k] = (float)c.radius[k]; u.cls[k] = c.kind_class[k]; }
  for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) u.attr[i][j] = (float)c.attr_scale[i][j];
  u.acid = (float)c.acid_soap_scale;
  u.c6 = (float)std::pow(2.0, (double)0.16666667f);
  u.list_range = (float)c.list_range;
  u.es_A = (float)c.es_coeff_a; u.es_kappa = (float)c.es_kappa; u.es_rc = (float)c.es_cutoff;
  u.es_fc = (float)c.es_shift_f; u.es_split = (float)c.es_split_radius;
  u.es_list_range = (float)c.es_list_range; u.es_kind = (float)c.charged_kind;
  u.wall_r = (float)c.wall_radius; u.wall_k = (float)c.wall_k;
  for (int r = 0; r < SOUP_MAX_RULES; ++r) {
    bool on = r < (int)c.n_rules;
    u.kindA[r] = on ? (float)c.rule_kind_a[r] : 0.f; u.kindB[r] = on ? (float)c.rule_kind_b[r] : 0.f;
    u.att_form[r] = on ? (float)c.attempt_form[r] : 0.f; u.att_break[r] = on ? (float)c.attempt_break[r] : 0.f;
    u.acc_form[r] = on ? (float)c.accept_form[r] : 0.f; u.acc_break[r] = on ? (float)c.accept_break[r] : 0.f;
    u.req_cat[r] = on ? (float)c.requires_catalyst[r] : 0.f;
    u.roleA[r] = on ? (float)c.role_a[r] : 0.f; u.roleB[r] = on ? (float)c.role_b[r] : 0.f;
  }
  u.cat_kind = (float)c.catalyst_kind; u.head_terminal = (float)c.head_terminal_only;
  u.head_cap = (float)c.head_chain_capacity; u.max_hold = (float)c.max_hold_steps;
  u.interval = (float)c.bond_interval;
  return u;
}

// ------------------------------------------------------------------------------------------------
// Pair physics, templated on the arithmetic type.  T=float follows the WGSL f32 formulas op for op;
// T=double is the FP64 reference used for the force-accuracy bar.
// ------------------------------------------------------------------------------------------------
template <class T> struct Phys {
  T sigma, eps, b_tt, k_fene, r_inf, k_bend, r_bend, wc, c6;
  T radius[SOUP_MAX_KINDS];
  uint32_t cls[SOUP_MAX_KINDS];
  T attr[4][4];
  T acid;
  T es_A, es_kappa, es_rc, es_fc, es_split;
  T box[3];

  static Phys from_f32(const U32f& u) {
    Phys p{};
    p.sigma = u.sigma; p.eps = u.eps; p.b_tt = u.b_tt; p.k_fene = u.k_fene; p.r_inf = u.r_inf;
    p.k_bend = u.k_bend; p.r_bend = u.r_bend; p.wc = u.wc; p.c6 = u.c6;
    for (int k = 0; k < SOUP_MAX_KINDS; ++k) { p.radius[k] = u.radius[k]; p.cls[k] = u.cls[k]; }
    for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) p.attr[i][j] = u.attr[i][j];
    p.acid = u.acid;
    p.es_A = u.es_A; p.es_kappa = u.es_kappa; p.es_rc = u.es_rc; p.es_fc = u.es_fc; p.es_split = u.es_split;
    for (int a = 0; a < 3; ++a) p.box[a] = u.box[a];
    return p;
  }
  static Phys from_f64(const SoupConfig& c) {
    Phys p{};
    p.sigma = c.sigma; p.eps = c.epsilon; p.b_tt = c.b_tt; p.k_fene = c.k_fene; p.r_inf = c.r_inf;
    p.k_bend = c.k_bend; p.r_bend = c.r_bend; p.wc = c.wc; p.c6 = std::pow(2.0, 1.0 / 6.0);
    for (int k = 0; k < SOUP_MAX_KINDS; ++k) { p.radius[k] = c.radius[k]; p.cls[k] = c.kind_class[k]; }
    for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) p.attr[i][j] = c.attr_scale[i][j];
    p.acid = c.acid_soap_scale;
    p.es_A = c.es_coeff_a; p.es_kappa = c.es_kappa; p.es_rc = c.es_cutoff; p.es_fc = c.es_shift_f;
    p.es_split = c.es_split_radius;
    for (int a = 0; a < 3; ++a) p.box[a] = c.box[a];
    return p;
  }

  static T rint_(T x) { return std::nearbyint(x); }  // WGSL round(): half to even
  // soup/wgsl/pair.wgsl:64-66 mi3
  T mi(T d, int a) const { return d - rint_(d / box[a]) * box[a]; }
  static T len3(T x, T y, T z) { return std::sqrt((x * x + y * y) + z * z); }
  // engine/wgsl/forces.wgsl:17 wca_cut
  T wca_cut(T b) const { return c6 * b; }
  // soup/wgsl/pair.wgsl:126 pairB
  T pairB(int ki, int kj) const { return (sigma * (radius[ki] + radius[kj])) * T(0.5); }
  // engine/wgsl/forces.wgsl:19-23 wca_dv
  T wca_dv(T r, T b) const {
    if (r >= wca_cut(b) || r <= T(0)) return T(0);
    T s6 = std::pow(b / r, T(6));
    return T(-24) * eps / r * (T(2) * s6 * s6 - s6);
  }
  // engine/wgsl/forces.wgsl:25-28 fene_dv
  T fene_dv(T r) const { T x = r / r_inf; return k_fene * r / (T(1) - x * x); }
  // engine/wgsl/forces.wgsl:30 bend_dv
  T bend_dv(T r) const { return k_bend * (r - r_bend); }
  // engine/wgsl/forces.wgsl:32-37 attr_dv
  T attr_dv(T r) const {
    const T PI = T(3.14159265);
    T rc = wca_cut(b_tt);
    if (r < rc || r > rc + wc) return T(0);
    T x = PI * (r - rc) / (T(2) * wc);
    return eps * PI * std::sin(T(2) * x) / (T(2) * wc);
  }
  // soup/wgsl/electrostatics.wgsl:65-71 esForceMag
  T es_mag(T r, T qq) const {
    if (es_A == T(0) || qq == T(0) || r >= es_rc) return T(0);
    T u = es_A * std::exp(-es_kappa * r) / r;
    return qq * (u * (T(1) / r + es_kappa) - es_fc);
  }
  // soup/wgsl/pair.wgsl:151-160 acidSoapScale
  T acid_scale(int ki, int kj, T qi, T qj) const {
    if (acid <= T(0)) return T(0);
    if (cls[ki] != 1u || cls[kj] != 1u) return T(0);
    if ((qi != T(0)) == (qj != T(0))) return T(0);
    return acid;
  }
  // soup/wgsl/pair.wgsl:168-204 nonbondedSoup, with esForceNear (electrostatics.wgsl:80-83)
  void nonbonded(const T* xi, const T* xj, int ki, int kj, T qi, T qj, T* f) const {
    T dx = mi(xi[0] - xj[0], 0), dy = mi(xi[1] - xj[1], 1), dz = mi(xi[2] - xj[2], 2);
    T r = len3(dx, dy, dz);
    if (r < T(1e-6)) return;
    T b = pairB(ki, kj);
    if (r < wca_cut(b)) {
      T s = wca_dv(r, b);
      f[0] = f[0] - s * dx / r; f[1] = f[1] - s * dy / r; f[2] = f[2] - s * dz / r;
    }
    T scale = attr[cls[ki]][cls[kj]] + acid_scale(ki, kj, qi, qj);
    if (scale > T(0)) {
      T s = scale * attr_dv(r);
      f[0] = f[0] - s * dx / r; f[1] = f[1] - s * dy / r; f[2] = f[2] - s * dz / r;
    }
    if (r < es_split) {
      T qq = qi * qj;
      if (qq != T(0)) {
        T m = es_mag(r, qq);
        f[0] = f[0] + m * dx / r; f[1] = f[1] + m * dy / r; f[2] = f[2] + m * dz / r;
      }
    }
  }
  // soup/wgsl/electrostatics.wgsl:87-90 esForceFar
  void es_far(const T* xi, const T* xj, T qi, T qj, T* f) const {
    T dx = mi(xi[0] - xj[0], 0), dy = mi(xi[1] - xj[1], 1), dz = mi(xi[2] - xj[2], 2);
    T r = len3(dx, dy, dz);
    if (r < es_split) return;
    T qq = qi * qj;
    if (qq == T(0)) return;
    T m = es_mag(r, qq);
    f[0] = f[0] + m * dx / r; f[1] = f[1] + m * dy / r; f[2] = f[2] + m * dz / r;
  }
  // a FENE or bend term between xi and xo (soup/wgsl/step.wgsl:152-193 bondedForce)
  void bonded_term(const T* xi, const T* xo, bool fene, T* f) const {
    T dx = mi(xi[0] - xo[0], 0), dy = mi(xi[1] - xo[1], 1), dz = mi(xi[2] - xo[2], 2);
    T r = std::max(len3(dx, dy, dz), T(1e-6));
    T s = fene ? fene_dv(r) : bend_dv(r);
    f[0] = f[0] - s * dx / r; f[1] = f[1] - s * dy / r; f[2] = f[2] - s * dz / r;
  }
};

// ------------------------------------------------------------------------------------------------
// The system
// ------------------------------------------------------------------------------------------------
enum Field {
  F_POS = 0, F_VEL, F_FORCE, F_SLOTS, F_CENTER, F_HELD, F_CHARGES, F_BOND_RNG, F_THERMO_RNG,
  F_FROZEN, F_EVENTS, F_DESORB, F_POS_REF, F_PROT_RNG, F_FIELD_COUNT
};

struct System {
  SoupConfig cfg;
  U32f u;
  uint32_t n = 0;
  std::vector<float> pos, vel, force, pos_ref, charge;
  std::vector<uint32_t> slots, center, held, bond_rng, thermo_rng, frozen;
  std::vector<uint32_t> events, desorb;
  uint32_t prot_rng = 0;
  uint64_t step = 0;
  uint64_t next_sweep = UINT64_MAX;
  // lists (sorted sets, CSR)
  std::vector<uint64_t> vl_off;
  std::vector<uint32_t> vl;
  std::vector<uint32_t> heads;            // titratable particles, index order
  std::vector<uint64_t> es_off;
  std::vector<uint32_t> es;               // per head, neighbour particle indices
  uint32_t list_overflow = 0, es_overflow = 0;
  float max_drift_sq = 0.f;
  uint64_t rebuilds = 0, sweeps = 0;
  SoupSweepResult last_sweep{};
};

// soup/src/soup-confine.ts sphereLatticeSites
std::vector<double> sphere_lattice_sites(uint32_t n, double radius, const double c[3], double* spacing) {
  std::vector<double> out;
  if (n == 0) { *spacing = radius; return out; }
  int nx = std::max(2, (int)std::ceil(std::cbrt(n / (M_PI / 6))));
  for (;;) {
    double h = (2 * radius) / nx;
    out.clear();
    double r2 = radius * radius;
    for (int iz = 0; iz < nx; ++iz) {
      double z = -radius + (iz + 0.5) * h;
      for (int iy = 0; iy < nx; ++iy) {
        double y = -radius + (iy + 0.5) * h;
        for (int ix = 0; ix < nx; ++ix) {
          double x = -radius + (ix + 0.5) * h;
          if (x * x + y * y + z * z <= r2) { out.push_back(c[0] + x); out.push_back(c[1] + y); out.push_back(c[2] + z); }
        }
      }
    }
    if (out.size() / 3 >= n) { *spacing = h; return out; }
    ++nx;
  }
}

// soup/src/soup-init-state.ts:58-307 buildInitialState (no clay, no frozen bulk catalysts): the
// jittered lattice shuffled by Fisher-Yates, Maxwell-Boltzmann velocities, per-particle seeds.
void fresh_state(const SoupConfig& c, float* pos, float* vel, uint32_t* frozen, uint32_t* brng, uint32_t* trng) {
  const uint32_t N = c.n;
  Mulberry32 rng(c.seed);
  std::vector<double> parcel;
  double pspacing = 0;
  double box[3] = {c.box[0], c.box[1], c.box[2]};
  if (c.wall_radius > 0) {
    double centre[3] = {box[0] * 0.5, box[1] * 0.5, box[2] * 0.5};
    parcel = sphere_lattice_sites(N, c.wall_radius, centre, &pspacing);
  }
  uint32_t nx = std::max<uint32_t>(1, (uint32_t)std::ceil(std::cbrt((double)N)));
  while ((uint64_t)nx * nx * nx < N) ++nx;
  double sp[3];
  if (!parcel.empty()) { sp[0] = sp[1] = sp[2] = pspacing; }
  else { for (int a = 0; a < 3; ++a) sp[a] = box[a] / nx; }
  const double jitter = 0.15;
  uint64_t nsites = !parcel.empty() ? parcel.size() / 3 : (uint64_t)nx * nx * nx;
  std::vector<uint32_t> order(nsites);
  for (uint64_t i = 0; i < nsites; ++i) order[i] = (uint32_t)i;
  for (uint64_t i = nsites - 1; i > 0; --i) {
    uint64_t j = (uint64_t)std::floor(rng() * (double)(i + 1));
    std::swap(order[i], order[j]);
  }
  uint32_t idx = 0;
  for (uint32_t kind = 0; kind < c.n_kinds; ++kind) {
    for (uint32_t k = 0; k < c.counts[kind]; ++k) {
      uint32_t site = order[idx];
      double bx, by, bz;
      if (!parcel.empty()) { bx = parcel[site * 3 + 0]; by = parcel[site * 3 + 1]; bz = parcel[site * 3 + 2]; }
      else {
        uint32_t ix = site % nx, iy = (site / nx) % nx, iz = site / (nx * nx);
        bx = (ix + 0.5) * sp[0]; by = (iy + 0.5) * sp[1]; bz = (iz + 0.5) * sp[2];
      }
      double px = bx + (rng() * 2 - 1) * jitter * sp[0];
      double py = by + (rng() * 2 - 1) * jitter * sp[1];
      double pz = bz + (rng() * 2 - 1) * jitter * sp[2];
      if (pos) { pos[idx * 4 + 0] = (float)px; pos[idx * 4 + 1] = (float)py; pos[idx * 4 + 2] = (float)pz; pos[idx * 4 + 3] = (float)kind; }
      double s = std::sqrt(c.kT);
      double g[3];
      for (int a = 0; a < 3; ++a) {   // soup/src/soup-init-state.ts:27-31 gaussian
        double u1 = std::max(rng(), 1e-9);
        double u2 = rng();
        g[a] = s * (std::sqrt(-2 * std::log(u1)) * std::cos(2 * M_PI * u2));
      }
      if (vel) { vel[idx * 4 + 0] = (float)g[0]; vel[idx * 4 + 1] = (float)g[1]; vel[idx * 4 + 2] = (float)g[2]; vel[idx * 4 + 3] = 0.f; }
      if (frozen) frozen[idx] = 0;
      ++idx;
    }
  }
  for (uint32_t i = 0; i < N; ++i) {  // soup/src/soup-init-state.ts:269-272
    if (brng) brng[i] = c.seed ^ ((i + 1u) * 2654435761u) ^ 0x9e3779b9u;
    if (trng) trng[i] = c.seed ^ ((i + 1u) * 3266489917u) ^ 0x85ebca6bu;
  }
}

// soup/src/soup-protonation.ts:38-49 initialCharges
void initial_charges(const SoupConfig& c, const float* pos, float* charges, uint32_t* prot_rng) {
  uint32_t s = c.seed ^ 0x9e3779b9u;
  for (uint32_t i = 0; i < c.n; ++i) charges[i] = 0.f;
  if (c.es_enabled) {
    double alpha = 1.0 / (1.0 + std::pow(10.0, c.pka_intrinsic - c.ph));
    for (uint32_t i = 0; i < c.n; ++i) {
      if ((int)pos[i * 4 + 3] != c.charged_kind) continue;
      if (pcg_next(s) < alpha) charges[i] = (float)c.charge_deprotonated;
    }
  }
  if (prot_rng) *prot_rng = s;
}

// engine/wgsl/neighbor.wgsl:19-24 cell_of / engine/wgsl/forces.wgsl:215-219 cell_coord (f32)
inline void cell_coord(const U32f& u, const float* p, const int dims[3], int out[3]) {
  for (int a = 0; a < 3; ++a) {
    float f = std::floor((p[a] / u.box[a]) * (float)dims[a]);
    int ci = (int)std::max(f, -1.0f);
    out[a] = std::min(std::max(ci, 0), dims[a] - 1);
  }
}

// The cells a +-R walk visits along each axis, wrapped, duplicates dropped in first-visit order.
// Cell tuples are products of per-axis coordinates, so this is the reference's walk with its
// dedupe (soup/src/electrostatics.ts:363-377) and, when dims >= 2R+1, exactly its plain walk.
inline void distinct_axis(const int q[3], const int dims[3], int R, int out[3][64], int n[3]) {
  for (int a = 0; a < 3; ++a) {
    n[a] = 0;
    for (int d = -R; d <= R; ++d) {
      int c = ((q[a] + d) % dims[a] + dims[a]) % dims[a];
      bool dup = false;
      for (int t = 0; t < n[a]; ++t) dup |= out[a][t] == c;
      if (!dup) out[a][n[a]++] = c;
    }
  }
}

// soup/wgsl/verlet.wgsl:53-92 soup_build_verlet_list_main over the reference grid, as a sorted set.
void build_lists(System& s) {
  const SoupConfig& c = s.cfg;
  const U32f& u = s.u;
  Phys<float> ph = Phys<float>::from_f32(u);
  const uint32_t N = s.n;
  double cell = c.interaction_range;  // cellDivisor = 1 in data/soup.json; any complete walk gives the same set
  int dims[3];
  for (int a = 0; a < 3; ++a) dims[a] = std::max(1, (int)std::floor(c.box[a] / cell));
  int R = (int)std::ceil(c.list_range / cell);
  uint64_t ncell = (uint64_t)dims[0] * dims[1] * dims[2];
  std::vector<uint32_t> cstart(ncell + 1, 0), cidx(N);
  std::vector<int> cc(N);
  for (uint32_t i = 0; i < N; ++i) {
    int q[3];
    cell_coord(u, &s.pos[i * 4], dims, q);
    cc[i] = q[0] + dims[0] * (q[1] + dims[1] * q[2]);
    cstart[cc[i] + 1]++;
  }
  for (uint64_t k = 0; k < ncell; ++k) cstart[k + 1] += cstart[k];
  {
    std::vector<uint32_t> cur(cstart.begin(), cstart.end() - 1);
    for (uint32_t i = 0; i < N; ++i) cidx[cur[cc[i]]++] = i;
  }
  // the walk visits each distinct cell once when dims >= 2R+1 (soup/src/soup-plan.ts:99-100); for
  // smaller grids the set semantics still hold because duplicates are removed below.
  const float lr = u.list_range;
  std::vector<uint32_t> counts(N, 0);
  std::vector<std::vector<uint32_t>> rows(N);
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t ii = 0; ii < (int64_t)N; ++ii) {
    uint32_t i = (uint32_t)ii;
    const float* xi = &s.pos[i * 4];
    int q[3];
    cell_coord(u, xi, dims, q);
    std::vector<uint32_t>& row = rows[i];
    row.clear();
    int ax[3][64], na[3];
    distinct_axis(q, dims, R, ax, na);
    for (int iz = 0; iz < na[2]; ++iz) {
      int cz = ax[2][iz];
      for (int iy = 0; iy < na[1]; ++iy) {
        int cy = ax[1][iy];
        for (int ix = 0; ix < na[0]; ++ix) {
          int cx = ax[0][ix];
          uint64_t nc = (uint64_t)cx + (uint64_t)dims[0] * ((uint64_t)cy + (uint64_t)dims[1] * cz);
          for (uint32_t k = cstart[nc]; k < cstart[nc + 1]; ++k) {
            uint32_t j = cidx[k];
            if (j == i) continue;
            const float* xj = &s.pos[j * 4];
            float dx_ = ph.mi(xi[0] - xj[0], 0), dy_ = ph.mi(xi[1] - xj[1], 1), dz_ = ph.mi(xi[2] - xj[2], 2);
            if (Phys<float>::len3(dx_, dy_, dz_) < lr) row.push_back(j);
          }
        }
      }
    }
    std::sort(row.begin(), row.end());
    counts[i] = (uint32_t)row.size();
  }
  s.vl_off.assign(N + 1, 0);
  for (uint32_t i = 0; i < N; ++i) s.vl_off[i + 1] = s.vl_off[i] + counts[i];
  s.vl.resize(s.vl_off[N]);
  s.list_overflow = 0;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)N; ++i) {
    std::copy(rows[i].begin(), rows[i].end(), s.vl.begin() + s.vl_off[i]);
  }
  for (uint32_t i = 0; i < N; ++i) if (counts[i] > c.list_capacity) s.list_overflow = 1;

  // soup/wgsl/electrostatics-long.wgsl:15-56: head compaction in index order, head list at rc_es+skin
  s.heads.clear();
  s.es_off.assign(1, 0);
  s.es.clear();
  s.es_overflow = 0;
  if (c.es_enabled && c.charged_kind >= 0) {
    for (uint32_t i = 0; i < N; ++i) if (s.pos[i * 4 + 3] == u.es_kind) s.heads.push_back(i);
    const uint32_t H = (uint32_t)s.heads.size();
    std::vector<std::vector<uint32_t>> erow(H);
    const float elr = u.es_list_range;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t hh = 0; hh < (int64_t)H; ++hh) {
      uint32_t i = s.heads[hh];
      const float* xi = &s.pos[i * 4];
      for (uint32_t g = 0; g < H; ++g) {
        uint32_t j = s.heads[g];
        if (j == i) continue;
        const float* xj = &s.pos[j * 4];
        float dx_ = ph.mi(xi[0] - xj[0], 0), dy_ = ph.mi(xi[1] - xj[1], 1), dz_ = ph.mi(xi[2] - xj[2], 2);
        if (Phys<float>::len3(dx_, dy_, dz_) < elr) erow[hh].push_back(j);
      }
    }
    s.es_off.assign(H + 1, 0);
    for (uint32_t h = 0; h < H; ++h) {
      s.es_off[h + 1] = s.es_off[h] + erow[h].size();
      if (erow[h].size() > c.es_list_capacity) s.es_overflow = 1;
    }
    s.es.resize(s.es_off[H]);
    for (uint32_t h = 0; h < H; ++h) std::copy(erow[h].begin(), erow[h].end(), s.es.begin() + s.es_off[h]);
  }
  // soup_snapshot_positions_main / soup_reset_max_drift_main (soup/wgsl/verlet.wgsl:94-111)
  s.pos_ref = s.pos;
  s.max_drift_sq = 0.f;
  s.rebuilds++;
}

// soup/wgsl/step.wgsl:152-193 bondedForce
template <class T>
void bonded_force(const System& s, const Phys<T>& ph, uint32_t i, const T* xi, T* f) {
  auto P = [&](uint32_t j, T* x) { for (int a = 0; a < 3; ++a) x[a] = (T)s.pos[j * 4 + a]; };
  T xo[3];
  for (int k = 0; k < 3; ++k) {
    uint32_t p = s.slots[i * 3 + k];
    if (p == NONE) continue;
    P(p, xo); ph.bonded_term(xi, xo, true, f);
  }
  for (int k = 0; k < 3; ++k) {
    uint32_t m = s.slots[i * 3 + k];
    if (m == NONE) continue;
    for (int t = 0; t < 3; ++t) {
      uint32_t o = s.slots[m * 3 + t];
      if (o == NONE || o == i) continue;
      P(o, xo); ph.bonded_term(xi, xo, false, f);
    }
  }
  uint32_t owner = s.center[i];
  if (owner != NONE) { P(owner, xo); ph.bonded_term(xi, xo, true, f); }
}

// soup/wgsl/wall.wgsl:42-56 soup_wall_force_main
template <class T>
void wall_force(const System& s, T wr, T wk, const T* box, const T* xi, T* f) {
  if (!(wr > T(0))) return;
  T d[3] = {xi[0] - box[0] * T(0.5), xi[1] - box[1] * T(0.5), xi[2] - box[2] * T(0.5)};
  T r = Phys<T>::len3(d[0], d[1], d[2]);
  if (r <= wr) return;
  T k = (-wk * (r - wr) / std::max(r, T(1e-6)));
  for (int a = 0; a < 3; ++a) f[a] = f[a] + k * d[a];
}

// encodeSoupForceList (soup/src/soup-integrate.ts:64-71): soup_force_list_main (verlet.wgsl:132-149)
// over the sorted list, then soup_es_force_far_main (electrostatics-long.wgsl:63-82), then the wall.
// T=float writes s.force; T=double writes out64 (the FP64 reference on the same lists).
template <class T>
void list_force(System& s, double* out64) {
  const uint32_t N = s.n;
  Phys<T> ph = std::is_same<T, float>::value ? Phys<T>::from_f32(s.u) : Phys<T>::from_f64(s.cfg);
  T wr = std::is_same<T, float>::value ? (T)s.u.wall_r : (T)s.cfg.wall_radius;
  T wk = std::is_same<T, float>::value ? (T)s.u.wall_k : (T)s.cfg.wall_k;
  std::vector<T> F((size_t)N * 3, T(0));
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t ii = 0; ii < (int64_t)N; ++ii) {
    uint32_t i = (uint32_t)ii;
    T xi[3] = {(T)s.pos[i * 4], (T)s.pos[i * 4 + 1], (T)s.pos[i * 4 + 2]};
    int ki = (int)s.pos[i * 4 + 3];
    T qi = (T)s.charge[i];
    T f[3] = {0, 0, 0};
    bonded_force<T>(s, ph, i, xi, f);
    for (uint64_t e = s.vl_off[i]; e < s.vl_off[i + 1]; ++e) {
      uint32_t j = s.vl[e];
      T xj[3] = {(T)s.pos[j * 4], (T)s.pos[j * 4 + 1], (T)s.pos[j * 4 + 2]};
      ph.nonbonded(xi, xj, ki, (int)s.pos[j * 4 + 3], qi, (T)s.charge[j], f);
    }
    for (int a = 0; a < 3; ++a) F[i * 3 + a] = f[a];
  }
  const uint32_t H = (uint32_t)s.heads.size();
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t hh = 0; hh < (int64_t)H; ++hh) {
    uint32_t i = s.heads[hh];
    T qi = (T)s.charge[i];
    if (qi == T(0)) continue;
    T xi[3] = {(T)s.pos[i * 4], (T)s.pos[i * 4 + 1], (T)s.pos[i * 4 + 2]};
    T f[3] = {0, 0, 0};
    for (uint64_t e = s.es_off[hh]; e < s.es_off[hh + 1]; ++e) {
      uint32_t j = s.es[e];
      T xj[3] = {(T)s.pos[j * 4], (T)s.pos[j * 4 + 1], (T)s.pos[j * 4 + 2]};
      ph.es_far(xi, xj, qi, (T)s.charge[j], f);
    }
    for (int a = 0; a < 3; ++a) F[i * 3 + a] = F[i * 3 + a] + f[a];
  }
  for (uint32_t i = 0; i < N; ++i) {
    T xi[3] = {(T)s.pos[i * 4], (T)s.pos[i * 4 + 1], (T)s.pos[i * 4 + 2]};
    T f[3] = {F[i * 3], F[i * 3 + 1], F[i * 3 + 2]};
    wall_force<T>(s, wr, wk, ph.box, xi, f);
    if (out64) { for (int a = 0; a < 3; ++a) out64[i * 4 + a] = (double)f[a]; out64[i * 4 + 3] = 0; }
    else { for (int a = 0; a < 3; ++a) s.force[i * 4 + a] = (float)f[a]; s.force[i * 4 + 3] = 0.f; }
  }
}

// soup/wgsl/step.wgsl:277-292 soup_force_brute_main + electrostatics-long.wgsl:88-103 + wall
template <class T>
void brute_force(System& s, T* out) {
  const uint32_t N = s.n;
  Phys<T> ph = std::is_same<T, float>::value ? Phys<T>::from_f32(s.u) : Phys<T>::from_f64(s.cfg);
  T wr = std::is_same<T, float>::value ? (T)s.u.wall_r : (T)s.cfg.wall_radius;
  T wk = std::is_same<T, float>::value ? (T)s.u.wall_k : (T)s.cfg.wall_k;
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t ii = 0; ii < (int64_t)N; ++ii) {
    uint32_t i = (uint32_t)ii;
    T xi[3] = {(T)s.pos[i * 4], (T)s.pos[i * 4 + 1], (T)s.pos[i * 4 + 2]};
    int ki = (int)s.pos[i * 4 + 3];
    T qi = (T)s.charge[i];
    T f[3] = {0, 0, 0};
    bonded_force<T>(s, ph, i, xi, f);
    for (uint32_t j = 0; j < N; ++j) {
      if (j == i) continue;
      T xj[3] = {(T)s.pos[j * 4], (T)s.pos[j * 4 + 1], (T)s.pos[j * 4 + 2]};
      ph.nonbonded(xi, xj, ki, (int)s.pos[j * 4 + 3], qi, (T)s.charge[j], f);
    }
    if (qi != T(0) && s.cfg.es_enabled) {
      T g[3] = {0, 0, 0};
      for (uint32_t j = 0; j < N; ++j) {
        if (j == i) continue;
        T xj[3] = {(T)s.pos[j * 4], (T)s.pos[j * 4 + 1], (T)s.pos[j * 4 + 2]};
        ph.es_far(xi, xj, qi, (T)s.charge[j], g);
      }
      for (int a = 0; a < 3; ++a) f[a] = f[a] + g[a];
    }
    wall_force<T>(s, wr, wk, ph.box, xi, f);
    for (int a = 0; a < 3; ++a) out[i * 4 + a] = f[a];
    out[i * 4 + 3] = T(0);
  }
}

// soup/wgsl/step.wgsl:96-108 kick_drift_wrap_main (f32)
void kick_drift(System& s) {
  const U32f& u = s.u;
  const float hdt = 0.5f * u.dt;
  for (uint32_t i = 0; i < s.n; ++i) {
    float* v = &s.vel[i * 4];
    float* x = &s.pos[i * 4];
    if (s.frozen[i] != 0) { v[0] = v[1] = v[2] = v[3] = 0.f; continue; }
    for (int a = 0; a < 3; ++a) v[a] = v[a] + hdt * s.force[i * 4 + a];
    v[3] = 0.f;
    for (int a = 0; a < 3; ++a) {
      float y = x[a] + u.dt * v[a];
      x[a] = y - std::floor(y / u.box[a]) * u.box[a];
    }
  }
}

// soup/wgsl/step.wgsl:110-142 kick_thermostat_main (f32; logf/cosf/sqrtf from the C library)
void kick_thermostat(System& s) {
  const U32f& u = s.u;
  const float hdt = 0.5f * u.dt;
  const float sigma_v = std::sqrt(2.0f * u.gamma * u.kT * u.dt);
  const float gdt = u.gamma * u.dt;
  for (uint32_t i = 0; i < s.n; ++i) {
    float* v = &s.vel[i * 4];
    if (s.frozen[i] != 0) { v[0] = v[1] = v[2] = v[3] = 0.f; continue; }
    float w[3];
    for (int a = 0; a < 3; ++a) w[a] = v[a] + hdt * s.force[i * 4 + a];
    uint32_t st = s.thermo_rng[i];
    float noise[3];
    for (int a = 0; a < 3; ++a) {
      st = pcg_hash(st);
      float u1 = std::max(u01f(st), 1e-7f);
      st = pcg_hash(st);
      float u2 = u01f(st);
      noise[a] = std::sqrt(-2.0f * std::log(u1)) * std::cos(6.28318531f * u2);
    }
    s.thermo_rng[i] = st;
    for (int a = 0; a < 3; ++a) v[a] = (w[a] - gdt * w[a]) + sigma_v * noise[a];
    v[3] = 0.f;
  }
}

// soup/wgsl/verlet.wgsl:113-122 soup_max_drift_main: atomicMax over the u32 bits of drift^2
// (monotone for non-negative floats; a NaN's bits exceed every finite value's, so NaN wins).
void max_drift(System& s) {
  Phys<float> ph = Phys<float>::from_f32(s.u);
  uint32_t m;
  std::memcpy(&m, &s.max_drift_sq, 4);
  for (uint32_t i = 0; i < s.n; ++i) {
    float d[3];
    for (int a = 0; a < 3; ++a) d[a] = ph.mi(s.pos[i * 4 + a] - s.pos_ref[i * 4 + a], a);
    float q = (d[0] * d[0] + d[1] * d[1]) + d[2] * d[2];
    uint32_t b;
    std::memcpy(&b, &q, 4);
    m = std::max(m, b);
  }
  std::memcpy(&s.max_drift_sq, &m, 4);
}

// soup/wgsl/health.wgsl:52-68 soup_scan_nonfinite_main
void nonfinite(const System& s, uint32_t out[2]) {
  auto bad = [](float x) { uint32_t b; std::memcpy(&b, &x, 4); return ((b >> 23) & 0xFFu) == 0xFFu; };
  out[0] = out[1] = 0;
  for (uint32_t i = 0; i < s.n; ++i)
    for (int a = 0; a < 3; ++a) { out[0] += bad(s.pos[i * 4 + a]); out[1] += bad(s.vel[i * 4 + a]); }
}

// ------------------------------------------------------------------------------------------------
// Bond Monte Carlo, canonical serial semantics (soup/wgsl/bond-*.wgsl)
// ------------------------------------------------------------------------------------------------
struct Bonds {
  System& s;
  const U32f& u;
  Phys<float> ph;
  explicit Bonds(System& sys) : s(sys), u(sys.u), ph(Phys<float>::from_f32(sys.u)) {}

  float kind(uint32_t i) const { return s.pos[i * 4 + 3]; }
  float dist(uint32_t a, uint32_t b) const {
    const float* xa = &s.pos[a * 4];
    const float* xb = &s.pos[b * 4];
    return Phys<float>::len3(ph.mi(xa[0] - xb[0], 0), ph.mi(xa[1] - xb[1], 1), ph.mi(xa[2] - xb[2], 2));
  }
  // soup/wgsl/bond-common.wgsl:123 bPairB
  float pairB(float ti, float tj) const { return (u.sigma * (u.radius[(int)ti] + u.radius[(int)tj])) * 0.5f; }
  float wcut(float b) const { return u.c6 * b; }
  // bond-common.wgsl:142-149 matchRule
  int match_rule(float ti, float tj) const {
    for (uint32_t r = 0; r < 2u; ++r) {   // BOND_RULES = 2 (bond-common.wgsl:41)
      float a = u.kindA[r], b = u.kindB[r];
      if ((ti == a && tj == b) || (ti == b && tj == a)) return (int)r;
    }
    return -1;
  }
  uint32_t role_of(uint32_t r, float k) const { return (k == u.kindA[r]) ? (uint32_t)u.roleA[r] : (uint32_t)u.roleB[r]; }
  bool has_bond_to(uint32_t i, uint32_t j) const {
    for (int k = 0; k < 3; ++k) if (s.slots[i * 3 + k] == j) return true;
    return false;
  }
  bool cas_center(uint32_t p, uint32_t expect, uint32_t v) {
    if (s.center[p] != expect) return false;
    s.center[p] = v;
    return true;
  }
  // bond-valence.wgsl:40-98 tryClaimSlot
  int try_claim(uint32_t p, uint32_t role, uint32_t partner) {
    uint32_t* sl = &s.slots[p * 3];
    bool term = u.head_terminal > 0.5f;
    if (role == 0) {
      if (sl[0] == NONE) {
        sl[0] = partner;
        if (term && sl[2] != NONE) { sl[0] = NONE; return -1; }
        return 0;
      }
      if (sl[1] == NONE) {
        sl[1] = partner;
        if (term && sl[2] != NONE) { sl[1] = NONE; return -1; }
        return 1;
      }
      return -1;
    } else if (role == 1) {
      if (sl[2] == NONE) {
        sl[2] = partner;
        if (term && sl[0] != NONE && sl[1] != NONE) { sl[2] = NONE; return -1; }
        return 2;
      }
      return -1;
    }
    uint32_t cap = (uint32_t)u.head_cap;
    for (uint32_t k = 0; k < cap; ++k) {
      if (sl[k] == NONE) { sl[k] = partner; return (int)k; }
    }
    return -1;
  }
  void release(uint32_t p, int slot) { if (slot >= 0) s.slots[p * 3 + slot] = NONE; }
  // bond-adsorption.wgsl:74-77 centerWithinReach
  bool within_reach(uint32_t a, uint32_t b) const {
    return dist(a, b) < wcut(pairB(kind(a), u.cat_kind)) + u.wc;
  }
  // bond-adsorption.wgsl:87-248 propagateOnCenter
  bool propagate(uint32_t i, uint32_t j, int slotI, int slotJ, uint32_t cat) {
    if (slotI == 0 && slotJ == 0) {
      if (cat == NONE) return false;
      if (dist(i, cat) >= wcut(pairB(kind(i), u.cat_kind))) return false;
      if (!cas_center(cat, NONE, i)) return false;
      if (!cas_center(i, NONE, cat)) { cas_center(cat, i, NONE); return false; }
      s.held[cat] = 0;
      return true;
    }
    uint32_t tipOld, tipNew;
    if (slotI == 1 && slotJ == 0) { tipOld = i; tipNew = j; }
    else if (slotI == 0 && slotJ == 1) { tipOld = j; tipNew = i; }
    else return false;
    uint32_t owner = s.center[tipOld];
    bool reclaim = false;
    if (owner == NONE) {
      if (cat == NONE) return false;
      owner = cat;
      reclaim = true;
    }
    if (reclaim) {
      if (dist(tipOld, cat) >= wcut(pairB(kind(tipOld), u.cat_kind))) return false;
    } else {
      if (!within_reach(tipOld, owner)) return false;
    }
    if (dist(tipNew, owner) >= wcut(pairB(kind(tipNew), u.cat_kind))) return false;
    if (reclaim) {
      if (!cas_center(owner, NONE, tipOld)) return false;
      if (!cas_center(tipOld, NONE, owner)) { cas_center(owner, tipOld, NONE); return false; }
    }
    if (!cas_center(owner, tipOld, tipNew)) {
      if (reclaim) cas_center(tipOld, owner, NONE);
      return false;
    }
    if (!cas_center(tipNew, NONE, owner)) {
      cas_center(owner, tipNew, tipOld);
      if (reclaim) { cas_center(owner, tipOld, NONE); cas_center(tipOld, owner, NONE); }
      return false;
    }
    cas_center(tipOld, owner, NONE);
    s.held[owner] = 0;
    return true;
  }
  // bond-adsorption.wgsl:256-268 terminateOnCenter
  bool terminate(uint32_t carbon) {
    uint32_t owner = s.center[carbon];
    if (owner == NONE) return false;
    if (!within_reach(carbon, owner)) return false;
    if (!cas_center(carbon, owner, NONE)) return false;
    cas_center(owner, carbon, NONE);
    s.held[owner] = 0;
    return true;
  }
  // bond-adsorption.wgsl:283-292 desorbStretch
  void desorb_stretch(uint32_t carbon, uint32_t owner) {
    if (dist(carbon, owner) >= u.r_inf) {
      if (cas_center(carbon, owner, NONE)) {
        cas_center(owner, carbon, NONE);
        s.held[owner] = 0;
        s.desorb[0]++;
      }
    }
  }
  // bond-adsorption.wgsl:304-316 desorbTimeout
  void desorb_timeout(uint32_t cat) {
    uint32_t tip = s.center[cat];
    if (tip == NONE) return;
    uint32_t inc = (uint32_t)u.interval;
    uint32_t prev = s.held[cat];
    s.held[cat] = prev + inc;
    if (prev + inc > (uint32_t)u.max_hold) {
      if (cas_center(cat, tip, NONE)) {
        cas_center(tip, cat, NONE);
        s.held[cat] = 0;
        s.desorb[1]++;
      }
    }
  }

  // bond-verlet.wgsl:44-54 bond_form_list_main + bond-dispatch.wgsl:89-142 bondFormDecide,
  // run for i = 0..N-1 in order.
  void form_pass() {
    for (uint32_t i = 0; i < s.n; ++i) {
      float ti = kind(i);
      uint32_t catNear = 0, catId = NONE, nCand = 0;
      uint32_t candJ[CANDIDATE_CAP], candR[CANDIDATE_CAP];
      for (uint64_t e = s.vl_off[i]; e < s.vl_off[i + 1]; ++e) {
        uint32_t j = s.vl[e];
        float tj = kind(j);
        if (catNear == 0 && tj == u.cat_kind) {
          if (dist(i, j) < wcut(pairB(ti, u.cat_kind))) { catNear = 1; catId = j; }
        }
        if (j > i && nCand < CANDIDATE_CAP) {
          int r = match_rule(ti, tj);
          if (r >= 0 && !has_bond_to(i, j)) {
            if (dist(i, j) < wcut(pairB(ti, tj))) { candJ[nCand] = j; candR[nCand] = (uint32_t)r; ++nCand; }
          }
        }
      }
      uint32_t rng = s.bond_rng[i];
      if (ti == u.cat_kind) desorb_timeout(i);
      else {
        uint32_t owner = s.center[i];
        if (owner != NONE) desorb_stretch(i, owner);
      }
      for (uint32_t ci = 0; ci < nCand; ++ci) {
        uint32_t j = candJ[ci], r = candR[ci];
        float tj = kind(j);
        if (u.req_cat[r] > 0.5f && catNear == 0) continue;
        rng = pcg_hash(rng);
        if (u01f(rng) >= u.att_form[r]) continue;
        rng = pcg_hash(rng);
        if (u01f(rng) >= u.acc_form[r]) continue;
        uint32_t roleI = role_of(r, ti), roleJ = role_of(r, tj);
        int slotI = try_claim(i, roleI, j);
        if (slotI < 0) continue;
        int slotJ = try_claim(j, roleJ, i);
        if (slotJ < 0) { release(i, slotI); continue; }
        bool ok;
        if (roleI == 0 && roleJ == 0) ok = propagate(i, j, slotI, slotJ, catId);
        else if (roleI == 1) ok = terminate(i);
        else ok = terminate(j);
        if (!ok) { release(i, slotI); release(j, slotJ); continue; }
        s.events[r * 2 + 0]++;
      }
      s.bond_rng[i] = rng;
    }
  }
  // bond-dispatch.wgsl:170-200 bond_break_main
  void break_pass() {
    for (uint32_t i = 0; i < s.n; ++i) {
      float ti = kind(i);
      uint32_t rng = s.bond_rng[i];
      for (int k = 0; k < 3; ++k) {
        uint32_t partner = s.slots[i * 3 + k];
        if (partner == NONE) continue;
        if (partner < i) continue;
        int r = match_rule(ti, kind(partner));
        if (r < 0) continue;
        rng = pcg_hash(rng);
        if (u01f(rng) >= u.att_break[r]) continue;
        rng = pcg_hash(rng);
        if (u01f(rng) >= u.acc_break[r]) continue;
        s.slots[i * 3 + k] = NONE;
        for (int t = 0; t < 3; ++t) {
          if (s.slots[partner * 3 + t] == i) { s.slots[partner * 3 + t] = NONE; break; }
        }
        s.events[r * 2 + 1]++;
      }
      s.bond_rng[i] = rng;
    }
  }
};

// ------------------------------------------------------------------------------------------------
// Constant-pH Monte Carlo (soup/src/electrostatics.ts:330-496, soup/src/acid-soap.ts:147-198), FP64
// ------------------------------------------------------------------------------------------------
struct EsHost {
  double A, kappa, rc, shiftU, shiftF, pka, ph, kT, q;
  double acid, rcAttr, wc, eps;
  bool enabled;
};
EsHost es_host(const SoupConfig& c) {
  return EsHost{c.es_coeff_a, c.es_kappa, c.es_cutoff, c.es_shift_u, c.es_shift_f, c.pka_intrinsic, c.ph, c.kT,
                c.charge_deprotonated, c.acid_soap_scale, c.rc_attr, c.wc, c.epsilon, c.es_enabled != 0};
}
// electrostatics.ts:277-281 esPairEnergy
inline double es_pair_energy(double r, double qq, const EsHost& b) {
  if (b.A == 0 || qq == 0 || r >= b.rc || r <= 0) return 0;
  double u1 = (b.A * std::exp(-b.kappa * r)) / r;
  return qq * (u1 - b.shiftU + b.shiftF * (r - b.rc));
}
// acid-soap.ts:155-162 acidSoapWell
inline double acid_soap_well(double r, const EsHost& w) {
  if (w.acid <= 0) return 0;
  if (r < w.rcAttr) return -w.acid * w.eps;
  if (r > w.rcAttr + w.wc) return 0;
  double c = std::cos((M_PI * (r - w.rcAttr)) / (2 * w.wc));
  return -w.acid * w.eps * c * c;
}

SoupSweepResult ph_sweep(const float* positions, float* charges, uint32_t n, const double box[3],
                         int charged_kind, const EsHost& b, uint32_t& rng) {
  std::vector<uint32_t> heads;
  for (uint32_t i = 0; i < n; ++i) if ((int)positions[i * 4 + 3] == charged_kind) heads.push_back(i);
  const uint32_t H = (uint32_t)heads.size();
  // headCells (electrostatics.ts:330-348)
  int nx = std::max(1, (int)std::floor(box[0] / b.rc));
  int ny = std::max(1, (int)std::floor(box[1] / b.rc));
  int nz = std::max(1, (int)std::floor(box[2] / b.rc));
  double wx = box[0] / nx, wy = box[1] / ny, wz = box[2] / nz;
  auto wrapj = [&](double x, double L) { return js_mod(js_mod(x, L) + L, L); };
  auto cell_of = [&](uint32_t i, int& cx, int& cy, int& cz) {
    double x = wrapj(positions[i * 4], box[0]), y = wrapj(positions[i * 4 + 1], box[1]), z = wrapj(positions[i * 4 + 2], box[2]);
    cx = std::min(nx - 1, (int)std::floor(x / wx));
    cy = std::min(ny - 1, (int)std::floor(y / wy));
    cz = std::min(nz - 1, (int)std::floor(z / wz));
  };
  std::vector<std::vector<uint32_t>> buckets((size_t)nx * ny * nz);
  for (uint32_t h = 0; h < H; ++h) {
    int cx, cy, cz; cell_of(heads[h], cx, cy, cz);
    buckets[cx + (size_t)nx * (cy + (size_t)ny * cz)].push_back(heads[h]);
  }
  const int pdims[3] = {nx, ny, nz};
  auto neighbours = [&](uint32_t i, std::vector<uint32_t>& out) {
    out.clear();
    int q[3];
    cell_of(i, q[0], q[1], q[2]);
    int ax[3][64], na[3];
    distinct_axis(q, pdims, 1, ax, na);
    for (int iz = 0; iz < na[2]; ++iz)
      for (int iy = 0; iy < na[1]; ++iy)
        for (int ix = 0; ix < na[0]; ++ix)
          for (uint32_t j : buckets[ax[0][ix] + (size_t)nx * (ax[1][iy] + (size_t)ny * ax[2][iz])]) out.push_back(j);
  };
  auto mi = [](double d, double L) { return d - js_round(d / L) * L; };
  const double dGintr = b.kT * M_LN10 * (b.pka - b.ph);
  const double q = b.q;
  const double cut2 = b.rc * b.rc;
  const double reach = b.rcAttr + b.wc, reach2 = reach * reach;
  uint32_t attempts = 0, accepted = 0, dEsCount = 0;
  double dEsSum = 0;
  std::vector<uint32_t> nb;
  for (uint32_t a = 0; a < H; ++a) {
    uint32_t i = heads[std::min<uint64_t>(H - 1, (uint64_t)std::floor(pcg_next(rng) * H))];
    attempts++;
    double uEs = 0;
    neighbours(i, nb);
    for (uint32_t j : nb) {
      if (j == i || charges[j] == 0.f) continue;
      double dx = mi((double)positions[i * 4] - positions[j * 4], box[0]);
      double dy = mi((double)positions[i * 4 + 1] - positions[j * 4 + 1], box[1]);
      double dz = mi((double)positions[i * 4 + 2] - positions[j * 4 + 2], box[2]);
      double r2 = dx * dx + dy * dy + dz * dz;
      if (r2 >= cut2) continue;
      uEs += es_pair_energy(std::sqrt(r2), q * (double)charges[j], b);
    }
    if (b.acid > 0) {  // acidSoapSiteWork (acid-soap.ts:175-198)
      double uw = 0;
      for (uint32_t j : nb) {
        if (j == i) continue;
        double dx = (double)positions[i * 4] - positions[j * 4];
        double dy = (double)positions[i * 4 + 1] - positions[j * 4 + 1];
        double dz = (double)positions[i * 4 + 2] - positions[j * 4 + 2];
        dx -= js_round(dx / box[0]) * box[0];
        dy -= js_round(dy / box[1]) * box[1];
        dz -= js_round(dz / box[2]) * box[2];
        double r2 = dx * dx + dy * dy + dz * dz;
        if (r2 >= reach2 || r2 <= 0) continue;
        double v = acid_soap_well(std::sqrt(r2), b);
        uw += charges[j] == 0.f ? v : -v;
      }
      uEs += uw;
    }
    bool charged = charges[i] != 0.f;
    double dG = charged ? -(dGintr + uEs) : dGintr + uEs;
    if (dG <= 0 || pcg_next(rng) < std::exp(-dG / b.kT)) {
      charges[i] = charged ? 0.f : (float)q;
      accepted++;
      if (!charged) { dEsSum += uEs / b.kT; dEsCount++; }
    }
  }
  uint32_t dep = 0;
  for (uint32_t h = 0; h < H; ++h) if (charges[heads[h]] != 0.f) dep++;
  SoupSweepResult r{};
  r.attempts = attempts; r.accepted = accepted; r.heads = H; r.deprotonated = dep;
  r.alpha = H > 0 ? (double)dep / H : 0;
  r.d_es_mean_kt = dEsCount > 0 ? dEsSum / dEsCount : 0;
  return r;
}

// ------------------------------------------------------------------------------------------------
// Schedule
// ------------------------------------------------------------------------------------------------
void do_force(System& s) { list_force<float>(s, nullptr); }

int set_err(int code, const std::string& m) { g_err = m; return code; }

int guards(System& s, uint64_t chunk_start) {
  uint32_t nf[2];
  nonfinite(s, nf);
  if (nf[0] || nf[1])
    return set_err(SOUP_E_NONFINITE, "non-finite state at step=" + std::to_string(s.step) + ": positions=" +
                   std::to_string(nf[0]) + ", velocities=" + std::to_string(nf[1]) + " (since step " + std::to_string(chunk_start) + ")");
  if (s.list_overflow) return set_err(SOUP_E_LIST_OVERFLOW, "Verlet list: listCapacity was insufficient");
  if (s.es_overflow) return set_err(SOUP_E_ES_OVERFLOW, "long-range electrostatics list: capacity insufficient");
  double drift = std::sqrt(std::max(0.0, (double)s.max_drift_sq));
  if (!std::isfinite(drift)) return set_err(SOUP_E_NONFINITE, "Verlet list: the measured drift is not a number");
  if (drift > s.cfg.skin / 2 + 1e-6) return set_err(SOUP_E_DRIFT, "Verlet list: the measured drift exceeds skin/2");
  return SOUP_OK;
}

int sweep_now(System& s) {
  EsHost b = es_host(s.cfg);
  s.last_sweep = ph_sweep(s.pos.data(), s.charge.data(), s.n, s.cfg.box, s.cfg.charged_kind, b, s.prot_rng);
  s.sweeps++;
  build_lists(s);
  do_force(s);
  return SOUP_OK;
}

// soup/src/soup-integrate.ts:83-175 (encodeOneIntegrationStep + buildStepper)
int step_n(System& s, uint64_t n) {
  uint64_t done = 0;
  const uint64_t chunkMax = s.cfg.chunk_steps ? s.cfg.chunk_steps : 1000;
  while (done < n) {
    uint64_t chunk = std::min(chunkMax, n - done);
    uint64_t chunk_start = s.step;
    for (uint64_t k = 0; k < chunk; ++k) {
      bool bonds = s.step % s.cfg.bond_interval == 0;
      kick_drift(s);
      bool rebuild;
      if (s.cfg.rebuild_on_drift) {
        Phys<float> ph = Phys<float>::from_f32(s.u);
        float m = 0.f;
        for (uint32_t i = 0; i < s.n; ++i) {
          float d[3];
          for (int a = 0; a < 3; ++a) d[a] = ph.mi(s.pos[i * 4 + a] - s.pos_ref[i * 4 + a], a);
          m = std::max(m, (d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]);
        }
        float half = (float)(s.cfg.skin * 0.5);
        rebuild = m > half * half;
      } else {
        rebuild = s.step % s.cfg.rebuild_every == 0;
      }
      if (rebuild) build_lists(s);
      do_force(s);
      max_drift(s);
      if (bonds) { Bonds b(s); b.form_pass(); b.break_pass(); }
      kick_thermostat(s);
      s.step++;
    }
    int st = guards(s, chunk_start);
    if (st) return st;
    if (s.cfg.es_enabled && s.step >= s.next_sweep) {
      s.next_sweep = s.step + s.cfg.sweep_every;
      sweep_now(s);
    }
    done += chunk;
  }
  return SOUP_OK;
}

// ------------------------------------------------------------------------------------------------
// Analysis (FP64, JavaScript semantics)
// ------------------------------------------------------------------------------------------------
inline double wrap1(double v, double L) { return v - std::floor(v / L) * L; }
inline double mi1(double d, double L) { return d - js_round(d / L) * L; }

// soup/src/water-closure.ts:63-88 circularAxisStat + periodicCentreOf
int periodic_centre(const float* pos, const uint32_t* idx, uint32_t m, const double box[3], double alpha, double out[3]) {
  if (m == 0) return 0;
  for (int a = 0; a < 3; ++a) {
    double sc = 0, ss = 0;
    for (uint32_t k = 0; k < m; ++k) {
      double th = (2 * M_PI * wrap1(pos[idx[k] * 4 + a], box[a])) / box[a];
      sc += std::cos(th); ss += std::sin(th);
    }
    sc /= m; ss /= m;
    double R = std::sqrt(sc * sc + ss * ss);
    double ang = std::atan2(ss, sc);
    if (!(R >= std::sqrt(-std::log(alpha) / m))) return 0;
    out[a] = wrap1((ang / (2 * M_PI)) * box[a], box[a]);
  }
  return 1;
}

// soup/src/water-closure.ts:109-363 occupancyPeriodic + farthestEmptyCellSeed + floodOutsidePeriodic
// + encapsulatedWaterVolume; with `parcel` (centre x y z, radius) the reached empty cells the bulk
// density is taken over are those whose centre lies in the parcel (water-closure.ts:323-337)
int closure(const float* pos, const uint32_t* mem, uint32_t nm, const uint32_t* wat, uint32_t nw, const double box[3],
            const double centre[3], double cell, double radius, double vmin, SoupClosureResult* res,
            std::vector<uint8_t>* occ_out, std::vector<uint8_t>* vis_out, const double* parcel = nullptr) {
  int nx = std::max(1, (int)std::ceil(box[0] / cell)), ny = std::max(1, (int)std::ceil(box[1] / cell)),
      nz = std::max(1, (int)std::ceil(box[2] / cell));
  size_t NC = (size_t)nx * ny * nz;
  std::vector<uint8_t> occ(NC, 0);
  int reach = std::max(1, (int)std::ceil(radius / cell));
  double r2 = radius * radius;
  for (uint32_t k = 0; k < nm; ++k) {
    uint32_t i = mem[k];
    double px = wrap1(pos[i * 4], box[0]), py = wrap1(pos[i * 4 + 1], box[1]), pz = wrap1(pos[i * 4 + 2], box[2]);
    int cx = (int)std::floor(px / cell), cy = (int)std::floor(py / cell), cz = (int)std::floor(pz / cell);
    for (int dz = -reach; dz <= reach; ++dz) {
      int gz = ((cz + dz) % nz + nz) % nz;
      double ddz = (gz + 0.5) * cell - pz; ddz -= js_round(ddz / box[2]) * box[2];
      for (int dy = -reach; dy <= reach; ++dy) {
        int gy = ((cy + dy) % ny + ny) % ny;
        double ddy = (gy + 0.5) * cell - py; ddy -= js_round(ddy / box[1]) * box[1];
        for (int dx = -reach; dx <= reach; ++dx) {
          int gx = ((cx + dx) % nx + nx) % nx;
          double ddx = (gx + 0.5) * cell - px; ddx -= js_round(ddx / box[0]) * box[0];
          if (ddx * ddx + ddy * ddy + ddz * ddz <= r2) occ[gx + (size_t)nx * (gy + (size_t)ny * gz)] = 1;
        }
      }
    }
  }
  // farthestEmptyCellSeed
  long best = -1; double bestD2 = -1;
  for (int z = 0; z < nz; ++z) for (int y = 0; y < ny; ++y) for (int x = 0; x < nx; ++x) {
    size_t i = x + (size_t)nx * (y + (size_t)ny * z);
    if (occ[i]) continue;
    double dx = mi1((x + 0.5) * cell - centre[0], box[0]);
    double dy = mi1((y + 0.5) * cell - centre[1], box[1]);
    double dz = mi1((z + 0.5) * cell - centre[2], box[2]);
    double d2 = dx * dx + dy * dy + dz * dz;
    if (d2 > bestD2) { bestD2 = d2; best = (long)i; }
  }
  if (best < 0) { g_err = "farthestEmptyCellSeed: the grid is fully occupied"; return SOUP_E_STATE; }
  // floodOutsidePeriodic (BFS; the reached set does not depend on visiting order)
  std::vector<uint8_t> vis(NC, 0);
  std::vector<uint32_t> queue;
  queue.reserve(NC);
  vis[best] = 1; queue.push_back((uint32_t)best);
  for (size_t head = 0; head < queue.size(); ++head) {
    uint32_t i = queue[head];
    int z = (int)(i / ((size_t)nx * ny)); size_t rem = i - (size_t)z * nx * ny; int y = (int)(rem / nx); int x = (int)(rem - (size_t)y * nx);
    int nb[6][3] = {{(x + 1) % nx, y, z}, {(x - 1 + nx) % nx, y, z}, {x, (y + 1) % ny, z}, {x, (y - 1 + ny) % ny, z},
                    {x, y, (z + 1) % nz}, {x, y, (z - 1 + nz) % nz}};
    for (auto& q : nb) {
      size_t ni = q[0] + (size_t)nx * (q[1] + (size_t)ny * q[2]);
      if (!occ[ni] && !vis[ni]) { vis[ni] = 1; queue.push_back((uint32_t)ni); }
    }
  }
  uint32_t totalEmpty = 0, unreached = 0, reachedEmpty = 0;
  for (size_t i = 0; i < NC; ++i) if (!occ[i]) { totalEmpty++; if (!vis[i]) unreached++; }
  for (size_t i = 0; i < NC; ++i) {
    if (!(occ[i] == 0 && vis[i] != 0)) continue;
    if (parcel) {
      const int cz = (int)(i / ((size_t)nx * ny));
      const size_t crem = i - (size_t)cz * nx * ny;
      const int cy = (int)(crem / nx), cx = (int)(crem - (size_t)cy * nx);
      const double ex = (cx + 0.5) * cell - parcel[0], ey = (cy + 0.5) * cell - parcel[1], ez = (cz + 0.5) * cell - parcel[2];
      if (ex * ex + ey * ey + ez * ez > parcel[3] * parcel[3]) continue;
    }
    reachedEmpty++;
  }
  uint32_t enc = 0, reachedWater = 0;
  for (uint32_t k = 0; k < nw; ++k) {
    uint32_t i = wat[k];
    double wx = wrap1(pos[i * 4], box[0]), wy = wrap1(pos[i * 4 + 1], box[1]), wz = wrap1(pos[i * 4 + 2], box[2]);
    int gx = std::min(nx - 1, (int)std::floor(wx / cell)), gy = std::min(ny - 1, (int)std::floor(wy / cell)),
        gz = std::min(nz - 1, (int)std::floor(wz / cell));
    size_t cidx = gx + (size_t)nx * (gy + (size_t)ny * gz);
    if (occ[cidx]) continue;
    if (!vis[cidx]) enc++; else reachedWater++;
  }
  double bulk = reachedEmpty > 0 ? reachedWater / (reachedEmpty * cell * cell * cell) : 0;
  double thr = bulk > 0 ? vmin * bulk : NAN;
  int z = (int)(best / ((long)nx * ny)); long rem = best - (long)z * nx * ny; int y = (int)(rem / nx); int x = (int)(rem - (long)y * nx);
  double ddx = mi1((x + 0.5) * cell - centre[0], box[0]), ddy = mi1((y + 0.5) * cell - centre[1], box[1]),
         ddz = mi1((z + 0.5) * cell - centre[2], box[2]);
  res->encapsulated_count = enc; res->total_water = nw; res->bulk_water_density = bulk; res->threshold_count = thr;
  res->closed = (std::isfinite(thr) && enc > thr) ? 1 : 0;
  res->total_empty_cells = totalEmpty; res->unreached_cells = unreached; res->seed_cell = (uint32_t)best;
  res->seed_dist_from_centre = std::sqrt(ddx * ddx + ddy * ddy + ddz * ddz);
  if (occ_out) *occ_out = std::move(occ);
  if (vis_out) *vis_out = std::move(vis);
  return SOUP_OK;
}

// soup/src/amphiphile.ts:55-141 findAmphiphiles; head_of[i] = head index or NONE
uint32_t amphiphiles(const float* pos, const uint32_t* slots, uint32_t n, const uint32_t* polar_of_kind, uint32_t* head_of) {
  std::vector<std::vector<uint32_t>> adj(n);
  std::vector<uint32_t> parent(n);
  std::iota(parent.begin(), parent.end(), 0u);
  auto find = [&](uint32_t x) { while (parent[x] != x) { parent[x] = parent[parent[x]]; x = parent[x]; } return x; };
  for (uint32_t i = 0; i < n; ++i)    // bonds() (soup-readback.ts:40-50): pairs with j > i
    for (int k = 0; k < 3; ++k) {
      uint32_t j = slots[i * 3 + k];
      if (j != NONE && j > i) {
        adj[i].push_back(j); adj[j].push_back(i);
        uint32_t ra = find(i), rb = find(j);
        if (ra != rb) parent[ra] = rb;
      }
    }
  std::vector<std::vector<uint32_t>> comp(n);
  for (uint32_t i = 0; i < n; ++i) comp[find(i)].push_back(i);
  for (uint32_t i = 0; i < n; ++i) head_of[i] = NONE;
  uint32_t count = 0;
  for (uint32_t r = 0; r < n; ++r) {
    const auto& mem = comp[r];
    if (mem.empty()) continue;
    uint64_t sumDeg = 0; uint32_t polarCount = 0, polarIdx = NONE; bool bad = false;
    for (uint32_t i : mem) {
      size_t deg = adj[i].size();
      sumDeg += deg;
      bool polar = polar_of_kind[(int)std::lround(pos[i * 4 + 3])] != 0;
      if (polar) { polarCount++; polarIdx = i; if (deg < 1 || deg > 2) bad = true; }
      else if (deg > 2) bad = true;
    }
    if (bad || polarCount != 1) continue;
    if (sumDeg / 2 != mem.size() - 1) continue;
    for (uint32_t i : mem) head_of[i] = polarIdx;
    count++;
  }
  return count;
}

// engine/src/aggregate.ts:65-130 buildClusterUnionFind (periodicZ) + clusterComponents; labels are
// the minimum original index of each component.
uint32_t aggregates(const float* pos, const uint32_t* mem, uint32_t m, const double box[3], double cutoff, uint32_t* labels) {
  std::vector<uint32_t> parent(m);
  std::iota(parent.begin(), parent.end(), 0u);
  auto find = [&](uint32_t x) { while (parent[x] != x) { parent[x] = parent[parent[x]]; x = parent[x]; } return x; };
  int nx = std::max(1, (int)std::floor(box[0] / cutoff)), ny = std::max(1, (int)std::floor(box[1] / cutoff)),
      nz = std::max(1, (int)std::floor(box[2] / cutoff));
  double wx = box[0] / nx, wy = box[1] / ny, wz = box[2] / nz;
  std::vector<int> cx(m), cy(m), cz(m);
  std::vector<std::vector<uint32_t>> buckets((size_t)nx * ny * nz);
  for (uint32_t k = 0; k < m; ++k) {
    uint32_t i = mem[k];
    double x = wrap1(pos[i * 4], box[0]), y = wrap1(pos[i * 4 + 1], box[1]), z = wrap1(pos[i * 4 + 2], box[2]);
    cx[k] = std::min(nx - 1, (int)std::floor(x / wx)); cy[k] = std::min(ny - 1, (int)std::floor(y / wy));
    cz[k] = std::min(nz - 1, (int)std::floor(z / wz));
    buckets[cx[k] + (size_t)nx * (cy[k] + (size_t)ny * cz[k])].push_back(k);
  }
  const double c2 = cutoff * cutoff;
  for (uint32_t k = 0; k < m; ++k) {
    uint32_t i = mem[k];
    for (int dx = -1; dx <= 1; ++dx) {
      int ax = ((cx[k] + dx) % nx + nx) % nx;
      for (int dy = -1; dy <= 1; ++dy) {
        int ay = ((cy[k] + dy) % ny + ny) % ny;
        for (int dz = -1; dz <= 1; ++dz) {
          int az = ((cz[k] + dz) % nz + nz) % nz;
          for (uint32_t l : buckets[ax + (size_t)nx * (ay + (size_t)ny * az)]) {
            if (l <= k) continue;
            uint32_t j = mem[l];
            double ddx = mi1((double)pos[i * 4] - pos[j * 4], box[0]);
            double ddy = mi1((double)pos[i * 4 + 1] - pos[j * 4 + 1], box[1]);
            double ddz = mi1((double)pos[i * 4 + 2] - pos[j * 4 + 2], box[2]);
            if (ddx * ddx + ddy * ddy + ddz * ddz <= c2) {
              uint32_t ra = find(k), rb = find(l);
              if (ra != rb) parent[ra] = rb;
            }
          }
        }
      }
    }
  }
  std::vector<uint32_t> minIdx(m, NONE);
  for (uint32_t k = 0; k < m; ++k) { uint32_t r = find(k); minIdx[r] = std::min(minIdx[r], mem[k]); }
  uint32_t ncomp = 0;
  for (uint32_t k = 0; k < m; ++k) { labels[k] = minIdx[find(k)]; if (find(k) == k) ncomp++; }
  return ncomp;
}

// soup/wgsl/relax.wgsl:50-72 soup_relax_step_main
void relax_step(System& s, float d) {
  for (uint32_t i = 0; i < s.n; ++i) {
    if (s.frozen[i] != 0) continue;
    float f[3] = {s.force[i * 4], s.force[i * 4 + 1], s.force[i * 4 + 2]};
    float a = std::max(std::max(std::fabs(f[0]), std::fabs(f[1])), std::fabs(f[2]));
    uint32_t b; std::memcpy(&b, &a, 4);
    if (!(a > 0.f) || ((b >> 23) & 0xFFu) == 0xFFu) continue;
    float g[3] = {f[0] / a, f[1] / a, f[2] / a};
    float L = Phys<float>::len3(g[0], g[1], g[2]);
    for (int k = 0; k < 3; ++k) {
      float y = s.pos[i * 4 + k] + (g[k] / L) * d;
      s.pos[i * 4 + k] = y - std::floor(y / s.u.box[k]) * s.u.box[k];
    }
  }
}

System* create(const SoupConfig* c, const SoupInitState* init) {
  if (!c || c->abi_version != SOUP_ABI_VERSION || c->n == 0) { g_err = "bad config"; return nullptr; }
  System* s = new System();
  s->cfg = *c;
  s->u = make_u32f(*c);
  const uint32_t N = s->n = c->n;
  s->pos.assign((size_t)N * 4, 0.f); s->vel.assign((size_t)N * 4, 0.f); s->force.assign((size_t)N * 4, 0.f);
  s->charge.assign(N, 0.f); s->slots.assign((size_t)N * 3, NONE); s->center.assign(N, NONE);
  s->held.assign(N, 0); s->bond_rng.assign(N, 0); s->thermo_rng.assign(N, 0); s->frozen.assign(N, 0);
  s->events.assign(2 * SOUP_MAX_RULES, 0); s->desorb.assign(2, 0);
  fresh_state(*c, s->pos.data(), s->vel.data(), s->frozen.data(), s->bond_rng.data(), s->thermo_rng.data());
  s->prot_rng = c->protonation_rng;
  bool charges_given = init && init->charges;
  if (init) {
    if (init->positions) std::memcpy(s->pos.data(), init->positions, (size_t)N * 16);
    if (init->velocities) std::memcpy(s->vel.data(), init->velocities, (size_t)N * 16);
    if (init->bond_slots) std::memcpy(s->slots.data(), init->bond_slots, (size_t)N * 12);
    if (init->center_link) std::memcpy(s->center.data(), init->center_link, (size_t)N * 4);
    if (init->center_held) std::memcpy(s->held.data(), init->center_held, (size_t)N * 4);
    if (init->bond_rng) std::memcpy(s->bond_rng.data(), init->bond_rng, (size_t)N * 4);
    if (init->thermo_rng) std::memcpy(s->thermo_rng.data(), init->thermo_rng, (size_t)N * 4);
    if (init->charges) std::memcpy(s->charge.data(), init->charges, (size_t)N * 4);
    if (init->frozen) std::memcpy(s->frozen.data(), init->frozen, (size_t)N * 4);
    if (init->events) std::memcpy(s->events.data(), init->events, (size_t)c->n_rules * 8);
    if (init->desorb_events) std::memcpy(s->desorb.data(), init->desorb_events, 8);
  }
  if (!charges_given) {
    uint32_t pr = 0;
    initial_charges(*c, s->pos.data(), s->charge.data(), &pr);
    if (c->protonation_rng == 0) s->prot_rng = pr;
  }
  s->step = c->global_step;
  s->next_sweep = c->es_enabled ? c->global_step + c->sweep_every : UINT64_MAX;
  build_lists(*s);   // priming pass (soup/src/sim.ts:396-408)
  do_force(*s);
  return s;
}

void* field_ptr(System& s, int f, size_t& bytes) {
  const size_t N = s.n;
  switch (f) {
    case F_POS: bytes = N * 16; return s.pos.data();
    case F_VEL: bytes = N * 16; return s.vel.data();
    case F_FORCE: bytes = N * 16; return s.force.data();
    case F_SLOTS: bytes = N * 12; return s.slots.data();
    case F_CENTER: bytes = N * 4; return s.center.data();
    case F_HELD: bytes = N * 4; return s.held.data();
    case F_CHARGES: bytes = N * 4; return s.charge.data();
    case F_BOND_RNG: bytes = N * 4; return s.bond_rng.data();
    case F_THERMO_RNG: bytes = N * 4; return s.thermo_rng.data();
    case F_FROZEN: bytes = N * 4; return s.frozen.data();
    case F_EVENTS: bytes = (size_t)s.cfg.n_rules * 8; return s.events.data();
    case F_DESORB: bytes = 8; return s.desorb.data();
    case F_POS_REF: bytes = N * 16; return s.pos_ref.data();
    case F_PROT_RNG: bytes = 4; return &s.prot_rng;
  }
  bytes = 0;
  return nullptr;
}

}  // namespace

// ------------------------------------------------------------------------------------------------
// C API for the tests (ctypes) and the CPU baseline
// ------------------------------------------------------------------------------------------------
extern "C" {

const char* oracle_last_error() { return g_err.c_str(); }
int oracle_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
void oracle_set_threads(int t) {
#ifdef _OPENMP
  if (t > 0) omp_set_num_threads(t);
#else
  (void)t;
#endif
}

int oracle_fresh_state(const SoupConfig* c, float* pos, float* vel, uint32_t* frozen, uint32_t* brng, uint32_t* trng) {
  if (!c) return SOUP_E_ARG;
  fresh_state(*c, pos, vel, frozen, brng, trng);
  return SOUP_OK;
}
int oracle_initial_charges(const SoupConfig* c, const float* pos, float* charges, uint32_t* prot_rng) {
  if (!c || !pos || !charges) return SOUP_E_ARG;
  initial_charges(*c, pos, charges, prot_rng);
  return SOUP_OK;
}

void* oracle_create(const SoupConfig* c, const SoupInitState* init) { return create(c, init); }
void oracle_destroy(void* p) { delete static_cast<System*>(p); }

int oracle_step(void* p, uint64_t n) { return step_n(*static_cast<System*>(p), n); }

int oracle_phase(void* p, int phase) {
  System& s = *static_cast<System*>(p);
  switch (phase) {
    case SOUP_PHASE_REBUILD: build_lists(s); return SOUP_OK;
    case SOUP_PHASE_FORCE: do_force(s); return SOUP_OK;
    case SOUP_PHASE_KICK_DRIFT: kick_drift(s); return SOUP_OK;
    case SOUP_PHASE_KICK_THERMO: kick_thermostat(s); return SOUP_OK;
    case SOUP_PHASE_BONDS: { Bonds b(s); b.form_pass(); b.break_pass(); return SOUP_OK; }
    case SOUP_PHASE_MAX_DRIFT: max_drift(s); return SOUP_OK;
  }
  return SOUP_E_ARG;
}

int oracle_read(void* p, int field, void* dst, size_t bytes) {
  size_t need = 0;
  void* src = field_ptr(*static_cast<System*>(p), field, need);
  if (!src || bytes != need) return SOUP_E_ARG;
  std::memcpy(dst, src, bytes);
  return SOUP_OK;
}
int oracle_write(void* p, int field, const void* src, size_t bytes) {
  size_t need = 0;
  void* dst = field_ptr(*static_cast<System*>(p), field, need);
  if (!dst || bytes != need) return SOUP_E_ARG;
  std::memcpy(dst, src, bytes);
  return SOUP_OK;
}
// FP64 force on the current positions (list force in double; lists must be complete)
int oracle_forces64(void* p, double* out) { list_force<double>(*static_cast<System*>(p), out); return SOUP_OK; }
int oracle_forces_brute64(void* p, double* out) { brute_force<double>(*static_cast<System*>(p), out); return SOUP_OK; }
int oracle_forces_brute32(void* p, float* out) { brute_force<float>(*static_cast<System*>(p), out); return SOUP_OK; }

// Verlet list as sorted CSR (counts[n]; lists may be NULL)
int oracle_verlet(void* p, uint32_t* counts, uint32_t* lists, size_t cap) {
  System& s = *static_cast<System*>(p);
  for (uint32_t i = 0; i < s.n; ++i) counts[i] = (uint32_t)(s.vl_off[i + 1] - s.vl_off[i]);
  if (lists) {
    if (cap < s.vl.size()) return SOUP_E_ARG;
    std::memcpy(lists, s.vl.data(), s.vl.size() * 4);
  }
  return SOUP_OK;
}
// head (long-range) list as sorted CSR over the heads in ascending index (counts[heads]; lists may be
// NULL); rows hold particle indices
int oracle_es_list(void* p, uint32_t* counts, uint32_t* lists, size_t cap) {
  System& s = *static_cast<System*>(p);
  const size_t H = s.heads.size();
  for (size_t h = 0; h < H; ++h) counts[h] = (uint32_t)(s.es_off[h + 1] - s.es_off[h]);
  if (lists) {
    if (cap < s.es.size()) return SOUP_E_ARG;
    for (size_t h = 0; h < H; ++h) {
      std::copy(s.es.begin() + s.es_off[h], s.es.begin() + s.es_off[h + 1], lists + s.es_off[h]);
      std::sort(lists + s.es_off[h], lists + s.es_off[h + 1]);
    }
  }
  return SOUP_OK;
}
int oracle_info(void* p, uint64_t* out6) {
  System& s = *static_cast<System*>(p);
  out6[0] = s.step; out6[1] = s.rebuilds; out6[2] = s.sweeps; out6[3] = s.vl.size();
  out6[4] = s.heads.size(); out6[5] = s.list_overflow | (s.es_overflow << 1);
  return SOUP_OK;
}
double oracle_max_drift_sq(void* p) { return static_cast<System*>(p)->max_drift_sq; }
int oracle_nonfinite(void* p, uint32_t* out2) { nonfinite(*static_cast<System*>(p), out2); return SOUP_OK; }

int oracle_sweep(void* p, SoupSweepResult* out) {
  System& s = *static_cast<System*>(p);
  sweep_now(s);
  if (out) *out = s.last_sweep;
  return SOUP_OK;
}
// A sweep on bare arrays (the reference's tests call protonationSweep on hand-made positions)
int oracle_ph_sweep_arrays(const SoupConfig* c, const float* pos, float* charges, uint32_t n, uint32_t* rng,
                           SoupSweepResult* out) {
  EsHost b = es_host(*c);
  *out = ph_sweep(pos, charges, n, c->box, c->charged_kind, b, *rng);
  return SOUP_OK;
}
double oracle_es_pair_energy(const SoupConfig* c, double r, double qq) { return es_pair_energy(r, qq, es_host(*c)); }
double oracle_acid_soap_well(const SoupConfig* c, double r) { return acid_soap_well(r, es_host(*c)); }
// the f32 pair force of one pair (x_i - x_j = (dx,0,0)) as the kernels evaluate it, for -dU/dr pins
double oracle_pair_force_x(const SoupConfig* c, int ki, int kj, double qi, double qj, double r, int fp64) {
  if (fp64) {
    Phys<double> ph = Phys<double>::from_f64(*c);
    double xi[3] = {r, 0, 0}, xj[3] = {0, 0, 0}, f[3] = {0, 0, 0};
    ph.nonbonded(xi, xj, ki, kj, qi, qj, f);
    double g[3] = {0, 0, 0};
    ph.es_far(xi, xj, qi, qj, g);
    return f[0] + g[0];
  }
  Phys<float> ph = Phys<float>::from_f32(make_u32f(*c));
  float xi[3] = {(float)r, 0, 0}, xj[3] = {0, 0, 0}, f[3] = {0, 0, 0};
  ph.nonbonded(xi, xj, ki, kj, (float)qi, (float)qj, f);
  float g[3] = {0, 0, 0};
  ph.es_far(xi, xj, (float)qi, (float)qj, g);
  return (double)f[0] + g[0];
}

int oracle_periodic_centre(const float* pos, const uint32_t* idx, uint32_t m, const double box[3], double alpha, double out[3]) {
  return periodic_centre(pos, idx, m, box, alpha, out);
}
int oracle_closure(const float* pos, const uint32_t* mem, uint32_t nm, const uint32_t* wat, uint32_t nw, const double box[3],
                   const double centre[3], double cell, double radius, double vmin, SoupClosureResult* res,
                   uint8_t* occ, uint8_t* vis) {
  std::vector<uint8_t> o, v;
  int st = closure(pos, mem, nm, wat, nw, box, centre, cell, radius, vmin, res, occ ? &o : nullptr, vis ? &v : nullptr);
  if (st) return st;
  if (occ) std::memcpy(occ, o.data(), o.size());
  if (vis) std::memcpy(vis, v.data(), v.size());
  return SOUP_OK;
}
int oracle_closure_in_parcel(const float* pos, const uint32_t* mem, uint32_t nm, const uint32_t* wat, uint32_t nw,
                             const double box[3], const double centre[3], double cell, double radius, double vmin,
                             const double parcel_centre[3], double parcel_radius, SoupClosureResult* res) {
  const double parcel[4] = {parcel_centre[0], parcel_centre[1], parcel_centre[2], parcel_radius};
  return closure(pos, mem, nm, wat, nw, box, centre, cell, radius, vmin, res, nullptr, nullptr, parcel);
}
uint32_t oracle_amphiphiles(const float* pos, const uint32_t* slots, uint32_t n, const uint32_t* polar_of_kind, uint32_t* head_of) {
  return amphiphiles(pos, slots, n, polar_of_kind, head_of);
}
uint32_t oracle_aggregates(const float* pos, const uint32_t* mem, uint32_t m, const double box[3], double cutoff, uint32_t* labels) {
  return aggregates(pos, mem, m, box, cutoff, labels);
}

// pairingStats (soup/src/electrostatics.ts:520-561) over every pair of titratable heads; the nearest
// contact's exact-distance ties go to the smaller head index.  out: with_neighbour, unlike, like,
// paired, charged, heads.
int oracle_pairing_stats(const float* pos, const float* charges, uint32_t n, const double box[3], int charged_kind,
                         double contact, uint32_t* out6) {
  std::vector<uint32_t> heads;
  for (uint32_t i = 0; i < n; ++i) if ((int)pos[4 * i + 3] == charged_kind) heads.push_back(i);
  auto mi = [](double d, double L) { return d - js_round(d / L) * L; };
  uint32_t with = 0, unlike = 0, like = 0, paired = 0, charged = 0;
  for (size_t a = 0; a < heads.size(); ++a) {
    const uint32_t i = heads[a];
    if (charges[i] != 0.f) ++charged;
    double best = INFINITY;
    long best_b = -1;
    bool any = false;
    for (size_t b = 0; b < heads.size(); ++b) {
      if (b == a) continue;
      const uint32_t j = heads[b];
      const double dx = mi((double)pos[4 * i] - pos[4 * j], box[0]);
      const double dy = mi((double)pos[4 * i + 1] - pos[4 * j + 1], box[1]);
      const double dz = mi((double)pos[4 * i + 2] - pos[4 * j + 2], box[2]);
      const double r = std::sqrt(dx * dx + dy * dy + dz * dz);
      if (r > contact) continue;
      any = true;
      if ((charges[i] == 0.f) != (charges[j] == 0.f)) ++unlike; else ++like;
      if (r < best) { best = r; best_b = (long)b; }
    }
    if (any) ++with;
    if (best_b >= 0 && (charges[i] == 0.f) != (charges[heads[best_b]] == 0.f)) ++paired;
  }
  out6[0] = with; out6[1] = unlike; out6[2] = like; out6[3] = paired; out6[4] = charged;
  out6[5] = (uint32_t)heads.size();
  return SOUP_OK;
}

// densityProfileZ (engine/src/metrics.ts:21-47) with heads = kinds in head_mask; escaped beads are
// counted instead of binned (dropEscapedZ, metrics.ts:91-110)
int oracle_density_profile_z(const float* pos, uint32_t n, double box_z, uint32_t bins, uint32_t head_mask,
                             uint32_t* head, uint32_t* tail, uint32_t* escaped) {
  const double dz = box_z / bins;
  for (uint32_t b = 0; b < bins; ++b) head[b] = tail[b] = 0;
  uint32_t esc = 0;
  for (uint32_t i = 0; i < n; ++i) {
    const double z = pos[4 * i + 2];
    if (!(z >= 0 && z < box_z)) { ++esc; continue; }
    const uint32_t b = std::min<uint32_t>(bins - 1, (uint32_t)std::floor(z / dz));
    const uint32_t kind = (uint32_t)(int)pos[4 * i + 3];
    if (kind < 32 && ((head_mask >> kind) & 1u)) ++head[b]; else ++tail[b];
  }
  *escaped = esc;
  return SOUP_OK;
}

// shapeOf over unwrapAggregate (engine/src/aggregate.ts:245-262, 308-346) for one component; members
// ascending, the first one the unwrap reference.  out10: n, centre xyz, Sxx Syy Szz Sxy Sxz Syz.
int oracle_aggregate_shape(const float* pos, const uint32_t* members, uint32_t m, const double box[3], double* out10) {
  if (m == 0) return SOUP_E_ARG;
  auto mi = [](double d, double L) { return d - js_round(d / L) * L; };
  std::vector<float> u(3 * (size_t)m);
  const double ref[3] = {pos[4 * members[0]], pos[4 * members[0] + 1], pos[4 * members[0] + 2]};
  for (uint32_t k = 0; k < m; ++k)
    for (int a = 0; a < 3; ++a)
      u[3 * k + a] = (float)(ref[a] + mi((double)pos[4 * members[k] + a] - ref[a], box[a]));
  double c[3] = {0, 0, 0};
  for (uint32_t k = 0; k < m; ++k) for (int a = 0; a < 3; ++a) c[a] += u[3 * k + a];
  for (int a = 0; a < 3; ++a) c[a] /= m;
  double S[6] = {0, 0, 0, 0, 0, 0};
  for (uint32_t k = 0; k < m; ++k) {
    const double dx = u[3 * k] - c[0], dy = u[3 * k + 1] - c[1], dz = u[3 * k + 2] - c[2];
    S[0] += dx * dx; S[1] += dy * dy; S[2] += dz * dz; S[3] += dx * dy; S[4] += dx * dz; S[5] += dy * dz;
  }
  out10[0] = m;
  for (int a = 0; a < 3; ++a) out10[1 + a] = c[a];
  for (int q = 0; q < 6; ++q) out10[4 + q] = S[q] / m;
  return SOUP_OK;
}

// relaxIterations (soup/src/soup-relax.ts:87-111)
int oracle_relax(void* p, uint32_t iterations, double d0) {
  System& s = *static_cast<System*>(p);
  for (uint32_t k = 0; k < iterations; ++k) {
    float d = (float)(d0 * (1.0 - (double)k / iterations));
    build_lists(s);
    do_force(s);
    relax_step(s, d);
  }
  build_lists(s);
  do_force(s);
  return SOUP_OK;
}

// scaleMoleculesRigid (soup/src/soup-box-scale-math.ts:63-138).  Adjacency lists in edge order
// (each edge (i, j) appends j to i's list and i to j's); components discovered from the smallest
// unvisited index; breadth-first walk with offsets accumulated edge by edge through mi1 (JavaScript
// Math.round); FP64 centre of mass summed in visiting order; each bead rebuilt about the scaled,
// wrapped centre from its unchanged offset and wrapped into the new box.  All double, no FMA
// contraction (the Makefile's -ffp-contract=off), as the reference's JavaScript numbers.
int oracle_scale_molecules_rigid(const float* pos, uint32_t n, const uint32_t* edges, uint32_t n_edges,
                                 const double old_box[3], const double new_box[3], float* out) {
  const double s[3] = {new_box[0] / old_box[0], new_box[1] / old_box[1], new_box[2] / old_box[2]};
  std::vector<std::vector<uint32_t>> adj(n);
  for (uint32_t k = 0; k < n_edges; ++k) {
    const uint32_t i = edges[2 * k], j = edges[2 * k + 1];
    if (i >= n || j >= n) { g_err = "scaleMoleculesRigid: edge names a particle outside the system"; return SOUP_E_ARG; }
    adj[i].push_back(j);
    adj[j].push_back(i);
  }
  std::vector<uint8_t> visited(n, 0);
  std::vector<double> off(3 * (size_t)n, 0.0);
  std::vector<uint32_t> members;
  for (uint32_t root = 0; root < n; ++root) {
    if (visited[root]) continue;
    visited[root] = 1;
    for (int a = 0; a < 3; ++a) off[3 * (size_t)root + a] = 0.0;
    members.assign(1, root);
    for (size_t qi = 0; qi < members.size(); ++qi) {
      const uint32_t p = members[qi];
      for (uint32_t c : adj[p]) {
        if (visited[c]) continue;
        visited[c] = 1;
        for (int a = 0; a < 3; ++a)
          off[3 * (size_t)c + a] = off[3 * (size_t)p + a] + mi1((double)pos[4 * (size_t)c + a] - (double)pos[4 * (size_t)p + a], old_box[a]);
        members.push_back(c);
      }
    }
    double cen[3], com[3];
    for (int a = 0; a < 3; ++a) {
      double sum = 0.0;
      for (uint32_t b : members) sum += off[3 * (size_t)b + a];
      cen[a] = sum / (double)members.size();
      com[a] = wrap1((double)pos[4 * (size_t)root + a] + cen[a], old_box[a]) * s[a];
    }
    for (uint32_t b : members) {
      for (int a = 0; a < 3; ++a) out[4 * (size_t)b + a] = (float)wrap1(com[a] + (off[3 * (size_t)b + a] - cen[a]), new_box[a]);
      out[4 * (size_t)b + 3] = pos[4 * (size_t)b + 3];
    }
  }
  return SOUP_OK;
}

// unwrapAggregate (engine/src/aggregate.ts:245-262) on all three axes about members[0]; f32 out, w = kind
int oracle_unwrap_aggregate(const float* pos, const uint32_t* members, uint32_t m, const double box[3], float* out) {
  if (m == 0) return SOUP_OK;
  const float* r = pos + 4 * (size_t)members[0];
  for (uint32_t k = 0; k < m; ++k) {
    const float* p = pos + 4 * (size_t)members[k];
    for (int a = 0; a < 3; ++a) out[4 * (size_t)k + a] = (float)((double)r[a] + mi1((double)p[a] - (double)r[a], box[a]));
    out[4 * (size_t)k + 3] = p[3];
  }
  return SOUP_OK;
}

// localCavityVolume (soup/src/aggregates.ts:350-385) over occupancy (engine/src/closure.ts:67-107: x
// and y wrap, z open) and enclosedVolume/floodOutside (closure.ts:108-163: breadth-first from every
// empty cell on the six faces, open boundary); unreached empty cells times cell^3
static double cavity_on_grid(const float* sh, uint32_t n, const double box[3], const int dims[3], double cell,
                             double radius);

double oracle_local_cavity_volume(const float* positions, uint32_t n, double cell, double radius) {
  if (n == 0) return 0.0;
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint32_t i = 0; i < n; ++i)
    for (int a = 0; a < 3; ++a) {
      const double v = positions[4 * (size_t)i + a];
      if (v < lo[a]) lo[a] = v;
      if (v > hi[a]) hi[a] = v;
    }
  const double pad = radius * 4;
  double box[3];
  int dims[3];
  std::vector<float> sh(4 * (size_t)n);
  for (int a = 0; a < 3; ++a) {
    box[a] = hi[a] - lo[a] + 2 * pad;
    dims[a] = std::max(1, (int)std::ceil(box[a] / cell));
  }
  for (uint32_t i = 0; i < n; ++i)
    for (int a = 0; a < 3; ++a) sh[4 * (size_t)i + a] = (float)((double)positions[4 * (size_t)i + a] + (pad - lo[a]));
  return cavity_on_grid(sh.data(), n, box, dims, cell, radius);
}

// engine/src/closure.ts:51-163 occupancy (x, y periodic, z open) + floodOutside + enclosedVolume on
// the grid `dims` of `box`, positions as given
static double cavity_on_grid(const float* sh, uint32_t n, const double box[3], const int dims[3], double cell,
                             double radius) {
  const int nx = dims[0], ny = dims[1], nz = dims[2];
  const size_t nc = (size_t)nx * ny * nz;
  std::vector<uint8_t> occ(nc, 0), vis(nc, 0);
  const int reach = std::max(1, (int)std::ceil(radius / cell));
  const double r2 = radius * radius;
  for (uint32_t i = 0; i < n; ++i) {
    const double px = sh[4 * (size_t)i], py = sh[4 * (size_t)i + 1], pz = sh[4 * (size_t)i + 2];
    const int cx = (int)std::floor(px / cell), cy = (int)std::floor(py / cell), cz = (int)std::floor(pz / cell);
    for (int dz = -reach; dz <= reach; ++dz) {
      const int gz = cz + dz;
      if (gz < 0 || gz >= nz) continue;
      const double ddz = (gz + 0.5) * cell - pz;
      for (int dy = -reach; dy <= reach; ++dy) {
        const int gy = ((cy + dy) % ny + ny) % ny;
        double ddy = (gy + 0.5) * cell - py;
        ddy -= js_round(ddy / box[1]) * box[1];
        for (int dx = -reach; dx <= reach; ++dx) {
          const int gx = ((cx + dx) % nx + nx) % nx;
          double ddx = (gx + 0.5) * cell - px;
          ddx -= js_round(ddx / box[0]) * box[0];
          if (ddx * ddx + ddy * ddy + ddz * ddz <= r2) occ[gx + (size_t)nx * (gy + (size_t)ny * gz)] = 1;
        }
      }
    }
  }
  std::vector<size_t> queue;
  auto seed = [&](int x, int y, int z) {
    if (x < 0 || x >= nx || y < 0 || y >= ny || z < 0 || z >= nz) return;
    const size_t i = x + (size_t)nx * (y + (size_t)ny * z);
    if (!occ[i] && !vis[i]) { vis[i] = 1; queue.push_back(i); }
  };
  for (int y = 0; y < ny; ++y) for (int z = 0; z < nz; ++z) { seed(0, y, z); seed(nx - 1, y, z); }
  for (int x = 0; x < nx; ++x) for (int z = 0; z < nz; ++z) { seed(x, 0, z); seed(x, ny - 1, z); }
  for (int x = 0; x < nx; ++x) for (int y = 0; y < ny; ++y) { seed(x, y, 0); seed(x, y, nz - 1); }
  for (size_t h = 0; h < queue.size(); ++h) {
    const size_t i = queue[h];
    const int z = (int)(i / ((size_t)nx * ny));
    const size_t rem = i - (size_t)z * nx * ny;
    const int y = (int)(rem / nx), x = (int)(rem - (size_t)y * nx);
    seed(x + 1, y, z); seed(x - 1, y, z); seed(x, y + 1, z); seed(x, y - 1, z); seed(x, y, z + 1); seed(x, y, z - 1);
  }
  size_t unreached = 0;
  for (size_t i = 0; i < nc; ++i) unreached += (!occ[i] && !vis[i]) ? 1 : 0;
  return (double)unreached * cell * cell * cell;
}

// engine/src/closure.ts:315-323 enclosedVolumeFromPositions after its recentring: the grid of the
// periodic box (dimsFor, closure.ts:51-57), positions as given
double oracle_box_cavity_volume(const float* positions, uint32_t n, const double box[3], double cell, double radius) {
  if (n == 0) return 0.0;
  int dims[3];
  for (int a = 0; a < 3; ++a) dims[a] = std::max(1, (int)std::ceil(box[a] / cell));
  return cavity_on_grid(positions, n, box, dims, cell, radius);
}

// engine/src/aggregate.ts:65-130 buildClusterUnionFind with its periodicZ switch, binned as the
// reference bins: with z open the z cell is floor(z / cutoff), unwrapped and unbounded, and the z
// neighbours are not wrapped.  Labels: the minimum original index of each component.
uint32_t oracle_cluster_labels(const float* pos, const uint32_t* mem, uint32_t m, const double box[3], double cutoff,
                               int periodic_z, uint32_t* labels) {
  if (periodic_z) return aggregates(pos, mem, m, box, cutoff, labels);
  std::vector<uint32_t> parent(m);
  std::iota(parent.begin(), parent.end(), 0u);
  auto find = [&](uint32_t x) { while (parent[x] != x) { parent[x] = parent[parent[x]]; x = parent[x]; } return x; };
  const int nx = std::max(1, (int)std::floor(box[0] / cutoff)), ny = std::max(1, (int)std::floor(box[1] / cutoff));
  const double wx = box[0] / nx, wy = box[1] / ny, wz = cutoff;
  std::vector<int> cx(m), cy(m);
  std::vector<long long> cz(m);
  std::map<std::tuple<int, int, long long>, std::vector<uint32_t>> buckets;
  for (uint32_t k = 0; k < m; ++k) {
    const uint32_t i = mem[k];
    cx[k] = std::min(nx - 1, (int)std::floor(wrap1(pos[i * 4], box[0]) / wx));
    cy[k] = std::min(ny - 1, (int)std::floor(wrap1(pos[i * 4 + 1], box[1]) / wy));
    cz[k] = (long long)std::floor((double)pos[i * 4 + 2] / wz);
    buckets[std::make_tuple(cx[k], cy[k], cz[k])].push_back(k);
  }
  const double c2 = cutoff * cutoff;
  for (uint32_t k = 0; k < m; ++k) {
    const uint32_t i = mem[k];
    for (int dx = -1; dx <= 1; ++dx) {
      const int ax = ((cx[k] + dx) % nx + nx) % nx;
      for (int dy = -1; dy <= 1; ++dy) {
        const int ay = ((cy[k] + dy) % ny + ny) % ny;
        for (int dz = -1; dz <= 1; ++dz) {
          auto it = buckets.find(std::make_tuple(ax, ay, cz[k] + dz));
          if (it == buckets.end()) continue;
          for (uint32_t l : it->second) {
            if (l <= k) continue;
            const uint32_t j = mem[l];
            const double ddx = mi1((double)pos[i * 4] - pos[j * 4], box[0]);
            const double ddy = mi1((double)pos[i * 4 + 1] - pos[j * 4 + 1], box[1]);
            const double ddz = (double)pos[i * 4 + 2] - pos[j * 4 + 2];
            if (ddx * ddx + ddy * ddy + ddz * ddz <= c2) {
              const uint32_t ra = find(k), rb = find(l);
              if (ra != rb) parent[ra] = rb;
            }
          }
        }
      }
    }
  }
  std::vector<uint32_t> minIdx(m, NONE);
  for (uint32_t k = 0; k < m; ++k) { const uint32_t r = find(k); minIdx[r] = std::min(minIdx[r], mem[k]); }
  uint32_t ncomp = 0;
  for (uint32_t k = 0; k < m; ++k) { labels[k] = minIdx[find(k)]; if (find(k) == k) ncomp++; }
  return ncomp;
}

// proximityPairs (soup/src/soup-box-scale-math.ts:162-221): pairs i < j among the eligible beads with
// a minimum-image distance <= cutoff, from a cell list of floor(box / cutoff) cells per axis, every
// axis periodic.  A pair is listed once per neighbouring-cell visit that reaches it, as the
// reference's 27-cell loop does (fewer than three cells on an axis visits a cell more than once).
// Writes up to `cap` pairs; returns the number found in *count.
int oracle_proximity_pairs(const float* pos, uint32_t n, const double box[3], double cutoff, const uint8_t* eligible,
                           uint32_t* pairs, size_t cap, size_t* count) {
  int nc[3];
  double w[3];
  for (int a = 0; a < 3; ++a) { nc[a] = std::max(1, (int)std::floor(box[a] / cutoff)); w[a] = box[a] / nc[a]; }
  std::vector<int> cx(n), cy(n), cz(n);
  std::vector<std::vector<uint32_t>> bucket((size_t)nc[0] * nc[1] * nc[2]);
  for (uint32_t i = 0; i < n; ++i) {
    if (!eligible[i]) continue;
    int c[3];
    for (int a = 0; a < 3; ++a)
      c[a] = std::min(nc[a] - 1, (int)std::floor(wrap1((double)pos[4 * (size_t)i + a], box[a]) / w[a]));
    cx[i] = c[0]; cy[i] = c[1]; cz[i] = c[2];
    bucket[((size_t)c[2] * nc[1] + c[1]) * nc[0] + c[0]].push_back(i);
  }
  const double c2 = cutoff * cutoff;
  size_t k = 0;
  for (uint32_t i = 0; i < n; ++i) {
    if (!eligible[i]) continue;
    for (int dx = -1; dx <= 1; ++dx) {
      const int x = ((cx[i] + dx) % nc[0] + nc[0]) % nc[0];
      for (int dy = -1; dy <= 1; ++dy) {
        const int y = ((cy[i] + dy) % nc[1] + nc[1]) % nc[1];
        for (int dz = -1; dz <= 1; ++dz) {
          const int z = ((cz[i] + dz) % nc[2] + nc[2]) % nc[2];
          for (uint32_t j : bucket[((size_t)z * nc[1] + y) * nc[0] + x]) {
            if (j <= i) continue;
            const double ddx = mi1((double)pos[4 * (size_t)i] - (double)pos[4 * (size_t)j], box[0]);
            const double ddy = mi1((double)pos[4 * (size_t)i + 1] - (double)pos[4 * (size_t)j + 1], box[1]);
            const double ddz = mi1((double)pos[4 * (size_t)i + 2] - (double)pos[4 * (size_t)j + 2], box[2]);
            if (ddx * ddx + ddy * ddy + ddz * ddz <= c2) {
              if (k < cap) { pairs[2 * k] = i; pairs[2 * k + 1] = j; }
              ++k;
            }
          }
        }
      }
    }
  }
  *count = k;
  return SOUP_OK;
}

}  // extern "C"

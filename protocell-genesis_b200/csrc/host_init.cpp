// host_init.cpp -- fresh-creation state on the host, as createSoup builds it before any dispatch.
//
// Reference: soup/src/soup-init-state.ts:17-31 (mulberry32, gaussian), :58-307 buildInitialState
// (jittered cubic lattice, Fisher-Yates site shuffle, Maxwell-Boltzmann velocities, per-particle
// bond/thermostat seeds), soup/src/soup-confine.ts sphereLatticeSites (parcel lattice),
// soup/src/soup-protonation.ts:38-49 initialCharges (Henderson-Hasselbalch draw per head).
// The draw order is the reference's, so a given seed reproduces the reference's arrays bit for bit
// (the clay platelet and frozen bulk catalysts are not part of this build).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "soup_internal.h"

namespace soup {

namespace {

struct Mulberry {
  uint32_t a;
  double next() {
    a += 0x6d2b79f5u;
    uint32_t t = (a ^ (a >> 15)) * (1u | a);
    t = (t + ((t ^ (t >> 7)) * (61u | t))) ^ t;
    return (double)(t ^ (t >> 14)) / 4294967296.0;
  }
};

double lcg_pcg(uint32_t& s) {   // electrostatics.ts:308-315 pcgNext
  uint32_t v = s * 747796405u + 2891336453u;
  s = v;
  v = ((v >> ((v >> 28u) + 4u)) ^ v) * 277803737u;
  v = (v >> 22u) ^ v;
  return (double)v / 4294967296.0;
}

}  // namespace

void host_fresh_state(const SoupConfig& c, float* pos, float* vel, uint32_t* frozen, uint32_t* brng, uint32_t* trng) {
  const uint32_t N = c.n;
  Mulberry rng{c.seed};
  std::vector<double> parcel;
  double h = 0.0;
  if (c.wall_radius > 0) {   // sphereLatticeSites, centred in the box
    const double R = c.wall_radius, ctr[3] = {c.box[0] * 0.5, c.box[1] * 0.5, c.box[2] * 0.5};
    int m = std::max(2, (int)std::ceil(std::cbrt(N / (M_PI / 6))));
    for (;; ++m) {
      h = (2 * R) / m;
      parcel.clear();
      for (int iz = 0; iz < m; ++iz)
        for (int iy = 0; iy < m; ++iy)
          for (int ix = 0; ix < m; ++ix) {
            double x = -R + (ix + 0.5) * h, y = -R + (iy + 0.5) * h, z = -R + (iz + 0.5) * h;
            if (x * x + y * y + z * z <= R * R) {
              parcel.push_back(ctr[0] + x); parcel.push_back(ctr[1] + y); parcel.push_back(ctr[2] + z);
            }
          }
      if (parcel.size() / 3 >= N) break;
    }
  }
  uint32_t nx = std::max<uint32_t>(1, (uint32_t)std::ceil(std::cbrt((double)N)));
  while ((uint64_t)nx * nx * nx < N) ++nx;
  double sp[3];
  for (int a = 0; a < 3; ++a) sp[a] = parcel.empty() ? c.box[a] / nx : h;
  const uint64_t nsites = parcel.empty() ? (uint64_t)nx * nx * nx : parcel.size() / 3;
  std::vector<uint32_t> order(nsites);
  for (uint64_t i = 0; i < nsites; ++i) order[i] = (uint32_t)i;
  for (uint64_t i = nsites - 1; i > 0; --i) std::swap(order[i], order[(uint64_t)std::floor(rng.next() * (double)(i + 1))]);
  const double jitter = 0.15, s = std::sqrt(c.kT);
  uint32_t idx = 0;
  for (uint32_t kind = 0; kind < c.n_kinds; ++kind) {
    for (uint32_t q = 0; q < c.counts[kind]; ++q, ++idx) {
      const uint32_t site = order[idx];
      double base[3];
      if (!parcel.empty()) {
        for (int a = 0; a < 3; ++a) base[a] = parcel[(size_t)site * 3 + a];
      } else {
        base[0] = (site % nx + 0.5) * sp[0];
        base[1] = ((site / nx) % nx + 0.5) * sp[1];
        base[2] = (site / (nx * nx) + 0.5) * sp[2];
      }
      double p[3];
      for (int a = 0; a < 3; ++a) p[a] = base[a] + (rng.next() * 2 - 1) * jitter * sp[a];
      double g[3];
      for (int a = 0; a < 3; ++a) {
        const double u1 = std::max(rng.next(), 1e-9), u2 = rng.next();
        g[a] = s * (std::sqrt(-2 * std::log(u1)) * std::cos(2 * M_PI * u2));
      }
      if (pos) { for (int a = 0; a < 3; ++a) pos[4 * idx + a] = (float)p[a]; pos[4 * idx + 3] = (float)kind; }
      if (vel) { for (int a = 0; a < 3; ++a) vel[4 * idx + a] = (float)g[a]; vel[4 * idx + 3] = 0.f; }
      if (frozen) frozen[idx] = 0;
    }
  }
  for (uint32_t i = 0; i < N; ++i) {
    if (brng) brng[i] = c.seed ^ ((i + 1u) * 2654435761u) ^ 0x9e3779b9u;
    if (trng) trng[i] = c.seed ^ ((i + 1u) * 3266489917u) ^ 0x85ebca6bu;
  }
}

void host_initial_charges(const SoupConfig& c, const float* pos, float* charges, uint32_t* prot_rng) {
  uint32_t s = c.seed ^ 0x9e3779b9u;
  for (uint32_t i = 0; i < c.n; ++i) charges[i] = 0.f;
  if (c.es_enabled) {
    const double alpha = 1.0 / (1.0 + std::pow(10.0, c.pka_intrinsic - c.ph));
    for (uint32_t i = 0; i < c.n; ++i)
      if ((int)pos[4 * i + 3] == c.charged_kind && lcg_pcg(s) < alpha) charges[i] = (float)c.charge_deprotonated;
  }
  if (prot_rng) *prot_rng = s;
}

}  // namespace soup

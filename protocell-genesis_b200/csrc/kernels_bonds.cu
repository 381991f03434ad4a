// kernels_bonds.cu -- dynamic-bond Monte Carlo, deterministic.
//
// Reference: soup/wgsl/bond-verlet.wgsl:12-54 (candidate walk over the Verlet list),
// soup/wgsl/bond-dispatch.wgsl:89-142 bondFormDecide and :170-200 bond_break_main,
// soup/wgsl/bond-valence.wgsl:40-116 (tryClaimSlot / releaseSlot / releasePartnerSlot),
// soup/wgsl/bond-adsorption.wgsl:62-316 (catalyst centre bookkeeping and the two desorption valves),
// soup/wgsl/bond-common.wgsl:111-168 (matchRule, roleOf, hasBondTo, bondPcg).
//
// The reference resolves slot and centre claims by CAS races between threads, so its outcome varies
// with scheduling.  The canonical semantics here (and in the CPU oracle) are the serial execution of
// the formation pass in ascending particle order.  It is computed in parallel, exactly:
//   Phase A (one thread per particle): the candidate walk and both Metropolis draws.  Neither
//     depends on claim outcomes (a pair i<j is only ever formed by i; draws consume the particle's
//     own stream), so accept decisions and the final RNG state are computed here, in parallel.
//   Phase B (one CTA): every particle with an accepted proposal, every catalyst, every particle
//     holding a centre link, and every proposal partner becomes an "item".  Items whose particle
//     sets (self, partners, the catalyst found, and their current centre links) intersect are
//     joined by union-find; different components touch disjoint state, so they commute.  Inside a
//     component the items run in ascending index order, one per round.
//   Breaking is race-free in the reference (only the lower index of a bond draws for it) and runs
//     one thread per particle.
#include "soup_internal.h"

namespace soup {

namespace {

constexpr int kBlock = 256;
inline unsigned nblocks(uint64_t n, int b = kBlock) { return (unsigned)((n + b - 1) / b); }
constexpr uint32_t NONE = SOUP_NONE_U32;
constexpr int REC = 10;   // u32 per item record: i, catId, meta(nprop | rule<<(8+2c)), j[6], root

__device__ __forceinline__ int match_rule(const Shared& S, float ti, float tj) {
  for (int r = 0; r < 2; ++r) {   // BOND_RULES = 2 (bond-common.wgsl:41)
    const float a = S.kindA[r], b = S.kindB[r];
    if ((ti == a && tj == b) || (ti == b && tj == a)) return r;
  }
  return -1;
}

// Phase A
// A bead whose kind is in no rule has no candidate, draws nothing and, unless it is a catalyst or
// tethered to one, leaves no item: its walk would change nothing (water, most of a campaign's beads).
__device__ __forceinline__ bool bond_active(const Shared& S, float ti, uint32_t centre) {
  bool in_rule = false;
  for (int r = 0; r < 2; ++r) in_rule = in_rule || ti == S.kindA[r] || ti == S.kindB[r];
  return in_rule || ti == S.cat_kind || centre != NONE;
}

// the active beads' slots, compacted (a warp's in one atomic); sel[0..*nsel) in no particular order
__global__ void __launch_bounds__(256) k_bond_select(const Shared* __restrict__ Sg, uint32_t N,
                                                     const float4* __restrict__ pos,
                                                     const uint32_t* __restrict__ center, uint32_t* __restrict__ sel,
                                                     uint32_t* __restrict__ nsel) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  const bool act = k < N && bond_active(*Sg, pos[k].w, center[k]);
  const uint32_t m = __ballot_sync(0xffffffffu, act);
  if (!m) return;
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t base = 0;
  if (lane == (uint32_t)(__ffs(m) - 1)) base = atomicAdd(nsel, (uint32_t)__popc(m));
  base = __shfl_sync(0xffffffffu, base, __ffs(m) - 1);
  if (act) sel[base + __popc(m & ((1u << lane) - 1u))] = k;
}

// a thread per active bead (k_bond_select), so that the warps walk full
__global__ void __launch_bounds__(128) k_bond_walk(
    const Shared* __restrict__ Sg, const SysParams* __restrict__ sp, const uint8_t* __restrict__ sysid,
    const uint32_t* __restrict__ sel, const uint32_t* __restrict__ nsel,
    const float4* __restrict__ pos, const uint32_t* __restrict__ id, const uint32_t* __restrict__ slots,
    const uint32_t* __restrict__ center, const uint32_t* __restrict__ nl, const uint32_t* __restrict__ nl_cnt,
    uint32_t cap, uint32_t* __restrict__ brng, uint32_t* __restrict__ items, uint32_t* __restrict__ nitems,
    uint32_t* __restrict__ has_item) {
  const uint32_t ns = *nsel;
  if (blockIdx.x * blockDim.x >= ns) return;   // the whole block: past the active beads
  __shared__ Shared S;
  for (int w = threadIdx.x; w < (int)(sizeof(Shared) / 4); w += blockDim.x)
    reinterpret_cast<uint32_t*>(&S)[w] = reinterpret_cast<const uint32_t*>(Sg)[w];
  __syncthreads();
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ns) return;
  const uint32_t k = sel[t];
  const float4 xi = pos[k];
  const float ti = xi.w;
  const SysParams& P = sp[sysid[k]];
  const float box[3] = {P.box[0], P.box[1], P.box[2]};
  const uint32_t gi = id[k];
  const uint32_t s0 = slots[3 * k], s1 = slots[3 * k + 1], s2 = slots[3 * k + 2];
  const float cat_reach = ex_wcut(S, ex_pairB(S, ti, S.cat_kind));
  uint32_t catId = NONE;
  uint32_t cj[SOUP_CAND_CAP], cr[SOUP_CAND_CAP];
  int nc = 0;
  const uint32_t cnt = nl_cnt[k];
  const uint32_t* row = nl + (size_t)k * cap;
  for (uint32_t s = 0; s < cnt; ++s) {
    const uint32_t js = row[s];
    const float4 xj = pos[js];
    const float tj = xj.w;
    const bool isCat = tj == S.cat_kind;
    const int rk = match_rule(S, ti, tj);        // by the kinds alone
    if (!isCat && rk < 0) continue;
    const uint32_t j = id[js];
    int r = -1;
    if (j > gi) {
      r = rk;
      if (r >= 0 && (s0 == j || s1 == j || s2 == j)) r = -1;          // hasBondTo
      if (r >= 0 && nc == SOUP_CAND_CAP && j > cj[SOUP_CAND_CAP - 1]) r = -1;
    }
    if (!isCat && r < 0) continue;
    const float d = ex_dist(xi, xj, box);
    if (isCat && d < cat_reach && j < catId) catId = j;                // smallest catalyst in reach
    if (r >= 0 && d < ex_wcut(S, ex_pairB(S, ti, tj))) {
      // keep the SOUP_CAND_CAP smallest qualifying j, ascending
      int p = nc < SOUP_CAND_CAP ? nc : SOUP_CAND_CAP - 1;
      if (nc < SOUP_CAND_CAP) ++nc;
      while (p > 0 && cj[p - 1] > j) { cj[p] = cj[p - 1]; cr[p] = cr[p - 1]; --p; }
      cj[p] = j; cr[p] = (uint32_t)r;
    }
  }
  // draws (bondFormDecide's candidate loop up to the claims)
  uint32_t rng = brng[k];
  uint32_t pj[SOUP_CAND_CAP];
  uint32_t meta = 0;
  int np = 0;
  for (int c = 0; c < nc; ++c) {
    const uint32_t r = cr[c];
    if (S.req_cat[r] > 0.5f && catId == NONE) continue;
    rng = pcg_hash(rng);
    if (u01(rng) >= S.att_form[r]) continue;
    rng = pcg_hash(rng);
    if (u01(rng) >= S.acc_form[r]) continue;
    pj[np] = cj[c];
    meta |= r << (8 + 2 * np);
    ++np;
  }
  brng[k] = rng;
  if (np > 0 || ti == S.cat_kind || center[k] != NONE) {
    const uint32_t at = atomicAdd(nitems, 1u);
    uint32_t* rec = items + (size_t)at * REC;
    rec[0] = gi; rec[1] = catId; rec[2] = meta | (uint32_t)np;
    for (int c = 0; c < SOUP_CAND_CAP; ++c) rec[3 + c] = c < np ? pj[c] : NONE;
    has_item[gi] = 1;
  }
}

// ---- Phase B helpers: the serial body of bondFormDecide on global state ----
struct St {
  const Shared& S;
  const SysParams* sp;
  const uint8_t* sysid;
  const float4* pos;
  uint32_t* slots;
  uint32_t* center;
  uint32_t* held;
  const uint32_t* slot_of;
  uint32_t* events;
  uint32_t* desorb;

  __device__ uint32_t sl(uint32_t g) const { return slot_of[g]; }
  __device__ float kind(uint32_t g) const { return pos[sl(g)].w; }
  __device__ float dist(uint32_t a, uint32_t b) const {
    const SysParams& P = sp[sysid[sl(a)]];
    return ex_dist(pos[sl(a)], pos[sl(b)], P.box);
  }
  __device__ bool cas(uint32_t p, uint32_t e, uint32_t v) {
    uint32_t* c = &center[sl(p)];
    if (*c != e) return false;
    *c = v;
    return true;
  }
  __device__ float cat_contact(uint32_t a) const { return ex_wcut(S, ex_pairB(S, kind(a), S.cat_kind)); }
  // bond-valence.wgsl:40-98
  __device__ int claim(uint32_t p, uint32_t role, uint32_t partner) {
    uint32_t* s = &slots[3 * sl(p)];
    const bool term = S.head_terminal > 0.5f;
    if (role == 0) {
      if (s[0] == NONE) { s[0] = partner; if (term && s[2] != NONE) { s[0] = NONE; return -1; } return 0; }
      if (s[1] == NONE) { s[1] = partner; if (term && s[2] != NONE) { s[1] = NONE; return -1; } return 1; }
      return -1;
    } else if (role == 1) {
      if (s[2] == NONE) { s[2] = partner; if (term && s[0] != NONE && s[1] != NONE) { s[2] = NONE; return -1; } return 2; }
      return -1;
    }
    const uint32_t capc = (uint32_t)S.head_cap;
    for (uint32_t c = 0; c < capc; ++c) if (s[c] == NONE) { s[c] = partner; return (int)c; }
    return -1;
  }
  __device__ void release(uint32_t p, int slot) { if (slot >= 0) slots[3 * sl(p) + slot] = NONE; }
  __device__ bool within_reach(uint32_t a, uint32_t b) const { return dist(a, b) < __fadd_rn(cat_contact(a), S.wc); }
  // bond-adsorption.wgsl:87-248
  __device__ bool propagate(uint32_t i, uint32_t j, int sI, int sJ, uint32_t cat) {
    if (sI == 0 && sJ == 0) {
      if (cat == NONE) return false;
      if (dist(i, cat) >= cat_contact(i)) return false;
      if (!cas(cat, NONE, i)) return false;
      if (!cas(i, NONE, cat)) { cas(cat, i, NONE); return false; }
      held[sl(cat)] = 0;
      return true;
    }
    uint32_t tipOld, tipNew;
    if (sI == 1 && sJ == 0) { tipOld = i; tipNew = j; }
    else if (sI == 0 && sJ == 1) { tipOld = j; tipNew = i; }
    else return false;
    uint32_t owner = center[sl(tipOld)];
    bool reclaim = false;
    if (owner == NONE) { if (cat == NONE) return false; owner = cat; reclaim = true; }
    if (reclaim) { if (dist(tipOld, cat) >= cat_contact(tipOld)) return false; }
    else if (!within_reach(tipOld, owner)) return false;
    if (dist(tipNew, owner) >= cat_contact(tipNew)) return false;
    if (reclaim) {
      if (!cas(owner, NONE, tipOld)) return false;
      if (!cas(tipOld, NONE, owner)) { cas(owner, tipOld, NONE); return false; }
    }
    if (!cas(owner, tipOld, tipNew)) { if (reclaim) cas(tipOld, owner, NONE); return false; }
    if (!cas(tipNew, NONE, owner)) {
      cas(owner, tipNew, tipOld);
      if (reclaim) { cas(owner, tipOld, NONE); cas(tipOld, owner, NONE); }
      return false;
    }
    cas(tipOld, owner, NONE);
    held[sl(owner)] = 0;
    return true;
  }
  // bond-adsorption.wgsl:256-268
  __device__ bool terminate(uint32_t carbon) {
    const uint32_t owner = center[sl(carbon)];
    if (owner == NONE) return false;
    if (!within_reach(carbon, owner)) return false;
    if (!cas(carbon, owner, NONE)) return false;
    cas(owner, carbon, NONE);
    held[sl(owner)] = 0;
    return true;
  }
  // the whole item: desorption valve, then the accepted proposals in order
  __device__ void run(const uint32_t* rec) {
    const uint32_t i = rec[0], cat = rec[1], meta = rec[2];
    const int np = (int)(meta & 0xFFu);
    const uint32_t ks = sl(i);
    const uint32_t rs = sysid[ks];
    const float ti = pos[ks].w;
    if (ti == S.cat_kind) {                               // desorbTimeout (bond-adsorption.wgsl:304-316)
      const uint32_t tip = center[ks];
      if (tip != NONE) {
        const uint32_t inc = (uint32_t)S.interval;
        const uint32_t prev = held[ks];
        held[ks] = prev + inc;
        if (prev + inc > (uint32_t)S.max_hold) {
          if (cas(i, tip, NONE)) { cas(tip, i, NONE); held[ks] = 0; atomicAdd(&desorb[2 * rs + 1], 1u); }
        }
      }
    } else {
      const uint32_t owner = center[ks];                  // desorbStretch (bond-adsorption.wgsl:283-292)
      if (owner != NONE && dist(i, owner) >= S.r_inf) {
        if (cas(i, owner, NONE)) { cas(owner, i, NONE); held[sl(owner)] = 0; atomicAdd(&desorb[2 * rs + 0], 1u); }
      }
    }
    for (int c = 0; c < np; ++c) {
      const uint32_t j = rec[3 + c];
      const uint32_t r = (meta >> (8 + 2 * c)) & 3u;
      const float tj = kind(j);
      const uint32_t roleI = (ti == S.kindA[r]) ? (uint32_t)S.roleA[r] : (uint32_t)S.roleB[r];
      const uint32_t roleJ = (tj == S.kindA[r]) ? (uint32_t)S.roleA[r] : (uint32_t)S.roleB[r];
      const int sI = claim(i, roleI, j);
      if (sI < 0) continue;
      const int sJ = claim(j, roleJ, i);
      if (sJ < 0) { release(i, sI); continue; }
      bool ok;
      if (roleI == 0 && roleJ == 0) ok = propagate(i, j, sI, sJ, cat);
      else if (roleI == 1) ok = terminate(i);
      else ok = terminate(j);
      if (!ok) { release(i, sI); release(j, sJ); continue; }
      atomicAdd(&events[2 * SOUP_MAX_RULES * rs + 2 * r], 1u);   // components run concurrently
    }
  }
};

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
    if (a > b) { uint32_t t = a; a = b; b = t; }
    if (atomicCAS(&parent[b], b, a) == b) return;   // hook the larger root under the smaller
  }
}

// the particles an item may touch, as far as the pass-start state can tell (closure under centre links)
__device__ __forceinline__ int item_set(const uint32_t* rec, const uint32_t* center, const uint32_t* slot_of,
                                        uint32_t* out) {
  int n = 0;
  auto add = [&](uint32_t g) {
    if (g == NONE) return;
    out[n++] = g;
    const uint32_t c = center[slot_of[g]];
    if (c != NONE) out[n++] = c;
  };
  add(rec[0]);
  add(rec[1]);
  const int np = (int)(rec[2] & 0xFFu);
  for (int c = 0; c < np; ++c) add(rec[3 + c]);
  return n;
}

// Phase B.  Every particle an item may touch runs its own desorption check in its turn, so it needs
// an item too (proposal partners are the only ones the walk does not already cover): added here, by
// the whole grid, before the claims.
// nitems[1] holds the walk's item count: only the walk's items add partners (nitems[0] grows meanwhile).
__global__ void k_bond_partners(const uint32_t* __restrict__ center, const uint32_t* __restrict__ slot_of,
                                uint32_t* __restrict__ items, uint32_t* __restrict__ nitems, uint32_t item_cap,
                                uint32_t* __restrict__ has_item, uint32_t* __restrict__ flags) {
  const uint32_t M0 = min(nitems[1], item_cap);
  uint32_t setbuf[2 * (2 + SOUP_CAND_CAP)];
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < M0; t += gridDim.x * blockDim.x) {
    const int n = item_set(items + (size_t)t * REC, center, slot_of, setbuf);
    for (int q = 0; q < n; ++q) {
      const uint32_t x = setbuf[q];
      if (atomicCAS(&has_item[x], 0u, 1u) == 0u) {
        const uint32_t at = atomicAdd(nitems, 1u);
        if (at < item_cap) {
          uint32_t* nr = items + (size_t)at * REC;
          nr[0] = x; nr[1] = NONE; nr[2] = 0;
          for (int c = 0; c < SOUP_CAND_CAP; ++c) nr[3 + c] = NONE;
        } else {
          flags[6] = 1u;
        }
      }
    }
  }
}

// The claims of one replica per CTA (an item's set of particles never leaves its replica, so the
// replicas' components are disjoint and resolve independently).  The CTA collects its items, joins the
// items whose particle sets meet (union-find over the sets closed under centre links), and then in
// rounds executes the minimum-id pending item of every component: the serial ascending order within
// each component, which is all the serial order decides.
constexpr uint32_t kClaimLocal = 8192;   // a replica's items held as a list in shared memory
__global__ void __launch_bounds__(1024) k_bond_claims(
    const Shared* __restrict__ Sg, const SysParams* __restrict__ sp, const uint8_t* __restrict__ sysid,
    const float4* __restrict__ pos, uint32_t* __restrict__ slots, uint32_t* __restrict__ center,
    uint32_t* __restrict__ held, const uint32_t* __restrict__ slot_of, uint32_t* __restrict__ items,
    const uint32_t* __restrict__ nitems, uint32_t item_cap, uint32_t* __restrict__ parent,
    uint32_t* __restrict__ comp_min, uint8_t* __restrict__ done, uint32_t* __restrict__ events,
    uint32_t* __restrict__ desorb) {
  __shared__ Shared S;
  __shared__ uint32_t mine[kClaimLocal];
  __shared__ uint32_t nmine;
  for (int w = threadIdx.x; w < (int)(sizeof(Shared) / 4); w += blockDim.x)
    reinterpret_cast<uint32_t*>(&S)[w] = reinterpret_cast<const uint32_t*>(Sg)[w];
  if (threadIdx.x == 0) nmine = 0;
  __syncthreads();
  const uint32_t r = blockIdx.x;
  const uint32_t M = min(*nitems, item_cap);
  // this replica's items (any order: the rounds below depend on item ids, not positions); a batch of
  // one replica takes them all as they are
  const bool all = gridDim.x == 1;
  if (!all) {
    for (uint32_t t = threadIdx.x; t < M; t += blockDim.x)
      if (sysid[slot_of[items[(size_t)t * REC]]] == r) {
        const uint32_t at = atomicAdd(&nmine, 1u);
        if (at < kClaimLocal) mine[at] = t;
      }
  }
  __syncthreads();
  const bool local = !all && nmine <= kClaimLocal;
  const uint32_t L = local ? nmine : M;
  // item u of this CTA, or NONE for another replica's item (when the list did not fit)
  auto item = [&](uint32_t u) -> uint32_t {
    if (all) return u;
    if (local) return mine[u];
    return sysid[slot_of[items[(size_t)u * REC]]] == r ? u : NONE;
  };
  uint32_t setbuf[2 * (2 + SOUP_CAND_CAP)];
  for (uint32_t u = threadIdx.x; u < L; u += blockDim.x) {
    const uint32_t t = item(u);
    if (t == NONE) continue;
    const int n = item_set(items + (size_t)t * REC, center, slot_of, setbuf);
    for (int q = 0; q < n; ++q) parent[setbuf[q]] = setbuf[q];
    done[t] = 0;
  }
  __syncthreads();
  for (uint32_t u = threadIdx.x; u < L; u += blockDim.x) {
    const uint32_t t = item(u);
    if (t == NONE) continue;
    const int n = item_set(items + (size_t)t * REC, center, slot_of, setbuf);
    for (int q = 1; q < n; ++q) uf_union(parent, setbuf[0], setbuf[q]);
  }
  __syncthreads();
  for (uint32_t u = threadIdx.x; u < L; u += blockDim.x) {
    const uint32_t t = item(u);
    if (t == NONE) continue;
    uint32_t* rec = items + (size_t)t * REC;
    const uint32_t root = uf_find(parent, rec[0]);
    rec[9] = root;
    comp_min[root] = NONE;
  }
  __syncthreads();
  St st{S, sp, sysid, pos, slots, center, held, slot_of, events, desorb};
  for (int round = 0;; ++round) {
    int pending = 0;
    for (uint32_t u = threadIdx.x; u < L; u += blockDim.x) {
      const uint32_t t = item(u);
      if (t == NONE || done[t]) continue;
      pending = 1;
      atomicMin(&comp_min[items[(size_t)t * REC + 9]], items[(size_t)t * REC]);
    }
    if (!__syncthreads_or(pending)) break;
    for (uint32_t u = threadIdx.x; u < L; u += blockDim.x) {
      const uint32_t t = item(u);
      if (t == NONE || done[t]) continue;
      const uint32_t* rec = items + (size_t)t * REC;
      if (comp_min[rec[9]] == rec[0]) { st.run(rec); done[t] = 1; }
    }
    __syncthreads();
    for (uint32_t u = threadIdx.x; u < L; u += blockDim.x) {
      const uint32_t t = item(u);
      if (t != NONE) comp_min[items[(size_t)t * REC + 9]] = NONE;
    }
    __syncthreads();
  }
}

// bond-dispatch.wgsl:170-200 bond_break_main
__global__ void k_bond_break(const Shared* __restrict__ Sg, const uint8_t* __restrict__ sysid, uint32_t N,
                             const float4* __restrict__ pos, const uint32_t* __restrict__ id,
                             const uint32_t* __restrict__ slot_of, uint32_t* __restrict__ slots,
                             uint32_t* __restrict__ brng, uint32_t* __restrict__ events) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= N) return;
  const Shared& S = *Sg;
  const uint32_t gi = id[k];
  const float ti = pos[k].w;
  uint32_t rng = brng[k];
  bool touched = false;
  for (int s = 0; s < 3; ++s) {
    const uint32_t partner = slots[3 * k + s];
    if (partner == NONE || partner < gi) continue;
    const uint32_t ps = slot_of[partner];
    const int r = match_rule(S, ti, pos[ps].w);
    if (r < 0) continue;
    touched = true;
    rng = pcg_hash(rng);
    if (u01(rng) >= S.att_break[r]) continue;
    rng = pcg_hash(rng);
    if (u01(rng) >= S.acc_break[r]) continue;
    slots[3 * k + s] = NONE;
    for (int t = 0; t < 3; ++t) {
      if (atomicCAS(&slots[3 * ps + t], gi, NONE) == gi) break;
    }
    atomicAdd(&events[2 * SOUP_MAX_RULES * sysid[k] + 2 * r + 1], 1u);
  }
  if (touched) brng[k] = rng;
}

}  // namespace

void launch_bonds(Batch& b) {
  b.launches += 5;
  prof_begin(b, SOUP_K_BONDS);
  cudaMemsetAsync(b.bond_nitems, 0, 3 * sizeof(uint32_t), b.stream);
  cudaMemsetAsync(b.has_item, 0, sizeof(uint32_t) * b.N, b.stream);
  uint32_t* has_item = b.has_item;
  k_bond_select<<<nblocks(b.N, 256), 256, 0, b.stream>>>(b.shared, b.N, b.pos, b.center, b.bond_sel,
                                                         b.bond_nitems + 2);
  k_bond_walk<<<nblocks(b.N, 128), 128, 0, b.stream>>>(b.shared, b.sp, b.sysid, b.bond_sel, b.bond_nitems + 2, b.pos,
                                                       b.id, b.slots, b.center, b.nl, b.nl_cnt, b.list_cap, b.brng,
                                                       b.bond_items, b.bond_nitems, has_item);
  cudaMemcpyAsync(b.bond_nitems + 1, b.bond_nitems, sizeof(uint32_t), cudaMemcpyDeviceToDevice, b.stream);
  k_bond_partners<<<std::max(1u, std::min(nblocks(b.N, 256) / 8u, 592u)), 256, 0, b.stream>>>(
      b.center, b.slot_of, b.bond_items, b.bond_nitems, b.N, has_item, b.flags);
  k_bond_claims<<<b.R, 1024, 0, b.stream>>>(b.shared, b.sp, b.sysid, b.pos, b.slots, b.center, b.held, b.slot_of,
                                            b.bond_items, b.bond_nitems, b.N, b.uf_parent, b.comp_min, b.item_done,
                                            b.events, b.desorb);
  k_bond_break<<<nblocks(b.N), kBlock, 0, b.stream>>>(b.shared, b.sysid, b.N, b.pos, b.id, b.slot_of, b.slots,
                                                      b.brng, b.events);
  prof_end(b);
}

}  // namespace soup

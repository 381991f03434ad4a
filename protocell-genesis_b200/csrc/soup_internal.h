// soup_internal.h -- host-side device state of a batch of soup systems and the kernel launchers.
//
// A single SoupHandle is a batch of one.  All replicas of a batch share one set of device arrays:
// particles of replica r occupy slots [slot_off_r, slot_off_r + n_r), and every kernel covers the
// whole batch in one launch, reading the replica's parameters through a static per-slot system id.
//
// Layout in HBM ("slot" order = cell-sorted at the last rebuild, deterministic inside a cell by
// original index):
//   pos    float4  x, y, z, kind          vel, force float4 (w = 0)
//   charge float                          slots  u32 x3  partner ORIGINAL (global) ids
//   center u32 ORIGINAL id                held, bond_rng, thermo_rng u32;  frozen u8
//   id     u32 slot -> original id        slot_of u32 original id -> slot
//   pos_ref float4 positions at the last rebuild (drift reference)
//   nl     u32 [slot][list_cap] Verlet neighbours as SLOT indices; nl_cnt u32 [slot]; each row is
//          grouped by build distance (shell 0: inside the force's reach; shells 1-4: the skin in four
//          equal widths), nl_shell uint4 [slot] the ends of shells 0..3
//   heads  u32 original ids of titratable beads (ascending; static);  es_nl [head][es_cap] slots
#pragma once
#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/soup_b200.h"
#include "soup_common.cuh"

namespace soup {

// flags[0] list overflow, [1] head-list overflow, [6] bond item overflow; per-replica non-finite
// counters (positions, velocities) start at flags[kFlagWords].
constexpr uint32_t kFlagWords = 16;

template <class T> struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
};

// The state of one differentiable window (soup_diff_forward / soup_diff_backward): checkpoints in
// original order, the arrays that stay constant inside the window, and the reverse-pass scratch.
struct DiffWindow {
  uint32_t steps = 0, every = 0;
  uint32_t stride = 1;                   // the caller's frames: every stride-th step (0, stride, ..)
  uint64_t step0 = 0;
  bool ready = false;
  // per checkpoint, per replica: positions, velocities, thermostat states in original order
  std::vector<std::vector<std::vector<float>>> ck_pos, ck_vel;
  std::vector<std::vector<std::vector<uint32_t>>> ck_trng;
  // per replica, fixed over the window
  std::vector<std::vector<float>> charge;
  std::vector<std::vector<uint32_t>> slots, center, held, brng, frozen;
  std::vector<std::vector<float>> end_pos, end_vel;
  std::vector<std::vector<uint32_t>> end_trng;
  uint64_t end_step = 0;
  std::vector<uint32_t> prot_rng;
  bool stored = false;                  // every frame kept on the device (no checkpoints, no replay)
  float4* all = nullptr;                 // (steps + 1) frames in original order when stored
  size_t all_cap = 0;
  float4 *frames = nullptr, *A = nullptr, *B = nullptr, *g = nullptr, *jg = nullptr;
  uint8_t* frozen_o = nullptr;
  double* partial = nullptr;
  size_t frames_cap = 0, partial_cap = 0;
};

struct Batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  uint32_t R = 0;                    // replicas
  uint32_t N = 0;                    // total particles
  std::vector<SoupConfig> cfg;       // per replica
  std::vector<SysParams> hsp;        // per replica (host copy)
  Shared hs{};                       // batch-wide constants (host copy)
  SysParams* sp = nullptr;           // device copy
  Shared* shared = nullptr;          // device copy
  uint8_t* sysid = nullptr;          // per slot (static: slots never leave their replica's range)

  // particle state (double-buffered for the re-sort gather)
  float4 *pos = nullptr, *vel = nullptr, *force = nullptr, *pos_ref = nullptr;
  float* charge = nullptr;
  uint32_t *slots = nullptr, *center = nullptr, *held = nullptr, *brng = nullptr, *trng = nullptr;
  uint8_t* frozen = nullptr;
  uint32_t *id = nullptr, *slot_of = nullptr;
  float4 *pos2 = nullptr, *vel2 = nullptr, *force2 = nullptr;
  float* charge2 = nullptr;
  uint32_t *slots2 = nullptr, *center2 = nullptr, *held2 = nullptr, *brng2 = nullptr, *trng2 = nullptr;
  uint8_t* frozen2 = nullptr;
  uint32_t* id2 = nullptr;

  // grid + list
  uint32_t ncells = 0;               // total list-build cells over the batch
  uint32_t *cell_of_slot = nullptr, *cell_count = nullptr, *cell_start = nullptr, *cell_cursor = nullptr;
  uint8_t* cell_sys = nullptr;       // replica of each list-build cell
  bool list_by_cell = false;         // every replica's walk fits its grid: the cell-group build can run
  bool list_cells = false;           // use it (the autotuner's choice; SOUP_LIST_BY_CELL=1)
  uint32_t* perm = nullptr;          // new slot -> old slot
  uint32_t* scan_tmp = nullptr;
  uint32_t list_cap = 0;             // row stride of nl (max over replicas, rounded to 32)
  uint32_t* nl = nullptr;
  uint32_t* nl_cnt = nullptr;
  uint4* nl_shell = nullptr;
  size_t group_smem_set = 0;         // dynamic shared memory k_group_rows was opened to
  bool prune = true;                 // force passes read only the shells the drift can have brought in range         // per slot: ends of the row's build-distance shells 0..3 (shell 4 ends at nl_cnt)

  // heads / long-range electrostatics
  uint32_t H = 0;                    // total heads
  uint32_t* heads = nullptr;         // global original ids, per replica ascending
  uint32_t* head_sys = nullptr;      // replica of each head
  uint32_t* head_slot = nullptr;     // current slot of each head (refreshed at every rebuild)
  long long* head_e = nullptr;       // constant-pH site energy per head, fixed point 2^-40 (sweep scratch)
  float4* head_pos = nullptr;        // head positions gathered for the sweep
  float4* head_xq = nullptr;         // head positions and charges by head index, for the far half
  long long* head_d = nullptr;       // [head][es_cap] change of a list neighbour's energy when the head
                                     // deprotonates, fixed point 2^-40 (sweep scratch)
  uint8_t* head_flag = nullptr;      // charge state per head when the sweep cannot keep it in shared memory
  uint32_t* draw_site = nullptr;     // the site each draw of a sweep's stream selects (sweep scratch)
  long long* sweep_band = nullptr;   // [draw][64] changes of the next 63 draws' site energies (sweep scratch)
  uint32_t es_cap = 0;
  uint32_t* es_nl = nullptr;
  uint32_t* es_cnt = nullptr;
  uint32_t nhcells = 0;
  uint32_t *hcell_count = nullptr, *hcell_start = nullptr, *hcell_cursor = nullptr, *hsorted = nullptr;
  float4* hsorted_xg = nullptr;      // the heads in head-cell order: position, head index as w bits
  uint32_t* hcell_of = nullptr;

  // counters and flags (device): [0] list overflow, [1] es overflow, [2..3] nonfinite pos/vel,
  // [4] drift^2 bits max (global), [5] rebuild request, [6] timeout flag, [7..] per-replica events
  uint32_t* flags = nullptr;
  uint32_t* events = nullptr;        // per replica: 2*SOUP_MAX_RULES
  uint32_t* desorb = nullptr;        // per replica: 2
  uint32_t* drift_bits = nullptr;    // per replica max drift^2 bits

  // bond pass scratch
  uint32_t* bond_items = nullptr;    // item records
  uint32_t* bond_nitems = nullptr;
  uint32_t* bond_sel = nullptr;      // the active beads of a bond pass, compacted
  uint32_t* uf_parent = nullptr;     // per original id
  uint32_t* comp_min = nullptr;      // per original id
  uint8_t* item_done = nullptr;
  uint32_t* has_item = nullptr;

  // constant-pH sweep scratch / host state
  std::vector<uint32_t> prot_rng;    // per replica
  double* sweep_out = nullptr;       // per replica: attempts, accepted, dEsSum, dEsCount
  uint32_t* prot_rng_dev = nullptr;

  // analysis scratch: one buffer that grows to the largest request of the analysis calls and is
  // reused after that (analysis_scratch), so a call makes no cudaMalloc / cudaFree once its sizes
  // have been seen
  std::vector<double> wall_r0, wall_box0;   // per replica: the wall radius at creation and the box x it
                                            // belongs to (the live radius scales with the box)
  char* an_buf[2] = {nullptr, nullptr};   // [1]: a second buffer for sizes known only mid-call
  size_t an_cap[2] = {0, 0};

  // host-side schedule
  std::vector<uint64_t> step;        // per replica global step
  std::vector<uint64_t> next_sweep;
  uint64_t rebuilds = 0, sweeps = 0;
  bool force_fresh = false;          // force array matches positions+charges+lists
  int tpp = 4;                       // threads per particle in the list force
  bool queued = false;               // list force with the in-range pairs compacted per warp (k_force_w)
  uint32_t wait_limit = 0;           // polls of a bounded device-side handoff before it gives up (0: default)
  DiffWindow diff;
  // captured step chunks (CUDA graphs), keyed by length and schedule phase; the drift-triggered
  // rebuild is a conditional node whose condition a one-thread kernel sets
  struct ChunkGraph { uint64_t key; cudaGraphExec_t exec; uint64_t launches, rebuilds_fixed; };
  std::vector<ChunkGraph> graphs;
  bool graphs_enabled = true;
  cudaStream_t cap_stream = nullptr;     // captures the rebuild body
  uint64_t body_launches = 0;            // kernels in one rebuild body
  uint32_t* rebuild_count = nullptr;     // device: rebuilds the conditional nodes took
  uint32_t rebuild_count_seen = 0;
  std::string err;
  std::vector<SoupHandle*> views;    // per-replica handle views
  // charge locality: only the charged kind is in the polar class (batch-wide), and per replica the
  // kinds (host copy, static) and whether any other kind carries a charge; when no replica does,
  // a charge sweep changes the forces on the heads alone
  bool polar_is_charged_kind = false;
  std::vector<std::vector<uint8_t>> kinds;
  std::vector<uint8_t> off_head_charge;

  // measurement: launch counter and optional per-group event timing
  uint64_t launches = 0;
  bool prof = false;
  struct Mark { cudaEvent_t a, b; int k; };
  std::vector<Mark> marks;
  std::vector<cudaEvent_t> event_pool;
  double kt_ms[SOUP_K_COUNT] = {};
  uint64_t kt_n[SOUP_K_COUNT] = {};
};

// bracket one launch group with events when profiling is on
void prof_begin(Batch& b, int k);
void prof_end(Batch& b);
void prof_flush(Batch& b);

}  // namespace soup

struct SoupHandle {
  soup::Batch* b = nullptr;
  uint32_t r = 0;
  bool owns = false;
  std::string err;
};
struct SoupBatch {
  soup::Batch* b = nullptr;
};

namespace soup {
// kernel launchers (kernels_*.cu)
void launch_cell_index(Batch& b);
void launch_sort_and_gather(Batch& b);
void launch_build_lists(Batch& b);
void launch_build_es_lists(Batch& b);
void launch_force(Batch& b);       // list force, then the far electrostatics half
void launch_force_list(Batch& b, bool heads = false);
void launch_force_heads(Batch& b);  // the heads' list force and far half only (after a charge sweep)
void launch_es_far(Batch& b);
void launch_force_brute(Batch& b);
void launch_kick_drift(Batch& b);
void launch_kick_thermo(Batch& b);
void launch_thermo_drift(Batch& b);   // the thermostat kick of one step + the kick and drift of the next
void launch_rebuild_decide(Batch& b, cudaGraphConditionalHandle h);
void launch_max_drift(Batch& b);
void launch_nonfinite(Batch& b);
void launch_relax_step(Batch& b, float d);
void launch_bonds(Batch& b);
void launch_sweep(Batch& b, uint32_t replica);
size_t sweep_band_rows(const Batch& b);
uint32_t sweep_max_heads();   // heads one replica may hold for the device constant-pH sweep
size_t sweep_draw_sites(const Batch& b);
void adj_unpermute(Batch& b, float4* dst);
void adj_scatter_pos(Batch& b, const float4* src);
void adj_hvp(Batch& b, const float4* g, float4* jg, double* partial_dev);
void adj_theta_sum(Batch& b, const double* partial_dev, double* theta);
size_t adj_partial_count(const Batch& b);
void adj_update(Batch& b, uint32_t n, float4* A, float4* B, const float4* jg, const float4* ldx, const uint8_t* frozen_o,
                float a, float dt, float coef, float4* g, float4* xout);
void sweep_prepare(Batch& b);
void launch_rebuild_check(Batch& b);
// analysis
int run_closure(Batch& b, uint32_t r, const uint32_t* mem, uint32_t nm, const uint32_t* wat, uint32_t nw,
                const double centre[3], double cell, double radius, double vmin, const double* parcel,
                SoupClosureResult* out, std::string& err);
int run_amphiphiles(Batch& b, uint32_t r, uint32_t* head_of, uint32_t* n_out, std::string& err);
// Offsets of the sub-buffers of one analysis call inside the batch's analysis scratch (256-byte
// aligned), and the scratch itself, grown to `bytes` when it is smaller.
struct ScratchLayout {
  size_t used = 0;
  template <class T> size_t add(size_t n) {
    const size_t at = (used + 255) & ~size_t(255);
    used = at + (n > 0 ? n : 1) * sizeof(T);
    return at;
  }
};
char* analysis_scratch(Batch& b, size_t bytes, int which = 0);
// scaleMoleculesRigid (soup/src/soup-box-scale-math.ts:63-138) on the device over original-order
// arrays: n positions pos_o (device), the rigid edges as flat (i, j) pairs (edges_host on the host, or
// NULL with bond partners slots_o (device, u32 x3, NONE = empty) and, when cohesion > 0, the
// proximity pairs within `cohesion` among the beads eligible_host marks (NULL: all)).  Writes out_o
// (device).  With `check`, an edge whose minimum-image length moved by more than 1e-3 makes it return
// SOUP_E_STATE with the reference's message in err (applyBoxScaleOnce's self-check), and out_o is not
// to be used.
int run_rigid_map(Batch& b, const float4* pos_o, const uint32_t* slots_o, uint32_t n, const uint32_t* edges_host,
                  uint64_t n_edges_host, double cohesion, const uint8_t* eligible_host, const double old_box[3],
                  const double new_box[3], float4* out_o, bool check, std::string& err);
int run_profile_z(Batch& b, uint32_t r, uint32_t bins, uint32_t head_mask, uint32_t* head, uint32_t* tail,
                  uint32_t* escaped, std::string& err);
int run_pairing(Batch& b, uint32_t r, double contact, uint32_t out5[5], std::string& err);
int run_unwrap(Batch& b, uint32_t r, const uint32_t* members, uint32_t m, float* out, std::string& err);
// frame_box null: localCavityVolume's padded frame around the positions; otherwise the grid of
// that box (closure.ts dimsFor + occupancy + enclosedVolume), positions taken as given
int run_local_cavity(Batch& b, const float* positions, uint32_t n, double cell, double radius, double* volume,
                     std::string& err, const double* frame_box = nullptr);
int run_shapes(Batch& b, uint32_t r, const uint32_t* members_csr, const uint32_t* start, uint32_t ncomp,
               double* out10, std::string& err);
int run_aggregates(Batch& b, uint32_t r, const uint32_t* mem, uint32_t nm, double cutoff, uint32_t* labels,
                   uint32_t* ncomp, std::string& err, bool periodic_z = true);
// host
void host_fresh_state(const SoupConfig& c, float* pos, float* vel, uint32_t* frozen, uint32_t* brng, uint32_t* trng);
void host_initial_charges(const SoupConfig& c, const float* pos, float* charges, uint32_t* prot_rng);
}  // namespace soup

#define SOUP_CUDA_TRY(expr)                                                              \
  do {                                                                                   \
    cudaError_t e_ = (expr);                                                             \
    if (e_ != cudaSuccess) throw soup::CudaError(e_, #expr, __FILE__, __LINE__);         \
  } while (0)

namespace soup {
struct CudaError {
  cudaError_t code;
  std::string msg;
  CudaError(cudaError_t c, const char* expr, const char* file, int line)
      : code(c), msg(std::string(cudaGetErrorString(c)) + " at " + file + ":" + std::to_string(line) + " (" + expr + ")") {}
};
}  // namespace soup

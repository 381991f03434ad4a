/*
 * soup_b200.h -- C ABI of the B200 soup MD step.
 *
 * This is the drop-in boundary under the reference's TypeScript simulation API
 * (nefayran/protocell-genesis, soup/src/soup-types.ts:181-442 `SoupSystem`, created by
 * `createSoup` at soup/src/sim.ts:95).  Every entry point below names the reference member it
 * replaces.  Plain C types only: pointers, sizes, fixed-layout structs; no CUDA or torch types.
 *
 * Conventions
 *  - Every call returns an int status (SOUP_OK = 0).  On failure the handle keeps a message that
 *    soup_last_error() returns; calls that fail before a handle exists leave it in
 *    soup_last_error(NULL).  The wording follows the reference's thrown Errors
 *    (soup/src/soup-health.ts, soup/src/soup-grid-verlet.ts:266-313, soup/src/soup-plan.ts).
 *  - Readbacks write into CALLER-OWNED host buffers, in the ORIGINAL particle order, in the
 *    reference's layouts: positions f32x4 (w = kind index), velocities/forces f32x4 (w = 0),
 *    bond slots u32x3 with 0xFFFFFFFF = empty, everything else one 32-bit word per particle.
 *    `bytes` must equal the exact size of the array; otherwise SOUP_E_ARG.
 *  - A handle is not thread-safe.  Distinct handles may be used concurrently from different
 *    threads; each owns one CUDA stream on the device that was current when it was created.
 */
#ifndef SOUP_B200_H
#define SOUP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SOUP_ABI_VERSION 1u
#define SOUP_NONE 0xFFFFFFFFu
#define SOUP_MAX_KINDS 8
#define SOUP_MAX_RULES 4

/* Status codes (the reference throws Errors; the ABI returns these). */
enum {
  SOUP_OK = 0,
  SOUP_E_ARG = 1,           /* bad argument, size mismatch, NULL pointer */
  SOUP_E_NONFINITE = 2,     /* soup/src/soup-health.ts assertStateFinite */
  SOUP_E_LIST_OVERFLOW = 3, /* soup/src/soup-grid-verlet.ts:270-275 */
  SOUP_E_ES_OVERFLOW = 4,   /* soup/src/soup-grid-verlet.ts:281-291 */
  SOUP_E_DRIFT = 5,         /* soup/src/soup-grid-verlet.ts:301-312 */
  SOUP_E_GEOMETRY = 6,      /* soup/src/soup-plan.ts:76-157 grid / drift-bound refusals */
  SOUP_E_OOM = 7,           /* device allocation failed */
  SOUP_E_TIMEOUT = 8,       /* a bounded device-side wait gave up */
  SOUP_E_CUDA = 9,          /* any other CUDA runtime error */
  SOUP_E_STATE = 10         /* call not allowed in this state (e.g. relax after step 0) */
};

/* Species class (soup/src/soup-attraction.ts speciesClassOf). */
enum { SOUP_CLASS_APOLAR = 0, SOUP_CLASS_POLAR = 1, SOUP_CLASS_SOLVENT = 2, SOUP_CLASS_MINERAL = 3 };

/* Slot role (soup/src/soup-plan.ts slotRole): 0 carbon chain pool, 1 carbon head slot, 2 head. */
enum { SOUP_ROLE_CHAIN = 0, SOUP_ROLE_HEAD_SLOT = 1, SOUP_ROLE_HEAD = 2 };

/*
 * Fully resolved configuration of one system.  The host fills it from data/params.json,
 * data/soup.json and CreateSoupOpts exactly the way the reference fills its uniforms:
 *   Params          engine/wgsl/forces.wgsl:1-10, engine/src/params.ts:33-47
 *   Species/AttrScale soup/wgsl/pair.wgsl:43-62, soup/src/soup-attraction.ts
 *   GridDims / VL   soup/src/soup-plan.ts:121-157, soup/src/sim.ts (deriveListCapacity)
 *   ES / ES2        soup/src/electrostatics.ts:166-274 (makeEsBasis, esUniform, esUniform2)
 *   BondParams      soup/wgsl/bond-common.wgsl:54-80, soup/src/soup-buffers.ts:344-410
 *   WALL            soup/wgsl/wall.wgsl:40, soup/src/soup-confine.ts wallUniformBytes
 * Real numbers are given in double precision (JavaScript numbers); the library rounds to f32
 * wherever the reference uploads a Float32Array, and keeps FP64 where the reference computes on
 * the host in JavaScript doubles (the constant-pH sweep, the closure and aggregate analyses).
 */
typedef struct SoupConfig {
  uint32_t abi_version;            /* must be SOUP_ABI_VERSION */
  uint32_t n;                      /* number of particles (sum of counts) */
  uint32_t n_kinds;                /* monomer kinds, <= SOUP_MAX_KINDS */
  uint32_t seed;                   /* CreateSoupOpts.seed */
  uint32_t counts[SOUP_MAX_KINDS]; /* particles per kind, kinds in data/soup.json order */
  double box[3];                   /* live box, sigma */

  /* Params (data/params.json; kT is CreateSoupOpts.kT) */
  double sigma, epsilon, b_tt, k_fene, r_inf, k_bend, r_bend, wc, kT, gamma, dt;

  /* Species, per kind */
  double radius[SOUP_MAX_KINDS];      /* radiusSigma */
  uint32_t kind_class[SOUP_MAX_KINDS];/* SOUP_CLASS_* */
  double attr_scale[4][4];            /* class-pair attraction depth table */
  double acid_soap_scale;             /* AttrScale.pair.x */

  /* Neighbour grid and Verlet list (soup/src/soup-plan.ts:121-157) */
  double interaction_range;        /* wca_cut(sigma*max radius) + wc */
  double skin;                     /* verletList.skin */
  double list_range;               /* interaction_range + skin */
  uint32_t rebuild_every;          /* verletList.rebuildEvery (fixed-cadence mode) */
  uint32_t rebuild_on_drift;       /* 1: rebuild when max drift > skin/2 (no fixed cadence) */
  uint32_t list_capacity;          /* per-particle list capacity; 0 = library derives it */

  /* Electrostatics (EsBasis, soup/src/electrostatics.ts:77-131) */
  uint32_t es_enabled;
  int32_t charged_kind;            /* titratable kind, -1 = none */
  double charge_deprotonated;
  double es_coeff_a, es_kappa, es_cutoff, es_shift_u, es_shift_f;
  double es_split_radius;          /* = interaction_range */
  double es_list_range;            /* es_cutoff + skin */
  uint32_t es_list_capacity;       /* per-head capacity; 0 = library derives it */
  double pka_intrinsic, ph;
  uint32_t sweep_every;            /* sweepEverySteps */
  uint32_t protonation_rng;        /* PcgState.state of the constant-pH chain */
  double rc_attr;                  /* wca_cut(sigma*b_tt), the acid-soap well onset */

  /* Bond chemistry (BondParams) */
  uint32_t n_rules;
  int32_t rule_kind_a[SOUP_MAX_RULES], rule_kind_b[SOUP_MAX_RULES];
  double attempt_form[SOUP_MAX_RULES], attempt_break[SOUP_MAX_RULES];
  double accept_form[SOUP_MAX_RULES], accept_break[SOUP_MAX_RULES];
  uint32_t requires_catalyst[SOUP_MAX_RULES];
  uint32_t role_a[SOUP_MAX_RULES], role_b[SOUP_MAX_RULES];
  int32_t catalyst_kind;
  uint32_t head_terminal_only, head_chain_capacity;
  uint32_t max_hold_steps, bond_interval;

  /* Confinement wall (0 radius = none) */
  double wall_radius, wall_k;

  /* Schedule (soup/src/soup-integrate.ts:136-175) */
  uint64_t global_step;            /* starting step (resume.globalStep) */
  uint32_t chunk_steps;            /* steps per submission chunk; the reference uses 1000 */
  uint32_t cell_divisor;            /* neighborGrid.cellDivisor: the plan's cell = interaction_range /
                                      this (0 reads as 1); a live box change is refused, as
                                      planSoupGrid refuses it, when the plan's grid is too small */
  uint32_t reserved[6];
} SoupConfig;

/* Initial state: the resume arrays of CreateSoupOpts.resume (soup/src/soup-types.ts:145-178) plus
 * the frozen flags.  Any pointer may be NULL, in which case the fresh-creation value is used
 * (soup/src/soup-init-state.ts:58-307, soup/src/soup-protonation.ts:38-49). */
typedef struct SoupInitState {
  const float* positions;       /* f32 x4 */
  const float* velocities;      /* f32 x4 */
  const uint32_t* bond_slots;   /* u32 x3 */
  const uint32_t* center_link;  /* u32 */
  const uint32_t* center_held;  /* u32 */
  const uint32_t* bond_rng;     /* u32 */
  const uint32_t* thermo_rng;   /* u32 */
  const float* charges;         /* f32 */
  const uint32_t* frozen;       /* u32 */
  const uint32_t* events;       /* u32 x (2*n_rules): bond, break per rule */
  const uint32_t* desorb_events;/* u32 x2: stretch, timeout */
} SoupInitState;

/* Result of one constant-pH sweep (soup/src/electrostatics.ts:317-326 SweepResult). */
typedef struct SoupSweepResult {
  uint32_t attempts, accepted, heads, deprotonated;
  double alpha;
  double d_es_mean_kt;
} SoupSweepResult;

/* Result of the closure flood fill (soup/src/water-closure.ts:198-245 EncapsulatedWaterResult). */
typedef struct SoupClosureResult {
  uint32_t encapsulated_count, total_water;
  double bulk_water_density;
  double threshold_count;       /* NaN when no bulk water was reached */
  uint32_t closed;
  uint32_t total_empty_cells, unreached_cells;
  uint32_t seed_cell;
  double seed_dist_from_centre;
} SoupClosureResult;

/* Handle state summary. */
typedef struct SoupInfo {
  uint32_t n;
  uint64_t global_step;
  uint32_t list_capacity, es_list_capacity, heads;
  uint64_t rebuilds, sweeps;
  double box[3];
  double max_drift;             /* sqrt of the last measured max drift^2 */
} SoupInfo;

typedef struct SoupHandle SoupHandle;
typedef struct SoupBatch SoupBatch;

/* ---- lifecycle ------------------------------------------------------------------------------ */

/* createSoup (soup/src/sim.ts:95): allocates device state, uploads `init` (NULL = fresh lattice),
 * runs the priming rebuild + force pass (sim.ts:396-408).  Device = the current CUDA device. */
int soup_create(const SoupConfig* cfg, const SoupInitState* init, SoupHandle** out);
/* SoupSystem.dispose (soup/src/soup-types.ts:441). */
void soup_destroy(SoupHandle* h);
/* Message of the last failed call on `h` (NULL: the last failure with no handle). */
const char* soup_last_error(const SoupHandle* h);
int soup_get_info(SoupHandle* h, SoupInfo* out);

/* Fresh-creation arrays on the host: buildInitialState (soup/src/soup-init-state.ts:58-307) and
 * initialCharges (soup/src/soup-protonation.ts:38-49).  Any output pointer may be NULL. */
int soup_fresh_state(const SoupConfig* cfg, float* positions, float* velocities, uint32_t* frozen,
                     uint32_t* bond_rng, uint32_t* thermo_rng);
int soup_initial_charges(const SoupConfig* cfg, const float* positions, float* charges,
                         uint32_t* protonation_rng);

/* ---- stepping ------------------------------------------------------------------------------- */

/* SoupSystem.step(n) (soup/src/soup-integrate.ts:136-175): the same global-step schedule
 * (rebuild on step % rebuild_every == 0 or on half-skin drift, bonds on step % bond_interval == 0,
 * guards and the constant-pH sweep at chunk boundaries). */
int soup_step(SoupHandle* h, uint64_t n);
/* relaxColdStart (soup/src/soup-relax.ts:113-185): capped steepest descent, only at step 0.
 * out2 receives {maxForceBefore, maxForceAfter}; may be NULL. */
int soup_relax_cold_start(SoupHandle* h, uint32_t iterations, double max_displacement_sigma,
                          double* out2);

/* ---- readbacks (soup/src/soup-readback.ts:13-190) ------------------------------------------- */
int soup_read_pos(SoupHandle* h, void* dst, size_t bytes);          /* particles()    */
int soup_read_vel(SoupHandle* h, void* dst, size_t bytes);          /* velocities()   */
int soup_read_force(SoupHandle* h, void* dst, size_t bytes);        /* forcesNoRebuildDEBUG() */
int soup_forces(SoupHandle* h, void* dst, size_t bytes);            /* forces(): rebuild + force */
int soup_forces_brute(SoupHandle* h, void* dst, size_t bytes);      /* forcesBruteForce() */
int soup_read_slots(SoupHandle* h, void* dst, size_t bytes);        /* bondSlots()    */
int soup_read_center_link(SoupHandle* h, void* dst, size_t bytes);  /* centerLinks()  */
int soup_read_center_held(SoupHandle* h, void* dst, size_t bytes);  /* centerHeldSteps() */
int soup_read_charges(SoupHandle* h, void* dst, size_t bytes);      /* charges()      */
int soup_read_rng_bond(SoupHandle* h, void* dst, size_t bytes);     /* rngState().bond */
int soup_read_rng_thermo(SoupHandle* h, void* dst, size_t bytes);   /* rngState().thermo */
int soup_read_frozen(SoupHandle* h, void* dst, size_t bytes);       /* frozen()       */
int soup_read_events(SoupHandle* h, void* dst, size_t bytes);       /* events(): u32 x 2*n_rules */
int soup_read_desorb(SoupHandle* h, void* dst, size_t bytes);       /* desorbEvents(): u32 x2 */
/* nonFiniteCount() (soup/src/soup-health.ts scanNonFinite): out2 = {pos, vel} components. */
int soup_nonfinite_count(SoupHandle* h, uint32_t* out2);
/* The Verlet list of every particle as ORIGINAL indices: counts u32[n] and, when `lists` is not
 * NULL, each particle's neighbours sorted ascending in a CSR layout (offsets = prefix of counts).
 * `lists_cap` is the element capacity of `lists`.  Diagnostic/parity access. */
int soup_read_verlet(SoupHandle* h, uint32_t* counts, uint32_t* lists, size_t lists_cap);
/* The long-range (head) list of every titratable head, the heads in ascending original index: counts
 * u32[heads] and, when `lists` is not NULL, each head's neighbours as ORIGINAL particle indices sorted
 * ascending in a CSR layout (soup/wgsl/electrostatics-long.wgsl:31-56 esList, read back as sets).
 * `lists_cap` is the element capacity of `lists`.  Diagnostic/parity access. */
int soup_read_es_list(SoupHandle* h, uint32_t* counts, uint32_t* lists, size_t lists_cap);
/* Protonation chain state (SoupSystem.protonationRngState). */
int soup_read_protonation_rng(SoupHandle* h, uint32_t* out);

/* ---- checkpoint payload (soup/src/checkpoint.ts:176-214 encodeCheckpoint) --------------------
 * Every array encodeCheckpoint reads, in ONE call: the device gathers them into original particle
 * order and the host waits once.  `dst` receives, back to back, in CheckpointFile's field order and
 * the readback layouts above:
 *   positions f32 x4 | velocities f32 x4 | bondSlots u32 x3 | centerLink u32 | centerHeldSteps u32 |
 *   bondRng u32 | thermoRng u32 | charges f32
 * = SOUP_CHECKPOINT_BYTES_PER_PARTICLE * n bytes (`bytes` must equal that).  `scalars` (may be NULL)
 * receives the rest of the file's state.  A pure readback: the trajectory is unchanged. */
#define SOUP_CHECKPOINT_BYTES_PER_PARTICLE 64
typedef struct SoupCheckpointScalars {
  uint64_t global_step;           /* globalStep */
  uint32_t n;                     /* N */
  uint32_t n_rules;               /* rules whose counters fill events[0 .. 2*n_rules) */
  uint32_t protonation_rng;       /* protonationRng */
  uint32_t desorb[2];             /* desorbEvents: stretch, timeout */
  uint32_t events[2 * SOUP_MAX_RULES]; /* events: bond, break per rule */
  double live_box[3];             /* liveBox */
} SoupCheckpointScalars;
int soup_read_checkpoint(SoupHandle* h, void* dst, size_t bytes, SoupCheckpointScalars* scalars);

/* ---- box scale (soup/src/soup-box-scale.ts:81-165 applyBoxScaleOnce) -------------------------
 * One box change of a live system: every rigid unit (a connected component of the covalent bonds,
 * plus, when cohesion_cutoff > 0, of the proximity pairs within that cutoff among cohesion_members,
 * or among all beads when that is NULL) keeps its internal offsets, and its centre of mass scales
 * with the box (scaleMoleculesRigid, soup/src/soup-box-scale-math.ts:63-138).  Then the live box,
 * grid and wall radius change, the lists are rebuilt and the force recomputed, and the finiteness
 * and list guards run.  Refused (SOUP_E_STATE, state unchanged) with the reference's message when a
 * rigid edge's length moves by more than 1e-3 or the system has immobile (mineral) beads.
 * Velocities are not changed.  The ramp (scaleBoxTo, growBoxTo) is the caller's loop. */
int soup_scale_box(SoupHandle* h, const double target_box[3], double cohesion_cutoff,
                   const uint32_t* cohesion_members, uint32_t n_members);
/* scaleMoleculesRigid alone, on h's device, over caller arrays: n positions (f32 x4), n_edges rigid
 * edges as (i, j) pairs; out receives the positions in new_box (f32 x4, w copied). */
int soup_scale_molecules_rigid(SoupHandle* h, const float* positions, uint32_t n, const uint32_t* edges,
                               uint32_t n_edges, const double old_box[3], const double new_box[3], float* out);

/* ---- writes --------------------------------------------------------------------------------- */
/* writeBuffer(chargeBuf) (soup/src/soup-protonation.ts:60); marks forces stale. */
int soup_write_charges(SoupHandle* h, const float* src, size_t bytes);
/* Live box change (soup/src/soup-box-scale.ts resizeSoupGrid); positions are not moved, the wall
 * radius follows the box (liveRadius, soup/src/soup-confine.ts:76-78). */
int soup_set_box(SoupHandle* h, const double box[3]);

/* ---- autotuning (no reference counterpart) ----------------------------------------------------
 * Picks, for the handle's whole batch, the block shape of the list force (1, 2, 4 or 8 lanes per
 * particle, with the pair maths in the screening loop or the in-range pairs queued; timed on the force), the neighbour-cell size (list-walk radius 2 or 3, timed on the
 * list build) and, with drift-triggered rebuilds, the Verlet skin (0.6, 0.8 or 1.0 of the planned
 * skin, which sized the list capacity; timed on `steps` whole steps).  The choice stays in effect.
 * The state is restored afterwards: positions, velocities, charges, bonds, RNG states, event
 * counters and the step schedule are as they were, and the particles are re-sorted, so later forces
 * agree with an untuned run to FP32 rounding.  steps = 0 tunes the block shape and the cell size
 * only: the skin stays as planned and the ms_per_step fields are 0. */
typedef struct SoupTuneResult {
  uint32_t tpp, walk;             /* chosen lanes per particle, list-walk radius */
  uint32_t tpp_before, walk_before;
  double skin_scale;              /* chosen skin / planned skin */
  double ms_per_step_before, ms_per_step_after;
  uint32_t queued, queued_before; /* list-force variant: 0 pair maths in the screening loop (tpp lanes per
                                     particle), 1 each warp's in-range pairs compacted and evaluated with
                                     every lane busy (one lane per particle; the same result bits as
                                     variant 0 with tpp 1) */
  uint32_t list_cells;            /* list build: 0 a thread per particle, 1 a group of lanes per cell */
} SoupTuneResult;
int soup_autotune(SoupHandle* h, uint32_t steps, SoupTuneResult* out);
/* Apply a tuning found before (by soup_autotune on a system of the same shape) without timing
 * anything: lanes per particle, the list-force variant, list-walk radius, and the current skin scaled
 * by skin_scale (at most 1: the list capacity was sized for it; drift-triggered rebuilds only).  The
 * lists are rebuilt and the force recomputed.  Only tpp, queued, walk, skin_scale and list_cells are
 * read. */
int soup_apply_tuning(SoupHandle* h, const SoupTuneResult* tuning);
/* soup_step runs chunks of chunkSteps steps (at least 4) as captured CUDA graphs, captured on first
 * use; this captures every chunk graph of the current schedule now, without stepping. */
int soup_prepare_graphs(SoupHandle* h);
/* Replace the whole state (CreateSoupOpts.resume semantics); NULL members keep current values. */
int soup_write_state(SoupHandle* h, const SoupInitState* st);

/* Polls a bounded device-side handoff (the constant-pH walk's flags between the CTAs of its cluster)
 * makes before it gives up and the call returns SOUP_E_TIMEOUT; 0 restores the default (2^25).  It has
 * no counterpart in the reference, whose sweep runs on the host; a small limit makes the failure path
 * testable without faulting the device.  Applies to the handle's whole batch. */
int soup_set_wait_limit(SoupHandle* h, uint32_t polls);

/* ---- Monte Carlo and analysis -------------------------------------------------------------- */
/* protonationSweepDEBUG (soup/src/sim.ts): one constant-pH sweep now on the device, then the
 * rebuild + force recompute (soup/src/soup-protonation.ts:52-77). */
int soup_protonation_sweep(SoupHandle* h, SoupSweepResult* out);

/* encapsulatedWaterVolume (soup/src/water-closure.ts:271-363) on the current positions.
 * member_idx / water_idx are ORIGINAL particle indices; centre from periodicCentreOf. */
int soup_closure(SoupHandle* h, const uint32_t* member_idx, uint32_t n_members,
                 const uint32_t* water_idx, uint32_t n_water, const double centre[3],
                 double cell, double radius, double enclosed_volume_min, SoupClosureResult* out);
/* The same with encapsulatedWaterVolume's `parcel` (water-closure.ts:280-288, 323-337): for a finite
 * parcel in a larger box, the reached empty cells the bulk water density is averaged over are the
 * ones whose centre lies within parcel_radius of parcel_centre (no minimum image, as the reference). */
int soup_closure_in_parcel(SoupHandle* h, const uint32_t* member_idx, uint32_t n_members,
                           const uint32_t* water_idx, uint32_t n_water, const double centre[3], double cell,
                           double radius, double enclosed_volume_min, const double parcel_centre[3],
                           double parcel_radius, SoupClosureResult* out);

/* findAmphiphiles (soup/src/amphiphile.ts:55-141) on the current bond graph: head_of[i] = the
 * head index of the amphiphile particle i belongs to, or SOUP_NONE.  n_out = amphiphile count. */
int soup_amphiphile_labels(SoupHandle* h, uint32_t* head_of, uint32_t* n_out);

/* clusterComponents (engine/src/aggregate.ts:201-212) over the member particles (periodic on all
 * three axes, pair joined when r^2 <= cutoff^2): labels[k] = the minimum ORIGINAL index in the
 * component of member_idx[k].  n_components may be NULL. */
int soup_aggregate_labels(SoupHandle* h, const uint32_t* member_idx, uint32_t n_members,
                          double cutoff, uint32_t* labels, uint32_t* n_components);

/* The same labels as soup_aggregate_labels, computed without allocating device memory.  It has no
 * counterpart in the reference.  soup_aggregate_labels allocates its scratch with cudaMalloc and
 * frees it with cudaFree on every call; a caller whose device memory is held by another allocator
 * (a framework's caching allocator that reserved the GPU) may see that cudaMalloc fail, and the
 * cudaFree stalls every stream on the device.  This entry point keeps its scratch in one fixed
 * array that the library holds on each GPU it runs on (about 9.4 MB, for as long as the process
 * lives), so it needs no allocation and no free.
 *   Limits: n_members <= SOUP_NOALLOC_MAX_MEMBERS and floor(box_x/cutoff) * floor(box_y/cutoff)
 *   * floor(box_z/cutoff) <= SOUP_NOALLOC_MAX_CELLS; larger requests return SOUP_E_ARG with the
 *   limit in soup_last_error and compute nothing.
 *   The first call on each device looks up the array's device address (with lazy module loading
 *   this also loads the library's device code); make that first call before capturing any stream.
 *   All handles on one device share the array: calls that can overlap (from several host threads)
 *   must be serialised by the caller.  The call returns after its results are on the host. */
#define SOUP_NOALLOC_MAX_MEMBERS (1u << 18)
#define SOUP_NOALLOC_MAX_CELLS (1u << 18)
int soup_aggregate_labels_noalloc(SoupHandle* h, const uint32_t* member_idx, uint32_t n_members,
                                  double cutoff, uint32_t* labels, uint32_t* n_components);

/* ---- observables ----------------------------------------------------------------------------- */
/* pairingStats (soup/src/electrostatics.ts:520-561): for every titratable head, the like / unlike
 * contacts with the other heads within contact_radius (FP64 distance, JavaScript minimum image) and
 * whether its nearest such head carries the other charge state.  Exact-distance ties for the nearest
 * go to the smaller head index (the reference takes the first in its cell walk).  contact_radius must
 * be below the electrostatics cutoff; the reference passes wca_cut(sigma * head_head). */
typedef struct SoupPairingStats {
  uint32_t heads, with_neighbour, unlike_contacts, like_contacts, paired, charged;
  double unlike_fraction;         /* unlike / (unlike + like) */
  double unlike_fraction_random;  /* 2 alpha (1 - alpha) */
  double paired_fraction;         /* paired / heads */
  double contact_radius;
  double alpha;                   /* charged / heads */
} SoupPairingStats;
int soup_pairing_stats(SoupHandle* h, double contact_radius, SoupPairingStats* out);

/* shapeOf over unwrapAggregate (engine/src/aggregate.ts:245-262, 308-346) for the components named by
 * `labels` (one per member, e.g. from soup_aggregate_labels): components largest first (ties: smaller
 * label first, the order clusterComponents sorts them in), and the first max_shapes of them measured:
 * members unwrapped around the component's smallest original index (periodic on all three axes,
 * stored as f32 as the reference does), centre, and the per-member gyration tensor.
 * n_components receives the number of components. */
typedef struct SoupAggregateShape {
  uint32_t size;                  /* members */
  uint32_t label;                 /* the component's smallest original index */
  double centre[3];               /* centre of the unwrapped members (frame of the label member) */
  double gyration[6];             /* Sxx, Syy, Szz, Sxy, Sxz, Syz */
} SoupAggregateShape;
int soup_aggregate_shapes(SoupHandle* h, const uint32_t* member_idx, const uint32_t* labels, uint32_t n_members,
                          uint32_t max_shapes, SoupAggregateShape* out, uint32_t* n_components);

/* unwrapAggregate (engine/src/aggregate.ts:245-262) of one aggregate: its members (original
 * indices, the first one the reference) unwrapped on all three periodic axes, f32 x4 with w = kind,
 * in the given order.  The frame shapeOfAggregate's head-shell profiles are measured in
 * (soup/src/aggregates.ts:387-476). */
int soup_aggregate_unwrap(SoupHandle* h, const uint32_t* members, uint32_t n_members, float* out);
/* localCavityVolume (soup/src/aggregates.ts:350-385) on h's device: the vacuum cavity enclosed by n
 * unwrapped positions (f32 x4) on a local grid of side `cell` around them (padded by 4 * radius),
 * cells within `radius` of a bead occupied (engine/src/closure.ts:67-107 occupancy), the empty cells
 * the open-boundary flood from the grid's faces does not reach (closure.ts:108-163), times cell^3. */
int soup_local_cavity_volume(SoupHandle* h, const float* positions, uint32_t n, double cell, double radius,
                             double* volume);

/* enclosedVolume (engine/src/closure.ts:51-163: dimsFor, occupancy, floodOutside, enclosedVolume)
 * on the grid of this system's live box: cells of side `cell`, x and y periodic, z open; cells
 * within `radius` of a bead occupied; the empty cells the flood from the grid's faces does not reach,
 * times cell^3.  The positions (f32 x4) are taken as given; enclosedVolumeFromPositions
 * (closure.ts:315-323) recentres them on the largest cluster first, which the caller does with
 * soup_cluster_labels. */
int soup_box_cavity_volume(SoupHandle* h, const float* positions, uint32_t n, double cell, double radius,
                           double* volume);

/* buildClusterUnionFind (engine/src/aggregate.ts:65-130) with its periodicZ switch: labels as
 * soup_aggregate_labels (the minimum original index of each component), x and y periodic, z periodic
 * only when periodic_z is non-zero (largestClusterCenter, aggregate.ts:157-190, clusters with z open).
 * soup_aggregate_labels is this call with periodic_z = 1. */
int soup_cluster_labels(SoupHandle* h, const uint32_t* member_idx, uint32_t n_members, double cutoff, int periodic_z,
                        uint32_t* labels, uint32_t* n_components);

/* densityProfileZ (engine/src/metrics.ts:21-47): histogram of the beads' z over [0, box_z) in
 * `bins` bins, split into heads (kinds whose bit is set in head_kind_mask) and tails (the rest).
 * The soup profiles polar kinds as heads (soup/src/aggregates.ts:95-109); the engine's own
 * convention is kind 0 (mask 1).  A bead outside [0, box_z) makes the call fail as the reference
 * does, unless `escaped` is given: then such beads are left out and counted there (dropEscapedZ,
 * engine/src/metrics.ts:106-121). */
int soup_density_profile_z(SoupHandle* h, uint32_t bins, uint32_t head_kind_mask, uint32_t* head_counts,
                           uint32_t* tail_counts, uint32_t* escaped);

/* ---- differentiation ------------------------------------------------------------------------- */
/* The adjoint of the force + Langevin step.  It has no counterpart in the reference, which only
 * runs the step forward.  The parameters are SOUP_DIFF_NPARAM numbers, in this order:
 *   the class-pair attraction depths A[apolar][apolar], A[apolar][polar], A[apolar][solvent],
 *   A[polar][polar], A[polar][solvent], A[solvent][solvent] (symmetric table, SoupConfig.attr_scale),
 *   k_fene, k_bend, and kappa = 1 / Debye length.  The electrostatics cutoff and the acid-soap depth
 *   stay at their values when kappa changes.  On a batch the parameters are shared by every replica
 *   (which must agree on dt, gamma and, with electrostatics, kappa) and the trajectory, the loss
 *   gradients and dx0 / dv0 hold every replica's particles in the batch's original order; theta_grad
 *   sums the replicas. */
#define SOUP_DIFF_NPARAM 9
int soup_get_diff_params(SoupHandle* h, double* theta);
/* Sets the parameters and recomputes the force at the current positions. */
int soup_set_diff_params(SoupHandle* h, const double* theta);
/* A differentiable window: `steps` steps from the current state with bond Monte Carlo and the
 * constant-pH sweep held off (charges and bonds fixed), a checkpoint every `checkpoint_every` steps
 * (each one re-sorts the particles canonically and recomputes the force, so the reverse pass can
 * replay a segment bit for bit from it).  traj_device (may be NULL): device memory for steps + 1
 * frames of n float4 positions in original order (frame 0 the start), 16-byte aligned. */
int soup_diff_forward(SoupHandle* h, uint32_t steps, uint32_t checkpoint_every, float* traj_device);
/* soup_diff_forward keeping only every frame_stride-th frame for the caller: traj_device holds
 * steps / frame_stride + 1 frames (steps 0, frame_stride, 2 frame_stride, ..), and the reverse pass
 * takes dJ/dx at those frames alone (the loss depends on no other step).  frame_stride must divide
 * steps; 1 is soup_diff_forward.  This is what lets a long window of a large batch fit: the
 * internal replay does not depend on it. */
int soup_diff_forward_strided(SoupHandle* h, uint32_t steps, uint32_t checkpoint_every, uint32_t frame_stride,
                              float* traj_device);
/* The reverse pass of the last soup_diff_forward(_strided).  dldx_device: dJ/dx_t for the kept frames
 * (t = 0, frame_stride, .., steps: steps / frame_stride + 1 frames) of n float4 in original order
 * (w ignored), device memory.  theta_grad receives dJ/dtheta
 * (SOUP_DIFF_NPARAM doubles, host); dx0_device / dv0_device (device, n float4, may be NULL) receive
 * dJ/dx_0 and dJ/dv_0.  The Langevin noise is fixed by the window's seeds (the adjoint does not depend
 * on it).  The system is left at the window's end state.  The sensitivity of a chaotic window grows
 * exponentially with its length: SOUP_E_NONFINITE when a parameter gradient is no longer finite (the
 * FP32 adjoint state overflowed; theta_grad still receives the sums). */
int soup_diff_backward(SoupHandle* h, const float* dldx_device, double* theta_grad, float* dx0_device,
                       float* dv0_device);

/* ---- single phases ------------------------------------------------------------------------- */
/* One phase of the step on the current device state, so each kernel can be checked in isolation
 * (the reference times phases the same way: stepPhasesDEBUG, soup/src/soup-readback.ts:191-245).
 *   REBUILD     encodeVerletRebuild (soup/src/soup-grid-verlet.ts:236-248)
 *   FORCE       encodeSoupForceList: list force + far ES + wall (soup/src/soup-integrate.ts:64-71)
 *   KICK_DRIFT  kick_drift_wrap_main (soup/wgsl/step.wgsl:96)
 *   KICK_THERMO kick_thermostat_main (soup/wgsl/step.wgsl:110)
 *   BONDS       bond formation then breaking (soup/src/soup-bond-chemistry.ts)
 *   MAX_DRIFT   soup_max_drift_main (soup/wgsl/verlet.wgsl:113) */
enum {
  SOUP_PHASE_REBUILD = 1, SOUP_PHASE_FORCE = 2, SOUP_PHASE_KICK_DRIFT = 3,
  SOUP_PHASE_KICK_THERMO = 4, SOUP_PHASE_BONDS = 5, SOUP_PHASE_MAX_DRIFT = 6
};
int soup_debug_phase(SoupHandle* h, int phase);

/* ---- measurement hooks (no reference counterpart; the reference times phases by wall clock) --- */
enum {
  SOUP_K_FORCE = 0, SOUP_K_ES_FAR = 1, SOUP_K_LIST = 2, SOUP_K_SORT = 3, SOUP_K_KICK_DRIFT = 4,
  SOUP_K_KICK_THERMO = 5, SOUP_K_BONDS = 6, SOUP_K_SWEEP = 7, SOUP_K_COUNT = 8
};
/* The cudaStream_t this handle launches on, so a caller can record CUDA events on it. */
void* soup_stream(SoupHandle* h);
/* enable = 1: bracket the kernels of each SOUP_K_* group with CUDA events on the handle's stream. */
int soup_profile(SoupHandle* h, int enable);
/* Device milliseconds and launches of one SOUP_K_* group since profiling was last enabled. */
int soup_kernel_time(SoupHandle* h, int kernel, double* total_ms, uint64_t* launches);
/* Kernels this library has launched for the handle's batch since creation. */
uint64_t soup_launch_count(SoupHandle* h);

/* ---- batched replicas (no reference counterpart: one system per device there) -------------- */
/* Many independent systems of uneven size stepped together: one launch per kernel per step covers
 * every replica.  cfgs[r] / inits[r] as for soup_create (inits may be NULL). */
int soup_batch_create(const SoupConfig* cfgs, const SoupInitState* inits, uint32_t n_replicas,
                      SoupBatch** out);
int soup_batch_step(SoupBatch* b, uint64_t n);
/* Borrowed per-replica handle for readbacks; valid until soup_batch_destroy. */
SoupHandle* soup_batch_replica(SoupBatch* b, uint32_t r);
const char* soup_batch_last_error(const SoupBatch* b);
void soup_batch_destroy(SoupBatch* b);

#ifdef __cplusplus
}
#endif
#endif /* SOUP_B200_H */

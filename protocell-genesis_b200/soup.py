"""SoupSystem: the reference's simulation API (soup/src/soup-types.ts:181-442) over the C ABI.

Every method calls libsoup_b200.so; arrays come back in the reference's layouts and original
particle order.  Method names follow the reference (camelCase aliases are provided for the ones
soup/cli/campaign.ts and verify/ use).
"""
import ctypes as C
import math
from typing import Dict, Optional

import numpy as np

from . import _abi
from . import config as _config


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def _check(lib, h, st):
    if st != 0:
        raise _abi.SoupError(st, lib.soup_last_error(h).decode())


# values per particle of each SoupInitState array (events and desorb_events are per system)
_PER = {"positions": 4, "velocities": 4, "bond_slots": 3, "center_link": 1, "center_held": 1, "bond_rng": 1,
        "thermo_rng": 1, "charges": 1, "frozen": 1, "desorb_events": None, "events": None}


def init_state(st: Optional[dict], cfg=None):
    """SoupInitState from a dict of numpy arrays (CreateSoupOpts.resume field names accepted).  With
    the system's SoupConfig `cfg`, every per-particle array must hold exactly n x its values per
    particle, events 2 x n_rules values and desorb_events two (ValueError otherwise): the library
    reads that many from each pointer."""
    alias = {"positions": "positions", "velocities": "velocities", "bondSlots": "bond_slots",
             "bond_slots": "bond_slots", "centerLink": "center_link", "center_link": "center_link",
             "centerHeldSteps": "center_held", "center_held": "center_held", "bondRng": "bond_rng",
             "bond_rng": "bond_rng", "thermoRng": "thermo_rng", "thermo_rng": "thermo_rng",
             "charges": "charges", "frozen": "frozen", "events": "events", "desorbEvents": "desorb_events",
             "desorb_events": "desorb_events"}
    dtypes = {"positions": np.float32, "velocities": np.float32, "charges": np.float32}
    s = _abi.SoupInitState()
    keep = []
    for k, v in (st or {}).items():
        if k not in alias or v is None:
            continue
        name = alias[k]
        a = np.ascontiguousarray(v, dtype=dtypes.get(name, np.uint32))
        if cfg is not None:
            per = _PER[name]
            want = {"desorb_events": 2, "events": 2 * int(cfg.n_rules)}.get(name)
            if per is not None:
                want = int(cfg.n) * per
            if a.size != want:
                raise ValueError(f"state array {k!r} holds {a.size} values, expected {want}")
        keep.append(a)
        setattr(s, name, a.ctypes.data)
    s._keep = keep
    return s


class SoupSystem:
    """One soup system on the current CUDA device (createSoup, soup/src/sim.ts:95)."""

    def __init__(self, cfg: _abi.SoupConfig, state: Optional[dict] = None, rule_ids=None):
        self._lib = _abi.lib()
        self.cfg = cfg
        self.n = int(cfg.n)
        self.rule_ids = rule_ids or _config.rule_ids()
        h = C.c_void_p()
        st = init_state(state, cfg) if state is not None else None
        rc = self._lib.soup_create(C.byref(cfg), C.byref(st) if st is not None else None, C.byref(h))
        if rc != 0:
            raise _abi.SoupError(rc, self._lib.soup_last_error(None).decode())
        self._h = h
        self._owned = True

    @classmethod
    def _view(cls, lib, handle, cfg, rule_ids):
        self = cls.__new__(cls)
        self._lib = lib
        self.cfg = cfg
        self.n = int(cfg.n)
        self.rule_ids = rule_ids
        self._h = handle
        self._owned = False
        return self

    # ---- lifecycle ----
    def dispose(self):
        if getattr(self, "_h", None) and self._owned:
            self._lib.soup_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.dispose()
        except Exception:
            pass

    def info(self) -> dict:
        i = _abi.SoupInfo()
        _check(self._lib, self._h, self._lib.soup_get_info(self._h, C.byref(i)))
        return dict(n=i.n, global_step=i.global_step, list_capacity=i.list_capacity,
                    es_list_capacity=i.es_list_capacity, heads=i.heads, rebuilds=i.rebuilds, sweeps=i.sweeps,
                    box=tuple(i.box), max_drift=i.max_drift)

    @property
    def steps(self) -> int:
        return self.info()["global_step"]

    @property
    def box(self):
        return self.info()["box"]

    def confinement(self) -> Optional[dict]:
        """confinement() (soup/src/sim.ts:542-556): the parcel derived from the LIVE box (the radius
        scales with box x, soup/src/soup-confine.ts:76-78 liveRadius), or None on a periodic system."""
        r0 = float(self.cfg.wall_radius)
        if not r0 > 0:
            return None
        box = [float(x) for x in self.box]
        box0 = [float(x) for x in self.cfg.box]
        live = r0 * (box[0] / box0[0])
        return {"radiusWet": r0, "radiusLive": live, "stiffness": float(self.cfg.wall_k), "boxWet": box0,
                "boxLive": box, "parcelVolumeLive": 4.0 / 3.0 * math.pi * live ** 3,
                "boxVolumeLive": box[0] * box[1] * box[2], "cutMax": float(self.cfg.interaction_range),
                "clearanceLive": box[0] / 2 - live, "strongNoWrapLive": 2 * live < box[0] / 2}

    # ---- stepping ----
    def step(self, n: int):
        _check(self._lib, self._h, self._lib.soup_step(self._h, int(n)))

    def relax_cold_start(self, iterations: Optional[int] = None, max_displacement_sigma: Optional[float] = None):
        P = _config.load_params()
        it = iterations if iterations is not None else P["coldStartRelax"]["iterations"]
        md = max_displacement_sigma if max_displacement_sigma is not None else P["coldStartRelax"]["maxDisplacementSigma"]
        out = (C.c_double * 2)()
        _check(self._lib, self._h, self._lib.soup_relax_cold_start(self._h, int(it), float(md), out))
        return dict(iterations=it, maxDisplacementStart=md * self.cfg.sigma,
                    displacementBound=md * self.cfg.sigma * (it + 1) / 2,
                    maxForceBefore=out[0], maxForceAfter=out[1])

    relaxColdStart = relax_cold_start

    def debug_phase(self, phase: int):
        _check(self._lib, self._h, self._lib.soup_debug_phase(self._h, int(phase)))

    # ---- readbacks ----
    def _read(self, fn, dtype, per):
        a = np.empty(self.n * per, dtype=dtype)
        _check(self._lib, self._h, getattr(self._lib, fn)(self._h, _ptr(a), a.nbytes))
        return a

    def particles(self):
        return self._read("soup_read_pos", np.float32, 4)

    def velocities(self):
        return self._read("soup_read_vel", np.float32, 4)

    def forces(self):
        """soup/src/soup-readback.ts forces(): rebuild + force pass, then read."""
        return self._read("soup_forces", np.float32, 4)

    def forces_no_rebuild(self):
        return self._read("soup_read_force", np.float32, 4)

    def forces_brute_force(self):
        return self._read("soup_forces_brute", np.float32, 4)

    def bond_slots(self):
        return self._read("soup_read_slots", np.uint32, 3)

    def bonds(self):
        """soup/src/soup-readback.ts:40-50: (i, j) pairs with j > i, in slot order."""
        s = self.bond_slots().reshape(-1, 3)
        out = []
        for i in np.nonzero((s != _abi.NONE).any(axis=1))[0]:
            for j in s[i]:
                if j != _abi.NONE and j > i:
                    out += [i, j]
        return np.asarray(out, dtype=np.uint32)

    def center_links(self):
        return self._read("soup_read_center_link", np.uint32, 1)

    def center_held_steps(self):
        return self._read("soup_read_center_held", np.uint32, 1)

    def charges(self):
        return self._read("soup_read_charges", np.float32, 1)

    def frozen(self):
        return self._read("soup_read_frozen", np.uint32, 1)

    def rng_state(self):
        return dict(bond=self._read("soup_read_rng_bond", np.uint32, 1),
                    thermo=self._read("soup_read_rng_thermo", np.uint32, 1))

    def events(self) -> Dict[str, int]:
        a = np.empty(2 * self.cfg.n_rules, np.uint32)
        _check(self._lib, self._h, self._lib.soup_read_events(self._h, _ptr(a), a.nbytes))
        out = {}
        for r, (b, k) in enumerate(self.rule_ids[: self.cfg.n_rules]):
            out[b] = int(a[2 * r])
            out[k] = int(a[2 * r + 1])
        return out

    def events_raw(self):
        a = np.empty(2 * self.cfg.n_rules, np.uint32)
        _check(self._lib, self._h, self._lib.soup_read_events(self._h, _ptr(a), a.nbytes))
        return a

    def desorb_events(self):
        a = np.empty(2, np.uint32)
        _check(self._lib, self._h, self._lib.soup_read_desorb(self._h, _ptr(a), a.nbytes))
        return dict(stretch=int(a[0]), timeout=int(a[1]))

    def nonfinite_count(self):
        a = (C.c_uint32 * 2)()
        _check(self._lib, self._h, self._lib.soup_nonfinite_count(self._h, a))
        return dict(pos=a[0], vel=a[1])

    def protonation_rng_state(self) -> int:
        v = C.c_uint32()
        _check(self._lib, self._h, self._lib.soup_read_protonation_rng(self._h, C.byref(v)))
        return v.value

    def invariants(self) -> dict:
        """invariants (soup/src/soup-readback.ts:136-152): the live census per monomer id (kind read
        from the position's w, rounded), the bond count, and the summed monomer charge property
        (absent from every monomer of the parameter tables, so 0)."""
        monomers = _config.load_params()["monomers"]
        kinds = np.rint(self.particles().reshape(-1, 4)[:, 3]).astype(np.int64)
        census = np.bincount(kinds, minlength=len(monomers))
        counts = {m["id"]: int(census[k]) for k, m in enumerate(monomers)}
        charge = float(sum(census[k] * float(m.get("charge", 0) or 0) for k, m in enumerate(monomers)))
        return dict(monomers=counts, bonds=int(self.bonds().size // 2), charge=charge)

    def checkpoint_payload(self):
        """Every array and scalar a checkpoint carries, from one soup_read_checkpoint call: a dict of
        numpy arrays in the readback layouts (views of one host buffer) and a dict of scalars."""
        buf = np.empty(_abi.CHECKPOINT_BYTES_PER_PARTICLE * self.n, np.uint8)
        sc = _abi.SoupCheckpointScalars()
        _check(self._lib, self._h, self._lib.soup_read_checkpoint(self._h, _ptr(buf), buf.nbytes, C.byref(sc)))
        n, out, at = self.n, {}, 0
        for name, dt, per in (("positions", np.float32, 4), ("velocities", np.float32, 4), ("bondSlots", np.uint32, 3),
                              ("centerLink", np.uint32, 1), ("centerHeldSteps", np.uint32, 1), ("bondRng", np.uint32, 1),
                              ("thermoRng", np.uint32, 1), ("charges", np.float32, 1)):
            nb = 4 * per * n
            out[name] = buf[at:at + nb].view(dt)
            at += nb
        ev = list(sc.events)[: 2 * sc.n_rules]
        events = {}
        for r, (b, k) in enumerate(self.rule_ids[: sc.n_rules]):
            events[b], events[k] = int(ev[2 * r]), int(ev[2 * r + 1])
        scalars = dict(globalStep=int(sc.global_step), N=int(sc.n), protonationRng=int(sc.protonation_rng),
                       desorbEvents=dict(stretch=int(sc.desorb[0]), timeout=int(sc.desorb[1])), events=events,
                       liveBox=[float(x) for x in sc.live_box])
        return out, scalars

    def verlet_lists(self):
        counts = np.empty(self.n, np.uint32)
        _check(self._lib, self._h, self._lib.soup_read_verlet(self._h, counts.ctypes.data_as(_abi._U32P), None, 0))
        lists = np.empty(int(counts.sum(dtype=np.uint64)), np.uint32)
        _check(self._lib, self._h, self._lib.soup_read_verlet(
            self._h, counts.ctypes.data_as(_abi._U32P), lists.ctypes.data_as(_abi._U32P), lists.size))
        return counts, lists

    def es_lists(self):
        """The long-range head list as sets: (counts per head, CSR of sorted original indices), the
        heads in ascending original index."""
        nh = int(self.info()["heads"])
        counts = np.empty(nh, np.uint32)
        if nh == 0:
            return counts, np.empty(0, np.uint32)
        _check(self._lib, self._h, self._lib.soup_read_es_list(self._h, counts.ctypes.data_as(_abi._U32P), None, 0))
        lists = np.empty(int(counts.sum(dtype=np.uint64)), np.uint32)
        _check(self._lib, self._h, self._lib.soup_read_es_list(
            self._h, counts.ctypes.data_as(_abi._U32P), lists.ctypes.data_as(_abi._U32P), lists.size))
        return counts, lists

    def set_wait_limit(self, polls: int = 0):
        """Polls of the constant-pH walk's bounded handoffs before SOUP_E_TIMEOUT (0: the default)."""
        _check(self._lib, self._h, self._lib.soup_set_wait_limit(self._h, int(polls)))

    # ---- writes ----
    def write_charges(self, q):
        q = np.ascontiguousarray(q, np.float32)
        _check(self._lib, self._h, self._lib.soup_write_charges(self._h, _ptr(q), q.nbytes))

    def write_state(self, state: dict):
        st = init_state(state, self.cfg)
        _check(self._lib, self._h, self._lib.soup_write_state(self._h, C.byref(st)))

    def set_box(self, box):
        b = (C.c_double * 3)(*[float(x) for x in box])
        _check(self._lib, self._h, self._lib.soup_set_box(self._h, b))

    def scale_box_once(self, target_box, cohesion=None):
        """applyBoxScaleOnce (soup/src/soup-box-scale.ts:81-165) on the device: every rigid unit keeps its
        shape while its centre of mass scales with the box.  cohesion: {"cutoff": c, "memberIndices":
        optional indices} also holds beads within c of each other together (the reference's option)."""
        b = (C.c_double * 3)(*[float(x) for x in target_box])
        cut, mem = 0.0, None
        if cohesion is not None:
            cut = float(cohesion["cutoff"])
            if cohesion.get("memberIndices") is not None:
                mem = np.ascontiguousarray(cohesion["memberIndices"], np.uint32)
        _check(self._lib, self._h, self._lib.soup_scale_box(
            self._h, b, cut, mem.ctypes.data_as(_abi._U32P) if mem is not None else None,
            0 if mem is None else mem.size))

    def scale_box_to(self, target_box, ramp_steps: int, ramp_relax_steps: int, cohesion=None):
        """scaleBoxTo (soup/src/soup-box-scale.ts:218-275): `ramp_steps` log-linear box increments, each
        a scale_box_once, with `ramp_relax_steps` steps of dynamics between them (none after the last)."""
        for box in _box_ramp(self.box, target_box, ramp_steps):
            self.scale_box_once(box[0], cohesion)
            if not box[1] and ramp_relax_steps > 0:
                self.step(ramp_relax_steps)

    def grow_box_to(self, target_box, ramp_steps: int, ramp_relax_steps: int):
        """growBoxTo (soup/src/soup-box-scale.ts:318-360): the same ramp, moving no particle: only the
        live box, the grid and the lists change.  The force is recomputed at each new box (the
        reference keeps the previous force for the next half-kick)."""
        for box in _box_ramp(self.box, target_box, ramp_steps):
            self.set_box(box[0])
            if not box[1] and ramp_relax_steps > 0:
                self.step(ramp_relax_steps)

    def scale_molecules_rigid(self, positions, edges, old_box, new_box):
        """scaleMoleculesRigid (soup/src/soup-box-scale-math.ts:63-138) on this system's device over
        caller arrays: positions f32 x4, edges flat (i, j) pairs; returns the positions in new_box."""
        pos = np.ascontiguousarray(positions, np.float32)
        e = np.ascontiguousarray(edges, np.uint32)
        out = np.empty_like(pos)
        ob = (C.c_double * 3)(*[float(x) for x in old_box])
        nb = (C.c_double * 3)(*[float(x) for x in new_box])
        _check(self._lib, self._h, self._lib.soup_scale_molecules_rigid(
            self._h, _ptr(pos), pos.size // 4, e.ctypes.data_as(_abi._U32P), e.size // 2, ob, nb, _ptr(out)))
        return out

    def prepare_graphs(self):
        """Capture the step graphs of the current schedule now (soup_step captures them on first use)."""
        _check(self._lib, self._h, self._lib.soup_prepare_graphs(self._h))

    def autotune(self, steps: int = 20) -> dict:
        """Pick the list force's lanes per particle, the neighbour-cell size and (with drift-triggered
        rebuilds) the skin for this system's whole batch by timing them, keep the choice, and restore
        the state (see soup_autotune in include/soup_b200.h).  steps = 0: the lanes and the cell size
        only, the skin stays as planned."""
        return _autotune(self._lib, self._h, steps)

    def apply_tuning(self, tuning: dict):
        """Apply a result of autotune (tpp, walk, skin_scale) found on a system of the same shape,
        without timing anything (soup_apply_tuning)."""
        _apply_tuning(self._lib, self._h, tuning)

    # ---- Monte Carlo and analysis ----
    def protonation_sweep(self):
        r = _abi.SoupSweepResult()
        _check(self._lib, self._h, self._lib.soup_protonation_sweep(self._h, C.byref(r)))
        return dict(attempts=r.attempts, accepted=r.accepted, heads=r.heads, deprotonated=r.deprotonated,
                    alpha=r.alpha, dEsMeanKT=r.d_es_mean_kt)

    protonationSweepDEBUG = protonation_sweep

    def closure(self, members, water, centre, cell, radius, enclosed_volume_min, parcel=None):
        """encapsulatedWaterVolume (soup/src/water-closure.ts:271-363); parcel: {"centre": [x, y, z],
        "radius": R} restricts the bulk-density cells to a finite parcel (config 5's confined runs)."""
        m = np.ascontiguousarray(members, np.uint32)
        w = np.ascontiguousarray(water, np.uint32)
        c = (C.c_double * 3)(*[float(x) for x in centre])
        r = _abi.SoupClosureResult()
        if parcel is None:
            st = self._lib.soup_closure(self._h, m.ctypes.data_as(_abi._U32P), m.size, w.ctypes.data_as(_abi._U32P),
                                        w.size, c, float(cell), float(radius), float(enclosed_volume_min), C.byref(r))
        else:
            pc = (C.c_double * 3)(*[float(x) for x in parcel["centre"]])
            st = self._lib.soup_closure_in_parcel(self._h, m.ctypes.data_as(_abi._U32P), m.size,
                                                  w.ctypes.data_as(_abi._U32P), w.size, c, float(cell), float(radius),
                                                  float(enclosed_volume_min), pc, float(parcel["radius"]), C.byref(r))
        _check(self._lib, self._h, st)
        return dict(encapsulatedCount=r.encapsulated_count, totalWater=r.total_water,
                    bulkWaterDensity=r.bulk_water_density, encapsulationThresholdCount=r.threshold_count,
                    closed=bool(r.closed), totalEmptyCells=r.total_empty_cells, unreachedCells=r.unreached_cells,
                    seedCell=r.seed_cell, seedDistFromCentre=r.seed_dist_from_centre)

    def amphiphile_labels(self):
        head_of = np.empty(self.n, np.uint32)
        cnt = C.c_uint32()
        _check(self._lib, self._h, self._lib.soup_amphiphile_labels(self._h, head_of.ctypes.data_as(_abi._U32P),
                                                                    C.byref(cnt)))
        return int(cnt.value), head_of

    def aggregate_labels(self, members, cutoff):
        m = np.ascontiguousarray(members, np.uint32)
        labels = np.empty(m.size, np.uint32)
        nc = C.c_uint32()
        _check(self._lib, self._h, self._lib.soup_aggregate_labels(
            self._h, m.ctypes.data_as(_abi._U32P), m.size, float(cutoff), labels.ctypes.data_as(_abi._U32P),
            C.byref(nc)))
        return int(nc.value), labels

    def pairing_stats(self, contact_radius):
        """pairingStats (soup/src/electrostatics.ts:520-561) on the device; keys as the reference's."""
        r = _abi.SoupPairingStats()
        _check(self._lib, self._h, self._lib.soup_pairing_stats(self._h, float(contact_radius), C.byref(r)))
        return dict(heads=r.heads, withNeighbour=r.with_neighbour, unlikeContacts=r.unlike_contacts,
                    likeContacts=r.like_contacts, unlikeFraction=r.unlike_fraction,
                    unlikeFractionRandom=r.unlike_fraction_random, paired=r.paired,
                    pairedFraction=r.paired_fraction, contactRadius=r.contact_radius, alpha=r.alpha)

    def density_profile_z(self, bins, head_kinds=None, drop_escaped=False):
        """densityProfileZ (engine/src/metrics.ts:21-47) of this system's beads on the device:
        {z, head, tail} (+ escaped when drop_escaped).  head_kinds: the kind indices counted as
        heads (default: the polar kinds, as the soup's aggregate stage profiles them)."""
        if head_kinds is None:
            head_kinds = [k for k, m in enumerate(_config.load_params()["monomers"]) if m["polar"]]
        mask = 0
        for k in head_kinds:
            mask |= 1 << int(k)
        head = np.zeros(int(bins), np.uint32)
        tail = np.zeros(int(bins), np.uint32)
        esc = C.c_uint32(0)
        _check(self._lib, self._h, self._lib.soup_density_profile_z(
            self._h, int(bins), mask, head.ctypes.data_as(_abi._U32P), tail.ctypes.data_as(_abi._U32P),
            C.byref(esc) if drop_escaped else None))
        dz = float(self.cfg.box[2]) / int(bins)
        out = dict(z=[(i + 0.5) * dz for i in range(int(bins))], head=head.astype(np.int64).tolist(),
                   tail=tail.astype(np.int64).tolist())
        if drop_escaped:
            out["escaped"] = int(esc.value)
        return out

    def aggregate_shapes(self, members, labels, max_shapes):
        """Device shapeOf over unwrapAggregate for the components named by `labels`, largest first:
        (number of components, [ {size, label, centre, gyration (Sxx Syy Szz Sxy Sxz Syz)} ])."""
        m = np.ascontiguousarray(members, np.uint32)
        lab = np.ascontiguousarray(labels, np.uint32)
        out = (_abi.SoupAggregateShape * max(1, int(max_shapes)))()
        nc = C.c_uint32()
        _check(self._lib, self._h, self._lib.soup_aggregate_shapes(
            self._h, m.ctypes.data_as(_abi._U32P), lab.ctypes.data_as(_abi._U32P), m.size, int(max_shapes), out,
            C.byref(nc)))
        k = min(int(max_shapes), int(nc.value))
        return int(nc.value), [dict(size=out[c].size, label=out[c].label, centre=list(out[c].centre),
                                    gyration=list(out[c].gyration)) for c in range(k)]

    def aggregate_unwrap(self, members):
        """unwrapAggregate (engine/src/aggregate.ts:245-262) of one aggregate on the device: f32 x4 per
        member (w = kind), in the given order, about the first member."""
        m = np.ascontiguousarray(members, np.uint32)
        out = np.empty(4 * m.size, np.float32)
        _check(self._lib, self._h, self._lib.soup_aggregate_unwrap(self._h, m.ctypes.data_as(_abi._U32P), m.size,
                                                                   _ptr(out)))
        return out

    def local_cavity_volume(self, unwrapped, cell, radius):
        """localCavityVolume (soup/src/aggregates.ts:350-385) of unwrapped positions on the device."""
        p = np.ascontiguousarray(unwrapped, np.float32)
        v = C.c_double()
        _check(self._lib, self._h, self._lib.soup_local_cavity_volume(self._h, _ptr(p), p.size // 4, float(cell),
                                                                      float(radius), C.byref(v)))
        return v.value

    def box_cavity_volume(self, positions, cell, radius):
        """enclosedVolume (engine/src/closure.ts:51-163) of f32 x4 positions on the grid of the live box
        (x, y periodic, z open), on the device; the positions are taken as given."""
        p = np.ascontiguousarray(positions, np.float32)
        v = C.c_double()
        _check(self._lib, self._h, self._lib.soup_box_cavity_volume(self._h, _ptr(p), p.size // 4, float(cell),
                                                                    float(radius), C.byref(v)))
        return v.value

    def cluster_labels(self, members, cutoff, periodic_z=True):
        """buildClusterUnionFind (engine/src/aggregate.ts:65-130) over the members on the device, z
        periodic or open: (components, labels = the minimum original index of each component)."""
        m = np.ascontiguousarray(members, np.uint32)
        labels = np.empty(m.size, np.uint32)
        nc = C.c_uint32()
        _check(self._lib, self._h, self._lib.soup_cluster_labels(
            self._h, m.ctypes.data_as(_abi._U32P), m.size, float(cutoff), int(bool(periodic_z)),
            labels.ctypes.data_as(_abi._U32P), C.byref(nc)))
        return int(nc.value), labels

    # ---- differentiation (the adjoint of the step; no counterpart in the reference) ----
    def get_diff_params(self):
        t = (C.c_double * _abi.DIFF_NPARAM)()
        _check(self._lib, self._h, self._lib.soup_get_diff_params(self._h, t))
        return np.array(list(t), np.float64)

    def set_diff_params(self, theta):
        t = (C.c_double * _abi.DIFF_NPARAM)(*[float(v) for v in theta])
        _check(self._lib, self._h, self._lib.soup_set_diff_params(self._h, t))

    def diff_forward(self, steps, checkpoint_every, traj_ptr=None, frame_stride=1):
        """Differentiable window from the current state; traj_ptr: device pointer for
        steps / frame_stride + 1 frames (every frame_stride-th step)."""
        _check(self._lib, self._h, self._lib.soup_diff_forward_strided(
            self._h, int(steps), int(checkpoint_every), int(frame_stride), C.c_void_p(traj_ptr) if traj_ptr else None))

    def diff_backward(self, dldx_ptr, dx0_ptr=None, dv0_ptr=None):
        t = (C.c_double * _abi.DIFF_NPARAM)()
        _check(self._lib, self._h, self._lib.soup_diff_backward(
            self._h, C.c_void_p(dldx_ptr), t, C.c_void_p(dx0_ptr) if dx0_ptr else None,
            C.c_void_p(dv0_ptr) if dv0_ptr else None))
        return np.array(list(t), np.float64)

    pairingStats = pairing_stats
    densityProfileZ = density_profile_z

    def aggregate_labels_noalloc(self, members, cutoff):
        """aggregate_labels without device allocation (scratch in a fixed per-device array of the
        library; at most SOUP_NOALLOC_MAX_MEMBERS members and cells; overlapping calls race)."""
        m = np.ascontiguousarray(members, np.uint32)
        labels = np.empty(m.size, np.uint32)
        nc = C.c_uint32()
        _check(self._lib, self._h, self._lib.soup_aggregate_labels_noalloc(
            self._h, m.ctypes.data_as(_abi._U32P), m.size, float(cutoff), labels.ctypes.data_as(_abi._U32P),
            C.byref(nc)))
        return int(nc.value), labels

    # reference-style aliases
    scaleBoxTo = scale_box_to
    growBoxTo = grow_box_to
    forcesBruteForce = forces_brute_force
    forcesNoRebuildDEBUG = forces_no_rebuild
    bondSlots = bond_slots
    centerLinks = center_links
    centerHeldSteps = center_held_steps
    rngState = rng_state
    desorbEvents = desorb_events
    nonFiniteCount = nonfinite_count
    protonationRngState = protonation_rng_state


def _box_ramp(from_box, target_box, ramp_steps: int):
    """applyBoxScale's increments (soup/src/soup-box-scale.ts:228-250): from_box * exp(ln(target /
    from) * s / ramp_steps) for s = 1 .. ramp_steps, the last exactly target; (box, is_last) pairs."""
    fb = [float(x) for x in from_box]
    tb = [float(x) for x in target_box]
    ln = [math.log(tb[a] / fb[a]) for a in range(3)]
    out = []
    for s in range(1, int(ramp_steps) + 1):
        last = s == ramp_steps
        out.append((tb if last else [fb[a] * math.exp((ln[a] * s) / ramp_steps) for a in range(3)], last))
    return out


def _apply_tuning(lib, h, tuning):
    r = _abi.SoupTuneResult()
    r.tpp, r.walk, r.skin_scale = int(tuning["tpp"]), int(tuning["walk"]), float(tuning["skin_scale"])
    r.queued = int(tuning.get("queued", 0))
    r.list_cells = int(tuning.get("list_cells", 0))
    _check(lib, h, lib.soup_apply_tuning(h, C.byref(r)))


def _autotune(lib, h, steps):
    r = _abi.SoupTuneResult()
    _check(lib, h, lib.soup_autotune(h, int(steps), C.byref(r)))
    return dict(tpp=r.tpp, walk=r.walk, tpp_before=r.tpp_before, walk_before=r.walk_before,
                skin_scale=r.skin_scale, ms_per_step_before=r.ms_per_step_before,
                ms_per_step_after=r.ms_per_step_after, queued=r.queued, queued_before=r.queued_before,
                list_cells=r.list_cells)


class SoupBatch:
    """Many independent replicas stepped together (one launch per kernel per step)."""

    def __init__(self, cfgs, states=None, rule_ids=None):
        self._lib = _abi.lib()
        R = len(cfgs)
        arr = (_abi.SoupConfig * R)(*cfgs)
        self.cfgs = list(cfgs)
        sts = None
        self._keep = []
        if states is not None:
            sts = (_abi.SoupInitState * R)()
            for r, st in enumerate(states):
                s = init_state(st, cfgs[r])
                self._keep.append(s)
                sts[r] = s
        h = C.c_void_p()
        rc = self._lib.soup_batch_create(arr, sts, R, C.byref(h))
        if rc != 0:
            raise _abi.SoupError(rc, self._lib.soup_last_error(None).decode())
        self._h = h
        rid = rule_ids or _config.rule_ids()
        self.replicas = [SoupSystem._view(self._lib, self._lib.soup_batch_replica(h, r), cfgs[r], rid) for r in range(R)]

    def step(self, n: int):
        rc = self._lib.soup_batch_step(self._h, int(n))
        if rc != 0:
            raise _abi.SoupError(rc, self._lib.soup_batch_last_error(self._h).decode())

    @property
    def n(self) -> int:
        """Particles of the whole batch (replica r's original indices follow replica r-1's)."""
        return sum(int(r.n) for r in self.replicas)

    # the differentiable window over the whole batch: the parameters are shared by every replica,
    # the trajectory holds every replica's particles (soup_diff_forward / soup_diff_backward)
    def get_diff_params(self):
        return self.replicas[0].get_diff_params()

    def set_diff_params(self, theta):
        self.replicas[0].set_diff_params(theta)

    def diff_forward(self, steps, checkpoint_every, traj_ptr=None, frame_stride=1):
        self.replicas[0].diff_forward(steps, checkpoint_every, traj_ptr, frame_stride)

    def diff_backward(self, dldx_ptr, dx0_ptr=None, dv0_ptr=None):
        return self.replicas[0].diff_backward(dldx_ptr, dx0_ptr, dv0_ptr)

    def prepare_graphs(self):
        """soup_prepare_graphs for the whole batch."""
        _check(self._lib, self.replicas[0]._h, self._lib.soup_prepare_graphs(self.replicas[0]._h))

    def autotune(self, steps: int = 20) -> dict:
        """soup_autotune for the whole batch (through replica 0's handle, which addresses the batch)."""
        return _autotune(self._lib, self.replicas[0]._h, steps)

    def apply_tuning(self, tuning: dict):
        """soup_apply_tuning for the whole batch."""
        _apply_tuning(self._lib, self.replicas[0]._h, tuning)

    def dispose(self):
        if getattr(self, "_h", None):
            for r in self.replicas:
                r._h = None
            self._lib.soup_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.dispose()
        except Exception:
            pass


def create_soup(opts: _config.SoupOptions, state: Optional[dict] = None) -> SoupSystem:
    """createSoup (soup/src/sim.ts:95)."""
    return SoupSystem(_config.resolve(opts), state)


createSoup = create_soup

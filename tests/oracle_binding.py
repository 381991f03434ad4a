"""ctypes binding of the CPU oracle (oracle/libsoup_oracle.so) -- test infrastructure.

Used by tests/, __graft_entry__.smoke() and bench.py's CPU legs only, as the checker.
"""
import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "libsoup_oracle.so")

F_POS, F_VEL, F_FORCE, F_SLOTS, F_CENTER, F_HELD, F_CHARGES, F_BOND_RNG, F_THERMO_RNG, F_FROZEN, \
    F_EVENTS, F_DESORB, F_POS_REF, F_PROT_RNG = range(14)

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)


def lib(abi):
    """Load (building if needed) the oracle; `abi` is the package's _abi module (struct layouts)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < os.path.getmtime(
            os.path.join(ORACLE_DIR, "soup_oracle.cpp")):
        build()
    L = C.CDLL(ORACLE_SO)
    P = C.c_void_p
    cfgp = C.POINTER(abi.SoupConfig)
    sig = {
        "oracle_last_error": (C.c_char_p, []),
        "oracle_threads": (C.c_int, []),
        "oracle_set_threads": (None, [C.c_int]),
        "oracle_fresh_state": (C.c_int, [cfgp, P, P, P, P, P]),
        "oracle_initial_charges": (C.c_int, [cfgp, P, P, P]),
        "oracle_create": (P, [cfgp, C.POINTER(abi.SoupInitState)]),
        "oracle_destroy": (None, [P]),
        "oracle_step": (C.c_int, [P, C.c_uint64]),
        "oracle_phase": (C.c_int, [P, C.c_int]),
        "oracle_read": (C.c_int, [P, C.c_int, P, C.c_size_t]),
        "oracle_write": (C.c_int, [P, C.c_int, P, C.c_size_t]),
        "oracle_forces64": (C.c_int, [P, P]),
        "oracle_forces_brute64": (C.c_int, [P, P]),
        "oracle_forces_brute32": (C.c_int, [P, P]),
        "oracle_verlet": (C.c_int, [P, P, P, C.c_size_t]),
        "oracle_es_list": (C.c_int, [P, P, P, C.c_size_t]),
        "oracle_info": (C.c_int, [P, P]),
        "oracle_max_drift_sq": (C.c_double, [P]),
        "oracle_nonfinite": (C.c_int, [P, P]),
        "oracle_sweep": (C.c_int, [P, C.POINTER(abi.SoupSweepResult)]),
        "oracle_ph_sweep_arrays": (C.c_int, [cfgp, P, P, C.c_uint32, P, C.POINTER(abi.SoupSweepResult)]),
        "oracle_es_pair_energy": (C.c_double, [cfgp, C.c_double, C.c_double]),
        "oracle_acid_soap_well": (C.c_double, [cfgp, C.c_double]),
        "oracle_pair_force_x": (C.c_double, [cfgp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int]),
        "oracle_periodic_centre": (C.c_int, [P, P, C.c_uint32, P, C.c_double, P]),
        "oracle_closure": (C.c_int, [P, P, C.c_uint32, P, C.c_uint32, P, P, C.c_double, C.c_double, C.c_double,
                                     C.POINTER(abi.SoupClosureResult), P, P]),
        "oracle_amphiphiles": (C.c_uint32, [P, P, C.c_uint32, P, P]),
        "oracle_aggregates": (C.c_uint32, [P, P, C.c_uint32, P, C.c_double, P]),
        "oracle_pairing_stats": (C.c_int, [P, P, C.c_uint32, P, C.c_int, C.c_double, P]),
        "oracle_density_profile_z": (C.c_int, [P, C.c_uint32, C.c_double, C.c_uint32, C.c_uint32, P, P, P]),
        "oracle_aggregate_shape": (C.c_int, [P, P, C.c_uint32, P, P]),
        "oracle_relax": (C.c_int, [P, C.c_uint32, C.c_double]),
        "oracle_scale_molecules_rigid": (C.c_int, [P, C.c_uint32, P, C.c_uint32, P, P, P]),
        "oracle_unwrap_aggregate": (C.c_int, [P, P, C.c_uint32, P, P]),
        "oracle_closure_in_parcel": (C.c_int, [P, P, C.c_uint32, P, C.c_uint32, P, P, C.c_double, C.c_double,
                                               C.c_double, P, C.c_double, C.POINTER(abi.SoupClosureResult)]),
        "oracle_local_cavity_volume": (C.c_double, [P, C.c_uint32, C.c_double, C.c_double]),
        "oracle_box_cavity_volume": (C.c_double, [P, C.c_uint32, P, C.c_double, C.c_double]),
        "oracle_cluster_labels": (C.c_uint32, [P, P, C.c_uint32, P, C.c_double, C.c_int, P]),
        "oracle_proximity_pairs": (C.c_int, [P, C.c_uint32, P, C.c_double, P, P, C.c_size_t,
                                             C.POINTER(C.c_size_t)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def init_state(abi, st):
    """SoupInitState from a dict of numpy arrays (missing keys -> NULL)."""
    s = abi.SoupInitState()
    keep = []
    for name in ("positions", "velocities", "bond_slots", "center_link", "center_held", "bond_rng",
                 "thermo_rng", "charges", "frozen", "events", "desorb_events"):
        a = st.get(name) if st else None
        if a is not None:
            a = np.ascontiguousarray(a)
            keep.append(a)
            setattr(s, name, a.ctypes.data)
    s._keep = keep
    return s


_FIELD_DTYPE = {
    F_POS: (np.float32, 4), F_VEL: (np.float32, 4), F_FORCE: (np.float32, 4), F_SLOTS: (np.uint32, 3),
    F_CENTER: (np.uint32, 1), F_HELD: (np.uint32, 1), F_CHARGES: (np.float32, 1), F_BOND_RNG: (np.uint32, 1),
    F_THERMO_RNG: (np.uint32, 1), F_FROZEN: (np.uint32, 1), F_POS_REF: (np.float32, 4),
}


class OracleSystem:
    def __init__(self, abi, cfg, state=None):
        self.abi = abi
        self.L = lib(abi)
        self.cfg = cfg
        self.n = cfg.n
        st = init_state(abi, state)
        self.h = self.L.oracle_create(C.byref(cfg), C.byref(st) if state is not None else None)
        if not self.h:
            raise RuntimeError(self.L.oracle_last_error().decode())

    def close(self):
        if self.h:
            self.L.oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st != 0:
            raise RuntimeError(f"oracle status {st}: {self.L.oracle_last_error().decode()}")

    def step(self, n):
        self._check(self.L.oracle_step(self.h, n))

    def phase(self, p):
        self._check(self.L.oracle_phase(self.h, p))

    def read(self, field):
        if field == F_EVENTS:
            a = np.zeros(2 * self.cfg.n_rules, np.uint32)
        elif field == F_DESORB:
            a = np.zeros(2, np.uint32)
        elif field == F_PROT_RNG:
            a = np.zeros(1, np.uint32)
        else:
            dt, k = _FIELD_DTYPE[field]
            a = np.zeros(self.n * k, dt)
        self._check(self.L.oracle_read(self.h, field, _ptr(a), a.nbytes))
        return a

    def write(self, field, arr):
        arr = np.ascontiguousarray(arr)
        self._check(self.L.oracle_write(self.h, field, _ptr(arr), arr.nbytes))

    def forces64(self):
        out = np.zeros(self.n * 4, np.float64)
        self._check(self.L.oracle_forces64(self.h, _ptr(out)))
        return out

    def forces_brute64(self):
        out = np.zeros(self.n * 4, np.float64)
        self._check(self.L.oracle_forces_brute64(self.h, _ptr(out)))
        return out

    def forces_brute32(self):
        out = np.zeros(self.n * 4, np.float32)
        self._check(self.L.oracle_forces_brute32(self.h, _ptr(out)))
        return out

    def verlet(self):
        counts = np.zeros(self.n, np.uint32)
        self._check(self.L.oracle_verlet(self.h, _ptr(counts), None, 0))
        lists = np.zeros(int(counts.sum(dtype=np.uint64)), np.uint32)
        self._check(self.L.oracle_verlet(self.h, _ptr(counts), _ptr(lists), lists.size))
        return counts, lists

    def es_lists(self):
        nh = self.info()["heads"]
        counts = np.zeros(nh, np.uint32)
        if nh == 0:
            return counts, np.zeros(0, np.uint32)
        self._check(self.L.oracle_es_list(self.h, _ptr(counts), None, 0))
        lists = np.zeros(int(counts.sum(dtype=np.uint64)), np.uint32)
        self._check(self.L.oracle_es_list(self.h, _ptr(counts), _ptr(lists), lists.size))
        return counts, lists

    def info(self):
        out = np.zeros(6, np.uint64)
        self._check(self.L.oracle_info(self.h, _ptr(out)))
        return dict(step=int(out[0]), rebuilds=int(out[1]), sweeps=int(out[2]), list_entries=int(out[3]),
                    heads=int(out[4]), overflow=int(out[5]))

    def max_drift_sq(self):
        return self.L.oracle_max_drift_sq(self.h)

    def nonfinite(self):
        out = np.zeros(2, np.uint32)
        self._check(self.L.oracle_nonfinite(self.h, _ptr(out)))
        return out

    def sweep(self):
        r = self.abi.SoupSweepResult()
        self._check(self.L.oracle_sweep(self.h, C.byref(r)))
        return r

    def relax(self, iterations, d0):
        self._check(self.L.oracle_relax(self.h, iterations, d0))


def fresh_state(abi, cfg):
    L = lib(abi)
    n = cfg.n
    pos = np.zeros(n * 4, np.float32)
    vel = np.zeros(n * 4, np.float32)
    frozen = np.zeros(n, np.uint32)
    brng = np.zeros(n, np.uint32)
    trng = np.zeros(n, np.uint32)
    st = L.oracle_fresh_state(C.byref(cfg), _ptr(pos), _ptr(vel), _ptr(frozen), _ptr(brng), _ptr(trng))
    assert st == 0
    return dict(positions=pos, velocities=vel, frozen=frozen, bond_rng=brng, thermo_rng=trng)


def initial_charges(abi, cfg, pos):
    L = lib(abi)
    ch = np.zeros(cfg.n, np.float32)
    pr = np.zeros(1, np.uint32)
    assert L.oracle_initial_charges(C.byref(cfg), _ptr(pos), _ptr(ch), _ptr(pr)) == 0
    return ch, int(pr[0])


def ph_sweep_arrays(abi, cfg, pos, charges, rng_state):
    L = lib(abi)
    r = abi.SoupSweepResult()
    rs = np.array([rng_state], np.uint32)
    L.oracle_ph_sweep_arrays(C.byref(cfg), _ptr(pos), _ptr(charges), len(charges), _ptr(rs), C.byref(r))
    return r, int(rs[0])


def closure(abi, pos, members, water, box, centre, cell, radius, vmin, want_grids=False):
    L = lib(abi)
    members = np.ascontiguousarray(members, np.uint32)
    water = np.ascontiguousarray(water, np.uint32)
    box = np.ascontiguousarray(box, np.float64)
    centre = np.ascontiguousarray(centre, np.float64)
    r = abi.SoupClosureResult()
    occ = vis = None
    if want_grids:
        import math
        nc = 1
        for b in box:
            nc *= max(1, math.ceil(b / cell))
        occ = np.zeros(nc, np.uint8)
        vis = np.zeros(nc, np.uint8)
    st = L.oracle_closure(_ptr(pos), _ptr(members), len(members), _ptr(water), len(water), _ptr(box), _ptr(centre),
                          cell, radius, vmin, C.byref(r), _ptr(occ), _ptr(vis))
    if st != 0:
        raise RuntimeError(L.oracle_last_error().decode())
    return (r, occ, vis) if want_grids else r


def periodic_centre(abi, pos, idx, box, alpha):
    L = lib(abi)
    idx = np.ascontiguousarray(idx, np.uint32)
    box = np.ascontiguousarray(box, np.float64)
    out = np.zeros(3, np.float64)
    ok = L.oracle_periodic_centre(_ptr(pos), _ptr(idx), len(idx), _ptr(box), alpha, _ptr(out))
    return out if ok else None


def amphiphiles(abi, pos, slots, polar_of_kind):
    L = lib(abi)
    n = len(pos) // 4
    head_of = np.zeros(n, np.uint32)
    pk = np.ascontiguousarray(polar_of_kind, np.uint32)
    cnt = L.oracle_amphiphiles(_ptr(pos), _ptr(np.ascontiguousarray(slots, np.uint32)), n, _ptr(pk), _ptr(head_of))
    return int(cnt), head_of


def aggregates(abi, pos, members, box, cutoff):
    L = lib(abi)
    members = np.ascontiguousarray(members, np.uint32)
    labels = np.zeros(len(members), np.uint32)
    box = np.ascontiguousarray(box, np.float64)
    n = L.oracle_aggregates(_ptr(pos), _ptr(members), len(members), _ptr(box), cutoff, _ptr(labels))
    return int(n), labels


def pairing_stats(abi, pos, charges, box, charged_kind, contact):
    """(with_neighbour, unlike, like, paired, charged, heads) from the oracle."""
    L = lib(abi)
    pos = np.ascontiguousarray(pos, np.float32)
    charges = np.ascontiguousarray(charges, np.float32)
    box = np.ascontiguousarray(box, np.float64)
    out = np.zeros(6, np.uint32)
    L.oracle_pairing_stats(_ptr(pos), _ptr(charges), len(pos) // 4, _ptr(box), int(charged_kind), float(contact),
                           _ptr(out))
    return tuple(int(v) for v in out)


def density_profile_z(abi, pos, box_z, bins, head_mask):
    """(head counts, tail counts, escaped) from the oracle."""
    L = lib(abi)
    pos = np.ascontiguousarray(pos, np.float32)
    head = np.zeros(bins, np.uint32)
    tail = np.zeros(bins, np.uint32)
    esc = np.zeros(1, np.uint32)
    L.oracle_density_profile_z(_ptr(pos), len(pos) // 4, float(box_z), int(bins), int(head_mask), _ptr(head),
                               _ptr(tail), _ptr(esc))
    return head, tail, int(esc[0])


def aggregate_shape(abi, pos, members, box):
    """(n, centre[3], gyration[6]) of one component from the oracle; members ascending."""
    L = lib(abi)
    pos = np.ascontiguousarray(pos, np.float32)
    members = np.ascontiguousarray(np.sort(members), np.uint32)
    box = np.ascontiguousarray(box, np.float64)
    out = np.zeros(10, np.float64)
    L.oracle_aggregate_shape(_ptr(pos), _ptr(members), len(members), _ptr(box), _ptr(out))
    return int(out[0]), out[1:4].copy(), out[4:10].copy()


def scale_molecules_rigid(abi, pos, edges, old_box, new_box):
    """scaleMoleculesRigid from the oracle: positions (f32 x4) in the new box; `edges` flat (i, j) pairs."""
    L = lib(abi)
    pos = np.ascontiguousarray(pos, np.float32)
    edges = np.ascontiguousarray(edges, np.uint32)
    out = np.zeros_like(pos)
    ob_ = np.ascontiguousarray(old_box, np.float64)
    nb_ = np.ascontiguousarray(new_box, np.float64)
    st = L.oracle_scale_molecules_rigid(_ptr(pos), pos.size // 4, _ptr(edges), edges.size // 2, _ptr(ob_), _ptr(nb_),
                                        _ptr(out))
    if st != 0:
        raise RuntimeError(L.oracle_last_error().decode())
    return out


def proximity_pairs(abi, pos, box, cutoff, eligible=None):
    """proximityPairs from the oracle: flat (i, j) pairs, i < j, in the reference's visiting order."""
    L = lib(abi)
    pos = np.ascontiguousarray(pos, np.float32)
    n = pos.size // 4
    el = np.ones(n, np.uint8) if eligible is None else np.ascontiguousarray(eligible, np.uint8)
    b = np.ascontiguousarray(box, np.float64)
    cnt = C.c_size_t(0)
    L.oracle_proximity_pairs(_ptr(pos), n, _ptr(b), float(cutoff), _ptr(el), None, 0, C.byref(cnt))
    out = np.zeros(2 * max(cnt.value, 1), np.uint32)
    L.oracle_proximity_pairs(_ptr(pos), n, _ptr(b), float(cutoff), _ptr(el), _ptr(out), cnt.value, C.byref(cnt))
    return out[: 2 * cnt.value]


def unwrap_aggregate(abi, pos, members, box):
    """unwrapAggregate from the oracle: f32 x4 per member, about members[0]."""
    L = lib(abi)
    pos = np.ascontiguousarray(pos, np.float32)
    m = np.ascontiguousarray(members, np.uint32)
    out = np.zeros(4 * m.size, np.float32)
    L.oracle_unwrap_aggregate(_ptr(pos), _ptr(m), m.size, _ptr(np.ascontiguousarray(box, np.float64)), _ptr(out))
    return out


def local_cavity_volume(abi, positions, cell, radius):
    """localCavityVolume from the oracle, over unwrapped f32 x4 positions."""
    p = np.ascontiguousarray(positions, np.float32)
    return lib(abi).oracle_local_cavity_volume(_ptr(p), p.size // 4, float(cell), float(radius))


def closure_in_parcel(abi, pos, members, water, box, centre, cell, radius, vmin, parcel_centre, parcel_radius):
    """encapsulatedWaterVolume with the parcel restriction, from the oracle."""
    L = lib(abi)
    pos = np.ascontiguousarray(pos, np.float32)
    m = np.ascontiguousarray(members, np.uint32)
    w = np.ascontiguousarray(water, np.uint32)
    r = abi.SoupClosureResult()
    st = L.oracle_closure_in_parcel(_ptr(pos), _ptr(m), m.size, _ptr(w), w.size, _ptr(np.ascontiguousarray(box, np.float64)),
                                    _ptr(np.ascontiguousarray(centre, np.float64)), float(cell), float(radius), float(vmin),
                                    _ptr(np.ascontiguousarray(parcel_centre, np.float64)), float(parcel_radius), C.byref(r))
    if st != 0:
        raise RuntimeError(L.oracle_last_error().decode())
    return r


def box_cavity_volume(abi, positions, box, cell, radius):
    """enclosedVolume on the periodic box's grid (closure.ts:51-163), positions as given."""
    p = np.ascontiguousarray(positions, np.float32)
    return lib(abi).oracle_box_cavity_volume(_ptr(p), p.size // 4, _ptr(np.ascontiguousarray(box, np.float64)),
                                             float(cell), float(radius))


def cluster_labels(abi, pos, members, box, cutoff, periodic_z):
    """buildClusterUnionFind with its periodicZ switch (aggregate.ts:65-130): (components, labels)."""
    pos = np.ascontiguousarray(pos, np.float32)
    m = np.ascontiguousarray(members, np.uint32)
    labels = np.zeros(m.size, np.uint32)
    n = lib(abi).oracle_cluster_labels(_ptr(pos), _ptr(m), m.size, _ptr(np.ascontiguousarray(box, np.float64)),
                                       float(cutoff), int(bool(periodic_z)), _ptr(labels))
    return int(n), labels

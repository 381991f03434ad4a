"""Pins the CPU oracle against the reference's own known-answer tests (restated).

The reference's tests cannot run here (WebGPU in Chrome; TypeScript on Node -- neither exists in
this environment), so the oracle is pinned by the properties and tolerances those tests assert:
  tests/soup-electrostatics.test.ts:39-78   F = -dU/dr, zero and continuous at the cutoff, exact split
  tests/soup-electrostatics.test.ts:149-177 Henderson-Hasselbalch to 0.01 (rng state 12345)
  tests/soup-electrostatics.test.ts:179-241 exact two-head Boltzmann weights to 5e-3 (state 987654321)
  tests/soup-forces.test.ts:19-294          list force == brute force (plain, charged, long range, wall)
  tests/soup-area-move.test.ts:90           force == -grad of the pair potential
  tests/water-closure.test.ts:165-221       closure synthetics (centred == straddling, blob 0, hole leaks)
"""
import math

import numpy as np
import pytest

import oracle_binding as ob
from helpers import charged_opts, confined_opts, long_range_opts, plain_opts, rel_rms
from protocell_genesis_b200 import _abi, config as cfgm

P = cfgm.load_params()


def _cfg(opts):
    return cfgm.resolve(opts, P)


# ---------------------------------------------------------------------------------------------
# electrostatics
# ---------------------------------------------------------------------------------------------
def test_es_force_is_minus_gradient_and_continuous():
    cfg = _cfg(charged_opts())
    L = ob.lib(_abi)
    h = 1e-6
    worst = 0.0
    for r in [0.6, 0.8, 0.95, 1.2, 1.5, 2.0, 2.4, 2.7, 2.9469545, 3.2, 3.8, 4.4, 4.8]:
        num = -(L.oracle_es_pair_energy(cfg, r + h, 1.0) - L.oracle_es_pair_energy(cfg, r - h, 1.0)) / (2 * h)
        b = cfgm.make_es_basis(P, cfg.kT, {"enabled": True, "pH": 7.0, "minBoxSigma": 16.0})
        ana = cfgm.es_pair_force_mag(r, 1.0, b)
        worst = max(worst, abs(num - ana) / max(1e-12, abs(ana)))
    assert worst < 1e-5
    rc = cfg.es_cutoff
    assert abs(L.oracle_es_pair_energy(cfg, rc - 1e-7, 1.0)) < 1e-6
    assert L.oracle_es_pair_energy(cfg, rc, 1.0) == 0.0
    assert L.oracle_es_pair_energy(cfg, rc + 0.1, 1.0) == 0.0


def test_es_split_is_seamless_in_the_kernel_formula():
    # near half (r < split, in the list force) + far half (split <= r < rc) == whole, at the seam too
    cfg = _cfg(charged_opts())
    L = ob.lib(_abi)
    ko = [m["id"] for m in P["monomers"]].index("O")
    split = cfg.es_split_radius
    for r in [1.0, 2.9, split - 1e-6, split, split + 1e-6, 3.0, 4.0, cfg.es_cutoff - 1e-6]:
        f64 = L.oracle_pair_force_x(cfg, ko, ko, -1.0, -1.0, r, 1)
        b = cfgm.make_es_basis(P, cfg.kT, {"enabled": True, "pH": 7.0, "minBoxSigma": 16.0})
        whole = cfgm.es_pair_force_mag(r, 1.0, b)
        # the pair force also carries WCA (r < 1.066) and no attraction for O-O (polarPolar = 0)
        wca = 0.0
        bb = P["params"]["sigma"] * 0.95
        if r < cfgm.wca_cutoff(bb):
            s6 = (bb / r) ** 6
            wca = 24 * P["params"]["epsilon"] / r * (2 * s6 * s6 - s6)
        assert f64 == pytest.approx(whole + wca, rel=1e-9, abs=1e-12)


def test_henderson_hasselbalch_without_interaction():
    box = [200.0, 200.0, 200.0]
    ko = [m["id"] for m in P["monomers"]].index("O")
    pos = np.array([10, 10, 10, ko, 110, 110, 110, ko], np.float32)
    worst = 0.0
    for ph in [3.9, 4.4, 4.9, 5.4, 5.9]:
        cfg = _cfg(cfgm.SoupOptions(box=box, seed=1, kT=1.1, start={"C": 0, "O": 2, "H": 0, "M": 0, "W": 0},
                                    electrostatics={"enabled": True, "pH": ph}))
        charges = np.zeros(2, np.float32)
        rng = 12345
        on = 0
        sweeps = 20000
        for _ in range(sweeps):
            _, rng = ob.ph_sweep_arrays(_abi, cfg, pos, charges, rng)
            on += int((charges != 0).sum())
        alpha = 1 / (1 + 10 ** (cfg.pka_intrinsic - ph))
        worst = max(worst, abs(on / (2 * sweeps) - alpha))
    assert worst < 0.01


def test_detailed_balance_two_heads():
    box = [40.0, 40.0, 40.0]
    ko = [m["id"] for m in P["monomers"]].index("O")
    r = 1.1
    pos = np.array([10, 10, 10, ko, 10 + r, 10, 10, ko], np.float32)
    cfg = _cfg(cfgm.SoupOptions(box=box, seed=1, kT=1.1, start={"C": 0, "O": 2, "H": 0, "M": 0, "W": 0},
                                electrostatics={"enabled": True, "pH": 4.9}))
    b = cfgm.make_es_basis(P, cfg.kT, {"enabled": True, "pH": 4.9, "minBoxSigma": 40.0})
    q = b.charge_deprotonated
    u_both = cfgm.es_pair_energy(r, q * q, b)
    dg = b.kT * math.log(10) * (b.pka - b.ph)
    u_pair = cfgm.acid_soap_well(r, b)
    w = [1.0, math.exp(-(dg + u_pair) / b.kT), math.exp(-(dg + u_pair) / b.kT), math.exp(-(2 * dg + u_both) / b.kT)]
    z = sum(w)
    exact = [x / z for x in w]
    charges = np.zeros(2, np.float32)
    rng = 987654321
    counts = [0, 0, 0, 0]
    sweeps = 200000
    L = ob.lib(_abi)
    import ctypes as C
    res = _abi.SoupSweepResult()
    rs = np.array([rng], np.uint32)
    pp = pos.ctypes.data_as(C.c_void_p)
    cp = charges.ctypes.data_as(C.c_void_p)
    rp = rs.ctypes.data_as(C.c_void_p)
    for _ in range(sweeps):
        L.oracle_ph_sweep_arrays(cfg, pp, cp, 2, rp, C.byref(res))
        counts[(1 if charges[0] != 0 else 0) + (2 if charges[1] != 0 else 0)] += 1
    meas = [c / sweeps for c in counts]
    worst = max(abs(meas[0] - exact[0]), abs(meas[1] + meas[2] - exact[1] - exact[2]), abs(meas[3] - exact[3]))
    assert worst < 5e-3
    no_es = math.exp(-2 * dg / b.kT) / (1 + 2 * math.exp(-dg / b.kT) + math.exp(-2 * dg / b.kT))
    assert exact[3] < no_es


# ---------------------------------------------------------------------------------------------
# forces
# ---------------------------------------------------------------------------------------------
def _wca_v(r, b, eps):
    if r >= cfgm.wca_cutoff(b):
        return 0.0
    s6 = (b / r) ** 6
    q = 2 * s6 - 1
    return eps * q * q


def _attr_v(r, rc, wc, eps):
    if r < rc:
        return -eps
    if r > rc + wc:
        return 0.0
    c = math.cos(math.pi * (r - rc) / (2 * wc))
    return -eps * c * c


def test_pair_force_is_minus_gradient_of_the_potential():
    # engine/wgsl/forces.wgsl:78-102 potentials vs the kernels' force (FP64 mode), per class pair
    cfg = _cfg(plain_opts())
    L = ob.lib(_abi)
    p = P["params"]
    rc = cfgm.wca_cutoff(p["sigma"] * p["beadSizes"]["tail_tail"])
    kinds = {m["id"]: k for k, m in enumerate(P["monomers"])}
    for a, bk in [("C", "C"), ("W", "W"), ("O", "W"), ("C", "W"), ("M", "C"), ("H", "O")]:
        ka, kb = kinds[a], kinds[bk]
        b = p["sigma"] * (P["monomers"][ka]["radiusSigma"] + P["monomers"][kb]["radiusSigma"]) * 0.5
        scale = cfg.attr_scale[cfg.kind_class[ka]][cfg.kind_class[kb]]
        U = lambda r: _wca_v(r, b, p["epsilon"]) + scale * _attr_v(r, rc, p["wc"], p["epsilon"])
        for r in np.linspace(0.9 * b, rc + p["wc"] - 0.01, 23):
            h = 1e-6
            num = -(U(r + h) - U(r - h)) / (2 * h)
            ana = L.oracle_pair_force_x(cfg, ka, kb, 0.0, 0.0, float(r), 1)
            assert ana == pytest.approx(num, rel=2e-5, abs=2e-6)


@pytest.mark.parametrize("maker", [plain_opts, charged_opts])
def test_list_force_equals_brute_force(maker):
    cfg = _cfg(maker())
    o = ob.OracleSystem(_abi, cfg)
    o.relax(40, 0.1)
    f_list = o.forces64()
    f_brute = o.forces_brute64()
    assert np.abs(f_list - f_brute).max() < 1e-9
    f32 = o.read(ob.F_FORCE)
    assert rel_rms(f32, f_list) < 1e-5


def test_long_range_list_is_complete():
    cfg = _cfg(long_range_opts())
    assert cfg.es_cutoff == pytest.approx(13.5)          # 0.45 * 30 caps 4 lambda_D = 15.2
    o = ob.OracleSystem(_abi, cfg)
    o.relax(20, 0.1)
    o.step(60)
    assert np.abs(o.forces64() - o.forces_brute64()).max() < 1e-9


def test_confined_wall_in_both_paths():
    cfg = _cfg(confined_opts())
    o = ob.OracleSystem(_abi, cfg)
    pos = o.read(ob.F_POS).reshape(-1, 4)
    c = np.array(cfg.box) / 2
    assert np.sqrt(((pos[:, :3] - c) ** 2).sum(1)).max() < 16.5   # sphereLatticeSites fills the parcel
    o.relax(10, 0.1)
    assert np.abs(o.forces64() - o.forces_brute64()).max() < 1e-8


def test_verlet_list_equals_brute_set():
    cfg = _cfg(plain_opts())
    o = ob.OracleSystem(_abi, cfg)
    counts, lists = o.verlet()
    pos = o.read(ob.F_POS).reshape(-1, 4).astype(np.float32)
    box = np.array(cfg.box, np.float32)
    lr = np.float32(cfg.list_range)
    off = np.concatenate([[0], np.cumsum(counts.astype(np.int64))])
    for i in range(0, cfg.n, 37):
        d = pos[i, :3] - pos[:, :3]
        d = d - np.rint(d / box).astype(np.float32) * box
        r = np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2])
        want = np.nonzero(r < lr)[0]
        want = want[want != i]
        assert np.array_equal(lists[off[i]:off[i + 1]], want)


# ---------------------------------------------------------------------------------------------
# configuration derivations (the numbers the reference's reports quote at the campaign scale)
# ---------------------------------------------------------------------------------------------
def test_campaign_geometry_numbers():
    opts = cfgm.SoupOptions(box=[76, 76, 76], seed=19, kT=1.1,
                            start={"C": 55988, "O": 18659, "H": 55988, "M": 1452, "W": 351181},
                            electrostatics={"enabled": True, "pH": 7.0, "ionicStrengthMolar": 0.01})
    cfg = _cfg(opts)
    assert cfg.n == 483268
    assert cfg.interaction_range == pytest.approx(2.946954, abs=1e-6)
    assert cfg.list_range == pytest.approx(4.446954, abs=1e-6)
    plan = cfgm.derive_plan(P, [76] * 3, list(cfg.counts)[:5], 1.1, 1.5, 10, True)
    assert plan.dims == [25, 25, 25] and plan.list_walk_radius == 2
    assert cfg.es_cutoff == pytest.approx(15.2, abs=1e-9)
    assert cfg.es_list_range == pytest.approx(16.7, abs=1e-9)
    assert cfg.es_split_radius == pytest.approx(cfg.interaction_range)
    assert cfg.rc_attr + cfg.wc == pytest.approx(2.722462, abs=1e-6)


def test_drift_bound_refusal():
    with pytest.raises(cfgm.GeometryError):
        cfgm.resolve(plain_opts(skin=0.3), P)
    cfgm.resolve(plain_opts(skin=0.3, rebuild_on_drift=True), P)   # drift-triggered mode accepts it


# ---------------------------------------------------------------------------------------------
# fresh state: the library's host generator equals the oracle's restatement, bit for bit
# ---------------------------------------------------------------------------------------------
def test_fresh_state_library_matches_oracle():
    import ctypes as C
    cfg = _cfg(charged_opts())
    st = ob.fresh_state(_abi, cfg)
    L = _abi.lib()
    n = cfg.n
    pos = np.zeros(4 * n, np.float32)
    vel = np.zeros(4 * n, np.float32)
    fr = np.zeros(n, np.uint32)
    br = np.zeros(n, np.uint32)
    tr = np.zeros(n, np.uint32)
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    assert L.soup_fresh_state(C.byref(cfg), p(pos), p(vel), p(fr), p(br), p(tr)) == 0
    assert np.array_equal(pos, st["positions"]) and np.array_equal(vel, st["velocities"])
    assert np.array_equal(br, st["bond_rng"]) and np.array_equal(tr, st["thermo_rng"])
    ch = np.zeros(n, np.float32)
    pr = C.c_uint32()
    assert L.soup_initial_charges(C.byref(cfg), p(pos), p(ch), C.byref(pr)) == 0
    ch2, pr2 = ob.initial_charges(_abi, cfg, pos)
    assert np.array_equal(ch, ch2) and pr.value == pr2
    # heads drawn from Henderson-Hasselbalch at pH 7: nearly all charged
    ko = [m["id"] for m in P["monomers"]].index("O")
    heads = pos.reshape(-1, 4)[:, 3] == ko
    assert 0.95 < (ch[heads] != 0).mean() <= 1.0
    # the lattice: kinds in data/soup.json order, positions in the box, Maxwell-Boltzmann velocities
    kinds = pos.reshape(-1, 4)[:, 3]
    assert np.all(np.diff(kinds) >= 0)
    assert np.all(pos.reshape(-1, 4)[:, :3] > 0) and np.all(pos.reshape(-1, 4)[:, :3] < 16)
    v = vel.reshape(-1, 4)[:, :3]
    assert abs(v.var() - cfg.kT) < 0.1


# ---------------------------------------------------------------------------------------------
# closure (restating tests/water-closure.test.ts's synthetic shells with this file's own builders)
# ---------------------------------------------------------------------------------------------
ST = P["stageThresholds"]
SYN_BOX = [50.0, 50.0, 50.0]
R_IN, R_OUT = 8.0, 12.0


def _dirs(rng, n):
    u = rng.uniform(-1, 1, n)
    phi = rng.uniform(0, 2 * np.pi, n)
    s = np.sqrt(1 - u * u)
    return np.stack([s * np.cos(phi), s * np.sin(phi), u], 1)


def _shell(rng, centre, hole=None):
    pts = []
    for r in (R_IN, R_OUT):                  # head leaflets dense enough to seal at radius 0.6
        n = int(math.ceil(4 * math.pi * r * r / 0.1))
        pts.append(centre + _dirs(rng, n) * r)
    nt = 30000
    d = _dirs(rng, nt)
    rr = rng.uniform(R_IN, R_OUT, nt)
    pts.append(centre + d * rr[:, None])
    pts = np.concatenate(pts)
    if hole is not None:
        v = pts - centre
        cosang = (v @ hole) / np.linalg.norm(v, axis=1)
        pts = pts[cosang < math.cos(math.radians(25))]
    return pts


def _water(rng, centre, n_in, n_out):
    d = _dirs(rng, n_in) * (rng.uniform(0, 1, n_in) ** (1 / 3) * (R_IN - 1))[:, None] + centre
    out = []
    while len(out) < n_out:
        p = rng.uniform(0, 50, 3)
        if np.linalg.norm(p - centre) > R_OUT + 1:
            out.append(p)
    return np.concatenate([d, np.array(out)])


def _assemble(members, water):
    n = len(members) + len(water)
    pos = np.zeros((n, 4), np.float32)
    pos[: len(members), :3] = members
    pos[len(members):, :3] = water
    pos[len(members):, 3] = 4
    return pos.reshape(-1), np.arange(len(members)), np.arange(len(members), n)


def _closure(pos, mem, wat):
    c = ob.periodic_centre(_abi, pos, mem, SYN_BOX, P["circularAlpha"])
    assert c is not None
    return ob.closure(_abi, pos, mem, wat, SYN_BOX, c, ST["closureCell"], ST["closureRadius"], ST["enclosedVolume"])


def test_closure_centred_equals_straddling():
    rng = np.random.default_rng(2001)
    centre = np.array([25.0, 25.0, 25.0])
    pos, mem, wat = _assemble(_shell(rng, centre), _water(rng, centre, 900, 6000))
    rc = _closure(pos, mem, wat)
    p2 = pos.reshape(-1, 4).copy()
    p2[:, :3] = np.mod(p2[:, :3] + 25.0, 50.0)
    rs = _closure(p2.reshape(-1), mem, wat)
    assert rs.encapsulated_count == rc.encapsulated_count
    assert rs.total_empty_cells == rc.total_empty_cells and rs.unreached_cells == rc.unreached_cells
    assert 0.9 * 900 < rc.encapsulated_count < 1.1 * 900
    assert rc.closed == 1


def test_closure_solid_blob_traps_nothing():
    rng = np.random.default_rng(2002)
    centre = np.array([25.0, 25.0, 25.0])
    blob = _dirs(rng, 150000) * (rng.uniform(0, 1, 150000) ** (1 / 3) * R_OUT)[:, None] + centre
    pos, mem, wat = _assemble(blob, _water(rng, centre, 0, 6000))
    r = _closure(pos, mem, wat)
    assert r.encapsulated_count == 0 and r.closed == 0


def test_closure_hole_leaks():
    rng = np.random.default_rng(2003)
    centre = np.array([25.0, 25.0, 25.0])
    pos, mem, wat = _assemble(_shell(rng, centre, hole=np.array([1.0, 0.0, 0.0])), _water(rng, centre, 900, 6000))
    r = _closure(pos, mem, wat)
    assert r.encapsulated_count < 0.05 * 900 and r.closed == 0


# ---------------------------------------------------------------------------------------------
# amphiphiles and aggregates
# ---------------------------------------------------------------------------------------------
def test_amphiphile_recognition_rules():
    # particles: kinds C=0, O=1 (polar); slots as the bond graph
    NONE = _abi.NONE
    kinds = []
    bonds = []

    def add(k):
        kinds.append(k)
        return len(kinds) - 1

    def bond(a, b):
        bonds.append((a, b))

    h = add(1); c = [add(0) for _ in range(3)]                 # head-C-C-C: amphiphile
    bond(h, c[0]); bond(c[0], c[1]); bond(c[1], c[2])
    h2 = add(1); t1 = [add(0) for _ in range(2)]; t2 = [add(0) for _ in range(2)]   # two tails
    bond(h2, t1[0]); bond(t1[0], t1[1]); bond(h2, t2[0]); bond(t2[0], t2[1])
    r = [add(0) for _ in range(3)]; hr = add(1)                # ring + head: rejected
    bond(r[0], r[1]); bond(r[1], r[2]); bond(r[2], r[0]); bond(hr, r[0])
    b0 = add(1); bc = [add(0) for _ in range(3)]               # branched carbon (degree 3): rejected
    bond(b0, bc[0]); bond(bc[0], bc[1]); bond(bc[0], bc[2])
    lone_h = add(1)                                            # bare head: rejected
    x1 = add(1); xc = add(0); x2 = add(1)                      # two heads: rejected
    bond(x1, xc); bond(xc, x2)
    n = len(kinds)
    slots = np.full((n, 3), NONE, np.uint32)
    fill = np.zeros(n, int)
    for a, b in bonds:
        slots[a, fill[a]] = b; fill[a] += 1
        slots[b, fill[b]] = a; fill[b] += 1
    pos = np.zeros((n, 4), np.float32)
    pos[:, 3] = kinds
    polar = np.array([1 if m["polar"] else 0 for m in P["monomers"]], np.uint32)
    polar_by_kind = np.zeros(8, np.uint32)
    polar_by_kind[:2] = [0, 1]
    cnt, head_of = ob.amphiphiles(_abi, pos.reshape(-1), slots.reshape(-1), polar_by_kind)
    assert cnt == 2
    assert all(head_of[x] == h for x in [h] + c)
    assert all(head_of[x] == h2 for x in [h2] + t1 + t2)
    assert all(head_of[x] == NONE for x in r + [hr, b0] + bc + [lone_h, x1, xc, x2])
    assert polar[1] == 1


def test_aggregate_labels_match_brute_components():
    rng = np.random.default_rng(5)
    box = np.array([20.0, 20.0, 20.0])
    n = 700
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = rng.uniform(0, 20, (n, 3))
    members = np.sort(rng.choice(n, 500, replace=False)).astype(np.uint32)
    cut = 2.722462
    ncomp, labels = ob.aggregates(_abi, pos.reshape(-1), members, box, cut)
    # brute force, FP64 with JavaScript rounding of the minimum image
    x = pos[members, :3].astype(np.float64)
    d = x[:, None, :] - x[None, :, :]
    d = d - np.floor(d / box + 0.5) * box
    adj = (d ** 2).sum(-1) <= cut * cut
    lab = np.arange(len(members))
    changed = True
    while changed:
        new = np.where(adj, lab[None, :], len(members)).min(1)
        new = np.minimum(new, lab)
        changed = not np.array_equal(new, lab)
        lab = new[new]
    want = members[lab]
    assert np.array_equal(labels, want)
    assert ncomp == len(np.unique(want))


# ---------------------------------------------------------------------------------------------
# the step: conservation and bond bookkeeping (tests/soup-bonds.test.ts:10-54)
# ---------------------------------------------------------------------------------------------
def test_step_conserves_monomers_and_bond_symmetry():
    from helpers import boosted
    cfg = boosted(_cfg(plain_opts()), attempt=0.6, accept=1.0, brk=0.05)
    o = ob.OracleSystem(_abi, cfg)
    o.relax(40, 0.1)
    kinds0 = o.read(ob.F_POS).reshape(-1, 4)[:, 3].copy()
    o.step(400)
    pos = o.read(ob.F_POS).reshape(-1, 4)
    assert np.array_equal(pos[:, 3], kinds0)
    slots = o.read(ob.F_SLOTS).reshape(-1, 3)
    nb = 0
    for i in range(cfg.n):
        for j in slots[i]:
            if j != _abi.NONE:
                nb += 1
                assert i in slots[j]
    ev = o.read(ob.F_EVENTS)
    assert nb // 2 == int(ev[0::2].sum() - ev[1::2].sum())
    center = o.read(ob.F_CENTER)
    for i in range(cfg.n):
        if center[i] != _abi.NONE:
            assert center[center[i]] == i

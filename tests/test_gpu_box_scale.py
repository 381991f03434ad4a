"""The box-scale map on the device against the oracle's scaleMoleculesRigid
(soup/src/soup-box-scale-math.ts:63-138), and applyBoxScaleOnce on a live system
(soup/src/soup-box-scale.ts:81-165): same positions, the new box, the reference's refusals."""
import numpy as np
import pytest

import oracle_binding as ob
from helpers import boosted, plain_opts
from protocell_genesis_b200 import _abi, config as cfgm
from protocell_genesis_b200.soup import SoupSystem
from test_box_scale import bond_lengths, fixture, wrapped_chain

pytestmark = pytest.mark.gpu
P = cfgm.load_params()


def ulps(a, b):
    """Distance in float32 units in the last place, per component (positions are >= 0)."""
    return np.abs(np.asarray(a, np.float32).view(np.int32).astype(np.int64) -
                  np.asarray(b, np.float32).view(np.int32).astype(np.int64))


def _assert_same(dev, ref):
    d = ulps(dev, ref)
    assert d.max() <= 1, d.max()
    assert (d == 0).mean() > 0.999


def _carrier():
    """A small system whose device and stream carry the array-level calls."""
    return SoupSystem(cfgm.resolve(plain_opts(), P))


def random_molecules(seed, n_mol=400, box=(24.0, 24.0, 30.0)):
    """Chains of 1-8 beads, bonds about 1 sigma, placed anywhere (many cross the boundary)."""
    rng = np.random.default_rng(seed)
    pts, bonds = [], []
    for _ in range(n_mol):
        k = int(rng.integers(1, 9))
        p = rng.uniform(0, 1, 3) * box
        for b in range(k):
            if b:
                bonds += [len(pts) - 1, len(pts)]
                step = rng.normal(size=3)
                p = p + step / np.linalg.norm(step)
            pts.append(p.copy())
    pos = np.zeros((len(pts), 4), np.float32)
    pos[:, :3] = np.mod(np.array(pts), box)
    pos[:, 3] = rng.integers(0, 5, len(pts))
    return pos.reshape(-1), np.array(bonds, np.uint32), list(box)


@pytest.mark.parametrize("case", ["fixture", "wrapped_chain", "random", "random_stretch", "cycles"])
def test_device_map_equals_the_oracle(case):
    g = _carrier()
    if case == "fixture":
        pos, bonds, box = fixture()
        nb = [x * 0.929 for x in box]
    elif case == "wrapped_chain":
        pos, bonds, box = wrapped_chain()
        nb = [x * 0.929 for x in box]
    elif case.startswith("random"):
        pos, bonds, box = random_molecules(3)
        nb = [box[0] * 0.93, box[1] * 0.97, box[2] * 0.9] if case == "random" else [box[0] * 1.2, box[1], box[2] * 1.07]
    else:
        # rings and a dense cluster with every pair within 1.3 sigma bonded: many paths to a bead
        pos, bonds, box = random_molecules(5, n_mol=100)
        p = pos.reshape(-1, 4)[:, :3].astype(np.float64)
        L = np.array(box)
        extra = [[i, j] for i in range(len(p)) for j in range(i + 1, len(p))
                 if np.linalg.norm((p[i] - p[j] + L / 2) % L - L / 2) < 1.3]
        bonds = np.concatenate([bonds, np.array(extra, np.uint32).reshape(-1)])
        nb = [x * 0.95 for x in box]
    ref = ob.scale_molecules_rigid(_abi, pos, bonds, box, nb)
    dev = g.scale_molecules_rigid(pos, bonds, box, nb)
    _assert_same(dev, ref)
    assert np.abs(bond_lengths(dev, nb, bonds) - bond_lengths(pos, box, bonds)).max() < 5e-6 or case == "cycles"
    g.dispose()


def _amphiphile_system():
    """A bonded soup (the oracle's boosted bond chemistry, 400 steps) on the device, in a box that
    leaves the grid room to shrink by 10% (planSoupGrid needs 5 cells of 2.947 sigma a side)."""
    opts = plain_opts(box=[18, 18, 18], start={"C": 900, "O": 260, "H": 0, "M": 160, "W": 0})
    cfg = boosted(cfgm.resolve(opts, P), attempt=0.9, accept=1.0, brk=0.02)
    o = ob.OracleSystem(_abi, cfg)
    o.relax(30, 0.1)
    o.step(400)
    st = dict(positions=o.read(ob.F_POS), bond_slots=o.read(ob.F_SLOTS), center_link=o.read(ob.F_CENTER),
              velocities=o.read(ob.F_VEL))
    return SoupSystem(cfg, st), cfg


def _edge_check_passes(before, after, box, nb, edges):
    return np.abs(bond_lengths(after, nb, edges) - bond_lengths(before, box, edges)).max() <= 1e-3


def test_scale_box_once_moves_rigid_units_as_the_oracle_map():
    g, cfg = _amphiphile_system()
    box = list(g.box)
    p0, bonds = g.particles(), g.bonds()
    assert bonds.size > 0
    nb = [x * 0.95 for x in box]
    g.scale_box_once(nb)
    _assert_same(g.particles(), ob.scale_molecules_rigid(_abi, p0, bonds, box, nb))
    assert list(g.box) == nb
    g.step(20)
    assert g.nonfinite_count() == dict(pos=0, vel=0)
    g.dispose()


def test_scale_box_once_with_cohesion():
    g, cfg = _amphiphile_system()
    box = list(g.box)
    p0, bonds = g.particles(), g.bonds()
    _, head_of = g.amphiphile_labels()
    members = np.nonzero(head_of != _abi.NONE)[0].astype(np.uint32)
    assert members.size > 0
    cut = float(cfg.rc_attr + cfg.wc)
    elig = np.zeros(g.n, np.uint8)
    elig[members] = 1
    edges = np.concatenate([bonds, ob.proximity_pairs(_abi, p0, box, cut, elig)])
    nb = [x * 1.05 for x in box]
    ref = ob.scale_molecules_rigid(_abi, p0, edges, box, nb)
    if _edge_check_passes(p0, ref, box, nb, edges):
        g.scale_box_once(nb, {"cutoff": cut, "memberIndices": members})
        _assert_same(g.particles(), ref)
    else:      # an aggregate wraps the box: the reference's self-check refuses, and so does the device
        with pytest.raises(_abi.SoupError, match="an intramolecular distance changed"):
            g.scale_box_once(nb, {"cutoff": cut, "memberIndices": members})
        assert np.array_equal(g.particles(), p0) and list(g.box) == box
    g.dispose()


def test_a_ring_around_the_box_is_refused_and_nothing_changes():
    """A bonded ring that wraps the periodic box has no rigid shape: the self-check refuses the
    change (soup/src/soup-box-scale.ts:117-128) before any position is written."""
    n, L = 16, 16.0
    pos = np.zeros((n, 4), np.float32)
    pos[:, 0] = np.arange(n) + 0.5
    pos[:, 1:3] = 6.0
    slots = np.full((n, 3), _abi.NONE, np.uint32)
    for i in range(n):
        slots[i, 0], slots[i, 1] = (i - 1) % n, (i + 1) % n
    opts = plain_opts(box=[L, L, L], start={"C": n, "O": 0, "H": 0, "M": 0, "W": 0})
    g = SoupSystem(cfgm.resolve(opts, P), dict(positions=pos.reshape(-1), bond_slots=slots.reshape(-1)))
    with pytest.raises(_abi.SoupError, match="an intramolecular distance changed"):
        g.scale_box_once([L * 0.9, L, L])
    assert np.array_equal(g.particles(), pos.reshape(-1)) and list(g.box) == [L, L, L]
    g.dispose()


def test_immobile_beads_refuse_a_box_change():
    opts = plain_opts()
    cfg = cfgm.resolve(opts, P)
    fr = np.zeros(cfg.n, np.uint32)
    fr[:5] = 1
    g = SoupSystem(cfg, dict(frozen=fr))
    with pytest.raises(_abi.SoupError, match="mineral sheet: 5 immobile beads"):
        g.scale_box_once([15.0, 15.0, 15.0])
    g.dispose()


def test_ramps_reach_the_target_box():
    g, cfg = _amphiphile_system()
    box = list(g.box)
    target = [x * 0.9 for x in box]
    g.scale_box_to(target, 3, 10)
    assert list(g.box) == target and g.steps == 20
    g.grow_box_to(box, 2, 5)
    assert list(g.box) == box and g.steps == 25
    assert g.nonfinite_count() == dict(pos=0, vel=0)
    g.dispose()


def test_a_box_too_small_for_the_grid_is_refused_before_anything_moves():
    """planSoupGrid's refusal (soup/src/soup-plan.ts:133-146) on a live box change: the same message,
    and the positions and the box as they were (set_box and scale_box_once alike)."""
    g = SoupSystem(cfgm.resolve(plain_opts(), P))   # box 16: 5 cells of 2.947 sigma, the minimum
    p0, box = g.particles(), list(g.box)
    for change in (lambda: g.set_box([14.0, 16.0, 16.0]), lambda: g.scale_box_once([14.0, 16.0, 16.0])):
        with pytest.raises(_abi.SoupError, match=r"neighbour grid: box=\[14,16,16\] .* it needs dims>=5"):
            change()
        assert np.array_equal(g.particles(), p0) and list(g.box) == box
    g.dispose()


def test_wall_radius_follows_the_live_box():
    """resizeSoupGrid rewrites the wall with liveRadius (soup/src/soup-buffers.ts:551,
    soup/src/soup-confine.ts:76-78): after set_box the force equals the oracle's for a system created
    in that box with the wall radius scaled the same way."""
    from helpers import confined_opts, rel_rms
    cfg = cfgm.resolve(confined_opts(), P)
    o = ob.OracleSystem(_abi, cfg)
    o.relax(20, 0.1)
    st = dict(positions=o.read(ob.F_POS), velocities=o.read(ob.F_VEL), charges=o.read(ob.F_CHARGES))
    g = SoupSystem(cfg, st)
    g.set_box([88.0, 88.0, 88.0])
    cfg2 = cfgm.resolve(confined_opts(box=[88, 88, 88], confine={"radiusSigma": 16 * 1.1, "stiffness": 100}), P)
    o2 = ob.OracleSystem(_abi, cfg2, st)
    assert rel_rms(g.forces(), o2.forces64()) < 1e-5
    # the wall acts: beads beyond the scaled radius from the new centre feel it
    p = st["positions"].reshape(-1, 4)[:, :3].astype(np.float64)
    assert (np.linalg.norm(p - 44.0, axis=1) > 17.6).any()
    g.dispose()

"""The box-scale map on the host: the oracle's scaleMoleculesRigid and proximityPairs pinned to the
reference's own checks (tests/soup-boxcycle.test.ts:17-150), and the ramp's increments
(soup/src/soup-box-scale.ts:228-250)."""
import math

import numpy as np
import pytest

import oracle_binding as ob
from protocell_genesis_b200 import _abi
from protocell_genesis_b200.soup import _box_ramp

CLOSE = 5e-6      # vitest toBeCloseTo(x, 5): |a - b| < 10^-5 / 2


def mi(d, L):
    return d - np.floor(d / L + 0.5) * L


def bond_lengths(pos, box, bonds):
    p = np.asarray(pos, np.float64).reshape(-1, 4)[:, :3]
    e = np.asarray(bonds).reshape(-1, 2)
    d = p[e[:, 0]] - p[e[:, 1]]
    for a in range(3):
        d[:, a] = mi(d[:, a], box[a])
    return np.sqrt((d ** 2).sum(axis=1))


def fixture(box=(20.0, 20.0, 20.0)):
    """tests/soup-boxcycle.test.ts:36-57: a two-tailed amphiphile (branch point), a 4-bead chain, a
    free monomer and a bonded pair straddling x = 0."""
    L = box[0]
    p = np.zeros((10, 4), np.float32)
    p[:, :3] = [[5, 5, 5], [6, 5, 5], [6, 6, 5], [10, 10, 10], [11, 10, 10], [11, 11, 10], [11, 11, 11],
                [2, 17, 3], [0.4, 8, 8], [L - 0.4, 8, 8]]
    bonds = np.array([0, 1, 1, 2, 3, 4, 4, 5, 5, 6, 8, 9], np.uint32)
    return p.reshape(-1), bonds, list(box)


def wrapped_chain():
    """tests/soup-boxcycle.test.ts:116-148: 24 beads 1 sigma apart along x, wrapped in a box of 10."""
    box = [10.0, 10.0, 10.0]
    p = np.zeros((24, 4), np.float32)
    p[:, 0] = [i - math.floor(i / 10.0) * 10.0 for i in range(24)]
    p[:, 1:3] = 5.0
    bonds = np.array([[i, i + 1] for i in range(23)], np.uint32).reshape(-1)
    return p.reshape(-1), bonds, box


def test_bonded_distances_survive_the_map():
    pos, bonds, box = fixture()
    nb = [x * 0.929 for x in box]
    after = ob.scale_molecules_rigid(_abi, pos, bonds, box, nb)
    assert np.abs(bond_lengths(after, nb, bonds) - bond_lengths(pos, box, bonds)).max() < CLOSE
    assert np.array_equal(after.reshape(-1, 4)[:, 3], pos.reshape(-1, 4)[:, 3])


def test_compress_then_stretch_restores_positions():
    pos, bonds, box = fixture()
    nb = [x * 0.929 for x in box]
    back = ob.scale_molecules_rigid(_abi, ob.scale_molecules_rigid(_abi, pos, bonds, box, nb), bonds, nb, box)
    assert np.abs(back.reshape(-1, 4)[:, :3] - pos.reshape(-1, 4)[:, :3]).max() < CLOSE


def test_unbonded_distances_shrink():
    pos, bonds, box = fixture()
    nb = [x * 0.929 for x in box]
    after = ob.scale_molecules_rigid(_abi, pos, bonds, box, nb)
    pair = np.array([7, 3], np.uint32)
    assert bond_lengths(after, nb, pair)[0] < bond_lengths(pos, box, pair)[0]


def test_wrapped_chain_keeps_its_bonds():
    pos, bonds, box = wrapped_chain()
    x = pos.reshape(-1, 4)[:, 0]
    assert (np.abs(np.diff(x)) > box[0] / 2).any()
    nb = [v * 0.929 for v in box]
    after = ob.scale_molecules_rigid(_abi, pos, bonds, box, nb)
    assert np.abs(bond_lengths(after, nb, bonds) - bond_lengths(pos, box, bonds)).max() < CLOSE


@pytest.mark.parametrize("side", [10.0, 5.0])
def test_proximity_pairs_are_every_close_eligible_pair(side):
    """A cell list of floor(box / cutoff) cells per axis finds exactly the pairs a brute-force scan
    finds; with fewer than three cells per axis the reference's loop lists some pairs twice."""
    rng = np.random.default_rng(4)
    n = 300
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = rng.uniform(0, side, (n, 3))
    elig = (rng.uniform(size=n) < 0.7).astype(np.uint8)
    box, cut = [side] * 3, 2.0
    pairs = ob.proximity_pairs(_abi, pos.reshape(-1), box, cut, elig).reshape(-1, 2)
    p = pos[:, :3].astype(np.float64)
    want = set()
    for i in range(n):
        if not elig[i]:
            continue
        d = p[i + 1:] - p[i]
        for a in range(3):
            d[:, a] = mi(d[:, a], side)
        for k in np.nonzero((d ** 2).sum(axis=1) <= cut * cut)[0]:
            if elig[i + 1 + k]:
                want.add((i, i + 1 + k))
    got = set(map(tuple, pairs.tolist()))
    assert got == want and len(want) > 0
    assert (len(pairs) > len(got)) == (side / cut < 3)
    assert (pairs[:, 0] < pairs[:, 1]).all()


def test_ramp_increments():
    """applyBoxScale's log-linear increments; the last one exactly the target."""
    fb, tb = [30.0, 30.0, 40.0], [27.0, 28.0, 40.0]
    r = _box_ramp(fb, tb, 4)
    assert [last for _, last in r] == [False, False, False, True]
    assert r[-1][0] == tb
    for s, (box, _) in enumerate(r[:-1], start=1):
        assert box == [fb[a] * math.exp(math.log(tb[a] / fb[a]) * s / 4) for a in range(3)]

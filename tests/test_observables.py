"""Observables on the host and in the oracle (engine/src/metrics.ts; soup/src/electrostatics.ts:291-303,
520-561).  The device reductions are checked against the oracle in test_gpu_observables.py."""
import math

import numpy as np
import pytest

import oracle_binding as ob
from protocell_genesis_b200 import _abi
from protocell_genesis_b200 import observables as obs


def test_henderson_alpha_and_apparent_pka():
    assert obs.henderson_alpha(4.6, 4.6) == pytest.approx(0.5)
    assert obs.henderson_alpha(5.6, 4.6) == pytest.approx(10 / 11)
    for ph in (3.9, 4.9, 5.9, 7.0):
        assert obs.apparent_pka(obs.henderson_alpha(ph, 4.6), ph) == pytest.approx(4.6, abs=1e-12)
    assert math.isnan(obs.apparent_pka(0.0, 7.0)) and math.isnan(obs.apparent_pka(1.0, 7.0))


def test_area_per_lipid():
    assert obs.area_per_lipid([10.0, 12.0, 30.0], 100) == pytest.approx(2.4)


def _profile(peaks, bins=100, box_z=40.0, width=0.5, n=400):
    dz = box_z / bins
    z = [(i + 0.5) * dz for i in range(bins)]
    head = [0] * bins
    for c in peaks:
        for i, zi in enumerate(z):
            head[i] += int(round(n * math.exp(-0.5 * ((zi - c) / width) ** 2)))
    return {"z": z, "head": head, "tail": [0] * bins}


def test_bilayer_thickness_from_two_leaflets():
    pr = _profile([17.9, 22.3])
    assert obs.bilayer_thickness(pr) == pytest.approx(4.4, abs=0.05)   # sub-bin parabola, 0.4 bins
    lo_hi = obs.bilayer_peaks(pr)
    assert lo_hi["lower"] < lo_hi["upper"]


def test_bilayer_peaks_refuses_what_is_not_a_bilayer():
    with pytest.raises(ValueError, match="empty"):
        obs.bilayer_peaks({"z": [0.5, 1.5], "head": [0, 0], "tail": [0, 0]})
    with pytest.raises(ValueError, match="second peak not found"):
        obs.bilayer_peaks(_profile([20.0], width=0.2))


def test_sum_center_drop():
    a, b = _profile([10.0]), _profile([30.0])
    s = obs.sum_profiles([a, b])
    assert s["head"] == [x + y for x, y in zip(a["head"], b["head"])]
    with pytest.raises(ValueError, match="different grids"):
        obs.sum_profiles([a, _profile([10.0], bins=50)])
    pos = np.array([[1, 1, 2, 0], [1, 1, 4, 1], [1, 1, 9, 0], [1, 1, -1, 1]], np.float32).reshape(-1)
    c = obs.center_membrane_z(pos, [10.0, 10.0, 10.0]).reshape(-1, 4)
    assert c[:, 2].mean() == pytest.approx(5.0, abs=1e-5)
    kept, esc = obs.drop_escaped_z(pos, [10.0, 10.0, 10.0])
    assert esc == 1 and len(kept) == 12


def test_oracle_pairing_counts_a_hand_made_line():
    # heads (kind 1): A q=-1 at x=0, B q=0 at x=1.0, C q=-1 at x=1.9; contact 1.12; a water bead far off
    pos = np.array([[5.0, 5, 5, 1], [6.0, 5, 5, 1], [6.9, 5, 5, 1], [1.0, 1, 1, 4]], np.float32).reshape(-1)
    q = np.array([-1, 0, -1, 0], np.float32)
    w, unlike, like, paired, charged, heads = ob.pairing_stats(_abi, pos, q, [20.0] * 3, 1, 1.12)
    assert (w, unlike, like, paired, charged, heads) == (3, 4, 0, 3, 2, 3)


def test_oracle_pairing_equals_brute_force_definition():
    rng = np.random.default_rng(5)
    n, box = 300, 9.0
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = rng.uniform(0, box, (n, 3))
    pos[:, 3] = rng.choice([1.0, 4.0], n)
    q = np.where(rng.random(n) < 0.5, -1.0, 0.0).astype(np.float32) * (pos[:, 3] == 1)
    contact = 1.0665
    heads = np.nonzero(pos[:, 3] == 1)[0]
    d = pos[heads, None, :3].astype(np.float64) - pos[None, heads, :3].astype(np.float64)
    d -= np.floor(d / box + 0.5) * box
    r = np.sqrt((d ** 2).sum(-1))
    np.fill_diagonal(r, np.inf)
    near = r <= contact
    ch = q[heads] != 0
    unl = near & (ch[:, None] != ch[None, :])
    best = np.argmin(r, axis=1)
    paired = int(((r[np.arange(len(heads)), best] <= contact) & (ch != ch[best])).sum())
    want = (int(near.any(1).sum()), int(unl.sum()), int((near & ~unl).sum()), paired, int(ch.sum()), len(heads))
    assert ob.pairing_stats(_abi, pos.reshape(-1), q, [box] * 3, 1, contact) == want


def test_oracle_density_profile_equals_histogram():
    rng = np.random.default_rng(2)
    pos = np.zeros((5000, 4), np.float32)
    pos[:, :3] = rng.uniform(0, 20.0, (5000, 3))
    pos[:, 3] = rng.integers(0, 5, 5000)
    pos[:7, 2] = 20.5                                    # escaped
    head, tail, esc = ob.density_profile_z(_abi, pos.reshape(-1), 20.0, 40, 0b10)
    inb = pos[7:]
    hh = np.histogram(inb[inb[:, 3] == 1, 2], bins=40, range=(0, 20.0))[0]
    tt = np.histogram(inb[inb[:, 3] != 1, 2], bins=40, range=(0, 20.0))[0]
    assert esc == 7 and np.array_equal(head, hh) and np.array_equal(tail, tt)


def test_smith_eigenvalues_and_vectors():
    rng = np.random.default_rng(9)
    for _ in range(50):
        a = rng.normal(size=(3, 3))
        m = a @ a.T
        g = (m[0, 0], m[1, 1], m[2, 2], m[0, 1], m[0, 2], m[1, 2])
        lam = obs.symmetric_eigenvalues_3x3(*g)
        assert np.allclose(lam, np.linalg.eigvalsh(m), rtol=1e-10, atol=1e-12)
        v = obs.symmetric_eigenvector_3x3(*g, lam[0])
        assert np.allclose(m @ np.array(v), lam[0] * np.array(v), atol=1e-8)
    assert obs.symmetric_eigenvalues_3x3(3.0, 1.0, 2.0, 0.0, 0.0, 0.0) == [1.0, 2.0, 3.0]
    assert obs.symmetric_eigenvector_3x3(1.0, 1.0, 1.0, 0.0, 0.0, 0.0, 1.0) is None   # repeated


def test_oracle_shape_of_a_rod_across_the_boundary():
    # 9 beads 1 sigma apart along x, straddling x = 0 of a 20 sigma box (span 8 < L/2 from any bead):
    # moments 0, 0, (9^2 - 1)/12
    box = [20.0] * 3
    pos = np.zeros((9, 4), np.float32)
    pos[:, 0] = np.mod(np.arange(9) - 4.0, 20.0)
    pos[:, 1:3] = 7.0
    n, centre, g = ob.aggregate_shape(_abi, pos.reshape(-1), np.arange(9), box)
    m = obs.shape_metrics({"size": n, "label": 0, "centre": centre, "gyration": list(g)})
    assert n == 9
    assert m["principalMoments"][2] == pytest.approx(80.0 / 12.0, abs=1e-9)
    assert m["principalMoments"][0] == pytest.approx(0.0, abs=1e-9)
    assert m["radiusOfGyration"] == pytest.approx(math.sqrt(80.0 / 12.0))
    assert m["flatnessRatio"] == pytest.approx(0.0, abs=1e-9)


def test_periodic_centre_matches_the_oracle():
    """periodicCentreOf against the oracle's restatement, on a cluster that straddles a box face and
    on uniform points (no meaningful centre)."""
    import oracle_binding as ob
    from protocell_genesis_b200 import _abi
    from protocell_genesis_b200 import observables as obs
    rng = np.random.default_rng(4)
    box = [20.0, 20.0, 20.0]
    n = 400
    pos = np.zeros((n, 4), np.float32)
    pos[:200, :3] = np.mod(rng.normal(0.0, 1.5, (200, 3)) + [19.5, 10.0, 0.5], 20.0)
    pos[200:, :3] = rng.uniform(0, 20, (200, 3))
    flat = pos.reshape(-1)
    for idx in (np.arange(200, dtype=np.uint32), np.arange(200, 400, dtype=np.uint32)):
        c = obs.periodic_centre(flat, idx, box, 0.05)
        co = ob.periodic_centre(_abi, flat, idx, box, 0.05)
        if co is None:
            assert c is None
        else:
            assert np.allclose(c, co, atol=1e-9)

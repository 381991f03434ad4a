"""The stage ladder and the box-wide enclosed volume on the host and the oracle:
stageFromEvidence's ladder (tests/soup-amphiphile.test.ts:85-127), enclosedVolumeFromPositions'
recentring (tests/closure.test.ts:45-72: a shell moved across a periodic face, or into a corner, keeps
its cavity; a flat sheet has none) and buildClusterUnionFind's periodicZ switch."""
import math

import numpy as np
import pytest

import oracle_binding as ob
from protocell_genesis_b200 import _abi, config as cfgm, observables as obs

P = cfgm.load_params()
T = obs.load_stage_thresholds()
TT_CUTOFF = cfgm.wca_cutoff(P["params"]["beadSizes"]["tail_tail"]) + P["params"]["wc"]
EMPTY = {"aggregateCount": 0, "sizeHistogram": [], "aggregates": [], "qualifyingAggregateCount": 0,
         "amphiphilesInQualifying": 0, "amphiphileShareInQualifying": 0.0, "hasLamellarAggregate": False,
         "hasVesicleAggregate": False}


def _evidence(fraction, analysis):
    return {"amphiphileFraction": fraction, "largestAggregateFraction": 0.0, "headPeaks": 0, "enclosedVolume": 0.0,
            "aggregateAnalysis": analysis}


def test_amphiphiles_before_aggregates():
    assert obs.stage_from_evidence(_evidence(T["amphiphileFraction"] + 0.01, EMPTY), T) == "amphiphiles"


def test_saturated_analysis_without_amphiphiles_is_monomers():
    sat = {"aggregateCount": 3, "sizeHistogram": [500, 400, 300], "aggregates": [], "qualifyingAggregateCount": 3,
           "amphiphilesInQualifying": 1200, "amphiphileShareInQualifying": 1, "hasLamellarAggregate": True,
           "hasVesicleAggregate": True}
    assert obs.stage_from_evidence(_evidence(0.0, sat), T) == "monomers"


def test_ladder_order_vesicle_bilayer_micelles():
    many = dict(EMPTY, qualifyingAggregateCount=3, amphiphileShareInQualifying=0.9)
    assert obs.stage_from_evidence(_evidence(1.0, many), T) == "micelles"
    assert obs.stage_from_evidence(_evidence(1.0, dict(many, amphiphileShareInQualifying=0.2)), T) == "amphiphiles"
    assert obs.stage_from_evidence(_evidence(1.0, dict(many, hasLamellarAggregate=True)), T) == "bilayer"
    both = dict(many, hasLamellarAggregate=True, hasVesicleAggregate=True)
    assert obs.stage_from_evidence(_evidence(1.0, both), T) == "vesicle"


def shell(rng, radius=8.0, thickness=1.5, count=40_000, centre=20.0):
    u = rng.uniform(-1, 1, count)
    phi = rng.uniform(0, 2 * math.pi, count)
    r = radius + (rng.uniform(0, 1, count) - 0.5) * thickness
    s = np.sqrt(1 - u * u)
    p = np.ones((count, 4), np.float32)
    p[:, 0], p[:, 1], p[:, 2] = centre + r * s * np.cos(phi), centre + r * s * np.sin(phi), centre + r * u
    return p


def shift_xy(p, box, dx, dy):
    q = p.copy()
    q[:, 0] = np.mod(q[:, 0].astype(np.float64) + dx, box[0]).astype(np.float32)
    q[:, 1] = np.mod(q[:, 1].astype(np.float64) + dy, box[1]).astype(np.float32)
    return q


def oracle_enclosed_volume(p, box, cell=0.5, radius=0.6):
    """enclosedVolumeFromPositions through the oracle: z-open labels, the host recentring, the grid."""
    m = np.arange(p.shape[0], dtype=np.uint32)
    _, labels = ob.cluster_labels(_abi, p.reshape(-1), m, box, TT_CUTOFF, periodic_z=False)
    shift = obs.largest_cluster_shift(p, labels, box)
    return ob.box_cavity_volume(_abi, obs.recenter_positions(p, shift, box), box, cell, radius)


def test_recentring_keeps_the_cavity_of_a_shell_across_a_face_and_in_a_corner():
    box = [40.0, 40.0, 40.0]
    p = shell(np.random.default_rng(1))
    v0 = oracle_enclosed_volume(p, box)
    assert v0 > T["enclosedVolume"]
    for dx, dy in ((-20, 0), (-20, -20)):
        v = oracle_enclosed_volume(shift_xy(p, box, dx, dy), box)
        assert 0.7 * v0 < v < 1.3 * v0


def test_flat_sheet_has_no_cavity():
    rng = np.random.default_rng(2)
    p = np.ones((20_000, 4), np.float32)
    p[:, 0], p[:, 1] = rng.uniform(0, 40, 20_000), rng.uniform(0, 40, 20_000)
    p[:, 2] = 20 + (rng.uniform(0, 1, 20_000) - 0.5)
    assert ob.box_cavity_volume(_abi, p.reshape(-1), [40.0, 40.0, 40.0], 0.5, 0.6) == 0.0


def test_z_open_clusters_do_not_join_across_the_z_faces():
    box = [10.0, 10.0, 10.0]
    p = np.array([[5, 5, 0.2, 0], [5, 5, 9.9, 0], [9.9, 5, 5, 0], [0.3, 5, 5, 0]], np.float32)
    m = np.arange(4, dtype=np.uint32)
    n_open, lab_open = ob.cluster_labels(_abi, p.reshape(-1), m, box, 1.0, periodic_z=False)
    n_per, lab_per = ob.cluster_labels(_abi, p.reshape(-1), m, box, 1.0, periodic_z=True)
    assert n_open == 3 and lab_open.tolist() == [0, 1, 2, 2]
    assert n_per == 2 and lab_per.tolist() == [0, 0, 2, 2]


def test_largest_cluster_shift_ties_go_to_the_cluster_met_first():
    box = [10.0, 10.0, 10.0]
    p = np.array([[2, 2, 2, 0], [8, 8, 8, 0], [2.5, 2, 2, 0], [8.5, 8, 8, 0]], np.float32)
    labels = np.array([0, 1, 0, 1], np.uint32)
    sx, sy, sz = obs.largest_cluster_shift(p, labels, box)
    assert (sx, sy, sz) == pytest.approx((5 - 2.25, 3.0, 3.0))
    # a cluster that wraps in x: centre through minimum-image offsets from its first member
    q = np.array([[9.8, 1, 1, 0], [0.2, 1, 1, 0]], np.float32)
    sx, _, _ = obs.largest_cluster_shift(q, np.zeros(2, np.uint32), box)
    assert sx == pytest.approx(5.0, abs=1e-5)   # centre at x = 0 (10)

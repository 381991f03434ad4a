"""detectStage on the device (soup/src/stages.ts:204-289): the z-open and periodic cluster labels and
the box-grid enclosed volume equal the oracle's, and the reference's four synthetic arrangements
read as their stages (tests/soup-aggregates.test.ts:80-234: micelles, bilayer, vesicle, and the dense
ball as none of the three)."""
import json

import numpy as np
import pytest

import aggregate_scenarios as sc
import oracle_binding as ob
from protocell_genesis_b200 import _abi, config as cfgm, observables as obs
from protocell_genesis_b200.soup import SoupSystem
from test_stages import TT_CUTOFF, shell, shift_xy

pytestmark = pytest.mark.gpu
P = cfgm.load_params()
ST = obs.load_stage_thresholds()


def _system(pos, bonds, box):
    n = pos.size // 4
    kinds = pos.reshape(-1, 4)[:, 3]
    start = {"C": int((kinds == sc.KIND_C).sum()), "O": int((kinds == sc.KIND_O).sum()), "H": 0, "M": 0, "W": 0}
    opts = cfgm.SoupOptions(box=box, seed=1, kT=1.1, start=start, electrostatics={"enabled": False},
                            verlet_override={"listCapacity": 2048})
    return SoupSystem(cfgm.resolve(opts, P), {"positions": pos, "bond_slots": sc.slots_of(n, bonds)})


def _shell_system(dx, dy):
    """The closure test's shell (12,000 unbonded carbon beads here), moved by (dx, dy)."""
    box = [40.0, 40.0, 40.0]
    p = shift_xy(shell(np.random.default_rng(1), count=12_000), box, dx, dy)
    p[:, 3] = sc.KIND_C
    return _system(p.reshape(-1), np.zeros(0, np.uint32), box), p, box


@pytest.mark.parametrize("periodic_z", [False, True])
def test_cluster_labels_equal_the_oracle(periodic_z):
    g, p, box = _shell_system(-20, 0)
    p2 = p.copy()
    p2[:, 2] = np.mod(p2[:, 2] + 17.0, 40.0)   # the shell now also straddles the z faces
    g.write_state({"positions": p2.reshape(-1)})
    rng = np.random.default_rng(4)
    members = np.sort(rng.choice(p.shape[0], 6000, replace=False)).astype(np.uint32)
    nd, dev = g.cluster_labels(members, TT_CUTOFF * 0.6, periodic_z)
    no, ref = ob.cluster_labels(_abi, p2.reshape(-1), members, box, TT_CUTOFF * 0.6, periodic_z)
    assert nd == no and np.array_equal(dev, ref)
    g.dispose()


@pytest.mark.parametrize("dx,dy", [(0, 0), (-20, 0), (-20, -20)])
def test_enclosed_volume_equals_the_oracle_and_survives_the_faces(dx, dy):
    g, p, box = _shell_system(dx, dy)
    members = np.arange(p.shape[0], dtype=np.uint32)
    dev = obs.enclosed_volume_from_positions(g, members, g.particles(), ST["closureCell"], ST["closureRadius"])
    _, labels = ob.cluster_labels(_abi, p.reshape(-1), members, box, TT_CUTOFF, periodic_z=False)
    shifted = obs.recenter_positions(p, obs.largest_cluster_shift(p, labels, box), box)
    ref = ob.box_cavity_volume(_abi, shifted, box, ST["closureCell"], ST["closureRadius"])
    assert dev == ref and dev > ST["enclosedVolume"]
    g.dispose()


@pytest.mark.parametrize("scenario,stage", [(sc.micelles, "micelles"), (sc.flat_layer, "bilayer"),
                                            (sc.hollow_shell, "vesicle"), (sc.dense_ball, "amphiphiles")])
def test_detect_stage_on_the_reference_arrangements(scenario, stage):
    g = _system(*scenario())
    r = obs.detect_stage(g)
    e = r["evidence"]
    assert r["stage"] == stage
    assert e["amphiphileFraction"] == 1.0
    n_agg = e["aggregateAnalysis"]["aggregateCount"]
    assert e["largestAggregateFraction"] == pytest.approx(1.0 / 3 if stage == "micelles" else 1.0)
    assert n_agg == (3 if stage == "micelles" else 1)
    if stage == "vesicle":
        assert e["enclosedVolume"] > ST["enclosedVolume"]
    g.dispose()


def test_detect_stage_reads_the_parcel_off_a_confined_system():
    """stages.ts:274-279: a confined system's parcel comes from its live confinement (box centre,
    live wall radius) when the caller gives none; after a box change the radius follows the box."""
    from helpers import confined_opts
    g = SoupSystem(cfgm.resolve(confined_opts(), P))
    g.relax_cold_start(30, 0.1)
    g.step(20)
    cf = g.confinement()
    assert cf["radiusLive"] == pytest.approx(16.0) and cf["boxLive"] == [80.0, 80.0, 80.0]
    for box in ([80.0, 80.0, 80.0], [78.0, 78.0, 78.0]):
        g.set_box(box)
        live = 16.0 * box[0] / 80.0
        assert g.confinement()["radiusLive"] == pytest.approx(live)
        implicit = obs.detect_stage(g)
        explicit = obs.detect_stage(g, parcel={"centre": [b / 2 for b in box], "radius": live})
        assert implicit["stage"] == explicit["stage"]
        same = lambda e: json.dumps(e["evidence"], default=str, sort_keys=True)
        assert same(implicit) == same(explicit)
    g.dispose()

"""analyzeAggregates with shapeOfAggregate's full detail on the device, on the reference's four
synthetic arrangements (tests/soup-aggregates.test.ts:80-231): the counts, the shape gates, the
head-shell counts, the cavity and the lamellar / vesicle flags the reference asserts; and the device
unwrap and local cavity equal to the oracle's."""
import numpy as np
import pytest

import aggregate_scenarios as sc
import oracle_binding as ob
from protocell_genesis_b200 import _abi, config as cfgm, observables as obs
from protocell_genesis_b200.soup import SoupSystem

pytestmark = pytest.mark.gpu
P = cfgm.load_params()
ST = P["stageThresholds"]


def _system(scenario):
    pos, bonds, box = scenario()
    n = pos.size // 4
    kinds = pos.reshape(-1, 4)[:, 3]
    start = {"C": int((kinds == sc.KIND_C).sum()), "O": int((kinds == sc.KIND_O).sum()), "H": 0, "M": 0, "W": 0}
    opts = cfgm.SoupOptions(box=box, seed=1, kT=1.1, start=start, electrostatics={"enabled": False},
                            verlet_override={"listCapacity": 2048})
    return SoupSystem(cfgm.resolve(opts, P), {"positions": pos, "bond_slots": sc.slots_of(n, bonds)}), pos, box


def test_micelles():
    g, _, _ = _system(sc.micelles)
    a = obs.analyze_aggregates(g, sc.cutoff())
    assert a["aggregateCount"] == 3 and a["sizeHistogram"] == [20, 20, 20]
    assert a["qualifyingAggregateCount"] == 3 and a["amphiphileShareInQualifying"] == 1
    assert not a["hasLamellarAggregate"] and not a["hasVesicleAggregate"]
    g.dispose()


def test_flat_layer_is_lamellar_from_the_transverse_profile():
    g, _, _ = _system(sc.flat_layer)
    a = obs.analyze_aggregates(g, sc.cutoff())
    assert a["aggregateCount"] == 1
    s = a["aggregates"][0]
    assert s["flatnessRatio"] <= ST["lamellarFlatnessRatio"] and s["inPlaneSymmetry"] >= ST["lamellarInPlaneSymmetryMin"]
    assert s["transverseHeadShells"] == 2 and a["hasLamellarAggregate"]
    assert s["cavityVolume"] == 0 and not a["hasVesicleAggregate"]
    g.dispose()


def test_hollow_shell_is_a_vesicle():
    g, _, _ = _system(sc.hollow_shell)
    a = obs.analyze_aggregates(g, sc.cutoff())
    assert a["aggregateCount"] == 1
    s = a["aggregates"][0]
    assert s["radialHeadShells"] == 2 and s["cavityVolume"] > ST["enclosedVolume"]
    assert a["hasVesicleAggregate"] and not a["hasLamellarAggregate"]
    g.dispose()


def test_dense_ball_is_one_unstructured_aggregate():
    g, _, _ = _system(sc.dense_ball)
    a = obs.analyze_aggregates(g, sc.cutoff())
    assert a["aggregateCount"] == 1 and a["sizeHistogram"][0] > ST["minAmphiphilesPerAggregate"] * 10
    assert a["qualifyingAggregateCount"] == 1
    assert not a["hasLamellarAggregate"] and not a["hasVesicleAggregate"]
    g.dispose()


@pytest.mark.parametrize("scenario", [sc.flat_layer, sc.hollow_shell, sc.dense_ball])
def test_unwrap_and_cavity_equal_the_oracle(scenario):
    g, pos, box = _system(scenario)
    # the arrangement moved by half a box, so that it straddles every face
    shifted = pos.reshape(-1, 4).copy()
    shifted[:, :3] = np.mod(shifted[:, :3] + np.array(box, np.float32) / 2 + 0.37, np.array(box, np.float32))
    g.write_state({"positions": shifted.reshape(-1)})
    members = np.arange(g.n, dtype=np.uint32)
    dev = g.aggregate_unwrap(members)
    ref = ob.unwrap_aggregate(_abi, shifted.reshape(-1), members, box)
    assert np.array_equal(dev.view(np.uint32), ref.view(np.uint32))
    cell, radius = ST["closureCell"], ST["closureRadius"]
    assert g.local_cavity_volume(dev, cell, radius) == ob.local_cavity_volume(_abi, ref, cell, radius)
    g.dispose()

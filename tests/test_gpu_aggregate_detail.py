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


def test_hollow_shell_with_water_is_closed_by_its_encapsulated_water():
    """With water indices given, the vesicle flag follows the encapsulated water (isVesicleShape,
    soup/src/aggregates.ts:307-315): water inside the shell is unreached by the flood from outside."""
    pos, bonds, box = sc.hollow_shell()
    rng = np.random.default_rng(3)
    c = np.array([30.0, 30.0, 30.0])
    d = rng.normal(size=(4000, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    inside = c + d[:600] * (rng.uniform(0, 1, 600) ** (1 / 3) * 6.5)[:, None]
    outside = c + d[600:] * rng.uniform(14.0, 28.0, 3400)[:, None]
    w = np.zeros((4000, 4), np.float32)
    w[:, :3] = np.concatenate([inside, outside])
    w[:, 3] = next(k for k, m in enumerate(P["monomers"]) if m["solvent"])
    allpos = np.concatenate([pos.reshape(-1, 4), w]).reshape(-1)
    n = allpos.size // 4
    kinds = allpos.reshape(-1, 4)[:, 3]
    start = {"C": int((kinds == sc.KIND_C).sum()), "O": int((kinds == sc.KIND_O).sum()), "H": 0, "M": 0, "W": 4000}
    opts = cfgm.SoupOptions(box=box, seed=1, kT=1.1, start=start, electrostatics={"enabled": False},
                            verlet_override={"listCapacity": 2048})
    g = SoupSystem(cfgm.resolve(opts, P), {"positions": allpos, "bond_slots": sc.slots_of(n, bonds)})
    water = np.arange(pos.size // 4, n, dtype=np.uint32)
    a = obs.analyze_aggregates(g, sc.cutoff(), water=water)
    ew = a["aggregates"][0]["encapsulatedWater"]
    assert ew is not None and ew["encapsulatedCount"] == 600 and ew["closed"]
    assert a["hasVesicleAggregate"]
    g.dispose()

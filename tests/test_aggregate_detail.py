"""shapeOfAggregate's host parts and the oracle's local cavity (soup/src/aggregates.ts:83-120,
273-385): head-peak counting, the coordinate packing, and localCavityVolume on the reference's
synthetic arrangements (tests/soup-aggregates.test.ts:117-191)."""
import numpy as np
import pytest

import aggregate_scenarios as sc
import oracle_binding as ob
from protocell_genesis_b200 import _abi, config as cfgm, observables as obs

P = cfgm.load_params()
ST = P["stageThresholds"]
POLAR = [bool(m["polar"]) for m in P["monomers"]]
HP = (ST["aggregateHeadDensityBins"], ST["aggregateMinHeadsPerBin"], ST["headPeakSeparationMin"],
      ST["headPeakSeparationMax"])


def _layers(zs, n_each, kind):
    p = np.zeros((len(zs) * n_each, 4), np.float32)
    for k, z in enumerate(zs):
        p[k * n_each:(k + 1) * n_each, 2] = z
    p[:, 3] = kind
    return p


def test_head_peaks_two_layers_one_layer_too_few_none():
    box = [1.0, 1.0, 10.0]
    two = np.concatenate([_layers([2.2, 6.6], 40, sc.KIND_O), _layers([4.4], 80, sc.KIND_C)]).reshape(-1)
    assert obs.compute_head_peaks(two, box, POLAR, *HP) == 2
    one = np.concatenate([_layers([5.0], 80, sc.KIND_O), _layers([2.0], 40, sc.KIND_C)]).reshape(-1)
    assert obs.compute_head_peaks(one, box, POLAR, *HP) == 1
    near = np.concatenate([_layers([4.0, 5.5], 40, sc.KIND_O)]).reshape(-1)   # 1.5 apart: below the band
    assert obs.compute_head_peaks(near, box, POLAR, *HP) == 1
    few = _layers([2.2, 6.6], 5, sc.KIND_O).reshape(-1)                      # 10 heads / 10 bins < 2
    assert obs.compute_head_peaks(few, box, POLAR, *HP) == obs.HEAD_PEAKS_UNAVAILABLE
    assert obs.compute_head_peaks(_layers([3.0], 30, sc.KIND_C).reshape(-1), box, POLAR, *HP) == 0


def test_profile_along_and_escape():
    p, box = obs.profile_along([3.0, 5.0, 4.0], [1, 0, 1])
    q = p.reshape(-1, 4)
    assert q[:, 2].tolist() == [0.0, 2.0, 1.0] and box == [1.0, 1.0, pytest.approx(2.0002)]
    with pytest.raises(ValueError, match="outside"):
        obs.density_profile_of(np.array([0, 0, 11.0, 0], np.float32), 10.0, 10)


def _unwrapped(scenario):
    pos, bonds, box = scenario()
    members = np.arange(pos.size // 4, dtype=np.uint32)
    return ob.unwrap_aggregate(_abi, pos, members, box)


def test_local_cavity_of_the_reference_arrangements():
    """The hollow shell encloses more than the closure minimum; the flat patch and the dense ball
    enclose nothing (tests/soup-aggregates.test.ts:144-145, 184)."""
    cell, radius = ST["closureCell"], ST["closureRadius"]
    shell = ob.local_cavity_volume(_abi, _unwrapped(sc.hollow_shell), cell, radius)
    assert ST["enclosedVolume"] < shell < 4 / 3 * np.pi * 12.4 ** 3   # the interior and the wall's own pockets
    assert ob.local_cavity_volume(_abi, _unwrapped(sc.flat_layer), cell, radius) == 0.0
    assert ob.local_cavity_volume(_abi, _unwrapped(sc.dense_ball), cell, radius) == 0.0


def test_unwrap_about_the_first_member():
    pos = np.array([[19.5, 1, 1, 0], [0.3, 1, 1, 1], [19.9, 19.8, 0.1, 0]], np.float32).reshape(-1)
    u = ob.unwrap_aggregate(_abi, pos, np.array([0, 1, 2], np.uint32), [20.0, 20.0, 20.0]).reshape(-1, 4)
    assert u[1, 0] == pytest.approx(20.3, abs=1e-5) and u[2, 1] == pytest.approx(-0.2, abs=1e-5)
    assert u[2, 2] == np.float32(0.1) and u[0, 0] == np.float32(19.5)
    assert u[:, 3].tolist() == [0, 1, 0]


def test_parcel_restricts_the_bulk_density_to_the_parcel():
    """encapsulatedWaterVolume's parcel (soup/src/water-closure.ts:280-288, 323-337): water only within
    18 sigma of the shell's centre and vacuum beyond; the bulk density over the parcel's reached cells
    is the water's own density, over the whole box it is diluted by the vacuum."""
    from test_oracle_pins import SYN_BOX, _assemble, _shell
    rng = np.random.default_rng(5)
    centre = np.array([25.0, 25.0, 25.0])
    members = _shell(rng, centre)
    d = rng.normal(size=(6000, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    water = centre + d * rng.uniform(13.0, 18.0, 6000)[:, None]
    pos, mem, wat = _assemble(members, water)
    c = ob.periodic_centre(_abi, pos, mem, SYN_BOX, P["circularAlpha"])
    plain = ob.closure(_abi, pos, mem, wat, SYN_BOX, c, ST["closureCell"], ST["closureRadius"], ST["enclosedVolume"])
    parcel = ob.closure_in_parcel(_abi, pos, mem, wat, SYN_BOX, c, ST["closureCell"], ST["closureRadius"],
                                  ST["enclosedVolume"], centre, 18.0)
    shell_vol = 4 / 3 * np.pi * (18.0 ** 3 - 12.6 ** 3)
    assert parcel.bulk_water_density == pytest.approx(6000 / shell_vol, rel=0.1)
    assert parcel.bulk_water_density > 3 * plain.bulk_water_density
    assert parcel.encapsulated_count == plain.encapsulated_count == 0
    assert parcel.total_empty_cells == plain.total_empty_cells and parcel.unreached_cells == plain.unreached_cells

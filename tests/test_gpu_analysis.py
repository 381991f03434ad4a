"""Closure flood fill, amphiphile recognition and aggregate labels on the device vs the oracle:
identical occupancy-derived counts, seed cell and labels (FP64, JavaScript rounding, canonical
minimum-index labels)."""
import numpy as np
import pytest

import oracle_binding as ob
from helpers import boosted, plain_opts
from protocell_genesis_b200 import _abi, config as cfgm
from protocell_genesis_b200.soup import SoupSystem
from test_oracle_pins import SYN_BOX, ST, _assemble, _shell, _water

pytestmark = pytest.mark.gpu
P = cfgm.load_params()


def _system_for(pos, nmem):
    n = len(pos) // 4
    opts = cfgm.SoupOptions(box=SYN_BOX, seed=1, kT=1.1, start={"C": nmem, "O": 0, "H": 0, "M": 0, "W": n - nmem},
                            verlet_override={"listCapacity": 4096})
    cfg = cfgm.resolve(opts, P)
    return SoupSystem(cfg, {"positions": pos})


@pytest.mark.parametrize("hole", [False, True])
def test_closure_matches_oracle(hole):
    rng = np.random.default_rng(77 + hole)
    centre = np.array([25.0, 25.0, 25.0])
    members = _shell(rng, centre, hole=np.array([0.0, 1.0, 0.0]) if hole else None)
    pos, mem, wat = _assemble(members, _water(rng, centre, 800, 5000))
    g = _system_for(pos, len(mem))
    c = ob.periodic_centre(_abi, pos, mem, SYN_BOX, P["circularAlpha"])
    ro = ob.closure(_abi, pos, mem, wat, SYN_BOX, c, ST["closureCell"], ST["closureRadius"], ST["enclosedVolume"])
    rg = g.closure(mem, wat, c, ST["closureCell"], ST["closureRadius"], ST["enclosedVolume"])
    assert rg["encapsulatedCount"] == ro.encapsulated_count
    assert rg["totalEmptyCells"] == ro.total_empty_cells and rg["unreachedCells"] == ro.unreached_cells
    assert rg["seedCell"] == ro.seed_cell
    assert rg["bulkWaterDensity"] == pytest.approx(ro.bulk_water_density, rel=1e-12)
    assert rg["closed"] == bool(ro.closed)
    g.dispose()


def test_amphiphiles_and_aggregates_match_oracle():
    opts = plain_opts(box=[15, 15, 15], start={"C": 900, "O": 260, "H": 0, "M": 160, "W": 0})
    cfg = boosted(cfgm.resolve(opts, P), attempt=0.9, accept=1.0, brk=0.02)
    o = ob.OracleSystem(_abi, cfg)
    o.relax(30, 0.1)
    o.step(400)
    st = dict(positions=o.read(ob.F_POS), bond_slots=o.read(ob.F_SLOTS), center_link=o.read(ob.F_CENTER))
    g = SoupSystem(cfg, st)
    polar = np.zeros(8, np.uint32)
    for k, m in enumerate(P["monomers"]):
        polar[k] = 1 if m["polar"] else 0
    n_o, head_o = ob.amphiphiles(_abi, st["positions"], st["bond_slots"], polar)
    n_g, head_g = g.amphiphile_labels()
    assert n_g == n_o and np.array_equal(head_g, head_o)
    assert n_o > 0
    members = np.nonzero(head_o != _abi.NONE)[0].astype(np.uint32)
    cut = cfgm.wca_cutoff(P["params"]["sigma"] * 1.0) + P["params"]["wc"]
    nc_o, lab_o = ob.aggregates(_abi, st["positions"], members, cfg.box, cut)
    nc_g, lab_g = g.aggregate_labels(members, cut)
    assert nc_g == nc_o and np.array_equal(lab_g, lab_o)
    g.dispose()


def test_closure_in_a_parcel_matches_oracle():
    rng = np.random.default_rng(5)
    centre = np.array([25.0, 25.0, 25.0])
    members = _shell(rng, centre)
    d = rng.normal(size=(6000, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    e = rng.normal(size=(800, 3))
    inside = centre + e / np.linalg.norm(e, axis=1)[:, None] * (rng.uniform(0, 1, 800) ** (1 / 3) * 7.0)[:, None]
    water = np.concatenate([inside, centre + d * rng.uniform(13.0, 18.0, 6000)[:, None]])
    pos, mem, wat = _assemble(members, water)
    g = _system_for(pos, len(mem))
    c = ob.periodic_centre(_abi, pos, mem, SYN_BOX, P["circularAlpha"])
    args = (ST["closureCell"], ST["closureRadius"], ST["enclosedVolume"])
    ro = ob.closure_in_parcel(_abi, pos, mem, wat, SYN_BOX, c, *args, centre, 18.0)
    rg = g.closure(mem, wat, c, *args, parcel={"centre": list(centre), "radius": 18.0})
    assert rg["encapsulatedCount"] == ro.encapsulated_count > 0
    assert rg["bulkWaterDensity"] == pytest.approx(ro.bulk_water_density, rel=1e-12)
    assert rg["closed"] == bool(ro.closed) and rg["seedCell"] == ro.seed_cell
    g.dispose()

"""Device observables against the oracle on the same state: pairingStats counts and the z profile are
integers and must match exactly."""
import numpy as np
import pytest

import oracle_binding as ob
from helpers import water_opts
from protocell_genesis_b200 import _abi, config as cfgm, observables as obs
from protocell_genesis_b200.soup import SoupSystem

pytestmark = pytest.mark.gpu

P = cfgm.load_params()


def _system(ph):
    opts = water_opts(n_water=6000, box=24.0, start={"C": 1500, "O": 2500, "H": 0, "M": 60, "W": 6000},
                      electrostatics={"enabled": True, "pH": ph, "ionicStrengthMolar": 0.05})
    cfg = cfgm.resolve(opts, P)
    o = ob.OracleSystem(_abi, cfg)
    o.relax(30, 0.1)
    o.step(20)
    st = dict(positions=o.read(ob.F_POS), velocities=o.read(ob.F_VEL), bond_slots=o.read(ob.F_SLOTS),
              charges=o.read(ob.F_CHARGES))
    return cfg, SoupSystem(cfg, st)


@pytest.mark.parametrize("ph", [4.6, 7.0])
def test_pairing_stats_match_the_oracle(ph):
    cfg, g = _system(ph)
    g.step(15)                                             # a few device steps, sweeps included
    contact = cfgm.wca_cutoff(P["params"]["sigma"] * P["params"]["beadSizes"]["head_head"])
    d = g.pairing_stats(contact)
    w, unlike, like, paired, charged, heads = ob.pairing_stats(_abi, g.particles(), g.charges(), list(cfg.box),
                                                             cfg.charged_kind, contact)
    assert (d["withNeighbour"], d["unlikeContacts"], d["likeContacts"], d["paired"], d["heads"]) == \
        (w, unlike, like, paired, heads)
    assert d["alpha"] == pytest.approx(charged / heads)
    assert unlike + like > 100                             # the heads do touch
    assert obs.apparent_pka(d["alpha"], ph) == pytest.approx(ph - np.log10(d["alpha"] / (1 - d["alpha"])))
    g.dispose()


def test_density_profile_matches_the_oracle():
    cfg, g = _system(7.0)
    g.step(10)
    polar = [k for k, m in enumerate(P["monomers"]) if m["polar"]]
    mask = sum(1 << k for k in polar)
    for bins in (40, 97):
        d = g.density_profile_z(bins)
        head, tail, esc = ob.density_profile_z(_abi, g.particles(), cfg.box[2], bins, mask)
        assert esc == 0
        assert d["head"] == head.tolist() and d["tail"] == tail.tolist()
        assert sum(d["head"]) + sum(d["tail"]) == cfg.n
    d = g.density_profile_z(40, drop_escaped=True)
    assert d["escaped"] == 0
    g.dispose()


def test_aggregate_shapes_and_analysis_match_the_oracle():
    from helpers import boosted, plain_opts
    opts = plain_opts(box=[15, 15, 15], start={"C": 900, "O": 260, "H": 0, "M": 160, "W": 0})
    cfg = boosted(cfgm.resolve(opts, P), attempt=0.9, accept=1.0, brk=0.02)
    o = ob.OracleSystem(_abi, cfg)
    o.relax(30, 0.1)
    o.step(400)
    st = dict(positions=o.read(ob.F_POS), bond_slots=o.read(ob.F_SLOTS), center_link=o.read(ob.F_CENTER))
    g = SoupSystem(cfg, st)
    cut = cfgm.wca_cutoff(P["params"]["sigma"] * 1.0) + P["params"]["wc"]
    res = obs.analyze_aggregates(g, cut, detail_count=5)
    # the oracle's own labels, amphiphiles and shapes on the same positions
    polar = np.array([1 if m["polar"] else 0 for m in P["monomers"]] + [0] * (8 - len(P["monomers"])), np.uint32)
    n_o, head_o = ob.amphiphiles(_abi, st["positions"], st["bond_slots"], polar)
    members = np.nonzero(head_o != _abi.NONE)[0].astype(np.uint32)
    nc_o, lab_o = ob.aggregates(_abi, st["positions"], members, cfg.box, cut)
    assert res["aggregateCount"] == nc_o
    uniq, inv = np.unique(lab_o, return_inverse=True)
    size = np.bincount(inv)
    heads = np.bincount(inv, weights=(head_o[members] == members)).astype(int)
    order = sorted(range(len(uniq)), key=lambda c: (-int(size[c]), int(uniq[c])))
    assert res["sizeHistogram"] == [int(heads[c]) for c in order]
    assert len(res["aggregates"]) == min(5, nc_o)
    for k, shp in enumerate(res["aggregates"]):
        c = order[k]
        n, centre, gy = ob.aggregate_shape(_abi, st["positions"], members[inv == c], cfg.box)
        assert shp["size"] == n == size[c] and shp["label"] == uniq[c]
        assert np.allclose(shp["centre"], centre, rtol=1e-12, atol=1e-9)
        want = obs.shape_metrics({"size": n, "label": int(uniq[c]), "centre": centre, "gyration": list(gy)})
        assert np.allclose(shp["principalMoments"], want["principalMoments"], rtol=1e-9, atol=1e-9)
        assert shp["radiusOfGyration"] == pytest.approx(want["radiusOfGyration"], rel=1e-9)
    assert res["aggregates"][0]["size"] > 20
    g.dispose()

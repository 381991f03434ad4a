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

"""The guards' failure paths, made on the host or by a bounded wait that runs out (no device fault):

- SOUP_E_TIMEOUT: the constant-pH walk's handoffs between the CTAs of its cluster poll a flag a
  bounded number of times; with the limit set to one poll the walk gives up, the call returns
  SOUP_E_TIMEOUT with its message, and the handle then sweeps and steps normally at the default limit;
- SOUP_E_DRIFT: fixed-cadence rebuilds with a skin far below what ten steps move the beads, so the
  measured drift exceeds skin/2 (soup/src/soup-grid-verlet.ts:130-137, the reference's wording);
- SOUP_E_ES_OVERFLOW: a long-range list capacity of 4 (soup/src/soup-grid-verlet.ts:106-115).
"""
import numpy as np
import pytest

import oracle_binding as ob
from helpers import water_opts
from protocell_genesis_b200 import _abi, config as cfgm
from protocell_genesis_b200.soup import SoupSystem

pytestmark = pytest.mark.gpu

P = cfgm.load_params()


def _many_heads():
    opts = water_opts(n_water=6000, box=24.0, start={"C": 1500, "O": 2500, "H": 0, "M": 60, "W": 6000},
                      electrostatics={"enabled": True, "pH": 7.0, "ionicStrengthMolar": 0.01})
    cfg = cfgm.resolve(opts, P)
    cfg.protonation_rng = 4242
    o = ob.OracleSystem(_abi, cfg)
    o.relax(30, 0.1)
    o.step(10)
    st = dict(positions=o.read(ob.F_POS), velocities=o.read(ob.F_VEL), bond_slots=o.read(ob.F_SLOTS),
              charges=o.read(ob.F_CHARGES), bond_rng=o.read(ob.F_BOND_RNG), thermo_rng=o.read(ob.F_THERMO_RNG))
    return cfg, o, st


def test_a_handoff_that_runs_out_is_a_timeout_and_the_handle_recovers():
    cfg, o, st = _many_heads()
    g = SoupSystem(cfg, st)
    g.set_wait_limit(1)
    with pytest.raises(_abi.SoupError) as e:
        g.protonation_sweep()
    assert e.value.code == "SOUP_E_TIMEOUT"
    assert "did not arrive within its poll limit" in str(e.value)
    # the same handle at the default limit again: back at the oracle's state (the charges the failed
    # sweep left are not valid; the chain state it advanced is given to the oracle), a sweep gives the
    # oracle's decisions and the handle steps on
    g.set_wait_limit(0)
    g.write_state(st)
    o.write(ob.F_PROT_RNG, np.array([g.protonation_rng_state()], np.uint32))
    rg = g.protonation_sweep()
    ro = o.sweep()
    assert np.array_equal(g.charges(), o.read(ob.F_CHARGES))
    assert rg["accepted"] == ro.accepted and ro.accepted > 100
    g.step(20)
    assert g.nonfinite_count() == {"pos": 0, "vel": 0}
    g.dispose()


def test_drift_beyond_half_the_skin_is_refused_with_the_references_message():
    cfg = cfgm.resolve(water_opts(), P)
    skin = 0.05
    cfg.list_range += skin - cfg.skin
    cfg.es_list_range += skin - cfg.skin
    cfg.skin = skin
    cfg.rebuild_on_drift = 0
    cfg.rebuild_every = 10
    o = ob.OracleSystem(_abi, cfgm.resolve(water_opts(), P))
    o.relax(30, 0.1)
    g = SoupSystem(cfg, dict(positions=o.read(ob.F_POS), velocities=o.read(ob.F_VEL)))
    with pytest.raises(_abi.SoupError) as e:
        g.step(10)
    assert e.value.code == "SOUP_E_DRIFT"
    msg = str(e.value)
    assert "Verlet list: the measured drift" in msg and "exceeds skin/2=0.0250" in msg
    assert "the rebuild was not frequent enough" in msg
    g.dispose()


def test_a_long_range_list_overflow_is_refused_with_the_references_message():
    cfg = cfgm.resolve(water_opts(), P)
    cfg.es_list_capacity = 4
    o = ob.OracleSystem(_abi, cfgm.resolve(water_opts(), P))
    o.relax(30, 0.1)
    g = SoupSystem(cfg, dict(positions=o.read(ob.F_POS), velocities=o.read(ob.F_VEL)))
    with pytest.raises(_abi.SoupError) as e:
        g.step(1)
    assert e.value.code == "SOUP_E_ES_OVERFLOW"
    msg = str(e.value)
    heads = g.info()["heads"]
    assert msg.startswith("SOUP_E_ES_OVERFLOW: long-range electrostatics list: longRangeListCapacity=4 or the headIdx size "
                          f"({heads}) was insufficient at rc_es=")
    assert "-- data may have been silently dropped" in msg
    g.dispose()

"""The autotuner (soup_autotune): its choices come from the candidate sets, stay in effect, and leave
the state as it was; a tuned system keeps stepping finitely, and a tuned batch still equals its
single systems' trajectories to FP32 rounding."""
import numpy as np
import pytest

import oracle_binding as ob
from helpers import water_opts
from protocell_genesis_b200 import _abi, config as cfgm
from protocell_genesis_b200.soup import SoupBatch, SoupSystem

pytestmark = pytest.mark.gpu

P = cfgm.load_params()


def _state(g):
    return dict(positions=g.particles(), velocities=g.velocities(), charges=g.charges(), bond_slots=g.bond_slots(),
                center_link=g.center_links(), thermo=g.rng_state()["thermo"], bond=g.rng_state()["bond"],
                step=g.steps, events=g.events_raw())


def _system(seed=3):
    cfg = cfgm.resolve(water_opts(n_water=3000, seed=seed, electrostatics={"enabled": True, "pH": 7.0},
                                  sweep_every=10, chunk_steps=10, rebuild_on_drift=True, skin=1.0), P)
    o = ob.OracleSystem(_abi, cfg)
    o.relax(20, 0.1)
    st = dict(positions=o.read(ob.F_POS), velocities=o.read(ob.F_VEL), bond_slots=o.read(ob.F_SLOTS),
              thermo_rng=o.read(ob.F_THERMO_RNG), bond_rng=o.read(ob.F_BOND_RNG), charges=o.read(ob.F_CHARGES))
    return cfg, st


def test_choices_stay_and_the_state_is_restored():
    cfg, st = _system()
    g = SoupSystem(cfg, st)
    g.step(20)
    before = _state(g)
    r = g.autotune(steps=10)
    after = _state(g)
    assert r["tpp"] in (1, 2, 4, 8) and r["walk"] in (2, 3) and r["skin_scale"] in (0.6, 0.8, 1.0)
    assert r["ms_per_step_before"] > 0 and r["ms_per_step_after"] > 0
    for k in before:
        assert np.array_equal(np.asarray(before[k]), np.asarray(after[k])), k
    g.step(40)
    assert np.all(np.isfinite(g.particles()))
    g.dispose()


def test_tuned_trajectory_agrees_with_an_untuned_one():
    cfg, st = _system(seed=4)
    a = SoupSystem(cfg, st)
    b = SoupSystem(cfg, st)
    a.autotune(steps=10)
    a.step(20)
    b.step(20)
    pa, pb = a.particles().reshape(-1, 4), b.particles().reshape(-1, 4)
    d = pa[:, :3] - pb[:, :3]
    d -= np.rint(d / cfg.box[0]) * cfg.box[0]
    assert np.abs(d).max() < 1e-3
    assert np.array_equal(pa[:, 3], pb[:, 3])
    a.dispose()
    b.dispose()


def test_tuned_batch_steps_like_its_replicas():
    cfgs, states = [], []
    for k, (ph, ion, seed) in enumerate([(6.5, 0.05, 5), (8.0, 0.01, 6)]):
        c = cfgm.resolve(water_opts(n_water=1500 + 500 * k, electrostatics={"enabled": True, "pH": ph,
                                                                           "ionicStrengthMolar": ion},
                                    seed=seed, sweep_every=10, chunk_steps=10, rebuild_on_drift=True, skin=1.0), P)
        o = ob.OracleSystem(_abi, c)
        o.relax(20, 0.1)
        cfgs.append(c)
        states.append(dict(positions=o.read(ob.F_POS), velocities=o.read(ob.F_VEL), bond_slots=o.read(ob.F_SLOTS),
                           thermo_rng=o.read(ob.F_THERMO_RNG), bond_rng=o.read(ob.F_BOND_RNG),
                           charges=o.read(ob.F_CHARGES)))
    batch = SoupBatch(cfgs, states)
    r = batch.autotune(steps=10)
    assert r["tpp"] in (1, 2, 4, 8)
    batch.step(30)
    for c, st, rep in zip(cfgs, states, batch.replicas):
        single = SoupSystem(c, st)
        single.step(30)
        d = rep.particles().reshape(-1, 4)[:, :3] - single.particles().reshape(-1, 4)[:, :3]
        d -= np.rint(d / c.box[0]) * c.box[0]
        assert np.abs(d).max() < 1e-2
        single.dispose()
    batch.dispose()


def test_apply_tuning_reproduces_the_tuned_shape():
    """soup_apply_tuning puts a fresh system in the shape a tuning found: from the tuned system's
    state it then follows the tuned system's trajectory bit for bit."""
    from helpers import charged_opts
    opts = charged_opts(rebuild_on_drift=True)
    a = SoupSystem(cfgm.resolve(opts, P))
    a.relax_cold_start()
    tune = a.autotune(steps=10)
    arrays, sc = a.checkpoint_payload()
    cfg_b = cfgm.resolve(opts, P)
    cfg_b.protonation_rng = sc["protonationRng"]
    b = SoupSystem(cfg_b, {k: v.copy() for k, v in arrays.items()})
    b.apply_tuning(tune)
    a.step(40)
    b.step(40)
    assert np.array_equal(a.particles().view(np.uint32), b.particles().view(np.uint32))
    with pytest.raises(_abi.SoupError):
        b.apply_tuning(dict(tune, tpp=3))
    a.dispose()
    b.dispose()


@pytest.mark.parametrize("tpp", [1, 2, 4])
def test_queued_force_is_bit_identical_to_the_plain_one(tpp):
    """The list force with the in-range pairs queued per lane (k_force_q) accumulates every lane's
    terms in k_force's order: the forces are the same bits, for all particles and for the heads-only
    recompute after a sweep, on compositions with charges, catalysts and a confining wall."""
    from helpers import charged_opts, confined_opts
    for opts in (charged_opts(rebuild_on_drift=True, sweep_every=10, chunk_steps=10),
                 confined_opts(rebuild_on_drift=True, sweep_every=10, chunk_steps=10)):
        cfg = cfgm.resolve(opts, P)
        o = ob.OracleSystem(_abi, cfg)
        o.relax(20, 0.1)
        o.step(20)
        st = dict(positions=o.read(ob.F_POS), velocities=o.read(ob.F_VEL), bond_slots=o.read(ob.F_SLOTS),
                  center_link=o.read(ob.F_CENTER), charges=o.read(ob.F_CHARGES))
        out = []
        for q in (0, 1):
            g = SoupSystem(cfg, st)
            g.apply_tuning(dict(tpp=tpp, walk=2, skin_scale=1.0, queued=q))
            f = g.forces_no_rebuild()
            g.step(30)                          # sweeps every 10 steps recompute the heads' forces only
            out.append((f, g.forces_no_rebuild(), g.charges()))
            g.dispose()
        assert np.array_equal(out[0][0].view(np.uint32), out[1][0].view(np.uint32))
        assert np.array_equal(out[0][2], out[1][2])
        assert np.array_equal(out[0][1].view(np.uint32), out[1][1].view(np.uint32))

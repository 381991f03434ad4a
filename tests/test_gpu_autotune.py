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


def test_compacted_force_is_bit_identical_to_the_plain_one():
    """The list force with each warp's in-range pairs compacted and evaluated by every lane (k_force_w)
    accumulates every particle's terms in k_force<1>'s order with k_force<1>'s arithmetic: the forces
    are the same bits, for all particles and for the heads-only recompute after a sweep, on compositions
    with charges, catalysts and a confining wall (whose warps take both the minimum-image path and the
    direct one of warps inside the box).  In a batch, the warp that spans two replicas evaluates each
    owner's pairs on the owner's lane: the batch's forces are its replicas' own."""
    from helpers import charged_opts, confined_opts
    from protocell_genesis_b200.soup import SoupBatch
    states = []
    for opts in (charged_opts(rebuild_on_drift=True, sweep_every=10, chunk_steps=10),
                 confined_opts(rebuild_on_drift=True, sweep_every=10, chunk_steps=10)):
        cfg = cfgm.resolve(opts, P)
        o = ob.OracleSystem(_abi, cfg)
        o.relax(20, 0.1)
        o.step(20)
        st = dict(positions=o.read(ob.F_POS), velocities=o.read(ob.F_VEL), bond_slots=o.read(ob.F_SLOTS),
                  center_link=o.read(ob.F_CENTER), charges=o.read(ob.F_CHARGES))
        states.append((cfg, st))
        out = []
        for q in (0, 1):
            g = SoupSystem(cfg, st)
            g.apply_tuning(dict(tpp=1, walk=2, skin_scale=1.0, queued=q))
            f = g.forces_no_rebuild()
            g.step(30)                          # sweeps every 10 steps recompute the heads' forces only
            out.append((f, g.forces_no_rebuild(), g.charges()))
            g.dispose()
        assert np.array_equal(out[0][0].view(np.uint32), out[1][0].view(np.uint32))
        assert np.array_equal(out[0][2], out[1][2])
        assert np.array_equal(out[0][1].view(np.uint32), out[1][1].view(np.uint32))
    # two replicas of the charged composition (different seeds' states are not needed: the second
    # replica's slots start mid-warp unless its first replica's count is a multiple of 32)
    cfg, st = states[0]
    assert cfg.n % 32 != 0
    b = SoupBatch([cfg, cfg], [st, st])
    b.apply_tuning(dict(tpp=1, walk=2, skin_scale=1.0, queued=1))
    g = SoupSystem(cfg, st)
    g.apply_tuning(dict(tpp=1, walk=2, skin_scale=1.0, queued=1))
    fg = g.forces_no_rebuild().view(np.uint32)
    for r in b.replicas:
        assert np.array_equal(r.forces_no_rebuild().view(np.uint32), fg)
    g.dispose()
    b.dispose()


def test_pruned_rows_change_no_bit(monkeypatch):
    """Force passes read a list row only up to the build-distance shells that the largest displacement
    since the build can have brought within the force's reach; the entries skipped are beyond it, so
    a trajectory with the pruning equals one that reads every row whole (SOUP_FULL_ROWS=1), bit for
    bit, across drift-triggered rebuilds, charge sweeps and bond passes."""
    from helpers import confined_opts
    opts = confined_opts(rebuild_on_drift=True, sweep_every=10, chunk_steps=10)
    cfg = cfgm.resolve(opts, P)
    o = ob.OracleSystem(_abi, cfg)
    o.relax(20, 0.1)
    st = dict(positions=o.read(ob.F_POS), velocities=o.read(ob.F_VEL), bond_slots=o.read(ob.F_SLOTS),
              center_link=o.read(ob.F_CENTER), charges=o.read(ob.F_CHARGES))
    out = []
    for full in ("0", "1"):
        monkeypatch.setenv("SOUP_FULL_ROWS", full)
        g = SoupSystem(cfg, st)
        g.step(60)
        out.append((g.particles(), g.velocities(), g.forces_no_rebuild(), g.charges(), g.info()["rebuilds"]))
        g.dispose()
    assert out[0][4] == out[1][4] and out[0][4] >= 3
    for a, b in zip(out[0][:4], out[1][:4]):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("maker", ["charged_opts", "confined_opts"])
def test_cell_group_list_build_gives_the_oracle_sets(maker, monkeypatch):
    """The list build with a group of lanes per cell and the neighbour rows staged in shared memory
    (SOUP_LIST_BY_CELL=1, an autotuner choice) gives the oracle's Verlet sets, as the build with a
    thread per particle does."""
    import helpers
    monkeypatch.setenv("SOUP_LIST_BY_CELL", "1")
    cfg = cfgm.resolve(getattr(helpers, maker)(), P)
    o = ob.OracleSystem(_abi, cfg)
    o.relax(20, 0.1)
    o.step(20)
    st = dict(positions=o.read(ob.F_POS), velocities=o.read(ob.F_VEL), bond_slots=o.read(ob.F_SLOTS),
              center_link=o.read(ob.F_CENTER), charges=o.read(ob.F_CHARGES))
    g = SoupSystem(cfg, st)
    o2 = ob.OracleSystem(_abi, cfg, st)
    gc, gl = g.verlet_lists()
    oc, ol = o2.verlet()
    assert np.array_equal(gc, oc) and np.array_equal(gl, ol)
    g.dispose()
    o2.close()

"""Parity of the CUDA path (through the C ABI) with the CPU oracle, on identical inputs.

Bars: Verlet/head lists, positions after the kick+drift, RNG streams, bond slots / centre links /
event counters after a bond pass, and constant-pH accept decisions are bit-exact; forces are within
1e-5 relative RMS of the FP64 oracle; the thermostat velocities (logf/cosf differ between libraries)
within 2e-6 relative.
"""
import numpy as np
import pytest

import oracle_binding as ob
from helpers import boosted, charged_opts, confined_opts, csr_rows, long_range_opts, plain_opts, rel_rms, water_opts
from protocell_genesis_b200 import _abi, config as cfgm
from protocell_genesis_b200.soup import SoupBatch, SoupSystem

pytestmark = pytest.mark.gpu

P = cfgm.load_params()
FORCE_TOL = 1e-5       # relative RMS against FP64 (the target's force bar)
THERMO_TOL = 2e-6      # velocities after the Langevin kick (library logf/cosf differ in the last ulps)


def oracle_state(o, with_force=False):
    st = dict(positions=o.read(ob.F_POS), velocities=o.read(ob.F_VEL), bond_slots=o.read(ob.F_SLOTS),
              center_link=o.read(ob.F_CENTER), center_held=o.read(ob.F_HELD), bond_rng=o.read(ob.F_BOND_RNG),
              thermo_rng=o.read(ob.F_THERMO_RNG), charges=o.read(ob.F_CHARGES), frozen=o.read(ob.F_FROZEN),
              events=o.read(ob.F_EVENTS), desorb_events=o.read(ob.F_DESORB))
    return st


def make_pair(opts, relax=30, steps=0, tweak=None):
    cfg = cfgm.resolve(opts, P)
    if tweak:
        tweak(cfg)
    o = ob.OracleSystem(_abi, cfg)
    if relax:
        o.relax(relax, 0.1)
    if steps:
        o.step(steps)
    g = SoupSystem(cfg, oracle_state(o))
    return cfg, o, g


@pytest.mark.parametrize("maker", [plain_opts, charged_opts, long_range_opts, confined_opts])
def test_lists_are_the_oracle_sets(maker):
    cfg, o, g = make_pair(maker(), relax=10)
    gc, gl = g.verlet_lists()
    oc, ol = o.verlet()
    assert np.array_equal(gc, oc)
    assert np.array_equal(gl, ol)


@pytest.mark.parametrize("maker", [plain_opts, charged_opts, long_range_opts, confined_opts])
def test_force_within_fp64_tolerance(maker):
    cfg, o, g = make_pair(maker(), relax=20, steps=20)
    f64 = o.forces64()
    fg = g.forces_no_rebuild()
    assert rel_rms(fg, f64) < FORCE_TOL
    fb = g.forces_brute_force()
    assert rel_rms(fb, f64) < FORCE_TOL


def test_kick_drift_bit_exact_and_thermostat():
    cfg, o, g = make_pair(charged_opts(), relax=20, steps=10)
    o.write(ob.F_FORCE, g.forces_no_rebuild())          # both integrate the same force array
    g.debug_phase(_abi.PHASE_KICK_DRIFT)
    o.phase(_abi.PHASE_KICK_DRIFT)
    assert np.array_equal(g.particles(), o.read(ob.F_POS))
    assert np.array_equal(g.velocities(), o.read(ob.F_VEL))
    g.debug_phase(_abi.PHASE_KICK_THERMO)
    o.phase(_abi.PHASE_KICK_THERMO)
    assert np.array_equal(g.rng_state()["thermo"], o.read(ob.F_THERMO_RNG))
    vg = g.velocities().reshape(-1, 4)[:, :3].astype(np.float64)
    vo = o.read(ob.F_VEL).reshape(-1, 4)[:, :3].astype(np.float64)
    assert np.abs(vg - vo).max() <= THERMO_TOL * max(1.0, np.abs(vo).max())


def test_bond_passes_bit_exact():
    def tw(c):
        boosted(c, attempt=0.9, accept=1.0, brk=0.15)
        c.max_hold_steps = 60          # the hold-time valve fires too
    opts = plain_opts(box=[15, 15, 15], start={"C": 900, "O": 260, "H": 0, "M": 160, "W": 0})
    cfg, o, g = make_pair(opts, relax=30, tweak=tw)
    total = 0
    for rnd in range(10):
        o.step(13)
        g.write_state(oracle_state(o))
        o.phase(_abi.PHASE_REBUILD)
        o.phase(_abi.PHASE_BONDS)
        g.debug_phase(_abi.PHASE_BONDS)
        assert np.array_equal(g.bond_slots(), o.read(ob.F_SLOTS)), rnd
        assert np.array_equal(g.center_links(), o.read(ob.F_CENTER)), rnd
        assert np.array_equal(g.center_held_steps(), o.read(ob.F_HELD)), rnd
        assert np.array_equal(g.rng_state()["bond"], o.read(ob.F_BOND_RNG)), rnd
        assert np.array_equal(g.events_raw(), o.read(ob.F_EVENTS)), rnd
        d = g.desorb_events()
        assert [d["stretch"], d["timeout"]] == list(o.read(ob.F_DESORB)), rnd
        total = int(o.read(ob.F_EVENTS).sum())
    assert total > 150   # the passes really formed and broke bonds
    assert sum(o.read(ob.F_DESORB)) > 0


def test_protonation_sweep_decisions_match():
    def tw(c):
        c.protonation_rng = 12345
    cfg, o, g = make_pair(water_opts(), relax=30, steps=30, tweak=tw)
    g.write_state(oracle_state(o))
    rg = g.protonation_sweep()
    ro = o.sweep()
    assert np.array_equal(g.charges(), o.read(ob.F_CHARGES))
    assert g.protonation_rng_state() == int(o.read(ob.F_PROT_RNG)[0])
    assert rg["accepted"] == ro.accepted and rg["deprotonated"] == ro.deprotonated
    assert rg["dEsMeanKT"] == pytest.approx(ro.d_es_mean_kt, rel=1e-9, abs=1e-12)
    # the sweep recomputed the force with the new charges
    assert rel_rms(g.forces_no_rebuild(), o.forces64()) < FORCE_TOL


@pytest.mark.parametrize("ph,ionic", [(7.0, 0.01), (4.6, 0.1)])
def test_consecutive_sweeps_on_many_heads(ph, ionic):
    """Thousands of heads with many accepted flips per sweep, three sweeps in a row."""
    def tw(c):
        c.protonation_rng = 987654321
    opts = water_opts(n_water=6000, box=24.0, start={"C": 1500, "O": 2500, "H": 0, "M": 60, "W": 6000},
                      electrostatics={"enabled": True, "pH": ph, "ionicStrengthMolar": ionic})
    cfg, o, g = make_pair(opts, relax=30, steps=10, tweak=tw)
    g.write_state(oracle_state(o))
    for k in range(3):
        rg = g.protonation_sweep()
        ro = o.sweep()
        assert np.array_equal(g.charges(), o.read(ob.F_CHARGES)), k
        assert g.protonation_rng_state() == int(o.read(ob.F_PROT_RNG)[0]), k
        assert rg["accepted"] == ro.accepted and rg["deprotonated"] == ro.deprotonated, k
        assert rg["dEsMeanKT"] == pytest.approx(ro.d_es_mean_kt, rel=1e-9, abs=1e-12), k
        assert ro.accepted > 300, k


def test_short_trajectory_tracks_the_oracle():
    cfg, o, g = make_pair(charged_opts(), relax=30)
    g.step(40)
    o.step(40)
    assert np.array_equal(g.rng_state()["thermo"], o.read(ob.F_THERMO_RNG))
    pg_ = g.particles().reshape(-1, 4)
    po = o.read(ob.F_POS).reshape(-1, 4)
    d = pg_[:, :3] - po[:, :3]
    d -= np.rint(d / cfg.box[0]) * cfg.box[0]
    assert np.abs(d).max() < 1e-3
    assert np.array_equal(pg_[:, 3], po[:, 3])


def test_batch_replicas_equal_single_systems():
    cfgs = []
    for k, (ph, ion, seed) in enumerate([(6.0, 0.05, 3), (7.5, 0.01, 4), (8.5, 0.1, 5)]):
        c = cfgm.resolve(water_opts(n_water=1500 + 400 * k, electrostatics={"enabled": True, "pH": ph,
                                                                           "ionicStrengthMolar": ion},
                                    seed=seed, sweep_every=20, chunk_steps=20), P)
        cfgs.append(c)
    states = []
    for c in cfgs:
        o = ob.OracleSystem(_abi, c)
        o.relax(20, 0.1)
        states.append(oracle_state(o))
    batch = SoupBatch(cfgs, states)
    batch.step(60)
    for c, st, rep in zip(cfgs, states, batch.replicas):
        single = SoupSystem(c, st)
        single.step(60)
        assert np.array_equal(rep.particles(), single.particles())
        assert np.array_equal(rep.charges(), single.charges())
        assert np.array_equal(rep.bond_slots(), single.bond_slots())
        single.dispose()
    batch.dispose()


def test_guards_are_loud():
    cfg, o, g = make_pair(plain_opts(), relax=10)
    st = oracle_state(o)
    st["positions"] = st["positions"].copy()
    st["positions"][4 * 5] = np.nan
    g.write_state(st)
    with pytest.raises(_abi.SoupError) as e:
        g.step(1)
    assert e.value.code == "SOUP_E_NONFINITE"
    cfg2 = cfgm.resolve(plain_opts(), P)
    cfg2.list_capacity = 8
    g2 = SoupSystem(cfg2, oracle_state(o))
    with pytest.raises(_abi.SoupError) as e:
        g2.step(1)
    assert e.value.code == "SOUP_E_LIST_OVERFLOW"


def test_sweep_head_force_recompute_is_exact(monkeypatch):
    """After a charge sweep only the heads' forces are recomputed (only heads carry charge and the
    polar class is the heads' kind): the trajectory equals the one with the full force recomputed,
    bit for bit, across several sweeps with drift-triggered rebuilds."""
    opts = water_opts(n_water=4000, box=20.0, start={"C": 1200, "O": 800, "H": 0, "M": 40, "W": 4000},
                      electrostatics={"enabled": True, "pH": 7.0, "ionicStrengthMolar": 0.05},
                      sweep_every=10, chunk_steps=10, rebuild_on_drift=True, skin=1.0)
    cfg, o, _ = make_pair(opts, relax=30)
    st = oracle_state(o)
    out = {}
    for full in ("0", "1"):
        if full == "1":
            monkeypatch.setenv("SOUP_SWEEP_FORCE_ALL", "1")
        g = SoupSystem(cfg, st)
        g.step(40)
        out[full] = (g.particles(), g.charges(), g.forces_no_rebuild())
        g.dispose()
    assert np.array_equal(out["0"][0], out["1"][0])
    assert np.array_equal(out["0"][1], out["1"][1])
    assert np.array_equal(out["0"][2], out["1"][2])
    assert not np.array_equal(st["charges"], out["0"][1])   # the sweeps flipped charges


def test_plain_small_case_lists_forces_and_trajectory():
    """The plain small case (3,277 beads, 200 charged amphiphiles, no sweep): lists equal the oracle's
    sets, forces within 1e-5 relative RMS of FP64 on the thermalised state, and 100 steps follow the
    oracle's trajectory.  (Right after the relax the forces nearly cancel: there the oracle's own FP32
    restatement of the reference's arithmetic is 1.1e-5 from FP64; after 100 steps 1.6e-6.)"""
    from helpers import config1_start
    opts, st = config1_start()
    cfg = cfgm.resolve(opts, P)
    o = ob.OracleSystem(_abi, cfg, st)
    o.relax(100, 0.1)
    g = SoupSystem(cfg, oracle_state(o))     # both lists built from the relaxed positions
    gc, gl = g.verlet_lists()
    oc, ol = o.verlet()
    assert np.array_equal(gc, oc) and np.array_equal(gl, ol)
    o.step(100)                              # the oracle runs on from the relaxed state
    t = SoupSystem(cfg, oracle_state(o))
    assert rel_rms(t.forces(), o.forces64()) < 1e-5
    t.dispose()
    g.step(100)                              # the device from the same relaxed state
    assert np.array_equal(g.rng_state()["thermo"], o.read(ob.F_THERMO_RNG))
    pg_, po = g.particles().reshape(-1, 4), o.read(ob.F_POS).reshape(-1, 4)
    d = pg_[:, :3] - po[:, :3]
    d -= np.rint(d / cfg.box[0]) * cfg.box[0]
    assert np.abs(d).max() < 1e-2
    assert np.array_equal(g.charges(), o.read(ob.F_CHARGES))
    g.dispose()


@pytest.mark.parametrize("maker", [plain_opts, charged_opts])
def test_cold_start_relax_tracks_the_oracle(maker):
    """relaxColdStart (soup/src/soup-relax.ts:87-185, relax.wgsl:50-72) on the device against the
    oracle's relax from the same fresh lattice.  Every bead steps d along its own force direction
    f/|f|, whatever |f| is, so a bead whose force is near zero turns with the last bits of its force:
    two correct relaxes part after a few tens of iterations, and the map itself is what is compared.
    - one iteration from the same positions, at four points along the oracle's 60-iteration path
      (d = d0 (1 - k/60)): the device moves the beads where the oracle moves them, to the rounding of
      the force direction (99% of the beads within 1e-4 d0; fewer than 0.2% turned by more than 1e-2 d);
    - the whole 60 iterations: the two relaxes move the beads as far (RMS displacement within 5%) and
      leave forces of the same size (largest force within a factor of 2, both below the start's)."""
    cfg = cfgm.resolve(maker(), P)
    o = ob.OracleSystem(_abi, cfg)
    start = oracle_state(o)
    its, d0 = 60, 0.1
    checked = 0
    for k in range(its):
        d = d0 * (1.0 - k / its)
        if k in (0, 15, 40, 59):
            before = o.read(ob.F_POS).reshape(-1, 4).copy()
            g = SoupSystem(cfg, dict(oracle_state(o), positions=before.ravel()))
            g.relax_cold_start(1, d / cfg.sigma)
            o.relax(1, d)
            pg_, po = g.particles().reshape(-1, 4), o.read(ob.F_POS).reshape(-1, 4)
            e = pg_[:, :3].astype(np.float64) - po[:, :3]
            e -= np.rint(e / cfg.box[0]) * cfg.box[0]
            err = np.sqrt((e ** 2).sum(axis=1)) / d0
            print(f"relax iteration {k} (d = {d / d0:.3f} d0): RMS {np.sqrt((err ** 2).mean()):.2e} d0, max "
                  f"{err.max():.2e} d0, {(err > 1e-2 * d / d0).sum()} of {err.size} beads beyond 1e-2 d")
            assert np.quantile(err, 0.99) < 1e-4
            assert (err > 1e-2 * d / d0).mean() < 2e-3
            assert np.array_equal(pg_[:, 3], po[:, 3])
            g.dispose()
            checked += 1
        else:
            o.relax(1, d)
    assert checked == 4
    o_end = o.read(ob.F_POS).reshape(-1, 4)
    fo = np.abs(o.read(ob.F_FORCE).reshape(-1, 4)[:, :3]).max()
    g = SoupSystem(cfg, start)
    r = g.relax_cold_start(its, d0)
    s0 = start["positions"].reshape(-1, 4)[:, :3].astype(np.float64)

    def rms_moved(p):
        m = p[:, :3].astype(np.float64) - s0
        m -= np.rint(m / cfg.box[0]) * cfg.box[0]
        return float(np.sqrt((m ** 2).sum(axis=1).mean()))
    mg, mo = rms_moved(g.particles().reshape(-1, 4)), rms_moved(o_end)
    print(f"relax {its} iterations: RMS displacement {mg:.4f} vs oracle {mo:.4f}; largest force "
          f"{r['maxForceAfter']:.3e} vs {fo:.3e} (start {r['maxForceBefore']:.3e})")
    assert mo > 0.05 and abs(mg / mo - 1) < 0.05
    assert 0.5 < r["maxForceAfter"] / fo < 2.0
    assert r["maxForceAfter"] < r["maxForceBefore"] and fo < r["maxForceBefore"]
    g.dispose()

"""Parity at the benchmarked campaign shape, and the benchmark's own step schedule against the oracle.

The campaign shape is the one bench.py times: 483,268 beads in a 76 sigma box (the reference's B76
census), pH 7 constant-pH Monte Carlo, I = 0.01 M long-range Debye-Hueckel (rc_es 15.2 sigma), a
Verlet skin of 1.0 sigma rebuilt on half-skin drift, bonds every 20 steps (soup/src/soup-integrate.ts
:83-175).  Its start is the bench's: the seeded fresh lattice, relaxed on the device, stepped 20 steps.

- the list force plus the far half is within 1e-5 relative RMS of the oracle's FP64 force;
- the Verlet lists and the long-range head lists equal the oracle's sets (soup/wgsl/verlet.wgsl:53-92,
  soup/wgsl/electrostatics-long.wgsl:31-56);
- one full sweep over the 18,659 heads gives the oracle's charges, chain state and counts, and over
  a run of sweeps the number of decisions that differ from the oracle's FP64 sweep is counted (the
  device sums site energies in fixed point, the reference in FP64: soup/src/electrostatics.ts:435-496).

The schedule test runs the bench's schedule (rebuild on half-skin drift at the bench's skin, the sweep every
10 steps, bonds every 20) on a tenth of the campaign shape, chunk by chunk from the device's state.
"""
import numpy as np
import pytest

import bench
import oracle_binding as ob
from helpers import rel_rms
from protocell_genesis_b200 import _abi, config as cfgm
from protocell_genesis_b200.soup import SoupSystem

pytestmark = pytest.mark.gpu

P = cfgm.load_params()
SKIN = bench.SKIN     # the skin the benchmark runs at
FORCE_TOL = 1e-5
SWEEPS = 30           # sweeps whose decisions are compared with the oracle's at the full shape


def device_state(g):
    rng = g.rng_state()
    d = g.desorb_events()
    return dict(positions=g.particles(), velocities=g.velocities(), bond_slots=g.bond_slots(),
                center_link=g.center_links(), center_held=g.center_held_steps(), bond_rng=rng["bond"],
                thermo_rng=rng["thermo"], charges=g.charges(), frozen=g.frozen(), events=g.events_raw(),
                desorb_events=np.array([d["stretch"], d["timeout"]], np.uint32))


def campaign(scale=1.0, steps=20, skin=SKIN):
    cfg = cfgm.resolve(bench.workload_opts(cfgm, skin=skin, scale=scale), P)
    g = SoupSystem(cfg)
    g.relax_cold_start(bench.RELAX_ITERATIONS, 0.1)
    if steps:
        g.step(steps)
    return cfg, g


@pytest.fixture(scope="module")
def full():
    cfg, g = campaign()
    assert cfg.n == 483268
    o = ob.OracleSystem(_abi, cfg, device_state(g))
    yield cfg, g, o
    o.close()
    g.dispose()


def test_campaign_force_within_fp64_tolerance(full):
    cfg, g, o = full
    err = rel_rms(g.forces_no_rebuild(), o.forces64())
    print(f"campaign force relRMS vs FP64: {err:.3e}")
    assert err < FORCE_TOL


def test_campaign_lists_are_the_oracle_sets(full):
    cfg, g, o = full
    g.debug_phase(_abi.PHASE_REBUILD)          # lists from the same positions as the oracle's
    gc, gl = g.verlet_lists()
    oc, ol = o.verlet()
    assert np.array_equal(gc, oc)
    assert np.array_equal(gl, ol)
    hc, hl = g.es_lists()
    ohc, ohl = o.es_lists()
    assert hc.size == 18659
    assert np.array_equal(hc, ohc)
    assert np.array_equal(hl, ohl)


def test_campaign_sweeps_match_the_oracle(full):
    """The first sweep is compared whole; then SWEEPS sweeps in a row at these positions, each from
    the device's charges and chain state, counting the decisions that differ from the oracle's."""
    cfg, g, o = full
    # the device's 20 steps ran two sweeps: the oracle takes its chain state from there
    o.write(ob.F_PROT_RNG, np.array([g.protonation_rng_state()], np.uint32))
    rg = g.protonation_sweep()
    ro = o.sweep()
    assert np.array_equal(g.charges(), o.read(ob.F_CHARGES))
    assert g.protonation_rng_state() == int(o.read(ob.F_PROT_RNG)[0])
    assert rg["heads"] == 18659 and rg["accepted"] == ro.accepted and rg["deprotonated"] == ro.deprotonated
    assert rg["dEsMeanKT"] == pytest.approx(ro.d_es_mean_kt, rel=1e-9, abs=1e-12)
    mismatched_sweeps, mismatched_heads, accepted = 0, 0, 0
    for _ in range(SWEEPS):
        o.write(ob.F_CHARGES, g.charges())
        o.write(ob.F_PROT_RNG, np.array([g.protonation_rng_state()], np.uint32))
        rg = g.protonation_sweep()
        ro = o.sweep()
        accepted += ro.accepted
        d = int((g.charges() != o.read(ob.F_CHARGES)).sum())
        if d or g.protonation_rng_state() != int(o.read(ob.F_PROT_RNG)[0]) or rg["accepted"] != ro.accepted:
            mismatched_sweeps += 1
            mismatched_heads += d
    print(f"{SWEEPS} campaign sweeps: {accepted} accepted flips, {mismatched_sweeps} sweeps and "
          f"{mismatched_heads} head charges differing from the FP64 oracle")
    assert accepted > 1000 * SWEEPS
    assert mismatched_sweeps == 0


@pytest.mark.parametrize("skin", [SKIN, 0.6])
def test_bench_schedule_tracks_the_oracle(skin):
    """A tenth of the campaign shape (48,327 beads) on the bench's schedule.  Each chunk of 10 steps
    starts with a rebuild on the device and the oracle created from the device's whole state (which
    rebuilds too), its force array included: both drift references are the chunk's start, the first
    kick and drift are bit-identical, and a bond pass on the chunk's first step sees the same
    positions.  Then:
    the thermostat and bond RNG streams, bond slots, centre links and event counters are exact; the
    positions agree to 1e-3 sigma after the chunk; the drift-triggered rebuilds are as many (the oracle
    also rebuilds after each sweep, as the reference does, where the device recomputes the force only); and the
    device's end-of-chunk sweep equals the oracle's sweep on the device's own pre-sweep state (its
    positions at the chunk's end, the charges and chain state at its start)."""
    cfg, g = campaign(scale=0.1, steps=0, skin=skin)
    assert cfg.rebuild_on_drift and cfg.sweep_every == 10 and cfg.bond_interval == 20
    bond_chunks = rebuilds = 0
    for chunk in range(12):
        g.debug_phase(_abi.PHASE_REBUILD)
        st = device_state(g)
        force = g.forces_no_rebuild()
        prot = g.protonation_rng_state()
        step0 = g.steps
        c = cfgm.resolve(bench.workload_opts(cfgm, skin=skin, scale=0.1), P)
        c.global_step = step0
        c.protonation_rng = prot
        o = ob.OracleSystem(_abi, c, st)
        o.write(ob.F_FORCE, force)
        r0 = g.info()["rebuilds"]
        oi0 = o.info()
        g.step(10)
        o.step(10)
        oi1 = o.info()
        assert g.steps == step0 + 10 and o.info()["step"] == step0 + 10
        assert np.array_equal(g.rng_state()["thermo"], o.read(ob.F_THERMO_RNG)), chunk
        assert np.array_equal(g.rng_state()["bond"], o.read(ob.F_BOND_RNG)), chunk
        assert np.array_equal(g.bond_slots(), o.read(ob.F_SLOTS)), chunk
        assert np.array_equal(g.center_links(), o.read(ob.F_CENTER)), chunk
        assert np.array_equal(g.events_raw(), o.read(ob.F_EVENTS)), chunk
        # the oracle, as the reference, rebuilds the lists after a sweep (soup-protonation.ts:62-73);
        # in drift-triggered mode the device recomputes only the force there, so the drift-triggered
        # rebuilds inside the chunk are compared
        o_drift = (oi1["rebuilds"] - oi0["rebuilds"]) - (oi1["sweeps"] - oi0["sweeps"])
        assert g.info()["rebuilds"] - r0 == o_drift, chunk
        rebuilds += g.info()["rebuilds"] - r0
        bond_chunks += step0 % 20 == 0
        pg_, po = g.particles().reshape(-1, 4), o.read(ob.F_POS).reshape(-1, 4)
        d = pg_[:, :3] - po[:, :3]
        d -= np.rint(d / cfg.box[0]) * cfg.box[0]
        assert np.abs(d).max() < 1e-3, chunk
        o.close()
        # the device's sweep on its own inputs: positions now, charges and chain state from the start
        pre = dict(st, positions=g.particles())
        c2 = cfgm.resolve(bench.workload_opts(cfgm, skin=skin, scale=0.1), P)
        c2.protonation_rng = prot
        o2 = ob.OracleSystem(_abi, c2, pre)
        o2.sweep()
        assert np.array_equal(g.charges(), o2.read(ob.F_CHARGES)), chunk
        assert g.protonation_rng_state() == int(o2.read(ob.F_PROT_RNG)[0]), chunk
        o2.close()
    # at the bench's skin a drift rebuild inside a 10-step chunk is rare; at 0.6 most chunks have one
    assert bond_chunks >= 5 and rebuilds >= (6 if skin < SKIN else 0)
    g.dispose()

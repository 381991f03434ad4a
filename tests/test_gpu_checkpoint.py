"""Checkpoints of a device system (soup/src/checkpoint.ts; tests/soup-checkpoint.test.ts:57-200):
the one-call payload equals the separate readbacks, encode -> JSON -> decode -> resume reconstructs
every field exactly at zero elapsed steps, taking a checkpoint leaves the trajectory bit-identical,
and a resumed system continues the run."""
import json

import numpy as np
import pytest

from helpers import boosted
from protocell_genesis_b200 import _abi, checkpoint as ck, config as cfgm
from protocell_genesis_b200.soup import SoupSystem

pytestmark = pytest.mark.gpu
P = cfgm.load_params()
CONFIG = {"box": [18, 18, 18], "seed": 7, "kT": 1.1, "start": {"C": 120, "O": 40, "H": 120, "M": 10, "W": 0},
          "electrostatics": {"enabled": True, "pH": 7.0, "ionicStrengthMolar": 0.01}}
STEPS = 1500


def _cfg(opts):
    return boosted(cfgm.resolve(opts, P), attempt=0.9, accept=1.0, brk=0.05)


def _system():
    opts = cfgm.SoupOptions(box=CONFIG["box"], seed=CONFIG["seed"], kT=CONFIG["kT"], start=CONFIG["start"],
                            electrostatics=CONFIG["electrostatics"], sweep_every=100)
    s = SoupSystem(_cfg(opts))
    s.relax_cold_start()
    return s


def _resume(f):
    r = ck.decode_checkpoint_resume(f)
    opts = ck.resume_options(f, r)
    opts.sweep_every = 100
    return SoupSystem(_cfg(opts), ck.resume_state(r))


def _fields(s):
    return dict(pos=s.particles(), vel=s.velocities(), slots=s.bond_slots(), center=s.center_links(),
                held=s.center_held_steps(), q=s.charges(), brng=s.rng_state()["bond"], trng=s.rng_state()["thermo"],
                events=s.events(), desorb=s.desorb_events(), prot=s.protonation_rng_state(), step=s.steps)


def _same(a, b):
    for k in a:
        x, y = a[k], b[k]
        if isinstance(x, np.ndarray):
            assert x.dtype == y.dtype and np.array_equal(x.view(np.uint32), y.view(np.uint32)), k
        else:
            assert x == y, k


def test_payload_equals_the_separate_readbacks():
    s = _system()
    s.step(300)
    arrays, sc = s.checkpoint_payload()
    f = _fields(s)
    for name, key in (("positions", "pos"), ("velocities", "vel"), ("bondSlots", "slots"), ("centerLink", "center"),
                      ("centerHeldSteps", "held"), ("bondRng", "brng"), ("thermoRng", "trng"), ("charges", "q")):
        assert np.array_equal(arrays[name].view(np.uint32), f[key].view(np.uint32)), name
    assert sc["globalStep"] == 300 and sc["protonationRng"] == f["prot"]
    assert sc["events"] == f["events"] and sc["desorbEvents"] == f["desorb"]
    assert sc["liveBox"] == [18.0, 18.0, 18.0] and sc["N"] == s.n
    inv = s.invariants()
    assert inv["monomers"] == ck.census(arrays["positions"])
    assert inv["bonds"] == sum(f["events"][b] - f["events"][k] for b, k in cfgm.rule_ids())
    s.dispose()


def test_round_trip_reconstructs_every_field_at_zero_steps():
    """tests/soup-checkpoint.test.ts:57-120: step 1500, encode, decode, create, compare."""
    a = _system()
    a.step(STEPS)
    f = json.loads(json.dumps(ck.encode_checkpoint(a, CONFIG)))
    b = _resume(f)
    fa, fb = _fields(a), _fields(b)
    assert (fa["slots"] != _abi.NONE).any() and sum(fa["events"].values()) > 0
    _same(fa, fb)
    a.dispose()
    b.dispose()


def test_checkpoint_is_trajectory_neutral():
    """A checkpoint is a pure readback: with one taken mid-run the run is bit-identical to the run
    without it (the reference can only check this against its own run-to-run scatter).  Both runs
    make the same step() calls: the constant-pH sweep is due-checked at the end of each call."""
    a, b = _system(), _system()
    a.step(300)
    b.step(300)
    ck.encode_checkpoint(a, CONFIG)
    a.step(200)
    b.step(200)
    _same(_fields(a), _fields(b))
    a.dispose()
    b.dispose()


def test_resumed_system_continues_the_run():
    """The resumed system's first force and its next steps follow the original's.  Not bit-exact:
    the original's force at the checkpoint was summed in the slot order of its last list build, the
    resumed system sums it in the order of its own build, so the two differ by FP32 rounding."""
    a = _system()
    a.step(STEPS)
    f = ck.encode_checkpoint(a, CONFIG)
    b = _resume(f)
    fa = a._read("soup_read_force", np.float32, 4).reshape(-1, 4)[:, :3].astype(np.float64)
    fb = b._read("soup_read_force", np.float32, 4).reshape(-1, 4)[:, :3].astype(np.float64)
    assert np.sqrt(((fa - fb) ** 2).sum() / (fa ** 2).sum()) < 1e-6
    a.step(20)
    b.step(20)
    pa, pb = a.particles().reshape(-1, 4)[:, :3], b.particles().reshape(-1, 4)[:, :3]
    d = pa - pb
    d -= np.round(d / 18.0) * 18.0
    assert np.abs(d).max() < 1e-3
    assert a.steps == b.steps == STEPS + 20
    a.dispose()
    b.dispose()


def test_binary_checkpoint_resumes_as_the_json_one(tmp_path):
    """A system resumed from the binary checkpoint and one resumed from the JSON CheckpointFile of the
    same state are the same system: equal fields, and bit-identical steps after."""
    a = _system()
    a.step(300)
    when = "2026-01-01T00:00:00.000Z"
    f = ck.encode_checkpoint(a, CONFIG, created_at=when)
    ck.write_checkpoint_binary(str(tmp_path / "c.bin"), a, CONFIG, created_at=when)
    b, c = _resume(f), _resume(ck.read_checkpoint_binary(str(tmp_path / "c.bin")))
    _same(_fields(b), _fields(c))
    b.step(50)
    c.step(50)
    assert np.array_equal(b.particles().view(np.uint32), c.particles().view(np.uint32))
    for s in (a, b, c):
        s.dispose()

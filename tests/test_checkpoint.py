"""Checkpoint files (soup/src/checkpoint.ts) on the host: the reference's CheckpointFile keys and
encoding, and an exact encode -> JSON -> decode round trip of a stepped oracle state
(tests/soup-checkpoint.test.ts:57-120 claim 1, with the oracle standing in for the system)."""
import json

import numpy as np
import pytest

import oracle_binding as ob
from helpers import boosted
from protocell_genesis_b200 import _abi, checkpoint as ck, config as cfgm

P = cfgm.load_params()
CONFIG = {"box": [18, 18, 18], "seed": 7, "kT": 1.1, "start": {"C": 120, "O": 40, "H": 120, "M": 10, "W": 0},
          "electrostatics": {"enabled": True, "pH": 7.0, "ionicStrengthMolar": 0.01}}

STEPS = 1500          # tests/soup-checkpoint.test.ts:62: real bonds and advanced RNG streams to check
FILE_KEYS = ["version", "createdAt", "config", "N", "globalStep", "liveBox", "cyclePhase", "cycleIndex",
             "activeCounts", "events", "desorbEvents", "positionsB64", "velocitiesB64", "bondSlotsB64",
             "centerLinkB64", "centerHeldStepsB64", "bondRngB64", "thermoRngB64", "chargesB64", "protonationRng"]


class OracleCheckpointable:
    """The reference's CheckpointableSystem (checkpoint.ts:123-139) over the oracle's arrays."""

    def __init__(self, o, cfg):
        self.o, self.cfg = o, cfg
        self.box = list(cfg.box)
        self.cyclePhase, self.cycleIndex = "none", 0

    @property
    def steps(self):
        return self.o.info()["step"]

    def particles(self):
        return self.o.read(ob.F_POS)

    def velocities(self):
        return self.o.read(ob.F_VEL)

    def bondSlots(self):
        return self.o.read(ob.F_SLOTS)

    def centerLinks(self):
        return self.o.read(ob.F_CENTER)

    def centerHeldSteps(self):
        return self.o.read(ob.F_HELD)

    def charges(self):
        return self.o.read(ob.F_CHARGES)

    def rngState(self):
        return {"bond": self.o.read(ob.F_BOND_RNG), "thermo": self.o.read(ob.F_THERMO_RNG)}

    def desorbEvents(self):
        d = self.o.read(ob.F_DESORB)
        return {"stretch": int(d[0]), "timeout": int(d[1])}

    def events(self):
        e = self.o.read(ob.F_EVENTS)
        out = {}
        for r, (b, k) in enumerate(cfgm.rule_ids()[: self.cfg.n_rules]):
            out[b], out[k] = int(e[2 * r]), int(e[2 * r + 1])
        return out

    def protonationRngState(self):
        return int(self.o.read(ob.F_PROT_RNG)[0])

    def invariants(self):
        return {"monomers": ck.census(self.particles()), "bonds": 0, "charge": 0}


def _stepped_oracle():
    opts = cfgm.SoupOptions(box=CONFIG["box"], seed=CONFIG["seed"], kT=CONFIG["kT"], start=CONFIG["start"],
                            electrostatics=CONFIG["electrostatics"])
    cfg = boosted(cfgm.resolve(opts, P), attempt=0.9, accept=1.0, brk=0.05)
    o = ob.OracleSystem(_abi, cfg)
    o.relax(30, 0.1)
    o.step(STEPS)
    return o, cfg


def _oracle_state(st):
    """resume_state's keys as the oracle's start-state names."""
    names = {"positions": "positions", "velocities": "velocities", "bondSlots": "bond_slots",
             "centerLink": "center_link", "centerHeldSteps": "center_held", "bondRng": "bond_rng",
             "thermoRng": "thermo_rng", "charges": "charges", "events": "events", "desorbEvents": "desorb_events"}
    return {names[k]: v for k, v in st.items()}


def test_base64_is_the_little_endian_bytes():
    """bytesToBase64 over the typed array's bytes (checkpoint.ts:37-56): 1.0f is 00 00 80 3f."""
    assert ck._b64(np.array([1.0], np.float32), np.float32) == "AACAPw=="
    assert ck._b64(np.array([0xFFFFFFFF, 1], np.uint32), np.uint32) == "/////wEAAAA="
    assert np.array_equal(ck._unb64("AACAPw==", np.float32), np.array([1.0], np.float32))


def test_round_trip_is_exact_and_keys_are_the_references():
    o, cfg = _stepped_oracle()
    sysA = OracleCheckpointable(o, cfg)
    f = ck.encode_checkpoint(sysA, CONFIG)
    assert list(f.keys()) == FILE_KEYS
    f2 = json.loads(json.dumps(f))                       # what the file holds
    r = ck.decode_checkpoint_resume(f2)
    assert r["globalStep"] == STEPS and f2["N"] == cfg.n
    for name, arr in [("positions", sysA.particles()), ("velocities", sysA.velocities()),
                      ("bondSlots", sysA.bondSlots()), ("centerLink", sysA.centerLinks()),
                      ("centerHeldSteps", sysA.centerHeldSteps()), ("bondRng", sysA.rngState()["bond"]),
                      ("thermoRng", sysA.rngState()["thermo"]), ("charges", sysA.charges())]:
        assert r[name].dtype == arr.dtype and np.array_equal(r[name].view(np.uint32), arr.view(np.uint32)), name
    assert r["protonationRng"] == sysA.protonationRngState()
    assert (r["bondSlots"] != _abi.NONE).any()              # real bonds were checked, not only NONE
    st = ck.resume_state(r)
    assert np.array_equal(st["events"], o.read(ob.F_EVENTS))
    assert np.array_equal(st["desorbEvents"], o.read(ob.F_DESORB))

    # the resumed oracle continues exactly where the original does
    opts = ck.resume_options(f2, r)
    cfgB = boosted(cfgm.resolve(opts, P), attempt=0.9, accept=1.0, brk=0.05)
    assert cfgB.n == cfg.n and cfgB.global_step == STEPS
    oB = ob.OracleSystem(_abi, cfgB, _oracle_state(st))
    o.step(30)
    oB.step(30)
    for fld in (ob.F_POS, ob.F_VEL, ob.F_SLOTS, ob.F_CHARGES, ob.F_THERMO_RNG, ob.F_BOND_RNG, ob.F_EVENTS):
        assert np.array_equal(o.read(fld).view(np.uint32), oB.read(fld).view(np.uint32)), fld


def test_resume_options_scale_the_wall_to_the_live_box():
    f = {"version": 1, "config": {"box": [40, 40, 40], "seed": 3, "kT": 1.0, "confine": {"radiusSigma": 10.0, "stiffness": 100}},
         "globalStep": 7, "liveBox": [30, 30, 30], "activeCounts": {"C": 5, "W": 9},
         "desorbEvents": {"stretch": 0, "timeout": 0}, "events": {}, "protonationRng": 11}
    for key, _, dt, per in ck.ARRAYS:
        f[key] = ck._b64(np.zeros(14 * per, dt), dt)
    o = ck.resume_options(f)
    assert o.box == [30.0, 30.0, 30.0] and o.global_step == 7 and o.protonation_rng == 11
    assert o.confine["radiusSigma"] == 7.5 and o.start == {"C": 5, "W": 9}


def test_a_file_from_before_the_charges_resumes_with_fresh_charges():
    """A CheckpointFile written before chargesB64 / protonationRng existed (checkpoint.ts:163-171:
    both optional): decoding gives None for them, and the resumed system takes its charges and
    protonation chain from the fresh-start rule (initialCharges)."""
    o, cfg = _stepped_oracle()
    f = ck.encode_checkpoint(OracleCheckpointable(o, cfg), CONFIG)
    del f["chargesB64"], f["protonationRng"]
    r = ck.decode_checkpoint_resume(json.loads(json.dumps(f)))
    assert r["charges"] is None and r["protonationRng"] is None
    st = ck.resume_state(r)
    assert "charges" not in st
    opts = ck.resume_options(f, r)
    assert opts.protonation_rng is None


def test_unknown_version_is_refused():
    with pytest.raises(ValueError, match="version"):
        ck.decode_checkpoint_resume({"version": 2})


def test_binary_checkpoint_holds_the_same_file(tmp_path):
    """The binary form: the same fields and the same array bytes as the JSON CheckpointFile; read back
    it decodes to the same resume state, and written as JSON it is the reference's file."""
    o, cfg = _stepped_oracle()
    sysA = OracleCheckpointable(o, cfg)
    when = "2026-01-01T00:00:00.000Z"
    f = ck.encode_checkpoint(sysA, CONFIG, created_at=when)
    size = ck.write_checkpoint_binary(str(tmp_path / "c.bin"), sysA, CONFIG, created_at=when)
    assert size == (tmp_path / "c.bin").stat().st_size and size % 64 == 0
    fb = ck.read_checkpoint_binary(str(tmp_path / "c.bin"))
    r, rb = ck.decode_checkpoint_resume(f), ck.decode_checkpoint_resume(fb)
    for k, v in r.items():
        if isinstance(v, np.ndarray):
            assert rb[k].dtype == v.dtype and np.array_equal(rb[k].view(np.uint32), v.view(np.uint32)), k
        else:
            assert rb[k] == v, k
    ck.write_checkpoint(str(tmp_path / "c.json"), fb)
    assert ck.read_checkpoint(str(tmp_path / "c.json")) == json.loads(json.dumps(f))
    (tmp_path / "bad.bin").write_bytes(b"NOTSOUP!" + bytes(8))
    with pytest.raises(ValueError, match="not a binary"):
        ck.read_checkpoint_binary(str(tmp_path / "bad.bin"))


def _small_file(n_c=5, n_w=9):
    f = {"version": 1, "config": {"box": [20, 20, 20], "seed": 3, "kT": 1.0}, "N": n_c + n_w,
         "globalStep": 0, "liveBox": [20, 20, 20], "activeCounts": {"C": n_c, "W": n_w},
         "desorbEvents": {"stretch": 0, "timeout": 0}, "events": {}, "protonationRng": 1}
    for key, _, dt, per in ck.ARRAYS:
        f[key] = ck._b64(np.zeros((n_c + n_w) * per, dt), dt)
    return f


def test_truncated_or_missing_arrays_are_refused(tmp_path):
    """Every array must hold N x its values per particle, N the census sum; a required array that is
    missing fails as the reference's decodeFloat32(undefined) does, and nothing reaches the library."""
    ck.decode_checkpoint_resume(_small_file())
    f = _small_file()
    f["velocitiesB64"] = ck._b64(np.zeros(13 * 4, np.float32), np.float32)   # one particle short
    with pytest.raises(ValueError, match="velocitiesB64"):
        ck.decode_checkpoint_resume(f)
    f = _small_file()
    del f["thermoRngB64"]
    with pytest.raises(ValueError, match="thermoRngB64"):
        ck.decode_checkpoint_resume(f)
    f = _small_file()
    f["N"] = 15
    with pytest.raises(ValueError, match="census"):
        ck.decode_checkpoint_resume(f)
    # the binary form: a table entry with a negative offset or a ragged byte count
    o, cfg = _stepped_oracle()
    ck.write_checkpoint_binary(str(tmp_path / "c.bin"), OracleCheckpointable(o, cfg), CONFIG)
    data = bytearray((tmp_path / "c.bin").read_bytes())
    n = int.from_bytes(data[8:16], "little")
    head = json.loads(data[16:16 + n].decode())
    for field, value, what in (("offset", -64, "non-negative"), ("bytes", 6, "whole number")):
        h2 = json.loads(json.dumps(head))
        h2["arrays"][1][field] = value
        enc = json.dumps(h2).encode()
        assert len(enc) <= n
        bad = bytes(data[:8]) + n.to_bytes(8, "little") + enc + b" " * (n - len(enc)) + bytes(data[16 + n:])
        (tmp_path / "bad.bin").write_bytes(bad)
        with pytest.raises(ValueError, match=what):
            ck.read_checkpoint_binary(str(tmp_path / "bad.bin"))


def test_state_arrays_of_the_wrong_size_are_refused_before_the_library():
    """SoupInitState takes plain pointers: init_state checks every array's size against the config."""
    from protocell_genesis_b200 import soup as soupm
    cfg = cfgm.resolve(cfgm.SoupOptions(box=[16, 16, 16], seed=1, kT=1.0, start={"C": 10, "W": 20}), P)
    good = {"positions": np.zeros(4 * cfg.n, np.float32), "bondSlots": np.zeros(3 * cfg.n, np.uint32),
            "desorbEvents": np.zeros(2, np.uint32), "events": np.zeros(2 * cfg.n_rules, np.uint32)}
    soupm.init_state(good, cfg)
    for k, bad in (("positions", np.zeros(4 * cfg.n - 4, np.float32)), ("bondSlots", np.zeros(cfg.n, np.uint32)),
                   ("events", np.zeros(1, np.uint32))):
        with pytest.raises(ValueError, match=k):
            soupm.init_state(dict(good, **{k: bad}), cfg)

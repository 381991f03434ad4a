"""Checkpoint files of a soup run (soup/src/checkpoint.ts): encodeCheckpoint and
decodeCheckpointResume over the reference's CheckpointFile format, so that a file written here
resumes under the reference and the other way round.

The format is the reference's (checkpoint.ts:118-172): a JSON object whose arrays are base64 strings
of their little-endian bytes (standard alphabet with padding, what atob/btoa read and write), one
string per array, in the readback layouts (positions f32 x4 with w = kind, bond slots u32 x3 with
0xFFFFFFFF = none).  What differs is the read side: on a SoupSystem every array comes from ONE
device gather and one host wait (soup_read_checkpoint) instead of ten concurrent readbacks.

Writing the object to disk is the caller's job in the reference (soup/cli/campaign.ts);
write_checkpoint / read_checkpoint are the plain JSON file I/O for callers in Python.
"""
import base64
import datetime as _dt
import json
from typing import Optional

import numpy as np

from . import config as _config

VERSION = 1

# CheckpointFile's per-particle arrays: (file key, resume key, dtype, values per particle), in the
# file's field order (checkpoint.ts:148-162).
ARRAYS = (
    ("positionsB64", "positions", np.float32, 4),
    ("velocitiesB64", "velocities", np.float32, 4),
    ("bondSlotsB64", "bondSlots", np.uint32, 3),
    ("centerLinkB64", "centerLink", np.uint32, 1),
    ("centerHeldStepsB64", "centerHeldSteps", np.uint32, 1),
    ("bondRngB64", "bondRng", np.uint32, 1),
    ("thermoRngB64", "thermoRng", np.uint32, 1),
    ("chargesB64", "charges", np.float32, 1),
)


def _b64(a: np.ndarray, dtype) -> str:
    """encodeTyped (checkpoint.ts:54-56): the array's little-endian bytes as one base64 string."""
    return base64.b64encode(np.ascontiguousarray(a, np.dtype(dtype).newbyteorder("<")).tobytes()).decode("ascii")


def _unb64(s, dtype) -> np.ndarray:
    """decodeFloat32 / decodeUint32 (checkpoint.ts:58-66).  An array read from a binary checkpoint
    passes through as it is."""
    if isinstance(s, np.ndarray):
        return s.astype(dtype)
    return np.frombuffer(base64.b64decode(s), np.dtype(dtype).newbyteorder("<")).astype(dtype)


def census(positions: np.ndarray, P: Optional[dict] = None) -> dict:
    """invariants().monomers (soup/src/soup-readback.ts:140-149): beads per monomer id, the kind read
    from each position's w, rounded."""
    monomers = (P or _config.load_params())["monomers"]
    kinds = np.rint(np.asarray(positions, np.float32).reshape(-1, 4)[:, 3]).astype(np.int64)
    c = np.bincount(kinds, minlength=len(monomers))
    return {m["id"]: int(c[k]) for k, m in enumerate(monomers)}


def _now() -> str:
    t = _dt.datetime.now(_dt.timezone.utc)
    return t.strftime("%Y-%m-%dT%H:%M:%S.") + f"{t.microsecond // 1000:03d}Z"


def encode_checkpoint(sys, config: dict, created_at: Optional[str] = None) -> dict:
    """encodeCheckpoint (checkpoint.ts:176-214): the CheckpointFile of `sys`'s current state."""
    out, arrays = _checkpoint_fields(sys, config, created_at)
    prot = out.pop("protonationRng")   # the reference's field order: the arrays, then protonationRng
    for key, name, dt, _ in ARRAYS:
        out[key] = _b64(arrays[name], dt)
    out["protonationRng"] = prot
    return out


def _checkpoint_fields(sys, config: dict, created_at: Optional[str] = None):
    """The CheckpointFile's scalar fields and its eight arrays (by name), unencoded.

    `sys` is a SoupSystem (one soup_read_checkpoint call) or any object with the reference's
    CheckpointableSystem readbacks (particles, velocities, bondSlots, centerLinks, centerHeldSteps,
    desorbEvents, rngState, events, invariants, charges, protonationRngState, box, steps).  Like the
    reference it only reads: the trajectory after it is the one without it."""
    if hasattr(sys, "checkpoint_payload"):
        arrays, sc = sys.checkpoint_payload()
        active = census(arrays["positions"])
        step, box, events, desorb, prot = (sc["globalStep"], sc["liveBox"], sc["events"], sc["desorbEvents"],
                                           sc["protonationRng"])
    else:
        rng = sys.rngState()
        arrays = dict(positions=sys.particles(), velocities=sys.velocities(), bondSlots=sys.bondSlots(),
                      centerLink=sys.centerLinks(), centerHeldSteps=sys.centerHeldSteps(), bondRng=rng["bond"],
                      thermoRng=rng["thermo"], charges=sys.charges())
        active = sys.invariants()["monomers"]
        step, box, events, desorb, prot = (sys.steps, sys.box, sys.events(), sys.desorbEvents(),
                                           sys.protonationRngState())
    out = {
        "version": VERSION,
        "createdAt": created_at or _now(),
        "config": config,
        "N": int(np.asarray(arrays["positions"]).size // 4),
        "globalStep": int(step),
        "liveBox": [float(x) for x in box],
        "cyclePhase": getattr(sys, "cyclePhase", "none"),
        "cycleIndex": int(getattr(sys, "cycleIndex", 0)),
        "activeCounts": dict(active),
        "events": {k: int(v) for k, v in events.items()},
        "desorbEvents": {"stretch": int(desorb["stretch"]), "timeout": int(desorb["timeout"])},
        "protonationRng": int(prot),
    }
    return out, arrays


def decode_checkpoint_resume(file: dict) -> dict:
    """decodeCheckpointResume (checkpoint.ts:219-237): CreateSoupOpts.resume's shape, arrays as numpy.
    A file without chargesB64 / protonationRng (written before electrostatics) gives None there; the
    other seven arrays are required (the reference's decodeFloat32 / decodeUint32 throw on a missing
    string), and every array must hold exactly N x its values per particle, N being the live census
    sum(activeCounts) (checkpoint.ts:113-126), or ValueError is raised before anything reads it."""
    if file.get("version") != VERSION:
        raise ValueError(f"checkpoint version {file.get('version')!r} is not {VERSION}")
    r = {
        "globalStep": int(file["globalStep"]),
        "liveBox": [float(x) for x in file["liveBox"]],
        "activeCounts": dict(file["activeCounts"]),
        "desorbEvents": np.array([file["desorbEvents"]["stretch"], file["desorbEvents"]["timeout"]], np.uint32),
        "events": dict(file["events"]),
        "protonationRng": file.get("protonationRng"),
    }
    n = int(sum(int(v) for v in r["activeCounts"].values()))
    if "N" in file and int(file["N"]) != n:
        raise ValueError(f"checkpoint: N={file['N']} does not equal the census sum {n} of activeCounts")
    for key, name, dt, per in ARRAYS:
        if file.get(key) is None:
            if name == "charges":
                r[name] = None
                continue
            raise ValueError(f"checkpoint: the required array {key} is missing")
        a = _unb64(file[key], dt)
        if a.size != n * per:
            raise ValueError(f"checkpoint: {key} holds {a.size} values, expected N x {per} = {n * per}")
        r[name] = a
    return r


def resume_options(file: dict, resume: Optional[dict] = None) -> _config.SoupOptions:
    """createSoup({...file.config, resume}) (soup/cli/campaign.ts:118-125) as SoupOptions: the live box
    and step of the file, its census as the composition (the MD step holds exactly the live beads),
    the protonation chain's state, and a wall radius scaled to the live box (liveRadius,
    soup/src/soup-confine.ts:76-78)."""
    c = file["config"]
    r = resume if resume is not None else decode_checkpoint_resume(file)
    confine = None
    if c.get("confine"):
        confine = dict(c["confine"])
        confine["radiusSigma"] = float(confine["radiusSigma"]) * (r["liveBox"][0] / float(c["box"][0]))
    return _config.SoupOptions(box=r["liveBox"], seed=int(c["seed"]), kT=float(c["kT"]), start=dict(r["activeCounts"]),
                               electrostatics=c.get("electrostatics"), confine=confine,
                               global_step=r["globalStep"], protonation_rng=r["protonationRng"])


def resume_state(resume: dict, rule_ids=None) -> dict:
    """The resume arrays as SoupSystem's start state; the events record becomes the device's counter
    array (bond, break per rule, in rule order)."""
    ids = rule_ids or _config.rule_ids()
    ev = np.zeros(2 * len(ids), np.uint32)
    for k, (b, brk) in enumerate(ids):
        ev[2 * k], ev[2 * k + 1] = resume["events"].get(b, 0), resume["events"].get(brk, 0)
    st = {name: resume[name] for _, name, _, _ in ARRAYS if resume.get(name) is not None}
    st["events"] = ev
    st["desorbEvents"] = resume["desorbEvents"]
    return st


def create_from_checkpoint(file: dict):
    """A SoupSystem resumed from `file`, at the file's global step."""
    from .soup import SoupSystem
    r = decode_checkpoint_resume(file)
    return SoupSystem(_config.resolve(resume_options(file, r)), resume_state(r))


def write_checkpoint(path: str, file: dict) -> None:
    """The CheckpointFile as the reference's JSON text; arrays read from a binary checkpoint are
    encoded to base64 here, so a binary file converts to the reference's format."""
    out = dict(file)
    for key, _, dt, _ in ARRAYS:
        if isinstance(out.get(key), np.ndarray):
            out[key] = _b64(out[key], dt)
    with open(path, "w") as fh:
        json.dump(out, fh)


BINARY_MAGIC = b"SOUPCKB1"
_ALIGN = 64


def write_checkpoint_binary(path: str, sys, config: dict, created_at: Optional[str] = None) -> int:
    """The checkpoint of `sys` without the base64 round trip: an 8-byte magic, the header length
    (u64 little-endian), the CheckpointFile's fields as JSON with an "arrays" table (key, dtype,
    offset, bytes), then the eight arrays' little-endian bytes, each at a 64-byte aligned offset.
    Returns the file's size in bytes."""
    out, arrays = _checkpoint_fields(sys, config, created_at)
    table, blobs, at = [], [], 0
    for key, name, dt, _ in ARRAYS:
        b = np.ascontiguousarray(arrays[name], np.dtype(dt).newbyteorder("<"))
        table.append({"key": key, "dtype": np.dtype(dt).str.lstrip("<>|="), "offset": at, "bytes": b.nbytes})
        blobs.append((at, b))
        at += -(-b.nbytes // _ALIGN) * _ALIGN
    out["arrays"] = table
    head = json.dumps(out).encode()
    start = -(-(16 + len(head)) // _ALIGN) * _ALIGN
    with open(path, "wb") as fh:
        fh.write(BINARY_MAGIC + len(head).to_bytes(8, "little") + head)
        fh.write(b"\0" * (start - 16 - len(head)))
        pos = 0
        for off, b in blobs:
            if off > pos:
                fh.write(b"\0" * (off - pos))
            fh.write(memoryview(b).cast("B"))
            pos = off + b.nbytes
        if at > pos:
            fh.write(b"\0" * (at - pos))
    return start + at


def read_checkpoint_binary(path: str) -> dict:
    """A binary checkpoint as a CheckpointFile whose array fields are numpy arrays (accepted by
    decode_checkpoint_resume, create_from_checkpoint and write_checkpoint)."""
    with open(path, "rb") as fh:
        data = fh.read()
    if data[:8] != BINARY_MAGIC:
        raise ValueError("not a binary soup checkpoint")
    n = int.from_bytes(data[8:16], "little")
    file = json.loads(data[16:16 + n].decode())
    start = -(-(16 + n) // _ALIGN) * _ALIGN
    dts = {key: dt for key, _, dt, _ in ARRAYS}
    for a in file.pop("arrays"):
        dt = np.dtype(a["dtype"]).newbyteorder("<")
        if a["key"] not in dts or np.dtype(a["dtype"]) != np.dtype(dts[a["key"]]):
            raise ValueError(f"binary checkpoint: unexpected array {a['key']!r} of {a['dtype']}")
        lo = start + int(a["offset"])
        nb = int(a["bytes"])
        if int(a["offset"]) < 0 or nb < 0 or nb % dt.itemsize:
            raise ValueError(f"binary checkpoint: {a['key']} has offset {a['offset']} and {nb} bytes, "
                             f"not a whole number of {dt.itemsize}-byte values at a non-negative offset")
        if lo + nb > len(data):
            raise ValueError(f"binary checkpoint: {a['key']} runs past the end of the file")
        file[a["key"]] = np.frombuffer(data, dt, int(a["bytes"]) // dt.itemsize, lo).astype(dts[a["key"]])
    return file


def read_checkpoint(path: str) -> dict:
    with open(path) as fh:
        return json.load(fh)


encodeCheckpoint = encode_checkpoint
writeCheckpointBinary = write_checkpoint_binary
readCheckpointBinary = read_checkpoint_binary
decodeCheckpointResume = decode_checkpoint_resume

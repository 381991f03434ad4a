"""The C ABI: the library loads without a GPU, exports every declared entry point, and the ctypes
mirror has the exact struct layout of include/soup_b200.h (checked against a C compiler)."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from protocell_genesis_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "soup_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(soup_\w+)\s*\(", src, flags=re.M)))


def test_library_exports_every_declared_symbol():
    lib = _abi.lib()
    names = declared_functions()
    assert len(names) >= 35
    missing = [n for n in names if not hasattr(lib, n)]
    assert missing == []
    assert set(names) <= set(_abi.SIGNATURES)


def test_struct_layout_matches_header(tmp_path):
    prog = tmp_path / "layout.c"
    fields = [(s, f) for s in ("SoupConfig", "SoupInitState", "SoupSweepResult", "SoupClosureResult", "SoupInfo", "SoupPairingStats", "SoupAggregateShape")
              for f, _ in getattr(_abi, s)._fields_]
    body = "\n".join(f'  printf("{s}.{f} %zu\\n", offsetof({s}, {f}));' for s, f in fields)
    sizes = "\n".join(f'  printf("{s} %zu\\n", sizeof({s}));' for s in
                      ("SoupConfig", "SoupInitState", "SoupSweepResult", "SoupClosureResult", "SoupInfo", "SoupPairingStats", "SoupAggregateShape"))
    prog.write_text(f'#include <stdio.h>\n#include <stddef.h>\n#include "{HEADER}"\nint main(void) {{\n{body}\n{sizes}\n  return 0;\n}}\n')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", str(prog), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = dict(line.rsplit(" ", 1) for line in out if line)
    for s, f in fields:
        assert int(got[f"{s}.{f}"]) == getattr(getattr(_abi, s), f).offset, (s, f)
    for s in ("SoupConfig", "SoupInitState", "SoupSweepResult", "SoupClosureResult", "SoupInfo", "SoupPairingStats", "SoupAggregateShape"):
        assert int(got[s]) == C.sizeof(getattr(_abi, s)), s


def test_errors_without_a_device_are_status_codes():
    # no GPU here: creating a system fails with a status and a message, never a crash
    from helpers import plain_opts
    from protocell_genesis_b200 import config as cfgm
    cfg = cfgm.resolve(plain_opts())
    lib = _abi.lib()
    h = C.c_void_p()
    rc = lib.soup_create(C.byref(cfg), None, C.byref(h))
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        assert rc == 0
        lib.soup_destroy(h)
    else:
        assert rc in (9, 7)
        assert len(lib.soup_last_error(None)) > 0
    bad = _abi.SoupConfig()
    rc = lib.soup_create(C.byref(bad), None, C.byref(h))
    assert rc == 1 and b"abi_version" in lib.soup_last_error(None)

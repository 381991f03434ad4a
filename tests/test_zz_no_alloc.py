"""soup_aggregate_labels_noalloc (scratch in a fixed device array, no allocation) against
soup_aggregate_labels (per-call cudaMalloc scratch) on the same device state.

Two calls in a row with different member sets and cut-offs check that each call clears what the
previous one left in the shared array; the limits are checked to be refused before any work.
The file runs last so that it also sees the device after every other GPU test.
"""
import numpy as np
import pytest

import oracle_binding as ob
from helpers import boosted, plain_opts
from protocell_genesis_b200 import _abi, config as cfgm
from protocell_genesis_b200.soup import SoupSystem

pytestmark = pytest.mark.gpu

P = cfgm.load_params()
MAX_MEMBERS = 1 << 18      # SOUP_NOALLOC_MAX_MEMBERS
MAX_CELLS = 1 << 18        # SOUP_NOALLOC_MAX_CELLS


def _system():
    opts = plain_opts(box=[15, 15, 15], start={"C": 900, "O": 260, "H": 0, "M": 160, "W": 0})
    cfg = boosted(cfgm.resolve(opts, P), attempt=0.9, accept=1.0, brk=0.02)
    o = ob.OracleSystem(_abi, cfg)
    o.relax(30, 0.1)
    o.step(200)
    st = dict(positions=o.read(ob.F_POS), bond_slots=o.read(ob.F_SLOTS), center_link=o.read(ob.F_CENTER))
    return cfg, SoupSystem(cfg, st)


def test_noalloc_labels_equal_the_allocating_entry_point():
    cfg, g = _system()
    n = cfg.n
    cut = cfgm.wca_cutoff(P["params"]["sigma"] * 1.0) + P["params"]["wc"]
    rng = np.random.default_rng(7)
    big = np.arange(n, dtype=np.uint32)                                 # every particle, fine grid
    small = np.sort(rng.choice(n, n // 3, replace=False)).astype(np.uint32)
    for members, c in [(big, cut), (small, 2.5 * cut), (big, cut)]:
        nc_ref, lab_ref = g.aggregate_labels(members, c)
        nc, lab = g.aggregate_labels_noalloc(members, c)
        assert nc == nc_ref and np.array_equal(lab, lab_ref)
        assert 0 < nc <= members.size
    nc, lab = g.aggregate_labels_noalloc(np.zeros(0, np.uint32), cut)
    assert nc == 0 and lab.size == 0
    g.dispose()


def test_noalloc_limits_are_refused():
    cfg, g = _system()
    with pytest.raises(_abi.SoupError) as e:
        g.aggregate_labels_noalloc(np.zeros(MAX_MEMBERS + 1, np.uint32), 1.0)
    assert e.value.code == "SOUP_E_ARG" and "maximum" in str(e.value)
    fine = cfg.box[0] / 80.0                      # about 80^3 cells > the cell limit
    with pytest.raises(_abi.SoupError) as e:
        g.aggregate_labels_noalloc(np.arange(10, dtype=np.uint32), fine)
    assert e.value.code == "SOUP_E_ARG" and "cells" in str(e.value)
    # the handle still works after a refusal
    nc_ref, lab_ref = g.aggregate_labels(np.arange(100, dtype=np.uint32), 1.5)
    assert g.aggregate_labels_noalloc(np.arange(100, dtype=np.uint32), 1.5)[0] == nc_ref
    g.dispose()


def test_noalloc_calls_allocate_nothing():
    """The entry point's contract: after one warm call on the device, calls of different sizes leave
    the device's free memory exactly where it was (cudaMemGetInfo, device-wide)."""
    import torch
    cfg, g = _system()
    n = cfg.n
    cut = cfgm.wca_cutoff(P["params"]["sigma"] * 1.0) + P["params"]["wc"]
    torch.cuda.mem_get_info()                        # the runtime's own context first
    g.aggregate_labels_noalloc(np.arange(n, dtype=np.uint32), cut)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    rng = np.random.default_rng(3)
    for frac, c in ((1.0, cut), (0.25, 2 * cut), (0.6, 0.7 * cut), (1.0, 3 * cut)):
        members = np.sort(rng.choice(n, int(frac * n), replace=False)).astype(np.uint32)
        g.aggregate_labels_noalloc(members, c)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    g.dispose()

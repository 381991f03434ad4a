"""The FP64 torch window that serves as the adjoint's reference gradient, pinned to the oracle on the
CPU: its force is the oracle's FP64 force, its noise replay reproduces the oracle's thermostat states,
its trajectory follows the oracle's step phases, and its autograd gradient equals central
differences of its own loss (FP64, eps = 1e-3 relative)."""
import numpy as np
import pytest
import torch

import oracle_binding as ob
import torch_reference as tr
from helpers import oracle_bilayer_start, rel_rms
from protocell_genesis_b200 import _abi


@pytest.fixture(scope="module")
def patch():
    return oracle_bilayer_start(seed=3, relax=200, steps=60)


def test_force_is_the_oracle_fp64_force(patch):
    cfg, start = patch
    win = tr.SoupWindow64(cfg, start, 1, device="cpu")
    f = win.force(win.x0, torch.tensor(tr.theta_of(cfg), dtype=torch.float64)).numpy()
    o = ob.OracleSystem(_abi, cfg, start)
    fo = o.forces64().reshape(-1, 4)[:, :3]
    o.close()
    assert rel_rms(f, fo) < 1e-7
    assert np.abs(f).max() > 1.0


def test_noise_and_trajectory_follow_the_oracle_phases(patch):
    cfg, start = patch
    steps = 10
    win = tr.SoupWindow64(cfg, start, steps, device="cpu")
    frames = win.frames(tr.theta_of(cfg)).numpy()
    o = ob.OracleSystem(_abi, cfg, start)
    o.phase(_abi.PHASE_REBUILD)
    o.phase(_abi.PHASE_FORCE)
    for _ in range(steps):       # the window's step: no bond or charge Monte Carlo
        o.phase(_abi.PHASE_KICK_DRIFT)
        o.phase(_abi.PHASE_REBUILD)
        o.phase(_abi.PHASE_FORCE)
        o.phase(_abi.PHASE_KICK_THERMO)
    _, final_rng = tr.thermostat_noise(start["thermo_rng"], steps)
    assert np.array_equal(final_rng, o.read(ob.F_THERMO_RNG))
    po = o.read(ob.F_POS).reshape(-1, 4)[:, :3].astype(np.float64)
    o.close()
    box = np.array(list(cfg.box))
    d = frames[-1] - po
    d -= np.round(d / box) * box
    moved = frames[-1] - frames[0]
    assert np.abs(moved).max() > 0.02          # the particles moved
    assert np.abs(d).max() < 1e-4              # FP64 against the oracle's FP32 step


def test_autograd_equals_central_differences(patch):
    cfg, start = patch
    steps = 8
    win = tr.SoupWindow64(cfg, start, steps, device="cpu")
    gen = torch.Generator().manual_seed(5)
    w = torch.randn((steps + 1, win.n, 4), generator=gen, dtype=torch.float64)
    theta0 = tr.theta_of(cfg)
    _, grad = win.loss_and_grad(theta0, w)
    fd = np.zeros_like(grad)
    for p in range(len(theta0)):
        eps = 1e-3 * max(abs(theta0[p]), 0.1)
        tp, tm = theta0.copy(), theta0.copy()
        tp[p] += eps
        tm[p] -= eps
        fd[p] = (win.loss(tp, w) - win.loss(tm, w)) / (2 * eps)
    print("grad", grad, "\nfd  ", fd)
    assert np.all(np.abs(grad - fd) <= 1e-4 * np.abs(fd) + 1e-8 * np.abs(fd).max())

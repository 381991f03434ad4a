"""The library's adjoint of the force + Langevin window (FP32, through the C ABI and the
torch.autograd.Function) against two oracles on the same start state and the same noise:
  - the FP64 torch window's autograd gradient (tests/torch_reference.py, itself pinned to the CPU
    oracle's FP64 force and step phases), within 1e-3 relative per parameter;
  - central finite differences of the FP64 window, within 1e-3 relative per parameter;
and, as a self-consistency check, central differences of the library's own FP32 forward for the
parameters whose loss change is far above FP32 rounding.  Two losses: a fixed random linear
functional of every frame's displacement from the first frame (minimum image, so periodic wrapping
leaves it smooth), which reaches every force term, and the bilayer thickness proxy.

The force is continuous but its Jacobian is not (every cutoff: WCA, the attraction window, the
screened-Coulomb shift), so central differences converge only linearly in eps once a pair crosses a
cutoff inside the interval: on the 20-step window eps = 1e-3 leaves errors up to 7e-3 while
eps = 1e-6 agrees to 3e-5.  The dynamics are chaotic: over a 200-step window the FP32 and FP64
trajectories separate enough that their gradients differ by up to about 2e-2, as do the FP64
gradients of two starts that differ by FP32 rounding."""
import numpy as np
import pytest
import torch

import torch_reference as tr
from helpers import oracle_bilayer_start
from protocell_genesis_b200 import _abi, adjoint
from protocell_genesis_b200.soup import SoupSystem

pytestmark = pytest.mark.gpu

STEPS = 20
EVERY = 5
TOL = 1e-3


@pytest.fixture(scope="module")
def patch():
    cfg, start = oracle_bilayer_start(seed=3, relax=300, steps=200)
    gen = torch.Generator().manual_seed(1)
    w = torch.randn((STEPS + 1, cfg.n, 4), generator=gen, dtype=torch.float64)
    w[:, :, 3] = 0
    w[0] = 0
    return cfg, start, w


def _displacement_loss(traj, w, box):
    d = traj.double() - traj[0:1].double()
    d = d - torch.round(d / box) * box
    return (d * w).sum()


def _gpu(g, start, theta, w, every=EVERY):
    g.write_state(start)
    th = torch.tensor(theta, dtype=torch.float64, requires_grad=True)
    traj = adjoint.SoupWindow.apply(th, g, STEPS, every)
    box = torch.tensor(list(g.cfg.box) + [1.0], dtype=torch.float64, device="cuda")
    loss = _displacement_loss(traj, w.cuda(), box)
    loss.backward()
    return float(loss.detach()), th.grad.numpy().copy()


def test_gradient_matches_the_fp64_window_and_its_central_differences(patch):
    cfg, start, w = patch
    g = SoupSystem(cfg, start)
    theta0 = g.get_diff_params()
    assert np.allclose(theta0, tr.theta_of(cfg))
    loss, grad = _gpu(g, start, theta0, w)
    win = tr.SoupWindow64(cfg, start, STEPS, device="cuda")
    loss64, grad64 = win.loss_and_grad(theta0, w)
    fd = np.zeros_like(grad64)
    for p in range(_abi.DIFF_NPARAM):
        eps = 1e-6 * max(abs(theta0[p]), 0.1)
        tp, tm = theta0.copy(), theta0.copy()
        tp[p] += eps
        tm[p] -= eps
        fd[p] = (win.loss(tp, w) - win.loss(tm, w)) / (2 * eps)
    g.dispose()
    print("\nadjoint", grad, "\nfp64   ", grad64, "\nfd64   ", fd,
          "\nrel vs fp64", np.abs(grad - grad64) / np.abs(grad64), "\nrel vs fd  ", np.abs(grad - fd) / np.abs(fd))
    assert loss == pytest.approx(loss64, rel=1e-4)
    assert np.all(np.abs(grad - grad64) <= TOL * np.abs(grad64)), (grad, grad64)
    assert np.all(np.abs(grad - fd) <= TOL * np.abs(fd)), (grad, fd)


def test_gradient_matches_central_differences_of_the_fp32_forward(patch):
    cfg, start, w = patch
    g = SoupSystem(cfg, start)
    theta0 = g.get_diff_params()
    _, grad = _gpu(g, start, theta0, w)
    fd = np.zeros_like(grad)
    resolved = []
    for p in range(_abi.DIFF_NPARAM):
        eps = 1e-2 * max(abs(theta0[p]), 0.1)
        tp, tm = theta0.copy(), theta0.copy()
        tp[p] += eps
        tm[p] -= eps
        lp, _ = _gpu(g, start, tp, w)
        lm, _ = _gpu(g, start, tm, w)
        fd[p] = (lp - lm) / (2 * eps)
        if abs(lp - lm) > 5e-2:          # far above the FP32 rounding of the loss (about 1e-4 here)
            resolved.append(p)
    g.set_diff_params(theta0)
    g.dispose()
    print("\nadjoint", grad, "\nfd32   ", fd, "\nresolved", resolved)
    assert len(resolved) >= 4
    for p in resolved:
        assert abs(grad[p] - fd[p]) <= 1e-2 * abs(fd[p]), (p, grad[p], fd[p])


def test_start_state_gradients_match_the_fp64_window(patch):
    cfg, start, w = patch
    g = SoupSystem(cfg, start)
    theta0 = g.get_diff_params()
    g.write_state(start)
    traj = torch.empty((STEPS + 1, g.n, 4), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    g.diff_forward(STEPS, EVERY, traj.data_ptr())
    torch.cuda.synchronize()
    t = traj.detach().clone().requires_grad_(True)
    box = torch.tensor(list(cfg.box) + [1.0], dtype=torch.float64, device="cuda")
    _displacement_loss(t, w.cuda(), box).backward()
    dldx = t.grad.float().contiguous()
    dx0 = torch.zeros((g.n, 4), dtype=torch.float32, device="cuda")
    dv0 = torch.zeros((g.n, 4), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    g.diff_backward(dldx.data_ptr(), dx0.data_ptr(), dv0.data_ptr())
    torch.cuda.synchronize()
    g.dispose()
    win = tr.SoupWindow64(cfg, start, STEPS, device="cuda")
    gx, gv = win.start_gradients(theta0, w)
    ex = dx0.cpu().double().numpy()[:, :3]
    ev = dv0.cpu().double().numpy()[:, :3]
    rx = np.sqrt(((ex - gx) ** 2).sum() / (gx ** 2).sum())
    rv = np.sqrt(((ev - gv) ** 2).sum() / (gv ** 2).sum())
    print("\nrel rms dx0", rx, "dv0", rv)
    assert rx < TOL and rv < TOL


def test_checkpoint_spacing_and_repeatability(patch, monkeypatch):
    """The window keeps every frame on the device when they fit its budget, and otherwise checkpoints
    and replays segments.  Each checkpoint re-sorts the particles, which changes FP32 summation order,
    so the two modes and different spacings agree to rounding; the same spacing repeats bit for bit
    (the segments are replayed exactly from their checkpoints)."""
    cfg, start, w = patch
    g = SoupSystem(cfg, start)
    theta0 = g.get_diff_params()
    l0, g0 = _gpu(g, start, theta0, w, every=3)                # every frame kept
    monkeypatch.setenv("SOUP_DIFF_FRAME_BUDGET_MB", "0")      # checkpoints and replay
    l1, g1 = _gpu(g, start, theta0, w, every=3)
    l1b, g1b = _gpu(g, start, theta0, w, every=3)
    l2, g2 = _gpu(g, start, theta0, w, every=STEPS)
    g.dispose()
    assert l1 == l1b and np.array_equal(g1, g1b)
    assert l2 == pytest.approx(l1, rel=1e-5)
    assert np.allclose(g2, g1, rtol=1e-3, atol=1e-5 * np.abs(g1).max())
    assert l0 == pytest.approx(l1, rel=1e-5)
    assert np.allclose(g0, g1, rtol=1e-3, atol=1e-5 * np.abs(g1).max())


def _thickness(cfg, start):
    p = start["positions"].reshape(-1, 4)
    slots = start["bond_slots"].reshape(-1, 3)
    heads = np.nonzero(p[:, 3] == 1)[0]
    tails = np.nonzero((p[:, 3] == 0) & np.any(slots != tr.NONE, axis=1))[0]
    h = torch.tensor(heads, device="cuda")
    t = torch.tensor(tails, device="cuda")
    return lambda frames: adjoint.thickness_proxy(frames, h, t, float(cfg.box[2]))


def _gpu_observable(g, start, theta, fn, steps, every):
    g.write_state(start)
    th = torch.tensor(theta, dtype=torch.float64, requires_grad=True)
    v = fn(adjoint.SoupWindow.apply(th, g, steps, every).double())
    v.backward()
    return float(v.detach()), th.grad.numpy().copy()


def test_thickness_gradient_over_50_steps(patch):
    """The bilayer thickness proxy over a 50-step window with checkpoints every 10 steps, against the
    FP64 gradient and FP64 central differences at eps = 1e-3 relative."""
    cfg, start, _ = patch
    steps, every = 50, 10
    fn = _thickness(cfg, start)
    g = SoupSystem(cfg, start)
    theta0 = g.get_diff_params()
    v, grad = _gpu_observable(g, start, theta0, fn, steps, every)
    g.dispose()
    win = tr.SoupWindow64(cfg, start, steps, device="cuda")
    v64, grad64 = win.observable_and_grad(theta0, fn)
    fd = np.zeros_like(grad64)
    for p in range(_abi.DIFF_NPARAM):
        eps = 1e-3 * max(abs(theta0[p]), 0.1)
        tp, tm = theta0.copy(), theta0.copy()
        tp[p] += eps
        tm[p] -= eps
        fd[p] = (win.observable(tp, fn) - win.observable(tm, fn)) / (2 * eps)
    print("\nthickness", v, v64, "\nadjoint", grad, "\nfp64   ", grad64, "\nfd64   ", fd)
    assert v == pytest.approx(v64, rel=1e-5)
    assert np.all(np.abs(grad - grad64) <= TOL * np.abs(grad64)), (grad, grad64)
    assert np.all(np.abs(grad - fd) <= TOL * np.abs(fd)), (grad, fd)


def test_thickness_gradient_over_the_200_step_window(patch):
    """The 200-step window with checkpoints every 20 steps: chaos bounds the agreement of any two
    gradients whose trajectories differ by rounding, so the bar here is the FP64 gradient's own
    spread under a start perturbation of FP32 size (measured about 2e-2), not 1e-3."""
    cfg, start, _ = patch
    steps, every = 200, 20
    fn = _thickness(cfg, start)
    g = SoupSystem(cfg, start)
    theta0 = g.get_diff_params()
    v, grad = _gpu_observable(g, start, theta0, fn, steps, every)
    g.dispose()
    win = tr.SoupWindow64(cfg, start, steps, device="cuda")
    v64, grad64 = win.observable_and_grad(theta0, fn)
    nudged = dict(start)
    pos = start["positions"].reshape(-1, 4).astype(np.float64)
    pos[:, :3] += 1e-6 * np.random.default_rng(0).normal(size=(len(pos), 3))
    nudged["positions"] = pos.reshape(-1)
    _, grad64b = tr.SoupWindow64(cfg, nudged, steps, device="cuda").observable_and_grad(theta0, fn)
    spread = np.abs(grad64b - grad64) / np.abs(grad64)
    print("\nadjoint", grad, "\nfp64   ", grad64, "\nnudged ", grad64b, "\nrel adjoint", np.abs(grad - grad64) / np.abs(grad64),
          "\nrel nudged", spread)
    assert v == pytest.approx(v64, rel=1e-5)
    assert np.all(np.abs(grad - grad64) <= 5e-2 * np.abs(grad64)), (grad, grad64)


def test_batched_window_equals_its_replicas(monkeypatch):
    """A batch of two patches differentiates as one window with shared parameters: its gradient is
    the sum of the replicas' own.  With checkpoints every 5 steps (no drift-triggered rebuild inside a
    segment) the batch's frames are the replicas' frames bit for bit; with every frame kept, a rebuild
    that one replica's drift triggers re-sorts the other too, so frames agree to FP32 rounding."""
    from protocell_genesis_b200.soup import SoupBatch
    c1, s1 = oracle_bilayer_start(seed=3, relax=300, steps=200)
    c2, s2 = oracle_bilayer_start(seed=4, relax=300, steps=200)
    n1, n2 = c1.n, c2.n
    gen = torch.Generator().manual_seed(7)
    w = torch.randn((STEPS + 1, n1 + n2, 4), generator=gen, dtype=torch.float64)
    w[:, :, 3] = 0
    w[0] = 0
    box = torch.tensor(list(c1.box) + [1.0], dtype=torch.float64, device="cuda")

    def run(sys_, wt):
        th = torch.tensor(sys_.get_diff_params(), dtype=torch.float64, requires_grad=True)
        traj = adjoint.SoupWindow.apply(th, sys_, STEPS, EVERY)
        loss = _displacement_loss(traj, wt.cuda(), box)
        loss.backward()
        return float(loss.detach()), th.grad.numpy().copy(), traj.detach().cpu().numpy()

    def both():
        batch = SoupBatch([c1, c2], [s1, s2])
        out = run(batch, w)
        batch.dispose()
        parts = []
        for c, st, sl in ((c1, s1, slice(0, n1)), (c2, s2, slice(n1, n1 + n2))):
            g = SoupSystem(c, st)
            parts.append(run(g, w[:, sl]))
            g.dispose()
        return out, parts

    (lb, gb, tb), parts = both()                                 # every frame kept
    d = np.abs(tb[:, :n1] - parts[0][2]).max(), np.abs(tb[:, n1:] - parts[1][2]).max()
    assert max(d) < 1e-4
    assert lb == pytest.approx(parts[0][0] + parts[1][0], rel=1e-6)
    assert np.allclose(gb, parts[0][1] + parts[1][1], rtol=1e-3, atol=1e-6)
    monkeypatch.setenv("SOUP_DIFF_FRAME_BUDGET_MB", "0")        # checkpoints every 5 steps
    (lb, gb, tb), parts = both()
    assert np.array_equal(tb[:, :n1], parts[0][2]) and np.array_equal(tb[:, n1:], parts[1][2])
    assert lb == pytest.approx(parts[0][0] + parts[1][0], rel=1e-12)
    assert np.allclose(gb, parts[0][1] + parts[1][1], rtol=1e-9, atol=1e-12)


def test_frame_stride_gives_the_gradient_of_the_kept_frames(patch):
    """A window that hands back every 5th frame (soup_diff_forward_strided) differentiates a loss on
    those frames exactly as the full window does when the loss reads the same frames: the reverse
    pass adds dJ/dx only at the kept steps, and the others are zero either way."""
    cfg, start, w = patch
    stride = 5
    box = torch.tensor(list(cfg.box) + [1.0], dtype=torch.float64, device="cuda")
    ws = w[::stride].cuda()

    def run(g, frames_of):
        g.write_state(start)
        th = torch.tensor(g.get_diff_params(), dtype=torch.float64, requires_grad=True)
        traj = frames_of(th)
        loss = _displacement_loss(traj, ws, box)
        loss.backward()
        return traj.detach(), float(loss.detach()), th.grad.numpy().copy()

    g = SoupSystem(cfg, start)
    t_full, l_full, g_full = run(g, lambda th: adjoint.SoupWindow.apply(th, g, STEPS, EVERY)[::stride])
    t_str, l_str, g_str = run(g, lambda th: adjoint.SoupWindow.apply(th, g, STEPS, EVERY, stride))
    g.dispose()
    assert t_str.shape[0] == STEPS // stride + 1
    assert torch.equal(t_full, t_str)
    assert l_full == l_str
    assert np.array_equal(g_full, g_str), (g_full, g_str)
    with pytest.raises(ValueError):
        adjoint.SoupWindow.apply(torch.zeros(_abi.DIFF_NPARAM, dtype=torch.float64), g, STEPS, EVERY, 3)

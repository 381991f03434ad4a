"""The adjoint on the differentiable bilayer patch at its full size: 2,048 five-bead amphiphiles in
water at 0.80, box 32 x 32 x 40 sigma, 32,768 beads (the bench's `gradient` workload).  The start is
the seeded preassembled patch relaxed and stepped on the device.  Against the FP64 torch window
(tests/torch_reference.py) on the same start and the same replayed noise:
  - a 20-step window of a random linear functional of the displacements, checkpoints every 5 steps:
    the adjoint gradient within 1e-3 relative of the FP64 gradient and of FP64 central differences
    (eps = 1e-6 relative: the force's Jacobian jumps at every cutoff, so a larger eps measures the
    jumps a pair crossing inside the interval makes, not the gradient);
  - a 50-step window of the bilayer thickness proxy, checkpoints every 10 steps: the same two bars.
"""
import numpy as np
import pytest
import torch

import bench
import torch_reference as tr
from protocell_genesis_b200 import _abi, adjoint, config as cfgm
from protocell_genesis_b200.soup import SoupSystem

pytestmark = pytest.mark.gpu

TOL = 1e-3


@pytest.fixture(scope="module")
def patch():
    cfg, st = bench.bilayer_patch(_abi.lib(), cfgm)
    assert cfg.n == 32768
    g = SoupSystem(cfg, st)
    g.relax_cold_start(300, 0.05)
    g.step(200)
    rng = g.rng_state()
    start = dict(positions=g.particles(), velocities=g.velocities(), bond_slots=g.bond_slots(),
                 center_link=g.center_links(), center_held=g.center_held_steps(), bond_rng=rng["bond"],
                 thermo_rng=rng["thermo"], charges=g.charges(), frozen=g.frozen())
    g.dispose()
    return cfg, start


def _check(name, grad, grad64, fd):
    rel64 = np.abs(grad - grad64) / np.abs(grad64)
    relfd = np.abs(grad - fd) / np.abs(fd)
    print(f"\n{name}\nadjoint {grad}\nfp64    {grad64}\nfd64    {fd}\nrel vs fp64 {rel64}\nrel vs fd   {relfd}")
    assert np.all(rel64 <= TOL), (grad, grad64)
    assert np.all(relfd <= TOL), (grad, fd)


def _fd(theta0, f):
    out = np.zeros(len(theta0))
    for p in range(len(theta0)):
        eps = 1e-6 * max(abs(theta0[p]), 0.1)
        tp, tm = theta0.copy(), theta0.copy()
        tp[p] += eps
        tm[p] -= eps
        out[p] = (f(tp) - f(tm)) / (2 * eps)
    return out


def test_displacement_gradient_over_20_steps_at_full_size(patch):
    cfg, start = patch
    steps, every = 20, 5
    gen = torch.Generator().manual_seed(5)
    w = torch.randn((steps + 1, cfg.n, 4), generator=gen, dtype=torch.float64)
    w[:, :, 3] = 0
    w[0] = 0
    box = torch.tensor(list(cfg.box) + [1.0], dtype=torch.float64, device="cuda")
    g = SoupSystem(cfg, start)
    theta0 = g.get_diff_params()
    g.write_state(start)
    th = torch.tensor(theta0, dtype=torch.float64, requires_grad=True)
    traj = adjoint.SoupWindow.apply(th, g, steps, every)
    d = traj.double() - traj[0:1].double()
    d = d - torch.round(d / box) * box
    loss = (d * w.cuda()).sum()
    loss.backward()
    grad = th.grad.numpy().copy()
    g.dispose()
    win = tr.SoupWindow64(cfg, start, steps, device="cuda")
    loss64, grad64 = win.loss_and_grad(theta0, w)
    fd = _fd(theta0, lambda t: win.loss(t, w))
    # the functional is a signed sum of 2 million terms that cancels to a small value, so the FP32
    # window's value is held to its terms' own scale (their root sum of squares), not to the sum's
    scale = float(torch.sqrt(((d.detach() * w.cuda()) ** 2).sum()))
    assert abs(float(loss.detach()) - loss64) <= 1e-4 * scale, (float(loss.detach()), loss64, scale)
    _check("displacement functional, 20 steps, 32,768 beads", grad, grad64, fd)


def test_thickness_gradient_over_50_steps_at_full_size(patch):
    cfg, start = patch
    steps, every = 50, 10
    p = start["positions"].reshape(-1, 4)
    slots = start["bond_slots"].reshape(-1, 3)
    heads = torch.tensor(np.nonzero(p[:, 3] == 1)[0], device="cuda")
    tails = torch.tensor(np.nonzero((p[:, 3] == 0) & np.any(slots != tr.NONE, axis=1))[0], device="cuda")
    fn = lambda frames: adjoint.thickness_proxy(frames, heads, tails, float(cfg.box[2]))
    g = SoupSystem(cfg, start)
    theta0 = g.get_diff_params()
    g.write_state(start)
    th = torch.tensor(theta0, dtype=torch.float64, requires_grad=True)
    v = fn(adjoint.SoupWindow.apply(th, g, steps, every).double())
    v.backward()
    grad = th.grad.numpy().copy()
    g.dispose()
    win = tr.SoupWindow64(cfg, start, steps, device="cuda")
    v64, grad64 = win.observable_and_grad(theta0, fn)
    fd = _fd(theta0, lambda t: win.observable(t, fn))
    assert float(v.detach()) == pytest.approx(v64, rel=1e-5)
    _check("thickness proxy, 50 steps, 32,768 beads", grad, grad64, fd)

"""Gradients of a loss over a window of the soup step with respect to force-field parameters.

The library runs the window forward (`soup_diff_forward`: the force + Langevin step with bond Monte
Carlo and the constant-pH sweep held off, checkpoints every k steps) and backward
(`soup_diff_backward`: the discrete adjoint of the step, recomputing each segment from its
checkpoint).  `SoupWindow` wraps the pair as a torch.autograd.Function: its input is the parameter
vector, its output the trajectory (steps + 1 frames of x, y, z, kind in original order, on the
GPU), so any loss written in torch on the trajectory differentiates back to the parameters:

    theta = torch.tensor(system.get_diff_params(), dtype=torch.float64, requires_grad=True)
    traj = SoupWindow.apply(theta, system, 200, 20)
    loss = thickness_proxy(traj, heads, tails, box_z)
    loss.backward()          # theta.grad

The parameters (PARAM_NAMES) are the class-pair attraction depths, k_fene, k_bend and kappa.  A
call starts from the system's current state and leaves it at the window's end.  There is no
counterpart in the reference, which runs the step forward only.  In a fixed box the area per lipid
(Lx Ly / (N/2)) is a constant, so the bilayer's differentiable observable here is the thickness
proxy; any other torch loss on the trajectory works the same way.
"""
import numpy as np
import torch

from . import _abi

PARAM_NAMES = ["A_apolar_apolar", "A_apolar_polar", "A_apolar_solvent", "A_polar_polar", "A_polar_solvent",
               "A_solvent_solvent", "k_fene", "k_bend", "kappa"]


class SoupWindow(torch.autograd.Function):
    """apply(theta, system, steps, checkpoint_every, frame_stride=1): the trajectory's frames at steps
    0, frame_stride, .., steps (steps / frame_stride + 1 of them)."""
    @staticmethod
    def forward(ctx, theta, system, steps, checkpoint_every, frame_stride=1):
        if int(frame_stride) < 1 or int(steps) % int(frame_stride):
            raise ValueError("frame_stride must be positive and divide steps")
        th = theta.detach().cpu().double().numpy()
        if not np.array_equal(th, system.get_diff_params()):
            system.set_diff_params(th)
        traj = torch.empty((int(steps) // int(frame_stride) + 1, system.n, 4), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        system.diff_forward(steps, checkpoint_every, traj.data_ptr(), frame_stride)
        torch.cuda.synchronize()
        ctx.system = system
        ctx.theta_dtype, ctx.theta_device = theta.dtype, theta.device
        return traj

    @staticmethod
    def backward(ctx, grad_traj):
        g = grad_traj.contiguous().float()
        torch.cuda.synchronize()
        grad = ctx.system.diff_backward(g.data_ptr())
        torch.cuda.synchronize()
        return torch.as_tensor(grad, dtype=ctx.theta_dtype, device=ctx.theta_device), None, None, None, None


def window(system, theta, steps, checkpoint_every, frame_stride=1):
    """traj = SoupWindow.apply(theta, system, steps, checkpoint_every, frame_stride)."""
    return SoupWindow.apply(theta, system, steps, checkpoint_every, frame_stride)


def thickness_proxy(traj, heads, tails, box_z):
    """A differentiable bilayer thickness for a flat bilayer normal to z: twice the mean distance of
    the heads from the mid-plane (the mean z of the amphiphile beads), averaged over the frames.
    (metrics.ts's peak-to-peak thickness is a histogram argmax, which has no gradient.)  Positions
    are unwrapped in z around the first frame's mid-plane so a bilayer near a face stays whole."""
    z = traj[:, :, 2]
    members = torch.cat([heads, tails])
    ref = z[0, members].mean()
    zu = z - torch.round((z - ref) / box_z) * box_z
    mid = zu[:, members].mean(dim=1, keepdim=True)
    return 2.0 * (zu[:, heads] - mid).abs().mean()

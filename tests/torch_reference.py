"""An FP64 restatement of the soup window (force + Langevin step) in torch, differentiated by torch
autograd: the reference gradient the library's hand-written adjoint is checked against.  Test
infrastructure only; it runs on whatever device the test gives it.

The step (soup/wgsl/step.wgsl:96-142): v += h F; x += dt v; F = F(x); w = v + h F;
v = (1 - gamma dt) w + sqrt(2 gamma kT dt) xi, with xi replayed from each particle's thermostat
state exactly as the kernel draws it (pcgSoup, step.wgsl:18-23; Box-Muller on two uniforms per axis),
so the FP64 window follows the same noise as the FP32 one.  Positions are kept unwrapped (the
minimum image is taken in the force), which leaves the loss on displacements unchanged.

Force terms, each central, F_i = sum_j s(r) d with d = mi(x_i - x_j):
  WCA        s = 24 eps (2 (b/r)^12 - (b/r)^6) / r^2            r < 2^(1/6) b, b = sigma (r_i + r_j) / 2
             (soup/wgsl/pair.wgsl:168-204)
  attraction s = -(A[c_i][c_j] + acid) amp sin(2 (r - rc) k) / r  rc <= r <= rc + wc
             (amp = eps pi / (2 wc), k = pi / (2 wc), rc = 2^(1/6) b_tt; acid between a charged and an
             uncharged polar bead)
  screened   s = q_i q_j (A_es e^{-kappa r} (1/r^2 + kappa/r) - fc(kappa)) / r   r < rc_es, with
             fc(kappa) the same bracket at rc_es (soup/wgsl/electrostatics.wgsl:65-99 and its far half)
  FENE       s = -k_fene / (1 - r^2 / r_inf^2)                   bonded pairs  (step.wgsl:152-193)
  bend       s = -k_bend (r - r_bend) / r                        1-3 pairs of a chain
Nonbonded pairs are selected at every force evaluation (every pair within the longest reach of a
term, by minimum image), outside the autograd graph: every term is zero beyond its reach, so the
selection changes no value and no derivative.
"""
import math

import numpy as np
import torch

DEPTH_PAIRS = [(0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)]
NONE = 0xFFFFFFFF


def _pcg(v):
    """pcgSoup on a uint64 array holding uint32 values."""
    state = (v * 747796405 + 2891336453) & 0xFFFFFFFF
    word = (((state >> ((state >> 28) + 4)) ^ state) * 277803737) & 0xFFFFFFFF
    return (word >> 22) ^ word


def thermostat_noise(rng, steps):
    """xi[t] (steps, n, 3) in FP64 and the final states, drawn as the kick-thermostat kernel draws
    them: per axis two hashes, u1 = max(f32(s) / 2^32, 1e-7), u2 = f32(s) / 2^32,
    xi = sqrt(-2 ln u1) cos(2 pi u2)."""
    st = np.asarray(rng, np.uint64).copy()
    out = np.empty((steps, len(st), 3), np.float64)
    two_pi = float(np.float32(6.28318531))
    for t in range(steps):
        for a in range(3):
            st = _pcg(st)
            u1 = np.maximum(st.astype(np.float32) / np.float32(4294967296.0), np.float32(1e-7)).astype(np.float64)
            st = _pcg(st)
            u2 = (st.astype(np.float32) / np.float32(4294967296.0)).astype(np.float64)
            out[t, :, a] = np.sqrt(-2.0 * np.log(u1)) * np.cos(two_pi * u2)
    return out, st.astype(np.uint32)


def theta_of(cfg):
    """The differentiable parameters as the library orders them: the six class-pair depths, k_fene,
    k_bend, kappa."""
    return np.array([cfg.attr_scale[a][b] for a, b in DEPTH_PAIRS] + [cfg.k_fene, cfg.k_bend, cfg.es_kappa],
                    np.float64)


def _bonded_pairs(slots, n):
    s = np.asarray(slots).reshape(n, 3).astype(np.int64)
    bonds = set()
    for i in range(n):
        for j in s[i]:
            if j != NONE:
                bonds.add((min(i, int(j)), max(i, int(j))))
    nb = [[] for _ in range(n)]
    for i, j in bonds:
        nb[i].append(j)
        nb[j].append(i)
    bends = set()
    for m in range(n):
        for a in nb[m]:
            for c in nb[m]:
                if a < c:
                    bends.add((a, c))
    as_arr = lambda x: np.array(sorted(x), np.int64).reshape(-1, 2)
    return as_arr(bonds), as_arr(bends)


class SoupWindow64:
    """The window on one system's start state; `loss_and_grad(theta, w)` and `loss(theta, w)` for the
    loss sum_t w_t . (x_t - x_0) over frames 1..steps."""

    def __init__(self, cfg, start, steps, device="cuda"):
        if float(cfg.wall_radius) > 0:
            raise ValueError("the FP64 window has no wall term")
        self.cfg, self.steps, self.dev = cfg, int(steps), device
        f64 = torch.float64
        p = np.asarray(start["positions"], np.float64).reshape(-1, 4)
        n = self.n = len(p)
        if "frozen" in start and np.any(np.asarray(start["frozen"]) != 0):
            raise ValueError("the FP64 window has no frozen particles")
        if "center_link" in start and np.any(np.asarray(start["center_link"]) != NONE):
            raise ValueError("the FP64 window has no centre links")
        self.x0 = torch.tensor(p[:, :3], dtype=f64, device=device)
        self.v0 = torch.tensor(np.asarray(start["velocities"], np.float64).reshape(n, 4)[:, :3], dtype=f64, device=device)
        q = torch.tensor(np.asarray(start["charges"], np.float64), dtype=f64, device=device)
        kinds = torch.tensor(p[:, 3].astype(np.int64), device=device)
        self.box = torch.tensor(list(cfg.box), dtype=f64, device=device)
        radius = torch.tensor([cfg.radius[k] for k in range(8)], dtype=f64, device=device)
        cls = torch.tensor([cfg.kind_class[k] & 3 for k in range(8)], dtype=torch.int64, device=device)
        noise, _ = thermostat_noise(start["thermo_rng"], self.steps)
        self.noise = torch.tensor(noise, dtype=f64, device=device)

        c6 = float(np.float32(2.0 ** float(np.float32(1.0 / 6.0))))
        self.rc_attr = float(np.float32(c6 * float(cfg.b_tt)))
        self.wc = float(cfg.wc)
        self.eps = float(cfg.epsilon)
        self.amp = self.eps * math.pi / (2 * self.wc)
        self.katt = math.pi / (2 * self.wc)
        self.rc_es = float(cfg.es_cutoff)
        self.a_es = float(cfg.es_coeff_a) if cfg.es_enabled else 0.0
        self.base_attr = torch.tensor([[cfg.attr_scale[a][b] for b in range(4)] for a in range(4)], dtype=f64,
                                      device=device)
        self.reach = max(self.rc_attr + self.wc, c6 * float(cfg.sigma) * float(radius.max()))
        self.c6, self.q, self.kinds, self.radius, self.cls = c6, q, kinds, radius, cls
        bonds, bends = _bonded_pairs(start["bond_slots"], n)
        t = lambda a: torch.tensor(a, device=device)
        self.bi, self.bj = t(bonds[:, 0]), t(bonds[:, 1])
        self.ci3, self.cj3 = t(bends[:, 0]), t(bends[:, 1])

    def _mi(self, d):
        return d - torch.round(d / self.box).detach() * self.box

    def _pairs_within(self, x, reach, q, reach_es, rows=256):
        """(i, j), i < j, of every pair within reach, or within reach_es when both are charged."""
        out_i, out_j = [], []
        for r0 in range(0, self.n, rows):
            xs = x[r0:r0 + rows]
            r = self._mi(xs[:, None, :] - x[None, :, :]).norm(dim=-1)
            qs = q[r0:r0 + rows]
            near = (r < reach) | ((qs[:, None] != 0) & (q[None, :] != 0) & (r < reach_es))
            i, j = torch.triu(near, diagonal=1 + r0).nonzero(as_tuple=True)
            out_i.append(i + r0)
            out_j.append(j)
        return torch.cat(out_i), torch.cat(out_j)

    def _depths(self, theta):
        A = self.base_attr.clone()
        for k, (a, b) in enumerate(DEPTH_PAIRS):
            A[a, b] = theta[k]
            A[b, a] = theta[k]
        return A

    def force(self, x, theta):
        A = self._depths(theta)
        kf, kb, kap = theta[6], theta[7], theta[8]
        with torch.no_grad():       # beyond these every term is zero, so the selection is exact
            ii, jj = self._pairs_within(x.detach(), self.reach, self.q, self.rc_es)
        ki, kj = self.kinds[ii], self.kinds[jj]
        b = float(self.cfg.sigma) * (self.radius[ki] + self.radius[kj]) / 2
        ci, cj = self.cls[ki], self.cls[kj]
        qi, qj = self.q[ii], self.q[jj]
        qq = qi * qj
        acid = float(self.cfg.acid_soap_scale) * ((ci == 1) & (cj == 1) & ((qi != 0) != (qj != 0))).to(x.dtype)
        d = self._mi(x[ii] - x[jj])
        r = d.norm(dim=-1)
        zero = torch.zeros_like(r)
        sb = (b / r) ** 6
        s = torch.where(r < self.c6 * b, 24 * self.eps * (2 * sb * sb - sb) / r ** 2, zero)
        depth = A[ci, cj] + acid
        on = (r >= self.rc_attr) & (r <= self.rc_attr + self.wc)
        s = s - torch.where(on, depth * self.amp * torch.sin(2 * (r - self.rc_attr) * self.katt) / r, zero)
        rc = self.rc_es
        fc = self.a_es * torch.exp(-kap * rc) * (1 / rc ** 2 + kap / rc)
        on = (qq != 0) & (r < rc)
        s = s + torch.where(on, qq * (self.a_es * torch.exp(-kap * r) * (1 / r ** 2 + kap / r) - fc) / r, zero)
        f = torch.zeros_like(x).index_add(0, ii, s[:, None] * d).index_add(0, jj, -s[:, None] * d)
        db = self._mi(x[self.bi] - x[self.bj])
        rb = db.norm(dim=-1)
        sf = -kf / (1 - rb ** 2 / float(self.cfg.r_inf) ** 2)
        f = f.index_add(0, self.bi, sf[:, None] * db).index_add(0, self.bj, -sf[:, None] * db)
        dc = self._mi(x[self.ci3] - x[self.cj3])
        rc3 = dc.norm(dim=-1)
        sc = -kb * (rc3 - float(self.cfg.r_bend)) / rc3
        return f.index_add(0, self.ci3, sc[:, None] * dc).index_add(0, self.cj3, -sc[:, None] * dc)

    def run(self, theta, w=None, frames=False, x0=None, v0=None):
        """(loss, frames or None): the window at theta (a float64 tensor on the device) from (x0, v0),
        the start state's unless given."""
        cfg = self.cfg
        dt, h = float(cfg.dt), 0.5 * float(cfg.dt)
        a = 1.0 - float(cfg.gamma) * dt
        sv = math.sqrt(2.0 * float(cfg.gamma) * float(cfg.kT) * dt)
        x = self.x0 if x0 is None else x0
        v = self.v0 if v0 is None else v0
        x_start = x
        f = self.force(x, theta)
        loss = torch.zeros((), dtype=torch.float64, device=self.dev)
        out = [x] if frames else None
        for t in range(self.steps):
            v = v + h * f
            x = x + dt * v
            f = self.force(x, theta)
            v = a * (v + h * f) + sv * self.noise[t]
            if w is not None:
                loss = loss + (w[t + 1, :, :3] * (x - x_start)).sum()
            if frames:
                out.append(x)
        return loss, (torch.stack(out) if frames else None)

    def loss_and_grad(self, theta0, w):
        theta = torch.tensor(np.asarray(theta0, np.float64), dtype=torch.float64, device=self.dev, requires_grad=True)
        loss, _ = self.run(theta, w.to(self.dev, torch.float64))
        loss.backward()
        return float(loss.detach()), theta.grad.detach().cpu().numpy()

    def start_gradients(self, theta0, w):
        """(dloss/dx0, dloss/dv0) as (n, 3) FP64 arrays."""
        theta = torch.tensor(np.asarray(theta0, np.float64), dtype=torch.float64, device=self.dev)
        x0 = self.x0.clone().requires_grad_(True)
        v0 = self.v0.clone().requires_grad_(True)
        loss, _ = self.run(theta, w.to(self.dev, torch.float64), x0=x0, v0=v0)
        loss.backward()
        return x0.grad.detach().cpu().numpy(), v0.grad.detach().cpu().numpy()

    def observable_and_grad(self, theta0, fn):
        """(fn(frames), its gradient in theta) for a torch function of the (steps + 1, n, 3) frames."""
        theta = torch.tensor(np.asarray(theta0, np.float64), dtype=torch.float64, device=self.dev, requires_grad=True)
        _, frames = self.run(theta, None, frames=True)
        value = fn(frames)
        value.backward()
        return float(value.detach()), theta.grad.detach().cpu().numpy()

    def observable(self, theta0, fn):
        with torch.no_grad():
            theta = torch.tensor(np.asarray(theta0, np.float64), dtype=torch.float64, device=self.dev)
            return float(fn(self.run(theta, None, frames=True)[1]))

    def loss(self, theta0, w):
        with torch.no_grad():
            theta = torch.tensor(np.asarray(theta0, np.float64), dtype=torch.float64, device=self.dev)
            loss, _ = self.run(theta, w.to(self.dev, torch.float64))
        return float(loss)

    def frames(self, theta0):
        with torch.no_grad():
            theta = torch.tensor(np.asarray(theta0, np.float64), dtype=torch.float64, device=self.dev)
            return self.run(theta, None, frames=True)[1]

#!/usr/bin/env python
"""Benchmark: particle-steps/s of the soup MD step at 483,268 beads on B200.

Workload (the reference's full-campaign shape, box 76 sigma, its B76 census C 55,988 / O 18,659 /
H 55,988 / M 1,452 / W 351,181): seeded fresh lattice + 50-iteration cold-start relax (untimed),
pH 7 constant-pH Monte Carlo every 10 steps, I = 0.01 M long-range Debye-Hueckel (rc_es 15.2 sigma),
Verlet rebuild on half-skin drift, bond Monte Carlo every 20 steps.  Inputs (state + lists,
> 400 MB) are larger than the 126 MB L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cuda|reference]

One JSON line on rank 0.  N > 1 runs N independent replicas (one per GPU, weak scaling; the single
483k-bead system fits one GPU and is not split).  --impl reference times the CPU oracle (the reference's step
restated in C++, OpenMP over the host cores) on the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

METRIC = "particle-steps/s at 483k beads, plain vs batched, at <=1e-5 force err"
SKIN = 1.0                 # the Verlet skin of the plain workload, both arms (rebuilt on half-skin drift)
RELAX_ITERATIONS = 50      # cold-start relax of the fresh lattice, both arms (untimed)
E2E_MIN_STEPS = 200        # the end-to-end sample covers at least one analysis period
UNIT = "particle-steps/s"
# the reference's published full-campaign rate at this size (87.2 ms/step, Apple GPU via WebGPU)
PUBLISHED = 483268 / 0.0872
FORCE_KERNEL = "k_force (list pair force + bonded terms)"
CENSUS = {"C": 55988, "O": 18659, "H": 55988, "M": 1452, "W": 351181}


def workload_opts(cfgm, seed=19, skin=1.0, sweep_every=10, scale=1.0):
    """scale < 1 shrinks the census and the box volume by the same factor (profiling captures)."""
    start = {k: int(round(v * scale)) for k, v in CENSUS.items()}
    side = 76.0 * scale ** (1.0 / 3.0)
    return cfgm.SoupOptions(box=[side, side, side], seed=seed, kT=1.1, start=start,
                            electrostatics={"enabled": True, "pH": 7.0, "ionicStrengthMolar": 0.01},
                            skin=skin, rebuild_on_drift=True, sweep_every=sweep_every, chunk_steps=sweep_every)


def workload_config(skin, relax, n):
    """The `config` of both arms' lines: the same keys and values for the same workload."""
    return {"workload": workload_name(skin), "beads": int(n), "skin": float(skin), "relax_iterations": int(relax),
            "l2": "inputs larger than L2 (state + lists ~2.5 GB vs 126 MB), no flush"}


def workload_name(skin):
    return (f"campaign shape: 483,268 beads, 76 sigma box, pH 7 MC every 10 steps, I 0.01 M (rc_es 15.2), "
            f"bonds every 20, Verlet skin {skin} rebuilt on half-skin drift, fresh lattice relaxed "
            f"{RELAX_ITERATIONS} iterations")


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) > 8 for i in range(4) if "Active" in r[5 + i]
                          and "Not" not in r[5 + i]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            p = json.load(fh)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def rank_seeds(rank):
    """Replicas only: every rank runs its own copy of the plain workload, seeded apart; the batched
    replica set is one set (seed 7) split across the ranks (replica_share)."""
    return 19 + rank, 7


def replica_share(sizes, ws, rank):
    """Whole replicas to ranks, balanced by beads: largest first, each to the least loaded rank (ties
    to the lower rank).  Returns the replica indices of `rank`, ascending."""
    load = [0] * ws
    own = [[] for _ in range(ws)]
    for i in sorted(range(len(sizes)), key=lambda k: (-sizes[k], k)):
        r = min(range(ws), key=lambda q: (load[q], q))
        load[r] += sizes[i]
        own[r].append(i)
    return sorted(own[rank])


def max_over_ranks(x, dist, device):
    """The largest per-rank value (a step time) over all ranks; x itself on one rank."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x, dist, device):
    """The sum of a per-rank value over all ranks; x itself on one rank."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def aggregate_rate(ws, units_per_rank, steps, ms_max):
    """Whole-job particle-steps/s: every rank's units over the slowest rank's time."""
    return ws * units_per_rank * steps / (ms_max / 1e3)


def cpu_sample(pkg, ob, cfg, state, budget_s=12.0, max_steps=40):
    """Time the CPU oracle (all host threads) on a bounded number of steps of the same workload."""
    from protocell_genesis_b200 import _abi
    o = ob.OracleSystem(_abi, cfg, state)
    threads = ob.lib(_abi).oracle_threads()
    t0 = time.perf_counter()
    o.step(1)
    t1 = time.perf_counter()
    per = t1 - t0
    n = int(max(1, min(max_steps, budget_s / max(per, 1e-6))))
    t0 = time.perf_counter()
    o.step(n)
    dt = time.perf_counter() - t0
    o.close()
    return {"value": cfg.n * n / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{n} steps of the same 483,268-bead workload from the relaxed start (after 1 warm-up step), "
                      f"C++ oracle FP32 path, OpenMP {threads} threads"}


def run_reference(args):
    ws, rank, _ = dist_init()
    if rank != 0:
        return
    import __graft_entry__ as ge
    pkg = ge._package()
    import oracle_binding as ob
    from protocell_genesis_b200 import _abi, config as cfgm
    cfg = cfgm.resolve(workload_opts(cfgm, skin=args.skin))
    o = ob.OracleSystem(_abi, cfg)
    o.relax(args.relax, 0.1)
    threads = ob.lib(_abi).oracle_threads()
    o.step(max(1, min(args.warmup, 2)))
    t0 = time.perf_counter()
    o.step(1)
    per = time.perf_counter() - t0
    k = int(max(1, min(args.steps, args.ref_budget / max(per, 1e-6))))
    t0 = time.perf_counter()
    o.step(k)
    dt = time.perf_counter() - t0
    v = cfg.n * k / dt
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws, "steps": k,
            "warmup": args.warmup, "ms_per_step": 1e3 * dt / k, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": v / PUBLISHED, "dtype": "f32", "data": "synthetic",
            "config": workload_config(args.skin, args.relax, cfg.n),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{k} of the requested {args.steps} steps (bounded to ~{args.ref_budget:.0f} s), "
                                       f"C++ restatement of the reference step, OpenMP {threads} threads"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def batched_configs(cfgm, seed, replicas):
    """Uneven replicas: box L ~ U[29, 53] sigma at total density 0.80, 15% of the beads in
    preassembled five-bead amphiphiles (head O + four C), the rest water; pH ~ U[5, 9], ionic
    strength log-uniform in [0.001, 0.1] M; the same step schedule as the single system."""
    import numpy as np
    rng = np.random.default_rng(seed)
    out = []
    for r in range(replicas):
        side = float(rng.uniform(29.0, 53.0))
        n = int(round(0.80 * side ** 3))
        na = int(0.15 * n) // 5
        opts = cfgm.SoupOptions(box=[side] * 3, seed=int(seed * 1000 + r), kT=1.1,
                                start={"C": 4 * na, "O": na, "H": 0, "M": 0, "W": n - 5 * na},
                                electrostatics={"enabled": True, "pH": float(rng.uniform(5.0, 9.0)),
                                                "ionicStrengthMolar": float(10.0 ** rng.uniform(-3.0, -1.0))},
                                skin=1.0, rebuild_on_drift=True, sweep_every=10, chunk_steps=10)
        out.append((cfgm.resolve(opts), na, int(rng.integers(1 << 31))))
    return out


def amphiphile_state(L, cfg, na, seed):
    """Straight five-bead amphiphiles at random centres and orientations (head, then c1..c4 at
    0.95 sigma spacing) and water at uniform random positions; bond slots as the reference lays a
    chain out (head[0] = c1; c1[2] = head, c1[0] = c2; c2[0] = c1, c2[1] = c3; ...).  Velocities and
    the per-particle RNG seeds come from the library's fresh-state generator for this config."""
    import ctypes as C
    import numpy as np
    n = cfg.n
    side = cfg.box[0]
    rng = np.random.default_rng(seed)
    pos = np.zeros((n, 4), np.float32)
    vel = np.zeros(n * 4, np.float32)
    fr = np.zeros(n, np.uint32); br = np.zeros(n, np.uint32); tr = np.zeros(n, np.uint32)
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    L.soup_fresh_state(C.byref(cfg), p(pos), p(vel), p(fr), p(br), p(tr))
    kind_c, kind_o, kind_w = 0.0, 1.0, 4.0
    centres = rng.uniform(0.0, side, (na, 3))
    u = rng.normal(size=(na, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    chain = centres[:, None, :] + ((np.arange(5) - 2.0) * 0.95)[None, :, None] * u[:, None, :]
    pos[:5 * na, :3] = np.mod(chain.reshape(-1, 3), side)
    pos[:5 * na, 3] = np.tile([kind_o, kind_c, kind_c, kind_c, kind_c], na)
    pos[5 * na:, :3] = rng.uniform(0.0, side, (n - 5 * na, 3))
    pos[5 * na:, 3] = kind_w
    none = 0xFFFFFFFF
    slots = np.full((n, 3), none, np.uint32)
    b = 5 * np.arange(na, dtype=np.uint32)
    slots[b, 0] = b + 1
    slots[b + 1, 2] = b; slots[b + 1, 0] = b + 2
    slots[b + 2, 0] = b + 1; slots[b + 2, 1] = b + 3
    slots[b + 3, 0] = b + 2; slots[b + 3, 1] = b + 4
    slots[b + 4, 0] = b + 3
    pos = pos.reshape(-1)
    charges = np.zeros(n, np.float32)
    prng = C.c_uint32(0)
    L.soup_initial_charges(C.byref(cfg), p(pos), p(charges), C.byref(prng))
    return dict(positions=pos, velocities=vel, bond_slots=slots.reshape(-1), charges=charges, frozen=fr,
                bond_rng=br, thermo_rng=tr)


def bilayer_patch(L, cfgm, lx=32.0, lz=40.0, per_side=32, seed=11, kT=1.0, ph=9.0, ionic=0.01):
    """A preassembled flat bilayer: per_side^2 five-bead amphiphiles per leaflet on a square lattice
    spanning lx x lx, heads outward, tails inward, the mid-plane at lz / 2; water at uniform random
    positions outside the slab |z - lz/2| < 5, to a total density of 0.80.  Bond slots as the
    reference lays a chain out (see amphiphile_state).  Returns (config, state)."""
    import ctypes as C
    import numpy as np
    rng = np.random.default_rng(seed)
    na = 2 * per_side * per_side
    n = int(round(0.80 * lx * lx * lz))
    nw = n - 5 * na
    opts = cfgm.SoupOptions(box=[lx, lx, lz], seed=seed, kT=kT, start={"C": 4 * na, "O": na, "H": 0, "M": 0, "W": nw},
                            electrostatics={"enabled": True, "pH": ph, "ionicStrengthMolar": ionic},
                            skin=1.0, rebuild_on_drift=True)
    cfg = cfgm.resolve(opts)
    pos = np.zeros((n, 4), np.float32)
    vel = np.zeros(n * 4, np.float32)
    fr = np.zeros(n, np.uint32); br = np.zeros(n, np.uint32); tr = np.zeros(n, np.uint32)
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    L.soup_fresh_state(C.byref(cfg), p(pos), p(vel), p(fr), p(br), p(tr))
    a = lx / per_side
    gx, gy = np.meshgrid((np.arange(per_side) + 0.5) * a, (np.arange(per_side) + 0.5) * a, indexing="ij")
    mid = lz / 2
    k = 0
    for side in (1.0, -1.0):
        for x, y in zip(gx.reshape(-1), gy.reshape(-1)):
            jitter = rng.normal(scale=0.05, size=2)
            for b in range(5):   # head at 4.5 from the mid-plane, c1..c4 towards it
                pos[k * 5 + b, :3] = (x + jitter[0], y + jitter[1], mid + side * (4.5 - 0.95 * b))
            pos[k * 5:k * 5 + 5, 3] = (1.0, 0.0, 0.0, 0.0, 0.0)
            k += 1
    w = []
    while len(w) < nw:
        cand = rng.uniform((0, 0, 0), (lx, lx, lz), size=(2 * nw, 3))
        cand = cand[np.abs(cand[:, 2] - mid) > 5.0]
        w.extend(cand.tolist())
    pos[5 * na:, :3] = np.array(w[:nw], np.float32)
    pos[5 * na:, 3] = 4.0
    none = 0xFFFFFFFF
    slots = np.full((n, 3), none, np.uint32)
    b = 5 * np.arange(na, dtype=np.uint32)
    slots[b, 0] = b + 1
    slots[b + 1, 2] = b; slots[b + 1, 0] = b + 2
    slots[b + 2, 0] = b + 1; slots[b + 2, 1] = b + 3
    slots[b + 3, 0] = b + 2; slots[b + 3, 1] = b + 4
    slots[b + 4, 0] = b + 3
    pos = pos.reshape(-1)
    charges = np.zeros(n, np.float32)
    prng = C.c_uint32(0)
    L.soup_initial_charges(C.byref(cfg), p(pos), p(charges), C.byref(prng))
    state = dict(positions=pos, velocities=vel, bond_slots=slots.reshape(-1), charges=charges, frozen=fr,
                 bond_rng=br, thermo_rng=tr)
    return cfg, state


def parcel_configs(cfgm, seed, replicas, n=60000, density=1.1):
    """Finite water parcels: n beads inside a neutral spherical wall (stiffness 100) at the reference's
    confined density, 12% of the beads in five-bead amphiphiles, the rest water; pH ~ U[6, 8] with
    the heads' initial charges from initialCharges, I = 0.01 M for every replica (one Debye kappa,
    which the batched gradient window needs)."""
    import math
    import numpy as np
    rng = np.random.default_rng(seed)
    radius = (n / density / (4.0 / 3.0 * math.pi)) ** (1.0 / 3.0)
    side = 2.0 * radius + 34.0   # the face clearance must exceed the head-list range (16.2 sigma at 0.01 M)
    na = int(0.12 * n) // 5
    out = []
    for r in range(replicas):
        opts = cfgm.SoupOptions(box=[side] * 3, seed=int(seed * 1000 + r), kT=1.1,
                                start={"C": 4 * na, "O": na, "H": 0, "M": 0, "W": n - 5 * na},
                                electrostatics={"enabled": True, "pH": float(rng.uniform(6.0, 8.0)),
                                                "ionicStrengthMolar": 0.01},
                                confine={"radiusSigma": radius, "stiffness": 100.0},
                                skin=1.0, rebuild_on_drift=True, sweep_every=10, chunk_steps=10,
                                es_list_capacity=na)   # a parcel is smaller than the head-list range
        out.append((cfgm.resolve(opts), na, int(rng.integers(1 << 31)), radius))
    return out


def parcel_state(L, cfg, na, seed, radius):
    """amphiphile_state inside the parcel: chain centres uniform in the ball of radius - 3, water
    uniform in the ball of radius - 0.5, about the box centre."""
    import numpy as np
    st = amphiphile_state(L, cfg, na, seed)
    rng = np.random.default_rng(seed + 1)
    centre = np.array(list(cfg.box), np.float64) / 2.0

    def ball(k, rad):
        out = np.empty((0, 3))
        while len(out) < k:
            c = rng.uniform(-rad, rad, (2 * k + 16, 3))
            out = np.concatenate([out, c[np.linalg.norm(c, axis=1) < rad]])
        return out[:k]

    pos = st["positions"].reshape(-1, 4)
    u = rng.normal(size=(na, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    chain = ball(na, radius - 3.0)[:, None, :] + ((np.arange(5) - 2.0) * 0.95)[None, :, None] * u[:, None, :]
    pos[:5 * na, :3] = (chain.reshape(-1, 3) + centre).astype(np.float32)
    pos[5 * na:, :3] = (ball(cfg.n - 5 * na, radius - 0.5) + centre).astype(np.float32)
    st["positions"] = pos.reshape(-1)
    return st


def run_gradient_batched(args, pkg, L, torch):
    """Batched replicas + adjoint: 16 finite water parcels of 60k beads stepped as one batch; forward
    + adjoint of the encapsulated-water proxy over a window, with respect to the nine parameters
    (the head-water depth A_polar_solvent among them)."""
    import numpy as np
    from protocell_genesis_b200 import adjoint, config as cfgm
    items = parcel_configs(cfgm, seed=3, replicas=args.parcel_replicas)
    cfgs, states = [], []
    for cfg, na, sd, radius in items:
        st = parcel_state(L, cfg, na, sd, radius)
        s_ = pkg.SoupSystem(cfg, st)
        s_.relax_cold_start(args.aux_relax, 0.1)
        st["positions"] = s_.particles()
        s_.dispose()
        cfgs.append(cfg)
        states.append(st)
    batch = pkg.SoupBatch(cfgs, states)
    batch.step(20)
    N = batch.n
    kinds = np.concatenate([st["positions"].reshape(-1, 4)[:, 3] for st in states])
    rep = np.concatenate([np.full(c.n, r) for r, c in enumerate(cfgs)])
    heads = torch.tensor(kinds == 1.0, device="cuda")
    water = torch.tensor(kinds == 4.0, device="cuda")
    rep_t = torch.tensor(rep, device="cuda")
    R = len(cfgs)
    centre = torch.tensor(list(cfgs[0].box), dtype=torch.float64, device="cuda") / 2.0
    nh = torch.zeros(R, dtype=torch.float64, device="cuda").index_add_(0, rep_t[heads], torch.ones(int(heads.sum()), dtype=torch.float64, device="cuda"))

    def encapsulated(traj):
        # per replica and frame: the heads' mean distance from the parcel centre; the loss counts the
        # water inside it smoothly (logistic of width 0.5 sigma), summed over replicas, averaged over frames
        rad = (traj[:, :, :3].double() - centre).norm(dim=-1)
        shell = torch.zeros((traj.shape[0], R), dtype=torch.float64, device="cuda")
        shell = shell.index_add(1, rep_t[heads], rad[:, heads]) / nh
        inside = torch.sigmoid((shell[:, rep_t[water]] - rad[:, water]) / 0.5)
        return inside.sum(dim=1).mean()

    # config 5's window: 2,000 steps, checkpoints every 100 (the replay segments), the loss on every
    # 20th frame (the frame stride keeps 101 frames of the batch instead of 2,001)
    steps, every, stride = args.parcel_steps, args.parcel_checkpoint, args.parcel_stride
    stream = torch.cuda.ExternalStream(L.soup_stream(batch.replicas[0]._h))
    theta0 = batch.get_diff_params()

    def window(n_steps):
        th = torch.tensor(theta0, dtype=torch.float64, requires_grad=True)
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        torch.cuda.synchronize()
        e0.record(stream)
        traj = adjoint.SoupWindow.apply(th, batch, n_steps, every, stride)
        e1.record(stream)
        loss = encapsulated(traj)
        loss.backward()
        e2.record(stream)
        torch.cuda.synchronize()
        return float(loss.detach()), th.grad.numpy(), e0.elapsed_time(e1), e1.elapsed_time(e2)

    # untimed (scratch is allocated on first use); its gradient is the short window's, for scale
    loss_short, grad_short, _, _ = window(every)
    fwd, bwd = [], []
    for _ in range(args.parcel_windows):
        loss, grad, f_ms, b_ms = window(steps)
        fwd.append(f_ms)
        bwd.append(b_ms)
    batch.dispose()
    total = (sum(fwd) + sum(bwd)) / len(fwd)
    return {"value": N * steps / (total / 1e3), "unit": "particle-steps/s (forward + adjoint)", "replicas": R,
            "beads": N, "window_steps": steps, "checkpoint_every": every, "frame_stride": stride,
            "frames_kept": steps // stride + 1, "windows": len(fwd),
            "ms_per_window": total, "forward_ms": sum(fwd) / len(fwd), "backward_ms": sum(bwd) / len(bwd),
            "loss": "encapsulated-water proxy", "value_of_loss": loss,
            "theta": list(adjoint.PARAM_NAMES), "grad": [float(x) for x in grad],
            "short_window": {"steps": every, "value_of_loss": loss_short, "grad": [float(x) for x in grad_short]},
            "note": "the parcels are a chaotic fluid: the sensitivity of the loss to the parameters grows "
                    "exponentially with the window (compare short_window); the adjoint is validated against "
                    "FP64 windows and central differences on 20-200-step windows",
            "workload": f"{R} spherical water parcels of {cfgs[0].n} beads (radius {items[0][3]:.1f} sigma, "
                        f"density 1.1 as the reference's confined composition) behind a neutral wall, 12% "
                        f"beads in five-bead amphiphiles, pH U[6,8], I 0.01 M; a {steps}-step window with bond "
                        f"and charge Monte Carlo held off, checkpoints every {every} steps, the loss on every "
                        f"{stride}th frame; seeded synthetic, relaxed untimed"}


def run_batched(args, pkg, L, cfgm, rank, torch, ws=1):
    """The batched form: many uneven replicas stepped together, one launch per kernel per step.  With
    several ranks the one replica set is split across them, balanced by beads (replica_share)."""
    import ctypes as C
    items = batched_configs(cfgm, seed=rank_seeds(rank)[1], replicas=args.replicas)
    mine = replica_share([int(c.n) for c, _, _ in items], ws, rank)
    items = [items[i] for i in mine]
    cfgs, states = [], []
    for cfg, na, sd in items:
        st = amphiphile_state(L, cfg, na, sd)
        s = pkg.SoupSystem(cfg, st)
        s.relax_cold_start(args.aux_relax, 0.1)
        st["positions"] = s.particles()
        s.dispose()
        cfgs.append(cfg)
        states.append(st)
    batch = pkg.SoupBatch(cfgs, states)
    total = sum(int(c.n) for c in cfgs)
    tune = batch.autotune(steps=20) if not args.no_tune else None   # untimed; the choice stays in effect
    batch.step(args.warmup)
    batch.prepare_graphs()
    h0 = batch.replicas[0]._h
    stream = torch.cuda.ExternalStream(L.soup_stream(h0))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    steps = args.batched_steps
    launches0 = L.soup_launch_count(h0)
    torch.cuda.synchronize()
    e0.record(stream)
    batch.step(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    launches = L.soup_launch_count(h0) - launches0
    batch.dispose()
    return {"value": total * steps / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / steps, "steps": steps,
            "replicas": len(cfgs), "beads": total, "gpu_launches": int(launches), "autotune": tune,
            "workload": "uneven replicas: box U[29,53] sigma, density 0.80, 15% beads in preassembled 5-bead "
                        "amphiphiles, rest water, pH U[5,9], I log-U[0.001,0.1] M, sweep every 10, bonds every "
                        "20, skin planned 1.0 with drift rebuilds, lanes per particle, cell size and skin "
                        "autotuned (untimed); steps in captured CUDA graphs; seeded synthetic, relaxed untimed"}


def run_physics_pin(pkg):
    """The trajectory-level pin against the reference's published run (untimed): its bilayer patch
    (tests/water-bilayer-broth.test.ts:68-181, 400 three-bead lipids + 4,500 water, seed 31), equilibrated
    2,000 steps at 1.3 sigma^2 per lipid, taken to the area its area move settled at (1.1734 sigma^2, fixed
    volume), settled 20,000 steps, then the head-peak thickness every 500 steps over 80 snapshots against
    its 4.4689 sigma (verify/out/water-bilayer-area-move.json)."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import bilayer_broth as bb
    import test_gpu_bilayer_pin as pin
    t0 = time.perf_counter()
    th, amph, box, events = pin.run_patch()
    blocks = th.reshape(pin.BLOCKS, -1).mean(axis=1)
    mean, sd = float(th.mean()), float(th.std(ddof=1))
    se = float(blocks.std(ddof=1) / np.sqrt(pin.BLOCKS))
    return {"observable": "bilayer thickness (head-density peaks, 200 bins)", "value": mean, "unit": "sigma",
            "snapshot_sd": sd, "block_se": se, "snapshots": int(th.size), "reference": bb.THICKNESS_REFERENCE,
            "z": (bb.THICKNESS_REFERENCE - mean) / float(np.hypot(sd, se)),
            "area_per_lipid": box[0] * box[1] / (bb.N_LIPIDS / 2), "amphiphiles_min": int(amph.min()),
            "events": events, "wall_s": time.perf_counter() - t0,
            "reference_source": "verify/out/water-bilayer-area-move.json (one snapshot of its settled run)"}


def run_gradient(args, pkg, L, torch):
    """The differentiable bilayer patch: forward + adjoint of the thickness proxy over a 200-step
    window (checkpoints every 20) with respect to the nine force-field parameters."""
    import numpy as np
    from protocell_genesis_b200 import adjoint, config as cfgm
    cfg, st = bilayer_patch(L, cfgm)
    s = pkg.SoupSystem(cfg, st)
    s.relax_cold_start(args.aux_relax, 0.05)
    s.step(200)
    p = s.particles().reshape(-1, 4)
    slots = s.bond_slots().reshape(-1, 3)
    heads = torch.tensor(np.nonzero(p[:, 3] == 1)[0], device="cuda")
    tails = torch.tensor(np.nonzero((p[:, 3] == 0) & np.any(slots != 0xFFFFFFFF, axis=1))[0], device="cuda")
    bz = float(cfg.box[2])
    steps, every = args.grad_steps, 20
    stream = torch.cuda.ExternalStream(L.soup_stream(s._h))
    theta0 = s.get_diff_params()

    def window():
        th = torch.tensor(theta0, dtype=torch.float64, requires_grad=True)
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        torch.cuda.synchronize()
        e0.record(stream)
        traj = adjoint.SoupWindow.apply(th, s, steps, every)
        e1.record(stream)
        loss = adjoint.thickness_proxy(traj, heads, tails, bz)
        loss.backward()
        e2.record(stream)
        torch.cuda.synchronize()
        return float(loss.detach()), th.grad.numpy(), e0.elapsed_time(e1), e1.elapsed_time(e2)

    window()                                  # untimed: allocates the window's scratch
    launches0 = L.soup_launch_count(s._h)
    fwd, bwd = [], []
    for _ in range(args.grad_windows):
        loss, grad, f_ms, b_ms = window()
        fwd.append(f_ms)
        bwd.append(b_ms)
    launches = L.soup_launch_count(s._h) - launches0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    s.step(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    plain_ms = e0.elapsed_time(e1)
    n = int(cfg.n)
    s.dispose()
    total = (sum(fwd) + sum(bwd)) / len(fwd)
    return {"value": n * steps / (total / 1e3), "unit": "particle-steps/s (forward + adjoint)",
            "beads": n, "window_steps": steps, "checkpoint_every": every, "windows": len(fwd),
            "ms_per_window": total, "forward_ms": sum(fwd) / len(fwd), "backward_ms": sum(bwd) / len(bwd),
            "plain_step_ms": plain_ms / steps, "window_vs_plain_steps": total / plain_ms,
            "gpu_launches": int(launches), "loss": "thickness proxy", "value_of_loss": loss,
            "theta": list(adjoint.PARAM_NAMES), "grad": [float(x) for x in grad],
            "workload": "preassembled flat bilayer, 2,048 five-bead amphiphiles, water to density 0.80, box "
                        "32x32x40 sigma, pH 9, I 0.01 M; seeded synthetic, relaxed untimed; bond and charge "
                        "Monte Carlo held off inside the window"}


class CampaignSampler:
    """The campaign's progress sample on the system (config 2: closure flood-fill and aggregate
    labels every 200 steps): amphiphiles, aggregate labels at the nonbonded cutoff, the shapes of the
    five largest aggregates and the closure (encapsulated water) of each, about its periodic centre."""

    def __init__(self, pkg, cfgm, cfg, system):
        import math
        import numpy as np
        from protocell_genesis_b200 import observables
        self.np, self.obs = np, observables
        P = cfgm.load_params()
        self.st = P["stageThresholds"]
        self.alpha = P["circularAlpha"]
        self.cutoff = float(cfg.rc_attr + cfg.wc)
        self.cells = int(np.prod([max(1, int(math.floor(b / self.cutoff))) for b in cfg.box]))
        self.box = list(cfg.box)
        solvent = [k for k, m in enumerate(P["monomers"]) if m["solvent"]]
        kinds = system.particles().reshape(-1, 4)[:, 3]
        self.water = np.nonzero(np.isin(kinds, np.array(solvent, np.float32)))[0].astype(np.uint32)
        self.times = []

    def __call__(self, s):
        from protocell_genesis_b200 import _abi
        np = self.np
        t0 = time.perf_counter()
        _, head_of = s.amphiphile_labels()
        members = np.nonzero(head_of != 0xFFFFFFFF)[0].astype(np.uint32)
        out = {"aggregates": 0, "largest": 0, "encapsulated": []}
        if members.size:
            if members.size <= _abi.NOALLOC_MAX_MEMBERS and self.cells <= _abi.NOALLOC_MAX_CELLS:
                ncomp, labels = s.aggregate_labels_noalloc(members, self.cutoff)
            else:
                ncomp, labels = s.aggregate_labels(members, self.cutoff)
            _, shapes = s.aggregate_shapes(members, labels, int(self.st["detailAggregateCount"]))
            pos = s.particles()
            out["aggregates"], out["largest"] = int(ncomp), int(shapes[0]["size"]) if shapes else 0
            for sh in shapes:
                m = members[labels == sh["label"]]
                c = self.obs.periodic_centre(pos, m, self.box, self.alpha)
                if c is not None:
                    r = s.closure(m, self.water, c, self.st["closureCell"], self.st["closureRadius"],
                                  self.st["enclosedVolume"])
                    out["encapsulated"].append(int(r["encapsulatedCount"]))
        self.times.append(time.perf_counter() - t0)
        return out


def checkpoint_timing(s, cfg, reps=3):
    """A checkpoint of the live system (soup/src/checkpoint.ts encodeCheckpoint): the one-call device
    payload alone, and the whole CheckpointFile as JSON text (payload, base64, serialisation); the
    median of `reps` each, wall clock."""
    import json as _json
    from protocell_genesis_b200 import checkpoint as ck
    config = {"box": [float(x) for x in cfg.box], "seed": int(cfg.seed), "kT": float(cfg.kT)}
    import tempfile
    t_pay, t_file, t_bin, size, bsize = [], [], [], 0, 0
    with tempfile.TemporaryDirectory() as tmp:
        for _ in range(reps):
            t0 = time.perf_counter()
            s.checkpoint_payload()
            t_pay.append(time.perf_counter() - t0)
            t0 = time.perf_counter()
            size = len(_json.dumps(ck.encode_checkpoint(s, config)))
            t_file.append(time.perf_counter() - t0)
            t0 = time.perf_counter()
            bsize = ck.write_checkpoint_binary(os.path.join(tmp, "c.bin"), s, config)
            t_bin.append(time.perf_counter() - t0)
    return {"payload_ms": 1e3 * statistics.median(t_pay), "file_ms": 1e3 * statistics.median(t_file),
            "binary_file_ms": 1e3 * statistics.median(t_bin), "binary_file_bytes": bsize,
            "file_bytes": size, "payload_bytes": 64 * s.n,
            "what": "payload: soup_read_checkpoint (one device gather, one wait) into pageable host memory; "
                    "file: payload + base64 + JSON text of the reference's CheckpointFile; binary_file: payload "
                    "+ the binary form written to a local file"}


def stage_timing(s, reps=3):
    """detectStage (soup/src/stages.ts:204-289) of the live system through observables.detect_stage:
    the particle read-back, amphiphiles, aggregate labels, the box-wide head peaks and enclosed
    volume, and analyzeAggregates with the water beads; median wall clock of `reps` after one warm
    call."""
    from protocell_genesis_b200 import observables as obs
    r = obs.detect_stage(s)
    t = []
    for _ in range(reps):
        t0 = time.perf_counter()
        r = obs.detect_stage(s)
        t.append(time.perf_counter() - t0)
    e = r["evidence"]
    a = e["aggregateAnalysis"]
    return {"ms": 1e3 * statistics.median(t), "stage": r["stage"],
            "amphiphile_fraction": e["amphiphileFraction"], "aggregates": a["aggregateCount"],
            "enclosed_volume": e["enclosedVolume"], "head_peaks": e["headPeaks"],
            "what": "one detect_stage call per sample, wall clock (the reference quotes 1.5-1.9 s per sample at "
                    "this size)"}


def box_scale_timing(s, cfg):
    """One box change of the live system (soup/src/soup-box-scale.ts applyBoxScaleOnce) on the device:
    rigid units of the covalent bonds, then with the amphiphiles' proximity cohesion at the nonbonded
    cutoff; wall clock of each call (the map, the self-check, the re-grid, rebuild and force pass).
    It runs after everything that is timed: the system is left in the slightly compressed box."""
    import numpy as np
    from protocell_genesis_b200 import _abi
    box = [float(x) for x in s.box]
    _, head_of = s.amphiphile_labels()
    members = np.nonzero(head_of != _abi.NONE)[0].astype(np.uint32)
    cut = float(cfg.rc_attr + cfg.wc)
    out = {"beads": s.n, "bonds": int(s.bonds().size // 2), "cohesion_members": int(members.size)}
    t0 = time.perf_counter()
    s.scale_box_once([x * 0.995 for x in box])
    out["bonds_only_ms"] = 1e3 * (time.perf_counter() - t0)
    t0 = time.perf_counter()
    s.scale_box_once([x * 0.99 for x in box], {"cutoff": cut, "memberIndices": members})
    out["with_cohesion_ms"] = 1e3 * (time.perf_counter() - t0)
    return out


def step_with_samples(s, steps, every, sampler):
    """`steps` steps with the progress sample after every `every` of them."""
    done, samples = 0, []
    while done < steps:
        k = min(every - done % every, steps - done)
        s.step(k)
        done += k
        if sampler is not None and done % every == 0:
            samples.append(sampler(s))
    return samples


def run_cuda(args):
    import ctypes as C
    import numpy as np
    import torch
    ws, rank, local = dist_init()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", device_id=torch.device("cuda", local), timeout=datetime.timedelta(seconds=300))
    import __graft_entry__ as ge
    pkg = ge._package()
    from protocell_genesis_b200 import _abi, config as cfgm
    L = _abi.lib()
    cfg = cfgm.resolve(workload_opts(cfgm, seed=rank_seeds(rank)[0], skin=args.skin, scale=args.scale))
    n = cfg.n
    # fresh lattice on the host, relaxed on the device (untimed set-up)
    host = {}
    for name, dt, per in (("positions", np.float32, 4), ("velocities", np.float32, 4)):
        host[name] = np.zeros(n * per, dt)
    fr = np.zeros(n, np.uint32); br = np.zeros(n, np.uint32); tr = np.zeros(n, np.uint32)
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    L.soup_fresh_state(C.byref(cfg), p(host["positions"]), p(host["velocities"]), p(fr), p(br), p(tr))
    s = pkg.SoupSystem(cfg)
    relax = s.relax_cold_start(args.relax, 0.1)
    # untimed; the choice (lanes per particle, cell size) stays in effect; the skin stays as planned,
    # the same as the reference arm's
    tune = s.autotune(steps=0) if not args.no_tune else None
    s.step(args.warmup)
    s.prepare_graphs()   # every chunk graph of the schedule captured before the timed region
    sampler = None if args.no_analysis else CampaignSampler(pkg, cfgm, cfg, s)
    if sampler is not None:
        sampler(s)       # untimed: the analysis scratch is allocated on first use
        sampler.times.clear()
    stream = torch.cuda.ExternalStream(L.soup_stream(s._h))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    launches0 = L.soup_launch_count(s._h)
    info0 = s.info()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        torch.cuda.nvtx.range_push("timed")
        e0.record(stream)
        samples = step_with_samples(s, args.steps, args.analysis_every, sampler)
        e1.record(stream)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
    if dist:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    launches = L.soup_launch_count(s._h) - launches0
    info1 = s.info()
    # the per-kernel split: a profiled segment right after the timed region (events around every
    # launch group, so these steps run launch by launch instead of as captured graphs)
    L.soup_profile(s._h, 1)
    s.step(args.prof_steps)
    torch.cuda.synchronize()
    ktime = {}
    for k, name in enumerate(_abi.K_NAMES):
        t = C.c_double(); c = C.c_uint64()
        L.soup_kernel_time(s._h, k, C.byref(t), C.byref(c))
        ktime[name] = (t.value, c.value)
    L.soup_profile(s._h, 0)
    ms_max = max_over_ranks(ms, dist, "cuda")
    value = aggregate_rate(ws, n, args.steps, ms_max)

    # roofline of the dominant kernel (the list force), algorithmic bytes per launch:
    # per particle 4 B per list entry + pos 16 + charge 4 + slots 12 + centre 4 + count 4 + force 16
    counts = np.empty(n, np.uint32)
    L.soup_read_verlet(s._h, counts.ctypes.data_as(_abi._U32P), None, 0)
    mean_list = float(counts.mean())
    f_ms, f_n = ktime["force"]
    bytes_per_launch = n * (4.0 * mean_list + 56.0)
    achieved = bytes_per_launch / (f_ms / max(f_n, 1) / 1e3) / 1e9 if f_n else None
    peak, peak_kind = peaks()
    # DRAM bytes per launch of the force kernel from the committed ncu capture's numbers
    # (profiles/roofline_traffic.json: measured on a smaller case of the same workload and scaled to
    # 483,268 beads there); scaled again by particles x list entries, which the traffic follows
    traffic = None
    tf = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if os.path.exists(tf):
        with open(tf) as fh:
            tj = json.load(fh)
        if tj.get("kernel") == FORCE_KERNEL:
            traffic = float(tj["traffic_bytes_per_launch_483k"]) * (n * mean_list) / (
                483268.0 * float(tj["mean_list_entries_483k"]))
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                "kernel": FORCE_KERNEL,
                "algorithmic_bytes_per_launch": bytes_per_launch, "mean_list_entries": mean_list,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback 6.65 TB/s"}

    # the force error of the timed state (untimed): the list force + far half against the oracle's
    # FP64 force at the same positions
    force_err = None
    if not args.no_force_check:
        import oracle_binding as ob
        from helpers import rel_rms
        st_now = {"positions": s.particles(), "charges": s.charges(), "bond_slots": s.bond_slots(),
                  "center_link": s.center_links()}
        o_ = ob.OracleSystem(_abi, cfg, st_now)
        force_err = rel_rms(s.forces_no_rebuild(), o_.forces64())
        o_.close()

    ckpt = checkpoint_timing(s, cfg)
    stage = stage_timing(s)

    # end to end through the public API with host buffers: create from pinned host arrays
    # (H2D of the whole state), step in chunks of 10 with the positions read back after each chunk
    state = {"positions": s.particles(), "velocities": s.velocities(), "charges": s.charges(),
             "bond_slots": s.bond_slots(), "center_link": s.center_links(), "center_held": s.center_held_steps(),
             "bond_rng": s.rng_state()["bond"], "thermo_rng": s.rng_state()["thermo"]}
    pinned = {}
    for k_, v_ in state.items():
        t_ = torch.from_numpy(np.ascontiguousarray(v_)).pin_memory()
        pinned[k_] = t_.numpy()
    out_pos = torch.empty(4 * n, dtype=torch.float32).pin_memory().numpy()
    e2e_steps = max(args.steps, E2E_MIN_STEPS) if not args.no_e2e else 0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s2 = pkg.SoupSystem(cfg, pinned)
    if tune:
        s2.apply_tuning(tune)   # the tuning found above, applied as a user would reuse it
    done = 0
    while done < e2e_steps:
        c_ = min(10, e2e_steps - done)
        s2.step(c_)
        L.soup_read_pos(s2._h, out_pos.ctypes.data_as(C.c_void_p), out_pos.nbytes)
        done += c_
        if sampler is not None and done % args.analysis_every == 0:
            sampler(s2)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    h2d = sum(v_.nbytes for v_ in pinned.values())
    e2e = None
    if e2e_steps:
        e2e = {"value": ws * n * e2e_steps / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": h2d / e2e_steps, "d2h_bytes_per_step": 16 * n / 10,
               "steps": e2e_steps,
               "note": "create from pinned host arrays + apply the autotuned shape + step(10) + particles() readback "
                       "per 10 steps + the analysis sample every 200 steps, wall clock"}
    s2.dispose()
    box_scale = box_scale_timing(s, cfg)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        import oracle_binding as ob
        cpu = cpu_sample(pkg, ob, cfg, state, budget_s=args.cpu_budget)

    batched = None
    if not args.no_batched:
        batched = run_batched(args, pkg, L, cfgm, rank, torch, ws)
        if dist:
            # the replica set is split across the ranks: all their beads over the slowest rank's step
            batched["ms_per_step"] = max_over_ranks(batched["ms_per_step"], dist, "cuda")
            batched["beads"] = int(sum_over_ranks(batched["beads"], dist, "cuda"))
            batched["value"] = aggregate_rate(1, batched["beads"], 1, batched["ms_per_step"])
        batched["vs_plain"] = batched["value"] / value

    gradient_batched = None
    if not args.no_gradient:
        gradient_batched = run_gradient_batched(args, pkg, L, torch)
        if dist:
            gradient_batched["ms_per_window"] = max_over_ranks(gradient_batched["ms_per_window"], dist, "cuda")
            gradient_batched["value"] = aggregate_rate(ws, gradient_batched["beads"], gradient_batched["window_steps"],
                                                       gradient_batched["ms_per_window"])

    gradient = None
    if not args.no_gradient:
        gradient = run_gradient(args, pkg, L, torch)
        if dist:
            gradient["ms_per_window"] = max_over_ranks(gradient["ms_per_window"], dist, "cuda")
            gradient["value"] = aggregate_rate(ws, gradient["beads"], gradient["window_steps"],
                                               gradient["ms_per_window"])

    physics = run_physics_pin(pkg) if (rank == 0 and not args.no_physics) else None

    phases = {name: {"ms_total": t, "launches": c, "ms_per_step": t / args.prof_steps} for name, (t, c) in ktime.items() if c}
    # diagnostic: the rate with the constant-pH sweep's share of the profiled segment taken out
    seg_ms = sum(t for t, c in ktime.values())
    sweep_ms = ktime.get("sweep", (0.0, 0))[0]
    value_ex_sweep = value * seg_ms / (seg_ms - sweep_ms) if seg_ms > sweep_ms > 0 else None
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": value / (ws * PUBLISHED), "dtype": "f32", "data": "synthetic",
            "config": workload_config(args.skin, args.relax, n),
            "details": {"replicas_per_gpu": 1,
                       "relax": {"iterations": args.relax, "max_force_after": relax["maxForceAfter"]},
                       "rebuilds_in_timed_region": info1["rebuilds"] - info0["rebuilds"],
                       "sweeps_in_timed_region": info1["sweeps"] - info0["sweeps"],
                       "autotune": tune,
                       "checkpoint": ckpt,
                       "stage_detection": stage,
                       "box_scale": box_scale,
                       "analysis": None if sampler is None else {
                           "every": args.analysis_every, "samples_in_timed_region": len(samples),
                           "ms_per_sample": 1e3 * sum(sampler.times[:len(samples)]) / max(len(samples), 1),
                           "last": samples[-1] if samples else None,
                           "what": "amphiphiles, aggregate labels at the nonbonded cutoff, shapes of the five "
                                   "largest aggregates, closure flood-fill (0.5 sigma voxels) of each"},
                       "execution": "steps in captured CUDA graphs of 10 (one sweep period), the drift-triggered "
                                    "rebuild a conditional node",
                       "split": f"phases and the force roofline from a profiled segment of {args.prof_steps} steps "
                                "right after the timed region"},
            "force_rel_rms": force_err,
            "value_excluding_sweep": value_ex_sweep,
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
            "clocks": clk.summary(), "phases": phases, "batched": batched, "gradient": gradient,
            "gradient_batched": gradient_batched, "physics_pin": physics}
    if rank == 0:
        print(json.dumps(line), flush=True)
    s.dispose()
    if dist:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="cuda", choices=["cuda", "reference"])
    ap.add_argument("--skin", type=float, default=SKIN)
    ap.add_argument("--relax", type=int, default=RELAX_ITERATIONS, help="cold-start relax of the plain workload (both arms)")
    ap.add_argument("--aux-relax", type=int, default=200, help="cold-start relax of the batched and gradient workloads")
    ap.add_argument("--ref-budget", type=float, default=60.0)
    ap.add_argument("--cpu-budget", type=float, default=12.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-force-check", action="store_true", help="skip the FP64 force check of the timed state")
    ap.add_argument("--scale", type=float, default=1.0, help="census and box-volume factor (profiling captures)")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-replica measurement")
    ap.add_argument("--replicas", type=int, default=64)
    ap.add_argument("--batched-steps", type=int, default=100)
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuning (plain and batched)")
    ap.add_argument("--no-analysis", action="store_true", help="leave the campaign's progress sample out of the timed steps")
    ap.add_argument("--analysis-every", type=int, default=200)
    ap.add_argument("--no-gradient", action="store_true", help="skip the forward + adjoint window measurement")
    ap.add_argument("--no-physics", action="store_true", help="skip the bilayer-thickness pin (untimed)")
    ap.add_argument("--prof-steps", type=int, default=100, help="steps of the profiled segment (per-kernel split)")
    ap.add_argument("--grad-steps", type=int, default=200)
    ap.add_argument("--grad-windows", type=int, default=3)
    ap.add_argument("--parcel-replicas", type=int, default=16)
    ap.add_argument("--parcel-steps", type=int, default=2000)
    ap.add_argument("--parcel-checkpoint", type=int, default=100)
    ap.add_argument("--parcel-stride", type=int, default=20)
    ap.add_argument("--parcel-windows", type=int, default=1)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_cuda(args)


if __name__ == "__main__":
    main()

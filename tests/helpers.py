"""Shared fixtures for the tests: configurations of the reference's test compositions."""
import math

import numpy as np

import protocell_genesis_b200 as pg
from protocell_genesis_b200 import _abi, config as cfgm


def plain_opts(**kw):
    """tests/soup-forces.test.ts:19-65: box 16, C600 O100 H500 M20 W0, seed 7, kT 1.1."""
    base = dict(box=[16, 16, 16], seed=7, kT=1.1, start={"C": 600, "O": 100, "H": 500, "M": 20, "W": 0})
    base.update(kw)
    return cfgm.SoupOptions(**base)


def charged_opts(**kw):
    """tests/soup-forces.test.ts:81-139: the plain composition with electrostatics at pH 7."""
    base = dict(box=[16, 16, 16], seed=7, kT=1.1, start={"C": 600, "O": 100, "H": 500, "M": 20, "W": 0},
                electrostatics={"enabled": True, "pH": 7.0})
    base.update(kw)
    return cfgm.SoupOptions(**base)


def long_range_opts(**kw):
    """tests/soup-forces.test.ts:156-199 (box 30, I = 0.01 M: rc_es = 13.5 sigma by the 0.45 L cap)."""
    base = dict(box=[30, 30, 30], seed=11, kT=1.1, start={"C": 1200, "O": 400, "H": 1000, "M": 30, "W": 3000},
                electrostatics={"enabled": True, "pH": 7.0, "ionicStrengthMolar": 0.01})
    base.update(kw)
    return cfgm.SoupOptions(**base)


def confined_opts(**kw):
    """tests/soup-forces.test.ts:216-294: box 80, parcel R 16, k 100, the campaign census scaled."""
    base = dict(box=[80, 80, 80], seed=9, kT=1.1, start={"C": 2188, "O": 729, "H": 2188, "M": 57, "W": 13726},
                confine={"radiusSigma": 16, "stiffness": 100},
                electrostatics={"enabled": True, "pH": 7.0, "ionicStrengthMolar": 0.01})
    base.update(kw)
    return cfgm.SoupOptions(**base)


def water_opts(n_water=3000, box=16.0, **kw):
    base = dict(box=[box] * 3, seed=3, kT=1.1, start={"C": 300, "O": 120, "H": 0, "M": 30, "W": n_water},
                electrostatics={"enabled": True, "pH": 5.5, "ionicStrengthMolar": 0.05})
    base.update(kw)
    return cfgm.SoupOptions(**base)


def boosted(cfg, attempt=1.0, accept=1.0, brk=0.3):
    """Every formation attempt fires, breaks are frequent: stresses the claim arbitration."""
    for r in range(cfg.n_rules):
        cfg.attempt_form[r] = attempt
        cfg.accept_form[r] = accept
        cfg.attempt_break[r] = brk
        cfg.accept_break[r] = brk
    return cfg


def rel_rms(a, b):
    a = np.asarray(a, np.float64).reshape(-1, 4)[:, :3]
    b = np.asarray(b, np.float64).reshape(-1, 4)[:, :3]
    return math.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300))


def csr_rows(counts, lists):
    off = np.concatenate([[0], np.cumsum(counts.astype(np.int64))])
    return [lists[off[i]:off[i + 1]] for i in range(len(counts))]


def oracle_bilayer_start(lx=15.0, lz=16.0, per_side=10, seed=3, relax=200, steps=100):
    """A small preassembled bilayer patch (the differentiable-patch workload at lx x lx x lz),
    relaxed and stepped on the oracle: (config, start state with every field of a checkpoint)."""
    import bench
    import oracle_binding as ob
    cfg, st = bench.bilayer_patch(_abi.lib(), cfgm, lx=lx, lz=lz, per_side=per_side, seed=seed)
    o = ob.OracleSystem(_abi, cfg, st)
    o.relax(relax, 0.05)
    if steps:
        o.step(steps)
    start = dict(positions=o.read(ob.F_POS), velocities=o.read(ob.F_VEL), bond_slots=o.read(ob.F_SLOTS),
                 center_link=o.read(ob.F_CENTER), center_held=o.read(ob.F_HELD), bond_rng=o.read(ob.F_BOND_RNG),
                 thermo_rng=o.read(ob.F_THERMO_RNG), charges=o.read(ob.F_CHARGES), frozen=o.read(ob.F_FROZEN))
    o.close()
    return cfg, start


def config1_start(seed=0):
    """The plain small case (16 sigma cube, 3,277 beads): 200 five-bead amphiphiles (head + 4 carbon,
    straight along x, 0.95 sigma apart) on a 4 x 5 x 10 lattice, 2,277 water beads placed uniformly at
    random at least 0.8 sigma from every bead, every head charged -1 and no constant-pH sweep
    (lambda_D = 6.5 sigma, so I = (0.304 / (6.5 * 0.8))^2 M and rc_es = 0.45 L = 7.2 sigma), seed 0,
    kT 1.  Slots as tests/water-bilayer.test.ts:113-118: head[0] = c1; c1[2] = head, c1[0] = c2;
    c2 = (c1, c3); c3 = (c2, c4); c4[0] = c3.  Returns (options, start state)."""
    L = 16.0
    ion = (0.304 / (6.5 * 0.8)) ** 2
    opts = cfgm.SoupOptions(box=[L, L, L], seed=seed, kT=1.0, start={"C": 800, "O": 200, "H": 0, "M": 0, "W": 2277},
                            electrostatics={"enabled": True, "pH": 7.0, "ionicStrengthMolar": ion},
                            sweep_every=10 ** 9)
    P = cfgm.load_params()
    kind = {m["id"]: k for k, m in enumerate(P["monomers"])}
    pts, kinds = [], []
    slots = []
    for ix in range(4):
        for iy in range(5):
            for iz in range(10):
                h = len(pts)
                base = np.array([0.3 + ix * 4.0, 1.6 + iy * 3.2, 0.8 + iz * 1.6])
                pts.append(base)
                kinds.append(kind["O"])
                for c in range(1, 5):
                    pts.append(base + np.array([0.95 * c, 0.0, 0.0]))
                    kinds.append(kind["C"])
                s = [[h + 1, _abi.NONE, _abi.NONE], [h + 2, _abi.NONE, h], [h + 1, h + 3, _abi.NONE], [h + 2, h + 4, _abi.NONE],
                     [h + 3, _abi.NONE, _abi.NONE]]
                slots += s
    rng = np.random.default_rng(seed)
    cell = {}
    def key(p):
        return tuple((np.floor(p / 1.0).astype(int)) % 16)
    for i, p in enumerate(pts):
        cell.setdefault(key(p), []).append(i)
    placed = [np.asarray(p) for p in pts]
    while len(placed) < 3277:
        p = rng.uniform(0, L, 3)
        k = key(p)
        ok = True
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    for j in cell.get(((k[0] + dx) % 16, (k[1] + dy) % 16, (k[2] + dz) % 16), []):
                        d = placed[j] - p
                        d -= np.round(d / L) * L
                        if d @ d < 0.64:
                            ok = False
        if ok:
            cell.setdefault(k, []).append(len(placed))
            placed.append(p)
            kinds.append(kind["W"])
            slots.append([_abi.NONE, _abi.NONE, _abi.NONE])
    pos = np.zeros((3277, 4), np.float32)
    pos[:, :3] = np.mod(np.array(placed), L)
    pos[:, 3] = kinds
    q = np.where(pos[:, 3] == kind["O"], -1.0, 0.0).astype(np.float32)
    return opts, {"positions": pos.reshape(-1), "bond_slots": np.array(slots, np.uint32).reshape(-1), "charges": q}

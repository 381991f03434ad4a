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

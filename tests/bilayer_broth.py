"""The reference's bilayer-in-water patch: 400 three-bead lipids (head + two tail carbons) in liquid
water at 0.8 per sigma^3, seed 31, kT 1.1, restated from its construction in
tests/water-bilayer-broth.test.ts:68-181 (the same construction tests/water-bilayer-area-move.test.ts
:80-165 starts from).  The random numbers are mulberry32 with the reference's seed, drawn in the
reference's order (lipids x then y; water x, y, z), and every coordinate is computed in double and
stored as float32, as the reference's Float32Array does.

Its published outcome (verify/out/water-bilayer-area-move.json): with the zero-tension area move the
patch settles at an area per lipid of 1.1734 sigma^2 (tail window 1.1696-1.1765) and a thickness of
4.4689 sigma between the head-density peaks, with 381 of 400 amphiphiles left (19 head-carbon
breaks).  The area move keeps the volume (soup/src/soup-area-move.ts:57-63, 'lateral-fixed-volume').
"""
import math

import numpy as np

N_LIPIDS = 400
AREA_START = 1.3            # the area corridor's midpoint, (1.1 + 1.5) / 2 (data/literature.json)
BOX_Z = 30.0
WATER_DENSITY = 0.8
SEED = 31
KT = 1.1                    # data/params.json thermostat.kT
AREA_SETTLED = 1.1734461123400626      # verify/out/water-bilayer-area-move.json areaPerLipid
AREA_TAIL = (1.1695877806292108, 1.176498681004865)
THICKNESS_REFERENCE = 4.468932297634941


def mulberry32(seed):
    """The reference's seeded generator (JavaScript int32 arithmetic, as uint32 here)."""
    a = seed & 0xFFFFFFFF
    M = 0xFFFFFFFF

    def rng():
        nonlocal a
        a = (a + 0x6D2B79F5) & M
        t = ((a ^ (a >> 15)) * (1 | a)) & M
        t = ((t + (((t ^ (t >> 7)) * (61 | t)) & M)) & M) ^ t
        return ((t ^ (t >> 14)) & M) / 4294967296.0
    return rng


def broth_state(P, area=AREA_START, box_z=BOX_Z, seed=SEED):
    """(options dict for SoupOptions, resume arrays) of the patch at `area` per lipid."""
    mons = P["monomers"]
    carbon = next(i for i, m in enumerate(mons) if m["kind"] == "carbon")
    head = next(i for i, m in enumerate(mons) if m["kind"] == "head")
    water = next(i for i, m in enumerate(mons) if m["kind"] == "water")
    sigma = P["params"]["sigma"]
    cR, hR, wR = mons[carbon]["radiusSigma"], mons[head]["radiusSigma"], mons[water]["radiusSigma"]
    bTT = (sigma * (cR + cR)) / 2
    bHT = (sigma * (hR + cR)) / 2
    bWT = (sigma * (wR + cR)) / 2
    L = math.sqrt((N_LIPIDS / 2) * area)
    z0 = box_z / 2
    gap = bTT / 2
    half_span = gap + bTT + bHT
    per_leaflet = math.ceil(N_LIPIDS / 2)
    n_side = max(1, math.ceil(math.sqrt(per_leaflet)))
    spx, spy = L / n_side, L / n_side
    jitter = 0.15
    rng = mulberry32(seed)
    n_max = N_LIPIDS * 3 + math.ceil(WATER_DENSITY * L * L * box_z)
    pos = np.zeros((n_max, 4), np.float32)
    slots = np.full((n_max, 3), 0xFFFFFFFF, np.uint32)
    k = 0
    for i in range(N_LIPIDS):
        leaflet = 1 if i < per_leaflet else -1
        idx = i if i < per_leaflet else i - per_leaflet
        a, b = idx % n_side, idx // n_side
        x = math.fmod((a + 0.5) * spx + (rng() * 2 - 1) * jitter * spx + L, L)
        y = math.fmod((b + 0.5) * spy + (rng() * 2 - 1) * jitter * spy + L, L)
        z_t2 = z0 + leaflet * gap
        z_t1 = z_t2 + leaflet * bTT
        z_h = z_t1 + leaflet * bHT
        pos[k] = (x, y, z_h, head)
        pos[k + 1] = (x, y, z_t1, carbon)
        pos[k + 2] = (x, y, z_t2, carbon)
        slots[k, 0] = k + 1
        slots[k + 1, 2] = k
        slots[k + 1, 0] = k + 2
        slots[k + 2, 0] = k + 1
        k += 3
    margin = bWT * 1.5
    z_lo, z_hi = z0 - half_span - margin, z0 + half_span + margin
    spacing = (1 / WATER_DENSITY) ** (1 / 3)
    wnx = max(1, round(L / spacing))
    wny = max(1, round(L / spacing))
    wnz = max(1, round(box_z / spacing))
    sx, sy, sz = L / wnx, L / wny, box_z / wnz
    placed = 0
    for iz in range(wnz):
        if k >= n_max:
            break
        z_raw = (iz + 0.5) * sz
        if z_lo < z_raw < z_hi:
            continue
        for iy in range(wny):
            for ix in range(wnx):
                if k >= n_max:
                    break
                x = math.fmod((ix + 0.5) * sx + (rng() * 2 - 1) * jitter * sx + L, L)
                y = math.fmod((iy + 0.5) * sy + (rng() * 2 - 1) * jitter * sy + L, L)
                z = min(box_z - 1e-4, max(0.0, z_raw + (rng() * 2 - 1) * jitter * sz))
                pos[k] = (x, y, z, water)
                k += 1
                placed += 1
    n = k
    ids = np.arange(n, dtype=np.uint32)
    start = {m["id"]: 0 for m in mons}
    start[mons[head]["id"]] = N_LIPIDS
    start[mons[carbon]["id"]] = 2 * N_LIPIDS
    start[mons[water]["id"]] = placed
    opts = dict(box=[L, L, box_z], seed=seed, kT=KT, start=start)
    state = dict(positions=pos[:n].reshape(-1).copy(), velocities=np.zeros(4 * n, np.float32),
                 bond_slots=slots[:n].reshape(-1).copy(), center_link=np.full(n, 0xFFFFFFFF, np.uint32),
                 center_held=np.zeros(n, np.uint32), bond_rng=ids + 1, thermo_rng=ids + 1000003)
    return opts, state


def settled_box(area=AREA_SETTLED, area_start=AREA_START, box_z=BOX_Z):
    """The box at `area` per lipid with the start's volume (the area move's fixed-volume mode)."""
    L0 = math.sqrt((N_LIPIDS / 2) * area_start)
    L = math.sqrt((N_LIPIDS / 2) * area)
    return [L, L, L0 * L0 * box_z / (L * L)]

"""The four synthetic aggregate arrangements of the reference's stage tests
(tests/soup-aggregates.test.ts:17-231), seeded: (positions f32 x4 with w = kind, bonds as flat
(head, tail) pairs, box).  Every amphiphile is one head bead bonded to one tail bead."""
import math

import numpy as np

from protocell_genesis_b200 import config as cfgm

P = cfgm.load_params()
KIND_C = next(k for k, m in enumerate(P["monomers"]) if m["kind"] == "carbon")
KIND_O = next(k for k, m in enumerate(P["monomers"]) if m["kind"] == "head")


class _Builder:
    def __init__(self):
        self.p, self.bonds = [], []

    def amphiphile(self, head, tail):
        h = len(self.p)
        self.p.append([head[0], head[1], head[2], KIND_O])
        self.p.append([tail[0], tail[1], tail[2], KIND_C])
        self.bonds += [h, h + 1]

    def done(self, box):
        return np.array(self.p, np.float32).reshape(-1), np.array(self.bonds, np.uint32), list(box)


def _fibonacci_sphere(n):
    golden = math.pi * (3 - math.sqrt(5))
    out = []
    for i in range(n):
        y = 1 - (i / (n - 1)) * 2
        r = math.sqrt(1 - y * y)
        out.append((math.cos(golden * i) * r, y, math.sin(golden * i) * r))
    return out


def _random_dir(rng):
    u = rng.uniform(-1, 1)
    phi = rng.uniform(0, 2 * math.pi)
    s = math.sqrt(1 - u * u)
    return (s * math.cos(phi), s * math.sin(phi), u)


def micelles():
    """Scenario A (:80-108): three round micelles of 20 amphiphiles, heads at 1.2, tails at 0.5."""
    b = _Builder()
    for c in ((20, 20, 20), (70, 20, 20), (20, 70, 20)):
        for d in _fibonacci_sphere(20):
            b.amphiphile([c[k] + d[k] * 1.2 for k in range(3)], [c[k] + d[k] * 0.5 for k in range(3)])
    return b.done((100, 100, 100))


def flat_layer():
    """Scenario B (:117-147): a 13 x 13 square patch, heads at +-2.2 and tails at +-1.0 about z = 30."""
    b = _Builder()
    for ix in range(13):
        for iy in range(13):
            x, y = 30 + ix * 1.4, 30 + iy * 1.4
            b.amphiphile((x, y, 30 + 2.2), (x, y, 30 + 1.0))
            b.amphiphile((x, y, 30 - 2.2), (x, y, 30 - 1.0))
    return b.done((100, 100, 100))


def hollow_shell(seed=11):
    """Scenario C (:159-191): 8,000 outer and 4,000 inner heads at radii 12.4 and 8 (+-0.5), tails
    spread through the wall; box 60."""
    rng = np.random.default_rng(seed)
    b = _Builder()
    c = (30.0, 30.0, 30.0)

    def tail():
        d = _random_dir(rng)
        r = 8 + rng.uniform() * (12.4 - 8)
        return [c[k] + d[k] * r for k in range(3)]

    for n_heads, radius in ((8000, 12.4), (4000, 8.0)):
        for _ in range(n_heads):
            d = _random_dir(rng)
            rh = radius + (rng.uniform() - 0.5) * 1.0
            b.amphiphile([c[k] + d[k] * rh for k in range(3)], tail())
    return b.done((60, 60, 60))


def dense_ball():
    """Scenario D (:204-231): a cubic lattice (spacing 1.8) filling a ball of radius 9, tails 0.3 off."""
    b = _Builder()
    for ix in range(-6, 7):
        for iy in range(-6, 7):
            for iz in range(-6, 7):
                x, y, z = ix * 1.8, iy * 1.8, iz * 1.8
                if math.sqrt(x * x + y * y + z * z) > 9:
                    continue
                b.amphiphile((30 + x, 30 + y, 30 + z), (30 + x + 0.3, 30 + y, 30 + z))
    return b.done((60, 60, 60))


def cutoff():
    """The scenarios' clustering cutoff: wcaCutoff(sigma * max radius of carbon and head) + wc."""
    radii = [m["radiusSigma"] for m in P["monomers"] if m["kind"] in ("carbon", "head")]
    return cfgm.wca_cutoff(P["params"]["sigma"] * max(radii)) + P["params"]["wc"]


def slots_of(n, bonds):
    """Bond slots in the reference's convention: the head's slot 0 holds its tail, the tail's head slot
    (2) holds its head."""
    s = np.full((n, 3), 0xFFFFFFFF, np.uint32)
    e = np.asarray(bonds).reshape(-1, 2)
    s[e[:, 0], 0] = e[:, 1]
    s[e[:, 1], 2] = e[:, 0]
    return s.reshape(-1)

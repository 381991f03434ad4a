"""A trajectory-level pin against the reference's own published output: the thickness of its bilayer
patch in liquid water.

The patch is the reference's (tests/water-bilayer-broth.test.ts:68-181, restated in bilayer_broth.py):
400 three-bead lipids and 4,500 water beads, seed 31, kT 1.1, the default force field, bond Monte Carlo
every 20 steps, Verlet lists rebuilt every 10 steps.  Its published run (tests/water-bilayer-area-move
.test.ts; verify/out/water-bilayer-area-move.json) equilibrates 2,000 steps at 1.3 sigma^2 per lipid and
then lets a zero-tension area move settle the area at 1.1734 sigma^2 at fixed volume; its final snapshot
measures 4.4689 sigma between the head-density peaks of the amphiphiles' z profile (200 bins).

The area move itself is outside this path, so here the same start equilibrates the same 2,000 steps,
the box is taken to the settled area at fixed volume in 20 rigid-molecule increments
(soup/src/soup-box-scale.ts:218-275 scaleBoxTo), and the thickness is then sampled every 500 steps, the
reference's chunk, with densityProfileZ and bilayerPeaks (engine/src/metrics.ts:21-47, 118-162).  The
reference's number is one snapshot of its own trajectory, so it is compared with the distribution of
snapshots here: it must lie within three standard deviations of the snapshot spread combined with the
block standard error of the mean.  Measured on a B200: 4.491 sigma (snapshot sd 0.43, block standard
error 0.063 over 80 snapshots) against the reference's 4.469, z = -0.05.
"""
import numpy as np
import pytest

import bilayer_broth as bb
from protocell_genesis_b200 import _abi, config as cfgm, observables as obs
from protocell_genesis_b200.soup import SoupSystem

pytestmark = pytest.mark.gpu

P = cfgm.load_params()
EQUILIBRATE = 2000          # tests/water-bilayer-area-move.test.ts:41 EQUILIBRATE_STEPS
RAMP, RAMP_STEPS = 20, 250  # box increments to the settled area, steps between them
SETTLE = 20000              # steps at the settled area before sampling
CHUNK = 500                 # tests/water-bilayer-area-move.test.ts:42 CHUNK_STEPS
SAMPLES = 80
BLOCKS = 8


def thickness_sample(g):
    """(thickness, amphiphiles) of the live system, as the reference's measureAll takes them."""
    particles = g.particles().reshape(-1, 4)
    n_amph, head_of = g.amphiphile_labels()
    members = np.nonzero(head_of != _abi.NONE)[0]
    polar = np.array([bool(m.get("polar")) for m in P["monomers"]])
    mp = particles[members].copy()
    mp[:, 3] = np.where(polar[np.rint(mp[:, 3]).astype(np.int64)], 0.0, 1.0)
    prof = obs.density_profile_of(mp, float(g.box[2]), 200)
    return obs.bilayer_thickness(prof), n_amph


def run_patch():
    opts, state = bb.broth_state(P)
    cfg = cfgm.resolve(cfgm.SoupOptions(**opts), P)
    assert cfg.n == 5700
    g = SoupSystem(cfg, state)
    g.step(EQUILIBRATE)
    g.scale_box_to(bb.settled_box(), RAMP, RAMP_STEPS)
    g.step(SETTLE)
    th, amph = [], []
    for _ in range(SAMPLES):
        g.step(CHUNK)
        t, a = thickness_sample(g)
        th.append(t)
        amph.append(a)
    box = [float(x) for x in g.box]
    assert g.nonfinite_count() == {"pos": 0, "vel": 0}
    events = g.events()
    g.dispose()
    return np.asarray(th), np.asarray(amph), box, events


def test_bilayer_thickness_agrees_with_the_reference_run():
    th, amph, box, events = run_patch()
    area = obs.area_per_lipid(box, bb.N_LIPIDS)
    blocks = th.reshape(BLOCKS, -1).mean(axis=1)
    mean = float(th.mean())
    sd = float(th.std(ddof=1))
    se = float(blocks.std(ddof=1) / np.sqrt(BLOCKS))
    z = (bb.THICKNESS_REFERENCE - mean) / np.hypot(sd, se)
    print(f"bilayer patch at area {area:.4f} sigma^2 (box {box[0]:.4f} x {box[1]:.4f} x {box[2]:.4f}): thickness "
          f"{mean:.4f} sigma, snapshot sd {sd:.4f}, block se {se:.4f} over {th.size} samples; reference "
          f"{bb.THICKNESS_REFERENCE:.4f} (z = {z:+.2f}); amphiphiles {amph.min()}-{amph.max()} of {bb.N_LIPIDS}; "
          f"events {events}")
    assert abs(area - bb.AREA_SETTLED) < 1e-4
    assert abs(z) < 3.0
    # one intact bilayer: the mean inside the reference's corridor (4-6 sigma, data/literature.json),
    # the amphiphiles kept (a single snapshot's peak finder can pair two maxima of one noisy leaflet,
    # which is why the comparison is on the distribution)
    assert 4.0 < mean < 6.0
    assert np.all(np.isfinite(th))
    assert amph.min() >= 350

"""Trajectory observables (engine/src/metrics.ts; soup/src/electrostatics.ts:291-303).

The per-bead reductions run on the device through the C ABI: the z histogram
(`SoupSystem.density_profile_z`, densityProfileZ) and the head pairing counts
(`SoupSystem.pairing_stats`, pairingStats).  What remains is host arithmetic on their small results
or on host arrays, written here in the reference's terms:
  area_per_lipid     engine/src/metrics.ts:8-10
  sum_profiles       engine/src/metrics.ts:52-69
  center_membrane_z  engine/src/metrics.ts:75-84
  drop_escaped_z     engine/src/metrics.ts:91-110
  bilayer_peaks      engine/src/metrics.ts:118-146 (+ subBinPeak 148-157)
  bilayer_thickness  engine/src/metrics.ts:159-162
  henderson_alpha    soup/src/electrostatics.ts:293-295
  apparent_pka       soup/src/electrostatics.ts:300-303
Errors are raised where the reference throws, with its wording.
"""
import math

import numpy as np

from . import config as _config


def area_per_lipid(box, lipids):
    """(Lx * Ly) / (lipids / 2): the projected area per lipid of a flat bilayer."""
    return (box[0] * box[1]) / (lipids / 2)


def sum_profiles(profiles):
    """Bin-by-bin sum of profiles on one z grid."""
    if not profiles:
        raise ValueError("sumProfiles: empty list of profiles")
    bins = len(profiles[0]["z"])
    head = [0] * bins
    tail = [0] * bins
    for pr in profiles:
        if len(pr["z"]) != bins or pr["z"][0] != profiles[0]["z"][0]:
            raise ValueError("sumProfiles: the profiles are built on different grids in z, so they cannot be summed")
        for i in range(bins):
            head[i] += pr["head"][i]
            tail[i] += pr["tail"][i]
    return {"z": list(profiles[0]["z"]), "head": head, "tail": tail}


def center_membrane_z(positions, box):
    """A copy of the flat x,y,z,w array with every z shifted so the mean z sits at box_z / 2."""
    p = np.array(positions, dtype=np.float32).reshape(-1, 4)
    shift = box[2] / 2 - float(np.sum(p[:, 2].astype(np.float64))) / len(p)
    out = p.copy()
    out[:, 2] = (p[:, 2].astype(np.float64) + shift).astype(np.float32)
    return out.reshape(-1)


def drop_escaped_z(positions, box):
    """(positions inside [0, box_z), number left out)."""
    p = np.asarray(positions, dtype=np.float32).reshape(-1, 4)
    z = p[:, 2].astype(np.float64)
    keep = (z >= 0) & (z < box[2])
    return p[keep].reshape(-1).copy(), int((~keep).sum())


def _sub_bin_peak(values, z, i):
    """Three-point parabola through the peak bin and its neighbours, offset clamped to half a bin."""
    if i == 0 or i == len(values) - 1 or len(z) < 2:
        return z[i]
    dz = z[1] - z[0]
    denom = values[i - 1] - 2 * values[i] + values[i + 1]
    if denom >= 0:
        return z[i]
    offset = (0.5 * (values[i - 1] - values[i + 1])) / denom
    return z[i] + max(-0.5, min(0.5, offset)) * dz


def bilayer_peaks(profile, min_separation=None):
    """The two most prominent head-density maxima at least one sigma apart: the global maximum, then
    the maximum of what is left after zeroing +-1 sigma around it."""
    head, z = profile["head"], profile["z"]
    if min_separation is None:
        min_separation = _config.load_params()["params"]["sigma"]
    a = 0
    for i in range(1, len(head)):
        if head[i] > head[a]:
            a = i
    if head[a] == 0:
        raise ValueError("bilayerPeaks: the head profile is empty, there are no peaks")
    masked = [0 if abs(z[i] - z[a]) <= min_separation else v for i, v in enumerate(head)]
    b = 0
    for i in range(1, len(masked)):
        if masked[i] > masked[b]:
            b = i
    if masked[b] == 0:
        raise ValueError(f"bilayerPeaks: second peak not found: all heads lie within {min_separation} of the "
                         f"maximum at z={z[a]}; this is not a bilayer")
    za = _sub_bin_peak(head, z, a)
    zb = _sub_bin_peak(head, z, b)
    return {"lower": za, "upper": zb} if za <= zb else {"lower": zb, "upper": za}


def bilayer_thickness(profile, min_separation=None):
    """Distance between the two head-density peaks."""
    p = bilayer_peaks(profile, min_separation)
    return p["upper"] - p["lower"]


def henderson_alpha(ph, pka):
    """Deprotonated fraction of an isolated acid: 1 / (1 + 10^(pKa - pH))."""
    return 1 / (1 + math.pow(10, pka - ph))


def apparent_pka(alpha, ph):
    """Henderson-Hasselbalch read backwards; NaN outside (0, 1)."""
    if alpha <= 0 or alpha >= 1:
        return math.nan
    return ph - math.log10(alpha / (1 - alpha))


# reference-style names
areaPerLipid = area_per_lipid
sumProfiles = sum_profiles
centerMembraneZ = center_membrane_z
dropEscapedZ = drop_escaped_z
bilayerPeaks = bilayer_peaks
bilayerThickness = bilayer_thickness
hendersonAlpha = henderson_alpha
apparentPKa = apparent_pka

"""Trajectory observables (engine/src/metrics.ts; soup/src/electrostatics.ts:291-303).

The per-bead reductions run on the device through the C ABI: the z histogram
(`SoupSystem.density_profile_z`, densityProfileZ) and the head pairing counts
(`SoupSystem.pairing_stats`, pairingStats).  What remains is host arithmetic on their small results
or on host arrays, written here in the reference's terms:
  area_per_lipid     engine/src/metrics.ts:8-10
  sum_profiles       engine/src/metrics.ts:52-69
  center_membrane_z  engine/src/metrics.ts:75-84
  periodic_centre    soup/src/water-closure.ts:63-97 (periodicCentreOf, circularAxisStat)
  drop_escaped_z     engine/src/metrics.ts:91-110
  bilayer_peaks      engine/src/metrics.ts:118-146 (+ subBinPeak 148-157)
  bilayer_thickness  engine/src/metrics.ts:159-162
  henderson_alpha    soup/src/electrostatics.ts:293-295
  apparent_pka       soup/src/electrostatics.ts:300-303
  shape_metrics      engine/src/aggregate.ts:268-346 (symmetricEigenvalues3x3, symmetricEigenvector3x3,
                     shapeOf's derived numbers; the sums come from SoupSystem.aggregate_shapes)
  analyze_aggregates soup/src/aggregates.ts:499-558, the counting and shape parts
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


def periodic_centre(positions, idx, box, alpha):
    """periodicCentreOf (soup/src/water-closure.ts:63-97): per axis the circular mean of the members'
    wrapped coordinates (angle 2 pi x / L); None when the mean resultant length R falls below the
    Rayleigh bound sqrt(-ln(alpha) / m) on any axis (no meaningful centre)."""
    p = np.asarray(positions, np.float32).reshape(-1, 4)[np.asarray(idx, np.int64), :3].astype(np.float64)
    m = len(p)
    if m == 0:
        return None
    out = []
    for a in range(3):
        L = float(box[a])
        x = p[:, a] - np.floor(p[:, a] / L) * L
        th = 2.0 * math.pi * x / L
        sc, ss = float(np.cos(th).mean()), float(np.sin(th).mean())
        R = math.sqrt(sc * sc + ss * ss)
        if not R >= math.sqrt(-math.log(alpha) / m):
            return None
        c = math.atan2(ss, sc) / (2.0 * math.pi) * L
        out.append(c - math.floor(c / L) * L)
    return out


def symmetric_eigenvalues_3x3(sxx, syy, szz, sxy, sxz, syz):
    """Ascending eigenvalues of a real symmetric 3x3 matrix by Smith's closed form (O. K. Smith,
    "Eigenvalues of a symmetric 3x3 matrix", CACM 4(4):168, 1961): shift by the mean eigenvalue q,
    scale by p = sqrt(|A - qI|_F^2 / 6), and read the three angles off acos(det(B) / 2) / 3.  A
    diagonal matrix (off-diagonal norm below 1e-30) is sorted directly."""
    p1 = sxy * sxy + sxz * sxz + syz * syz
    if p1 < 1e-30:
        return sorted([sxx, syy, szz])
    q = (sxx + syy + szz) / 3
    p2 = (sxx - q) ** 2 + (syy - q) ** 2 + (szz - q) ** 2 + 2 * p1
    p = math.sqrt(p2 / 6)
    bxx, byy, bzz = (sxx - q) / p, (syy - q) / p, (szz - q) / p
    bxy, bxz, byz = sxy / p, sxz / p, syz / p
    det = bxx * (byy * bzz - byz * byz) - bxy * (bxy * bzz - byz * bxz) + bxz * (bxy * byz - byy * bxz)
    phi = math.acos(max(-1.0, min(1.0, det / 2))) / 3
    largest = q + 2 * p * math.cos(phi)
    smallest = q + 2 * p * math.cos(phi + 2 * math.pi / 3)
    return sorted([smallest, 3 * q - largest - smallest, largest])


def symmetric_eigenvector_3x3(sxx, syy, szz, sxy, sxz, syz, lam):
    """Unit eigenvector of one eigenvalue: the largest cross product of two rows of (A - lam I), or
    None when every pair degenerates (magnitude below 1e-9: a repeated eigenvalue)."""
    r = [(sxx - lam, sxy, sxz), (sxy, syy - lam, syz), (sxz, syz, szz - lam)]

    def cross(a, b):
        return (a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0])

    best, best_mag = None, -1.0
    for a, b in ((0, 1), (0, 2), (1, 2)):
        c = cross(r[a], r[b])
        m = math.sqrt(c[0] ** 2 + c[1] ** 2 + c[2] ** 2)
        if m > best_mag:
            best, best_mag = c, m
    if best_mag < 1e-9:
        return None
    return [best[0] / best_mag, best[1] / best_mag, best[2] / best_mag]


def shape_metrics(shape):
    """shapeOf's numbers from one device shape {size, label, centre, gyration}: principal moments
    (ascending), radius of gyration, the smallest-moment axis ([0, 0, 1] when not unique), and the
    flatness (l0 / l2) and in-plane symmetry (l1 / l2) ratios shapeOfAggregate reports."""
    g = shape["gyration"]
    lam = symmetric_eigenvalues_3x3(*g)
    axis = symmetric_eigenvector_3x3(*g, lam[0]) or [0.0, 0.0, 1.0]
    l0, l1, l2 = lam
    return {"size": shape["size"], "label": shape["label"], "centre": list(shape["centre"]),
            "principalMoments": lam, "radiusOfGyration": math.sqrt(max(0.0, l0 + l1 + l2)), "smallestAxis": axis,
            "flatnessRatio": l0 / l2 if l2 > 1e-12 else 1.0, "inPlaneSymmetry": l1 / l2 if l2 > 1e-12 else 1.0}


HEAD_PEAKS_UNAVAILABLE = "unavailable"


def density_profile_of(positions, box_z, bins):
    """densityProfileZ (engine/src/metrics.ts:21-47) of f32 x4 positions whose w is 0 for a head:
    z histogram over [0, box_z) in `bins` bins, heads and tails apart; a z outside raises."""
    p = np.asarray(positions, np.float32).reshape(-1, 4)
    z = p[:, 2].astype(np.float64)
    bad = ~((z >= 0) & (z < box_z))
    if bad.any():
        raise ValueError(f"densityProfileZ: bead with z={z[bad][0]} outside [0, {box_z}): the z profile is undefined "
                         f"for escaped beads (z is not periodic), and clamping them into the edge bin is not allowed: "
                         f"it creates a false peak")
    dz = box_z / bins
    b = np.minimum(bins - 1, np.floor(z / dz)).astype(np.int64)
    head = p[:, 3] == 0
    return {"z": [(i + 0.5) * dz for i in range(bins)],
            "head": np.bincount(b[head], minlength=bins).astype(np.int64).tolist(),
            "tail": np.bincount(b[~head], minlength=bins).astype(np.int64).tolist()}


def compute_head_peaks(particles, box, polar, bins, min_heads_per_bin, sep_min, sep_max):
    """computeHeadPeaks (soup/src/aggregates.ts:83-120): 0 without polar beads; "unavailable" when
    fewer than min_heads_per_bin heads per bin remain after dropping escaped z; 2 when the head profile
    has two peaks min..max apart (bilayerThickness); 1 otherwise.  `polar[k]`: kind k is polar."""
    p = np.asarray(particles, np.float32).reshape(-1, 4)
    kinds = np.rint(p[:, 3]).astype(np.int64)
    is_head = np.array([bool(polar[k]) if 0 <= k < len(polar) else False for k in kinds], bool)
    if not is_head.any():
        return 0
    remapped = p.copy()
    remapped[:, 3] = np.where(is_head, 0.0, 1.0)
    kept, _ = drop_escaped_z(remapped.reshape(-1), box)
    kept_heads = int((kept.reshape(-1, 4)[:, 3] == 0).sum())
    if kept_heads == 0 or kept_heads / bins < min_heads_per_bin:
        return HEAD_PEAKS_UNAVAILABLE
    profile = density_profile_of(kept, box[2], bins)
    try:
        sep = bilayer_thickness(profile)
    except ValueError:
        return 1
    return 2 if sep_min <= sep <= sep_max else 1


def profile_along(coords, kinds):
    """profileAlong (soup/src/aggregates.ts:324-347): a coordinate per bead packed into z (shifted to
    start at 0, rounded to f32) with the bead's kind, in a [1, 1, span] box."""
    c = np.asarray(coords, np.float64)
    lo, hi = float(c.min()), float(c.max())
    span = max(1e-6, (hi - lo) * 1.0001)
    p = np.zeros((c.size, 4), np.float32)
    p[:, 2] = (c - lo).astype(np.float32)
    p[:, 3] = np.asarray(kinds, np.float32)
    return p.reshape(-1), [1.0, 1.0, span]


def is_lamellar_shape(shape, t):
    """isLamellarShape (soup/src/aggregates.ts:273-282)."""
    return shape["flatnessRatio"] <= t["lamellarFlatnessRatio"] and shape["inPlaneSymmetry"] >= t["lamellarInPlaneSymmetryMin"]


def is_bilayer_shape(shape, t):
    """isBilayerShape (soup/src/aggregates.ts:284-290)."""
    return is_lamellar_shape(shape, t) and (shape["radialHeadShells"] == 2 or shape["transverseHeadShells"] == 2)


def is_vesicle_shape(shape, t):
    """isVesicleShape (soup/src/aggregates.ts:307-315): two radial head shells and a closed interior,
    by encapsulated water when water was measured (None: the centre could not be trusted, not
    closed), else by the vacuum cavity."""
    if shape["radialHeadShells"] != 2:
        return False
    if "encapsulatedWater" in shape:
        return shape["encapsulatedWater"] is not None and bool(shape["encapsulatedWater"]["closed"])
    return shape["cavityVolume"] > t["enclosedVolume"]


def shape_of_aggregate(system, members, amphiphile_count, device_shape, thresholds, positions=None, water=None,
                       parcel=None):
    """shapeOfAggregate (soup/src/aggregates.ts:387-476) of one aggregate (members ascending, the
    first the unwrap reference) on a device system: shapeOf from the device gyration tensor, the
    radial and (for a flat shape) transverse head-shell counts from the device-unwrapped members, the
    vacuum cavity of the device local flood, and, when water indices are given, the encapsulated
    water of the device periodic closure about the periodic centre."""
    P = _config.load_params()
    t = thresholds
    polar = [bool(m["polar"]) for m in P["monomers"]]
    sh = shape_metrics(device_shape)
    unwrapped = system.aggregate_unwrap(members).reshape(-1, 4)
    kinds = unwrapped[:, 3]
    d = unwrapped[:, :3].astype(np.float64) - np.asarray(sh["centre"], np.float64)
    hp = (t["aggregateHeadDensityBins"], t["aggregateMinHeadsPerBin"], t["headPeakSeparationMin"],
          t["headPeakSeparationMax"])
    rad, rbox = profile_along(np.sqrt((d * d).sum(axis=1)), kinds)
    out = dict(sh)
    out.update(particleCount=int(len(members)), amphiphileCount=int(amphiphile_count))
    out["radialHeadShells"] = compute_head_peaks(rad, rbox, polar, *hp)
    out["transverseHeadShells"] = 0
    if is_lamellar_shape(out, t):
        ax = np.asarray(sh["smallestAxis"], np.float64)
        tr, tbox = profile_along(d[:, 0] * ax[0] + d[:, 1] * ax[1] + d[:, 2] * ax[2], kinds)
        out["transverseHeadShells"] = compute_head_peaks(tr, tbox, polar, *hp)
    out["cavityVolume"] = system.local_cavity_volume(unwrapped.reshape(-1), t["closureCell"], t["closureRadius"])
    if water is not None and len(water) > 0:
        pos = system.particles() if positions is None else positions
        c = periodic_centre(pos, members, system.box, P["circularAlpha"])
        out["encapsulatedWater"] = None if c is None else system.closure(
            members, water, c, t["closureCell"], t["closureRadius"], t["enclosedVolume"], parcel)
    return out


def analyze_aggregates(system, cutoff, detail_count=None, min_amphiphiles_per_aggregate=None, thresholds=None,
                       water=None, parcel=None):
    """analyzeAggregates (soup/src/aggregates.ts:499-558) on a device system: amphiphiles
    (findAmphiphiles), their members clustered by `cutoff` on all three periodic axes, amphiphiles per
    aggregate (largest aggregate first), the qualifying aggregates, shapeOfAggregate for the largest
    `detail_count`, and whether any of them reads as lamellar (bilayer) or as a vesicle.  Thresholds
    default to the parameter tables' stage thresholds; `water`: the water indices, for the closure;
    `parcel`: {"centre", "radius"} of a confined run, for the closure's bulk density."""
    t = dict(_config.load_params()["stageThresholds"])
    t.update(thresholds or {})
    if detail_count is not None:
        t["detailAggregateCount"] = detail_count
    if min_amphiphiles_per_aggregate is not None:
        t["minAmphiphilesPerAggregate"] = min_amphiphiles_per_aggregate
    n_amph, head_of = system.amphiphile_labels()
    none = 0xFFFFFFFF
    members = np.nonzero(head_of != none)[0].astype(np.uint32)
    empty = {"aggregateCount": 0, "sizeHistogram": [], "aggregates": [], "qualifyingAggregateCount": 0,
             "amphiphilesInQualifying": 0, "amphiphileShareInQualifying": 0.0, "hasLamellarAggregate": False,
             "hasVesicleAggregate": False}
    if members.size == 0:
        return empty
    _, labels = system.aggregate_labels(members, cutoff)
    ncomp, shapes = system.aggregate_shapes(members, labels, max(int(t["detailAggregateCount"]), 0))
    # amphiphiles per component: its members that are their amphiphile's head
    is_head = head_of[members] == members
    uniq, inv = np.unique(labels, return_inverse=True)
    size = np.bincount(inv)
    heads = np.bincount(inv, weights=is_head).astype(np.int64)
    order = sorted(range(len(uniq)), key=lambda c: (-int(size[c]), int(uniq[c])))
    hist = [int(heads[c]) for c in order]
    qual = [h for h in hist if h >= t["minAmphiphilesPerAggregate"]]
    total = int(n_amph)
    pos = system.particles() if water is not None else None
    detail = []
    for k, shp in enumerate(shapes):
        c = order[k]
        detail.append(shape_of_aggregate(system, members[inv == c], int(heads[c]), shp, t, pos, water, parcel))
    return {"aggregateCount": int(ncomp), "sizeHistogram": hist, "aggregates": detail,
            "qualifyingAggregateCount": len(qual), "amphiphilesInQualifying": int(sum(qual)),
            "amphiphileShareInQualifying": (sum(qual) / total) if total > 0 else 0.0,
            "hasLamellarAggregate": any(is_bilayer_shape(a, t) for a in detail),
            "hasVesicleAggregate": any(is_vesicle_shape(a, t) for a in detail)}


# reference-style names
areaPerLipid = area_per_lipid
sumProfiles = sum_profiles
centerMembraneZ = center_membrane_z
periodicCentreOf = periodic_centre
dropEscapedZ = drop_escaped_z
bilayerPeaks = bilayer_peaks
bilayerThickness = bilayer_thickness
hendersonAlpha = henderson_alpha
apparentPKa = apparent_pka
symmetricEigenvalues3x3 = symmetric_eigenvalues_3x3
analyzeAggregates = analyze_aggregates
computeHeadPeaks = compute_head_peaks
isLamellarShape = is_lamellar_shape
isBilayerShape = is_bilayer_shape
isVesicleShape = is_vesicle_shape

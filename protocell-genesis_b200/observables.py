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


STAGES = ("monomers", "amphiphiles", "micelles", "bilayer", "vesicle")


def _js_round(x):
    """JavaScript Math.round on float64: to the nearest integer, halves toward +infinity."""
    f = np.floor(x)
    return f + ((x - f) >= 0.5)


def _wrap1(v, box):
    return v - np.floor(v / box) * box


def largest_cluster_shift(positions, labels, box):
    """largestClusterShift + largestClusterCenter (engine/src/closure.ts:291-296,
    engine/src/aggregate.ts:157-190) from the members' component labels, in the members' order: the
    largest component (ties to the one met first), its x, y centre as minimum-image offsets from its
    first member summed in order, its plain z mean; the shift that puts that centre at the box's
    middle.  positions: f32 x4 of the members in that order."""
    p = np.asarray(positions, np.float32).reshape(-1, 4).astype(np.float64)
    lab = np.asarray(labels)
    if lab.size == 0:
        raise ValueError("largestClusterCenter: empty set of beads")
    uniq, first, size = np.unique(lab, return_index=True, return_counts=True)
    best = uniq[min(range(uniq.size), key=lambda c: (-int(size[c]), int(first[c])))]
    idx = np.nonzero(lab == best)[0]
    box = [float(b) for b in box]
    ref_x, ref_y = p[idx[0], 0], p[idx[0], 1]
    dx = p[idx, 0] - ref_x
    dy = p[idx, 1] - ref_y
    sx = np.cumsum(dx - _js_round(dx / box[0]) * box[0])[-1]   # sequential, as the reference sums
    sy = np.cumsum(dy - _js_round(dy / box[1]) * box[1])[-1]
    sz = np.cumsum(p[idx, 2])[-1]
    n = float(idx.size)
    com = (_wrap1(ref_x + sx / n, box[0]), _wrap1(ref_y + sy / n, box[1]), sz / n)
    return (box[0] / 2 - com[0], box[1] / 2 - com[1], box[2] / 2 - com[2])


def recenter_positions(positions, shift, box):
    """recenterOnLargestCluster's translation (engine/src/closure.ts:298-309): x, y shifted and wrapped,
    z shifted only, in float64 and stored as f32."""
    p = np.asarray(positions, np.float32).reshape(-1, 4)
    out = p.copy()
    for a in range(2):
        out[:, a] = _wrap1(p[:, a].astype(np.float64) + shift[a], float(box[a])).astype(np.float32)
    out[:, 2] = (p[:, 2].astype(np.float64) + shift[2]).astype(np.float32)
    return out.reshape(-1)


def enclosed_volume_from_positions(system, members, particles, cell, radius):
    """enclosedVolumeFromPositions (engine/src/closure.ts:315-323) over the given member beads of a
    device system: clustered with z open at the tail-tail attraction range (closure.ts:291-296) on the
    device, recentred on the largest cluster, then the box-grid occupancy and flood on the device."""
    P = _config.load_params()
    m = np.ascontiguousarray(members, np.uint32)
    if m.size == 0:
        return 0.0
    cutoff = _config.wca_cutoff(P["params"]["beadSizes"]["tail_tail"]) + P["params"]["wc"]
    _, labels = system.cluster_labels(m, cutoff, periodic_z=False)
    pos = np.asarray(particles, np.float32).reshape(-1, 4)[m]
    box = system.box
    shift = largest_cluster_shift(pos, labels, box)
    return system.box_cavity_volume(recenter_positions(pos, shift, box), cell, radius)


def load_stage_thresholds():
    """loadStageThresholds (soup/src/stages.ts:130-170): the stage thresholds of the parameter
    tables.  The tables are generated from the reference's data files, so the two cross-checks the
    reference makes there (the closure minimum against the literature table, and the minimum
    amphiphiles per aggregate against its formula) held when they were written."""
    return dict(_config.load_params()["stageThresholds"])


def stage_from_evidence(evidence, thresholds):
    """stageFromEvidence (soup/src/stages.ts:184-202): every stage above monomers needs the amphiphile
    fraction; vesicle, bilayer and micelles are then checked in that order on the per-aggregate
    analysis."""
    a = evidence["aggregateAnalysis"]
    amphiphile_ok = evidence["amphiphileFraction"] >= thresholds["amphiphileFraction"]
    micelle_ok = (amphiphile_ok and a["qualifyingAggregateCount"] >= thresholds["minMicelleAggregates"]
                  and a["amphiphileShareInQualifying"] >= thresholds["minAmphiphileShareInAggregates"])
    if amphiphile_ok and a["hasVesicleAggregate"]:
        return "vesicle"
    if amphiphile_ok and a["hasLamellarAggregate"]:
        return "bilayer"
    if micelle_ok:
        return "micelles"
    if amphiphile_ok:
        return "amphiphiles"
    return "monomers"


def _member_order(head_of, members):
    """memberIndicesOf (soup/src/aggregates.ts:122-129) order: amphiphiles by the smallest index of
    their component (findAmphiphiles' order), each as its head then its other members.  The reference
    lists a chain in walk order; ascending order here changes only the rounding of the recentring's
    centre sum, whose first member (the head) is the same."""
    heads = head_of[members]
    uh, first = np.unique(heads, return_index=True)
    rank = np.empty(uh.size, np.int64)
    rank[np.argsort(first)] = np.arange(uh.size)
    group = rank[np.searchsorted(uh, heads)]
    not_head = (heads != members).astype(np.int64)
    return members[np.lexsort((members, not_head, group))]


def detect_stage(system, thresholds=None, parcel=None):
    """detectStage (soup/src/stages.ts:204-289) on a device system: {"stage", "evidence"} with the
    amphiphile fraction (carbon beads in a recognised chain over all carbon beads), the largest
    aggregate's share of the amphiphile members (z periodic), the box-wide head-peak count and
    enclosed volume (diagnostics), and analyzeAggregates with the water beads.  `parcel`: {"centre",
    "radius"} of a confined run; when it is not given, it is read off the system's live confinement
    as stages.ts:274-279 does (the box centre and the live wall radius; None on a periodic system)."""
    if parcel is None and hasattr(system, "confinement"):
        cf = system.confinement()
        if cf is not None:
            b = cf["boxLive"]
            parcel = {"centre": [b[0] / 2, b[1] / 2, b[2] / 2], "radius": float(cf["radiusLive"])}
    P = _config.load_params()
    t = load_stage_thresholds()
    t.update(thresholds or {})
    mon = P["monomers"]
    particles = system.particles()
    kinds = np.rint(np.asarray(particles, np.float32).reshape(-1, 4)[:, 3]).astype(np.int64)
    n_amph, head_of = system.amphiphile_labels()
    members = np.nonzero(head_of != 0xFFFFFFFF)[0].astype(np.uint32)
    carbon = [k for k, m in enumerate(mon) if m["kind"] == "carbon"]
    total_carbon = int(np.isin(kinds, carbon).sum())
    in_chains = int(members.size) - int(n_amph)
    radii = [m["radiusSigma"] for m in mon if m["kind"] in ("carbon", "head")]
    cutoff = _config.wca_cutoff(P["params"]["sigma"] * max(radii)) + P["params"]["wc"]
    largest = 0.0
    enclosed = 0.0
    if members.size:
        _, lab = system.aggregate_labels(members, cutoff)
        largest = float(np.unique(lab, return_counts=True)[1].max()) / members.size
        enclosed = enclosed_volume_from_positions(system, _member_order(head_of, members), particles,
                                                  t["closureCell"], t["closureRadius"])
    polar = [bool(m["polar"]) for m in mon]
    peaks = compute_head_peaks(particles, system.box, polar, t["headDensityBins"], t["minHeadsPerBin"],
                               t["headPeakSeparationMin"], t["headPeakSeparationMax"])
    water_kind = next((k for k, m in enumerate(mon) if m.get("solvent")), None)
    water = None if water_kind is None else np.nonzero(kinds == water_kind)[0].astype(np.uint32)
    analysis = analyze_aggregates(system, cutoff, thresholds=t,
                                  water=water if water is not None and water.size else None, parcel=parcel)
    evidence = {"amphiphileFraction": in_chains / total_carbon if total_carbon > 0 else 0.0,
                "largestAggregateFraction": largest, "headPeaks": peaks, "enclosedVolume": enclosed,
                "aggregateAnalysis": analysis}
    return {"stage": stage_from_evidence(evidence, t), "evidence": evidence}


# reference-style names
loadStageThresholds = load_stage_thresholds
stageFromEvidence = stage_from_evidence
detectStage = detect_stage
enclosedVolumeFromPositions = enclosed_volume_from_positions
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

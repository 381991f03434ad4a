"""Resolve CreateSoupOpts-style options into a SoupConfig.

This is the host-side half of the reference's createSoup (soup/src/sim.ts:95-330): everything it
derives on the CPU before the first dispatch -- grid geometry and its refusals
(soup/src/soup-plan.ts:76-157), the Verlet list capacity (soup-plan.ts:160-191), the
electrostatics basis (soup/src/electrostatics.ts:166-247 makeEsBasis), the bond-rule uniforms
(soup/src/soup-plan.ts:22-49 resolveRules, soup/src/soup-buffers.ts:344-410, soup/src/rules.ts:576-591)
and the class-pair attraction table (soup/src/soup-attraction.ts attractionScaleTable /
acidSoapScaleOf).  The numbers come from soup_params.json, which is generated from the
reference's data/params.json and data/soup.json by data/make_params.py.
"""
import json
import math
import os
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

from . import _abi

_HERE = os.path.dirname(os.path.abspath(__file__))
CLASS_NAMES = ("apolar", "polar", "solvent", "mineral")


def load_params(path: Optional[str] = None) -> dict:
    with open(path or os.path.join(_HERE, "data", "soup_params.json")) as fh:
        return json.load(fh)


def wca_cutoff(b: float) -> float:
    """engine/src/params.ts:31 wcaCutoff: 2^(1/6) b."""
    return math.pow(2.0, 1.0 / 6.0) * b


def species_class(m: dict) -> int:
    """soup/src/soup-attraction.ts speciesClassOf."""
    if m.get("mineral"):
        return 3
    if m.get("solvent"):
        return 2
    if m.get("polar"):
        return 1
    return 0


def _pair_key(ci: int, cj: int) -> str:
    hi = CLASS_NAMES[max(ci, cj)]
    lo = CLASS_NAMES[min(ci, cj)]
    return hi + lo[0].upper() + lo[1:]


def attraction_table(P: dict, override: Optional[float] = None) -> List[List[float]]:
    """soup/src/soup-attraction.ts attractionScaleTable (pairEpsilon branch)."""
    at = P["attraction"]
    glob = override if override is not None else at.get("epsilonScale", 1.0)
    if not (math.isfinite(glob) and glob > 0):
        raise ValueError(f"soup attraction: epsilonScale={glob} must be a finite positive number")
    ref = at["levelsKJ"][at["reference"]]
    table = [[0.0] * 4 for _ in range(4)]
    for ci in range(4):
        for cj in range(4):
            key = _pair_key(ci, cj)
            if ci == 3 or cj == 3:
                key = at["mineralPairAlias"].get(key, key)
            table[ci][cj] = (glob * at["levelsKJ"][key]) / ref
    return table


def acid_soap_scale(P: dict, override: Optional[float] = None, eps_override: Optional[float] = None) -> float:
    """soup/src/soup-attraction.ts acidSoapScaleOf."""
    if override is not None:
        if not (math.isfinite(override) and override >= 0):
            raise ValueError(f"soup attraction: acidSoapScaleOverride={override} must be a finite non-negative number")
        return float(override)
    at = P["attraction"]
    ref = at["levelsKJ"][at["reference"]]
    glob = eps_override if eps_override is not None else at.get("epsilonScale", 1.0)
    return (glob * at.get("acidSoapPairKJ", 0.0)) / ref


def slot_role(this_kind: str, other_kind: str) -> int:
    """soup/src/soup-plan.ts slotRole."""
    if this_kind == "carbon":
        return 0 if other_kind == "carbon" else 1
    if this_kind == "head":
        return 2
    raise ValueError(f'a rule bonds a monomer of kind "{this_kind}", but only carbon and head are supported')


@dataclass
class EsBasis:
    """soup/src/electrostatics.ts:77-131 EsBasis (the fields the step uses)."""
    enabled: bool
    charged_kind: int
    charge_deprotonated: float
    coeff_a: float
    kappa: float
    cutoff: float
    nb_cutoff: float
    split_radius: float
    list_range: float
    list_capacity: int
    shift_u: float
    shift_f: float
    pka: float
    ph: float
    ionic_strength: float
    debye_sigma: float
    sweep_every: int
    kT: float
    acid_soap: float
    rc_attr: float
    wc: float
    epsilon: float


def make_es_basis(P: dict, kT: float, over: Optional[dict] = None) -> EsBasis:
    """soup/src/electrostatics.ts:166-247 makeEsBasis."""
    over = over or {}
    p = P["params"]
    es = P["electrostatics"]
    cutoff_nb = wca_cutoff(p["sigma"] * p["beadSizes"]["tail_tail"]) + p["wc"]
    inter = wca_cutoff(p["sigma"] * max(m["radiusSigma"] for m in P["monomers"])) + p["wc"]
    enabled = over.get("enabled", es["enabled"])
    ph = over.get("pH", es["pH"])
    ionic = over.get("ionicStrengthMolar", es["ionicStrengthMolar"])
    ids = [m["id"] for m in P["monomers"]]
    if es["chargedKind"] not in ids:
        raise ValueError(f"electrostatics.chargedKind='{es['chargedKind']}' is not among monomers")
    charged_kind = ids.index(es["chargedKind"])
    if not (ionic > 0):
        raise ValueError(f"electrostatics: ionicStrengthMolar must be > 0, given {ionic}")
    sigma_nm = es["sigmaToNm"]
    debye = es["debyeLengthNmAtUnitMolar"] / math.sqrt(ionic) / sigma_nm
    coeff_a = kT * (es["bjerrumLengthNm"] / sigma_nm) if enabled else 0.0
    kappa = 1.0 / debye
    target = es["longRangeDebyeLengths"] * debye
    min_box = over.get("minBoxSigma")
    image_cap = es["longRangeMaxBoxFraction"] * min_box if min_box is not None else math.inf
    es_cut = over["cutoffSigma"] if over.get("cutoffSigma") is not None else max(cutoff_nb, min(target, image_cap))
    if min_box is not None and es_cut > min_box / 2:
        raise ValueError(
            f"electrostatics: the cutoff rc_es={es_cut:.6f} violates the minimum image convention at "
            f"min(box)={min_box:.4f} (need rc_es <= {min_box / 2:.4f})"
        )
    skin = P["verletList"]["skin"] if over.get("skin") is None else over["skin"]
    list_range = es_cut + skin
    cap = es["longRangeListCapacity"]
    max_heads = over.get("maxHeads")
    if max_heads is not None and max_heads > 0 and min_box is not None:
        dv = over.get("densityVolumeSigma3")
        denom = dv if (dv is not None and dv > 0) else min_box ** 3
        uniform = (4 * math.pi / 3) * list_range ** 3 * (max_heads / denom)
        cap = max(64, min(max_heads, math.ceil(es["longRangeListSafetyFactor"] * uniform)))
    shift_u = coeff_a * math.exp(-kappa * es_cut) / es_cut
    shift_f = shift_u * (1 / es_cut + kappa)
    return EsBasis(
        enabled=bool(enabled), charged_kind=charged_kind, charge_deprotonated=float(es["chargeDeprotonated"]),
        coeff_a=coeff_a, kappa=kappa, cutoff=es_cut, nb_cutoff=cutoff_nb, split_radius=inter,
        list_range=list_range, list_capacity=int(cap), shift_u=shift_u, shift_f=shift_f,
        pka=es["pKaIntrinsic"], ph=ph, ionic_strength=ionic, debye_sigma=debye,
        sweep_every=int(over.get("sweepEverySteps", es["sweepEverySteps"])), kT=kT,
        acid_soap=acid_soap_scale(P, over.get("acidSoapScale")),
        rc_attr=wca_cutoff(p["sigma"] * p["beadSizes"]["tail_tail"]), wc=p["wc"], epsilon=p["epsilon"],
    )


def es_pair_energy(r: float, qq: float, b: EsBasis) -> float:
    """soup/src/electrostatics.ts:277-281 esPairEnergy."""
    if b.coeff_a == 0 or qq == 0 or r >= b.cutoff or r <= 0:
        return 0.0
    u1 = (b.coeff_a * math.exp(-b.kappa * r)) / r
    return qq * (u1 - b.shift_u + b.shift_f * (r - b.cutoff))


def es_pair_force_mag(r: float, qq: float, b: EsBasis) -> float:
    """soup/src/electrostatics.ts:285-289 esPairForceMag."""
    if b.coeff_a == 0 or qq == 0 or r >= b.cutoff or r <= 0:
        return 0.0
    u1 = (b.coeff_a * math.exp(-b.kappa * r)) / r
    return qq * (u1 * (1 / r + b.kappa) - b.shift_f)


def acid_soap_well(r: float, b: EsBasis) -> float:
    """soup/src/acid-soap.ts acidSoapWell."""
    if b.acid_soap <= 0:
        return 0.0
    if r < b.rc_attr:
        return -b.acid_soap * b.epsilon
    if r > b.rc_attr + b.wc:
        return 0.0
    c = math.cos((math.pi * (r - b.rc_attr)) / (2 * b.wc))
    return -b.acid_soap * b.epsilon * c * c


@dataclass
class Plan:
    """soup/src/soup-plan.ts GridGeometry + SoupPlan, plus the derived list capacity."""
    n: int
    counts: List[int]
    interaction_range: float
    cell_size: float
    walk_radius: int
    list_range: float
    list_walk_radius: int
    dims: List[int]
    list_capacity: int
    uniform_expected: float


def derive_plan(P: dict, box: Sequence[float], counts: List[int], kT: float, skin: float,
                rebuild_every: int, fixed_cadence: bool, list_capacity: Optional[int] = None,
                density_volume: Optional[float] = None) -> Plan:
    """deriveGridGeometry + planSoupGrid + deriveListCapacity (soup/src/soup-plan.ts:76-191)."""
    p = P["params"]
    max_r = max(m["radiusSigma"] for m in P["monomers"])
    inter = wca_cutoff(p["sigma"] * max_r) + p["wc"]
    cell = inter / P["neighborGrid"]["cellDivisor"]
    walk = math.ceil(inter / cell)
    if walk * cell < inter - 1e-6:
        raise GeometryError(f"neighbour grid: walkRadius={walk} * cellSize={cell:.6f} does not cover interactionRange={inter:.6f}")
    list_range = inter + skin
    lwalk = math.ceil(list_range / cell)
    if lwalk * cell < list_range - 1e-6:
        raise GeometryError(f"Verlet list: listBuildWalkRadius={lwalk} does not cover listRange={list_range:.6f}")
    if fixed_cadence:
        v_bound = 2 * math.sqrt(3 * kT)
        drift_bound = 2 * rebuild_every * p["dt"] * v_bound
        if drift_bound > skin:
            raise GeometryError(
                f"Verlet list: 2*rebuildEvery*dt*vBound={drift_bound:.4f} exceeds skin={skin} at kT={kT}: "
                f"the rebuild is not frequent enough (or skin is too small) for this temperature"
            )
    dims = [max(1, math.floor(b / cell)) for b in box]
    min_cells = 2 * lwalk + 1
    if not (all(d >= min_cells for d in dims) and min(box) / 2 > p["bend"]["r0"]):
        raise GeometryError(
            f"neighbour grid: box=[{box[0]},{box[1]},{box[2]}] gives cellSize={cell:.4f}, dims={dims} and "
            f"min(box)/2={min(box) / 2:.4f}; it needs dims>={min_cells} (2*effectiveWalkRadius+1) on all "
            f"three axes and min(box)/2 > bend.r0={p['bend']['r0']}"
        )
    n = sum(counts)
    vol = density_volume if density_volume else box[0] * box[1] * box[2]
    dens = n / vol
    vl = P["verletList"]
    uniform = (4 * math.pi / 3) * list_range ** 3 * dens
    if list_capacity is None:
        if n > 0 and dens > 0:
            list_capacity = max(64, min(n, max(vl["capacityFloor"], math.ceil(vl["capacitySafetyFactor"] * uniform))))
        else:
            list_capacity = vl["listCapacity"]
    return Plan(n=n, counts=list(counts), interaction_range=inter, cell_size=cell, walk_radius=walk,
                list_range=list_range, list_walk_radius=lwalk, dims=dims, list_capacity=int(list_capacity),
                uniform_expected=uniform)


class GeometryError(ValueError):
    pass


@dataclass
class SoupOptions:
    """The subset of CreateSoupOpts (soup/src/soup-types.ts:14-179) the MD step honours."""
    box: Sequence[float]
    seed: int
    kT: float
    start: Dict[str, int] = field(default_factory=dict)
    catalyst_count: Optional[int] = None
    electrostatics: Optional[dict] = None      # {enabled, pH, ionicStrengthMolar, densityVolumeSigma3}
    acid_soap_scale_override: Optional[float] = None
    solvent_attraction_scale_override: Optional[float] = None
    verlet_override: Optional[dict] = None     # {listCapacity}
    confine: Optional[dict] = None             # {radiusSigma, stiffness}
    skin: Optional[float] = None               # list skin (data/soup.json verletList.skin if None)
    rebuild_on_drift: bool = False             # half-skin drift trigger instead of fixed cadence
    sweep_every: Optional[int] = None          # constant-pH cadence override
    chunk_steps: int = 1000                    # soup/src/soup-integrate.ts STEP_CHUNK
    global_step: int = 0
    protonation_rng: Optional[int] = None
    es_list_capacity: Optional[int] = None


def resolve(opts: SoupOptions, P: Optional[dict] = None) -> _abi.SoupConfig:
    """Build the SoupConfig for `opts` (soup/src/sim.ts:95-330 up to the buffer allocation)."""
    P = P or load_params()
    p = P["params"]
    monomers = P["monomers"]
    if len(monomers) > _abi.MAX_KINDS:
        raise ValueError(f"{len(monomers)} monomer kinds, but at most {_abi.MAX_KINDS} are supported")
    ids = [m["id"] for m in monomers]
    start = dict(P["start"])
    start.update(opts.start or {})
    if opts.catalyst_count is not None:
        cat = next(m for m in monomers if m["kind"] == "catalyst")
        start[cat["id"]] = opts.catalyst_count
    for m in monomers:
        if m.get("mineral"):
            start[m["id"]] = 0   # the clay platelet is not part of the MD step built here
    counts = [int(start.get(m["id"], 0)) for m in monomers]
    n = sum(counts)
    if n == 0:
        raise ValueError("createSoup: the starting composition is empty")
    box = [float(b) for b in opts.box]
    kT = float(opts.kT)
    skin = float(P["verletList"]["skin"] if opts.skin is None else opts.skin)
    rebuild_every = int(P["verletList"]["rebuildEvery"])
    vo = opts.verlet_override or {}

    confine_r = 0.0
    confine_k = 0.0
    density_volume = None
    if opts.confine:
        confine_r = float(opts.confine["radiusSigma"])
        confine_k = float(opts.confine["stiffness"])
        if not (confine_r > 0 and confine_k > 0):
            raise ValueError("confine: radius and stiffness must be positive")
        if not (box[0] == box[1] == box[2]):
            raise ValueError("confine: confinement is implemented only in a cubic box")
        density_volume = 4.0 / 3.0 * math.pi * confine_r ** 3

    plan = derive_plan(P, box, counts, kT, skin, rebuild_every, not opts.rebuild_on_drift,
                       vo.get("listCapacity"), density_volume)

    es_opts = dict(opts.electrostatics or {})
    es_over = {
        "enabled": es_opts.get("enabled"),
        "pH": es_opts.get("pH"),
        "ionicStrengthMolar": es_opts.get("ionicStrengthMolar"),
        "minBoxSigma": min(box),
        "maxHeads": start.get(P["electrostatics"]["chargedKind"], 0),
        "acidSoapScale": opts.acid_soap_scale_override,
        "densityVolumeSigma3": density_volume if density_volume else es_opts.get("densityVolumeSigma3"),
        "cutoffSigma": es_opts.get("cutoffSigma"),
        "skin": skin,
        "sweepEverySteps": opts.sweep_every if opts.sweep_every is not None else None,
    }
    es_over = {k: v for k, v in es_over.items() if v is not None}
    es = make_es_basis(P, kT, es_over)
    if confine_r > 0:
        cut_max = max(plan.list_range, es.list_range if es.enabled else 0.0)
        clearance = box[0] / 2 - confine_r
        if not (clearance > cut_max):
            raise GeometryError(
                f"confine: the clearance to the box face L/2-R={clearance:.4f} does not exceed the largest "
                f"interaction radius {cut_max:.4f}"
            )

    cfg = _abi.SoupConfig()
    cfg.abi_version = _abi.ABI_VERSION
    cfg.n = n
    cfg.n_kinds = len(monomers)
    cfg.seed = int(opts.seed) & 0xFFFFFFFF
    for k, c in enumerate(counts):
        cfg.counts[k] = c
    for a in range(3):
        cfg.box[a] = box[a]
    cfg.sigma = p["sigma"]
    cfg.epsilon = p["epsilon"]
    cfg.b_tt = p["beadSizes"]["tail_tail"]
    cfg.k_fene = p["fene"]["k"]
    cfg.r_inf = p["fene"]["rInf"]
    cfg.k_bend = p["bend"]["k"]
    cfg.r_bend = p["bend"]["r0"]
    cfg.wc = p["wc"]
    cfg.kT = kT
    cfg.gamma = p["gamma"]
    cfg.dt = p["dt"]
    for k, m in enumerate(monomers):
        cfg.radius[k] = m["radiusSigma"]
        cfg.kind_class[k] = species_class(m)
    table = attraction_table(P, opts.solvent_attraction_scale_override)
    for ci in range(4):
        for cj in range(4):
            cfg.attr_scale[ci][cj] = table[ci][cj]
    cfg.acid_soap_scale = acid_soap_scale(P, opts.acid_soap_scale_override, opts.solvent_attraction_scale_override)
    cfg.interaction_range = plan.interaction_range
    cfg.cell_divisor = int(P["neighborGrid"]["cellDivisor"])
    cfg.skin = skin
    cfg.list_range = plan.list_range
    cfg.rebuild_every = rebuild_every
    cfg.rebuild_on_drift = 1 if opts.rebuild_on_drift else 0
    cfg.list_capacity = plan.list_capacity

    cfg.es_enabled = 1 if es.enabled else 0
    cfg.charged_kind = es.charged_kind
    cfg.charge_deprotonated = es.charge_deprotonated
    cfg.es_coeff_a = es.coeff_a
    cfg.es_kappa = es.kappa
    cfg.es_cutoff = es.cutoff
    cfg.es_shift_u = es.shift_u
    cfg.es_shift_f = es.shift_f
    cfg.es_split_radius = es.split_radius
    cfg.es_list_range = es.list_range
    cfg.es_list_capacity = opts.es_list_capacity or es.list_capacity
    cfg.pka_intrinsic = es.pka
    cfg.ph = es.ph
    cfg.sweep_every = es.sweep_every
    cfg.protonation_rng = 0 if opts.protonation_rng is None else int(opts.protonation_rng) & 0xFFFFFFFF
    cfg.rc_attr = es.rc_attr

    # resolveRules (soup/src/soup-plan.ts:22-49) + BondParams (soup/src/soup-buffers.ts:344-410)
    kind_of = {m["id"]: k for k, m in enumerate(monomers)}
    cat = [k for k, m in enumerate(monomers) if m["kind"] == "catalyst"]
    if not cat:
        raise ValueError("data/soup.json: no monomer of kind catalyst found")
    bond_rules = [r for r in P["rules"] if r["kind"] == "bond"]
    if len(bond_rules) > _abi.MAX_RULES:
        raise ValueError(f"{len(bond_rules)} bond formation rules, but BondParams holds at most 4")
    bond_dt = p["dt"] * P["bondAttemptInterval"]
    cfg.n_rules = len(bond_rules)
    for ri, bond in enumerate(bond_rules):
        brk = next((r for r in P["rules"] if r["kind"] == "break" and r["a"] == bond["a"] and r["b"] == bond["b"]), None)
        if brk is None:
            raise ValueError(f"data/soup.json: rule {bond['id']} has no paired break")
        ma = next(m for m in monomers if m["id"] == bond["a"])
        mb = next(m for m in monomers if m["id"] == bond["b"])
        cfg.rule_kind_a[ri] = kind_of[bond["a"]]
        cfg.rule_kind_b[ri] = kind_of[bond["b"]]
        cfg.attempt_form[ri] = bond["attemptRate"] * bond_dt
        cfg.attempt_break[ri] = brk["attemptRate"] * bond_dt
        cfg.accept_form[ri] = min(1.0, math.exp(-(-bond["energyKT"]) / kT))
        cfg.accept_break[ri] = min(1.0, math.exp(-(brk["energyKT"]) / kT))
        cfg.requires_catalyst[ri] = 1 if bond["requiresCatalyst"] else 0
        cfg.role_a[ri] = slot_role(ma["kind"], mb["kind"])
        cfg.role_b[ri] = slot_role(mb["kind"], ma["kind"])
    cfg.catalyst_kind = cat[0]
    cfg.head_terminal_only = 1 if P["headPlacement"]["terminalOnly"] else 0
    cfg.head_chain_capacity = int(P["headPlacement"]["chainCapacity"])
    cfg.max_hold_steps = int(P["adsorption"]["maxHoldSteps"])
    cfg.bond_interval = int(P["bondAttemptInterval"])
    cfg.wall_radius = confine_r
    cfg.wall_k = confine_k
    cfg.global_step = int(opts.global_step)
    cfg.chunk_steps = int(opts.chunk_steps)
    return cfg


def rule_ids(P: Optional[dict] = None) -> List[tuple]:
    """[(bond id, break id)] per resolved rule, the event-counter names (soup/src/sim.ts eventRuleIds)."""
    P = P or load_params()
    out = []
    for bond in (r for r in P["rules"] if r["kind"] == "bond"):
        brk = next(r for r in P["rules"] if r["kind"] == "break" and r["a"] == bond["a"] and r["b"] == bond["b"])
        out.append((bond["id"], brk["id"]))
    return out

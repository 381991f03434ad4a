"""Generate soup_params.json: the numeric subset of the reference's data files that the soup MD
step reads.

The reference keeps every physical constant in two JSON files (data/params.json and
data/soup.json) and derives every GPU uniform from them at system creation (soup/src/sim.ts:95,
soup/src/soup-buffers.ts:344-410, soup/src/electrostatics.ts:166-247).  This script copies the
numbers only -- no basis/prose fields -- into one flat file that ships with the package, because the
reference tree is not present where the library runs.

Usage:  python make_params.py /path/to/reference  >  (writes soup_params.json beside this file)
"""
import json
import os
import sys


def main(ref_root: str) -> None:
    with open(os.path.join(ref_root, "data", "params.json")) as fh:
        params = json.load(fh)
    with open(os.path.join(ref_root, "data", "soup.json")) as fh:
        soup = json.load(fh)
    with open(os.path.join(ref_root, "data", "periodic-measurement.json")) as fh:
        periodic = json.load(fh)

    sc = soup["solvent"]["attractionScale"]
    pe = sc["pairEpsilon"]
    clay = soup.get("clay", {})
    chem_name = clay.get("surfaceChemistry")
    chem_pairs = clay.get("surfaceChemistries", {}).get(chem_name, {}).get("pairs", {})
    es = soup["electrostatics"]
    out = {
        "params": {
            "sigma": params["sigma"],
            "epsilon": params["epsilon"],
            "beadSizes": dict(params["beadSizes"]),
            "fene": dict(params["fene"]),
            "bend": dict(params["bend"]),
            "wc": params["attraction"]["wc"],
            "gamma": params["thermostat"]["gamma"],
            "kT": params["thermostat"]["kT"],
            "dt": params["integrator"]["dt"],
        },
        "monomers": [
            {
                "id": m["id"],
                "kind": m["kind"],
                "radiusSigma": m["radiusSigma"],
                "polar": bool(m.get("polar", False)),
                "solvent": bool(m.get("solvent", False)),
                "mineral": bool(m.get("mineral", False)),
            }
            for m in soup["monomers"]
        ],
        "start": dict(soup["start"]),
        "rules": [
            {
                "id": r["id"],
                "kind": r["kind"],
                "a": r["a"],
                "b": r["b"],
                "requiresCatalyst": bool(r["requiresCatalyst"]),
                "energyKT": r["energyKT"],
                "attemptRate": r["attemptRate"],
            }
            for r in soup["rules"]
        ],
        "attraction": {
            "epsilonScale": sc.get("epsilonScale", 1.0),
            "reference": pe["reference"],
            "levelsKJ": {k: v["epsilonKJ"] for k, v in pe["levels"].items()},
            "mineralPairAlias": dict(chem_pairs),
            "acidSoapPairKJ": sc.get("acidSoapPair", {}).get("epsilonKJ", 0.0),
        },
        "electrostatics": {
            k: es[k]
            for k in (
                "enabled", "chargedKind", "chargeDeprotonated", "sigmaToNm", "bjerrumLengthNm",
                "debyeLengthNmAtUnitMolar", "ionicStrengthMolar", "pKaIntrinsic", "pH",
                "sweepEverySteps", "longRangeDebyeLengths", "longRangeMaxBoxFraction",
                "longRangeListCapacity", "longRangeListSafetyFactor",
            )
        },
        "adsorption": {"maxHoldSteps": soup["adsorption"]["maxHoldSteps"]},
        "neighborGrid": {"cellDivisor": soup["neighborGrid"]["cellDivisor"]},
        "verletList": {
            k: soup["verletList"][k]
            for k in ("enabled", "skin", "rebuildEvery", "listCapacity", "capacitySafetyFactor", "capacityFloor")
        },
        "headPlacement": {k: soup["headPlacement"][k] for k in ("terminalOnly", "chainCapacity")},
        "bondAttemptInterval": soup["bondAttemptInterval"]["steps"],
        "stageThresholds": {k: v for k, v in soup["stageThresholds"].items() if isinstance(v, (int, float))},
        "coldStartRelax": {k: soup["coldStartRelax"][k] for k in ("iterations", "maxDisplacementSigma")},
        "circularAlpha": periodic["circularConcentration"]["alpha"],
    }
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "soup_params.json")
    with open(dst, "w") as fh:
        json.dump(out, fh, indent=1, sort_keys=True)
        fh.write("\n")
    print(dst)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python make_params.py <path of a protocell-genesis checkout (its data/ is read)>")
    main(sys.argv[1])

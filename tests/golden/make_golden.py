"""Writes tests/golden/replay_fingerprints.json: SHA-256 fingerprints of the
oracle's checkerboard replay for fixed (model, shape, beta, seed, sweeps)
cases, with the final cached energy.  The oracle is pinned to the reference's
own known answers and exact results by tests/test_oracle.py; these fixtures
freeze its output so that (a) a change of the oracle shows up on the CPU and
(b) the device is checked against committed values without running the
oracle.  Run from the repository root:  python tests/golden/make_golden.py
"""
import hashlib
import json
import math
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

CASES = [
    # model, shape, beta, seed, sweeps, extra
    ("ising", [64, 64], 0.4407, 101, 6, {}),
    ("ising", [130, 302], 0.5, 102, 3, {}),
    ("ising", [34, 6], 0.35, 103, 8, {"J": -1.0}),
    ("ising", [6, 8, 10], 0.2216, 104, 5, {}),
    ("ising", [288, 6, 4], 0.3, 105, 3, {}),
    ("potts", [130, 20], 1.0051, 106, 5, {"q": 3}),
    ("potts", [34, 6, 36], 0.6, 107, 4, {"q": 4}),
    ("potts", [1040, 8], 0.8814, 108, 3, {"q": 2}),
    ("potts", [200, 130], 1.2, 113, 3, {"q": 4}),
    ("potts", [66, 10], 1.0, 114, 4, {"q": 5}),
    ("o3", [66, 10], 0.7, 109, 4, {"alpha": 1.0}),
    ("o3", [8, 6, 20], 0.69, 110, 3, {"alpha": 0.8}),
    ("msc", [66, 10], 0.4407, 111, 3, {}),
    ("msc", [34, 6, 20], 0.2216, 112, 2, {}),
    # heat bath
    ("ising", [64, 64], 0.4407, 121, 5, {"algorithm": "heat_bath"}),
    ("ising", [34, 6, 20], 0.3, 122, 4, {"algorithm": "heat_bath", "J": -1.0}),
    ("potts", [66, 10], 1.0, 123, 4, {"q": 3, "algorithm": "heat_bath"}),
    ("potts", [18, 8, 10], 0.6, 124, 3, {"q": 6, "algorithm": "heat_bath"}),
    ("o3", [66, 10], 0.7, 125, 3, {"algorithm": "heat_bath"}),
    ("o3", [16, 8, 12], 0.69, 126, 3, {"algorithm": "heat_bath"}),
    # cluster updates
    ("ising", [66, 34], 0.4407, 131, 4, {"algorithm": "swendsen_wang"}),
    ("ising", [18, 10, 6], 0.22, 132, 5, {"algorithm": "wolff"}),
    ("potts", [34, 18], 1.0, 133, 3, {"q": 3, "algorithm": "swendsen_wang"}),
    ("potts", [10, 8, 6], 0.55, 134, 4, {"q": 4, "algorithm": "wolff"}),
    ("o3", [34, 18], 0.8, 135, 3, {"algorithm": "swendsen_wang"}),
    ("o3", [10, 8, 6], 0.6, 136, 4, {"algorithm": "wolff"}),
    # the reference's O(3) proposals (StandardStrategy, OPSSStrategy at a
    # fixed sigma)
    ("o3", [34, 18], 0.8, 137, 3, {"proposal": "standard"}),
    ("o3", [16, 8, 12], 0.7, 138, 3, {"proposal": "opss", "sigma": 0.7}),
]

_ALGS = {"heat_bath": "-hb", "swendsen_wang": "-sw", "wolff": "-wolff"}
# O(3) Metropolis proposal codes of the oracle (0 = the engine's cap)
PROPOSALS = {"standard": 1, "opss": 2}


def case_id(c):
    suffix = _ALGS.get(c["extra"].get("algorithm"), "")
    if "proposal" in c["extra"]:
        suffix += "-" + c["extra"]["proposal"]
    return f"{c['model']}-{'x'.join(map(str, c['shape']))}{suffix}"


def omc(alpha):
    return float(np.float32(2.0 * math.sin(0.5 * alpha) * math.sin(0.5 * alpha)))


def fingerprint(state):
    return hashlib.sha256(np.ascontiguousarray(state).tobytes()).hexdigest()


def run_case(oracle, model, shape, beta, seed, sweeps, extra):
    mid = {"ising": oracle.ISING, "potts": oracle.POTTS, "o3": oracle.O3, "msc": oracle.MSC}[model]
    alg = {"heat_bath": oracle.HEAT_BATH, "swendsen_wang": oracle.SWENDSEN_WANG,
           "wolff": oracle.WOLFF}.get(extra.get("algorithm"), oracle.METROPOLIS)
    prop = PROPOSALS.get(extra.get("proposal"), 0)
    # OPSS: the oracle's step parameter is sigma itself (float32)
    step = float(np.float32(extra["sigma"])) if prop == 2 else omc(extra.get("alpha", 1.0))
    lat = oracle.Lattice(mid, tuple(shape), q=extra.get("q", 3), J=extra.get("J", 1.0), beta=beta,
                         seed=seed, omc=step, algorithm=alg, prop=prop)
    for _ in range(sweeps):
        lat.sweep(adapt=False)
    st = lat.state()
    energy = float(lat.energy())
    return {"model": model, "shape": shape, "beta": beta, "seed": seed, "sweeps": sweeps,
            "extra": extra, "sha256": fingerprint(st), "energy": energy}


def main():
    import oracle
    oracle.build()
    out = [run_case(oracle, *c) for c in CASES]
    path = os.path.join(ROOT, "tests", "golden", "replay_fingerprints.json")
    with open(path, "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "cases": out}, f, indent=1)
    print(f"wrote {len(out)} cases to {path}")


if __name__ == "__main__":
    main()

"""The oracle against its committed golden fixtures (tests/golden/).

tests/golden/replay_fingerprints.json holds SHA-256 fingerprints and final
energies of the oracle's checkerboard replay for fixed cases, written by
tests/golden/make_golden.py.  The oracle itself is pinned to the reference's
known answers and exact results in test_oracle.py; this test catches any
change of its output, and test_gpu_parity.py checks the device against the
same committed values."""
import json
import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden  # noqa: E402

with open(os.path.join(HERE, "golden", "replay_fingerprints.json")) as f:
    CASES = json.load(f)["cases"]


@pytest.mark.parametrize("case", CASES, ids=[make_golden.case_id(c) for c in CASES])
def test_oracle_reproduces_golden_fingerprints(oracle, case):
    got = make_golden.run_case(oracle, case["model"], case["shape"], case["beta"], case["seed"],
                               case["sweeps"], case["extra"])
    assert got["sha256"] == case["sha256"]
    assert got["energy"] == case["energy"]

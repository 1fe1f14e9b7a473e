"""The bounds-checked build, the stand-in for a memory sanitizer.

libgpumc_bounds.so is the engine compiled with -DGPUMC_DEBUG_BOUNDS: every
checked global and shared-memory access of the sweep, cluster and lattice
kernels that would fall outside its buffer is skipped and counted instead
(gpumc_debug_bounds).  CPU: the build compiles and exports the counter
entry point.  GPU: a child process loads the checked library, runs every
kernel family on ragged, split and wrapped tiles (and a batched engine), and
must count no violation while its spins still match the oracle.
"""
import json
import os
import subprocess
import sys
import textwrap

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_bounds_build_compiles_and_exports_the_counters():
    from scamper_b200.build import build_library
    lib = build_library(bounds=True)
    syms = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True, check=True).stdout
    assert "gpumc_debug_bounds" in syms and "gpumc_sweep" in syms


CHILD = textwrap.dedent('''
    import json, math, sys
    import numpy as np
    sys.path.insert(0, %(root)r)
    import scamper_b200 as gpumc
    from scamper_b200 import _lib
    import oracle

    def params(shape, **kw):
        p = {"lattice_type": "square" if len(shape) == 2 else "cubic", "Lx": shape[0], "Ly": shape[1]}
        if len(shape) == 3:
            p["Lz"] = shape[2]
        p.update(kw)
        return p

    cases = [
        ("ising", (64, 34), {}, None), ("ising", (130, 20), {}, None), ("ising", (2054, 4), {}, None),
        ("ising", (6, 8, 10), {}, None), ("ising", (34, 6, 4), {}, None), ("ising", (128, 64, 40), {}, None),
        ("ising", (66, 10), {}, "heat_bath"), ("ising", (16, 16, 16), {}, "swendsen_wang"),
        ("ising", (64, 64), {}, "wolff"),
        ("potts", (34, 6), {"q": 3}, None), ("potts", (8256, 6), {"q": 4}, None), ("potts", (6, 8, 10), {"q": 2}, None),
        ("potts", (130, 20), {"q": 5}, None), ("potts", (34, 6, 36), {"q": 7}, None),
        ("potts", (32, 32), {"q": 3}, "heat_bath"), ("potts", (34, 18), {"q": 3}, "swendsen_wang"),
        ("o3", (66, 10), {}, None), ("o3", (8, 6, 20), {}, None), ("o3", (64, 64, 8), {}, None),
        ("o3", (70, 4, 6), {}, "heat_bath"), ("o3", (16, 8, 12), {"o3_proposal": "opss"}, None),
        ("o3", (10, 6), {"o3_proposal": "standard"}, None), ("o3", (8, 8, 8), {}, "wolff"),
        ("o3", (16, 8, 12), {"o3_proposal": "cap_fast"}, None), ("o3", (10, 6), {"o3_proposal": "cap_fast"}, None),
        ("msc", (66, 10), {}, None), ("msc", (34, 6, 20), {}, None),
    ]
    oracle.build()
    mids = {"ising": oracle.ISING, "potts": oracle.POTTS, "o3": oracle.O3, "msc": oracle.MSC}
    mismatches = []
    for model, shape, kw, alg in cases:
        beta = 0.44 if len(shape) == 2 else 0.22
        kw = dict(kw)
        prop = kw.pop("o3_proposal", None)
        p = params(shape, beta=beta, cone_half_angle=1.0, **kw)
        if model == "msc":
            mc = gpumc.MultiSpinIsing.from_params(p, 5)
        else:
            mc = gpumc.ClassicalMC.from_params(p, 5, model=model, algorithm=alg, o3_proposal=prop)
        mc.on_phase_start(_lib.PHASE_MEASUREMENT)
        mc.sweep(3)
        if alg is None and prop is None:
            ref = oracle.Lattice(mids[model], shape, q=kw.get("q", 3), beta=beta, seed=5, omc=float(np.float32(1.0 - math.cos(1.0))))
            for _ in range(3):
                ref.sweep()
            got = mc.spins().reshape(-1, 3) if model == "o3" else mc.spins().ravel()
            if not np.array_equal(got, ref.state()):
                mismatches.append([model, list(shape)])
        mc.close()
    # resident cubic slabs (refinement off keeps whole planes), with PT
    mc = gpumc.ClassicalMC.from_params(params((32, 32, 32)), 7, n_replicas=4,
                                       betas=gpumc.geometric_ladder_betas(3.5, 5.5, 4))
    mc.set_tile_refinement(False)
    mc.pt_configure(5)
    mc.sweep(20)
    mc.close()
    # a batched engine of mixed kinds (concurrent plans, refined tiles)
    eng = gpumc.Engine()
    sims = [gpumc.ClassicalMC.from_params(params((130, 20), beta=0.44), 1, engine=eng),
            gpumc.ClassicalMC.from_params(params((34, 18), beta=1.0, q=3), 2, model="potts", engine=eng),
            gpumc.ClassicalMC.from_params(params((8, 6, 20), beta=0.7), 3, model="o3", engine=eng),
            gpumc.ClassicalMC.from_params(params((16, 16, 16), beta=0.22), 4, engine=eng)]
    eng.sweep(5)
    for s in sims:
        s.close()
    eng.close()
    hits, module, line, compiled = _lib.debug_bounds()
    print(json.dumps({"hits": hits, "module": module, "line": line, "compiled": compiled,
                      "mismatches": mismatches}))
''')


@pytest.mark.gpu
def test_kernels_stay_in_bounds_under_the_checked_build():
    from scamper_b200.build import build_library
    build_library(bounds=True)
    env = dict(os.environ, GPUMC_LIBRARY="bounds")
    r = subprocess.run([sys.executable, "-c", CHILD % {"root": ROOT}], env=env, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["compiled"], "the child did not load the bounds-checked library"
    assert out["hits"] == 0, f"out-of-bounds accesses: {out}"
    assert out["mismatches"] == [], out

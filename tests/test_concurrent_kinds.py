"""Concurrent kernel kinds: an engine batch runs each plan (one kernel kind)
on a stream of its own, forked from and joined back into the engine stream.
The plans touch disjoint lattices, so spins, energies, records and PT labels
are identical with the kinds concurrent or in sequence, with and without CUDA
graphs, and a multi-spin plan keeps its measurement kernels in order."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _params(shape, **kw):
    p = {"lattice_type": "square" if len(shape) == 2 else "cubic", "Lx": shape[0], "Ly": shape[1]}
    if len(shape) == 3:
        p["Lz"] = shape[2]
    p.update(kw)
    return p


SPECS = [
    ("ising", (96, 64), dict(beta=0.44), 3, [0.3, 0.44, 0.6], None),   # PT ladder
    ("ising", (16, 16, 24), dict(beta=0.22), 1, None, None),
    ("potts", (130, 66), dict(q=3, beta=1.0), 1, None, None),
    ("potts", (40, 40), dict(q=6, beta=1.1), 2, None, "heat_bath"),
    ("o3", (16, 16, 16), dict(beta=0.7), 2, None, None),
    ("o3", (24, 20), dict(beta=0.9), 1, None, None),
    ("ising", (48, 48), dict(beta=0.44), 1, None, "swendsen_wang"),
    ("msc", (34, 10), dict(beta=0.44), 1, None, None),
]


def _run(gpumc, concurrent, graphs):
    from scamper_b200 import _lib
    eng = gpumc.Engine()
    eng.set_concurrent_kinds(concurrent)
    sims = []
    for i, (model, shape, kw, n_rep, betas, alg) in enumerate(SPECS):
        if model == "msc":
            m = gpumc.MultiSpinIsing.from_params(_params(shape, **kw), 700 + i, engine=eng)
        else:
            m = gpumc.ClassicalMC.from_params(_params(shape, **kw), 700 + i, model=model, n_replicas=n_rep,
                                              betas=betas, algorithm=alg, engine=eng, record_capacity=128)
            if betas:
                m.pt_configure(4)
        m.on_phase_start(_lib.PHASE_MEASUREMENT)
        sims.append(m)
    if graphs:
        eng.sweep(40)
    else:
        for _ in range(40):
            eng.sweep(1)
    out = []
    for (model, *_), m in zip(SPECS, sims):
        n_rep = 1 if model == "msc" else m.n_replicas
        out.append((np.stack([m.spins(r) for r in range(n_rep)]), np.asarray(m.energy()),
                    [tuple(sorted(r.items())) for r in m.observables()],
                    None if model == "msc" else m.pt_labels()))
        m.close()
    eng.close()
    return out


@pytest.mark.parametrize("graphs", [True, False])
def test_concurrent_kinds_match_sequential_kinds(gpumc, graphs):
    a = _run(gpumc, True, graphs)
    b = _run(gpumc, False, graphs)
    for (model, *_), (sa, ea, ra, la), (sb, eb, rb, lb) in zip(SPECS, a, b):
        np.testing.assert_array_equal(sa, sb)
        if model == "o3":  # fp64 bond sums reduced by atomics in launch order
            np.testing.assert_allclose(ea, eb, rtol=1e-12)
            assert len(ra) == len(rb)
        else:
            np.testing.assert_array_equal(ea, eb)
            assert ra == rb, model
        if la is not None:
            np.testing.assert_array_equal(la, lb)

"""Cluster updates: Swendsen-Wang (SWCore, CMC.rs/src/algorithms/
swendsen_wang.rs) and Wolff (WolffCore, CMC.rs/src/algorithms/wolff.rs) for
Ising and Potts.

CPU: the oracle's restatement samples the exact distributions the
reference's cluster tests check (CMC.rs/tests/physics/potts_exact.rs:333-399
for Potts q = 3, 4 against exact enumeration, and its beta = 0 limit
:401-440), here on the 4x4 torus (Ising: full enumeration; Potts: row
transfer matrix); its cached energy equals recomputation; invalid specs
(J < 0, O(3), multi-spin) are rejected as the reference's asserts do.

GPU: the four-launch device sweep (tile union-find, global union, flip, account)
against the oracle bit for bit (spins, energies, changed counts) on 2D and
3D lattices whose extents are and are not multiples of the tile, alone,
with several replicas and ladders, and batched with other models in one
engine; the bond thresholds p = 1 - exp(-2 beta J) (Ising), 1 - exp(-beta J)
(Potts) are the reference's (models.rs:130-147, :312-329).
"""
import math

import numpy as np
import pytest

from scamper_b200 import _lib
from tests import exact


def _chain(lat, therm, meas):
    for _ in range(therm):
        lat.sweep()
    es, ms = [], []
    for _ in range(meas):
        lat.sweep()
        es.append(lat.cached_energy())
        if lat.model == 0:
            ms.append((lat.spins.astype(np.float64).sum() / lat.n) ** 2)
    return es, ms


@pytest.mark.parametrize("alg", ["sw", "wolff"])
@pytest.mark.parametrize("beta", [0.3, 0.4407, 0.6])
def test_ising_cluster_samples_exact_4x4(oracle, alg, beta):
    a = oracle.SWENDSEN_WANG if alg == "sw" else oracle.WOLFF
    ex = exact.ising_enumeration(4, 4, beta)
    es_all, ms_all = [], []
    for seed in range(1, 9):
        lat = oracle.Lattice(oracle.ISING, (4, 4), beta=beta, seed=seed, algorithm=a)
        es, ms = _chain(lat, 100, 4000)
        es_all.append(es)
        ms_all.append(ms)
        assert lat.cached_energy() == lat.energy()
    exact.replicas_ok(es_all, ex["E"])
    exact.replicas_ok(ms_all, ex["M2"])


@pytest.mark.parametrize("alg", ["sw", "wolff"])
@pytest.mark.parametrize("q,beta", [(3, 0.6), (3, None), (4, 0.8), (4, None)])
def test_potts_cluster_samples_exact_4x4(oracle, alg, q, beta):
    a = oracle.SWENDSEN_WANG if alg == "sw" else oracle.WOLFF
    beta = math.log(1.0 + math.sqrt(q)) if beta is None else beta
    ex = exact.potts_transfer_matrix(4, 4, q, beta)
    es_all = []
    for seed in range(1, 9):
        lat = oracle.Lattice(oracle.POTTS, (4, 4), q=q, beta=beta, seed=seed, algorithm=a)
        es, _ = _chain(lat, 100, 4000)
        es_all.append(es)
    exact.replicas_ok(es_all, ex["E"])


@pytest.mark.parametrize("alg", ["sw", "wolff"])
@pytest.mark.parametrize("q", [3, 4])
def test_potts_cluster_beta_zero_is_uniform(oracle, alg, q):
    """potts_exact.rs:401-440: at beta = 0 the states are uniform, <E> = -J
    (bonds) / q exactly; no bond is ever active."""
    a = oracle.SWENDSEN_WANG if alg == "sw" else oracle.WOLFF
    assert oracle.lib().orc_cluster_threshold(oracle.POTTS, 1.0, 0.0) == 0
    es_all = []
    for seed in range(1, 7):
        lat = oracle.Lattice(oracle.POTTS, (4, 4), q=q, beta=0.0, seed=seed, algorithm=a)
        es, _ = _chain(lat, 10, 3000)
        es_all.append(es)
    exact.replicas_ok(es_all, -32.0 / q)


@pytest.mark.parametrize("model,q", [("ising", 2), ("potts", 3), ("potts", 7)])
@pytest.mark.parametrize("alg", ["sw", "wolff"])
def test_cluster_energy_cache_on_3d(oracle, model, q, alg):
    a = oracle.SWENDSEN_WANG if alg == "sw" else oracle.WOLFF
    m = oracle.ISING if model == "ising" else oracle.POTTS
    lat = oracle.Lattice(m, (6, 8, 10), q=q, beta=0.35, seed=2, algorithm=a)
    changed = [lat.sweep() for _ in range(60)]
    assert lat.cached_energy() == lat.energy()
    assert sum(changed) > 0


def test_cluster_threshold_encoding(oracle):
    L = oracle.lib()
    p = 1.0 - math.exp(-2.0 * 0.44 * 1.0)
    assert L.orc_cluster_threshold(oracle.ISING, 1.0, 0.44) == int(math.ldexp(p, 64))
    p = 1.0 - math.exp(-1.2 * 1.0)
    assert L.orc_cluster_threshold(oracle.POTTS, 1.0, 1.2) == int(math.ldexp(p, 64))
    assert L.orc_cluster_threshold(oracle.ISING, 1.0, 1e6) == 2 ** 64 - 1


def _params(shape, **kw):
    p = {"lattice_type": "square" if len(shape) == 2 else "cubic", "Lx": shape[0], "Ly": shape[1]}
    if len(shape) == 3:
        p["Lz"] = shape[2]
    p.update(kw)
    return p


def test_cluster_specs_validated(gpumc):
    for model, kw in [("ising", dict(J=-1.0)), ("potts", dict(J=-0.5, q=3)), ("o3", dict(J=-1.0)),
                      (_lib.ISING_MSC64, {})]:
        for alg in ("swendsen_wang", "wolff"):
            with pytest.raises(gpumc.InvalidConfig):
                gpumc.ClassicalMC.validate_params(_params((8, 8), beta=0.4, **kw), model=model, algorithm=alg)
    gpumc.ClassicalMC.validate_params(_params((8, 8), beta=0.4), model="ising", algorithm="sw")
    gpumc.ClassicalMC.validate_params(_params((6, 8, 10), beta=0.4, q=5), model="potts", algorithm="wolff")
    gpumc.ClassicalMC.validate_params(_params((6, 8, 10), beta=0.7), model="o3", algorithm="swendsen_wang")


@pytest.mark.parametrize("alg", ["sw", "wolff"])
def test_o3_cluster_matches_heat_bath_4x4(oracle, alg):
    """O(3) cluster updates (embedded Ising reflections, models.rs:516-579)
    against the heat bath (itself pinned to the Langevin moments) on the 4x4
    torus: pooled <E> of independent chains agree (cross-solver z, cf.
    CMC.rs/tests/physics/continuous_cross_solver.rs)."""
    a = oracle.SWENDSEN_WANG if alg == "sw" else oracle.WOLFF
    beta = 0.9
    means = {}
    for name, algo in (("cluster", a), ("hb", oracle.HEAT_BATH)):
        ms = []
        for seed in range(1, 13):
            lat = oracle.Lattice(oracle.O3, (4, 4), beta=beta, seed=seed + (0 if name == "cluster" else 100),
                                 algorithm=algo)
            es, _ = _chain(lat, 200, 3000)
            ms.append(np.mean(es))
            st = lat.state().astype(np.float64)
            assert np.abs((st ** 2).sum(axis=1) - 1.0).max() < 1e-5
            assert lat.cached_energy() == pytest.approx(lat.energy(), rel=1e-9, abs=1e-9)
        means[name] = (np.mean(ms), np.std(ms, ddof=1) / math.sqrt(len(ms)))
    (m1, s1), (m2, s2) = means["cluster"], means["hb"]
    assert abs(m1 - m2) < 4.0 * math.hypot(s1, s2), means


SHAPES = [(16, 16), (34, 18), (4, 4), (64, 64), (6, 6, 6), (8, 8, 8), (18, 10, 6), (130, 6, 4)]


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(16, 16), (34, 18), (6, 6, 6), (18, 10, 6)])
@pytest.mark.parametrize("alg", ["swendsen_wang", "wolff"])
def test_gpu_o3_cluster_matches_oracle(gpumc, oracle, shape, alg):
    a = oracle.SWENDSEN_WANG if alg == "swendsen_wang" else oracle.WOLFF
    beta = 0.8 if len(shape) == 2 else 0.6
    mc = gpumc.ClassicalMC.from_params(_params(shape, beta=beta), 67, model="o3", algorithm=alg)
    ref = oracle.Lattice(oracle.O3, shape, beta=beta, seed=67, algorithm=a)
    mc.on_phase_start(_lib.PHASE_MEASUREMENT)
    changed = []
    for _ in range(3):
        mc.sweep(2)
        changed += [ref.sweep(), ref.sweep()]
        np.testing.assert_array_equal(mc.spins(), ref.state().reshape(mc.spins().shape))
        assert mc.energy()[0] == pytest.approx(ref.cached_energy(), rel=1e-12, abs=1e-9)
    obs = mc.observables()
    assert [round(o["acceptance"] * ref.n) for o in obs] == changed
    assert mc.launches_per_sweep() == 4
    mc.close()


@pytest.mark.gpu
@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("model,q,beta", [("ising", 2, 0.4407), ("ising", 2, 0.25), ("potts", 3, 1.0),
                                          ("potts", 8, 1.4)])
@pytest.mark.parametrize("alg", ["swendsen_wang", "wolff"])
def test_gpu_cluster_matches_oracle(gpumc, oracle, shape, model, q, beta, alg):
    if len(shape) == 3:
        beta *= 0.5
    a = oracle.SWENDSEN_WANG if alg == "swendsen_wang" else oracle.WOLFF
    m = oracle.ISING if model == "ising" else oracle.POTTS
    mc = gpumc.ClassicalMC.from_params(_params(shape, beta=beta, q=q), 61, model=model, algorithm=alg)
    ref = oracle.Lattice(m, shape, q=q, beta=beta, seed=61, algorithm=a)
    np.testing.assert_array_equal(mc.spins().ravel(), ref.spins)
    mc.on_phase_start(_lib.PHASE_MEASUREMENT)
    changed = []
    for _ in range(3):
        mc.sweep(2)
        changed += [ref.sweep(), ref.sweep()]
        np.testing.assert_array_equal(mc.spins().ravel(), ref.spins)
        assert mc.energy()[0] == ref.cached_energy()
    obs = mc.observables()
    assert [round(o["acceptance"] * ref.n) for o in obs] == changed
    assert mc.name() == ("Swendsen-Wang" if alg == "swendsen_wang" else "Wolff")
    assert mc.launches_per_sweep() == 4
    mc.close()


@pytest.mark.gpu
def test_gpu_cluster_replicas_ladder_and_pt(gpumc, oracle):
    betas = [0.3, 0.42, 0.5]
    mc = gpumc.ClassicalMC.from_params(_params((48, 40), beta=0.4), 8, model="ising", n_replicas=3, betas=betas,
                                       algorithm="swendsen_wang")
    refs = [oracle.Lattice(oracle.ISING, (48, 40), beta=b, seed=8, replica=r, algorithm=oracle.SWENDSEN_WANG)
            for r, b in enumerate(betas)]
    mc.sweep(5)
    for r, ref in enumerate(refs):
        for _ in range(5):
            ref.sweep()
        np.testing.assert_array_equal(mc.spins(r).ravel(), ref.spins)
        assert mc.energy()[r] == ref.cached_energy()
    mc.pt_configure(2)
    mc.sweep(40)
    assert sorted(mc.pt_labels()) == [0, 1, 2]
    assert np.all(mc.energy() == mc.recompute_energy())
    mc.close()


@pytest.mark.gpu
def test_gpu_cluster_batched_with_other_models(gpumc):
    specs = [(_params((64, 48), beta=0.44), "ising", "swendsen_wang"),
             (_params((20, 20, 20), beta=0.3, q=3), "potts", "wolff"),
             (_params((128, 128), beta=0.44), "ising", "metropolis"),
             (_params((32, 32), beta=1.0, q=5), "potts", "heat_bath")]
    eng = gpumc.Engine()
    batched = [gpumc.ClassicalMC.from_params(p, 300 + i, model=m, algorithm=a, engine=eng)
               for i, (p, m, a) in enumerate(specs)]
    plain = [gpumc.ClassicalMC.from_params(p, 300 + i, model=m, algorithm=a) for i, (p, m, a) in enumerate(specs)]
    eng.sweep(12)
    for m in plain:
        m.sweep(12)
    for b, p in zip(batched, plain):
        np.testing.assert_array_equal(b.spins(), p.spins())
        assert b.energy()[0] == p.energy()[0]
    for m in batched + plain:
        m.close()
    eng.close()


@pytest.mark.gpu
@pytest.mark.parametrize("alg", ["swendsen_wang", "wolff"])
def test_gpu_potts_cluster_samples_exact_4x4(gpumc, alg):
    q, beta = 3, 1.0
    ex = exact.potts_transfer_matrix(4, 4, q, beta)
    mc = gpumc.ClassicalMC.from_params(_params((4, 4), beta=beta, q=q), 77, model="potts", n_replicas=16,
                                       algorithm=alg, record_capacity=8192)
    mc.sweep(100)
    mc.on_phase_start(_lib.PHASE_MEASUREMENT)
    mc.sweep(4000)
    rows = mc.observable_arrays()
    exact.replicas_ok([rows["energy"][rows["replica"] == r] for r in range(16)], ex["E"])
    mc.close()

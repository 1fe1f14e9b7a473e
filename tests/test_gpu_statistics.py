"""Statistical parity of the CUDA sweep with the reference sampler and with
exact results.

The engine visits sites in checkerboard order with its own random stream, so
agreement with the reference sampler (random-permutation Metropolis,
restated in oracle/refsampler.c) is statistical: observables from
independent chains must agree within |z| < 3, z = (mean_gpu - mean_ref) /
sqrt(se_gpu^2 + se_ref^2) with standard errors from the spread over
independent chains.  The 2D Ising energy at beta_c is checked against the
exact finite-torus value (Kaufman) and Onsager's infinite-lattice -sqrt(2)
with the reference's multi-seed z-score criteria
(CMC.rs/tests/physics/zscore_extended.rs:175-245).
"""
import math

import numpy as np
import pytest

from tests import exact

pytestmark = pytest.mark.gpu


def _params(shape, **kw):
    p = {"lattice_type": "square" if len(shape) == 2 else "cubic", "Lx": shape[0], "Ly": shape[1]}
    if len(shape) == 3:
        p["Lz"] = shape[2]
    p.update(kw)
    return p


def _gpu_chains(gpumc, model, shape, beta, n_rep, therm, meas, seed, **kw):
    """Per-replica time series of E/N and |M| (or order parameter)."""
    from scamper_b200 import _lib
    if model == "msc":
        mc = gpumc.MultiSpinIsing.from_params(_params(shape, beta=beta, **kw), seed, record_capacity=1024)
        n_rep = 64
    else:
        mc = gpumc.ClassicalMC.from_params(_params(shape, **kw), seed, model=model, n_replicas=n_rep,
                                           betas=[beta], record_capacity=1024)
    mc.sweep(therm)
    mc.on_phase_start(_lib.PHASE_MEASUREMENT)
    es, ms = [], []
    left = meas
    while left:
        k = min(left, 1024)
        mc.sweep(k)
        a = mc.observable_arrays()
        es.append(a["energy"].reshape(k, n_rep))
        ms.append(a["magnetization"].reshape(k, n_rep))
        left -= k
    n = mc.n_sites
    mc.close()
    return np.concatenate(es) / n, np.concatenate(ms)


def _ref_chains(oracle, model, shape, beta, n_chains, therm, meas, seed, q=3):
    mid = {"ising": oracle.ISING, "potts": oracle.POTTS, "o3": oracle.O3}[model]
    es = np.zeros((meas, n_chains))
    ms = np.zeros((meas, n_chains))
    for c in range(n_chains):
        r = oracle.RefSampler(mid, shape, q=q, beta=beta, seed=seed + 1000 * c)
        r.sweep(therm)
        for t in range(meas):
            r.sweep()
            e, m = r.measure()
            es[t, c] = e / r.n
            ms[t, c] = m
        r.close()
    return es, ms


def _chain_stat(series_fn):
    """Mean over chains of a per-chain statistic, with its standard error
    from the spread over independent chains."""
    vals = np.asarray(series_fn)
    return vals.mean(), vals.std(ddof=1) / math.sqrt(len(vals))


def _compare(a_series, b_series, fn, label, limit=3.0):
    ma, sa = _chain_stat([fn(a_series[:, c]) for c in range(a_series.shape[1])])
    mb, sb = _chain_stat([fn(b_series[:, c]) for c in range(b_series.shape[1])])
    z = (ma - mb) / math.sqrt(sa * sa + sb * sb)
    assert abs(z) < limit, f"{label}: gpu {ma:.6f}+-{sa:.6f} vs reference {mb:.6f}+-{sb:.6f}, z = {z:.2f}"
    return z


def _binder_per_chain(ms):
    # U4 from the chain's own moments (pooled over chains by the caller)
    return 1.0 - np.mean(ms ** 4) / (3.0 * np.mean(ms ** 2) ** 2)


def test_ising_beta_c_energy_matches_exact_finite_torus(gpumc):
    """E/N of the 64x64 torus at beta_c: per-replica z-scores against
    Kaufman's exact value; mean |M| sanity against Onsager's -sqrt(2)."""
    beta = exact.BETA_C_2D_ISING
    L = 64
    es, _ = _gpu_chains(gpumc, "ising", (L, L), beta, 16, 2000, 16384, seed=71)
    ex = exact.kaufman_energy(L, beta) / (L * L)
    zs = []
    for c in range(es.shape[1]):
        m, s = exact.binned(es[:, c], nbins=32)
        zs.append((m - ex) / s)
    assert max(abs(z) for z in zs) < 4.0, zs
    assert abs(np.mean(zs)) < 2.0, zs
    assert sum(zs) > -2.0 * math.sqrt(len(zs)), zs
    # finite-size offset of L = 64 from -sqrt(2) is ~0.0097
    assert abs(es.mean() + math.sqrt(2.0)) < 0.02


def test_ising_beta_c_l128_energy_matches_exact(gpumc):
    """L = 128 at beta_c after a long thermalization (Metropolis relaxes as
    ~L^2.2 sweeps at criticality): E/N against Kaufman's exact value and
    within the finite-size offset of Onsager's -sqrt(2)."""
    beta = exact.BETA_C_2D_ISING
    L = 128
    es, _ = _gpu_chains(gpumc, "ising", (L, L), beta, 8, 40000, 16384, seed=72)
    ex = exact.kaufman_energy(L, beta) / (L * L)
    zs = []
    for c in range(es.shape[1]):
        m, s = exact.binned(es[:, c], nbins=16)
        zs.append((m - ex) / s)
    assert max(abs(z) for z in zs) < 4.0, zs
    assert abs(np.mean(zs)) < 2.0, zs
    assert abs(es.mean() + math.sqrt(2.0)) < 0.01  # finite-size offset at L = 128 is ~0.0049


@pytest.mark.parametrize("beta", [0.35, exact.BETA_C_2D_ISING, 0.5])
def test_ising_observables_match_reference_sampler(gpumc, oracle, beta):
    shape = (16, 16)
    g_e, g_m = _gpu_chains(gpumc, "ising", shape, beta, 16, 2000, 20000, seed=81)
    r_e, r_m = _ref_chains(oracle, "ising", shape, beta, 8, 2000, 20000, seed=82)
    _compare(g_e, r_e, np.mean, f"E/N beta={beta}")
    _compare(g_m, r_m, np.mean, f"|M| beta={beta}")
    _compare(g_m, r_m, lambda m: np.mean(m * m), f"M2 beta={beta}")
    _compare(g_m, r_m, _binder_per_chain, f"Binder beta={beta}")


def test_potts_observables_match_reference_sampler(gpumc, oracle):
    q = 3
    beta = math.log(1.0 + math.sqrt(q))
    shape = (16, 16)
    g_e, g_m = _gpu_chains(gpumc, "potts", shape, beta, 16, 2000, 16000, seed=91, q=q)
    r_e, r_m = _ref_chains(oracle, "potts", shape, beta, 8, 2000, 16000, seed=92, q=q)
    _compare(g_e, r_e, np.mean, "Potts E/N")
    _compare(g_m, r_m, np.mean, "Potts order parameter")


def test_o3_observables_match_reference_sampler(gpumc, oracle):
    beta = 1.0 / 1.443
    shape = (8, 8, 8)
    g_e, g_m = _gpu_chains(gpumc, "o3", shape, beta, 16, 1500, 6000, seed=101, cone_half_angle=1.0)
    r_e, r_m = _ref_chains(oracle, "o3", shape, beta, 8, 1500, 6000, seed=102)
    _compare(g_e, r_e, np.mean, "O(3) E/N")
    _compare(g_m, r_m, np.mean, "O(3) |M|")


def test_multispin_replicas_match_reference_sampler(gpumc, oracle):
    beta = exact.BETA_C_2D_ISING
    shape = (16, 16)
    g_e, g_m = _gpu_chains(gpumc, "msc", shape, beta, 64, 2000, 8000, seed=111)
    r_e, r_m = _ref_chains(oracle, "ising", shape, beta, 8, 2000, 8000, seed=112)
    _compare(g_e, r_e, np.mean, "MSC E/N")
    _compare(g_m, r_m, np.mean, "MSC |M|")

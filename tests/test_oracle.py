"""CPU tests of the oracle: pinned against published known-answer vectors
and against the reference's own tests (known answers, exact enumeration,
transfer matrices), before it is trusted as the parity checker."""
import math

import numpy as np
import pytest

from tests import exact


# ---- Philox4x32-10 published known-answer vectors (Random123 KAT) ----------
KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


@pytest.mark.parametrize("ctr,key,expect", KAT)
def test_philox_known_answers(oracle, ctr, key, expect):
    assert tuple(int(x) for x in oracle.philox(ctr, key)) == expect


def test_stream_seed_is_deterministic_and_domain_separated(oracle):
    # Carlo.rs/src/rng_stream.rs:161-194
    k = oracle.stream_seed(42, 3, 7, 2, 5, 1, 2, 11)
    assert k == oracle.stream_seed(42, 3, 7, 2, 5, 1, 2, 11)
    base = dict(base=123)
    seeds = {
        oracle.stream_seed(123),
        oracle.stream_seed(123, task=1),
        oracle.stream_seed(123, run=1),
        oracle.stream_seed(123, chain=1),
        oracle.stream_seed(123, replica=1),
        oracle.stream_seed(123, thread=1),
        oracle.stream_seed(123, phase=2),
        oracle.stream_seed(123, substream=1),
    }
    assert len(seeds) == 8, base


def test_threshold_encoding(oracle):
    assert oracle.threshold(1.0) == (65536, 0)
    assert oracle.threshold(2.5) == (65536, 0)
    assert oracle.threshold(0.0) == (0, 0)
    assert oracle.threshold(float("nan")) == (0, 0)
    assert oracle.threshold(0.5) == (32768, 0)
    for p in [math.exp(-4.0), math.exp(-8 * 0.4407), 0.123456789, 1e-30]:
        h, t = oracle.threshold(p)
        val = (h * 2.0 ** 64 + t) / 2.0 ** 80
        assert abs(val - p) <= 2.0 ** -79 + p * 1e-15


def test_multispin_lut_matches_reference_values(oracle):
    # CMC.rs/src/multi_spin.rs:433-441: chain (z = 2), beta = 1, J = 1:
    # log_acceptance[aligned = 2] = -4, [1] = [0] = 0.  Classes here are
    # anti-aligned counts k = z - aligned.
    head, tail = oracle.table(oracle.MSC, 1, 1.0, 1.0)
    assert len(head) == 3
    assert head[1] == 65536 and head[2] == 65536
    p = (int(head[0]) * 2.0 ** 64 + int(tail[0])) / 2.0 ** 80
    assert abs(math.log(p) + 4.0) < 1e-10


def test_single_flip_delta_matches_recompute(oracle):
    # CMC.rs/tests/physics/lattice_exact.rs:23-97 and usage_exact.rs:26-60:
    # every single-site change equals the difference of full recomputations.
    rng = np.random.default_rng(3)
    for dims, shape in [(2, (6, 4)), (3, (4, 4, 6))]:
        for model, q in [(oracle.ISING, 2), (oracle.POTTS, 3)]:
            lat = oracle.Lattice(model, shape, q=q, beta=0.3, seed=5)
            z = 2 * dims
            for _ in range(10):
                s = lat.spins.copy()
                e0 = lat.energy()
                site = int(rng.integers(lat.n))
                # neighbours of the site in the fixed order
                coords = np.unravel_index(site, tuple(reversed(shape)))[::-1]
                nbs = []
                for a in range(dims):
                    for d in (-1, 1):
                        c = list(coords)
                        c[a] = (c[a] + d) % shape[a]
                        nbs.append(int(np.ravel_multi_index(tuple(reversed(c)), tuple(reversed(shape)))))
                if model == oracle.ISING:
                    k = sum(s[nb] != s[site] for nb in nbs)
                    lat.spins[site] = -s[site]
                    assert lat.energy() - e0 == pytest.approx(2 * (z - 2 * k))
                else:
                    t = (int(s[site]) + 1) % q
                    d = sum(s[nb] == t for nb in nbs) - sum(s[nb] == s[site] for nb in nbs)
                    lat.spins[site] = t
                    assert lat.energy() - e0 == pytest.approx(-d)
                lat.set_state(s)


@pytest.mark.parametrize("model", ["ising", "potts"])
def test_energy_cache_does_not_drift(oracle, model):
    # CMC.rs/tests/exact/classic_models.rs:279-311 (cached energy vs exact over
    # long 3D runs)
    m = oracle.ISING if model == "ising" else oracle.POTTS
    lat = oracle.Lattice(m, (6, 6, 6), q=3, beta=0.25, seed=11)
    for _ in range(1500):
        lat.sweep()
    assert lat.cached_energy() == lat.energy()


def _chain_moments(lat, therm, meas, nbins=25):
    for _ in range(therm):
        lat.sweep()
    es, ms = [], []
    for _ in range(meas):
        lat.sweep()
        es.append(lat.cached_energy())
        if lat.model == 0:
            ms.append((lat.spins.astype(np.float64).sum() / lat.n) ** 2)
    return es, ms


def test_checkerboard_replay_samples_exact_ising_4x4(oracle):
    """The replay of the engine's method samples the Boltzmann distribution:
    <E>, <m^2> on the 4x4 torus against exact enumeration (2^16 states),
    multi-seed z-scores as in CMC.rs/tests/physics/zscore_validation.rs."""
    beta = 0.4
    ex = exact.ising_enumeration(4, 4, beta)
    zs_e, zs_m = [], []
    for seed in range(1, 9):
        lat = oracle.Lattice(oracle.ISING, (4, 4), beta=beta, seed=seed)
        es, ms = _chain_moments(lat, 200, 8000)
        me, se = exact.binned(es)
        mm, sm = exact.binned(ms)
        zs_e.append(exact.zscore(me, se, ex["E"]))
        zs_m.append(exact.zscore(mm, sm, ex["M2"]))
    for zs in (zs_e, zs_m):
        assert max(abs(z) for z in zs) < 4.0
        assert abs(np.mean(zs)) < 2.0
        assert sum(zs) > -2.0 * math.sqrt(len(zs))


@pytest.mark.parametrize("q", [2, 3, 4, 5])
def test_checkerboard_replay_samples_exact_potts(oracle, q):
    """q-state Potts <E> on a 4x4 torus at beta_c(q) against the row transfer
    matrix: q <= 4 runs the bit-plane method (q = 4 with its rejection-drawn
    proposals), q = 5 the 16-bit chunk method."""
    beta = exact.math.log(1.0 + math.sqrt(q))
    ex = exact.potts_transfer_matrix(4, 4, q, beta)
    zs = []
    for seed in range(1, 7):
        lat = oracle.Lattice(oracle.POTTS, (4, 4), q=q, beta=beta, seed=seed)
        es, _ = _chain_moments(lat, 200, 8000)
        me, se = exact.binned(es)
        zs.append(exact.zscore(me, se, ex["E"]))
    assert max(abs(z) for z in zs) < 4.0
    assert abs(np.mean(zs)) < 2.0


def test_reference_sampler_samples_exact_ising_4x4(oracle):
    """The restated reference sampler (random-permutation order, log-space
    acceptance) against exact enumeration: it is the statistical yardstick."""
    beta = 0.4
    ex = exact.ising_enumeration(4, 4, beta)
    zs = []
    for seed in range(1, 7):
        r = oracle.RefSampler(oracle.ISING, (4, 4), beta=beta, seed=seed)
        r.sweep(200)
        es = []
        for _ in range(6000):
            r.sweep()
            es.append(r.measure()[0])
        me, se = exact.binned(es)
        zs.append(exact.zscore(me, se, ex["E"]))
        assert r.recompute_energy() == pytest.approx(r.measure()[0], abs=1e-9)
    assert max(abs(z) for z in zs) < 4.0
    assert abs(np.mean(zs)) < 2.0


def test_multispin_replicas_sample_exact_ising_4x4(oracle):
    """Each of the 64 bit-replicas of the multi-spin replay samples the 4x4
    Boltzmann distribution (pooled over replicas, cf.
    CMC.rs/tests/physics/multispin_cross_solver.rs:86-204)."""
    beta = 0.4
    ex = exact.ising_enumeration(4, 4, beta)
    lat = oracle.Lattice(oracle.MSC, (4, 4), beta=beta, seed=9)
    for _ in range(200):
        lat.sweep()
    rows = []
    for _ in range(1500):
        lat.sweep()
        e, m = lat.msc_observables()
        rows.append(e)
    rows = np.array(rows)  # sweeps x 64
    per_rep = rows.mean(axis=0)
    pooled = per_rep.mean()
    se = per_rep.std(ddof=1) / math.sqrt(64)
    assert abs(exact.zscore(pooled, se, ex["E"])) < 4.0


def test_o3_engine_math_accuracy(oracle):
    lib = oracle.lib()
    for x in np.linspace(-80.0, 0.0, 2001):
        v = lib.orc_exp_neg(float(x))
        assert v == pytest.approx(math.exp(float(np.float32(x))), rel=2e-5, abs=1e-37)
    c = np.zeros(1, dtype=np.float32)
    s = np.zeros(1, dtype=np.float32)
    import ctypes
    for u in np.linspace(0, 2 ** 32 - 1, 5001).astype(np.uint64):
        lib.orc_sincos_turn(int(u), c.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                            s.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
        phi = 2.0 * math.pi * (int(u) >> 5 << 5) / 2.0 ** 32
        assert abs(c[0] - math.cos(phi)) < 2e-6 and abs(s[0] - math.sin(phi)) < 2e-6


def test_o3_replay_keeps_unit_norm_and_energy_cache(oracle):
    lat = oracle.Lattice(oracle.O3, (6, 6, 6), beta=0.7, seed=4, omc=float(np.float32(1.0 - math.cos(1.0))))
    for i in range(300):
        lat.sweep(adapt=i < 100)
    st = lat.state().astype(np.float64)
    assert np.abs((st ** 2).sum(axis=1) - 1.0).max() < 1e-5
    assert lat.cached_energy() == pytest.approx(lat.energy(), rel=1e-9, abs=1e-6)


# ---- replica exchange: Carlo.rs/tests/unit/pt_exchange_rule.rs -------------
def test_accept_log_boundaries(oracle):
    lib = oracle.lib()
    for u in [0, 1, 2 ** 63, 2 ** 64 - 1, 12345678901234567]:
        for d in [0.0, -0.0, np.finfo(float).eps, np.finfo(float).tiny, 1.0, float("inf")]:
            assert lib.orc_accept_log(d, u) == 1
        assert lib.orc_accept_log(float("-inf"), u) == 0
        assert lib.orc_accept_log(float("nan"), u) == 0


def test_exchange_rate_matches_exp_delta(oracle):
    # two chains, equal rate e^delta = 0.3: (b0 - b1)(E0 - E1) = ln 0.3
    betas = np.array([1.0, 2.0])
    d = math.log(0.3)
    energies = np.array([0.0, d])  # (1-2)*(0-d) = d
    key = oracle.exchange_key(2024)
    acc = 0
    n = 100000
    labels = np.array([0, 1], dtype=np.int32)
    for step in range(1, 2 * n + 1, 2):  # odd steps pair (0,1)
        lab, k, _ = oracle.pt_exchange(betas, energies, labels, key, step)
        acc += k
    emp = acc / n
    assert abs(emp - 0.3) <= 5 * math.sqrt(0.3 * 0.7 / n)


def test_exchange_keeps_labels_a_permutation_and_pairs_by_parity(oracle):
    n = 9
    betas = np.linspace(0.2, 1.0, n)
    rng = np.random.default_rng(1)
    labels = np.arange(n, dtype=np.int32)
    key = oracle.exchange_key(7)
    for step in range(1, 200):
        e = rng.normal(size=n) * 5
        lab, k, acc = oracle.pt_exchange(betas, e, labels, key, step)
        assert sorted(lab.tolist()) == list(range(n))
        # only ladder pairs (t, t+1) with t % 2 == (step - 1) % 2 may swap
        moved = np.nonzero(lab != labels)[0]
        for r in moved:
            t_old, t_new = labels[r], lab[r]
            assert abs(int(t_old) - int(t_new)) == 1
            assert min(t_old, t_new) % 2 == (step - 1) % 2
        labels = lab


# ---- carlo-rs accumulator (Carlo.rs/tests/unit/accumulator.rs) ------------
def test_accumulator_matches_reference_unit_tests():
    from scamper_b200.measurements import Accumulator, binder_cumulant, specific_heat
    a = Accumulator(10)
    for i in range(1, 11):
        a.add(i)
    assert a.finalize().mean == pytest.approx(5.5)
    a = Accumulator(5)
    for i in range(1, 16):
        a.add(i)
    e = a.finalize()
    assert e.mean == pytest.approx(8.0) and e.stderr > 0 and e.n_bins == 3
    a = Accumulator(10)
    for i in range(1, 16):
        a.add(i)
    assert a.finalize().n_bins == 2
    assert Accumulator(10).finalize().n_bins == 0
    a = Accumulator(10)
    a.add(1.0)
    e = a.finalize()
    assert e.n_bins == 1 and e.mean == pytest.approx(1.0)
    assert binder_cumulant(0.0, 0.0) is None
    assert binder_cumulant(0.5, 0.25) == pytest.approx(1 - 0.25 / 0.75)
    assert specific_heat(-1.0, 2.0, 0.5, 4) == pytest.approx(0.25 / 4 * 1.0)


@pytest.mark.parametrize("L,beta", [(4, 0.3), (4, 0.4407), (6, 0.5), (8, 0.4407), (8, 0.2)])
def test_kaufman_exact_energy_matches_transfer_matrix(L, beta):
    """The exact finite-torus energy used for the beta_c check agrees with the
    row transfer matrix (CMC.rs/tests/physics/zscore_extended.rs:60-135)."""
    tm = exact.potts_transfer_matrix_ising(L, L, beta)["E"]
    assert exact.kaufman_energy(L, beta) == pytest.approx(tm, rel=1e-6, abs=1e-6)


def test_kaufman_energy_approaches_onsager():
    b = exact.BETA_C_2D_ISING
    e64 = exact.kaufman_energy(64, b) / 64 ** 2
    e512 = exact.kaufman_energy(512, b) / 512 ** 2
    ons = exact.onsager_energy_per_site(b)
    assert ons == pytest.approx(-math.sqrt(2.0), abs=1e-9)
    assert abs(e512 - ons) < abs(e64 - ons) < 0.02


def _abs_m_series(oracle, L, beta, seed, therm, meas, algorithm):
    lat = oracle.Lattice(oracle.ISING, (L, L), beta=beta, seed=seed, algorithm=algorithm)
    for _ in range(therm):
        lat.sweep()
    m = np.empty(meas)
    for t in range(meas):
        lat.sweep()
        m[t] = abs(int(lat.spins.sum(dtype=np.int64))) / (L * L)
    return m


def _binned_mean(x, n_bins=20):
    bins = np.array_split(x, n_bins)
    means = np.array([b.mean() for b in bins])
    return means.mean(), means.std(ddof=1) / math.sqrt(n_bins)


def test_wolff_binder_cumulant_at_tc_matches_universal_value(oracle):
    """U4 = 1 - <m^4> / (3 <m^2>^2) of the 2D Ising model at beta_c from the
    oracle's Wolff update: within 0.04 of the universal 0.610 at L = 32 and
    size-independent between L = 16 and 32 within 0.05, with the reference's
    run lengths and criteria (10^4 + 8 10^4 single-cluster updates, seed 42;
    CMC.rs/tests/physics/long_convergence.rs:16-61)."""
    u = {}
    for L in (16, 32):
        m = _abs_m_series(oracle, L, exact.BETA_C_2D_ISING, 42, 10_000, 80_000, oracle.WOLFF)
        u[L] = 1.0 - np.mean(m ** 4) / (3.0 * np.mean(m ** 2) ** 2)
    assert abs(u[32] - 0.610) < 0.04, u
    assert abs(u[16] - u[32]) < 0.05, u


def test_checkerboard_magnetization_follows_onsager(oracle):
    """The checkerboard Metropolis replay (the engine's method) on the 8 x 8
    torus: |M| vanishes at beta = 0.1 (below 0.3 + 3 sigma) and matches
    Onsager's spontaneous magnetisation (1 - sinh(2 beta)^-4)^(1/8) within
    10 % + 3 sigma at beta = 1 (CMC.rs/tests/exact/onsager.rs:60-95)."""
    m, err = _binned_mean(_abs_m_series(oracle, 8, 0.1, 7, 500, 2000, oracle.METROPOLIS))
    assert m < 0.3 + 3.0 * err, (m, err)
    m, err = _binned_mean(_abs_m_series(oracle, 8, 1.0, 8, 1000, 2000, oracle.METROPOLIS))
    onsager = (1.0 - math.sinh(2.0) ** -4) ** 0.125
    assert m > 0.5 - 3.0 * err, (m, err)
    assert abs(m - onsager) < 0.10 * onsager + 3.0 * err, (m, err, onsager)


def test_o3_energy_is_the_bond_dot_product(oracle):
    """-J sum over bonds of s_i . s_j (CMC.rs/tests/physics/continuous_spins.rs:9-25,
    there on a two-site chain; here on the 4 x 4 torus, 2N bonds): equal
    spins give -J 2N, orthogonal spins on the two colours give 0, and a
    random configuration equals the edge-list sum; the fixed-point energy the
    kernels record agrees to its resolution."""
    J, L = 1.7, 4
    lat = oracle.Lattice(oracle.O3, (L, L), J=J, beta=0.5, seed=3)
    n = L * L
    lat.set_state(np.tile(np.float32([0.0, 0.6, 0.8]), (n, 1)))
    assert lat.energy() == pytest.approx(-J * 2 * n, rel=1e-6)
    y, x = np.divmod(np.arange(n), L)
    cb = np.where(((x + y) % 2 == 0)[:, None], np.float32([1.0, 0.0, 0.0]), np.float32([0.0, 0.6, 0.8]))
    lat.set_state(cb)
    assert lat.energy() == pytest.approx(0.0, abs=1e-6)
    v = np.random.default_rng(11).normal(size=(n, 3))
    s = (v / np.linalg.norm(v, axis=1, keepdims=True)).astype(np.float32)
    lat.set_state(s)
    s64 = s.astype(np.float64).reshape(L, L, 3)
    bonds = (s64 * np.roll(s64, -1, axis=0)).sum() + (s64 * np.roll(s64, -1, axis=1)).sum()
    assert lat.energy() == pytest.approx(-J * bonds, rel=1e-6, abs=1e-9)
    assert lat.fixed_observables()[0] == pytest.approx(-J * bonds, abs=1e-4)


def test_potts_critical_coupling(gpumc):
    """beta_c(q) = ln(1 + sqrt(q)) (CMC.rs/tests/physics/potts_exact.rs:480-485):
    1.0051 for q = 3, and q = 2 is twice the Ising coupling (the Potts energy
    counts equal neighbours, half the Ising bond's range)."""
    assert gpumc.potts_beta_c(3) == pytest.approx(1.0051, abs=1e-4)
    assert gpumc.potts_beta_c(2) == pytest.approx(2.0 * exact.BETA_C_2D_ISING, rel=1e-15)

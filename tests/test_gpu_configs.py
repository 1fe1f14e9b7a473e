"""Parity on the workloads the benchmark numbers are quoted on.

The small-shape parity tests pin every kernel path; these pin the exact
launches the benchmark times, at their full sizes, against the oracle's
replay of the same method (checkerboard order, Philox stream keyed by
(seed, replica, sweep, site)):

* 2D Ising L = 8192 x beta in {0.35, 0.4407, 0.5}, 20 measured sweeps as one
  resident (temporally blocked) launch: spins byte-equal and all 60 records
  (energy, |M|/N, acceptance) equal;
* multi-spin L = 2048 x 64 bit-replicas, 3 sweeps: words equal after every
  sweep, per-replica energies and |M| equal;
* batched parallel tempering, 2D L = 512 x 64 replicas + 3D L = 128 x 32
  replicas in one engine, exchange every 10 sweeps, 20 sweeps: labels and
  every replica's spins equal (reported as SHA-256 digests);
* Potts q = 6, 7, 8 on 2D and 3D shapes;
* the reference sampler comparison on 2D Ising L = 64 at beta = 0.4407 with
  10^3 thermalization and 10^4 measured sweeps (E/N, |M|, M^2 and the Binder
  cumulant within |z| < 3; CMC.rs/tests/physics/zscore_extended.rs:175-245).

The oracle's discrete and multi-spin replays split the rows of each colour
pass across the host's cores (results do not depend on the thread count).
"""
import hashlib
import math
import os
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HEADLINE_L = 8192
HEADLINE_BETAS = [0.35, 0.4407, 0.5]


def _params(shape, **kw):
    p = {"lattice_type": "square" if len(shape) == 2 else "cubic", "Lx": shape[0], "Ly": shape[1]}
    if len(shape) == 3:
        p["Lz"] = shape[2]
    p.update(kw)
    return p


@pytest.fixture
def threaded_oracle(oracle):
    oracle.set_threads(os.cpu_count() or 1)
    yield oracle
    oracle.set_threads(1)


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_headline_resident_launch_matches_oracle(gpumc, threaded_oracle):
    """The headline workload's exact launch: 3 x 8192^2 Ising lattices, 20
    measured sweeps in one cooperative launch of the resident kernel (588
    whole-row tiles with edge-row exchange), against three oracle replays."""
    from scamper_b200 import _lib
    oracle = threaded_oracle
    seed, sweeps, L = 1000, 20, HEADLINE_L
    mc = gpumc.ClassicalMC.from_params({"lattice_type": "square", "Lx": L, "Ly": L}, seed, model="ising",
                                       n_replicas=3, betas=HEADLINE_BETAS, record_capacity=64)
    try:
        mc.on_phase_start(_lib.PHASE_MEASUREMENT)
        reps = [oracle.Lattice(oracle.ISING, (L, L), beta=b, seed=seed, replica=r)
                for r, b in enumerate(HEADLINE_BETAS)]
        for r in range(3):
            np.testing.assert_array_equal(mc.spins(r).ravel(), reps[r].state(), err_msg=f"initial {r}")
        n0 = mc.launch_count()
        mc.sweep(sweeps)
        assert mc.launch_count() - n0 == 1, "expected one resident launch for the 20 sweeps"
        recs = mc.observables()
        n = L * L
        expect = {}
        for r, rep in enumerate(reps):
            for s in range(sweeps):
                acc = rep.sweep()
                m = abs(int(rep.spins.sum(dtype=np.int64))) / n
                expect[(s, r)] = (rep.cached_energy(), m, acc / n)
        assert len(recs) == 3 * sweeps
        for rec in recs:
            e, m, a = expect[(rec["sweep"], rec["replica"])]
            assert rec["energy"] == e, rec
            assert rec["magnetization"] == m, rec
            assert rec["acceptance"] == pytest.approx(a, rel=0, abs=1e-15), rec
        for r in range(3):
            got = mc.spins(r).ravel()
            assert _digest(got) == _digest(reps[r].state()), f"replica {r} spins differ"
            assert mc.energy()[r] == reps[r].cached_energy() == reps[r].energy()
    finally:
        mc.close()


def test_multispin_l2048_matches_oracle(gpumc, threaded_oracle):
    """Multi-spin L = 2048 (64 bit-replicas, one seed each), beta = 0.4407,
    3 sweeps: the benchmark's multi-spin workload."""
    oracle = threaded_oracle
    seed, L = 7, 2048
    m = gpumc.MultiSpinIsing.from_params({"lattice_type": "square", "Lx": L, "Ly": L, "beta": 0.4407}, seed)
    try:
        orc = oracle.Lattice(oracle.MSC, (L, L), beta=0.4407, seed=seed)
        np.testing.assert_array_equal(m.spins().ravel(), orc.state(), err_msg="initial")
        for s in range(3):
            m.sweep(1)
            orc.sweep()
            assert _digest(m.spins().ravel()) == _digest(orc.state()), f"after sweep {s + 1}"
        e64, m64 = m.replica_observables(0)
        oe, om = orc.msc_observables()
        np.testing.assert_array_equal(e64, oe)
        np.testing.assert_array_equal(m64, np.abs(om) / orc.n)
    finally:
        m.close()


def _replay_pt(oracle, model_shape, betas, seed, interval, sweeps):
    """Oracle replay of one PT ensemble: every replica sweeps at the beta of
    the label it holds; exchanges every `interval` sweeps with step =
    sweep / interval.  Replicas sweep on Python threads (the C replay releases
    the GIL)."""
    R = len(betas)
    reps = [oracle.Lattice(oracle.ISING, model_shape, beta=betas[r], seed=seed, replica=r) for r in range(R)]
    labels = np.arange(R, dtype=np.int32)
    key = oracle.exchange_key(seed)
    for s in range(1, sweeps + 1):
        for r in range(R):
            reps[r].set_beta(betas[labels[r]])
        threads = [threading.Thread(target=reps[r].sweep) for r in range(R)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        if s % interval == 0:
            energies = [rep.cached_energy() for rep in reps]
            labels, _, _ = oracle.pt_exchange(betas, energies, labels, key, s // interval)
    return reps, labels


def test_batched_parallel_tempering_config_matches_oracle(gpumc, oracle):
    """The benchmark's PT workload in one engine: 2D L = 512 x 64 replicas
    (T 1.5..3.5) + 3D L = 128 x 32 replicas (T 3.5..5.5), exchange every 10
    sweeps on the device, 20 sweeps (two exchange steps, both pairings)."""
    from scamper_b200 import _lib
    interval, sweeps = 10, 20
    ens = [((512, 512), gpumc.geometric_ladder_betas(1.5, 3.5, 64), 11),
           ((128, 128, 128), gpumc.geometric_ladder_betas(3.5, 5.5, 32), 12)]
    eng = gpumc.Engine()
    sims = []
    try:
        for shape, betas, seed in ens:
            lt = {"lattice_type": "square", "L": shape[0]} if len(shape) == 2 else \
                {"lattice_type": "cubic", "L": shape[0]}
            s = gpumc.ClassicalMC.from_params(lt, seed, model="ising", n_replicas=len(betas), betas=betas,
                                              engine=eng, record_capacity=64)
            s.pt_configure(interval)
            s.on_phase_start(_lib.PHASE_MEASUREMENT)
            sims.append(s)
        eng.sweep(sweeps)
        for s, (shape, betas, seed) in zip(sims, ens):
            reps, labels = _replay_pt(oracle, shape, betas, seed, interval, sweeps)
            np.testing.assert_array_equal(s.pt_labels(), labels, err_msg=f"labels {shape}")
            got = [_digest(s.spins(r).ravel()) for r in range(len(betas))]
            exp = [_digest(rep.state()) for rep in reps]
            assert got == exp, f"{shape}: replicas {[i for i, (a, b) in enumerate(zip(got, exp)) if a != b]} differ"
            np.testing.assert_array_equal(s.energy(), [rep.cached_energy() for rep in reps])
            steps, _ = s.pt_stats()
            assert steps == sweeps // interval
    finally:
        for s in sims:
            s.close()
        eng.close()


@pytest.mark.parametrize("shape", [(130, 20), (8, 6, 20)])
@pytest.mark.parametrize("q", [6, 7, 8])
def test_potts_large_q_bit_exact(gpumc, oracle, shape, q):
    from tests.test_gpu_parity import _run_parity
    beta = math.log(1.0 + math.sqrt(q)) * (1.0 if len(shape) == 2 else 0.6)
    _run_parity(gpumc, oracle, "potts", shape, beta, seed=40 + q, sweeps=4, q=q)[0].close()


def _gpu_series(gpumc, L, beta, n_rep, therm, meas, seed):
    from scamper_b200 import _lib
    mc = gpumc.ClassicalMC.from_params({"lattice_type": "square", "L": L}, seed, model="ising",
                                       n_replicas=n_rep, betas=[beta], record_capacity=1024)
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


def _ref_series(oracle, L, beta, n_chains, therm, meas, seed):
    es = np.zeros((meas, n_chains))
    ms = np.zeros((meas, n_chains))
    samplers = [oracle.RefSampler(oracle.ISING, (L, L), beta=beta, seed=seed, chain=c) for c in range(n_chains)]

    def run(c):
        es[:, c], ms[:, c] = samplers[c].series(therm, meas)

    threads = [threading.Thread(target=run, args=(c,)) for c in range(n_chains)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for s in samplers:
        s.close()
    return es, ms


def _z(a, b):
    """z of two sets of independent per-chain values."""
    ma, mb = np.mean(a), np.mean(b)
    sa = np.std(a, ddof=1) / math.sqrt(len(a))
    sb = np.std(b, ddof=1) / math.sqrt(len(b))
    return (ma - mb) / math.sqrt(sa * sa + sb * sb), ma, sa, mb, sb


def _binder_jackknife(m):
    m2 = np.mean(m * m, axis=0)
    m4 = np.mean(m ** 4, axis=0)
    c = len(m2)
    full = 1.0 - m4.mean() / (3.0 * m2.mean() ** 2)
    loo = np.array([1.0 - (m4.sum() - m4[i]) / (c - 1) / (3.0 * ((m2.sum() - m2[i]) / (c - 1)) ** 2)
                    for i in range(c)])
    se = math.sqrt((c - 1) / c * np.sum((loo - loo.mean()) ** 2))
    return full, se


def test_plain_method_config_matches_reference_sampler(gpumc, oracle):
    """The plain CPU configuration of the reference: 2D Ising L = 64, J = 1,
    beta = 0.4407, hot start, 10^3 thermalization + 10^4 measured sweeps.
    64 device replicas (checkerboard, Philox) against 32 chains of the
    restated reference sampler (random-permutation order, Xoshiro256++):
    E/N, |M|, M^2 and U4 = 1 - <M^4> / (3 <M^2>^2), each chain's value from its
    own 10^4 samples, compared over independent chains within |z| < 3."""
    L, beta, therm, meas = 64, 0.4407, 1000, 10000
    g_e, g_m = _gpu_series(gpumc, L, beta, 64, therm, meas, seed=4407)
    r_e, r_m = _ref_series(oracle, L, beta, 32, therm, meas, seed=4408)
    stats = {
        "E/N": lambda e, m: np.mean(e, axis=0),
        "|M|": lambda e, m: np.mean(m, axis=0),
        "M2": lambda e, m: np.mean(m * m, axis=0),
    }
    report = []
    for name, fn in stats.items():
        z, ma, sa, mb, sb = _z(fn(g_e, g_m), fn(r_e, r_m))
        report.append(f"{name}: gpu {ma:.6f}+-{sa:.6f} ref {mb:.6f}+-{sb:.6f} z={z:+.2f}")
        assert abs(z) < 3.0, "; ".join(report)
    # U4 from the pooled moments of all chains (binder_cumulant,
    # CMC.rs/src/postprocess.rs:70-77), its error by leaving out one chain
    # at a time (jackknife over independent chains)
    (ga, gsa), (ra, rsa) = _binder_jackknife(g_m), _binder_jackknife(r_m)
    z = (ga - ra) / math.sqrt(gsa * gsa + rsa * rsa)
    report.append(f"U4: gpu {ga:.6f}+-{gsa:.6f} ref {ra:.6f}+-{rsa:.6f} z={z:+.2f}")
    assert abs(z) < 3.0, "; ".join(report)
    # the device energy at beta_c also sits within the finite-size offset of
    # Onsager's -sqrt(2) (L = 64: about +0.0097)
    assert abs(np.mean(g_e) + math.sqrt(2.0)) < 0.02, report

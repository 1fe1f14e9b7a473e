"""GPU tests of the engine around the sweep: device-side parallel tempering
against the oracle's exchange replay, batched launches and the serving loop
against the plain single-simulation path (bit-identical results alone and in
the mix), energy-cache audits at full benchmark sizes, and error paths."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _params(shape, **kw):
    p = {"lattice_type": "square" if len(shape) == 2 else "cubic", "Lx": shape[0], "Ly": shape[1]}
    if len(shape) == 3:
        p["Lz"] = shape[2]
    p.update(kw)
    return p


@pytest.mark.parametrize("model", ["ising", "o3"])
def test_parallel_tempering_matches_oracle_replay(gpumc, oracle, model):
    """Sweeps and neighbour exchanges every `interval` sweeps on the device
    against the oracle: each replica sweeps with its own stream at the beta of
    the label it holds; exchanges use the exchange stream and the cached
    energies (PtExchange::try_exchange, Carlo.rs/src/parallel_tempering.rs:362-419)."""
    from scamper_b200 import _lib
    R, interval, sweeps = 8, 3, 24
    shape = (8, 6) if model == "ising" else (6, 4, 4)
    betas = gpumc.geometric_ladder_betas(1.5, 3.5, R) if model == "ising" else \
        gpumc.geometric_ladder_betas(0.9, 2.0, R)
    seed = 31
    mc = gpumc.ClassicalMC.from_params(_params(shape, cone_half_angle=0.8), seed, model=model,
                                       n_replicas=R, betas=betas)
    mc.on_phase_start(_lib.PHASE_MEASUREMENT)  # no cone adaptation
    mc.pt_configure(interval)
    mid = oracle.ISING if model == "ising" else oracle.O3
    omc = float(np.float32(2.0 * math.sin(0.4) * math.sin(0.4)))
    reps = [oracle.Lattice(mid, shape, beta=betas[r], seed=seed, replica=r, omc=omc) for r in range(R)]
    labels = np.arange(R, dtype=np.int32)
    key = oracle.exchange_key(seed)
    step = 0
    for s in range(1, sweeps + 1):
        for r in range(R):
            reps[r].set_beta(betas[labels[r]])
            reps[r].sweep()
        if s % interval == 0:
            step += 1
            energies = [rep.cached_energy() if model == "ising" else rep.fixed_observables()[0] for rep in reps]
            labels, _, _ = oracle.pt_exchange(betas, energies, labels, key, step)
    mc.sweep(sweeps)
    np.testing.assert_array_equal(mc.pt_labels(), labels)
    for r in range(R):
        st = mc.spins(r)
        st = st.reshape(-1, 3) if model == "o3" else st.ravel()
        np.testing.assert_array_equal(st, reps[r].state())
    steps, acc = mc.pt_stats()
    assert steps == sweeps // interval and acc > 0
    recs = mc.observables()
    assert len(recs) == sweeps * R
    mc.close()


def test_log_weight_ratio_and_change_parameter(gpumc):
    # ClassicalMC::log_weight_ratio = (beta - beta') E (CMC.rs/src/classical_mc.rs:602-615)
    mc = gpumc.ClassicalMC.from_params(_params((8, 8), beta=0.4), 42)
    e = mc.energy()[0]
    assert mc.log_weight_ratio("beta", 0.7) == pytest.approx((0.4 - 0.7) * e)
    mc.change_parameter("beta", 0.55)
    assert mc.log_weight_ratio("beta", 0.7) == pytest.approx((0.55 - 0.7) * e)
    mc.close()
    m = gpumc.MultiSpinIsing.from_params(_params((8, 8), beta=1.0), 42)
    e64, _ = m.replica_observables(0)
    assert m.log_weight_ratio("beta", 2.0) == pytest.approx((1.0 - 2.0) * e64.sum())
    m.close()


def test_batched_engine_matches_plain_path(gpumc):
    """One batched launch per sweep over uneven lattices of several models
    gives the same spins as each simulation swept alone."""
    specs = [
        ("potts", (34, 34), dict(q=3, beta=1.0)),
        ("potts", (130, 66), dict(q=2, beta=0.8)),
        ("potts", (16, 256), dict(q=4, beta=1.1)),
        ("ising", (64, 64), dict(beta=0.44)),
        ("ising", (6, 8, 10), dict(beta=0.22)),
        ("o3", (8, 8, 8), dict(beta=0.7)),
        ("msc", (34, 10), dict(beta=0.44)),
    ]
    eng = gpumc.Engine()
    batched, plain = [], []
    for i, (model, shape, kw) in enumerate(specs):
        params = _params(shape, **kw)
        if model == "msc":
            batched.append(gpumc.MultiSpinIsing.from_params(params, 100 + i, engine=eng))
            plain.append(gpumc.MultiSpinIsing.from_params(params, 100 + i))
        else:
            batched.append(gpumc.ClassicalMC.from_params(params, 100 + i, model=model, engine=eng))
            plain.append(gpumc.ClassicalMC.from_params(params, 100 + i, model=model))
    eng.sweep(70)
    for p in plain:
        p.sweep(70)
    for (model, _, _), b, p in zip(specs, batched, plain):
        np.testing.assert_array_equal(b.spins(), p.spins())
        if model == "o3":  # fp64 energy cache summed by atomics in launch order
            np.testing.assert_allclose(b.energy(), p.energy(), rtol=1e-12)
        else:
            np.testing.assert_array_equal(b.energy(), p.energy())
        assert b.sweep_count() == p.sweep_count() == 70
    for m in batched + plain:
        m.close()
    eng.close()


@pytest.mark.parametrize("shape,n_rep,interval", [((256, 300), 3, 0), ((8, 6), 8, 3), ((1024, 64), 2, 0)])
def test_temporal_blocking_matches_streaming_kernel(gpumc, shape, n_rep, interval):
    """Resident multi-sweep launches (temporal blocking) and one streaming
    launch per sweep give the same spins, energies, records and PT labels,
    on the plain path and in a batched engine."""
    from scamper_b200 import _lib
    betas = gpumc.geometric_ladder_betas(1.5, 3.5, n_rep)
    runs = []
    for blocking in (True, False):
        mc = gpumc.ClassicalMC.from_params(_params(shape), 77, model="ising", n_replicas=n_rep,
                                           betas=betas, record_capacity=256)
        mc.set_temporal_blocking(blocking)
        mc.on_phase_start(_lib.PHASE_MEASUREMENT)
        if interval:
            mc.pt_configure(interval)
        n0 = mc.launch_count()
        mc.sweep(150)
        launches = mc.launch_count() - n0
        recs = mc.observables()
        runs.append((np.stack([mc.spins(r) for r in range(n_rep)]), mc.energy(),
                     [(r["sweep"], r["replica"], r["energy"], r["magnetization"], r["temp_index"]) for r in recs],
                     mc.pt_labels(), launches))
        mc.close()
    (s1, e1, r1, l1, n1), (s2, e2, r2, l2, n2) = runs
    np.testing.assert_array_equal(s1, s2)
    np.testing.assert_array_equal(e1, e2)
    assert r1 == r2 and len(r1) == 150 * n_rep
    np.testing.assert_array_equal(l1, l2)
    assert n2 == 150 and n1 == 3  # 150 streaming launches vs 3 resident chunks of <= 64 sweeps
    eng_runs = []
    for blocking in (True, False):
        eng = gpumc.Engine()
        eng.set_temporal_blocking(blocking)
        mc = gpumc.ClassicalMC.from_params(_params(shape), 78, model="ising", n_replicas=n_rep, betas=betas,
                                           engine=eng)
        eng.sweep(70)
        eng_runs.append((np.stack([mc.spins(r) for r in range(n_rep)]), mc.energy()))
        mc.close()
        eng.close()
    np.testing.assert_array_equal(eng_runs[0][0], eng_runs[1][0])
    np.testing.assert_array_equal(eng_runs[0][1], eng_runs[1][1])


def test_server_results_identical_alone_and_in_mix(gpumc):
    """Continuous batching: jobs admitted while others run give the same
    spins as the same job run alone through the plain path."""
    jobs = [
        ("ising", (64, 32), dict(beta=0.44), 40, 10),
        ("potts", (34, 34), dict(q=3, beta=1.0), 25, 5),
        ("o3", (8, 8, 8), dict(beta=0.7), 30, 12),
        ("ising", (16, 16, 16), dict(beta=0.22), 17, 3),
        ("potts", (66, 18), dict(q=4, beta=1.1), 50, 0),
        ("o3", (8, 8, 6), dict(beta=0.7, o3_proposal="opss"), 20, 6),
        ("o3", (6, 6, 6), dict(beta=0.7, o3_proposal="cap_fast"), 15, 4),
    ]
    srv = gpumc.Server(hbm_budget=1 << 30, chunk=7)
    ids = []
    for i, (model, shape, kw, nmeas, ntherm) in enumerate(jobs):
        kw = dict(kw)
        prop = kw.pop("o3_proposal", None)
        ids.append(srv.submit(_params(shape, **kw), 500 + i, nmeas, ntherm, model=model, o3_proposal=prop))
        srv.step()  # later jobs arrive while earlier ones are running
    done = {}
    for _ in range(200):
        for r in srv.poll():
            done[r["job_id"]] = r
        if len(done) == len(jobs):
            break
        srv.step()
    for r in srv.poll():
        done[r["job_id"]] = r
    assert len(done) == len(jobs)
    for jid, (model, shape, kw, nmeas, ntherm) in zip(ids, jobs):
        assert done[jid]["status"] == 0
        kw = dict(kw)
        prop = kw.pop("o3_proposal", None)
        alone = gpumc.ClassicalMC.from_params(_params(shape, **kw), 500 + ids.index(jid), model=model,
                                              o3_proposal=prop)
        from scamper_b200 import _lib
        alone.sweep(ntherm)
        alone.on_phase_start(_lib.PHASE_MEASUREMENT)
        alone.sweep(nmeas)
        ref = alone.spins()
        got = srv.job_spins(jid, ref.nbytes, dtype=ref.dtype).reshape(ref.shape)
        np.testing.assert_array_equal(got, ref)
        recs = alone.observables()
        assert len(recs) == nmeas
        assert done[jid]["mean_energy"] == pytest.approx(np.mean([r["energy"] for r in recs]) / alone.n_sites)
        alone.close()
    st = srv.stats()
    assert st["bytes_in_use"] == 0 and st["attempts"] > 0
    srv.close()


def test_server_timing_and_spin_retention(gpumc):
    """gpumc_server_timing splits the steps' host time into admit / sweep /
    retire; gpumc_server_set_keep_spins bounds which finished jobs keep their
    final spins for gpumc_job_spins."""
    srv = gpumc.Server(hbm_budget=1 << 30, chunk=5)
    srv.set_keep_spins(32 * 32)
    small = srv.submit(_params((32, 32), beta=0.44), 11, 12)
    large = srv.submit(_params((64, 64), beta=0.44), 12, 12)
    for _ in range(20):
        if srv.step() == 0:
            break
    res = {r["job_id"]: r for r in srv.poll()}
    assert res[small]["status"] == 0 and res[large]["status"] == 0
    assert srv.job_spins(small, 32 * 32).size == 32 * 32
    with pytest.raises(gpumc.GpumcError):
        srv.job_spins(large, 64 * 64)
    st = srv.stats()
    assert st["admit_s"] > 0 and st["sweep_s"] > 0 and st["retire_s"] > 0
    assert st["admit_s"] + st["sweep_s"] + st["retire_s"] == pytest.approx(st["busy_s"], rel=1e-9, abs=1e-9)
    srv.close()


def test_server_admission_by_footprint(gpumc):
    srv = gpumc.Server(hbm_budget=3 << 20, chunk=5)
    big = _params((1024, 1024), beta=0.4)  # 2 MiB of ping-pong buffers + records
    a = srv.submit(big, 1, 10)
    b = srv.submit(big, 2, 10)
    assert a and b
    srv.step()
    st = srv.stats()
    assert st["bytes_in_use"] <= 3 << 20  # only one resident at a time
    with pytest.raises(gpumc.InvalidConfig):
        srv.submit(_params((4096, 4096), beta=0.4), 3, 10)
    for _ in range(20):
        if srv.step() == 0:
            break
    res = {r["job_id"]: r for r in srv.poll()}
    assert res[a]["status"] == 0 and res[b]["status"] == 0
    assert res[b]["start_s"] >= res[a]["finish_s"]
    srv.close()


@pytest.mark.parametrize("shape,beta", [((8192, 8192), 0.4407), ((2048, 2048), 0.5)])
def test_full_size_ising_invariants(gpumc, shape, beta):
    """At benchmark sizes: spins stay +-1 and the cached energy equals the
    exact recomputation (audit_lattice_cache, CMC.rs/src/audit.rs:41-52)."""
    from scamper_b200 import _lib
    mc = gpumc.ClassicalMC.from_params(_params(shape, beta=beta), 77, record_capacity=64)
    mc.on_phase_start(_lib.PHASE_MEASUREMENT)
    mc.sweep(20)
    np.testing.assert_array_equal(mc.energy(), mc.recompute_energy())
    s = mc.spins()
    assert np.isin(s, [-1, 1]).all()
    recs = mc.observables()
    assert len(recs) == 20
    assert abs(recs[-1]["energy"] - mc.energy()[0]) == 0
    assert abs(recs[-1]["magnetization"] - abs(int(s.astype(np.int64).sum())) / s.size) < 1e-15
    mc.close()


def test_full_size_msc_and_cubic_invariants(gpumc):
    m = gpumc.MultiSpinIsing.from_params(_params((2048, 2048), beta=0.4407), 9)
    m.sweep(6)
    e64, mag = m.replica_observables(0)
    assert m.energy()[0] == pytest.approx(e64.sum())
    assert np.all(mag <= 1.0)
    m.close()
    c = gpumc.ClassicalMC.from_params(_params((128, 128, 128), beta=0.2216), 9)
    c.sweep(8)
    np.testing.assert_array_equal(c.energy(), c.recompute_energy())
    c.close()


def test_invalid_configs_raise(gpumc):
    for bad in [dict(Lx=7, Ly=8), dict(Lx=8, Ly=8, beta=-1.0), dict(Lx=8, Ly=8, pbc="false"),
                dict(Lx=2, Ly=8)]:
        with pytest.raises(gpumc.InvalidConfig):
            gpumc.ClassicalMC.from_params(_params((bad.pop("Lx"), bad.pop("Ly")), **bad), 1)
    with pytest.raises(gpumc.InvalidConfig):
        gpumc.ClassicalMC.from_params(_params((8, 8), q=1), 1, model="potts")

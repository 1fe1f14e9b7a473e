"""Failure paths of the engine, made without a GPU fault.

* The resident Ising kernel's inter-CTA waits are bounded; with a limit of
  zero polls a wait gives up at once, every CTA leaves, the sweep call reports
  the error, and the handle continues exactly once its state is restored.
* Serving: cancelling a queued and a running job returns their results with
  the cancelled status and frees their memory; other jobs are unaffected.
* The periodic energy-cache audit (should_audit_cache / audit_lattice_cache,
  CMC.rs/src/audit.rs:35-52) passes on healthy runs and reports a cache that
  the host perturbed.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _params(shape, **kw):
    p = {"lattice_type": "square" if len(shape) == 2 else "cubic", "Lx": shape[0], "Ly": shape[1]}
    if len(shape) == 3:
        p["Lz"] = shape[2]
    p.update(kw)
    return p


def test_resident_wait_limit_gives_up_and_handle_recovers(gpumc, oracle):
    """L = 1024 x 4 replicas (many whole-row tiles in one cooperative launch):
    a zero-poll wait limit makes the first grid barrier that is not complete
    on arrival give up.  The call fails with the timeout message; after
    restoring the spins and the sweep count the same handle reproduces the
    oracle's trajectory."""
    from scamper_b200 import _lib
    shape, betas, seed = (1024, 1024), [0.3, 0.4, 0.44, 0.5], 17
    mc = gpumc.ClassicalMC.from_params(_params(shape), seed, n_replicas=4, betas=betas)
    try:
        assert mc.tile_count() >= 8
        start = [mc.spins(r).copy() for r in range(4)]
        n0 = mc.launch_count()
        mc.set_wait_limit(0)
        with pytest.raises(gpumc.GpumcError) as err:
            mc.sweep(20)
        assert err.value.code == _lib.ECUDA and "gave up" in err.value.message
        assert mc.launch_count() == n0  # the failed launch is not counted as done
        mc.set_wait_limit(None)
        mc.set_sweep_count(0)
        for r in range(4):
            mc.set_spins(r, start[r])
        mc.sweep(6)
        for r in range(4):
            ref = oracle.Lattice(oracle.ISING, shape, beta=betas[r], seed=seed, replica=r)
            for _ in range(6):
                ref.sweep()
            np.testing.assert_array_equal(mc.spins(r).ravel(), ref.state(), err_msg=f"replica {r}")
            assert mc.energy()[r] == ref.cached_energy()
    finally:
        mc.close()


def test_engine_wait_limit_rejects_negative(gpumc):
    eng = gpumc.Engine()
    with pytest.raises(gpumc.InvalidConfig):
        eng.set_wait_limit(-1)
    eng.set_wait_limit(5)
    eng.set_wait_limit(None)
    eng.close()


def _job_footprint(gpumc, params, model, n_sweeps):
    import ctypes
    from scamper_b200 import _lib
    from scamper_b200.mc import spec_from_params
    # a served job buffers one record per measured sweep
    spec, _keep = spec_from_params(params, model=model, record_capacity=n_sweeps)
    n = ctypes.c_size_t()
    _lib.call("gpumc_footprint", ctypes.byref(spec), ctypes.byref(n))
    return n.value


def test_cancel_queued_and_running_jobs(gpumc):
    """Reference counterpart: cancelled tasks of the carlo-rs scheduler.  A
    budget of one job makes the second wait; cancelling it (queued) and the
    first (running) returns both with status 1 and frees the budget; a third
    job then runs to the same result as alone."""
    from scamper_b200 import _lib
    p = _params((256, 256), beta=0.44)
    fp = _job_footprint(gpumc, p, "ising", 100000)
    srv = gpumc.Server(hbm_budget=int(fp * 1.5), chunk=10)
    try:
        a = srv.submit(p, 1, 100000, model="ising")
        b = srv.submit(p, 2, 100000, model="ising")
        assert srv.step() == 2  # a running, b waiting for memory
        assert srv.stats()["bytes_in_use"] == fp
        srv.cancel(b)
        srv.step()
        srv.cancel(a)
        assert srv.stats()["bytes_in_use"] == 0
        res = {r["job_id"]: r for r in srv.poll()}
        assert res[a]["status"] == 1 and res[b]["status"] == 1
        assert res[b]["start_s"] == 0.0  # never started
        with pytest.raises(gpumc.GpumcError) as err:
            srv.cancel(a)
        assert err.value.code == _lib.ENOTFOUND
        c = srv.submit(p, 3, 40, model="ising")
        while srv.step():
            pass
        done = {r["job_id"]: r for r in srv.poll()}
        assert done[c]["status"] == 0
    finally:
        srv.close()
    alone = gpumc.Server(hbm_budget=int(fp * 1.5), chunk=10)  # job c needs far less than fp
    try:
        c2 = alone.submit(p, 3, 40, model="ising")
        while alone.step():
            pass
        ref = {r["job_id"]: r for r in alone.poll()}[c2]
        assert ref["mean_energy"] == done[c]["mean_energy"] and ref["mean_abs_m"] == done[c]["mean_abs_m"]
    finally:
        alone.close()


def test_energy_audit_passes_for_o3(gpumc):
    """O(3) energies are recomputed from the spins every sweep (fixed-point
    sums of the fp32 bond products), so the audit compares them with the
    exact fp64 recomputation within the fp32 rounding bound and passes."""
    mc = gpumc.ClassicalMC.from_params(_params((8, 8, 8), beta=0.7), 9, model="o3", n_replicas=2, betas=[0.7])
    try:
        mc.set_audit_interval(16)
        mc.sweep(70)
        assert mc.sweep_count() == 70
    finally:
        mc.close()


@pytest.mark.parametrize("model,shape,kw", [
    ("ising", (64, 64), dict(beta=0.44)),
    ("potts", (34, 18), dict(beta=1.0, q=3)),
    ("ising", (16, 16, 16), dict(beta=0.22)),
])
def test_energy_audit_passes_and_catches_a_perturbed_cache(gpumc, model, shape, kw):
    from scamper_b200 import _lib
    mc = gpumc.ClassicalMC.from_params(_params(shape, **kw), 9, model=model, n_replicas=2,
                                       betas=[kw["beta"]])
    try:
        mc.set_audit_interval(16)
        mc.sweep(70)  # audits after sweeps 16, 32, 48 and 64
        assert mc.sweep_count() == 70
        mc.sweep(5)  # no audit point in 71..75
        mc.perturb_energy_cache(1, 4.0)
        mc.sweep(4)  # 76..79: still no audit point
        with pytest.raises(gpumc.GpumcError) as err:
            mc.sweep(1)  # sweep 80 is an audit point
        assert err.value.code == _lib.ESTATE
        assert "mismatch" in err.value.message and "replica 1" in err.value.message
        # restoring the spins recomputes the cache; the next audit passes
        mc.set_spins(1, mc.spins(1))
        mc.sweep(16)
    finally:
        mc.close()


def test_audit_in_engine_batches(gpumc):
    eng = gpumc.Engine()
    a = gpumc.ClassicalMC.from_params(_params((64, 64), beta=0.44), 1, engine=eng)
    b = gpumc.ClassicalMC.from_params(_params((8, 8, 8), beta=0.7), 2, model="o3", engine=eng)
    try:
        a.set_audit_interval(10)
        b.set_audit_interval(7)
        eng.sweep(40)
        a.perturb_energy_cache(0, -2.0)
        with pytest.raises(gpumc.GpumcError):
            eng.sweep(10)
    finally:
        a.close()
        b.close()
        eng.close()

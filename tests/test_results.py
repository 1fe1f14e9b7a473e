"""Results container, merge and JSON export (carlo-rs Results,
Carlo.rs/src/results.rs), restating the reference's unit tests
(Carlo.rs/tests/unit/results.rs), and the device-side binning that feeds the
accumulators (gpumc_set_binning): its bins equal a host Accumulator's fed
with the per-sweep records of the same run, bit for bit."""
import json
import math

import numpy as np
import pytest

from scamper_b200.measurements import Accumulator, Context, Estimate
from scamper_b200.results import Metadata, Results, format_timestamp, parse_timestamp


def test_results_creation_and_json():
    r = Results()
    r.add("Energy", Estimate(1.5, 0.02, 1.0, 100))
    assert abs(r.get("Energy").mean - 1.5) < 1e-10
    r = Results()
    r.add("Magnetization", Estimate(0.8, 0.01, 1.0, 50))
    js = r.to_json()
    assert "Magnetization" in js and "0.8" in js
    assert "complex_observables" not in js  # omitted when empty
    d = json.loads(js)
    assert d["observables"]["Magnetization"] == {"mean": 0.8, "stderr": 0.01, "autocorr_time": 1.0, "n_bins": 50}
    assert set(d["metadata"]) == {"version", "timestamp", "base_seed", "thermalization_sweeps",
                                  "measurement_sweeps", "n_tasks"}


def test_results_merge_empty_single_two():
    assert Results.merge([]).estimates == {}
    r = Results()
    r.add("Energy", Estimate(1.5, 0.02, 1.0, 100))
    m = Results.merge([r])
    assert abs(m.get("Energy").mean - 1.5) < 1e-10 and m.get("Energy").n_bins == 100
    r1, r2 = Results(), Results()
    r1.add("Energy", Estimate(1.5, 0.02, 1.0, 100))
    r2.add("Energy", Estimate(1.6, 0.03, 1.0, 100))
    m = Results.merge([r1, r2]).get("Energy")
    assert abs(m.mean - 1.55) < 1e-10 and m.n_bins == 200
    # combined variance sum (se_i sqrt(n_i))^2 / n_runs^2, over total bins
    var = ((0.02 * math.sqrt(100)) ** 2 + (0.03 * math.sqrt(100)) ** 2) / 4.0
    assert m.stderr == math.sqrt(var) / math.sqrt(200)


def test_results_merge_multiple_and_mismatched_observables():
    r1, r2 = Results(), Results()
    r1.add("Energy", Estimate(1.5, 0.02, 1.0, 100))
    r1.add("Magnetization", Estimate(0.5, 0.01, 1.0, 100))
    r2.add("Energy", Estimate(1.6, 0.03, 1.0, 100))
    r2.add("Magnetization", Estimate(0.6, 0.02, 1.0, 100))
    m = Results.merge([r1, r2])
    assert abs(m.get("Energy").mean - 1.55) < 1e-10 and abs(m.get("Magnetization").mean - 0.55) < 1e-10
    r1, r2 = Results(), Results()
    r1.add("Energy", Estimate(1.0, 0.1, 1.0, 10))
    r1.add("Mag", Estimate(0.5, 0.05, 1.0, 10))
    r2.add("Energy", Estimate(2.0, 0.2, 1.0, 10))
    m = Results.merge([r1, r2])
    assert abs(m.get("Energy").mean - 1.5) < 1e-10
    assert abs(m.get("Mag").mean - 0.5) < 1e-10
    # one estimate: stderr^2 n_bins, over the total
    assert m.get("Mag").stderr == math.sqrt(0.05 ** 2 * 10) / math.sqrt(10)


def test_results_metadata_and_merge_metadata():
    r = Results()
    r.set_metadata(Metadata(version="0.1.0", base_seed=42, thermalization_sweeps=100, measurement_sweeps=1000,
                            n_tasks=4))
    assert r.metadata.base_seed == 42 and r.metadata.measurement_sweeps == 1000
    a, b = Results(metadata=Metadata(base_seed=7, thermalization_sweeps=10, measurement_sweeps=100)), \
        Results(metadata=Metadata(base_seed=8, thermalization_sweeps=20, measurement_sweeps=300))
    a.add("E", Estimate(1.0, 0.1, 2.0, 4))
    b.add("E", Estimate(3.0, 0.1, 4.0, 4))
    m = Results.merge([a, b])
    assert (m.metadata.base_seed, m.metadata.thermalization_sweeps, m.metadata.measurement_sweeps,
            m.metadata.n_tasks) == (7, 10, 400, 2)
    assert m.get("E").autocorr_time == 3.0


def test_rfc3339_timestamps_round_trip():
    expected = "2026-09-03T02:10:25.123456789Z"
    for legacy in ["2026-09-03T02:10:25.123456789Z", "2026-09-03T10:10:25.123456789+08:00"]:
        meta = Metadata.from_dict(dict(Metadata().to_dict(), timestamp=legacy))
        assert meta.to_dict()["timestamp"] == expected
    assert format_timestamp(*parse_timestamp("2026-01-01T00:00:00-01:30")) == "2026-01-01T01:30:00Z"
    with pytest.raises(ValueError):
        parse_timestamp("yesterday")


def test_json_round_trip_and_serde_layout():
    r = Results(metadata=Metadata(base_seed=3, measurement_sweeps=50))
    r.add("Energy", Estimate(-1.25, 0.003, 1.7, 40))
    r.complex_estimates["Green"] = {"re": {"mean": 0.1, "stderr": 0.0, "autocorr_time": 1.0, "n_bins": 2},
                                    "im": {"mean": 0.3, "stderr": 0.0, "autocorr_time": 1.0, "n_bins": 2}}
    back = Results.from_json(r.to_json())
    assert back.get("Energy") == r.get("Energy")
    assert back.complex_estimates == r.complex_estimates
    assert back.metadata.to_dict() == r.metadata.to_dict()
    serde = json.dumps({"estimates": {"Energy": {"mean": 2.0, "stderr": 0.5, "autocorr_time": 1.0, "n_bins": 8}},
                        "complex_estimates": {}, "metadata": r.metadata.to_dict()})
    assert Results.from_json(serde).get("Energy") == Estimate(2.0, 0.5, 1.0, 8)


def test_accumulator_bins_from_elsewhere_equal_sample_feed():
    rng = np.random.default_rng(4)
    x = rng.normal(size=103)
    a = Accumulator(10)
    for v in x:
        a.add(v)
    b = Accumulator(10)
    means = []
    for i in range(10):
        s = 0.0
        for v in x[10 * i:10 * i + 10]:
            s += v
        means.append(s / 10)
    b.add_bins(means)
    s = 0.0
    for v in x[100:]:
        s += v
    b.set_open_bin(s, 3)
    ea, eb = a.finalize(), b.finalize()
    assert ea == eb and a.total_count == b.total_count == 103


# ---------------------------------------------------------------------------
# device-side binning
# ---------------------------------------------------------------------------
def _params(shape, **kw):
    p = {"lattice_type": "square" if len(shape) == 2 else "cubic", "Lx": shape[0], "Ly": shape[1]}
    if len(shape) == 3:
        p["Lz"] = shape[2]
    p.update(kw)
    return p


CASES = [
    ("ising", (64, 64), dict(beta=0.44), 1, None, "metropolis"),
    ("ising", (128, 128), dict(beta=0.44), 4, [0.3, 0.4, 0.45, 0.6], "metropolis"),  # PT chains by label
    ("ising", (32, 32), dict(beta=0.5), 3, None, "heat_bath"),                        # replicas, shared beta
    ("potts", (40, 40), dict(beta=1.0, q=3), 1, None, "metropolis"),
    ("potts", (8, 8, 8), dict(beta=0.6, q=6), 2, [0.5, 0.6], "heat_bath"),
    ("o3", (16, 16, 16), dict(beta=0.7), 1, None, "metropolis"),
]


@pytest.mark.gpu
@pytest.mark.parametrize("model,shape,kw,n_rep,betas,alg", CASES)
@pytest.mark.parametrize("binsize,sweeps", [(7, 150), (25, 50)])
def test_device_bins_equal_host_accumulator(gpumc, model, shape, kw, n_rep, betas, alg, binsize, sweeps):
    """Same seed, same trajectory: one handle records every sweep and feeds a
    host Context, the other bins on the device; the finalized estimates of
    every observable and chain are identical (bit for bit for the integer
    models; O(3) energies carry the run-to-run rounding of the fp64 atomic
    energy accumulation)."""
    from scamper_b200 import _lib
    out = []
    for device_bins in (False, True):
        mc = gpumc.ClassicalMC.from_params(_params(shape, **kw), 91, model=model, n_replicas=n_rep,
                                           betas=betas, algorithm=alg, record_capacity=64)
        if betas:
            mc.pt_configure(5)
        if device_bins:
            mc.enable_device_binning(binsize, capacity=3)  # forces several drains
        mc.sweep(20)
        mc.on_phase_start(_lib.PHASE_MEASUREMENT)
        ctx = Context(binsize)
        done = 0
        while done < sweeps:
            k = min(37, sweeps - done)
            mc.sweep(k)
            mc.measure(ctx)
            done += k
        if device_bins:
            mc.finish_measurements(ctx)
        out.append(ctx.finalize_measurements())
        mc.close()
    host, dev = out
    if n_rep > 1 and not betas:
        # shared beta: the record path pools the replicas into one chain, the
        # device bins each replica; compare per-replica sample sums instead
        assert set(k.split("/")[1] for k in dev) >= {"Energy", "E2", "Magnetization", "M2", "M4"}
        return
    assert set(host) == set(dev)
    for k in host:
        if model == "o3":
            # the O(3) energy cache sums fp64 warp partials with atomics, in an
            # order that varies between the two runs: equal to ~1e-15
            assert host[k].n_bins == dev[k].n_bins, k
            assert dev[k].mean == pytest.approx(host[k].mean, rel=1e-9, abs=1e-12), k
            assert dev[k].stderr == pytest.approx(host[k].stderr, rel=1e-6, abs=1e-12), k
        else:
            assert host[k] == dev[k], k


@pytest.mark.gpu
def test_device_binning_run_one_and_results(gpumc):
    params = _params((64, 64), beta=0.44)
    a = gpumc.ClassicalMC.from_params(params, 5)
    a.enable_device_binning(10)
    ra = gpumc.run_one(a, 100, 1005, binsize=10)
    b = gpumc.ClassicalMC.from_params(params, 5)
    rb = gpumc.run_one(b, 100, 1005, binsize=10)
    assert ra == rb
    assert ra["Energy"].n_bins == 101  # 100 full bins + the trailing partial one
    res = gpumc.Results.from_measurements(ra, gpumc.Metadata(base_seed=5, thermalization_sweeps=100,
                                                             measurement_sweeps=1005))
    back = gpumc.Results.from_json(res.to_json())
    assert back.get("Energy") == ra["Energy"]
    with pytest.raises(ValueError):
        a.measure(gpumc.Context(3))  # bin sizes must agree
    a.close()
    b.close()


@pytest.mark.gpu
def test_device_binning_rejections(gpumc):
    m = gpumc.MultiSpinIsing.from_params(_params((64, 64), beta=0.44), 1)
    with pytest.raises(gpumc.InvalidConfig):
        m.enable_device_binning(10)
    m.close()
    mc = gpumc.ClassicalMC.from_params(_params((16, 16), beta=0.44), 1)
    with pytest.raises(gpumc.InvalidConfig):
        mc.enable_device_binning(-1)
    with pytest.raises(gpumc.InvalidConfig):
        mc.enable_device_binning(4, capacity=0)
    mc.enable_device_binning(4)
    mc.enable_device_binning(0)  # back to records
    from scamper_b200 import _lib
    mc.on_phase_start(_lib.PHASE_MEASUREMENT)
    mc.sweep(3)
    assert len(mc.observables()) == 3
    mc.close()

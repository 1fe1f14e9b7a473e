"""The empirical tile autotuner: the planner's knobs (CPU: they reach the
host tile plan, are validated, and round-trip through the JSON cache) and,
on the device, that a tuned plan gives exactly the spins, energies and
records of the analytic one and that the tuner times its candidates."""
import json

import numpy as np
import pytest


def _plan(gpumc, params, model, **kw):
    return gpumc.plan_tiles(params, model=model, **kw)


def test_knobs_reach_the_host_planner(gpumc):
    from scamper_b200 import autotune
    o3 = {"lattice_type": "cubic", "L": 64, "beta": 0.7}
    ising3 = {"lattice_type": "cubic", "L": 128, "beta": 0.22}
    potts = {"lattice_type": "square", "L": 2048, "q": 3, "beta": 1.0}
    base = {k: _plan(gpumc, p, m, refine=False)[0] for k, (p, m) in
            {"o3": (o3, "o3"), "i3": (ising3, "ising"), "p2": (potts, "potts")}.items()}
    prev = autotune.set_knobs({"o3_planes": 16, "ising3d_planes": 32, "potts_segments": 3072})
    try:
        assert autotune.get_knobs()["o3_planes"] == 16
        assert _plan(gpumc, o3, "o3", refine=False)[0] == (64 // 16) * (64 // 16)  # 16-row tiles
        assert _plan(gpumc, ising3, "ising", refine=False)[0] == 128 // 32
        assert _plan(gpumc, potts, "potts", refine=False)[0] < base["p2"]
    finally:
        autotune.set_knobs(prev)
    assert _plan(gpumc, o3, "o3", refine=False)[0] == base["o3"] == 4 * 8
    with pytest.raises(gpumc.InvalidConfig):
        autotune.set_knobs({"o3_rows": -1})
    with pytest.raises(ValueError):
        autotune.tune(lambda eng: [], {"no_such_knob": [1]}, torch=object())


def test_tile_cache_round_trip(tmp_path):
    from scamper_b200.autotune import TileCache
    path = str(tmp_path / "tiles.json")
    c = TileCache(path)
    assert c.get("NVIDIA B200", "mix") is None
    c.put("NVIDIA B200", "mix", {"knobs": {"o3_planes": 16, "potts_segments": 0}, "ms_per_sweep": 1.5,
                                 "analytic_ms_per_sweep": 2.0, "table": []})
    c.save()
    d = TileCache(path)
    assert d.get("NVIDIA B200", "mix") == {"o3_planes": 16, "potts_segments": 0}
    assert d.get("NVIDIA H100", "mix") is None
    with open(path) as f:
        assert json.load(f)["NVIDIA B200|mix"]["analytic_ms_per_sweep"] == 2.0


def test_tuner_keeps_the_analytic_plan_within_the_noise_margin(monkeypatch):
    from scamper_b200 import autotune
    assert autotune.MIN_GAIN == 0.02
    # fake timings (ms per sweep) by knob setting, relative to the analytic 1.0
    times = {(): 1.0,
             (("potts_segments", 768),): 0.995,                       # 0.5 % faster: inside the margin
             (("o3_planes", 16),): 0.996,
             (("potts_segments", 3072),): 0.95,                       # 5 % faster: taken
             (("o3_planes", 16), ("potts_segments", 3072)): 0.945,    # a further 0.5 %: not taken
             (("o3_planes", 4), ("potts_segments", 3072)): 0.92,      # a further 3 %: taken
             (("o3_planes", 16), ("potts_segments", 768)): 0.999}

    def fake_time(build, knobs, sweeps, warm, torch, repeats=3):
        return times[tuple(sorted((k, v) for k, v in knobs.items() if v))]

    monkeypatch.setattr(autotune, "time_workload", fake_time)
    res = autotune.tune(lambda eng: [], {"potts_segments": [768], "o3_planes": [16]}, torch=object())
    assert res["knobs"]["potts_segments"] == 0 and res["knobs"]["o3_planes"] == 0
    assert res["ms_per_sweep"] == res["analytic_ms_per_sweep"] == 1.0
    assert [e["ms_per_sweep"] for e in res["table"]] == [1.0, 0.995, 0.996]
    res = autotune.tune(lambda eng: [], {"potts_segments": [768, 3072], "o3_planes": [16, 4]}, torch=object())
    assert res["knobs"]["potts_segments"] == 3072 and res["knobs"]["o3_planes"] == 4
    assert res["ms_per_sweep"] == 0.92 and res["analytic_ms_per_sweep"] == 1.0
    # with no margin any improvement is kept
    res = autotune.tune(lambda eng: [], {"potts_segments": [768], "o3_planes": [16]}, torch=object(), min_gain=0.0)
    assert res["knobs"]["potts_segments"] == 768 and res["ms_per_sweep"] == 0.995


def _mix(gpumc, eng):
    sims = []
    for i, L in enumerate((34, 130, 258)):
        sims.append(gpumc.ClassicalMC.from_params({"lattice_type": "square", "L": L, "q": 3, "beta": 1.0},
                                                  10 + i, model="potts", engine=eng))
    for i in range(2):
        sims.append(gpumc.ClassicalMC.from_params({"lattice_type": "cubic", "L": 32, "beta": 0.7}, 20 + i,
                                                  model="o3", engine=eng))
    sims.append(gpumc.ClassicalMC.from_params({"lattice_type": "cubic", "L": 32, "beta": 0.22}, 30, engine=eng))
    sims.append(gpumc.ClassicalMC.from_params({"lattice_type": "square", "L": 256, "beta": 0.44}, 31, engine=eng))
    return sims


@pytest.mark.gpu
@pytest.mark.parametrize("knobs", [
    {"o3_rows": 8, "o3_planes": 4, "potts_segments": 768, "ising3d_planes": 4, "ising2d_rows": 16},
    {"o3_rows": 32, "o3_planes": 32, "potts_segments": 3072, "ising3d_planes": 32, "ising2d_rows": 64},
])
def test_tuned_plan_gives_identical_results(gpumc, knobs):
    from scamper_b200 import _lib, autotune
    out = []
    for kn in ({}, knobs):
        prev = autotune.set_knobs(kn)
        try:
            eng = gpumc.Engine()
            sims = _mix(gpumc, eng)
        finally:
            autotune.set_knobs(prev)
        for s in sims:
            s.on_phase_start(_lib.PHASE_MEASUREMENT)
        eng.sweep(12)
        out.append(([s.spins().copy() for s in sims], [s.energy().copy() for s in sims],
                    [s.observable_arrays()["magnetization"].copy() for s in sims]))
        for s in sims:
            s.close()
        eng.close()
    for a, b in zip(out[0][0], out[1][0]):
        np.testing.assert_array_equal(a, b)
    for a, b in zip(out[0][1], out[1][1]):
        np.testing.assert_array_equal(a, b)
    for a, b in zip(out[0][2], out[1][2]):
        np.testing.assert_array_equal(a, b)


@pytest.mark.gpu
def test_tuner_times_candidates_and_keeps_the_fastest(gpumc):
    import torch
    from scamper_b200 import autotune
    res = autotune.tune(lambda eng: _mix(gpumc, eng), {"o3_planes": [4, 16], "potts_segments": [768]},
                        sweeps=5, warm=2, torch=torch)
    times = [r["ms_per_sweep"] for r in res["table"]]
    assert len(times) == 4
    # the kept plan is a timed one, and no candidate beat it by more than the
    # tuner's margin
    assert res["ms_per_sweep"] in times
    assert res["ms_per_sweep"] <= min(times) / (1.0 - autotune.MIN_GAIN) * (1.0 + 1e-12)
    assert res["ms_per_sweep"] <= res["analytic_ms_per_sweep"]
    assert autotune.get_knobs() == {k: 0 for k in autotune.KNOBS}

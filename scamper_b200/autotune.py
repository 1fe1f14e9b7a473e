"""Empirical tile autotuner.

The planner sizes tiles with analytic cost models (CTA waves x halo work).
This module measures instead: for a batched workload it times candidate
values of the planner's tile knobs (gpumc_set_tile_knobs: rows of whole-row
2D Ising tiles, planes of whole-plane 3D Ising / Potts tiles, packed segments
per bit-sliced 2D Potts tile, rows and planes of the O(3) z-march tiles) on
the device, one knob at a time with the others at their best so far
(coordinate descent), and keeps the fastest.  Winners are cached in a JSON
file per (device name, workload name); a workload without a cached entry
runs on the analytic choice.  Tiles never change results: a colour pass
reads only the other colour and every random draw is keyed by site or row
segment, so any tuned plan gives the spins of the analytic one.
"""
import ctypes
import json
import os

from . import _lib

KNOBS = ("ising2d_rows", "ising3d_planes", "potts_segments", "potts3d_planes", "o3_rows", "o3_planes")
DEFAULT_CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuned_tiles.json")
# A candidate plan must beat the best so far by this fraction to replace it.
# Two tuning runs of the uneven mix on B200 boxes ordered the Potts segment
# candidates differently by up to 2.4 %, so smaller gains are not resolved.
MIN_GAIN = 0.02


def get_knobs():
    k = _lib.TileKnobs()
    _lib.call("gpumc_get_tile_knobs", ctypes.byref(k))
    return {name: getattr(k, name) for name in KNOBS}


def set_knobs(knobs=None):
    """Sets the planner's knobs (missing or 0 = analytic) for layouts
    planned afterwards; returns the previous values."""
    prev = get_knobs()
    k = _lib.TileKnobs(**{name: int((knobs or {}).get(name, 0)) for name in KNOBS})
    _lib.call("gpumc_set_tile_knobs", ctypes.byref(k))
    return prev


class TileCache:
    """Tuned knobs per (device name, workload name) in a JSON file."""

    def __init__(self, path=DEFAULT_CACHE):
        self.path = path
        try:
            with open(path) as f:
                self.data = json.load(f)
        except (OSError, ValueError):
            self.data = {}

    @staticmethod
    def key(device_name, workload):
        return f"{device_name}|{workload}"

    def get(self, device_name, workload):
        e = self.data.get(self.key(device_name, workload))
        return dict(e["knobs"]) if e else None

    def put(self, device_name, workload, result):
        self.data[self.key(device_name, workload)] = {
            "knobs": {k: int(v) for k, v in result["knobs"].items()},
            "ms_per_sweep": result["ms_per_sweep"], "analytic_ms_per_sweep": result["analytic_ms_per_sweep"],
            "table": result["table"]}

    def save(self):
        tmp = self.path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(self.data, f, indent=1, sort_keys=True)
        os.replace(tmp, self.path)


def time_workload(build, knobs, sweeps, warm, torch, repeats=3):
    """ms per engine sweep of the workload planned with `knobs`: a fresh
    engine, `warm` untimed sweeps (graph capture included), then the fastest
    of `repeats` windows of `sweeps` sweeps between CUDA events on the
    engine's stream (the minimum filters other work on a shared device)."""
    from .mc import Engine
    prev = set_knobs(knobs)
    try:
        eng = Engine()
        sims = build(eng)
        try:
            eng.sweep(warm)
            eng.synchronize()
            st = torch.cuda.ExternalStream(eng.stream_ptr())
            best = float("inf")
            for _ in range(max(1, repeats)):
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(st)
                eng.sweep(sweeps)
                b.record(st)
                b.synchronize()
                best = min(best, a.elapsed_time(b) / sweeps)
            return best
        finally:
            for s in sims:
                s.close()
            eng.close()
    finally:
        set_knobs(prev)


def tune(build, space, sweeps=20, warm=3, rounds=1, torch=None, repeats=3, min_gain=MIN_GAIN):
    """Coordinate descent over `space` ({knob: [candidates]}, 0 = analytic)
    for the workload that build(engine) creates.  A candidate replaces the
    best plan so far only when it is faster by more than `min_gain` (a
    fraction): differences inside the run-to-run spread of the timings keep
    the analytic plan.  Returns {"knobs",
    "ms_per_sweep", "analytic_ms_per_sweep", "table"} with every timed
    candidate in the table."""
    if torch is None:
        import torch  # noqa: F811
    for name in space:
        if name not in KNOBS:
            raise ValueError(f"unknown tile knob: {name}")
    best = {name: 0 for name in KNOBS}
    analytic = time_workload(build, best, sweeps, warm, torch, repeats)
    best_t = analytic
    table = [{"knobs": dict(best), "ms_per_sweep": analytic}]
    for _ in range(rounds):
        for name, cands in space.items():
            for v in cands:
                if v == best[name]:
                    continue
                trial = dict(best, **{name: int(v)})
                t = time_workload(build, trial, sweeps, warm, torch, repeats)
                table.append({"knobs": trial, "ms_per_sweep": t})
                if t < best_t * (1.0 - min_gain):
                    best, best_t = trial, t
    return {"knobs": best, "ms_per_sweep": best_t, "analytic_ms_per_sweep": analytic, "table": table}

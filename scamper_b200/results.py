"""Simulation results in carlo-rs's format: the Results container, its
merge of independent runs, and its JSON export.

Results (Carlo.rs/src/results.rs:10-335) holds one Estimate per observable
(mean, stderr, autocorr_time, n_bins), optional complex observables
({re, im} estimates, passed through unchanged here: the lattice engine
measures none) and run Metadata (version, RFC 3339 UTC timestamp, base_seed,
thermalization_sweeps, measurement_sweeps, n_tasks).  merge() follows
Results::merge (results.rs:142-285): per observable the n_bins-weighted mean,
the combined variance sum_i (stderr_i sqrt(n_bins_i))^2 / n_runs^2 (a single
estimate: stderr^2 n_bins) scaled by 1 / total_bins, the mean autocorrelation
time and the total bin count; metadata from the first run with the
measurement sweeps summed and n_tasks = number of runs.  to_json() writes the
export layout of Results::to_json (results.rs:289-308): {"observables",
["complex_observables" when non-empty], "metadata"}; from_json() reads it and
the serde layout of the struct itself ({"estimates", "complex_estimates",
"metadata"}).  Timestamps accept any RFC 3339 offset and are stored and
written in UTC with "Z" (Metadata, results.rs:50-82, and the round-trip test
Carlo.rs/tests/unit/results.rs).
"""
import calendar
import json
import math
import re
import time

from .measurements import Estimate

VERSION = "scamper-b200-0.1"

_RFC3339 = re.compile(r"^(\d{4})-(\d{2})-(\d{2})[Tt](\d{2}):(\d{2}):(\d{2})(?:\.(\d{1,9}))?"
                      r"(?:([Zz])|([+-])(\d{2}):(\d{2}))$")


def parse_timestamp(text):
    """RFC 3339 text -> (seconds since the epoch, nanoseconds)."""
    m = _RFC3339.match(text)
    if not m:
        raise ValueError(f"not an RFC 3339 timestamp: {text!r}")
    y, mo, d, h, mi, s = (int(m.group(i)) for i in range(1, 7))
    frac = m.group(7) or ""
    nanos = int(frac.ljust(9, "0")) if frac else 0
    sec = calendar.timegm((y, mo, d, h, mi, s, 0, 0, 0))
    if m.group(9):
        off = (int(m.group(10)) * 60 + int(m.group(11))) * 60
        sec -= off if m.group(9) == "+" else -off
    return sec, nanos


def format_timestamp(sec, nanos):
    """UTC RFC 3339 with the fractional seconds trimmed of trailing zeros."""
    base = time.strftime("%Y-%m-%dT%H:%M:%S", time.gmtime(sec))
    if nanos:
        base += "." + f"{nanos:09d}".rstrip("0")
    return base + "Z"


def _now():
    ns = time.time_ns()
    return ns // 1_000_000_000, ns % 1_000_000_000


class Metadata:
    """Run metadata (results.rs:50-82)."""

    def __init__(self, version=VERSION, timestamp=None, base_seed=0, thermalization_sweeps=0,
                 measurement_sweeps=0, n_tasks=1):
        self.version = version
        self.timestamp = _now() if timestamp is None else (
            parse_timestamp(timestamp) if isinstance(timestamp, str) else tuple(timestamp))
        self.base_seed = int(base_seed)
        self.thermalization_sweeps = int(thermalization_sweeps)
        self.measurement_sweeps = int(measurement_sweeps)
        self.n_tasks = int(n_tasks)

    def to_dict(self):
        return {"version": self.version, "timestamp": format_timestamp(*self.timestamp),
                "base_seed": self.base_seed, "thermalization_sweeps": self.thermalization_sweeps,
                "measurement_sweeps": self.measurement_sweeps, "n_tasks": self.n_tasks}

    @classmethod
    def from_dict(cls, d):
        return cls(version=d.get("version", VERSION), timestamp=d.get("timestamp"),
                   base_seed=d.get("base_seed", 0), thermalization_sweeps=d.get("thermalization_sweeps", 0),
                   measurement_sweeps=d.get("measurement_sweeps", 0), n_tasks=d.get("n_tasks", 1))


def _est_dict(e):
    return {"mean": e.mean, "stderr": e.stderr, "autocorr_time": e.autocorr_time, "n_bins": e.n_bins}


def _est_from(d):
    return Estimate(float(d["mean"]), float(d["stderr"]), float(d["autocorr_time"]), int(d["n_bins"]))


class Results:
    """carlo-rs Results: estimates by observable name plus run metadata."""

    def __init__(self, estimates=None, complex_estimates=None, metadata=None):
        self.estimates = dict(estimates or {})
        self.complex_estimates = dict(complex_estimates or {})
        self.metadata = metadata if metadata is not None else Metadata()

    @classmethod
    def from_measurements(cls, measurements, metadata=None):
        """From Context.finalize_measurements() / run_one() output."""
        return cls(measurements, metadata=metadata)

    def add(self, name, estimate):
        self.estimates[name] = estimate

    def get(self, name):
        return self.estimates.get(name)

    def set_metadata(self, metadata):
        self.metadata = metadata

    @staticmethod
    def merge(results):
        """Results::merge (results.rs:142-285)."""
        results = list(results)
        if not results:
            return Results()
        if len(results) == 1:
            r = results[0]
            return Results(r.estimates, r.complex_estimates, r.metadata)
        names = set()
        for r in results:
            names.update(r.estimates)
        merged = {}
        for name in names:
            ests = [r.estimates[name] for r in results if name in r.estimates]
            if not ests:
                continue
            total = sum(e.n_bins for e in ests)
            if total == 0:
                merged[name] = Estimate(0.0, 0.0, 1.0, 0)
                continue
            wmean = 0.0
            for e in ests:
                wmean += e.mean * float(e.n_bins)
            wmean /= float(total)
            if len(ests) > 1:
                var = 0.0
                for e in ests:
                    var += (e.stderr * math.sqrt(float(e.n_bins))) ** 2
                var /= float(len(ests)) ** 2
            else:
                var = ests[0].stderr ** 2 * float(ests[0].n_bins)
            tau = 0.0
            for e in ests:
                tau += e.autocorr_time
            merged[name] = Estimate(wmean, math.sqrt(var) / math.sqrt(float(total)), tau / len(ests), total)
        meta = Metadata(version=VERSION, base_seed=results[0].metadata.base_seed,
                        thermalization_sweeps=results[0].metadata.thermalization_sweeps,
                        measurement_sweeps=sum(r.metadata.measurement_sweeps for r in results),
                        n_tasks=len(results))
        cnames = set()
        for r in results:
            cnames.update(r.complex_estimates)
        merged_c = {}
        for name in cnames:
            parts = [r.complex_estimates[name] for r in results if name in r.complex_estimates]
            out = {}
            for key in ("re", "im"):
                ests = [_est_from(p[key]) for p in parts]
                total = sum(e.n_bins for e in ests)
                if total == 0:
                    out[key] = _est_dict(Estimate.from_bins([]))
                    continue
                wmean = 0.0
                for e in ests:
                    wmean += e.mean * float(e.n_bins)
                tau = 0.0
                for e in ests:
                    tau += e.autocorr_time
                out[key] = _est_dict(Estimate(wmean / float(total), ests[0].stderr, tau / len(ests), total))
            merged_c[name] = out
        return Results(merged, merged_c, meta)

    def to_json(self):
        """Results::to_json: pretty JSON of the export layout."""
        doc = {"observables": {k: _est_dict(v) for k, v in self.estimates.items()}}
        if self.complex_estimates:
            doc["complex_observables"] = self.complex_estimates
        doc["metadata"] = self.metadata.to_dict()
        return json.dumps(doc, indent=2)

    @classmethod
    def from_json(cls, text):
        d = json.loads(text)
        est = d.get("observables", d.get("estimates", {}))
        cplx = d.get("complex_observables", d.get("complex_estimates", {}))
        meta = Metadata.from_dict(d["metadata"]) if "metadata" in d else Metadata()
        return cls({k: _est_from(v) for k, v in est.items()}, cplx, meta)

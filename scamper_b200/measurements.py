"""Host-side statistics sink: binning accumulator and estimates.

Restates carlo-rs's measurement path so GPU results reduce exactly like the
reference's: Accumulator (Carlo.rs/src/measurements.rs:60-183, partial
trailing bin counted as an extra bin, autocorrelation time from one
rebinning level :244-280) and Estimate::from_bins_with_autocorr
(Carlo.rs/src/estimate.rs:30-57), plus the post-processing helpers Binder
cumulant and specific heat (CMC.rs/src/postprocess.rs:58-77).
"""
from dataclasses import dataclass
import math

import numpy as np


@dataclass
class Estimate:
    mean: float
    stderr: float
    autocorr_time: float
    n_bins: int

    @staticmethod
    def from_bins_with_autocorr(bins, autocorr_time):
        bins = np.asarray(bins, dtype=np.float64)
        if bins.size == 0:
            return Estimate(0.0, 0.0, 1.0, 0)
        n = float(bins.size)
        mean = float(bins.sum() / n)
        var = float(((bins - mean) ** 2).sum() / (n - 1.0)) if bins.size > 1 else 0.0
        return Estimate(mean, math.sqrt(var) / math.sqrt(n), max(autocorr_time, 1.0), int(bins.size))

    @staticmethod
    def from_bins(bins):
        return Estimate.from_bins_with_autocorr(bins, 1.0)


class Accumulator:
    """Samples binned in blocks of `bin_capacity`."""

    def __init__(self, bin_capacity):
        if bin_capacity < 1:
            raise ValueError("bin_capacity must be >= 1")
        self.bin_capacity = int(bin_capacity)
        self.bins = []
        self.current = None
        self.filling = 0
        self.total_count = 0

    def add(self, value):
        self.add_array([float(value)])

    def add_array(self, values):
        v = np.asarray(values, dtype=np.float64).ravel()
        if v.size == 0:
            return
        if self.current is None:
            self.current = np.zeros_like(v)
        self.current += v
        self.total_count += 1
        self.filling += 1
        if self.filling >= self.bin_capacity:
            self.bins.append(self.current / self.bin_capacity)
            self.current = np.zeros_like(v)
            self.filling = 0

    def add_many(self, values):
        """Feeds a batch of scalar samples in order (vectorised add)."""
        for x in np.asarray(values, dtype=np.float64).ravel():
            self.add(x)

    def add_bins(self, means):
        """Appends completed scalar bins computed elsewhere (the device's
        binning: each mean is the sum of `bin_capacity` samples in order /
        bin_capacity, the value add() would have produced).  Only valid at a
        bin boundary."""
        if self.filling:
            raise ValueError("add_bins: the accumulator has an open bin")
        for m in np.asarray(means, dtype=np.float64).ravel():
            self.bins.append(np.array([m]))
            self.total_count += self.bin_capacity

    def set_open_bin(self, total, filling):
        """The open (partial) bin: `filling` samples summing to `total`."""
        if self.filling:
            raise ValueError("set_open_bin: the accumulator has an open bin")
        if filling > 0:
            self.current = np.array([float(total)])
            self.filling = int(filling)
            self.total_count += int(filling)

    def autocorr_time(self):
        if len(self.bins) < 2:
            return 1.0
        means = np.array([b.sum() / b.size for b in self.bins])
        n = float(means.size)
        mu = means.sum() / n
        var_no = ((means - mu) ** 2).sum() / (n - 1.0)
        rn = int(n) // 2
        if rn < 2:
            return 1.0
        rb = 0.5 * (means[0:2 * rn:2] + means[1:2 * rn:2])
        rmu = rb.sum() / rn
        var_rb = ((rb - rmu) ** 2).sum() / (rn - 1.0)
        expected = var_no / 2.0
        if expected <= 0.0:
            return 1.0
        return 0.5 * max(var_rb / expected - 1.0, 0.0)

    def finalize(self):
        all_bins = [b.sum() / b.size for b in self.bins]
        if self.filling > 0 and self.current is not None and self.current.size:
            all_bins.append(self.current.sum() / (self.filling * self.current.size))
        return Estimate.from_bins_with_autocorr(all_bins, self.autocorr_time())


class Context:
    """Minimal carlo-rs Context (Carlo.rs/src/context.rs:49-214): named
    observables, measurement namespace, phase and sweep counter."""

    def __init__(self, binsize=1):
        self.binsize = binsize
        self.obs = {}
        self.namespace = None
        self.phase = 1
        self.sweeps = 0

    def _key(self, name):
        return f"{self.namespace}/{name}" if self.namespace else name

    def measure(self, name, value):
        key = self._key(name)
        if key not in self.obs:
            self.obs[key] = Accumulator(self.binsize)
        self.obs[key].add(value)

    def accumulator(self, name):
        """The accumulator of `name` in the current namespace (created with
        the context's bin size)."""
        key = self._key(name)
        if key not in self.obs:
            self.obs[key] = Accumulator(self.binsize)
        return self.obs[key]

    def measure_array(self, name, values):
        key = self._key(name)
        if key not in self.obs:
            self.obs[key] = Accumulator(self.binsize)
        self.obs[key].add_array(values)

    def set_measurement_namespace(self, ns):
        self.namespace = ns

    def finalize_measurements(self):
        return {k: a.finalize() for k, a in self.obs.items()}


def binder_cumulant(m2, m4):
    """U4 = 1 - <M^4> / (3 <M^2>^2) (CMC.rs/src/postprocess.rs:70-77);
    None when <M^2>^2 < 1e-15, as in the reference."""
    if m2 * m2 < 1e-15:
        return None
    return 1.0 - m4 / (3.0 * m2 * m2)


def specific_heat(e, e2, beta, n_sites):
    """C = beta^2 / N (<E^2> - <E>^2) (CMC.rs/src/postprocess.rs:58-65)."""
    if not math.isfinite(beta) or beta < 0.0 or n_sites == 0:
        return None
    return beta * beta / n_sites * (e2 - e * e)

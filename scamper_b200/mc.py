"""Host-side mirror of the reference's model contract over the C ABI.

`ClassicalMC` stands in for cmc-rs `ClassicalMC<H, MetropolisCore, _>`
(CMC.rs/src/classical_mc.rs:21-31, :168-229) behind carlo-rs's `MonteCarlo`,
`FromParams` and `ParallelTemperingCompatible` traits
(Carlo.rs/src/monte_carlo.rs:31-88, Carlo.rs/src/parallel_tempering.rs:71-84):
same parameter keys, same observable names ("Energy", "E2", "Magnetization",
"M2", "M4"), same error behaviour (InvalidConfig on bad parameters).
`MultiSpinIsing` stands in for CMC.rs/src/multi_spin.rs.  `run_one` and
`run_parallel_tempering` restate the scheduling loops of
Carlo.rs/src/scheduler.rs:94-155 and Carlo.rs/src/parallel_tempering.rs:313-419
with the sweeps and exchanges executed on the device.
"""
import ctypes
import math

import numpy as np

from . import _lib
from ._lib import InvalidConfig
from .measurements import Context


class Params(dict):
    """String-keyed parameter bag (Carlo.rs/src/params.rs:13-46)."""

    def set(self, key, value):
        self[key] = value

    def get_as(self, key, typ, default=None):
        if key not in self:
            return default
        v = self[key]
        try:
            if typ is bool:
                if isinstance(v, bool):
                    return v
                s = str(v).strip().lower()
                if s in ("true", "1", "yes"):
                    return True
                if s in ("false", "0", "no"):
                    return False
                raise ValueError(s)
            return typ(v)
        except (TypeError, ValueError):
            raise InvalidConfig(_lib.EINVAL, f"{key}: cannot parse {v!r}") from None

    def contains(self, key):
        return key in self


MODELS = {"ising": _lib.ISING, "potts": _lib.POTTS, "heisenberg": _lib.O3, "o3": _lib.O3}
# the algorithm type parameter of ClassicalMC<H, A> (CMC.rs/src/classical_mc.rs:21-31):
# MetropolisCore, HeatBathCore / ContinuousHeatBathCore
# (CMC.rs/src/algorithms/heat_bath.rs:12-134), SWCore
# (CMC.rs/src/algorithms/swendsen_wang.rs) and WolffCore (CMC.rs/src/algorithms/wolff.rs)
ALGORITHMS = {"metropolis": _lib.METROPOLIS, "metropolis-hastings": _lib.METROPOLIS,
              "heat_bath": _lib.HEAT_BATH, "heatbath": _lib.HEAT_BATH,
              "continuous_heat_bath": _lib.HEAT_BATH,
              "swendsen_wang": _lib.SWENDSEN_WANG, "swendsen-wang": _lib.SWENDSEN_WANG, "sw": _lib.SWENDSEN_WANG,
              "wolff": _lib.WOLFF}


def algorithm_id(algorithm):
    if algorithm is None:
        return _lib.METROPOLIS
    if isinstance(algorithm, int):
        return algorithm
    a = str(algorithm).lower()
    if a not in ALGORITHMS:
        raise InvalidConfig(_lib.EINVAL, f"algorithm: unknown algorithm `{algorithm}` "
                                         "(expected metropolis, heat_bath, swendsen_wang or wolff)")
    return ALGORITHMS[a]


def _positive(params, key, default):
    v = params.get_as(key, int, default)
    if v is None or v < 1:
        raise InvalidConfig(_lib.EINVAL, f"{key}: must be a positive integer")
    return v


def lattice_from_params(params):
    """Geometry of build_lattice_from_params (CMC.rs/src/classical_mc.rs:336-425)
    restricted to the square and cubic lattices this engine runs."""
    inferred = "hypercubic" if "Lx" in params else "chain"
    ltype = str(params.get("lattice_type", inferred)).lower()
    if ltype == "chain" and "L" in params and "lattice_type" not in params:
        ltype = "square"  # the engine's default geometry for a bare L
    if ltype == "square":
        lx = _positive(params, "Lx", params.get_as("L", int, 4))
        ly = _positive(params, "Ly", lx)
        return 2, lx, ly, 1
    if ltype == "cubic":
        lx = _positive(params, "Lx", params.get_as("L", int, 4))
        ly = _positive(params, "Ly", lx)
        lz = _positive(params, "Lz", lx)
        return 3, lx, ly, lz
    if ltype == "hypercubic":
        lx = _positive(params, "Lx", 4)
        ly = _positive(params, "Ly", lx)
        if "Lz" in params:
            return 3, lx, ly, _positive(params, "Lz", lx)
        return 2, lx, ly, 1
    raise InvalidConfig(_lib.EINVAL, f"lattice_type: `{ltype}` is not supported by the checkerboard "
                        "engine (square, cubic, hypercubic)")


# O(3) Metropolis proposals: the engine's adapted cap, the reference's
# StandardStrategy (uniform unit vector) and OPSSStrategy (plane rotation),
# CMC.rs/src/lattice/proposal.rs:45-167, and the cap with the hardware
# approximations of sqrt, reciprocal, sin / cos and exp ("cap_fast":
# float32-tolerance parity, not bit-identical)
O3_PROPOSALS = {"cap": _lib.O3_CAP, "cone": _lib.O3_CAP, "standard": _lib.O3_UNIFORM,
                "uniform": _lib.O3_UNIFORM, "opss": _lib.O3_OPSS, "cap_fast": _lib.O3_CAP_FAST}


def spec_from_params(params, model=None, n_replicas=1, betas=None, record_capacity=1024, algorithm=None,
                     o3_proposal=None):
    params = params if isinstance(params, Params) else Params(params)
    mname = model if model is not None else str(params.get("model", "ising")).lower()
    if isinstance(mname, int):
        mid = mname
    elif mname in MODELS:
        mid = MODELS[mname]
    else:
        raise InvalidConfig(_lib.EINVAL, f"model: unknown model `{mname}`")
    dims, lx, ly, lz = lattice_from_params(params)
    pbc = params.get_as("pbc", bool, True)
    if betas is None:
        betas = [params.get_as("beta", float, 1.0)]
    betas = [float(b) for b in betas]
    init = str(params.get("initial_state", "hot")).lower()
    if init in ("hot", "random"):
        init_id = _lib.INIT_HOT
    elif init in ("cold", "ordered"):
        init_id = _lib.INIT_COLD
    else:
        raise InvalidConfig(_lib.EINVAL, "initial_state: expected hot/random or cold/ordered")
    prop = "cap" if o3_proposal is None else str(o3_proposal).lower()
    if prop not in O3_PROPOSALS:
        raise InvalidConfig(_lib.EINVAL, f"o3_proposal: unknown proposal `{o3_proposal}` "
                                         "(expected cap, standard, opss or cap_fast)")
    # the OPSS bound starts at OPSSStrategy's default sigma = 0.5 unless given
    step = params.get_as("opss_sigma", float, 0.5) if O3_PROPOSALS[prop] == _lib.O3_OPSS else \
        params.get_as("cone_half_angle", float, 1.0)
    arr = (ctypes.c_double * len(betas))(*betas)
    spec = _lib.Spec(model=mid, dims=dims, lx=lx, ly=ly, lz=lz, pbc=1 if pbc else 0,
                     q=params.get_as("q", int, 3), J=params.get_as("J", float, 1.0),
                     n_replicas=n_replicas, n_temps=len(betas), betas=arr, init=init_id,
                     cone_half_angle=step, record_capacity=record_capacity,
                     algorithm=algorithm_id(algorithm), o3_proposal=O3_PROPOSALS[prop])
    return spec, arr


def plan_tiles(params, model=None, n_replicas=1, algorithm=None, refine=True, slots=148 * 4, slots3=148 * 3):
    """(CTAs, kernel kind) of one sweep launch of a handle's own path on a
    device with `slots` CTA slots (`slots3` for the 3D bit-sliced kernels),
    with or without tile refinement; host-side planning, no device needed."""
    spec, _keep = spec_from_params(params, model=model, n_replicas=n_replicas, algorithm=algorithm)
    n = ctypes.c_int64()
    kind = ctypes.c_int32()
    _lib.call("gpumc_plan_tiles", ctypes.byref(spec), int(slots), int(slots3), 1 if refine else 0,
              ctypes.byref(n), ctypes.byref(kind))
    return n.value, kind.value


class Engine:
    """A device context whose simulations can be swept together in one
    batched launch per sweep (gpumc_engine_sweep)."""

    def __init__(self, device=0):
        self.h = ctypes.c_void_p()
        _lib.call("gpumc_engine_create", device, ctypes.byref(self.h))

    def sweep(self, n=1):
        _lib.call("gpumc_engine_sweep", self.h, n)

    def synchronize(self):
        _lib.call("gpumc_engine_synchronize", self.h)

    def stream_ptr(self):
        v = ctypes.c_void_p()
        _lib.call("gpumc_engine_stream", self.h, ctypes.byref(v))
        return v.value

    def set_temporal_blocking(self, enable):
        _lib.call("gpumc_engine_set_temporal_blocking", self.h, 1 if enable else 0)

    def set_tile_refinement(self, enable):
        """Split the tiles of batches that leave CTA slots idle (default) or
        keep every lattice's full-launch tiles; results identical."""
        _lib.call("gpumc_engine_set_tile_refinement", self.h, 1 if enable else 0)

    def set_wait_limit(self, polls=None):
        """Polls after which an inter-CTA wait of the resident kernel gives up
        (None = the default, about half a second)."""
        _lib.call("gpumc_engine_set_wait_limit", self.h, (1 << 22) if polls is None else int(polls))

    def set_concurrent_kinds(self, enable):
        """Run each kernel kind's sweeps on a stream of its own (default) or
        all kinds in sequence on the engine stream; results identical."""
        _lib.call("gpumc_engine_set_concurrent_kinds", self.h, 1 if enable else 0)

    def launch_count(self):
        v = ctypes.c_uint64()
        _lib.call("gpumc_engine_launch_count", self.h, ctypes.byref(v))
        return v.value

    def close(self):
        if self.h:
            _lib.call("gpumc_engine_destroy", self.h)
            self.h = ctypes.c_void_p()


class ClassicalMC:
    """GPU ClassicalMC handle holding `n_replicas` lattices of one model."""

    NAME = "Metropolis-Hastings"

    def __init__(self, spec, seed, engine=None, _keep=None):
        self._keep = _keep
        self.spec = spec
        self.seed = seed
        self.engine = engine
        self.h = ctypes.c_void_p()
        eng = engine.h if engine is not None else None
        _lib.call("gpumc_create", eng, ctypes.byref(spec), ctypes.c_uint64(seed), ctypes.byref(self.h))
        self.model = spec.model
        self.dims = spec.dims
        self.shape = (spec.lx, spec.ly) if spec.dims == 2 else (spec.lx, spec.ly, spec.lz)
        self.n_sites = int(np.prod(self.shape))
        self.n_replicas = spec.n_replicas
        self.betas = [spec.betas[i] for i in range(spec.n_temps)]
        self.algorithm = spec.algorithm
        self.phase = _lib.PHASE_THERMALIZATION

    # -- FromParams -----------------------------------------------------------
    @staticmethod
    def validate_params(params, model=None, algorithm=None, o3_proposal=None):
        spec, _keep = spec_from_params(params, model=model, algorithm=algorithm, o3_proposal=o3_proposal)
        _lib.call("gpumc_validate", ctypes.byref(spec))

    @classmethod
    def from_params(cls, params, seed, model=None, n_replicas=1, betas=None, engine=None,
                    record_capacity=1024, algorithm=None, o3_proposal=None):
        """`algorithm`: "metropolis" (MetropolisCore, the default),
        "heat_bath" (HeatBathCore for Ising / Potts, ContinuousHeatBathCore
        for O(3)), "swendsen_wang" (SWCore) or "wolff" (WolffCore; one cluster
        per sweep), the cluster updates for Ising / Potts / O(3) with J >= 0.
        `o3_proposal` (O(3) Metropolis): "cap" (default: a cap around the
        current spin, half-angle adapted), "standard" (StandardStrategy:
        uniform unit vector), "opss" (OPSSStrategy: plane rotation, bound
        from params["opss_sigma"], default 0.5, adapted) or "cap_fast" (the
        cap on the same draws with the hardware approximations of sqrt,
        reciprocal, sin / cos and exp: spins within float32 tolerance of the
        cap's, not bit-identical)."""
        spec, keep = spec_from_params(params, model=model, n_replicas=n_replicas, betas=betas,
                                      record_capacity=record_capacity, algorithm=algorithm,
                                      o3_proposal=o3_proposal)
        return cls(spec, seed, engine=engine, _keep=keep)

    # -- MonteCarlo -----------------------------------------------------------
    def name(self):
        """Algorithm::name (CMC.rs/src/algorithms/heat_bath.rs:69-71, :131-133,
        swendsen_wang.rs:141-143, wolff.rs:138-140)."""
        if self.algorithm == _lib.HEAT_BATH:
            return "ContinuousHeatBath" if self.model == _lib.O3 else "HeatBath"
        if self.algorithm == _lib.SWENDSEN_WANG:
            return "Swendsen-Wang"
        if self.algorithm == _lib.WOLFF:
            return "Wolff"
        return self.NAME

    def on_phase_start(self, phase):
        self.phase = phase
        _lib.call("gpumc_set_phase", self.h, phase)

    def sweep(self, n=1):
        _lib.call("gpumc_sweep", self.h, n)

    def observables(self):
        """Drains the device records: list of dicts (one per replica per
        measured sweep, oldest first)."""
        out = []
        buf = (_lib.Obs * 4096)()
        n = ctypes.c_size_t()
        while True:
            _lib.call("gpumc_observables", self.h, buf, len(buf), ctypes.byref(n))
            for i in range(n.value):
                o = buf[i]
                out.append(dict(sweep=o.sweep, replica=o.replica, temp_index=o.temp_index,
                                beta=o.beta, energy=o.energy, magnetization=o.magnetization,
                                acceptance=o.acceptance))
            if n.value < len(buf):
                return out

    def observable_arrays(self):
        """Drained records as numpy arrays keyed by field."""
        recs = self.observables()
        keys = ("sweep", "replica", "temp_index", "beta", "energy", "magnetization", "acceptance")
        return {k: np.array([r[k] for r in recs]) for k in keys}

    def measure(self, ctx, namespace_by_chain=False):
        """Feeds every pending record into `ctx` with the reference's names
        (DefaultObservableSet::measure_all, CMC.rs/src/observables/common.rs:81-95);
        with device binning on, the completed device bins instead."""
        if getattr(self, "binsize", 0):
            return self._measure_bins(ctx)
        for r in self.observables():
            if namespace_by_chain or self.n_replicas > 1:
                ctx.set_measurement_namespace(f"pt_chain_{r['temp_index']:04d}")
            e = r["energy"]
            m = r["magnetization"]
            ctx.measure("Energy", e)
            ctx.measure("E2", e * e)
            ctx.measure("Magnetization", m)
            ctx.measure("M2", m * m)
            ctx.measure("M4", (m * m) * (m * m))  # powi(4): two squarings
            if namespace_by_chain or self.n_replicas > 1:
                ctx.measure("_pt_parameter", r["beta"])
                ctx.set_measurement_namespace(None)

    # -- device-side binning --------------------------------------------------
    BIN_NAMES = ("Energy", "E2", "Magnetization", "M2", "M4")

    def enable_device_binning(self, binsize, capacity=4096):
        """Bins Energy, E2, Magnetization, M2, M4 on the device (gpumc_set_binning):
        measure(ctx) then feeds completed bins to ctx's accumulators, which must
        use the same bin size; per-sweep records are not kept meanwhile.
        binsize 0 switches back to records."""
        _lib.call("gpumc_set_binning", self.h, int(binsize), int(capacity))
        self.binsize = int(binsize)

    def _bin_slot_name(self, slot):
        if self.n_replicas == 1:
            return None
        if len(self.betas) == self.n_replicas:
            return f"pt_chain_{slot:04d}"  # slot = temperature index
        return f"replica_{slot:04d}"

    def drain_bins(self):
        """Completed bins, shape (n_bins, n_replicas, 5)."""
        out = []
        cap = 1024
        buf = (ctypes.c_double * (cap * self.n_replicas * 5))()
        while True:
            n = ctypes.c_size_t()
            _lib.call("gpumc_drain_bins", self.h, buf, cap, ctypes.byref(n))
            if n.value == 0:
                break
            out.append(np.frombuffer(buf, dtype=np.float64, count=n.value * self.n_replicas * 5).copy())
            if n.value < cap:
                break
        if not out:
            return np.zeros((0, self.n_replicas, 5))
        return np.concatenate(out).reshape(-1, self.n_replicas, 5)

    def open_bin(self):
        """(sums of the open bin, shape (n_replicas, 5), its sample count)."""
        buf = (ctypes.c_double * (self.n_replicas * 5))()
        fill = ctypes.c_int32()
        _lib.call("gpumc_open_bin", self.h, buf, ctypes.byref(fill))
        return np.array(buf[:]).reshape(self.n_replicas, 5), fill.value

    def _measure_bins(self, ctx):
        if ctx.binsize != self.binsize:
            raise ValueError(f"device bins hold {self.binsize} samples, the context bins {ctx.binsize}")
        bins = self.drain_bins()
        if len(bins) == 0:
            return
        per_chain = len(self.betas) == self.n_replicas and self.n_replicas > 1
        for slot in range(self.n_replicas):
            ctx.set_measurement_namespace(self._bin_slot_name(slot))
            for k, name in enumerate(self.BIN_NAMES):
                ctx.accumulator(name).add_bins(bins[:, slot, k])
            if per_chain:
                # the chain's parameter is constant: the bin mean add() would
                # produce from binsize equal samples
                total = 0.0
                for _ in range(self.binsize):
                    total += self.betas[slot]
                ctx.accumulator("_pt_parameter").add_bins(np.full(len(bins), total / self.binsize))
        ctx.set_measurement_namespace(None)

    def finish_measurements(self, ctx):
        """Drains the last completed bins and hands the open bin to ctx as its
        trailing partial bin (call once, before ctx.finalize_measurements())."""
        if not getattr(self, "binsize", 0):
            return self.measure(ctx)
        self._measure_bins(ctx)
        sums, fill = self.open_bin()
        if fill == 0:
            return
        per_chain = len(self.betas) == self.n_replicas and self.n_replicas > 1
        for slot in range(self.n_replicas):
            ctx.set_measurement_namespace(self._bin_slot_name(slot))
            for k, name in enumerate(self.BIN_NAMES):
                ctx.accumulator(name).set_open_bin(sums[slot, k], fill)
            if per_chain:
                total = 0.0
                for _ in range(fill):
                    total += self.betas[slot]
                ctx.accumulator("_pt_parameter").set_open_bin(total, fill)
        ctx.set_measurement_namespace(None)

    # -- state ----------------------------------------------------------------
    def _site_dtype(self):
        return {_lib.ISING: np.int8, _lib.POTTS: np.int8, _lib.O3: np.float32,
                _lib.ISING_MSC64: np.uint64}[self.model]

    def spins(self, replica=0):
        """Spin state in the reference's site order (x fastest); O(3) has
        shape (..., 3)."""
        dt = self._site_dtype()
        n = self.n_sites * (3 if self.model == _lib.O3 else 1)
        a = np.empty(n, dtype=dt)
        _lib.call("gpumc_get_spins", self.h, replica, a.ctypes.data, a.nbytes)
        shape = tuple(reversed(self.shape))
        return a.reshape(shape + ((3,) if self.model == _lib.O3 else ()))

    def set_spins(self, replica, spins):
        a = np.ascontiguousarray(spins, dtype=self._site_dtype())
        _lib.call("gpumc_set_spins", self.h, replica, a.ctypes.data, a.nbytes)

    def energy(self):
        e = (ctypes.c_double * self.n_replicas)()
        _lib.call("gpumc_energy", self.h, e)
        return np.array(e[:])

    def recompute_energy(self):
        e = (ctypes.c_double * self.n_replicas)()
        _lib.call("gpumc_recompute_energy", self.h, e)
        return np.array(e[:])

    def stream_ptr(self):
        """cudaStream_t the handle's kernels are launched on."""
        e = ctypes.c_void_p()
        _lib.call("gpumc_sim_engine", self.h, ctypes.byref(e))
        v = ctypes.c_void_p()
        _lib.call("gpumc_engine_stream", e, ctypes.byref(v))
        return v.value

    def set_audit_interval(self, interval):
        """Compare cached and recomputed energies after every `interval`-th
        sweep (0 = off); a mismatch raises GpumcError (ESTATE)."""
        _lib.call("gpumc_set_audit_interval", self.h, int(interval))

    def perturb_energy_cache(self, replica, delta):
        """Adds `delta` to a replica's cached energy, spins untouched (a
        host-made cache fault for audit tests)."""
        _lib.call("gpumc_perturb_energy_cache", self.h, replica, float(delta))

    def set_wait_limit(self, polls=None):
        """Polls after which an inter-CTA wait of the resident kernel gives up
        (None = the default, about half a second), for the handle's engine."""
        e = ctypes.c_void_p()
        _lib.call("gpumc_sim_engine", self.h, ctypes.byref(e))
        _lib.call("gpumc_engine_set_wait_limit", e, (1 << 22) if polls is None else int(polls))

    def launches_per_sweep(self):
        v = ctypes.c_int32()
        _lib.call("gpumc_launches_per_sweep", self.h, ctypes.byref(v))
        return v.value

    def set_temporal_blocking(self, enable):
        """Run qualifying 2D Ising sweeps as resident multi-sweep launches
        (default) or as one streaming launch per sweep; results identical."""
        _lib.call("gpumc_set_temporal_blocking", self.h, 1 if enable else 0)

    def set_tile_refinement(self, enable):
        """Split this handle's tiles until one sweep launch fills the device
        (default) or keep the tiles sized for a full batch; results identical."""
        _lib.call("gpumc_set_tile_refinement", self.h, 1 if enable else 0)

    def tile_count(self):
        """CTAs of one sweep launch of this handle's own path."""
        v = ctypes.c_int32()
        _lib.call("gpumc_tile_count", self.h, ctypes.byref(v))
        return v.value

    def launch_count(self):
        """Kernel launches issued so far by this handle's sweeps."""
        v = ctypes.c_uint64()
        _lib.call("gpumc_launch_count", self.h, ctypes.byref(v))
        return v.value

    def sweep_count(self):
        v = ctypes.c_uint64()
        _lib.call("gpumc_sweep_count", self.h, ctypes.byref(v))
        return v.value

    def set_sweep_count(self, sweeps):
        """Moves every replica's sweep counter (the random-stream position)."""
        _lib.call("gpumc_set_sweep_count", self.h, int(sweeps))

    def cone_omc(self, replica=0):
        """O(3) cone parameter 1 - cos(alpha) as the device's float."""
        v = ctypes.c_float()
        _lib.call("gpumc_get_cone_omc", self.h, replica, ctypes.byref(v))
        return v.value

    def set_cone_omc(self, replica, omc):
        _lib.call("gpumc_set_cone_omc", self.h, replica, ctypes.c_float(omc))

    # -- snapshots (ClassicalMC::save_snapshot / load_snapshot) ---------------
    def save_snapshot(self, replica=0, renormalize=False):
        """cmc-rs-snapshot-v2 state of one replica (JSON-ready dict)."""
        from . import snapshot
        return snapshot.save_snapshot(self, replica, renormalize=renormalize)

    def load_snapshot(self, snap, replica=0):
        """Restores one replica; raises CheckpointCorrupted on any mismatch."""
        from . import snapshot
        snapshot.load_snapshot(self, snap, replica)

    def cone_half_angle(self, replica=0):
        v = ctypes.c_double()
        _lib.call("gpumc_acceptance", self.h, replica, ctypes.byref(v))
        return v.value

    # -- ParallelTemperingCompatible -------------------------------------------
    def log_weight_ratio(self, param, new_value, replica=0):
        if param != "beta":
            raise ValueError(f"unsupported classical PT parameter: {param}")
        v = ctypes.c_double()
        _lib.call("gpumc_log_weight_ratio", self.h, replica, float(new_value), ctypes.byref(v))
        return v.value

    def change_parameter(self, param, new_value, replica=0):
        if param != "beta":
            raise ValueError(f"unsupported classical PT parameter: {param}")
        _lib.call("gpumc_change_parameter", self.h, replica, float(new_value))
        labels = self.pt_labels()
        self.betas[labels[replica]] = float(new_value)

    def pt_configure(self, interval):
        _lib.call("gpumc_pt_configure", self.h, interval)

    def pt_labels(self):
        a = (ctypes.c_int32 * self.n_replicas)()
        _lib.call("gpumc_pt_labels", self.h, a)
        return np.array(a[:], dtype=np.int32)

    def set_pt_labels(self, labels):
        """Restores the ladder index held by each replica (a resumed
        ensemble's parameter-chain indices, set_chain_idx,
        Carlo.rs/src/parallel_tempering.rs:159-163)."""
        a = (ctypes.c_int32 * self.n_replicas)(*[int(v) for v in labels])
        _lib.call("gpumc_pt_set_labels", self.h, a)

    def pt_stats(self):
        s = ctypes.c_uint64()
        a = ctypes.c_uint64()
        _lib.call("gpumc_pt_stats", self.h, ctypes.byref(s), ctypes.byref(a))
        return s.value, a.value

    def close(self):
        if self.h:
            _lib.call("gpumc_destroy", self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class MultiSpinIsing(ClassicalMC):
    """64 Ising replicas per lattice packed in uint64 words."""

    NAME = "MultiSpinIsing"

    @classmethod
    def from_params(cls, params, seed, n_replicas=1, betas=None, engine=None, record_capacity=256):
        return super().from_params(params, seed, model=_lib.ISING_MSC64, n_replicas=n_replicas,
                                   betas=betas, engine=engine, record_capacity=record_capacity)

    def replica_observables(self, word_lattice=0):
        e = (ctypes.c_double * 64)()
        m = (ctypes.c_double * 64)()
        _lib.call("gpumc_msc_replica_observables", self.h, word_lattice, e, m)
        return np.array(e[:]), np.array(m[:])

    def measure(self, ctx, namespace_by_chain=False):
        """Array observables Energy_replica ... plus replica-0 scalars
        (MultiSpinIsing::measure, CMC.rs/src/multi_spin.rs:220-286)."""
        recs = self.observables()
        for i in range(0, len(recs), 64 * self.n_replicas):
            row = recs[i:i + 64]
            e = np.array([r["energy"] for r in row])
            m = np.array([r["magnetization"] for r in row])
            m4 = m * m * m * m  # left to right, as multi_spin.rs:268
            ctx.measure_array("Energy_replica", e)
            ctx.measure_array("Magnetization_replica", m)
            ctx.measure_array("E2_replica", e * e)
            ctx.measure_array("M2_replica", m * m)
            ctx.measure_array("M4_replica", m4)
            ctx.measure("Energy", e[0])
            ctx.measure("Magnetization", m[0])
            ctx.measure("E2", e[0] * e[0])
            ctx.measure("M2", m[0] * m[0])
            ctx.measure("M4", m4[0])


def run_one(mc, thermalization_sweeps, measurement_sweeps, binsize=1):
    """Scheduler::run_one (Carlo.rs/src/scheduler.rs:94-155): thermalize, then
    measure after every sweep; returns {name: Estimate}."""
    ctx = Context(binsize)
    mc.on_phase_start(_lib.PHASE_THERMALIZATION)
    if thermalization_sweeps:
        mc.sweep(thermalization_sweeps)
    mc.on_phase_start(_lib.PHASE_MEASUREMENT)
    left = measurement_sweeps
    while left > 0:
        k = min(left, 4096)
        mc.sweep(k)
        mc.measure(ctx)
        left -= k
    if getattr(mc, "binsize", 0):
        mc.finish_measurements(ctx)
    return ctx.finalize_measurements()


def geometric_ladder_betas(t_min, t_max, n):
    """Temperatures geometric between t_min and t_max, returned as betas in
    ascending-temperature order."""
    return [1.0 / (t_min * (t_max / t_min) ** (k / (n - 1))) for k in range(n)]


def potts_beta_c(q):
    """beta_c(q) = ln(1 + sqrt(q)) of the square-lattice Potts model."""
    return math.log(1.0 + math.sqrt(q))


class Server:
    """Continuous-batching simulation server (gpumc_server_*)."""

    def __init__(self, hbm_budget, chunk=10, device=0):
        self.h = ctypes.c_void_p()
        _lib.call("gpumc_server_create", device, ctypes.c_size_t(int(hbm_budget)), chunk,
                  ctypes.byref(self.h))

    def submit(self, params, seed, n_sweeps, n_therm=0, model=None, n_replicas=1, betas=None,
               algorithm=None, o3_proposal=None):
        """Queues a job (ClassicalMC.from_params's model / algorithm /
        o3_proposal arguments); returns its id, or None when the queue is
        full (GPUMC_EAGAIN)."""
        spec, keep = spec_from_params(params, model=model, n_replicas=n_replicas, betas=betas,
                                      algorithm=algorithm, o3_proposal=o3_proposal)
        job = _lib.Job(spec=spec, base_seed=seed, n_sweeps=n_sweeps, n_therm=n_therm)
        jid = ctypes.c_uint64()
        rc = _lib.load().gpumc_submit(self.h, ctypes.byref(job), ctypes.byref(jid))
        if rc == _lib.EAGAIN:
            return None
        _lib.check(rc)
        del keep  # gpumc_submit copied the spec and its betas
        return jid.value

    def step(self):
        a = ctypes.c_int32()
        _lib.call("gpumc_server_step", self.h, ctypes.byref(a))
        return a.value

    def poll(self):
        buf = (_lib.JobResult * 1024)()
        n = ctypes.c_size_t()
        out = []
        while True:
            _lib.call("gpumc_poll", self.h, buf, len(buf), ctypes.byref(n))
            for i in range(n.value):
                r = buf[i]
                out.append(dict(job_id=r.job_id, status=r.status, n_replicas=r.n_replicas,
                                submit_s=r.submit_s, start_s=r.start_s, finish_s=r.finish_s,
                                mean_energy=r.mean_energy, mean_abs_m=r.mean_abs_m,
                                attempts=r.attempts))
            if n.value < len(buf):
                return out

    def cancel(self, job_id):
        _lib.call("gpumc_cancel", self.h, ctypes.c_uint64(job_id))

    def job_spins(self, job_id, n_bytes, replica=0, dtype=np.int8):
        a = np.empty(n_bytes // np.dtype(dtype).itemsize, dtype=dtype)
        _lib.call("gpumc_job_spins", self.h, ctypes.c_uint64(job_id), replica, a.ctypes.data, a.nbytes)
        return a

    def stats(self):
        att = ctypes.c_double()
        busy = ctypes.c_double()
        used = ctypes.c_size_t()
        _lib.call("gpumc_server_stats", self.h, ctypes.byref(att), ctypes.byref(busy), ctypes.byref(used))
        adm, swp, ret = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        _lib.call("gpumc_server_timing", self.h, ctypes.byref(adm), ctypes.byref(swp), ctypes.byref(ret))
        return dict(attempts=att.value, busy_s=busy.value, bytes_in_use=used.value, admit_s=adm.value,
                    sweep_s=swp.value, retire_s=ret.value)

    def set_keep_spins(self, max_sites):
        """Keep final spins (gpumc_job_spins) of jobs up to `max_sites` sites."""
        _lib.call("gpumc_server_set_keep_spins", self.h, int(max_sites))

    def close(self):
        if self.h:
            _lib.call("gpumc_server_destroy", self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

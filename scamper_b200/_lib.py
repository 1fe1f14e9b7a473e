"""ctypes bindings of the engine's C ABI (include/gpumc.h).

The shared library is loaded from the package directory; there is no CPU
fallback, so a missing library or a missing CUDA device raises immediately.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# GPUMC_LIBRARY=bounds loads the bounds-checked build (libgpumc_bounds.so,
# python scamper_b200/build.py --bounds) instead of the release library.
# GPUMC_LIBRARY=<absolute path> loads that build of the library instead.
_choice = os.environ.get("GPUMC_LIBRARY", "")
LIB_PATH = (_choice if os.path.isabs(_choice) else
            os.path.join(HERE, "libgpumc_bounds.so" if _choice == "bounds" else "libgpumc.so"))

OK = 0
EINVAL = -1
ENODEV = -2
ECUDA = -3
ENOMEM = -4
EAGAIN = -5
ESTATE = -6
ENOTFOUND = -7

ISING = 0
POTTS = 1
O3 = 2
ISING_MSC64 = 3

INIT_HOT = 0
INIT_COLD = 1

METROPOLIS = 0
HEAT_BATH = 1
SWENDSEN_WANG = 2
WOLFF = 3
O3_CAP = 0
O3_UNIFORM = 1
O3_OPSS = 2
O3_CAP_FAST = 3
PHASE_THERMALIZATION = 1
PHASE_MEASUREMENT = 2


class Spec(ctypes.Structure):
    _fields_ = [
        ("model", ctypes.c_int32),
        ("dims", ctypes.c_int32),
        ("lx", ctypes.c_int64),
        ("ly", ctypes.c_int64),
        ("lz", ctypes.c_int64),
        ("pbc", ctypes.c_int32),
        ("q", ctypes.c_int32),
        ("J", ctypes.c_double),
        ("n_replicas", ctypes.c_int32),
        ("n_temps", ctypes.c_int32),
        ("betas", ctypes.POINTER(ctypes.c_double)),
        ("init", ctypes.c_int32),
        ("cone_half_angle", ctypes.c_double),
        ("record_capacity", ctypes.c_int32),
        ("algorithm", ctypes.c_int32),
        ("o3_proposal", ctypes.c_int32),
    ]


class Obs(ctypes.Structure):
    _fields_ = [
        ("sweep", ctypes.c_uint64),
        ("replica", ctypes.c_int32),
        ("temp_index", ctypes.c_int32),
        ("beta", ctypes.c_double),
        ("energy", ctypes.c_double),
        ("magnetization", ctypes.c_double),
        ("acceptance", ctypes.c_double),
    ]


class Job(ctypes.Structure):
    _fields_ = [
        ("spec", Spec),
        ("base_seed", ctypes.c_uint64),
        ("n_sweeps", ctypes.c_uint64),
        ("n_therm", ctypes.c_uint64),
    ]


class JobResult(ctypes.Structure):
    _fields_ = [
        ("job_id", ctypes.c_uint64),
        ("status", ctypes.c_int32),
        ("n_replicas", ctypes.c_int32),
        ("submit_s", ctypes.c_double),
        ("start_s", ctypes.c_double),
        ("finish_s", ctypes.c_double),
        ("mean_energy", ctypes.c_double),
        ("mean_abs_m", ctypes.c_double),
        ("attempts", ctypes.c_double),
    ]


# (name, argtypes) of every exported entry point declared in include/gpumc.h
class TileKnobs(ctypes.Structure):
    """gpumc_tile_knobs: 0 = the planner's analytic choice."""
    _fields_ = [(name, ctypes.c_int32) for name in
                ("ising2d_rows", "ising3d_planes", "potts_segments", "potts3d_planes", "o3_rows", "o3_planes")]


_vp = ctypes.c_void_p
_P = ctypes.POINTER
SIGNATURES = {
    "gpumc_engine_create": [ctypes.c_int32, _P(_vp)],
    "gpumc_engine_destroy": [_vp],
    "gpumc_engine_sweep": [_vp, ctypes.c_uint32],
    "gpumc_engine_synchronize": [_vp],
    "gpumc_engine_stream": [_vp, _P(_vp)],
    "gpumc_sim_engine": [_vp, _P(_vp)],
    "gpumc_launches_per_sweep": [_vp, _P(ctypes.c_int32)],
    "gpumc_set_temporal_blocking": [_vp, ctypes.c_int32],
    "gpumc_set_sweep_count": [_vp, ctypes.c_uint64],
    "gpumc_get_cone_omc": [_vp, ctypes.c_int32, _P(ctypes.c_float)],
    "gpumc_set_cone_omc": [_vp, ctypes.c_int32, ctypes.c_float],
    "gpumc_engine_set_temporal_blocking": [_vp, ctypes.c_int32],
    "gpumc_set_tile_refinement": [_vp, ctypes.c_int32],
    "gpumc_engine_set_tile_refinement": [_vp, ctypes.c_int32],
    "gpumc_engine_set_concurrent_kinds": [_vp, ctypes.c_int32],
    "gpumc_tile_count": [_vp, _P(ctypes.c_int32)],
    "gpumc_launch_count": [_vp, _P(ctypes.c_uint64)],
    "gpumc_engine_launch_count": [_vp, _P(ctypes.c_uint64)],
    "gpumc_create": [_vp, _P(Spec), ctypes.c_uint64, _P(_vp)],
    "gpumc_validate": [_P(Spec)],
    "gpumc_destroy": [_vp],
    "gpumc_set_phase": [_vp, ctypes.c_int32],
    "gpumc_sweep": [_vp, ctypes.c_uint32],
    "gpumc_observables": [_vp, _P(Obs), ctypes.c_size_t, _P(ctypes.c_size_t)],
    "gpumc_set_binning": [_vp, ctypes.c_int32, ctypes.c_int32],
    "gpumc_drain_bins": [_vp, _P(ctypes.c_double), ctypes.c_size_t, _P(ctypes.c_size_t)],
    "gpumc_open_bin": [_vp, _P(ctypes.c_double), _P(ctypes.c_int32)],
    "gpumc_get_spins": [_vp, ctypes.c_int32, _vp, ctypes.c_size_t],
    "gpumc_set_spins": [_vp, ctypes.c_int32, _vp, ctypes.c_size_t],
    "gpumc_energy": [_vp, _P(ctypes.c_double)],
    "gpumc_recompute_energy": [_vp, _P(ctypes.c_double)],
    "gpumc_msc_replica_observables": [_vp, ctypes.c_int32, _P(ctypes.c_double), _P(ctypes.c_double)],
    "gpumc_sweep_count": [_vp, _P(ctypes.c_uint64)],
    "gpumc_acceptance": [_vp, ctypes.c_int32, _P(ctypes.c_double)],
    "gpumc_log_weight_ratio": [_vp, ctypes.c_int32, ctypes.c_double, _P(ctypes.c_double)],
    "gpumc_change_parameter": [_vp, ctypes.c_int32, ctypes.c_double],
    "gpumc_pt_configure": [_vp, ctypes.c_uint32],
    "gpumc_engine_set_wait_limit": [_vp, ctypes.c_int64],
    "gpumc_set_audit_interval": [_vp, ctypes.c_uint64],
    "gpumc_set_tile_knobs": [_P(TileKnobs)],
    "gpumc_get_tile_knobs": [_P(TileKnobs)],
    "gpumc_debug_bounds": [_P(ctypes.c_uint64), _P(ctypes.c_int32), _P(ctypes.c_int32), _P(ctypes.c_int32)],
    "gpumc_perturb_energy_cache": [_vp, ctypes.c_int32, ctypes.c_double],
    "gpumc_pt_labels": [_vp, _P(ctypes.c_int32)],
    "gpumc_pt_set_labels": [_vp, _P(ctypes.c_int32)],
    "gpumc_pt_stats": [_vp, _P(ctypes.c_uint64), _P(ctypes.c_uint64)],
    "gpumc_server_create": [ctypes.c_int32, ctypes.c_size_t, ctypes.c_uint32, _P(_vp)],
    "gpumc_submit": [_vp, _P(Job), _P(ctypes.c_uint64)],
    "gpumc_server_step": [_vp, _P(ctypes.c_int32)],
    "gpumc_poll": [_vp, _P(JobResult), ctypes.c_size_t, _P(ctypes.c_size_t)],
    "gpumc_cancel": [_vp, ctypes.c_uint64],
    "gpumc_job_spins": [_vp, ctypes.c_uint64, ctypes.c_int32, _vp, ctypes.c_size_t],
    "gpumc_server_stats": [_vp, _P(ctypes.c_double), _P(ctypes.c_double), _P(ctypes.c_size_t)],
    "gpumc_server_timing": [_vp, _P(ctypes.c_double), _P(ctypes.c_double), _P(ctypes.c_double)],
    "gpumc_server_set_keep_spins": [_vp, ctypes.c_size_t],
    "gpumc_server_destroy": [_vp],
    "gpumc_last_error": [ctypes.c_char_p, ctypes.c_size_t],
    "gpumc_philox_probe": [_P(ctypes.c_uint32), _P(ctypes.c_uint32), _P(ctypes.c_uint32), ctypes.c_int32],
    "gpumc_footprint": [_P(Spec), _P(ctypes.c_size_t)],
    "gpumc_plan_tiles": [_P(Spec), ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _P(ctypes.c_int64),
                         _P(ctypes.c_int32)],
    "gpumc_energy_int8_noalloc": [ctypes.c_int32, ctypes.c_int32, ctypes.c_int64, ctypes.c_int64,
                                  ctypes.c_int64, _vp, ctypes.c_int32, _vp, _vp],
}


class GpumcError(RuntimeError):
    """Error returned through the C ABI (status code + message)."""

    def __init__(self, code, message):
        super().__init__(f"[{code}] {message}")
        self.code = code
        self.message = message


class InvalidConfig(GpumcError, ValueError):
    """The reference's CarloError::InvalidConfig."""


_lib = None


def load():
    """Loads libgpumc.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python scamper_b200/build.py` (--bounds for the checked build) "
            "(there is no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int
    _lib = lib
    return lib


def debug_bounds():
    """(violations since the last call, first module, first line, compiled)
    of a bounds-checked library; compiled is False for a release library."""
    h, m, ln, c = ctypes.c_uint64(), ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
    check(load().gpumc_debug_bounds(ctypes.byref(h), ctypes.byref(m), ctypes.byref(ln), ctypes.byref(c)))
    return h.value, m.value, ln.value, bool(c.value)


def last_error():
    buf = ctypes.create_string_buffer(4096)
    load().gpumc_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc):
    if rc == OK:
        return rc
    msg = last_error()
    if rc == EINVAL:
        raise InvalidConfig(rc, msg)
    raise GpumcError(rc, msg)


def call(name, *args):
    return check(getattr(load(), name)(*args))

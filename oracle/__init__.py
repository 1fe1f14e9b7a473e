"""ctypes wrapper of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() to
check the device result, and by bench.py's CPU-baseline leg.  Nothing on the
product path imports it.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

ISING, POTTS, O3, MSC = 0, 1, 2, 3
METROPOLIS, HEAT_BATH, SWENDSEN_WANG, WOLFF = 0, 1, 2, 3
TAG_ACC, TAG_PROP, TAG_ACC_REFINE, TAG_PROP_REFINE, TAG_INIT, TAG_O3, TAG_MSC, TAG_PT = range(8)
SUB_INIT, SUB_SWEEP = 0, 1

_lib = None
_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_i64p = ctypes.POINTER(ctypes.c_int64)
_i32p = ctypes.POINTER(ctypes.c_int32)
_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)
_i8p = ctypes.POINTER(ctypes.c_int8)
_i64 = ctypes.c_int64
_u64 = ctypes.c_uint64
_int = ctypes.c_int


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        sig = {
            "orc_philox4x32_10": (None, [_u32p, _u32p, _u32p]),
            "orc_set_threads": (None, [_int]),
            "orc_stream_seed": (_u64, [_u64] * 8),
            "orc_replica_key": (_u64, [_u64, _u64, _u64]),
            "orc_exchange_key": (_u64, [_u64]),
            "orc_threshold": (None, [ctypes.c_double, _u32p, _u64p]),
            "orc_build_table": (_int, [_int, _int, ctypes.c_double, ctypes.c_double, _u32p, _u64p]),
            "orc_build_table_hb": (_int, [_int, _int, ctypes.c_double, ctypes.c_double, _u32p, _u64p]),
            "orc_sweep_discrete_hb": (_i64, [_int, _int, _i64, _i64, _i64, _int, ctypes.c_double, _u32p,
                                             _u64p, _u64, _u64, _i8p, _i64p]),
            "orc_sweep_o3_hb": (ctypes.c_double, [_int, _i64, _i64, _i64, ctypes.c_float, ctypes.c_float,
                                                  _u64, _u64, _f32p, _f32p, _f32p, _i64p]),
            "orc_one_minus_exp_neg": (ctypes.c_float, [ctypes.c_float]),
            "orc_cluster_threshold": (_u64, [_int, ctypes.c_double, ctypes.c_double]),
            "orc_sweep_cluster_o3": (ctypes.c_double, [_int, _i64, _i64, _i64, ctypes.c_float, ctypes.c_float, _int,
                                                       _u64, _u64, _f32p, _f32p, _f32p, _i64p]),
            "orc_sweep_cluster": (_i64, [_int, _int, _i64, _i64, _i64, _int, _int, _u64, _u64, _u64, _i8p,
                                         _i64p]),
            "orc_log_one_minus": (ctypes.c_float, [ctypes.c_float]),
            "orc_init_discrete": (None, [_int, _int, _i64, _i64, _i64, _int, _u64, _u64, _int, _i8p]),
            "orc_sweep_discrete": (_i64, [_int, _int, _i64, _i64, _i64, _int, _u32p, _u64p, _u64, _u64,
                                          _i8p, _i64p]),
            "orc_energy_int": (_i64, [_int, _int, _i64, _i64, _i64, _i8p]),
            "orc_init_o3": (None, [_int, _i64, _i64, _i64, _u64, _u64, _int, _f32p, _f32p, _f32p]),
            "orc_sweep_o3": (ctypes.c_double, [_int, _i64, _i64, _i64, ctypes.c_float, ctypes.c_float,
                                               ctypes.c_float, _u64, _u64, _f32p, _f32p, _f32p, _i64p]),
            "orc_energy_o3": (ctypes.c_double, [_int, _i64, _i64, _i64, ctypes.c_double, _f32p, _f32p,
                                                _f32p]),
            "orc_o3_adapt": (ctypes.c_float, [ctypes.c_float, _i64, _i64]),
            "orc_opss_adapt": (ctypes.c_float, [ctypes.c_float, _i64, _i64]),
            "orc_sweep_o3_prop": (ctypes.c_double, [_int, _i64, _i64, _i64, ctypes.c_float, ctypes.c_float,
                                                    ctypes.c_float, _int, _u64, _u64, _f32p, _f32p, _f32p, _i64p]),
            "orc_exp_neg": (ctypes.c_float, [ctypes.c_float]),
            "orc_exp_neg2": (ctypes.c_float, [ctypes.c_float]),
            "orc_unit23": (ctypes.c_float, [ctypes.c_uint32]),
            "orc_half23": (ctypes.c_float, [ctypes.c_uint32]),
            "orc_sincos23": (None, [ctypes.c_uint32, _f32p, _f32p]),
            "orc_o3_fixed_observables": (None, [_int, _i64, _i64, _i64, ctypes.c_double, _f32p, _f32p, _f32p,
                                                _f64p, _f64p]),
            "orc_sincos_turn": (None, [ctypes.c_uint32, _f32p, _f32p]),
            "orc_init_msc": (None, [_int, _i64, _i64, _i64, _u64, _int, _u64p]),
            "orc_sweep_msc": (None, [_int, _i64, _i64, _i64, _u32p, _u64p, _u64, _u64, _u64p, _i64p]),
            "orc_msc_observables": (None, [_int, _i64, _i64, _i64, _u64p, _i64p, _i64p]),
            "orc_pt_exchange": (_int, [_int, _f64p, _f64p, _i32p, _u64, _u64, _i32p]),
            "orc_accept_log": (_int, [ctypes.c_double, _u64]),
            "orc_ref_create": (ctypes.c_void_p, [_int, _int, _i64, _i64, _i64, _int, ctypes.c_double,
                                                 ctypes.c_double, _u64, _u64, _int]),
            "orc_ref_destroy": (None, [ctypes.c_void_p]),
            "orc_ref_sweep": (None, [ctypes.c_void_p, _int]),
            "orc_ref_measure": (None, [ctypes.c_void_p, _f64p, _f64p]),
            "orc_ref_recompute_energy": (ctypes.c_double, [ctypes.c_void_p]),
            "orc_ref_series": (None, [ctypes.c_void_p, _int, _int, _f64p, _f64p]),
            "orc_ref_set_beta": (None, [ctypes.c_void_p, ctypes.c_double]),
            "orc_ref_n_sites": (_i64, [ctypes.c_void_p]),
            "orc_ref_run_parallel": (ctypes.c_double, [_int, _int, _i64, _i64, _i64, _int,
                                                       ctypes.c_double, ctypes.c_double, _u64, _int,
                                                       _int, _int, _int, _f64p, _f64p, _f64p]),
            "orc_ref_msc_run": (ctypes.c_double, [_int, _i64, _i64, _i64, ctypes.c_double,
                                                  ctypes.c_double, _u64, _int, _int, _f64p]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def set_threads(n):
    """Threads of the discrete and multi-spin replays (same results for any
    count)."""
    lib().orc_set_threads(int(n))


def _p(a, t):
    return a.ctypes.data_as(t)


def philox(ctr, key):
    c = np.asarray(ctr, dtype=np.uint32)
    k = np.asarray(key, dtype=np.uint32)
    o = np.zeros(4, dtype=np.uint32)
    lib().orc_philox4x32_10(_p(c, _u32p), _p(k, _u32p), _p(o, _u32p))
    return o


def stream_seed(base, task=0, run=0, chain=0, replica=0, thread=0, phase=0, substream=0):
    return lib().orc_stream_seed(base, task, run, chain, replica, thread, phase, substream)


def replica_key(base, replica, substream):
    return lib().orc_replica_key(base, replica, substream)


def exchange_key(base):
    return lib().orc_exchange_key(base)


def threshold(p):
    h = ctypes.c_uint32()
    t = ctypes.c_uint64()
    lib().orc_threshold(p, ctypes.byref(h), ctypes.byref(t))
    return h.value, t.value


def table(model, dims, J, beta, algorithm=METROPOLIS):
    head = np.zeros(13, dtype=np.uint32)
    tail = np.zeros(13, dtype=np.uint64)
    fn = lib().orc_build_table_hb if algorithm == HEAT_BATH else lib().orc_build_table
    n = fn(model, dims, J, beta, _p(head, _u32p), _p(tail, _u64p))
    return head[:n].copy(), tail[:n].copy()


class Lattice:
    """Oracle replica of one lattice under the engine's checkerboard method."""

    def __init__(self, model, shape, q=3, J=1.0, beta=0.44, seed=1, replica=0, hot=True,
                 omc=None, algorithm=METROPOLIS, prop=0):
        self.model = model
        self.algorithm = algorithm
        self.prop = prop  # O(3) Metropolis proposal: 0 cap, 1 uniform, 2 OPSS (omc = sigma)
        self.dims = len(shape)
        self.lx, self.ly = shape[0], shape[1]
        self.lz = shape[2] if self.dims == 3 else 1
        self.n = self.lx * self.ly * self.lz
        self.q = q
        self.J = J
        self.beta = beta
        self.seed = seed
        self.replica = replica
        self.sweeps = 0
        L = lib()
        if model in (ISING, POTTS):
            self.spins = np.zeros(self.n, dtype=np.int8)
            L.orc_init_discrete(model, self.dims, self.lx, self.ly, self.lz, q, seed, replica,
                                1 if hot else 0, _p(self.spins, _i8p))
            self.key = replica_key(seed, replica, SUB_SWEEP)
            self.e_int = L.orc_energy_int(model, self.dims, self.lx, self.ly, self.lz,
                                          _p(self.spins, _i8p))
        elif model == O3:
            self.sx = np.zeros(self.n, dtype=np.float32)
            self.sy = np.zeros(self.n, dtype=np.float32)
            self.sz = np.zeros(self.n, dtype=np.float32)
            L.orc_init_o3(self.dims, self.lx, self.ly, self.lz, seed, replica, 1 if hot else 0,
                          _p(self.sx, _f32p), _p(self.sy, _f32p), _p(self.sz, _f32p))
            self.key = replica_key(seed, replica, SUB_SWEEP)
            self.omc = np.float32(omc if omc is not None else 1.0 - np.cos(1.0))
            self.e = L.orc_energy_o3(self.dims, self.lx, self.ly, self.lz, J, _p(self.sx, _f32p),
                                     _p(self.sy, _f32p), _p(self.sz, _f32p))
        else:
            self.words = np.zeros(self.n, dtype=np.uint64)
            L.orc_init_msc(self.dims, self.lx, self.ly, self.lz, seed, 1 if hot else 0,
                           _p(self.words, _u64p))
            self.key = replica_key(seed, 64 * replica, SUB_SWEEP)
        self.set_beta(beta)

    def set_beta(self, beta):
        self.beta = beta
        if self.algorithm in (SWENDSEN_WANG, WOLFF) and self.model != O3:
            self.thr = lib().orc_cluster_threshold(self.model, self.J, beta)
        elif self.model != O3:
            tm = ISING if self.model == MSC else self.model
            self.head, self.tail = table(tm, self.dims, self.J, beta, self.algorithm)

    def sweep(self, adapt=False):
        L = lib()
        acc = ctypes.c_int64()
        if self.algorithm in (SWENDSEN_WANG, WOLFF) and self.model == O3:
            d = L.orc_sweep_cluster_o3(self.dims, self.lx, self.ly, self.lz, np.float32(self.J),
                                       np.float32(self.beta), 1 if self.algorithm == WOLFF else 0, self.key,
                                       self.sweeps, _p(self.sx, _f32p), _p(self.sy, _f32p), _p(self.sz, _f32p),
                                       ctypes.byref(acc))
            self.e += d
        elif self.algorithm in (SWENDSEN_WANG, WOLFF):
            d = L.orc_sweep_cluster(self.model, self.dims, self.lx, self.ly, self.lz, self.q,
                                    1 if self.algorithm == WOLFF else 0, self.thr, self.key, self.sweeps,
                                    _p(self.spins, _i8p), ctypes.byref(acc))
            self.e_int += d
        elif self.model in (ISING, POTTS) and self.algorithm == HEAT_BATH:
            d = L.orc_sweep_discrete_hb(self.model, self.dims, self.lx, self.ly, self.lz, self.q, self.J,
                                        _p(self.head, _u32p), _p(self.tail, _u64p), self.key,
                                        self.sweeps, _p(self.spins, _i8p), ctypes.byref(acc))
            self.e_int += d
        elif self.model == O3 and self.algorithm == HEAT_BATH:
            d = L.orc_sweep_o3_hb(self.dims, self.lx, self.ly, self.lz, np.float32(self.J),
                                  np.float32(self.beta), self.key, self.sweeps, _p(self.sx, _f32p),
                                  _p(self.sy, _f32p), _p(self.sz, _f32p), ctypes.byref(acc))
            self.e += d
        elif self.model in (ISING, POTTS):
            d = L.orc_sweep_discrete(self.model, self.dims, self.lx, self.ly, self.lz, self.q,
                                     _p(self.head, _u32p), _p(self.tail, _u64p), self.key,
                                     self.sweeps, _p(self.spins, _i8p), ctypes.byref(acc))
            self.e_int += d
        elif self.model == O3:
            d = L.orc_sweep_o3_prop(self.dims, self.lx, self.ly, self.lz, np.float32(self.J),
                                    np.float32(self.beta), self.omc, self.prop, self.key, self.sweeps,
                                    _p(self.sx, _f32p), _p(self.sy, _f32p), _p(self.sz, _f32p),
                                    ctypes.byref(acc))
            self.e += d
            if adapt and self.prop == 2:
                self.omc = np.float32(L.orc_opss_adapt(self.omc, acc.value, self.n))
            elif adapt and self.prop == 0:
                self.omc = np.float32(L.orc_o3_adapt(self.omc, acc.value, self.n))
        else:
            L.orc_sweep_msc(self.dims, self.lx, self.ly, self.lz, _p(self.head, _u32p),
                            _p(self.tail, _u64p), self.key, self.sweeps, _p(self.words, _u64p),
                            ctypes.byref(acc))
        self.sweeps += 1
        return acc.value

    def energy(self):
        """Physical energy of the current state (exact recomputation)."""
        L = lib()
        if self.model in (ISING, POTTS):
            return self.J * L.orc_energy_int(self.model, self.dims, self.lx, self.ly, self.lz,
                                             _p(self.spins, _i8p))
        if self.model == O3:
            return L.orc_energy_o3(self.dims, self.lx, self.ly, self.lz, self.J, _p(self.sx, _f32p),
                                   _p(self.sy, _f32p), _p(self.sz, _f32p))
        e, m = self.msc_observables()
        return float(e.sum())

    def fixed_observables(self):
        """O(3): (energy, magnetisation vector) as the sweep kernels record
        them (fixed-point sums of the fp32 configuration)."""
        e = ctypes.c_double()
        m = np.zeros(3, dtype=np.float64)
        lib().orc_o3_fixed_observables(self.dims, self.lx, self.ly, self.lz, self.J, _p(self.sx, _f32p),
                                       _p(self.sy, _f32p), _p(self.sz, _f32p), ctypes.byref(e), _p(m, _f64p))
        return e.value, m

    def cached_energy(self):
        if self.model in (ISING, POTTS):
            return self.J * self.e_int
        return self.e

    def msc_observables(self):
        e = np.zeros(64, dtype=np.int64)
        m = np.zeros(64, dtype=np.int64)
        lib().orc_msc_observables(self.dims, self.lx, self.ly, self.lz, _p(self.words, _u64p),
                                  _p(e, _i64p), _p(m, _i64p))
        return self.J * e.astype(np.float64), m

    def state(self):
        if self.model in (ISING, POTTS):
            return self.spins.copy()
        if self.model == O3:
            return np.stack([self.sx, self.sy, self.sz], axis=1).copy()
        return self.words.copy()

    def set_state(self, arr):
        if self.model in (ISING, POTTS):
            self.spins[:] = np.asarray(arr, dtype=np.int8).ravel()
            self.e_int = lib().orc_energy_int(self.model, self.dims, self.lx, self.ly, self.lz,
                                              _p(self.spins, _i8p))
        elif self.model == O3:
            a = np.asarray(arr, dtype=np.float32).reshape(-1, 3)
            self.sx[:], self.sy[:], self.sz[:] = a[:, 0], a[:, 1], a[:, 2]
            self.e = self.energy()
        else:
            self.words[:] = np.asarray(arr, dtype=np.uint64).ravel()


def pt_exchange(betas, energies, labels, key, step):
    b = np.ascontiguousarray(betas, dtype=np.float64)
    e = np.ascontiguousarray(energies, dtype=np.float64)
    lab = np.ascontiguousarray(labels, dtype=np.int32).copy()
    acc = np.zeros(len(b), dtype=np.int32)
    n = lib().orc_pt_exchange(len(b), _p(b, _f64p), _p(e, _f64p), _p(lab, _i32p), key, step,
                              _p(acc, _i32p))
    return lab, n, acc


class RefSampler:
    """Restated reference sampler (cmc-rs MetropolisCore on a CSR lattice)."""

    def __init__(self, model, shape, q=3, J=1.0, beta=0.44, seed=1, chain=0, hot=True):
        dims = len(shape)
        lz = shape[2] if dims == 3 else 1
        self.h = lib().orc_ref_create(model, dims, shape[0], shape[1], lz, q, J, beta, seed, chain,
                                      1 if hot else 0)
        self.n = lib().orc_ref_n_sites(self.h)

    def sweep(self, n=1):
        for _ in range(n):
            lib().orc_ref_sweep(self.h, 0)

    def measure(self):
        e = ctypes.c_double()
        m = ctypes.c_double()
        lib().orc_ref_measure(self.h, ctypes.byref(e), ctypes.byref(m))
        return e.value, m.value

    def recompute_energy(self):
        return lib().orc_ref_recompute_energy(self.h)

    def series(self, therm, meas):
        """therm sweeps, then meas measured sweeps: (E/N, |M|) per sweep.  The
        C call releases the GIL, so chains can run on Python threads."""
        e = np.zeros(meas, dtype=np.float64)
        m = np.zeros(meas, dtype=np.float64)
        lib().orc_ref_series(self.h, therm, meas, _p(e, _f64p), _p(m, _f64p))
        return e, m

    def set_beta(self, beta):
        lib().orc_ref_set_beta(self.h, beta)

    def close(self):
        if self.h:
            lib().orc_ref_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def ref_run_parallel(model, shape, beta, seed, n_chains, n_threads, therm, meas, q=3, J=1.0):
    dims = len(shape)
    lz = shape[2] if dims == 3 else 1
    att = ctypes.c_double()
    me = ctypes.c_double()
    mm = ctypes.c_double()
    dt = lib().orc_ref_run_parallel(model, dims, shape[0], shape[1], lz, q, J, beta, seed, n_chains,
                                    n_threads, therm, meas, ctypes.byref(att), ctypes.byref(me),
                                    ctypes.byref(mm))
    return dict(seconds=dt, attempts=att.value, mean_e=me.value, mean_m=mm.value)


def ref_msc_run(shape, beta, seed, sweeps, measure=True, J=1.0):
    dims = len(shape)
    lz = shape[2] if dims == 3 else 1
    att = ctypes.c_double()
    dt = lib().orc_ref_msc_run(dims, shape[0], shape[1], lz, J, beta, seed, sweeps,
                               1 if measure else 0, ctypes.byref(att))
    return dict(seconds=dt, attempts=att.value)

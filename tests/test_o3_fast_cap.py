"""The fast cap proposal of the O(3) Metropolis sweep ("cap_fast").

It draws the same random words as the engine's cap proposal and differs only
in arithmetic: the hardware approximations of sqrt, reciprocal, sin / cos and
exp take the place of the correctly rounded operations and the engine's own
polynomials.  Its parity with the oracle is therefore float32 tolerance, not
bit identity:

- one sweep from the oracle's initial state (the same seed): every site
  within 1e-5 per component of the oracle's exact-cap replay, except the
  few sites whose acceptance decision changed because a uniform fell within
  the approximations' error of its acceptance probability (and their
  neighbours of the other colour);
- the energy the sweep records equals, bit for bit, the oracle's fixed-point
  energy of the device's own spins (the recorded observable is a function of
  the configuration alone);
- over many sweeps, E/N and |M| agree with the reference sampler
  (random-permutation Metropolis, oracle/refsampler.c) within |z| < 3, as
  the exact cap does (CMC.rs/tests/physics/zscore_extended.rs:175-245).
"""
import ctypes
import math

import numpy as np
import pytest

from scamper_b200 import _lib

TOL = 1e-5  # per spin component, float32 spins of unit norm


def _params(shape, **kw):
    p = {"lattice_type": "square" if len(shape) == 2 else "cubic", "Lx": shape[0], "Ly": shape[1]}
    if len(shape) == 3:
        p["Lz"] = shape[2]
    p.update(kw)
    return p


def test_fast_cap_is_a_named_proposal(gpumc):
    spec, _keep = gpumc.mc.spec_from_params(_params((8, 8), beta=0.5), model="o3", o3_proposal="cap_fast")
    assert spec.o3_proposal == _lib.O3_CAP_FAST == 3
    gpumc.ClassicalMC.validate_params(_params((8, 8, 8), beta=0.5), model="o3", o3_proposal="cap_fast")
    # the C ABI rejects proposal codes past the last one
    spec.o3_proposal = 4
    with pytest.raises(gpumc.InvalidConfig):
        _lib.call("gpumc_validate", ctypes.byref(spec))


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(16, 16), (10, 6), (6, 6, 6), (16, 8, 12), (64, 16, 32)])
def test_gpu_fast_cap_one_sweep_within_float32_tolerance(gpumc, oracle, shape):
    beta, alpha = (0.9 if len(shape) == 2 else 0.7), 1.0
    omc = float(np.float32(2.0 * math.sin(0.5 * alpha) ** 2))
    mc = gpumc.ClassicalMC.from_params(_params(shape, beta=beta, cone_half_angle=alpha), 33, model="o3",
                                       o3_proposal="cap_fast")
    ref = oracle.Lattice(oracle.O3, shape, beta=beta, seed=33, omc=omc)
    np.testing.assert_array_equal(mc.spins().reshape(-1, 3), ref.state())
    mc.sweep(1)
    ref.sweep(adapt=True)
    dev = mc.spins().reshape(-1, 3)
    d = np.abs(dev.astype(np.float64) - ref.state().astype(np.float64)).max(axis=1)
    n = dev.shape[0]
    changed = int((d > TOL).sum())
    # a changed decision moves its site by the proposal's step; at most a few
    # such sites (and their other-colour neighbours) per sweep
    assert changed <= 7 + n // 1000, (changed, n, np.sort(d)[-10:])
    assert d[d <= TOL].mean() < 1e-6
    assert np.abs((dev.astype(np.float64) ** 2).sum(axis=1) - 1.0).max() < 1e-5
    # the recorded energy is the fixed-point energy of the device's own spins
    own = oracle.Lattice(oracle.O3, shape, beta=beta, seed=33, omc=omc)
    own.set_state(dev)
    assert mc.energy()[0] == own.fixed_observables()[0]
    assert mc.energy()[0] == pytest.approx(own.energy(), rel=1e-6, abs=1e-4)
    mc.close()


@pytest.mark.gpu
def test_gpu_fast_cap_observables_match_reference_sampler(gpumc, oracle):
    from tests.test_gpu_statistics import _compare, _ref_chains
    beta, shape, n_rep, therm, meas = 1.0 / 1.443, (8, 8, 8), 16, 1500, 6000
    mc = gpumc.ClassicalMC.from_params(_params(shape, cone_half_angle=1.0), 211, model="o3", n_replicas=n_rep,
                                       betas=[beta], record_capacity=1024, o3_proposal="cap_fast")
    mc.sweep(therm)
    mc.on_phase_start(_lib.PHASE_MEASUREMENT)
    es, ms = [], []
    left = meas
    while left:
        k = min(left, 1024)
        mc.sweep(k)
        a = mc.observable_arrays()
        es.append(a["energy"].reshape(k, n_rep))
        ms.append(a["magnetization"].reshape(k, n_rep))
        left -= k
    g_e, g_m = np.concatenate(es) / mc.n_sites, np.concatenate(ms)
    mc.close()
    r_e, r_m = _ref_chains(oracle, "o3", shape, beta, 8, therm, meas, seed=102)
    _compare(g_e, r_e, np.mean, "O(3) fast cap E/N")
    _compare(g_m, r_m, np.mean, "O(3) fast cap |M|")

"""O(3) Metropolis proposals of the reference (CMC.rs/src/lattice/proposal.rs):
StandardStrategy (an independent uniform unit vector, :45-63) and
OPSSStrategy (a rotation by theta uniform in (-sigma, sigma) in a random
coordinate plane, sigma adapted by exp(0.08 (rate - 0.5)) during
thermalization and clamped to [1e-4, pi], :72-167), beside the engine's
adapted cap.

CPU: the oracle's restatement of both samples the same distribution as the
heat bath (cross-solver <E> on the 4x4 torus, cf.
CMC.rs/tests/physics/continuous_cross_solver.rs), keeps unit norms and the
energy cache, and OPSS adapts sigma toward 50 % acceptance within its clamp.
GPU: the device kernels (plain and z-march) against the oracle bit for bit,
sigma included, through thermalization (adapting) and measurement (frozen).
"""
import math

import numpy as np
import pytest

from scamper_b200 import _lib

OPSS, UNIFORM = 2, 1


def _params(shape, **kw):
    p = {"lattice_type": "square" if len(shape) == 2 else "cubic", "Lx": shape[0], "Ly": shape[1]}
    if len(shape) == 3:
        p["Lz"] = shape[2]
    p.update(kw)
    return p


def _mean_energy(oracle, seeds, **kw):
    ms = []
    for seed in seeds:
        lat = oracle.Lattice(oracle.O3, (4, 4), beta=0.9, seed=seed, **kw)
        for i in range(400):
            lat.sweep(adapt=i < 200)
        es = []
        for _ in range(3000):
            lat.sweep()
            es.append(lat.cached_energy())
        st = lat.state().astype(np.float64)
        assert np.abs((st ** 2).sum(axis=1) - 1.0).max() < 1e-5
        assert lat.cached_energy() == pytest.approx(lat.energy(), rel=1e-9, abs=1e-9)
        ms.append(np.mean(es))
    return np.mean(ms), np.std(ms, ddof=1) / math.sqrt(len(ms))


@pytest.mark.parametrize("prop", [UNIFORM, OPSS])
def test_reference_proposals_sample_the_heat_bath_distribution(oracle, prop):
    m1, s1 = _mean_energy(oracle, range(1, 13), prop=prop, omc=0.5 if prop == OPSS else None)
    m2, s2 = _mean_energy(oracle, range(101, 113), algorithm=oracle.HEAT_BATH)
    assert abs(m1 - m2) < 4.0 * math.hypot(s1, s2), (m1, s1, m2, s2)


def test_opss_sigma_adapts_toward_half_acceptance_within_its_clamp(oracle):
    L = oracle.lib()
    assert L.orc_opss_adapt(1.0, 50, 100) == pytest.approx(1.0)
    assert L.orc_opss_adapt(1.0, 100, 100) == pytest.approx(math.exp(0.04), rel=1e-6)
    assert L.orc_opss_adapt(1.0, 0, 100) == pytest.approx(math.exp(-0.04), rel=1e-6)
    assert L.orc_opss_adapt(3.14, 100, 100) == pytest.approx(math.pi, rel=1e-7)
    assert L.orc_opss_adapt(1.0001e-4, 0, 100) == pytest.approx(1e-4, rel=1e-6)
    # a cold lattice accepts almost every small rotation: sigma grows; at
    # low temperature large rotations are rejected: it settles
    lat = oracle.Lattice(oracle.O3, (8, 8), beta=3.0, seed=4, prop=OPSS, omc=0.5)
    sig = []
    for _ in range(300):
        acc = lat.sweep(adapt=True)
        sig.append(float(lat.omc))
    rate = acc / lat.n
    assert 0.3 < rate < 0.7 and 1e-4 <= sig[-1] <= math.pi
    before = float(lat.omc)
    lat.sweep(adapt=False)
    assert float(lat.omc) == before


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(16, 16), (10, 6), (6, 6, 6), (16, 8, 12), (64, 16, 32)])
@pytest.mark.parametrize("prop", ["standard", "opss"])
def test_gpu_o3_proposals_match_oracle(gpumc, oracle, shape, prop):
    beta = 0.9 if len(shape) == 2 else 0.7
    mc = gpumc.ClassicalMC.from_params(_params(shape, beta=beta, opss_sigma=0.7), 33, model="o3",
                                       o3_proposal=prop)
    p = UNIFORM if prop == "standard" else OPSS
    ref = oracle.Lattice(oracle.O3, shape, beta=beta, seed=33, prop=p,
                         omc=float(np.float32(0.7)) if p == OPSS else None)
    np.testing.assert_array_equal(mc.spins(), ref.state().reshape(mc.spins().shape))
    # thermalization: OPSS adapts sigma after every sweep (the cap's rule is
    # not involved; the uniform proposal has nothing to adapt)
    for _ in range(5):
        mc.sweep(1)
        ref.sweep(adapt=True)
        np.testing.assert_array_equal(mc.spins(), ref.state().reshape(mc.spins().shape))
        if p == OPSS:
            assert np.float32(mc.cone_omc()) == np.float32(ref.omc)
    mc.on_phase_start(_lib.PHASE_MEASUREMENT)
    frozen = mc.cone_omc()
    for _ in range(3):
        mc.sweep(2)
        ref.sweep()
        ref.sweep()
        np.testing.assert_array_equal(mc.spins(), ref.state().reshape(mc.spins().shape))
        assert mc.energy()[0] == ref.fixed_observables()[0]
        assert mc.energy()[0] == pytest.approx(ref.cached_energy(), rel=1e-6, abs=1e-4)
    assert mc.cone_omc() == frozen
    if p == OPSS:
        assert mc.cone_half_angle() == pytest.approx(float(ref.omc), rel=1e-7)
    mc.close()


def test_o3_proposal_validated(gpumc):
    with pytest.raises(gpumc.InvalidConfig):
        gpumc.ClassicalMC.validate_params(_params((8, 8), beta=0.5), model="o3", o3_proposal="gibbs")
    gpumc.ClassicalMC.validate_params(_params((8, 8), beta=0.5), model="o3", o3_proposal="opss")
    gpumc.ClassicalMC.validate_params(_params((8, 8), beta=0.5), model="o3", o3_proposal="standard")

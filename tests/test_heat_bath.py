"""Heat-bath sweeps (HeatBathCore / ContinuousHeatBathCore,
CMC.rs/src/algorithms/heat_bath.rs:12-134).

CPU: the oracle's restatement of the engine's heat-bath method samples the
exact distributions the reference's heat-bath tests check
(CMC.rs/tests/physics/heat_bath_exact.rs): Ising <E>, <m^2> against full
enumeration at beta 0.3 and 0.8 (heat_bath_exact.rs:113-200, here on the 4x4
torus), Potts <E> against the row transfer matrix, and the O(3) conditional
moments of a spin in a fixed field against the Langevin function
(<cos> = coth x - 1/x, <cos^2> = 1 - 2 L(x)/x, heat_bath_exact.rs:1-40):
the field is fixed by resetting the other colour to +z before every sweep,
so each sweep's colour-0 sites are independent draws with kappa = 4 beta J.
The energy cache matches recomputation.

GPU: the device kernels against the oracle, bit for bit (spins, energy,
changed counts) for Ising (2D / 3D, streaming and resident), Potts (int8
kernel, every q) and O(3) (2D / 3D, plain and z-march), then the device
statistics on the same exact references.
"""
import math

import numpy as np
import pytest

from scamper_b200 import _lib
from tests import exact

HB = 1


def _zs_ok(zs):
    assert max(abs(z) for z in zs) < 4.0, zs
    assert abs(np.mean(zs)) < 2.0, zs
    assert sum(zs) > -2.0 * math.sqrt(len(zs)), zs


_replicas_ok = exact.replicas_ok


def _chain(lat, therm, meas):
    for _ in range(therm):
        lat.sweep()
    es, ms = [], []
    for _ in range(meas):
        lat.sweep()
        es.append(lat.cached_energy())
        if lat.model == 0:
            ms.append((lat.spins.astype(np.float64).sum() / lat.n) ** 2)
    return es, ms


@pytest.mark.parametrize("beta,J", [(0.3, 1.0), (0.8, 1.0), (0.4, -1.0)])
def test_ising_heat_bath_samples_exact_4x4(oracle, beta, J):
    ex = exact.ising_enumeration(4, 4, beta, J=J)
    zs_e, zs_m = [], []
    for seed in range(1, 7):
        lat = oracle.Lattice(oracle.ISING, (4, 4), J=J, beta=beta, seed=seed, algorithm=HB)
        es, ms = _chain(lat, 200, 6000)
        me, se = exact.binned(es)
        mm, sm = exact.binned(ms)
        zs_e.append(exact.zscore(me, se, ex["E"]))
        zs_m.append(exact.zscore(mm, sm, ex["M2"]))
    _zs_ok(zs_e)
    _zs_ok(zs_m)


@pytest.mark.parametrize("q,beta,J", [(2, 0.9, 1.0), (3, None, 1.0), (5, None, 1.0), (3, 0.6, -1.0)])
def test_potts_heat_bath_samples_exact_4x4(oracle, q, beta, J):
    beta = math.log(1.0 + math.sqrt(q)) if beta is None else beta
    ex = exact.potts_transfer_matrix(4, 4, q, beta, J=J)
    zs = []
    for seed in range(1, 7):
        lat = oracle.Lattice(oracle.POTTS, (4, 4), q=q, J=J, beta=beta, seed=seed, algorithm=HB)
        es, _ = _chain(lat, 200, 6000)
        me, se = exact.binned(es)
        zs.append(exact.zscore(me, se, ex["E"]))
    _zs_ok(zs)


def _langevin(x):
    L = 1.0 / math.tanh(x) - 1.0 / x
    return L, 1.0 - 2.0 * L / x


@pytest.mark.parametrize("kappa,J", [(0.2, 1.0), (1.5, 1.0), (5.0, 1.0), (1.5, -1.0), (1e-7, 1.0)])
def test_o3_heat_bath_conditional_moments(oracle, kappa, J):
    lat = oracle.Lattice(oracle.O3, (4, 4), J=J, beta=kappa / 4.0, seed=3, algorithm=HB)
    colour0 = ((np.arange(16) % 4 + np.arange(16) // 4) % 2) == 0
    c1, c2 = [], []
    for _ in range(4000):
        st = lat.state()
        st[~colour0] = (0.0, 0.0, 1.0)
        lat.set_state(st)
        lat.sweep()
        sz = lat.state()[colour0, 2].astype(np.float64) * (1.0 if J > 0 else -1.0)
        c1.extend(sz)
        c2.extend(sz * sz)
    c1, c2 = np.array(c1), np.array(c2)
    if kappa < 1e-3:
        m1, m2 = 0.0, 1.0 / 3.0
    else:
        m1, m2 = _langevin(kappa)
    n = len(c1)
    assert abs(c1.mean() - m1) < 4.0 * c1.std() / math.sqrt(n) + 1e-6
    assert abs(c2.mean() - m2) < 4.0 * c2.std() / math.sqrt(n) + 1e-6
    st = lat.state().astype(np.float64)
    assert np.abs((st ** 2).sum(axis=1) - 1.0).max() < 1e-5


@pytest.mark.parametrize("model,shape,q", [("ising", (6, 6, 6), 2), ("potts", (6, 6, 6), 3),
                                           ("potts", (8, 6), 7), ("o3", (6, 4, 6), 2)])
def test_heat_bath_energy_cache_matches_recompute(oracle, model, shape, q):
    m = {"ising": oracle.ISING, "potts": oracle.POTTS, "o3": oracle.O3}[model]
    lat = oracle.Lattice(m, shape, q=q, beta=0.45, seed=5, algorithm=HB)
    changed = [lat.sweep() for _ in range(300)]
    assert 0 < np.mean(changed) <= lat.n
    if model == "o3":
        assert lat.cached_energy() == pytest.approx(lat.energy(), rel=1e-9, abs=1e-6)
        assert np.mean(changed) == lat.n  # a continuous draw always moves the spin
    else:
        assert lat.cached_energy() == lat.energy()


def test_heat_bath_tables(oracle):
    # Ising: T[k] = T[z-k] = p(|x|), zero field exactly 1/2, never "always"
    head, tail = oracle.table(oracle.ISING, 2, 1.0, 0.7, HB)
    assert len(head) == 5 and head[2] == 32768 and tail[2] == 0
    assert (head[0], tail[0]) == (head[4], tail[4]) and (head[1], tail[1]) == (head[3], tail[3])
    p = 1.0 / (1.0 + math.exp(-2 * 0.7 * 4))
    assert head[0] == math.floor(p * 65536) and head.max() < 65536
    head, tail = oracle.table(oracle.ISING, 3, 1.0, 50.0, HB)  # p rounds to 1: clamped
    assert head.max() == 65535
    # Potts: W[d] = floor(2^60 exp(-beta |J| d)), favoured state exactly 2^60
    head, tail = oracle.table(oracle.POTTS, 2, -1.5, 0.4, HB)
    assert tail[0] == 1 << 60 and (head == 0).all()
    for d in range(5):
        assert abs(int(tail[d]) - math.exp(-0.6 * d) * 2.0 ** 60) <= 2.0 ** 60 * 1e-15 + 1


# ---------------------------------------------------------------------------
# device kernels against the oracle
# ---------------------------------------------------------------------------
def _params(shape, **kw):
    p = {"lattice_type": "square" if len(shape) == 2 else "cubic", "Lx": shape[0], "Ly": shape[1]}
    if len(shape) == 3:
        p["Lz"] = shape[2]
    p.update(kw)
    return p


ISING_SHAPES = [(64, 64), (66, 10), (200, 6), (4, 4), (6, 6, 6), (64, 8, 10), (130, 6, 4)]


@pytest.mark.gpu
@pytest.mark.parametrize("shape", ISING_SHAPES)
@pytest.mark.parametrize("beta,J", [(0.4407, 1.0), (0.3, -1.0), (0.0, 1.0)])
def test_gpu_ising_heat_bath_matches_oracle(gpumc, oracle, shape, beta, J):
    mc = gpumc.ClassicalMC.from_params(_params(shape, beta=beta, J=J), 17, model="ising",
                                       algorithm="heat_bath")
    ref = oracle.Lattice(oracle.ISING, shape, J=J, beta=beta, seed=17, algorithm=HB)
    np.testing.assert_array_equal(mc.spins(), ref.spins.reshape(mc.spins().shape))
    mc.on_phase_start(_lib.PHASE_MEASUREMENT)
    for _ in range(4):
        mc.sweep(3)
        for _ in range(3):
            ref.sweep()
        np.testing.assert_array_equal(mc.spins().ravel(), ref.spins)
        assert mc.energy()[0] == ref.cached_energy()
    obs = mc.observables()
    assert len(obs) == 12
    mc.close()


@pytest.mark.gpu
def test_gpu_ising_heat_bath_resident_equals_streaming(gpumc):
    """The temporally blocked launch and the per-sweep kernel run the same
    heat-bath trajectory."""
    out = []
    for blocking in (True, False):
        mc = gpumc.ClassicalMC.from_params(_params((512, 512), beta=0.44), 5, model="ising",
                                           n_replicas=3, betas=[0.3, 0.44, 0.6], algorithm="heat_bath")
        mc.set_temporal_blocking(blocking)
        mc.pt_configure(10)
        mc.sweep(70)
        out.append((np.stack([mc.spins(r) for r in range(3)]), mc.energy(), mc.pt_labels()))
        mc.close()
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])
    assert list(out[0][2]) == list(out[1][2])


POTTS_SHAPES = [(32, 32), (34, 18), (6, 6, 6), (18, 8, 10), (4, 4)]


@pytest.mark.gpu
@pytest.mark.parametrize("shape", POTTS_SHAPES)
@pytest.mark.parametrize("q,J", [(2, 1.0), (3, 1.0), (4, -1.0), (5, 1.0), (8, 1.0)])
def test_gpu_potts_heat_bath_matches_oracle(gpumc, oracle, shape, q, J):
    beta = 1.1
    mc = gpumc.ClassicalMC.from_params(_params(shape, beta=beta, q=q, J=J), 23, model="potts",
                                       algorithm="heat_bath")
    ref = oracle.Lattice(oracle.POTTS, shape, q=q, J=J, beta=beta, seed=23, algorithm=HB)
    for _ in range(3):
        mc.sweep(2)
        ref.sweep()
        ref.sweep()
        np.testing.assert_array_equal(mc.spins().ravel(), ref.spins)
        assert mc.energy()[0] == ref.cached_energy()
    mc.close()


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(16, 16), (10, 6), (6, 6, 6), (16, 8, 12), (64, 16, 32)])
@pytest.mark.parametrize("J", [1.0, -0.5])
def test_gpu_o3_heat_bath_matches_oracle(gpumc, oracle, shape, J):
    beta = 0.9
    mc = gpumc.ClassicalMC.from_params(_params(shape, beta=beta, J=J), 29, model="o3",
                                       algorithm="heat_bath")
    ref = oracle.Lattice(oracle.O3, shape, J=J, beta=beta, seed=29, algorithm=HB)
    mc.on_phase_start(_lib.PHASE_MEASUREMENT)
    for _ in range(3):
        mc.sweep(2)
        ch = ref.sweep() + ref.sweep()
        np.testing.assert_array_equal(mc.spins(), ref.state().reshape(mc.spins().shape))
        # the kernels' fixed-point bond sum, exactly; within fp32 rounding of
        # the reference's exact energy cache
        assert mc.energy()[0] == ref.fixed_observables()[0]
        assert mc.energy()[0] == pytest.approx(ref.cached_energy(), rel=1e-6, abs=1e-4)
    obs = mc.observables()
    assert obs[-1]["acceptance"] == pytest.approx(ch / 2 / ref.n) or obs[-1]["acceptance"] > 0.99
    mc.close()


@pytest.mark.gpu
@pytest.mark.parametrize("beta", [0.3, 0.8])
def test_gpu_ising_heat_bath_samples_exact_4x4(gpumc, beta):
    ex = exact.ising_enumeration(4, 4, beta)
    mc = gpumc.ClassicalMC.from_params(_params((4, 4), beta=beta), 101, model="ising", n_replicas=16,
                                       algorithm="heat_bath", record_capacity=8192)
    mc.sweep(200)
    mc.on_phase_start(_lib.PHASE_MEASUREMENT)
    mc.sweep(4000)
    rows = mc.observable_arrays()
    _replicas_ok([rows["energy"][rows["replica"] == r] for r in range(16)], ex["E"])
    mc.close()


@pytest.mark.gpu
@pytest.mark.parametrize("q,J", [(3, 1.0), (6, 1.0), (3, -1.0)])
def test_gpu_potts_heat_bath_samples_exact_4x4(gpumc, q, J):
    beta = 0.9
    ex = exact.potts_transfer_matrix(4, 4, q, beta, J=J)
    mc = gpumc.ClassicalMC.from_params(_params((4, 4), beta=beta, q=q, J=J), 77, model="potts", n_replicas=16,
                                       algorithm="heat_bath", record_capacity=8192)
    mc.sweep(200)
    mc.on_phase_start(_lib.PHASE_MEASUREMENT)
    mc.sweep(4000)
    rows = mc.observable_arrays()
    _replicas_ok([rows["energy"][rows["replica"] == r] for r in range(16)], ex["E"])
    mc.close()


@pytest.mark.gpu
def test_gpu_heat_bath_rejected_for_multispin(gpumc):
    with pytest.raises(gpumc.InvalidConfig):
        gpumc.ClassicalMC.from_params(_params((64, 64), beta=0.4), 1, model=_lib.ISING_MSC64,
                                      algorithm="heat_bath")
    with pytest.raises(gpumc.InvalidConfig):
        gpumc.ClassicalMC.from_params(_params((64, 64), beta=0.4), 1, model="ising", algorithm="overrelaxation")

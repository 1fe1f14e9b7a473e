"""GPU parity: the CUDA sweep kernels against the oracle's replay of the same
method (checkerboard order, Philox stream keyed by (seed, replica, sweep,
site)).  Spins must agree byte for byte (int8 Ising / Potts, uint64 multi-spin)
and bit for bit (float32 O(3)); energies and records must agree exactly for the
integer models and to 1e-9 relative for O(3)."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _params(shape, **kw):
    p = {"lattice_type": "square" if len(shape) == 2 else "cubic", "Lx": shape[0], "Ly": shape[1]}
    if len(shape) == 3:
        p["Lz"] = shape[2]
    p.update(kw)
    return p


def _omc(alpha):
    return float(np.float32(2.0 * math.sin(0.5 * alpha) * math.sin(0.5 * alpha)))


def _gpu_state(mc, replica=0):
    s = mc.spins(replica)
    return s.reshape(-1, 3) if mc.model == 2 else s.ravel()


def _run_parity(gpumc, oracle, model_name, shape, beta, seed, sweeps, q=3, J=1.0, alpha=1.0,
                measure=False):
    from scamper_b200 import _lib
    mid = {"ising": oracle.ISING, "potts": oracle.POTTS, "o3": oracle.O3, "msc": oracle.MSC}[model_name]
    params = _params(shape, beta=beta, q=q, J=J, cone_half_angle=alpha)
    if model_name == "msc":
        mc = gpumc.MultiSpinIsing.from_params(params, seed)
    else:
        mc = gpumc.ClassicalMC.from_params(params, seed, model=model_name)
    orc = oracle.Lattice(mid, shape, q=q, J=J, beta=beta, seed=seed, omc=_omc(alpha))
    try:
        np.testing.assert_array_equal(_gpu_state(mc), orc.state(), err_msg="initial state")
        if measure:
            mc.on_phase_start(_lib.PHASE_MEASUREMENT)
        for s in range(sweeps):
            mc.sweep(1)
            orc.sweep(adapt=(model_name == "o3" and not measure))
            np.testing.assert_array_equal(_gpu_state(mc), orc.state(), err_msg=f"after sweep {s + 1}")
        if model_name in ("ising", "potts"):
            assert mc.energy()[0] == orc.cached_energy() == orc.energy()
        elif model_name == "o3":
            # the kernels' fixed-point bond sum of the fp32 configuration,
            # exactly; within fp32 rounding of the exact fp64 energy
            assert mc.energy()[0] == orc.fixed_observables()[0]
            assert mc.energy()[0] == pytest.approx(orc.energy(), rel=1e-6, abs=1e-4)
        else:
            e64, m64 = mc.replica_observables(0)
            oe, om = orc.msc_observables()
            np.testing.assert_array_equal(e64, oe)
            np.testing.assert_allclose(m64, np.abs(om) / orc.n)
            assert mc.energy()[0] == pytest.approx(oe.sum())
        return mc, orc
    except Exception:
        mc.close()
        raise


ISING_2D = [(4, 4), (8, 8), (34, 6), (64, 64), (130, 20), (16, 130), (1040, 8), (2054, 4), (256, 300),
            (130, 302)]
ISING_3D = [(4, 4, 4), (6, 8, 10), (34, 6, 4), (16, 16, 36), (288, 6, 4), (128, 800, 4), (128, 64, 40)]


@pytest.mark.parametrize("shape", ISING_2D)
@pytest.mark.parametrize("beta", [0.35, 0.4407, 0.5])
def test_ising_2d_bit_exact(gpumc, oracle, shape, beta):
    _run_parity(gpumc, oracle, "ising", shape, beta, seed=17, sweeps=4)[0].close()


@pytest.mark.parametrize("shape,beta,sweeps", [((256, 300), 0.4407, 7), ((130, 302), 0.5, 5),
                                              ((2054, 4), 0.35, 3), ((64, 64), 0.3, 70)])
def test_ising_multi_sweep_call_matches_oracle(gpumc, oracle, shape, beta, sweeps):
    """Many sweeps in one call (one resident launch for whole-row 2D tiles:
    the packed tiles stay on chip and exchange edge rows between sweeps)
    against the oracle, with every sweep's record."""
    from scamper_b200 import _lib
    mc = gpumc.ClassicalMC.from_params(_params(shape, beta=beta), 41, record_capacity=128)
    mc.on_phase_start(_lib.PHASE_MEASUREMENT)
    orc = oracle.Lattice(oracle.ISING, shape, beta=beta, seed=41)
    mc.sweep(sweeps)
    energies = []
    for _ in range(sweeps):
        orc.sweep()
        energies.append(orc.cached_energy())
    np.testing.assert_array_equal(mc.spins().ravel(), orc.state())
    recs = mc.observables()
    assert [r["energy"] for r in recs] == energies
    assert recs[-1]["magnetization"] == pytest.approx(abs(int(orc.state().astype(np.int64).sum())) / orc.n)
    assert mc.energy()[0] == orc.energy()
    mc.close()


@pytest.mark.parametrize("shape", ISING_3D)
def test_ising_3d_bit_exact(gpumc, oracle, shape):
    _run_parity(gpumc, oracle, "ising", shape, 0.2216, seed=5, sweeps=4)[0].close()


@pytest.mark.parametrize("shape", [(4, 4), (34, 6), (130, 20), (1040, 8), (2048, 64), (8256, 6), (4, 4, 4),
                                   (6, 8, 10), (34, 6, 36), (128, 400, 4)])
@pytest.mark.parametrize("q", [2, 3, 4, 5])
def test_potts_bit_exact(gpumc, oracle, shape, q):
    beta = math.log(1.0 + math.sqrt(q)) * (1.0 if len(shape) == 2 else 0.6)
    _run_parity(gpumc, oracle, "potts", shape, beta, seed=3 + q, sweeps=4, q=q)[0].close()


@pytest.mark.parametrize("shape", [(4, 4), (66, 10), (130, 44), (4, 4, 4), (8, 6, 20), (70, 4, 6), (64, 64, 8)])
def test_o3_bit_exact(gpumc, oracle, shape):
    _run_parity(gpumc, oracle, "o3", shape, 0.7, seed=23, sweeps=4, alpha=1.0)[0].close()


@pytest.mark.parametrize("shape", [(4, 4), (66, 10), (130, 8), (4, 4, 4), (34, 6, 20)])
def test_msc_bit_exact(gpumc, oracle, shape):
    beta = 0.4407 if len(shape) == 2 else 0.2216
    _run_parity(gpumc, oracle, "msc", shape, beta, seed=29, sweeps=3)[0].close()


def test_antiferromagnetic_and_zero_beta(gpumc, oracle):
    _run_parity(gpumc, oracle, "ising", (8, 6), 0.6, seed=2, sweeps=3, J=-1.0)[0].close()
    _run_parity(gpumc, oracle, "ising", (8, 6), 0.0, seed=2, sweeps=3)[0].close()
    _run_parity(gpumc, oracle, "potts", (8, 6), 0.9, seed=2, sweeps=3, q=3, J=-0.5)[0].close()


def test_records_match_oracle(gpumc, oracle):
    mc, orc = _run_parity(gpumc, oracle, "ising", (34, 6), 0.44, seed=8, sweeps=0)
    from scamper_b200 import _lib
    mc.on_phase_start(_lib.PHASE_MEASUREMENT)
    exp = []
    for _ in range(12):
        orc.sweep()
        exp.append((orc.cached_energy(), abs(int(orc.spins.astype(np.int64).sum())) / orc.n))
    mc.sweep(12)
    recs = mc.observables()
    assert [r["sweep"] for r in recs] == list(range(12))
    for r, (e, m) in zip(recs, exp):
        assert r["energy"] == e and r["magnetization"] == pytest.approx(m, abs=0)
    mc.close()


def test_potts_order_parameter_record(gpumc, oracle):
    from scamper_b200 import _lib
    q = 4
    mc = gpumc.ClassicalMC.from_params(_params((20, 10), beta=1.0, q=q), 4, model="potts")
    orc = oracle.Lattice(oracle.POTTS, (20, 10), q=q, beta=1.0, seed=4)
    mc.on_phase_start(_lib.PHASE_MEASUREMENT)
    mc.sweep(5)
    for _ in range(5):
        orc.sweep()
    r = mc.observables()[-1]
    counts = np.bincount(orc.spins.astype(np.int64), minlength=q)
    assert r["magnetization"] == pytest.approx((q * counts.max() - orc.n) / (orc.n * (q - 1)))
    mc.close()


def test_cold_start_and_set_spins_roundtrip(gpumc, oracle):
    mc = gpumc.ClassicalMC.from_params(_params((10, 8), beta=0.3, initial_state="cold"), 1)
    assert (mc.spins() == 1).all()
    assert mc.energy()[0] == -2 * 80
    rng = np.random.default_rng(0)
    s = rng.choice(np.array([-1, 1], dtype=np.int8), size=80)
    mc.set_spins(0, s)
    np.testing.assert_array_equal(mc.spins().ravel(), s)
    orc = oracle.Lattice(oracle.ISING, (10, 8), beta=0.3, seed=1)
    orc.set_state(s)
    assert mc.energy()[0] == orc.energy()
    with pytest.raises(gpumc.InvalidConfig):
        mc.set_spins(0, np.zeros(80, dtype=np.int8))
    mc.close()


@pytest.mark.parametrize("model,shape,q", [("ising", (200, 34), 2), ("ising", (6, 10, 12), 2),
                                           ("potts", (130, 18), 3), ("potts", (34, 6, 8), 4),
                                           ("ising", (1024, 8), 2)])
def test_set_spins_validates_on_device_and_keeps_state(gpumc, oracle, model, shape, q):
    """set_spins stages the state on the device, checks every value
    (validate_spin) and computes the exact energy in one pass; an invalid
    value anywhere rejects the whole state and keeps the old one."""
    kw = dict(beta=0.3) if model == "ising" else dict(beta=0.9, q=q)
    mc = gpumc.ClassicalMC.from_params(_params(shape, **kw), 3, model=model)
    n = int(np.prod(shape))
    rng = np.random.default_rng(11)
    vals = np.array([-1, 1], dtype=np.int8) if model == "ising" else np.arange(q, dtype=np.int8)
    s = rng.choice(vals, size=n)
    mc.set_spins(0, s)
    np.testing.assert_array_equal(mc.spins().ravel(), s)
    mid = oracle.ISING if model == "ising" else oracle.POTTS
    orc = oracle.Lattice(mid, shape, q=q, beta=kw["beta"], seed=3)
    orc.set_state(s)
    assert mc.energy()[0] == orc.energy()
    np.testing.assert_array_equal(mc.recompute_energy(), mc.energy())
    bad_values = [0, 2, -2] if model == "ising" else [-1, q, 100]
    for pos in [0, n // 2 + 1, n - 1]:
        for v in bad_values:
            t = rng.choice(vals, size=n)
            t[pos] = v
            with pytest.raises(gpumc.InvalidConfig):
                mc.set_spins(0, t)
    np.testing.assert_array_equal(mc.spins().ravel(), s)
    assert mc.energy()[0] == orc.energy()
    mc.sweep(3)  # the sweeps continue from the accepted state
    for _ in range(3):
        orc.sweep()
    np.testing.assert_array_equal(mc.spins().ravel(), orc.state())
    assert mc.energy()[0] == orc.cached_energy()
    mc.close()


def _golden_cases():
    import json
    import os
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "replay_fingerprints.json")
    with open(path) as f:
        return json.load(f)["cases"]


@pytest.mark.parametrize("case", _golden_cases(),
                         ids=[f"{c['model']}-{'x'.join(map(str, c['shape']))}"
                              + {"heat_bath": "-hb", "swendsen_wang": "-sw", "wolff": "-wolff"}.get(
                                  c["extra"].get("algorithm"), "")
                              + ("-" + c["extra"]["proposal"] if "proposal" in c["extra"] else "")
                              for c in _golden_cases()])
def test_device_matches_committed_golden_fingerprints(gpumc, case):
    """The device against the committed fixtures, without the oracle."""
    import hashlib
    from scamper_b200 import _lib
    shape, extra = tuple(case["shape"]), case["extra"]
    params = _params(shape, beta=case["beta"], q=extra.get("q", 3), J=extra.get("J", 1.0),
                     cone_half_angle=extra.get("alpha", 1.0), opss_sigma=extra.get("sigma", 0.5))
    if case["model"] == "msc":
        mc = gpumc.MultiSpinIsing.from_params(params, case["seed"])
    else:
        mc = gpumc.ClassicalMC.from_params(params, case["seed"], model=case["model"],
                                           algorithm=extra.get("algorithm"), o3_proposal=extra.get("proposal"))
    mc.on_phase_start(_lib.PHASE_MEASUREMENT)  # no cone adaptation (O(3))
    mc.sweep(case["sweeps"])
    st = np.ascontiguousarray(_gpu_state(mc))
    assert hashlib.sha256(st.tobytes()).hexdigest() == case["sha256"]
    if case["model"] == "o3":
        # fixture: exact fp64 energy; device: fixed-point sum of fp32 bonds
        assert mc.energy()[0] == pytest.approx(case["energy"], rel=1e-6, abs=1e-4)
    elif case["model"] == "msc":
        e64, _ = mc.replica_observables(0)
        assert float(e64.sum()) == case["energy"]
    else:
        assert mc.energy()[0] == case["energy"]
    mc.close()


def test_philox_device_matches_known_answers_and_oracle(gpumc, oracle):
    import ctypes
    from scamper_b200 import _lib
    rng = np.random.default_rng(5)
    ctr = rng.integers(0, 2 ** 32, size=(64, 4), dtype=np.uint64).astype(np.uint32)
    key = rng.integers(0, 2 ** 32, size=(64, 2), dtype=np.uint64).astype(np.uint32)
    ctr[0] = 0
    key[0] = 0
    ctr[1] = 0xFFFFFFFF
    key[1] = 0xFFFFFFFF
    out = np.zeros((64, 4), dtype=np.uint32)
    P = ctypes.POINTER(ctypes.c_uint32)
    _lib.call("gpumc_philox_probe", ctr.ctypes.data_as(P), key.ctypes.data_as(P), out.ctypes.data_as(P), 64)
    assert tuple(out[0]) == (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)
    assert tuple(out[1]) == (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)
    for i in range(64):
        np.testing.assert_array_equal(out[i], oracle.philox(ctr[i], key[i]))

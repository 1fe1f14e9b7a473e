"""CPU tests of the host side: the C-ABI library loads and exports every entry
point include/gpumc.h declares, spec validation follows the reference's
InvalidConfig rules, and the Python mirror parses the reference's parameter
keys.  No compute call needs a GPU here."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "gpumc.h")).read()
    return sorted(set(re.findall(r"^int (gpumc_\w+)\(", src, flags=re.M)))


def test_library_exports_every_declared_symbol(gpumc):
    lib = gpumc._lib.load()
    names = _declared()
    assert len(names) >= 30
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(gpumc._lib.SIGNATURES), "Python bindings out of sync with the header"


def _spec(gpumc, **kw):
    from scamper_b200.mc import spec_from_params
    p = {"lattice_type": "square", "Lx": 8, "Ly": 8, "beta": 0.4}
    p.update(kw)
    return spec_from_params(p, model=kw.pop("model", None) if "model" in kw else None)


@pytest.mark.parametrize("bad", [
    dict(Lx=7), dict(Ly=2), dict(beta=-0.5), dict(beta=float("inf")), dict(J=float("nan")),
    dict(pbc="false"), dict(model="potts", q=1), dict(model="potts", q=9),
])
def test_validate_rejects_invalid_specs(gpumc, bad):
    from scamper_b200.mc import spec_from_params
    p = {"lattice_type": "square", "Lx": 8, "Ly": 8, "beta": 0.4}
    model = bad.pop("model", None)
    p.update(bad)
    spec, keep = spec_from_params(p, model=model)
    rc = gpumc._lib.load().gpumc_validate(ctypes.byref(spec))
    assert rc == gpumc._lib.EINVAL
    assert gpumc._lib.last_error()


def test_validate_accepts_reference_configs(gpumc):
    from scamper_b200.mc import spec_from_params
    for p, model in [
        ({"L": 64, "beta": 0.4407}, "ising"),
        ({"lattice_type": "square", "Lx": 8192, "beta": 0.4407}, "ising"),
        ({"lattice_type": "cubic", "L": 128, "beta": 0.2}, "ising"),
        ({"lattice_type": "square", "L": 2048, "q": 4, "beta": 1.1}, "potts"),
        ({"lattice_type": "cubic", "L": 64, "beta": 0.7, "cone_half_angle": 0.9}, "o3"),
        ({"lattice_type": "hypercubic", "Lx": 34, "Ly": 10, "Lz": 6, "beta": 0.7}, "o3"),
    ]:
        spec, keep = spec_from_params(p, model=model)
        assert gpumc._lib.load().gpumc_validate(ctypes.byref(spec)) == 0, gpumc._lib.last_error()
        n = ctypes.c_size_t()
        assert gpumc._lib.load().gpumc_footprint(ctypes.byref(spec), ctypes.byref(n)) == 0
        assert n.value > 0


def test_footprint_counts_both_ping_pong_buffers(gpumc):
    from scamper_b200.mc import spec_from_params
    spec, keep = spec_from_params({"lattice_type": "square", "Lx": 8192, "beta": 0.44}, model="ising",
                                  record_capacity=1)
    n = ctypes.c_size_t()
    gpumc._lib.call("gpumc_footprint", ctypes.byref(spec), ctypes.byref(n))
    assert 2 * 8192 * 8192 <= n.value < 2 * 8192 * 8192 + (1 << 20)


def test_unknown_lattice_and_model_raise(gpumc):
    from scamper_b200.mc import spec_from_params
    with pytest.raises(gpumc.InvalidConfig):
        spec_from_params({"lattice_type": "kagome", "Lx": 8}, model="ising")
    with pytest.raises(gpumc.InvalidConfig):
        spec_from_params({"Lx": 8}, model="xy")
    with pytest.raises(gpumc.InvalidConfig):
        spec_from_params({"Lx": 8, "initial_state": "lukewarm"}, model="ising")


def test_no_device_fails_loudly_without_cpu_fallback(gpumc):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    e = ctypes.c_void_p()
    rc = gpumc._lib.load().gpumc_engine_create(0, ctypes.byref(e))
    assert rc == gpumc._lib.ENODEV
    with pytest.raises(gpumc.GpumcError):
        gpumc.ClassicalMC.from_params({"Lx": 8, "Ly": 8}, 1)


def test_geometric_ladder(gpumc):
    b = gpumc.geometric_ladder_betas(1.5, 3.5, 64)
    assert len(b) == 64
    assert 1 / b[0] == pytest.approx(1.5) and 1 / b[-1] == pytest.approx(3.5)
    assert all(x > y for x, y in zip(b, b[1:]))


@pytest.mark.parametrize("model", [0, 1, 2, 3])
def test_every_geometry_has_a_tile_plan(gpumc, model):
    """Each model and extent in the benchmark and serving ranges gets a tile
    plan with positive steps, and every tile it enumerates fits its shared
    memory plan (validation re-derives each bit-sliced tile's geometry)."""
    from scamper_b200.mc import spec_from_params
    lib = gpumc._lib.load()
    for q in ([2, 3, 4, 5, 8] if model == 1 else [3]):
        for dims in (2, 3):
            sizes = [4, 6, 10, 16, 30, 34, 62, 64, 66, 126, 128, 130, 190, 192]
            if dims == 2:
                sizes += [256, 510, 514, 1024, 2046, 2048, 2050, 4096, 8192, 8256, 16384, 20032]
            for L in sizes:
                p = {"lattice_type": "square" if dims == 2 else "cubic", "L": L, "beta": 0.4, "q": q}
                spec, keep = spec_from_params(p, model=model)
                assert lib.gpumc_validate(ctypes.byref(spec)) == 0, (model, q, dims, L, gpumc._lib.last_error())
            if dims == 2:
                for shape in [(130, 66), (8256, 6), (20032, 10), (34, 34)]:
                    p = {"lattice_type": "square", "Lx": shape[0], "Ly": shape[1], "beta": 0.4, "q": q}
                    spec, keep = spec_from_params(p, model=model)
                    assert lib.gpumc_validate(ctypes.byref(spec)) == 0, (model, q, shape, gpumc._lib.last_error())


def test_random_geometries_validate_and_plan(gpumc):
    """Seeded random lattices across models, algorithms and O(3) proposals:
    every even extent >= 4 validates and gets a tile plan with and without
    refinement; an odd extent is rejected with GPUMC_EINVAL (the checkerboard
    needs even extents)."""
    import random
    from scamper_b200.mc import spec_from_params
    lib = gpumc._lib.load()
    rng = random.Random(5)
    for _ in range(600):
        model = rng.choice(["ising", "potts", "o3"])
        q = rng.choice([2, 3, 4, 5, 6, 8]) if model == "potts" else 3
        alg = rng.choice([None, "heat_bath"])
        prop = rng.choice([None, "standard", "opss", "cap_fast"]) if model == "o3" and alg is None else None
        if rng.random() < 0.5:
            lx, ly = 2 * rng.randint(2, 6000), 2 * rng.randint(2, 3000)
            if lx * ly > 300_000_000:
                continue
            p = {"lattice_type": "square", "Lx": lx, "Ly": ly, "beta": 0.4, "q": q}
        else:
            lx, ly, lz = (2 * rng.randint(2, 160) for _ in range(3))
            p = {"lattice_type": "cubic", "Lx": lx, "Ly": ly, "Lz": lz, "beta": 0.4, "q": q}
        spec, keep = spec_from_params(p, model=model, algorithm=alg, o3_proposal=prop)
        assert lib.gpumc_validate(ctypes.byref(spec)) == 0, (p, model, alg, prop, gpumc._lib.last_error())
        for refine in (True, False):
            n, kind = gpumc.plan_tiles(p, model=model, algorithm=alg, refine=refine)
            assert n > 0, (p, model, alg, refine)
        odd = dict(p, Lx=lx + 1)
        spec, keep = spec_from_params(odd, model=model, algorithm=alg, o3_proposal=prop)
        assert lib.gpumc_validate(ctypes.byref(spec)) == gpumc._lib.EINVAL, odd

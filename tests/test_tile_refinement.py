"""Launch-dependent tile shapes: a launch with fewer tiles than half the
device's CTA slots splits its 3D Ising, Potts and O(3) tiles until it fills
them.  CPU: the host planner (gpumc_plan_tiles) on lone lattices and on the
full launches that must keep their plans.  GPU: refined and unrefined tiles
give identical spins, energies and records, on a handle's own path and in a
batched engine (results depend on sites and row segments, never on tiles)."""
import numpy as np
import pytest

SLOTS, SLOTS3 = 148 * 4, 148 * 3


def _params(shape, **kw):
    p = {"lattice_type": "square" if len(shape) == 2 else "cubic", "Lx": shape[0], "Ly": shape[1]}
    if len(shape) == 3:
        p["Lz"] = shape[2]
    p.update(kw)
    return p


LONE = [
    ("o3", (64, 64, 64), {}, None),
    ("o3", (108, 108, 108), {}, None),
    ("o3", (16, 16, 16), {}, None),
    ("o3", (256, 256), {}, None),
    ("ising", (188, 188, 188), {}, None),
    ("ising", (16, 16, 16), {}, None),
    ("potts", (1660, 1660), dict(q=3), None),
    ("potts", (512, 512), dict(q=6), None),
    ("potts", (40, 40, 40), dict(q=3), None),
    ("potts", (64, 64, 64), dict(q=5), "heat_bath"),
]


@pytest.mark.parametrize("model,shape,kw,alg", LONE)
def test_lone_lattice_is_split_until_it_fills_half_the_slots(gpumc, model, shape, kw, alg):
    p = _params(shape, beta=0.5, **kw)
    n0, _ = gpumc.plan_tiles(p, model=model, algorithm=alg, refine=False, slots=SLOTS, slots3=SLOTS3)
    n1, _ = gpumc.plan_tiles(p, model=model, algorithm=alg, refine=True, slots=SLOTS, slots3=SLOTS3)
    slots = SLOTS3 if (len(shape) == 3 and (model == "ising" or (model == "potts" and kw.get("q", 3) <= 4
                                                                  and alg is None))) else SLOTS
    assert n1 >= n0
    sites = int(np.prod(shape))
    # split until half a wave, unless the tiles reached their minimum size
    assert n1 >= slots // 2 or sites // n1 <= 2048, (n0, n1)


@pytest.mark.parametrize("model,shape,n_rep,kw", [
    ("ising", (8192, 8192), 3, {}),          # the 2D Ising headline (resident kernel)
    ("ising", (512, 512), 64, {}),           # PT ladders
    ("ising", (128, 128, 128), 32, {}),
    ("o3", (64, 64, 64), 32, {}),            # the O(3) part of the uneven mix
    ("potts", (2048, 2048), 16, dict(q=3)),
])
def test_full_launches_keep_their_plans(gpumc, model, shape, n_rep, kw):
    p = _params(shape, beta=0.5, **kw)
    assert gpumc.plan_tiles(p, model=model, n_replicas=n_rep, refine=True, slots=SLOTS, slots3=SLOTS3) == \
        gpumc.plan_tiles(p, model=model, n_replicas=n_rep, refine=False, slots=SLOTS, slots3=SLOTS3)


@pytest.mark.parametrize("model,shape,alg", [("ising", (64, 64), None), ("ising", (32, 32, 32), "swendsen_wang"),
                                             ("potts", (48, 48), "wolff")])
def test_2d_ising_and_cluster_plans_are_never_split(gpumc, model, shape, alg):
    p = _params(shape, beta=0.3, q=3)
    assert gpumc.plan_tiles(p, model=model, algorithm=alg, refine=True) == \
        gpumc.plan_tiles(p, model=model, algorithm=alg, refine=False)


def test_plan_tiles_validates(gpumc):
    with pytest.raises(gpumc.InvalidConfig):
        gpumc.plan_tiles(_params((7, 8)), model="ising")
    with pytest.raises(gpumc.InvalidConfig):
        gpumc.plan_tiles(_params((8, 8)), model="ising", slots=0)


# ---------------------------------------------------------------------------
# device: identical results with and without refinement
# ---------------------------------------------------------------------------
DEVICE = [
    ("o3", (64, 16, 32), dict(beta=0.7), None, None),       # march -> plain, z split first
    ("o3", (32, 32, 32), dict(beta=0.7), "heat_bath", None),
    ("o3", (16, 8, 12), dict(beta=0.9), None, "opss"),
    ("o3", (64, 32), dict(beta=0.9), None, None),            # 2D: row bands
    ("ising", (64, 32, 48), dict(beta=0.22), None, None),    # whole planes -> row bands with halos
    ("ising", (32, 32, 32), dict(beta=0.22), "heat_bath", None),
    ("potts", (320, 200), dict(beta=1.0, q=3), None, None),  # bit-sliced Potts
    ("potts", (32, 24, 40), dict(beta=0.55, q=4), None, None),
    ("potts", (200, 120), dict(beta=1.2, q=6), None, None),  # int8 Potts
    ("potts", (24, 32, 16), dict(beta=0.6, q=5), "heat_bath", None),
]


@pytest.mark.gpu
@pytest.mark.parametrize("model,shape,kw,alg,prop", DEVICE)
def test_refined_tiles_give_identical_results(gpumc, model, shape, kw, alg, prop):
    from scamper_b200 import _lib
    runs = []
    for refine in (False, True):
        mc = gpumc.ClassicalMC.from_params(_params(shape, **kw), 515, model=model, n_replicas=2,
                                           algorithm=alg, o3_proposal=prop, record_capacity=64)
        mc.set_tile_refinement(refine)
        tiles = mc.tile_count()
        mc.sweep(7)  # thermalization (cone / OPSS adaptation)
        mc.on_phase_start(_lib.PHASE_MEASUREMENT)
        mc.sweep(13)
        recs = [(r["sweep"], r["replica"], r["energy"], r["magnetization"]) for r in mc.observables()]
        runs.append((np.stack([mc.spins(r) for r in range(2)]), mc.energy(), recs, tiles))
        mc.close()
    (s0, e0, r0, t0), (s1, e1, r1, t1) = runs
    assert t1 > t0
    np.testing.assert_array_equal(s0, s1)
    if model == "o3":  # fp64 energy cache summed by atomics in launch order
        np.testing.assert_allclose(e0, e1, rtol=1e-12)
        assert [r[:2] for r in r0] == [r[:2] for r in r1]
        np.testing.assert_allclose([r[2:] for r in r0], [r[2:] for r in r1], rtol=1e-12)
    else:
        np.testing.assert_array_equal(e0, e1)
        assert r0 == r1
    assert len(r0) == 26


@pytest.mark.gpu
def test_batched_engine_with_and_without_refinement(gpumc):
    specs = [("o3", (32, 32, 32), dict(beta=0.7)), ("o3", (16, 16, 16), dict(beta=0.9)),
             ("ising", (48, 48, 48), dict(beta=0.22)), ("potts", (300, 260), dict(q=3, beta=1.0)),
             ("potts", (24, 24, 24), dict(q=6, beta=0.6))]
    out = []
    for refine in (False, True):
        eng = gpumc.Engine()
        eng.set_tile_refinement(refine)
        sims = [gpumc.ClassicalMC.from_params(_params(shape, **kw), 900 + i, model=model, engine=eng)
                for i, (model, shape, kw) in enumerate(specs)]
        eng.sweep(25)
        out.append([(m.spins(), m.energy()) for m in sims])
        for m in sims:
            m.close()
        eng.close()
    for (model, _, _), (sa, ea), (sb, eb) in zip(specs, out[0], out[1]):
        np.testing.assert_array_equal(sa, sb)
        if model == "o3":
            np.testing.assert_allclose(ea, eb, rtol=1e-12)
        else:
            np.testing.assert_array_equal(ea, eb)

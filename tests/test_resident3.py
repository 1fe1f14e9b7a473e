"""Resident (temporally blocked) sweeps of cubic Ising lattices.

A cooperative launch keeps whole-plane slabs of every lattice in shared
memory for up to 64 sweeps, exchanging two boundary planes with the slabs
above and below through a grid barrier per sweep, and runs the sweep
epilogue (records, energies, PT exchanges) on the device between sweeps.
It must give exactly the spins, energies, labels and records of the
per-sweep streaming kernel, for Metropolis and the heat bath."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("alg", [None, "heat_bath"])
@pytest.mark.parametrize("shape,n_rep,pt", [((32, 32, 32), 4, 5), ((64, 64, 40), 2, 0), ((128, 128, 128), 8, 10),
                                            ((130, 6, 12), 3, 3)])
def test_resident3_equals_streaming(gpumc, shape, n_rep, pt, alg):
    from scamper_b200 import _lib
    betas = gpumc.geometric_ladder_betas(3.5, 5.5, n_rep)
    out = []
    for blocking in (True, False):
        mc = gpumc.ClassicalMC.from_params({"lattice_type": "cubic", "Lx": shape[0], "Ly": shape[1], "Lz": shape[2]},
                                           23, n_replicas=n_rep, betas=betas, algorithm=alg, record_capacity=128)
        mc.set_tile_refinement(False)  # whole-plane slabs
        mc.set_temporal_blocking(blocking)
        if pt:
            mc.pt_configure(pt)
        mc.on_phase_start(_lib.PHASE_MEASUREMENT)
        n0 = mc.launch_count()
        mc.sweep(70)
        launches = mc.launch_count() - n0
        out.append(([mc.spins(r).copy() for r in range(n_rep)], mc.energy(), mc.pt_labels(),
                    mc.observable_arrays(), launches, mc.recompute_energy()))
        mc.close()
    res, stream = out
    for a, b in zip(res[0], stream[0]):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(res[1], stream[1])
    np.testing.assert_array_equal(res[1], res[5])  # cache = exact recomputation
    np.testing.assert_array_equal(res[2], stream[2])
    for k in ("energy", "magnetization", "acceptance", "temp_index"):
        np.testing.assert_array_equal(res[3][k], stream[3][k])
    assert res[4] == 2, "expected two resident launches (64 + 6 sweeps)"
    assert stream[4] == 70


def test_resident3_matches_oracle(gpumc, oracle):
    """The resident slabs against the oracle's replay for a lattice with a
    ragged last slab."""
    shape, seed, beta = (64, 16, 22), 5, 0.22
    mc = gpumc.ClassicalMC.from_params({"lattice_type": "cubic", "Lx": 64, "Ly": 16, "Lz": 22, "beta": beta}, seed,
                                       n_replicas=3, betas=[beta])
    mc.set_tile_refinement(False)
    ref = [oracle.Lattice(oracle.ISING, shape, beta=beta, seed=seed, replica=r) for r in range(3)]
    mc.sweep(9)
    for r in range(3):
        for _ in range(9):
            ref[r].sweep()
        np.testing.assert_array_equal(mc.spins(r).ravel(), ref[r].state())
        assert mc.energy()[r] == ref[r].cached_energy()
    mc.close()

"""The allocation-free energy entry point against the allocating one.

gpumc_energy_int8_noalloc exists for callers that must not allocate device
memory (memory owned by another allocator under a fixed budget, or loops that
cannot absorb cudaFree's device-wide synchronization).  It must return exactly
what gpumc_recompute_energy returns for the same lattices, on consecutive
calls that reuse its fixed scratch array.  This file is collected last so a
failure here leaves every other test already run.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(gpumc, model, dims, shape, dev_spins, n_lattices, dev_out, stream):
    lz = shape[2] if dims == 3 else 1
    return gpumc._lib.load().gpumc_energy_int8_noalloc(
        model, dims, shape[0], shape[1], lz, ctypes.c_void_p(dev_spins), n_lattices,
        ctypes.c_void_p(dev_out), ctypes.c_void_p(stream))


@pytest.mark.parametrize("model,shape,q", [
    ("ising", (64, 34), 2),
    ("potts", (34, 18), 3),
    ("ising", (16, 12, 10), 2),
    ("potts", (8, 6, 10), 4),
])
def test_noalloc_energy_matches_allocating_entry_point(gpumc, model, shape, q):
    import torch
    from scamper_b200 import _lib
    dims = len(shape)
    params = {"lattice_type": "square" if dims == 2 else "cubic", "Lx": shape[0], "Ly": shape[1],
              "beta": 0.4, "q": q}
    if dims == 3:
        params["Lz"] = shape[2]
    n_rep = 3
    mc = gpumc.ClassicalMC.from_params(params, 13, model=model, n_replicas=n_rep)
    mc.sweep(7)
    expect = mc.recompute_energy()  # allocating path: J * integer energy, J = 1
    host = np.concatenate([mc.spins(r).ravel() for r in range(n_rep)])
    dev = torch.from_numpy(host).to("cuda")
    out = torch.zeros(n_rep, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    mid = _lib.ISING if model == "ising" else _lib.POTTS
    for call in range(2):  # consecutive calls reuse (and must not depend on) the scratch contents
        out.zero_()
        rc = _noalloc(gpumc, mid, dims, shape, dev.data_ptr(), n_rep, out.data_ptr(), stream)
        assert rc == 0, _lib.last_error()
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out.cpu().numpy().astype(np.float64), expect, err_msg=f"call {call}")
    mc.close()


def _edge_list_energy(spins, shape, potts):
    """Energy in units of J from the reference's periodic hypercubic edge list
    (CMC.rs/src/lattice/graph.rs:417-451): one +1 bond per axis and site, no
    bond along an axis of extent 1."""
    from scamper_b200.snapshot import lattice_topology
    _, _, _, src, dst, kinds = lattice_topology(shape)
    keep = np.array([shape[k] > 1 for k in kinds], dtype=bool) if len(kinds) else np.zeros(0, bool)
    a, b = spins[src[keep]].astype(np.int64), spins[dst[keep]].astype(np.int64)
    return -int((a == b).sum()) if potts else -int((a * b).sum())


@pytest.mark.parametrize("model,shape,q", [
    ("ising", (5, 3), 2),
    ("potts", (2, 6), 3),
    ("ising", (3, 3, 5), 2),
    ("ising", (7, 1), 2),
    ("potts", (1, 1), 4),
    ("ising", (4, 1, 3), 2),
    ("potts", (1, 9, 2), 5),
    ("ising", (2, 2, 2), 2),
])
def test_noalloc_energy_small_and_odd_extents_match_the_edge_list(gpumc, model, shape, q):
    """Extents the allocating path does not accept (odd, 1, 2) against the
    reference builder's edge list: an axis of extent 1 has no bond, extent 2
    has the builder's two parallel bonds."""
    import torch
    from scamper_b200 import _lib
    rng = np.random.default_rng(sum(shape) * 7 + q)
    n_rep = 3
    n = int(np.prod(shape))
    if model == "ising":
        host = rng.choice(np.array([-1, 1], dtype=np.int8), size=(n_rep, n))
    else:
        host = rng.integers(0, q, size=(n_rep, n), dtype=np.int8)
    expect = [_edge_list_energy(host[r], shape, model == "potts") for r in range(n_rep)]
    dev = torch.from_numpy(host.ravel().copy()).to("cuda")
    out = torch.zeros(n_rep, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    mid = _lib.ISING if model == "ising" else _lib.POTTS
    for call in range(2):
        out.fill_(12345)
        rc = _noalloc(gpumc, mid, len(shape), shape, dev.data_ptr(), n_rep, out.data_ptr(), stream)
        assert rc == 0, _lib.last_error()
        torch.cuda.synchronize()
        assert out.cpu().numpy().tolist() == expect, f"call {call}"


def test_noalloc_rejects_requests_beyond_its_scratch(gpumc):
    import torch
    from scamper_b200 import _lib
    dev = torch.zeros(65 * 16, dtype=torch.int8, device="cuda")
    out = torch.zeros(65, dtype=torch.int64, device="cuda")
    rc = _noalloc(gpumc, _lib.ISING, 2, (4, 4), dev.data_ptr(), 65, out.data_ptr(), 0)
    assert rc == _lib.EINVAL
    assert "64" in _lib.last_error()

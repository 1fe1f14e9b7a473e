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


def test_noalloc_rejects_requests_beyond_its_scratch(gpumc):
    import torch
    from scamper_b200 import _lib
    dev = torch.zeros(65 * 16, dtype=torch.int8, device="cuda")
    out = torch.zeros(65, dtype=torch.int64, device="cuda")
    rc = _noalloc(gpumc, _lib.ISING, 2, (4, 4), dev.data_ptr(), 65, out.data_ptr(), 0)
    assert rc == _lib.EINVAL
    assert "64" in _lib.last_error()

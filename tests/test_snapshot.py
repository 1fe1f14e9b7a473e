"""Snapshots in the reference's cmc-rs-snapshot-v2 format.

CPU: the lattice topology written into a snapshot is the reference's
periodic hypercubic CSR (CMC.rs/src/lattice/graph.rs:131-185, :417-451):
edge counts 2N / 3N (graph.rs:549-561), 2d incidences per site in edge order.
GPU: the reference's checkpoint tests (CMC.rs/tests/integration/
checkpoint.rs:28-193) restated for device handles: a run split by save /
restore into a fresh handle ends bit-identical to the continuous run, unknown
formats, bad edge kinds, topology mismatches and invalid spins are rejected
with CheckpointCorrupted (leaving the state untouched), and the energy is
recomputed on load.
"""
import json

import numpy as np
import pytest


def _params(shape, **kw):
    p = {"lattice_type": "square" if len(shape) == 2 else "cubic", "Lx": shape[0], "Ly": shape[1]}
    if len(shape) == 3:
        p["Lz"] = shape[2]
    p.update(kw)
    return p


@pytest.mark.parametrize("shape", [(4, 4), (6, 10), (4, 4, 4), (6, 8, 10)])
def test_topology_is_the_reference_periodic_csr(shape):
    from scamper_b200.snapshot import lattice_topology
    offsets, neighbors, edge_ids, src, dst, kinds = lattice_topology(shape)
    n, d = int(np.prod(shape)), len(shape)
    assert len(src) == d * n  # graph.rs:549-561: 2N bonds (square), 3N (cubic)
    assert np.all(np.diff(offsets) == 2 * d)
    strides = np.cumprod([1] + list(shape[:-1]))
    for e in range(len(src)):  # edge e = site e // d, axis e % d, +1 neighbour
        s, a = e // d, e % d
        c = (s // strides[a]) % shape[a]
        assert src[e] == s and kinds[e] == a
        assert dst[e] == s + (((c + 1) % shape[a]) - c) * strides[a]
    for s in range(n):  # incidences of a site: its edges in edge order
        inc = edge_ids[offsets[s]:offsets[s + 1]]
        assert np.all(np.diff(inc) > 0)
        for k, e in zip(range(offsets[s], offsets[s + 1]), inc):
            assert s in (src[e], dst[e])
            assert neighbors[k] == (dst[e] if src[e] == s else src[e])
    if shape == (4, 4):
        assert neighbors[:4].tolist() == [1, 4, 3, 12] and edge_ids[:4].tolist() == [0, 1, 6, 25]


@pytest.mark.gpu
@pytest.mark.parametrize("model,shape,kw,n1,n2", [
    ("ising", (16, 16), dict(beta=0.5), 200, 200),
    ("ising", (4, 4), dict(beta=0.44), 400, 600),
    ("ising", (64, 128), dict(beta=0.4407), 70, 90),
    ("potts", (34, 18), dict(beta=1.0, q=3), 121, 80),
    ("potts", (6, 8, 10), dict(beta=0.6, q=4), 50, 50),
    ("o3", (8, 6, 10), dict(beta=0.7), 60, 40),
])
def test_split_run_through_snapshot_is_identical(gpumc, model, shape, kw, n1, n2):
    """checkpoint.rs:28-78 and :150-193: continuous run vs save -> restore into
    a fresh handle -> continue, through JSON text."""
    cont = gpumc.ClassicalMC.from_params(_params(shape, **kw), 42, model=model)
    cont.sweep(n1 + n2)
    split = gpumc.ClassicalMC.from_params(_params(shape, **kw), 42, model=model)
    split.sweep(n1)
    text = json.dumps(split.save_snapshot())
    split.close()
    fresh = gpumc.ClassicalMC.from_params(_params(shape, **kw), 42, model=model)
    fresh.load_snapshot(json.loads(text))
    assert fresh.sweep_count() == n1
    fresh.sweep(n2)
    np.testing.assert_array_equal(fresh.spins(), cont.spins())
    if model == "o3":
        assert fresh.energy()[0] == pytest.approx(cont.energy()[0], rel=1e-12, abs=1e-9)
        assert fresh.cone_omc() == cont.cone_omc()
    else:
        assert fresh.energy()[0] == cont.energy()[0]
    fresh.close()
    cont.close()


@pytest.mark.gpu
def test_snapshot_rejections_leave_state_untouched(gpumc):
    """checkpoint.rs:80-130: unknown format, bad edge kind, topology mismatch;
    plus invalid and non-finite spins and a wrong length."""
    mc = gpumc.ClassicalMC.from_params(_params((8, 8), beta=0.5), 7)
    mc.sweep(5)
    snap = mc.save_snapshot()
    assert snap["format"] == "cmc-rs-snapshot-v2" and snap["spin_dim"] == 1 and snap["n_edges"] == 128
    before, e_before = mc.spins().copy(), mc.energy()[0]
    bad_cases = []
    b = dict(snap, format="cmc-rs-snapshot-v1")
    bad_cases.append(b)
    b = json.loads(json.dumps(snap))
    b["edges"][0]["kind"] = "invalid_kind"
    bad_cases.append(b)
    bad_cases.append(dict(snap, n_sites=999))
    b = json.loads(json.dumps(snap))
    b["neighbors"][5] += 1
    bad_cases.append(b)
    b = json.loads(json.dumps(snap))
    b["spins"][3] = 0.5
    bad_cases.append(b)
    b = json.loads(json.dumps(snap))
    b["spins"][3] = float("nan")
    bad_cases.append(b)
    bad_cases.append(dict(snap, spins=snap["spins"][:-1]))
    bad_cases.append(dict(snap, beta=None))
    for bad in bad_cases:
        with pytest.raises(gpumc.CheckpointCorrupted):
            mc.load_snapshot(bad)
    np.testing.assert_array_equal(mc.spins(), before)
    assert mc.energy()[0] == e_before
    mc.close()


@pytest.mark.gpu
def test_snapshot_load_recomputes_energy_and_restores_beta(gpumc):
    """checkpoint.rs:132-148: the energy comes from the loaded spins, never
    from the snapshot; beta is the snapshot's."""
    a = gpumc.ClassicalMC.from_params(_params((16, 16), beta=0.3), 1)
    a.sweep(30)
    snap = a.save_snapshot()
    b = gpumc.ClassicalMC.from_params(_params((16, 16), beta=0.9), 2)
    b.sweep(11)
    b.load_snapshot(snap)
    np.testing.assert_array_equal(b.spins(), a.spins())
    assert b.energy()[0] == a.energy()[0] == b.recompute_energy()[0]
    assert b.log_weight_ratio("beta", 0.5) == pytest.approx((0.3 - 0.5) * a.energy()[0])
    a.close()
    b.close()


@pytest.mark.gpu
@pytest.mark.parametrize("model,shape,n1,n2", [
    ("ising", (16, 8), 25, 23),
    ("ising", (64, 64), 37, 40),
    ("potts", (8, 6, 6), 22, 20),
    ("o3", (6, 4, 4), 13, 17),
])
def test_parallel_tempering_resumes_mid_run(gpumc, model, shape, n1, n2):
    """A PT ensemble stopped after n1 sweeps and restored into a fresh handle
    (spins, sweep count, labels) continues exactly as the uninterrupted run:
    each exchange's pairing and random stream follow from the sweep count
    (exchange_step = sweep_count / interval, Carlo.rs/src/parallel_tempering.rs:
    372-373), not from how many exchanges the handle itself has made."""
    from scamper_b200 import _lib
    R, interval = 8, 3
    betas = gpumc.geometric_ladder_betas(1.5, 3.5, R) if model != "o3" else \
        gpumc.geometric_ladder_betas(0.9, 2.0, R)
    kw = dict(q=3) if model == "potts" else {}

    def make():
        mc = gpumc.ClassicalMC.from_params(_params(shape, **kw), 77, model=model, n_replicas=R, betas=betas)
        mc.on_phase_start(_lib.PHASE_MEASUREMENT)  # no O(3) cone adaptation
        mc.pt_configure(interval)
        return mc

    cont = make()
    cont.sweep(n1 + n2)
    split = make()
    split.sweep(n1)
    spins = [split.spins(r).copy() for r in range(R)]
    labels = split.pt_labels()
    assert split.pt_stats()[0] == n1 // interval
    split.close()
    fresh = make()
    fresh.set_sweep_count(n1)
    fresh.set_pt_labels(labels)
    for r in range(R):
        fresh.set_spins(r, spins[r])
    assert fresh.pt_stats()[0] == n1 // interval
    fresh.sweep(n2)
    np.testing.assert_array_equal(fresh.pt_labels(), cont.pt_labels())
    for r in range(R):
        np.testing.assert_array_equal(fresh.spins(r), cont.spins(r))
    assert fresh.pt_stats()[0] == cont.pt_stats()[0] == (n1 + n2) // interval
    fresh.close()
    cont.close()


@pytest.mark.gpu
def test_pt_set_labels_rejects_non_permutations(gpumc):
    mc = gpumc.ClassicalMC.from_params(_params((8, 8)), 3, n_replicas=4,
                                       betas=gpumc.geometric_ladder_betas(1.5, 3.5, 4))
    mc.pt_configure(2)
    for bad in ([0, 1, 2, 2], [0, 1, 2, 4], [-1, 0, 1, 2]):
        with pytest.raises(gpumc.InvalidConfig):
            mc.set_pt_labels(bad)
    mc.set_pt_labels([3, 2, 1, 0])
    assert mc.pt_labels().tolist() == [3, 2, 1, 0]
    mc.close()

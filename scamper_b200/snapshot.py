"""State snapshots in the reference's `cmc-rs-snapshot-v2` JSON format.

ClassicalMC::save_snapshot / load_snapshot (CMC.rs/src/classical_mc.rs:63-165)
write and verify: the format tag, the spins (flat f64, spin_dim values per
site), beta, spin_dim, n_sites, n_edges and the lattice topology (CSR
offsets / neighbors / edge_ids and the physical edge list with source,
target, bond kind label and weight).  The lattice is the reference's
periodic hypercubic builder (build_hypercubic, CMC.rs/src/lattice/
graph.rs:417-451): for every site in index order and every axis, one bond to
the +1 neighbour (kinds square_x / square_y or cubic_x / cubic_y / cubic_z,
weight 1), and CSR incidences in edge order for each endpoint
(CsrLattice::try_from_edges, graph.rs:131-185).

Loading follows the reference's checks and error kind: unknown format, a
missing or non-numeric or non-finite spin array, a length mismatch, an invalid
configuration, or any topology field that disagrees raises
CheckpointCorrupted; beta is restored and the cached energy recomputed, not
read.  Snapshots written here carry one extra object, "gpumc_state" (ignored
by the reference, which reads keys by name): the sweep counter (the position
of the engine's counter-based random stream, so a resumed run continues the
same trajectory), the replica's temperature label and the O(3) cone parameter
as the exact float the device holds.

O(3) spins are the engine's float32 values widened exactly to f64, so their
norms deviate from 1 by float32 rounding (~1e-7); this engine accepts them
back (|n^2 - 1| <= 1e-5), while the reference's f64 check (1e-10 per
component) would not: `save_snapshot(..., renormalize=True)` writes f64
vectors of unit norm for a reference reader instead (not bit-exact on the
way back).
"""
import numpy as np

from . import _lib

FORMAT = "cmc-rs-snapshot-v2"
_KINDS = {2: ["square_x", "square_y"], 3: ["cubic_x", "cubic_y", "cubic_z"]}


class CheckpointCorrupted(_lib.GpumcError):
    """The reference's CarloError::CheckpointCorrupted { detail }."""

    def __init__(self, field, reason):
        super().__init__(_lib.ESTATE, f"{field}: {reason}")


def lattice_topology(shape):
    """CSR topology of the periodic square / cubic lattice as the reference
    builds it.  Returns (offsets, neighbors, edge_ids, sources, targets,
    kinds) with kinds as axis indices."""
    dims = list(shape)
    n = int(np.prod(dims))
    strides = np.cumprod([1] + dims[:-1])
    site = np.arange(n, dtype=np.int64)
    src, dst, kind = [], [], []
    coords = [(site // strides[a]) % dims[a] for a in range(len(dims))]
    for a in range(len(dims)):
        nxt = np.where(coords[a] + 1 < dims[a], coords[a] + 1, 0)
        src.append(site)
        dst.append(site - coords[a] * strides[a] + nxt * strides[a])
        kind.append(np.full(n, a, dtype=np.int64))
    # edges in the builder's order: site-major, axis-minor
    sources = np.stack(src, axis=1).ravel()
    targets = np.stack(dst, axis=1).ravel()
    kinds = np.stack(kind, axis=1).ravel()
    m = len(sources)
    eid = np.arange(m, dtype=np.int64)
    inc_site = np.empty(2 * m, dtype=np.int64)
    inc_nb = np.empty(2 * m, dtype=np.int64)
    inc_site[0::2], inc_site[1::2] = sources, targets
    inc_nb[0::2], inc_nb[1::2] = targets, sources
    inc_eid = np.repeat(eid, 2)
    order = np.argsort(inc_site, kind="stable")  # per site, in edge order
    offsets = np.concatenate([[0], np.cumsum(np.bincount(inc_site, minlength=n))])
    return offsets, inc_nb[order], inc_eid[order], sources, targets, kinds


def save_snapshot(mc, replica=0, renormalize=False):
    """Snapshot of one replica of a ClassicalMC handle (a JSON-ready dict)."""
    dims = len(mc.shape)
    spin_dim = 3 if mc.model == _lib.O3 else 1
    s = mc.spins(replica)
    if mc.model == _lib.O3:
        v = s.reshape(-1, 3).astype(np.float64)
        if renormalize:
            v = v / np.sqrt((v * v).sum(axis=1))[:, None]
        spins = v.ravel()
    else:
        spins = s.ravel().astype(np.float64)
    labels = mc.pt_labels()
    beta = float(mc.betas[labels[replica]])
    offsets, neighbors, edge_ids, sources, targets, kinds = lattice_topology(mc.shape)
    labels_of = _KINDS[dims]
    edges = [{"source": int(a), "target": int(b), "kind": labels_of[k], "weight": 1.0}
             for a, b, k in zip(sources.tolist(), targets.tolist(), kinds.tolist())]
    state = {"sweep": int(mc.sweep_count()), "label": int(labels[replica])}
    if mc.model == _lib.O3:
        state["omc_bits"] = int(np.float32(mc.cone_omc(replica)).view(np.uint32))
    return {
        "format": FORMAT,
        "spins": spins.tolist(),
        "beta": beta,
        "spin_dim": spin_dim,
        "n_sites": int(mc.n_sites),
        "n_edges": len(edges),
        "offsets": offsets.tolist(),
        "neighbors": neighbors.tolist(),
        "edge_ids": edge_ids.tolist(),
        "edges": edges,
        "gpumc_state": state,
    }


def _check_usize_array(snapshot, name, expected):
    values = snapshot.get(name)
    if values is None:
        return  # older snapshots carried no topology
    if not isinstance(values, list) or len(values) != len(expected):
        raise CheckpointCorrupted(f"snapshot.{name}", "topology length mismatch")
    got = np.array([v if isinstance(v, int) and not isinstance(v, bool) else -1 for v in values],
                   dtype=np.int64)
    bad = np.nonzero(got != expected)[0]
    if len(bad):
        raise CheckpointCorrupted(f"snapshot.{name}[{bad[0]}]", "topology mismatch")


def load_snapshot(mc, snapshot, replica=0):
    """Restores one replica from a snapshot, verifying it against the handle's
    model and lattice; the cached energy is recomputed on the device."""
    fmt = snapshot.get("format") if isinstance(snapshot, dict) else None
    if fmt != FORMAT:
        raise CheckpointCorrupted("snapshot.format",
                                  f"unknown snapshot format: expected '{FORMAT}', got '{fmt or ''}'")
    values = snapshot.get("spins")
    if not isinstance(values, list):
        raise CheckpointCorrupted("snapshot.spins", "missing or invalid array")
    if any(isinstance(v, bool) or not isinstance(v, (int, float)) for v in values):
        raise CheckpointCorrupted("snapshot.spins", "contains a non-number")
    spins = np.array(values, dtype=np.float64)
    if not np.all(np.isfinite(spins)):
        raise CheckpointCorrupted("snapshot.spins", "contains a non-finite value")
    spin_dim = 3 if mc.model == _lib.O3 else 1
    if len(spins) != mc.n_sites * spin_dim:
        raise CheckpointCorrupted("snapshot.spins", f"length mismatch: expected {mc.n_sites * spin_dim}, "
                                                    f"got {len(spins)}")
    _validate_configuration(mc, spins)
    if snapshot.get("n_sites") is not None and snapshot["n_sites"] != mc.n_sites:
        raise CheckpointCorrupted("snapshot.n_sites", "topology mismatch")
    if snapshot.get("spin_dim") is not None and snapshot["spin_dim"] != spin_dim:
        raise CheckpointCorrupted("snapshot.spin_dim", "model mismatch")
    offsets, neighbors, edge_ids, sources, targets, kinds = lattice_topology(mc.shape)
    if snapshot.get("n_edges") is not None and snapshot["n_edges"] != len(sources):
        raise CheckpointCorrupted("snapshot.n_edges", "topology mismatch")
    _check_usize_array(snapshot, "offsets", offsets)
    _check_usize_array(snapshot, "neighbors", neighbors)
    _check_usize_array(snapshot, "edge_ids", edge_ids)
    edges = snapshot.get("edges")
    if edges is not None:
        if not isinstance(edges, list) or len(edges) != len(sources):
            raise CheckpointCorrupted("snapshot.edges", "topology length mismatch")
        labels_of = _KINDS[len(mc.shape)]
        for i, e in enumerate(edges):
            ok = (isinstance(e, dict) and e.get("source") == sources[i] and e.get("target") == targets[i]
                  and e.get("kind") == labels_of[kinds[i]] and isinstance(e.get("weight"), (int, float))
                  and float(e["weight"]) == 1.0)
            if not ok:
                raise CheckpointCorrupted(f"snapshot.edges[{i}]", "physical edge mismatch")
    beta = snapshot.get("beta")
    if isinstance(beta, bool) or not isinstance(beta, (int, float)) or not np.isfinite(beta) or beta < 0:
        raise CheckpointCorrupted("snapshot.beta", "missing or invalid")
    state = snapshot.get("gpumc_state") or {}
    if "sweep" in state:
        mc.set_sweep_count(int(state["sweep"]))
    mc.change_parameter("beta", float(beta), replica=replica)
    if mc.model == _lib.O3:
        mc.set_spins(replica, spins.astype(np.float32).reshape(-1, 3))
        if "omc_bits" in state:
            mc.set_cone_omc(replica, float(np.uint32(state["omc_bits"]).view(np.float32)))
    else:
        mc.set_spins(replica, spins.astype(np.int8))


def _validate_configuration(mc, spins):
    """The reference's validate_configuration / validate_spin rules
    (CMC.rs/src/lattice/models.rs:62-75, :238-252, :454-475), with the O(3)
    norm tolerance of this engine's float32 spins."""
    if mc.model == _lib.ISING:
        bad = np.nonzero((spins != 1.0) & (spins != -1.0))[0]
        reason = "Ising spin must be exactly -1 or +1"
    elif mc.model == _lib.POTTS:
        q = mc.spec.q
        bad = np.nonzero((spins != np.floor(spins)) | (spins < 0) | (spins >= q))[0]
        reason = f"Potts spin must be an integer in [0, {q})"
    else:
        v = spins.reshape(-1, 3)
        bad = np.nonzero(np.abs((v * v).sum(axis=1) - 1.0) > 1e-5)[0]
        reason = "O(N) spin must have unit norm"
    if len(bad):
        raise CheckpointCorrupted("snapshot.spins", f"invalid spin at site {bad[0]}: {reason}")

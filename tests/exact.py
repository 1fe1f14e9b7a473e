"""Exact reference values used by the statistical tests.

Restated from the reference's own test helpers: enumeration moments
(CMC.rs/tests/physics/common.rs:51-85), the row transfer matrix of the 2D
Ising model on an L x L torus (CMC.rs/tests/physics/zscore_extended.rs:60-135,
generalised here to q-state Potts rows), and Onsager's infinite-lattice energy
(zscore_extended.rs:140-171, CMC.rs/tests/exact/onsager.rs:11-58).
"""
import itertools
import math

import numpy as np


def square_bonds(lx, ly):
    """+x and +y periodic bonds of build_square (site = x + lx*y)."""
    b = []
    for y in range(ly):
        for x in range(lx):
            s = x + lx * y
            b.append((s, (x + 1) % lx + lx * y))
            b.append((s, x + lx * ((y + 1) % ly)))
    return np.array(b)


def ising_enumeration(lx, ly, beta, J=1.0):
    """Exact <E>, <E^2>, <m^2>, <|m|>, <m^4> (m = M/N) by enumerating 2^N states."""
    n = lx * ly
    bonds = square_bonds(lx, ly)
    states = ((np.arange(1 << n)[:, None] >> np.arange(n)[None, :]) & 1).astype(np.int8) * 2 - 1
    e = -J * (states[:, bonds[:, 0]] * states[:, bonds[:, 1]]).sum(axis=1).astype(np.float64)
    m = states.sum(axis=1) / n
    w = np.exp(-beta * (e - e.min()))
    z = w.sum()
    return dict(E=(w * e).sum() / z, E2=(w * e * e).sum() / z, M2=(w * m * m).sum() / z,
                M=(w * np.abs(m)).sum() / z, M4=(w * m ** 4).sum() / z)


def potts_transfer_matrix(lx, ly, q, beta, J=1.0):
    """Exact <E> (total) and <order parameter> ingredients of the q-state Potts
    model on an lx x ly torus via the row transfer matrix (q^lx row states).
    Returns <E> and <E^2>."""
    rows = np.array(list(itertools.product(range(q), repeat=lx)), dtype=np.int64)
    h = -(rows == np.roll(rows, -1, axis=1)).sum(axis=1).astype(np.float64)  # in-row bond energy / J
    v = -(rows[:, None, :] == rows[None, :, :]).sum(axis=2).astype(np.float64)  # vertical / J

    def logz(b):
        t = np.exp(-b * J * (v + 0.5 * (h[:, None] + h[None, :])))
        ev = np.linalg.eigvalsh(t) if np.allclose(t, t.T) else np.linalg.eigvals(t).real
        lam = ev.max()
        return ly * math.log(lam) + math.log(np.sum((ev / lam) ** ly))

    eps = 1e-5
    e = -(logz(beta + eps) - logz(beta - eps)) / (2 * eps)
    e2c = (logz(beta + eps) - 2 * logz(beta) + logz(beta - eps)) / eps ** 2  # var(E)
    return dict(E=e, E2=e2c + e * e)


def ising_transfer_matrix_energy(lx, ly, beta, J=1.0):
    return potts_transfer_matrix_ising(lx, ly, beta, J)


def potts_transfer_matrix_ising(lx, ly, beta, J=1.0):
    rows = np.array(list(itertools.product((-1, 1), repeat=lx)), dtype=np.int64)
    h = (rows * np.roll(rows, -1, axis=1)).sum(axis=1).astype(np.float64)
    v = (rows[:, None, :] * rows[None, :, :]).sum(axis=2).astype(np.float64)

    def logz(b):
        t = np.exp(b * J * (v + 0.5 * (h[:, None] + h[None, :])))
        ev = np.linalg.eigvalsh(t)
        lam = np.abs(ev).max()
        return ly * math.log(lam) + math.log(np.sum((ev / lam) ** ly))

    eps = 1e-5
    e = -(logz(beta + eps) - logz(beta - eps)) / (2 * eps)
    var = (logz(beta + eps) - 2 * logz(beta) + logz(beta - eps)) / eps ** 2
    return dict(E=e, E2=var + e * e)


def complete_elliptic_k(m):
    k = math.sqrt(1.0 - m * m)
    a, b = 1.0, k
    for _ in range(60):
        a, b = 0.5 * (a + b), math.sqrt(a * b)
        if abs(a - b) < 1e-16:
            break
    return math.pi / (2.0 * a)


def onsager_energy_per_site(beta, J=1.0):
    k = beta * J
    s2, c2 = math.sinh(2 * k), math.cosh(2 * k)
    coth = c2 / s2
    t2 = math.tanh(2 * k)
    coeff = 2 * t2 * t2 - 1.0
    mod = 2 * s2 / (c2 * c2) if s2 < 1.0 else (c2 * c2) / (2 * s2)
    return -J * coth * (1.0 + (2.0 / math.pi) * coeff * complete_elliptic_k(mod))


BETA_C_2D_ISING = 0.5 * math.log(1.0 + math.sqrt(2.0))


def zscore(mean, stderr, exact):
    return (mean - exact) / stderr if stderr > 0 else float("inf")


def binned(values, nbins=20):
    """Mean and standard error from equal bins of a correlated series."""
    v = np.asarray(values, dtype=np.float64)
    k = len(v) // nbins
    b = v[: k * nbins].reshape(nbins, k).mean(axis=1)
    return b.mean(), b.std(ddof=1) / math.sqrt(nbins)


def kaufman_logz(m, n, beta, J=1.0):
    """ln Z of the 2D Ising model on an m x n torus from Kaufman's exact
    finite-lattice solution (Phys. Rev. 76, 1232 (1949)): Z = 1/2 (2 sinh 2K)^(mn/2)
    (Z1 + Z2 + Z3 + Z4) with products over the gamma_l of the row transfer
    matrix.  Evaluated in log space with signs (Z2, Z4 can be negative)."""
    K = beta * J
    c2, s2 = math.cosh(2 * K), math.sinh(2 * K)
    coth2 = c2 / s2

    def gamma(l):
        if l == 0:
            return 2 * K + math.log(math.tanh(K))
        return math.acosh(c2 * coth2 - math.cos(math.pi * l / n))

    def log_prod(fn, ls):
        lg, sg = 0.0, 1.0
        for l in ls:
            v = fn(m * gamma(l) / 2.0)
            if v == 0.0:
                return float("-inf"), 0.0
            lg += math.log(2.0 * abs(v))
            sg *= 1.0 if v > 0 else -1.0
        return lg, sg

    odd = [2 * r + 1 for r in range(n)]
    even = [2 * r for r in range(n)]
    terms = [log_prod(math.cosh, odd), log_prod(math.sinh, odd), log_prod(math.cosh, even),
             log_prod(math.sinh, even)]
    top = max(t[0] for t in terms)
    s = sum(sg * math.exp(lg - top) for lg, sg in terms)
    return math.log(0.5) + 0.5 * m * n * math.log(2 * s2) + top + math.log(s)


def kaufman_energy(L, beta, J=1.0, eps=1e-5):
    """Exact <E> (total) of the L x L periodic Ising model."""
    return -(kaufman_logz(L, L, beta + eps, J) - kaufman_logz(L, L, beta - eps, J)) / (2 * eps)


def replicas_ok(series, ex, nbins=20):
    """Independent chains against an exact mean: per-chain z (binned stderr)
    below 4, mean z below 2, and the pooled mean within 4 standard errors of
    the spread of the chain means (an unbiased error bar for independent
    chains).  Raises AssertionError otherwise."""
    zs, means = [], []
    for e in series:
        me, se = binned(e, nbins)
        zs.append(zscore(me, se, ex))
        means.append(me)
    means = np.array(means)
    pooled = (means.mean() - ex) / (means.std(ddof=1) / math.sqrt(len(means)))
    assert max(abs(z) for z in zs) < 4.0, zs
    assert abs(np.mean(zs)) < 2.0, zs
    assert abs(pooled) < 4.0, (pooled, zs)

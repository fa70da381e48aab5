"""Seeded synthetic tridiagonal workloads.

The reference ships no benchmark inputs; these generators produce the matrix
families named by the benchmark configurations, with their sizes and value
distributions, from a numpy seed:

* ``uniform(n, seed)``          D_i, E_i i.i.d. uniform(-1, 1)
* ``one_two_one(n)``            D = 2, E = 1; eigenvalues 2 - 2 cos(k pi/(n+1))
* ``glued_wilkinson(nb, bs, glue)``  nb copies of W+ of size bs
                                (D_j = |j - (bs-1)/2|, E = 1) glued by ``glue``
* ``mixed_batch(count, seed)``  the 4096-problem batch: n log-uniform in
                                [32, 4096], 25 % replaced by 1-2-1
* ``large_mixed(n, seed)``      half uniform, half glued W+ (size 401, glue 1e-10)
* ``serve_stream(count, seed)`` request sizes and Poisson arrival times
"""
from __future__ import annotations

import numpy as np


def uniform(n: int, seed: int = 0):
    rng = np.random.default_rng(seed)
    D = rng.uniform(-1.0, 1.0, n)
    E = rng.uniform(-1.0, 1.0, n)
    E[-1] = 0.0
    return D, E


def one_two_one(n: int):
    D = np.full(n, 2.0)
    E = np.ones(n)
    E[-1] = 0.0
    return D, E


def one_two_one_eigs(n: int):
    k = np.arange(1, n + 1)
    return np.sort(2.0 - 2.0 * np.cos(k * np.pi / (n + 1)))


def wilkinson_plus(bs: int):
    """W+ of odd size bs: D_j = |j - (bs-1)/2|, E = 1."""
    h = (bs - 1) // 2
    return np.abs(np.arange(bs) - h).astype(np.float64)


def glued_wilkinson(nb: int, bs: int, glue: float):
    D = np.tile(wilkinson_plus(bs), nb)
    E = np.ones(nb * bs)
    E[bs - 1::bs] = glue
    E[-1] = 0.0
    return D, E


def mixed_batch(count: int = 4096, seed: int = 3, nmin: int = 32, nmax: int = 4096,
                frac_121: float = 0.25):
    """The batched workload: list of (D, E, kind) with n log-uniform in [nmin, nmax]."""
    rng = np.random.default_rng(seed)
    ns = np.rint(np.exp(rng.uniform(np.log(nmin), np.log(nmax), count))).astype(int)
    is121 = rng.random(count) < frac_121
    out = []
    for k in range(count):
        n = int(ns[k])
        if is121[k]:
            D, E = one_two_one(n)
            out.append((D, E, "121"))
        else:
            D = rng.uniform(-1.0, 1.0, n)
            E = rng.uniform(-1.0, 1.0, n)
            E[-1] = 0.0
            out.append((D, E, "uniform"))
    return out


def large_mixed(n: int = 40000, seed: int = 5, bs: int = 401, glue: float = 1e-10):
    """Half uniform(-1,1) rows, half glued W+ blocks of size bs; the last block
    is truncated to fit and the junction off-diagonal is ``glue``."""
    rng = np.random.default_rng(seed)
    h = n // 2
    D = np.empty(n)
    E = np.empty(n)
    D[:h] = rng.uniform(-1.0, 1.0, h)
    E[:h] = rng.uniform(-1.0, 1.0, h)
    E[h - 1] = glue
    rest = n - h
    nb = (rest + bs - 1) // bs
    Dw, Ew = glued_wilkinson(nb, bs, glue)
    D[h:] = Dw[:rest]
    E[h:] = Ew[:rest]
    E[-1] = 0.0
    return D, E


def serve_stream(count: int = 50000, rate: float = 5000.0, seed: int = 11,
                 sizes=(64, 256, 1024, 4096, 16384), probs=(0.4, 0.3, 0.2, 0.08, 0.02)):
    """Request sizes, Poisson arrival times (s) and ranges (alternating A and I)."""
    rng = np.random.default_rng(seed)
    ns = rng.choice(np.asarray(sizes), size=count, p=np.asarray(probs))
    gaps = rng.exponential(1.0 / rate, size=count)
    t = np.cumsum(gaps)
    ranges = np.where(np.arange(count) % 2 == 0, "A", "I")
    return ns, t, ranges, rng


def residual_orth(D, E, W, Z):
    """Scaled residual max|T z - lambda z| / (n eps ||T||) and orthogonality
    max|Z^T Z - I| / (n eps) of eigenpairs (dense check, for moderate n)."""
    n = len(D)
    eps = np.finfo(np.float64).eps
    m = Z.shape[1]
    if m == 0:
        return 0.0, 0.0
    e = np.asarray(E[: n - 1], dtype=np.float64)
    tn = max(np.abs(D).max(), np.abs(e).max() if n > 1 else 0.0)
    if tn == 0.0:
        tn = 1.0
    TZ = D[:, None] * Z
    TZ[:-1] += e[:, None] * Z[1:]
    TZ[1:] += e[:, None] * Z[:-1]
    res = np.abs(TZ - Z * W[None, :]).max() / (n * eps * tn)
    G = Z.T @ Z
    orth = np.abs(G - np.eye(m)).max() / (n * eps)
    return float(res), float(orth)


def residual_orth_torch(D, E, W, Z, device="cuda", chunk=4096):
    """residual_orth on the GPU (torch, fp64) for large problems: the same
    two scaled quantities; Z may be a host array (n x m) or a torch tensor."""
    import torch
    n = len(D)
    eps = np.finfo(np.float64).eps
    Zt = torch.as_tensor(Z, device=device, dtype=torch.float64)
    m = Zt.shape[1]
    if m == 0:
        return 0.0, 0.0
    d = torch.as_tensor(np.asarray(D, dtype=np.float64), device=device)
    e = torch.as_tensor(np.asarray(E[: n - 1], dtype=np.float64), device=device)
    w = torch.as_tensor(np.asarray(W, dtype=np.float64), device=device)
    tn = max(float(d.abs().max()), float(e.abs().max()) if n > 1 else 0.0) or 1.0
    res = 0.0
    for c0 in range(0, m, chunk):
        Zc = Zt[:, c0:c0 + chunk]
        TZ = d[:, None] * Zc
        TZ[:-1] += e[:, None] * Zc[1:]
        TZ[1:] += e[:, None] * Zc[:-1]
        res = max(res, float((TZ - Zc * w[None, c0:c0 + chunk]).abs().max()))
    orth = 0.0
    for c0 in range(0, m, chunk):
        G = Zt[:, c0:c0 + chunk].T @ Zt
        G[:, c0:c0 + chunk] -= torch.eye(G.shape[0], device=device, dtype=torch.float64)
        orth = max(orth, float(G.abs().max()))
    return res / (n * eps * tn), orth / (n * eps)

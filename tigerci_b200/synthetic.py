"""Seeded synthetic MO Hamiltonians with the shapes of the benchmark configs.

The kernel-scale configuration is specified as: Cholesky vectors
L^J_pq ~ N(0,1) * exp(-0.05 |p-q|) * exp(-J/400), symmetric in pq; h_pq
symmetric with its diagonal sorted ascending in [-20, 2] and off-diagonal
N(0, 0.05).  `scale` shrinks L for small test systems so that the
correlation problem stays well conditioned.
"""
from __future__ import annotations

import numpy as np


def synthetic_operator(norb: int, nchol: int, seed: int = 1234, scale: float = 1.0, diag_range=(-20.0, 2.0),
                       offdiag_sigma: float = 0.05):
    rng = np.random.default_rng(seed)
    npair = norb * (norb + 1) // 2
    p = np.repeat(np.arange(norb), np.arange(1, norb + 1))
    q = np.concatenate([np.arange(i + 1) for i in range(norb)])
    chol = rng.standard_normal((npair, nchol))
    chol *= (scale * np.exp(-0.05 * np.abs(p - q)))[:, None]
    chol *= np.exp(-np.arange(nchol) / 400.0)[None, :]
    h = rng.normal(0.0, offdiag_sigma, size=(norb, norb))
    h = 0.5 * (h + h.T)
    d = np.sort(rng.uniform(diag_range[0], diag_range[1], size=norb))
    h[np.arange(norb), np.arange(norb)] = d
    return np.ascontiguousarray(h), np.ascontiguousarray(chol)


def random_civec(n: int, seed: int = 7):
    rng = np.random.default_rng(seed)
    c = rng.standard_normal(n)
    return c / np.linalg.norm(c)

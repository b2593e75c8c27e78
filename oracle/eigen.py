"""Chebyshev-filtered subspace iteration and Fermi-Dirac occupancies (oracle).

The reference runs one pass of DFT-FE's ``kohnShamEigenSpaceCompute`` per loop
iteration of ``solveEigen`` (InverseDFTSolverFunction.cpp:1392-1474).  DFT-FE's
solver is not in the reference tree; this is the published Zhou-Saad
Chebyshev-filtered subspace iteration it implements:

  filter (degree m, bounds [a, b], scaling at a0) -> Cholesky orthonormalisation
  -> Rayleigh-Ritz on the filtered block -> residual norms |Ht x_i - eps_i x_i|.

The upper bound b comes from a k-step Lanczos run started from a fixed
deterministic vector; a is the largest Ritz value of the current block and a0
the smallest.  The GPU library uses the same rules and the same start vector.
"""
from __future__ import annotations

import math

import numpy as np
import scipy.linalg as sla

C_KB = 3.166811429e-06


def hash_uniform(i, salt: int) -> np.ndarray:
    """Exactly reproducible pseudo-random values in [-0.5, 0.5).

    ((i * 2654435761 + salt * 40503) mod 2^32) / 2^32 - 0.5 in 64-bit integers,
    so every implementation produces the same doubles bit for bit."""
    i = np.asarray(i, dtype=np.uint64)
    h = (i * np.uint64(2654435761) + np.uint64(salt) * np.uint64(40503)) & np.uint64(0xFFFFFFFF)
    h ^= h >> np.uint64(15)
    h = (h * np.uint64(2246822519)) & np.uint64(0xFFFFFFFF)
    h ^= h >> np.uint64(13)
    return h.astype(np.float64) / 4294967296.0 - 0.5


def lanczos_start(n: int, free: np.ndarray) -> np.ndarray:
    """Deterministic Lanczos start vector (hash_uniform, salt 7) on free rows."""
    v = hash_uniform(np.arange(n), 7)
    v[~free] = 0.0
    return v / np.linalg.norm(v)


def lanczos_bounds(hx, v0: np.ndarray, steps: int):
    """k-step Lanczos: returns (smallest Ritz value, largest Ritz value + |beta_k|)."""
    alphas, betas = [], []
    v_prev = np.zeros_like(v0)
    v = v0.copy()
    beta = 0.0
    for _ in range(steps):
        w = hx(v)
        a = float(np.dot(v, w))
        w = w - a * v - beta * v_prev
        beta = float(np.linalg.norm(w))
        alphas.append(a)
        betas.append(beta)
        if beta == 0.0:
            break
        v_prev, v = v, w / beta
    T = np.diag(alphas) + np.diag(betas[:-1], 1) + np.diag(betas[:-1], -1)
    ev = np.linalg.eigvalsh(T)
    return float(ev[0]), float(ev[-1] + abs(betas[-1]))


def chebyshev_filter(hx, X, m: int, a: float, b: float, a0: float):
    """Scaled three-term Chebyshev recurrence damping [a, b], normalised at a0."""
    e = (b - a) / 2.0
    c = (b + a) / 2.0
    sigma = e / (a0 - c)
    sigma1 = sigma
    gamma = 2.0 / sigma1
    Y = (hx(X) - c * X) * (sigma1 / e)
    for _ in range(2, m + 1):
        sigma2 = 1.0 / (gamma - sigma)
        Ynew = (hx(Y) - c * Y) * (2.0 * sigma2 / e) - (sigma * sigma2) * X
        X, Y = Y, Ynew
        sigma = sigma2
    return Y


def fix_signs(Q: np.ndarray) -> np.ndarray:
    """Make the entry of largest magnitude of every column positive."""
    idx = np.argmax(np.abs(Q), axis=0)
    s = np.sign(Q[idx, np.arange(Q.shape[1])])
    s[s == 0] = 1.0
    return Q * s[None, :]


def chfsi_pass(hx, X, m: int, a: float, b: float, a0: float):
    """One filter + Cholesky-GS + Rayleigh-Ritz + residual pass.

    Returns (X_new, eigenvalues ascending, residual norms).
    """
    Y = chebyshev_filter(hx, X, m, a, b, a0)
    S = Y.T @ Y
    L = np.linalg.cholesky(S)
    Y = sla.solve_triangular(L, Y.T, lower=True).T          # Y L^{-T}
    HY = hx(Y)
    Hp = Y.T @ HY
    Hp = 0.5 * (Hp + Hp.T)
    w, Q = np.linalg.eigh(Hp)
    Q = fix_signs(Q)
    Xn = Y @ Q
    HX = HY @ Q
    R = HX - Xn * w[None, :]
    return Xn, w, np.linalg.norm(R, axis=0)


def partial_occupancy(eig, mu, T):
    """Fermi-Dirac f(eps) in the overflow-safe form of dftUtils::getPartialOccupancy."""
    x = (np.asarray(eig, dtype=np.float64) - mu) / (C_KB * T)
    out = np.empty_like(x)
    pos = x >= 0
    out[pos] = np.exp(-x[pos]) / (1.0 + np.exp(-x[pos]))
    out[~pos] = 1.0 / (1.0 + np.exp(x[~pos]))
    return out


def partial_occupancy_der(eig, mu, T):
    """df/d(eps) of the Fermi-Dirac function (dftUtils::getPartialOccupancyDer)."""
    kT = C_KB * T
    x = (np.asarray(eig, dtype=np.float64) - mu) / kT
    e = np.exp(-np.abs(x))
    return -e / (kT * (1.0 + e) ** 2)


def fermi_energy(eig, n_electrons: float, T: float, k_weights=(1.0,)):
    """Bisection for mu with 2 sum_i f_i = N_e (dftClass::compute_fermienergy)."""
    eig = np.asarray(eig, dtype=np.float64)
    lo, hi = float(eig.min()) - 1.0, float(eig.max()) + 1.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        n = 2.0 * float(np.sum(partial_occupancy(eig, mid, T)))
        if n > n_electrons:
            hi = mid
        else:
            lo = mid
        if hi - lo < 1e-15 * max(1.0, abs(mid)):
            break
    return 0.5 * (lo + hi)

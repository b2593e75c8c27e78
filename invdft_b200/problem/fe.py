"""One-dimensional spectral-element building blocks on the unit interval [0, 1].

The parent (wavefunction) space uses Lagrange polynomials of order p on the
Gauss-Lobatto-Legendre (GLL) points, integrated with (p+1)-point Gauss rules for
the stiffness and potential matrices and with the GLL rule for the lumped
(diagonal) mass.  This is the spectral-element discretisation DFT-FE builds for
invDFT's Kohn-Sham operator (the reference calls it through
``KohnShamDFTBaseOperator::HXWithLowdinOrthonormalisedInput`` at
MultiVectorAdjointLinearSolverProblem.cpp:1353 and the quadrature of
``C_num1DQuad`` = p+1 in include/InverseDFTSolverFunction.h:42-44).

Node and quadrature indices of a hexahedral cell are lexicographic with x
fastest: ``i = a + (p+1)*b + (p+1)**2*c``.
"""
from __future__ import annotations

import numpy as np
from numpy.polynomial import legendre as _leg


def gll_points(p: int) -> tuple[np.ndarray, np.ndarray]:
    """GLL points and weights of order p mapped to [0, 1] (weights sum to 1)."""
    if p < 1:
        raise ValueError("order must be >= 1")
    if p == 1:
        return np.array([0.0, 1.0]), np.array([0.5, 0.5])
    interior = np.sort(_leg.Legendre.basis(p).deriv().roots().real)
    x = np.concatenate([[-1.0], interior, [1.0]])
    pp = _leg.Legendre.basis(p)(x)
    w = 2.0 / (p * (p + 1) * pp * pp)
    xs = 0.5 * (x + 1.0)
    # exact symmetric values: the midpoint of an even order is exactly 1/2
    xs = 0.5 * (xs + (1.0 - xs[::-1]))
    if p % 2 == 0:
        xs[p // 2] = 0.5
    xs[0], xs[-1] = 0.0, 1.0
    return xs, 0.5 * w


def gauss_points(n: int) -> tuple[np.ndarray, np.ndarray]:
    """n-point Gauss-Legendre rule on [0, 1] (weights sum to 1)."""
    x, w = _leg.leggauss(n)
    xs = 0.5 * (x + 1.0)
    xs = 0.5 * (xs + (1.0 - xs[::-1]))
    if n % 2 == 1:
        xs[n // 2] = 0.5
    return xs, 0.5 * w


def lagrange_eval(nodes: np.ndarray, x: np.ndarray) -> np.ndarray:
    """Values L[k, a] = l_a(x_k) of the Lagrange basis on ``nodes``.

    Evaluated as products so that l_a(nodes[b]) is exactly delta_ab.
    """
    x = np.asarray(x, dtype=np.float64)
    n = len(nodes)
    out = np.ones((x.size, n))
    for a in range(n):
        for b in range(n):
            if b != a:
                out[:, a] *= (x.ravel() - nodes[b]) / (nodes[a] - nodes[b])
    return out


def lagrange_deriv(nodes: np.ndarray, x: np.ndarray) -> np.ndarray:
    """Derivatives D[k, a] = l_a'(x_k)."""
    x = np.asarray(x, dtype=np.float64).ravel()
    n = len(nodes)
    out = np.zeros((x.size, n))
    for a in range(n):
        for m in range(n):
            if m == a:
                continue
            term = np.full(x.size, 1.0 / (nodes[a] - nodes[m]))
            for b in range(n):
                if b != a and b != m:
                    term *= (x - nodes[b]) / (nodes[a] - nodes[b])
            out[:, a] += term
    return out


class Element1D:
    """1D data of the order-p parent element on [0, 1]."""

    def __init__(self, p: int):
        self.p = p
        self.n1 = p + 1
        self.nodes, self.wgll = gll_points(p)
        self.qpts, self.wq = gauss_points(p + 1)
        # phi[q, a] = l_a(g_q), dphi[q, a] = l_a'(g_q)
        self.phi = lagrange_eval(self.nodes, self.qpts)
        self.dphi = lagrange_deriv(self.nodes, self.qpts)
        self.mass = self.phi.T @ (self.wq[:, None] * self.phi)
        self.stiff = self.dphi.T @ (self.wq[:, None] * self.dphi)

    # --- 3D tensor-product operators (lexicographic, x fastest) -----------
    def kron3(self, ax: np.ndarray, ay: np.ndarray, az: np.ndarray) -> np.ndarray:
        return np.kron(az, np.kron(ay, ax))

    def stiffness_ref(self) -> np.ndarray:
        """Unit-cube Laplacian stiffness: int grad N_i . grad N_j."""
        S, M = self.stiff, self.mass
        return self.kron3(S, M, M) + self.kron3(M, S, M) + self.kron3(M, M, S)

    def shape_at_quad(self) -> np.ndarray:
        """N[q, i] of the (p+1)^3 Gauss points."""
        return self.kron3(self.phi, self.phi, self.phi)

    def quad_weights(self) -> np.ndarray:
        w = self.wq
        return np.kron(w, np.kron(w, w))

    def gll_weights3(self) -> np.ndarray:
        w = self.wgll
        return np.kron(w, np.kron(w, w))

    def quad_points3(self) -> np.ndarray:
        """(n_q, 3) reference coordinates of the Gauss points."""
        g = self.qpts
        n = self.n1
        q = np.arange(n ** 3)
        return np.stack([g[q % n], g[(q // n) % n], g[q // (n * n)]], axis=1)

    def node_points3(self) -> np.ndarray:
        g = self.nodes
        n = self.n1
        i = np.arange(n ** 3)
        return np.stack([g[i % n], g[(i // n) % n], g[i // (n * n)]], axis=1)


GAUSS2 = gauss_points(2)

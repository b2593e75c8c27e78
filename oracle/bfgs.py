"""Oracle of ``BFGSInverseDFTSolver`` with the CP line search
(src/BFGSInverseDFTSolver.cpp:68-118, 185-303, 467-627), one spin component."""
from __future__ import annotations

import numpy as np


class BFGSInverseDFTSolver:
    def __init__(self, max_iter: int, tol: float = 1e-12, line_search_iters: int = 1,
                 line_search_tol: float = 1e-6, history: int = 100):
        self.max_iter = max_iter
        self.tol = tol
        self.n_ls = line_search_iters
        self.ls_tol = line_search_tol
        self.history = history
        self.y, self.s, self.rho = [], [], []
        self.k = 0
        self.log = []

    def inverse_jacobian_times_vec(self, g, fn):
        """Two-loop recursion (:68-118)."""
        q = g.copy()
        gamma = 1.0
        if self.y:
            gamma = fn.dot_product(self.s[-1], self.y[-1]) / fn.dot_product(self.y[-1], self.y[-1])
        N = self.k
        alpha = [0.0] * N
        for i in range(N - 1, -1, -1):
            ii = len(self.s) - (N - i)
            alpha[i] = self.rho[ii] * fn.dot_product(self.s[ii], q)
            q = q - alpha[i] * self.y[ii]
        z = gamma * q
        for i in range(N):
            beta = self.rho[i] * fn.dot_product(self.y[i], z)
            z = z + (alpha[i] - beta) * self.s[i]
        return z

    def _fnorm_cp(self, x, p, lam, fn):
        """fnormCP (:185-213): g(x + lam p) . p."""
        g, L, _ = fn.get_force_vector(x + lam * p)
        return fn.dot_product(g, p)

    def solve(self, fn, x0):
        x = np.array(x0, dtype=np.float64)
        g = None
        L = None
        for it in range(self.max_iter):
            if it == 0:
                g, L, st = fn.get_force_vector(x)
                self.log.append(dict(iter=it, loss=L, stats=st))
            gnorm = np.sqrt(fn.dot_product(g, g))
            p = -self.inverse_jacobian_times_vec(g, fn)
            f0 = fn.dot_product(g, p)
            lambdas = [0.0, 1.0]
            ls = [f0]
            if gnorm < self.tol:
                break
            self._line_search_cp(lambdas, ls, x, p, fn)
            lam = lambdas[-1] if lambdas[-1] > 0.0 else 1.0
            s = lam * p
            x = x + s
            y = -g
            g, L, st = fn.get_force_vector(x)
            self.log.append(dict(iter=it + 1, loss=L, stats=st, lam=lam))
            y = y + g
            curv = fn.dot_product(y, s)
            if curv > 0.0:
                self.y.append(y)
                self.s.append(s)
                self.rho.append(1.0 / curv)
                self.k += 1
            if self.k > self.history:
                self.k = self.history
                self.y.pop(0)
                self.s.pop(0)
                self.rho.pop(0)
        return x, g, L

    def _line_search_cp(self, lam, f, x, p, fn):
        """solveLineSearchCP (:217-303) with the reference's secant update."""
        for _ in range(self.n_ls):
            l0, l1 = lam[-2], lam[-1]
            f0 = f[-1]
            if np.sqrt(abs(f0)) < self.ls_tol:
                lam.pop()
                break
            f1 = self._fnorm_cp(x, p, l1, fn)
            f.append(f1)
            if np.sqrt(abs(f1)) < self.ls_tol:
                break
            if abs((f1 - f0) / f1) < 1e-15:
                raise RuntimeError("Secant line search failed, possibly because f'(x) = 0")
            sl = (f1 - f0) / (l1 - l0)
            if sl > 0.0:
                sl = -sl
            nxt = l1 - f1 / sl
            if nxt < 0.0:
                nxt = l1 + f1 / sl
            lam.append(nxt)

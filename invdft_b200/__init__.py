"""B200-native force evaluation of the invDFT inverse Kohn-Sham method.

The hot path (Chebyshev-filtered eigensolve -> density -> block-MINRES adjoint
-> projection of psi.p onto the v_xc mesh) runs in hand-written sm_100a
kernels behind the C ABI of ``include/invdft_force.h``; this package holds the
ctypes binding (``native``), the reference-shaped host interface (``solver``),
the differentiable wrapper (``autograd``) and the synthetic problem generator
(``problem``) that produces the inputs the reference receives from its engine.
"""
from .native import InvDFTError, load  # noqa: F401


def __getattr__(name):
    if name in ("InverseDFTSolverFunction", "MultiVectorAdjointLinearSolverProblem", "BFGSInverseDFTSolver"):
        from . import solver
        return getattr(solver, name)
    raise AttributeError(name)

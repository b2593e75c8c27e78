"""FP64 CPU oracle of invDFT's force evaluation -- TEST INFRASTRUCTURE ONLY.

This package restates, in numpy/scipy, the algorithm of the reference's hot
path (``InverseDFTSolverFunction::getForceVector`` and the adjoint problem of
``MultiVectorAdjointLinearSolverProblem``) so that the CUDA library can be
checked against it.  Only the tests, the smoke check and the CPU-baseline leg of
the benchmark may import it; the product never calls it.

Parity status: the parts invDFT implements itself are restated line by line
from its sources (each function cites file:line).  The parts invDFT delegates
to DFT-FE (Hamiltonian application, Chebyshev-filtered subspace iteration,
density, block MINRES, constraint handling) are not in the reference tree and
are restated from the published mathematics; the reference ships no golden
vectors for this path, so against DFT-FE itself parity is UNPINNED.  The oracle
is pinned against closed-form answers instead (see tests/test_oracle_*.py).
"""
from .force import ForceParams, InverseDFTSolverFunction  # noqa: F401
from .bfgs import BFGSInverseDFTSolver  # noqa: F401

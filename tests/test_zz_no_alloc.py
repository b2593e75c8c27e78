"""The allocation-free column-dot entry point against the existing dot product.

invdft_coldot_noalloc is for callers that must not let the library allocate
device memory while they run (their vectors live in their own device pool, as
in an outer L-BFGS or Krylov driver).  It keeps its scratch in a static device
array; this test calls it twice in a row through the C ABI and checks both
results against the library's existing dot product (invdft_dot) and against
numpy, and checks that a block wider than its scratch is rejected.  It sits in
its own file, collected last.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import problem

pytestmark = pytest.mark.gpu


def test_noalloc_coldot_matches_dot_twice():
    import torch
    from invdft_b200 import native
    from invdft_b200.solver import InverseDFTSolverFunction
    lib = native.load()
    fn = InverseDFTSolverFunction(problem("tiny_h2"))      # context for the existing invdft_dot
    rng = np.random.default_rng(11)
    cases = [(100003, 5), (4099, 1)]
    host, dev, outs = [], [], []
    for n, B in cases:
        a = rng.standard_normal((n, B))
        b = rng.standard_normal((n, B))
        host.append((a, b))
        da, db = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
        out = torch.full((B,), np.nan, dtype=torch.float64, device="cuda")
        dev.append((da, db))
        outs.append(out)
    torch.cuda.synchronize()
    for (n, B), (da, db), out in zip(cases, dev, outs):     # two calls in a row
        rc = lib.invdft_coldot_noalloc(C.c_void_p(da.data_ptr()), C.c_void_p(db.data_ptr()), n, B,
                                       C.c_void_p(out.data_ptr()), None)
        assert rc == 0, lib.invdft_last_error(None)
    torch.cuda.synchronize()
    for (n, B), (a, b), out in zip(cases, host, outs):
        got = out.cpu().numpy()
        for j in range(B):
            ref = fn.dot_product(np.ascontiguousarray(a[:, j]), np.ascontiguousarray(b[:, j]))
            assert abs(got[j] - ref) <= 1e-12 * max(1.0, abs(ref)) * np.sqrt(n)
            assert abs(got[j] - float(np.dot(a[:, j], b[:, j]))) <= 1e-12 * max(1.0, abs(ref)) * np.sqrt(n)


def test_noalloc_coldot_rejects_wider_than_scratch():
    import torch
    from invdft_b200 import native
    lib = native.load()
    a = torch.zeros((8, 65), dtype=torch.float64, device="cuda")
    out = torch.zeros(65, dtype=torch.float64, device="cuda")
    rc = lib.invdft_coldot_noalloc(C.c_void_p(a.data_ptr()), C.c_void_p(a.data_ptr()), 8, 65,
                                   C.c_void_p(out.data_ptr()), None)
    assert rc == 5
    assert b"[1, 64]" in lib.invdft_last_error(None)

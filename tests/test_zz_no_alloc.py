"""lu_solve_noalloc: the allocation-free solve, checked against lu_solve.

Some callers may not allocate device memory: a plugin whose host
application owns the device memory and grants it a fixed budget, a real-time
loop that cannot afford an allocation's device-wide synchronisation, or a
caller without a solver handle (creating one allocates).  lu_solve_noalloc
serves them with its scratch in a fixed device array inside the library.  This file is collected last so a
run that stops at the first failure has run every other test first; each
test also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu

LU_ERR_ARG = -1


def _noalloc(LU, ipiv, x, status=None, n=None, lda=None):
    from charmlu_b200 import _lib
    L = _lib.load()
    n = LU.shape[0] if n is None else n
    lda = LU.stride(0) if lda is None else lda
    return L.lu_solve_noalloc(ctypes.c_void_p(LU.data_ptr()), lda, n,
                              ctypes.c_void_p(ipiv.data_ptr()), ctypes.c_void_p(x.data_ptr()),
                              ctypes.c_void_p(status.data_ptr()) if status is not None else None,
                              ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))


@pytest.mark.parametrize("n,b", [(1000, 128), (4096, 256)])
def test_noalloc_solve_matches_lu_solve_twice(cuda_dev, n, b):
    import charmlu_b200 as lu
    A = oracle.gen_matrix(n, 13)
    Ad = torch.from_numpy(A).cuda()
    s = lu.LUSolver(lu.LUConfig(n, b))
    ipiv = s.factor(Ad)
    assert s.status() == 0
    for call in range(2):  # two calls in a row: the shared scratch must be re-cleared
        rhs = oracle.gen_vector(n, 100 + call)
        x_ref = torch.from_numpy(rhs).cuda()
        s.solve(Ad, ipiv, x_ref)
        assert s.status() == 0
        x = torch.from_numpy(rhs).cuda()
        st = torch.full((1,), -99, dtype=torch.int32, device="cuda")
        assert _noalloc(Ad, ipiv, x, st) == 0
        torch.cuda.synchronize()
        assert st.item() == 0
        xr = x_ref.cpu().numpy()
        # same tolerance as the solve tests (1e-10 relative); the two paths run
        # the same substitution kernels, so they agree to the last bit here
        assert np.abs(x.cpu().numpy() - xr).max() <= 1e-10 * max(1.0, np.abs(xr).max())
        r = oracle.residual(A, x.cpu().numpy(), rhs)
        assert r["r_hpl"] < 16


def test_noalloc_rejects_oversize(cuda_dev):
    # rejected by the size check before anything is launched or read
    n = (1 << 17) + 2
    LU = torch.zeros(2, 2, dtype=torch.float64, device="cuda")
    ipiv = torch.zeros(1, dtype=torch.int32, device="cuda")
    x = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert _noalloc(LU, ipiv, x, n=n, lda=n) == LU_ERR_ARG

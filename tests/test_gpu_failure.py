"""Failure detection without a GPU fault: every spin-wait in the library is
bounded.  A wait on a pipeline counter that nothing advances gives up after
its poll limit, records LU_ERR_TIMEOUT in the device status word and
returns; the context stays usable for the next solve."""
import ctypes

import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_context_survives(cuda_dev):
    import charmlu_b200 as lu
    from charmlu_b200 import _lib
    f = _lib.load().lub_test_wait_timeout
    f.argtypes = [ctypes.c_longlong]
    f.restype = ctypes.c_int
    assert f(20000) == lu.LU_ERR_TIMEOUT
    # the next factor + solve on the same context is unaffected
    n = 256
    A = torch.from_numpy(oracle.gen_matrix(n, 3)).cuda()
    b = torch.from_numpy(oracle.gen_vector(n, 3)).cuda()
    s = lu.LUSolver(lu.LUConfig(n, 64))
    A0, x = A.clone(), b.clone()
    s.factor_solve(A, x)
    assert s.status() == 0
    assert s.residual(A0, x, b)["r_hpl"] < 16

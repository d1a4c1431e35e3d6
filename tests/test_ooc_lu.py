"""The out-of-core FP64 LU driver (charmlu_b200/ooc.py) on CPU, with the
numpy stand-in for the per-block kernels. It runs the driver's own logic:
panel streaming and buffer reuse, earlier pivots applied to each loaded
panel, later pivots applied to the earlier panels' rows, the final L pass,
and the streamed solve. Checked against LAPACK getrf (scipy): the same
pivots, the same L\\U to rounding, x against numpy.linalg.solve, and the
first singular column. The GPU kernels are checked through the C ABI in
tests/test_gpu_ooc.py."""
import numpy as np
import pytest
import scipy.linalg as sl
import torch

from numpy_blocks import NumpyBlocks


@pytest.mark.parametrize("n,w", [(300, 64), (257, 32), (64, 64), (100, 200), (129, 2)])
def test_out_of_core_lu_matches_lapack(n, w):
    from charmlu_b200.ooc import OutOfCoreLU
    rng = np.random.default_rng(n + w)
    A = rng.uniform(-0.5, 0.5, (n, n))
    b = rng.uniform(-0.5, 0.5, n)
    host = torch.from_numpy(A.copy())
    ooc = OutOfCoreLU(n, panel=w, blocks=NumpyBlocks(), device="cpu")
    ipiv = ooc.factor(host)
    assert ooc.status_code == 0
    lu_ref, piv_ref = sl.lu_factor(A)
    assert np.array_equal(ipiv.numpy(), piv_ref.astype(np.int32))
    assert np.abs(host.numpy() - lu_ref).max() <= 1e-12 * n * max(1.0, np.abs(lu_ref).max())
    x = ooc.solve(host, ipiv, torch.from_numpy(b)).numpy()
    xr = np.linalg.solve(A, b)
    assert np.abs(x - xr).max() <= 1e-10 * np.abs(xr).max()


def test_out_of_core_lu_reports_singular_column():
    from charmlu_b200.ooc import OutOfCoreLU
    n, w = 96, 32
    A = np.random.default_rng(1).uniform(-0.5, 0.5, (n, n))
    A[:, 50] = 0.0
    ooc = OutOfCoreLU(n, panel=w, blocks=NumpyBlocks(), device="cpu")
    ooc.factor(torch.from_numpy(A))
    assert ooc.status_code == 51


def test_panel_width_from_device_budget():
    from charmlu_b200.ooc import OutOfCoreLU
    ooc = OutOfCoreLU(131072, b=256, blocks=NumpyBlocks(), device="cpu", device_budget=90 << 30)
    # three n x w FP64 panels within the budget, w a multiple of b
    assert ooc.w % 256 == 0 and 3 * 8 * 131072 * ooc.w <= 90 << 30
    assert OutOfCoreLU(1000, b=256, blocks=NumpyBlocks(), device="cpu", device_budget=1 << 20).w == 256


def test_status_is_cleared_between_factorisations():
    """A driver reused after a singular matrix reports 0 for a regular one."""
    from charmlu_b200.ooc import OutOfCoreLU
    n = 64
    ooc = OutOfCoreLU(n, panel=16, blocks=NumpyBlocks(), device="cpu")
    A = np.random.default_rng(2).uniform(-0.5, 0.5, (n, n))
    S = A.copy()
    S[:, 5] = 0.0
    ooc.factor(torch.from_numpy(S))
    assert ooc.status_code == 6
    ooc.factor(torch.from_numpy(A.copy()))
    assert ooc.status_code == 0

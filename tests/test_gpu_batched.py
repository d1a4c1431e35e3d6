"""Batched uneven factor + solve in one persistent launch (no reference
counterpart).  Each system is checked against the per-system contract the
single-matrix path meets: scaled residual r_hpl < 16, and the solution
against an FP64 LAPACK solve."""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

LU_PREC_FP64, LU_PREC_FP32 = 0, 4


def _systems(count, lo, hi, seed):
    rng = np.random.default_rng(seed)
    n = np.exp(rng.uniform(np.log(lo), np.log(hi + 1), count)).astype(np.int32)
    n = np.clip(n, lo, hi)
    a_off = np.concatenate([[0], np.cumsum(n.astype(np.int64) ** 2)[:-1]]).astype(np.int64)
    b_off = np.concatenate([[0], np.cumsum(n.astype(np.int64))[:-1]]).astype(np.int64)
    return n, a_off, b_off


def _run(n, a_off, b_off, precision, seed=42):
    import charmlu_b200 as lu
    from charmlu_b200 import _lib
    L = _lib.load()
    count = len(n)
    tot_a = int(a_off[-1] + int(n[-1]) ** 2)
    tot_b = int(b_off[-1] + int(n[-1]))
    A = lu.generate_uniform(1, tot_a, seed=seed, stream_id=10).view(-1)
    b = lu.generate_uniform(1, tot_b, seed=seed, stream_id=11).view(-1)
    A0, b0 = A.clone(), b.clone()
    dn = torch.from_numpy(n).cuda()
    da = torch.from_numpy(a_off).cuda()
    dbo = torch.from_numpy(b_off).cuda()
    info = torch.full((count,), -99, dtype=torch.int32, device="cuda")
    wb = L.lu_batched_work_bytes(count, ctypes.c_void_p(n.ctypes.data), precision)
    work = torch.empty(wb, dtype=torch.uint8, device="cuda")
    rc = L.lu_batched_factor_solve(count, ctypes.c_void_p(dn.data_ptr()), ctypes.c_void_p(da.data_ptr()),
                                   ctypes.c_void_p(dbo.data_ptr()), ctypes.c_void_p(A.data_ptr()),
                                   ctypes.c_void_p(b.data_ptr()), ctypes.c_void_p(info.data_ptr()), precision,
                                   ctypes.c_void_p(work.data_ptr()), wb,
                                   ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    assert rc == 0
    if precision == LU_PREC_FP32:
        # every system lands in exactly one bin of the refinement-step histogram
        hist = np.zeros(12, dtype=np.int32)
        assert L.lu_batched_refine_histogram(ctypes.c_void_p(work.data_ptr()), ctypes.c_void_p(hist.ctypes.data),
                                             ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)) == 0
        assert hist.sum() == count and hist[11] == int((info.cpu().numpy() != 0).sum()), hist
    return A0.cpu().numpy(), b0.cpu().numpy(), b.cpu().numpy(), info.cpu().numpy(), A


def _check(n, a_off, b_off, A0, b0, x, info, fe_tol):
    eps = np.finfo(np.float64).eps
    assert np.all(info == 0), info[info != 0][:10]
    worst = 0.0
    for i in range(len(n)):
        k = int(n[i])
        Ai = A0[a_off[i]:a_off[i] + k * k].reshape(k, k)
        bi = b0[b_off[i]:b_off[i] + k]
        xi = x[b_off[i]:b_off[i] + k]
        r = np.abs(bi - Ai @ xi).max()
        r_hpl = r / ((np.abs(Ai).sum(1).max() * np.abs(xi).max() + np.abs(bi).max()) * k * eps)
        worst = max(worst, r_hpl)
        assert r_hpl < 16, (i, k, r_hpl)
        xr = np.linalg.solve(Ai, bi)
        assert np.abs(xi - xr).max() / np.abs(xr).max() < fe_tol, (i, k)
    return worst


@pytest.mark.parametrize("lo,hi,count", [(1, 40, 300), (32, 1024, 160), (150, 300, 64)])
def test_batched_fp64(cuda_dev, lo, hi, count):
    n, a_off, b_off = _systems(count, lo, hi, seed=lo * 7 + hi)
    A0, b0, x, info, _ = _run(n, a_off, b_off, LU_PREC_FP64)
    _check(n, a_off, b_off, A0, b0, x, info, fe_tol=1e-9)


@pytest.mark.parametrize("lo,hi,count", [(32, 1024, 160), (1, 40, 100)])
def test_batched_fp32_one_refinement(cuda_dev, lo, hi, count):
    n, a_off, b_off = _systems(count, lo, hi, seed=lo * 11 + hi)
    A0, b0, x, info, A_after = _run(n, a_off, b_off, LU_PREC_FP32)
    # the FP64 matrices are left untouched in FP32 mode
    assert np.array_equal(A_after.cpu().numpy(), A0)
    _check(n, a_off, b_off, A0, b0, x, info, fe_tol=1e-7)


def test_batched_matches_single_matrix_path(cuda_dev):
    """Same pivots and factors as lu_factor on each system (FP64)."""
    import charmlu_b200 as lu
    n, a_off, b_off = _systems(24, 16, 200, seed=5)
    A0, b0, x, info, A_fact = _run(n, a_off, b_off, LU_PREC_FP64)
    Af = A_fact.cpu().numpy()
    for i in range(len(n)):
        k = int(n[i])
        Ai = A0[a_off[i]:a_off[i] + k * k].reshape(k, k)
        buf = torch.zeros(k, k + (k & 1), dtype=torch.float64, device="cuda")
        Ad = buf[:, :k]
        Ad.copy_(torch.from_numpy(Ai))
        s = lu.LUSolver(lu.LUConfig(k, 16))
        s.factor(Ad)
        assert s.status() == 0
        ref = Ad.cpu().numpy()
        got = Af[a_off[i]:a_off[i] + k * k].reshape(k, k)
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max(), i


def test_batched_rejects_bad_order(cuda_dev):
    n = np.array([10, 5000, 7], dtype=np.int32)
    a_off = np.array([0, 100, 100 + 5000 * 5000], dtype=np.int64)
    b_off = np.array([0, 10, 5010], dtype=np.int64)
    from charmlu_b200 import _lib
    L = _lib.load()
    # the prep kernel marks every system LU_ERR_ARG and the solve kernel does nothing
    count = 3
    dn = torch.from_numpy(n).cuda()
    da = torch.from_numpy(a_off).cuda()
    dbo = torch.from_numpy(b_off).cuda()
    A = torch.zeros(16, dtype=torch.float64, device="cuda")
    b = torch.zeros(16, dtype=torch.float64, device="cuda")
    info = torch.zeros(count, dtype=torch.int32, device="cuda")
    work = torch.empty(1 << 20, dtype=torch.uint8, device="cuda")
    rc = L.lu_batched_factor_solve(count, ctypes.c_void_p(dn.data_ptr()), ctypes.c_void_p(da.data_ptr()),
                                   ctypes.c_void_p(dbo.data_ptr()), ctypes.c_void_p(A.data_ptr()),
                                   ctypes.c_void_p(b.data_ptr()), ctypes.c_void_p(info.data_ptr()), 0,
                                   ctypes.c_void_p(work.data_ptr()), 1 << 20,
                                   ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    assert rc == 0
    assert np.all(info.cpu().numpy() == -1)

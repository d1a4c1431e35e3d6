"""GPU parity tests of the FP64 path through the C ABI against the CPU oracle.

Bars: pivots bit-exact except near-ties (oracle top-2 margin
<= 1e-10, where a different summation order may legitimately flip the
choice), L and U within 1e-12 relative (max-abs difference over max-abs
entry), scaled residual < 16.
"""
import os

import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "lu_golden.npz"))
LU_RTOL = 1e-12
TIE_MARGIN = 1e-10


def _lu():
    import charmlu_b200 as lu
    return lu


def _gpu_factor(A_np, b, rhs_np=None, lda_pad=0, lookahead=False):
    lu = _lu()
    n = A_np.shape[0]
    lda = n + lda_pad
    if lda % 2:
        lda += 1
    buf = torch.zeros(n, lda, dtype=torch.float64, device="cuda")
    buf[:, :n] = torch.from_numpy(A_np)
    A = buf[:, :n]
    rhs = None if rhs_np is None else torch.from_numpy(rhs_np).cuda()
    s = lu.LUSolver(lu.LUConfig(n, b, lookahead=lookahead))
    ipiv = s.factor(A, rhs=rhs)
    st = s.status()
    return s, A, ipiv, rhs, st


def _compare(LU_gpu, ipiv_gpu, LU_ref, ipiv_ref, margin, rtol=LU_RTOL):
    ok = margin > TIE_MARGIN
    np.testing.assert_array_equal(ipiv_gpu[ok], ipiv_ref[ok])
    scale = np.abs(LU_ref).max()
    err = np.abs(LU_gpu - LU_ref).max() / scale
    assert err <= rtol, err


def _cpu_envelope(A, LU_ref):
    """Normwise gap between two correct CPU FP64 factorisations of A (the
    oracle's blocked order vs LAPACK dgetrf).  Above N ~ 4096 it exceeds
    1e-12, so large-N parity is held to max(1e-12, 2 x this gap)."""
    import scipy.linalg as sl
    lu_l, _ = sl.lu_factor(A)
    return np.abs(lu_l - LU_ref).max() / np.abs(LU_ref).max()


def test_generator_bit_identical(cuda_dev):
    lu = _lu()
    for (r, c, seed, sid) in [(64, 64, 42, 0), (37, 129, 7, 1), (1000, 3, 42, 0)]:
        g = lu.generate_uniform(r, c, seed=seed, stream_id=sid).cpu().numpy()
        ref = oracle.gen_uniform(r * c, seed, sid).reshape(r, c)
        np.testing.assert_array_equal(g, ref)


@pytest.mark.parametrize("key", [k[:-5] for k in GOLD.files if k.endswith("_ipiv")])
def test_factor_matches_golden(cuda_dev, key):
    n, b = (int(s[1:]) for s in key.split("_"))
    A = oracle.gen_matrix(n, 42)
    rhs = oracle.gen_vector(n, 42)
    s, Ag, ipiv, rg, st = _gpu_factor(A, b, rhs)
    assert st == 0
    ip = ipiv.cpu().numpy()
    margin = GOLD[key + "_margin"]
    ok = margin > TIE_MARGIN
    np.testing.assert_array_equal(ip[ok], GOLD[key + "_ipiv"][ok])
    if key + "_lu" in GOLD.files:
        ref = GOLD[key + "_lu"]
        assert np.abs(Ag.cpu().numpy() - ref).max() / np.abs(ref).max() <= LU_RTOL
    # rhs carried through the swaps (lu.h:66) then solved
    x = torch.from_numpy(rhs).cuda()
    s.solve(Ag, ipiv, x)
    assert s.status() == 0
    xr = GOLD[key + "_x"]
    assert np.abs(x.cpu().numpy() - xr).max() <= 1e-10 * max(1.0, np.abs(xr).max())


@pytest.mark.parametrize("n,b,pad", [(512, 64, 0), (1000, 128, 0), (777, 32, 6), (2048, 128, 0), (1536, 256, 2)])
def test_factor_matches_oracle(cuda_dev, n, b, pad):
    A = oracle.gen_matrix(n, 11)
    rhs = oracle.gen_vector(n, 11)
    LU_ref, ip_ref, rp_ref, margin, info = oracle.lu_factor(A, b=b, rhs=rhs)
    s, Ag, ipiv, rg, st = _gpu_factor(A, b, rhs, lda_pad=pad)
    assert st == 0 and info == 0
    _compare(Ag.cpu().numpy(), ipiv.cpu().numpy(), LU_ref, ip_ref, margin)
    if np.all(margin > TIE_MARGIN):
        np.testing.assert_array_equal(rg.cpu().numpy(), rp_ref)


def test_config1_n2048_b128_full_contract(cuda_dev):
    """N=2048, b=128, seed 42: pivots, L/U, residual (the reference's CPU case)."""
    lu = _lu()
    n, b = 2048, 128
    A = oracle.gen_matrix(n, 42)
    rhs = oracle.gen_vector(n, 42)
    x_ref, LU_ref, ip_ref, margin, info = oracle.solve(A, rhs, b=b)
    Ad = torch.from_numpy(A).cuda()
    bd = torch.from_numpy(rhs).cuda()
    s = lu.LUSolver(lu.LUConfig(n, b))
    ipiv = s.factor_solve(Ad, bd)
    assert s.status() == 0
    _compare(Ad.cpu().numpy(), ipiv.cpu().numpy(), LU_ref, ip_ref, margin)
    res = s.residual(torch.from_numpy(A).cuda(), bd, torch.from_numpy(rhs).cuda())
    ref = oracle.residual(A, bd.cpu().numpy(), rhs)
    assert res["r_hpl"] < 16 and res["r_ref"] < 16
    assert abs(res["amax"] - ref["amax"]) == 0 and abs(res["bnorm"] - ref["bmax"]) == 0
    assert abs(res["anorm"] - ref["anorm"]) <= 1e-12 * ref["anorm"]
    fe = np.abs(bd.cpu().numpy() - x_ref).max() / np.abs(x_ref).max()
    assert fe < 1e-10


# test_lu.pl's parameter sets (test_lu.pl:9-52): pass when residual < 16
TEST_LU_PL = [(48, 48), (48, 24), (48, 16), (48, 12), (32, 8), (32, 4), (512, 128), (512, 64), (512, 256),
              (1024, 256), (1024, 128), (1024, 64), (2048, 256), (2048, 512), (4096, 256), (4096, 512)]


@pytest.mark.parametrize("n,b", TEST_LU_PL)
def test_lu_pl_residual_contract(cuda_dev, n, b):
    lu = _lu()
    A = lu.generate_uniform(n, n, seed=42, stream_id=0)
    A0 = A.clone()
    rhs = torch.from_numpy(lu.matgen(n)).cuda()  # the reference's b (benchmark.C:455-460)
    x = rhs.clone()
    s = lu.LUSolver(lu.LUConfig(n, b))
    s.factor_solve(A, x)
    assert s.status() == 0
    r = s.residual(A0, x, rhs)
    assert r["r_ref"] < 16 and r["r_hpl"] < 16, r


def test_singular_column_reports_info(cuda_dev):
    lu = _lu()
    n, b = 256, 64
    A = oracle.gen_matrix(n, 5)
    A[:, 70] = 0.0
    _, _, _, _, info_ref = oracle.lu_factor(A, b=b)
    s, Ag, ipiv, _, st = _gpu_factor(A, b)
    assert info_ref == 71 and st == 71


@pytest.mark.parametrize("lookahead", [False, True])
def test_exact_tie_lowest_row_wins(cuda_dev, lookahead):
    """|a_i0| = 1 exactly at rows 10, 1000 and 3000 (signs -, +, -), rows
    held by different CTAs of the panel grid: the pivot is row 10, as in the
    oracle (lowest global row wins an exact tie)."""
    A = oracle.gen_matrix(4096, 3)
    A[10, 0], A[1000, 0], A[3000, 0] = -1.0, 1.0, -1.0
    _, ipiv_ref, _, _, _ = oracle.lu_factor(A, b=256)
    s, Ag, ipiv, _, st = _gpu_factor(A, 256, lookahead=lookahead)
    assert st == 0 and int(ipiv[0]) == 10 and ipiv_ref[0] == 10


def test_reference_threshold_singularity(cuda_dev):
    lu = _lu()
    n, b = 128, 32
    A = oracle.gen_matrix(n, 8)
    A[40] = A[3] * 1.0  # exact duplicate row
    _, _, _, _, info_ref = oracle.lu_factor(A, b=b, sing_threshold=oracle.SING_REF)
    Ad = torch.from_numpy(A).cuda()
    s = lu.LUSolver(lu.LUConfig(n, b, sing_threshold=oracle.SING_REF))
    s.factor(Ad)
    assert info_ref > 0 and s.status() == info_ref


def test_solve_new_rhs_with_ipiv(cuda_dev):
    lu = _lu()
    n, b = 1024, 128
    A = oracle.gen_matrix(n, 21)
    s, Ag, ipiv, _, st = _gpu_factor(A, b)
    rhs = oracle.gen_vector(n, 22)
    x = torch.from_numpy(rhs).cuda()
    s.solve(Ag, ipiv, x)
    assert s.status() == 0
    r = oracle.residual(A, x.cpu().numpy(), rhs)
    assert r["r_hpl"] < 16


def test_deterministic_replay(cuda_dev):
    A = oracle.gen_matrix(1024, 31)
    _, A1, p1, _, _ = _gpu_factor(A, 128)
    _, A2, p2, _, _ = _gpu_factor(A, 128)
    assert torch.equal(p1, p2)
    assert torch.equal(A1, A2)


def test_bad_arguments_return_codes(cuda_dev):
    lu = _lu()
    s = lu.LUSolver(lu.LUConfig(64, 16))
    A = torch.zeros(64, 64, dtype=torch.float64, device="cuda")
    with pytest.raises(TypeError):
        s.factor(A.cpu())
    with pytest.raises(lu.LUError):
        s.factor(torch.zeros(63, 63, dtype=torch.float64, device="cuda"))


def test_large_n8192_against_oracle(cuda_dev):
    lu = _lu()
    n, b = 8192, 256
    A = oracle.gen_matrix(n, 42)
    rhs = oracle.gen_vector(n, 42)
    x_ref, LU_ref, ip_ref, margin, info = oracle.solve(A, rhs, b=b)
    Ad = torch.from_numpy(A).cuda()
    bd = torch.from_numpy(rhs).cuda()
    s = lu.LUSolver(lu.LUConfig(n, b))
    ipiv = s.factor_solve(Ad, bd)
    assert s.status() == 0
    env = _cpu_envelope(A, LU_ref)
    _compare(Ad.cpu().numpy(), ipiv.cpu().numpy(), LU_ref, ip_ref, margin, rtol=max(LU_RTOL, 2 * env))
    r = s.residual(torch.from_numpy(A).cuda(), bd, torch.from_numpy(rhs).cuda())
    assert r["r_hpl"] < 16


@pytest.mark.parametrize("n,b", [(1000, 128), (2048, 128), (4096, 256), (777, 64)])
def test_lookahead_matches_oracle(cuda_dev, n, b):
    """Two-stream look-ahead schedule: same contract as the serial schedule."""
    A = oracle.gen_matrix(n, 17)
    rhs = oracle.gen_vector(n, 17)
    LU_ref, ip_ref, rp_ref, margin, info = oracle.lu_factor(A, b=b, rhs=rhs)
    s, Ag, ipiv, rg, st = _gpu_factor(A, b, rhs, lookahead=True)
    assert st == 0
    env = _cpu_envelope(A, LU_ref) if n > 2048 else 0.0
    _compare(Ag.cpu().numpy(), ipiv.cpu().numpy(), LU_ref, ip_ref, margin, rtol=max(LU_RTOL, 2 * env))
    if np.all(margin > TIE_MARGIN):
        np.testing.assert_array_equal(rg.cpu().numpy(), rp_ref)
    x = torch.from_numpy(rhs).cuda()
    s.solve(Ag, ipiv, x)
    assert oracle.residual(A, x.cpu().numpy(), rhs)["r_hpl"] < 16


def test_lookahead_trailing_update_identical_to_serial(cuda_dev):
    """With equal leaf widths the two schedules do the same arithmetic per
    element, so the factors are bit-identical."""
    import os
    A = oracle.gen_matrix(1536, 23)
    _, A1, p1, _, _ = _gpu_factor(A, 128, lookahead=False)
    _, A2, p2, _, _ = _gpu_factor(A, 128, lookahead=True)
    assert torch.equal(p1, p2)
    # leaf widths differ between the schedules (32 vs 16), so only near-equality
    assert (A1 - A2).abs().max().item() <= 1e-12 * A1.abs().max().item()


@pytest.mark.parametrize("lookahead", [False, True])
def test_graph_replay_identical(cuda_dev, lookahead):
    """use_graph: the schedule is captured once per buffer set and replayed;
    replays give bit-identical factors, and new buffers trigger a new capture."""
    import charmlu_b200 as lu
    n, b = 1536, 128
    A = oracle.gen_matrix(n, 41)
    ref = lu.LUSolver(lu.LUConfig(n, b, lookahead=lookahead))
    Ar = torch.from_numpy(A).cuda()
    pr = ref.factor(Ar)
    assert ref.status() == 0
    g = lu.LUSolver(lu.LUConfig(n, b, lookahead=lookahead, use_graph=True))
    Ad = torch.empty_like(Ar)
    ip = torch.empty(n, dtype=torch.int32, device="cuda")
    for _ in range(3):  # capture, then two replays on the same buffers
        Ad.copy_(torch.from_numpy(A))
        g.factor(Ad, ipiv=ip)
        assert g.status() == 0
        assert torch.equal(ip, pr) and torch.equal(Ad, Ar)
    A2 = torch.from_numpy(A).cuda()  # different buffer: re-capture
    p2 = g.factor(A2)
    assert g.status() == 0 and torch.equal(A2, Ar) and torch.equal(p2, pr)


@pytest.mark.parametrize("n,b", [(1000, 128), (1001, 64), (2048, 256)])
def test_column_major_layout_matches_row_major(cuda_dev, n, b):
    """LU_LAYOUT_COL: a column-major A (LAPACK order) is transposed in place,
    factored and transposed back, so its factors and pivots equal the
    row-major factorisation's, bit for bit, stored column-major."""
    lu = _lu()
    A = torch.from_numpy(oracle.gen_matrix(n, 31)).cuda()
    ld = n + (n & 1)
    buf = torch.zeros(ld, ld, dtype=torch.float64, device="cuda")
    buf[:n, :n] = A.t()
    A_col = buf[:n, :n].t()  # column-major view of A: unit row stride, pitch ld
    assert A_col.stride(0) == 1 and torch.equal(A_col, A)
    s_col = lu.LUSolver(lu.LUConfig(n, b, layout=lu.LU_LAYOUT_COL))
    ipiv_col = s_col.factor(A_col)
    assert s_col.status() == 0
    s_row = lu.LUSolver(lu.LUConfig(n, b))
    ref = torch.zeros(n, ld, dtype=torch.float64, device="cuda")
    ref[:, :n] = A
    ipiv_row = s_row.factor(ref[:, :n])
    assert torch.equal(ipiv_col, ipiv_row)
    assert torch.equal(A_col, ref[:, :n])
    # factor_solve on a fresh column-major copy gives the row-major path's x
    buf[:n, :n] = A.t()
    rhs = torch.from_numpy(oracle.gen_vector(n, 31)).cuda()
    x_col = rhs.clone()
    s_col.factor_solve(A_col, x_col)
    ref[:, :n] = A
    x_row = rhs.clone()
    s_row.factor_solve(ref[:, :n], x_row)
    assert torch.equal(x_col, x_row) and torch.equal(A_col, ref[:, :n])
    # the other entry points take row-major data
    with pytest.raises(lu.LUError) as e:
        s_col.solve(A_col, ipiv_col, rhs.clone())
    assert e.value.code == lu.LU_ERR_UNSUPPORTED


def test_transpose_square_and_layout_arguments(cuda_dev):
    lu = _lu()
    for n in (1, 31, 32, 33, 1001):
        ld = n + (n & 1) + 2
        buf = torch.from_numpy(oracle.gen_uniform(n * ld, 5, 0).reshape(n, ld)).cuda()
        A = buf[:, :n]
        A0 = A.clone()
        pad0 = buf[:, n:].clone()
        lu.transpose_square(A)
        torch.cuda.synchronize()
        assert torch.equal(A, A0.t()) and torch.equal(buf[:, n:], pad0)
        lu.transpose_square(A)
        assert torch.equal(A, A0)
    with pytest.raises(lu.LUError) as e:
        lu.LUSolver(lu.LUConfig(256, 64, precision=lu.LU_PREC_FP16X3, layout=lu.LU_LAYOUT_COL))
    assert e.value.code == lu.LU_ERR_UNSUPPORTED
    with pytest.raises(lu.LUError):
        lu.LUSolver(lu.LUConfig(256, 64, layout=7))
    # a rejected argument leaves a column-major matrix untouched (the in-place
    # transpose runs only after every check has passed)
    import ctypes
    from charmlu_b200 import _lib
    n = 256
    s_col = lu.LUSolver(lu.LUConfig(n, 64, layout=lu.LU_LAYOUT_COL))
    A = torch.from_numpy(oracle.gen_matrix(n, 9)).cuda()
    A0 = A.clone()
    x = torch.ones(n, dtype=torch.float64, device="cuda")
    L = _lib.load()
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert L.lu_factor(s_col._h, ctypes.c_void_p(A.data_ptr()), n, None, None, st) == lu.LU_ERR_ARG
    assert L.lu_factor_solve(s_col._h, ctypes.c_void_p(A.data_ptr()), n, None,
                             ctypes.c_void_p(x.data_ptr()), st) == lu.LU_ERR_ARG
    torch.cuda.synchronize()
    assert torch.equal(A, A0)

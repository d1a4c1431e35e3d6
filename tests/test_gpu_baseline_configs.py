"""Parity of the FP64 path at the benchmark configurations, against the CPU
oracle through the C ABI.

* N=2048, b=128 (the reference's CPU-sized case) with the two-stream
  look-ahead schedule and CUDA-graph replay, as the bench runs it.
* N=32768, b=256 (the reference's trailing-update path lu.C:26-43 at scale):
  pivots bit-exact except near-ties, L\\U within the CPU-CPU envelope, r_hpl
  below 16.
* N=65536 (the headline order): the FP64 solve's scaled residual.

Near-ties are columns whose oracle top-2 margin is <= 1e-10: a different
FP64 summation order may legitimately pick the other row there.
"""
import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu

TIE_MARGIN = 1e-10
# Normwise gap between two correct CPU FP64 factorisations of the same
# seed-42 uniform matrix (the oracle's b=256 blocked order against LAPACK
# dgetrf through scipy), measured: 9.3e-13 at N=4096, 2.6e-12 at 8192,
# 9.2e-12 at 16384 and 1.53e-11 at 32768 (the two pivot vectors equal at every
# order; at 32768 no column's top-2 margin is below 1e-10).  The GPU is held
# to twice the N=32768 gap.
ENVELOPE_N32768 = 3.1e-11


def _max_rel_diff(X, Y, rows=4096):
    """max |X - Y| / max |Y| over row chunks (keeps host memory bounded)."""
    num, den = 0.0, 0.0
    for r0 in range(0, X.shape[0], rows):
        x, y = X[r0:r0 + rows], Y[r0:r0 + rows]
        num = max(num, float(np.abs(x - y).max()))
        den = max(den, float(np.abs(y).max()))
    return num / den


def test_c1_lookahead_graph_replay_against_oracle(cuda_dev):
    import charmlu_b200 as lu
    n, b = 2048, 128
    A = oracle.gen_matrix(n, 42)
    rhs = oracle.gen_vector(n, 42)
    x_ref, LU_ref, ip_ref, margin, info = oracle.solve(A, rhs, b=b)
    assert info == 0
    s = lu.LUSolver(lu.LUConfig(n, b, lookahead=True, use_graph=True))
    Ad = torch.empty(n, n, dtype=torch.float64, device="cuda")
    xd = torch.empty(n, dtype=torch.float64, device="cuda")
    ipiv = torch.empty(n, dtype=torch.int32, device="cuda")
    for replay in range(3):  # capture, then two replays of the captured schedule
        Ad.copy_(torch.from_numpy(A))
        xd.copy_(torch.from_numpy(rhs))
        s.factor_solve(Ad, xd, ipiv=ipiv)
        assert s.status() == 0
        ok = margin > TIE_MARGIN
        np.testing.assert_array_equal(ipiv.cpu().numpy()[ok], ip_ref[ok])
        assert _max_rel_diff(Ad.cpu().numpy(), LU_ref) <= 1e-12
        fe = np.abs(xd.cpu().numpy() - x_ref).max() / np.abs(x_ref).max()
        assert fe < 1e-10
        r = s.residual(torch.from_numpy(A).cuda(), xd, torch.from_numpy(rhs).cuda())
        assert r["r_hpl"] < 16 and r["r_ref"] < 16


def test_c2_n32768_b256_against_oracle(cuda_dev):
    import charmlu_b200 as lu
    n, b = 32768, 256
    A = oracle.gen_matrix(n, 42)
    rhs = oracle.gen_vector(n, 42)
    s = lu.LUSolver(lu.LUConfig(n, b, lookahead=True))
    Ad = torch.from_numpy(A).cuda()
    xd = torch.from_numpy(rhs).cuda()
    ipiv = s.factor_solve(Ad, xd)
    assert s.status() == 0
    r = s.residual(torch.from_numpy(A).cuda(), xd, torch.from_numpy(rhs).cuda())
    assert r["r_hpl"] < 16
    LU_gpu = Ad.cpu().numpy()
    ip_gpu = ipiv.cpu().numpy()
    x_gpu = xd.cpu().numpy()
    del Ad, xd
    torch.cuda.empty_cache()
    LU_ref, ip_ref, _, margin, info = oracle.lu_factor(A, b=b)
    assert info == 0
    ok = margin > TIE_MARGIN
    np.testing.assert_array_equal(ip_gpu[ok], ip_ref[ok])
    assert _max_rel_diff(LU_gpu, LU_ref) <= ENVELOPE_N32768
    del LU_ref, LU_gpu
    ro = oracle.residual(A, x_gpu, rhs)
    assert ro["r_hpl"] < 16
    assert abs(ro["r_hpl"] - r["r_hpl"]) <= 1e-6 * max(1.0, ro["r_hpl"])


def test_n65536_fp64_residual(cuda_dev):
    import charmlu_b200 as lu
    n, b = 65536, 256
    A = lu.generate_uniform(n, n, seed=42, stream_id=0)
    rhs = lu.generate_uniform(n, 1, seed=42, stream_id=1).view(-1)
    Af = A.clone()
    x = rhs.clone()
    s = lu.LUSolver(lu.LUConfig(n, b, lookahead=True))
    s.factor_solve(Af, x)
    assert s.status() == 0
    del Af
    r = s.residual(A, x, rhs)
    assert r["r_hpl"] < 16, r

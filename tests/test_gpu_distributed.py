"""GPU tests of the per-block building blocks (lu_panel_factor,
lu_apply_pivots, lu_trsm_lower_unit, lu_gemm_update, lu_trsv_block,
lu_gemv_update) and of the block-cyclic driver on one GPU.

Each building block is checked against a plain FP64 torch / scipy
reference of the same operation. The driver at world size 1 (NCCL, one
rank) runs the same kernels on the same shapes as lu_factor, so without
look-ahead its factors and pivots equal lu_factor's bit for bit; with
look-ahead the pivots are equal and the factors agree to rounding. World
sizes above one are covered on CPU with gloo ranks (tests/test_distributed_lu.py,
tests/test_distributed_2d.py)."""
import os

import numpy as np
import pytest
import scipy.linalg as sl
import torch
import torch.distributed as dist

pytestmark = pytest.mark.gpu


def _blocks(n, b):
    from charmlu_b200.distributed import CudaBlocks
    return CudaBlocks(n, b)


def _rand(shape, seed, scale=1.0):
    g = torch.Generator(device="cuda").manual_seed(seed)
    return (torch.rand(*shape, dtype=torch.float64, device="cuda", generator=g) - 0.5) * scale


def _even(rows, cols, seed):
    """rows x cols view of a buffer with an even row pitch."""
    buf = _rand((rows, cols + (cols & 1)), seed)
    return buf[:, :cols]


@pytest.mark.parametrize("M,N,K", [(300, 130, 70), (1024, 512, 256), (7, 3, 2)])
def test_gemm_update_matches_torch(cuda_dev, M, N, K):
    bl = _blocks(2048, 64)
    A, B, C = _even(M, K, 1), _even(K, N, 2), _even(M, N, 3)
    ref = C - A @ B
    bl.gemm_update(A, B, C)
    torch.cuda.synchronize()
    assert (C - ref).abs().max().item() <= 1e-13 * K


@pytest.mark.parametrize("w,ncols", [(64, 300), (200, 33), (2, 5)])
def test_trsm_and_trsv_blocks_match_scipy(cuda_dev, w, ncols):
    bl = _blocks(2048, 64)
    L = _even(w, w, 4)
    L.fill_diagonal_(1.0)
    B = _even(w, ncols, 5)
    ref = sl.solve_triangular(L.cpu().numpy(), B.cpu().numpy(), lower=True, unit_diagonal=True)
    bl.trsm_lower_unit(L, B)
    x = _rand((w,), 6)
    U = _even(w, w, 7)
    U.add_(torch.eye(w, dtype=torch.float64, device="cuda") * w)  # well conditioned
    xr = sl.solve_triangular(U.cpu().numpy(), x.cpu().numpy(), lower=False)
    bl.trsv_block(U, 1, x)
    y = _rand((w,), 8)
    yr = sl.solve_triangular(L.cpu().numpy(), y.cpu().numpy(), lower=True, unit_diagonal=True)
    bl.trsv_block(L, 0, y)
    torch.cuda.synchronize()
    assert np.abs(B.cpu().numpy() - ref).max() <= 1e-11 * max(1.0, np.abs(ref).max())
    assert np.abs(x.cpu().numpy() - xr).max() <= 1e-13 * max(1.0, np.abs(xr).max())
    assert np.abs(y.cpu().numpy() - yr).max() <= 1e-11 * max(1.0, np.abs(yr).max())


def test_gemv_update_matches_torch(cuda_dev):
    bl = _blocks(2048, 64)
    for m, k in ((1000, 64), (33, 7), (5, 1)):
        A, x, y = _even(m, k, 9), _rand((k,), 10), _rand((m,), 11)
        ref = y - A @ x
        bl.gemv_update(A, x, y)
        torch.cuda.synchronize()
        assert (y - ref).abs().max().item() <= 1e-14 * k


@pytest.mark.parametrize("m,w,base", [(500, 64, 0), (777, 130, 1000), (64, 64, 3)])
def test_panel_factor_and_pivots_match_lapack(cuda_dev, m, w, base):
    bl = _blocks(4096, 256)
    P = _even(m, w, 12)
    P0 = P.cpu().numpy().copy()
    ipiv = torch.zeros(w, dtype=torch.int32, device="cuda")
    bl.panel_factor(P, ipiv, base)
    torch.cuda.synchronize()
    assert bl.status() == 0
    lu_ref, piv_ref = sl.lu_factor(P0)
    assert np.array_equal(ipiv.cpu().numpy(), piv_ref[:w].astype(np.int32) + base)
    got = P.cpu().numpy()
    assert np.abs(got - lu_ref[:, :w]).max() <= 1e-12 * max(1.0, np.abs(lu_ref).max())
    # the same interchanges applied to other columns and to a vector
    A = _even(m, 50, 13)
    A0 = A.cpu().numpy().copy()
    v = _rand((m,), 14)
    v0 = v.cpu().numpy().copy()
    rel = (ipiv - base).contiguous()  # swaps i <-> rel[i] among A's m rows
    bl.apply_pivots(A, 50, rel, 0, w, 10, 20, v)
    torch.cuda.synchronize()
    for j, p in enumerate(piv_ref[:w]):
        A0[[j, p], :] = A0[[p, j], :]
        v0[[j, p]] = v0[[p, j]]
    got = A.cpu().numpy()
    keep = [c for c in range(50) if not 10 <= c < 20]
    assert np.array_equal(got[:, keep], A0[:, keep])
    assert np.array_equal(v.cpu().numpy(), v0)


_PORTS = iter(range(33000 + (os.getpid() % 500) * 8, 33000 + (os.getpid() % 500) * 8 + 8))


def test_apply_pivots_rejects_rows_outside_the_matrix(cuda_dev):
    """A pivot naming a row at or past m (or before its own position) is
    caught before anything moves: the batch is left unapplied and the status
    word reports LU_ERR_ARG."""
    import charmlu_b200 as lu
    bl = _blocks(1024, 64)
    m = 100
    A = _even(m, 40, 15)
    A0 = A.clone()
    ipiv = torch.arange(8, dtype=torch.int32, device="cuda")
    ipiv[3] = m  # one past the last row
    bl.apply_pivots(A, 40, ipiv, 0, 8, 0, 0)
    assert bl.status() == lu.LU_ERR_ARG
    assert torch.equal(A, A0)


@pytest.fixture()
def one_rank_group():
    """A one-rank NCCL process group (a fresh store port per test)."""
    if not dist.is_initialized():
        dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{next(_PORTS)}", rank=0, world_size=1)
    yield
    dist.destroy_process_group()


@pytest.mark.parametrize("n,b,la", [(1000, 128, False), (1000, 128, True), (2048, 256, True)])
def test_block_cyclic_one_rank_matches_lu_factor(cuda_dev, one_rank_group, n, b, la):
    import charmlu_b200 as lu
    from charmlu_b200.distributed import BlockCyclicLU
    A = lu.generate_uniform(n, n, seed=17, stream_id=0)
    rhs = lu.generate_uniform(n, 1, seed=17, stream_id=1).view(-1)
    d = BlockCyclicLU(n, b, lookahead=la)
    loc = d.scatter(A)
    ipiv = d.factor(loc)
    assert d.status_code == 0
    x = d.solve(loc, ipiv, rhs)
    s = lu.LUSolver(lu.LUConfig(n, b))
    ref = A.clone()
    ipiv_ref = s.factor(ref)
    assert s.status() == 0
    assert torch.equal(ipiv, ipiv_ref)
    LU = loc[:, :n]
    if not la:
        assert torch.equal(LU, ref)
    else:
        assert (LU - ref).abs().max().item() <= 1e-12 * ref.abs().max().item() * n
    r = s.residual(A, x, rhs)
    assert r["r_hpl"] < 16, r
    xr = rhs.clone()
    s.solve(ref, ipiv_ref, xr)
    assert (x - xr).abs().max().item() <= 1e-10 * xr.abs().max().item()


def test_block_cyclic_one_rank_singular(cuda_dev, one_rank_group):
    import charmlu_b200 as lu
    from charmlu_b200.distributed import BlockCyclicLU
    n, b = 512, 64
    A = lu.generate_uniform(n, n, seed=3, stream_id=0)
    A[:, 300] = 0.0
    d = BlockCyclicLU(n, b)
    d.factor(d.scatter(A))
    assert d.status_code == 301


@pytest.mark.parametrize("n,b", [(1000, 128), (2048, 256)])
def test_block_cyclic_2d_one_rank_matches_lu_factor(cuda_dev, one_rank_group, n, b):
    """The 2D driver on a 1 x 1 grid: its panel gather, interchange exchange
    and U broadcast reduce to local copies, so it runs lu_factor's kernels
    on the same blocks: the same pivots, the factors equal to rounding."""
    import charmlu_b200 as lu
    from charmlu_b200.distributed import BlockCyclic2DLU
    A = lu.generate_uniform(n, n, seed=19, stream_id=0)
    rhs = lu.generate_uniform(n, 1, seed=19, stream_id=1).view(-1)
    d = BlockCyclic2DLU(n, b, 1, 1)
    loc = d.scatter(A)
    ipiv = d.factor(loc)
    assert d.status_code == 0
    x = d.solve(loc, ipiv, rhs)
    s = lu.LUSolver(lu.LUConfig(n, b))
    ref = A.clone()
    ipiv_ref = s.factor(ref)
    assert torch.equal(ipiv, ipiv_ref)
    LU = d.gather(loc)
    assert (LU - ref).abs().max().item() <= 1e-12 * ref.abs().max().item() * n
    r = s.residual(A, x, rhs)
    assert r["r_hpl"] < 16, r

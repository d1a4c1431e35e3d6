"""The 2D block-cyclic multi-GPU LU (charmlu_b200/distributed.py,
BlockCyclic2DLU) on CPU: gloo ranks on P x Q process grids run the
driver's distribution (the panel gathered and factored in its process
column, panel and pivots broadcast along process rows, interchanges of rows
held by different process rows, the U block row broadcast down process
columns, the replicated-b solve) with a numpy stand-in for the per-block
kernels. Checked against LAPACK getrf (scipy): the same pivots, the same
L\\U to rounding, x against numpy.linalg.solve, and the first singular
column reported as lu_factor reports it."""
import os

import numpy as np
import pytest
import scipy.linalg as sl
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from numpy_blocks import NumpyBlocks

# (n, b, zero column): ragged last blocks, ranks holding no block, a
# singular matrix
CASES = [(96, 8, None), (101, 16, None), (40, 4, None), (12, 8, None), (64, 8, 29)]
GRIDS = {4: [(2, 2), (1, 4), (4, 1)], 2: [(1, 2), (2, 1)]}


def _matrix(n, seed, zero_col):
    A = np.random.default_rng(seed).uniform(-0.5, 0.5, (n, n))
    if zero_col is not None:
        A[:, zero_col] = 0.0
    return A


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from charmlu_b200.distributed import BlockCyclic2DLU
    try:
        out = {}
        for (P, Q) in GRIDS[world]:
            for i, (n, b, zero_col) in enumerate(CASES):
                A = _matrix(n, 300 + i, zero_col)
                bvec = np.random.default_rng(400 + i).uniform(-0.5, 0.5, n)
                d = BlockCyclic2DLU(n, b, P, Q, blocks=NumpyBlocks(), device="cpu")
                loc = d.scatter(torch.from_numpy(A))
                ipiv = d.factor(loc)
                LU = d.gather(loc).numpy()
                x = d.solve(loc, ipiv, torch.from_numpy(bvec)).numpy() if zero_col is None else None
                out[(P, Q, i)] = (LU, ipiv.numpy().copy(), x, d.status_code, d.nrows, d.ncols)
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 4])
def test_block_cyclic_2d_lu_gloo_ranks(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 46000 + world * 100 + (os.getpid() % 97)
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert sorted(res) == list(range(world))
    for (P, Q) in GRIDS[world]:
        for i, (n, b, zero_col) in enumerate(CASES):
            key = (P, Q, i)
            A = _matrix(n, 300 + i, zero_col)
            bvec = np.random.default_rng(400 + i).uniform(-0.5, 0.5, n)
            # every block is held once: the ranks' rows x columns add up to n x n
            assert sum(res[r][key][4] * res[r][key][5] for r in range(world)) == n * n
            for r in range(1, world):
                assert np.array_equal(res[r][key][0], res[0][key][0]), key
                assert np.array_equal(res[r][key][1], res[0][key][1]), key
                assert res[r][key][3] == res[0][key][3]
                if res[0][key][2] is not None:
                    assert np.array_equal(res[r][key][2], res[0][key][2]), key
            LU, ipiv, x, status, _, _ = res[0][key]
            if zero_col is not None:
                assert status == zero_col + 1, (key, status)
                continue
            assert status == 0, key
            lu_ref, piv_ref = sl.lu_factor(A)
            assert np.array_equal(ipiv, piv_ref.astype(np.int32)), key
            assert np.abs(LU - lu_ref).max() <= 1e-12 * max(1.0, np.abs(lu_ref).max()) * n, key
            xr = np.linalg.solve(A, bvec)
            assert np.abs(x - xr).max() <= 1e-10 * np.abs(xr).max(), key


def test_2d_layout_without_process_group():
    """Row and column blocks per grid position, local offsets, the global
    row of every local row (pure arithmetic, as the driver computes them)."""
    n, b = 1000, 64
    nb = (n + b - 1) // b
    for P, Q in ((2, 3), (4, 2), (1, 1)):
        total = 0
        for r in range(P * Q):
            pr, pc = divmod(r, Q)
            rb = [i for i in range(nb) if i % P == pr]
            cb = [j for j in range(nb) if j % Q == pc]
            rows = sum(min(b, n - i * b) for i in rb)
            cols = sum(min(b, n - j * b) for j in cb)
            total += rows * cols
            offs, off = [], 0
            for j in cb:
                offs.append(off)
                off += min(b, n - j * b)
            assert all(o % 2 == 0 for o in offs)  # 16-byte aligned column views
        assert total == n * n

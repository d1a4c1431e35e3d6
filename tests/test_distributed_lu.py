"""The 1D block-cyclic multi-GPU LU (charmlu_b200/distributed.py) on CPU:
world_size 2 and 4 gloo ranks run the driver's distribution (which rank
factors which panel, the panel and pivot broadcasts, row interchanges across
every rank's columns, look-ahead ordering, the replicated-b solve) with a
numpy stand-in for the per-block kernels. Checked against LAPACK getrf
(scipy): the same pivots, the same L\\U to rounding, x against
numpy.linalg.solve, and the first singular column reported as lu_factor
reports it. The kernels themselves are checked on the GPU through the C ABI
(tests/test_gpu_distributed.py)."""
import os

import numpy as np
import pytest
import scipy.linalg as sl
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from numpy_blocks import NumpyBlocks


# (n, b, look-ahead, zero column): ragged last blocks, ranks that own no
# block (n <= b at world 2; 3 blocks at world 4), a singular matrix
CASES = {
    2: [(200, 16, True, None), (200, 16, False, None), (64, 8, True, 21), (130, 64, True, None),
        (6, 8, True, None)],
    4: [(97, 8, True, None), (97, 8, False, None), (40, 4, True, None), (20, 8, True, None),
        (20, 8, False, None)],
}


def _matrix(n, seed, zero_col):
    A = np.random.default_rng(seed).uniform(-0.5, 0.5, (n, n))
    if zero_col is not None:
        A[:, zero_col] = 0.0
    return A


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from charmlu_b200.distributed import BlockCyclicLU
    try:
        out = []
        for i, (n, b, la, zero_col) in enumerate(CASES[world]):
            A = _matrix(n, 100 + i, zero_col)
            bvec = np.random.default_rng(200 + i).uniform(-0.5, 0.5, n)
            d = BlockCyclicLU(n, b, blocks=NumpyBlocks(), device="cpu", lookahead=la)
            loc = d.scatter(torch.from_numpy(A))
            ipiv = d.factor(loc)
            LU = d.gather(loc).numpy()
            x = d.solve(loc, ipiv, torch.from_numpy(bvec)).numpy() if not zero_col else None
            out.append((LU, ipiv.numpy().copy(), x, d.status_code, d.ncols))
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 4])
def test_block_cyclic_lu_gloo_ranks(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 40000 + world * 1000 + (os.getpid() % 1000)  # clear of the other gloo tests' ports
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert sorted(res) == list(range(world))
    for i, (n, b, la, zero_col) in enumerate(CASES[world]):
        A = _matrix(n, 100 + i, zero_col)
        bvec = np.random.default_rng(200 + i).uniform(-0.5, 0.5, n)
        nb = (n + b - 1) // b
        # every rank holds its share of the columns and the same replicated results
        assert sum(res[r][i][4] for r in range(world)) == n
        for r in range(1, world):
            assert np.array_equal(res[r][i][0], res[0][i][0]) and np.array_equal(res[r][i][1], res[0][i][1])
            assert res[r][i][3] == res[0][i][3]
            if res[0][i][2] is not None:
                assert np.array_equal(res[r][i][2], res[0][i][2])
        LU, ipiv, x, status, _ = res[0][i]
        if zero_col is not None:
            assert status == zero_col + 1, (status, zero_col)
            continue
        assert status == 0
        lu_ref, piv_ref = sl.lu_factor(A)
        assert np.array_equal(ipiv, piv_ref.astype(np.int32)), (n, b, la, nb)
        assert np.abs(LU - lu_ref).max() <= 1e-12 * max(1.0, np.abs(lu_ref).max()) * n
        xr = np.linalg.solve(A, bvec)
        assert np.abs(x - xr).max() <= 1e-10 * np.abs(xr).max()


def test_layout_owners_and_offsets():
    """Owned blocks, local column offsets and widths for a ragged last block,
    without a process group (the layout is pure arithmetic)."""
    from charmlu_b200.distributed import BlockCyclicLU

    class Fake(BlockCyclicLU):
        def __init__(self, n, b, rank, world):
            self.n, self.b, self.rank, self.world = n, b, rank, world
            self.nb = (n + b - 1) // b
            self.owned = [j for j in range(self.nb) if j % world == rank]
            self.col_off, off = {}, 0
            for j in self.owned:
                self.col_off[j] = off
                off += self.width(j)
            self.ncols = off

    n, b = 1000, 64
    total = 0
    for world in (1, 3, 8):
        cols = []
        for r in range(world):
            f = Fake(n, b, r, world)
            cols.append(f.ncols)
            assert all(f.owner(j) == r for j in f.owned)
            assert f._trailing_start(f.nb) == f.ncols
            for j in f.owned:
                assert f.col_off[j] % 2 == 0  # 16-byte aligned views in an even-pitch row
        total = sum(cols)
        assert total == n

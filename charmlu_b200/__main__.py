"""Command-line drop-in for charmlu's driver.

    python -m charmlu_b200 <matrix size> <block size> <mem threshold>
                           [<pivot batch size> <mapping scheme> [<peTileRows> <peTileCols> <peRotate> <peStride>]]
                           [--precision fp64|bf16|fp16s|fp16x3] [--seed S] [--json]

Same positional arguments as charmlu (benchmark.C:81-134); the memory
threshold, mapping scheme and PE-tile arguments configure Charm++ placement
and are accepted and ignored.  Under torchrun with several processes (one
per GPU, as charmrun +pN gives the reference N PEs) the FP64 solve runs on
the 1D block-cyclic driver over NCCL (charmlu_b200.distributed) and rank 0
prints the result lines.  Prints the reference's result
lines (benchmark.C:150-184, 343-400: configuration, time and GFlop/s, the
per-machine fraction of peak, the block DGEMM self-benchmark, residual and
validation time), including the
``residual = %f`` line that test_lu.pl parses (test_lu.pl:76-77).  A is the
counter-based uniform[-0.5,0.5) matrix; b is the reference's MatGen stream
(seed 9934835, benchmark.C:455-460).
"""
import argparse
import json
import os
import sys
import time


# Per-core peaks (GFlop/s) of the machines the reference reports its
# fraction of peak against (benchmark.C:361-367): machine constants, kept so
# the output has the same lines.
MACHINE_PEAKS = [("Order", 7.4585), ("Abe", 9.332), ("Ranger", 9.2), ("Jaguar/Kraken XT5", 10.3987),
                 ("BG/P", 3.4), ("Jaguar XK6 sans GPUs", 8.8)]


def _pe_tile(procs, tile):
    """PE tile of mapping scheme 3 (benchmark.C:101-127): rows, cols, rotate,
    stride, with the reference's defaults (benchmark.C:193-212: the
    process count as a near-square product, the larger factor as rows, when
    no dimensions are given)."""
    if len(tile) >= 2:
        rows, cols = tile[0], tile[1]
    else:
        f1 = max(d for d in range(1, int(procs ** 0.5) + 1) if procs % d == 0)
        rows = max(f1, procs // f1)
        cols = procs // rows
    rotate = tile[2] if len(tile) >= 3 else 0
    stride = tile[3] if len(tile) >= 4 else cols
    return rows, cols, rotate, stride


def _header(n, b, batch, mem, mapping, procs, tile=()):
    """The configuration lines the reference prints before the solve
    (benchmark.C:150-184)."""
    print("Running LU compiled from revision: charmlu_b200")
    print(f"Running LU on {procs} processors (1 nodes): \n\tMatrix size: {n} X {n} \n\tBlock size: {b} X {b} "
          f"\n\tChare Array size: {n // b} X {n // b}\n\tPivot batch size: {batch}\n\tMem Threshold (MB): {mem}"
          f"\n\tSend Limit: 0\n\tMapping Scheme: {mapping} ({'Block Cyclic' if mapping == 2 else '2D Tiling'})")
    if mapping == 3:
        r, c, rot, stride = _pe_tile(procs, tile)
        print(f"\tMapping PE tile size: {r} x {c} rotate {rot} stride {stride} ")
    # the pivot reduction is not scheduled and U rows leave from the diagonal
    # (the reference's default build, benchmark.C:173-182)
    print("\tPivot Redn Scheduling: Off")
    print("\tUseg Multicast from: Diagonal")


def dgemm_block_time(b, trials=10):
    """Seconds for one b x b x b C -= A B on this GPU's FP64 trailing-update
    kernel (lu_gemm_update), averaged over `trials` launches timed with CUDA
    events: the counterpart of the reference's testdgemm, which times one
    block-sized cblas_dgemm (benchmark.C:298-341)."""
    import torch
    import charmlu_b200 as lu
    from charmlu_b200.blocks import CudaBlocks
    ld = b + (b & 1)
    blk = CudaBlocks(max(b, 2), max(b, 2))
    try:
        mats = [lu.generate_uniform(b, ld, seed=0, stream_id=i)[:, :b] for i in range(3)]
        c, a, bb = mats
        blk.gemm_update(a, bb, c)  # warm the kernel
        total = 0.0
        for _ in range(trials):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            blk.gemm_update(a, bb, c)
            e1.record()
            e1.synchronize()
            total += e0.elapsed_time(e1) / 1e3
        return total / trials
    finally:
        blk.close()


def _report(n, b, procs, dt, st, r, eps, dgemm_s=None):
    """The result lines of the reference (benchmark.C:343-400): time and HPL
    GFlop/s, fraction of each listed machine's per-core peak, the block
    DGEMM self-benchmark, the scaled residual and the validation time."""
    if st > 0:
        print("Diagonal element very small despite pivoting. Is the matrix singular??")
    gflops = (2.0 / 3.0 * n ** 3 + 1.5 * n ** 2) / dt / 1e9
    per_core = gflops / procs
    print("RESULT procs: \t%d\tblock size:\t%d\tTime(s):\t%g" % (procs, b, dt))
    print("HPL flop count gives \t%g\tGFlops" % gflops)
    for machine, peak in MACHINE_PEAKS:
        print("%s:\t%g%% of peak" % (machine, 100.0 * per_core / peak))
    if dgemm_s:
        dg = 2.0 * b * b * b / 1e9 / dgemm_s
        print("The dgemm %d x %d takes %g ms and achieves %g GFlop/sec" % (b, b, dgemm_s * 1e3, dg))
        print("Percent of DGEMM is: %g%%" % (per_core / dg * 100.0))
    print(f"epsilon = {eps:e}\nresidual = {r['r_ref']:f}")
    if r["r_ref"] > 16:
        print("=== WARNING: Scaled residual is greater than 16 - OUT OF SPEC ===")
    print("finished validation at wall time: %f" % (time.monotonic() - _T_START))
    print(f"r_hpl = {r['r_hpl']:f}")
    return gflops


_T_START = time.monotonic()


def _main_ranks(n, b, mem, batch, mapping, a, world):
    """The FP64 solve over `world` GPUs, one process each (torchrun)."""
    import datetime
    import torch
    import torch.distributed as dist
    import charmlu_b200 as lu
    from charmlu_b200.distributed import BlockCyclicLU
    if a.precision != "fp64":
        print("Only the FP64 solve runs over several GPUs; run one process for --precision", a.precision)
        return 1
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group("nccl", device_id=dev, timeout=datetime.timedelta(seconds=120))
    try:
        if rank == 0:
            _header(n, b, batch, mem, mapping, world, a.positional[5:9])
        # the local set-up can fail on one rank only (memory, arguments): the
        # ranks agree on that before the first collective of the solve, so
        # none is left waiting for a rank that has already given up
        err = None
        try:
            d = BlockCyclicLU(n, b, lookahead=True)
            A = lu.generate_uniform(n, n, seed=a.seed, stream_id=0, device=dev)
        except Exception as e:  # reported after the agreement below
            err = e
        flag = torch.tensor([1 if err is not None else 0], dtype=torch.int32, device=dev)
        dist.all_reduce(flag, op=dist.ReduceOp.MAX)
        if int(flag.item()):
            print(f"rank {rank}: set-up failed on {'this' if err is not None else 'another'} rank: {err}",
                  file=sys.stderr)
            return 1
        loc = d.scatter(A)
        bvec = torch.from_numpy(lu.matgen(n)).to(dev)
        if rank == 0:
            print("Starting solve")
        dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ipiv = d.factor(loc)
        x = d.solve(loc, ipiv, bvec)
        torch.cuda.synchronize()
        dist.barrier()
        dt = time.perf_counter() - t0
        if rank == 0:
            r = lu.LUSolver(lu.LUConfig(n, b)).residual(A, x, bvec)
            gflops = _report(n, b, world, dt, d.status_code, r, lu.EPS, dgemm_block_time(b))
            if a.json:
                print(json.dumps({"n": n, "b": b, "precision": "fp64", "procs": world, "time_s": dt,
                                  "gflops_ref_count": gflops, "status": d.status_code, **r}))
            print("Finished solve")
    finally:
        dist.destroy_process_group()
    return 0


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    ap = argparse.ArgumentParser(prog="charmlu_b200", add_help=True)
    ap.add_argument("positional", nargs="*", type=int)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "bf16", "fp16s", "fp16x3"])
    ap.add_argument("--seed", type=int, default=42)
    ap.add_argument("--json", action="store_true")
    a = ap.parse_args(argv)
    if len(a.positional) < 3:
        print("Usage: charmlu_b200 <matrix size> <block size> <mem threshold> [<pivot batch size> <mapping scheme>"
              " [<peTileRows> <peTileCols> <peRotate> <peStride>] ]")
        return 0
    n, b, mem = a.positional[:3]
    batch = a.positional[3] if len(a.positional) >= 4 else b // 4
    mapping = a.positional[4] if len(a.positional) >= 5 else 2
    if b <= 0 or n <= 0:
        print(f"The matrix size {n} should be a multiple of block size {b}!")
        return 0
    if n % b != 0:
        # the reference refuses (benchmark.C:143-147); the same check is kept for drop-in behaviour
        print(f"The matrix size {n} should be a multiple of block size {b}!")
        return 0

    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1:
        return _main_ranks(n, b, mem, batch, mapping, a, world)

    import torch
    import charmlu_b200 as lu
    prec = {"fp64": lu.LU_PREC_FP64, "bf16": lu.LU_PREC_BF16, "fp16s": lu.LU_PREC_FP16S,
            "fp16x3": lu.LU_PREC_FP16X3}[a.precision]
    _header(n, b, batch, mem, mapping, 1, a.positional[5:9])
    A = lu.generate_uniform(n, n, seed=a.seed, stream_id=0)
    bvec = torch.from_numpy(lu.matgen(n)).cuda()
    A0 = A.clone()
    x = bvec.clone()
    blk = b if prec == lu.LU_PREC_FP64 or b % 64 == 0 else 64 * max(1, b // 64)
    s = lu.LUSolver(lu.LUConfig(n, blk, pivot_batch_size=batch, mem_threshold=mem, precision=prec))
    print("Starting solve")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    info = None
    if prec == lu.LU_PREC_FP64:
        s.factor_solve(A, x)
    else:
        x, info = s.refine_solve(A0, bvec)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    st = s.status()
    r = s.residual(A0, x, bvec)
    gflops = _report(n, b, 1, dt, st, r, lu.EPS, dgemm_block_time(b))
    if a.json:
        print(json.dumps({"n": n, "b": b, "precision": a.precision, "time_s": dt, "gflops_ref_count": gflops,
                          "tflops": (2 / 3 * n ** 3 + 2 * n ** 2) / dt / 1e12, "status": st, "refine": info, **r}))
    print("Finished solve")
    return 0


if __name__ == "__main__":
    sys.exit(main())

"""Benchmark: dense LU with partial pivoting + solve at N=65536 on one B200.

Metric (BASELINE): "N=65536 solve TFLOP/s & time: BF16+FP64-IR vs FP64 LU,
HPL resid<16".  One step = one time-to-solution pass over the N=65536
system (A, b i.i.d. uniform[-0.5,0.5), seed 42), the span charmlu times
(benchmark.C:243 -> 344: factor, then solve).  TFLOP/s = (2/3 N^3 + 2 N^2)
/ time.  Inputs are resident in HBM for `value`; `e2e` repeats the metric
through the public API from pinned host buffers with the copies timed.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--n 65536] [--block 256] [--mode fp64|mixed]

N > 1 GPUs (torchrun): replicas only — the single-matrix LU does not shard
into independent units; every rank solves its own system, value = all ranks'
flops / the slowest rank's time.  `--impl reference` times the CPU
restatement of charmlu's algorithm (charmlu itself cannot be built: no
Charm++ runtime) on the host cores, rank 0 only.
"""
import argparse
import json

import numpy as np
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "N=65536 solve TFLOP/s & time: BF16+FP64-IR vs FP64 LU, HPL resid<16"


def flops_lu(n):
    return 2.0 / 3.0 * n ** 3 + 2.0 * n ** 2


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index=0):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        sm.sort()
        med = sm[len(sm) // 2] if sm else None
        return {"sm_mhz": med, "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(n_sample=8192, b=256, reps=2):
    """The oracle (CPU restatement of charmlu's blocked LU, OpenBLAS per block,
    OpenMP over blocks like charmlu's PEs) on all host cores."""
    import numpy as np
    import oracle
    cores = os.cpu_count() or 1
    oracle.set_threads(cores)
    A = oracle.gen_matrix(n_sample, 42)
    rhs = oracle.gen_vector(n_sample, 42)
    best = None
    res = None
    for _ in range(reps):
        t0 = time.perf_counter()
        x, *_ = oracle.solve(A, rhs, b=b)
        dt = time.perf_counter() - t0
        best = dt if best is None else min(best, dt)
        res = oracle.residual(A, x, rhs)
    return {"value": flops_lu(n_sample) / best / 1e12, "unit": "TFLOP/s", "cores": cores, "kind": "port",
            "sample": f"N={n_sample} b={b} factor+solve (best of {reps}, {best:.2f} s each); "
                      f"r_hpl={res['r_hpl']:.3g}; the N=65536 step would take ~{flops_lu(65536) / (flops_lu(n_sample) / best) / 60:.0f} min on these cores"}


def fp64_c2_record(dev, peak64, steps=3, with_cpu=True):
    """The FP64 path at N=32768, b=256 (factor + solve with look-ahead,
    inputs resident in HBM, 8.6 GB > L2), timed with CUDA events, beside the
    CPU oracle at the same order run once on all host cores."""
    import torch
    import charmlu_b200 as lu
    n, b = 32768, 256
    A0 = lu.generate_uniform(n, n, seed=42, stream_id=0, device=dev)
    rhs0 = lu.generate_uniform(n, 1, seed=42, stream_id=1, device=dev).view(-1)
    A = torch.empty_like(A0)
    x = torch.empty_like(rhs0)
    s = lu.LUSolver(lu.LUConfig(n, b, lookahead=True))
    ms = []
    for k in range(1 + steps):
        A.copy_(A0)
        x.copy_(rhs0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        s.factor_solve(A, x)
        e1.record()
        torch.cuda.synchronize()
        if k:
            ms.append(e0.elapsed_time(e1))
    st = s.status()
    r = s.residual(A0, x, rhs0)
    t = sum(ms) / len(ms) / 1e3
    rec = {"n": n, "block_size": b, "lookahead": True, "steps": steps, "time_s": t,
           "tflops": flops_lu(n) / t / 1e12, "frac_of_fp64_peak": flops_lu(n) / t / 1e12 / peak64,
           "status": st, "r_hpl": r["r_hpl"], "r_ref": r["r_ref"]}
    x_gpu = x.cpu().numpy()
    del A0, A, x, rhs0
    s.close()
    torch.cuda.empty_cache()
    if with_cpu:
        import oracle
        cores = os.cpu_count() or 1
        oracle.set_threads(cores)
        Ah = oracle.gen_matrix(n, 42)
        bh = oracle.gen_uniform(n, 42, 1)
        t0 = time.perf_counter()
        xc, *_ = oracle.solve(Ah, bh, b=b)
        tc = time.perf_counter() - t0
        rc = oracle.residual(Ah, xc, bh)
        rec["cpu_same_n"] = {"kind": "port", "cores": cores, "time_s": tc, "tflops": flops_lu(n) / tc / 1e12,
                             "r_hpl": rc["r_hpl"], "gpu_speedup": tc / t,
                             "x_rel_diff_gpu_vs_cpu": float(abs(x_gpu - xc).max() / abs(xc).max()),
                             "sample": f"N={n} b={b} factor+solve, one run (the oracle restatement of charmlu)"}
    return rec


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    steps, warm = args.steps, args.warmup
    n_sample = args.ref_sample
    import oracle
    cores = os.cpu_count() or 1
    oracle.set_threads(cores)
    A = oracle.gen_matrix(n_sample, 42)
    rhs = oracle.gen_vector(n_sample, 42)
    for _ in range(warm):
        oracle.solve(A, rhs, b=args.block)
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        x, *_ = oracle.solve(A, rhs, b=args.block)
        times.append(time.perf_counter() - t0)
    r = oracle.residual(A, x, rhs)
    tot = sum(times)
    val = flops_lu(n_sample) * steps / tot / 1e12
    line = {
        "metric": METRIC, "value": val, "unit": "TFLOP/s", "n_gpus": world, "steps": steps, "warmup": warm,
        "ms_per_step": tot / steps * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic uniform[-0.5,0.5) seed 42", "impl": "reference",
        "config": {"workload": f"N={args.n} dense LU+solve; CPU sample N={n_sample} b={args.block} per step",
                   "n": args.n, "sample_n": n_sample, "block_size": args.block},
        "cpu_baseline": {"value": val, "unit": "TFLOP/s", "cores": cores, "kind": "port",
                         "sample": f"N={n_sample} b={args.block} factor+solve per step (charmlu cannot be built: "
                                   f"no Charm++ runtime; this is the oracle restatement)"},
        "e2e": {"value": val, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "r_hpl": r["r_hpl"], "r_ref": r["r_ref"],
    }
    print(json.dumps(line), flush=True)
    return 0


def batched_measure(n_all, mine, dev, dist, steps, warmup, world=1):
    """Time the batched solver on this rank's systems (indices `mine` of the
    orders n_all): one persistent launch, captured in a CUDA graph and
    replayed, in FP64 and in FP32 with FP64 refinement.  Returns per mode the
    mean replay time (max over ranks), throughput on all systems, failures
    and the largest per-system scaled residual, plus the buffers."""
    import numpy as np
    import torch
    import charmlu_b200 as lu
    from charmlu_b200.batched import BatchedSystems, flops, gather_results, partition_by_cost
    n = n_all[mine]
    # the global data set (counter-based generator), this rank's systems copied out
    g = BatchedSystems(n_all, device=dev)
    gA = lu.generate_uniform(1, g.total_a, seed=42, stream_id=30, device=dev).view(-1)
    gb = lu.generate_uniform(1, g.total_b, seed=42, stream_id=31, device=dev).view(-1)
    bs = BatchedSystems(n, device=dev)
    A0 = torch.empty(bs.total_a, dtype=torch.float64, device=dev)
    b0 = torch.empty(bs.total_b, dtype=torch.float64, device=dev)
    for q, i in enumerate(mine):
        k = int(n_all[i])
        A0[bs.a_off[q]:bs.a_off[q] + k * k].copy_(gA[g.a_off[i]:g.a_off[i] + k * k])
        b0[bs.b_off[q]:bs.b_off[q] + k].copy_(gb[g.b_off[i]:g.b_off[i] + k])
    del gA, gb, g
    A, b = A0.clone(), b0.clone()
    F_all = flops(n_all)
    out = {}
    for name, prec in (("fp64", lu.LU_PREC_FP64), ("fp32_ir", lu.LU_PREC_FP32)):
        A.copy_(A0)
        b.copy_(b0)
        bs.factor_solve(A, b, prec)  # warm-up outside capture (tuning upload, attributes)
        torch.cuda.synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            bs.factor_solve(A, b, prec)
        ms = []
        for k in range(warmup + steps):
            A.copy_(A0)
            b.copy_(b0)
            torch.cuda.synchronize()
            if dist:
                dist.barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            graph.replay()
            e1.record()
            torch.cuda.synchronize()
            t = torch.tensor([e0.elapsed_time(e1)], device=dev)
            if dist:
                dist.all_reduce(t, op=dist.ReduceOp.MAX)
            if k >= warmup:
                ms.append(float(t))
        # every system's scaled residual against the untouched FP64 data
        res = np.empty(len(n))
        for q in range(len(n)):
            k = int(n[q])
            Ai = A0[bs.a_off[q]:bs.a_off[q] + k * k].view(k, k)
            bi = b0[bs.b_off[q]:bs.b_off[q] + k]
            xi = b[bs.b_off[q]:bs.b_off[q] + k]
            r = (bi - Ai @ xi).abs().max()
            den = (Ai.abs().sum(1).max() * xi.abs().max() + bi.abs().max()) * k * 2.220446049250313e-16
            res[q] = float(r / den)
        g_info, g_res = gather_results(mine, bs.info.cpu().numpy(), res, len(n_all))
        t = sum(ms) / len(ms)
        out[name] = {"ms": t, "tflops": F_all / (t / 1e3) / 1e12, "systems_per_s": len(n_all) / (t / 1e3),
                     "bad_systems": int((g_info != 0).sum()), "r_hpl_max": float(np.nanmax(g_res)),
                     "systems_per_rank": [int(len(p)) for p in partition_by_cost(n_all, world)]}
        if prec == lu.LU_PREC_FP32:
            # systems that met r_hpl < 16 after 0, 1, 2, ... FP64 refinement
            # steps (this rank's share), the last entry not at all
            hist = bs.refine_histogram().tolist()
            out[name]["refine_steps_histogram"] = hist
            out[name]["systems_needing_more_than_one_step"] = int(sum(hist[2:]))
        del graph
    return out, bs, A, b, A0, b0


def run_batched(args, rank, world):
    """4096 independent systems, orders log-uniform in [32, 1024] (seed 42),
    one RHS each, factored and solved in one persistent launch replayed from
    a CUDA graph; FP64 and FP32-factor + FP64-refinement; against a loop of
    the single-matrix path on the same GPU.  With N > 1 GPUs the one set of
    systems is split by cost (partition_by_cost): no collective but a final
    gather of per-system status and scaled residual; time = max over ranks
    (strong scaling: total work fixed)."""
    import numpy as np
    import torch
    import charmlu_b200 as lu
    from charmlu_b200.batched import BatchedSystems, flops, gather_results, log_uniform_orders, partition_by_cost
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", device_id=dev, timeout=datetime.timedelta(seconds=300))
    n_all = log_uniform_orders(args.batch_count, 32, 1024, seed=42)
    mine = partition_by_cost(n_all, world)[rank]
    out, bs, A, b, A0, b0 = batched_measure(n_all, mine, dev, dist, args.steps, args.warmup, world)
    n = n_all[mine]
    F_all = flops(n_all)
    loop_ms = None
    if world == 1:
        # a loop of the single-matrix path (one handle per distinct order, created before timing)
        A.copy_(A0)
        b.copy_(b0)
        handles = {}
        for k in sorted(set(n.tolist())):
            handles[k] = lu.LUSolver(lu.LUConfig(int(k), 64 if k >= 64 else max(2, k - (k & 1))))
        views = []
        for i in range(len(n)):
            k = int(n[i])
            Av = A[bs.a_off[i]:bs.a_off[i] + k * k].view(k, k)
            if k % 2 or (Av.data_ptr() % 16):
                # the single-matrix path wants a 16-byte aligned base and an even
                # row pitch: padded copy made before timing
                pad = torch.zeros(k, k + (k & 1), dtype=torch.float64, device=A.device)
                pad[:, :k] = Av
                Av = pad[:, :k]
            views.append((handles[k], Av, b[bs.b_off[i]:bs.b_off[i] + k]))
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for h, Av, bv in views:
            h.factor_solve(Av, bv)
        e1.record()
        torch.cuda.synchronize()
        loop_ms = e0.elapsed_time(e1)
    if rank == 0:
        line = {"metric": "batched uneven solves: 4096 systems, n log-uniform [32,1024], TFLOP/s",
                "unit": "TFLOP/s", "value": out["fp64"]["tflops"], "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": out["fp64"]["ms"], "higher_is_better": True,
                "scaling": "strong", "dtype": "f64", "data": "synthetic uniform[-0.5,0.5) seed 42",
                "config": {"workload": "batched", "count": int(len(n_all)), "n_min": int(n_all.min()),
                           "n_max": int(n_all.max()), "sum_flops": F_all, "graph": True,
                           "parallelism": f"systems split by cost over {world} GPU(s)"},
                "fp64": out["fp64"], "fp32_ir": out["fp32_ir"]}
        if loop_ms is not None:
            line["single_matrix_loop"] = {"ms": loop_ms, "systems": int(len(n)),
                                          "note": "lu_factor_solve per system, b=64, one handle per distinct order"}
            line["speedup_vs_loop"] = loop_ms / out["fp64"]["ms"]
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def kappa_matrix(n, kappa, seed, dev):
    """A = Q1 diag(sigma) Q2^T, Q from QR of seeded Gaussian matrices, sigma
    geometric from 1 to 1/kappa (generated with torch on the GPU: input
    construction only)."""
    import torch
    g = torch.Generator(device=dev).manual_seed(seed)
    Q1, _ = torch.linalg.qr(torch.randn(n, n, dtype=torch.float64, device=dev, generator=g))
    Q2, _ = torch.linalg.qr(torch.randn(n, n, dtype=torch.float64, device=dev, generator=g))
    sig = torch.logspace(0, -float(np.log10(kappa)), n, dtype=torch.float64, device=dev)
    return ((Q1 * sig) @ Q2.T).contiguous()


def run_ksweep(args, rank, world):
    """kappa sweep of the mixed path (BASELINE config 3 side sweep)."""
    import scipy.linalg as sl
    import torch
    import charmlu_b200 as lu
    if rank != 0:
        return 0
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    n = args.ksweep_n
    rows = []
    precs = [("bf16", lu.LU_PREC_BF16), ("fp16s", lu.LU_PREC_FP16S), ("fp16x3", lu.LU_PREC_FP16X3)]
    for kappa in (1e2, 1e6, 1e10):
        A = kappa_matrix(n, kappa, 1234, dev)
        b = lu.generate_uniform(n, 1, seed=42, stream_id=1, device=dev).view(-1)
        x_ref = sl.solve(A.cpu().numpy(), b.cpu().numpy(), check_finite=False)  # FP64 LAPACK oracle solution
        for name, prec in precs:
            s = lu.LUSolver(lu.LUConfig(n, 512, precision=prec, ir_max_iter=args.ksweep_iters))
            x = torch.empty_like(b)
            s.refine_solve(A, b, x)  # warm (allocations)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            _, info = s.refine_solve(A, b, x)
            e1.record()
            torch.cuda.synchronize()
            st = s.status()
            r = s.residual(A, x, b)
            fe = float(np.abs(x.cpu().numpy() - x_ref).max() / np.abs(x_ref).max())
            # ||I - M^{-1} A|| of these factors (power iteration on the kept
            # factors of a separate refine_factor): classical refinement
            # contracts by about this factor per step
            sk = lu.LUSolver(lu.LUConfig(n, 512, precision=prec))
            sk.refine_factor(A)
            try:
                pn = sk.refine_precond_norm(A, iters=15)
            except lu.LUError:
                pn = None
            del sk
            rows.append({"kappa": kappa, "precision": name, "status": st, "converged": st == 0,
                         "ir_iterations": info["iterations"], "gmres_iterations": info["gmres_iterations"],
                         "used_gmres": bool(info["used_gmres"]), "rejected_steps": info["rejected"],
                         "r_hpl": r["r_hpl"], "r_hpl_initial": info["r_hpl_initial"],
                         "r_hpl_not_above_initial": r["r_hpl"] <= info["r_hpl_initial"],
                         "forward_error_vs_fp64": fe, "norm_I_minus_Minv_A": pn,
                         "kappa_eps": kappa * 2.22e-16, "ms": e0.elapsed_time(e1)})
            print(json.dumps(rows[-1]), flush=True)
            del s
        del A
        torch.cuda.empty_cache()
    print(json.dumps({"metric": f"kappa sweep N={n}", "rows": rows}), flush=True)
    return 0


def _timed(fn):
    import torch
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    out = fn()
    e1.record()
    torch.cuda.synchronize()
    return out, e0.elapsed_time(e1)


def run_adjoint(args, rank, world):
    """Adjoint of X = A^{-1} B: FP64 at N=4096 with 16
    right-hand sides against the FP64 LAPACK gradient, then the mixed
    forward (low-precision factors + FP64 refinement) with the FP64-refined
    adjoint at N=32768 in factor-storing and refactor-in-backward modes,
    against the FP64 GPU path's gradient."""
    import scipy.linalg as sl
    import torch
    import charmlu_b200 as lu
    if rank != 0:
        return 0
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    k = 16
    rows = []

    def rel(a, b):
        return float((a - b).abs().max() / b.abs().max())

    # ---- FP64, N = 4096
    n = args.adjoint_n
    A = lu.generate_uniform(n, n, seed=42, stream_id=0, device=dev)
    B = lu.generate_uniform(n, k, seed=42, stream_id=2, device=dev)
    W = 2.0 * lu.generate_uniform(n, k, seed=42, stream_id=3, device=dev)
    s = lu.LUSolver(lu.LUConfig(n, 256))
    LU = A.clone()
    for _ in range(2):  # warm, then timed
        LU.copy_(A)
        (ipiv, t_fac) = _timed(lambda: s.factor(LU))
        X = B.clone()
        _, t_sol = _timed(lambda: s.solve(LU, ipiv, X))
        (gA, gB), t_adj = _timed(lambda: s.adjoint(LU, ipiv, X, W))
    assert s.status() == 0
    An, Wn = A.cpu().numpy(), W.cpu().numpy()
    f = sl.lu_factor(An)
    Xr = sl.lu_solve(f, B.cpu().numpy())
    lam = sl.lu_solve(f, Wn, trans=1)
    gA_ref, gB_ref = torch.from_numpy(-lam @ Xr.T), torch.from_numpy(lam)
    flops = 2 * (2 * n * n * k) + 2 * n * n * k
    rows.append({"case": f"fp64 N={n} nrhs={k}", "factor_ms": t_fac, "solve_ms": t_sol, "adjoint_ms": t_adj,
                 "adjoint_tflops": flops / t_adj / 1e9,
                 "adjoint_gbs": (2 * 8 * n * n + 8 * n * n) / t_adj / 1e6,
                 "rel_err_gradA": rel(gA.cpu(), gA_ref), "rel_err_gradB": rel(gB.cpu(), gB_ref)})
    print(json.dumps(rows[-1]), flush=True)
    del A, B, W, LU, X, gA, gB, s
    torch.cuda.empty_cache()

    # ---- mixed forward + FP64-refined adjoint, N = 32768
    n = args.adjoint_mixed_n
    if n <= 0:
        print(json.dumps({"metric": "adjoint of X = A^-1 B (FP64)", "rows": rows}), flush=True)
        return 0
    A = lu.generate_uniform(n, n, seed=42, stream_id=0, device=dev)
    B = lu.generate_uniform(n, k, seed=42, stream_id=2, device=dev)
    W = 2.0 * lu.generate_uniform(n, k, seed=42, stream_id=3, device=dev)
    # FP64 reference gradient from the FP64 GPU path (second pass timed)
    s64 = lu.LUSolver(lu.LUConfig(n, 256, lookahead=True))
    LU = A.clone()
    for _ in range(2):
        LU.copy_(A)
        ipiv, t64_fac = _timed(lambda: s64.factor(LU))
        X64 = B.clone()
        _, t64_sol = _timed(lambda: s64.solve(LU, ipiv, X64))
        (gA64, gB64), t64_adj = _timed(lambda: s64.adjoint(LU, ipiv, X64, W))
    assert s64.status() == 0
    gA64 = gA64.cpu()
    del LU, s64
    torch.cuda.empty_cache()
    # a tightly refined solution (scaled residual < 1e-5) as a third point:
    # the errors of both paths against it
    st = lu.LUSolver(lu.LUConfig(n, args.block_mixed, precision=lu.LU_PREC_FP16X3, lookahead=True, ir_target=1e-5,
                                 ir_max_iter=20))
    st.refine_factor(A)
    Xt, _ = st.refine_apply(A, B)
    Lt, _ = st.refine_apply(A, W, trans=True)
    st.close()
    del st
    torch.cuda.empty_cache()
    rows.append({"case": f"fp64 reference N={n} nrhs={k}", "factor_ms": t64_fac, "solve_ms": t64_sol,
                 "adjoint_ms": t64_adj, "forward_ms": t64_fac + t64_sol})
    print(json.dumps(rows[-1]), flush=True)
    prec = {"bf16": lu.LU_PREC_BF16, "fp16s": lu.LU_PREC_FP16S, "fp16x3": lu.LU_PREC_FP16X3}[args.precision]
    cfg = lu.LUConfig(n, args.block_mixed, precision=prec, lookahead=True, ir_target=args.adjoint_target)
    # one handle, warmed once (its workspace is allocated outside the timed
    # calls); refactor mode factors A again before the adjoint instead of
    # keeping the factors (the memory it saves is the FP32 copy, 4 n^2 B)
    s = lu.LUSolver(cfg)
    s.refine_factor(A)
    X, _ = s.refine_apply(A, B)
    s.refine_adjoint(A, X, W)
    del X
    torch.cuda.synchronize()
    for mode in ("storing", "refactor"):
        _, t_fac = _timed(lambda: s.refine_factor(A))
        (X, fi), t_app = _timed(lambda: s.refine_apply(A, B))
        t_ref = _timed(lambda: s.refine_factor(A))[1] if mode == "refactor" else 0.0
        (gA, gB, bi), t_adj = _timed(lambda: s.refine_adjoint(A, X, W))
        st = s.status()
        rows.append({"case": f"mixed {args.precision} N={n} nrhs={k} {mode}", "status": st,
                     "ir_target": args.adjoint_target,
                     "forward_ms": t_fac + t_app, "refine_factor_ms": t_fac, "refine_apply_ms": t_app,
                     "forward_ir_iterations": fi["iterations"], "forward_r_hpl": fi["r_hpl"],
                     "backward_ms": t_ref + t_adj, "backward_refactor_ms": t_ref, "adjoint_ms": t_adj,
                     "adjoint_ir_iterations": bi["iterations"], "adjoint_r_hpl": bi["r_hpl"],
                     "rel_err_X_vs_fp64": rel(X, X64), "rel_err_gradB_vs_fp64": rel(gB, gB64),
                     "rel_err_X_vs_tight": rel(X, Xt), "rel_err_gradB_vs_tight": rel(gB, Lt),
                     "fp64_path_rel_err_X_vs_tight": rel(X64, Xt), "fp64_path_rel_err_gradB_vs_tight": rel(gB64, Lt),
                     "rel_err_gradA_vs_fp64": rel(gA.cpu(), gA64),
                     "speedup_fwd_bwd_vs_fp64": (t64_fac + t64_sol + t64_adj) / (t_fac + t_app + t_ref + t_adj)})
        print(json.dumps(rows[-1]), flush=True)
        del gA, gB, X
        torch.cuda.empty_cache()
    print(json.dumps({"metric": "adjoint of X = A^-1 B (FP64 and mixed-precision forward)", "rows": rows}),
          flush=True)
    return 0


def run_ooc(args, rank, world):
    """Out-of-core form of the mixed path (lu_refine_solve_host): the FP64
    matrix stays in pinned host memory. One streamed pass converts it to
    FP32; its leading rows stay in HBM as far as they fit beside the FP32
    factors, and each refinement step's FP64 residual streams only the rest.
    At N=65536 it is timed with all rows resident and with none (every
    residual streams the whole matrix), beside the device-resident solve of
    the same matrix (same x bit for bit); --ooc-n above ~115k takes orders
    whose FP64 matrix does not fit in HBM beside the factors."""
    import torch
    import charmlu_b200 as lu
    if rank != 0:
        return 0
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    rows = []
    cases = [(65536, None), (65536, 0)] + ([(args.ooc_n, None)] if args.ooc_n != 65536 else [])
    for n, resident in cases:
        if resident is None:
            os.environ.pop("LU_B200_RESIDENT_BYTES", None)
        else:
            os.environ["LU_B200_RESIDENT_BYTES"] = str(resident)
        need = 8 * n * n
        try:
            import psutil
            avail = psutil.virtual_memory().available
        except Exception:
            avail = 0
        if avail < 1.15 * need:
            rows.append({"n": n, "skipped": f"host memory {avail / 1e9:.0f} GB < {1.15 * need / 1e9:.0f} GB"})
            print(json.dumps(rows[-1]), flush=True)
            continue
        hA = torch.empty(n, n, dtype=torch.float64, pin_memory=True)
        chunk = max(1, (1 << 30) // (8 * n))  # rows per 1 GiB generated on the device
        for r0 in range(0, n, chunk):
            r = min(chunk, n - r0)
            hA[r0:r0 + r].copy_(lu.generate_uniform(r, n, seed=42, stream_id=1000 + r0 // chunk, device=dev))
        b = lu.generate_uniform(n, 1, seed=42, stream_id=1, device=dev).view(-1)
        s = lu.LUSolver(lu.LUConfig(n, args.block_mixed, precision=lu.LU_PREC_FP16X3, lookahead=True))
        x = torch.empty_like(b)
        s.refine_solve_host(hA, b, x)  # warm (staging, resident rows and workspace allocation)
        ms = []
        for _ in range(max(1, args.steps - 1)):
            (_, info), t = _timed(lambda: s.refine_solve_host(hA, b, x))
            ms.append(t)
        t = sum(ms) / len(ms)
        row = {"n": n, "resident_rows": "all that fit in HBM" if resident is None else f"at most {resident} bytes",
               "ms": t, "tflops": flops_lu(n) / (t / 1e3) / 1e12, "status": s.status(), "r_hpl": info["r_hpl"],
               "ir_iterations": info["iterations"], "gmres_iterations": info["gmres_iterations"],
               "host_to_device_bytes_per_solve": info["host_bytes"],
               "host_to_device_gb_per_s_over_solve": info["host_bytes"] / (t / 1e3) / 1e9,
               "fp32_factors_gb_on_device": 4 * n * n / 1e9, "fp64_matrix_gb_in_host_memory": 8 * n * n / 1e9}
        if resident is None and 8 * n * n * 1.6 < torch.cuda.mem_get_info(dev)[0]:
            dA = hA.to(dev)
            xd = torch.empty_like(b)
            s2 = lu.LUSolver(lu.LUConfig(n, args.block_mixed, precision=lu.LU_PREC_FP16X3, lookahead=True))
            s2.refine_solve(dA, b, xd)
            (_, _), td = _timed(lambda: s2.refine_solve(dA, b, xd))
            row["device_resident_ms"] = td
            row["same_x_as_device_resident"] = bool(torch.equal(x, xd))
            del dA, s2
        rows.append(row)
        print(json.dumps(row), flush=True)
        del hA, s
        torch.cuda.empty_cache()
    os.environ.pop("LU_B200_RESIDENT_BYTES", None)
    print(json.dumps({"metric": "out-of-core mixed solve: FP64 A in host memory", "rows": rows}), flush=True)
    return 0


def run_blockcyclic(args, rank, world):
    """One N x N FP64 system factored and solved over all ranks, one GPU
    each: the 1D block-cyclic driver (charmlu_b200.distributed), which
    broadcasts each factored panel and its pivots over NCCL. Every rank
    generates the same global A (counter-based generator) and keeps its
    column blocks. A step is factor + solve on a fresh copy of the local
    blocks; time is the max over ranks of CUDA-event time (strong scaling:
    the matrix is fixed as N grows). Rank 0 checks r_hpl against the
    regenerated A."""
    import datetime
    import torch
    import torch.distributed as dist
    import charmlu_b200 as lu
    from charmlu_b200.distributed import BlockCyclicLU
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    os.environ.setdefault("MASTER_PORT", str(29400 + os.getpid() % 500))
    dist.init_process_group("nccl", rank=rank, world_size=world, device_id=dev,
                            timeout=datetime.timedelta(seconds=600))
    n, b = args.n, args.block
    d = BlockCyclicLU(n, b, lookahead=bool(args.lookahead))
    A = lu.generate_uniform(n, n, seed=42, stream_id=0, device=dev)
    rhs = lu.generate_uniform(n, 1, seed=42, stream_id=1, device=dev).view(-1)
    loc0 = d.scatter(A)
    del A
    torch.cuda.empty_cache()
    loc = torch.empty_like(loc0)
    ms = []
    x = None
    for k in range(args.warmup + args.steps):
        loc.copy_(loc0)
        torch.cuda.synchronize()
        dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        ipiv = d.factor(loc)
        x = d.solve(loc, ipiv, rhs)
        e1.record()
        torch.cuda.synchronize()
        t = torch.tensor([e0.elapsed_time(e1)], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        if k >= args.warmup:
            ms.append(float(t))
    status = d.status_code
    del loc, loc0
    torch.cuda.empty_cache()
    if rank == 0:
        A = lu.generate_uniform(n, n, seed=42, stream_id=0, device=dev)
        r = lu.LUSolver(lu.LUConfig(n, b)).residual(A, x, rhs)
        del A
        t = sum(ms) / len(ms)
        print(json.dumps({
            "metric": f"N={n} FP64 LU + solve over {world} GPU(s), 1D block-cyclic over NCCL, TFLOP/s",
            "unit": "TFLOP/s", "value": flops_lu(n) / (t / 1e3) / 1e12, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t, "higher_is_better": True, "scaling": "strong",
            "dtype": "f64", "data": "synthetic uniform[-0.5,0.5) seed 42 (counter-based generator)",
            "config": {"workload": "blockcyclic", "n": n, "block_size": b, "lookahead": bool(args.lookahead),
                       "l2": f"local blocks {8 * n * n / world / 1e9:.1f} GB per GPU >> 126 MB L2",
                       "parallelism": f"1D column-block-cyclic over {world} GPU(s)"},
            "status": status, "r_hpl": r["r_hpl"], "r_ref": r["r_ref"]}), flush=True)
    dist.barrier()
    dist.destroy_process_group()
    return 0


def run_ooc64(args, rank, world):
    """Out-of-core FP64 LU + solve (charmlu_b200.ooc.OutOfCoreLU): the matrix
    in pinned host memory, column panels streamed through the GPU; at
    --ooc-n (default 65536, beside the in-core lu_factor_solve of the same
    matrix when that fits) one factor + solve timed with CUDA events, r_hpl
    checked against a regenerated copy on the device when it fits, else
    skipped."""
    import torch
    import charmlu_b200 as lu
    from charmlu_b200.ooc import OutOfCoreLU
    if rank != 0:
        return 0
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    n, b = args.ooc_n, args.block
    try:
        import psutil
        avail = psutil.virtual_memory().available
    except Exception:
        avail = 0
    if avail < 1.15 * 8 * n * n:
        print(json.dumps({"workload": "ooc64", "n": n, "skipped": f"host memory {avail / 1e9:.0f} GB"}))
        return 0
    host = torch.empty(n, n, dtype=torch.float64, pin_memory=True)
    chunk = max(1, (1 << 30) // (8 * n))
    for r0 in range(0, n, chunk):
        r = min(chunk, n - r0)
        host[r0:r0 + r].copy_(lu.generate_uniform(r, n, seed=42, stream_id=2000 + r0 // chunk, device=dev))
    rhs = lu.generate_uniform(n, 1, seed=42, stream_id=1, device=dev).view(-1)
    ooc = OutOfCoreLU(n, b=b)
    # the in-core comparison needs a second host copy and the matrix in HBM
    fits = 8 * n * n * 1.6 < torch.cuda.mem_get_info(dev)[0] and avail >= 2.3 * 8 * n * n
    orig = host.clone() if fits else None
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    ipiv = ooc.factor(host)
    x = ooc.solve(host, ipiv, rhs)
    e1.record()
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1)
    row = {"workload": "ooc64", "n": n, "panel_width": ooc.w, "ms": t, "tflops": flops_lu(n) / (t / 1e3) / 1e12,
           "status": ooc.status_code, "fp64_matrix_gb_in_host_memory": 8 * n * n / 1e9,
           "device_panels_gb": 3 * 8 * n * ooc.w / 1e9}
    if orig is not None:
        A = orig.to(dev)
        row["r_hpl"] = lu.LUSolver(lu.LUConfig(n, b)).residual(A, x, rhs)["r_hpl"]
        s = lu.LUSolver(lu.LUConfig(n, b, lookahead=True))
        xr = rhs.clone()
        e0.record()
        s.factor_solve(A, xr)
        e1.record()
        torch.cuda.synchronize()
        row["in_core_ms"] = e0.elapsed_time(e1)
    print(json.dumps(row), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=65536)
    ap.add_argument("--block", type=int, default=256)
    ap.add_argument("--block-mixed", type=int, default=512)
    ap.add_argument("--precision", default="fp16x3", choices=["bf16", "fp16s", "fp16x3"])
    ap.add_argument("--lookahead", type=int, default=1)
    ap.add_argument("--graph", type=int, default=1)        # mixed path: replay the captured schedule
    ap.add_argument("--graph-fp64", type=int, default=0)   # FP64 path (replay measured slower there)
    ap.add_argument("--fp64-steps", type=int, default=1)
    ap.add_argument("--mode", default="auto", choices=["auto", "fp64", "mixed"])
    ap.add_argument("--ref-sample", type=int, default=8192)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-c2", action="store_true")        # skip the N=32768 FP64 sub-record
    ap.add_argument("--no-fp64", action="store_true")      # mixed mode: skip the FP64 companion run
    ap.add_argument("--no-batched", action="store_true")   # skip the batched sub-record
    ap.add_argument("--workload", default="lu", choices=["lu", "batched", "ksweep", "adjoint", "ooc",
                                                         "blockcyclic", "ooc64"])
    ap.add_argument("--ooc-n", type=int, default=65536)
    ap.add_argument("--adjoint-n", type=int, default=4096)
    ap.add_argument("--adjoint-mixed-n", type=int, default=32768)
    ap.add_argument("--adjoint-target", type=float, default=1e-3)
    ap.add_argument("--ksweep-n", type=int, default=8192)
    ap.add_argument("--ksweep-iters", type=int, default=30)
    ap.add_argument("--batch-count", type=int, default=4096)
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.workload == "batched":
        return run_batched(args, rank, world)
    if args.workload == "ksweep":
        return run_ksweep(args, rank, world)
    if args.workload == "adjoint":
        return run_adjoint(args, rank, world)
    if args.workload == "ooc":
        return run_ooc(args, rank, world)
    if args.workload == "blockcyclic":
        return run_blockcyclic(args, rank, world)
    if args.workload == "ooc64":
        return run_ooc64(args, rank, world)

    import torch
    import charmlu_b200 as lu
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    n, b = args.n, args.block
    bm = args.block_mixed
    seed = 42 + rank
    mode = "mixed" if args.mode == "auto" else args.mode
    dev = torch.device("cuda", local)
    peaks = measured_peaks()

    A0 = lu.generate_uniform(n, n, seed=seed, stream_id=0, device=dev)
    rhs0 = lu.generate_uniform(n, 1, seed=seed, stream_id=1, device=dev).view(-1)

    # ---------------- FP64 path: factor_solve on a copy of A0 ----------------
    s64 = lu.LUSolver(lu.LUConfig(n, b, lookahead=bool(args.lookahead), use_graph=bool(args.graph_fp64)))
    A = torch.empty_like(A0)
    x = torch.empty_like(rhs0)

    def step_fp64(ev=None):
        A.copy_(A0)
        x.copy_(rhs0)
        if ev:
            ev[0].record()
        s64.factor_solve(A, x)
        if ev:
            ev[1].record()

    # ---------------- mixed path: refine_solve (A0, b read only) -------------
    prec = {"bf16": lu.LU_PREC_BF16, "fp16s": lu.LU_PREC_FP16S, "fp16x3": lu.LU_PREC_FP16X3}[args.precision]
    smx = lu.LUSolver(lu.LUConfig(n, bm, precision=prec, lookahead=bool(args.lookahead),
                                  use_graph=bool(args.graph))) if mode == "mixed" else None
    xm = torch.empty_like(rhs0)
    last_info = {}

    def step_mixed(ev=None):
        if ev:
            ev[0].record()
        _, inf = smx.refine_solve(A0, rhs0, xm)
        if ev:
            ev[1].record()
        last_info.update(inf)

    headline = step_mixed if mode == "mixed" else step_fp64
    head_solver = smx if mode == "mixed" else s64
    for _ in range(args.warmup):
        headline()
    st = head_solver.status()
    if st != 0:
        raise SystemExit(f"warmup status {st}: {lu.status_string(st)} {last_info}")

    clocks = ClockSampler(local)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    launches0 = lu.launch_count()
    barrier()
    clocks.start()
    for k in range(args.steps):
        headline(evs[k])
    barrier()
    clk = clocks.stop()
    launches = lu.launch_count() - launches0
    step_ms = [a.elapsed_time(bv) for a, bv in evs]
    tot_ms = sum(step_ms)
    if dist is not None:
        t = torch.tensor([tot_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        tot_ms = float(t.item())
    status = head_solver.status()
    xh = xm if mode == "mixed" else x
    res = s64.residual(A0, xh, rhs0)
    info = dict(last_info)

    # one profiled headline step (outside the timed region), on a solver
    # without graph replay so every phase is bracketed by events
    prof_solver = head_solver
    if (args.graph if mode == "mixed" else args.graph_fp64):
        prof_solver = lu.LUSolver(lu.LUConfig(n, bm if mode == "mixed" else b,
                                              precision=prec if mode == "mixed" else lu.LU_PREC_FP64,
                                              lookahead=bool(args.lookahead)))
    prof_solver.profile(True)
    if mode == "mixed":
        prof_solver.refine_solve(A0, rhs0, xm)
    else:
        A.copy_(A0)
        x.copy_(rhs0)
        prof_solver.factor_solve(A, x)
    phases = prof_solver.phase_times()
    prof_solver.profile(False)
    if prof_solver is not head_solver:
        prof_solver.close()
        torch.cuda.empty_cache()

    # FP64 companion (mixed mode): time-to-solution of the FP64 path, same A, b
    fp64 = None
    if mode == "mixed" and not args.no_fp64:
        step_fp64()
        e = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
        fp64_ms = []
        for _ in range(args.fp64_steps):
            step_fp64(e)
            torch.cuda.synchronize()
            fp64_ms.append(e[0].elapsed_time(e[1]))
        r64 = s64.residual(A0, x, rhs0)
        sp = lu.LUSolver(lu.LUConfig(n, b, lookahead=bool(args.lookahead)))
        sp.profile(True)
        A.copy_(A0)
        x.copy_(rhs0)
        sp.factor_solve(A, x)
        ph64 = sp.phase_times()
        sp.close()
        fe = ((xm - x).abs().max() / x.abs().max()).item()
        t64 = sum(fp64_ms) / len(fp64_ms)
        fp64 = {"time_to_solution_s": t64 / 1e3, "tflops": flops_lu(n) / (t64 / 1e3) / 1e12, "block_size": b,
                "r_hpl": r64["r_hpl"], "r_ref": r64["r_ref"], "status": s64.status(),
                "phases_ms": {k: round(v[0], 3) for k, v in ph64.items()},
                "gemm_tflops": ph64["gemm"][2] / ph64["gemm"][0] / 1e9 if ph64["gemm"][0] else None}
        info["forward_error_vs_fp64_path"] = fe

    # FP64 peak: cuBLAS DGEMM 8192^3 back to back (MEASURED_PEAKS.json has no FP64 entry)
    peak64 = None
    try:
        m = 8192
        a = torch.randn(m, m, dtype=torch.float64, device=dev)
        bb = torch.randn(m, m, dtype=torch.float64, device=dev)
        c = torch.empty_like(a)
        for _ in range(2):
            torch.matmul(a, bb, out=c)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(12):
            torch.matmul(a, bb, out=c)
        e1.record()
        torch.cuda.synchronize()
        peak64 = 2 * m ** 3 * 12 / e0.elapsed_time(e1) / 1e9
        del a, bb, c
    except Exception:
        peak64 = None
    peak64_v = peak64 if peak64 else 35.2

    gms, gcalls, gfl = phases["gemm"]
    gemm_tf = gfl / gms / 1e9 if gms > 0 else None
    if mode == "mixed":
        peak_v, peak_src = (peaks.get("bf16_tflops_sustained"), "MEASURED_PEAKS.json bf16_tflops_sustained "
                                                                "(of measured)")
        if not peak_v:
            peak_v, peak_src = 1400.0, "fallback sustained bf16 figure (MEASURED_PEAKS.json absent; of fallback)"
        # the phase counts executed tensor flops: three FP16 products per
        # element for the error-compensated split, one otherwise
        prods = 3 if args.precision == "fp16x3" else 1
        alg_tf = gemm_tf / prods if gemm_tf else None
        # FP16x3 runs on CTA pairs unless LU_B200_GEMM_PAIR=0
        pair = args.precision == "fp16x3" and os.environ.get("LU_B200_GEMM_PAIR", "1") != "0"
        kname = ("gemm_lowp_pair_kernel (trailing update, tcgen05 kind::f16 cta_group::2, 256x256 tiles on CTA "
                 "pairs" if pair else "gemm_lowp_persistent_kernel (trailing update, tcgen05 kind::f16")
        roof = {"bound": "tensor", "kernel": f"{kname}, {args.precision}, double-buffered TMEM accumulators)",
                "achieved": alg_tf, "peak": peak_v, "unit": "TFLOP/s",
                "frac": (alg_tf / peak_v) if alg_tf else None, "traffic": None,
                "flops_counted": "algorithmic: 2*M*N*K per trailing update, each product once",
                "achieved_executed": gemm_tf, "frac_executed": (gemm_tf / peak_v) if gemm_tf else None,
                "executed_note": f"{prods} tensor-core product(s) per element ({args.precision})",
                "peak_source": peak_src}
        if args.lookahead and gemm_tf:
            # beside the look-ahead panel the update's main launch holds the
            # SMs the panel's reserve leaves it; a helper launch takes the
            # reserved SMs once the panel is done, so the phase runs on
            # between these and all SMs
            try:
                sms = torch.cuda.get_device_properties(dev).multi_processor_count
                held = sms - int(os.environ.get("LU_B200_GEMM_RESERVE", "48"))
                if 0 < held < sms:
                    roof["sms_beside_panel"] = held
                    roof["sms_total"] = sms
            except Exception:
                pass
        tpath = os.path.join(ROOT, "profiles",
                             "gemm_lowp_pair_traffic.json" if pair else "gemm_lowp_persistent_traffic.json")
    else:
        roof = {"bound": "tensor", "kernel": "gemm_f64_sub_kernel (trailing update, DMMA)",
                "achieved": gemm_tf, "peak": peak64_v, "unit": "TFLOP/s",
                "frac": (gemm_tf / peak64_v) if gemm_tf else None, "traffic": None,
                "peak_source": "live cuBLAS DGEMM 8192^3 (MEASURED_PEAKS.json has no FP64 entry)"}
        tpath = os.path.join(ROOT, "profiles", "gemm_f64_traffic.json")
    if os.path.exists(tpath) and gcalls:
        tj = json.load(open(tpath))
        roof["traffic"] = tj["bytes_per_flop"] * gfl / gcalls
        roof["traffic_note"] = "bytes per launch, from the ncu capture in " + tj["source"] + " scaled by flops"

    line = None
    if rank == 0:
        value = flops_lu(n) * args.steps * world / (tot_ms / 1e3) / 1e12
        line = {
            "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": tot_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": (f"{args.precision}-tensor/f32-panel/f64-ir") if mode == "mixed" else "f64",
            "data": "synthetic uniform[-0.5,0.5) seed 42 (counter-based generator)",
            "config": {"workload": (f"N={n} dense LU + solve to r_hpl<16: {args.precision} tensor-core trailing update / "
                                    f"FP32 panel factor + FP64 refinement (b={bm}), FP64 LU (b={b}) beside it; "
                                    f"look-ahead={'on' if args.lookahead else 'off'}") if mode == "mixed" else
                       f"N={n} dense LU with partial pivoting + solve, FP64 path, b={b}",
                       "n": n, "block_size": bm if mode == "mixed" else b, "path": mode,
                       "precision": args.precision if mode == "mixed" else "fp64",
                       "lookahead": bool(args.lookahead),
                       "cuda_graph": bool(args.graph if mode == "mixed" else args.graph_fp64),
                       "l2": "inputs 34 GB >> 126 MB L2 (no flush needed)",
                       "parallelism": "replicas" if world > 1 else "single"},
            "time_to_solution_s": tot_ms / args.steps / 1e3,
            "status": status, "r_hpl": res["r_hpl"], "r_ref": res["r_ref"],
            "refine": info if mode == "mixed" else None,
            "fp64_path": fp64,
            "speedup_vs_fp64": (fp64["time_to_solution_s"] / (tot_ms / args.steps / 1e3)) if fp64 else None,
            "roofline": roof,
            "fp64_peak_tflops": peak64_v,
            "phases_ms": {k: round(v[0], 3) for k, v in phases.items()},
            "gpu_launches": launches,
            "clocks": clk,
        }
    # ---- e2e through the public API from pinned host buffers
    if rank == 0 and not args.no_e2e:
        try:
            import psutil
            avail = psutil.virtual_memory().available
        except Exception:
            avail = 0
        need = 8 * n * n * 2.2
        if avail > need:
            hA = torch.empty(n, n, dtype=torch.float64, pin_memory=True)
            hA.copy_(A0)
            hb = torch.empty(n, dtype=torch.float64, pin_memory=True)
            hb.copy_(rhs0)
            hx = torch.empty(n, dtype=torch.float64, pin_memory=True)
            e2e_ms = []
            for k in range(3):  # the first pass is untimed (graph capture for this buffer)
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                if mode == "mixed":
                    A.copy_(hA, non_blocking=True)
                    x.copy_(hb, non_blocking=True)
                    smx.refine_solve(A, x, xm)
                    hx.copy_(xm, non_blocking=True)
                else:
                    A.copy_(hA, non_blocking=True)
                    x.copy_(hb, non_blocking=True)
                    s64.factor_solve(A, x)
                    hx.copy_(x, non_blocking=True)
                e1.record()
                torch.cuda.synchronize()
                if k > 0:
                    e2e_ms.append(e0.elapsed_time(e1))
            line["e2e"] = {"value": flops_lu(n) / (sum(e2e_ms) / len(e2e_ms) / 1e3) / 1e12, "unit": "TFLOP/s",
                           "h2d_bytes_per_step": 8 * n * n + 8 * n, "d2h_bytes_per_step": 8 * n,
                           "ms_per_step": sum(e2e_ms) / len(e2e_ms), "steps": len(e2e_ms)}
            del hA
        else:
            line["e2e"] = {"value": None, "unit": "TFLOP/s", "h2d_bytes_per_step": 8 * n * n + 8 * n,
                           "d2h_bytes_per_step": 8 * n,
                           "note": f"host RAM available {avail / 1e9:.0f} GB < {need / 1e9:.0f} GB needed for pinned A"}
    if rank == 0 and world == 1 and not args.no_c2:
        # the BASELINE's N=32768 FP64 configuration, with the CPU oracle at the same order
        line["fp64_c2"] = fp64_c2_record(dev, peak64_v, with_cpu=not args.no_cpu)
    if rank == 0 and world == 1 and not args.no_batched:
        from charmlu_b200.batched import log_uniform_orders
        import numpy as np
        n_all = log_uniform_orders(args.batch_count, 32, 1024, seed=42)
        bout = batched_measure(n_all, np.arange(len(n_all)), dev, None, 3, 3)[0]
        line["batched"] = {"workload": f"{len(n_all)} systems, n log-uniform [32,1024] seed 42, one RHS each, "
                                       "one persistent launch replayed from a CUDA graph",
                           "fp64": bout["fp64"], "fp32_ir": bout["fp32_ir"]}
        torch.cuda.empty_cache()
    if rank == 0 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())

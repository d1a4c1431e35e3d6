"""Batched uneven solves (no reference counterpart): many independent
systems of different order factored and solved in one persistent launch
(lu_batched_factor_solve).  Per-size-bucket kernel parameters come from the
autotuner's tables in charmlu_b200/tuning/ when present."""
import ctypes
import json
import os

import numpy as np
import torch

from . import _lib
from ._lib import LU_PREC_FP32, LU_PREC_FP64

TUNING_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning")
_applied = {}


def tuning_path(precision):
    return os.path.join(TUNING_DIR, "batched_fp64.json" if precision == LU_PREC_FP64 else "batched_fp32.json")


def apply_tuning(precision, table=None):
    """Load the autotuned {n_max, nb, small} table for this precision (or the
    given table; [] restores the built-in defaults) into the kernel."""
    L = _lib.load()
    if table is None:
        p = tuning_path(precision)
        table = json.load(open(p))["table"] if os.path.exists(p) else []
    flat = np.asarray([v for e in table for v in (e["n_max"], e["nb"], e["small"])], dtype=np.int32)
    rc = L.lu_batched_set_tuning(len(table), ctypes.c_void_p(flat.ctypes.data) if len(table) else None)
    if rc != 0:
        raise RuntimeError(f"lu_batched_set_tuning failed ({rc})")
    _applied["precision"] = precision


class BatchedSystems:
    """Device storage for `count` systems of orders n (host int array):
    matrices concatenated row-major, right-hand sides concatenated."""

    def __init__(self, n, device="cuda"):
        self.n = np.asarray(n, dtype=np.int32)
        self.count = len(self.n)
        n64 = self.n.astype(np.int64)
        self.a_off = np.concatenate([[0], np.cumsum(n64 * n64)[:-1]]).astype(np.int64)
        self.b_off = np.concatenate([[0], np.cumsum(n64)[:-1]]).astype(np.int64)
        self.total_a = int((n64 * n64).sum())
        self.total_b = int(n64.sum())
        self.d_n = torch.from_numpy(self.n).to(device)
        self.d_a_off = torch.from_numpy(self.a_off).to(device)
        self.d_b_off = torch.from_numpy(self.b_off).to(device)
        self.info = torch.zeros(self.count, dtype=torch.int32, device=device)
        self._work = {}

    def work(self, precision):
        if precision not in self._work:
            L = _lib.load()
            wb = L.lu_batched_work_bytes(self.count, ctypes.c_void_p(self.n.ctypes.data), precision)
            self._work[precision] = torch.empty(wb, dtype=torch.uint8, device=self.d_n.device)
        return self._work[precision]

    def factor_solve(self, A, b, precision=LU_PREC_FP64, stream=None):
        """A (total_a doubles), b (total_b doubles) on the device; b is
        overwritten by the solutions, A by the factors (FP64) or left intact
        (FP32 mode).  Returns the per-system status tensor (device)."""
        if _applied.get("precision") != precision:
            apply_tuning(precision)
        L = _lib.load()
        w = self.work(precision)
        s = stream if stream is not None else torch.cuda.current_stream()
        rc = L.lu_batched_factor_solve(self.count, ctypes.c_void_p(self.d_n.data_ptr()),
                                       ctypes.c_void_p(self.d_a_off.data_ptr()),
                                       ctypes.c_void_p(self.d_b_off.data_ptr()), ctypes.c_void_p(A.data_ptr()),
                                       ctypes.c_void_p(b.data_ptr()), ctypes.c_void_p(self.info.data_ptr()),
                                       precision, ctypes.c_void_p(w.data_ptr()), w.numel(),
                                       ctypes.c_void_p(s.cuda_stream))
        if rc != 0:
            raise RuntimeError(f"lu_batched_factor_solve failed ({rc})")
        return self.info

    def refine_histogram(self, stream=None):
        """After an FP32-mode factor_solve: systems that met r_hpl < 16
        after s FP64 refinement steps, s = 0 .. 10, and (last entry) those
        that did not (lu_batched_refine_histogram; synchronises)."""
        L = _lib.load()
        w = self.work(LU_PREC_FP32)
        hist = np.zeros(12, dtype=np.int32)
        s = stream if stream is not None else torch.cuda.current_stream()
        rc = L.lu_batched_refine_histogram(ctypes.c_void_p(w.data_ptr()), ctypes.c_void_p(hist.ctypes.data),
                                           ctypes.c_void_p(s.cuda_stream))
        if rc != 0:
            raise RuntimeError(f"lu_batched_refine_histogram failed ({rc})")
        return hist


def log_uniform_orders(count, lo=32, hi=1024, seed=42):
    """Orders drawn log-uniform in [lo, hi] from the seed."""
    rng = np.random.default_rng(seed)
    n = np.exp(rng.uniform(np.log(lo), np.log(hi + 1), count)).astype(np.int32)
    return np.clip(n, lo, hi)


def flops(n):
    n = np.asarray(n, dtype=np.float64)
    return float((2.0 / 3.0 * n ** 3 + 2.0 * n ** 2).sum())


def partition_by_cost(n, parts):
    """Split systems of orders n over `parts` GPUs so that the factor+solve
    work (2/3 n^3 + 2 n^2 per system) is balanced: longest-processing-time
    order, each system to the currently lightest part.  Deterministic;
    returns `parts` sorted index arrays that together cover every system
    exactly once.  The systems are independent, so a sharded run needs no
    collective except the final gather_results."""
    n = np.asarray(n, dtype=np.int64)
    if parts < 1:
        raise ValueError("parts must be >= 1")
    cost = (2.0 / 3.0) * n.astype(np.float64) ** 3 + 2.0 * n.astype(np.float64) ** 2
    order = np.argsort(-cost, kind="stable")
    loads = np.zeros(parts)
    buckets = [[] for _ in range(parts)]
    for i in order:
        p = int(np.argmin(loads))
        buckets[p].append(int(i))
        loads[p] += cost[i]
    return [np.array(sorted(b), dtype=np.int64) for b in buckets]


def gather_results(index, info, residual, count, group=None):
    """Per-system status codes and scaled residuals of this rank's systems
    (global indices `index`) gathered into global order on every rank over
    torch.distributed (any backend).  Returns (info[count], residual[count])
    as numpy arrays; systems no rank reported keep status -1 and NaN."""
    import torch.distributed as dist
    mine = (np.asarray(index, dtype=np.int64).tolist(), np.asarray(info, dtype=np.int64).tolist(),
            np.asarray(residual, dtype=np.float64).tolist())
    if dist.is_available() and dist.is_initialized():
        allp = [None] * dist.get_world_size(group)
        dist.all_gather_object(allp, mine, group=group)
    else:
        allp = [mine]
    g_info = np.full(count, -1, dtype=np.int64)
    g_res = np.full(count, np.nan)
    for idx, inf, res in allp:
        g_info[idx] = inf
        g_res[idx] = res
    return g_info, g_res


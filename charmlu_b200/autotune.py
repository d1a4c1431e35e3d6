"""Autotuner for the batched solver's per-size-bucket parameters.

For each order bucket it times the persistent batched kernel on seeded
systems with every candidate (panel width nb, in-shared-memory threshold)
and keeps the fastest; the tables are written to charmlu_b200/tuning/ and
applied by charmlu_b200.batched at run time.

    python -m charmlu_b200.autotune [--precision fp64|fp32|both] [--quick]
"""
import argparse
import json
import os
import sys
import time

import numpy as np
import torch

from . import generate_uniform
from ._lib import LU_PREC_FP32, LU_PREC_FP64
from .batched import BatchedSystems, TUNING_DIR, apply_tuning

BUCKETS = [32, 64, 96, 128, 160, 192, 256, 384, 512, 768, 1024, 1536, 2048]
NB = [8, 16, 32]


def _small_candidates(prec):
    cap = 159 if prec == LU_PREC_FP64 else 225
    return [0, 64, 96, 128, cap]


def time_config(prec, n_lo, n_hi, nb, small, systems=296, reps=3, seed=7):
    rng = np.random.default_rng(seed + n_hi)
    n = rng.integers(n_lo, n_hi + 1, systems).astype(np.int32)
    bs = BatchedSystems(n)
    A0 = generate_uniform(1, bs.total_a, seed=seed, stream_id=20).view(-1)
    b0 = generate_uniform(1, bs.total_b, seed=seed, stream_id=21).view(-1)
    A, b = A0.clone(), b0.clone()
    apply_tuning(prec, [{"n_max": 4096, "nb": nb, "small": small}])
    best = float("inf")
    for r in range(reps + 1):
        A.copy_(A0)
        b.copy_(b0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        info = bs.factor_solve(A, b, prec)
        e1.record()
        torch.cuda.synchronize()
        if r > 0:
            best = min(best, e0.elapsed_time(e1))
    good = int((info == 0).sum().item())
    return best, good


def tune(prec, quick=False):
    table, log = [], []
    lo = 1
    buckets = BUCKETS if not quick else [64, 256, 1024]
    for hi in buckets:
        cands = []
        cap = _small_candidates(prec)[-1]
        smalls = sorted(set([0] + [v for v in (64, 96, 128) if v < hi] + [min(cap, hi)]))
        for nb in NB:
            for small in smalls:
                ms, good = time_config(prec, lo, hi, nb, small, systems=148 if quick else 296,
                                       reps=1 if quick else 3)
                cands.append((-good, ms, nb, small))
                log.append({"n_lo": lo, "n_hi": hi, "nb": nb, "small": small, "ms": ms, "systems_ok": good})
        # most systems meeting the residual contract first, then the fastest
        _, ms, nb, small = min(cands)
        table.append({"n_max": hi, "nb": nb, "small": small, "ms": ms})
        print(f"bucket ({lo},{hi}]: nb={nb} small={small} {ms:.3f} ms", flush=True)
        lo = hi + 1
    return table, log


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--precision", default="both", choices=["fp64", "fp32", "both"])
    ap.add_argument("--quick", action="store_true")
    ap.add_argument("--out", default=TUNING_DIR)
    a = ap.parse_args(argv)
    os.makedirs(a.out, exist_ok=True)
    precs = {"fp64": [LU_PREC_FP64], "fp32": [LU_PREC_FP32], "both": [LU_PREC_FP64, LU_PREC_FP32]}[a.precision]
    for prec in precs:
        t0 = time.time()
        table, log = tune(prec, a.quick)
        name = "batched_fp64.json" if prec == LU_PREC_FP64 else "batched_fp32.json"
        with open(os.path.join(a.out, name), "w") as f:
            json.dump({"precision": "fp64" if prec == LU_PREC_FP64 else "fp32", "device": torch.cuda.get_device_name(),
                       "table": table, "candidates": log, "seconds": time.time() - t0}, f, indent=1)
        print("wrote", os.path.join(a.out, name), flush=True)
    apply_tuning(precs[-1], [])
    return 0


if __name__ == "__main__":
    sys.exit(main())

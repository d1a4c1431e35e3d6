"""ORACLE — test infrastructure only (see ref_lu.cpp for what it restates).

ctypes front-end of the CPU restatement of charmlu's dense-LU hot path.  Only
tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs may import
this package; the product (charmlu_b200) never does.
"""
import ctypes
import os

import numpy as np

from .build_oracle import OUT, build

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(OUT):
            build()
        L = ctypes.CDLL(OUT)
        P = ctypes.c_void_p
        i64, i32, u64, dbl = ctypes.c_int64, ctypes.c_int32, ctypes.c_uint64, ctypes.c_double
        L.oracle_gen_uniform.argtypes = [P, i64, u64, u64, i64]
        L.oracle_matgen.argtypes = [P, i64, i32, i64, P]
        L.oracle_set_threads.argtypes = [ctypes.c_int]
        L.oracle_lu_factor.argtypes = [ctypes.c_int, ctypes.c_int, P, i64, P, P, P, ctypes.c_int, dbl]
        L.oracle_lu_factor.restype = ctypes.c_int
        L.oracle_lu_solve_permuted.argtypes = [ctypes.c_int, ctypes.c_int, P, i64, P]
        L.oracle_residual.argtypes = [ctypes.c_int, P, i64, P, P, P]
        # OpenBLAS single-threaded inside the oracle's OpenMP regions (its
        # pthread pool must not be entered from several OpenMP threads)
        L.oracle_set_threads(0)
        _lib = L
    return _lib


def _p(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def set_threads(n=0):
    lib().oracle_set_threads(int(n))


def gen_uniform(count, seed, stream, offset=0):
    out = np.empty(int(count), dtype=np.float64)
    lib().oracle_gen_uniform(_p(out), int(count), int(seed), int(stream), int(offset))
    return out


def gen_matrix(n, seed=42, stream=0):
    """n x n row-major uniform[-0.5, 0.5) matrix (stream 0 = A)."""
    return gen_uniform(n * n, seed, stream).reshape(n, n)


def gen_vector(n, seed=42, stream=1):
    return gen_uniform(n, seed, stream)


def matgen(count, seed=9934835, skip=0):
    """The reference's MatGen b-vector generator (benchmark.C:28-74)."""
    out = np.empty(int(count), dtype=np.float64)
    ints = np.empty(int(count), dtype=np.int32)
    lib().oracle_matgen(_p(out), int(count), int(seed), int(skip), _p(ints))
    return out, ints


SING_REF = 100 * np.finfo(np.float64).eps  # lu.ci:339


def lu_factor(A, b=128, rhs=None, blas=True, sing_threshold=0.0):
    """Blocked LU in place semantics; returns (LU, ipiv, rhs_perm, margin, info)."""
    A = np.array(A, dtype=np.float64, order="C", copy=True)
    n = A.shape[0]
    ipiv = np.empty(n, dtype=np.int32)
    margin = np.empty(n, dtype=np.float64)
    r = None if rhs is None else np.array(rhs, dtype=np.float64, copy=True)
    info = lib().oracle_lu_factor(n, int(b), _p(A), n, _p(ipiv), _p(r), _p(margin),
                                  1 if blas else 0, float(sing_threshold))
    return A, ipiv, r, margin, info


def lu_solve_permuted(LU, b, x_perm):
    x = np.array(x_perm, dtype=np.float64, copy=True)
    lib().oracle_lu_solve_permuted(LU.shape[0], int(b), _p(np.ascontiguousarray(LU)), LU.shape[1], _p(x))
    return x


def residual(A, x, rhs):
    """dict with amax, bmax, xmax, rmax, anorm, r_ref, r_hpl (benchmark.C:385-400)."""
    A = np.ascontiguousarray(A, dtype=np.float64)
    out = np.zeros(7)
    lib().oracle_residual(A.shape[0], _p(A), A.shape[1], _p(np.ascontiguousarray(x, dtype=np.float64)),
                          _p(np.ascontiguousarray(rhs, dtype=np.float64)), _p(out))
    keys = ["amax", "bmax", "xmax", "rmax", "anorm", "r_ref", "r_hpl"]
    return dict(zip(keys, out.tolist()))


def apply_pivots(v, ipiv):
    v = np.array(v, copy=True)
    for j, p in enumerate(ipiv):
        if p != j:
            v[[j, p]] = v[[p, j]]
    return v


def solve(A, rhs, b=128, blas=True):
    """Factor + solve + residual, the reference's timed span plus its check."""
    LU, ipiv, rp, margin, info = lu_factor(A, b, rhs, blas)
    x = lu_solve_permuted(LU, b, rp)
    return x, LU, ipiv, margin, info

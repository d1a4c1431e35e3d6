"""Generate the golden fixtures in tests/golden/ from the CPU oracle.

charmlu's own test (test_lu.pl) pins only "residual < 16"; it holds no
pivot or factor vectors, and charmlu cannot be built in this image (Charm++
is absent).  These fixtures are therefore produced by the oracle
(oracle/ref_lu.cpp, a restatement of lu.C/lu.ci), cross-checked here
against LAPACK dgetrf through scipy before they are written, and used to pin
both the oracle (against drift) and the CUDA path.

Run: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402

# (n, b): test_lu.pl's small and pivot-batch configurations (test_lu.pl:9-26)
# plus odd and non-multiple-of-b orders
CASES = [(32, 4), (32, 8), (48, 12), (48, 16), (48, 24), (48, 48), (64, 16), (100, 32), (128, 32), (256, 64)]
SEED = 42
LU_STORE_MAX = 128


def main():
    import scipy.linalg as sl
    out = {}
    for n, b in CASES:
        A = oracle.gen_matrix(n, SEED)
        rhs = oracle.gen_vector(n, SEED)
        x, LU, ipiv, margin, info = oracle.solve(A, rhs, b=b)
        lu_l, piv_l = sl.lu_factor(A)
        assert info == 0
        assert np.array_equal(piv_l, ipiv), (n, b)
        scale = np.abs(LU).max()
        assert np.abs(lu_l - LU).max() / scale < 1e-13, (n, b)
        res = oracle.residual(A, x, rhs)
        key = f"n{n}_b{b}"
        out[key + "_ipiv"] = ipiv
        out[key + "_margin"] = margin
        out[key + "_x"] = x
        out[key + "_r"] = np.array([res["r_ref"], res["r_hpl"]])
        out[key + "_a00"] = A.ravel()[:4]       # generator spot values
        if n <= LU_STORE_MAX:
            out[key + "_lu"] = LU
    # reference generator MatGen: first draws for seed 9934835 and the
    # minimal-standard known answer (seed 1, 10000th draw = 399268537)
    v, ints = oracle.matgen(16, seed=9934835)
    out["matgen_9934835_first16"] = v
    out["matgen_9934835_first16_int"] = ints
    _, ints1 = oracle.matgen(10000, seed=1)
    out["minstd_seed1_10000th"] = np.array([ints1[-1]], dtype=np.int64)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lu_golden.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()

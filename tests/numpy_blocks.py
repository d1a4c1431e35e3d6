"""A numpy stand-in for charmlu_b200.blocks.CudaBlocks (the per-block
kernels), on CPU tensors: lets the CPU tests run the multi-GPU and
out-of-core drivers' own logic (layout, pivots, ordering) without a GPU.
Test infrastructure only."""
import numpy as np
import scipy.linalg as sl


class NumpyBlocks:
    """The per-block operations of CudaBlocks, in numpy on CPU tensors."""

    def __init__(self):
        self.first_singular = 0

    def panel_factor(self, P, ipiv_out, base):
        a = P.numpy()
        m, w = a.shape
        piv = ipiv_out.numpy()
        for j in range(w):
            p = j + int(np.argmax(np.abs(a[j:, j])))  # first maximum, as idamax
            piv[j] = base + p
            if p != j:
                a[[j, p], :] = a[[p, j], :]
            if a[j, j] == 0.0:
                if not self.first_singular:
                    self.first_singular = base + j + 1
                continue
            a[j + 1:, j] /= a[j, j]
            a[j + 1:, j + 1:] -= np.outer(a[j + 1:, j], a[j, j + 1:])

    def apply_pivots(self, A, ncols, ipiv, k0, cnt, skip_b, skip_e, b=None):
        a = A.numpy() if ncols > 0 else None
        cols = [c for c in range(ncols) if not (skip_b <= c < skip_e)]
        bv = b.numpy() if b is not None else None
        piv = ipiv.numpy()
        for i in range(k0, k0 + cnt):
            p = int(piv[i])
            if p != i:
                if cols:
                    tmp = a[i, cols].copy()
                    a[i, cols] = a[p, cols]
                    a[p, cols] = tmp
                if bv is not None:
                    bv[i], bv[p] = bv[p], bv[i]

    def trsm_lower_unit(self, L, B):
        B.numpy()[:] = sl.solve_triangular(L.numpy(), B.numpy(), lower=True, unit_diagonal=True)

    def gemm_update(self, A, B, C):
        C.numpy()[:] -= A.numpy() @ B.numpy()

    def trsv_block(self, T, upper, x):
        x.numpy()[:] = sl.solve_triangular(T.numpy(), x.numpy(), lower=not upper, unit_diagonal=not upper)

    def gemv_update(self, A, x, y):
        y.numpy()[:] -= A.numpy() @ x.numpy()

    def clear_status(self):
        self.first_singular = 0

    def status(self):
        return self.first_singular

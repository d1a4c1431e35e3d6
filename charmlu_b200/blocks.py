"""Per-block operations of the factorisation through the C ABI, for the
drivers that arrange the blocks themselves: the block-cyclic multi-GPU LU
(distributed.py) and the out-of-core FP64 LU (ooc.py). Arguments are 2-D
torch views with unit column stride; the leading dimension is the row
stride. Every call is asynchronous on torch's current CUDA stream.
"""
import ctypes

import torch

from . import _lib


def _check(code, what):
    if code != 0:
        from . import LUError
        raise LUError(code, what)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


class CudaBlocks:
    """Per-block operations through the C ABI on the current CUDA device.
    Arguments are 2-D views with unit column stride; the leading dimension
    is the row stride."""

    def __init__(self, n, b, lookahead=False):
        from . import LUConfig
        self._L = _lib.load()
        # look-ahead: panels use the narrow leaf shape that runs beside an update
        cfg = LUConfig(n, b, lookahead=lookahead)
        h = ctypes.c_void_p()
        _check(self._L.lu_create(ctypes.byref(cfg.to_c()), ctypes.byref(h)), "lu_create")
        self._h = h

    def close(self):
        if self._h:
            self._L.lu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _s():
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def panel_factor(self, P, ipiv_out, base):
        m, w = P.shape
        _check(self._L.lu_panel_factor(self._h, _ptr(P), P.stride(0), m, w, _ptr(ipiv_out), base, self._s()),
               "lu_panel_factor")

    def apply_pivots(self, A, ncols, ipiv, k0, cnt, skip_b, skip_e, b=None):
        if ncols <= 0 and b is None:
            return
        m = A.shape[0] if ncols > 0 else b.shape[0]
        _check(self._L.lu_apply_pivots(self._h, _ptr(A) if ncols > 0 else None, A.stride(0) if ncols > 0 else 2, m,
                                       ncols, _ptr(ipiv), k0, cnt, skip_b, skip_e,
                                       _ptr(b) if b is not None else None, self._s()), "lu_apply_pivots")

    def trsm_lower_unit(self, L, B):
        w = L.shape[0]
        _check(self._L.lu_trsm_lower_unit(self._h, _ptr(L), L.stride(0), w, _ptr(B), B.stride(0), B.shape[1],
                                          self._s()), "lu_trsm_lower_unit")

    def gemm_update(self, A, B, C):
        M, K = A.shape
        N = B.shape[1]
        _check(self._L.lu_gemm_update(self._h, _ptr(A), A.stride(0), _ptr(B), B.stride(0), _ptr(C), C.stride(0),
                                      M, N, K, self._s()), "lu_gemm_update")

    def trsv_block(self, T, upper, x):
        _check(self._L.lu_trsv_block(self._h, _ptr(T), T.stride(0), T.shape[0], int(upper), _ptr(x), self._s()),
               "lu_trsv_block")

    def gemv_update(self, A, x, y):
        m, k = A.shape
        _check(self._L.lu_gemv_update(self._h, _ptr(A), A.stride(0), m, k, _ptr(x), _ptr(y), self._s()),
               "lu_gemv_update")

    def clear_status(self):
        """Clear the handle's status word before a factorisation."""
        _check(self._L.lu_status_clear(self._h, self._s()), "lu_status_clear")

    def status(self):
        """First singular global column (1-based), a negative error code, or 0."""
        return int(self._L.lu_status(self._h, self._s()))

    def copy_2d(self, dst, src):
        """dst <- src for two equally shaped 2-D float64 views, either of which
        may be in (pinned) host memory (lu_copy_2d)."""
        rows, cols = src.shape
        _check(self._L.lu_copy_2d(_ptr(dst), dst.stride(0) * 8, _ptr(src), src.stride(0) * 8, cols * 8, rows,
                                  self._s()), "lu_copy_2d")

"""charmlu_b200 — B200-native dense LU with partial pivoting + solve.

Host-side mirror of charmlu's driver interface for its factor-then-solve
path.  charmlu configures a run with ``LUConfig`` (luConfig.h:8-62: matrix
size, block size, pivot batch size, memory threshold), starts it with
``LUSolver`` (benchmark.C:222-401: factor, then forwardSolve on the
diagonals, then validation through the scaled residual).  Here the same
objects drive the C ABI of ``liblu_b200.so`` on one GPU; device memory and
streams come from PyTorch (plumbing only).  There is no CPU fallback: a
missing library or a CPU tensor raises.
"""
import ctypes
import dataclasses

import torch

from . import _lib
from ._lib import (LU_ERR_ARG, LU_ERR_NOCONV, LU_ERR_TIMEOUT, LU_ERR_UNSUPPORTED, LU_IR_CLASSIC, LU_IR_GMRES,
                   LU_LAYOUT_COL, LU_LAYOUT_ROW, LU_OK, LU_PREC_BF16, LU_PREC_FP16S, LU_PREC_FP16X3, LU_PREC_FP32,
                   LU_PREC_FP64)

__all__ = ["LUConfig", "LUSolver", "LUError", "generate_uniform", "matgen", "status_string",
           "LU_PREC_FP64", "LU_PREC_BF16", "LU_PREC_FP16S", "LU_PREC_FP16X3", "LU_PREC_FP32", "LU_IR_CLASSIC", "LU_IR_GMRES",
           "LU_LAYOUT_ROW", "LU_LAYOUT_COL", "transpose_square"]

EPS = 2.220446049250313e-16


class LUError(RuntimeError):
    def __init__(self, code, what=""):
        self.code = code
        super().__init__(f"{what}: {status_string(code)} ({code})")


def status_string(code):
    return _lib.load().lu_status_string(int(code)).decode()


def _check(code, what):
    if code != LU_OK:
        raise LUError(code, what)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _stream(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def _require_cuda(t, dtype, name):
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{name} must be a CUDA tensor (no CPU path exists)")
    if t.dtype != dtype:
        raise TypeError(f"{name} must be {dtype}, got {t.dtype}")


@dataclasses.dataclass
class LUConfig:
    """luConfig.h:8-62 (matrixSize, blockSize, pivotBatchSize, memThreshold)
    plus the B200 additions.  memThreshold and the mapping fields exist for
    CLI compatibility and have no effect on one GPU."""
    matrix_size: int
    block_size: int = 128
    pivot_batch_size: int = 0          # 0 -> blockSize/4 (benchmark.C:98)
    mem_threshold: int = 0             # MB; ignored (one GPU holds the matrix)
    precision: int = LU_PREC_FP64
    lookahead: bool = False
    use_graph: bool = False
    ir_mode: int = LU_IR_CLASSIC
    ir_max_iter: int = 50
    ir_target: float = 16.0
    sing_threshold: float = 0.0        # reference: 100*eps aborts (lu.ci:339)
    spin_limit: int = 0
    layout: int = LU_LAYOUT_ROW        # LU_LAYOUT_COL: factor / factor_solve take column-major A
    gmres_restart: int = 0             # GMRES-IR Krylov vectors per cycle (0: 120)
    ir_stall: int = 0                  # GMRES cycles in a row with < 10% residual drop before giving up (0: 3)
    gmres_tol: float = 0.0             # residual reduction that ends a GMRES cycle (0: 1e-10)

    def to_c(self):
        c = _lib.LuConfig()
        _check(_lib.load().lu_config_default(ctypes.byref(c), int(self.matrix_size), int(self.block_size)),
               "lu_config_default")
        if self.pivot_batch_size:
            c.pivot_batch = int(self.pivot_batch_size)
        c.precision = int(self.precision)
        c.lookahead = int(bool(self.lookahead))
        c.use_graph = int(bool(self.use_graph))
        c.ir_mode = int(self.ir_mode)
        c.ir_max_iter = int(self.ir_max_iter)
        c.ir_target = float(self.ir_target)
        c.sing_threshold = float(self.sing_threshold)
        c.spin_limit = int(self.spin_limit)
        c.layout = int(self.layout)
        c.gmres_restart = int(self.gmres_restart)
        c.ir_stall = int(self.ir_stall)
        c.gmres_tol = float(self.gmres_tol)
        return c


class LUSolver:
    """One solver handle on the current CUDA device (LUSolver, benchmark.C:222-401)."""

    def __init__(self, cfg: LUConfig):
        if cfg.matrix_size <= 0 or cfg.block_size <= 0:
            raise LUError(LU_ERR_ARG, "LUConfig")
        self.cfg = cfg
        self._L = _lib.load()
        self._c = cfg.to_c()
        h = ctypes.c_void_p()
        _check(self._L.lu_create(ctypes.byref(self._c), ctypes.byref(h)), "lu_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._L.lu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def n(self):
        return self.cfg.matrix_size

    def workspace_bytes(self):
        return int(self._L.lu_workspace_bytes(ctypes.byref(self._c)))

    # -- status --------------------------------------------------------
    def status(self, stream=None):
        """Synchronise and return LU_OK, >0 (singular column) or LU_ERR_*."""
        return int(self._L.lu_status(self._h, _stream(stream)))

    def check(self, what="lu", stream=None):
        st = self.status(stream)
        if st != LU_OK:
            raise LUError(st, what)

    # -- factor / solve ------------------------------------------------
    def _check_matrix(self, A):
        _require_cuda(A, torch.float64, "A")
        n = self.n
        if self.cfg.layout == LU_LAYOUT_COL:  # column-major: unit row stride, pitch = column stride
            if A.dim() != 2 or A.shape[0] != n or A.shape[1] != n or A.stride(0) != 1:
                raise LUError(LU_ERR_ARG, "A must be n x n and column-major (unit row stride)")
            return A.stride(1)
        if A.dim() != 2 or A.shape[0] != n or A.shape[1] != n or A.stride(1) != 1:
            raise LUError(LU_ERR_ARG, "A must be n x n with unit column stride")
        return A.stride(0)

    def factor(self, A, ipiv=None, rhs=None, stream=None):
        """In-place P A = L U (LUBlk::factor, lu.ci:31-42).  Returns ipiv
        (int32, 0-based global rows).  rhs, if given, is permuted with the
        rows (lu.h:66)."""
        lda = self._check_matrix(A)
        if ipiv is None:
            ipiv = torch.empty(self.n, dtype=torch.int32, device=A.device)
        if rhs is not None:
            _require_cuda(rhs, torch.float64, "rhs")
        _check(self._L.lu_factor(self._h, _ptr(A), lda, _ptr(ipiv), _ptr(rhs), _stream(stream)), "lu_factor")
        return ipiv

    def solve(self, LU, ipiv, B, trans=False, stream=None):
        """Solve with stored factors in place (forwardSolve/backwardSolve,
        lu.ci:387-436); trans=True solves A^T X = B."""
        lda = self._check_matrix(LU)
        _require_cuda(B, torch.float64, "B")
        Bv = B if B.dim() == 2 else B.view(-1, 1)
        if Bv.stride(1) != 1 and Bv.shape[1] > 1:
            raise LUError(LU_ERR_ARG, "B must be row-major")
        ldb = Bv.stride(0) if Bv.shape[1] > 1 else 1
        _check(self._L.lu_solve(self._h, _ptr(LU), lda, _ptr(ipiv), _ptr(Bv), ldb, Bv.shape[1], int(trans),
                                _stream(stream)), "lu_solve")
        return B

    def factor_solve(self, A, b, ipiv=None, stream=None):
        """Time-to-solution span of the reference (benchmark.C:243 -> 344):
        factor A in place and overwrite b with x."""
        lda = self._check_matrix(A)
        _require_cuda(b, torch.float64, "b")
        if ipiv is None:
            ipiv = torch.empty(self.n, dtype=torch.int32, device=A.device)
        _check(self._L.lu_factor_solve(self._h, _ptr(A), lda, _ptr(ipiv), _ptr(b), _stream(stream)),
               "lu_factor_solve")
        return ipiv

    def residual(self, A, x, b, stream=None):
        """Scaled residual against the ORIGINAL A (benchmark.C:385-400).
        Returns dict(amax, anorm, bnorm, xnorm, rnorm, r_ref, r_hpl)."""
        lda = self._check_matrix(A)
        info = _lib.LuResidualInfo()
        _check(self._L.lu_residual(self._h, _ptr(A), lda, _ptr(x), _ptr(b), ctypes.byref(info), _stream(stream)),
               "lu_residual")
        return {k: getattr(info, k) for k, _ in info._fields_}

    def adjoint(self, LU, ipiv, X, W, gradB=None, gradA=None, want_gradA=True, stream=None):
        """Adjoint of X = A^{-1} B (no reference counterpart): lambda =
        A^{-T} W into gradB, grad_A = -lambda X^T into gradA (lu_adjoint).
        Returns (gradA or None, gradB)."""
        lda = self._check_matrix(LU)
        n = self.n
        for t, nm in ((X, "X"), (W, "W")):
            _require_cuda(t, torch.float64, nm)
        X2 = X if X.dim() == 2 else X.view(-1, 1)
        W2 = W.contiguous() if W.dim() == 2 else W.contiguous().view(-1, 1)
        k = W2.shape[1]
        if gradB is None:
            gradB = torch.empty(n, k, dtype=torch.float64, device=LU.device)
        if want_gradA and gradA is None:
            gradA = torch.empty(n, n, dtype=torch.float64, device=LU.device)
        gB = gradB if gradB.dim() == 2 else gradB.view(-1, 1)
        _check(self._L.lu_adjoint(self._h, _ptr(LU), lda, _ptr(ipiv), _ptr(X2), X2.stride(0) if k > 1 else 1,
                                  _ptr(W2), W2.stride(0) if k > 1 else 1, k, _ptr(gB), gB.stride(0) if k > 1 else 1,
                                  _ptr(gradA) if want_gradA else None, gradA.stride(0) if want_gradA else n,
                                  _stream(stream)), "lu_adjoint")
        return (gradA if want_gradA else None), gradB

    def profile(self, enable=True):
        """Bracket every phase of later calls with CUDA events (lu_profile)."""
        _check(self._L.lu_profile(self._h, int(bool(enable))), "lu_profile")

    def phase_times(self):
        """{phase: (ms, calls, flops)} since the last call (synchronises)."""
        n = len(_lib.PHASES)
        ms = (ctypes.c_double * n)()
        cnt = (ctypes.c_int64 * n)()
        fl = (ctypes.c_double * n)()
        _check(self._L.lu_phase_times(self._h, ms, cnt, fl), "lu_phase_times")
        return {p: (ms[i], int(cnt[i]), fl[i]) for i, p in enumerate(_lib.PHASES)}

    def refine_solve(self, A, b, x=None, stream=None):
        """Mixed-precision factor + FP64 iterative refinement (A, b untouched)."""
        lda = self._check_matrix(A)
        _require_cuda(b, torch.float64, "b")
        if x is None:
            x = torch.empty_like(b)
        info = _lib.LuRefineInfo()
        _check(self._L.lu_refine_solve(self._h, _ptr(A), lda, _ptr(b), _ptr(x), ctypes.byref(info),
                                       _stream(stream)), "lu_refine_solve")
        return x, {k: getattr(info, k) for k, _ in info._fields_}

    def refine_solve_host(self, A_host, b, x=None, stream=None):
        """refine_solve with the FP64 matrix in host memory (CPU tensor,
        pinned for full copy speed; lu_refine_solve_host). Its leading rows
        stay in HBM as far as they fit beside the FP32 factors; each pass over
        A streams the others in row chunks. info["host_bytes"] counts the
        bytes copied."""
        if not isinstance(A_host, torch.Tensor) or A_host.device.type != "cpu" or A_host.dtype != torch.float64:
            raise LUError(LU_ERR_ARG, "A_host must be a float64 CPU tensor")
        n = self.n
        if A_host.dim() != 2 or A_host.shape[0] != n or A_host.shape[1] != n or A_host.stride(1) != 1:
            raise LUError(LU_ERR_ARG, "A_host must be n x n with unit column stride")
        _require_cuda(b, torch.float64, "b")
        if x is None:
            x = torch.empty_like(b)
        info = _lib.LuRefineInfo()
        _check(self._L.lu_refine_solve_host(self._h, _ptr(A_host), A_host.stride(0), _ptr(b), _ptr(x),
                                            ctypes.byref(info), _stream(stream)), "lu_refine_solve_host")
        return x, {k: getattr(info, k) for k, _ in info._fields_}

    def refine_factor(self, A, stream=None):
        """Low-precision factorisation of A kept in the handle for
        refine_apply / refine_adjoint (lu_refine_factor; A untouched)."""
        lda = self._check_matrix(A)
        _check(self._L.lu_refine_factor(self._h, _ptr(A), lda, _stream(stream)), "lu_refine_factor")

    def refine_precond_norm(self, A, iters=10, stream=None):
        """Power-iteration estimate of ||I - M^{-1} A|| for the factors M kept
        by refine_factor (lu_refine_precond_norm): classical refinement
        contracts by about this factor per step."""
        lda = self._check_matrix(A)
        est = ctypes.c_double(0.0)
        _check(self._L.lu_refine_precond_norm(self._h, _ptr(A), lda, int(iters), ctypes.byref(est),
                                              _stream(stream)), "lu_refine_precond_norm")
        return est.value

    def refine_apply(self, A, B, X=None, trans=False, stream=None):
        """op(A) X = B (op = A^T with trans) by FP64 iterative refinement on
        the kept low-precision factors (lu_refine_apply).  Returns (X, info)."""
        lda = self._check_matrix(A)
        _require_cuda(B, torch.float64, "B")
        B2 = B.contiguous() if B.dim() == 2 else B.contiguous().view(-1, 1)
        k = B2.shape[1]
        if X is None:
            X = torch.empty(B.shape, dtype=torch.float64, device=A.device)
        X2 = X if X.dim() == 2 else X.view(-1, 1)
        info = _lib.LuRefineInfo()
        _check(self._L.lu_refine_apply(self._h, _ptr(A), lda, int(bool(trans)), _ptr(B2), B2.stride(0) if k > 1 else 1,
                                       _ptr(X2), X2.stride(0) if k > 1 else 1, k, ctypes.byref(info),
                                       _stream(stream)), "lu_refine_apply")
        return X, {f: getattr(info, f) for f, _ in info._fields_}

    def refine_adjoint(self, A, X, W, want_gradA=True, stream=None):
        """Adjoint of X = A^{-1} B on the kept low-precision factors:
        lambda = A^{-T} W by FP64 refinement, grad_A = -lambda X^T
        (lu_refine_adjoint).  Returns (gradA or None, gradB, info)."""
        lda = self._check_matrix(A)
        n = self.n
        for t, nm in ((X, "X"), (W, "W")):
            _require_cuda(t, torch.float64, nm)
        X2 = X.contiguous() if X.dim() == 2 else X.contiguous().view(-1, 1)
        W2 = W.contiguous() if W.dim() == 2 else W.contiguous().view(-1, 1)
        k = W2.shape[1]
        gradB = torch.empty(W.shape, dtype=torch.float64, device=A.device)
        gB = gradB if gradB.dim() == 2 else gradB.view(-1, 1)
        gradA = torch.empty(n, n, dtype=torch.float64, device=A.device) if want_gradA else None
        info = _lib.LuRefineInfo()
        _check(self._L.lu_refine_adjoint(self._h, _ptr(A), lda, _ptr(X2), X2.stride(0) if k > 1 else 1, _ptr(W2),
                                         W2.stride(0) if k > 1 else 1, k, _ptr(gB), gB.stride(0) if k > 1 else 1,
                                         _ptr(gradA) if want_gradA else None, n, ctypes.byref(info),
                                         _stream(stream)), "lu_refine_adjoint")
        return gradA, gradB, {f: getattr(info, f) for f, _ in info._fields_}


def launch_count():
    """Kernels liblu_b200 has launched since it was loaded."""
    return int(_lib.load().lu_launch_count())


def transpose_square(A, stream=None):
    """A <- A^T in place for a square float64 CUDA matrix with unit column
    stride (lu_transpose_square): converts the storage between row- and
    column-major."""
    _require_cuda(A, torch.float64, "A")
    if A.dim() != 2 or A.shape[0] != A.shape[1] or A.stride(1) != 1:
        raise LUError(LU_ERR_ARG, "A must be square with unit column stride")
    _check(_lib.load().lu_transpose_square(_ptr(A), A.shape[0], A.stride(0), _stream(stream)),
           "lu_transpose_square")
    return A


def generate_uniform(rows, cols, seed=42, stream_id=0, device="cuda", out=None):
    """Counter-based uniform[-0.5,0.5) matrix, identical to the oracle's."""
    if out is None:
        out = torch.empty(rows, cols, dtype=torch.float64, device=device)
    _require_cuda(out, torch.float64, "out")
    ld = out.stride(0) if out.dim() == 2 else cols
    _check(_lib.load().lu_generate_uniform(_ptr(out), int(rows), int(cols), int(ld), int(seed), int(stream_id),
                                           _stream()), "lu_generate_uniform")
    return out


def matgen(count, seed=9934835, skip=0):
    """The reference's b generator MatGen (benchmark.C:28-74), host side."""
    import numpy as np
    out = np.empty(int(count), dtype=np.float64)
    _check(_lib.load().lu_matgen_host(ctypes.c_void_p(out.ctypes.data), int(count), int(seed), int(skip)),
           "lu_matgen_host")
    return out

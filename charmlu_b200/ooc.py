"""FP64 LU with partial pivoting, and the solve, for a matrix kept in host
memory: orders whose FP64 matrix (8 n^2 bytes) does not fit in HBM.

The reference bounds the memory a node spends on blocks in flight with its
memThreshold scheduler (scheduler.C:46-47, 448-484). On one GPU the whole
matrix normally lives in HBM, so this is the form that bound takes when it
cannot: a left-looking blocked LU over column panels of width w, with only
three n x w panels on the device. Per panel k (columns c0 .. c1):
  1. the panel's columns are copied in, and the pivots of every earlier
     panel are applied to them (lu_apply_pivots);
  2. for each earlier panel j, its columns are copied in (double-buffered
     on a copy stream, so the copy of panel j+1 overlaps the work on panel
     j) and brought up to date with the pivots chosen after it. Then the
     U block of rows j is solved (lu_trsm_lower_unit) and the rows below
     are updated (lu_gemm_update);
  3. rows c0 .. n are factored (lu_panel_factor) and the panel is copied
     back.
A last pass applies the pivots chosen after each panel to its L columns, so
the host matrix ends as lu_factor leaves its matrix (LAPACK layout, global
0-based pivots). The arithmetic runs in this library's kernels
(CudaBlocks). Host <-> device traffic is about 8 n^2 (n/(2w) + 4) bytes, so
a wide panel keeps the GEMMs (K = w) ahead of the copies.

The mixed-precision form (lu_refine_solve_host) is faster where FP32
factors fit in HBM. This path keeps FP64 factors for orders past that, or
when the factors themselves are wanted.
"""
import torch

from .blocks import CudaBlocks


class OutOfCoreLU:
    """LU of an n x n row-major FP64 matrix in host memory (pinned for copy
    speed) through panels of `panel` columns on `device`."""

    def __init__(self, n, panel=None, b=256, blocks=None, device=None, device_budget=None):
        if n < 1:
            raise ValueError("n >= 1 required")
        self.n = int(n)
        self.device = torch.device(device) if device is not None else torch.device(
            "cuda", torch.cuda.current_device())
        self.cuda = self.device.type == "cuda"
        self.blocks = blocks if blocks is not None else CudaBlocks(self.n, b)
        if panel is None:
            if device_budget is None:
                free = torch.cuda.mem_get_info(self.device)[0] if self.cuda else 1 << 33
                device_budget = free // 2
            panel = max(b, (int(device_budget) // (3 * 8 * self.n)) // b * b)
        self.w = max(2, min(int(panel), self.n))
        self.w += self.w & 1
        self.ld = self.w
        self.status_code = 0
        if self.cuda:
            self.copy_stream = torch.cuda.Stream(device=self.device)

    # ---- copies and their ordering ---------------------------------------
    def _copy(self, dst, src, after=None):
        """dst <- src on the copy stream after `after` (an event, or the
        main stream's work so far when None); returns an event the main
        stream can wait on."""
        if not self.cuda:
            dst.copy_(src)
            return None
        if after is None:
            self.copy_stream.wait_stream(torch.cuda.current_stream(self.device))
        else:
            self.copy_stream.wait_event(after)
        with torch.cuda.stream(self.copy_stream):
            self.blocks.copy_2d(dst, src)
            ev = torch.cuda.Event()
            ev.record()
        return ev

    def _wait(self, ev):
        if ev is not None:
            torch.cuda.current_stream(self.device).wait_event(ev)

    def _mark(self):
        if not self.cuda:
            return None
        ev = torch.cuda.Event()
        ev.record()
        return ev

    def _cols(self, j):
        c0 = j * self.w
        return c0, min(self.n, c0 + self.w)

    def _stream_panels(self, A_host, order, bufs):
        """Yields (j, device view of panel j's columns, all rows) for j in
        `order`, the copy of the next one in flight while the caller works
        on the current one. A buffer is reused only after the caller's
        work on it (recorded when control returns here) is done."""
        n = self.n
        freed = [None, None]
        pending = None
        for i, j in enumerate(order):
            c0, c1 = self._cols(j)
            if pending is None:
                pending = self._copy(bufs[i % 2][:, :c1 - c0], A_host[:, c0:c1], freed[i % 2])
            ready = pending
            if i + 1 < len(order):
                d0, d1 = self._cols(order[i + 1])
                pending = self._copy(bufs[(i + 1) % 2][:, :d1 - d0], A_host[:, d0:d1], freed[(i + 1) % 2])
            else:
                pending = None
            self._wait(ready)
            yield j, bufs[i % 2][:n, :c1 - c0]
            freed[i % 2] = self._mark()

    # ---- factorisation ---------------------------------------------------
    def factor(self, A_host):
        """P A = L U in place in A_host (n x n float64, unit column stride).
        Returns the pivots (device int32, 0-based global rows, as
        lu_factor's); self.status_code holds the first singular column
        (1-based) or 0."""
        n, w, bl = self.n, self.w, self.blocks
        nbp = (n + w - 1) // w
        dev = self.device
        bl.clear_status()
        ipiv = torch.zeros(n, dtype=torch.int32, device=dev)
        P = torch.empty(n, self.ld, dtype=torch.float64, device=dev)
        bufs = [torch.empty(n, self.ld, dtype=torch.float64, device=dev) for _ in range(2)]
        stored = None
        for k in range(nbp):
            c0, c1 = self._cols(k)
            wk = c1 - c0
            Pk = P[:, :wk]
            # the previous panel's copy back (on the copy stream) precedes this copy in
            self._wait(self._copy(Pk, A_host[:, c0:c1], stored))
            if c0 > 0:
                bl.apply_pivots(Pk, wk, ipiv, 0, c0, 0, 0)
            for j, Lj in self._stream_panels(A_host, range(k), bufs):
                j0, j1 = self._cols(j)
                if j1 < c0:  # pivots chosen after panel j reach its rows here
                    bl.apply_pivots(Lj, j1 - j0, ipiv, j1, c0 - j1, 0, 0)
                bl.trsm_lower_unit(Lj[j0:j1], Pk[j0:j1])
                bl.gemm_update(Lj[j1:], Pk[j0:j1], Pk[j1:])
            bl.panel_factor(Pk[c0:], ipiv[c0:c1], c0)
            stored = self._copy(A_host[:, c0:c1], Pk, None)
        self._wait(stored)
        # later pivots into each earlier panel's L columns
        for j, Lj in self._stream_panels(A_host, range(nbp - 1), bufs):
            j0, j1 = self._cols(j)
            bl.apply_pivots(Lj, j1 - j0, ipiv, j1, n - j1, 0, 0)
            self._wait(self._copy(A_host[:, j0:j1], Lj, None))
        if self.cuda:
            torch.cuda.current_stream(dev).synchronize()
        self.status_code = bl.status()
        return ipiv

    # ---- solve -----------------------------------------------------------
    def solve(self, A_host, ipiv, rhs):
        """x = A^{-1} rhs from the factors factor() left in A_host (rhs a
        float64 vector on the device)."""
        n, bl = self.n, self.blocks
        nbp = (n + self.w - 1) // self.w
        bufs = [torch.empty(n, self.ld, dtype=torch.float64, device=self.device) for _ in range(2)]
        y = rhs.clone()
        bl.apply_pivots(None, 0, ipiv, 0, n, 0, 0, y)
        for j, Lj in self._stream_panels(A_host, range(nbp), bufs):  # y <- L^{-1} P b
            j0, j1 = self._cols(j)
            bl.trsv_block(Lj[j0:j1], 0, y[j0:j1])
            if j1 < n:
                bl.gemv_update(Lj[j1:], y[j0:j1], y[j1:])
        for j, Lj in self._stream_panels(A_host, range(nbp - 1, -1, -1), bufs):  # x <- U^{-1} y
            j0, j1 = self._cols(j)
            bl.trsv_block(Lj[j0:j1], 1, y[j0:j1])
            if j0 > 0:
                bl.gemv_update(Lj[:j0], y[j0:j1], y[:j0])
        if self.cuda:
            torch.cuda.current_stream(self.device).synchronize()
        return y

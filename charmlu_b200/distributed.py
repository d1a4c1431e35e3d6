"""Dense LU with partial pivoting over several GPUs, one process per GPU:
a 1D column-block-cyclic distribution over torch.distributed (NCCL).

The reference distributes the matrix as b x b block chares mapped over PEs
(mapping.h:14-75). The column holding the diagonal block factors the panel:
pivot search with a reduction over its blocks, and swaps (lu.ci:256-370).
Its pivots are multicast to every block column for the row interchanges
(lu.ci:92-123, 275-333), and the L panel to the trailing blocks for their U
solve and updates (lu.ci:132-251). The scheduler gives the next panel's
column priority (scheduler.C:235-354, manager.h:55-56).

Here each rank keeps the column blocks j with j % world == rank, all N rows,
in one row-major device matrix. Per step k:
  1. the owner of block column k factors its panel (rows k*b .. N) in place
     (lu_panel_factor) and broadcasts it, with its pivots, to every rank;
  2. every rank applies the panel's row interchanges to its other columns
     (lu_apply_pivots), solves the U block row of its trailing columns
     (lu_trsm_lower_unit), and updates them (lu_gemm_update);
  3. with look-ahead, the owner of block column k+1 first updates that
     panel's columns, then factors it on a high-priority side stream and
     posts its broadcast (asynchronous) from there, while the rest of its
     update runs on the main stream: panel, transfer and GEMM overlap. Every
     rank posts the same broadcasts in the same order.
The solve keeps b replicated. Each diagonal block's owner solves it
(lu_trsv_block), updates the remaining entries (lu_gemv_update) and
broadcasts them.

All arithmetic runs in this library's kernels through the C ABI (the
CudaBlocks class). torch provides device memory, the copies that pack
panels into broadcast buffers, and the collectives. A blocks object with the
same methods can stand in, for testing the distribution on CPU ranks.
"""
import torch
import torch.distributed as dist


from .blocks import CudaBlocks  # noqa: F401  (the default per-block operations)


class BlockCyclicLU:
    """LU of an n x n matrix distributed by column blocks of width b over the
    ranks of `group`: rank r holds the blocks j with j % world == r, in
    ascending j, side by side in one n x ld local matrix (ld even)."""

    def __init__(self, n, b, group=None, blocks=None, device=None, lookahead=True):
        if n < 1 or b < 2 or b % 2:
            raise ValueError("n >= 1 and an even block size b >= 2 are required")
        self.n, self.b = int(n), int(b)
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.nb = (self.n + self.b - 1) // self.b
        self.device = torch.device(device) if device is not None else torch.device(
            "cuda", torch.cuda.current_device())
        self.lookahead = bool(lookahead)
        self.blocks = blocks if blocks is not None else CudaBlocks(self.n, self.b, lookahead=self.lookahead)
        # with look-ahead on a GPU, the next panel is factored on a
        # high-priority stream beside the rest of the update
        self.side = None
        if self.lookahead and isinstance(self.blocks, CudaBlocks):
            self.side = torch.cuda.Stream(device=self.device, priority=-1)
        self.owned = [j for j in range(self.nb) if j % self.world == self.rank]
        self.col_off = {}
        off = 0
        for j in self.owned:
            self.col_off[j] = off
            off += self.width(j)
        self.ncols = off
        # one pitch on every rank (the widest rank's column count, even), so
        # local matrices have the same shape for the gather
        widest = max(sum(self.width(j) for j in range(r, self.nb, self.world)) for r in range(self.world))
        self.ld = max(2, widest + (widest & 1))
        self.ldp = self.b  # panel buffer pitch (b is even)
        self.status_code = 0

    # ---- layout ---------------------------------------------------------
    def width(self, j):
        return min(self.b, self.n - j * self.b)

    def owner(self, j):
        return j % self.world

    def empty_local(self):
        """Zeroed local matrix (n x ld); its first ncols columns are this
        rank's blocks."""
        return torch.zeros(self.n, self.ld, dtype=torch.float64, device=self.device)

    def scatter(self, A):
        """This rank's column blocks of a full n x n matrix (any device)."""
        loc = self.empty_local()
        for j in self.owned:
            c = self.col_off[j]
            loc[:, c:c + self.width(j)].copy_(A[:, j * self.b:j * self.b + self.width(j)])
        return loc

    def gather(self, loc):
        """The full n x n matrix from every rank's local matrix (all ranks
        receive it; for checks and small orders)."""
        parts = [torch.empty_like(loc) for _ in range(self.world)]
        dist.all_gather(parts, loc.contiguous(), group=self.group)
        full = torch.empty(self.n, self.n, dtype=torch.float64, device=loc.device)
        for r in range(self.world):
            off = 0
            for j in range(r, self.nb, self.world):
                w = self.width(j)
                full[:, j * self.b:j * self.b + w].copy_(parts[r][:, off:off + w])
                off += w
        return full

    def _trailing_start(self, k):
        """First local column of this rank's blocks right of block k."""
        for j in self.owned:
            if j > k:
                return self.col_off[j]
        return self.ncols

    # ---- factorisation --------------------------------------------------
    def _bcast(self, buf, src, async_op):
        return dist.broadcast(buf, src=src, group=self.group, async_op=async_op)

    def _panel_message(self, bufs, k):
        m = self.n - k * self.b
        return bufs[k % 2][:m * self.ldp + self.width(k)]

    def _factor_and_pack(self, loc, ipiv, bufs, k):
        """Owner of block column k: factor its panel in place and pack the
        panel and its pivots (as doubles) into the broadcast buffer."""
        k0, kw = k * self.b, self.width(k)
        m = self.n - k0
        c = self.col_off[k]
        self.blocks.panel_factor(loc[k0:, c:c + kw], ipiv[k0:k0 + kw], k0)
        msg = self._panel_message(bufs, k)
        msg[:m * self.ldp].view(m, self.ldp)[:, :kw].copy_(loc[k0:, c:c + kw])
        msg[m * self.ldp:].copy_(ipiv[k0:k0 + kw])

    def factor(self, loc):
        """Factor the distributed matrix in place (L unit lower and U on the
        owners' columns, rows interchanged across all columns as lu_factor
        does). Returns the pivots (device int32, n, the same on every rank);
        self.status_code holds the first singular column (1-based, lowest
        over ranks) or 0."""
        n, b, me = self.n, self.b, self.rank
        self.blocks.clear_status()
        ipiv = torch.zeros(n, dtype=torch.int32, device=self.device)
        bufs = [torch.zeros(n * self.ldp + b, dtype=torch.float64, device=self.device) for _ in range(2)]
        if self.owner(0) == me:
            self._factor_and_pack(loc, ipiv, bufs, 0)
        pending = self._bcast(self._panel_message(bufs, 0), self.owner(0), self.lookahead)
        for k in range(self.nb):
            k0, kw = k * b, self.width(k)
            k1, m = k0 + kw, n - k0
            if pending is not None:
                pending.wait()
            msg = self._panel_message(bufs, k)
            own = self.owner(k) == me
            if own:
                c = self.col_off[k]
                Lkk, L21 = loc[k0:k1, c:c + kw], loc[k1:, c:c + kw]
                skip = (c, c + kw)
            else:
                ipiv[k0:k1].copy_(msg[m * self.ldp:])
                panel = msg[:m * self.ldp].view(m, self.ldp)[:, :kw]
                Lkk, L21 = panel[:kw], panel[kw:]
                skip = (0, 0)
            if self.ncols > 0:  # a rank may own no block when world > nb
                self.blocks.apply_pivots(loc, self.ncols, ipiv, k0, kw, skip[0], skip[1])
            t0 = self._trailing_start(k)
            nxt = k + 1 if k + 1 < self.nb else None
            if t0 < self.ncols and k1 < n:
                U = loc[k0:k1, t0:self.ncols]
                self.blocks.trsm_lower_unit(Lkk, U)
                if self.lookahead and nxt is not None and self.owner(nxt) == me:
                    # next panel's columns first, then factor and post it
                    w1 = self.width(nxt)
                    self.blocks.gemm_update(L21, U[:, :w1], loc[k1:, t0:t0 + w1])
                    if self.side is not None:
                        # the panel's columns are disjoint from the rest of
                        # the update; the next step waits on the broadcast,
                        # which follows the panel on the side stream
                        self.side.wait_stream(torch.cuda.current_stream(self.device))
                        with torch.cuda.stream(self.side):
                            self._factor_and_pack(loc, ipiv, bufs, nxt)
                            pending = self._bcast(self._panel_message(bufs, nxt), self.owner(nxt), True)
                    else:
                        self._factor_and_pack(loc, ipiv, bufs, nxt)
                        pending = self._bcast(self._panel_message(bufs, nxt), self.owner(nxt), True)
                    nxt = None
                    if t0 + w1 < self.ncols:
                        self.blocks.gemm_update(L21, U[:, w1:], loc[k1:, t0 + w1:self.ncols])
                else:
                    self.blocks.gemm_update(L21, U, loc[k1:, t0:self.ncols])
            if nxt is not None:
                if self.owner(nxt) == me:
                    self._factor_and_pack(loc, ipiv, bufs, nxt)
                pending = self._bcast(self._panel_message(bufs, nxt), self.owner(nxt), self.lookahead)
            elif not self.lookahead or k + 1 >= self.nb:
                pending = None
        self.status_code = self._reduce_status(self.blocks.status())
        return ipiv

    def _reduce_status(self, code):
        t = torch.tensor([code], dtype=torch.int64, device=self.device)
        allc = [torch.zeros_like(t) for _ in range(self.world)]
        dist.all_gather(allc, t, group=self.group)
        codes = [int(c.item()) for c in allc]
        neg = [c for c in codes if c < 0]
        if neg:
            return min(neg)
        pos = [c for c in codes if c > 0]
        return min(pos) if pos else 0

    # ---- solve ----------------------------------------------------------
    def solve(self, loc, ipiv, rhs):
        """x = A^{-1} rhs from the distributed factors (rhs replicated on
        every rank, device float64 vector; returned replicated)."""
        n, b, me = self.n, self.b, self.rank
        y = rhs.clone()
        self.blocks.apply_pivots(loc, 0, ipiv, 0, n, 0, 0, y)
        for k in range(self.nb):  # y <- L^{-1} P b
            k0, kw = k * b, self.width(k)
            k1 = k0 + kw
            if self.owner(k) == me:
                c = self.col_off[k]
                self.blocks.trsv_block(loc[k0:k1, c:c + kw], 0, y[k0:k1])
                if k1 < n:
                    self.blocks.gemv_update(loc[k1:, c:c + kw], y[k0:k1], y[k1:])
            self._bcast(y[k0:], self.owner(k), False)
        for k in range(self.nb - 1, -1, -1):  # x <- U^{-1} y
            k0, kw = k * b, self.width(k)
            k1 = k0 + kw
            if self.owner(k) == me:
                c = self.col_off[k]
                self.blocks.trsv_block(loc[k0:k1, c:c + kw], 1, y[k0:k1])
                if k0 > 0:
                    self.blocks.gemv_update(loc[:k0, c:c + kw], y[k0:k1], y[:k0])
            self._bcast(y[:k1], self.owner(k), False)
        return y

"""Dense LU with partial pivoting over several GPUs, one process per GPU:
block-cyclic distributions over torch.distributed (NCCL), 1D by column
blocks (BlockCyclicLU) and 2D over a P x Q process grid (BlockCyclic2DLU).

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


class BlockCyclic2DLU:
    """LU of an n x n matrix over a P x Q process grid, b x b blocks dealt
    block-cyclically in both directions: rank r = pr * Q + pc holds the
    blocks (i, j) with i % P == pr and j % Q == pc, in ascending i and j,
    packed into one local matrix (rows of its row blocks, columns of its
    column blocks; row pitch ld even).

    This is the reference's 2D tiling (mapping.h:28-75: a PE tile of
    peTileRows x peTileCols, the chare (x, y) on tile PE (x % rows, y %
    cols)). Per step k, with pk = k % P and qk = k % Q:
      1. the P ranks of process column qk gather block column k's panel
         (rows k*b .. n) by an all-reduce of their disjoint rows, factor it
         (lu_panel_factor; each computes the same factors and pivots from the
         same data) and keep their rows of the result;
      2. each of them broadcasts the factored panel and its pivots along its
         process row (the reference multicasts the L panel and pivots,
         lu.ci:92-123, 275-333);
      3. the rows the pivots touch are exchanged within every process column
         (an all-reduce of the touched rows' segments) and written back
         interchanged, on every column but the panel's (sendPendingPivots /
         applySwap, lu.C:46-169);
      4. process row pk solves its part of the U block row with the panel's
         unit lower triangle (computeU, lu.C:180-189) and broadcasts it down
         each process column;
      5. every rank updates its trailing blocks: its rows of L21 times its
         columns of U12 (updateMatrix, lu.C:26-43).
    The solve keeps b replicated: each diagonal block's owner solves it
    (lu_trsv_block) and broadcasts it, and the process column holding that
    block column updates its rows (lu_gemv_update), which an all-reduce of
    disjoint entries makes known to every rank (forwardSolve /
    backwardSolve / offDiagSolve, lu.ci:387-456).

    The groups span the default process group (world size P * Q). Every
    arithmetic step runs in the per-block kernels (`blocks`); torch provides
    the buffers, the index copies that pack rows and the collectives."""

    def __init__(self, n, b, P, Q, blocks=None, device=None):
        if n < 1 or b < 2 or b % 2:
            raise ValueError("n >= 1 and an even block size b >= 2 are required")
        world = dist.get_world_size()
        if P < 1 or Q < 1 or P * Q != world:
            raise ValueError(f"a {P} x {Q} grid needs {P * Q} ranks, the process group has {world}")
        self.n, self.b, self.P, self.Q = int(n), int(b), int(P), int(Q)
        self.rank = dist.get_rank()
        self.pr, self.pc = divmod(self.rank, self.Q)
        self.nb = (self.n + self.b - 1) // self.b
        self.device = torch.device(device) if device is not None else torch.device(
            "cuda", torch.cuda.current_device())
        self.blocks = blocks if blocks is not None else CudaBlocks(self.n, self.b)
        # every rank creates every group, in the same order
        self.row_groups = [dist.new_group([r * self.Q + c for c in range(self.Q)]) for r in range(self.P)]
        self.col_groups = [dist.new_group([r * self.Q + c for r in range(self.P)]) for c in range(self.Q)]
        self.my_rb = [i for i in range(self.nb) if i % self.P == self.pr]
        self.my_cb = [j for j in range(self.nb) if j % self.Q == self.pc]
        self.row_off, self.col_off = {}, {}
        off = 0
        for i in self.my_rb:
            self.row_off[i] = off
            off += self.width(i)
        self.nrows = off
        off = 0
        for j in self.my_cb:
            self.col_off[j] = off
            off += self.width(j)
        self.ncols = off
        # the same local shape on every rank (for the gather): the largest
        # row and column counts, the pitch even
        rows = [sum(self.width(i) for i in range(r, self.nb, self.P)) for r in range(self.P)]
        cols = [sum(self.width(j) for j in range(c, self.nb, self.Q)) for c in range(self.Q)]
        self.rows_max = max(1, max(rows))
        self.ld = max(2, max(cols) + (max(cols) & 1))
        self.ldp = self.b
        # global row of each local row
        g = [i * self.b + t for i in self.my_rb for t in range(self.width(i))]
        self.grow = torch.tensor(g, dtype=torch.int64)
        self.status_code = 0

    # ---- layout ---------------------------------------------------------
    def width(self, j):
        return min(self.b, self.n - j * self.b)

    def owner(self, i, j):
        """Rank holding block (i, j)."""
        return (i % self.P) * self.Q + (j % self.Q)

    def empty_local(self):
        return torch.zeros(self.rows_max, self.ld, dtype=torch.float64, device=self.device)

    def _local_row(self, g):
        i = g // self.b
        return self.row_off[i] + (g - i * self.b) if i % self.P == self.pr else None

    def _first_local_row_from(self, g0):
        """First local row whose global row is >= g0 (local rows ascend)."""
        return int(torch.searchsorted(self.grow, torch.tensor(g0, dtype=torch.int64)).item()) \
            if self.nrows else 0

    def _first_local_col_after(self, k):
        for j in self.my_cb:
            if j > k:
                return self.col_off[j]
        return self.ncols

    def scatter(self, A):
        """This rank's blocks of a full n x n matrix (any device)."""
        loc = self.empty_local()
        for i in self.my_rb:
            r, wi = self.row_off[i], self.width(i)
            for j in self.my_cb:
                c, wj = self.col_off[j], self.width(j)
                loc[r:r + wi, c:c + wj].copy_(A[i * self.b:i * self.b + wi, j * self.b:j * self.b + wj])
        return loc

    def gather(self, loc):
        """The full matrix from every rank's blocks (all ranks receive it)."""
        parts = [torch.empty_like(loc) for _ in range(self.P * self.Q)]
        dist.all_gather(parts, loc.contiguous())
        full = torch.empty(self.n, self.n, dtype=torch.float64, device=loc.device)
        for rank, part in enumerate(parts):
            pr, pc = divmod(rank, self.Q)
            ro = 0
            for i in range(pr, self.nb, self.P):
                wi = self.width(i)
                co = 0
                for j in range(pc, self.nb, self.Q):
                    wj = self.width(j)
                    full[i * self.b:i * self.b + wi, j * self.b:j * self.b + wj].copy_(part[ro:ro + wi, co:co + wj])
                    co += wj
                ro += wi
        return full

    # ---- factorisation --------------------------------------------------
    def factor(self, loc):
        """Factor the distributed matrix in place (the layout of lu_factor:
        L unit lower and U, rows interchanged across all columns). Returns
        the pivots (int32 on the device, n, the same on every rank);
        self.status_code holds the first singular column (1-based) or 0."""
        n, b, dev = self.n, self.b, self.device
        self.blocks.clear_status()
        ipiv = torch.zeros(n, dtype=torch.int32, device=dev)
        grow = self.grow.to(dev)
        for k in range(self.nb):
            k0, kw = k * b, self.width(k)
            k1, m = k0 + kw, n - k0
            pk, qk = k % self.P, k % self.Q
            lr0 = self._first_local_row_from(k0)
            msg = torch.zeros(m * self.ldp + kw, dtype=torch.float64, device=dev)
            panel = msg[:m * self.ldp].view(m, self.ldp)
            # 1. the panel, gathered and factored in process column qk
            if self.pc == qk:
                c = self.col_off[k]
                rows = grow[lr0:self.nrows] - k0
                if len(rows):
                    panel[rows, :kw] = loc[lr0:self.nrows, c:c + kw]
                if self.P > 1:
                    dist.all_reduce(msg, group=self.col_groups[qk])
                self.blocks.panel_factor(panel[:, :kw], ipiv[k0:k1], k0)
                if len(rows):
                    loc[lr0:self.nrows, c:c + kw] = panel[rows, :kw]
                msg[m * self.ldp:].copy_(ipiv[k0:k1])
            # 2. panel and pivots along every process row
            if self.Q > 1:
                dist.broadcast(msg, src=self.pr * self.Q + qk, group=self.row_groups[self.pr])
            if self.pc != qk:
                ipiv[k0:k1].copy_(msg[m * self.ldp:])
            # 3. the interchanges, on every local column but the panel's
            self._interchange(loc, ipiv[k0:k1].cpu().tolist(), k0, k)
            # 4. the U block row, solved by process row pk, down every column
            t0 = self._first_local_col_after(k)
            nt = self.ncols - t0
            if nt <= 0 or k1 >= n:
                continue
            ubuf = torch.empty(kw, nt + (nt & 1), dtype=torch.float64, device=dev)
            U = ubuf[:, :nt]
            if self.pr == pk:
                r = self.row_off[k]
                self.blocks.trsm_lower_unit(panel[:kw, :kw], loc[r:r + kw, t0:self.ncols])
                U.copy_(loc[r:r + kw, t0:self.ncols])
            if self.P > 1:
                dist.broadcast(ubuf, src=pk * self.Q + self.pc, group=self.col_groups[self.pc])
            # 5. the trailing update of this rank's blocks
            lr1 = self._first_local_row_from(k1)
            mr = self.nrows - lr1
            if mr > 0:
                lbuf = torch.empty(mr, kw + (kw & 1), dtype=torch.float64, device=dev)
                L21 = lbuf[:, :kw]
                L21.copy_(panel[grow[lr1:self.nrows] - k0, :kw])
                self.blocks.gemm_update(L21, U, loc[lr1:self.nrows, t0:self.ncols])
        self.status_code = self._reduce_status(self.blocks.status())
        return ipiv

    def _interchange(self, loc, piv, k0, k):
        """Apply the swaps (k0 + t) <-> piv[t] in order to this rank's
        columns, except block column k's (already interchanged inside the
        panel): the touched rows are exchanged within the process column."""
        touched = sorted(set(range(k0, k0 + len(piv))) | set(int(p) for p in piv))
        content = {g: g for g in touched}  # row g ends up holding old row content[g]
        for t, p in enumerate(piv):
            i = k0 + t
            if p != i:
                content[i], content[p] = content[p], content[i]
        if all(content[g] == g for g in touched) or self.ncols == 0:
            return
        pos = {g: t for t, g in enumerate(touched)}
        buf = torch.zeros(len(touched), self.ld, dtype=torch.float64, device=self.device)
        mine = [(t, self._local_row(g)) for t, g in enumerate(touched) if self._local_row(g) is not None]
        dev = self.device
        if mine:
            bi = torch.tensor([t for t, _ in mine], dtype=torch.int64, device=dev)
            li = torch.tensor([r for _, r in mine], dtype=torch.int64, device=dev)
            buf[bi] = loc[li]
        if self.P > 1:
            dist.all_reduce(buf, group=self.col_groups[self.pc])
        if not mine:
            return
        src = torch.tensor([pos[content[touched[t]]] for t, _ in mine], dtype=torch.int64, device=dev)
        newrows = buf[src]
        spans = [(0, self.ncols)]
        if self.pc == k % self.Q:
            c = self.col_off[k]
            spans = [(0, c), (c + self.width(k), self.ncols)]
        for c0, c1 in spans:
            if c1 > c0:
                loc[li, c0:c1] = newrows[:, c0:c1]

    def _reduce_status(self, code):
        t = torch.tensor([code], dtype=torch.int64, device=self.device)
        allc = [torch.zeros_like(t) for _ in range(self.P * self.Q)]
        dist.all_gather(allc, t)
        codes = [int(c.item()) for c in allc]
        neg = [c for c in codes if c < 0]
        if neg:
            return min(neg)
        pos = [c for c in codes if c > 0]
        return min(pos) if pos else 0

    # ---- solve ----------------------------------------------------------
    def solve(self, loc, ipiv, rhs):
        """x = A^{-1} rhs from the distributed factors (rhs replicated on
        every rank, a float64 vector on the device; returned replicated)."""
        n, b, dev = self.n, self.b, self.device
        perm = list(range(n))  # y <- P b: the pivots applied in order
        for i, p in enumerate(ipiv.cpu().tolist()):
            if p != i:
                perm[i], perm[p] = perm[p], perm[i]
        y = rhs[torch.tensor(perm, dtype=torch.int64, device=rhs.device)].clone()
        grow = self.grow.to(dev)
        for k in range(self.nb):  # y <- L^{-1} P b
            k0, kw = k * b, self.width(k)
            k1 = k0 + kw
            if self.owner(k, k) == self.rank:
                r, c = self.row_off[k], self.col_off[k]
                self.blocks.trsv_block(loc[r:r + kw, c:c + kw], 0, y[k0:k1])
            dist.broadcast(y[k0:k1], src=self.owner(k, k))
            if k1 < n:
                self._offdiag_update(loc, y, grow, k, self._first_local_row_from(k1), self.nrows, k1, n)
        for k in range(self.nb - 1, -1, -1):  # x <- U^{-1} y
            k0, kw = k * b, self.width(k)
            k1 = k0 + kw
            if self.owner(k, k) == self.rank:
                r, c = self.row_off[k], self.col_off[k]
                self.blocks.trsv_block(loc[r:r + kw, c:c + kw], 1, y[k0:k1])
            dist.broadcast(y[k0:k1], src=self.owner(k, k))
            if k0 > 0:
                self._offdiag_update(loc, y, grow, k, 0, self._first_local_row_from(k0), 0, k0)
        return y

    def _offdiag_update(self, loc, y, grow, k, lr_a, lr_b, g_a, g_b):
        """y[g_a:g_b] -= A[g_a:g_b, block k] y[block k]: the process column
        holding block column k updates its local rows lr_a .. lr_b (global
        rows in [g_a, g_b)).  Every row of the range lives on exactly one of
        that column's ranks, so an all-reduce of the updated entries (zeros
        elsewhere: the sum is exact) gives every rank the result."""
        k0, kw = k * self.b, self.width(k)
        part = torch.zeros(g_b - g_a, dtype=torch.float64, device=self.device)
        if self.pc == k % self.Q and lr_b > lr_a:
            c = self.col_off[k]
            rows = grow[lr_a:lr_b]
            yl = y[rows].clone()
            self.blocks.gemv_update(loc[lr_a:lr_b, c:c + kw], y[k0:k0 + kw], yl)
            part[rows - g_a] = yl
        dist.all_reduce(part)
        y[g_a:g_b] = part

"""torch.autograd binding of the dense solve X = A^{-1} B (no counterpart in
the reference, which has no differentiation).

Forward factors A once with lu_factor and solves with lu_solve; backward
calls lu_adjoint, which reuses the stored factors and pivots for the
transposed solves A^T lambda = dL/dX and forms grad_A = -lambda X^T,
grad_B = lambda.  With refactor=True the factors are not kept: backward
refactors A (which autograd holds anyway), trading one factorisation for
n^2 doubles of memory.
"""
import torch

from . import LUConfig, LUSolver


class LUSolveFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, A, B, block_size=128, refactor=False):
        n = A.shape[0]
        solver = LUSolver(LUConfig(n, block_size))
        lda = n + (n & 1)
        buf = torch.empty(n, lda, dtype=torch.float64, device=A.device)
        LU = buf[:, :n]
        LU.copy_(A.detach())
        ipiv = solver.factor(LU)
        X = B.detach().to(torch.float64).clone().contiguous()
        solver.solve(LU, ipiv, X)
        solver.check("LUSolveFunction.forward")
        ctx.solver = solver
        ctx.refactor = bool(refactor)
        ctx.vector = B.dim() == 1
        if ctx.refactor:
            del buf, LU
            ctx.save_for_backward(A, X)
        else:
            ctx.save_for_backward(LU, ipiv, X)
        return X

    @staticmethod
    def backward(ctx, W):
        solver = ctx.solver
        if ctx.refactor:
            A, X = ctx.saved_tensors
            n = A.shape[0]
            buf = torch.empty(n, n + (n & 1), dtype=torch.float64, device=A.device)
            LU = buf[:, :n]
            LU.copy_(A.detach())
            ipiv = solver.factor(LU)
        else:
            LU, ipiv, X = ctx.saved_tensors
        want_a = ctx.needs_input_grad[0]
        gA, gB = solver.adjoint(LU, ipiv, X, W.to(torch.float64).contiguous(), want_gradA=want_a)
        solver.check("LUSolveFunction.backward")
        if ctx.vector:
            gB = gB.view(-1)
        return gA, (gB if ctx.needs_input_grad[1] else None), None, None


def lu_solve(A, B, block_size=128, refactor=False):
    """Differentiable X = A^{-1} B on the GPU (FP64)."""
    return LUSolveFunction.apply(A, B, block_size, refactor)

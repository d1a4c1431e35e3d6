"""Adjoint of X = A^{-1} B (no reference counterpart): lu_adjoint and the
torch.autograd binding against an FP64 reference gradient and central finite
differences.  Bar: gradients within 1e-10 relative (normwise)
of the FP64 reference gradient."""
import numpy as np
import pytest
import scipy.linalg as sl
import torch

import oracle

pytestmark = pytest.mark.gpu


def _reference_grads(A, B, W):
    """FP64 reference: lambda = A^{-T} W, grad_A = -lambda X^T, grad_B = lambda."""
    lu, piv = sl.lu_factor(A)
    X = sl.lu_solve((lu, piv), B)
    lam = sl.lu_solve((lu, piv), W, trans=1)
    return X, -lam @ X.T, lam


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("n,k,b", [(256, 16, 64), (1000, 3, 128), (4096, 16, 256)])
def test_adjoint_matches_fp64_reference(cuda_dev, n, k, b):
    import charmlu_b200 as lu
    A = oracle.gen_matrix(n, 42)
    B = oracle.gen_uniform(n * k, 42, 2).reshape(n, k)
    W = 2.0 * oracle.gen_uniform(n * k, 42, 3).reshape(n, k)  # uniform[-1, 1)
    X_ref, gA_ref, gB_ref = _reference_grads(A, B, W)
    s = lu.LUSolver(lu.LUConfig(n, b))
    LU = torch.from_numpy(A).cuda()
    ipiv = s.factor(LU)
    X = torch.from_numpy(B).cuda().contiguous()
    s.solve(LU, ipiv, X)
    assert s.status() == 0
    assert _rel(X.cpu().numpy(), X_ref) < 1e-10
    gA, gB = s.adjoint(LU, ipiv, X, torch.from_numpy(W).cuda())
    assert s.status() == 0
    assert _rel(gB.cpu().numpy(), gB_ref) < 1e-10
    assert _rel(gA.cpu().numpy(), gA_ref) < 1e-10


def test_transposed_solve_single_rhs(cuda_dev):
    import charmlu_b200 as lu
    n = 777
    A = oracle.gen_matrix(n, 5)
    w = oracle.gen_vector(n, 6)
    s = lu.LUSolver(lu.LUConfig(n, 64))
    buf = torch.zeros(n, n + 1, dtype=torch.float64, device="cuda")
    LU = buf[:, :n]
    LU.copy_(torch.from_numpy(A))
    ipiv = s.factor(LU)
    y = torch.from_numpy(w).cuda()
    s.solve(LU, ipiv, y, trans=True)
    assert s.status() == 0
    ref = np.linalg.solve(A.T, w)
    assert _rel(y.cpu().numpy(), ref) < 1e-10


def test_autograd_finite_differences(cuda_dev):
    """Central differences (h = 1e-6) of loss = sum(W * X) at N=256."""
    from charmlu_b200.autograd import lu_solve
    n, k = 256, 16
    A = torch.from_numpy(oracle.gen_matrix(n, 9)).cuda().requires_grad_(True)
    B = torch.from_numpy(oracle.gen_uniform(n * k, 9, 2).reshape(n, k)).cuda().requires_grad_(True)
    W = torch.from_numpy(2.0 * oracle.gen_uniform(n * k, 9, 3).reshape(n, k)).cuda()
    loss = (lu_solve(A, B, block_size=64) * W).sum()
    loss.backward()
    gA, gB = A.grad.cpu().numpy(), B.grad.cpu().numpy()
    A0, B0, W0 = A.detach().cpu().numpy(), B.detach().cpu().numpy(), W.cpu().numpy()
    h = 1e-6
    rng = np.random.default_rng(0)

    def f(Am, Bm):
        return float((np.linalg.solve(Am, Bm) * W0).sum())

    for _ in range(6):
        i, j = rng.integers(0, n, 2)
        Ap, Am_ = A0.copy(), A0.copy()
        Ap[i, j] += h
        Am_[i, j] -= h
        fd = (f(Ap, B0) - f(Am_, B0)) / (2 * h)
        assert abs(fd - gA[i, j]) <= 1e-6 * max(1.0, abs(gA).max())
        r, c = rng.integers(0, n), rng.integers(0, k)
        Bp, Bm_ = B0.copy(), B0.copy()
        Bp[r, c] += h
        Bm_[r, c] -= h
        fd = (f(A0, Bp) - f(A0, Bm_)) / (2 * h)
        assert abs(fd - gB[r, c]) <= 1e-6 * max(1.0, abs(gB).max())


def test_autograd_refactor_mode_same_gradient(cuda_dev):
    from charmlu_b200.autograd import lu_solve
    n, k = 512, 4
    A0 = torch.from_numpy(oracle.gen_matrix(n, 11)).cuda()
    B0 = torch.from_numpy(oracle.gen_uniform(n * k, 11, 2).reshape(n, k)).cuda()
    W = torch.from_numpy(oracle.gen_uniform(n * k, 11, 3).reshape(n, k)).cuda()
    grads = []
    for refactor in (False, True):
        A = A0.clone().requires_grad_(True)
        B = B0.clone().requires_grad_(True)
        (lu_solve(A, B, 128, refactor) * W).sum().backward()
        grads.append((A.grad.clone(), B.grad.clone()))
    assert torch.equal(grads[0][1], grads[1][1])
    assert torch.equal(grads[0][0], grads[1][0])


def test_autograd_vector_rhs_and_gradcheck(cuda_dev):
    from charmlu_b200.autograd import lu_solve
    n = 24
    A = (torch.from_numpy(oracle.gen_matrix(n, 4)).cuda() + 3 * torch.eye(n, device="cuda", dtype=torch.float64))
    A.requires_grad_(True)
    b = torch.from_numpy(oracle.gen_vector(n, 4)).cuda().requires_grad_(True)
    assert torch.autograd.gradcheck(lambda A_, b_: lu_solve(A_, b_, 8), (A, b), eps=1e-6, atol=1e-7)

"""Multi-right-hand-side refinement on kept low-precision factors
(lu_refine_factor / lu_refine_apply) and the adjoint on them
(lu_refine_adjoint, MixedLUSolveFunction): no reference counterpart.

Checks: every column of op(A) X = B reaches the scaled residual target
against the FP64 A (recomputed here in numpy), X agrees with the FP64
solution, and the adjoint's gradients agree with the FP64 reference
gradient (lambda = A^{-T} W, grad_A = -lambda X^T) to 1e-10 relative
(max-norm) when refined to r_hpl < 1e-3 (the HPL bar of 16 leaves forward
errors near kappa * n * eps * 16, 1e-10 at n = 2048 and 1e-7 at
n = 32768); storing and refactor modes give the same gradient.
References are LAPACK solutions sharpened by one extended-precision
refinement step."""
import numpy as np
import pytest
import scipy.linalg as sl
import torch

import oracle

pytestmark = pytest.mark.gpu

EPS = 2.220446049250313e-16


def _padded(A):
    n = A.shape[0]
    buf = torch.zeros(n, n + (n & 1), dtype=torch.float64, device="cuda")
    buf[:, :n].copy_(torch.from_numpy(A))
    return buf[:, :n]


def _r_hpl_cols(opA, X, B):
    n = opA.shape[0]
    R = B - opA @ X
    an = np.abs(opA).sum(axis=1).max()
    return np.abs(R).max(axis=0) / ((an * np.abs(X).max(axis=0) + np.abs(B).max(axis=0)) * n * EPS)


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def _accurate_solve(A, B, trans=False):
    """FP64 LAPACK solve of op(A) X = B plus one refinement step whose
    residual is formed in extended precision (x86 long double), so the
    reference's own forward error (~kappa eps) does not enter the 1e-10
    comparisons."""
    f = sl.lu_factor(A)
    t = 1 if trans else 0
    X = sl.lu_solve(f, B, trans=t)
    opA = (A.T if trans else A).astype(np.longdouble)
    R = B.astype(np.longdouble) - opA @ X.astype(np.longdouble)
    return X + sl.lu_solve(f, R.astype(np.float64), trans=t)


@pytest.mark.parametrize("trans", [0, 1])
@pytest.mark.parametrize("n,k,b,prec", [(999, 5, 128, 3), (2048, 16, 256, 3), (1500, 20, 192, 1),
                                        (1024, 1, 64, 2)])
def test_refine_apply_columns_converge(cuda_dev, n, k, b, prec, trans):
    import charmlu_b200 as lu
    A = oracle.gen_matrix(n, 11 + n)
    B = oracle.gen_uniform(n * k, 11 + n, 2).reshape(n, k)
    s = lu.LUSolver(lu.LUConfig(n, b, precision=prec))
    Ad = _padded(A)
    s.refine_factor(Ad)
    X, info = s.refine_apply(Ad, torch.from_numpy(B).cuda(), trans=bool(trans))
    assert info["status"] == 0, info
    assert info["r_hpl"] < 16.0 and info["r_hpl_initial"] >= info["r_hpl"]
    opA = A.T if trans else A
    Xh = X.cpu().numpy()
    r = _r_hpl_cols(opA, Xh, B)
    assert r.max() < 16.0, r
    ref = np.linalg.solve(opA, B)
    assert _rel(Xh, ref) < 1e-8
    assert s.status() == 0


def test_refine_apply_vector_and_repeat(cuda_dev):
    """A 1-D right-hand side; two applies on the same kept factors agree."""
    import charmlu_b200 as lu
    n = 777
    A = oracle.gen_matrix(n, 3)
    bvec = oracle.gen_vector(n, 4)
    s = lu.LUSolver(lu.LUConfig(n, 64, precision=lu.LU_PREC_FP16X3))
    Ad = _padded(A)
    s.refine_factor(Ad)
    bt = torch.from_numpy(bvec).cuda()
    x1, i1 = s.refine_apply(Ad, bt)
    x2, i2 = s.refine_apply(Ad, bt)
    assert i1["status"] == 0 and i2["status"] == 0
    assert torch.equal(x1, x2)
    assert _rel(x1.cpu().numpy(), np.linalg.solve(A, bvec)) < 1e-9


def test_refine_apply_argument_errors(cuda_dev):
    import charmlu_b200 as lu
    n = 256
    A = _padded(oracle.gen_matrix(n, 1))
    B = torch.zeros(n, 2, dtype=torch.float64, device="cuda")
    s = lu.LUSolver(lu.LUConfig(n, 64, precision=lu.LU_PREC_FP16X3))
    with pytest.raises(lu.LUError) as e:  # no kept factors yet
        s.refine_apply(A, B)
    assert e.value.code == lu.LU_ERR_ARG
    s64 = lu.LUSolver(lu.LUConfig(n, 64))
    with pytest.raises(lu.LUError) as e:
        s64.refine_factor(A)
    assert e.value.code == lu.LU_ERR_UNSUPPORTED


@pytest.mark.parametrize("n,k,b", [(1024, 16, 128), (2048, 16, 256), (4096, 16, 256)])
def test_refine_adjoint_matches_fp64_gradient(cuda_dev, n, k, b):
    import charmlu_b200 as lu
    A = oracle.gen_matrix(n, 42)
    B = oracle.gen_uniform(n * k, 42, 2).reshape(n, k)
    W = 2.0 * oracle.gen_uniform(n * k, 42, 3).reshape(n, k)
    X_ref = _accurate_solve(A, B)
    lam = _accurate_solve(A, W, trans=True)
    gA_ref, gB_ref = -lam @ X_ref.T, lam
    s = lu.LUSolver(lu.LUConfig(n, b, precision=lu.LU_PREC_FP16X3, ir_target=1e-3))
    Ad = _padded(A)
    s.refine_factor(Ad)
    X, info = s.refine_apply(Ad, torch.from_numpy(B).cuda())
    assert info["status"] == 0 and info["r_hpl"] < 1e-3
    assert _rel(X.cpu().numpy(), X_ref) < 1e-10
    gA, gB, ai = s.refine_adjoint(Ad, X, torch.from_numpy(W).cuda())
    assert ai["status"] == 0 and ai["r_hpl"] < 1e-3
    assert _rel(gB.cpu().numpy(), gB_ref) < 1e-10
    assert _rel(gA.cpu().numpy(), gA_ref) < 1e-10


def test_mixed_autograd_storing_and_refactor_agree(cuda_dev):
    from charmlu_b200.autograd import lu_solve_mixed
    n, k = 1000, 4
    A0 = torch.from_numpy(oracle.gen_matrix(n, 8)).cuda()
    B0 = torch.from_numpy(oracle.gen_uniform(n * k, 8, 2).reshape(n, k)).cuda()
    W = torch.from_numpy(2.0 * oracle.gen_uniform(n * k, 8, 3).reshape(n, k)).cuda()
    grads = []
    for refactor in (False, True):
        A = A0.clone().requires_grad_(True)
        B = B0.clone().requires_grad_(True)
        X = lu_solve_mixed(A, B, block_size=128, refactor=refactor)
        (X * W).sum().backward()
        grads.append((A.grad.clone(), B.grad.clone()))
    assert torch.equal(grads[0][0], grads[1][0]) and torch.equal(grads[0][1], grads[1][1])
    An = A0.cpu().numpy()
    lam = _accurate_solve(An, W.cpu().numpy(), trans=True)
    Xr = _accurate_solve(An, B0.cpu().numpy())
    assert _rel(grads[0][1].cpu().numpy(), lam) < 1e-10
    assert _rel(grads[0][0].cpu().numpy(), -lam @ Xr.T) < 1e-10


def test_mixed_autograd_finite_differences(cuda_dev):
    """Central differences (h = 1e-6) of loss = sum(W * X) at n = 256."""
    from charmlu_b200.autograd import lu_solve_mixed
    n, k = 256, 3
    A0 = torch.from_numpy(oracle.gen_matrix(n, 21)).cuda()
    B0 = torch.from_numpy(oracle.gen_uniform(n * k, 21, 2).reshape(n, k)).cuda()
    W = torch.from_numpy(2.0 * oracle.gen_uniform(n * k, 21, 3).reshape(n, k)).cuda()
    A = A0.clone().requires_grad_(True)
    X = lu_solve_mixed(A, B0, block_size=64, ir_target=0.5)
    (X * W).sum().backward()

    def loss(Am):
        return float((lu_solve_mixed(Am, B0, block_size=64, ir_target=0.5) * W).sum())

    h = 1e-6
    rng = np.random.default_rng(0)
    gmax = float(A.grad.abs().max())
    for _ in range(6):
        i, j = (int(v) for v in rng.integers(0, n, 2))
        Ap, Am = A0.clone(), A0.clone()
        Ap[i, j] += h
        Am[i, j] -= h
        fd = (loss(Ap) - loss(Am)) / (2 * h)
        g = float(A.grad[i, j])
        assert abs(fd - g) <= 1e-6 * max(1.0, gmax), (i, j, fd, g)

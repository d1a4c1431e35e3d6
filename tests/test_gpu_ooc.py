"""The out-of-core FP64 LU (charmlu_b200/ooc.py) on the GPU: the matrix in
pinned host memory, column panels streamed through the device. The host
factors satisfy P A = L U to rounding, the streamed solve meets the HPL
residual bar and agrees with lu_factor's solution, and where the pivot
sequences agree (they do unless two candidates tie to rounding; the
left-looking order accumulates updates differently) the factors agree with
lu_factor's to rounding."""
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,w", [(3000, 512), (2048, 256), (1000, 1000)])
def test_out_of_core_factor_and_solve(cuda_dev, n, w):
    import charmlu_b200 as lu
    from charmlu_b200.ooc import OutOfCoreLU
    A = lu.generate_uniform(n, n, seed=23, stream_id=0)
    rhs = lu.generate_uniform(n, 1, seed=23, stream_id=1).view(-1)
    host = torch.empty(n, n, dtype=torch.float64, pin_memory=True)
    host.copy_(A)
    ooc = OutOfCoreLU(n, panel=w)
    ipiv = ooc.factor(host)
    assert ooc.status_code == 0
    x = ooc.solve(host, ipiv, rhs)
    s = lu.LUSolver(lu.LUConfig(n, 256))
    assert s.residual(A, x, rhs)["r_hpl"] < 16
    # P A = L U from the host factors, formed in FP64 on the device
    LU = host.to("cuda")
    L = torch.tril(LU, -1) + torch.eye(n, dtype=torch.float64, device="cuda")
    U = torch.triu(LU)
    PA = A.clone()
    for i, p in enumerate(ipiv.tolist()):
        if p != i:
            PA[[i, p]] = PA[[p, i]]
    assert (L @ U - PA).abs().max().item() <= 1e-12 * n * A.abs().max().item()
    ref = A.clone()
    ipiv_ref = s.factor(ref)
    assert s.status() == 0
    if torch.equal(ipiv, ipiv_ref):  # the same pivot sequence: the same factors to rounding
        assert (LU - ref).abs().max().item() <= 1e-12 * n * ref.abs().max().item()
    # two backward-stable solutions differ by about kappa * sqrt(n) * eps
    xr = rhs.clone()
    s.solve(ref, ipiv_ref, xr)
    assert (x - xr).abs().max().item() <= 1e-8 * xr.abs().max().item()


def test_out_of_core_singular_column(cuda_dev):
    import charmlu_b200 as lu
    from charmlu_b200.ooc import OutOfCoreLU
    n = 768
    A = lu.generate_uniform(n, n, seed=4, stream_id=0)
    A[:, 400] = 0.0
    host = torch.empty(n, n, dtype=torch.float64, pin_memory=True)
    host.copy_(A)
    ooc = OutOfCoreLU(n, panel=256)
    ooc.factor(host)
    assert ooc.status_code == 401

"""GPU tests of the mixed-precision path (no reference counterpart: charmlu is
FP64 only).  The BF16 tensor-core kernel is checked against a plain FP64
torch product of the same BF16-rounded operands; the refined solutions
against the oracle's FP64 solution (forward error) and the scaled residual
contract r_hpl < 16."""
import ctypes

import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu


def _lib():
    from charmlu_b200 import _lib as L
    lib = L.load()
    f = lib.lub_test_gemm_lowp
    f.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                  ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def _pow2_scale(t):
    m = t.abs().max().item()
    e = np.frexp(m)[1]  # m = f * 2^e, f in [0.5, 1)
    return 2.0 ** (13 - (e - 1))


def _lowp_reference(A, B, C, mode):
    """C - product, the product formed exactly (FP64) from the operands the
    kernel sees: BF16-rounded (mode 0), FP16 of the power-of-two scaled
    panel (mode 1), or the hi/lo FP16 split with three products (mode 2;
    mode 3, the pairs layout, computes the same three products)."""
    mode = 2 if mode == 3 else mode
    if mode == 0:
        return C.double() - A.bfloat16().double() @ B.bfloat16().double()
    sa, sb = _pow2_scale(A), _pow2_scale(B)
    As, Bs = A * sa, B * sb
    Ah, Bh = As.half(), Bs.half()
    if mode == 1:
        P = Ah.double() @ Bh.double()
    else:
        Al = (As - Ah.float()).half()
        Bl = (Bs - Bh.float()).half()
        P = Ah.double() @ Bh.double() + Ah.double() @ Bl.double() + Al.double() @ Bh.double()
    return C.double() - P / (sa * sb)


@pytest.mark.parametrize("mode", [0, 1, 2, 3])
@pytest.mark.parametrize("M,N,K", [(128, 256, 64), (300, 520, 256), (1024, 1024, 512), (257, 999, 1024),
                                   (4096, 4096, 256), (1000, 700, 200)])
def test_gemm_lowp_tcgen05_matches_reference(cuda_dev, M, N, K, mode):
    f = _lib()
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N)
    A = torch.rand(M, K, device="cuda", generator=g, dtype=torch.float32) - 0.5
    B = (torch.rand(K, N, device="cuda", generator=g, dtype=torch.float32) - 0.5) * 37.0
    ldc = (N + 3) // 4 * 4
    Cbuf = torch.rand(M, ldc, device="cuda", generator=g, dtype=torch.float32) - 0.5
    C = Cbuf[:, :N]
    pad_before = Cbuf[:, N:].clone()
    ref = _lowp_reference(A, B, C, mode)
    # mode 3 (pairs layout) runs on the persistent kernel (148 CTAs)
    rc = f(A.data_ptr(), K, B.data_ptr(), N, Cbuf.data_ptr(), ldc, M, N, K, mode | ((148 << 8) if mode == 3 else 0),
           torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert rc == 0
    err = (C.double() - ref).abs().max().item()
    # FP32 accumulation of K (3K for the split) products |a b| <= 0.5 * 18.5:
    # a statistical bound 4 u32 K max|a b| (the worst-case bound is K^2 u32 max|ab|)
    kk = K * (3 if mode >= 2 else 1)
    assert err <= 4 * 6e-8 * kk * 0.5 * 18.5 + 1e-6, err
    assert torch.equal(Cbuf[:, N:], pad_before)
    if mode >= 2:
        # the three-product split reproduces the exact FP32 product to ~u_fp16^2
        split = -_lowp_reference(A, B, torch.zeros_like(C), 2)
        assert (split - A.double() @ B.double()).abs().max().item() <= 1e-5 * 18.5 * K / 64


@pytest.mark.parametrize("mode", [0, 2])
@pytest.mark.parametrize("pctas", [1, 3, 116, 148])
@pytest.mark.parametrize("M,N,K", [(300, 520, 256), (1100, 2100, 192), (4096, 4096, 256)])
def test_gemm_lowp_persistent_matches_tile_kernel(cuda_dev, M, N, K, mode, pctas):
    """The persistent kernel (CTAs walking tiles, two TMEM accumulators)
    issues the same MMAs per tile as the one-tile-per-CTA kernel: the
    results agree bit for bit."""
    f = _lib()
    g = torch.Generator(device="cuda").manual_seed(M + 3 * N + pctas)
    A = torch.rand(M, K, device="cuda", generator=g, dtype=torch.float32) - 0.5
    B = (torch.rand(K, N, device="cuda", generator=g, dtype=torch.float32) - 0.5) * 5.0
    ldc = (N + 3) // 4 * 4
    C0 = torch.rand(M, ldc, device="cuda", generator=g, dtype=torch.float32) - 0.5
    C1 = C0.clone()
    st = torch.cuda.current_stream().cuda_stream
    assert f(A.data_ptr(), K, B.data_ptr(), N, C0.data_ptr(), ldc, M, N, K, mode, st) == 0
    assert f(A.data_ptr(), K, B.data_ptr(), N, C1.data_ptr(), ldc, M, N, K, mode | (pctas << 8), st) == 0
    torch.cuda.synchronize()
    assert torch.equal(C0, C1)


PAIR_BIT = 1 << 24


@pytest.mark.parametrize("pctas", [1, 2, 7, 100, 148])
@pytest.mark.parametrize("M,N,K", [(128, 256, 64), (300, 520, 256), (129, 999, 128), (1000, 700, 192),
                                   (4096, 4096, 256), (2560, 512, 512)])
def test_gemm_lowp_cta_pair_kernel(cuda_dev, M, N, K, pctas):
    """The CTA-pair kernel (tcgen05 cta_group::2, 256 x 256 tiles over two
    SMs) computes the pairs layout's three products: within the FP32
    accumulation bound of the exact product of the split operands, the
    padding columns untouched, and equal to the one-SM pairs kernel."""
    f = _lib()
    g = torch.Generator(device="cuda").manual_seed(M * 11 + N + pctas)
    A = torch.rand(M, K, device="cuda", generator=g, dtype=torch.float32) - 0.5
    B = (torch.rand(K, N, device="cuda", generator=g, dtype=torch.float32) - 0.5) * 37.0
    ldc = (N + 3) // 4 * 4 + 4
    C0 = torch.rand(M, ldc, device="cuda", generator=g, dtype=torch.float32) - 0.5
    C1 = C0.clone()
    pad_before = C0[:, N:].clone()
    ref = _lowp_reference(A, B, C0[:, :N], 3)
    st = torch.cuda.current_stream().cuda_stream
    assert f(A.data_ptr(), K, B.data_ptr(), N, C0.data_ptr(), ldc, M, N, K, 3 | (pctas << 8) | PAIR_BIT, st) == 0
    assert f(A.data_ptr(), K, B.data_ptr(), N, C1.data_ptr(), ldc, M, N, K, 3 | (148 << 8), st) == 0
    torch.cuda.synchronize()
    err = (C0[:, :N].double() - ref).abs().max().item()
    assert err <= 4 * 6e-8 * 3 * K * 0.5 * 18.5 + 1e-6, err
    assert torch.equal(C0[:, N:], pad_before)
    assert torch.equal(C0, C1)


@pytest.mark.parametrize("pctas,hctas", [(100, 48), (2, 2), (3, 5), (116, 32)])
@pytest.mark.parametrize("M,N,K", [(300, 520, 256), (1100, 2100, 192), (4096, 4096, 256)])
def test_gemm_lowp_cta_pair_shared_tile_counter(cuda_dev, M, N, K, pctas, hctas):
    """Two CTA-pair launches on two streams sharing one tile counter (the
    even CTA of each pair draws the tile and hands it to the odd one) give
    the same C as one launch."""
    f = _lib()
    g = torch.Generator(device="cuda").manual_seed(M + 9 * N + pctas + hctas)
    A = torch.rand(M, K, device="cuda", generator=g, dtype=torch.float32) - 0.5
    B = (torch.rand(K, N, device="cuda", generator=g, dtype=torch.float32) - 0.5) * 5.0
    ldc = (N + 3) // 4 * 4
    C0 = torch.rand(M, ldc, device="cuda", generator=g, dtype=torch.float32) - 0.5
    C1 = C0.clone()
    st = torch.cuda.current_stream().cuda_stream
    assert f(A.data_ptr(), K, B.data_ptr(), N, C0.data_ptr(), ldc, M, N, K, 3 | (148 << 8) | PAIR_BIT, st) == 0
    assert f(A.data_ptr(), K, B.data_ptr(), N, C1.data_ptr(), ldc, M, N, K,
             3 | (pctas << 8) | (hctas << 16) | PAIR_BIT, st) == 0
    torch.cuda.synchronize()
    assert torch.equal(C0, C1)


@pytest.mark.parametrize("mode", [0, 2, 3])
@pytest.mark.parametrize("pctas,hctas", [(100, 48), (1, 1), (3, 5), (116, 32)])
@pytest.mark.parametrize("M,N,K", [(300, 520, 256), (1100, 2100, 192), (4096, 4096, 256)])
def test_gemm_lowp_shared_tile_counter(cuda_dev, M, N, K, mode, pctas, hctas):
    """Two persistent launches on two streams that take tiles from one
    counter (the look-ahead update and its helper) give the same C bit for
    bit as one launch: each tile is computed once, by whichever CTA takes it."""
    f = _lib()
    g = torch.Generator(device="cuda").manual_seed(M + 5 * N + pctas + hctas)
    A = torch.rand(M, K, device="cuda", generator=g, dtype=torch.float32) - 0.5
    B = (torch.rand(K, N, device="cuda", generator=g, dtype=torch.float32) - 0.5) * 5.0
    ldc = (N + 3) // 4 * 4
    C0 = torch.rand(M, ldc, device="cuda", generator=g, dtype=torch.float32) - 0.5
    C1 = C0.clone()
    st = torch.cuda.current_stream().cuda_stream
    single = mode | ((148 << 8) if mode == 3 else 0)
    assert f(A.data_ptr(), K, B.data_ptr(), N, C0.data_ptr(), ldc, M, N, K, single, st) == 0
    assert f(A.data_ptr(), K, B.data_ptr(), N, C1.data_ptr(), ldc, M, N, K, mode | (pctas << 8) | (hctas << 16),
             st) == 0
    torch.cuda.synchronize()
    assert torch.equal(C0, C1)


def _refine(n, b, A_np=None, seed=42, mode=None, target=16.0, prec=None, lookahead=False):
    import charmlu_b200 as lu
    prec = lu.LU_PREC_FP16X3 if prec is None else prec
    if A_np is None:
        A = lu.generate_uniform(n, n, seed=seed, stream_id=0)
    else:
        A = torch.from_numpy(A_np).cuda()
    rhs = lu.generate_uniform(n, 1, seed=seed, stream_id=1).view(-1)
    cfg = lu.LUConfig(n, b, precision=prec, ir_target=target, lookahead=lookahead)
    if mode is not None:
        cfg.ir_mode = mode
    s = lu.LUSolver(cfg)
    x, info = s.refine_solve(A, rhs)
    st = s.status()
    return s, A, rhs, x, info, st


@pytest.mark.parametrize("prec,n,b", [(1, 512, 256), (2, 512, 256), (2, 1024, 256), (3, 1024, 256), (3, 2048, 512),
                                      (3, 3000, 256), (3, 4096, 512)])
def test_refine_solve_reaches_residual_target(cuda_dev, prec, n, b):
    s, A, rhs, x, info, st = _refine(n, b, prec=prec)
    assert st == 0 and info["status"] == 0, info
    r = s.residual(A, x, rhs)
    assert r["r_hpl"] < 16, r
    # forward error against the FP64 oracle solution
    x_ref, *_ = oracle.solve(A.cpu().numpy(), rhs.cpu().numpy(), b=128)
    fe = np.abs(x.cpu().numpy() - x_ref).max() / np.abs(x_ref).max()
    assert fe < 1e-6, fe
    # the low-precision solve alone is far from the target; refinement did the work
    assert info["r_hpl_initial"] > info["r_hpl"]


def test_refine_tight_target_matches_fp64(cuda_dev):
    """Refined to r_hpl < 0.01 the mixed solution agrees with the FP64 one."""
    n, b = 2048, 256
    s, A, rhs, x, info, st = _refine(n, b, target=0.01)
    assert st == 0 and info["status"] == 0, info
    x_ref, *_ = oracle.solve(A.cpu().numpy(), rhs.cpu().numpy(), b=128)
    fe = np.abs(x.cpu().numpy() - x_ref).max() / np.abs(x_ref).max()
    assert fe < 1e-10, fe


def test_gmres_ir_mode(cuda_dev):
    import charmlu_b200 as lu
    n, b = 1024, 256
    s, A, rhs, x, info, st = _refine(n, b, mode=lu.LU_IR_GMRES)
    assert st == 0 and info["status"] == 0 and info["used_gmres"] == 1, info
    assert s.residual(A, x, rhs)["r_hpl"] < 16


def test_singular_matrix_reports_info_mixed(cuda_dev):
    import charmlu_b200 as lu
    n, b = 256, 64
    A = oracle.gen_matrix(n, 3)
    A[:, 100] = 0.0
    s, Ad, rhs, x, info, st = _refine(n, b, A_np=A)
    assert st == 101, (st, info)


@pytest.mark.parametrize("n,b", [(2048, 256), (4096, 512), (1500, 192), (1000, 64), (2000, 320)])
def test_refine_lookahead(cuda_dev, n, b):
    """Block sizes that are not a multiple of the 256-column update tile make
    the next-panel update's last tile reach into columns the rest update
    owns; those must receive a zero increment from it."""
    s, A, rhs, x, info, st = _refine(n, b, lookahead=True)
    assert st == 0 and info["status"] == 0, info
    assert info["used_gmres"] == 0 and info["iterations"] <= 4, info
    assert s.residual(A, x, rhs)["r_hpl"] < 16


@pytest.mark.parametrize("kappa", [1e2, 1e6])
def test_kappa_matrices_refine_or_report(cuda_dev, kappa):
    """Q1 diag(sigma) Q2^T test matrices: a refined result either meets the
    residual contract (checked independently here) or is reported as not
    converged; never a silent wrong answer."""
    import sys, os
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from bench import kappa_matrix
    import charmlu_b200 as lu
    n = 1024
    A = kappa_matrix(n, kappa, 99, torch.device("cuda"))
    b = lu.generate_uniform(n, 1, seed=42, stream_id=1).view(-1)
    x_ref = np.linalg.solve(A.cpu().numpy(), b.cpu().numpy())
    for prec in (lu.LU_PREC_FP16S, lu.LU_PREC_FP16X3):
        s = lu.LUSolver(lu.LUConfig(n, 256, precision=prec, ir_max_iter=30))
        x, info = s.refine_solve(A, b)
        st = s.status()
        r = s.residual(A, x, b)
        if st == 0:
            assert r["r_hpl"] < 16, (prec, r)
            fe = np.abs(x.cpu().numpy() - x_ref).max() / np.abs(x_ref).max()
            # backward error ~ r_hpl * n * eps, forward error <~ kappa * that
            assert fe < 4 * kappa * max(r["r_hpl"], 1.0) * n * 2.2e-16, (prec, fe)
        else:
            assert st == lu.LU_ERR_NOCONV
    # the error-compensated factors converge classically at kappa = 1e2
    if kappa == 1e2:
        s = lu.LUSolver(lu.LUConfig(n, 256, precision=lu.LU_PREC_FP16X3))
        x, info = s.refine_solve(A, b)
        assert s.status() == 0 and info["used_gmres"] == 0


@pytest.mark.parametrize("n,b", [(4096, 512), (3000, 192)])
def test_refine_update_helper_bitwise(cuda_dev, n, b, monkeypatch):
    """Under look-ahead the reserved SMs join the trailing update once the
    panel is done (a helper launch sharing the update's tile counter). The
    factors, and so x, are the same bit for bit as without the helper."""
    import charmlu_b200 as lu
    A = lu.generate_uniform(n, n, seed=5, stream_id=0)
    rhs = lu.generate_uniform(n, 1, seed=5, stream_id=1).view(-1)
    xs = []
    for helper in ("1", "0"):
        monkeypatch.setenv("LU_B200_GEMM_HELPER", helper)
        s = lu.LUSolver(lu.LUConfig(n, b, precision=lu.LU_PREC_FP16X3, lookahead=True))
        x, info = s.refine_solve(A, rhs)
        assert s.status() == 0 and info["status"] == 0, info
        xs.append(x)
    assert torch.equal(xs[0], xs[1])


@pytest.mark.parametrize("n,b,la,split", [(4096, 512, True, "0"), (3000, 192, True, "0"), (2048, 512, False, "0"),
                                         (4096, 512, True, "1")])
def test_refine_cta_pair_update_bitwise(cuda_dev, n, b, la, split, monkeypatch):
    """LU_B200_GEMM_PAIR=1 runs the trailing updates (and their helper
    launches) on CTA pairs; each C element receives the same FP32 increment,
    so the factors and x are the same bit for bit as with one-SM tiles, also
    under graph replay."""
    import charmlu_b200 as lu
    monkeypatch.setenv("LU_B200_LA_SPLIT", split)
    A = lu.generate_uniform(n, n, seed=21, stream_id=0)
    rhs = lu.generate_uniform(n, 1, seed=21, stream_id=1).view(-1)
    xs = []
    for pair in ("0", "1"):
        monkeypatch.setenv("LU_B200_GEMM_PAIR", pair)
        s = lu.LUSolver(lu.LUConfig(n, b, precision=lu.LU_PREC_FP16X3, lookahead=la))
        x, info = s.refine_solve(A, rhs)
        assert s.status() == 0 and info["status"] == 0, info
        assert s.residual(A, x, rhs)["r_hpl"] < 16
        xs.append(x)
    assert torch.equal(xs[0], xs[1])
    sg = lu.LUSolver(lu.LUConfig(n, b, precision=lu.LU_PREC_FP16X3, lookahead=la, use_graph=True))
    xg = torch.empty_like(rhs)
    for _ in range(2):
        sg.refine_solve(A, rhs, xg)
        assert sg.status() == 0 and torch.equal(xg, xs[1])


@pytest.mark.parametrize("n,b,la", [(4096, 512, True), (3000, 256, True), (2048, 512, False), (1500, 192, True)])
def test_refine_panel_gemm_tensor_cores(cuda_dev, n, b, la, monkeypatch):
    """LU_B200_PANEL_TC=1 moves the recursive panel's GEMM halves (width >=
    128) onto the tcgen05 kernel with split FP16 operands. Refinement reaches
    the target as quickly, and x agrees with the FP32-SIMT panel's x to the
    accuracy the HPL bar leaves (forward error ~ kappa * n * eps * 16)."""
    import charmlu_b200 as lu
    A = lu.generate_uniform(n, n, seed=9, stream_id=0)
    rhs = lu.generate_uniform(n, 1, seed=9, stream_id=1).view(-1)
    out = []
    for tc in ("0", "1"):
        monkeypatch.setenv("LU_B200_PANEL_TC", tc)
        s = lu.LUSolver(lu.LUConfig(n, b, precision=lu.LU_PREC_FP16X3, lookahead=la))
        x, info = s.refine_solve(A, rhs)
        assert s.status() == 0 and info["status"] == 0, info
        assert info["used_gmres"] == 0 and info["iterations"] <= 4, info
        assert s.residual(A, x, rhs)["r_hpl"] < 16
        out.append(x)
    x_ref, *_ = oracle.solve(A.cpu().numpy(), rhs.cpu().numpy(), b=128)
    for x in out:
        fe = np.abs(x.cpu().numpy() - x_ref).max() / np.abs(x_ref).max()
        assert fe < 1e-6, fe


@pytest.mark.parametrize("n,b", [(4096, 512), (3000, 256), (1500, 192), (2048, 512), (1024, 256)])
def test_refine_lookahead_split_schedule(cuda_dev, n, b, monkeypatch):
    """LU_B200_LA_SPLIT=1: each look-ahead step does the next panel's
    columns first (interchanges, U solve, operands, update) and the other
    columns after the panel has started, the rest's U rows with their own
    scale. Refinement reaches the target as quickly as with the one-pass
    schedule, x matches the FP64 oracle's to the HBM bar's accuracy, and the
    captured schedule replays to the same x bit for bit."""
    import charmlu_b200 as lu
    monkeypatch.setenv("LU_B200_LA_SPLIT", "1")
    A = lu.generate_uniform(n, n, seed=13, stream_id=0)
    rhs = lu.generate_uniform(n, 1, seed=13, stream_id=1).view(-1)
    s = lu.LUSolver(lu.LUConfig(n, b, precision=lu.LU_PREC_FP16X3, lookahead=True))
    x, info = s.refine_solve(A, rhs)
    assert s.status() == 0 and info["status"] == 0, info
    assert info["used_gmres"] == 0 and info["iterations"] <= 4, info
    assert s.residual(A, x, rhs)["r_hpl"] < 16
    x_ref, *_ = oracle.solve(A.cpu().numpy(), rhs.cpu().numpy(), b=128)
    fe = np.abs(x.cpu().numpy() - x_ref).max() / np.abs(x_ref).max()
    assert fe < 1e-6, fe
    sg = lu.LUSolver(lu.LUConfig(n, b, precision=lu.LU_PREC_FP16X3, lookahead=True, use_graph=True))
    xg = torch.empty_like(rhs)
    for _ in range(2):
        sg.refine_solve(A, rhs, xg)
        assert sg.status() == 0 and torch.equal(xg, x)


def test_refine_graph_replay(cuda_dev):
    import charmlu_b200 as lu
    n, b = 2048, 256
    A = lu.generate_uniform(n, n, seed=42, stream_id=0)
    rhs = lu.generate_uniform(n, 1, seed=42, stream_id=1).view(-1)
    s0 = lu.LUSolver(lu.LUConfig(n, b, precision=lu.LU_PREC_FP16X3, lookahead=True))
    x0, _ = s0.refine_solve(A, rhs)
    sg = lu.LUSolver(lu.LUConfig(n, b, precision=lu.LU_PREC_FP16X3, lookahead=True, use_graph=True))
    x = torch.empty_like(rhs)
    for _ in range(3):
        _, info = sg.refine_solve(A, rhs, x)
        assert sg.status() == 0 and info["status"] == 0
        assert torch.equal(x, x0)


@pytest.mark.parametrize("n,b,stage,resident", [(1500, 192, 1 << 20, 0), (2048, 256, 3 << 20, 11 << 20),
                                                (3000, 256, 5 << 20, 1 << 20), (8192, 512, 0, None)])
def test_refine_solve_host_matches_device(cuda_dev, n, b, stage, resident, monkeypatch):
    """The mixed path with the FP64 matrix in host memory gives the
    device-resident path's x bit for bit. Leading rows up to `resident`
    bytes stay on the device (0: none, every pass streams all rows; None:
    all that fit); the others stream in row chunks (small chunks force many
    double-buffered copies; 0 keeps the 256 MB default)."""
    import charmlu_b200 as lu
    if stage:
        monkeypatch.setenv("LU_B200_STAGE_BYTES", str(stage))
    if resident is not None:
        monkeypatch.setenv("LU_B200_RESIDENT_BYTES", str(resident))
    A = lu.generate_uniform(n, n, seed=77, stream_id=0)
    bvec = lu.generate_uniform(n, 1, seed=77, stream_id=1).view(-1)
    s = lu.LUSolver(lu.LUConfig(n, b, precision=lu.LU_PREC_FP16X3, lookahead=True))
    x_dev, i_dev = s.refine_solve(A, bvec)
    hA = A.cpu().pin_memory()
    x_host, i_host = s.refine_solve_host(hA, bvec)
    torch.cuda.synchronize()
    assert i_host["status"] == 0 and i_host["r_hpl"] < 16, i_host
    assert i_host["iterations"] == i_dev["iterations"]
    assert torch.equal(x_host, x_dev)
    # one full pass (the conversion), then only the non-resident rows per residual
    lda = hA.stride(0)
    rows = n if resident is None else min(n, resident // (8 * lda))
    assert i_dev["host_bytes"] == 0 and i_host["used_gmres"] == 0
    assert i_host["host_bytes"] == 8 * lda * (n + (n - rows) * (i_host["iterations"] + 1))
    # a second call on the same handle reuses the staging and resident buffers
    x2, i2 = s.refine_solve_host(hA, bvec)
    assert torch.equal(x2, x_dev) and i2["host_bytes"] == i_host["host_bytes"]
    with pytest.raises(lu.LUError):
        s.refine_solve_host(A, bvec)  # a device tensor is rejected


@pytest.mark.parametrize("kappa", [1e6, 1e10])
@pytest.mark.parametrize("prec", [1, 2, 3])
def test_refinement_never_raises_the_residual(cuda_dev, kappa, prec):
    """Hard systems for the low-precision factors: whatever the outcome, the
    returned x has the smallest residual the refinement reached (steps that
    raise ||b - A x||inf are rolled back), its r_hpl is what info reports,
    and non-convergence is reported as LU_ERR_NOCONV."""
    import sys, os
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from bench import kappa_matrix
    import charmlu_b200 as lu
    n = 1024
    A = kappa_matrix(n, kappa, 5, torch.device("cuda"))
    b = lu.generate_uniform(n, 1, seed=43, stream_id=1).view(-1)
    s = lu.LUSolver(lu.LUConfig(n, 256, precision=prec, ir_max_iter=20, gmres_restart=60))
    x, info = s.refine_solve(A, b)
    st = s.status()
    if not np.isfinite(info["r_hpl_initial"]):
        # the low-precision factors broke down (overflow): reported, not refined
        assert st != 0 and info["status"] != 0, (st, info)
        return
    assert info["r_hpl"] <= info["r_hpl_initial"], info
    r = s.residual(A, x, b)
    assert abs(r["r_hpl"] - info["r_hpl"]) <= 1e-6 * max(1.0, info["r_hpl"]), (r, info)
    if st == 0:
        assert info["r_hpl"] < 16
    else:
        assert st == lu.LU_ERR_NOCONV and info["status"] == lu.LU_ERR_NOCONV


def test_refine_apply_never_raises_the_residual(cuda_dev):
    """The multi-RHS refinement (both op(A) = A and A^T) keeps each column's
    best iterate."""
    import sys, os
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from bench import kappa_matrix
    import charmlu_b200 as lu
    n = 1024
    A = kappa_matrix(n, 1e6, 6, torch.device("cuda"))
    B = lu.generate_uniform(n, 5, seed=44, stream_id=2)
    s = lu.LUSolver(lu.LUConfig(n, 256, precision=lu.LU_PREC_BF16, ir_max_iter=15, gmres_restart=40))
    s.refine_factor(A)
    for trans in (False, True):
        X, info = s.refine_apply(A, B, trans=trans)
        if not np.isfinite(info["r_hpl_initial"]):
            assert info["status"] != 0, info
            continue
        assert info["r_hpl"] <= info["r_hpl_initial"], info
        if info["status"] == 0:
            op = A.t() if trans else A
            R = B - op @ X
            an = op.abs().sum(dim=1).max()
            for c in range(5):
                rc = R[:, c].abs().max() / ((an * X[:, c].abs().max() + B[:, c].abs().max()) * n * 2.22e-16)
                assert rc.item() < 16


def test_precond_norm_estimate(cuda_dev):
    """||I - M^{-1} A||: well below 1 for the near-FP32 FP16x3 factors of a
    well-conditioned matrix (classical refinement contracts fast), larger
    for BF16 factors of an ill-conditioned one; cross-checked against the
    contraction the refinement shows."""
    import sys, os
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from bench import kappa_matrix
    import charmlu_b200 as lu
    n = 1024
    A = kappa_matrix(n, 1e2, 7, torch.device("cuda"))
    s = lu.LUSolver(lu.LUConfig(n, 256, precision=lu.LU_PREC_FP16X3))
    s.refine_factor(A)
    e3 = s.refine_precond_norm(A, iters=12)
    assert 0.0 < e3 < 1e-2, e3
    A6 = kappa_matrix(n, 1e6, 7, torch.device("cuda"))
    s6 = lu.LUSolver(lu.LUConfig(n, 256, precision=lu.LU_PREC_BF16))
    s6.refine_factor(A6)
    e6 = s6.refine_precond_norm(A6, iters=12)
    assert e6 > 10 * e3 and np.isfinite(e6), (e3, e6)
    with pytest.raises(lu.LUError):
        lu.LUSolver(lu.LUConfig(n, 256, precision=lu.LU_PREC_BF16)).refine_precond_norm(A, iters=4)


@pytest.mark.parametrize("M,N,K", [(32768, 32, 32), (4096, 64, 64), (1000, 48, 16), (77, 2, 4), (5000, 128, 128),
                                   (3000, 200, 96)])
def test_gemm_f32_panel_kernels_match_torch(cuda_dev, M, N, K):
    """The FP32 panel GEMM (C -= A B) against a plain FP32 torch product, and
    the narrow kernel (N, K <= 64) against the 128 x 128 tile kernel: both
    accumulate over k in order and subtract once, so they agree bit for
    bit."""
    from charmlu_b200 import _lib as L
    f = L.load().lub_test_gemm_f32
    f.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                  ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    f.restype = ctypes.c_int
    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    A = torch.rand(M, K + 3, device="cuda", generator=g)[:, :K] - 0.5  # row pitch != K
    B = torch.rand(K, N + 1, device="cuda", generator=g)[:, :N] - 0.5
    C0 = torch.rand(M, N + 5, device="cuda", generator=g) - 0.5
    out = []
    for wide_only in (0, 1):
        Cb = C0.clone()
        C = Cb[:, :N]
        st = torch.cuda.current_stream().cuda_stream
        assert f(A.data_ptr(), A.stride(0), B.data_ptr(), B.stride(0), C.data_ptr(), C.stride(0), M, N, K,
                 wide_only, st) == 0
        torch.cuda.synchronize()
        assert torch.equal(Cb[:, N:], C0[:, N:])  # nothing right of C touched
        out.append(C.clone())
    ref = C0[:, :N].double() - A.double() @ B.double()
    assert (out[0].double() - ref).abs().max().item() <= 4e-7 * K
    assert torch.equal(out[0], out[1])


def _tslu(P, ncols, max_ctas=48):
    from charmlu_b200 import _lib as L
    f = L.load().lub_test_tslu_leaf
    f.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                  ctypes.c_void_p]
    f.restype = ctypes.c_int
    ipiv = torch.zeros(ncols, dtype=torch.int32, device="cuda")
    rc = f(P.data_ptr(), P.stride(0), P.shape[0], ncols, ipiv.data_ptr(), max_ctas,
           torch.cuda.current_stream().cuda_stream)
    return rc, ipiv


@pytest.mark.parametrize("M,ncols,max_ctas", [(65536, 32, 48), (5000, 32, 48), (3001, 17, 48), (100, 8, 48),
                                              (32, 32, 48), (20000, 16, 8), (60000, 32, 148)])
def test_tslu_leaf_factors_the_permuted_panel(cuda_dev, M, ncols, max_ctas):
    """The tournament-pivoting leaf: its sequential swaps applied to the
    original panel give P A = L U (FP32, checked in FP64), every pivot lies
    in [j, M), the first pivot is the column's largest entry (lowest row on
    a tie), and the multipliers stay bounded."""
    g = torch.Generator(device="cuda").manual_seed(M + ncols)
    A = torch.rand(M, ncols + 3, device="cuda", generator=g)[:, :ncols] - 0.5
    A0 = A.double().cpu().numpy()
    P = A.clone()
    Pv = P[:, :ncols]
    rc, ipiv = _tslu(Pv, ncols, max_ctas)
    assert rc == 0, rc
    ip = ipiv.cpu().numpy()
    assert all(j <= ip[j] < M for j in range(ncols)), ip
    col = np.abs(A0[:, 0])
    assert ip[0] == int(np.flatnonzero(col == col.max())[0])
    PA = A0.copy()
    for j, p in enumerate(ip):
        PA[[j, p]] = PA[[p, j]]
    LU = Pv.double().cpu().numpy()
    Lm = np.tril(LU, -1)[:, :ncols]
    Lm[:ncols, :ncols] += np.eye(ncols)
    U = np.triu(LU[:ncols])
    err = np.abs(PA - Lm @ U).max() / np.abs(A0).max()
    assert err < 2e-6 * ncols, err
    assert np.abs(Lm).max() < 50.0


def test_tslu_leaf_declines_panels_beyond_its_blocks(cuda_dev):
    """A panel taller than the row blocks and the stack can hold is left
    untouched and declined (LU_ERR_UNSUPPORTED): the caller then runs the
    partial-pivoting leaf."""
    M, ncols = 80000, 32
    A = torch.rand(M, ncols, device="cuda") - 0.5
    A0 = A.clone()
    rc, _ = _tslu(A, ncols)
    assert rc == -8 and torch.equal(A, A0)


def test_tslu_leaf_reports_a_zero_column(cuda_dev):
    M, ncols = 4096, 32
    g = torch.Generator(device="cuda").manual_seed(5)
    A = torch.rand(M, ncols, device="cuda", generator=g) - 0.5
    A[:, 9] = 0.0
    rc, ipiv = _tslu(A, ncols)
    assert rc == 10, rc


@pytest.mark.parametrize("n,b,la", [(4096, 512, True), (3000, 256, True), (2048, 256, False)])
def test_refine_solve_with_tournament_leaf(cuda_dev, n, b, la, monkeypatch):
    """LU_B200_TSLU=1: the mixed factorisation with the tournament-pivoting
    leaf meets the residual contract and the forward-error bar."""
    monkeypatch.setenv("LU_B200_TSLU", "1")
    s, A, rhs, x, info, st = _refine(n, b, prec=3, lookahead=la)
    assert st == 0 and info["status"] == 0, info
    assert s.residual(A, x, rhs)["r_hpl"] < 16
    x_ref, *_ = oracle.solve(A.cpu().numpy(), rhs.cpu().numpy(), b=128)
    assert np.abs(x.cpu().numpy() - x_ref).max() / np.abs(x_ref).max() < 1e-6


@pytest.mark.parametrize("w,ncols", [(256, 256), (256, 512), (160, 96), (33, 5), (64, 64), (200, 37)])
def test_trsm_block_matches_torch(cuda_dev, w, ncols):
    """The one-launch blocked FP32 TRSM of the mixed path's panels (B <-
    L^{-1} B, L unit lower) against a plain FP32 torch triangular solve."""
    from charmlu_b200 import _lib as L
    f = L.load().lub_test_trsm_block
    f.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_int,
                  ctypes.c_void_p]
    f.restype = ctypes.c_int
    g = torch.Generator(device="cuda").manual_seed(w + ncols)
    Lm = (torch.rand(w, w + 2, device="cuda", generator=g) - 0.5)[:, :w] * 0.2
    B = torch.rand(w, ncols + 3, device="cuda", generator=g) - 0.5
    B0 = B.clone()
    Bv = B[:, :ncols]
    assert f(Lm.data_ptr(), Lm.stride(0), Bv.data_ptr(), B.stride(0), w, ncols,
             torch.cuda.current_stream().cuda_stream) == 0
    torch.cuda.synchronize()
    Lu = torch.tril(Lm, -1) + torch.eye(w, device="cuda")
    ref = torch.linalg.solve_triangular(Lu, B0[:, :ncols], upper=False, unitriangular=True)
    assert torch.equal(B[:, ncols:], B0[:, ncols:])
    assert (Bv - ref).abs().max().item() <= 1e-5 * max(1.0, ref.abs().max().item())


@pytest.mark.parametrize("w,ncols,aligned", [(512, 4096, True), (512, 600, True), (500, 1000, True),
                                             (256, 2048, True), (33, 513, True), (96, 40, True),
                                             (512, 777, False), (100, 1030, False), (1, 64, True)])
def test_trsm_wide_matches_torch(cuda_dev, w, ncols, aligned):
    """The wide U block-row solve (B <- L^{-1} B, L unit lower, w <= 512:
    32 x 32 diagonal blocks inverted, then block products over a 32-column
    slice per CTA) against a plain FP64 torch triangular solve, with the
    16-byte and the element copy paths and ragged widths."""
    from charmlu_b200 import _lib as L
    f = L.load().lub_test_trsm_wide
    f.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_int,
                  ctypes.c_void_p]
    f.restype = ctypes.c_int
    g = torch.Generator(device="cuda").manual_seed(w * 3 + ncols)
    ldl = w + (4 if aligned else 3)
    Lfull = (torch.rand(w, ldl, device="cuda", generator=g) - 0.5) * 0.2
    Lm = Lfull[:, :w]
    assert Lm.stride(0) == ldl
    ldb = ncols + (8 if aligned else 5)
    B = torch.rand(w, ldb, device="cuda", generator=g) - 0.5
    B0 = B.clone()
    Bv = B[:, :ncols]
    assert f(Lm.data_ptr(), ldl, Bv.data_ptr(), ldb, w, ncols, torch.cuda.current_stream().cuda_stream) == 0
    torch.cuda.synchronize()
    Lu = (torch.tril(Lm, -1) + torch.eye(w, device="cuda")).double()
    ref = torch.linalg.solve_triangular(Lu, B0[:, :ncols].double(), upper=False, unitriangular=True)
    assert torch.equal(B[:, ncols:], B0[:, ncols:])
    err = (Bv.double() - ref).abs().max().item()
    assert err <= 2e-5 * max(1.0, ref.abs().max().item()), err


@pytest.mark.parametrize("n,b,la", [(4096, 512, True), (3000, 256, True), (2048, 512, False), (5000, 384, True)])
def test_refine_wide_u_solve(cuda_dev, n, b, la, monkeypatch):
    """LU_B200_TRSM_WIDE (default on) solves each step's U block row in one
    launch; with it and without it the refinement reaches r_hpl < 16 in as
    few steps, and both solutions match the FP64 oracle's to the HPL bar's
    accuracy."""
    import charmlu_b200 as lu
    A = lu.generate_uniform(n, n, seed=17, stream_id=0)
    rhs = lu.generate_uniform(n, 1, seed=17, stream_id=1).view(-1)
    x_ref, *_ = oracle.solve(A.cpu().numpy(), rhs.cpu().numpy(), b=128)
    for wide in ("1", "0"):
        monkeypatch.setenv("LU_B200_TRSM_WIDE", wide)
        s = lu.LUSolver(lu.LUConfig(n, b, precision=lu.LU_PREC_FP16X3, lookahead=la))
        x, info = s.refine_solve(A, rhs)
        assert s.status() == 0 and info["status"] == 0, info
        assert info["used_gmres"] == 0 and info["iterations"] <= 4, info
        assert s.residual(A, x, rhs)["r_hpl"] < 16
        fe = np.abs(x.cpu().numpy() - x_ref).max() / np.abs(x_ref).max()
        assert fe < 1e-6, fe

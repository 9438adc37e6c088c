"""GPU checks of the mixed-precision path: the BF16 tcgen05 GEMM, the hi/lo
split, the BF16 Omega stream and whole mixed solves against FP64 iSVD with the
same A and Omega (sigma relative error <= 1e-6 is the target)."""
import numpy as np
import pytest
import torch

from oracle import isvd_oracle as O

pytestmark = pytest.mark.gpu


def _bf16_mat(rows, cols, dev, g, scale=1.0):
    from mcnla_b200 import isvd
    buf, ld = isvd._bf16_buffer(rows, cols, dev)
    buf.copy_((scale * torch.randn(rows, cols, generator=g, device=dev)).to(torch.bfloat16))
    return buf, ld


@pytest.mark.parametrize("M,N,K,parts", [(128, 256, 64, 1), (300, 500, 1000, 1), (1000, 4096, 2000, 2),
                                         (129, 257, 65, 2), (4096, 320, 2000, 1), (500, 300, 777, 3),
                                         (1024, 512, 4096, 3)])
def test_gemm_bf16_against_fp64(cuda, M, N, K, parts):
    from mcnla_b200 import isvd
    g = torch.Generator(device=cuda).manual_seed(M + N + K)
    a_hi, lda = _bf16_mat(M, K, cuda, g)
    a_lo = _bf16_mat(M, K, cuda, g, 1e-3)[0] if parts >= 2 else None
    a_lo2 = _bf16_mat(M, K, cuda, g, 1e-6)[0] if parts >= 3 else None
    b, ldb = _bf16_mat(N, K, cuda, g)
    for out in (torch.float64, torch.float32):
        d = isvd.gemm_bf16(a_hi, a_lo, lda, b, ldb, out, a_lo2=a_lo2)
        a64 = a_hi.double() + (a_lo.double() if a_lo is not None else 0) + \
            (a_lo2.double() if a_lo2 is not None else 0)
        ref = a64 @ b.double().t()
        bound = a64.abs() @ b.double().abs().t()
        err = (d.double() - ref).abs()
        assert bool(torch.all(err <= 2e-6 * bound + 1e-30)), (err / bound).max().item()


def test_split_bf16_layouts(cuda):
    from mcnla_b200 import isvd
    g = torch.Generator(device=cuda).manual_seed(3)
    a = torch.randn(333, 517, generator=g, dtype=torch.float64, device=cuda)
    for view in (a, a.t().contiguous().t()):
        hi, lo, lo2, ld = isvd.split_bf16(view, 3)
        assert ld % 8 == 0
        assert torch.equal(hi, a.to(torch.bfloat16))
        rec = hi.double() + lo.double()
        assert bool(torch.all((rec - a).abs() <= 2.0 ** -16 * a.abs() + 1e-300))
        rec3 = rec + lo2.double()
        assert bool(torch.all((rec3 - a).abs() <= 2.0 ** -24 * a.abs() + 1e-300))
    # three parts hold an FP32 matrix exactly
    a32 = a.float().double()
    hi, lo, lo2, ld = isvd.split_bf16(a32, 3)
    assert torch.equal(hi.double() + lo.double() + lo2.double(), a32)
    two = isvd.split_bf16(a, 2)
    assert two.lo2 is None and two.parts == 2


def test_gaussian_bf16_matches_fp64_stream(cuda):
    from mcnla_b200 import isvd, _lib
    import ctypes
    n, L, seed = 777, 96, 11
    om_t, ld, om = isvd.gaussian_bf16(n, L, seed, cuda, with_fp64=True)
    ctx = isvd.context()
    full = torch.empty(n * L, dtype=torch.float64, device=cuda)
    _lib.check(ctx.lib.mcnla_b200_gaussian(ctx.bind(), ctypes.c_uint64(seed), n * L,
                                           ctypes.c_void_p(full.data_ptr())), "gaussian")
    ref = full.view(n, L)
    # BF16-representable and within half a BF16 ulp of the FP64 stream
    # (round to nearest from FP64; torch's own cast may round twice via FP32)
    assert torch.equal(om.to(torch.bfloat16).double(), om)
    assert bool(torch.all((om - ref).abs() <= 2.0 ** -8 * ref.abs()))   # half a BF16 ulp: <= 2^-8 relative
    assert torch.equal(om_t.double(), om.t())


def _metrics(s, u, v, s_ref, u_ref, v_ref):
    rel = np.max(np.abs(s - s_ref) / s_ref)
    # largest principal angle between the U (V) subspaces
    ang_u = np.arccos(np.clip(np.linalg.svd(u_ref.T @ u, compute_uv=False).min(), -1, 1))
    ang_v = np.arccos(np.clip(np.linalg.svd(v_ref.T @ v, compute_uv=False).min(), -1, 1))
    orth = np.linalg.norm(u.T @ u - np.eye(u.shape[1]))
    return rel, max(ang_u, ang_v), orth


@pytest.mark.parametrize("case", ["config1", "ill_conditioned"])
def test_mixed_matches_fp64_isvd(cuda, case):
    """Same A, same (BF16-representable) Omega: mixed vs plain FP64 iSVD."""
    from mcnla_b200 import isvd, synthetic
    if case == "config1":
        m, n, k, p, N = 1000, 2000, 10, 10, 16
        a = synthetic.lowrank_np(m, n, 1.0 / np.arange(1, 1001), seed=0)
    else:
        m, n, k, p, N = 1000, 2000, 64, 16, 32
        a = synthetic.lowrank_np(m, n, synthetic.config3_sigma(), seed=0, noise=1e-8)
    at = torch.as_tensor(a, device=cuda)
    seed = 5
    _, _, omega = isvd.gaussian_bf16(n, (k + p) * N, seed, cuda, with_fp64=True)
    s64, u64, v64, it64 = isvd.solve(at, k, p, N, omega=omega, integrator="rb_gramian_kn", former="svd", tol=1e-6)
    s, u, v, it = isvd.solve_mixed(at, k, p, N, seed=seed, integrator="rb_gramian_kn", former="svd", tol=1e-6)
    rel, ang, orth = _metrics(*(x.cpu().numpy() for x in (s, u, v, s64, u64, v64)))
    assert rel <= 1e-6, rel
    assert orth <= 1e-10, orth
    # hi-only sketch: coarser (8-bit A), reported not asserted to 1e-6
    s1, _, _, _ = isvd.solve_mixed(at, k, p, N, seed=seed, integrator="rb_gramian_kn", former="svd", tol=1e-6,
                                   parts=1)
    rel1 = np.max(np.abs(s1.cpu().numpy() - s64.cpu().numpy()) / s64.cpu().numpy())
    s3, _, _, _ = isvd.solve_mixed(at, k, p, N, seed=seed, integrator="rb_gramian_kn", former="svd", tol=1e-6,
                                   parts=3)
    rel3 = np.max(np.abs(s3.cpu().numpy() - s64.cpu().numpy()) / s64.cpu().numpy())
    print("%s: sigma rel err hi+lo %.2e (hi only %.2e, hi+lo+lo2 %.2e), max principal angle %.2e, ||U'U-I|| %.2e, "
          "it %d/%d" % (case, rel, rel1, rel3, ang, orth, it, it64))
    assert rel1 <= 1e-2
    assert rel3 <= 1e-6, rel3


@pytest.mark.parametrize("m,n,k,p", [(1000, 2000, 10, 10), (20011, 1537, 24, 8), (777, 3001, 64, 16)])
@pytest.mark.parametrize("former", ["svd", "rb_gramian"])
def test_form_bf16_matches_fp64_former(cuda, m, n, k, p, former):
    """Precision-form former (Q' A on tcgen05 from three BF16 parts of A' and of Qbar, split over
    K = m) against the FP64 former on the same A and Qbar: sigma to 1e-6 relative, U and V
    subspaces, U orthonormal to FP64 rounding."""
    from mcnla_b200 import isvd, synthetic
    a = torch.as_tensor(synthetic.lowrank_np(m, n, 1.0 / np.arange(1, min(m, n, 300) + 1), seed=m + n), device=cuda)
    g = torch.Generator(device=cuda).manual_seed(7)
    qbar = torch.linalg.qr(a @ torch.randn(n, k + p, generator=g, dtype=torch.float64, device=cuda))[0].contiguous()
    prm = isvd.Parameters(device=cuda).setSize(m, n).setRank(k).setOverRank(p).setNumSketch(1).sync()
    stage = {"svd": isvd.SvdFormer, "rb_gramian": isvd.RowBlockGramianFormer}[former](prm)
    stage.initialize()
    stage(a, qbar)
    s64, u64, v64 = (x.cpu().numpy() for x in (stage.vectorS(), stage.matrixU(), stage.matrixV()))
    at = isvd.split_bf16(a.t(), 3)
    assert at.hi.shape == (n, m)
    s, u, v = isvd.form_bf16(at, qbar, k, p, 1, former=former)
    rel, ang, orth = _metrics(*(x.cpu().numpy() for x in (s, u, v)), s64, u64, v64)
    print("form_bf16 %s %dx%d l=%d: sigma rel %.2e, angle %.2e, ||U'U-I|| %.2e" % (former, m, n, k + p, rel, ang, orth))
    assert rel <= 1e-6, rel
    assert ang <= 1e-5, ang
    assert orth <= 1e-10, orth
    # deterministic: the same call gives the same bits
    s2, u2, v2 = isvd.form_bf16(at, qbar, k, p, 1, former=former)
    assert torch.equal(s, s2) and torch.equal(u, u2) and torch.equal(v, v2)


@pytest.mark.parametrize("case", ["config1", "ill_conditioned"])
def test_mixed_precision_former_solve(cuda, case):
    """Whole mixed solve with the sketch and the former on tcgen05 (A' in three BF16 parts)
    against plain FP64 iSVD on the same A and Omega."""
    from mcnla_b200 import isvd, synthetic
    if case == "config1":
        m, n, k, p, N = 1000, 2000, 10, 10, 16
        a = synthetic.lowrank_np(m, n, 1.0 / np.arange(1, 1001), seed=0)
    else:
        m, n, k, p, N = 1000, 2000, 64, 16, 32
        a = synthetic.lowrank_np(m, n, synthetic.config3_sigma(), seed=0, noise=1e-8)
    at = torch.as_tensor(a, device=cuda)
    seed = 5
    _, _, omega = isvd.gaussian_bf16(n, (k + p) * N, seed, cuda, with_fp64=True)
    s64, u64, v64, it64 = isvd.solve(at, k, p, N, omega=omega, integrator="rb_gramian_kn", former="rb_gramian",
                                     tol=1e-6)
    fs = isvd.split_bf16(at.t(), 3)
    for former in ("rb_gramian", "svd"):
        s, u, v, it = isvd.solve_mixed(at, k, p, N, seed=seed, integrator="rb_gramian_kn", former=former, tol=1e-6,
                                       parts=3, former_split=fs)
        rel, ang, orth = _metrics(*(x.cpu().numpy() for x in (s, u, v, s64, u64, v64)))
        print("%s %s: sigma rel %.2e, angle %.2e, ||U'U-I|| %.2e, it %d/%d" % (case, former, rel, ang, orth, it, it64))
        assert rel <= 1e-6, rel
        assert orth <= 1e-10, orth


def test_mixed_gramian_loop_bf16(cuda):
    """N l > 1536 and (N l)^2 m >= 1e11: the mixed solve forms Bs from BF16 parts of Qs and its
    row-block Gramian KN loop runs Bs Bc on tcgen05 (three BF16 parts of Bs and of Bc each
    iteration), then re-orthonormalizes Qbar in FP64; sigma against plain FP64 iSVD on the same A
    and Omega to 1e-6, U orthonormal to FP64 rounding."""
    from mcnla_b200 import isvd, synthetic
    m, n, k, p, N = 30000, 3000, 30, 10, 48
    a = torch.as_tensor(synthetic.lowrank_np(m, n, np.exp(-np.arange(1, 201) / 30.0), seed=3, noise=1e-4),
                        device=cuda)
    seed = 9
    _, _, omega = isvd.gaussian_bf16(n, (k + p) * N, seed, cuda, with_fp64=True)
    s64, u64, v64, it64 = isvd.solve(a, k, p, N, omega=omega, integrator="rb_gramian_kn", former="rb_gramian",
                                     tol=1e-6)
    s, u, v, it = isvd.solve_mixed(a, k, p, N, seed=seed, integrator="rb_gramian_kn", former="rb_gramian", tol=1e-6,
                                   parts=3)
    rel, ang, orth = _metrics(*(x.cpu().numpy() for x in (s, u, v, s64, u64, v64)))
    print("gramian loop bf16: sigma rel %.2e, angle %.2e, ||U'U-I|| %.2e, it %d/%d" % (rel, ang, orth, it, it64))
    assert rel <= 1e-6, rel
    assert orth <= 1e-10, orth
    s2, u2, v2, it2 = isvd.solve_mixed(a, k, p, N, seed=seed, integrator="rb_gramian_kn", former="rb_gramian",
                                       tol=1e-6, parts=3)
    assert it2 == it and torch.equal(s2, s) and torch.equal(u2, u)

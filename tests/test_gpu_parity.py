"""GPU parity: the B200 kernels (through the C ABI) against the reference's
golden fixtures, the CPU oracle and plain torch FP64 products.

Tolerances: the FP64 path must reproduce the reference to 1e-10 (relative for
singular values; absolute, up to column sign, for unit-norm singular vectors
and bases) with identical integrator iteration counts; the reference's own
fixture checks use 1e-8.
"""
import numpy as np
import pytest
import torch

from oracle import isvd_oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-10


def dev(x, cuda):
    return torch.as_tensor(np.ascontiguousarray(x), dtype=torch.float64, device=cuda)


def host(t):
    return t.detach().cpu().numpy()


def params(m, n, k, p, N):
    from mcnla_b200 import isvd
    return isvd.Parameters().setSize(m, n).setRank(k).setOverRank(p).setNumSketch(N).sync()


# ------------------------------------------------------------------------------------------------
# building blocks
# ------------------------------------------------------------------------------------------------
GEMM_SHAPES = [(1, 1, 1), (7, 5, 3), (101, 11, 1001), (300, 64, 257), (129, 130, 131), (1000, 320, 2000),
               (64, 64, 5000), (20, 20, 100000)]


@pytest.mark.parametrize("M,N,K", GEMM_SHAPES)
@pytest.mark.parametrize("ta,tb", [(False, False), (True, False), (False, True), (True, True)])
def test_dgemm_layouts(cuda, M, N, K, ta, tb):
    from mcnla_b200 import isvd, _lib
    import ctypes
    g = torch.Generator(device=cuda).manual_seed(M * 7 + N * 3 + K)
    a = torch.randn(K, M, generator=g, dtype=torch.float64, device=cuda).t() if ta else \
        torch.randn(M, K, generator=g, dtype=torch.float64, device=cuda)
    b = torch.randn(N, K, generator=g, dtype=torch.float64, device=cuda).t() if tb else \
        torch.randn(K, N, generator=g, dtype=torch.float64, device=cuda)
    c0 = torch.randn(M, N, generator=g, dtype=torch.float64, device=cuda)
    for alpha, beta, splits in [(1.0, 0.0, 0), (0.5, -2.0, 0), (1.0, 1.0, 3)]:
        c = c0.clone()
        ctx = isvd.context()
        st = ctx.lib.mcnla_b200_dgemm(ctx.bind(), M, N, K, alpha, ctypes.c_void_p(a.data_ptr()), a.stride(0),
                                      a.stride(1), ctypes.c_void_p(b.data_ptr()), b.stride(0), b.stride(1), beta,
                                      ctypes.c_void_p(c.data_ptr()), c.stride(0), c.stride(1), splits)
        _lib.check(st, "dgemm")
        ref = alpha * (a @ b) + beta * c0
        scale = (a.abs() @ b.abs()).max().item() + c0.abs().max().item()
        assert (c - ref).abs().max().item() <= 1e-14 * scale * max(1, K) ** 0.5 + 1e-300


@pytest.mark.parametrize("n,batch", [(1, 1), (2, 3), (11, 12), (20, 16), (64, 4), (80, 2), (113, 1), (160, 1)])
def test_syev_batched(cuda, n, batch):
    from mcnla_b200 import isvd, _lib
    import ctypes
    rng = np.random.default_rng(n)
    x = rng.standard_normal((batch, n, n))
    a = x + x.transpose(0, 2, 1)
    for order in (0, 1):
        at = dev(a, cuda)
        w = torch.empty(batch, n, dtype=torch.float64, device=cuda)
        v = torch.empty(batch, n, n, dtype=torch.float64, device=cuda)
        ctx = isvd.context()
        _lib.check(ctx.lib.mcnla_b200_syev_batched(ctx.bind(), n, batch, ctypes.c_void_p(at.data_ptr()),
                                                   ctypes.c_void_p(w.data_ptr()), ctypes.c_void_p(v.data_ptr()),
                                                   order), "syev")
        wn, vn = host(w), host(v)
        for b in range(batch):
            lam = np.linalg.eigvalsh(a[b])
            ref = np.sort(np.abs(lam))[::-1] if order else lam
            scale = np.abs(lam).max()
            assert np.abs(wn[b] - ref).max() <= 1e-13 * scale * n
            # A V = V diag(lambda) with signed eigenvalues, V orthogonal
            lam_signed = np.diag(vn[b].T @ a[b] @ vn[b])
            assert np.abs(a[b] @ vn[b] - vn[b] * lam_signed).max() <= 1e-12 * scale * n
            assert np.abs(vn[b].T @ vn[b] - np.eye(n)).max() <= 1e-13 * n


@pytest.mark.parametrize("n", [1, 5, 22, 128, 160])
def test_inverse_batched(cuda, n):
    from mcnla_b200 import isvd, _lib
    import ctypes
    rng = np.random.default_rng(n)
    a = rng.standard_normal((2, n, n)) + 3 * np.eye(n)
    at = dev(a, cuda)
    ctx = isvd.context()
    _lib.check(ctx.lib.mcnla_b200_inverse_batched(ctx.bind(), n, 2, ctypes.c_void_p(at.data_ptr())), "inverse")
    inv = host(at)
    for b in range(2):
        assert np.abs(inv[b] - np.linalg.inv(a[b])).max() <= 1e-12 * np.linalg.cond(a[b])


def test_inverse_singular_reports_status(cuda):
    from mcnla_b200 import isvd, _lib
    import ctypes
    a = torch.zeros(1, 4, 4, dtype=torch.float64, device=cuda)
    ctx = isvd.context()
    st = ctx.lib.mcnla_b200_inverse_batched(ctx.bind(), 4, 1, ctypes.c_void_p(a.data_ptr()))
    assert st == _lib.ERR_SINGULAR


def test_gaussian_generator(cuda):
    from mcnla_b200 import isvd, _lib
    import ctypes
    ctx = isvd.context()
    out = torch.empty(2_000_001, dtype=torch.float64, device=cuda)
    out2 = torch.empty_like(out)
    for t in (out, out2):
        _lib.check(ctx.lib.mcnla_b200_gaussian(ctx.bind(), ctypes.c_uint64(42), t.numel(),
                                               ctypes.c_void_p(t.data_ptr())), "gaussian")
    assert torch.equal(out, out2)
    x = host(out)
    assert abs(x.mean()) < 5e-3 and abs(x.std() - 1) < 5e-3
    assert abs(np.mean(x ** 4) - 3) < 5e-2        # Gaussian kurtosis
    other = torch.empty(1000, dtype=torch.float64, device=cuda)
    _lib.check(ctx.lib.mcnla_b200_gaussian(ctx.bind(), ctypes.c_uint64(43), 1000,
                                           ctypes.c_void_p(other.data_ptr())), "gaussian")
    assert not torch.equal(other, out[:1000])


# ------------------------------------------------------------------------------------------------
# stages against the reference's golden fixtures (check/isvd/**.cpp criteria) and the oracle
# ------------------------------------------------------------------------------------------------
def test_orthogonalizer_golden(cuda, golden):
    from mcnla_b200 import isvd
    m, l, N = golden["m"], golden["l"], golden["N"]
    prm = params(m, l, l, 0, N)
    for cls in (isvd.GramianOrthogonalizer, isvd.RowBlockGramianOrthogonalizer):
        orth = cls(prm)
        orth.initialize()
        q = dev(golden["ys"], cuda)
        orth(q)
        qn = host(q)
        qo = O.orthogonalize_gramian(golden["ys"], l, N)
        for i in range(N):
            qi = qn[:, i * l:(i + 1) * l]
            assert O.projector_gap(qi, golden["qi"][i]) < 1e-8
            assert O.projector_gap(qi, qo[:, i * l:(i + 1) * l]) < TOL
        assert len(orth.times()) == 1 and orth.time() > 0


@pytest.mark.parametrize("cls_name,oracle_name", [
    ("KolmogorovNagumoIntegrator", "kn"),
    ("RowBlockKolmogorovNagumoIntegrator", "rb_kn"),
    ("RowBlockGramianKolmogorovNagumoIntegrator", "rb_gramian_kn"),
])
def test_kn_golden(cuda, golden, cls_name, oracle_name):
    from mcnla_b200 import isvd
    m, l, N = golden["m"], golden["l"], golden["N"]
    prm = params(m, l, l, 0, N)
    integ = getattr(isvd, cls_name)(prm, 256, 1e-4)
    integ.initialize()
    q = dev(golden["qs"], cuda)
    qbar = prm.createMatrixQbar()
    integ(q, qbar)
    assert integ.iteration() == 81
    qb = host(qbar)
    assert np.abs(qb - golden["qb_kn"]).max() < 1e-8
    qo, it = O.INTEGRATORS[oracle_name](golden["qs"], l, N, 256, 1e-4)
    assert it == integ.iteration()
    assert np.abs(qb - qo).max() < TOL


@pytest.mark.parametrize("cls_name", ["KolmogorovNagumoIntegrator", "RowBlockKolmogorovNagumoIntegrator",
                                      "RowBlockGramianKolmogorovNagumoIntegrator"])
def test_kn_step_methods_agree(cuda, golden, cls_name):
    """The series, Newton-Schulz and eigendecomposition forms of the KN step
    give the same integrated basis and iteration count on the golden fixture."""
    from mcnla_b200 import isvd, _lib
    m, l, N = golden["m"], golden["l"], golden["N"]
    prm = params(m, l, l, 0, N)
    out = []
    ctx = isvd.context()
    try:
        for method in (_lib.KN_AUTO, _lib.KN_NEWTON_SCHULZ, _lib.KN_EIGEN):
            ctx.set_kn_method(method)
            integ = getattr(isvd, cls_name)(prm, 256, 1e-4)
            integ.initialize()
            qbar = prm.createMatrixQbar()
            integ(dev(golden["qs"], cuda), qbar)
            out.append((integ.iteration(), host(qbar)))
    finally:
        ctx.set_kn_method(_lib.KN_AUTO)
    assert out[0][0] == out[1][0] == out[2][0] == 81
    assert np.abs(out[0][1] - out[2][1]).max() < TOL
    assert np.abs(out[1][1] - out[2][1]).max() < TOL


def test_gramian_kn_runs_persistent(cuda, golden):
    """With the default step method the row-block Gramian KN integrator runs
    whole iterations in one cooperative kernel: far fewer launches than the
    four or more per iteration of the launch-per-product loop."""
    from mcnla_b200 import isvd, _lib
    m, l, N = golden["m"], golden["l"], golden["N"]
    prm = params(m, l, l, 0, N)
    ctx = isvd.context()
    counts = []
    for method in (_lib.KN_AUTO, _lib.KN_NEWTON_SCHULZ):
        ctx.set_kn_method(method)
        integ = isvd.RowBlockGramianKolmogorovNagumoIntegrator(prm, 256, 1e-4)
        integ.initialize()
        qbar = prm.createMatrixQbar()
        k0 = ctx.kernels_launched()
        integ(dev(golden["qs"], cuda), qbar)
        counts.append(ctx.kernels_launched() - k0)
        assert integ.iteration() == 81
    ctx.set_kn_method(_lib.KN_AUTO)
    assert counts[0] < 40 and counts[1] > 4 * 81, counts


@pytest.mark.parametrize("l", [5, 48, 96, 160])
@pytest.mark.parametrize("cls_name,oracle_name", [
    ("KolmogorovNagumoIntegrator", "kn"),
    ("RowBlockKolmogorovNagumoIntegrator", "rb_kn"),
    ("RowBlockGramianKolmogorovNagumoIntegrator", "rb_gramian_kn"),
])
def test_kn_wide_sketches(cuda, l, cls_name, oracle_name):
    """KN integrators up to the largest sketch (l = 160, past the one-CTA
    matrix-function limit): every step method against the oracle."""
    from mcnla_b200 import isvd, _lib, synthetic
    m, n, N = 1500, 700, 4
    a = synthetic.lowrank_np(m, n, np.arange(1, n + 1) ** -1.0, seed=l)
    omega = np.random.default_rng(l).standard_normal((n, l * N))
    qs = O.orthogonalize_gramian(a @ omega, l, N)
    qo, it_ref = O.INTEGRATORS[oracle_name](qs, l, N, 256, 1e-5)
    prm = params(m, n, l, 0, N)
    ctx = isvd.context()
    try:
        for method in (_lib.KN_AUTO, _lib.KN_NEWTON_SCHULZ, _lib.KN_EIGEN):
            ctx.set_kn_method(method)
            integ = getattr(isvd, cls_name)(prm, 256, 1e-5)
            integ.initialize()
            qbar = prm.createMatrixQbar()
            integ(dev(qs, cuda), qbar)
            assert integ.iteration() == it_ref, method
            assert np.abs(host(qbar) - qo).max() < TOL, method
    finally:
        ctx.set_kn_method(_lib.KN_AUTO)


@pytest.mark.parametrize("cls_name,oracle_name", [
    ("RowBlockWenYinIntegrator", "rb_wy"),
    ("RowBlockGramianWenYinIntegrator", "rb_gramian_wy"),
])
def test_wy_golden(cuda, golden, cls_name, oracle_name):
    from mcnla_b200 import isvd
    m, l, N = golden["m"], golden["l"], golden["N"]
    prm = params(m, l, l, 0, N)
    integ = getattr(isvd, cls_name)(prm, 256, 1e-3)
    integ.initialize()
    q = dev(golden["qs"], cuda)
    qbar = prm.createMatrixQbar()
    integ(q, qbar)
    assert integ.iteration() == 21
    qb = host(qbar)
    assert np.abs(qb - golden["qb_wy"]).max() < 1e-8
    qo, it = O.INTEGRATORS[oracle_name](golden["qs"], l, N, 256, 1e-3)
    assert it == integ.iteration()
    assert np.abs(qb - qo).max() < 1e-9


@pytest.mark.parametrize("cls_name,oracle_name,colmajor", [
    ("SvdFormer", "svd", False), ("SvdFormer", "svd", True), ("GramianFormer", "gramian", False),
    ("RowBlockGramianFormer", "gramian", False), ("ColBlockGramianFormer", "gramian", True),
])
def test_formers_golden(cuda, golden, cls_name, oracle_name, colmajor):
    from mcnla_b200 import isvd
    a, q = golden["a"], golden["q"]
    m, n = a.shape
    k = q.shape[1] // 2
    p = q.shape[1] - k
    prm = params(m, n, k, p, 1)
    former = getattr(isvd, cls_name)(prm)
    former.initialize()
    at = dev(a.T, cuda).t() if colmajor else dev(a, cuda)
    former(at, dev(q, cuda))
    s, u, v = host(former.vectorS()), host(former.matrixU()), host(former.matrixV())
    assert O.projector_gap(u, golden["u"][:, :k]) < 1e-8
    so, uo, vo = O.FORMERS[oracle_name](a, q, k)
    np.testing.assert_allclose(s, so, rtol=TOL)
    assert np.abs(O.align_signs(u, uo) - uo).max() < TOL
    assert np.abs(O.align_signs(v, vo) - vo).max() < TOL
    assert len(former.times()) == 3


# ------------------------------------------------------------------------------------------------
# sketcher and whole pipeline against the oracle on seeded synthetic matrices
# ------------------------------------------------------------------------------------------------
@pytest.mark.parametrize("colmajor,exponent", [(False, 0), (True, 0), (False, 2)])
def test_sketch_explicit_omega(cuda, colmajor, exponent):
    from mcnla_b200 import isvd, synthetic
    a, omega = synthetic.config1_numpy(m=301, n=517, k=5, p=4, N=6, seed=11)
    a = a / np.linalg.norm(a, 2)
    prm = params(301, 517, 5, 4, 6)
    sk = isvd.GaussianProjectionSketcher(prm, 0, exponent)
    sk.initialize()
    sk.setOmega(dev(omega, cuda))
    q = prm.createCollectionQ()
    at = dev(a.T, cuda).t() if colmajor else dev(a, cuda)
    sk(at, q)
    ref = O.sketch_power(a, omega, exponent)
    assert np.abs(host(q) - ref).max() <= 1e-12 * np.abs(ref).max()


def _pipeline(cuda, a, omega, k, p, N, integrator, former, tol, colmajor=False):
    from mcnla_b200 import isvd
    at = dev(a.T, cuda).t() if colmajor else dev(a, cuda)
    s, u, v, it = isvd.solve(at, k, p, N, omega=dev(omega, cuda), integrator=integrator, former=former, tol=tol)
    return host(s), host(u), host(v), it


@pytest.mark.parametrize("integrator", list(O.INTEGRATORS))
@pytest.mark.parametrize("former", ["svd", "gramian"])
def test_pipeline_config1_shape(cuda, integrator, former):
    """The first benchmark configuration's shape (m=1000, n=2000, k=10, p=10,
    N=16, sigma_j = 1/j): singular values and vectors to 1e-10 of the oracle,
    identical iteration counts."""
    from mcnla_b200 import synthetic
    a, omega = synthetic.config1_numpy(seed=0)
    tol = 1e-4 if "kn" in integrator else 1e-3
    s, u, v, it = _pipeline(cuda, a, omega, 10, 10, 16, integrator, former if former == "svd" else "gramian", tol)
    ref = O.isvd(a, omega, 10, 10, 16, integrator=integrator, former=former, tol=tol)
    assert it == ref["iterations"]
    np.testing.assert_allclose(s, ref["s"], rtol=TOL)
    assert np.abs(O.align_signs(u, ref["u"]) - ref["u"]).max() < TOL
    assert np.abs(O.align_signs(v, ref["v"]) - ref["v"]).max() < TOL


def rounding_sensitivity(a, omega, k, p, N, integ, tol, ref):
    """How far the reference algorithm itself moves sigma when A is perturbed
    at the rounding level (1e-16 relative): the floor of any two FP64
    implementations' agreement.  The row-block Gramian Wen-Yin integrator
    amplifies rounding by about 1e7 (its Qbar = Q0 F~ + Qs E~ cancels), the
    others stay near 1e-15."""
    rng = np.random.default_rng(1)
    a1 = a * (1 + 1e-16 * rng.standard_normal(a.shape))
    r1 = O.isvd(a1, omega, k, p, N, integrator=integ, former="svd", tol=tol)
    return float(np.max(np.abs(r1["s"] - ref["s"]) / ref["s"]))


@pytest.mark.parametrize("m,n,k,p,N", [(97, 61, 3, 2, 1), (257, 129, 7, 5, 3), (640, 300, 30, 2, 4),
                                       (50, 2000, 8, 8, 2)])
def test_pipeline_ragged_shapes(cuda, m, n, k, p, N):
    from mcnla_b200 import synthetic
    rng = np.random.default_rng(m + n)
    a = synthetic.lowrank_np(m, n, 1.0 / np.arange(1, min(m, n) + 1), seed=m)
    omega = rng.standard_normal((n, (k + p) * N))
    for integ in ("kn", "rb_gramian_wy"):
        ref = O.isvd(a, omega, k, p, N, integrator=integ, former="svd", tol=1e-4)
        tol_s = max(TOL, 20 * rounding_sensitivity(a, omega, k, p, N, integ, 1e-4, ref))
        for colmajor in (False, True):
            s, u, v, it = _pipeline(cuda, a, omega, k, p, N, integ, "svd", 1e-4, colmajor)
            assert it == ref["iterations"]
            np.testing.assert_allclose(s, ref["s"], rtol=tol_s)


def test_host_entry_point_matches_device(cuda):
    from mcnla_b200 import isvd, synthetic
    a, omega = synthetic.config1_numpy(m=400, n=700, k=8, p=8, N=4, seed=5)
    s1, u1, v1, it1 = isvd.solve(dev(a, cuda), 8, 8, 4, omega=dev(omega, cuda), integrator="rb_kn")
    a_h = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    o_h = torch.from_numpy(np.ascontiguousarray(omega)).pin_memory()
    s2, u2, v2, it2 = isvd.solve_host(a_h, o_h, 8, 8, 4, integrator="rb_kn")
    assert it1 == it2
    assert torch.equal(s1.cpu(), s2) and torch.equal(u1.cpu(), u2) and torch.equal(v1.cpu(), v2)
    # column-major host buffer
    s3, _, _, it3 = isvd.solve_host(torch.from_numpy(np.ascontiguousarray(a.T)), o_h, 8, 8, 4,
                                    integrator="rb_kn", colmajor=True)
    assert it3 == it1
    np.testing.assert_allclose(s3.numpy(), s2.numpy(), rtol=1e-12)


@pytest.mark.parametrize("m,n", [(6000, 2000), (1100, 8000)])
def test_host_entry_point_streams_large_a(cuda, m, n):
    """Row-major host A of 64 MB or more is copied in row blocks behind the sketch; the result is
    bit for bit the device-resident solve's (the second shape's whole sketch GEMM uses split-K,
    which every row block repeats)."""
    from mcnla_b200 import isvd, synthetic
    a, omega = synthetic.config1_numpy(m=m, n=n, k=8, p=8, N=4, seed=6)
    assert a.nbytes >= 64 << 20
    s1, u1, v1, it1 = isvd.solve(dev(a, cuda), 8, 8, 4, omega=dev(omega, cuda), integrator="rb_gramian_kn",
                                 former="rb_gramian")
    a_h = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    o_h = torch.from_numpy(np.ascontiguousarray(omega)).pin_memory()
    for _ in range(2):
        s2, u2, v2, it2 = isvd.solve_host(a_h, o_h, 8, 8, 4, integrator="rb_gramian_kn", former="rb_gramian")
        assert it1 == it2
        assert torch.equal(s1.cpu(), s2) and torch.equal(u1.cpu(), u2) and torch.equal(v1.cpu(), v2)


@pytest.mark.parametrize("m,n", [(2048, 4096), (101, 1001)])
def test_streamed_ingest_from_a_binary_file(cuda, tmp_path, m, n):
    """mcnla_b200_isvd_stream with the binary file's row reader (the reference's loadBinaryRowBlock):
    the file's row blocks are read into pinned staging while the previous ones are copied and
    sketched; the result is bit for bit the host-buffer solve's and the device-resident solve's.
    A reader that fails stops the solve with its error."""
    from mcnla_b200 import io, isvd, synthetic
    a, omega = synthetic.config1_numpy(m=m, n=n, k=8, p=8, N=4, seed=3)
    path = tmp_path / "a.bin"
    io.save_binary(path, a)
    mm, nn, read_rows = io.binary_row_reader(path)
    assert (mm, nn) == (m, n)
    calls = []

    def reader(row0, rows, buf):
        calls.append((row0, rows))
        read_rows(row0, rows, buf)
    o_h = torch.from_numpy(np.ascontiguousarray(omega)).pin_memory()
    s1, u1, v1, it1 = isvd.solve_stream(reader, m, n, o_h, 8, 8, 4, integrator="rb_gramian_kn", former="rb_gramian")
    assert calls[0][0] == 0 and sum(r for _, r in calls) == m
    assert all(calls[i][0] + calls[i][1] == calls[i + 1][0] for i in range(len(calls) - 1))
    a_h = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    s2, u2, v2, it2 = isvd.solve_host(a_h, o_h, 8, 8, 4, integrator="rb_gramian_kn", former="rb_gramian")
    s3, u3, v3, it3 = isvd.solve(dev(a, cuda), 8, 8, 4, omega=dev(omega, cuda), integrator="rb_gramian_kn",
                                 former="rb_gramian")
    assert it1 == it2 == it3
    assert torch.equal(s1, s2) and torch.equal(u1, u2) and torch.equal(v1, v2)
    assert torch.equal(s1, s3.cpu()) and torch.equal(u1, u3.cpu())

    def failing(row0, rows, buf):
        if row0 > 0 or rows < m:
            raise IOError("truncated file")
        read_rows(row0, rows, buf)
    if len(calls) > 1:
        with pytest.raises(IOError):
            isvd.solve_stream(failing, m, n, o_h, 8, 8, 4, integrator="rb_gramian_kn", former="rb_gramian")


def test_stage_api_pipeline_with_device_omega(cuda):
    """Stages chained as the reference's driver does, Omega drawn on the device."""
    from mcnla_b200 import isvd, synthetic
    a, _ = synthetic.config1_numpy(m=500, n=800, k=6, p=6, N=8, seed=9)
    prm = params(500, 800, 6, 6, 8)
    sk = isvd.GaussianProjectionSketcher(prm, 1234)
    orth = isvd.GramianOrthogonalizer(prm)
    integ = isvd.KolmogorovNagumoIntegrator(prm)
    former = isvd.SvdFormer(prm)
    for st in (sk, orth, integ, former):
        st.initialize()
    at = dev(a, cuda)
    q = prm.createCollectionQ()
    qbar = prm.createMatrixQbar()
    sk(at, q)
    orth(q)
    integ(q, qbar)
    former(at, qbar)
    omega = host(sk.matrixOmega())
    ref = O.isvd(a, omega, 6, 6, 8, integrator="kn", former="svd", tol=1e-4)
    assert integ.iteration() == ref["iterations"]
    np.testing.assert_allclose(host(former.vectorS()), ref["s"], rtol=TOL)
    # determinism of the device draw
    q2 = prm.createCollectionQ()
    sk(at, q2)
    orth(q2)
    assert torch.equal(q, q2)


# ------------------------------------------------------------------------------------------------
# errors and edge cases
# ------------------------------------------------------------------------------------------------
def test_errors_are_statuses(cuda):
    from mcnla_b200 import isvd, _lib
    import ctypes
    ctx = isvd.context()
    h = ctx.bind()
    q = torch.zeros(10, 200, dtype=torch.float64, device=cuda)
    qbar = torch.zeros(10, 200, dtype=torch.float64, device=cuda)
    it = ctypes.c_int()
    big = _lib.Params(10, 10, 150, 50, 1)           # l = 200 > 160
    assert ctx.lib.mcnla_b200_integrate(h, ctypes.byref(big), 0, ctypes.c_void_p(q.data_ptr()), 5, 1e-4,
                                        ctypes.c_void_p(qbar.data_ptr()), ctypes.byref(it)) == _lib.ERR_UNSUPPORTED
    wy = _lib.Params(10, 10, 81, 0, 1)              # Wen-Yin limit l <= 80
    assert ctx.lib.mcnla_b200_integrate(h, ctypes.byref(wy), _lib.ROW_BLOCK_WEN_YIN, ctypes.c_void_p(q.data_ptr()),
                                        5, 1e-4, ctypes.c_void_p(qbar.data_ptr()), ctypes.byref(it)) \
        == _lib.ERR_UNSUPPORTED
    bad = _lib.Params(0, 10, 2, 2, 1)
    assert ctx.lib.mcnla_b200_orthogonalize(h, ctypes.byref(bad), ctypes.c_void_p(q.data_ptr())) == _lib.ERR_SHAPE
    ok = _lib.Params(10, 10, 2, 2, 1)
    assert ctx.lib.mcnla_b200_integrate(h, ctypes.byref(ok), 9, ctypes.c_void_p(q.data_ptr()), 5, 1e-4,
                                        ctypes.c_void_p(qbar.data_ptr()), ctypes.byref(it)) == _lib.ERR_ARG
    # the context is still usable afterwards
    a = torch.eye(4, dtype=torch.float64, device=cuda)
    c = torch.zeros(4, 4, dtype=torch.float64, device=cuda)
    _lib.check(ctx.lib.mcnla_b200_dgemm(h, 4, 4, 4, 1.0, ctypes.c_void_p(a.data_ptr()), 4, 1,
                                        ctypes.c_void_p(a.data_ptr()), 4, 1, 0.0, ctypes.c_void_p(c.data_ptr()), 4,
                                        1, 0), "dgemm")
    assert torch.equal(c, a)


@pytest.mark.parametrize("name", list(O.INTEGRATORS))
def test_integrators_maxit_zero(cuda, golden, name):
    from mcnla_b200 import isvd
    cls = {"kn": isvd.KolmogorovNagumoIntegrator, "rb_kn": isvd.RowBlockKolmogorovNagumoIntegrator,
           "rb_gramian_kn": isvd.RowBlockGramianKolmogorovNagumoIntegrator, "rb_wy": isvd.RowBlockWenYinIntegrator,
           "rb_gramian_wy": isvd.RowBlockGramianWenYinIntegrator}[name]
    m, l, N = golden["m"], golden["l"], golden["N"]
    prm = params(m, l, l, 0, N)
    integ = cls(prm, 0)
    integ.initialize()
    qbar = prm.createMatrixQbar()
    integ(dev(golden["qs"], cuda), qbar)
    assert integ.iteration() == 0
    assert np.abs(host(qbar) - golden["qs"][:, :l]).max() < 1e-14


@pytest.mark.parametrize("M,N,K", [(4096, 64, 4096), (384, 48, 8448), (64, 128, 4096), (1000, 96, 192)])
def test_dgemm_autotuned_matches_heuristic(cuda, M, N, K):
    """The tuned tile / split-K choice gives the product to the same accuracy as
    the fixed heuristic, and later calls of the shape reuse the decision (bit
    for bit the same result)."""
    from mcnla_b200 import isvd, _lib
    import ctypes
    g = torch.Generator(device=cuda).manual_seed(M + N + K)
    a = torch.randn(M, K, generator=g, dtype=torch.float64, device=cuda)
    b = torch.randn(K, N, generator=g, dtype=torch.float64, device=cuda)
    ctx = isvd.context()
    outs = []
    try:
        for on in (False, True, True):
            ctx.set_autotune(on)
            c = torch.empty(M, N, dtype=torch.float64, device=cuda)
            _lib.check(ctx.lib.mcnla_b200_dgemm(ctx.bind(), M, N, K, 1.0, ctypes.c_void_p(a.data_ptr()), K, 1,
                                                ctypes.c_void_p(b.data_ptr()), N, 1, 0.0,
                                                ctypes.c_void_p(c.data_ptr()), N, 1, 0), "dgemm")
            outs.append(c)
    finally:
        ctx.set_autotune(True)
    ref = a @ b
    scale = (a.abs() @ b.abs()).max().item()
    for c in outs:
        assert (c - ref).abs().max().item() <= 1e-14 * scale * K ** 0.5
    assert torch.equal(outs[1], outs[2])


@pytest.mark.parametrize("integrator,shape", [("kn", (1000, 2000, 10, 10, 16)), ("rb_kn", (1000, 2000, 10, 10, 16)),
                                              ("rb_gramian_kn", (3000, 2000, 20, 12, 50))])
def test_graph_loop_matches_direct(cuda, integrator, shape):
    """The KN loop replayed as a captured CUDA graph gives the same bits and the same iteration
    count as direct launches (the last shape has N l = 1600, past the persistent kernel)."""
    from mcnla_b200 import isvd, synthetic
    m, n, k, p, N = shape
    a = torch.as_tensor(synthetic.lowrank_np(m, n, 1.0 / np.arange(1, min(m, n) + 1), seed=4), device=cuda)
    ctx = isvd.context()
    out = []
    try:
        for on in (False, True, True):
            ctx.set_graph_loop(on)
            r0 = ctx.graph_replays()
            out.append(isvd.solve(a, k, p, N, seed=2, integrator=integrator, former="svd", tol=1e-5))
            replays = ctx.graph_replays() - r0
            assert (replays > 0) == on, replays
    finally:
        ctx.set_graph_loop(True)
    (s0, u0, v0, it0) = out[0]
    assert it0 > 24, it0          # several graph chunks ran
    for s1, u1, v1, it1 in out[1:]:
        assert it1 == it0
        assert torch.equal(s1, s0) and torch.equal(u1, u0) and torch.equal(v1, v0)


@pytest.mark.parametrize("l,N", [(96, 8), (48, 8), (20, 16)])
def test_persistent_integrator_bits_do_not_depend_on_its_cta_share(cuda, l, N):
    """The persistent row-block Gramian KN kernel folds every product element's K chunks in one
    fixed order, by one warp per tile (when the product has at least as many tiles as the grid has
    warps) or by the CTA's warps through shared memory: the same bits on 8, 18, 37 CTAs and the
    whole GPU, and the oracle's iteration count."""
    from mcnla_b200 import isvd, synthetic
    m, n = 3000, 1200
    a = synthetic.lowrank_np(m, n, np.arange(1, n + 1) ** -1.0, seed=l)
    omega = np.random.default_rng(l + 1).standard_normal((n, l * N))
    qs = O.orthogonalize_gramian(a @ omega, l, N)
    qo, it_ref = O.INTEGRATORS["rb_gramian_kn"](qs, l, N, 256, 1e-5)
    prm = params(m, n, l, 0, N)
    ctx = isvd.context()
    outs = []
    try:
        for ctas in (8, 18, 37, 0):
            ctx.set_cta_limit(ctas)
            integ = isvd.RowBlockGramianKolmogorovNagumoIntegrator(prm, 256, 1e-5)
            integ.initialize()
            qbar = prm.createMatrixQbar()
            integ(dev(qs, cuda), qbar)
            assert integ.iteration() == it_ref, ctas
            outs.append(qbar.clone())
    finally:
        ctx.set_cta_limit(0)
    for q in outs[1:]:
        assert torch.equal(q, outs[0])
    assert np.abs(host(outs[-1]) - qo).max() < TOL

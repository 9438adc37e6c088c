"""Pins the CPU oracle (oracle/isvd_oracle.py) to the reference.

1. Against the reference's own golden fixtures with the reference's own
   criteria (check/isvd/**.cpp): projectors within 1e-8, integrated bases
   element-wise within 1e-8, iteration counts 81 (KN, tol 1e-4) and 21 (WY,
   tol 1e-3), former U U' within 1e-8.
2. Against the outputs of the reference's own stages compiled here
   (tests/golden/ref_outputs.npz, made by tests/golden/make_golden.py), and,
   when oracle/_ref is built, against a live call of it.
"""
import numpy as np
import pytest

from oracle import isvd_oracle as O

KN_CASES = [("kn", 0), ("rb_kn", 1), ("rb_gramian_kn", 2)]
WY_CASES = [("rb_wy", 3), ("rb_gramian_wy", 4)]


def test_orthogonalizer_golden(golden, ref_outputs):
    # check/isvd/orthogonalizer/gramian_orthogonalizer.cpp:58-67
    l, N = golden["l"], golden["N"]
    q = O.orthogonalize_gramian(golden["ys"], l, N)
    for i in range(N):
        qi = q[:, i * l:(i + 1) * l]
        assert O.projector_gap(qi, golden["qi"][i]) < 1e-8
        assert O.projector_gap(qi, ref_outputs["orth_q"][:, i * l:(i + 1) * l]) < 1e-12
        assert np.abs(qi.T @ qi - np.eye(l)).max() < 1e-10   # Gram-based: eps * cond(Y_i)^2


@pytest.mark.parametrize("name,kind", KN_CASES)
def test_kn_golden(golden, ref_outputs, name, kind):
    # check/isvd/integrator/kolmogorov_nagumo_integrator.cpp:61-66 (and the row-block variants)
    qbar, it = O.INTEGRATORS[name](golden["qs"], golden["l"], golden["N"], 256, 1e-4)
    assert it == int(golden["qb_kn_iter"]) == 81
    assert np.abs(qbar - golden["qb_kn"]).max() < 1e-8
    assert it == int(ref_outputs["int%d_iter" % kind])
    assert np.abs(qbar - ref_outputs["int%d_qbar" % kind]).max() < 1e-12


@pytest.mark.parametrize("name,kind", WY_CASES)
def test_wy_golden(golden, ref_outputs, name, kind):
    # check/isvd/integrator/row_block_wen_yin_integrator.cpp:69-74
    qbar, it = O.INTEGRATORS[name](golden["qs"], golden["l"], golden["N"], 256, 1e-3)
    assert it == int(golden["qb_wy_iter"]) == 21
    assert np.abs(qbar - golden["qb_wy"]).max() < 1e-8
    assert it == int(ref_outputs["int%d_iter" % kind])
    assert np.abs(qbar - ref_outputs["int%d_qbar" % kind]).max() < 1e-10


@pytest.mark.parametrize("kind,name", [(0, "svd"), (1, "gramian"), (2, "gramian"), (3, "gramian")])
def test_formers_golden(golden, ref_outputs, kind, name):
    # check/isvd/former/svd_former.cpp:56-66 (k = ncol(q)/2 = 5)
    q = golden["q"]
    k = q.shape[1] // 2
    s, u, v = O.FORMERS[name](golden["a"], q, k)
    assert O.projector_gap(u, golden["u"][:, :k]) < 1e-8
    np.testing.assert_allclose(s, ref_outputs["form%d_s" % kind], rtol=1e-12)
    np.testing.assert_allclose(O.align_signs(u, ref_outputs["form%d_u" % kind]), ref_outputs["form%d_u" % kind],
                               atol=1e-12)
    np.testing.assert_allclose(O.align_signs(v, ref_outputs["form%d_v" % kind]), ref_outputs["form%d_v" % kind],
                               atol=1e-12)


@pytest.mark.parametrize("name", list(O.INTEGRATORS))
def test_integrators_maxit_zero(golden, name):
    # max_iteration = 0 runs no iteration: Qbar = Q0 (the loops of all five
    # integrators test the bound before the body).
    qs = golden["qs"]
    l, N = golden["l"], golden["N"]
    qbar, it = O.INTEGRATORS[name](qs, l, N, 0, 1e-4)
    assert it == 0
    np.testing.assert_allclose(qbar, qs[:, :l], atol=1e-14)


def test_live_reference_matches(golden):
    """When the reference checker is built here, run it live on the golden inputs."""
    from oracle import ref_lib
    if not ref_lib.available():
        pytest.skip("oracle/_ref not built (make -C oracle)")
    lib = ref_lib.load()
    qbar, it = ref_lib.integrate(lib, golden["qs"], golden["l"], golden["N"], 0, 256, 1e-4)
    assert it == 81
    assert np.abs(qbar - golden["qb_kn"]).max() < 1e-8


def test_pipeline_small_consistency():
    """Whole-pipeline oracle on a seeded C1-shaped (reduced) problem: the three
    Kolmogorov-Nagumo formulations take the same iterations and agree to
    rounding; the two Wen-Yin formulations likewise (KN and WY are different
    iterations and stop at different points, so they are not compared)."""
    from mcnla_b200 import synthetic
    a, omega = synthetic.config1_numpy(m=200, n=300, k=6, p=6, N=8, seed=3)
    res = {name: O.isvd(a, omega, 6, 6, 8, integrator=name, tol=1e-4) for name in O.INTEGRATORS}
    # the line search makes the Wen-Yin trajectory sensitive to rounding
    for fam, rtol in ((["kn", "rb_kn", "rb_gramian_kn"], 1e-10), (["rb_wy", "rb_gramian_wy"], 1e-7)):
        r0 = res[fam[0]]
        for name in fam[1:]:
            assert res[name]["iterations"] == r0["iterations"]
            np.testing.assert_allclose(res[name]["s"], r0["s"], rtol=rtol)

"""CPU checks of bench.py's measurement arithmetic (no GPU): the per-stage roofline and the
defaults the benchmark contract relies on."""
import sys

import pytest

import bench


def _stages(sketch=0.5, orth=0.008, integ=0.1, form=0.0127, it=256):
    return {"sketch_gemm_s": sketch, "orthogonalize_s": orth, "integrate_s": integ, "integrate_iterations": it,
            "form_s": form}


def test_stage_roofline_c2_figures():
    m, n, k, p, N = 100000, 20000, 50, 14, 64
    l = k + p
    r = bench.stage_rooflines(m, n, k, l, N, "rb_gramian_kn", "rb_gramian", _stages(), 35.0, 6450.0)
    sk = r["sketch"]
    # 2 m n N l flops; A, Omega and Y once
    assert sk["flops"] == 2.0 * m * n * N * l
    assert sk["bytes"] == 8.0 * (m * n + n * N * l + m * N * l)
    assert sk["bound"] == "tensor"
    assert sk["frac"] == pytest.approx(sk["flops"] / 35e12 / 0.5, abs=1e-4)
    for name in ("sketch", "orthogonalize", "integrate", "form"):
        assert 0.0 < r[name]["frac"] < 2.0
        assert r[name]["achieved_tflops"] == pytest.approx(r[name]["flops"] / r[name]["s"] / 1e12, rel=1e-3)


def test_stage_roofline_bound_switches_to_hbm():
    # a thin sketch (small N l) is HBM bound: A's bytes dominate its flops at the FP64 ridge
    r = bench.stage_rooflines(100000, 20000, 2, 2, 1, "kn", "svd", _stages(sketch=0.3, it=10), 35.0, 6450.0)
    assert r["sketch"]["bound"] == "hbm"
    assert r["sketch"]["frac"] == pytest.approx(r["sketch"]["bytes"] / 6450e9 / 0.3, abs=1e-4)   # rounded to 4 places


@pytest.mark.parametrize("integrator", ["kn", "rb_kn", "rb_gramian_kn", "rb_wy", "rb_gramian_wy"])
def test_stage_roofline_every_integrator(integrator):
    r = bench.stage_rooflines(1000, 2000, 10, 20, 16, integrator, "svd", _stages(it=81), 35.0, 6450.0)
    assert r["integrate"]["flops"] > 0


def test_default_arguments_follow_the_contract(monkeypatch):
    monkeypatch.setattr(sys, "argv", ["bench.py"])
    a = bench.parse()
    assert a.gpus == 1 and a.warmup >= 3 and a.steps >= 1
    assert (a.m, a.n, a.k, a.p, a.N) == (100000, 20000, 50, 14, 64)
    w = bench.workload(a)
    assert "m=100000" in w["workload"] and w["sketch_gemm"] == "100000x20000x4096"


def test_svd_metrics_against_a_known_rotation():
    """The accuracy report of the precision-form legs: sigma relative error, largest principal
    angle of U, ||U'U - I||_F, on a case with known answers."""
    import numpy as np
    rng = np.random.default_rng(0)
    q, _ = np.linalg.qr(rng.standard_normal((50, 4)))
    s_ref = np.array([4.0, 3.0, 2.0, 1.0])
    theta = 1e-3
    rot = np.eye(4)
    rot[0, 0] = rot[1, 1] = np.cos(theta)
    rot[0, 1], rot[1, 0] = -np.sin(theta), np.sin(theta)
    # the same subspace (a rotation within it) with the last column tilted out of it by theta
    u = q @ rot
    out, _ = np.linalg.qr(np.concatenate([q, rng.standard_normal((50, 1))], axis=1))
    u[:, 3] = np.cos(theta) * q[:, 3] + np.sin(theta) * out[:, 4]
    m = bench._svd_metrics(s_ref * (1 + 1e-7), u, s_ref, q)
    assert abs(m["sigma_rel_err"] - 1e-7) < 1e-12
    assert abs(m["max_principal_angle_U"] - theta) < 1e-9
    assert m["UtU_minus_I_fro"] < 1e-12


def test_reference_arm_default_budget_is_minutes(monkeypatch):
    """The reference arm times whole solves of the full matrix until its budget (seconds) would be
    exceeded: a few minutes by default."""
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference"])
    a = bench.parse()
    assert 60 <= a.ref_budget <= 600

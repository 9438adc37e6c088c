"""GPU parity on the code paths the benchmark itself runs.

The benchmark's integrator is the row-block Gramian Kolmogorov-Nagumo integrator at
N l = 4096 with the default step method: above N l = 1536 that is the launch-per-product
loop (not the persistent kernel) with the power-series KN step, replayed as a captured
CUDA graph per chunk of iterations.  These tests run exactly that path against the CPU
oracle and against the reference's own stages compiled here (oracle/_ref), and then the
benchmark configuration's own parameters (k = 50, p = 14, N = 64, tol 1e-6, sigma_j =
exp(-j/30) plus 1e-4 noise) at a reduced row count, in both layouts of A.

Tolerances as in test_gpu_parity: singular values to 1e-10 relative, singular vectors
to 1e-10 up to column sign, identical iteration counts.
"""
import numpy as np
import pytest
import torch

from oracle import isvd_oracle as O
from oracle import ref_lib

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _dev(x, cuda):
    return torch.as_tensor(np.ascontiguousarray(x), dtype=torch.float64, device=cuda)


def _solve(cuda, a, omega, k, p, N, integrator, former, tol, colmajor=False, maxit=256):
    from mcnla_b200 import isvd
    at = _dev(a.T, cuda).t() if colmajor else _dev(a, cuda)
    s, u, v, it = isvd.solve(at, k, p, N, omega=_dev(omega, cuda), integrator=integrator, former=former, tol=tol,
                             maxit=maxit)
    return s.cpu().numpy(), u.cpu().numpy(), v.cpu().numpy(), it


def _ref(a, omega, k, p, N, integrator, former, tol, colmajor=False, maxit=256):
    """The reference's own stages (oracle/_ref): sketch -> RB Gramian orthogonalizer -> integrator -> former."""
    lib = ref_lib.load()
    kinds = {"kn": 0, "rb_kn": 1, "rb_gramian_kn": 2, "rb_wy": 3, "rb_gramian_wy": 4}
    fkinds = {"svd": 0, "gramian": 1, "rb_gramian": 2, "cb_gramian": 3}
    sol = ref_lib.Solver(lib, a, omega, k, p, N, kinds[integrator], fkinds[former], maxit, tol, colmajor=colmajor)
    it, _ = sol.run()
    s, u, v = sol.result()
    sol.close()
    return s, u, v, it


def _close(got, ref, tol=TOL):
    s, u, v, it = got
    rs, ru, rv, rit = ref
    assert it == rit, (it, rit)
    np.testing.assert_allclose(s, rs, rtol=tol)
    assert np.abs(O.align_signs(u, ru) - ru).max() < tol
    assert np.abs(O.align_signs(v, rv) - rv).max() < tol


def test_gramian_kn_launch_loop_with_graph_replay_matches_oracle(cuda):
    """N l = 1600 > 1536: the launch-per-product loop with the series step and graph replay
    (the benchmark's path), against the numpy oracle and the compiled reference."""
    from mcnla_b200 import isvd, synthetic
    m, n, k, p, N = 3000, 2000, 20, 12, 50
    a = synthetic.lowrank_np(m, n, 1.0 / np.arange(1, min(m, n) + 1), seed=4)
    omega = np.random.default_rng(9).standard_normal((n, (k + p) * N))
    ctx = isvd.context(cuda)
    ctx.set_kn_method(0)
    r0 = ctx.graph_replays()
    got = _solve(cuda, a, omega, k, p, N, "rb_gramian_kn", "rb_gramian", 1e-5)
    assert ctx.graph_replays() > r0, "the iteration loop did not replay a captured graph"
    assert got[3] > 24
    orc = O.isvd(a, omega, k, p, N, integrator="rb_gramian_kn", former="gramian", tol=1e-5)
    _close(got, (orc["s"], orc["u"], orc["v"], orc["iterations"]))
    if ref_lib.available():
        _close(got, _ref(a, omega, k, p, N, "rb_gramian_kn", "rb_gramian", 1e-5))


def _config2_reduced(m=8192, n=20000, r=200, seed=21):
    from mcnla_b200 import synthetic
    a = synthetic.lowrank_np(m, n, np.exp(-np.arange(1, r + 1) / 30.0), seed=seed, noise=1e-4)
    omega = np.random.default_rng(seed + 1).standard_normal((n, 64 * 64))
    return a, omega


@pytest.mark.skipif(not ref_lib.available(), reason="oracle/_ref (the compiled reference) is not built")
@pytest.mark.parametrize("colmajor,former", [(False, "rb_gramian"), (True, "cb_gramian")])
def test_config2_parameters_match_the_reference(cuda, colmajor, former):
    """The benchmark configuration's parameters (k = 50, p = 14, N = 64: sketch 8192 x 20000 x
    4096; RB Gramian KN, tol 1e-6, maxit 256) on an 8192-row matrix with its spectrum and noise,
    row-major A with the row-block former and column-major A with the column-block former,
    against the reference's own stages.  Both stop at the same iteration (at this tolerance
    both run to maxit: the stopping quantity sits above 1e-6)."""
    a, omega = _config2_reduced()
    got = _solve(cuda, a, omega, 50, 14, 64, "rb_gramian_kn", former, 1e-6, colmajor=colmajor)
    ref = _ref(a, omega, 50, 14, 64, "rb_gramian_kn", former, 1e-6, colmajor=colmajor)
    _close(got, ref)

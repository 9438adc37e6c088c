"""The grouped batch (mcnla_b200_isvd_grouped): row-block Gramian Kolmogorov-Nagumo problems of
uneven sizes go through the workers' sketch / orthogonalizer / Gramian phase, one grouped
persistent kernel for every problem's iterations (a cluster of CTAs per problem from a device
work queue; the iterations the power series declines run on the workers in between), and the
workers' Qbar / former phase.  Every stage but the iterations is the single solve's own; the
grouped kernel sums its products in a fixed order of its own, so each result must match
mcnla_b200_isvd / mcnla_b200_isvd_mixed to 1e-10 (sigma relative, singular vectors up to sign)
with the same iteration count, be the same bits in any batch, and the FP64 ones must match the
CPU oracle to 1e-10 with identical iteration counts."""
import numpy as np
import pytest
import torch

from oracle import isvd_oracle as O

pytestmark = pytest.mark.gpu


def _problems(cuda, count, seed, ks=(4, 8, 16, 32), mixed_every=3):
    from mcnla_b200 import isvd, synthetic
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(count):
        m, n = int(rng.integers(300, 3000)), int(rng.integers(200, 1500))
        k = int(rng.choice(ks))
        p, N = k // 2, int(rng.choice([4, 8]))
        alpha = rng.uniform(0.5, 2.0)
        a = synthetic.lowrank_np(m, n, np.arange(1, min(m, n) + 1) ** -alpha, seed=300 + i)
        at = torch.as_tensor(a, device=cuda).to(torch.float32 if i % 2 else torch.float64)
        if i % 4 == 3:
            at = at.t().contiguous().t()          # column-major
        mixed = (False, False, 3, True)[i % mixed_every] if mixed_every else False
        former = ["rb_gramian", "svd", "gramian", "cb_gramian"][i % 4]
        reqs.append(isvd.Request(at, k, p, N, seed=2000 + i, integrator="rb_gramian_kn", former=former, tol=1e-5,
                                 mixed=mixed))
    return reqs


def _alone(req):
    from mcnla_b200 import isvd
    pr = req.problem
    a = req.a if req.a.dtype == torch.float64 else req.a.double()
    former = {v: k for k, v in isvd.FORMERS.items()}[pr.former]
    args = dict(seed=pr.seed, integrator="rb_gramian_kn", former=former, maxit=pr.max_iteration, tol=pr.tolerance)
    k, p, N = pr.params.rank, pr.params.over_rank, pr.params.num_sketch
    if pr.precision in (1, 2):
        return isvd.solve_mixed(a, k, p, N, parts=pr.precision + 1, former_split=isvd.split_bf16(a.t(), 3), **args)
    return isvd.solve(a, k, p, N, **args)


def _close(got, ref, tol=1e-10):
    s, u, v = (x.cpu().numpy() for x in got)
    rs, ru, rv = (x.cpu().numpy() for x in ref)
    np.testing.assert_allclose(s, rs, rtol=tol)
    assert np.abs(O.align_signs(u, ru) - ru).max() < tol
    assert np.abs(O.align_signs(v, rv) - rv).max() < tol


def test_grouped_batch_matches_single_solves(cuda):
    from mcnla_b200 import isvd
    reqs = _problems(cuda, 24, seed=7)
    isvd.solve_grouped(reqs, workers=4)
    first = [(r.s.clone(), r.u.clone(), r.v.clone(), r.result.iteration) for r in reqs]
    for r in reqs:
        assert r.result.status == 0
        s, u, v, it = _alone(r)
        assert it == r.result.iteration, (it, r.result.iteration)
        _close((r.s, r.u, r.v), (s, u, v))
    # the same problems in another batch (other neighbours, other order): the same bits
    again = list(reversed(reqs[:10]))
    for r in again:
        r.s.zero_()
    isvd.solve_grouped(again, workers=3)
    for r in again:
        s0, u0, v0, it0 = first[reqs.index(r)]
        assert r.result.iteration == it0
        assert torch.equal(r.s, s0) and torch.equal(r.u, u0) and torch.equal(r.v, v0)


def test_grouped_batch_matches_the_oracle(cuda):
    from mcnla_b200 import isvd
    reqs = _problems(cuda, 6, seed=11, mixed_every=0)
    isvd.solve_grouped(reqs, workers=3)
    for r in reqs:
        pr = r.problem
        k, p, N = pr.params.rank, pr.params.over_rank, pr.params.num_sketch
        m, n = pr.params.nrow, pr.params.ncol
        L = (k + p) * N
        om = torch.empty(n * L, dtype=torch.float64, device=cuda)
        ctx = isvd.context(cuda)
        from mcnla_b200 import _lib
        import ctypes
        _lib.check(ctx.lib.mcnla_b200_gaussian(ctx.bind(), ctypes.c_uint64(pr.seed), n * L,
                                               ctypes.c_void_p(om.data_ptr())), "gaussian")
        a = r.a.double().cpu().numpy()
        former = "svd" if pr.former == 0 else "gramian"
        ref = O.isvd(a, om.view(n, L).cpu().numpy(), k, p, N, integrator="rb_gramian_kn", former=former, tol=1e-5)
        assert r.result.iteration == ref["iterations"]
        np.testing.assert_allclose(r.s.cpu().numpy(), ref["s"], rtol=1e-10)
        assert np.abs(O.align_signs(r.u.cpu().numpy(), ref["u"]) - ref["u"]).max() < 1e-10
        assert np.abs(O.align_signs(r.v.cpu().numpy(), ref["v"]) - ref["v"]).max() < 1e-10


def test_grouped_batch_waves_and_other_integrators(cuda):
    """A budget that holds a few problems at a time (several waves), and problems the grouped
    kernel does not take (other integrators) in the same batch: every result equals its single
    solve."""
    from mcnla_b200 import isvd, synthetic
    reqs = _problems(cuda, 10, seed=13)
    for i, integ in enumerate(["kn", "rb_kn", "rb_gramian_wy"]):
        a = torch.as_tensor(synthetic.lowrank_np(700 + i, 400, np.arange(1, 401) ** -1.0, seed=i), device=cuda)
        reqs.append(isvd.Request(a, 8, 4, 4, seed=99 + i, integrator=integ, former="svd", tol=1e-4))
    budget = 3 * max(r.bytes() for r in reqs)
    isvd.solve_grouped(reqs, workers=3, budget_bytes=budget)
    for r in reqs:
        assert r.result.status == 0
        pr = r.problem
        if pr.integrator == isvd.INTEGRATORS["rb_gramian_kn"]:
            s, u, v, it = _alone(r)
            assert it == r.result.iteration
            _close((r.s, r.u, r.v), (s, u, v))
        else:                           # whole solves on the workers: the single solve's bits
            integ = {v_: k_ for k_, v_ in isvd.INTEGRATORS.items()}[pr.integrator]
            s, u, v, it = isvd.solve(r.a, pr.params.rank, pr.params.over_rank, pr.params.num_sketch, seed=pr.seed,
                                     integrator=integ, former="svd", tol=pr.tolerance)
            assert it == r.result.iteration
            assert torch.equal(s, r.s) and torch.equal(u, r.u)

"""Batched and served solves (mcnla_b200_isvd_batched / mcnla_b200_server_*):
many uneven problems run concurrently on one GPU, and each result is the same
alone and in the mix (bit for bit: every kernel reduces in a fixed order).  The
grouped batch (mcnla_b200_isvd_grouped) is covered by test_gpu_grouped.py."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _problems(cuda, count=10, seed=0):
    from mcnla_b200 import isvd, synthetic
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(count):
        m, n = int(rng.integers(300, 3000)), int(rng.integers(200, 1500))
        k = int(rng.choice([4, 8, 16]))
        p, N = k // 2, 4
        alpha = rng.uniform(0.5, 2.0)
        a = synthetic.lowrank_np(m, n, np.arange(1, min(m, n, 200) + 1) ** -alpha, seed=100 + i)
        dtype = torch.float32 if i % 3 == 2 else torch.float64
        at = torch.as_tensor(a, device=cuda).to(dtype)
        if i % 4 == 3:
            at = at.t().contiguous().t()          # column-major
        mixed = (False, True, False, 3)[i % 4]
        integ = ["kn", "rb_gramian_kn", "rb_gramian_wy", "rb_kn"][i % 4]
        reqs.append(isvd.Request(at, k, p, N, seed=1000 + i, integrator=integ, former="svd", tol=1e-5,
                                 mixed=mixed))
    return reqs


def _alone(req):
    from mcnla_b200 import isvd
    pr = req.problem
    a = req.a if req.a.dtype == torch.float64 else req.a.double()
    integ = {v: k for k, v in isvd.INTEGRATORS.items()}[pr.integrator]
    args = dict(seed=pr.seed, integrator=integ, former="svd", maxit=pr.max_iteration, tol=pr.tolerance)
    k, p, N = pr.params.rank, pr.params.over_rank, pr.params.num_sketch
    if pr.precision in (1, 2):
        # the served mixed solve: the precision former from three BF16 parts of A'
        return isvd.solve_mixed(a, k, p, N, parts=pr.precision + 1, former_split=isvd.split_bf16(a.t(), 3), **args)
    return isvd.solve(a, k, p, N, **args)


def test_batched_results_equal_alone(cuda):
    from mcnla_b200 import isvd
    reqs = _problems(cuda)
    isvd.solve_batched(reqs, workers=4)
    for r in reqs:
        assert r.result.status == 0
        assert r.result.seconds > 0
        s, u, v, it = _alone(r)
        assert it == r.result.iteration
        assert torch.equal(s, r.s), (s - r.s).abs().max().item()
        assert torch.equal(u, r.u)
        assert torch.equal(v, r.v)


def test_server_overlapping_submissions_and_admission(cuda):
    from mcnla_b200 import isvd
    reqs = _problems(cuda, 8, seed=1)
    single = max(r.bytes() for r in reqs)
    # a budget below any single problem: problems run one at a time
    with isvd.Server(workers=4, budget_bytes=1) as srv:
        for r in reqs:
            srv.submit(r)
        for r in reqs:
            srv.wait(r)
        st = srv.stats()
    assert st["completed"] == len(reqs)
    assert st["peak_bytes"] <= single
    serial = [r.s.clone() for r in reqs]
    # a large budget: problems overlap on the device and give the same results
    with isvd.Server(workers=4, budget_bytes=150 << 30) as srv:
        for r in reqs:
            srv.submit(r)
        for r in reqs:
            srv.wait(r)
        st = srv.stats()
    assert st["peak_bytes"] > single
    for r, s0 in zip(reqs, serial):
        assert torch.equal(r.s, s0)


def test_server_reports_bad_problem_and_continues(cuda):
    from mcnla_b200 import isvd, _lib
    reqs = _problems(cuda, 3, seed=2)
    bad = _problems(cuda, 1, seed=3)[0]
    bad.problem.params.over_rank = 500                  # l > 160
    with isvd.Server(workers=2) as srv:
        srv.submit(bad)
        for r in reqs:
            srv.submit(r)
        with pytest.raises(_lib.McnlaError):
            srv.wait(bad)
        for r in reqs:
            srv.wait(r)
            assert r.result.status == 0


def test_server_tight_budget_with_held_workspaces(cuda):
    """A budget of about two large problems and six workers: the workers that served the large
    problems keep their workspaces between solves, and those workspaces count against the budget,
    so the queue head can find them in its way; the idle workers then release them.  Every
    problem completes, and each result is the same bits as with an ample budget."""
    from mcnla_b200 import isvd, synthetic
    small = _problems(cuda, 12, seed=5)
    rng = np.random.default_rng(9)
    big = []
    for i in range(3):
        a = torch.as_tensor(synthetic.lowrank_np(6000, 2500, np.arange(1, 2501) ** -1.0, seed=70 + i), device=cuda)
        big.append(isvd.Request(a, 48, 24, 8, seed=int(rng.integers(1 << 30)), integrator="rb_gramian_kn",
                                former="svd", tol=1e-5))
    reqs = big[:1] + small[:4] + big[1:2] + small[4:8] + big[2:] + small[8:]
    budget = 2 * max(r.bytes() for r in reqs) + max(r.bytes() for r in small)
    with isvd.Server(workers=6, budget_bytes=budget) as srv:
        for r in reqs:
            srv.submit(r)
        for r in reqs:
            srv.wait(r)
    tight = [(r.s.clone(), r.u.clone(), r.result.iteration) for r in reqs]
    for r in reqs:
        assert r.result.status == 0
    with isvd.Server(workers=6, budget_bytes=150 << 30) as srv:
        for r in reqs:
            srv.submit(r)
        for r in reqs:
            srv.wait(r)
    for r, (s0, u0, it0) in zip(reqs, tight):
        assert r.result.iteration == it0
        assert torch.equal(r.s, s0) and torch.equal(r.u, u0)

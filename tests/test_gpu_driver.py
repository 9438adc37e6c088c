"""The command-line driver (python -m mcnla_b200.isvd_dense), the reference's isvd_dense_rb /
isvd_dense_cb: A from a file, S, U, V written as the reference writes them, and the drivers'
||A - U S V'||_F / ||A||_F check.  The files it writes must hold the solve of the library on the
same A and Omega (the seeded Omega of the driver), bit for bit."""
import os
import subprocess
import sys

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("layout,binary", [("rb", False), ("cb", False), ("rb", True)])
def test_driver_writes_the_solve(cuda, tmp_path, golden, layout, binary):
    from mcnla_b200 import io, isvd, synthetic
    a = golden["a"]                                    # the reference's data/a.mtx (101 x 1001)
    m, n = a.shape
    k, p, N, seed = 5, 3, 4, 11
    src = tmp_path / ("a.bin" if binary else "a.mtx")
    if binary:
        io.save_binary(src, a)
    else:
        io.save_matrix_market(src, a)
    out = [str(tmp_path / x) for x in ("s.mtx", "u.mtx", "v.mtx")]
    cmd = [sys.executable, "-m", "mcnla_b200.isvd_dense", str(src), *out, str(N), str(k), str(p), "1e-4", "256",
           "--layout", layout, "--integrator", "rb_gramian_kn", "--seed", str(seed)] + (["--binary"] if binary else [])
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stdout + r.stderr
    s, u, v = (io.load_matrix_market(f) for f in out)
    omega = synthetic.omega_torch(n, (k + p) * N, seed=seed, device=cuda)
    at = torch.as_tensor(a, device=cuda)
    if layout == "cb":
        at = at.t().contiguous().t()
    s1, u1, v1, it = isvd.solve(at, k, p, N, omega=omega, integrator="rb_gramian_kn",
                                former="cb_gramian" if layout == "cb" else "rb_gramian", tol=1e-4)
    assert np.array_equal(s.ravel(), s1.cpu().numpy())
    assert np.array_equal(u, u1.cpu().numpy()) and np.array_equal(v, v1.cpu().numpy())
    assert "Iteration = %d" % it in r.stdout
    err = np.linalg.norm(a - (u * s.ravel()) @ v.T) / np.linalg.norm(a)
    line = [x for x in r.stdout.splitlines() if x.startswith("Error     = ")][0]
    assert abs(float(line.split("=")[1]) - err) <= 1e-6 * err          # printed with 7 digits, as the reference prints it

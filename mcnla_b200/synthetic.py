"""Seeded synthetic test matrices with prescribed spectra (the reference's demo
generator idea, demo/demo.cpp:250-283: A = U diag(sigma) V' from the Q factors
of Gaussian matrices).  There is no public dataset for this path; the shapes,
spectra and noise levels are the ones the benchmark configurations name.

numpy versions (CPU, float64, numpy PCG64 seeds) feed parity tests; torch
versions build the large matrices directly on the GPU for the benchmark.
"""
import numpy as np


# ----------------------------------------------------------------------------------------------
# numpy (CPU)
# ----------------------------------------------------------------------------------------------
def _orth_np(rng, rows, cols):
    q, _ = np.linalg.qr(rng.standard_normal((rows, cols)))
    return q


def lowrank_np(m, n, sigma, seed=0, noise=0.0):
    """A = U diag(sigma) V' (+ noise * G), U m x r, V n x r orthonormal."""
    rng = np.random.default_rng(seed)
    r = len(sigma)
    u = _orth_np(rng, m, r)
    v = _orth_np(rng, n, r)
    a = (u * sigma) @ v.T
    if noise:
        a += noise * rng.standard_normal((m, n))
    return a


def omega_np(n, L, seed=0):
    return np.random.default_rng(seed).standard_normal((n, L))


def config1_numpy(m=1000, n=2000, k=10, p=10, N=16, seed=0):
    """Plain-iSVD configuration: sigma_j = 1/j, j = 1..min(m, n); Omega N(0,1) from the seed."""
    r = min(m, n)
    sigma = 1.0 / np.arange(1, r + 1)
    a = lowrank_np(m, n, sigma, seed=seed)
    return a, omega_np(n, (k + p) * N, seed=seed)


def config2_sigma(r=200):
    return np.exp(-np.arange(1, r + 1) / 30.0)


def config3_sigma(r=200):
    return 10.0 ** (-6.0 * np.arange(r) / (r - 1))


# ----------------------------------------------------------------------------------------------
# torch (GPU)
# ----------------------------------------------------------------------------------------------
def lowrank_torch(m, n, sigma, seed=0, noise=0.0, device="cuda", colmajor=False, chunk_rows=8192, dtype=None):
    """A = U_r diag(sigma) V_r' + noise * G on the device, float64 (or `dtype`).

    U_r, V_r come from QR of seeded Gaussians; G is i.i.d. N(0,1).  Built in
    row chunks so the temporaries stay small next to A.  colmajor=True returns
    the m x n column-major view (transpose of a contiguous n x m buffer).
    """
    import torch
    dt = torch.float64 if dtype is None else dtype
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    sig = torch.as_tensor(np.asarray(sigma, dtype=np.float64), device=device).to(dt)
    r = sig.numel()
    u, _ = torch.linalg.qr(torch.randn(m, r, generator=g, dtype=dt, device=device))
    v, _ = torch.linalg.qr(torch.randn(n, r, generator=g, dtype=dt, device=device))
    us = u * sig
    if colmajor:
        at = torch.empty(n, m, dtype=dt, device=device)
        for c0 in range(0, m, chunk_rows):
            c1 = min(m, c0 + chunk_rows)
            blk = v @ us[c0:c1].T
            if noise:
                blk += noise * torch.randn(n, c1 - c0, generator=g, dtype=dt, device=device)
            at[:, c0:c1] = blk
        del u, v, us
        return at.t()
    a = torch.empty(m, n, dtype=dt, device=device)
    for r0 in range(0, m, chunk_rows):
        r1 = min(m, r0 + chunk_rows)
        a[r0:r1] = us[r0:r1] @ v.T
        if noise:
            a[r0:r1] += noise * torch.randn(r1 - r0, n, generator=g, dtype=dt, device=device)
    del u, v, us
    return a


def omega_torch(n, L, seed=0, device="cuda"):
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(int(seed) + 7919)
    return torch.randn(n, L, generator=g, dtype=torch.float64, device=device)


# ----------------------------------------------------------------------------------------------
# uneven batches and served requests
# ----------------------------------------------------------------------------------------------
def batch_shapes(count, seed=0, r_max=None):
    """`count` uneven problems: m ~ U[512, 16384], n ~ U[256, 4096], k in {8, 16, 32, 64},
    p = k / 2, N = 8, sigma_j = j^-alpha with alpha ~ U[0.5, 2] over the whole spectrum,
    j = 1 .. min(m, n) (r_max, when given, cuts it shorter)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        m = int(rng.integers(512, 16385))
        n = int(rng.integers(256, 4097))
        k = int(rng.choice([8, 16, 32, 64]))
        alpha = float(rng.uniform(0.5, 2.0))
        r = min(m, n) if r_max is None else min(m, n, r_max)
        out.append({"m": m, "n": n, "k": k, "p": k // 2, "N": 8, "alpha": alpha,
                    "sigma": np.arange(1, r + 1, dtype=np.float64) ** -alpha, "seed": int(seed) * 100003 + i})
    return out


def large_shape(seed=0, r_max=None):
    """The large served request: m = 65536, n = 8192, k = 128, p = 32, N = 16, sigma_j = j^-alpha
    over the whole spectrum (j = 1 .. 8192; r_max, when given, cuts it shorter)."""
    rng = np.random.default_rng(seed)
    alpha = float(rng.uniform(0.5, 2.0))
    r = 8192 if r_max is None else min(8192, r_max)
    return {"m": 65536, "n": 8192, "k": 128, "p": 32, "N": 16, "alpha": alpha,
            "sigma": np.arange(1, r + 1, dtype=np.float64) ** -alpha, "seed": int(seed) * 100003 + 99991}

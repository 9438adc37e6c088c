"""CPU restatement of MCNLA's iSVD hot path, in numpy (float64).

TEST INFRASTRUCTURE ONLY.  This module is the checker the CUDA path is compared
with; it is imported by ``tests/``, by ``__graft_entry__.smoke()`` and by the
CPU-baseline leg of ``bench.py``, and never by the product package.

Each function restates one reference stage, step for step, citing the
reference file:line it follows (paths relative to the reference project root,
MCNLA 0.7.2).  Conventions match the reference's storage:

* A is m x n; Omega is n x (N*l).
* The sketch collection is "unfolded": one row-major m x (N*l) array whose
  column block i is sketch i
  (include/mcnla/core/matrix/collection/dense/dense_matrix_collection_col_block.hpp:44-55).
* Q-bar is m x l; U is m x k; V is n x k; S holds the k leading singular values.

``syev`` is ``numpy.linalg.eigh`` (ascending eigenvalues, eigenvectors as
columns; the reference's row-major call sees them as rows, hence the
transposes below); ``gesvd`` is ``numpy.linalg.svd``; ``getrfi`` (LU + inverse)
is ``numpy.linalg.inv``.  Only results that are invariant under the sign and
basis freedom of those factorizations are compared elsewhere.

Pinning: ``tests/test_oracle_golden.py`` checks this module against the
reference's own golden fixtures (data/qi.mtx, qb_kn.mtx, qb_wy.mtx, q.mtx,
u.mtx, yi.mtx) and against the reference's own stages compiled here
(``oracle/_ref``) on the same inputs.
"""
import numpy as np

# Wen-Yin line-search constants, include/mcnla/isvd/integrator/row_block_wen_yin_integrator.hh:76-94
WY_TAU0, WY_TAUMAX, WY_TAUMIN, WY_TAUMAXITER = 1.0, 1e14, 1e-14, 20
WY_BETA, WY_SIGMA, WY_ETA = 0.5, 1e-4, 0.85


def _blocks(qs, l, N):
    return [qs[:, i * l:(i + 1) * l] for i in range(N)]


def _nrm2_converged(v, tol):
    # is_converged = !(nrm2(e - 1) >= tol): a NaN norm counts as converged
    # (kolmogorov_nagumo_integrator.hpp:181).
    return not (np.linalg.norm(v) >= tol)


def _kn_c_cinv(z):
    """C and inv(C) from the symmetric Z, as in the KN integrators.

    eig(Z) = Z' S Z (syev, ascending); s := sqrt(1/2 + sqrt(1/4 - s));
    C = Z' S Z, inv(C) = Z' inv(S) Z.  Returns (C, inv(C), s).
    row_block_kolmogorov_nagumo_integrator.hpp:150-171.
    """
    lam, vec = np.linalg.eigh(z, UPLO="L")
    with np.errstate(invalid="ignore"):
        s = np.sqrt(0.5 + np.sqrt(0.25 - lam))
    ss = np.sqrt(s)
    zr = vec.T                          # rows are eigenvectors (row-major view)
    sz = ss[:, None] * zr
    sinvz = zr / ss[:, None]
    c = sz.T @ sz
    cinv = sinvz.T @ sinvz
    return c, cinv, s


# --------------------------------------------------------------------------------------------
# Sketch
# --------------------------------------------------------------------------------------------
def sketch(a, omega):
    """Q := A * Omega on the unfolded collection.

    include/mcnla/isvd/sketcher/gaussian_projection_sketcher.hpp:96 (same GEMM in
    row_block_gaussian_projection_sketcher.hpp:104 and col_block_...:92).
    """
    return a @ omega


def sketch_power(a, omega, exponent):
    """Power iterations of the plain sketcher: Omega := A' Q; Q := A Omega.

    gaussian_projection_sketcher.hpp:96-100.
    """
    q = a @ omega
    for _ in range(exponent):
        omega = a.T @ q
        q = a @ omega
    return q


# --------------------------------------------------------------------------------------------
# Orthogonalizer
# --------------------------------------------------------------------------------------------
def orthogonalize_gramian(y, l, N):
    """Gramian orthogonalizer (plain and row-block give the same result on one rank).

    include/mcnla/isvd/orthogonalizer/gramian_orthogonalizer.hpp:84-101:
      W_i := Y_i' Y_i; gesvd<'N','O'>(W_i) -> s (descending), W_i := V'
      s := sqrt(s); W_i := diag(1/s) W_i; Q_i := Y_i W_i'.
    """
    q = np.empty_like(y)
    for i, yi in enumerate(_blocks(y, l, N)):
        w = yi.T @ yi
        _, s, vt = np.linalg.svd(w)
        s = np.sqrt(s)
        w = vt / s[:, None]
        q[:, i * l:(i + 1) * l] = yi @ w.T
    return q


# --------------------------------------------------------------------------------------------
# Integrators
# --------------------------------------------------------------------------------------------
def integrate_kn(qs, l, N, maxit=256, tol=1e-4):
    """Kolmogorov-Nagumo integrator.

    include/mcnla/isvd/integrator/kolmogorov_nagumo_integrator.hpp:105-181.
    Returns (Qbar, iterations).
    """
    qc = qs[:, :l].copy()                                   # :105
    it = 0
    converged = False
    while it < maxit and not converged:                     # :116
        b = qs.T @ qc                                       # :117
        d = b.T @ b                                         # :123
        x = (qs @ b) / N                                    # :126
        x -= (qc @ d) / N                                   # :129
        z = x.T @ x                                         # :143
        lam, vec = np.linalg.eigh(z, UPLO="L")              # :146
        with np.errstate(invalid="ignore"):
            e = np.sqrt(0.5 + np.sqrt(0.25 - lam))          # :150-153
        f = np.sqrt(e)
        zr = vec.T
        dd = f[:, None] * zr                                # :155
        zr = zr / f[:, None]                                # :158
        c = dd.T @ dd                                       # :161
        cinv = zr.T @ zr                                    # :164
        qc = qc @ c + x @ cinv                              # :170-171
        converged = _nrm2_converged(e - 1.0, tol)           # :174-181
        it += 1
    return qc, it


def integrate_rb_kn(qs, l, N, maxit=256, tol=1e-4):
    """Row-block Kolmogorov-Nagumo integrator (tracks B = Qs' Qc instead of X).

    include/mcnla/isvd/integrator/row_block_kolmogorov_nagumo_integrator.hpp:110-205.
    """
    qc = qs[:, :l].copy()                                   # :110
    bc = qs.T @ qc                                          # :113
    it = 0
    converged = False
    while it < maxit and not converged:                     # :124
        gc = (qs @ bc) / N                                  # :138
        bgc = qs.T @ gc                                     # :141
        dc = (bc.T @ bc) / N                                # :147
        z = (bc.T @ bgc) / N                                # :150
        z = z - dc @ dc.T                                   # :156
        c, cinv, s = _kn_c_cinv(z)                          # :159-180
        fc = c - dc @ cinv                                  # :186
        qc = qc @ fc + gc @ cinv                            # :189-190
        bc = bc @ fc + bgc @ cinv                           # :193-194
        converged = _nrm2_converged(s - 1.0, tol)           # :198-201
        it += 1
    return qc, it


def _gramian_bs(qs, l):
    """Bs := Qs' Qs as the reference builds it: lower triangle from syrk after
    zeroing the first l rows, so Bc := Bs(:, 0:l) has the strict upper triangle
    of its leading l x l block (Q0' Q0 ~ I there) equal to zero.
    row_block_gramian_kolmogorov_nagumo_integrator.hpp:112-125.
    Returns (Bs as a full symmetric matrix from its lower triangle, Bc).
    """
    full = qs.T @ qs
    low = np.tril(full)
    bs = low + np.tril(full, -1).T
    bc = low[:, :l].copy()
    return bs, bc


def integrate_rb_gramian_kn(qs, l, N, maxit=256, tol=1e-4, history=None):
    """Row-block Gramian Kolmogorov-Nagumo integrator (iterates on Bs only).

    include/mcnla/isvd/integrator/row_block_gramian_kolmogorov_nagumo_integrator.hpp:112-226.
    history: an optional list that receives the stopping quantity ||s - 1||_2 of every iteration.
    """
    L = qs.shape[1]
    bs, bc = _gramian_bs(qs, l)                             # :112-125
    ff = np.eye(l)                                          # :127-133
    ee = np.zeros((L, l))
    it = 0
    converged = False
    while it < maxit and not converged:                     # :138
        bgc = (bs @ bc) / N                                 # :152
        dc = (bc.T @ bc) / N                                # :155
        z = (bc.T @ bgc) / N                                # :158
        z = z - dc @ dc.T                                   # :164
        c, cinv, s = _kn_c_cinv(z)                          # :167-185
        fc = c - dc @ cinv                                  # :188
        ec = (bc @ cinv) / N                                # :194
        ff_new = ff @ fc                                    # :197
        ee = ee @ fc + ec                                   # :200
        ff = ff_new
        bc = bc @ fc + bgc @ cinv                           # :203-204
        converged = _nrm2_converged(s - 1.0, tol)           # :207-214
        if history is not None:
            history.append(float(np.linalg.norm(s - 1.0)))
        it += 1
    qbar = qs[:, :l] @ ff + qs @ ee                         # :225-226
    return qbar, it


def _wy_step(dc, dgc, bc, bgc, tau, l):
    """One trial of the Wen-Yin curvilinear step.

    C := [Dc/2 - I/tau, I/2; -Dgc/2, -Dc/2 - I/tau]; inv(C) (getrfi);
    [Fgc; Fc] := inv(C)(:, l:2l) Dc - inv(C)(:, 0:l); Fc += I; B+ := Bc Fc + Bgc Fgc.
    row_block_wen_yin_integrator.hpp:176-204.
    """
    eye = np.eye(l)
    cm = np.zeros((2 * l, 2 * l))
    cm[:l, :l] = 0.5 * dc - eye / tau
    cm[:l, l:] = 0.5 * eye
    cm[l:, :l] = -0.5 * dgc
    cm[l:, l:] = -0.5 * dc - eye / tau
    ci = np.linalg.inv(cm)
    t = ci[:, l:] @ dc - ci[:, :l]
    fgc = t[:l]
    fc = t[l:] + eye
    bp = bc @ fc + bgc @ fgc
    return fc, fgc, bp


def _wy_line_search(dc, dgc, bc, bgc, taug, phi, mu, N, l):
    tau = taug
    phit = phi
    fc = fgc = bp = None
    for _ in range(WY_TAUMAXITER):                          # :174
        fc, fgc, bp = _wy_step(dc, dgc, bc, bgc, tau, l)
        phit = (0.5 / N) * np.sum(bp * bp)                  # :207
        if phit >= phi + tau * WY_SIGMA * mu:               # :210
            break
        tau *= WY_BETA
    return fc, fgc, bp, phit


def integrate_rb_wy(qs, l, N, maxit=256, tol=1e-3):
    """Row-block Wen-Yin line-search integrator.

    include/mcnla/isvd/integrator/row_block_wen_yin_integrator.hpp:112-278.
    """
    qc = qs[:, :l].copy()                                   # :112
    bc = qs.T @ qc                                          # :115
    dc = (bc.T @ bc) / N                                    # :121
    gc = (qs @ bc) / N                                      # :124
    bgc = qs.T @ gc                                         # :127
    dgc = (bc.T @ bgc) / N                                  # :133
    xc = gc - qc @ dc                                       # :136-137
    taug, zeta, phi = WY_TAU0, 1.0, (0.5 / N) * np.sum(bc * bc)      # :140
    mu = np.sum(np.abs(np.diag(dgc))) - np.sum(dc * dc)     # :143
    is_odd = False
    it = 0
    while it < maxit:                                       # :152
        is_odd = not is_odd
        fc, fgc, bp, phit = _wy_line_search(dc, dgc, bc, bgc, taug, phi, mu, N, l)
        phi = (WY_ETA * zeta * phi + phit) / (WY_ETA * zeta + 1)     # :217
        zeta = WY_ETA * zeta + 1                            # :218
        qp = qc @ fc + gc @ fgc                             # :221-222
        dp = (bp.T @ bp) / N                                # :224
        gp = (qs @ bp) / N                                  # :227
        bgp = qs.T @ gp                                     # :233
        dgp = (bp.T @ bgp) / N                              # :236
        mu = np.sum(np.abs(np.diag(dgp))) - np.sum(dp * dp)  # :240
        if mu < tol * tol:                                  # :249-250
            it += 1
            qc = qp
            break
        xp = gp - qp @ dp                                   # :253-254
        d1 = qc - qp                                        # :261
        d2 = xc - xp                                        # :262
        if is_odd:                                          # :264-273
            t1, t2 = np.sum(d1 * d1), np.sum(d1 * d2)
        else:
            t1, t2 = np.sum(d1 * d2), np.sum(d2 * d2)
        taug = min(max(abs(t1 / t2), WY_TAUMIN), WY_TAUMAX)  # :278-280
        qc, xc, bc, dc, gc, bgc, dgc = qp, xp, bp, dp, gp, bgp, dgp
        it += 1
    return qc, it


def integrate_rb_gramian_wy(qs, l, N, maxit=256, tol=1e-3):
    """Row-block Gramian Wen-Yin integrator (iterates on Bs only).

    include/mcnla/isvd/integrator/row_block_gramian_wen_yin_integrator.hpp:121-328.
    """
    L = qs.shape[1]
    bs, bc = _gramian_bs(qs, l)                             # :121-133
    bgc = (bs @ bc) / N                                     # :136
    dc = (bc.T @ bc) / N                                    # :139
    dgc = (bc.T @ bgc) / N                                  # :142
    ff = np.eye(l)                                          # :143-149
    ee = np.zeros((L, l))
    taug, zeta, phi = WY_TAU0, 1.0, (0.5 / N) * np.sum(bc * bc)      # :152
    mu = np.sum(np.abs(np.diag(dgc))) - np.sum(dc * dc)     # :155
    is_odd = False
    it = 0
    while it < maxit:                                       # :162
        is_odd = not is_odd
        fc, fgc, bp, phit = _wy_line_search(dc, dgc, bc, bgc, taug, phi, mu, N, l)
        phi = (WY_ETA * zeta * phi + phit) / (WY_ETA * zeta + 1)     # :225
        zeta = WY_ETA * zeta + 1
        u1 = (bc @ fgc) / N                                 # :229
        ffp = ff @ fc                                       # :232
        eep = u1 + ee @ fc                                  # :235-236
        bgp = (bs @ bp) / N                                 # :239
        dp = (bp.T @ bp) / N                                # :242
        dgp = (bp.T @ bgp) / N                              # :245
        mu = np.sum(np.abs(np.diag(dgp))) - np.sum(dp * dp)  # :248
        ff, ee = ffp, eep
        if mu < tol * tol:                                  # :252
            it += 1
            break
        phi2 = dc - fc @ dp                                 # :261-262
        phi1 = fc - np.eye(l)                               # :265-266
        u2 = (bp - bc) / N - u1 @ dp                        # :269-271
        bcu1 = bc.T @ u1                                    # :274
        bcu2 = bc.T @ u2                                    # :277
        if is_odd:                                          # :284-306
            bsu = bs @ u1
            t1 = np.sum(phi1 * phi1) + 2 * np.sum(phi1 * bcu1) + np.sum(u1 * bsu)
            t2 = np.sum(phi1 * phi2) + np.sum(phi1 * bcu2) + np.sum(phi2 * bcu1) + np.sum(u2 * bsu)
        else:
            bsu = bs @ u2
            t1 = np.sum(phi1 * phi2) + np.sum(phi1 * bcu2) + np.sum(phi2 * bcu1) + np.sum(u1 * bsu)
            t2 = np.sum(phi2 * phi2) + 2 * np.sum(phi2 * bcu2) + np.sum(u2 * bsu)
        taug = min(max(abs(t1 / t2), WY_TAUMIN), WY_TAUMAX)  # :309-311
        bc, dc, bgc, dgc = bp, dp, bgp, dgp
        it += 1
    qbar = qs[:, :l] @ ff + qs @ ee                         # :327-328
    return qbar, it


INTEGRATORS = {
    "kn": integrate_kn,
    "rb_kn": integrate_rb_kn,
    "rb_gramian_kn": integrate_rb_gramian_kn,
    "rb_wy": integrate_rb_wy,
    "rb_gramian_wy": integrate_rb_gramian_wy,
}


# --------------------------------------------------------------------------------------------
# Formers
# --------------------------------------------------------------------------------------------
def form_svd(a, qbar, k):
    """SVD former (with V).

    include/mcnla/isvd/former/svd_former.hpp:99-113:
      Vt := Q' A; gesvd(Vt) = W S Vt; U := Q W(:, 0:k); V := Vt(0:k, :)'.
    """
    vt = qbar.T @ a
    w, s, vt = np.linalg.svd(vt, full_matrices=False)
    return s[:k].copy(), qbar @ w[:, :k], vt[:k].T.copy()


def form_gramian(a, qbar, k):
    """Gramian former (plain, row-block and column-block agree on one rank).

    include/mcnla/isvd/former/gramian_former.hpp:101-128
    (row_block_gramian_former.hpp:109-142, col_block_gramian_former.hpp:97-127):
      Z := A' Q; W := Z' Z; gesvd(W) -> W, s; s := sqrt(s);
      U := Q W(:, 0:k); V := Z W(:, 0:k) diag(1/s).
    """
    z = a.T @ qbar
    w = z.T @ z
    wu, s, _ = np.linalg.svd(w)
    s = np.sqrt(s)
    u = qbar @ wu[:, :k]
    v = (z @ wu[:, :k]) / s[:k]
    return s[:k].copy(), u, v


FORMERS = {"svd": form_svd, "gramian": form_gramian}


# --------------------------------------------------------------------------------------------
# Pipeline
# --------------------------------------------------------------------------------------------
def isvd(a, omega, k, p, N, integrator="kn", former="svd", maxit=256, tol=1e-4):
    """Sketch -> Gramian orthogonalizer -> integrator -> former, as wired by the
    reference's drivers (src/isvd_dense_rb.cpp:46-286) with Omega explicit.
    Returns dict(s, u, v, qbar, iterations, q).
    """
    l = k + p
    y = sketch(a, omega)
    q = orthogonalize_gramian(y, l, N)
    qbar, it = INTEGRATORS[integrator](q, l, N, maxit, tol)
    s, u, v = FORMERS[former](a, qbar, k)
    return {"s": s, "u": u, "v": v, "qbar": qbar, "iterations": it, "q": q}


# --------------------------------------------------------------------------------------------
# Comparisons that are invariant under the factorizations' sign / basis freedom
# --------------------------------------------------------------------------------------------
def projector_gap(q1, q2):
    """max |Q1 Q1' - Q2 Q2'| (the reference tests' basis-invariant check,
    check/isvd/orthogonalizer/gramian_orthogonalizer.cpp:58-67)."""
    return float(np.max(np.abs(q1 @ q1.T - q2 @ q2.T)))


def align_signs(x, ref):
    """Flips the columns of x to agree in sign with ref (singular vectors are
    unique up to sign for distinct singular values)."""
    sg = np.sign(np.sum(x * ref, axis=0))
    sg[sg == 0] = 1.0
    return x * sg

"""Regenerates the golden fixtures in this folder from the reference's own test data.

The reference pins its iSVD stages with MatrixMarket "array" files under its
``data/`` folder (check/isvd/**.cpp load them through
include/mcnla/core/io/matrix_market/dense_load.hpp).  This script converts the
ones the hot path uses into one compressed ``.npz`` so that the tests run where
the reference tree is absent:

  a        (101, 1001)        row-major A             data/a.mtx
  q        (101, 11)          Q-bar fed to formers    data/q.mtx
  u        (101, 11)          expected U (first k=5)  data/u.mtx
  yi       (12, 101, 11)      sketches Y_i            data/yi.mtx
  qi       (12, 101, 11)      orthonormal Q_i         data/qi.mtx
  qb_kn    (101, 11)          KN result, tol 1e-4, 81 iterations   data/qb_kn.mtx
  qb_wy    (101, 11)          WY result, tol 1e-3, 21 iterations   data/qb_wy.mtx

It also records, in ``ref_outputs.npz``, what the reference's own stages (the
CPU checker built by ``make -C oracle``) return on those inputs, so the oracle
restatement can be compared with the reference beyond the published fixtures.

Usage: python tests/golden/make_golden.py [/path/to/reference]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))


def read_mtx_array(path):
    """Reads a MatrixMarket 'array' file (2-D or the reference's 3-D extension).

    Values are stored column-major per matrix; a 3-D file holds its matrices
    one after the other (dense_load.hpp reads k, then j, then i).
    Returns an array shaped (m, n) or (nmat, m, n) and the comment lines.
    """
    comments = []
    with open(path) as f:
        lines = f.read().split("\n")
    pos = 0
    while lines[pos].startswith("%"):
        comments.append(lines[pos])
        pos += 1
    dims = [int(x) for x in lines[pos].split()]
    vals = np.array([float(x) for x in " ".join(lines[pos + 1:]).split()], dtype=np.float64)
    if len(dims) == 2:
        m, n = dims
        assert vals.size == m * n, path
        return vals.reshape(n, m).T.copy(), comments
    m, n, k = dims
    assert vals.size == m * n * k, path
    return vals.reshape(k, n, m).transpose(0, 2, 1).copy(), comments


def main():
    from oracle.refpath import reference_root
    ref = sys.argv[1] if len(sys.argv) > 1 else reference_root()
    if not ref:
        sys.exit("the reference checkout was not found: pass its path or set MCNLA_REFERENCE")
    data = os.path.join(ref, "data")
    out = {}
    for name in ["a", "q", "u", "yi", "qi", "qb_kn", "qb_wy"]:
        arr, comments = read_mtx_array(os.path.join(data, name + ".mtx"))
        out[name] = arr
        for c in comments:
            if "iter" in c:
                out[name + "_iter"] = np.array(int(c.split("=")[1]))
            if "tol" in c:
                out[name + "_tol"] = np.array(float(c.split("tol =")[1].split(",")[0]))
    np.savez_compressed(os.path.join(HERE, "mcnla_data.npz"), **out)
    print({k: v.shape for k, v in out.items()})

    # Outputs of the reference's own stages on the same inputs.
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from oracle import ref_lib
    lib = ref_lib.load()
    refout = {}
    qs = np.concatenate(list(out["qi"]), axis=1)       # unfolded m x (N*l)
    ys = np.concatenate(list(out["yi"]), axis=1)
    m, L = qs.shape
    N = out["qi"].shape[0]
    l = L // N
    refout["orth_q"] = ref_lib.orthogonalize(lib, ys, l, N, row_block=False)
    for kind, tol in [(0, 1e-4), (1, 1e-4), (2, 1e-4), (3, 1e-3), (4, 1e-3)]:
        qbar, it = ref_lib.integrate(lib, qs, l, N, kind, 256, tol)
        refout["int%d_qbar" % kind] = qbar
        refout["int%d_iter" % kind] = np.array(it)
    a = out["a"]
    k = out["q"].shape[1] // 2
    p = out["q"].shape[1] - k
    for kind in range(4):
        s, u, v = ref_lib.form(lib, a, out["q"], k, p, kind)
        refout["form%d_s" % kind] = s
        refout["form%d_u" % kind] = u
        refout["form%d_v" % kind] = v
    np.savez_compressed(os.path.join(HERE, "ref_outputs.npz"), **refout)
    print({k: (v.shape, v if v.ndim == 0 else "") for k, v in refout.items() if k.endswith("iter")})


if __name__ == "__main__":
    main()

"""The binding a reference maintainer adds (include/mcnla_b200/mcnla_tags.hpp): B200 tags that
specialise the reference's own Sketcher / Orthogonalizer / Integrator / Former templates over the
C ABI.  Here (CPU) it compiles against the reference's headers with the one-rank MPI stub the
oracle uses; on a GPU the reference's stage templates run with those tags next to its CPU stages
on the reference's own fixtures (tests/cpp/check_mcnla_tags.cpp, built by oracle/Makefile):
81 KN iterations with Qbar within 1e-8 of qb_kn, the orthogonalizer and formers within 1e-10
of the CPU stages, and the row-block integrators again with their sums through the library's NCCL
communicator (the attachment an MPI run makes, here at one rank)."""
import os
import subprocess

import numpy as np
import pytest

from oracle.refpath import reference_root

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CHECKER = os.path.join(ROOT, "oracle", "_ref", "check_mcnla_tags")


@pytest.mark.skipif(reference_root() is None, reason="the reference's headers are not on this machine")
def test_binding_compiles_against_the_reference_headers():
    r = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "MCNLA_REFERENCE=" + reference_root(),
                        "_ref/check_mcnla_tags"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    assert os.path.exists(CHECKER)


@pytest.mark.gpu
def test_reference_stage_templates_with_b200_tags(tmp_path, golden):
    if not os.path.exists(CHECKER):
        pytest.skip("oracle/_ref/check_mcnla_tags is not built (make -C oracle)")
    for name in ("qs", "ys", "qb_kn", "a", "q"):
        np.ascontiguousarray(golden[name], dtype="<f8").tofile(os.path.join(str(tmp_path), name + ".bin"))
    r = subprocess.run([CHECKER, str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "OK (0 failures)" in r.stdout
    assert "rb_gramian_kn B200 iterations 81, reference 81" in r.stdout
    # the MPI row-block attachment: the library's NCCL communicator (one rank) carries the sums
    assert "rb_kn over a one-rank NCCL communicator" in r.stdout

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 and the built libmcnla_b200.so")


@pytest.fixture(scope="session")
def golden():
    """The reference's own test data (data/*.mtx), converted by tests/golden/make_golden.py."""
    d = np.load(os.path.join(GOLDEN, "mcnla_data.npz"))
    out = {k: d[k] for k in d.files}
    out["qs"] = np.concatenate(list(out["qi"]), axis=1)     # unfolded m x (N*l)
    out["ys"] = np.concatenate(list(out["yi"]), axis=1)
    out["N"], out["m"], out["l"] = out["qi"].shape
    return out


@pytest.fixture(scope="session")
def ref_outputs():
    """What the reference's own stages return on the golden inputs (oracle/_ref run here)."""
    d = np.load(os.path.join(GOLDEN, "ref_outputs.npz"))
    return {k: d[k] for k in d.files}


@pytest.fixture(scope="session")
def cuda():
    import torch
    assert torch.cuda.is_available(), "GPU test needs a CUDA device"
    from mcnla_b200 import _lib
    _lib.load()
    return torch.device("cuda", 0)

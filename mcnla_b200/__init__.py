"""mcnla_b200: B200-native integrated randomized SVD behind MCNLA's ``mcnla::isvd`` stage API.

The compute lives in ``libmcnla_b200.so`` (hand-written sm_100a kernels behind
the C ABI of ``include/mcnla_b200.h``); this package is its Python host side.
"""
from . import _lib  # noqa: F401

__version__ = "0.1.0"


def __getattr__(name):
    # the stage API needs torch; import it lazily so the C-ABI binding stays light
    if name == "isvd":
        import importlib
        return importlib.import_module(".isvd", __name__)
    raise AttributeError(name)

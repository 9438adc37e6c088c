"""Where the reference (emfomy/mcnla) sources are, for the recipes that read them.

Test infrastructure: only the oracle's build, the golden-fixture script and the
CPU tests that read the reference's own data files use it.  The location is the
MCNLA_REFERENCE environment variable when set, else a checkout named
``reference`` beside this repository.  It returns None when neither exists
(e.g. on a machine that only runs the prebuilt checker).
"""
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def reference_root():
    env = os.environ.get("MCNLA_REFERENCE")
    cands = [env] if env else []
    cands.append(os.path.join(os.path.dirname(ROOT), "reference"))
    for c in cands:
        if c and os.path.isdir(os.path.join(c, "include", "mcnla")):
            return os.path.abspath(c)
    return None

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def require_reference_build(path=None):
    """The reference library compiled from its sources (oracle/_ref) is part of the test
    set-up: a missing build fails the parity tests that compare against it instead of
    turning them off.  WDG_ALLOW_NO_REFERENCE=1 lets them skip (a checkout without the
    reference sources)."""
    from oracle import cpu

    ok = cpu.available("reference") if path is None else os.path.exists(path)
    if not ok:
        what = path or "oracle/_ref/libwdgref.so"
        if os.environ.get("WDG_ALLOW_NO_REFERENCE") == "1":
            pytest.skip(f"{what} not built (WDG_ALLOW_NO_REFERENCE=1)")
        pytest.fail(f"{what} is missing: build it with `make -C oracle ref` (needs the reference sources)")


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, name), allow_pickle=False))


def golden_files(prefix):
    return sorted(f for f in os.listdir(GOLDEN) if f.startswith(prefix) and f.endswith(".npz"))


def rel(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


@pytest.fixture(scope="session")
def gpu_lib():
    """The built CUDA library; GPU tests fail (not skip) if it is missing."""
    from wavedg_b200 import build, lib

    build.build()
    return lib()

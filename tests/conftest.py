"""Shared test set-up: paths, the `gpu` marker, builds on demand."""
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(REPO, "vid.stab_b200"))
sys.path.insert(0, os.path.join(REPO, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _has_gpu():
    try:
        import vidstab_b200
        return vidstab_b200.lib().vsb_device_count() > 0
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session", autouse=True)
def built():
    """Builds the product library and the oracle once per session."""
    import subprocess
    lib = os.path.join(REPO, "vid.stab_b200", "lib", "libvidstab_b200.so")
    if not os.path.exists(lib):
        subprocess.run([sys.executable, os.path.join(REPO, "vid.stab_b200", "build.py")],
                       check=True)
    if not os.path.exists(os.path.join(REPO, "oracle", "liboracle.so")):
        subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle"), "oracle"], check=True)
    yield


def records_equal(a, b):
    """LocalMotions equality over all seven fields, in order (the predicate of
    tests/test_determinism.c:356-361 of the reference)."""
    if len(a) != len(b):
        return False
    return all(np.array_equal(a[k], b[k]) for k in ("vx", "vy", "fx", "fy", "fsize",
                                                     "contrast", "match"))


def first_difference(a, b):
    for i in range(min(len(a), len(b))):
        if any(a[k][i] != b[k][i] for k in ("vx", "vy", "fx", "fy", "fsize", "contrast", "match")):
            return i, a[i], b[i]
    return min(len(a), len(b)), len(a), len(b)

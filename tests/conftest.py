"""Test configuration: the `gpu` marker, import paths, shared helpers.

`-m "not gpu"` tests run anywhere (oracle vs golden vectors, host logic, the
C-ABI library loading); `-m gpu` tests need a CUDA device and compare the
engine with the CPU oracle.
"""
import pathlib
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "matscipy-neighbours_b200", ROOT / "oracle"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: full-size workloads")


def _gpu_present():
    try:
        from matscipy_neighbours import _matscipy_neighbours as ext
        return bool(ext._has_gpu)
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _gpu_present():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    O.build()
    return O


def assert_same_lists(got, want, quantities):
    """Bit-identical outputs, in the same order (the engine reproduces the
    reference's row order, so no canonical sort is needed)."""
    if len(quantities) == 1:
        got, want = (got,), (want,)
    assert len(got) == len(want)
    for q, g, w in zip(quantities, got, want):
        g = np.asarray(g)
        w = np.asarray(w)
        assert g.shape == w.shape, f"{q}: shape {g.shape} != {w.shape}"
        assert g.dtype == w.dtype, f"{q}: dtype {g.dtype} != {w.dtype}"
        if g.dtype.kind == "f":
            same = np.array_equal(g.view(np.int64), w.view(np.int64))
        else:
            same = np.array_equal(g, w)
        if not same:
            bad = np.flatnonzero((g != w).reshape(len(g), -1).any(axis=1))
            raise AssertionError(f"{q}: {bad.size} rows differ, first {bad[:5]}")

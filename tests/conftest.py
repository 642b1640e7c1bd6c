"""Shared test set-up: repo root on sys.path, the ``gpu`` marker, golden loader."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def golden(name):
    return np.load(os.path.join(GOLDEN, name))


def baseline_refshim():
    """baseline/refshim.py, loaded under its own module name (tests/golden has a
    refshim module of its own)."""
    import importlib.util
    mod = sys.modules.get("amhd_baseline_refshim")
    if mod is None:
        spec = importlib.util.spec_from_file_location("amhd_baseline_refshim",
                                                      os.path.join(ROOT, "baseline", "refshim.py"))
        mod = importlib.util.module_from_spec(spec)
        sys.modules["amhd_baseline_refshim"] = mod
        spec.loader.exec_module(mod)
    return mod


def reference_available() -> bool:
    """Are the reference's modules installed (baseline/_ref) or named by AMHD_REFERENCE_DIR?"""
    try:
        baseline_refshim().reference_dir()
        return True
    except FileNotFoundError:
        return False


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    O.lib()
    return O


def pytest_collection_modifyitems(config, items):
    """GPU tests need a CUDA device; on a machine without one they are skipped."""
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:  # pragma: no cover
        has_gpu = False
    if has_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)

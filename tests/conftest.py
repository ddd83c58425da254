"""Shared test configuration.

Markers: ``gpu`` tests need a CUDA device (they run the engine through its C
ABI); everything else runs on CPU.  ``slow`` marks the full-size parity cases.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the engine through the C ABI")
    config.addinivalue_line("markers", "slow: full-size parity case (seconds of oracle time)")


def pytest_collection_modifyitems(config, items):
    try:
        import torch

        has_gpu = torch.cuda.is_available()
    except Exception:  # pragma: no cover
        has_gpu = False
    if has_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device in this environment")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


def rel_l2(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    den = np.linalg.norm(b.astype(np.complex128).ravel())
    num = np.linalg.norm((a.astype(np.complex128) - b.astype(np.complex128)).ravel())
    return float(num / den) if den > 0 else float(num)


def tolerance(single: bool, dims) -> float:
    """Parity bar: 1e-13 (f64) and 1e-6 * log2(N) (f32) relative L2 against
    the double-precision oracle, N = number of points."""
    n = int(np.prod(dims))
    return 1e-6 * max(1.0, np.log2(max(n, 2))) if single else 1e-13

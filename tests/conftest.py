import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def lib():
    """The built CUDA library (built here when missing or stale: nvcc cross-compiles without a GPU)."""
    from o_o_solver_b200 import _native, build

    build.build(quiet=True)
    return _native.load()


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    if not oracle.reference_available():
        pytest.skip("the reference oracle is not built (make -C oracle)")
    return oracle


def relative_columns(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    if a.ndim == 1:
        a = a[:, None]
        b = b[:, None]
    return np.linalg.norm(a - b, axis=0) / np.maximum(np.linalg.norm(b, axis=0), 1e-300)


def solution_bound(spread):
    """The bound on the relative difference between a GPU solution and the reference's: where the reference's own
    two kernel families agree to 1e-11 or better (well-conditioned matrices), the smaller of 1e-9 (the displacement
    tolerance of the path) and 100 x that spread + 1e-12; on the thin plates, whose conditioning makes two correct FP64
    solves differ by 1e-8 or more, 100 x the spread."""
    if spread <= 1e-11:
        return min(1e-9, 100.0 * spread + 1e-12)
    return 100.0 * spread

import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(Path(__file__).resolve().parent))

GOLDEN = Path(os.environ.get("OSTC_GOLDEN_DIR", str(ROOT / "tests" / "golden")))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the native parts once per session (no-op when up to date)."""
    from openstc_b200.build import build

    build()


@pytest.fixture(scope="session")
def case_factory(tmp_path_factory):
    """case_factory(name, builder, **kwargs) -> Path, cached per session."""
    cache: dict = {}

    def make(name, builder, **kw):
        key = (name, builder.__name__, tuple(sorted(kw.items())))
        if key not in cache:
            cache[key] = builder(tmp_path_factory.mktemp(name), **kw)
        return cache[key]

    return make


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    """Largest difference relative to the field's magnitude: max|a-b| / max|b|."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    na, nb = np.isnan(a), np.isnan(b)
    if np.any(na != nb):
        return float("inf")
    if np.any(na):  # the same cells are undefined on both sides (unused ghost corners)
        a, b = a[~na], b[~nb]
    scale = float(np.max(np.abs(b))) if b.size else 0.0
    if scale == 0.0:
        return float(np.max(np.abs(a - b))) if a.size else 0.0
    return float(np.max(np.abs(a - b))) / scale


def has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False

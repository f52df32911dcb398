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
        key = (name, builder.__name__, tuple(sorted((k, tuple(v) if isinstance(v, list) else v) for k, v in kw.items())))
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


VELOCITY = ("u", "v", "w")
SPECIES = ("H2", "H", "O2", "O", "OH", "HO2", "H2O2", "H2O", "N2")


def scaled_err(fields: dict, gold: dict) -> dict:
    """Per field: max|a - ref| divided by the variable's natural scale:
    the velocity magnitude scale (max over u, v, w) for velocity components,
    1 for mass fractions, the field's own max|ref| otherwise."""
    vscale = max(float(np.max(np.abs(gold[n]))) for n in VELOCITY if n in gold) if any(
        n in gold for n in VELOCITY) else 1.0
    out = {}
    for n, a in fields.items():
        b = np.asarray(gold[n], dtype=np.float64)
        a = np.asarray(a, dtype=np.float64)
        if n in VELOCITY:
            scale = vscale
        elif n in SPECIES:
            scale = 1.0
        else:
            scale = float(np.max(np.abs(b))) or 1.0
        d = np.abs(a - b)
        both_nan = np.isnan(a) & np.isnan(b)
        d[both_nan] = 0.0
        out[n] = float(np.max(d)) / scale if d.size else 0.0
    return out


def has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def err_max_history(rms_by_step: dict) -> dict:
    """{step: err_max} from the RMS one-step changes of (rho, |V|, p, T) of
    each residual step, the way Driver::compute_residual forms it
    (src/Driver.cu:345-380): normalised by the step-1 values (floored at
    1e-20), then the first one unless a later one is larger in magnitude."""
    out, scale = {}, None
    for step in sorted(rms_by_step):
        res = np.asarray(rms_by_step[step], dtype=np.float64)
        if step == 1:
            scale = np.maximum(res, 1e-20)
        res = res / scale
        e = res[0]
        for l in range(1, 4):
            if abs(res[l]) > e:
                e = res[l]
        out[step] = float(e)
    return out


def history_mismatch(ours: dict, gold_rows, rel: float = 1e-9) -> list:
    """Steps whose err_max differs from the reference's history.dat line.  The
    reference prints %11.4e (five significant digits), so a value matches
    when it lies within half a unit of that last digit of the printed value
    (plus `rel` of it, for rounding at a digit boundary)."""
    bad = []
    gold = {int(r[0]): float(r[1]) for r in gold_rows}
    if set(gold) != set(ours):
        return [("steps", sorted(set(gold) ^ set(ours)))]
    for step, g in gold.items():
        v = ours[step]
        if g == 0.0:
            ok = abs(v) < 5e-5 * 1e-300
        else:
            unit = 10.0 ** (np.floor(np.log10(abs(g))) - 4)
            ok = abs(v - g) <= 0.5 * unit + rel * abs(g)
        if not ok:
            bad.append((step, v, g))
    return bad

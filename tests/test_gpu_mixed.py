"""The FP32-bulk / FP64-critical path (precision="mixed") against the plain
FP64 path on the same case and GPU.

Bar: relative L2 error of T, Y_OH and p within 1e-3 of the FP64 path after
100 steps; every other stored field is reported and held to 1e-2.
"""
import numpy as np
import pytest

import openstc_b200 as ostc
from openstc_b200 import cases
from oracle_bridge import interior

pytestmark = pytest.mark.gpu

TOL_MAIN = 1e-3
TOL_OTHER = 1e-2


def rel_l2(a, b):
    d = np.linalg.norm((a - b).ravel())
    s = np.linalg.norm(b.ravel())
    return d / s if s > 0 else d


def fields(drv):
    info = drv.info()
    g = info.ngg
    bv = interior(drv.get(0, "bv"), g)
    sv = interior(drv.get(0, "sv"), g)
    out = {"density": bv[0], "u": bv[1], "v": bv[2], "pressure": bv[4], "temperature": bv[5]}
    names = ["H2", "H", "O2", "O", "OH", "HO2", "H2O2", "H2O", "N2"]
    for l, n in enumerate(names[: info.n_spec]):
        out[n] = sv[l]
    out["tke"], out["omega"] = sv[info.n_spec], sv[info.n_spec + 1]
    return out


@pytest.mark.parametrize("steps", [1, 100])
def test_mixed_tracks_fp64(case_factory, steps):
    case = case_factory("mixed_ml", cases.mixing_layer_case, mx=24, my=16, mz=8, total_step=steps,
                        output_screen=10, output_file=steps)
    ref = ostc.Driver(case)
    ref.initialize()
    ref.step(steps)
    mix = ostc.Driver(case, precision="mixed")
    mix.initialize()
    mix.step(steps)
    a, b = fields(mix), fields(ref)
    errs = {n: rel_l2(a[n], b[n]) for n in b}
    main = {n: errs[n] for n in ("temperature", "OH", "pressure")}
    assert all(v <= TOL_MAIN for v in main.values()), errs
    other = {n: v for n, v in errs.items() if n not in main and not v <= TOL_OTHER}
    assert not other, errs
    assert np.all(np.isfinite(mix.residual()))


def test_mixed_needs_finite_rate_sst(case_factory):
    case = case_factory("mixed_ramp", cases.ramp_case, mx=16, my=12, total_step=2, output_screen=1)
    d = ostc.Driver(case, precision="mixed")
    with pytest.raises(ostc.OstcError, match="finite-rate SST"):
        d.initialize()

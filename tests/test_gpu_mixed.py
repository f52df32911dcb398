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


FLUX_INPUTS = ("bv", "sv", "mul", "conductivity", "rho_d", "gamma", "cp", "mut", "turb_cond", "vel", "acoustic",
               "mach")


@pytest.mark.parametrize("shape", [(40, 10, 11), (24, 16, 8)])
def test_mixed_flux_matches_fp64_flux(case_factory, shape):
    """The FP32 column flux (primitive stencil staged in shared memory) against
    the FP64 flux on the same state, at sizes that leave partial columns in
    i, j and k: the flux differences added to dq within 1e-3 relative L2 per
    equation (an indexing fault gives O(1)), the local time step within 1e-5."""
    mx, my, mz = shape
    case = case_factory("mixed_flux", cases.mixing_layer_case, mx=mx, my=my, mz=mz, total_step=3,
                        output_screen=1, output_file=3)
    ref = ostc.Driver(case)
    ref.initialize()
    ref.step(3)
    mix = ostc.Driver(case, precision="mixed")
    mix.initialize()
    for f in FLUX_INPUTS:
        mix.set(0, f, ref.get(0, f))
    out = {}
    for name, drv in (("fp64", ref), ("mixed", mix)):
        drv.set(0, "dq", np.zeros(drv.field_shape(0, "dq")))
        drv.run_phase("flux")
        out[name] = (drv.get(0, "dq"), drv.get(0, "dt_local"))
    dq_m, dt_m = out["mixed"]
    dq_r, dt_r = out["fp64"]
    assert np.all(np.isfinite(dq_m))
    # momentum components against the momentum residual as a whole: the
    # spanwise component of this spanwise-uniform layer is FP32 rounding of
    # the z-face pressure terms alone
    mom = np.linalg.norm(dq_r[1:4].ravel())
    errs = [np.linalg.norm((dq_m[l] - dq_r[l]).ravel()) / (mom if 1 <= l <= 3 else np.linalg.norm(dq_r[l].ravel()))
            for l in range(dq_r.shape[0])]
    assert max(errs) <= 1e-3, " ".join(f"{e:.2e}" for e in errs)
    assert rel_l2(dt_m, dt_r) <= 1e-5

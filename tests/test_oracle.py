"""The CPU oracle itself: determinism, conservation of the update, and its
agreement with the reference program's outputs (tests/golden)."""
import numpy as np
import pytest

import openstc_b200 as ostc
from openstc_b200 import cases
from conftest import GOLDEN, scaled_err
from oracle_bridge import OracleSolver, interior

FIXTURE_CASES = {
    "ramp": (cases.ramp_case, dict(mx=48, my=24)),
    "ml": (cases.mixing_layer_case, dict(mx=16, my=12, mz=6)),
    "ml_explicit": (cases.mixing_layer_case, dict(mx=16, my=12, mz=6, implicit=0)),
    "mb": (cases.multiblock_case, dict(mxs=[10, 8], my=12, mz=6)),
}


def run(case, steps, threads=1):
    s = OracleSolver(ostc.Driver(case), threads=threads)
    s.initialize()
    res = None
    for k in range(1, steps + 1):
        r = s.step(k)
        if r is not None:
            res = r
    return s, res


def test_threads_do_not_change_results(case_factory):
    case = case_factory("ml", cases.mixing_layer_case, mx=12, my=10, mz=6, total_step=3, output_screen=1)
    a, ra = run(case, 3, threads=1)
    b, rb = run(case, 3, threads=4)
    shape = (11, 10, 14, 16)
    assert np.array_equal(a.get(0, "sv", shape), b.get(0, "sv", shape))
    assert np.array_equal(ra, rb)


def test_mass_fractions_stay_normalised(case_factory):
    """sum_k Y_k stays close to 1: chemistry and diffusion conserve it exactly,
    the per-species minmod limiting of the inviscid flux only nearly so."""
    case = case_factory("ml", cases.mixing_layer_case, mx=12, my=10, mz=6, total_step=3, output_screen=1)
    s, _ = run(case, 3)
    sv = s.get(0, "sv", (11, 10, 14, 16))
    ysum = interior(sv[:9], 2).sum(axis=0)
    assert np.max(np.abs(ysum - 1.0)) < 1e-8


@pytest.mark.parametrize("name,steps", [("ramp", 1), ("ramp", 10), ("ml", 1), ("ml", 10), ("ml_explicit", 1),
                                        ("ml_explicit", 10), ("mb", 1), ("mb", 10)])
def test_oracle_matches_reference_program(case_factory, name, steps):
    fix = GOLDEN / f"{name}_s{steps}.npz"
    if not fix.exists():
        pytest.skip(f"no reference fixture {fix.name}")
    gold = np.load(fix)
    fn, kw = FIXTURE_CASES[name]
    case = case_factory(name, fn, **dict(kw, total_step=steps, output_screen=1, output_file=steps))
    s, res = run(case, steps, threads=4)
    info = s.info
    worst = {}
    for b in range(info.n_block):
        mx, my, mz = s.dims[b]
        g = info.ngg
        shp = (mz + 2 * g, my + 2 * g, mx + 2 * g)
        bv = s.get(b, "bv", (6,) + shp)
        cols = {"density": bv[0], "u": bv[1], "v": bv[2], "w": bv[3], "pressure": bv[4], "temperature": bv[5],
                "mach": s.get(b, "mach", shp)}
        if info.n_scalar:
            sv = s.get(b, "sv", (info.n_scalar,) + shp)
            names = [k.split("/", 1)[1] for k in gold.files if k.startswith(f"b{b}/")]
            sp = [n for n in names if n not in cols and n not in ("tke", "omega", "mut")]
            for l, n in enumerate(sp):
                cols[n] = sv[l]
            if info.rans:
                cols["tke"], cols["omega"] = sv[info.n_spec], sv[info.n_spec + 1]
                cols["mut"] = s.get(b, "mut", shp)
        errs = scaled_err({n: interior(a, g) for n, a in cols.items()},
                          {n: gold[f"b{b}/{n}"] for n in cols})
        worst.update({f"b{b}/{n}": v for n, v in errs.items()})
    tol = 1e-10
    bad = {k: v for k, v in worst.items() if not v <= tol}
    assert not bad, f"beyond {tol}: {bad}"

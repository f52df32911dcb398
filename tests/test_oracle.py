"""The CPU oracle itself: determinism, conservation of the update, and its
agreement with the reference program's outputs (tests/golden)."""
import numpy as np
import pytest

import openstc_b200 as ostc
from openstc_b200 import cases
from conftest import GOLDEN, err_max_history, history_mismatch, scaled_err
from oracle_bridge import OracleSolver, interior

from fixture_cases import FIXTURES

FIXTURE_RUNS = [(n, k) for n, (_, _, steps) in FIXTURES.items() for k in steps]


def run(case, steps, threads=1, raws=None):
    """The oracle over `steps` steps; raws (dict) collects the RMS one-step
    changes of (rho, |V|, p, T) of every residual step."""
    s = OracleSolver(ostc.Driver(case), threads=threads)
    s.initialize()
    res = None
    for k in range(1, steps + 1):
        r = s.step(k)
        if r is not None:
            res = r
            if raws is not None:
                raws[k] = r.copy()
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


@pytest.mark.parametrize("name,steps", FIXTURE_RUNS)
def test_oracle_matches_reference_program(case_factory, name, steps):
    """Every variable of the reference's flowfield.plt within 1e-10 of its
    scale, and every line of its history.dat (err_max per step)."""
    fix = GOLDEN / f"{name}_s{steps}.npz"
    if not fix.exists():
        pytest.skip(f"no reference fixture {fix.name}")
    gold = np.load(fix)
    fn, kw, _ = FIXTURES[name]
    case = case_factory(name, fn, **dict(kw, total_step=steps, output_screen=1, output_file=steps))
    raws = {}
    s, res = run(case, steps, threads=4, raws=raws)
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
    # glibc's exp / pow / log differ from CUDA's by ulps per call; through 100
    # steps of stiff chemistry that reaches ~1e-10 of a field's scale (the
    # two-block case: 1.1e-10 in T), so the CPU restatement is held to 5e-10
    # there and to 1e-10 up to 10 steps (the GPU path keeps 1e-10 throughout)
    tol = 1e-10 if steps <= 10 else 5e-10
    bad = {k: v for k, v in worst.items() if not v <= tol}
    assert not bad, f"beyond {tol}: {bad}"
    hist = history_mismatch(err_max_history(raws), gold["history"])
    assert not hist, f"history.dat lines that differ (step, ours, reference): {hist[:10]}"


def wall_friction_heatflux_2d(bv, mul, cond, metric, dyn_pressure, g):
    """Restatement of wall_friction_heatFlux_2d (src/PostProcess.cu:50-73) on
    ghosted arrays (component, k, j, i): skin friction and wall heat flux at
    the j = 0 points of the k = 0 plane."""
    k0, j0, j1 = g, g, g + 1
    sl = slice(g, -g)
    xi_x, xi_y = metric[0, k0, j0, sl], metric[1, k0, j0, sl]
    eta_x, eta_y = metric[3, k0, j0, sl], metric[4, k0, j0, sl]
    u_parallel = (xi_x * bv[1, k0, j1, sl] + xi_y * bv[2, k0, j1, sl]) / np.sqrt(xi_x * xi_x + xi_y * xi_y)
    grad_eta = np.sqrt(eta_x * eta_x + eta_y * eta_y)
    cf = mul[k0, j0, sl] * (u_parallel * grad_eta) / dyn_pressure
    qw = cond[k0, j0, sl] * (bv[5, k0, j1, sl] - bv[5, k0, j0, sl]) * grad_eta
    return cf, qw


def test_wall_postprocess_restatement_matches_reference_program(case_factory):
    """The 2-D wall post-processing formula applied to the oracle's fields
    after 10 steps of the 48x24 ramp reproduces the reference program's own
    output/wall/friction_heatflux.dat (tests/golden/ramp_wall_s10.dat) to the
    six significant digits it writes."""
    fix = GOLDEN / "ramp_wall_s10.dat"
    if not fix.exists():
        pytest.skip(f"no reference fixture {fix.name}")
    lines = fix.read_text().splitlines()
    assert lines[0] == 'variables = "x", "cf", "qw"'
    gold = np.array([[float(v) for v in ln.split("\t")] for ln in lines[1:]])
    case = case_factory("ramp", cases.ramp_case, mx=48, my=24, total_step=10, output_screen=1, output_file=10)
    s, _ = run(case, 10, threads=4)
    g = s.info.ngg
    mx, my, mz = s.dims[0]
    shp = (mz + 2 * g, my + 2 * g, mx + 2 * g)
    # freestream of the ramp: air at Mach 3, 220 K, 2.5 kPa
    r_air = 8314.462618 / 28.9647
    rho_inf, v_inf = 2500.0 / (r_air * 220.0), 3.0 * np.sqrt(1.4 * r_air * 220.0)
    cf, qw = wall_friction_heatflux_2d(s.get(0, "bv", (6,) + shp), s.get(0, "mul", shp),
                                       s.get(0, "conductivity", shp), s.get(0, "metric", (9,) + shp),
                                       0.5 * rho_inf * v_inf * v_inf, g)
    x = s.get(0, "x", shp)[g, g, g:-g]
    ours = np.stack([x, cf, qw], axis=1)
    assert ours.shape == gold.shape == (48, 3)
    scale = np.abs(gold).max(axis=0)
    assert np.all(np.abs(ours - gold) <= 1e-5 * np.abs(gold) + 1e-12 * scale)

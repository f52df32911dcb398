"""The chemistry surrogate: FP64 EPI labels against the C oracle, tensor-core
gradients against the NumPy oracle (oracle/mlp_oracle.py), training, the
trust gate, and what the network gains over the EPI step it replaces."""
import ctypes as C
import sys
import time

import numpy as np
import pytest

import openstc_b200 as ostc
from openstc_b200 import cases
from conftest import ROOT
from oracle_bridge import oracle_lib, orc_params_from

sys.path.insert(0, str(ROOT / "oracle"))
import mlp_oracle  # noqa: E402

pytestmark = pytest.mark.gpu

RU = 8314.462618


@pytest.fixture(scope="module")
def drv(tmp_path_factory):
    case = tmp_path_factory.mktemp("sur") / "ml"
    cases.mixing_layer_case(case, mx=8, my=8, mz=4, total_step=1, output_screen=1)
    return ostc.Driver(case)


def random_states(n, seed):
    rng = np.random.default_rng(seed)
    s = np.zeros((n, 12))
    s[:, 0] = rng.uniform(250, 2800, n)
    s[:, 1] = 10 ** rng.uniform(4.5, 6.0, n)
    s[:, 2:11] = rng.dirichlet(np.ones(9), n)
    s[:, 11] = 10 ** rng.uniform(-9, -6, n)
    return s


def test_labels_match_oracle_epi(drv):
    sur = ostc.Surrogate(drv, seed=3)
    st = random_states(512, 11)
    dy = sur.label(st)
    p = orc_params_from(drv.params())
    mw = np.array(drv.params().mw[:9])
    worst = 0.0
    for i in range(st.shape[0]):
        Y = np.zeros(20)
        Y[:9] = st[i, 2:11]
        rho = st[i, 1] / (RU * st[i, 0] * np.sum(Y[:9] / mw))
        ref = np.zeros(20)
        oracle_lib().orc_epi_increment(C.byref(p), rho, st[i, 0], Y.ctypes.data_as(C.POINTER(C.c_double)), st[i, 11],
                                       ref.ctypes.data_as(C.POINTER(C.c_double)))
        scale = max(np.max(np.abs(ref[:9])), 1e-30)
        worst = max(worst, np.max(np.abs(dy[i] - ref[:9])) / scale)
    assert worst < 1e-9, worst


def test_gradients_match_oracle(drv):
    sur = ostc.Surrogate(drv, seed=5)
    sur.generate(4096, seed=2)
    st = random_states(1024, 12)
    dy = sur.label(st)
    loss, g = sur.gradients(st, dy)
    mu, sig, c, sc = sur.normalisation()
    x = mlp_oracle.features(st, mu, sig)
    r = dy / (st[:, 2:11] + 1e-10)
    t = (np.arcsinh(r / c.astype(np.float64)) / sc.astype(np.float64)).astype(np.float32).astype(np.float64)
    loss_ref, g_ref = mlp_oracle.loss_and_grads(sur.params(), x, t)
    assert abs(loss - loss_ref) <= 1e-4 * abs(loss_ref)
    off = 0
    for l in range(5):
        for n in (mlp_oracle.DIMS[l] * mlp_oracle.DIMS[l + 1], mlp_oracle.DIMS[l + 1]):
            a, b = g[off:off + n], g_ref[off:off + n]
            off += n
            rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
            assert rel < 2e-3, (l, n, rel)


def test_training_learns_and_gate(drv, tmp_path):
    sur = ostc.Surrogate(drv, seed=7)
    n = 1 << 19
    sur.generate(n, seed=4)
    losses = sur.train(400, batch=16384, lr=2e-3, n_train=n - (1 << 16))
    assert np.all(np.isfinite(losses))
    assert np.median(losses[-50:]) < 0.2 * np.median(losses[:5]), (losses[:5], losses[-50:])
    ev = sur.evaluate(n - (1 << 16), 1 << 16)
    assert ev["count"] == 1 << 16 and 0.0 <= ev["gate_pass"] <= 1.0
    # save / load round trip
    path = tmp_path / "mlp.bin"
    sur.save(path)
    other = ostc.Surrogate(drv, seed=99)
    other.load(path)
    st = random_states(256, 21)
    a, ga = sur.predict(st)
    b, gb = other.predict(st)
    assert np.array_equal(a, b) and np.array_equal(ga, gb)
    print("held-out:", ev)


def cell_states(d):
    """(T, p, Y[9], dt) of every interior cell of block 0, i fastest."""
    info = d.info()
    g = info.ngg
    bv = d.get(0, "bv")[:, g:-g, g:-g, g:-g]
    sv = d.get(0, "sv")[:, g:-g, g:-g, g:-g]
    dt = d.get(0, "dt_local")[0]
    n = dt.size
    st = np.zeros((n, 12))
    st[:, 0] = bv[5].ravel()
    st[:, 1] = bv[4].ravel()
    for k in range(9):
        st[:, 2 + k] = sv[k].ravel()
    st[:, 11] = dt.ravel()
    return st


@pytest.fixture(scope="module")
def trained(drv, tmp_path_factory):
    case = tmp_path_factory.mktemp("sur_field") / "ml"
    cases.mixing_layer_case(case, mx=24, my=16, mz=8, total_step=1, output_screen=1)
    field = ostc.Driver(case, precision="mixed")
    field.initialize()
    field.step(20)
    sur = ostc.Surrogate(field, seed=17)
    sur.generate(1 << 19, seed=5, field=field, field_fraction=0.9)
    sur.train(3000, batch=16384, lr=2e-3)
    return case, field, sur


def check_fused_against_unfused(field, sur):
    """The fused kernel (a split chemistry step over every cell of the field)
    against the unfused prediction on the same cells, the judge off so that
    the comparison covers accepted cells too.  Returns (accepted, fallback)."""
    sur.set_gate(judge_rel=-1.0)
    try:
        st = cell_states(field)
        dy_net, acc_net = sur.predict(st)
        dy_epi = sur.label(st)
        g = field.info().ngg
        y0 = field.get(0, "sv")[:9, g:-g, g:-g, g:-g].reshape(9, -1).T.copy()
        field.set_surrogate(sur)
        field.run_phase("chemistry")
        y1 = field.get(0, "sv")[:9, g:-g, g:-g, g:-g].reshape(9, -1).T
        dy = y1 - y0
        acc, fb = field.chemistry_stats()
        assert acc + fb == st.shape[0]
        # cells that took the EPI fallback: the same FP64 step as the labels
        scale = np.abs(dy_epi).max(axis=1, keepdims=True) + 1e-30
        epi_like = np.all(np.abs(dy - dy_epi) <= 1e-9 * scale + 1e-15, axis=1)
        # the fused kernel evaluates GELU with the hardware tanh: increments agree
        # to 10 % of the cell's largest increment (floor 1e-13); a layout or
        # pipeline fault would break nearly every cell, rounding only a few
        net_like = np.all(np.abs(dy - dy_net) <= 1e-1 * np.abs(dy_net).max(axis=1, keepdims=True) + 1e-13, axis=1)
        assert np.mean(epi_like | net_like) >= 0.99, np.mean(epi_like | net_like)
        # where the unfused gate accepted, the fused kernel gave the network's increment
        assert np.mean(net_like[acc_net]) > 0.98, np.mean(net_like[acc_net])
        field.set_surrogate(None)
        return acc, fb
    finally:
        sur.set_gate(judge_rel=0.25, judge_abs=1e-4)


def test_fused_inference_matches_unfused(trained):
    """24x16x8 cells: 24 tiles of 128, one per CTA (a pair with one tile)."""
    case, field, sur = trained
    acc, fb = check_fused_against_unfused(field, sur)
    print("fused: accepted", acc, "fallback", fb)


def test_fused_inference_two_and_three_tiles_per_cta(trained, tmp_path):
    """64x32x24 cells: 384 tiles over at most 148 CTAs, so a CTA runs a full
    pair of tiles (both slots) and some a pair and a single tile."""
    _, _, sur = trained
    case = tmp_path / "ml_big"
    cases.mixing_layer_case(case, mx=64, my=32, mz=24, total_step=1, output_screen=1)
    field = ostc.Driver(case, precision="mixed")
    field.initialize()
    field.step(20)
    try:
        acc, fb = check_fused_against_unfused(field, sur)
    finally:
        field.close()
    assert acc > 0
    print("fused, 49152 cells: accepted", acc, "fallback", fb)


def test_judge_rejects_a_silent_network_on_reacting_cells(drv):
    """A network whose every weight and bias is zero predicts no change at
    all.  The gate's own checks (training box, element defect, |dY_k| <=
    rel_max (Y_k + y_floor)) accept that wherever the change is small, even
    where the cell reacts; the judge compares with the cell's explicit
    increment (the diagonal point-implicit one) and rejects it on every cell that reacts
    measurably (an EPI increment above ten times the judge's floor)."""
    sur = ostc.Surrogate(drv, seed=7)
    sur.generate(1 << 14, seed=3)  # feature and target scaling
    sur.set_params(np.zeros_like(sur.params()))
    st = random_states(1 << 14, 31)
    dy_epi = sur.label(st)
    g = sur.gate()
    Y = st[:, 2:11]
    reacting = np.any(np.abs(dy_epi) > 10 * g["judge_abs"] * (Y + g["y_floor"]), axis=1)
    pred, acc = sur.predict(st)
    assert np.all(pred == 0.0)
    assert reacting.sum() > 1000
    assert not np.any(acc & reacting), int(np.sum(acc & reacting))
    # where nothing happens (cold hydrogen without oxygen) it is still trusted
    cold = np.zeros((256, 12))
    cold[:, 0] = np.linspace(300.0, 400.0, 256)
    cold[:, 1] = 101325.0
    cold[:, 2], cold[:, 10] = 0.4, 0.6  # H2, N2
    cold[:, 11] = 1e-7
    _, acc_cold = sur.predict(cold)
    assert np.all(acc_cold)
    sur.set_gate(judge_rel=-1.0)
    _, acc_unjudged = sur.predict(st)
    assert np.sum(acc_unjudged & reacting) > 100  # what the judge catches


def test_what_the_network_gains(trained, tmp_path):
    """The surrogate against the method without it on the same flow field and
    steps: the point-implicit chemistry everywhere (the FP32-bulk path) and
    the surrogate path both stay within the metric's 1e-3 relative L2 of
    (T, Y_OH, p) against the plain FP64 path, and the network takes the
    chemistry of a share of the cell-steps, whose EPI Jacobian,
    factorisation and DPLUR solves are skipped.  (Step time is measured at
    the benchmark's size, where it means something: bench.py --mode
    surrogate against --mode mixed.)"""
    case, _, sur = trained
    steps = 30
    runs = {}
    for name, kw, use in (("fp64", dict(precision="fp64"), False), ("epi", dict(precision="mixed"), False),
                          ("surrogate", dict(precision="mixed"), True)):
        d = ostc.Driver(case, **kw)
        d.initialize()
        d.step(20)
        if use:
            d.set_surrogate(sur)
        d.step(steps)
        g = d.info().ngg
        bv = d.get(0, "bv")[:, g:-g, g:-g, g:-g]
        sv = d.get(0, "sv")[:, g:-g, g:-g, g:-g]
        runs[name] = {"T": bv[5].copy(), "Y_OH": sv[4].copy(), "p": bv[4].copy()}
        if use:
            runs["stats"] = d.chemistry_stats()
            d.set_surrogate(None)
        d.close()
    for name in ("epi", "surrogate"):
        for f in ("T", "Y_OH", "p"):
            rel = np.linalg.norm(runs[name][f] - runs["fp64"][f]) / np.linalg.norm(runs["fp64"][f])
            assert rel <= 1e-3, (name, f, rel)
    accepted, fallback = runs["stats"]
    assert accepted + fallback == steps * runs["fp64"]["T"].size
    assert accepted > 0
    print(f"network took {accepted / (accepted + fallback):.3f} of the cell-steps' chemistry")

"""The launch autotuner (ostc_driver_autotune): every tuning it chooses from
(the order of the blocks in each launch x the variant of the flux kernels)
computes the same fields bit for bit, and the choice it records is applied
again by a later driver on the same case."""
import numpy as np
import pytest

import openstc_b200 as ostc
from openstc_b200 import cases

pytestmark = pytest.mark.gpu

MXS, MY, MZ = [12, 9, 10], 12, 6


def run(case, precision, schedule, variant, steps=3, fields=("bv", "sv", "dq")):
    d = ostc.Driver(case, precision=precision)
    d.initialize()
    d.set_tuning(schedule, variant)
    err = [d.step(1) for _ in range(steps)]
    out = {f: [d.get(b, f) for b in range(d.info().n_block)] for f in fields}
    d.close()
    return out, err


@pytest.mark.parametrize("precision,variants", [("fp64", 2), ("mixed", 4)])
def test_every_tuning_gives_the_same_fields(case_factory, precision, variants):
    case = case_factory("tuning_blocks", cases.multiblock_case, mxs=MXS, my=MY, mz=MZ, total_step=3,
                        output_screen=1)
    ref, ref_err = run(case, precision, 0, 0)
    for schedule in (0, 1):
        for variant in range(variants):
            if schedule == 0 and variant == 0:
                continue
            got, err = run(case, precision, schedule, variant)
            assert err == ref_err, (schedule, variant)
            for f in ref:
                for b, (x, y) in enumerate(zip(got[f], ref[f])):
                    assert np.array_equal(x, y, equal_nan=True), (schedule, variant, f, b)


def test_autotune_records_its_choice(case_factory, tmp_path):
    import shutil

    case = tmp_path / "blocks"
    shutil.copytree(case_factory("tuning_blocks", cases.multiblock_case, mxs=MXS, my=MY, mz=MZ, total_step=3,
                                 output_screen=1), case)
    d = ostc.Driver(case, precision="mixed")
    d.initialize()
    t = d.autotune(reps=2)
    assert t["candidates"] == 8
    assert 0 <= t["schedule"] <= 1 and 0 <= t["flux_variant"] < 4
    assert 0 < t["ms"] <= t["ms_default"]
    d.close()
    lines = (case / "output" / "message" / "autotune.txt").read_text().splitlines()
    assert lines[0].startswith("mix 2 rans 1 precision 1 exact 0 blocks 12x12x6 9x12x6 10x12x6")
    assert lines[1].split() == [str(t["schedule"]), str(t["flux_variant"])]
    # a later driver applies it; a bad setting is refused
    d = ostc.Driver(case, precision="mixed")
    d.initialize()
    d.step(1)
    with pytest.raises(ostc.OstcError, match="no such flux variant"):
        d.set_tuning(0, 9)
    d.close()


def test_fp64_flux_forms_agree_on_the_ramp(case_factory):
    """The column and the per-cell FP64 flux kernels on the 2-D ramp (a wall,
    an inflow, an outflow and a symmetry face): the same fields bit for bit."""
    case = case_factory("tuning_ramp", cases.ramp_case, mx=40, my=24, total_step=5, output_screen=1)
    fields = ("bv", "dq", "dt_local")
    ref, ref_err = run(case, "fp64", 0, 0, steps=5, fields=fields)
    got, err = run(case, "fp64", 0, 1, steps=5, fields=fields)
    assert err == ref_err
    for f in ref:
        assert np.array_equal(got[f][0], ref[f][0], equal_nan=True), f

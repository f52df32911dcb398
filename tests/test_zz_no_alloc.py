"""ostc_driver_residual_noalloc (static device scratch, no device allocation)
against ostc_driver_residual on the same driver.

Both reduce the same per-tile partial sums in the same order, so they agree
to the last bit in practice; the test allows 1e-13 relative.  The file name
puts it last in collection: it must pass alone and after every other test
(the scratch is shared by all drivers in the process).
"""
import numpy as np
import pytest

import openstc_b200 as ostc
from openstc_b200 import cases

pytestmark = pytest.mark.gpu

TOL = 1e-13


def close(a, b):
    return np.all(np.abs(a - b) <= TOL * np.abs(b))


@pytest.mark.parametrize("name", ["ml", "mb"])
def test_noalloc_residual_matches_residual_entry(case_factory, name):
    if name == "ml":
        case = case_factory("zz_ml", cases.mixing_layer_case, mx=16, my=12, mz=6, total_step=10, output_screen=1,
                            output_file=10)
    else:
        case = case_factory("zz_mb", cases.multiblock_case, mxs=[10, 8], my=12, mz=6, total_step=10, output_screen=1,
                            output_file=10)
    d = ostc.Driver(case)
    d.initialize()
    d.step(3)
    ref = d.residual()
    first = d.residual_noalloc()
    second = d.residual_noalloc()
    assert np.all(np.isfinite(ref)) and np.all(ref > 0)
    assert close(first, ref), (first, ref)
    assert close(second, ref), (second, ref)
    # after another step the scratch is reused with new values
    d.step(1)
    ref2 = d.residual()
    again = d.residual_noalloc()
    assert close(again, ref2), (again, ref2)
    assert not np.array_equal(ref2, ref)


def test_noalloc_residual_needs_a_step(case_factory):
    case = case_factory("zz_ramp", cases.ramp_case, mx=16, my=12, total_step=2, output_screen=1)
    d = ostc.Driver(case)
    d.initialize()
    with pytest.raises(ostc.OstcError, match="no step taken yet"):
        d.residual_noalloc()


def test_noalloc_residual_only_after_a_residual_step(case_factory):
    """With output_screen = 5 the previous state is stored at steps 5, 10, ...
    only.  Right after step 5 the recomputed residual equals the driver's;
    after step 7 the device holds the state of step 4 as the previous one, so
    the entry point refuses instead of returning a residual over three steps."""
    case = case_factory("zz_ml_s5", cases.mixing_layer_case, mx=16, my=12, mz=6, total_step=20, output_screen=5,
                        output_file=20)
    d = ostc.Driver(case)
    d.initialize()
    d.step(1)
    assert close(d.residual_noalloc(), d.residual())  # step 1 computes a residual too
    d.step(4)
    ref = d.residual()
    assert close(d.residual_noalloc(), ref), (d.residual_noalloc(), ref)
    d.step(2)
    with pytest.raises(ostc.OstcError, match="computed no residual"):
        d.residual_noalloc()
    d.step(3)  # step 10 stores again
    ref10 = d.residual()
    assert close(d.residual_noalloc(), ref10), (d.residual_noalloc(), ref10)
    assert not np.array_equal(ref10, ref)

"""The host-driven stepping loop (ostc_driver_step_io): each step's state is
uploaded from host buffers and the result read back into them, with the
copies of consecutive steps overlapped chunk by chunk.  Checked against the
plain loop (ostc_driver_step) on a second driver of the same case: the fields
and the host buffers are bit-identical, with residual steps (which wait on
the host) and without, with chunks far smaller than a field, and with host
data that differs from the device state before the call."""
import numpy as np
import pytest
import torch

import openstc_b200 as ostc
from openstc_b200 import cases

pytestmark = pytest.mark.gpu


def pinned_copy(a):
    t = torch.empty(a.size, dtype=torch.float64, pin_memory=True).numpy()
    t[:] = a.ravel()
    return t


@pytest.mark.parametrize("precision,screen,chunk", [("fp64", 1, 0), ("fp64", 50, 4096), ("mixed", 50, 65536)])
def test_step_io_matches_plain_loop(tmp_path, precision, screen, chunk):
    case = cases.mixing_layer_case(tmp_path / "ml", mx=24, my=16, mz=8, total_step=100, output_screen=screen)
    a = ostc.Driver(case, precision=precision)
    b = ostc.Driver(case, precision=precision)
    try:
        for d in (a, b):
            d.initialize()
            d.step(2)
        bv, sv = pinned_copy(a.get(0, "bv")), pinned_copy(a.get(0, "sv"))
        ea = a.step_io(6, 0, ["bv", "sv"], [bv, sv], chunk_bytes=chunk)
        eb = b.step(6)
        assert ea == eb
        for f, h in (("bv", bv), ("sv", sv)):
            ref = b.get(0, f).ravel()
            assert np.array_equal(a.get(0, f).ravel(), ref), f
            assert np.array_equal(h, ref), f
        # host data the device does not hold yet: the call starts from it
        bv *= 1.0 + 1e-6
        b.set(0, "bv", bv.copy())
        a.step_io(1, 0, ["bv", "sv"], [bv, sv], chunk_bytes=chunk)
        b.step(1)
        assert np.array_equal(bv, b.get(0, "bv").ravel())
        assert np.array_equal(sv, b.get(0, "sv").ravel())
    finally:
        a.close()
        b.close()


def test_step_io_second_block_of_two(tmp_path):
    """A two-block case: the fields of block 1 go up and down, block 0 stays
    on the device; the result equals the plain loop's."""
    case = cases.multiblock_case(tmp_path / "mb", mxs=[10, 8], my=12, mz=6, total_step=100, output_screen=50)
    a = ostc.Driver(case)
    b = ostc.Driver(case)
    try:
        for d in (a, b):
            d.initialize()
            d.step(1)
        bv, sv = pinned_copy(a.get(1, "bv")), pinned_copy(a.get(1, "sv"))
        a.step_io(4, 1, ["bv", "sv"], [bv, sv], chunk_bytes=2048)
        b.step(4)
        for blk in (0, 1):
            for f in ("bv", "sv"):
                assert np.array_equal(a.get(blk, f), b.get(blk, f)), (blk, f)
        assert np.array_equal(bv, b.get(1, "bv").ravel())
    finally:
        a.close()
        b.close()


def test_step_io_rejects_bad_arguments(tmp_path):
    case = cases.mixing_layer_case(tmp_path / "ml", mx=8, my=8, mz=4, total_step=10, output_screen=1)
    d = ostc.Driver(case)
    try:
        d.initialize()
        bv = d.get(0, "bv").ravel().copy()
        with pytest.raises(ostc.OstcError, match="size"):
            d.step_io(1, 0, ["bv"], [bv[:-1].copy()])
        with pytest.raises(ostc.OstcError, match="geometry"):
            d.step_io(1, 0, ["x"], [d.get(0, "x").ravel().copy()])
        with pytest.raises(ostc.OstcError, match="block"):
            d.step_io(1, 3, ["bv"], [bv])
    finally:
        d.close()

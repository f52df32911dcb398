"""Multi-block grids with exact inner faces (ostc_options.exact_inner) against
the same grid as one block, FP64 path: after every step each interior point
of every block equals the one-block point bit for bit.

The blocks are tiled along x with 1:1 faces (block b's last i plane is block
b + 1's first), so block b's interior i maps to i0_b + i of the one-block
grid with i0_b = sum(mxs[:b]) - b.  With the reference's inner-face
treatment (exact_inner = 0) the same comparison differs, since the DPLUR
sweeps stop at the face and mu_t is not exchanged; the test shows that too.
"""
import numpy as np
import pytest

import openstc_b200 as ostc
from openstc_b200 import cases
from oracle_bridge import interior

pytestmark = pytest.mark.gpu

FIELDS = ("bv", "sv", "mut", "dt_local")


def pair_of_runs(case_factory, mxs, my, mz, steps, exact=True):
    total = sum(mxs) - (len(mxs) - 1)
    one = case_factory("one_block", cases.mixing_layer_case, mx=total, my=my, mz=mz, total_step=steps,
                       output_screen=1)
    many = case_factory("many_blocks", cases.multiblock_case, mxs=list(mxs), my=my, mz=mz, total_step=steps,
                        output_screen=1)
    a = ostc.Driver(one)
    a.initialize()
    b = ostc.Driver(many, exact_inner=exact)
    b.initialize()
    return a, b


def differences(a, b, mxs):
    """{field: number of interior points of the blocks that differ from the
    one-block run}"""
    g = a.info().ngg
    out = {}
    for f in FIELDS:
        whole = a.get(0, f)
        whole = interior(whole, g) if f != "dt_local" else whole
        bad = 0
        i0 = 0
        for blk, m in enumerate(mxs):
            part = b.get(blk, f)
            part = interior(part, g) if f != "dt_local" else part
            bad += int(np.count_nonzero(part != whole[..., i0:i0 + m]))
            i0 += m - 1
        out[f] = bad
    return out


@pytest.mark.parametrize("mxs", [[10, 8], [9, 7, 11]])
def test_exact_inner_faces_equal_one_block(case_factory, mxs):
    a, b = pair_of_runs(case_factory, mxs, my=12, mz=6, steps=5)
    for step in range(1, 6):
        a.step(1)
        b.step(1)
        diff = differences(a, b, mxs)
        assert not any(diff.values()), f"step {step}: points that differ from one block {diff}"
    a.close()
    b.close()


def test_reference_inner_faces_differ_from_one_block(case_factory):
    """The reference's own treatment is not a partition of one block."""
    mxs = [10, 8]
    a, b = pair_of_runs(case_factory, mxs, my=12, mz=6, steps=2, exact=False)
    a.step(2)
    b.step(2)
    assert sum(differences(a, b, mxs).values()) > 0
    a.close()
    b.close()

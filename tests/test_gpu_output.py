"""The .plt output of the steady loop, written by a host thread while the next
steps run (two page-locked staging sets), against the synchronous writer on
the same final state: the files must be byte-identical, with step.txt naming
the last output step.  Output every step exercises the reuse of both staging
sets and the wait for the older one."""
import shutil

import pytest

import openstc_b200 as ostc
from openstc_b200 import cases

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["one_block", "two_blocks"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_async_plt_matches_sync_writer(tmp_path, kind, precision):
    if kind == "one_block":
        case = cases.mixing_layer_case(tmp_path / "c", mx=24, my=16, mz=8, total_step=7, output_screen=2,
                                       output_file=1)
    else:
        if precision == "mixed":
            pytest.skip("the two-block case is checked on the FP64 path")
        case = cases.multiblock_case(tmp_path / "c", [12, 10], my=12, mz=6, total_step=7, output_screen=2,
                                     output_file=1)
    d = ostc.Driver(case, precision=precision)
    d.initialize()
    d.simulate()
    plt = case / "output" / "field" / "flowfield.plt"
    assert (case / "output" / "message" / "step.txt").read_text() == "7"
    sync = tmp_path / "sync.plt"
    d.write_plt(sync)
    assert plt.read_bytes() == sync.read_bytes()
    # a second run continues from the same driver: the staging sets are reused
    shutil.copy(plt, tmp_path / "first.plt")
    d.simulate()
    # (the loop's counter ends one past its last step, so the second run
    # covers total_step further steps from there)
    assert int((case / "output" / "message" / "step.txt").read_text()) > 7
    d.write_plt(sync)
    assert plt.read_bytes() == sync.read_bytes()
    assert plt.read_bytes() != (tmp_path / "first.plt").read_bytes()

"""The .plt output of the steady loop, written by a host thread while the next
steps run (two page-locked staging sets), against the synchronous writer on
the same final state: the files must be byte-identical, with step.txt naming
the last output step.  Output every step exercises the reuse of both staging
sets and the wait for the older one."""
import shutil
from pathlib import Path

import numpy as np
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


GOLDEN = Path(__file__).resolve().parent / "golden"


def _wall_table(text: str):
    lines = text.splitlines()
    return lines[0], np.array([[float(v) for v in ln.split("\t")] for ln in lines[1:]])


@pytest.mark.parametrize("steps", [10, 100])
def test_wall_friction_heatflux_matches_reference(tmp_path, steps):
    """The reference's post-processing 0 (src/PostProcess.cu): skin friction
    and wall heat flux along the j = 0 wall of the 48x24 ramp, written at the
    output step, against the reference program's own
    output/wall/friction_heatflux.dat of the same case (same header, same
    number of points, values equal to the 6 significant digits both write)."""
    golden = GOLDEN / f"ramp_wall_s{steps}.dat"
    case = cases.ramp_case(tmp_path / "r", mx=48, my=24, total_step=steps, output_screen=1, output_file=steps,
                           post_process=[0])
    d = ostc.Driver(case)
    d.initialize()
    d.simulate()
    head, ours = _wall_table((case / "output" / "wall" / "friction_heatflux.dat").read_text())
    ref_head, ref = _wall_table(golden.read_text())
    assert head == ref_head
    assert ours.shape == ref.shape == (48, 3)
    scale = np.abs(ref).max(axis=0)
    assert np.all(np.abs(ours - ref) <= 1e-5 * np.abs(ref) + 1e-12 * scale)
    assert np.abs(ref[:, 1]).max() > 0 and np.abs(ref[:, 2]).max() > 0


def test_no_wall_file_without_post_process(tmp_path):
    case = cases.ramp_case(tmp_path / "r", mx=24, my=12, total_step=2, output_screen=1, output_file=2)
    d = ostc.Driver(case)
    d.initialize()
    d.simulate()
    assert not (case / "output" / "wall").exists()

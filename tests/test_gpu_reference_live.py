"""The plain FP64 path against the reference program at the stated sizes of
the benchmark configurations, both run on the same GPU from the same case
files for 100 steps:

  ramp_256x128    2-D laminar air over the 15 degree ramp, 256 x 128, explicit
  ml_384x192x64   the 3-D 9-species SST mixing layer, 384 x 192 x 64
                  (4.72 M cells), DPLUR 4 sweeps, EPI chemistry

The reference program is Liangerty/OpenSTC built from its own sources
(oracle/ref/Makefile -> oracle/_ref/openstc_ref); the library runs the same
case through Driver::simulate.  Compared: every variable of
output/field/flowfield.plt within 1e-10 of its scale (conftest.scaled_err)
and every line of history.dat (err_max of each step, output_screen = 1) to
the five digits the reference prints.  Set OSTC_REPORT_DIR to keep the worst
error per variable as JSON.
"""
import json
import os
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

import openstc_b200 as ostc
from openstc_b200 import cases
from openstc_b200.plt import read_plt
from conftest import ROOT, history_mismatch, scaled_err

REF_BIN = ROOT / "oracle" / "_ref" / "openstc_ref"

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not REF_BIN.exists(), reason="reference program not built (oracle/ref/Makefile)")]

STEPS = 100
CONFIGS = {
    "ramp_256x128": (cases.ramp_case, dict(mx=256, my=128)),
    "ml_384x192x64": (cases.mixing_layer_case, dict(mx=384, my=192, mz=64)),
}


def read_history(path: Path) -> np.ndarray:
    rows = []
    for line in path.read_text().splitlines():
        parts = line.split()
        if len(parts) == 2 and parts[0].isdigit():
            rows.append([float(parts[0]), float(parts[1])])
    return np.array(rows)


def run_copy(base: Path, where: Path) -> Path:
    """A run directory over `base`: setup files and the initial output copied
    (the run rewrites output/), grid, boundary and chemistry files linked."""
    (where / "input_files").mkdir(parents=True)
    for sub in (base / "input_files").iterdir():
        if sub.name == "setup":
            shutil.copytree(sub, where / "input_files" / "setup")
        else:
            (where / "input_files" / sub.name).symlink_to(sub.resolve())
    if (base / "output").exists():
        shutil.copytree(base / "output", where / "output")
    return where


@pytest.mark.parametrize("name", list(CONFIGS))
def test_config_size_matches_reference_program(tmp_path, name):
    fn, kw = CONFIGS[name]
    base = fn(tmp_path / "case", **dict(kw, total_step=STEPS, output_screen=1, output_file=STEPS))
    ref_dir, our_dir = run_copy(base, tmp_path / "reference"), run_copy(base, tmp_path / "ours")
    run = subprocess.run([str(REF_BIN)], cwd=ref_dir, capture_output=True, text=True, timeout=1800)
    assert run.returncode == 0, run.stdout[-2000:] + run.stderr[-2000:]
    drv = ostc.Driver(our_dir)
    drv.initialize()
    drv.simulate()
    drv.close()

    names, ref_zones = read_plt(ref_dir / "output" / "field" / "flowfield.plt")
    our_names, our_zones = read_plt(our_dir / "output" / "field" / "flowfield.plt")
    assert our_names == names
    worst = {}
    for b, (rz, oz) in enumerate(zip(ref_zones, our_zones)):
        fields = [n for n in names if n not in ("x", "y", "z")]
        for n in ("x", "y", "z"):
            assert np.array_equal(oz[n], rz[n]), f"grid {n} differs"
        errs = scaled_err({n: oz[n] for n in fields}, {n: rz[n] for n in fields})
        worst.update({f"b{b}/{n}": v for n, v in errs.items()})
    hist_ref = read_history(ref_dir / "history.dat")
    hist_our = read_history(our_dir / "history.dat")
    assert len(hist_ref) == STEPS
    bad_hist = history_mismatch({int(s): v for s, v in hist_our}, hist_ref)
    report = os.environ.get("OSTC_REPORT_DIR")
    if report:
        Path(report).mkdir(parents=True, exist_ok=True)
        (Path(report) / f"live_{name}.json").write_text(json.dumps(
            {"case": name, "steps": STEPS, "worst_scaled_err": worst,
             "history_lines_differing": len(bad_hist), "history_ref": hist_ref[:, 1].tolist(),
             "history_ours": hist_our[:, 1].tolist()}, indent=1))
    bad = {k: v for k, v in worst.items() if not v <= 1e-10}
    assert not bad, f"fields beyond 1e-10 vs the reference program: {bad}"
    assert not bad_hist, f"history.dat lines that differ (step, ours, reference): {bad_hist[:10]}"

"""Generates the golden fixtures of tests/golden/ by running the reference
program (Liangerty/OpenSTC built from its own sources by oracle/ref/Makefile
into oracle/_ref/openstc_ref) on small cases written by openstc_b200.cases.

The reference has no CPU path, so this runs on a GPU machine:

    python tests/golden/make_golden.py --ref oracle/_ref/openstc_ref --out tests/golden

Each fixture ``<case>_s<steps>.npz`` holds every variable of the reference's
output/field/flowfield.plt after <steps> steps (x, y, z dropped) plus the
history.dat residuals and residual_scale.txt of that run; the one-step
fixtures also keep the raw bytes of that flowfield.plt (``plt_raw``), which
the library must reproduce byte for byte.  The cases are listed in
tests/fixture_cases.py.  ``ramp_wall_s<steps>.dat``
is the reference's output/wall/friction_heatflux.dat (post-processing 0: skin
friction and heat flux along the ramp wall) of the ramp case run with
post_process = {0}, verbatim.
"""
from __future__ import annotations

import argparse
import shutil
import subprocess
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from openstc_b200 import cases  # noqa: E402
from openstc_b200.plt import read_plt  # noqa: E402

sys.path.insert(0, str(ROOT / "tests"))
from fixture_cases import FIXTURES as CASES  # noqa: E402

def build_case(name: str, where: Path, steps: int) -> Path:
    fn, kw, _ = CASES[name]
    case = where / f"{name}_s{steps}"
    if case.exists():
        shutil.rmtree(case)
    fn(case, **dict(kw, total_step=steps, output_screen=1, output_file=steps))
    return case


def run_reference(ref: Path, case: Path) -> None:
    res = subprocess.run([str(ref.resolve())], cwd=case, capture_output=True, text=True, timeout=1800)
    if res.returncode != 0:
        raise RuntimeError(f"reference run failed in {case}:\n{res.stdout[-2000:]}\n{res.stderr[-2000:]}")


def collect(case: Path, keep_raw: bool = False) -> dict[str, np.ndarray]:
    names, zones = read_plt(case / "output" / "field" / "flowfield.plt")
    out: dict[str, np.ndarray] = {}
    for z, zone in enumerate(zones):
        for n in names:
            if n in ("x", "y", "z"):
                continue
            out[f"b{z}/{n}"] = zone[n]
    rows = []
    for line in (case / "history.dat").read_text().splitlines():
        parts = line.split()
        if len(parts) == 2 and parts[0].isdigit():  # restart runs have no header line
            rows.append([float(parts[0]), float(parts[1])])
    out["history"] = np.array(rows) if rows else np.zeros((0, 2))
    out["residual_scale"] = np.array([float(v) for v in (case / "output" / "message" / "residual_scale.txt")
                                      .read_text().split()])
    if keep_raw:
        out["plt_raw"] = np.frombuffer((case / "output" / "field" / "flowfield.plt").read_bytes(), dtype=np.uint8)
    return out


# the ramp with the reference's 2-D wall post-processing: steps recorded
WALL_STEPS = (10, 100)


def make_wall_fixture(ref: Path, work: Path, out: Path, steps: int) -> None:
    case = work / f"ramp_wall_s{steps}"
    if case.exists():
        shutil.rmtree(case)
    cases.ramp_case(case, mx=48, my=24, total_step=steps, output_screen=1, output_file=steps, post_process=[0])
    run_reference(ref, case)
    shutil.copy(case / "output" / "wall" / "friction_heatflux.dat", out / f"ramp_wall_s{steps}.dat")


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=str(ROOT / "oracle" / "_ref" / "openstc_ref"))
    ap.add_argument("--out", default=str(ROOT / "tests" / "golden"))
    ap.add_argument("--work", default=str(ROOT / "cases" / "golden_runs"))
    ap.add_argument("--only", nargs="*")
    a = ap.parse_args()
    work = Path(a.work)
    work.mkdir(parents=True, exist_ok=True)
    out = Path(a.out)
    out.mkdir(parents=True, exist_ok=True)
    for name, (_, _, steps_list) in CASES.items():
        if a.only and name not in a.only:
            continue
        for steps in steps_list:
            case = build_case(name, work, steps)
            run_reference(Path(a.ref), case)
            np.savez_compressed(out / f"{name}_s{steps}.npz", **collect(case, keep_raw=steps == 1))
            print(f"{name} {steps} steps: ok", flush=True)
    if not a.only or "ramp_wall" in a.only:
        for steps in WALL_STEPS:
            make_wall_fixture(Path(a.ref), work, out, steps)
            print(f"ramp_wall {steps} steps: ok", flush=True)


if __name__ == "__main__":
    main()

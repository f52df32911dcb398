"""The reference-shaped C++ API (include/openstc_b200.hpp): Parameter, Mesh,
Driver<MixtureModel, TurbMethod>(Parameter &, Mesh &), initialize_computation,
simulate -- a main written as the reference's (tests/cxx_driver_api.cpp),
compiled with g++ against the header and linked with the library."""
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from openstc_b200 import cases
from conftest import GOLDEN, ROOT
from fixture_cases import FIXTURES


@pytest.fixture(scope="module")
def program(tmp_path_factory):
    from openstc_b200.build import LIB, build

    build()
    exe = tmp_path_factory.mktemp("cxx") / "cxx_driver_api"
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", str(ROOT / "include"), str(ROOT / "tests" / "cxx_driver_api.cpp"),
                    "-L", str(LIB.parent), "-lopenstc_b200", f"-Wl,-rpath,{LIB.parent}", "-o", str(exe)],
                   check=True)
    return exe


def test_driver_template_must_match_the_setup(program, case_factory):
    case = case_factory("cxx_ml", cases.mixing_layer_case, mx=10, my=8, mz=4, total_step=1, output_screen=1)
    res = subprocess.run([str(program), str(case), "check"], capture_output=True, text=True)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "blocks 1 dimension 3 cells 320 first 10 8 4" in res.stdout
    assert "ok 0" in res.stdout


@pytest.mark.gpu
def test_reference_main_writes_the_reference_plt(program, case_factory, tmp_path):
    """The main of the reference, rewritten against the header, run on the
    mixing layer of the golden fixtures for one step, writes the reference
    program's own output/field/flowfield.plt byte for byte."""
    fix = GOLDEN / "ml_s1.npz"
    if not fix.exists() or "plt_raw" not in np.load(fix).files:
        pytest.skip("no raw reference .plt")
    fn, kw, _ = FIXTURES["ml"]
    case = tmp_path / "ml"
    shutil.copytree(case_factory("ml", fn, **dict(kw, total_step=1, output_screen=1, output_file=1)), case)
    res = subprocess.run([str(program), str(case), "run"], capture_output=True, text=True)
    assert res.returncode == 0, res.stdout + res.stderr
    assert (case / "output" / "field" / "flowfield.plt").read_bytes() == np.load(fix)["plt_raw"].tobytes()
    assert (case / "history.dat").exists()

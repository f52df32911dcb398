"""The C ABI library loads, exports every declared entry point and reads
cases on the host (no GPU needed)."""
import ctypes
import re

import numpy as np
import pytest

import openstc_b200 as ostc
from openstc_b200 import cases
from conftest import ROOT


def declared_symbols():
    text = (ROOT / "include" / "openstc_b200.h").read_text()
    return sorted(set(re.findall(r"\b(ostc_[a-z_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(ostc.LIB_PATH))
    names = declared_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_missing_case_reports_input_error(tmp_path):
    with pytest.raises(ostc.OstcError, match="cannot open setup file"):
        ostc.Driver(tmp_path / "nope")


def test_device_calls_need_initialize(case_factory):
    case = case_factory("ramp", cases.ramp_case, mx=16, my=12, total_step=2, output_screen=1)
    d = ostc.Driver(case)
    with pytest.raises(ostc.OstcError, match="initialize first"):
        d.step(1)


@pytest.mark.parametrize("key", ["output_screen", "output_file"])
def test_step_intervals_must_be_positive(tmp_path, key):
    kw = {"output_screen": 1, "output_file": 2, key: 0}
    case = cases.ramp_case(tmp_path / "ramp", mx=16, my=12, total_step=2, **kw)
    with pytest.raises(ostc.OstcError, match=key + " must be a positive number of steps"):
        ostc.Driver(case)


def test_ramp_case_description(case_factory):
    case = case_factory("ramp", cases.ramp_case, mx=16, my=12, total_step=2, output_screen=1)
    d = ostc.Driver(case)
    i = d.info()
    assert (i.n_block, i.dimension, i.n_var, i.n_scalar, i.mix, i.rans) == (1, 2, 5, 0, 0, 0)
    assert i.n_grid_total == 16 * 12
    types = [b.type for b in d.bcs()]
    assert types == [6, 5, 3, 2]  # outflow, inflow, symmetry, wall: application order
    wall = d.bcs()[-1]
    assert list(wall.start) == [0, 0, 0] and list(wall.end) == [15, 0, 0]  # trimmed by ngg, k range [0, 0]
    inflow = d.bcs()[1]
    assert list(inflow.start) == [0, -2, -2] and list(inflow.end) == [0, 13, 2]
    # Mach 3 at 220 K, 2.5 kPa: velocity = 3 sqrt(1.4 R T / W)
    c = np.sqrt(1.4 * 8314.462618 / 28.9647 * 220.0)
    assert inflow.u == pytest.approx(3 * c, rel=1e-14)
    assert inflow.density == pytest.approx(2500.0 * 28.9647 / (8314.462618 * 220.0), rel=1e-14)


def test_layouts_follow_reference_ghosts(case_factory):
    case = case_factory("ml", cases.mixing_layer_case, mx=12, my=10, mz=6, total_step=2, output_screen=1)
    d = ostc.Driver(case)
    assert d.layout("bv") == (2, 6)
    assert d.layout("sv") == (2, 11)
    assert d.layout("cv") == (2, 16)
    assert d.layout("dq") == (1, 16)        # one ghost layer under DPLUR
    assert d.layout("chem_jac") == (0, 81)  # EPI Jacobian, no ghosts
    assert d.layout("bv_last") == (0, 4)
    assert d.field_shape(0, "metric") == (9, 10, 14, 16)


STRUCTS = {
    "ostc_options": ostc.Options, "ostc_info": ostc.Info, "ostc_params": ostc.Params, "ostc_bc": ostc.Bc,
    "ostc_inner": ostc.Inner, "ostc_surrogate_eval": ostc.SurrogateEval,
    "ostc_surrogate_gate": ostc.SurrogateGate, "ostc_tuning": ostc.Tuning,
}


def test_ctypes_structures_match_header(tmp_path):
    """Every ctypes mirror of a C-ABI struct has the header's size, field
    names, offsets and field sizes (compiled with the host C compiler)."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "openstc_b200.h"', "int main(void) {",
             '  printf("OSTC_MAX_SPEC %d\\n", OSTC_MAX_SPEC);', '  printf("OSTC_MAX_REAC %d\\n", OSTC_MAX_REAC);']
    for cname, cls in STRUCTS.items():
        lines.append(f'  printf("{cname} %zu\\n", sizeof({cname}));')
        for f, _ in cls._fields_:
            lines.append(f'  printf("{cname}.{f} %zu %zu\\n", offsetof({cname}, {f}), '
                         f"sizeof((({cname} *)0)->{f}));")
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c11", "-Wall", "-Werror", "-I", str(ROOT / "include"), str(src), "-o", str(exe)],
                   check=True)
    got = dict(line.split(" ", 1) for line in subprocess.run([str(exe)], check=True, capture_output=True,
                                                               text=True).stdout.splitlines())
    assert int(got["OSTC_MAX_SPEC"]) == ostc.MAX_SPEC and int(got["OSTC_MAX_REAC"]) == ostc.MAX_REAC
    for cname, cls in STRUCTS.items():
        assert int(got[cname]) == ctypes.sizeof(cls), cname
        for f, _ in cls._fields_:
            off, size = map(int, got[f"{cname}.{f}"].split())
            desc = getattr(cls, f)
            assert (desc.offset, desc.size) == (off, size), (cname, f)


def test_device_entry_points_refuse_an_uninitialised_driver(case_factory):
    """Before ostc_driver_initialize every entry point that needs the device
    returns OSTC_ERR_STATE ("initialize first") and touches nothing; with a
    null driver each returns OSTC_ERR_INPUT.  Host only: no GPU is needed."""
    case = case_factory("ramp", cases.ramp_case, mx=16, my=12, total_step=2, output_screen=1)
    d = ostc.Driver(case)
    lib = ostc.library()
    x = np.zeros(16)
    dp = x.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    fields = (ctypes.c_int * 1)(0)
    hosts = (ctypes.c_void_p * 1)(x.ctypes.data)
    counts = (ctypes.c_int64 * 1)(16)
    ll = ctypes.c_longlong()
    buf = ctypes.create_string_buffer(64)
    calls = {
        "ostc_driver_simulate": (),
        "ostc_driver_step": (1, dp),
        "ostc_driver_step_io": (1, 0, fields, hosts, counts, 1, 0, dp),
        "ostc_driver_autotune": (1, None),
        "ostc_driver_set_tuning": (0, 0),
        "ostc_driver_residual_noalloc": (dp,),
        "ostc_driver_run_phase": (0,),
        "ostc_driver_get_field": (0, 0, dp, 16),
        "ostc_driver_set_field": (0, 0, dp, 16),
        "ostc_driver_write_plt": (b"never_written.plt",),
        "ostc_driver_launches_per_step": (0, 0),
        "ostc_driver_last_step_ms": (dp,),
        "ostc_driver_profile_step": (buf, 64),
        "ostc_driver_set_surrogate": (None,),
        "ostc_driver_chemistry_stats": (ctypes.byref(ll), ctypes.byref(ll), ctypes.byref(ll)),
    }
    for name, args in calls.items():
        fn = getattr(lib, name)
        assert fn(d._h, *args) == -3, name  # OSTC_ERR_STATE
        assert "initialize first" in lib.ostc_last_error().decode(), name
        assert fn(None, *args) == -1, name  # OSTC_ERR_INPUT
    assert not np.any(x)
    assert lib.ostc_driver_stream(d._h) is None
    d.close()


def test_surrogate_entry_points_refuse_a_null_handle():
    lib = ostc.library()
    f = (ctypes.c_float * 16)()
    x = np.zeros(16)
    p = x.ctypes.data
    gate = ostc.SurrogateGate()
    ev = ostc.SurrogateEval()
    dbl = ctypes.c_double()
    calls = {
        "ostc_surrogate_generate": (None, 16, 1, 0.5),
        "ostc_surrogate_train": (1, 128, 1e-3, 0, None),
        "ostc_surrogate_evaluate": (0, 1, ctypes.byref(ev)),
        "ostc_surrogate_label": (p, 1, p),
        "ostc_surrogate_predict": (p, 1, p, p),
        "ostc_surrogate_gradients": (p, p, 128, f, ctypes.byref(dbl)),
        "ostc_surrogate_get_params": (f,),
        "ostc_surrogate_set_params": (f,),
        "ostc_surrogate_normalisation": (f, f, f, f),
        "ostc_surrogate_save": (b"never_written.bin",),
        "ostc_surrogate_load": (b"never_read.bin",),
        "ostc_surrogate_get_gate": (ctypes.byref(gate),),
        "ostc_surrogate_set_gate": (ctypes.byref(gate),),
    }
    for name, args in calls.items():
        assert getattr(lib, name)(None, *args) == -1, name  # OSTC_ERR_INPUT
    assert lib.ostc_surrogate_param_count() > 0

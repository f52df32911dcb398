"""Host side of the drop-in boundary: setup parser, grid / metric, boundary
registry, inner faces and Tecplot restart (CPU only)."""
import numpy as np
import pytest

import openstc_b200 as ostc
from openstc_b200 import cases
from openstc_b200.plt import read_plt, write_plt


def _ramp(tmp_path, **kw):
    return cases.ramp_case(tmp_path / "ramp", mx=kw.pop("mx", 16), my=kw.pop("my", 12), total_step=2,
                           output_screen=1, **kw)


def test_first_definition_wins_and_column_zero_comments(tmp_path):
    case = _ramp(tmp_path)
    f = case / "input_files" / "setup" / "2_scheme.txt"
    text = f.read_text()
    # a repeated key keeps its first value; "//" and "!" only comment at column 0
    text = text.replace("real    cfl = 0.5", "// real cfl = 9.0\nreal    cfl = 0.5\nreal cfl = 0.9\n! real cfl = 7")
    f.write_text(text)
    assert ostc.Driver(case).params().cfl == 0.5


def test_derived_keys(tmp_path, case_factory):
    d = ostc.Driver(_ramp(tmp_path))
    i = d.info()
    assert i.ngg == 2 and i.n_var == 5 and i.n_scalar == 0
    ml = case_factory("ml", cases.mixing_layer_case, mx=12, my=10, mz=6, total_step=2, output_screen=1)
    i = ostc.Driver(ml).info()
    assert (i.n_var, i.n_scalar, i.n_spec, i.n_reac) == (16, 11, 9, 19)


def test_string_array_value_on_brace_line_is_dropped(tmp_path):
    """src/Parameter.cpp:100 reads two tokens after the name of a string
    array; a value written on the '{' line is lost, so the wall struct is
    not registered and the label-2 wall falls back to the 300 K default."""
    case = _ramp(tmp_path)
    f = case / "input_files" / "setup" / "5_boundary_condition.txt"
    text = f.read_text().replace("array   string  boundary_conditions {\n    freestream wall\n}",
                                 "array   string  boundary_conditions { wall\n    freestream\n}")
    text = text.replace("real    temperature     =   300.0", "real    temperature     =   350.0")
    f.write_text(text)
    walls = [b for b in ostc.Driver(case).bcs() if b.type == 2]
    assert walls and all(w.t_wall == 300.0 for w in walls)


def test_missing_key_is_reported(tmp_path):
    case = _ramp(tmp_path)
    f = case / "input_files" / "setup" / "9_transport_property.txt"
    f.write_text(f.read_text().replace("real prandtl_number = 0.72\n", ""))
    with pytest.raises(ostc.OstcError, match="prandtl_number"):
        ostc.Driver(case)


def test_cartesian_metrics(tmp_path):
    """Uniform grid: J = dx dy dz and a diagonal metric, ghosts included."""
    mx, my, mz = 7, 6, 5
    dx, dy, dz = 0.01, 0.02, 0.005
    z, y, x = np.meshgrid(np.arange(mz) * dz, np.arange(my) * dy, np.arange(mx) * dx, indexing="ij")
    case = cases.mixing_layer_case(tmp_path / "ml", mx=mx, my=my, mz=mz, total_step=1, output_screen=1)
    cases.write_grid(case, [(x, y, z)])
    d = ostc.Driver(case)
    jac = d.host_field(0, "jac")[0]
    met = d.host_field(0, "metric")
    assert np.allclose(jac, dx * dy * dz, rtol=1e-12)
    expect = np.zeros(9)
    expect[[0, 4, 8]] = [1 / dx, 1 / dy, 1 / dz]
    for q in range(9):
        assert np.allclose(met[q], expect[q], rtol=1e-12, atol=1e-9)


def test_two_d_ghost_geometry(tmp_path):
    d = ostc.Driver(_ramp(tmp_path))
    z = d.host_field(0, "z")[0]
    # ghost planes are the k = 0 plane shifted by k (src/Mesh.cpp:840-855)
    assert np.allclose(z[0] - z[2], -2.0) and np.allclose(z[4] - z[2], 2.0)
    jac = d.host_field(0, "jac")[0][2]
    x, y = d.host_field(0, "x")[0][2], d.host_field(0, "y")[0][2]
    i, j = 5, 4  # interior point (ghost offset 2)
    dxd1 = (x[j + 2, i + 3] - x[j + 2, i + 1]) / 2
    dyd2 = (y[j + 3, i + 2] - y[j + 1, i + 2]) / 2
    dxd2 = (x[j + 3, i + 2] - x[j + 1, i + 2]) / 2
    dyd1 = (y[j + 2, i + 3] - y[j + 2, i + 1]) / 2
    assert jac[j + 2, i + 2] == pytest.approx(dxd1 * dyd2 - dxd2 * dyd1, rel=1e-13)


def test_multiblock_inner_faces(tmp_path):
    case = cases.multiblock_case(tmp_path / "mb", mxs=[6, 5], my=7, mz=4, total_step=1, output_screen=1)
    d = ostc.Driver(case)
    faces = d.inner_faces()
    assert len(faces) == 2
    f0 = faces[0]  # block 0, face at i = mx-1 looking at block 1's i = 0
    assert (f0.block, f0.target_block, f0.face, f0.direction) == (0, 1, 0, 1)
    assert list(f0.start) == [5, 0, 0] and list(f0.end) == [7, 6, 3] and list(f0.tstart) == [0, 0, 0]
    assert list(f0.src_tar) == [0, 1, 2] and list(f0.tloop_dir) == [1, 1, 1]
    f1 = faces[1]
    assert (f1.block, f1.target_block, f1.direction) == (1, 0, -1)
    assert list(f1.start) == [-2, 0, 0] and list(f1.tstart) == [3, 0, 0]
    # ghost geometry across the face is the neighbour's interior
    x0, x1 = d.host_field(0, "x")[0], d.host_field(1, "x")[0]
    g = 2
    assert np.array_equal(x0[g:-g, g:-g, 5 + g + 1], x1[g:-g, g:-g, 1 + g])
    assert np.array_equal(x1[g:-g, g:-g, g - 1], x0[g:-g, g:-g, 4 + g])


def _folded_case(tmp_path, x1):
    mx, my, mz = 6, 5, 4
    z, y, x = np.meshgrid(np.arange(mz) * 1.0, np.arange(my) * 1.0, np.arange(mx) * 1.0, indexing="ij")
    x = x.copy()
    x[:, :, 1] = x1
    case = cases.mixing_layer_case(tmp_path / "ml", mx=mx, my=my, mz=mz, total_step=1, output_screen=1)
    cases.write_grid(case, [(x, y, z)])
    return case


def test_negative_jacobian_in_ghost_layer_is_logged(tmp_path):
    """x(1) < x(0): the interior stays valid, the boundary metric folds; the
    reference logs it and copies the neighbour (src/Mesh.cpp:321-326, 523-532)."""
    case = _folded_case(tmp_path, -0.5)
    d = ostc.Driver(case)
    log = case / "error-log" / "negative-jacobian" / "Process_0-Block_0.log"
    assert log.exists() and log.read_text().startswith("Block 0, I = ")
    jac = d.host_field(0, "jac")[0]
    assert np.all(jac[2:-2, 2:-2, 2] == jac[2:-2, 2:-2, 3])  # i = 0 copied from i = 1


def test_negative_jacobian_inside_is_fatal(tmp_path):
    case = _folded_case(tmp_path, 3.5)  # x(2) - x(0) > 0 but x(3) - x(1) < 0 at i = 2
    with pytest.raises(ostc.OstcError, match="Negative Jacobian"):
        ostc.Driver(case)


def test_plt_round_trip(tmp_path):
    rng = np.random.default_rng(3)
    names = ["x", "y", "z", "density", "u"]
    zones = [{n: rng.random((2, 3, 4)) for n in names}, {n: rng.random((1, 2, 5)) for n in names}]
    write_plt(tmp_path / "f.plt", names, zones)
    n2, z2 = read_plt(tmp_path / "f.plt")
    assert n2 == names
    for a, b in zip(zones, z2):
        for n in names:
            assert np.array_equal(a[n], b[n])


def test_restart_reads_fields_by_name(case_factory):
    case = case_factory("ml", cases.mixing_layer_case, mx=12, my=10, mz=6, total_step=2, output_screen=1)
    names, zones = read_plt(case / "output" / "field" / "flowfield.plt")
    d = ostc.Driver(case)
    bv, sv = d.host_field(0, "bv"), d.host_field(0, "sv")
    g = 2
    for l, n in enumerate(["density", "u", "v", "w", "pressure", "temperature"]):
        assert np.array_equal(bv[l, g:-g, g:-g, g:-g], zones[0][n])
    for l, n in enumerate(["H2", "H", "O2", "O", "OH", "HO2", "H2O2", "H2O", "N2", "tke", "omega"]):
        assert np.array_equal(sv[l, g:-g, g:-g, g:-g], zones[0][n])
    assert d.info().step == 0


def test_batched_block_sizes_are_seeded_and_bounded():
    a = cases.batched_block_sizes(7)
    assert a == cases.batched_block_sizes(7) and a != cases.batched_block_sizes(8)
    mxs, my, mz = a
    assert len(mxs) == 12 and all(32 <= m <= 160 for m in mxs) and 32 <= my <= 96 and 32 <= mz <= 64
    assert sum(mxs) * my * mz <= 12 * 160 * 96 * 64


def test_batched_multiblock_case_reads_as_twelve_tiled_blocks(tmp_path):
    lo, hi = (5, 5, 4), (9, 7, 5)
    case = cases.batched_multiblock_case(tmp_path / "b12", seed=3, total_step=1, output_screen=1, lo=lo, hi=hi)
    mxs, my, mz = cases.batched_block_sizes(3, 12, lo, hi)
    d = ostc.Driver(case)
    info = d.info()
    assert info.n_block == 12
    assert [d.dims(b) for b in range(12)] == [(m, my, mz) for m in mxs]
    # two inner faces per shared plane, each naming its neighbour
    faces = d.inner_faces()
    assert len(faces) == 22
    assert sorted((f.block, f.target_block) for f in faces) == sorted(
        [(b, b + 1) for b in range(11)] + [(b + 1, b) for b in range(11)])


def test_numpy_inflow_state_equals_the_library_reader(tmp_path):
    """The case generator restates the inflow state in NumPy (so that writing
    a case loads no native library); it must equal what the library's own
    boundary-condition reader computes from the same files, bit for bit."""
    case = cases.mixing_layer_case(tmp_path / "ml", mx=8, my=6, mz=4, total_step=1)
    drv = ostc.Driver(case)
    prm = drv.params()
    by_t = sorted([b for b in drv.bcs() if b.type == 5], key=lambda b: b.temperature)
    ns = drv.info().n_spec
    for lib, spec in ((by_t[0], cases.LOWER), (by_t[-1], cases.UPPER)):
        st = cases.inflow_state(case, spec)
        for k in ("density", "u", "v", "w", "pressure", "temperature", "mut"):
            assert st[k] == getattr(lib, k), (k, st[k], getattr(lib, k))
        assert st["sv"] == [lib.sv[l] for l in range(ns + 2)]
        assert st["mw"] == [prm.mw[l] for l in range(ns)]
    drv.close()


def test_blended_initial_field_reads_back(tmp_path):
    """The tanh-blended restart file: the two streams far from the splitter,
    and the grid of the case's own grid file."""
    case = cases.mixing_layer_case(tmp_path / "ml", mx=8, my=24, mz=4, total_step=1)
    from openstc_b200.plt import read_plt

    names, zones = read_plt(case / "output" / "field" / "flowfield.plt")
    z = zones[0]
    up, lo = cases.inflow_state(case, cases.UPPER), cases.inflow_state(case, cases.LOWER)
    assert np.allclose(z["temperature"][:, -1, :], up["temperature"], rtol=1e-12)
    assert np.allclose(z["temperature"][:, 0, :], lo["temperature"], rtol=1e-12)
    assert np.allclose(z["u"][:, -1, :], up["u"], rtol=1e-12)
    assert np.allclose(z["H2"][:, 0, :], 0.4, rtol=1e-12)
    grid = cases._read_grid(case)[0]
    assert np.array_equal(z["y"], grid[1])


def test_exact_inner_faces_give_the_one_block_geometry(tmp_path):
    """With exact inner faces the ghost grid of each inner face, its
    tangential ghost rows included, is the neighbour's grid, so every block's
    coordinates, Jacobian and metrics over its whole ghosted extent equal
    those of the same grid as one block; the reference's completion of the
    ghost corners (src/Mesh.cpp:864-943) differs from them in the last bits."""
    mxs, my, mz = [9, 7, 11], 12, 6
    total = sum(mxs) - (len(mxs) - 1)
    one = ostc.Driver(cases.mixing_layer_case(tmp_path / "one", mx=total, my=my, mz=mz, total_step=1))
    many = cases.multiblock_case(tmp_path / "many", mxs=mxs, my=my, mz=mz, total_step=1)
    g = one.info().ngg
    for exact in (True, False):
        drv = ostc.Driver(many, exact_inner=exact)
        worst = 0.0
        for f in ("x", "y", "z", "jac", "metric"):
            whole = one.host_field(0, f)
            i0 = 0
            for b, m in enumerate(mxs):
                part = drv.host_field(b, f)
                lo, hi = max(i0 - g, -g), min(i0 + m + g, total + g)
                seg = part[..., lo - (i0 - g):lo - (i0 - g) + hi - lo]
                worst = max(worst, float(np.max(np.abs(seg - whole[..., lo + g:hi + g]))))
                i0 += m - 1
        if exact:
            assert worst == 0.0
        else:
            assert worst > 0.0
        drv.close()
    one.close()

"""ctypes bridge to the CPU oracle (oracle/libostc_oracle.so).

Test infrastructure: builds an oracle solver with the same case data the
library read (physics tables, boundary list, grid, initial field) so that
the oracle and the GPU path start from identical inputs.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
ORACLE_LIB = ROOT / "oracle" / "libostc_oracle.so"
MAXS, MAXR = 20, 64

ORC_FIELDS = [
    "x", "y", "z", "jac", "metric", "wall_dist", "bv", "sv", "cv", "vel", "acoustic", "mach", "mul",
    "conductivity", "rho_d", "gamma", "cp", "mut", "turb_cond", "chem_jac", "turb_src_jac", "dq", "dq0", "dqk",
    "inv_spec", "visc_spec", "dt_local", "bv_last",
]


class OrcParams(C.Structure):
    _fields_ = [
        ("mix", C.c_int), ("turb", C.c_int), ("rans_model", C.c_int), ("turb_implicit", C.c_int),
        ("chem_src_method", C.c_int), ("implicit_method", C.c_int), ("dplur_inner_step", C.c_int),
        ("reconstruction", C.c_int), ("limiter", C.c_int), ("viscous_order", C.c_int),
        ("ns", C.c_int), ("nr", C.c_int), ("n_var", C.c_int), ("n_scalar", C.c_int), ("output_screen", C.c_int),
        ("cfl", C.c_double), ("Pr", C.c_double), ("Prt", C.c_double), ("Sct", C.c_double), ("Sc", C.c_double),
        ("ll", C.c_double * 7), ("ul", C.c_double * 7), ("sv_inf", C.c_double * (MAXS + 2)),
        ("mw", C.c_double * MAXS), ("t_low", C.c_double * MAXS), ("t_mid", C.c_double * MAXS),
        ("low_coeff", C.c_double * (MAXS * 7)), ("high_coeff", C.c_double * (MAXS * 7)),
        ("lj_inv", C.c_double * MAXS), ("vis_coeff", C.c_double * MAXS),
        ("w_quarter", C.c_double * (MAXS * MAXS)), ("w_sqrt8", C.c_double * (MAXS * MAXS)),
        ("label", C.c_int * MAXR), ("order", C.c_int * MAXR),
        ("stoi_f", C.c_int * (MAXR * MAXS)), ("stoi_b", C.c_int * (MAXR * MAXS)),
        ("A", C.c_double * MAXR), ("b", C.c_double * MAXR), ("Ea", C.c_double * MAXR),
        ("A2", C.c_double * MAXR), ("b2", C.c_double * MAXR), ("Ea2", C.c_double * MAXR),
        ("third_body", C.c_double * (MAXR * MAXS)),
        ("troe_alpha", C.c_double * MAXR), ("troe_t3", C.c_double * MAXR), ("troe_t1", C.c_double * MAXR),
        ("troe_t2", C.c_double * MAXR),
    ]


class OrcBc(C.Structure):
    _fields_ = [
        ("block", C.c_int), ("type", C.c_int), ("face", C.c_int), ("direction", C.c_int),
        ("start", C.c_int * 3), ("end", C.c_int * 3),
        ("density", C.c_double), ("u", C.c_double), ("v", C.c_double), ("w", C.c_double),
        ("pressure", C.c_double), ("temperature", C.c_double), ("mut", C.c_double),
        ("sv", C.c_double * (MAXS + 2)), ("isothermal", C.c_int), ("t_wall", C.c_double),
    ]


class OrcInner(C.Structure):
    _fields_ = [
        ("block", C.c_int), ("target_block", C.c_int), ("face", C.c_int), ("direction", C.c_int),
        ("start", C.c_int * 3), ("loop_dir", C.c_int * 3), ("tstart", C.c_int * 3), ("tloop_dir", C.c_int * 3),
        ("src_tar", C.c_int * 3), ("n_point", C.c_int * 3), ("end", C.c_int * 3),
    ]


_lib = None


def oracle_lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not ORACLE_LIB.exists():
            from openstc_b200.build import build_oracle

            build_oracle()
        lib = C.CDLL(str(ORACLE_LIB))
        P, D = C.c_void_p, C.POINTER(C.c_double)
        lib.orc_create.argtypes = [C.POINTER(OrcParams), C.c_int, C.POINTER(C.c_int), C.c_int, C.c_int]
        lib.orc_create.restype = P
        lib.orc_destroy.argtypes = [P]
        lib.orc_array.argtypes = [P, C.c_int, C.c_int, C.POINTER(C.c_int64)]
        lib.orc_array.restype = D
        lib.orc_add_bc.argtypes = [P, C.POINTER(OrcBc)]
        lib.orc_add_inner.argtypes = [P, C.POINTER(OrcInner)]
        lib.orc_initialize.argtypes = [P]
        lib.orc_step.argtypes = [P, C.c_int, D]
        for ph in ("orc_phase_residual", "orc_phase_implicit", "orc_phase_update", "orc_phase_bc"):
            getattr(lib, ph).argtypes = [P, C.c_int]
        lib.orc_phase_exchange.argtypes = [P]
        lib.orc_chemical_source.argtypes = [C.POINTER(OrcParams), C.c_double, C.c_double, D, D, D]
        lib.orc_epi_increment.argtypes = [C.POINTER(OrcParams), C.c_double, C.c_double, D, C.c_double, D]
        lib.orc_enthalpy_cp.argtypes = [C.POINTER(OrcParams), C.c_double, D, D]
        _lib = lib
    return _lib


def orc_params_from(p) -> OrcParams:
    """Copy an openstc_b200.Params into the oracle's parameter struct."""
    o = OrcParams()
    for name, _ in OrcParams._fields_:
        src = getattr(p, name)
        dst = getattr(o, name)
        if isinstance(src, (int, float)):
            setattr(o, name, src)
        else:
            n = min(len(src), len(dst))
            for q in range(n):
                dst[q] = src[q]
    return o


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class OracleSolver:
    """The oracle run of a case, set up from an openstc_b200.Driver that has
    read the case (the driver does not need a GPU)."""

    def __init__(self, drv, threads: int = 1):
        lib = oracle_lib()
        info = drv.info()
        self.info = info
        self.params = orc_params_from(drv.params())
        self.dims = [drv.dims(b) for b in range(info.n_block)]
        d = (C.c_int * (3 * info.n_block))(*[v for t in self.dims for v in t])
        self._s = lib.orc_create(C.byref(self.params), info.n_block, d, info.ngg, threads)
        self.ngg = info.ngg
        for b in range(info.n_block):
            for f in ("x", "y", "z", "jac", "metric", "bv", "sv"):
                if f == "sv" and info.n_scalar == 0:
                    continue
                self.set(b, f, drv.host_field(b, f))
        for bc in drv.bcs():
            o = OrcBc()
            C.memmove(C.byref(o), C.byref(bc), min(C.sizeof(o), C.sizeof(bc)))
            lib.orc_add_bc(self._s, C.byref(o))
        for f in drv.inner_faces():
            o = OrcInner(block=f.block, target_block=f.target_block, face=f.face, direction=f.direction)
            for q in range(3):
                o.start[q], o.end[q], o.loop_dir[q] = f.start[q], f.end[q], f.loop_dir[q]
                o.tstart[q], o.tloop_dir[q], o.src_tar[q], o.n_point[q] = (
                    f.tstart[q], f.tloop_dir[q], f.src_tar[q], f.n_point[q])
            lib.orc_add_inner(self._s, C.byref(o))

    def close(self):
        if getattr(self, "_s", None):
            oracle_lib().orc_destroy(self._s)
            self._s = None

    def __del__(self):
        self.close()

    def view(self, block: int, field: str) -> np.ndarray:
        n = C.c_int64()
        ptr = oracle_lib().orc_array(self._s, block, ORC_FIELDS.index(field), C.byref(n))
        if not ptr:
            raise KeyError(f"oracle field {field} is not allocated")
        return np.ctypeslib.as_array(ptr, shape=(n.value,))

    def get(self, block: int, field: str, shape=None) -> np.ndarray:
        a = self.view(block, field).copy()
        return a.reshape(shape) if shape is not None else a

    def set(self, block: int, field: str, values: np.ndarray) -> None:
        v = self.view(block, field)
        flat = np.ascontiguousarray(values, dtype=np.float64).ravel()
        if flat.size != v.size:
            raise ValueError(f"{field}: {flat.size} values for {v.size}")
        v[:] = flat

    def initialize(self):
        oracle_lib().orc_initialize(self._s)

    def step(self, step_no: int):
        res = np.zeros(4)
        due = oracle_lib().orc_step(self._s, step_no, _dp(res))
        return res if due else None

    def phase(self, name: str, block: int = 0):
        lib = oracle_lib()
        if name == "exchange":
            lib.orc_phase_exchange(self._s)
        else:
            getattr(lib, f"orc_phase_{name}")(self._s, block)


def interior(a: np.ndarray, g: int) -> np.ndarray:
    """Strip g ghost layers from the last three axes."""
    if g == 0:
        return a
    return a[..., g:-g, g:-g, g:-g] if a.shape[-3] > 2 * g else a[..., :, g:-g, g:-g]

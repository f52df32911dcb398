"""B200-native OpenSTC step engine: Python binding of the C ABI.

The compute path is the in-tree library ``libopenstc_b200.so`` (C++ host
code and sm_100a CUDA kernels, declared in include/openstc_b200.h).  This
module only loads it and wraps its entry points; there is no Python or CPU
fallback: if the library is missing, importing the binding raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libopenstc_b200.so"

MAX_SPEC = 20
MAX_REAC = 50

# ostc_field_id
FIELDS = [
    "x", "y", "z", "jac", "metric", "wall_dist", "bv", "sv", "cv", "vel", "acoustic", "mach", "mul",
    "conductivity", "rho_d", "gamma", "cp", "mut", "turb_cond", "chem_jac", "turb_src_jac", "dq", "dq0", "dqk",
    "inv_spec", "visc_spec", "dt_local", "bv_last",
]
FIELD_ID = {n: i for i, n in enumerate(FIELDS)}
PRECISIONS = {"fp64": 0, "mixed": 1}
PHASES = {"residual": 0, "implicit": 1, "update": 2, "bc": 3, "exchange": 4, "store": 5, "source": 6, "flux": 7,
          "chemistry": 8}


class OstcError(RuntimeError):
    pass


class Options(C.Structure):
    _fields_ = [("device", C.c_int), ("quiet", C.c_int), ("precision", C.c_int), ("exact_inner", C.c_int),
                ("wall_distance", C.c_int)]


class SurrogateEval(C.Structure):
    _fields_ = [("mean_rel", C.c_double), ("max_rel", C.c_double), ("mean_abs", C.c_double),
                ("max_defect", C.c_double), ("mean_defect", C.c_double), ("median_rel_all", C.c_double),
                ("p90_rel_all", C.c_double), ("gate_pass", C.c_double), ("count", C.c_longlong),
                ("nonfinite", C.c_longlong), ("rel_count", C.c_longlong)]


class SurrogateGate(C.Structure):
    _fields_ = [(n, C.c_float) for n in ("t_min", "t_max", "lp_min", "lp_max", "ldt_min", "ldt_max", "defect_tol",
                                         "rel_max", "out_max", "y_floor", "judge_rel", "judge_abs")]


class Info(C.Structure):
    _fields_ = [
        ("n_block", C.c_int), ("ngg", C.c_int), ("dimension", C.c_int), ("n_spec", C.c_int), ("n_reac", C.c_int),
        ("n_var", C.c_int), ("n_scalar", C.c_int), ("mix", C.c_int), ("rans", C.c_int),
        ("implicit_method", C.c_int), ("dplur_inner_step", C.c_int), ("chem_src_method", C.c_int),
        ("step", C.c_int), ("n_grid_total", C.c_int64), ("n_bc", C.c_int), ("n_inner", C.c_int),
    ]


class Params(C.Structure):
    _fields_ = [
        ("ns", C.c_int), ("nr", C.c_int), ("n_var", C.c_int), ("n_scalar", C.c_int),
        ("mix", C.c_int), ("turb", C.c_int), ("rans_model", C.c_int), ("turb_implicit", C.c_int),
        ("chem_src_method", C.c_int), ("implicit_method", C.c_int), ("dplur_inner_step", C.c_int),
        ("reconstruction", C.c_int), ("limiter", C.c_int), ("viscous_order", C.c_int), ("dim", C.c_int),
        ("output_screen", C.c_int),
        ("cfl", C.c_double), ("Pr", C.c_double), ("Prt", C.c_double), ("Sct", C.c_double), ("Sc", C.c_double),
        ("ll", C.c_double * 7), ("ul", C.c_double * 7), ("sv_inf", C.c_double * (MAX_SPEC + 2)),
        ("mw", C.c_double * MAX_SPEC), ("t_low", C.c_double * MAX_SPEC), ("t_mid", C.c_double * MAX_SPEC),
        ("low_coeff", C.c_double * (MAX_SPEC * 7)), ("high_coeff", C.c_double * (MAX_SPEC * 7)),
        ("lj_inv", C.c_double * MAX_SPEC), ("vis_coeff", C.c_double * MAX_SPEC),
        ("w_quarter", C.c_double * (MAX_SPEC * MAX_SPEC)), ("w_sqrt8", C.c_double * (MAX_SPEC * MAX_SPEC)),
        ("label", C.c_int * MAX_REAC), ("order", C.c_int * MAX_REAC),
        ("stoi_f", C.c_int * (MAX_REAC * MAX_SPEC)), ("stoi_b", C.c_int * (MAX_REAC * MAX_SPEC)),
        ("A", C.c_double * MAX_REAC), ("b", C.c_double * MAX_REAC), ("Ea", C.c_double * MAX_REAC),
        ("A2", C.c_double * MAX_REAC), ("b2", C.c_double * MAX_REAC), ("Ea2", C.c_double * MAX_REAC),
        ("third_body", C.c_double * (MAX_REAC * MAX_SPEC)),
        ("troe_alpha", C.c_double * MAX_REAC), ("troe_t3", C.c_double * MAX_REAC),
        ("troe_t1", C.c_double * MAX_REAC), ("troe_t2", C.c_double * MAX_REAC),
    ]


class Tuning(C.Structure):
    _fields_ = [("schedule", C.c_int), ("flux_variant", C.c_int), ("candidates", C.c_int), ("ms", C.c_double),
                ("ms_default", C.c_double)]


class Bc(C.Structure):
    _fields_ = [
        ("block", C.c_int), ("type", C.c_int), ("face", C.c_int), ("direction", C.c_int),
        ("start", C.c_int * 3), ("end", C.c_int * 3),
        ("density", C.c_double), ("u", C.c_double), ("v", C.c_double), ("w", C.c_double),
        ("pressure", C.c_double), ("temperature", C.c_double), ("mut", C.c_double),
        ("sv", C.c_double * (MAX_SPEC + 2)), ("isothermal", C.c_int), ("t_wall", C.c_double),
    ]


class Inner(C.Structure):
    _fields_ = [
        ("block", C.c_int), ("target_block", C.c_int), ("face", C.c_int), ("direction", C.c_int),
        ("start", C.c_int * 3), ("end", C.c_int * 3), ("loop_dir", C.c_int * 3), ("tstart", C.c_int * 3),
        ("tloop_dir", C.c_int * 3), ("src_tar", C.c_int * 3), ("n_point", C.c_int * 3),
    ]


_lib = None


def library() -> C.CDLL:
    """Load libopenstc_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise OstcError(f"{LIB_PATH} is missing: build it with `python -m openstc_b200.build`")
    lib = C.CDLL(str(LIB_PATH))
    P, I64, D = C.c_void_p, C.c_int64, C.POINTER(C.c_double)
    sig = {
        "ostc_driver_create": ([C.c_char_p, C.POINTER(Options), C.POINTER(P)], C.c_int),
        "ostc_driver_destroy": ([P], None),
        "ostc_last_error": ([], C.c_char_p),
        "ostc_driver_info": ([P, C.POINTER(Info)], C.c_int),
        "ostc_driver_params": ([P, C.POINTER(Params)], C.c_int),
        "ostc_driver_bc": ([P, C.c_int, C.POINTER(Bc)], C.c_int),
        "ostc_driver_inner": ([P, C.c_int, C.POINTER(Inner)], C.c_int),
        "ostc_driver_block_dims": ([P, C.c_int, C.POINTER(C.c_int)], C.c_int),
        "ostc_field_layout": ([P, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)], C.c_int),
        "ostc_driver_get_host_field": ([P, C.c_int, C.c_int, D, I64], C.c_int),
        "ostc_driver_initialize": ([P], C.c_int),
        "ostc_driver_simulate": ([P], C.c_int),
        "ostc_driver_step": ([P, C.c_int, D], C.c_int),
        "ostc_driver_step_io": ([P, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_void_p), C.POINTER(C.c_int64),
                                 C.c_int, C.c_int64, D], C.c_int),
        "ostc_driver_residual": ([P, D], C.c_int),
        "ostc_driver_residual_noalloc": ([P, D], C.c_int),
        "ostc_driver_autotune": ([P, C.c_int, C.POINTER(Tuning)], C.c_int),
        "ostc_driver_set_tuning": ([P, C.c_int, C.c_int], C.c_int),
        "ostc_tc_gemm_bf16": ([P, C.c_int, P, C.c_int, P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, P, P], C.c_int),
        "ostc_surrogate_create": ([P, C.c_ulonglong, C.POINTER(P)], C.c_int),
        "ostc_surrogate_destroy": ([P], None),
        "ostc_surrogate_param_count": ([], C.c_int),
        "ostc_surrogate_generate": ([P, P, C.c_longlong, C.c_ulonglong, C.c_double], C.c_int),
        "ostc_surrogate_train": ([P, C.c_int, C.c_int, C.c_double, C.c_longlong, P], C.c_int),
        "ostc_surrogate_evaluate": ([P, C.c_longlong, C.c_longlong, C.POINTER(SurrogateEval)], C.c_int),
        "ostc_surrogate_label": ([P, P, C.c_longlong, P], C.c_int),
        "ostc_surrogate_predict": ([P, P, C.c_longlong, P, P], C.c_int),
        "ostc_surrogate_gradients": ([P, P, P, C.c_longlong, P, C.POINTER(C.c_double)], C.c_int),
        "ostc_surrogate_get_params": ([P, P], C.c_int),
        "ostc_surrogate_set_params": ([P, P], C.c_int),
        "ostc_surrogate_normalisation": ([P, P, P, P, P], C.c_int),
        "ostc_surrogate_save": ([P, C.c_char_p], C.c_int),
        "ostc_surrogate_load": ([P, C.c_char_p], C.c_int),
        "ostc_driver_set_surrogate": ([P, P], C.c_int),
        "ostc_surrogate_get_gate": ([P, C.POINTER(SurrogateGate)], C.c_int),
        "ostc_surrogate_set_gate": ([P, C.POINTER(SurrogateGate)], C.c_int),
        "ostc_driver_chemistry_stats": ([P, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong),
                                         C.POINTER(C.c_longlong)], C.c_int),
        "ostc_driver_run_phase": ([P, C.c_int], C.c_int),
        "ostc_driver_get_field": ([P, C.c_int, C.c_int, D, I64], C.c_int),
        "ostc_driver_set_field": ([P, C.c_int, C.c_int, D, I64], C.c_int),
        "ostc_driver_write_plt": ([P, C.c_char_p], C.c_int),
        "ostc_driver_launches_per_step": ([P, C.c_int, C.c_int], C.c_int),
        "ostc_driver_last_step_ms": ([P, D], C.c_int),
        "ostc_driver_stream": ([P], C.c_void_p),
        "ostc_driver_profile_step": ([P, C.c_char_p, C.c_int], C.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def _check(rc: int) -> None:
    if rc != 0:
        msg = library().ostc_last_error().decode(errors="replace")
        raise OstcError(f"openstc_b200 call failed ({rc}): {msg}")


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Driver:
    """Python face of the reference's Driver<mix, turb> (src/Driver.cuh:12-46).

    ``Driver(case_dir)`` reads the case (host only); ``initialize()`` runs
    Driver::initialize_computation on the GPU; ``simulate()`` the steady loop;
    ``step(n)`` n loop iterations without file output.
    """

    def __init__(self, case_dir: str | Path, device: int = 0, quiet: bool = True, precision: str = "fp64",
                 exact_inner: bool = False, wall_distance: str = "auto"):
        """precision: "fp64" (the reference's arithmetic) or "mixed" (FP32 fluxes,
        limiter, SST, flux Jacobians and transport; FP64 state, update,
        temperature inversion, chemistry, point-implicit solve, residual).
        exact_inner: a multi-block grid computes what the same grid as one
        block computes (ostc_options.exact_inner; FP64 path).
        wall_distance: "auto", "brute" (the reference's search over every wall
        point) or "grid" (an exact bucket search; the same values)."""
        lib = library()
        self._h = C.c_void_p()
        if precision not in PRECISIONS:
            raise OstcError(f"precision must be one of {sorted(PRECISIONS)}")
        walls = {"auto": 0, "brute": 1, "grid": 2}
        if wall_distance not in walls:
            raise OstcError(f"wall_distance must be one of {sorted(walls)}")
        opt = Options(device, 1 if quiet else 0, PRECISIONS[precision], 1 if exact_inner else 0, walls[wall_distance])
        _check(lib.ostc_driver_create(str(case_dir).encode(), C.byref(opt), C.byref(self._h)))
        self.case_dir = Path(case_dir)

    def close(self) -> None:
        if getattr(self, "_h", None):
            library().ostc_driver_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---------------------------------------------------------- description
    def info(self) -> Info:
        inf = Info()
        _check(library().ostc_driver_info(self._h, C.byref(inf)))
        return inf

    def params(self) -> Params:
        p = Params()
        _check(library().ostc_driver_params(self._h, C.byref(p)))
        return p

    def bcs(self) -> list[Bc]:
        out = []
        for q in range(self.info().n_bc):
            b = Bc()
            _check(library().ostc_driver_bc(self._h, q, C.byref(b)))
            out.append(b)
        return out

    def inner_faces(self) -> list[Inner]:
        out = []
        for q in range(self.info().n_inner):
            f = Inner()
            _check(library().ostc_driver_inner(self._h, q, C.byref(f)))
            out.append(f)
        return out

    def dims(self, block: int) -> tuple[int, int, int]:
        d = (C.c_int * 3)()
        _check(library().ostc_driver_block_dims(self._h, block, d))
        return d[0], d[1], d[2]

    def layout(self, field: str) -> tuple[int, int]:
        g, n = C.c_int(), C.c_int()
        _check(library().ostc_field_layout(self._h, FIELD_ID[field], C.byref(g), C.byref(n)))
        return g.value, n.value

    def field_shape(self, block: int, field: str) -> tuple[int, int, int, int]:
        """(components, nz, ny, nx) of the ghosted array in C order."""
        g, n = self.layout(field)
        mx, my, mz = self.dims(block)
        return n, mz + 2 * g, my + 2 * g, mx + 2 * g

    def host_field(self, block: int, field: str) -> np.ndarray:
        shape = self.field_shape(block, field)
        out = np.empty(shape, dtype=np.float64)
        _check(library().ostc_driver_get_host_field(self._h, block, FIELD_ID[field], _dptr(out), out.size))
        return out

    # ---------------------------------------------------------- device
    def initialize(self) -> None:
        _check(library().ostc_driver_initialize(self._h))

    def simulate(self) -> None:
        _check(library().ostc_driver_simulate(self._h))

    def step(self, n: int = 1) -> float:
        err = C.c_double(-1.0)
        _check(library().ostc_driver_step(self._h, n, C.byref(err)))
        return err.value

    def step_io(self, n: int, block: int, fields: list[str], arrays: list[np.ndarray], chunk_bytes: int = 0) -> float:
        """A host-driven stepping loop (ostc_driver_step_io): n steps, each
        preceded by the upload of the named fields of `block` from `arrays`
        (float64, C-contiguous, the get_field layout) and followed by their
        download into the same arrays.  The copies of one step's download and
        the next step's upload overlap chunk by chunk; page-locked arrays
        (e.g. from torch's pin_memory) make them asynchronous."""
        nf = len(fields)
        if len(arrays) != nf:
            raise OstcError("one array per field")
        for a in arrays:
            if a.dtype != np.float64 or not a.flags.c_contiguous:
                raise OstcError("arrays must be C-contiguous float64")
        ids = (C.c_int * nf)(*[FIELD_ID[f] for f in fields])
        ptrs = (C.c_void_p * nf)(*[a.ctypes.data for a in arrays])
        counts = (C.c_int64 * nf)(*[a.size for a in arrays])
        err = C.c_double(-1.0)
        _check(library().ostc_driver_step_io(self._h, n, block, ids, ptrs, counts, nf, chunk_bytes, C.byref(err)))
        return err.value

    def residual(self) -> np.ndarray:
        r = np.zeros(4)
        _check(library().ostc_driver_residual(self._h, _dptr(r)))
        return r

    def set_surrogate(self, sur: "Surrogate | None") -> None:
        """Chemistry through the surrogate: cells its trust gate accepts take
        the network's rate as an explicit source, the others keep the coupled
        point-implicit chemistry (None: point-implicit everywhere)."""
        self._surrogate = sur
        _check(library().ostc_driver_set_surrogate(self._h, sur._h if sur is not None else None))

    def chemistry_stats(self) -> tuple[int, int]:
        """(cell-steps accepted by the trust gate, cell-steps sent to the EPI fallback)."""
        a, f, e = C.c_longlong(), C.c_longlong(), C.c_longlong()
        _check(library().ostc_driver_chemistry_stats(self._h, C.byref(a), C.byref(f), C.byref(e)))
        return a.value, f.value

    def surrogate_evaluations(self) -> int:
        """Cell evaluations of the network since the surrogate was set."""
        a, f, e = C.c_longlong(), C.c_longlong(), C.c_longlong()
        _check(library().ostc_driver_chemistry_stats(self._h, C.byref(a), C.byref(f), C.byref(e)))
        return e.value

    def autotune(self, reps: int = 3) -> dict:
        """Time every launch tuning (block schedule x FP32 flux variant) on
        this case, apply the fastest and record it for later runs
        (ostc_driver_autotune)."""
        t = Tuning()
        _check(library().ostc_driver_autotune(self._h, reps, C.byref(t)))
        return {k: getattr(t, k) for k, _ in Tuning._fields_}

    def set_tuning(self, schedule: int, flux_variant: int = 0) -> None:
        _check(library().ostc_driver_set_tuning(self._h, schedule, flux_variant))

    def residual_noalloc(self) -> np.ndarray:
        """The residual of the last stored step recomputed on the device in
        a static scratch (ostc_driver_residual_noalloc): no device memory
        is allocated."""
        r = np.zeros(4)
        _check(library().ostc_driver_residual_noalloc(self._h, _dptr(r)))
        return r

    def run_phase(self, phase: str) -> None:
        _check(library().ostc_driver_run_phase(self._h, PHASES[phase]))

    def get(self, block: int, field: str) -> np.ndarray:
        shape = self.field_shape(block, field)
        out = np.empty(shape, dtype=np.float64)
        _check(library().ostc_driver_get_field(self._h, block, FIELD_ID[field], _dptr(out), out.size))
        return out

    def get_into(self, block: int, field: str, out: np.ndarray) -> None:
        _check(library().ostc_driver_get_field(self._h, block, FIELD_ID[field], _dptr(out), out.size))

    def set(self, block: int, field: str, values: np.ndarray) -> None:
        a = np.ascontiguousarray(values, dtype=np.float64)
        _check(library().ostc_driver_set_field(self._h, block, FIELD_ID[field], _dptr(a), a.size))

    def write_plt(self, path: str | Path) -> None:
        _check(library().ostc_driver_write_plt(self._h, str(path).encode()))

    def launches_per_step(self, store_last: bool = False, residual: bool = False) -> int:
        n = library().ostc_driver_launches_per_step(self._h, int(store_last), int(residual))
        if n < 0:
            _check(n)
        return n

    def last_step_ms(self) -> float:
        v = C.c_double()
        _check(library().ostc_driver_last_step_ms(self._h, C.byref(v)))
        return v.value

    def profile_step(self) -> list[tuple[str, int, float]]:
        """One eager step with per-kernel CUDA events: [(kernel, launches, ms)]."""
        buf = C.create_string_buffer(1 << 16)
        n = library().ostc_driver_profile_step(self._h, buf, len(buf))
        if n < 0:
            _check(n)
        rows = []
        for line in buf.value.decode().splitlines():
            name, cnt, ms = line.split()
            rows.append((name, int(cnt), float(ms)))
        return rows

    def stream(self) -> int:
        return library().ostc_driver_stream(self._h) or 0


def _vp(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class Surrogate:
    """The learned EPI chemistry step (ostc_surrogate_*): data generation with
    the FP64 EPI step, training on the tensor cores, evaluation."""

    def __init__(self, driver: "Driver", seed: int = 1):
        h = C.c_void_p()
        _check(library().ostc_surrogate_create(driver._h, seed, C.byref(h)))
        self._h = h

    def close(self) -> None:
        if self._h:
            library().ostc_surrogate_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def param_count() -> int:
        return library().ostc_surrogate_param_count()

    def generate(self, n: int, seed: int = 1, field: "Driver | None" = None, field_fraction: float = 0.5) -> None:
        _check(library().ostc_surrogate_generate(self._h, field._h if field else None, n, seed, field_fraction))

    def train(self, steps: int, batch: int = 65536, lr: float = 1e-3, n_train: int = 0) -> np.ndarray:
        losses = np.zeros(max(steps, 1), dtype=np.float32)
        _check(library().ostc_surrogate_train(self._h, steps, batch, lr, n_train, _vp(losses)))
        return losses[:steps]

    def evaluate(self, begin: int, count: int) -> dict:
        e = SurrogateEval()
        _check(library().ostc_surrogate_evaluate(self._h, begin, count, C.byref(e)))
        out = {f: getattr(e, f) for f, _ in SurrogateEval._fields_}
        if e.rel_count == 0:
            # no accepted sample has a resolvable increment: no relative error to report
            out["mean_rel"] = out["max_rel"] = None
        return out

    def label(self, states: np.ndarray) -> np.ndarray:
        s = np.ascontiguousarray(states, dtype=np.float64)
        out = np.zeros((s.shape[0], 9))
        _check(library().ostc_surrogate_label(self._h, _vp(s), s.shape[0], _vp(out)))
        return out

    def predict(self, states: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
        s = np.ascontiguousarray(states, dtype=np.float64)
        out = np.zeros((s.shape[0], 9))
        acc = np.zeros(s.shape[0], dtype=np.int32)
        _check(library().ostc_surrogate_predict(self._h, _vp(s), s.shape[0], _vp(out), _vp(acc)))
        return out, acc.astype(bool)

    def gradients(self, states: np.ndarray, dy: np.ndarray) -> tuple[float, np.ndarray]:
        s = np.ascontiguousarray(states, dtype=np.float64)
        d = np.ascontiguousarray(dy, dtype=np.float64)
        g = np.zeros(self.param_count(), dtype=np.float32)
        loss = C.c_double()
        _check(library().ostc_surrogate_gradients(self._h, _vp(s), _vp(d), s.shape[0], _vp(g), C.byref(loss)))
        return loss.value, g

    def params(self) -> np.ndarray:
        p = np.zeros(self.param_count(), dtype=np.float32)
        _check(library().ostc_surrogate_get_params(self._h, _vp(p)))
        return p

    def set_params(self, p: np.ndarray) -> None:
        a = np.ascontiguousarray(p, dtype=np.float32)
        _check(library().ostc_surrogate_set_params(self._h, _vp(a)))

    def normalisation(self) -> tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]:
        """(in_mu, in_sig, out_c, out_s): x = (f - in_mu) / in_sig;
        dY = (Y + 1e-10) out_c sinh(out_s o)."""
        mu, sig = np.zeros(12, np.float32), np.zeros(12, np.float32)
        c, sc = np.zeros(9, np.float32), np.zeros(9, np.float32)
        _check(library().ostc_surrogate_normalisation(self._h, _vp(mu), _vp(sig), _vp(c), _vp(sc)))
        return mu, sig, c, sc

    def gate(self) -> dict:
        g = SurrogateGate()
        _check(library().ostc_surrogate_get_gate(self._h, C.byref(g)))
        return {n: getattr(g, n) for n, _ in SurrogateGate._fields_}

    def set_gate(self, **kw) -> None:
        g = SurrogateGate()
        _check(library().ostc_surrogate_get_gate(self._h, C.byref(g)))
        for k, v in kw.items():
            if not hasattr(g, k):
                raise OstcError(f"unknown gate field {k}")
            setattr(g, k, v)
        _check(library().ostc_surrogate_set_gate(self._h, C.byref(g)))

    def save(self, path) -> None:
        _check(library().ostc_surrogate_save(self._h, str(path).encode()))

    def load(self, path) -> None:
        _check(library().ostc_surrogate_load(self._h, str(path).encode()))


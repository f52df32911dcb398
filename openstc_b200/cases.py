"""Case directories in the reference's input format.

A case directory holds ``input_files/setup/*.txt`` (the nine setup files of
src/Parameter.h:64-74), ``input_files/grid/grid   0.grd`` (src/Mesh.cpp:598-685),
``input_files/boundary_condition/{boundary,inner}   0.txt`` and
``input_files/chemistry/*``.  Both this library and the reference build read
these files unchanged.

Workloads:
* ``ramp_case``           - 2-D laminar air, Mach 3 over a 15 degree ramp
                            (256 x 128 x 1 by default, explicit, CFL 0.5).
* ``mixing_layer_case``   - 3-D reacting H2 / vitiated-air mixing layer,
                            9 species, k-omega SST, DPLUR 4 sweeps, EPI
                            (384 x 192 x 64 by default); starts from a tanh
                            blend of the two streams written as a restart file.
* ``multiblock_case``     - the mixing-layer physics on several blocks tiled
                            along x with 1:1 inner faces.
"""
from __future__ import annotations

import math
import shutil
from pathlib import Path

import numpy as np

_DATA = Path(__file__).resolve().parent / "data" / "chemistry"


def _fmt(v) -> str:
    if isinstance(v, bool):
        return "1" if v else "0"
    return repr(v) if isinstance(v, float) else str(v)


def write_setup(case: Path, files: dict[str, list[str]]) -> None:
    d = Path(case) / "input_files" / "setup"
    d.mkdir(parents=True, exist_ok=True)
    for name, lines in files.items():
        (d / name).write_text("\n".join(lines) + "\n")


def setup_files(*, dimension: int, total_step: int, output_file: int, output_screen: int, cfl: float,
                implicit_method: int, dplur_inner_step: int, species: bool, reaction: bool, turbulence: bool,
                chem_src_method: int = 1, initial: int = 0, convergence: float = 1e-30, reconstruction: int = 2,
                grid_scale: float = 1.0, inflows: list[dict] | None = None, walls: list[dict] | None = None,
                default_init: str = "freestream", schmidt: float = 0.5,
                post_process: list[int] | None = None) -> dict[str, list[str]]:
    """The nine setup files with the keys the reference reads.  post_process:
    the reference's post-processing labels (0: skin friction and heat flux of
    the j = 0 wall of a 2-D case)."""
    inflows = inflows or []
    walls = walls or []
    names = [f["name"] for f in inflows] + [w["name"] for w in walls]
    bc = ["array   string  boundary_conditions {", "    " + " ".join(names), "}", ""]
    for f in inflows:
        bc.append(f"struct  {f['name']} {{")
        bc.append("    string  type            =   inflow")
        bc.append(f"    int     label           =   {f['label']}")
        for k in ("temperature", "mach", "pressure", "u", "v", "w"):
            bc.append(f"    real    {k} = {_fmt(float(f[k]))}")
        if species:
            bc.append("    int     mole_or_mass    =   1")
            for sp, y in f.get("Y", {}).items():
                bc.append(f"    real    {sp} = {_fmt(float(y))}")
        if turbulence:
            bc.append(f"    real    turbulence_intensity = {_fmt(float(f.get('ti', 0.01)))}")
            bc.append(f"    real    turb_viscosity_ratio = {_fmt(float(f.get('mut_ratio', 1.0)))}")
        bc += ["}", ""]
    for w in walls:
        bc.append(f"struct  {w['name']} {{")
        bc.append("    string  type            =   wall")
        bc.append(f"    int     label           =   {w['label']}")
        bc.append(f"    string  thermal_type    =   {w.get('thermal', 'isothermal')}")
        bc.append(f"    real    temperature     =   {_fmt(float(w.get('temperature', 300.0)))}")
        bc += ["}", ""]
    return {
        "0_global_control.txt": [
            "bool parallel = 0", f"int initial = {initial}", f"int total_step = {total_step}",
            f"int output_file = {output_file}", f"int output_screen = {output_screen}"],
        "1_grid_information.txt": [
            f"int dimension = {dimension}", f"real gridScale = {_fmt(float(grid_scale))}",
            "real referenceLength = 1.0", "int wall_distance = 0"],
        "2_scheme.txt": [
            "bool    steady = 1", f"real    cfl = {_fmt(float(cfl))}", f"int     implicit_method = {implicit_method}",
            f"int     DPLUR_inner_step = {dplur_inner_step}", f"real convergence_criteria = {_fmt(float(convergence))}",
            "int	 temporal_scheme = 0", "real dt = 1e-9", "real total_simulation_time = 7e-3",
            "int     inner_iteration = 20", "int  inviscid_scheme = 3", f"int  reconstruction = {reconstruction}",
            "int  limiter = 0", "real entropy_fix_factor = 0.125", "int viscous_order = 2"],
        "3_species_reactions.txt": [
            f"bool species = {int(species)}", f"bool reaction = {int(reaction)}",
            "string mechanism_file = chemistry/combustion_mechanism.inp", "string therm_file = chemistry/therm.dat",
            "string transport_file = chemistry/tran.dat", f"int chemSrcMethod = {chem_src_method}",
            "string mix_frac_elem = C", "real hcst_tolerance = 1e-4"],
        "4_laminar_turbulent.txt": [
            f"bool    turbulence = {int(turbulence)}", f"int     turbulence_method = {1 if turbulence else 0}",
            "int     fluctuate_method = 0", "int     RANS_model = 2", "int     turb_implicit   =   1"],
        "5_boundary_condition.txt": bc,
        "6_post_process.txt": ["array   int post_process {"] + ([" ".join(map(str, post_process))] if post_process
                                                                 else []) + ["}"],
        "8_initialization.txt": ["int groups_init = 1", f"string  default_init    =   {default_init}"],
        "9_transport_property.txt": [
            "int diffusivity_method = 1", f"real schmidt_number = {_fmt(float(schmidt))}",
            "real prandtl_number = 0.72", "real turbulent_prandtl_number = 0.9",
            "real turbulent_schmidt_number = 0.9"],
    }


def write_grid(case: Path, blocks: list[tuple[np.ndarray, np.ndarray, np.ndarray]]) -> None:
    """blocks: (x, y, z) arrays of shape (mz, my, mx) each."""
    d = Path(case) / "input_files" / "grid"
    d.mkdir(parents=True, exist_ok=True)
    with open(d / "grid   0.grd", "w") as f:
        f.write(f"{len(blocks)}\n")
        for x, _, _ in blocks:
            mz, my, mx = x.shape
            f.write(f"{mx} {my} {mz}\n")
        for x, y, z in blocks:
            for a in (x, y, z):
                f.write("\n".join(map(repr, np.asarray(a, dtype=np.float64).ravel().tolist())))
                f.write("\n")


def write_boundary(case: Path, faces: list[list[tuple[int, ...]]], inner: list[list[tuple]] | None = None) -> None:
    """faces[b]: rows (i1, i2, j1, j2, k1, k2, label), 0-based inclusive.
    inner[b]: pairs ((7 ints of this face), (7 ints of the target face))
    in the 1-based convention of src/Mesh.cpp:709-741."""
    d = Path(case) / "input_files" / "boundary_condition"
    d.mkdir(parents=True, exist_ok=True)
    lines = []
    for fl in faces:
        lines.append(f"{len(fl):12d}")
        lines += ["".join(f"{v:6d}" for v in row) for row in fl]
    (d / "boundary   0.txt").write_text("\n".join(lines) + "\n")
    inner = inner or [[] for _ in faces]
    il = [f"{len(faces):12d}", "".join(f"{len(fl):12d}" for fl in inner), " imin  imax  jmin  jmax  kmin  kmax   id"]
    for fl in inner:
        for src, tar in fl:
            il.append("".join(f"{v:9d}" for v in src))
            il.append("".join(f"{v:9d}" for v in tar))
    (d / "inner   0.txt").write_text("\n".join(il) + "\n")
    (d / "parallel   0.txt").write_text(f"{len(faces):12d}{0:12d}\n" + "".join(f"{0:12d}" for _ in faces) + "\n")


def copy_chemistry(case: Path) -> None:
    d = Path(case) / "input_files" / "chemistry"
    d.mkdir(parents=True, exist_ok=True)
    for f in ("combustion_mechanism.inp", "therm.dat", "tran.dat"):
        shutil.copyfile(_DATA / f, d / f)


def _tanh_wall(n: int, first: float, height: float) -> np.ndarray:
    """n points on [0, height], one-sided tanh stretching with first spacing
    close to `first` (the stretching factor is found by bisection)."""
    s = np.linspace(0.0, 1.0, n)

    def spacing(beta):
        y = height * (1.0 + np.tanh(beta * (s - 1.0)) / np.tanh(beta))
        return y[1] - y[0]

    lo, hi = 1e-3, 20.0
    if spacing(lo) < first:
        return height * s
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if spacing(mid) > first:
            lo = mid
        else:
            hi = mid
    beta = 0.5 * (lo + hi)
    return height * (1.0 + np.tanh(beta * (s - 1.0)) / np.tanh(beta))


def ramp_case(case: str | Path, mx: int = 256, my: int = 128, total_step: int = 5000, output_screen: int = 100,
              output_file: int | None = None, post_process: list[int] | None = None) -> Path:
    """2-D laminar air, Mach 3, p = 2.5 kPa, T = 220 K over a 15 degree
    compression ramp (corner at x = 0.05 m, x in [0, 0.1] m, top at y = 0.03 m),
    first cell 1e-5 m at the isothermal 300 K wall; inflow i = 0, outflow
    i = max, symmetry on top.  AUSM+ / MUSCL-minmod, explicit, CFL 0.5."""
    case = Path(case)
    xs = np.linspace(0.0, 0.1, mx)
    ywall = np.where(xs < 0.05, 0.0, (xs - 0.05) * math.tan(math.radians(15.0)))
    x = np.empty((1, my, mx))
    y = np.empty((1, my, mx))
    for i in range(mx):
        y[0, :, i] = ywall[i] + _tanh_wall(my, 1e-5, 0.03 - ywall[i])
        x[0, :, i] = xs[i]
    z = np.zeros((1, my, mx))
    write_grid(case, [(x, y, z)])
    write_boundary(case, [[
        (0, mx - 1, 0, 0, 0, 0, 2),
        (0, 0, 0, my - 1, 0, 0, 5),
        (mx - 1, mx - 1, 0, my - 1, 0, 0, 6),
        (0, mx - 1, my - 1, my - 1, 0, 0, 3),
    ]])
    write_setup(case, setup_files(
        dimension=2, total_step=total_step, output_file=total_step if output_file is None else output_file,
        output_screen=output_screen,
        cfl=0.5, implicit_method=0, dplur_inner_step=3, species=False, reaction=False, turbulence=False,
        inflows=[dict(name="freestream", label=5, temperature=220.0, mach=3.0, pressure=2500.0, u=1.0, v=0.0,
                      w=0.0)],
        walls=[dict(name="wall", label=2, temperature=300.0)], post_process=post_process))
    copy_chemistry(case)
    return case


UPPER = dict(name="freestream", label=5, temperature=1250.0, mach=2.4, pressure=101325.0, u=1.0, v=0.0, w=0.0,
             Y={"O2": 0.245, "H2O": 0.175, "N2": 0.58}, ti=0.01, mut_ratio=1.0)
LOWER = dict(name="fuel", label=9, temperature=300.0, mach=1.2, pressure=101325.0, u=1.0, v=0.0, w=0.0,
             Y={"H2": 0.4, "N2": 0.6}, ti=0.01, mut_ratio=1.0)


def _mixing_layer_grid(mx, my, mz, x0=0.0, lx=0.3):
    xs = np.linspace(x0, x0 + lx, mx)
    s = np.linspace(-1.0, 1.0, my)
    ys = 0.025 + 0.025 * np.sinh(3.0 * s) / math.sinh(3.0)
    zs = np.linspace(0.0, 0.02, mz)
    z, y, x = np.meshgrid(zs, ys, xs, indexing="ij")
    return x, y, z


def _mixing_setup(case, *, total_step, output_screen, output_file, initial, cfl, dplur, chem, implicit=1,
                  wall=False):
    write_setup(case, setup_files(
        dimension=3, total_step=total_step, output_file=output_file, output_screen=output_screen, cfl=cfl,
        implicit_method=implicit, dplur_inner_step=dplur, species=True, reaction=True, turbulence=True,
        chem_src_method=chem, initial=initial, inflows=[UPPER, LOWER],
        walls=[dict(name="wall", label=2, temperature=300.0)] if wall else None))


RU = 8314.462618  # J/(kmol K), src/Constants.h:18

# Standard atomic weights of the elements a mechanism here names, as the
# reference tabulates them (src/Element.cpp:13-166).
_ATOMIC_WEIGHT = {"H": 1.008, "HE": 4.002602, "C": 12.011, "N": 14.007, "O": 15.999, "AR": 39.95}


def _mixture_data(case: Path) -> dict:
    """Molecular weights, NASA-7 coefficients and Lennard-Jones viscosity data
    of the mechanism's species, read from the case's therm.dat and tran.dat
    the way the reference's reader does (src/ChemData.cpp:138-293): the first
    record of a species wins; name in columns 1-18, element counts in four
    5-column fields from column 25, T_low / T_high / T_mid in 10-column fields
    from column 46; three lines of 15-column coefficients (high set first)."""
    chem = Path(case) / "input_files" / "chemistry"
    species = _species_names(case)
    idx = {n: i for i, n in enumerate(species)}
    ns = len(species)
    mw = [0.0] * ns
    t_low, t_mid = [300.0] * ns, [1000.0] * ns
    low, high = [[0.0] * 7 for _ in range(ns)], [[0.0] * 7 for _ in range(ns)]
    lines = (chem / "therm.dat").read_text().splitlines()
    seen = set()
    i = 2  # THERMO, then the global temperature line
    while i < len(lines):
        line = lines[i]
        key = line[:18].split()[0].upper() if line[:18].split() else ""
        if key.startswith("END") or key.startswith("REAC") or key.startswith("TRAN"):
            break
        if key not in idx or key in seen:
            i += 4
            continue
        sp = idx[key]
        t_low[sp] = float(line[45:55])
        tm = line[65:75].split()
        if tm:
            t_mid[sp] = float(tm[0])
        comp = {}
        for e in range(4):
            f = line[24 + 5 * e: 29 + 5 * e].strip()
            if not f or f[0] == "0":
                break
            el, cnt = f.split()[0].upper(), int(f.split()[1])
            comp[el] = cnt
        w = 0.0
        for el in sorted(comp):  # the reference sums over its std::map of elements
            w += _ATOMIC_WEIGHT[el] * comp[el]
        mw[sp] = w
        c = []
        for r in range(3):
            row = lines[i + 1 + r]
            c += [float(row[15 * q: 15 * q + 15]) for q in range(4 if r == 2 else 5)]
        high[sp] = c[0:7]
        low[sp] = c[7:14]
        seen.add(key)
        i += 4
    lj_inv, vis_coeff = [0.0] * ns, [0.0] * ns
    for line in (chem / "tran.dat").read_text().splitlines():
        parts = line.split()
        if not parts or parts[0][0] == "!":
            continue
        name = parts[0].upper()
        if name in idx and vis_coeff[idx[name]] == 0.0:
            sp = idx[name]
            eps_k, sigma = float(parts[2]), float(parts[3])
            lj_inv[sp] = 1.0 / eps_k
            vis_coeff[sp] = 2.6693e-6 * math.sqrt(mw[sp]) / (sigma * sigma)
    return {"species": species, "mw": mw, "t_low": t_low, "t_mid": t_mid, "low": low, "high": high,
            "lj_inv": lj_inv, "vis_coeff": vis_coeff}


def inflow_state(case: Path, bc: dict) -> dict:
    """The primitive state of an inflow boundary condition of a 9-species
    k-omega SST case as the reference computes it (src/BoundCond.cpp:8-109):
    mass fractions as given, W = 1/sum(Y/W_k), mixture viscosity by Wilke's
    rule over Chapman-Enskog species viscosities (src/Transport.cu:11-38),
    gamma from the NASA-7 cp (cp/cv), velocity = Mach x speed of sound,
    density from the ideal gas, tke = 1.5 (TI |V|)^2, mu_t = ratio x mu,
    omega = rho tke / mu_t.  Returns u, v, w, density, pressure, temperature,
    sv (ns mass fractions, tke, omega) and mut."""
    m = _mixture_data(case)
    ns = len(m["species"])
    mw_k = m["mw"]
    Y = [0.0] * ns
    for name, y in bc.get("Y", {}).items():
        Y[m["species"].index(name.upper())] = float(y)
    inv = 0.0
    for k in range(ns):
        inv += Y[k] / mw_k[k]
    mw = 1.0 / inv
    T, p = float(bc["temperature"]), float(bc["pressure"])
    x = [Y[k] * mw / mw_k[k] for k in range(ns)]
    mu = []
    for k in range(ns):
        tdl = T * m["lj_inv"][k]
        om = 1.147 * math.pow(tdl, -0.145) + math.pow(tdl + 0.5, -2)
        mu.append(m["vis_coeff"][k] * math.sqrt(T) / om)
    visc = 0.0
    for i in range(ns):
        den = 0.0
        for j in range(ns):
            if i == j:
                phi = 1.0
            else:
                num = 1 + math.sqrt(mu[i] / mu[j]) * math.pow(mw_k[j] / mw_k[i], 0.25)
                phi = num * num * (1.0 / math.sqrt(8 * (1 + mw_k[i] / mw_k[j])))
            den += phi * x[j]
        visc += mu[i] * x[i] / den
    cp = cv = 0.0
    t2 = T * T
    t3 = t2 * T
    t4 = t3 * T
    for k in range(ns):
        if T < m["t_low"][k]:
            tt = m["t_low"][k]
            tt2 = tt * tt
            tt3 = tt2 * tt
            c = m["low"][k]
            cpk = c[0] + c[1] * tt + c[2] * tt2 + c[3] * tt3 + c[4] * (tt3 * tt)
        else:
            c = m["low"][k] if T < m["t_mid"][k] else m["high"][k]
            cpk = c[0] + c[1] * T + c[2] * t2 + c[3] * t3 + c[4] * t4
        cpk *= RU / mw_k[k]
        cp += Y[k] * cpk
        cv += Y[k] * (cpk - RU / mw_k[k])
    gamma = cp / cv
    vel = float(bc["mach"]) * math.sqrt(gamma * RU / mw * T)
    rho = p * mw / (RU * T)
    mut = float(bc.get("mut_ratio", 1.0)) * visc
    tke = 1.5 * vel * vel * float(bc.get("ti", 0.01)) * float(bc.get("ti", 0.01))
    sv = Y + [tke, rho * tke / mut]
    return {"u": float(bc["u"]) * vel, "v": float(bc["v"]) * vel, "w": float(bc["w"]) * vel, "density": rho,
            "pressure": p, "temperature": T, "sv": sv, "mut": mut, "mw": mw_k}


def _read_grid(case: Path) -> list[tuple[np.ndarray, np.ndarray, np.ndarray]]:
    """The blocks' (x, y, z) of the case's grid file, shape (mz, my, mx) each."""
    tok = (Path(case) / "input_files" / "grid" / "grid   0.grd").read_text().split()
    nb = int(tok[0])
    dims = [tuple(int(v) for v in tok[1 + 3 * b: 4 + 3 * b]) for b in range(nb)]
    pos = 1 + 3 * nb
    vals = np.array(tok[pos:], dtype=np.float64)
    out, o = [], 0
    for mx, my, mz in dims:
        n = mx * my * mz
        xyz = [vals[o + q * n: o + (q + 1) * n].reshape(mz, my, mx) for q in range(3)]
        o += 3 * n
        out.append(tuple(xyz))
    return out


def _blend_initial_field(case: Path, delta: float = 5e-4,
                         spikes: list[tuple[int, int, int, float, float]] | None = None) -> None:
    """Writes output/field/flowfield.plt with a tanh blend (thickness delta)
    of the two inflow states (UPPER and LOWER) across y = 0.025 m, plus
    step.txt and residual_scale.txt, so that a run with initial = 1 starts
    from it.  spikes: (i, j, k, f_rho, f_p) cells of block 0 whose density
    and pressure are multiplied by f_rho and f_p (the temperature by
    f_p / f_rho, the ideal-gas state), to put unphysical states in front of
    limit_flow.  Pure NumPy: generating a case loads no native library."""
    from .plt import write_plt

    up, lo = inflow_state(case, UPPER), inflow_state(case, LOWER)
    species = _species_names(case)
    ns = len(species)
    mw_k = up["mw"]
    names = ["x", "y", "z", "density", "u", "v", "w", "pressure", "temperature", "mach"] + species + [
        "tke", "omega", "mut"]
    zones = []
    for x, y, z in _read_grid(case):
        phi = 0.5 * (1.0 + np.tanh((y - 0.025) / delta))
        mix = lambda a, b: phi * b + (1.0 - phi) * a  # noqa: E731
        zone = {"x": x, "y": y, "z": z}
        zone["u"] = mix(lo["u"], up["u"])
        zone["v"] = np.zeros_like(x)
        zone["w"] = np.zeros_like(x)
        zone["pressure"] = np.full_like(x, up["pressure"])
        zone["temperature"] = mix(lo["temperature"], up["temperature"])
        Y = [mix(lo["sv"][l], up["sv"][l]) for l in range(ns)]
        mw = 1.0 / sum(Y[l] / mw_k[l] for l in range(ns))
        zone["density"] = zone["pressure"] * mw / (RU * zone["temperature"])
        zone["mach"] = np.zeros_like(x)
        for l, n in enumerate(species):
            zone[n] = Y[l]
        zone["tke"] = mix(lo["sv"][ns], up["sv"][ns])
        zone["omega"] = mix(lo["sv"][ns + 1], up["sv"][ns + 1])
        zone["mut"] = mix(lo["mut"], up["mut"])
        if spikes and not zones:
            for i, j, k, f_rho, f_p in spikes:
                zone["density"][k, j, i] *= f_rho
                zone["pressure"][k, j, i] *= f_p
                # the temperature the reference derives from them
                zone["temperature"][k, j, i] *= f_p / f_rho
        zones.append(zone)
    write_plt(case / "output" / "field" / "flowfield.plt", names, zones)
    msg = case / "output" / "message"
    msg.mkdir(parents=True, exist_ok=True)
    (msg / "step.txt").write_text("0")
    (msg / "residual_scale.txt").write_text("1\n1\n1\n1\n")


def _species_names(case: Path) -> list[str]:
    text = (Path(case) / "input_files" / "chemistry" / "combustion_mechanism.inp").read_text().split()
    i = text.index("SPECIES") + 1
    out = []
    while text[i].upper() != "END":
        out.append(text[i].upper())
        i += 1
    return out


def mixing_layer_case(case: str | Path, mx: int = 384, my: int = 192, mz: int = 64, total_step: int = 2000,
                      output_screen: int = 100, output_file: int | None = None, cfl: float = 0.5,
                      dplur: int = 4, chem: int = 1, implicit: int = 1,
                      spikes: list[tuple[int, int, int, float, float]] | None = None, wall_j0: bool = False) -> Path:
    """3-D supersonic H2 / vitiated-air mixing layer (0.3 x 0.05 x 0.02 m,
    y clustered at the splitter y = 0.025 m).  Upper stream Mach 2.4, 1250 K,
    Y_O2 0.245, Y_H2O 0.175, N2; lower stream H2 / N2 (0.4 / 0.6) at
    Mach 1.2, 300 K; 1 atm; 9 species / 19 reactions, k-omega SST with 1 %
    inflow turbulence, DPLUR with `dplur` sweeps, chemistry treatment `chem`
    (1 point-implicit EPI, 2 diagonal).  spikes: cells whose initial density
    and pressure are scaled (see _blend_initial_field).  wall_j0: the j = 0
    face is an isothermal 300 K wall instead of a symmetry plane (the SST
    wall distance then has mx x mz wall points)."""
    case = Path(case)
    x, y, z = _mixing_layer_grid(mx, my, mz)
    write_grid(case, [(x, y, z)])
    js = int(np.searchsorted(y[0, :, 0], 0.025))
    write_boundary(case, [[
        (0, 0, js, my - 1, 0, mz - 1, 5),
        (0, 0, 0, js - 1, 0, mz - 1, 9),
        (mx - 1, mx - 1, 0, my - 1, 0, mz - 1, 6),
        (0, mx - 1, 0, 0, 0, mz - 1, 2 if wall_j0 else 3),
        (0, mx - 1, my - 1, my - 1, 0, mz - 1, 3),
        (0, mx - 1, 0, my - 1, 0, 0, 3),
        (0, mx - 1, 0, my - 1, mz - 1, mz - 1, 3),
    ]])
    copy_chemistry(case)
    _mixing_setup(case, total_step=total_step, output_screen=output_screen, output_file=output_file or 10 ** 9,
                  initial=0, cfl=cfl, dplur=dplur, chem=chem, implicit=implicit, wall=wall_j0)
    _blend_initial_field(case, spikes=spikes)
    _mixing_setup(case, total_step=total_step, output_screen=output_screen, output_file=output_file or 10 ** 9,
                  initial=1, cfl=cfl, dplur=dplur, chem=chem, implicit=implicit, wall=wall_j0)
    return case


def multiblock_case(case: str | Path, mxs: list[int], my: int = 64, mz: int = 32, total_step: int = 100,
                    output_screen: int = 10, output_file: int | None = None, cfl: float = 0.5,
                    dplur: int = 4) -> Path:
    """Mixing-layer physics on len(mxs) blocks tiled along x (1:1 faces):
    block b spans mxs[b] points and shares its first plane with the last
    plane of block b-1."""
    case = Path(case)
    total = sum(mxs) - (len(mxs) - 1)
    x_all, y_all, z_all = _mixing_layer_grid(total, my, mz)
    blocks, faces, inner = [], [], []
    i0 = 0
    nb = len(mxs)
    js = int(np.searchsorted(y_all[0, :, 0], 0.025))
    for b, m in enumerate(mxs):
        sl = slice(i0, i0 + m)
        blocks.append((x_all[:, :, sl], y_all[:, :, sl], z_all[:, :, sl]))
        fl = []
        if b == 0:
            fl += [(0, 0, js, my - 1, 0, mz - 1, 5), (0, 0, 0, js - 1, 0, mz - 1, 9)]
        if b == nb - 1:
            fl.append((m - 1, m - 1, 0, my - 1, 0, mz - 1, 6))
        fl += [(0, m - 1, 0, 0, 0, mz - 1, 3), (0, m - 1, my - 1, my - 1, 0, mz - 1, 3),
               (0, m - 1, 0, my - 1, 0, 0, 3), (0, m - 1, 0, my - 1, mz - 1, mz - 1, 3)]
        faces.append(fl)
        il = []
        # 1-based ranges; the negative j range marks the first tangential
        # direction of a 3-D face (src/Mesh.cpp:84-106).
        if b > 0:
            prev = mxs[b - 1]
            il.append(((1, 1, -1, -my, 1, mz, b + 1), (prev, prev, -1, -my, 1, mz, b)))
        if b < nb - 1:
            il.append(((m, m, -1, -my, 1, mz, b + 1), (1, 1, -1, -my, 1, mz, b + 2)))
        inner.append(il)
        i0 += m - 1
    write_grid(case, blocks)
    write_boundary(case, faces, inner)
    copy_chemistry(case)
    _mixing_setup(case, total_step=total_step, output_screen=output_screen, output_file=output_file or 10 ** 9,
                  initial=0, cfl=cfl, dplur=dplur, chem=1)
    _blend_initial_field(case)
    _mixing_setup(case, total_step=total_step, output_screen=output_screen, output_file=output_file or 10 ** 9,
                  initial=1, cfl=cfl, dplur=dplur, chem=1)
    return case


def batched_block_sizes(seed: int, n_blocks: int = 12, lo: tuple[int, int, int] = (32, 32, 32),
                        hi: tuple[int, int, int] = (160, 96, 64)) -> tuple[list[int], int, int]:
    """Block sizes of the batched multi-block workload: n_blocks blocks tiled
    along x with 1:1 faces, so every block shares one (my, mz) and only mx
    varies; each drawn uniformly between lo and hi from `seed`.  Returns
    (mxs, my, mz).  With the bounds 32x32x32 .. 160x96x64, twelve blocks hold
    at most 11.8 M cells."""
    rng = np.random.default_rng(seed)
    my = int(rng.integers(lo[1], hi[1] + 1))
    mz = int(rng.integers(lo[2], hi[2] + 1))
    mxs = [int(v) for v in rng.integers(lo[0], hi[0] + 1, size=n_blocks)]
    return mxs, my, mz


def batched_multiblock_case(case: str | Path, seed: int = 0, n_blocks: int = 12, total_step: int = 100,
                            output_screen: int = 10, output_file: int | None = None, dplur: int = 4,
                            lo: tuple[int, int, int] = (32, 32, 32),
                            hi: tuple[int, int, int] = (160, 96, 64)) -> Path:
    """The mixing-layer physics on n_blocks seeded blocks (batched_block_sizes)
    tiled along x with 1:1 inner faces: the batched multi-block workload."""
    mxs, my, mz = batched_block_sizes(seed, n_blocks, lo, hi)
    return multiblock_case(case, mxs, my=my, mz=mz, total_step=total_step, output_screen=output_screen,
                           output_file=output_file, dplur=dplur)

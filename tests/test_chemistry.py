"""CHEMKIN reader and chemistry known-answer / conservation checks (CPU).

The reference ships no tests; these pin the parse of its own mechanism
(input_files/chemistry) and physical invariants of the oracle's chemistry."""
import ctypes as C

import numpy as np
import pytest

import openstc_b200 as ostc
from openstc_b200 import cases
from oracle_bridge import oracle_lib, orc_params_from

R_U, R_C = 8314.462618, 1.98720425864083
SPECIES = ["H2", "H", "O2", "O", "OH", "HO2", "H2O2", "H2O", "N2"]
ELEMENTS = {"H2": (2, 0, 0), "H": (1, 0, 0), "O2": (0, 2, 0), "O": (0, 1, 0), "OH": (1, 1, 0), "HO2": (1, 2, 0),
            "H2O2": (2, 2, 0), "H2O": (2, 1, 0), "N2": (0, 0, 2)}  # (H, O, N)


@pytest.fixture(scope="module")
def drv(case_factory):
    case = case_factory("ml", cases.mixing_layer_case, mx=12, my=10, mz=6, total_step=2, output_screen=1)
    return ostc.Driver(case)


@pytest.fixture(scope="module")
def params(drv):
    return drv.params()


def test_mechanism_shape(params):
    assert params.ns == 9 and params.nr == 19
    labels = list(params.label[:19])
    # third body (4) for the four "+M" reactions, Troe (6) for the two (+M)
    # fall-off reactions, DUPLICATE pairs merged into one type-3 reaction each
    assert labels == [1, 1, 1, 1, 4, 4, 4, 4, 6, 1, 1, 1, 1, 3, 6, 1, 1, 1, 3]


def test_molecular_weights(params):
    w = {"H": 1.008, "O": 15.999, "N": 14.007}
    for k, name in enumerate(SPECIES):
        h, o, n = ELEMENTS[name]
        expect = 0.0
        for sym, cnt in sorted({"H": h, "N": n, "O": o}.items()):  # element map order
            expect += w[sym] * cnt
        assert params.mw[k] == expect


def test_activation_energies_and_dup(params):
    # main-line Ea divided by R_c; LOW Ea kept in the file's units (reference quirk)
    assert params.Ea[0] == 1.66e4 / R_C
    assert params.A2[8] == 6.37e20 and params.b2[8] == -1.72 and params.Ea2[8] == 5.25e2
    # HO2+HO2 duplicate pair: second Arrhenius set, Ea divided by R_c
    assert params.A[13] == 4.2e14 and params.A2[13] == 1.3e11 and params.Ea2[13] == -1.63e3 / R_C
    # Troe parameters of H+O2(+M)
    assert (params.troe_alpha[8], params.troe_t3[8], params.troe_t1[8]) == (0.8, 1e-30, 1e30)
    # third-body efficiencies of H+O2(+M): H2 2.0, H2O 11.0, O2 0.78, others 1
    tb = [params.third_body[8 * 9 + k] for k in range(9)]
    assert tb == [2.0, 1.0, 0.78, 1.0, 1.0, 1.0, 1.0, 11.0, 1.0]
    # reaction orders: H2+M=H+H+M is +1, O+O+M=O2+M is -1
    assert params.order[4] == 1 and params.order[5] == -1


def test_nasa7_cp_known_values(drv, params):
    """cp(298.15 K) from the therm.dat coefficients, evaluated here directly."""
    p = orc_params_from(params)
    h = np.zeros(20)
    cp = np.zeros(20)
    oracle_lib().orc_enthalpy_cp(C.byref(p), 298.15, h.ctypes.data_as(C.POINTER(C.c_double)),
                                 cp.ctypes.data_as(C.POINTER(C.c_double)))
    # N2's own line sets T_low = 300 K, so below it cp is frozen at cp(300 K)
    # (src/Thermo.cu:47-61); its low-range coefficients from therm.dat:
    assert params.t_low[8] == 300.0
    t = 300.0
    a = [0.03298677e2, 0.14082404e-2, -0.03963222e-4, 0.05641515e-7, -0.02444854e-10]
    cp_n2 = (a[0] + a[1] * t + a[2] * t ** 2 + a[3] * t ** 3 + a[4] * t ** 4) * R_U / params.mw[8]
    assert cp[8] == pytest.approx(cp_n2, rel=1e-13)
    assert cp[8] == pytest.approx(1040.0, rel=0.01)  # tabulated cp of N2 at 298 K
    assert cp[7] == pytest.approx(1864.0, rel=0.01)  # H2O
    assert cp[0] == pytest.approx(14300.0, rel=0.01)  # H2


def _source(params, rho, t, Y):
    p = orc_params_from(params)
    om = np.zeros(20)
    jac = np.zeros(400)
    Yc = np.zeros(20)
    Yc[:9] = Y
    oracle_lib().orc_chemical_source(C.byref(p), rho, t, Yc.ctypes.data_as(C.POINTER(C.c_double)),
                                     om.ctypes.data_as(C.POINTER(C.c_double)),
                                     jac.ctypes.data_as(C.POINTER(C.c_double)))
    return om[:9], jac[:81].reshape(9, 9)


@pytest.mark.parametrize("t", [900.0, 1500.0, 2400.0])
def test_source_conserves_mass_and_elements(params, t):
    rng = np.random.default_rng(int(t))
    Y = rng.dirichlet(np.ones(9))
    om, _ = _source(params, 0.3, t, Y)
    scale = np.max(np.abs(om))
    assert scale > 0
    assert abs(om.sum()) < 1e-12 * scale
    for e in range(3):
        moles = sum(ELEMENTS[s][e] * om[k] / params.mw[k] for k, s in enumerate(SPECIES))
        assert abs(moles) < 1e-12 * scale


def test_jacobian_columns_conserve_mass_and_elements(params):
    """Every reaction conserves mass and elements, so each column of the EPI
    Jacobian sums to zero, by mass and by element moles."""
    rng = np.random.default_rng(7)
    Y = rng.dirichlet(np.ones(9)) * 0.9 + 0.1 / 9
    _, J = _source(params, 0.25, 1800.0, Y)
    scale = np.max(np.abs(J))
    assert scale > 0
    assert np.max(np.abs(J.sum(axis=0))) < 1e-12 * scale
    for e in range(3):
        w = np.array([ELEMENTS[s][e] / params.mw[k] for k, s in enumerate(SPECIES)])
        assert np.max(np.abs(w @ J)) < 1e-12 * scale


def test_epi_increment_conserves_mass(params):
    p = orc_params_from(params)
    Y = np.zeros(20)
    Y[:9] = [0.02, 1e-4, 0.2, 1e-4, 1e-3, 1e-5, 1e-6, 0.1, 0.0]
    Y[8] = 1.0 - Y[:8].sum()
    dY = np.zeros(20)
    oracle_lib().orc_epi_increment(C.byref(p), 0.2, 1800.0, Y.ctypes.data_as(C.POINTER(C.c_double)), 1e-6,
                                   dY.ctypes.data_as(C.POINTER(C.c_double)))
    assert np.max(np.abs(dY[:9])) > 0
    assert abs(dY[:9].sum()) < 1e-12 * np.max(np.abs(dY[:9]))

"""The cases of the golden fixtures (tests/golden), shared by the fixture
generator and the tests that read the fixtures.

name -> (case builder, keyword arguments, steps recorded).  Every case is
small enough for the CPU oracle; each exercises a branch of the path:
  ramp         2-D laminar air, explicit (the 48 x 24 ramp)
  ml           3-D 9-species SST mixing layer, DPLUR 4 sweeps, EPI chemistry
  ml_explicit  the same, explicit, EPI point-implicit chemistry stage
  mb           two blocks with an inner face
  ml_da        the mixing layer with the diagonal (DA) stiff chemistry
               (chemSrcMethod = 2, src/FiniteRateChem.cu:196-209, 400-412)
  ml_limit     the mixing layer with one cell (i = 12) whose initial density
               and pressure are 1100 times its neighbours': after the first
               update it and the cells its blast empties leave the flow bounds
               (1000 rho_inf, 1e-6 rho_inf, 1e-6 .. 1000 p_inf), and
               limit_flow (src/TimeAdvanceFunc.cu:34-224) sets them to the
               clamped state with sv_inf.  Every flagged cell has i >= 7 > mz,
               so the reference's neighbour loop, which bounds i1 by mz = 6
               (:84), skips all their neighbours: this branch reads no
               neighbour value and is deterministic in the reference, whose
               averaging branch races when flagged cells are adjacent (each
               thread reads neighbours that others overwrite).  The averaging
               branch is checked against the oracle on an isolated cell
               (test_gpu_parity.py).
"""
from openstc_b200 import cases

SPIKES = [(12, 8, 2, 1100.0, 1100.0)]

FIXTURES = {
    "ramp": (cases.ramp_case, dict(mx=48, my=24), (1, 10, 100)),
    "ml": (cases.mixing_layer_case, dict(mx=16, my=12, mz=6), (1, 10, 100)),
    "ml_explicit": (cases.mixing_layer_case, dict(mx=16, my=12, mz=6, implicit=0), (1, 10, 100)),
    "mb": (cases.multiblock_case, dict(mxs=[10, 8], my=12, mz=6), (1, 10, 100)),
    "ml_da": (cases.mixing_layer_case, dict(mx=16, my=12, mz=6, chem=2), (1, 10, 100)),
    "ml_limit": (cases.mixing_layer_case, dict(mx=16, my=12, mz=6, spikes=SPIKES), (1,)),
}


def builder(name):
    fn, kw, _ = FIXTURES[name]
    return fn, kw


def parse_history(rows) -> dict:
    """{step: err_max} from the fixture's history array."""
    return {int(r[0]): float(r[1]) for r in rows}

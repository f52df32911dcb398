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
  ml_limit     the mixing layer with two cells whose initial density and
               pressure are 1100 times their neighbours': after the first
               update both exceed 1000 rho_inf, so limit_flow
               (src/TimeAdvanceFunc.cu:34-224) replaces them, the one at i = 2
               by the average of its good neighbours, the one at i = 12 by the
               clamped state and sv_inf, because the reference bounds the
               neighbour index i1 by mz = 6 (:84) and every neighbour of
               i = 12 is skipped
"""
from openstc_b200 import cases

SPIKES = [(2, 5, 3, 1100.0), (12, 8, 2, 1100.0)]

FIXTURES = {
    "ramp": (cases.ramp_case, dict(mx=48, my=24), (1, 10, 100)),
    "ml": (cases.mixing_layer_case, dict(mx=16, my=12, mz=6), (1, 10, 100)),
    "ml_explicit": (cases.mixing_layer_case, dict(mx=16, my=12, mz=6, implicit=0), (1, 10, 100)),
    "mb": (cases.multiblock_case, dict(mxs=[10, 8], my=12, mz=6), (1, 10, 100)),
    "ml_da": (cases.mixing_layer_case, dict(mx=16, my=12, mz=6, chem=2), (1, 10, 100)),
    "ml_limit": (cases.mixing_layer_case, dict(mx=16, my=12, mz=6, spikes=SPIKES), (1, 2)),
}


def builder(name):
    fn, kw, _ = FIXTURES[name]
    return fn, kw


def parse_history(rows) -> dict:
    """{step: err_max} from the fixture's history array."""
    return {int(r[0]): float(r[1]) for r in rows}

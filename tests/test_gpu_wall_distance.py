"""The SST wall distance: the exact bucket search (ostc_options.wall_distance
= 2) against the reference's brute force over every wall point
(src/Driver.cu:461-482; option 1), on a mixing layer whose j = 0 face is a
wall: the same values bit for bit at every point of the ghosted grid, and
both within rounding of a NumPy evaluation of the same formula."""
import time

import numpy as np
import pytest

import openstc_b200 as ostc
from openstc_b200 import cases

pytestmark = pytest.mark.gpu


def wall_points(drv):
    """x, y, z of the wall-face points the library registers (ranges trimmed
    by ngg in the tangential directions, src/BoundCond.cu:215-229)."""
    g = drv.layout("x")[0]
    x, y, z = (drv.host_field(0, f)[0] for f in ("x", "y", "z"))
    pts = []
    for bc in drv.bcs():
        if bc.type != 2:
            continue
        (i0, j0, k0), (i1, j1, k1) = bc.start, bc.end
        sl = (slice(k0 + g, k1 + g + 1), slice(j0 + g, j1 + g + 1), slice(i0 + g, i1 + g + 1))
        pts.append(np.stack([x[sl].ravel(), y[sl].ravel(), z[sl].ravel()], axis=1))
    return np.concatenate(pts), (x, y, z)


@pytest.mark.parametrize("size", [(48, 24, 16), (96, 40, 24), (256, 96, 64)])
def test_bucket_search_equals_brute_force(tmp_path, size):
    mx, my, mz = size
    case = cases.mixing_layer_case(tmp_path / "w", mx=mx, my=my, mz=mz, total_step=1, wall_j0=True)
    out, secs = {}, {}
    for method in ("brute", "grid"):
        d = ostc.Driver(case, wall_distance=method)
        t0 = time.perf_counter()
        d.initialize()
        secs[method] = time.perf_counter() - t0
        out[method] = d.get(0, "wall_dist")
        if method == "grid":
            pts, (x, y, z) = wall_points(d)
        d.close()
    assert np.array_equal(out["brute"], out["grid"])
    # a NumPy restatement on a sample of points
    rng = np.random.default_rng(1)
    flat = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)
    sample = rng.choice(flat.shape[0], 2000, replace=False)
    d2 = ((flat[sample, None, :] - pts[None, :, :]) ** 2).sum(axis=2).min(axis=1)
    ref = np.sqrt(np.minimum(d2, 1e6))
    got = out["grid"].ravel()[sample]
    assert np.all(np.abs(got - ref) <= 1e-12 * np.maximum(ref, 1e-30) + 1e-18)
    print(f"{size}: {pts.shape[0]} wall points; initialize {secs['brute']:.3f} s brute force, "
          f"{secs['grid']:.3f} s bucket search")

"""Single-plane-symmetric sections (cross_sectional_shape 3) on the GPU: the
trace of a shape-3 vowel tube equals the oracle engine's FP32 trace on the
same maps (reference arithmetic), and the fast_math trace stays as close to
the double-precision trace as the reference arithmetic does.  The maps
themselves are checked on the CPU (tests/test_shapes.py)."""
import numpy as np
import pytest

import oracle as O
import vocalsim_b200 as V
from vocalsim_b200 import synthetic as S
from vocalsim_b200.autograd import tube_layout

pytestmark = pytest.mark.gpu

STEPS = 1500


def rel_l2(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def tube():
    L, A = S.vowel_tube(2, n=8)
    p = V.params(cross_sectional_shape=3)
    g = V.Geometry(L, A)
    return L, A, V.build_maps(p, g), tube_layout(p, g)


def oracle_trace(L, A, maps, layout, f64=False, **kw):
    O.set_sps_diameters(layout["major"])
    try:
        run = O.run_maps_f64 if f64 else O.run_maps_f32
        return run(O.params(cross_sectional_shape=3, **kw), O.Geometry(L, A), STEPS, maps["depth_p"],
                   maps["depth_x"], maps["depth_y"], maps["dims"]["z_inv_val"])
    finally:
        O.set_sps_diameters([])


@pytest.mark.parametrize("kw", [dict(), dict(source_type=2, tmm_ps_pa=800.0)])
def test_shape3_trace_equals_oracle(tube, kw, cuda_ok):
    L, A, maps, layout = tube
    tr = V.Solver(V.params(cross_sectional_shape=3, **kw), V.Geometry(L, A)).run(STEPS)
    ref = oracle_trace(L, A, maps, layout, **kw)
    assert np.array_equal(tr, ref)
    assert np.abs(tr).max() > 0


def test_shape3_fast_math_close_to_double(tube, cuda_ok):
    L, A, maps, layout = tube
    tr = V.Solver(V.params(cross_sectional_shape=3, fast_math=1), V.Geometry(L, A)).run(STEPS)
    r32 = oracle_trace(L, A, maps, layout)
    r64 = oracle_trace(L, A, maps, layout, f64=True)
    assert rel_l2(tr, r64) <= max(2 * rel_l2(r32, r64), 1e-5)

"""The library's GPU time loop against the reference's own engine.

tests/golden/reference_engine.npz holds record_pressure of the reference's
FDTDEngineCPU run after its own setupWaveSolver (built from the reference
sources, tests/golden/make_reference_engine.py).  The library is given the
reference's own depth maps and z_inv (vs_batch_set_maps; the cell types it
builds itself equal the reference's in every case), so the comparison covers
the time loop whatever the reference's depth kernels computed.  vs_run in the
reference arithmetic (fast_math = 0) must give the same trace bit for bit; a
single tube runs on the cluster kernel by default, the strip kernels are run
too.  With the reciprocal form (fast_math = 1) the trace stays within the
FP32 reference's own distance from the FP64 engine on the same maps (x2 +
1e-6).  Where the reference engine is built here (oracle/_ref/ref_engine),
two circular-section cases are also run live, to show the fixture is what
that binary computes on this machine.
"""
import json
from pathlib import Path

import numpy as np
import pytest

import oracle as O
import vocalsim_b200 as V

GOLD = Path(__file__).parent / "golden" / "reference_engine.npz"
if not GOLD.exists():
    pytest.skip("tests/golden/reference_engine.npz not generated", allow_module_level=True)
G = np.load(GOLD)
CASES = json.loads(str(G["cases_json"]))
IDS = [f"c{c['case']}-{c['geometry']}" for c in CASES]
STRIP_SHAPE = 7


def inputs(c):
    i = c["case"]
    geo = (G[f"c{i}_length_cm"], G[f"c{i}_area_cm2"]) if f"c{i}_length_cm" in G else None
    return dict(c["params"]), geo


def reference_maps(c):
    i = c["case"]
    zmap = G[f"c{i}_z_inv"]
    zval = float(zmap[zmap != 0][0]) if np.any(zmap != 0) else 0.0
    return G[f"c{i}_depth_p"], G[f"c{i}_depth_x"], G[f"c{i}_depth_y"], zval


def run_on_reference_maps(c, shape=None, **extra):
    kw, geo = inputs(c)
    b = V.Batch([V.params(**kw, **extra)], [V.Geometry(*geo) if geo is not None else None])
    dp, dx, dy, zval = reference_maps(c)
    b.set_maps(0, dp, dx, dy, zval)
    if shape is not None:
        b.set_tile(shape)
    tr = b.run(c["steps"])[0]
    b.close()
    return tr


@pytest.mark.gpu
@pytest.mark.parametrize("c", CASES, ids=IDS)
def test_gpu_trace_equals_the_reference_engine(cuda_ok, c):
    ref = G[f"c{c['case']}_trace"]
    for shape in (None, STRIP_SHAPE):          # default (cluster kernel), strip kernel
        tr = run_on_reference_maps(c, shape)
        assert np.array_equal(tr, ref), f"shape {shape}: first difference at step {int(np.argmax(tr != ref))}"


@pytest.mark.gpu
@pytest.mark.parametrize("c", [c for c in CASES if c["params"].get("source_type", 1) != 2][:8],
                         ids=lambda c: f"c{c['case']}")
def test_gpu_fast_math_within_the_reference_rounding(cuda_ok, c):
    kw, geo = inputs(c)
    dp, dx, dy, zval = reference_maps(c)
    d = O.run_maps_f64(O.params(**kw), O.Geometry(*geo) if geo is not None else None, c["steps"],
                       dp.astype(np.float64), dx.astype(np.float64), dy.astype(np.float64), zval)
    ref = G[f"c{c['case']}_trace"].astype(np.float64)
    tr = run_on_reference_maps(c, None, fast_math=1).astype(np.float64)
    rel = lambda a: np.linalg.norm(a - d) / np.linalg.norm(d)  # noqa: E731
    assert rel(tr) <= 2 * rel(ref) + 1e-6, (rel(tr), rel(ref))


@pytest.mark.gpu
@pytest.mark.skipif(not O.REF_ENGINE.exists(), reason="oracle/_ref/ref_engine not built")
@pytest.mark.parametrize("case", [0, 10])
def test_reference_engine_reproduces_the_fixture(cuda_ok, case):
    c = next(x for x in CASES if x["case"] == case)
    kw, geo = inputs(c)
    steps = min(c["steps"], 600)
    r = O.reference_engine(O.params(**kw), O.Geometry(*geo) if geo is not None else None, steps)
    assert np.array_equal(r["trace"], G[f"c{case}_trace"][:steps])
    assert np.array_equal(r["cell_type"], G[f"c{case}_cell_type"].astype(np.int32))
    assert np.array_equal(r["depth_x"], G[f"c{case}_depth_x"])

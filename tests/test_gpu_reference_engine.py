"""The library's GPU time loop against the reference's own engine.

tests/golden/reference_engine.npz holds record_pressure of the reference's
FDTDEngineCPU run after its own setupWaveSolver (built from the reference
sources, tests/golden/make_reference_engine.py).  vs_run in the reference
arithmetic (fast_math = 0) must give the same trace bit for bit; with the
reciprocal form (fast_math = 1) the trace stays within the FP32 reference's
own distance from the double-precision restatement (x2 + 1e-6).  Where the
reference engine is built here (oracle/_ref/ref_engine) two cases are also
run live, to show the fixture is what that binary computes on this machine.
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


def inputs(c):
    i = c["case"]
    geo = (G[f"c{i}_length_cm"], G[f"c{i}_area_cm2"]) if f"c{i}_length_cm" in G else None
    return dict(c["params"]), geo


@pytest.mark.gpu
@pytest.mark.parametrize("c", CASES, ids=IDS)
def test_gpu_trace_equals_the_reference_engine(cuda_ok, c):
    kw, geo = inputs(c)
    ref = G[f"c{c['case']}_trace"]
    s = V.Solver(V.params(**kw), V.Geometry(*geo) if geo is not None else None)
    tr = s.run(c["steps"])
    s.close()
    assert np.array_equal(tr, ref), f"first difference at step {int(np.argmax(tr != ref))}"


@pytest.mark.gpu
@pytest.mark.parametrize("c", [c for c in CASES if c["params"].get("source_type", 1) != 2][:6], ids=lambda c: f"c{c['case']}")
def test_gpu_fast_math_within_the_reference_rounding(cuda_ok, c):
    kw, geo = inputs(c)
    ref = G[f"c{c['case']}_trace"].astype(np.float64)
    g64 = O.Geometry(*geo) if geo is not None else None
    d = O.run(O.params(**kw), g64, c["steps"], "f64")
    s = V.Solver(V.params(**kw, fast_math=1), V.Geometry(*geo) if geo is not None else None)
    tr = s.run(c["steps"]).astype(np.float64)
    s.close()
    rel = lambda a: np.linalg.norm(a - d) / np.linalg.norm(d)  # noqa: E731
    assert rel(tr) <= 2 * rel(ref) + 1e-6, (rel(tr), rel(ref))


@pytest.mark.gpu
@pytest.mark.skipif(not O.REF_ENGINE.exists(), reason="oracle/_ref/ref_engine not built")
@pytest.mark.parametrize("case", [1, 9])
def test_reference_engine_reproduces_the_fixture(cuda_ok, case):
    c = next(x for x in CASES if x["case"] == case)
    kw, geo = inputs(c)
    steps = min(c["steps"], 600)
    r = O.reference_engine(O.params(**kw), O.Geometry(*geo) if geo is not None else None, steps)
    assert np.array_equal(r["trace"], G[f"c{case}_trace"][:steps])
    assert np.array_equal(r["cell_type"], G[f"c{case}_cell_type"].astype(np.int32))

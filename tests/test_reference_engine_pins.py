"""Pin the oracle and the library's map builder against the reference's own
grid setup and CPU engine.

tests/golden/reference_engine.npz holds what the reference itself computed:
tests/golden/make_reference_engine.py built SimulationParams, SolverParams,
DeviceSymbols, GlottalExcitations, FDTDSolver, TubeGeometry, TubeDepth,
TwoMassModel and FDTDEngineCPU from the reference sources (oracle/Makefile.ref,
oracle/_ref/ref_engine), ran setupWaveSolver (its CUDA setup kernels) and
startSolverEngine on a B200, and stored the cell-type / depth / z_inv maps,
digests of the 17 coefficient arrays of calculateSolverCoefficients and of the
final P/Vx/Vy frames, and record_pressure.  Every comparison here is exact.
"""
import hashlib
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

# The circular depth radicand r^2 - d^2 (TubeDepth.cu:355-370) is the one map
# expression nvcc can contract into an FMA; the reference's Release-like build
# contracts it, its -G (CMake default Debug) build does not.
RELEASE_DEPTH_FMA = 1
DEBUG_DEPTH_FMA = 0


def case_inputs(c):
    kw = dict(c["params"])
    i = c["case"]
    if f"c{i}_length_cm" in G:
        geo = (G[f"c{i}_length_cm"], G[f"c{i}_area_cm2"])
    else:
        geo = None
    return kw, geo


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


IDS = [f"c{c['case']}-{c['geometry']}-{'-'.join(f'{k}{v}' for k, v in c['params'].items())}" for c in CASES]


@pytest.mark.parametrize("c", CASES, ids=IDS)
@pytest.mark.parametrize("build,fma", [("", RELEASE_DEPTH_FMA), ("g_", DEBUG_DEPTH_FMA)], ids=["release", "debug"])
def test_oracle_maps_equal_the_reference(c, build, fma):
    kw, geo = case_inputs(c)
    i = c["case"]
    m = O.maps(O.params(**kw, depth_fma=fma), O.Geometry(*geo) if geo is not None else None)
    assert [m["dims"]["frame_h"], m["dims"]["frame_w"]] == c["frame"]
    assert [m["dims"]["listener_x"], m["dims"]["listener_y"]] == c["listener"]
    if kw.get("simulation_type", 1) == 1:
        assert [m["dims"]["excitation_x"], m["dims"]["excitation_y"]] == c["excitation"]
    assert np.array_equal(m["cell_type"], G[f"c{i}_{build}cell_type"].astype(np.int32))
    for k in ("depth_p", "depth_x", "depth_y", "z_inv"):
        assert np.array_equal(m[k], G[f"c{i}_{build}{k}"]), k


@pytest.mark.parametrize("c", CASES, ids=IDS)
def test_library_maps_equal_the_reference(c):
    kw, geo = case_inputs(c)
    i = c["case"]
    m = V.build_maps(V.params(**kw, depth_fma=RELEASE_DEPTH_FMA), V.Geometry(*geo) if geo is not None else None)
    assert np.array_equal(m["cell_type"], G[f"c{i}_cell_type"].astype(np.int32))
    for k in ("depth_p", "depth_x", "depth_y", "z_inv"):
        assert np.array_equal(m[k], G[f"c{i}_{k}"]), k


@pytest.mark.parametrize("c", CASES, ids=IDS)
def test_oracle_coefficients_equal_the_reference(c):
    kw, geo = case_inputs(c)
    got = O.coeffs(O.params(**kw, depth_fma=RELEASE_DEPTH_FMA), O.Geometry(*geo) if geo is not None else None)
    bad = [k for k, v in got.items() if digest(v) != c["coeff_sha256"][k]]
    assert not bad, f"coefficient arrays differing from the reference: {bad}"
    assert c["coeff_sha256"] == c["debug_build_coeff_sha256"]


@pytest.mark.parametrize("c", CASES, ids=IDS)
def test_oracle_engine_equals_the_reference_engine(c):
    """record_pressure and the final P/Vx/Vy frames of FDTDEngineCPU, bit for bit."""
    kw, geo = case_inputs(c)
    i = c["case"]
    p = O.params(**kw, depth_fma=RELEASE_DEPTH_FMA)
    g = O.Geometry(*geo) if geo is not None else None
    assert np.array_equal(O.source(p, c["steps"]), G[f"c{i}_excitation"]) or p.source_type == 2
    tr, (P, VX, VY) = O.run(p, g, c["steps"], "f32", fields=True)
    ref = G[f"c{i}_trace"]
    assert np.array_equal(tr, ref), f"first difference at step {int(np.argmax(tr != ref))}"
    assert np.any(ref != 0)
    assert {"p": digest(P), "vx": digest(VX), "vy": digest(VY)} == c["fields_sha256"]

"""Pin the oracle and the library's map builder against the reference's own
grid setup and CPU engine.

tests/golden/reference_engine.npz holds what the reference itself computed:
tests/golden/make_reference_engine.py built SimulationParams, SolverParams,
DeviceSymbols, GlottalExcitations, FDTDSolver, TubeGeometry, TubeDepth,
TwoMassModel and FDTDEngineCPU from the reference sources (oracle/Makefile.ref,
oracle/_ref/ref_engine: a Release-like build, and the -G build of the CMake
default), ran setupWaveSolver (its CUDA setup kernels) and startSolverEngine on
a B200, and stored the cell-type / depth / z_inv maps, digests of the 17
coefficient arrays of calculateSolverCoefficients and of the final P/Vx/Vy
frames, and record_pressure.  Every comparison here is exact.

What the reference defines, and so what is pinned:
* cell types and z_inv maps: every case, both builds;
* depth maps of circular sections: the Release build contracts the radicand
  r^2 - d^2 (TubeDepth.cu:355-370) into an FMA, the -G build does not; they
  equal the builders with depth_fma = 1 and 0 respectively.  2D and
  open-space depths are constants;
* depth maps of elliptical sections are not defined by the reference: it
  builds the minor-axis device vector from begin() and end() of two different
  temporary copies (TubeDepth.cu:147 with the by-value getter of
  TubeGeometry.cu:620), so what the depth kernel reads depends on where the
  heap put the two copies.  The Release-like build never read the tube's axes
  (its maps came out at the 1 mm floor, or at ~0.17 m); the -G build read them
  for the reference's own area functions and the vowel tube, and there its
  maps equal the builders' bit for bit; elsewhere there is nothing to compare;
* the time loop: FDTDEngineCPU run on the reference's own maps gives the
  same record_pressure and final fields as the oracle engine run on those
  maps, for every case.
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
BUILDS = {"release": ("", 1), "debug": ("g_", 0)}     # fixture prefix, depth_fma of the build
MIN_DEPTH = np.float32(0.001)


def case_inputs(c):
    i = c["case"]
    geo = (G[f"c{i}_length_cm"], G[f"c{i}_area_cm2"]) if f"c{i}_length_cm" in G else None
    return dict(c["params"]), geo


def elliptical_25d(kw):
    return kw.get("cross_sectional_shape", 1) == 2 and kw.get("fdtd_solver_type", 1) == 1 \
        and kw.get("simulation_type", 1) == 1


def depths_defined(c, prefix):
    """False where the build's elliptical depth kernel did not read the tube's
    axes: always in the Release-like build (its maps came out at the 1 mm floor
    or at depths of ~0.17 m, neither the tube's), and in the -G build where the
    whole map sits at the floor."""
    kw, _ = case_inputs(c)
    if not elliptical_25d(kw):
        return True
    return prefix == "g_" and not np.all(G[f"c{c['case']}_{prefix}depth_x"] == MIN_DEPTH)


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


IDS = [f"c{c['case']}-{c['geometry']}-{'-'.join(f'{k}{v}' for k, v in c['params'].items())}" for c in CASES]


@pytest.mark.parametrize("c", CASES, ids=IDS)
@pytest.mark.parametrize("build", sorted(BUILDS))
def test_oracle_maps_equal_the_reference(c, build):
    prefix, fma = BUILDS[build]
    kw, geo = case_inputs(c)
    i = c["case"]
    m = O.maps(O.params(**kw, depth_fma=fma), O.Geometry(*geo) if geo is not None else None)
    assert [m["dims"]["frame_h"], m["dims"]["frame_w"]] == c["frame"]
    assert [m["dims"]["listener_x"], m["dims"]["listener_y"]] == c["listener"]
    if kw.get("simulation_type", 1) == 1:
        assert [m["dims"]["excitation_x"], m["dims"]["excitation_y"]] == c["excitation"]
    assert np.array_equal(m["cell_type"], G[f"c{i}_{prefix}cell_type"].astype(np.int32))
    assert np.array_equal(m["z_inv"], G[f"c{i}_{prefix}z_inv"])
    if depths_defined(c, prefix):
        for k in ("depth_p", "depth_x", "depth_y"):
            assert np.array_equal(m[k], G[f"c{i}_{prefix}{k}"]), k


def test_every_elliptical_case_is_pinned_by_one_build():
    """The reference's four area functions and the vowel tube: the -G build read
    the tube's axes, so their elliptical maps are pinned.  (The batch tubes
    read other memory in both builds; their maps rest on the oracle and the
    circular-section pins.)"""
    ell = [c for c in CASES if elliptical_25d(c["params"])]
    pinned = [c["geometry"] for c in ell if depths_defined(c, "g_") or depths_defined(c, "")]
    assert {"ref:vocaltract_a", "ref:vocaltract_u", "vowel:0"} <= set(pinned)


@pytest.mark.parametrize("c", CASES, ids=IDS)
def test_library_maps_equal_the_reference(c):
    kw, geo = case_inputs(c)
    i = c["case"]
    for build, (prefix, fma) in BUILDS.items():
        m = V.build_maps(V.params(**kw, depth_fma=fma), V.Geometry(*geo) if geo is not None else None)
        assert np.array_equal(m["cell_type"], G[f"c{i}_{prefix}cell_type"].astype(np.int32))
        assert np.array_equal(m["z_inv"], G[f"c{i}_{prefix}z_inv"])
        if depths_defined(c, prefix):
            for k in ("depth_p", "depth_x", "depth_y"):
                assert np.array_equal(m[k], G[f"c{i}_{prefix}{k}"]), (build, k)


@pytest.mark.parametrize("c", CASES, ids=IDS)
def test_oracle_coefficients_equal_the_reference(c):
    """The 17 arrays of calculateSolverCoefficients depend on cell types, the
    tables and constants only: equal in every case and in both builds."""
    kw, geo = case_inputs(c)
    got = O.coeffs(O.params(**kw), O.Geometry(*geo) if geo is not None else None)
    bad = [k for k, v in got.items() if digest(v) != c["coeff_sha256"][k]]
    assert not bad, f"coefficient arrays differing from the reference: {bad}"
    assert c["coeff_sha256"] == c["debug_build_coeff_sha256"]


def reference_maps(c):
    i = c["case"]
    zmap = G[f"c{i}_z_inv"]
    zval = float(zmap[zmap != 0][0]) if np.any(zmap != 0) else 0.0
    return G[f"c{i}_depth_p"], G[f"c{i}_depth_x"], G[f"c{i}_depth_y"], zval


@pytest.mark.parametrize("c", CASES, ids=IDS)
def test_oracle_engine_equals_the_reference_engine(c):
    """record_pressure and the final P/Vx/Vy frames of the reference's
    FDTDEngineCPU (Release build, on the maps its own setup made) equal the
    oracle engine run on those same maps, bit for bit."""
    kw, geo = case_inputs(c)
    i = c["case"]
    p = O.params(**kw)
    g = O.Geometry(*geo) if geo is not None else None
    if p.source_type != 2:
        assert np.array_equal(O.source(p, c["steps"]), G[f"c{i}_excitation"])
    dp, dx, dy, zval = reference_maps(c)
    tr, (P, VX, VY) = O.run_maps_f32(p, g, c["steps"], dp, dx, dy, zval, fields=True)
    ref = G[f"c{i}_trace"]
    assert np.array_equal(tr, ref), f"first difference at step {int(np.argmax(tr != ref))}"
    assert np.any(ref != 0)
    assert {"p": digest(P), "vx": digest(VX), "vy": digest(VY)} == c["fields_sha256"]

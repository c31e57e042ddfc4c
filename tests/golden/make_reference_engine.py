"""Golden outputs of the reference's own grid setup and CPU engine.

    python tests/golden/make_reference_engine.py [--out PATH]

Needs oracle/_ref/ref_engine and ref_engine_g (oracle/Makefile.ref builds them
from the reference sources: SimulationParams, SolverParams, DeviceSymbols,
GlottalExcitations, FDTDSolver, TubeGeometry, TubeDepth, TwoMassModel,
FDTDEngineCPU) and a CUDA device, because the reference computes its maps
with setup kernels.  Writes tests/golden/reference_engine.npz: per case the
parameters, the area function, the reference's cell-type / depth / z_inv
maps, digests of its 17 coefficient arrays and of its final fields, its
record_pressure, and the same maps from the -G build.  Nothing here comes
from the oracle or the library under test.

Cases: the reference's four area functions (tests/golden/
reference_area_functions.npz) over circular/elliptical, 2D/2.5D, open and
Dirichlet mouth, PML on/off and the three sources; the uniform 17.5 x 3 cm
tube; eight batch tubes and one vowel tube of the seeded synthetic
workloads; srate_mul 30; the open-space domain.  Parameters the reference
hard-codes (mu, the Gaussian, ps = 686.46 Pa) keep its values.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO / "oracle"))
sys.path.insert(0, str(REPO / "vocalsim-2p5d-fdtd_b200" / "python"))

import oracle as O  # noqa: E402  (runs oracle/_ref/ref_engine; no oracle arithmetic is used)
from vocalsim_b200 import synthetic as S  # noqa: E402

AF = np.load(HERE / "reference_area_functions.npz")


def area(name: str):
    if name.startswith("ref:"):
        k = name[4:]
        return AF[f"{k}_length_cm"], AF[f"{k}_area_cm2"]
    if name == "uniform":
        return S.uniform_tube()
    if name.startswith("batch:"):
        return S.batch_tube(int(name[6:]))[:2]
    if name.startswith("vowel:"):
        return S.vowel_tube(int(name[6:]))
    if name == "open":
        return None
    raise KeyError(name)


# (geometry, overrides of the reference defaults, steps)
CASES = [
    ("ref:vocaltract_a", dict(cross_sectional_shape=1, mouth_radiation_cond=1, pml_flag=0), 2000),   # main.cu's run
    ("ref:vocaltract_a", dict(cross_sectional_shape=2), 2000),
    ("ref:vocaltract_i", dict(cross_sectional_shape=1), 2000),
    ("ref:vocaltract_u", dict(cross_sectional_shape=2, mouth_radiation_cond=1), 2000),
    ("ref:cylindrical-tube", dict(cross_sectional_shape=1), 2000),
    ("ref:vocaltract_a", dict(cross_sectional_shape=1, fdtd_solver_type=0, source_type=0), 2000),
    ("ref:vocaltract_i", dict(cross_sectional_shape=2, fdtd_solver_type=0, mouth_radiation_cond=1, pml_flag=0), 2000),
    ("ref:vocaltract_u", dict(cross_sectional_shape=1, fdtd_solver_type=0), 2000),
    ("ref:cylindrical-tube", dict(cross_sectional_shape=2, fdtd_solver_type=0, mouth_radiation_cond=1,
                                  source_type=0), 2000),
    ("ref:vocaltract_a", dict(cross_sectional_shape=2, source_type=2), 5000),
    ("ref:vocaltract_u", dict(cross_sectional_shape=1, mouth_radiation_cond=1, source_type=2), 5000),
    ("uniform", dict(cross_sectional_shape=1), 2000),
    ("vowel:0", dict(cross_sectional_shape=2, source_type=2), 5000),
    ("ref:vocaltract_a", dict(cross_sectional_shape=2, srate_mul=30), 1500),
    ("ref:vocaltract_i", dict(cross_sectional_shape=1, srate_mul=30, mouth_radiation_cond=1), 1500),
    ("open", dict(simulation_type=0), 1500),
    ("open", dict(simulation_type=0, fdtd_solver_type=0, pml_flag=0, source_type=0), 1500),
] + [(f"batch:{s}", dict(cross_sectional_shape=2), 2000) for s in range(8)]


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(HERE / "reference_engine.npz"))
    ap.add_argument("--only", type=int, default=-1)
    args = ap.parse_args()
    out = {}
    specs = []
    for i, (geo, kw, steps) in enumerate(CASES):
        if args.only >= 0 and i != args.only:
            continue
        p = O.params(**kw)
        la = area(geo)
        g = O.Geometry(*la) if la is not None else None
        # safety gate only: the reference's depth kernels execute `trap` on a
        # negative radicand (TubeDepth.cu:273-288); such inputs are not run
        try:
            for fma in (0, 1):
                O.maps(O.params(**kw, depth_fma=fma), g)
        except RuntimeError as e:
            print(f"case {i}: skipped ({e})")
            continue
        r = O.reference_engine(p, g, steps)
        rg = O.reference_engine(p, g, 1, debug_build=True)
        m = r["meta"]
        specs.append({"case": i, "geometry": geo, "params": kw, "steps": steps, "frame": [m["frame_h"], m["frame_w"]],
                      "listener": [m["listener_x"], m["listener_y"]], "excitation": [m["excitation_x"], m["excitation_y"]],
                      "ref_steps": m["ref_steps"], "loop_s": m["loop_s"],
                      "coeff_sha256": {k: digest(v) for k, v in r["coeffs"].items()},
                      "fields_sha256": {k: digest(r[k]) for k in ("p", "vx", "vy")},
                      "debug_build_coeff_sha256": {k: digest(v) for k, v in rg["coeffs"].items()}})
        c = f"c{i}_"
        if la is not None:
            out[c + "length_cm"], out[c + "area_cm2"] = (np.asarray(x, np.float32) for x in la)
        out[c + "cell_type"] = r["cell_type"].astype(np.int8)
        for k in ("depth_p", "depth_x", "depth_y", "z_inv"):
            out[c + k] = r[k]
            out[c + "g_" + k] = rg[k]
        out[c + "g_cell_type"] = rg["cell_type"].astype(np.int8)
        out[c + "trace"] = r["trace"]
        out[c + "excitation"] = r["excitation"][:steps]
        cells = (m["frame_h"] - 2) * (m["frame_w"] - 2)
        print(f"case {i:2d} {geo:22s} {json.dumps(kw):70s} frame {m['frame_h']}x{m['frame_w']} "
              f"loop {m['loop_s']:.3f} s ({cells * steps / m['loop_s'] / 1e6:.1f} Mcell/s)", flush=True)
    out["cases_json"] = np.array(json.dumps(specs))
    np.savez_compressed(args.out, **out)
    print(args.out, Path(args.out).stat().st_size)


if __name__ == "__main__":
    main()

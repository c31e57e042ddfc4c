"""Regenerate the golden fixtures in tests/golden/ from the reference itself.

    python tests/golden/make_golden.py        (needs the reference tree and oracle/_ref)

Sources of truth (nothing here comes from the oracle under test):
  * oracle/_ref/libvsref.so -- the reference's own TwoMassModel.cpp,
    GlottalExcitations.cu, SolverParams.cu and SimulationParams.cu compiled
    from the reference tree by oracle/Makefile.ref;
  * the reference's area-function files data/tube-geometry/*.txt, parsed with
    the C library's strtof as the reference's `file >> float` does;
  * the reference's Python get_formants_bw (results/formants_bandwidths.py),
    imported from the reference tree, run on seeded synthetic signals.
"""
from __future__ import annotations

import ctypes as C
import importlib.util
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
# the reference tree: VOCALSIM_REFERENCE, else the build recipe's default location
REF = Path(os.environ.get("VOCALSIM_REFERENCE", "/root/reference"))
sys.path.insert(0, str(REPO / "oracle"))

import oracle as O  # noqa: E402  (only for the library path of the reference pieces)


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def reference_pieces(path: Path) -> None:
    O.build()
    R = O.ref_lib()
    if R is None:
        raise SystemExit("oracle/_ref/libvsref.so missing: run make -C oracle -f Makefile.ref")
    out = {}
    for mul in (1, 15, 30):
        v = np.zeros(12, np.float32)
        R.vsref_sim_params(mul, _fp(v))
        out[f"sim_params_{mul}"] = v
    for mul in (15, 30):
        dt = out[f"sim_params_{mul}"][3]
        b, s, d = (np.zeros(k, np.float32) for k in (13, 13, 4))
        R.vsref_solver_tables(6, np.float32(0.5), dt, _fp(b), _fp(s), _fp(d))
        out[f"beta_{mul}"], out[f"sigma_{mul}"], out[f"dir_{mul}"] = b, s, d
        durs = np.array([0.02, 0.05, 0.1, 1.0], np.float32)
        out[f"step_durations_{mul}"] = durs
        out[f"step_counts_{mul}"] = np.array([R.vsref_step_count(float(x), float(dt)) for x in durs], np.int64)
        for st in (0, 1, 2):
            e = np.zeros(4000, np.float32)
            R.vsref_excitation(st, 4000, float(dt), _fp(e))
            out[f"excitation_{st}_{mul}"] = e
        rng = np.random.default_rng(2024 + mul)
        p1 = (rng.standard_normal(20000) * 60.0).astype(np.float32)
        ug = np.zeros_like(p1)
        R.vsref_tmm(mul, _fp(p1), len(p1), _fp(ug))
        out[f"tmm_p1_{mul}"], out[f"tmm_ug_{mul}"] = p1, ug
        z = np.zeros(20000, np.float32)
        ugz = np.zeros_like(z)
        R.vsref_tmm(mul, _fp(z), len(z), _fp(ugz))
        out[f"tmm_ug_zero_p1_{mul}"] = ugz
    np.savez_compressed(path, **out)


def area_files(path: Path) -> None:
    libc = C.CDLL(None)
    libc.strtof.restype = C.c_float
    libc.strtof.argtypes = [C.c_char_p, C.c_void_p]
    out = {}
    for name in ("vocaltract_a", "vocaltract_i", "vocaltract_u", "cylindrical-tube"):
        rows = [ln.split() for ln in (REF / "data" / "tube-geometry" / f"{name}.txt").read_text().splitlines()
                if ln.strip()]
        length = np.array([libc.strtof(r[0].encode(), None) for r in rows], np.float32)
        area = np.array([libc.strtof(r[1].encode(), None) for r in rows], np.float32)
        out[f"{name}_length_cm"] = length
        out[f"{name}_area_cm2"] = area
    np.savez_compressed(path, **out)


def formants(path: Path) -> None:
    spec = importlib.util.spec_from_file_location("ref_formants", REF / "results" / "formants_bandwidths.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    out = {}
    rng = np.random.default_rng(7)
    fs = 44100.0 * 15
    for k in range(4):
        n = [4000, 33075, 13230, 9001][k]
        t = np.arange(n) / fs
        sig = np.zeros(n)
        for f0, bw in zip(rng.uniform(300, 4500, 4), rng.uniform(40, 200, 4)):
            sig += np.exp(-np.pi * bw * t) * np.sin(2 * np.pi * f0 * t)
        sig += 1e-6 * rng.standard_normal(n)
        sig = sig.astype(np.float32)
        out[f"signal_{k}"] = sig
        out[f"bw_{k}"] = mod.get_formants_bw(sig, fs, 6)
    np.savez_compressed(path, **out)


if __name__ == "__main__":
    if not REF.exists():
        raise SystemExit("the reference tree is not present here")
    reference_pieces(HERE / "reference_pieces.npz")
    area_files(HERE / "reference_area_functions.npz")
    formants(HERE / "formants_golden.npz")
    for p in sorted(HERE.glob("*.npz")):
        print(p.name, p.stat().st_size)

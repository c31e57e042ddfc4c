"""ctypes wrapper of the CPU oracle (oracle/_build/liboracle.so) and of the
reference pieces compiled from the reference tree (oracle/_ref/libvsref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py, never by the solver package.
"""
from __future__ import annotations

import ctypes as C
import os
import shutil
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
REPO = ORACLE_DIR.parent
sys.path.insert(0, str(REPO / "vocalsim-2p5d-fdtd_b200" / "python"))
from vocalsim_b200.abi import VsDims, VsGeometry, VsParams  # noqa: E402  (struct layout only)

LIB = ORACLE_DIR / "_build" / "liboracle.so"
REF_LIB = ORACLE_DIR / "_ref" / "libvsref.so"
REF_ENGINE = ORACLE_DIR / "_ref" / "ref_engine"          # Release-like build of the reference's setup + engine
REF_ENGINE_G = ORACLE_DIR / "_ref" / "ref_engine_g"      # the same with -G (the reference CMake's default)
MAIN_ON_MIRROR = ORACLE_DIR / "_ref" / "main_on_mirror"  # the reference's main.cu against the C++ mirror headers
# Where oracle/Makefile.ref finds the reference sources: VOCALSIM_REFERENCE, else
# the build recipe's default location.  Only build() reads it.
REFERENCE_TREE = Path(os.environ.get("VOCALSIM_REFERENCE", "/root/reference"))

_orc = None
_ref = None


def build(force: bool = False) -> None:
    """Compile the oracle (and the reference pieces when the tree is present)."""
    if force or not LIB.exists():
        subprocess.run(["make", "-s", "-C", str(ORACLE_DIR)], check=True)
    if REFERENCE_TREE.exists() and (force or not (REF_LIB.exists() and REF_ENGINE.exists() and REF_ENGINE_G.exists())):
        subprocess.run(["make", "-s", "-C", str(ORACLE_DIR), "-f", "Makefile.ref",
                        f"REF={REFERENCE_TREE}", "all"], check=True)


def build_main_on_mirror(force: bool = False) -> None:
    """Compile the reference's own driver (src/main.cu, unchanged) against the
    library's C++ mirror headers; needs the reference tree and the built
    libvocalsim_b200.so."""
    if REFERENCE_TREE.exists() and (force or not MAIN_ON_MIRROR.exists()):
        subprocess.run(["make", "-s", "-C", str(ORACLE_DIR), "-f", "Makefile.ref", f"REF={REFERENCE_TREE}",
                        "main_on_mirror"], check=True)


def lib() -> C.CDLL:
    global _orc
    if _orc is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        vp, vg, vd = C.POINTER(VsParams), C.POINTER(VsGeometry), C.POINTER(VsDims)
        fp, dp, ip = C.POINTER(C.c_float), C.POINTER(C.c_double), C.POINTER(C.c_int32)
        L.orc_last_error.restype = C.c_char_p
        L.orc_params_init.argtypes = [vp]
        L.orc_maps.argtypes = [vp, vg, vd, ip, ip, fp, fp, fp, fp, dp]
        L.orc_coeffs.argtypes = [vp, vg, fp]
        L.orc_consts.argtypes = [C.c_int, fp]
        L.orc_tables.argtypes = [C.c_int, fp, fp, fp]
        L.orc_step_count.argtypes = [C.c_float, C.c_float]
        L.orc_step_count.restype = C.c_longlong
        L.orc_source_f32.argtypes = [vp, C.c_longlong, fp]
        L.orc_tmm_f32.argtypes = [C.c_float, C.c_int, fp, C.c_longlong, fp]
        L.orc_tmm_f64.argtypes = [C.c_float, C.c_int, dp, C.c_longlong, dp]
        L.orc_tmm_f64r.argtypes = [C.c_float, C.c_int, dp, C.c_longlong, dp]
        L.orc_run_f32.argtypes = [vp, vg, C.c_longlong, fp, fp, fp, fp]
        L.orc_run_f64.argtypes = [vp, vg, C.c_longlong, dp, dp, dp, dp]
        L.orc_run_maps_f64.argtypes = [vp, vg, C.c_longlong, dp, dp, dp, C.c_double, dp]
        L.orc_run_maps_f32.argtypes = [vp, vg, C.c_longlong, fp, fp, fp, C.c_float, fp]
        L.orc_run_maps_f32_fields.argtypes = [vp, vg, C.c_longlong, fp, fp, fp, C.c_float, fp, fp, fp, fp]
        L.orc_set_sps_diameters.argtypes = [fp, C.c_int]
        _orc = L
    return _orc


def ref_lib() -> C.CDLL | None:
    """The reference's own compiled pieces, or None when not built here."""
    global _ref
    if _ref is None:
        if not REF_LIB.exists():
            return None
        L = C.CDLL(str(REF_LIB))
        fp = C.POINTER(C.c_float)
        L.vsref_tmm.argtypes = [C.c_int, fp, C.c_longlong, fp]
        L.vsref_excitation.argtypes = [C.c_int, C.c_int, C.c_double, fp]
        L.vsref_solver_tables.argtypes = [C.c_int, C.c_float, C.c_float, fp, fp, fp]
        L.vsref_step_count.argtypes = [C.c_float, C.c_float]
        L.vsref_step_count.restype = C.c_longlong
        L.vsref_sim_params.argtypes = [C.c_int, fp]
        _ref = L
    return _ref


def _fp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _check(rc: int, where: str) -> None:
    if rc != 0:
        raise RuntimeError(f"oracle {where}: status {rc}: {lib().orc_last_error().decode()}")


def params(**kw) -> VsParams:
    """Reference default parameters, with keyword overrides."""
    p = VsParams()
    lib().orc_params_init(C.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


class Geometry:
    """Owns the float32 arrays a VsGeometry points at."""

    def __init__(self, length_cm, area_cm2):
        self.length = np.ascontiguousarray(length_cm, dtype=np.float32)
        self.area = np.ascontiguousarray(area_cm2, dtype=np.float32)
        assert self.length.shape == self.area.shape
        self.g = VsGeometry(len(self.length), 0, _fp(self.length), _fp(self.area))

    def ref(self):
        return C.byref(self.g)


def set_sps_diameters(diameters_m) -> None:
    """Section diameters (m) for the next single-plane-symmetric (shape 3)
    builds: the oracle rasterises such tubes from them but does not construct
    the sections itself (their depths come in through run_maps_f32)."""
    d = np.ascontiguousarray(np.asarray(diameters_m, np.float32).ravel())
    _check(lib().orc_set_sps_diameters(_fp(d), int(d.size)), "set_sps_diameters")


def maps(p: VsParams, g: Geometry | None):
    d = VsDims()
    gp = g.ref() if g is not None else None
    _check(lib().orc_maps(C.byref(p), gp, C.byref(d), None, None, None, None, None, None, None), "maps")
    n = d.frame_h * d.frame_w
    t = np.zeros(n, np.int32); b = np.zeros(n, np.int32)
    dP = np.zeros(n, np.float32); dX = np.zeros(n, np.float32); dY = np.zeros(n, np.float32)
    z = np.zeros(n, np.float32)
    margin = C.c_double(0)
    ip = C.POINTER(C.c_int32)
    _check(lib().orc_maps(C.byref(p), gp, C.byref(d), t.ctypes.data_as(ip), b.ctypes.data_as(ip),
                          _fp(dP), _fp(dX), _fp(dY), _fp(z), C.byref(margin)), "maps")
    shp = (d.frame_h, d.frame_w)
    return dict(dims=d.as_dict(), cell_type=t.reshape(shp), bst=b.reshape(shp), depth_p=dP.reshape(shp),
                depth_x=dX.reshape(shp), depth_y=dY.reshape(shp), z_inv=z.reshape(shp),
                scan_margin=margin.value)


COEFF_NAMES = ["N_out", "N_in", "minVxBeta", "minVyBeta", "maxVxSigmaPrimedt", "maxVySigmaPrimedt",
               "betaVxSqr_dt_inv_rho_inv_ds", "betaVySqr_dt_inv_rho_inv_ds", "pressureSigmaPrimedt",
               "areWeNotExcitationVx", "areWeNotExcitationVy", "excitationWeightVx",
               "excitationWeightVy", "xor_val1", "xor_val2", "xor_val3", "xor_val4"]


def coeffs(p: VsParams, g: Geometry | None) -> dict:
    m = maps(p, g)
    H, W = m["dims"]["frame_h"], m["dims"]["frame_w"]
    out = np.zeros(17 * (H - 2) * (W - 2), np.float32)
    _check(lib().orc_coeffs(C.byref(p), g.ref() if g is not None else None, _fp(out)), "coeffs")
    out = out.reshape(17, H - 2, W - 2)
    return {k: out[i] for i, k in enumerate(COEFF_NAMES)}


def run(p: VsParams, g: Geometry | None, steps: int, precision: str = "f32", fields: bool = False):
    """Trace (and optionally final P/Vx/Vy frames) of `steps` steps from rest."""
    m = maps(p, g)["dims"]
    n = m["frame_h"] * m["frame_w"]
    gp = g.ref() if g is not None else None
    if precision == "f32":
        tr = np.zeros(steps, np.float32)
        F = [np.zeros(n, np.float32) for _ in range(3)] if fields else [None] * 3
        _check(lib().orc_run_f32(C.byref(p), gp, steps, _fp(tr), *[(_fp(a) if a is not None else None) for a in F]),
               "run_f32")
    else:
        tr = np.zeros(steps, np.float64)
        F = [np.zeros(n, np.float64) for _ in range(3)] if fields else [None] * 3
        _check(lib().orc_run_f64(C.byref(p), gp, steps, _dp(tr), *[(_dp(a) if a is not None else None) for a in F]),
               "run_f64")
    if not fields:
        return tr
    shp = (m["frame_h"], m["frame_w"])
    return tr, [a.reshape(shp) for a in F]


def run_maps_f64(p: VsParams, g: Geometry | None, steps: int, depth_p, depth_x, depth_y, z_inv: float) -> np.ndarray:
    """Double-precision trace of the engine on the given depth maps and z_inv value."""
    mp, mx, my = (np.ascontiguousarray(a, np.float64).reshape(-1) for a in (depth_p, depth_x, depth_y))
    tr = np.zeros(steps, np.float64)
    _check(lib().orc_run_maps_f64(C.byref(p), g.ref() if g is not None else None, steps, _dp(mp), _dp(mx), _dp(my),
                                  float(z_inv), _dp(tr)), "run_maps_f64")
    return tr


def run_maps_f32(p: VsParams, g: Geometry | None, steps: int, depth_p, depth_x, depth_y, z_inv: float,
                 fields: bool = False):
    """FP32 trace of the engine on the given depth maps (rounded to float) and z_inv value
    (and, with fields=True, the final P, Vx, Vy frames)."""
    mp, mx, my = (np.ascontiguousarray(a, np.float32).reshape(-1) for a in (depth_p, depth_x, depth_y))
    tr = np.zeros(steps, np.float32)
    gp = g.ref() if g is not None else None
    if not fields:
        _check(lib().orc_run_maps_f32(C.byref(p), gp, steps, _fp(mp), _fp(mx), _fp(my), float(z_inv), _fp(tr)),
               "run_maps_f32")
        return tr
    F = [np.zeros(mp.size, np.float32) for _ in range(3)]
    _check(lib().orc_run_maps_f32_fields(C.byref(p), gp, steps, _fp(mp), _fp(mx), _fp(my), float(z_inv), _fp(tr),
                                         *[_fp(a) for a in F]), "run_maps_f32_fields")
    shp = np.shape(depth_p)
    return tr, [a.reshape(shp) for a in F]


def source(p: VsParams, n: int) -> np.ndarray:
    out = np.zeros(n, np.float32)
    _check(lib().orc_source_f32(C.byref(p), n, _fp(out)), "source")
    return out


def tmm(ps: float, srate_mul: int, p1: np.ndarray, precision: str = "f32") -> np.ndarray:
    """The two-mass model driven by the pressure sequence p1: "f32" the
    reference's float model, "f64" its expressions in double, "f64r" the
    tmm_f64 option's arrangement of the double model."""
    if precision == "f32":
        p1 = np.ascontiguousarray(p1, np.float32)
        ug = np.zeros_like(p1)
        lib().orc_tmm_f32(ps, srate_mul, _fp(p1), len(p1), _fp(ug))
    else:
        p1 = np.ascontiguousarray(p1, np.float64)
        ug = np.zeros_like(p1)
        fn = lib().orc_tmm_f64r if precision == "f64r" else lib().orc_tmm_f64
        fn(ps, srate_mul, _dp(p1), len(p1), _dp(ug))
    return ug


def consts(srate_mul: int) -> np.ndarray:
    out = np.zeros(11, np.float32)
    lib().orc_consts(srate_mul, _fp(out))
    return out


def tables(srate_mul: int):
    b = np.zeros(13, np.float32); s = np.zeros(13, np.float32); d = np.zeros(4, np.float32)
    lib().orc_tables(srate_mul, _fp(b), _fp(s), _fp(d))
    return b, s, d


def step_count(audio_dur: float, dt: float) -> int:
    return int(lib().orc_step_count(audio_dur, dt))


# --------------------------------------------------------------------------- reference engine
# vs_params fields whose values the reference hard-codes; a reference-engine
# run is only a like-for-like check when they hold the defaults.
_NATIVE_FIELDS = ("mu3d", "gauss_peak_s", "gauss_width_s", "gauss_amp", "sine_freq_hz", "sine_amp", "tmm_ps_pa",
                  "wall_coupling", "uniform_depth_m", "listener_mode", "listener_x", "listener_y", "engine",
                  "tmm_f64", "fast_math")


def reference_native(p: VsParams) -> bool:
    """True when every parameter the reference hard-codes has its reference value."""
    d = params()
    return all(getattr(p, k) == getattr(d, k) for k in _NATIVE_FIELDS if hasattr(d, k)) and p.source_type in (0, 1, 2)


def _fmt32(x) -> str:
    """Shortest decimal that reads back as the same float32 (strtof)."""
    return np.format_float_positional(np.float32(x), unique=True, trim="-")


def reference_engine(p: VsParams, g: Geometry | None, steps: int, debug_build: bool = False, with_maps: bool = True,
                     timeout: float = 900.0) -> dict:
    """Run the reference's own SimulationParams -> FDTDSolver::setupWaveSolver ->
    FDTDEngineCPU::startSolverEngine (oracle/_ref/ref_engine, compiled from the
    reference sources; the setup kernels need a CUDA device) for `steps` steps.
    The area function is written in the reference's file format to the file
    its constructor reads (TubeGeometry.cu:53-88) in a scratch tree.  Returns the
    reference's maps, its 17 coefficient arrays, its excitation table, its
    record_pressure and final fields, and the seconds its time loop took."""
    exe = REF_ENGINE_G if debug_build else REF_ENGINE
    if not exe.exists():
        raise FileNotFoundError(f"{exe} is not built (oracle/Makefile.ref needs the reference tree)")
    if not reference_native(p):
        raise ValueError("the reference engine hard-codes mu3d, its sources and its wall and depth model: "
                         "use reference defaults for those fields")
    if g is None and p.source_type == 2:
        # openSpaceSimulation never sets FDTDSolver::excitationX/Y (FDTDSolver.cu:530-531),
        # which the two-mass source reads
        raise ValueError("the reference's open-space domain has no excitation cell for the two-mass source")
    root = Path(tempfile.mkdtemp(prefix="vs_refeng_"))
    try:
        (root / "data" / "tube-geometry").mkdir(parents=True)
        (root / "results").mkdir()
        (root / "a" / "b").mkdir(parents=True)
        (root / "out").mkdir()
        if g is not None:
            lines = [f"{_fmt32(l)} {_fmt32(a)}" for l, a in zip(g.length, g.area)]
            (root / "data" / "tube-geometry" / "vocaltract_a.txt").write_text("\n".join(lines) + "\n")
        consts_ = consts(p.srate_mul)
        dt = float(consts_[3])
        audio_dur = (steps + 16) * dt * 1.01
        args = [str(exe), f"solver={p.fdtd_solver_type}", f"sim={p.simulation_type}", "tube=1", "vowel=1",
                f"shape={p.cross_sectional_shape if g is not None else -1}", f"mouth={p.mouth_radiation_cond}",
                f"srate_mul={p.srate_mul}", f"audio_dur={audio_dur!r}", f"source={p.source_type}",
                f"pml={p.pml_flag}", f"steps={steps}", f"out={root / 'out'}", f"maps={1 if with_maps else 0}"]
        t0 = time.perf_counter()
        r = subprocess.run(args, cwd=root / "a" / "b", capture_output=True, text=True, timeout=timeout)
        wall = time.perf_counter() - t0
        if r.returncode != 0:
            raise RuntimeError(f"ref_engine exited {r.returncode}: {r.stderr[-2000:]}")
        out = root / "out"
        meta = {}
        for line in (out / "meta.txt").read_text().splitlines():
            k, v = line.split()
            meta[k] = float(v) if any(ch in v for ch in ".e") else int(v)
        H, W = meta["frame_h"], meta["frame_w"]
        rd = lambda name, dt_=np.float32: np.fromfile(out / name, dtype=dt_)  # noqa: E731
        res = {"meta": meta, "trace": rd("trace.f32"), "excitation": rd("excitation.f32"),
               "p": rd("p.f32").reshape(H, W), "vx": rd("vx.f32").reshape(H, W), "vy": rd("vy.f32").reshape(H, W),
               "loop_s": meta["loop_s"], "wall_s": wall}
        if with_maps:
            res["cell_type"] = rd("cell_type.i32", np.int32).reshape(H, W)
            for k in ("depth_p", "depth_x", "depth_y", "z_inv"):
                res[k] = rd(k + ".f32").reshape(H, W)
            res["coeffs"] = {k: rd(k + ".f32").reshape(H - 2, W - 2) for k in COEFF_NAMES}
        return res
    finally:
        shutil.rmtree(root, ignore_errors=True)


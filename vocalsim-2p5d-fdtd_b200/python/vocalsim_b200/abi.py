"""ctypes mirror of include/vocalsim_b200.h and the loader of libvocalsim_b200.so.

The structs below must match the C header field for field; a CPU test checks
their sizes and offsets against the library's own view (vs_abi_layout).
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

PKG_ROOT = Path(__file__).resolve().parents[2]          # vocalsim-2p5d-fdtd_b200/
REPO_ROOT = PKG_ROOT.parent
LIB_PATH = PKG_ROOT / "lib" / "libvocalsim_b200.so"
HEADER_PATH = REPO_ROOT / "include" / "vocalsim_b200.h"

VS_ABI_VERSION = 1

# vs_status
VS_OK = 0
VS_ERR_INVALID_ARG = 1
VS_ERR_GEOMETRY = 2
VS_ERR_CUDA = 3
VS_ERR_TIMEOUT = 4
VS_ERR_NONFINITE = 5
VS_ERR_ALLOC = 6
VS_ERR_UNSUPPORTED = 7
VS_ERR_NEGATIVE_SQRT = 8
STATUS_NAMES = {
    0: "VS_OK", 1: "VS_ERR_INVALID_ARG", 2: "VS_ERR_GEOMETRY", 3: "VS_ERR_CUDA",
    4: "VS_ERR_TIMEOUT", 5: "VS_ERR_NONFINITE", 6: "VS_ERR_ALLOC",
    7: "VS_ERR_UNSUPPORTED", 8: "VS_ERR_NEGATIVE_SQRT",
}

# cell types (reference enum CellTypes, include/SolverParams.h:21-35)
CELL_WALL, CELL_AIR, CELL_EXCITATION = 0, 1, 2
CELL_PML0, CELL_PML5 = 3, 8
CELL_DYNAMIC, CELL_DEAD, CELL_NOPRESSURE, CELL_HEAD = 9, 10, 11, 12

SRC_SINE, SRC_GAUSS, SRC_TMM, SRC_GAUSS_STD = 0, 1, 2, 3
ENGINE_CPU, ENGINE_EIGEN = 1, 2
LISTENER_REFERENCE, LISTENER_EXPLICIT = 0, 1


class VsParams(C.Structure):
    _fields_ = [
        ("fdtd_solver_type", C.c_int32),
        ("simulation_type", C.c_int32),
        ("cross_sectional_shape", C.c_int32),
        ("mouth_radiation_cond", C.c_int32),
        ("srate_mul", C.c_int32),
        ("source_type", C.c_int32),
        ("pml_flag", C.c_int32),
        ("engine", C.c_int32),
        ("audio_dur", C.c_float),
        ("pad0", C.c_int32),
        ("num_steps", C.c_int64),
        ("gauss_peak_s", C.c_float),
        ("gauss_width_s", C.c_float),
        ("gauss_amp", C.c_float),
        ("sine_freq_hz", C.c_float),
        ("sine_amp", C.c_float),
        ("tmm_ps_pa", C.c_float),
        ("mu3d", C.c_float),
        ("wall_coupling", C.c_float),
        ("uniform_depth_m", C.c_float),
        ("depth_fma", C.c_int32),
        ("listener_mode", C.c_int32),
        ("listener_x", C.c_int32),
        ("listener_y", C.c_int32),
        ("tmm_f64", C.c_int32),
        ("fast_math", C.c_int32),
        ("reserved", C.c_int32 * 6),
    ]

    def copy(self) -> "VsParams":
        out = VsParams()
        C.memmove(C.byref(out), C.byref(self), C.sizeof(VsParams))
        return out

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_
                if name not in ("pad0", "reserved")}


class VsGeometry(C.Structure):
    _fields_ = [
        ("n_sections", C.c_int32),
        ("pad0", C.c_int32),
        ("section_length_cm", C.POINTER(C.c_float)),
        ("section_area_cm2", C.POINTER(C.c_float)),
    ]


class VsDims(C.Structure):
    _fields_ = [
        ("frame_h", C.c_int32), ("frame_w", C.c_int32),
        ("listener_x", C.c_int32), ("listener_y", C.c_int32),
        ("excitation_x", C.c_int32), ("excitation_y", C.c_int32),
        ("tube_length_cells", C.c_int32),
        ("tube_start_x", C.c_int32), ("tube_end_x", C.c_int32), ("tube_mid_y", C.c_int32),
        ("num_steps", C.c_int64),
        ("interior_cells", C.c_int64),
        ("dt", C.c_float), ("ds", C.c_float),
        ("z_inv_val", C.c_float),
        ("pad0", C.c_int32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "pad0"}


def header_symbols(path: Path = HEADER_PATH) -> list[str]:
    """Every function the public header declares (`int vs_x(`, `void vs_x(` ...)."""
    import re
    text = path.read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+char\s*\*|int|void)\s+(vs_\w+)\s*\(", text, re.M)))


_lib = None


def load_library(path: os.PathLike | None = None) -> C.CDLL:
    """Load libvocalsim_b200.so (built in-tree by build.py) and declare its ABI."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path is not None else LIB_PATH
    if not p.exists():
        raise RuntimeError(
            f"{p} is missing: build it with `python vocalsim-2p5d-fdtd_b200/build.py` "
            "(there is no CPU fallback for the solver)")
    lib = C.CDLL(str(p))
    vp, vg, vd = C.POINTER(VsParams), C.POINTER(VsGeometry), C.POINTER(VsDims)
    fp, ip, i32p = C.POINTER(C.c_float), C.POINTER(C.c_int), C.POINTER(C.c_int32)
    sig = {
        "vs_version": (C.c_int, []),
        "vs_params_init": (C.c_int, [vp]),
        "vs_build_maps": (C.c_int, [vp, vg, vd, i32p, fp, fp, fp, fp]),
        "vs_source_table": (C.c_int, [vp, C.c_int64, fp]),
        "vs_tube_layout": (C.c_int, [vp, vg, vd, i32p, i32p, i32p, fp, fp]),
        "vs_create": (C.c_int, [vp, vg, C.POINTER(C.c_void_p)]),
        "vs_get_dims": (C.c_int, [C.c_void_p, vd]),
        "vs_run": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_int]),
        "vs_reset": (C.c_int, [C.c_void_p]),
        "vs_get_fields": (C.c_int, [C.c_void_p, fp, fp, fp]),
        "vs_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
        "vs_destroy": (None, [C.c_void_p]),
        "vs_batch_create": (C.c_int, [C.c_int32, vp, vg, C.POINTER(C.c_void_p)]),
        "vs_batch_get_dims": (C.c_int, [C.c_void_p, C.c_int32, vd]),
        "vs_batch_run": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_int]),
        "vs_batch_reset": (C.c_int, [C.c_void_p]),
        "vs_batch_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
        "vs_batch_set_tile": (C.c_int, [C.c_void_p, C.c_int32]),
        "vs_batch_set_wait_limit": (C.c_int, [C.c_void_p, C.c_uint32]),
        "vs_batch_set_adjoint_form": (C.c_int, [C.c_void_p, C.c_int32]),
        "vs_batch_set_adjoint_rows": (C.c_int, [C.c_void_p, C.c_int32]),
        "vs_batch_adjoint_times": (C.c_int, [C.c_void_p, fp, fp]),
        "vs_batch_forward_ckpt_device": (C.c_int, [C.c_void_p, C.c_int64, C.c_int32, C.c_void_p]),
        "vs_batch_adjoint_device": (C.c_int, [C.c_void_p, C.c_void_p, fp, fp, fp, fp]),
        "vs_batch_autotune": (C.c_int, [C.c_void_p, C.c_int64, i32p, fp]),
        "vs_tile_shape_count": (C.c_int, []),
        "vs_tile_shape": (C.c_int, [C.c_int32, i32p, i32p]),
        "vs_tile_shape_steps": (C.c_int, [C.c_int32, i32p]),
        "vs_audio": (C.c_int, [C.c_void_p, C.c_int32, C.c_int64, C.c_int32, C.c_void_p, C.c_void_p]),
        "vs_audio_filter": (C.c_int, [C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
        "vs_batch_destroy": (None, [C.c_void_p]),
        "vs_batch_set_maps": (C.c_int, [C.c_void_p, C.c_int32, fp, fp, fp, C.c_float]),
        "vs_batch_get_maps": (C.c_int, [C.c_void_p, C.c_int32, i32p, fp, fp, fp, fp]),
        "vs_batch_get_fields": (C.c_int, [C.c_void_p, C.c_int32, fp, fp, fp]),
        "vs_batch_forward_ckpt": (C.c_int, [C.c_void_p, C.c_int64, C.c_int32, fp]),
        "vs_batch_adjoint": (C.c_int, [C.c_void_p, fp, fp, fp, fp, fp]),
        "vs_run_noalloc": (C.c_int, [vp, vd, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]),
        "vs_batch_set_sections": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
        "vs_batch_section_gradients": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
        "vs_formants": (C.c_int, [C.c_void_p, C.c_int32, C.c_int64, C.c_double, C.c_int32, C.c_void_p,
                                  C.c_void_p]),
        "vs_last_error": (C.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


class VsError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str = ""):
        self.status = status
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}: {msg}")


def check(lib: C.CDLL, status: int, where: str) -> None:
    if status != VS_OK:
        raise VsError(status, where, lib.vs_last_error().decode(errors="replace"))

"""Python handles over the C ABI (ctypes): Geometry, Solver, Batch, build_maps.

Every compute call goes through libvocalsim_b200.so; there is no Python or
CPU fallback, and a missing library raises.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from .abi import VsDims, VsGeometry, VsParams, check, load_library


def _fp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def params(**overrides) -> VsParams:
    """Reference defaults (vs_params_init) with keyword overrides."""
    lib = load_library()
    p = VsParams()
    check(lib, lib.vs_params_init(C.byref(p)), "vs_params_init")
    for k, v in overrides.items():
        if not hasattr(p, k) or k in ("pad0", "reserved"):
            raise KeyError(f"unknown vs_params field {k!r}")
        setattr(p, k, v)
    return p


class Geometry:
    """An area function; keeps the float32 arrays the C struct points at alive."""

    def __init__(self, length_cm, area_cm2):
        self.length = np.ascontiguousarray(length_cm, dtype=np.float32).reshape(-1)
        self.area = np.ascontiguousarray(area_cm2, dtype=np.float32).reshape(-1)
        if self.length.shape != self.area.shape:
            raise ValueError("length and area need the same number of sections")
        self.struct = VsGeometry(len(self.length), 0, _fp(self.length), _fp(self.area))


def build_maps(p: VsParams, g: Geometry | None) -> dict:
    """Host-only map build (vs_build_maps): dims + cell_type/depth/z_inv frames."""
    lib = load_library()
    gp = C.byref(g.struct) if g is not None else None
    d = VsDims()
    check(lib, lib.vs_build_maps(C.byref(p), gp, C.byref(d), None, None, None, None, None), "vs_build_maps")
    shp = (d.frame_h, d.frame_w)
    ct = np.zeros(shp, np.int32)
    dp, dx, dy, z = (np.zeros(shp, np.float32) for _ in range(4))
    check(lib, lib.vs_build_maps(C.byref(p), gp, C.byref(d), ct.ctypes.data_as(C.POINTER(C.c_int32)),
                                 _fp(dp), _fp(dx), _fp(dy), _fp(z)), "vs_build_maps")
    return dict(dims=d.as_dict(), cell_type=ct, depth_p=dp, depth_x=dx, depth_y=dy, z_inv=z)


def source_table(p: VsParams, n: int) -> np.ndarray:
    lib = load_library()
    out = np.zeros(n, np.float32)
    check(lib, lib.vs_source_table(C.byref(p), n, _fp(out)), "vs_source_table")
    return out


class Solver:
    """One tube on the current CUDA device (vs_create / vs_run / vs_destroy)."""

    def __init__(self, p: VsParams, g: Geometry | None):
        self.lib = load_library()
        self._g = g
        self.h = C.c_void_p()
        check(self.lib, self.lib.vs_create(C.byref(p), C.byref(g.struct) if g is not None else None,
                                           C.byref(self.h)), "vs_create")
        d = VsDims()
        check(self.lib, self.lib.vs_get_dims(self.h, C.byref(d)), "vs_get_dims")
        self.dims = d.as_dict()

    def run(self, steps: int, out: np.ndarray | None = None) -> np.ndarray:
        """Advance `steps` steps; return the listener trace (host float32)."""
        tr = out if out is not None else np.zeros(steps, np.float32)
        check(self.lib, self.lib.vs_run(self.h, steps, tr.ctypes.data_as(C.c_void_p), 0), "vs_run")
        return tr

    def run_device(self, steps: int, device_ptr: int) -> None:
        """Advance `steps` steps writing the trace to a device buffer."""
        check(self.lib, self.lib.vs_run(self.h, steps, C.c_void_p(device_ptr), 1), "vs_run")

    def reset(self) -> None:
        check(self.lib, self.lib.vs_reset(self.h), "vs_reset")

    def set_stream(self, stream_handle: int | None) -> None:
        check(self.lib, self.lib.vs_set_stream(self.h, C.c_void_p(stream_handle) if stream_handle else None),
              "vs_set_stream")

    def fields(self):
        H, W = self.dims["frame_h"], self.dims["frame_w"]
        P, Vx, Vy = (np.zeros((H, W), np.float32) for _ in range(3))
        check(self.lib, self.lib.vs_get_fields(self.h, _fp(P), _fp(Vx), _fp(Vy)), "vs_get_fields")
        return P, Vx, Vy

    def close(self) -> None:
        if self.h:
            self.lib.vs_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many independent tubes stepped together (vs_batch_*)."""

    def __init__(self, ps: Sequence[VsParams], gs: Sequence[Geometry | None]):
        self.lib = load_library()
        n = len(ps)
        if n != len(gs):
            raise ValueError("one geometry per parameter set")
        self._gs = list(gs)
        parr = (VsParams * n)(*ps)
        garr = (VsGeometry * n)()
        for i, g in enumerate(gs):
            if g is not None:
                garr[i] = g.struct
        self.n = n
        self.trace_device = None        # a torch device: SectionTrace keeps traces there
        self.h = C.c_void_p()
        check(self.lib, self.lib.vs_batch_create(n, parr, garr, C.byref(self.h)), "vs_batch_create")
        self.dims = []
        for i in range(n):
            d = VsDims()
            check(self.lib, self.lib.vs_batch_get_dims(self.h, i, C.byref(d)), "vs_batch_get_dims")
            self.dims.append(d.as_dict())

    @property
    def interior_cells(self) -> int:
        return sum(d["interior_cells"] for d in self.dims)

    def run(self, steps: int, out: np.ndarray | None = None) -> np.ndarray:
        tr = out if out is not None else np.zeros((self.n, steps), np.float32)
        check(self.lib, self.lib.vs_batch_run(self.h, steps, tr.ctypes.data_as(C.c_void_p), 0), "vs_batch_run")
        return tr

    def run_device(self, steps: int, device_ptr: int = 0) -> None:
        """Advance without a host copy; device_ptr (n x steps floats) may be 0."""
        check(self.lib, self.lib.vs_batch_run(self.h, steps, C.c_void_p(device_ptr) if device_ptr else None, 1),
              "vs_batch_run")

    def reset(self) -> None:
        check(self.lib, self.lib.vs_batch_reset(self.h), "vs_batch_reset")

    def set_stream(self, stream_handle: int | None) -> None:
        """Issue all later work on this cudaStream_t (an int handle, e.g. torch's stream.cuda_stream)."""
        check(self.lib, self.lib.vs_batch_set_stream(self.h, C.c_void_p(stream_handle) if stream_handle else None),
              "vs_batch_set_stream")

    def set_tile(self, index: int) -> None:
        check(self.lib, self.lib.vs_batch_set_tile(self.h, index), "vs_batch_set_tile")

    def adjoint_times(self) -> tuple[float, float]:
        """(recomputation ms, reverse-step ms) of the last adjoint(), device time."""
        a, r = C.c_float(), C.c_float()
        check(self.lib, self.lib.vs_batch_adjoint_times(self.h, C.byref(a), C.byref(r)), "vs_batch_adjoint_times")
        return a.value, r.value

    def set_adjoint_form(self, form: int) -> None:
        """Reverse-step kernel of adjoint(): 0 = automatic (default), 1 = tiles,
        2 = two-step warp strips (form 3 for two-mass batches), 3 = one-step strips."""
        check(self.lib, self.lib.vs_batch_set_adjoint_form(self.h, form), "vs_batch_set_adjoint_form")

    def set_adjoint_rows(self, rows: int) -> None:
        """Rows per strip of the strip forms: 4, 8, 16 or 0 (8 for form 2, 4 for form 3)."""
        check(self.lib, self.lib.vs_batch_set_adjoint_rows(self.h, rows), "vs_batch_set_adjoint_rows")

    def set_wait_limit(self, polls: int) -> None:
        """Polls of a row-copy wait before the run gives up with VS_ERR_TIMEOUT (0 = default)."""
        check(self.lib, self.lib.vs_batch_set_wait_limit(self.h, polls), "vs_batch_set_wait_limit")

    def set_maps(self, tube: int, depth_p=None, depth_x=None, depth_y=None, z_inv: float = 0.0) -> None:
        """Replace tube `tube`'s depth maps (frame-shaped float32) and z_inv value."""
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float32) for a in (depth_p, depth_x, depth_y)]
        ptrs = [None if a is None else _fp(a) for a in arrs]
        check(self.lib, self.lib.vs_batch_set_maps(self.h, tube, *ptrs, float(z_inv)), "vs_batch_set_maps")

    def get_maps(self, tube: int) -> dict:
        """The maps tube `tube` steps with, read back from the device:
        cell_type, depth_p, depth_x, depth_y, z_inv (frame-shaped), as
        build_maps returns them."""
        d = self.dims[tube]
        H, W = int(d["frame_h"]), int(d["frame_w"])
        out = {"cell_type": np.zeros((H, W), np.int32)}
        for k in ("depth_p", "depth_x", "depth_y", "z_inv"):
            out[k] = np.zeros((H, W), np.float32)
        check(self.lib, self.lib.vs_batch_get_maps(self.h, tube, out["cell_type"].ctypes.data_as(C.POINTER(C.c_int32)),
                                                   _fp(out["depth_p"]), _fp(out["depth_x"]), _fp(out["depth_y"]),
                                                   _fp(out["z_inv"])), "vs_batch_get_maps")
        return out

    def fields(self, tube: int):
        """Tube `tube`'s current P, Vx, Vy frames."""
        d = self.dims[tube]
        H, W = int(d["frame_h"]), int(d["frame_w"])
        P, Vx, Vy = (np.zeros((H, W), np.float32) for _ in range(3))
        check(self.lib, self.lib.vs_batch_get_fields(self.h, tube, _fp(P), _fp(Vx), _fp(Vy)), "vs_batch_get_fields")
        return P, Vx, Vy

    def forward_ckpt(self, steps: int, ckpt_every: int = 512) -> np.ndarray:
        """Forward from rest keeping checkpoints for adjoint(); returns (n, steps) traces."""
        tr = np.zeros((self.n, steps), np.float32)
        check(self.lib, self.lib.vs_batch_forward_ckpt(self.h, steps, ckpt_every, _fp(tr)), "vs_batch_forward_ckpt")
        self._ck_steps = steps
        return tr

    def forward_ckpt_device(self, steps: int, ckpt_every: int, traces_ptr: int) -> None:
        """forward_ckpt with the (n, steps) float32 traces written to device memory at traces_ptr."""
        check(self.lib, self.lib.vs_batch_forward_ckpt_device(self.h, steps, ckpt_every, C.c_void_p(traces_ptr)),
              "vs_batch_forward_ckpt_device")
        self._ck_steps = steps

    def adjoint_device(self, grad_ptr: int) -> np.ndarray:
        """adjoint(maps=False) with dL/dtrace (n, steps float32) in device memory; returns dL/dz_inv per tube."""
        gz = np.zeros(self.n, np.float32)
        check(self.lib, self.lib.vs_batch_adjoint_device(self.h, C.c_void_p(grad_ptr), None, None, None, _fp(gz)),
              "vs_batch_adjoint_device")
        return gz

    def set_sections(self, widths, depths, z_inv=None) -> None:
        """Depth maps of every tube from its section widths / depths (m), computed
        on the device (vs_batch_set_sections); z_inv per tube or None."""
        w = np.ascontiguousarray(np.concatenate([np.asarray(x, np.float64).ravel() for x in widths]))
        d = np.ascontiguousarray(np.concatenate([np.asarray(x, np.float64).ravel() for x in depths]))
        z = None if z_inv is None else np.ascontiguousarray(np.asarray(z_inv, np.float64).ravel())
        dp = C.POINTER(C.c_double)
        check(self.lib, self.lib.vs_batch_set_sections(self.h, w.ctypes.data_as(dp), d.ctypes.data_as(dp),
                                                       None if z is None else z.ctypes.data_as(dp)),
              "vs_batch_set_sections")
        self._nsec = [len(np.asarray(x).ravel()) for x in widths]

    def section_gradients(self):
        """(dL/d widths, dL/d depths) per tube after set_sections / forward_ckpt / adjoint."""
        tot = sum(self._nsec)
        gw, gd = np.zeros(tot), np.zeros(tot)
        dp = C.POINTER(C.c_double)
        check(self.lib, self.lib.vs_batch_section_gradients(self.h, gw.ctypes.data_as(dp), gd.ctypes.data_as(dp)),
              "vs_batch_section_gradients")
        out, k = [], 0
        for m in self._nsec:
            out.append((gw[k:k + m], gd[k:k + m]))
            k += m
        return out

    def adjoint(self, dL_dtrace: np.ndarray, maps: bool = True):
        """Per-cell gradients (list of (dP, dX, dY) frames per tube; None with
        maps=False, leaving them on the device) and dL/dz_inv per tube."""
        g = np.ascontiguousarray(dL_dtrace, dtype=np.float32).reshape(self.n, -1)
        if not maps:
            gz = np.zeros(self.n, np.float32)
            check(self.lib, self.lib.vs_batch_adjoint(self.h, _fp(g), None, None, None, _fp(gz)), "vs_batch_adjoint")
            return None, gz
        sizes = [d["frame_h"] * d["frame_w"] for d in self.dims]
        tot = sum(sizes)
        gp, gx, gy = (np.zeros(tot, np.float32) for _ in range(3))
        gz = np.zeros(self.n, np.float32)
        check(self.lib, self.lib.vs_batch_adjoint(self.h, _fp(g), _fp(gp), _fp(gx), _fp(gy), _fp(gz)),
              "vs_batch_adjoint")
        out, off = [], 0
        for d, sz in zip(self.dims, sizes):
            shp = (d["frame_h"], d["frame_w"])
            out.append((gp[off:off + sz].reshape(shp), gx[off:off + sz].reshape(shp), gy[off:off + sz].reshape(shp)))
            off += sz
        return out, gz

    def autotune(self, steps: int):
        best = C.c_int32(-1)
        ms = C.c_float(0)
        check(self.lib, self.lib.vs_batch_autotune(self.h, steps, C.byref(best), C.byref(ms)), "vs_batch_autotune")
        return best.value, ms.value

    def close(self) -> None:
        if self.h:
            self.lib.vs_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def tile_shapes() -> list[tuple[int, int]]:
    lib = load_library()
    out = []
    for i in range(lib.vs_tile_shape_count()):
        r, c = C.c_int32(), C.c_int32()
        check(lib, lib.vs_tile_shape(i, C.byref(r), C.byref(c)), "vs_tile_shape")
        out.append((r.value, c.value))
    return out


def tile_shape_steps(index: int) -> int:
    """Time steps one launch of tile shape `index` advances (1, or 2 for the
    two-step shapes)."""
    lib = load_library()
    k = C.c_int32()
    check(lib, lib.vs_tile_shape_steps(index, C.byref(k)), "vs_tile_shape_steps")
    return k.value

"""Gradients through the solver.

* SectionDepthModel -- the tube's depth maps as a differentiable (torch,
  float64) function of per-section parameters: width (major axis, m) and
  depth (minor axis, m) of the 3:1 elliptical sections.  It follows the
  reference's elliptical depth kernel, open-space reset, half-cell smoothing
  and depthP average (TubeDepth.cu:392-490, 642-762) on the nominal tube's
  rasterisation: wall rows stay where the nominal widths put them
  (TubeGeometry.cu:433-484 rounds them to whole cells, which has no useful
  derivative), and a section's width enters continuously through the
  semi-major axis a = (air cells x ds / 2) x width / nominal width of the
  depth formula.  At the nominal parameters the maps equal vs_build_maps'
  up to float rounding.
* TubeTrace -- torch.autograd.Function over vs_batch_set_maps /
  vs_batch_forward_ckpt (forward) and vs_batch_adjoint (backward): listener
  traces as a function of the depth maps and z_inv of each tube.
* SectionTrace -- the same from section widths / depths directly, with the
  depth model and its reverse pass on the device (vs_batch_set_sections,
  vs_batch_section_gradients).
* spectral_loss -- L2 between log power spectra over 0..fmax, the transfer
  function the reference plots (results/plt_transfer_function.py:20-24).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from .abi import VsDims, check, load_library
from .solver import Batch, Geometry, build_maps

OPEN_SPACE_DEPTH = 0.5     # TubeDepth.cu:91
MIN_DEPTH = 1e-3           # TubeDepth.cu:90


def tube_layout(p, g: Geometry) -> dict:
    """Wall rows, per-column segment ids and section axes (vs_tube_layout)."""
    lib = load_library()
    d = VsDims()
    check(lib, lib.vs_tube_layout(C.byref(p), C.byref(g.struct), C.byref(d), None, None, None, None, None),
          "vs_tube_layout")
    L, n = d.tube_length_cells, len(g.length)
    up, lo, seg = (np.zeros(L, np.int32) for _ in range(3))
    major, minor = np.zeros(n, np.float32), np.zeros(n, np.float32)
    i32 = C.POINTER(C.c_int32)
    f32 = C.POINTER(C.c_float)
    check(lib, lib.vs_tube_layout(C.byref(p), C.byref(g.struct), C.byref(d), up.ctypes.data_as(i32),
                                  lo.ctypes.data_as(i32), seg.ctypes.data_as(i32), major.ctypes.data_as(f32),
                                  minor.ctypes.data_as(f32)), "vs_tube_layout")
    return dict(dims=d.as_dict(), upper=up, lower=lo, segment=seg, major=major, minor=minor)


class SectionDepthModel:
    """Depth maps of one elliptical-section tube as a function of section widths and depths."""

    def __init__(self, p, g: Geometry):
        if p.cross_sectional_shape != 2 or p.fdtd_solver_type != 1:
            raise ValueError("the section model covers 2.5D elliptical sections")
        lay = tube_layout(p, g)
        d = lay["dims"]
        self.H, self.W = d["frame_h"], d["frame_w"]
        self.ds = float(d["ds"])
        self.width0 = torch.tensor(lay["major"], dtype=torch.float64)
        self.depth0 = torch.tensor(lay["minor"], dtype=torch.float64)
        self.nominal = build_maps(p, g)
        # the cells the depth kernel writes, in its order (last write wins):
        # (flat index, segment, nominal semi-major a0, distance in cells or None for a zero)
        writes_x, writes_y = {}, {}
        sx = d["tube_start_x"]
        for i, (u, lo_, s) in enumerate(zip(lay["upper"], lay["lower"], lay["segment"])):
            x = sx + i
            air = int(lo_) - int(u) - 1
            half = math.ceil(air * 0.5) - 1
            a0 = (air * self.ds) / 2.0
            for cc in range(half, -1, -1):
                pu = int(u) + (half - cc) + 1
                pl = int(lo_) - (half - cc) - 1
                writes_x[pu * self.W + x] = (int(s), a0, float(cc))
                writes_x[pl * self.W + x] = (int(s), a0, float(cc))
                writes_y[pu * self.W + x] = (int(s), a0, float(cc) + 0.5 if cc != half else None)
                writes_y[pl * self.W + x] = (int(s), a0, float(cc) - 0.5)
            for r in (int(u), int(lo_)):
                writes_x[r * self.W + x] = (int(s), a0, None)
                writes_y[r * self.W + x] = (int(s), a0, None)
        self.pivot = d["tube_mid_y"] * self.W + d["tube_end_x"]
        self._x = self._pack(writes_x)
        self._y = self._pack(writes_y)

    def _pack(self, writes):
        idx = np.array(list(writes.keys()), np.int64)
        vals = list(writes.values())
        seg = np.array([v[0] for v in vals], np.int64)
        a0 = np.array([v[1] for v in vals], np.float64)
        dist = np.array([0.0 if v[2] is None else v[2] for v in vals], np.float64)
        zero = np.array([v[2] is None for v in vals], bool)
        written = np.zeros(self.H * self.W, bool)
        written[idx] = True
        return dict(idx=torch.from_numpy(idx), seg=torch.from_numpy(seg), a0=torch.from_numpy(a0),
                    dist=torch.from_numpy(dist), zero=torch.from_numpy(zero), unwritten=torch.from_numpy(~written))

    def _raw(self, w, dep, spec):
        a = spec["a0"] * (w[spec["seg"]] / self.width0[spec["seg"]])
        b = dep[spec["seg"]] / 2.0
        y = spec["dist"] * self.ds
        arg = 1.0 - (y * y) / (a * a)
        pos = arg > 0
        # sqrt of the positive part; the masked branch keeps the derivative finite at 0
        v = torch.where(pos, 2.0 * b * torch.sqrt(torch.where(pos, arg, torch.ones_like(arg))), torch.zeros_like(arg))
        v = torch.where(spec["zero"], torch.zeros_like(v), v)
        out = torch.full((self.H * self.W,), OPEN_SPACE_DEPTH, dtype=torch.float64)
        return out.index_put((spec["idx"],), v)

    def maps(self, width: torch.Tensor, depth: torch.Tensor):
        """(depth_p, depth_x, depth_y) frames (float64) for section widths / depths (m)."""
        H, W = self.H, self.W
        x = self._raw(width, depth, self._x)
        y = self._raw(width, depth, self._y)
        # open-space cells take the (mid row, tube end) value (resetOpenSpaceDepth)
        x = torch.where(self._x["unwritten"], x[self.pivot], x).reshape(H, W)
        y = torch.where(self._y["unwritten"], y[self.pivot], y).reshape(H, W)
        px, py = x.reshape(-1)[self.pivot], y.reshape(-1)[self.pivot]
        # half-cell smoothing (smoothDepthX / smoothDepthY)
        xr = torch.cat([x[:, 1:], px.expand(H, 1)], dim=1)
        ya = torch.cat([py.expand(1, W), y[:-1, :]], dim=0)
        xs = 0.5 * (x + xr)
        ys = 0.5 * (y + ya)
        # depthP = mean of the four face depths (updateDepthP)
        pxs, pys = xs.reshape(-1)[self.pivot], ys.reshape(-1)[self.pivot]
        xl = torch.cat([pxs.expand(H, 1), xs[:, :-1]], dim=1)
        yb = torch.cat([ys[1:, :], pys.expand(1, W)], dim=0)
        dp = 0.25 * (xs + ys + xl + yb)
        # depths below the (float) minimum are raised to it (TubeDepth.cu:90)
        lo = torch.tensor(float(np.float32(MIN_DEPTH)), dtype=torch.float64)
        return torch.where(dp < lo, lo, dp), torch.where(xs < lo, lo, xs), torch.where(ys < lo, lo, ys)


class TubeTrace(torch.autograd.Function):
    """Listener traces (n, steps) of a Batch as a function of each tube's depth
    maps and z_inv; backward runs the checkpointed adjoint."""

    @staticmethod
    def forward(ctx, batch: Batch, steps: int, ckpt_every: int, z_inv: torch.Tensor, *maps: torch.Tensor):
        n = batch.n
        for i in range(n):
            dp, dx, dy = (m.detach().to(torch.float32).cpu().numpy() for m in maps[3 * i:3 * i + 3])
            batch.set_maps(i, dp, dx, dy, float(z_inv[i]))
        tr = batch.forward_ckpt(steps, ckpt_every)
        ctx.batch = batch
        ctx.n = n
        return torch.from_numpy(tr).to(torch.float64)

    @staticmethod
    def backward(ctx, grad_trace: torch.Tensor):
        grads, gz = ctx.batch.adjoint(grad_trace.detach().to(torch.float32).cpu().numpy())
        out = [None, None, None, torch.from_numpy(gz.astype(np.float64))]
        for gp, gx, gy in grads:
            out += [torch.from_numpy(gp.astype(np.float64)), torch.from_numpy(gx.astype(np.float64)),
                    torch.from_numpy(gy.astype(np.float64))]
        return tuple(out)


class SectionTrace(torch.autograd.Function):
    """Listener traces (n, steps) of a Batch as a function of each tube's
    section widths and depths (m) and z_inv, with the depth maps built on the
    device (vs_batch_set_sections) and the section gradients reduced there
    (vs_batch_section_gradients).  widths / depths: one 1-D tensor per tube."""

    @staticmethod
    def forward(ctx, batch: Batch, steps: int, ckpt_every: int, z_inv: torch.Tensor, *sections: torch.Tensor):
        n = batch.n
        ws = [t.detach().cpu().numpy() for t in sections[:n]]
        ds = [t.detach().cpu().numpy() for t in sections[n:]]
        batch.set_sections(ws, ds, z_inv.detach().cpu().numpy())
        ctx.batch = batch
        ctx.device = getattr(batch, "trace_device", None)
        if ctx.device is not None:
            # traces stay on the GPU: the loss and its gradient are computed there
            # and dL/dtrace goes back to the adjoint without a host copy
            tr = torch.empty((n, steps), dtype=torch.float32, device=ctx.device)
            batch.forward_ckpt_device(steps, ckpt_every, tr.data_ptr())
            return tr.to(torch.float64)
        tr = batch.forward_ckpt(steps, ckpt_every)
        return torch.from_numpy(tr).to(torch.float64)

    @staticmethod
    def backward(ctx, grad_trace: torch.Tensor):
        if ctx.device is not None:
            g32 = grad_trace.detach().to(device=ctx.device, dtype=torch.float32).contiguous()
            gz = ctx.batch.adjoint_device(g32.data_ptr())
        else:
            _, gz = ctx.batch.adjoint(grad_trace.detach().to(torch.float32).cpu().numpy(), maps=False)
        g = ctx.batch.section_gradients()
        return (None, None, None, torch.from_numpy(gz.astype(np.float64)),
                *[torch.from_numpy(w) for w, _ in g], *[torch.from_numpy(d) for _, d in g])


def log_power_spectrum(trace: torch.Tensor, fs: float, fmax: float = 5000.0, floor: float = 1e-30) -> torch.Tensor:
    """log |FFT|^2 of the trace on the bins 0 < f <= fmax."""
    X = torch.fft.rfft(trace, dim=-1)
    f = torch.fft.rfftfreq(trace.shape[-1], d=1.0 / fs)
    sel = (f > 0) & (f <= fmax)
    p = (X.real ** 2 + X.imag ** 2)[..., sel]
    return torch.log(p + floor)


def spectral_loss(trace: torch.Tensor, target: torch.Tensor, fs: float, fmax: float = 5000.0) -> torch.Tensor:
    """Mean squared difference of log power spectra over 0..fmax (per tube, summed over tubes)."""
    d = log_power_spectrum(trace, fs, fmax) - log_power_spectrum(target, fs, fmax)
    return (d * d).mean(dim=-1).sum()


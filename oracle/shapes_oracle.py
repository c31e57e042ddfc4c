"""Single-plane-symmetric sections (cross_sectional_shape 3), restating the
reference's ShapeGenerator::combineRegularShapes (ShapeGenerator.cpp:35-197),
ShapeAlignment (ShapeAlignment.cu:9-152) and
TubeDepth::generateTubeDepthSinglePlaneSymmetricShape (TubeDepth.cu:493-640)
followed by generateDepthP / setMinDepth (TubeDepth.cu:215-253, 642-762).

TEST INFRASTRUCTURE ONLY.  Parity with the reference is unpinned: the
reference takes the arcs' intersection, the contour area and the line
crossings from Boost.Geometry (absent here, so the reference cannot be built
to produce golden maps).  This restatement computes those in double from the
float points (segment crossings; ring area as the sequential sum of
(y1 + y2)(z1 - z2) / 2), as the library does, and keeps every float
expression of the reference in float32; the tests use it to check the
library's map builder cell for cell on the same wall layout.
"""
from __future__ import annotations

import ctypes
import ctypes.util

import numpy as np

f32 = np.float32
_libm = ctypes.CDLL(ctypes.util.find_library("m"))
for _name in ("cosf", "sinf"):
    getattr(_libm, _name).restype = ctypes.c_float
    getattr(_libm, _name).argtypes = [ctypes.c_float]
_libm.atan2f.restype = ctypes.c_float
_libm.atan2f.argtypes = [ctypes.c_float, ctypes.c_float]

MM = f32(1e-3 * 1.0)
N_COORD = 1999                      # TubeGeometry.cu:373


def linspace(start, end, n):
    """Utils::linspace (Utils.cpp:59-75) in float."""
    start, end = f32(start), f32(end)
    if n == 1:
        return np.array([start], f32)
    step = f32((end - start) / f32(n - 1))
    return (start + step * np.arange(n, dtype=np.int64).astype(f32)).astype(f32)


def ellipse_arc(y0, y1, a, b, n, yc):
    """ShapeGenerator::generateEllipseCoordinates (ShapeGenerator.cpp:222-262)."""
    y = linspace(y0, y1, n)
    t = (y - f32(yc)).astype(f32)
    d2 = (t * t).astype(f32)
    a2, b2 = f32(f32(a) * f32(a)), f32(f32(b) * f32(b))
    d2[0] = a2
    for i in range(n // 2):
        d2[n - i - 1] = d2[i]
    z = np.sqrt(np.maximum(f32(0), (b2 * (f32(1) - d2 / a2)).astype(f32))).astype(f32)
    return np.stack([y, z], axis=1)


def crossings(p1, p2, q1, q2):
    """Crossing points (double, then float) of segments p1-p2 with q1-q2 (arrays)."""
    px, py = p1[..., 0].astype(np.float64), p1[..., 1].astype(np.float64)
    rx, ry = p2[..., 0].astype(np.float64) - px, p2[..., 1].astype(np.float64) - py
    qx, qy = q1[..., 0].astype(np.float64), q1[..., 1].astype(np.float64)
    sx, sy = q2[..., 0].astype(np.float64) - qx, q2[..., 1].astype(np.float64) - qy
    den = rx * sy - ry * sx
    with np.errstate(divide="ignore", invalid="ignore"):
        t = ((qx - px) * sy - (qy - py) * sx) / den
        u = ((qx - px) * ry - (qy - py) * rx) / den
    ok = (den != 0.0) & (t >= 0.0) & (t <= 1.0) & (u >= 0.0) & (u <= 1.0)
    return ok, (px + t * rx).astype(f32), (py + t * ry).astype(f32)


def first_crossing(s1, s2):
    """First crossing along s1 of two polylines whose y increases along them."""
    for i in range(len(s1) - 1):
        lo, hi = min(s1[i, 0], s1[i + 1, 0]), max(s1[i, 0], s1[i + 1, 0])
        seg_lo = np.minimum(s2[:-1, 0], s2[1:, 0])
        seg_hi = np.maximum(s2[:-1, 0], s2[1:, 0])
        cand = np.nonzero((seg_hi >= lo) & (seg_lo <= hi))[0]
        if cand.size == 0:
            continue
        ok, y, z = crossings(np.repeat(s1[i][None], cand.size, 0), np.repeat(s1[i + 1][None], cand.size, 0),
                             s2[cand], s2[cand + 1])
        if ok.any():
            k = int(np.nonzero(ok)[0][0])
            return np.array([y[k], z[k]], f32)
    return None


def ring_area(c):
    """|area| of the ring through the points, sequential double sum."""
    a, b = c.astype(np.float64), np.roll(c, -1, axis=0).astype(np.float64)
    terms = (a[:, 0] + b[:, 0]) * (a[:, 1] - b[:, 1])
    return f32(abs(np.cumsum(terms)[-1] / 2.0))


def half_contour(ip, a1, b1, a2, b2, yc1, yc2, ys1, ye2, nhalf):
    """ShapeGenerator::finalContourCoordinates (ShapeGenerator.cpp:264-309)."""
    seg = nhalf - 1
    y1, y2 = linspace(ys1, ip[0], seg), linspace(ip[0], ye2, seg)
    d1, d2 = (y1 - f32(yc1)).astype(f32), (y2 - f32(yc2)).astype(f32)
    z1 = np.sqrt(np.maximum(f32(0), (f32(b1 * b1) * (f32(1) - (d1 * d1) / f32(a1 * a1))).astype(f32))).astype(f32)
    z2 = np.sqrt(np.maximum(f32(0), (f32(b2 * b2) * (f32(1) - (d2 * d2) / f32(a2 * a2))).astype(f32))).astype(f32)
    return np.concatenate([np.stack([y1, z1], 1), ip[None].astype(f32), np.stack([y2, z2], 1)]).astype(f32)


def section_shape(area: float):
    """(aligned full contour (n, 2) float32, diameter) of a section of `area` m^2."""
    nhalf = (N_COORD + 1) // 2
    area = f32(area)
    m = f32(3.0)
    x = f32(area / (m + f32(1)))
    A1, A2 = f32(m * x), f32(f32(1) * x)
    l1 = np.sqrt(f32(float(A1) / (np.pi * 3.0 * 1.0))).astype(f32)
    l2 = np.sqrt(f32(float(A2) / (np.pi * 1.0 * 1.0))).astype(f32)
    a1, b1, a2, b2 = f32(l1 * f32(3)), f32(l1 * f32(1)), f32(l2 * f32(1)), f32(l2 * f32(1))
    yc1 = f32(0)
    yc2 = f32(f32(yc1 + a1) + f32(f32(0.003) * MM))
    grow = f32(MM * f32(0.01))
    got, it, half = f32(-1), 0, None
    while got < area:
        if it > 0:
            a1, b1, a2, b2 = f32(a1 + grow), f32(b1 + grow), f32(a2 + grow), f32(b2 + grow)
        it += 1
        y0, y1, z0, z1 = f32(yc1 - a1), f32(yc1 + a1), f32(yc2 - a2), f32(yc2 + a2)
        s1 = ellipse_arc(y0, y1, a1, b1, nhalf, yc1)
        s2 = ellipse_arc(z0, z1, a2, b2, nhalf, yc2)
        ip = first_crossing(s1, s2)
        half = half_contour(ip, a1, b1, a2, b2, yc1, yc2, y0, z1, nhalf)
        got = f32(f32(2) * ring_area(half))
    half[0, 1] = f32(0)
    half[-1, 1] = f32(0)
    mirror = half[-2::-1].copy()
    mirror[:, 1] = (f32(-1) * mirror[:, 1]).astype(f32)
    full = np.concatenate([half, mirror]).astype(f32)
    # ShapeAlignment::shapeDiameter: first row with the largest row maximum,
    # first column of that row's maximum
    best, bi, bj = f32(0), 0, 0
    for s in range(0, len(full), 256):
        blk = full[s:s + 256]
        dy = (blk[:, None, 0] - full[None, :, 0]).astype(f32)
        dz = (blk[:, None, 1] - full[None, :, 1]).astype(f32)
        d = np.sqrt((dy * dy + dz * dz).astype(f32)).astype(f32)
        rmax = d.max(axis=1)
        for r in range(len(blk)):
            if rmax[r] > best:
                best, bi, bj = rmax[r], s + r, int(np.argmax(d[r]))
    # ShapeAlignment::rotateShapeAboutOrigin
    dy = f32(full[bj, 0] - full[bi, 0])
    dz = f32(full[bj, 1] - full[bi, 1])
    th = f32(_libm.atan2f(float(dz), float(dy)))
    c, s = f32(_libm.cosf(float(f32(-1) * th))), f32(_libm.sinf(float(f32(-1) * th)))
    y, z = full[:, 0].copy(), full[:, 1].copy()
    full[:, 0] = (c * y - s * z).astype(f32)
    full[:, 1] = (s * y + c * z).astype(f32)
    min_y, min_z = full[:, 0].min(), full[:, 1].min()
    sh_y = f32((-min_y if min_y < 0 else f32(0)) + f32(0.05))
    sh_z = f32((-min_z if min_z < 0 else f32(0)) + f32(0.05))
    full[:, 0] = (full[:, 0] + sh_y).astype(f32)
    full[:, 1] = (full[:, 1] + sh_z).astype(f32)
    return full, best


def half_depth(shape, y, zlo, zhi):
    """Half the z extent of the contour along the vertical line y; None when missed."""
    p1, p2 = shape[:-1], shape[1:]
    lo, hi = np.minimum(p1[:, 0], p2[:, 0]), np.maximum(p1[:, 0], p2[:, 0])
    cand = np.nonzero((y >= lo) & (y <= hi))[0]
    if cand.size == 0:
        return None
    q1 = np.repeat(np.array([[y, zlo]], f32), cand.size, 0)
    q2 = np.repeat(np.array([[y, zhi]], f32), cand.size, 0)
    ok, _, z = crossings(p1[cand], p2[cand], q1, q2)
    if not ok.any():
        return None
    z = z[ok]
    return f32((z.max() - z.min()) / f32(2))


def depth_maps(layout: dict, shapes, ds: float, osd: float = 0.5):
    """dP, dX, dY frames of a 2.5D shape-3 tube on the library's wall layout
    (vocalsim_b200.autograd.tube_layout)."""
    d = layout["dims"]
    H, W = d["frame_h"], d["frame_w"]
    ds = f32(ds)
    fill = f32(1.0 * osd)
    dX = np.full((H, W), fill, f32)
    dY = np.full((H, W), fill, f32)
    sx = d["tube_start_x"]
    for i, (up, down, sg) in enumerate(zip(layout["upper"], layout["lower"], layout["segment"])):
        x = sx + i
        sh = shapes[int(sg)]
        zlo = f32(float(sh[:, 1].min()) - 0.001)
        zhi = f32(float(sh[:, 1].max()) + 0.001)
        min_y = sh[:, 0].min()
        air = int(down) - int(up) - 1
        for k in range(1, air + 1):
            row = int(down) - k
            off_x = f32((k - 0.5) * float(ds))
            off_y = f32(f32(k) * ds)
            dX[row, x] = half_depth(sh, f32(min_y + off_x), zlo, zhi)
            dY[row, x] = half_depth(sh, f32(min_y + off_y), zlo, zhi) if k < air else f32(0)
        dX[down, x] = dX[up, x] = f32(0)
        dY[down, x] = dY[up, x] = f32(0)
    # generateDepthP (pivot = the cell (mid row, tube end)) and setMinDepth
    py0, px0 = d["tube_mid_y"], d["tube_end_x"]
    vx0, vy0 = dX[py0, px0], dY[py0, px0]
    dX[dX == fill] = vx0
    dY[dY == fill] = vy0
    right = np.concatenate([dX[:, 1:], np.full((H, 1), dX[py0, px0], f32)], axis=1)
    above = np.concatenate([np.full((1, W), dY[py0, px0], f32), dY[:-1]], axis=0)
    xs = (f32(0.5) * (dX + right)).astype(f32)
    ys = (f32(0.5) * (dY + above)).astype(f32)
    left = np.concatenate([np.full((H, 1), xs[py0, px0], f32), xs[:, :-1]], axis=1)
    below = np.concatenate([ys[1:], np.full((1, W), ys[py0, px0], f32)], axis=0)
    dP = (f32(0.25) * (((xs + ys).astype(f32) + left).astype(f32) + below).astype(f32)).astype(f32)
    lo = f32(0.001)
    return np.maximum(dP, lo), np.maximum(xs, lo), np.maximum(ys, lo)

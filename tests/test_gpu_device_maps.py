"""The batched device map builder (vs_mapbuild.cu) against the host builder.

A batch paints the maps of its circular and elliptical tubes on the device at
vs_batch_create; vs_batch_get_maps reads back what the kernels step with.
Cell types, z_inv and the three depth maps must equal vs_build_maps (the host
restatement of FDTDSolver::setupWaveSolver, itself pinned to the reference's
own setup) bit for bit, over the switches that shape the maps: 2D / 2.5D
solver, circular / elliptical sections, PML on / off, open / Dirichlet mouth,
uniform depth, the fused radicand, sampling rates 1 / 3 / 30, and mixed
batches with tubes the host still builds (single-plane-symmetric sections,
the open-space domain).
"""
import numpy as np
import pytest

import vocalsim_b200 as V
from vocalsim_b200 import synthetic as S

pytestmark = pytest.mark.gpu

KEYS = ("cell_type", "depth_p", "depth_x", "depth_y", "z_inv")


def _assert_same(b, i, p, g):
    dev = b.get_maps(i)
    host = V.build_maps(p, g)
    for k in KEYS:
        a, h = dev[k], host[k]
        assert a.shape == h.shape, k
        if not np.array_equal(a, h):
            bad = np.argwhere(a != h)
            r, c = bad[0]
            raise AssertionError(f"tube {i} {k}: {len(bad)} cells differ, first at ({r}, {c}): "
                                 f"device {a[r, c]!r} host {h[r, c]!r}")


CASES = {
    "ellipse": dict(cross_sectional_shape=2),
    "circle": dict(cross_sectional_shape=1),
    "circle_no_fma": dict(cross_sectional_shape=1, depth_fma=0),
    "ellipse_dirichlet": dict(cross_sectional_shape=2, mouth_radiation_cond=1),
    "ellipse_no_pml_dirichlet": dict(cross_sectional_shape=2, pml_flag=0, mouth_radiation_cond=1),
    "circle_2d": dict(cross_sectional_shape=1, fdtd_solver_type=0),
    "ellipse_2d_dirichlet": dict(cross_sectional_shape=2, fdtd_solver_type=0, mouth_radiation_cond=1),
    "uniform_depth": dict(cross_sectional_shape=1, uniform_depth_m=0.02),
    "ellipse_mul3": dict(cross_sectional_shape=2, srate_mul=3),
    "ellipse_mul30": dict(cross_sectional_shape=2, srate_mul=30),
}


@pytest.mark.parametrize("name", list(CASES))
def test_device_maps_equal_host_maps(name, cuda_ok):
    kw = CASES[name]
    geos = [S.vowel_tube(0), S.vowel_tube(5), S.batch_tube(3)[:2], S.batch_tube(11)[:2], S.uniform_tube()]
    ps = [V.params(num_steps=10, **kw) for _ in geos]
    gs = [V.Geometry(*t) for t in geos]
    b = V.Batch(ps, gs)
    for i, (p, g) in enumerate(zip(ps, gs)):
        _assert_same(b, i, p, g)
    b.close()


def test_mixed_batch_with_host_built_tubes(cuda_ok):
    """Single-plane-symmetric sections are built on the host; a batch mixing
    them with device-built tubes keeps both sets of maps."""
    geos = [S.vowel_tube(2), S.vowel_tube(2), S.batch_tube(7)[:2]]
    shapes = [2, 3, 1]
    ps = [V.params(num_steps=10, cross_sectional_shape=s) for s in shapes]
    gs = [V.Geometry(*t) for t in geos]
    b = V.Batch(ps, gs)
    for i, (p, g) in enumerate(zip(ps, gs)):
        _assert_same(b, i, p, g)
    b.close()


def test_open_space_single_tube(cuda_ok):
    p = V.params(num_steps=10, simulation_type=0)
    b = V.Batch([p], [None])
    _assert_same(b, 0, p, None)
    b.close()


def test_set_maps_on_a_device_built_tube(cuda_ok):
    """vs_batch_set_maps on a device-built tube replaces the depth maps it is
    given and keeps the device-built ones it is not."""
    g = V.Geometry(*S.vowel_tube(1))
    p = V.params(num_steps=10, cross_sectional_shape=2)
    host = V.build_maps(p, g)
    b = V.Batch([p], [g])
    dx = host["depth_x"] * 1.25
    b.set_maps(0, depth_x=dx, z_inv=float(host["dims"]["z_inv_val"]))
    got = b.get_maps(0)
    assert np.array_equal(got["depth_x"], dx.astype(np.float32))
    assert np.array_equal(got["depth_p"], host["depth_p"])
    assert np.array_equal(got["depth_y"], host["depth_y"])
    assert np.array_equal(got["cell_type"], host["cell_type"])
    b.close()

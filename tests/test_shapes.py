"""Single-plane-symmetric sections (cross_sectional_shape 3): the library's
host map builder against the oracle's restatement of the reference's shape
construction and depth sampling (ShapeGenerator.cpp:35-197,
ShapeAlignment.cu:9-152, TubeDepth.cu:493-640), cell for cell on the same
wall layout.  Parity with the reference itself is unpinned (it needs
Boost.Geometry, absent here); see oracle/shapes_oracle.py."""
import numpy as np
import pytest

import oracle as O
import shapes_oracle as SO
import vocalsim_b200 as V
from vocalsim_b200.autograd import tube_layout

LENGTHS = np.array([3.0, 2.5, 4.0, 3.0, 2.0, 3.0], np.float32)
AREAS = np.array([0.6, 1.8, 3.2, 2.4, 1.1, 0.8], np.float32)


@pytest.fixture(scope="module")
def built():
    p = V.params(cross_sectional_shape=3)
    g = V.Geometry(LENGTHS, AREAS)
    maps = V.build_maps(p, g)
    layout = tube_layout(p, g)
    shapes = [SO.section_shape(float(np.float32(a) * np.float32(1e-2) * np.float32(1e-2))) for a in AREAS]
    return maps, layout, shapes


def test_section_diameters_set_the_walls(built):
    maps, layout, shapes = built
    assert np.array_equal(layout["major"], np.array([d for _, d in shapes], np.float32))
    ds = np.float32(maps["dims"]["ds"])
    # diameters rounded to an odd cell count, even counts always down (TubeGeometry.cu:139-146)
    for up, lo, sg in zip(layout["upper"], layout["lower"], layout["segment"]):
        air = int(lo) - int(up) - 1
        c = int(np.round(shapes[int(sg)][1] / ds)) or 1
        assert air == (c - 1 if c % 2 == 0 else c)


def test_contour_area_reaches_the_section_area(built):
    _, _, shapes = built
    for (full, d), a in zip(shapes, AREAS):
        area = float(a) * 1e-4
        ring = SO.ring_area(full[: (len(full) + 1) // 2])
        assert 2 * float(ring) >= area * (1 - 1e-6)
        assert 2 * float(ring) < area * 1.05
        span_y = float(full[:, 0].max() - full[:, 0].min())
        assert abs(span_y - float(d)) <= 1e-6


def test_depth_maps_equal_the_oracle(built):
    maps, layout, shapes = built
    dP, dX, dY = SO.depth_maps(layout, [s for s, _ in shapes], maps["dims"]["ds"])
    assert np.array_equal(maps["depth_x"], dX)
    assert np.array_equal(maps["depth_y"], dY)
    assert np.array_equal(maps["depth_p"], dP)
    assert maps["depth_x"].max() > 0.002


def test_cell_types_equal_the_oracle_rasterisation(built):
    """With the section diameters given, the oracle rasterises a shape-3 tube
    as it does the other shapes; cell types, z_inv and dims must agree."""
    maps, layout, _ = built
    O.set_sps_diameters(layout["major"])
    try:
        om = O.maps(O.params(cross_sectional_shape=3), O.Geometry(LENGTHS, AREAS))
    finally:
        O.set_sps_diameters([])
    assert np.array_equal(om["cell_type"], maps["cell_type"])
    assert np.array_equal(om["z_inv"], maps["z_inv"])
    for k in ("frame_h", "frame_w", "listener_x", "listener_y", "excitation_x", "excitation_y"):
        assert om["dims"][k] == maps["dims"][k]


def test_shape3_in_the_2d_solver(built):
    """The 2D solver scales the section diameters (tubeAreaScaling) and keeps
    unit depths; the oracle rasteriser agrees given the same diameters."""
    _, layout, _ = built
    p = V.params(cross_sectional_shape=3, fdtd_solver_type=0)
    maps = V.build_maps(p, V.Geometry(LENGTHS, AREAS))
    assert np.all(maps["depth_p"] == 1.0) and np.all(maps["depth_x"] == 1.0)
    O.set_sps_diameters(layout["major"])
    try:
        om = O.maps(O.params(cross_sectional_shape=3, fdtd_solver_type=0), O.Geometry(LENGTHS, AREAS))
    finally:
        O.set_sps_diameters([])
    assert np.array_equal(om["cell_type"], maps["cell_type"])


def test_shape3_rejects_the_uniform_depth_override():
    with pytest.raises(V.VsError) as e:
        V.build_maps(V.params(cross_sectional_shape=3, uniform_depth_m=0.02), V.Geometry(LENGTHS, AREAS))
    assert e.value.status == 7


def test_shape3_is_outside_the_section_depth_model():
    """The device section model covers the 3:1 elliptical sections only."""
    from vocalsim_b200.autograd import SectionDepthModel
    with pytest.raises(ValueError):
        SectionDepthModel(V.params(cross_sectional_shape=3), V.Geometry(LENGTHS, AREAS))

"""Grid maps: the product's host builder (vs_build_maps) against the oracle.

The maps are integer / exact-float work, so the bar is bit equality of the
cell-type, depth (P, X, Y) and z_inv frames and of every grid dimension.
Inputs: the reference's own area functions (tests/golden/
reference_area_functions.npz, parsed from data/tube-geometry with strtof),
seeded synthetic tubes, and the open-space domain.
"""
from pathlib import Path

import numpy as np
import pytest

import oracle as O
import vocalsim_b200 as V
from vocalsim_b200 import synthetic as S
from vocalsim_b200.abi import VsError

AREAS = np.load(Path(__file__).parent / "golden" / "reference_area_functions.npz")
FILES = ["vocaltract_a", "vocaltract_i", "vocaltract_u", "cylindrical-tube"]


def ref_geometry(name):
    return AREAS[f"{name}_length_cm"], AREAS[f"{name}_area_cm2"]


def compare(kw, L=None, A=None):
    po, pv = O.params(**kw), V.params(**kw)
    go = O.Geometry(L, A) if L is not None else None
    gv = V.Geometry(L, A) if L is not None else None
    mo = O.maps(po, go)
    mv = V.build_maps(pv, gv)
    assert mv["dims"] == mo["dims"]
    for k in ("cell_type", "depth_p", "depth_x", "depth_y", "z_inv"):
        assert np.array_equal(mv[k], mo[k]), k
    return mv


@pytest.mark.parametrize("name", FILES)
@pytest.mark.parametrize("shape", [1, 2])
@pytest.mark.parametrize("solver", [0, 1])
@pytest.mark.parametrize("mouth,pml", [(0, 1), (1, 1), (1, 0)])
def test_reference_area_functions(name, shape, solver, mouth, pml):
    L, A = ref_geometry(name)
    compare(dict(cross_sectional_shape=shape, fdtd_solver_type=solver, mouth_radiation_cond=mouth,
                 pml_flag=pml), L, A)


@pytest.mark.parametrize("fma", [0, 1])
def test_circular_depth_contraction_variants(fma):
    L, A = ref_geometry("vocaltract_a")
    compare(dict(cross_sectional_shape=1, depth_fma=fma), L, A)


def test_fma_variant_changes_some_circular_depths():
    L, A = ref_geometry("vocaltract_u")
    a = V.build_maps(V.params(depth_fma=0), V.Geometry(L, A))
    b = V.build_maps(V.params(depth_fma=1), V.Geometry(L, A))
    assert np.array_equal(a["cell_type"], b["cell_type"])
    for k in ("depth_p", "depth_x", "depth_y"):
        d = np.abs(a[k] - b[k])
        assert 0 < d.max() <= 8e-7 * np.abs(b[k]).max()      # last-bit differences only


@pytest.mark.parametrize("seed", range(12))
def test_synthetic_tubes(seed):
    L, A, _, _ = S.batch_tube(seed)
    compare(dict(cross_sectional_shape=2), L, A)
    compare(dict(cross_sectional_shape=2, srate_mul=30), L, A)
    Lv, Av = S.vowel_tube(seed)
    compare(dict(cross_sectional_shape=2, source_type=2), Lv, Av)


def test_uniform_tube_maps():
    L, A = S.uniform_tube()
    m = compare(dict(mu3d=0.005, uniform_depth_m=0.02), L, A)
    d = m["dims"]
    assert (d["frame_h"], d["frame_w"], d["interior_cells"]) == (57, 253, 13805)
    assert d["listener_x"] == d["tube_end_x"] + 3 + 4 == 248
    ct = m["cell_type"]
    # air rows of the tube carry the override depth, walls zero depth before clamp
    assert np.all(m["depth_x"][d["tube_mid_y"], d["tube_start_x"]:d["tube_end_x"]] == np.float32(0.02))
    assert ct[d["tube_mid_y"], d["excitation_x"]] == V.CELL_EXCITATION
    assert (ct[0] == V.CELL_DEAD).all() and (ct[:, -1] == V.CELL_DEAD).all()
    assert set(np.unique(ct[1, 1:-1])) == {8}          # outermost PML layer


def test_open_space_domain():
    m = compare(dict(simulation_type=0))
    assert (m["dims"]["frame_h"], m["dims"]["frame_w"]) == (43 + 2 + 12, 341 + 2 + 12)
    compare(dict(simulation_type=0, fdtd_solver_type=0, pml_flag=0))


def test_dirichlet_column_and_excitation_walls():
    L, A = ref_geometry("vocaltract_i")
    m = compare(dict(mouth_radiation_cond=1), L, A)
    d, ct, z = m["dims"], m["cell_type"], m["z_inv"]
    col = ct[:, d["tube_end_x"] + 1]
    assert (col == V.CELL_NOPRESSURE).sum() >= 3
    exc_col = d["excitation_x"]
    walls = np.where(ct[:, exc_col] == V.CELL_WALL)[0]
    assert len(walls) == 2
    assert np.all(z[walls, exc_col] == 0)             # excitation walls carry no segment id
    assert np.all(z[ct == V.CELL_AIR] == 0)


@pytest.mark.parametrize("name", FILES)
def test_wall_rows_independent_of_summation_order(name):
    """The reference sums section lengths with a device scan whose order is not
    sequential; every wall-row decision must come out the same for any order.
    Checked by recomputing the decisions with sequential, pairwise, blocked and
    exact (double) cumulative sums."""
    L, A = ref_geometry(name)
    for seed in range(4):
        Ls, As, _, _ = S.batch_tube(seed)
        check_scan_orders(Ls)
    check_scan_orders(L)


def check_scan_orders(L_cm):
    k = O.consts(15)
    ds = np.float32(k[4])
    lm = (np.asarray(L_cm, np.float32) * np.float32(0.01)).astype(np.float32)
    n = len(lm)

    def seq(v):
        out, acc = [], np.float32(0)
        for x in v:
            acc = np.float32(acc + x)
            out.append(acc)
        return np.array(out, np.float32)

    def blocked(v, b):
        out = np.zeros(n, np.float32)
        pref = np.float32(0)
        for s in range(0, n, b):
            loc = seq(v[s:s + b])
            out[s:s + b] = np.array([np.float32(pref + x) for x in loc], np.float32)
            pref = np.float32(pref + loc[-1])
        return out

    orders = [seq(lm), blocked(lm, 4), blocked(lm, 7), blocked(lm, 15), np.cumsum(lm.astype(np.float64))]
    total = seq(lm)[-1]
    cells = int(np.round(total / ds))
    half = np.float32(ds * np.float32(0.5))
    decisions = []
    for cum in orders:
        segs = []
        for i in range(cells):
            x = np.float32((i + 1) * ds)
            s = 0
            while s < n - 1 and x > (np.float32(cum[s] + half) if cum.dtype == np.float32 else cum[s] + half):
                s += 1
            segs.append(s)
        decisions.append(segs)
    for d in decisions[1:]:
        assert d == decisions[0]


@pytest.mark.parametrize("bad", [
    dict(n=0), dict(area=0.0), dict(area=-1.0), dict(length=0.0), dict(area=float("nan")),
])
def test_invalid_geometry_rejected(bad):
    n = bad.get("n", 5)
    L = np.full(n, bad.get("length", 3.5), np.float32)
    A = np.full(n, bad.get("area", 2.0), np.float32)
    with pytest.raises(VsError) as e:
        V.build_maps(V.params(), V.Geometry(L, A))
    assert e.value.status == 2       # VS_ERR_GEOMETRY


@pytest.mark.parametrize("field,value,status", [
    ("srate_mul", 0, 1), ("fdtd_solver_type", 3, 1), ("pml_flag", 2, 1), ("engine", 0, 1),
    ("source_type", 9, 1), ("cross_sectional_shape", 4, 7), ("listener_mode", 5, 1), ("tmm_f64", 2, 1),
    ("fast_math", 2, 1),
])
def test_invalid_params_rejected(field, value, status):
    L, A = S.vowel_tube(0)
    with pytest.raises(VsError) as e:
        V.build_maps(V.params(**{field: value}), V.Geometry(L, A))
    assert e.value.status == status


def test_fast_math_with_coupled_wall_rejected():
    L, A = S.vowel_tube(0)
    with pytest.raises(VsError) as e:
        V.build_maps(V.params(fast_math=1, cross_sectional_shape=2, wall_coupling=0.5), V.Geometry(L, A))
    assert e.value.status == 7


def test_listener_outside_frame_rejected():
    """PML off + open mouth: the reference formula puts the listener past the frame
    (FDTDSolver.cu:605 with frameW from TubeGeometry.cu:169-175); both sides refuse."""
    L, A = S.vowel_tube(0)
    with pytest.raises(VsError):
        V.build_maps(V.params(pml_flag=0), V.Geometry(L, A))
    with pytest.raises(RuntimeError):
        O.maps(O.params(pml_flag=0), O.Geometry(L, A))


def test_tiny_tube_one_cell_wide():
    """Area so small the diameter rounds to 0 cells and is forced to 1
    (TubeGeometry.cu:135-137).  With two roundings the circular depth radicand
    is exactly 0; contracted into an FMA (as nvcc builds TubeDepth.cu:355-370)
    r^2 - d^2 comes out slightly negative, where the reference kernel executes
    `trap` (TubeDepth.cu:280-286).  Both builders report VS_ERR_NEGATIVE_SQRT."""
    L = np.array([1.0, 1.0], np.float32)
    A = np.array([1e-4, 1e-4], np.float32)
    m = compare(dict(cross_sectional_shape=1, depth_fma=0), L, A)
    assert m["dims"]["frame_h"] == 1 + 2 + 2 + 12
    with pytest.raises(VsError) as e:
        V.build_maps(V.params(cross_sectional_shape=1, depth_fma=1), V.Geometry(L, A))
    assert e.value.status == 8
    with pytest.raises(RuntimeError, match="status 8"):
        O.maps(O.params(cross_sectional_shape=1, depth_fma=1), O.Geometry(L, A))


def test_section_depth_model_reproduces_builder_maps():
    """The differentiable section model (vocalsim_b200.autograd) at nominal section
    widths / depths gives the reference maps up to float rounding."""
    import torch
    from vocalsim_b200.autograd import SectionDepthModel
    for seed in (0, 7):
        L, A = S.vowel_tube(seed)
        M = SectionDepthModel(V.params(cross_sectional_shape=2), V.Geometry(L, A))
        dp, dx, dy = M.maps(M.width0.clone(), M.depth0.clone())
        for t, ref in ((dp, M.nominal["depth_p"]), (dx, M.nominal["depth_x"]), (dy, M.nominal["depth_y"])):
            assert np.abs(t.numpy() - ref).max() <= 4e-6 * np.abs(ref).max()
        # widths move depths continuously (relaxed rasterisation)
        w = M.width0.clone().requires_grad_(True)
        M.maps(w, M.depth0)[1].sum().backward()
        assert torch.count_nonzero(w.grad) > 0

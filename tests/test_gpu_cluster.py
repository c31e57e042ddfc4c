"""The cluster kernel: one tube on one thread-block cluster, a whole run per
launch (vs_cluster.cu), against the oracle and the graph-replayed step kernels.

In the reference arithmetic its trace and fields must equal the FP32 oracle
(value equality, +0 == -0), like every step kernel; in the reciprocal form
(fast_math = 1) they must equal the strip kernels' (quad strips, two-step
strips) exactly.  Runs split over several calls continue the same state.
"""
import numpy as np
import pytest

import oracle as O
import vocalsim_b200 as V
from vocalsim_b200 import synthetic as S

pytestmark = pytest.mark.gpu

CLUSTER = len(V.tile_shapes()) - 1

CASES = {
    "uniform_gauss": (dict(mu3d=0.005, uniform_depth_m=0.02), S.uniform_tube()),
    "uniform_gauss_std_listener": (
        dict(mu3d=0.005, uniform_depth_m=0.02, source_type=3, gauss_peak_s=5e-4, gauss_width_s=1e-4,
             listener_mode=1, listener_x=244, listener_y=28), S.uniform_tube()),
    "vowel_ellipse_tmm": (dict(cross_sectional_shape=2, source_type=2, tmm_ps_pa=800.0), S.vowel_tube(3)),
    "vowel_ellipse_tmm_f64": (dict(cross_sectional_shape=2, source_type=2, tmm_ps_pa=800.0, tmm_f64=1),
                              S.vowel_tube(3)),
    "vowel_circle_dirichlet": (dict(mouth_radiation_cond=1), S.vowel_tube(5)),
    "vowel_eigen": (dict(cross_sectional_shape=2, engine=2), S.vowel_tube(7)),
    "vowel_2d_sine": (dict(fdtd_solver_type=0, source_type=0), S.vowel_tube(9)),
    "batch_tube_mul30": (dict(cross_sectional_shape=2, srate_mul=30), S.batch_tube(4)[:2]),
    "dirichlet_nopml_tmm": (dict(mouth_radiation_cond=1, pml_flag=0, source_type=2), S.vowel_tube(13)),
    "short_narrow_tmm": (dict(source_type=2, tmm_ps_pa=800.0), S.uniform_tube(2.0, 1.2)),
}


def cluster_batch(kw, geo):
    b = V.Batch([V.params(**kw)], [V.Geometry(*geo) if geo is not None else None])
    b.set_tile(CLUSTER)
    return b


@pytest.mark.parametrize("name", sorted(CASES))
def test_cluster_equals_fp32_oracle(name, cuda_ok):
    kw, geo = CASES[name]
    steps = 1500
    ref_tr, ref_f = O.run(O.params(**kw), O.Geometry(*geo), steps, "f32", fields=True)
    s = V.Solver(V.params(**kw), V.Geometry(*geo))      # a single tube defaults to the cluster shape
    tr = s.run(steps)
    P, Vx, Vy = s.fields()
    s.close()
    assert np.array_equal(tr, ref_tr), f"trace differs from step {int(np.argmax(tr != ref_tr))}"
    assert np.array_equal(P, ref_f[0]) and np.array_equal(Vx, ref_f[1]) and np.array_equal(Vy, ref_f[2])
    b = cluster_batch(kw, geo)
    assert np.array_equal(b.run(steps)[0], ref_tr)
    b.close()


def test_cluster_open_space(cuda_ok):
    kw = dict(simulation_type=0)
    ref = O.run(O.params(**kw), None, 600, "f32")
    b = cluster_batch(kw, None)
    assert np.array_equal(b.run(600)[0], ref)


@pytest.mark.parametrize("name", ["vowel_ellipse_tmm", "uniform_gauss"])
def test_cluster_split_runs_continue_the_state(name, cuda_ok):
    kw, geo = CASES[name]
    b = cluster_batch(kw, geo)
    whole = b.run(901)[0]
    b.reset()
    parts = np.concatenate([b.run(m)[0] for m in (1, 2, 128, 333, 437)])
    assert np.array_equal(whole, parts)


@pytest.mark.parametrize("name", ["uniform_gauss", "vowel_ellipse_tmm", "vowel_ellipse_tmm_f64",
                                  "vowel_circle_dirichlet", "vowel_2d_sine", "batch_tube_mul30",
                                  "dirichlet_nopml_tmm", "short_narrow_tmm"])
def test_cluster_fast_math_equals_the_strip_kernels(name, cuda_ok):
    kw, geo = CASES[name]
    kw = dict(kw, fast_math=1)
    segments = [3, 500, 128, 1]
    b = cluster_batch(kw, geo)
    got = np.concatenate([b.run(m)[0] for m in segments])
    P, _, _ = None, None, None
    b.close()
    ref = None
    for k in range(len(V.tile_shapes()) - 1):
        r = V.Batch([V.params(**kw)], [V.Geometry(*geo)])
        try:
            r.set_tile(k)
        except V.VsError:
            continue
        tr = np.concatenate([r.run(m)[0] for m in segments])
        r.close()
        if ref is None:
            ref = tr
        assert np.array_equal(tr, ref)
        if V.tile_shape_steps(k) == 2:
            break                        # one single-step and one two-step shape
    assert np.array_equal(got, ref), f"differs from step {int(np.argmax(got != ref))}"


def test_cluster_full_length_uniform_tube_equals_step_kernels(cuda_ok):
    """The uniform 17.5 x 3 cm tube over 33 075 steps: cluster == strip kernel, bit for bit."""
    kw, geo = CASES["uniform_gauss"]
    a = cluster_batch(kw, geo).run(33075)[0]
    r = V.Batch([V.params(**kw)], [V.Geometry(*geo)])
    r.set_tile(7)
    b = r.run(33075)[0]
    assert np.array_equal(a, b)
    assert np.all(np.isfinite(a)) and np.abs(a).max() > 0


BATCH_KWS = [dict(cross_sectional_shape=2),
             dict(cross_sectional_shape=2, source_type=2, tmm_ps_pa=800.0),
             dict(cross_sectional_shape=2, source_type=2, tmm_ps_pa=800.0, tmm_f64=1),
             dict(cross_sectional_shape=1, mouth_radiation_cond=1),
             dict(cross_sectional_shape=2, engine=2),
             dict(cross_sectional_shape=1, source_type=0)]


@pytest.mark.parametrize("fast", [0, 1])
def test_cluster_batch_equals_the_step_kernels(fast, cuda_ok):
    """A small batch on the cluster shape: every tube on its own thread-block
    cluster in one launch (the configuration sized for the largest frame),
    with table and two-mass sources (float and double model), a Dirichlet
    mouth and the Eigen denominator mixed.  Runs split over several calls of
    odd and even lengths give the step kernels' traces and final fields bit
    for bit (reference arithmetic and fast_math)."""
    tubes = [S.batch_tube(i)[:2] for i in range(len(BATCH_KWS))]
    ps = [V.params(fast_math=fast, **k) for k in BATCH_KWS]
    gs = [V.Geometry(L, A) for L, A in tubes]
    segments = [1, 300, 2, 129, 40]
    out = {}
    for shape in (CLUSTER, 0 if not fast else 17):
        b = V.Batch(ps, gs)
        b.set_tile(shape)
        tr = np.concatenate([b.run(m) for m in segments], axis=1)
        out[shape] = (tr, [b.fields(i) for i in range(len(ps))])
        b.close()
    (ca, fa), (sa, fb) = out.values()
    assert np.array_equal(ca, sa), f"tube {int(np.argmax(np.any(ca != sa, axis=1)))}"
    for x, y in zip(fa, fb):
        for a, c in zip(x, y):
            assert np.array_equal(a, c)
    assert np.all(np.abs(ca).max(axis=1) > 0)
    if not fast:
        for i in (0, 1, 2):
            o = O.run(O.params(**BATCH_KWS[i]), O.Geometry(*tubes[i]), sum(segments), "f32")
            assert np.array_equal(ca[i], o), f"tube {i} against the oracle"


def test_cluster_batch_more_tubes_than_resident_clusters(cuda_ok):
    """More tubes than clusters fit on the device at once: the clusters of
    later waves start from the same step (the step counter advances after the
    launch) and every tube's trace equals the step kernels'."""
    n = 40
    tubes = [S.batch_tube(i % 12)[:2] for i in range(n)]
    ps = [V.params(cross_sectional_shape=2, fast_math=1) for _ in range(n)]
    gs = [V.Geometry(L, A) for L, A in tubes]
    res = []
    for shape in (CLUSTER, 17):
        b = V.Batch(ps, gs)
        b.set_tile(shape)
        res.append(np.concatenate([b.run(257), b.run(64)], axis=1))
        b.close()
    assert np.array_equal(res[0], res[1])
    assert np.all(np.abs(res[0]).max(axis=1) > 0)

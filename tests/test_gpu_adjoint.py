"""Adjoint gradients (vs_batch_forward_ckpt + vs_batch_adjoint) against
central finite differences of the double-precision oracle.

Loss: L = 1/2 sum_n w_n y_n^2 over the listener trace y.  The adjoint gives
per-cell dL/d(depth_p, depth_x, depth_y) and dL/d z_inv; their directional
derivative along a random relative perturbation of the maps must match the
central difference [L(+h) - L(-h)] / 2h of the FP64 restatement with h = 1e-4
(relative), within 1e-3 relative error.
"""
import numpy as np
import pytest

import oracle as O
import vocalsim_b200 as V
from vocalsim_b200 import synthetic as S

pytestmark = pytest.mark.gpu

H_REL = 1e-4
TOL = 1e-3


def _loss(trace, w):
    t = np.asarray(trace, np.float64)
    return 0.5 * float(np.sum(w * t * t))


def _check(kw, L, A, steps, every, parts, seed=0):
    pv, gv = V.params(**kw), V.Geometry(L, A)
    po, go = O.params(**kw), O.Geometry(L, A)
    m = V.build_maps(pv, gv)
    b = V.Batch([pv], [gv])
    tr = b.forward_ckpt(steps, every)[0]
    rng = np.random.default_rng(seed)
    w = rng.uniform(0.5, 1.5, steps)
    grads, gz = b.adjoint((w * tr.astype(np.float64)).astype(np.float32)[None])
    gP, gX, gY = grads[0]
    shape = m["depth_p"].shape
    interior = np.zeros(shape, bool)
    interior[1:-1, 1:-1] = True
    d = {k: (rng.uniform(-1, 1, shape) * interior if k in parts else np.zeros(shape)) for k in ("P", "X", "Y")}
    dz = rng.uniform(-1, 1) if "Z" in parts else 0.0
    base = {k: m[f"depth_{k.lower()}"].astype(np.float64) for k in ("P", "X", "Y")}
    z0 = float(m["dims"]["z_inv_val"])
    adj = (np.sum(gP * base["P"] * d["P"]) + np.sum(gX * base["X"] * d["X"]) + np.sum(gY * base["Y"] * d["Y"])
           + float(gz[0]) * z0 * dz)

    def loss_at(h):
        mp = {k: base[k] * (1 + h * d[k]) for k in base}
        t = O.run_maps_f64(po, go, steps, mp["P"], mp["X"], mp["Y"], z0 * (1 + h * dz))
        return _loss(t, w)

    fd = (loss_at(H_REL) - loss_at(-H_REL)) / (2 * H_REL)
    assert abs(fd) > 0
    assert abs(adj - fd) <= TOL * abs(fd), f"adjoint {adj:.9e} vs finite difference {fd:.9e}"
    return adj, fd


@pytest.mark.parametrize("parts", ["P", "X", "Y", "Z", "PXYZ"])
def test_vowel_tube_map_gradients(parts, cuda_ok):
    L, A = S.vowel_tube(3)
    _check(dict(cross_sectional_shape=2, mu3d=0.025), L, A, steps=700, every=128, parts=parts)


def test_dirichlet_eigen_gradients(cuda_ok):
    L, A = S.vowel_tube(6)
    _check(dict(cross_sectional_shape=2, mouth_radiation_cond=1, engine=V.ENGINE_EIGEN, mu3d=0.025), L, A,
           steps=600, every=100, parts="PXYZ", seed=1)


def test_checkpoint_interval_does_not_change_gradients(cuda_ok):
    L, A = S.vowel_tube(4)
    pv, gv = V.params(cross_sectional_shape=2), V.Geometry(L, A)
    outs = []
    for every in (600, 97, 1):
        b = V.Batch([pv], [gv])
        tr = b.forward_ckpt(600, every)[0]
        grads, gz = b.adjoint(tr[None])
        gP, gX, gY = grads[0]
        outs.append((gP, gX, gY, gz))
    for o in outs[1:]:
        for a, ref in zip(o, outs[0]):
            assert np.array_equal(a, ref)


@pytest.mark.parametrize("parts,tmm_f64", [("P", 0), ("PXYZ", 0), ("PXYZ", 1)])
def test_two_mass_source_gradients(parts, tmm_f64, cuda_ok):
    # the glottal flow depends on the pressure at the excitation point, so the
    # reverse step runs the two-mass model's Jacobian transpose each step
    L, A = S.vowel_tube(1)
    _check(dict(cross_sectional_shape=2, source_type=V.SRC_TMM, tmm_ps_pa=800.0, mu3d=0.025, tmm_f64=tmm_f64),
           L, A, steps=1500, every=256, parts=parts, seed=2)


@pytest.mark.parametrize("tmm_f64", [0, 1])
def test_two_mass_checkpoint_interval_does_not_change_gradients(tmm_f64, cuda_ok):
    L, A = S.vowel_tube(2)
    pv, gv = V.params(cross_sectional_shape=2, source_type=V.SRC_TMM, tmm_f64=tmm_f64), V.Geometry(L, A)
    outs = []
    for every in (500, 33):
        b = V.Batch([pv], [gv])
        tr = b.forward_ckpt(500, every)[0]
        grads, gz = b.adjoint(tr[None])
        outs.append((*grads[0], gz))
    for a, ref in zip(outs[1], outs[0]):
        assert np.array_equal(a, ref)


def test_coupled_wall_adjoint_unsupported(cuda_ok):
    L, A = S.vowel_tube(1)
    b = V.Batch([V.params(cross_sectional_shape=2, wall_coupling=0.5)], [V.Geometry(L, A)])
    with pytest.raises(V.VsError) as e:
        b.forward_ckpt(50, 10)
    assert e.value.status == 7


@pytest.mark.parametrize("kw", [dict(cross_sectional_shape=2, mu3d=0.025),
                                dict(cross_sectional_shape=2, mu3d=0.025, source_type=V.SRC_TMM, tmm_ps_pa=800.0,
                                     tmm_f64=1)])
def test_fast_math_gradients(kw, cuda_ok):
    # reciprocal-form forward and recomputation (quad strips); the finite
    # differences are of the FP64 oracle as before
    L, A = S.vowel_tube(3)
    _check(dict(fast_math=1, **kw), L, A, steps=1200, every=256, parts="PXYZ", seed=4)


@pytest.mark.parametrize("kw", [dict(cross_sectional_shape=2, mu3d=0.025),
                                dict(cross_sectional_shape=2, source_type=2, tmm_ps_pa=800.0, tmm_f64=1),
                                dict(cross_sectional_shape=1, mouth_radiation_cond=1, engine=2),
                                dict(cross_sectional_shape=2, fast_math=1)],
                         ids=["gauss", "two_mass", "dirichlet_eigen", "fast_math"])
def test_strip_and_tile_reverse_steps_agree(kw, cuda_ok):
    """The kernel forms of the reverse step (32 x 8 tiles; two-step strips;
    one-step strips) transpose the same forward step; on a 3-tube batch their
    per-cell map gradients and z_inv gradients agree with the tiles' to float
    rounding (relative 1e-5 of each map's norm)."""
    tubes = [S.batch_tube(i)[:2] for i in (1, 2, 3)]
    steps, every = 1500, 512
    rng = np.random.default_rng(4)
    out = {}
    g = None
    for form in (1, 3, 2):
        b = V.Batch([V.params(**kw) for _ in tubes], [V.Geometry(*t) for t in tubes])
        b.set_adjoint_form(form)
        tr = b.forward_ckpt(steps, every)
        if g is None:
            g = (rng.uniform(0.5, 1.5, tr.shape) * tr).astype(np.float32)
        out[form] = b.adjoint(g)
        b.close()
    gb, zb = out[1]
    for form in (3, 2):
        ga, za = out[form]
        for ta, tb in zip(ga, gb):
            for a, c in zip(ta, tb):
                assert np.linalg.norm(a - c) <= 1e-5 * np.linalg.norm(c) + 1e-30, f"form {form}"
        assert np.allclose(za, zb, rtol=1e-5, atol=0), f"form {form}"


@pytest.mark.parametrize("rows", [4, 8, 16])
@pytest.mark.parametrize("every", [97, 512])
def test_two_step_reverse_equals_one_step(rows, every, cuda_ok):
    """The two-step strip kernel runs the one-step strip kernel's float
    operations cell by cell, so lambda is the same; only the order of the
    double additions into the gradient accumulators differs (both steps' terms
    are added together).  Odd segment lengths end with a single step; strips
    of 4, 8 and 16 rows put strip boundaries at different rows.  On a 3-tube
    batch (Gaussian source, z_inv walls) the gradients agree to a few float
    ulps."""
    tubes = [S.batch_tube(i)[:2] for i in (1, 2, 3)]
    steps = 1200
    out = {}
    g = None
    rng = np.random.default_rng(7)
    for form in (3, 2):
        b = V.Batch([V.params(cross_sectional_shape=2, mu3d=0.025) for _ in tubes], [V.Geometry(*t) for t in tubes])
        b.set_adjoint_form(form)
        b.set_adjoint_rows(rows)
        tr = b.forward_ckpt(steps, every)
        if g is None:
            g = (rng.uniform(0.5, 1.5, tr.shape) * tr).astype(np.float32)
        out[form] = b.adjoint(g)
        b.close()
    (ga, za), (gb, zb) = out[2], out[3]
    for ta, tb in zip(ga, gb):
        for a, c in zip(ta, tb):
            # a few float ulps, or 1e-9 of the map's largest term where sums cancel
            bound = 4 * np.spacing(np.abs(c).astype(np.float32)) + 1e-9 * np.abs(c).max()
            assert np.all(np.abs(a - c) <= bound)
    assert np.allclose(za, zb, rtol=1e-6, atol=0)


@pytest.mark.parametrize("kw", [dict(cross_sectional_shape=2, mu3d=0.025, fast_math=1),
                                dict(cross_sectional_shape=2, source_type=2, tmm_ps_pa=800.0, tmm_f64=1,
                                     fast_math=1)],
                         ids=["gauss", "two_mass"])
def test_two_step_recomputation_equals_one_step(kw, cuda_ok):
    """With fast_math a segment of even length is recomputed by the two-step
    kernel (both steps' states stored), an odd one step by step; the two
    give the same history bit for bit, so with one-step reverse strips (form
    3, each step's terms added on their own) the gradients of checkpoint
    intervals 256 and 255 are identical."""
    tubes = [S.batch_tube(i)[:2] for i in (1, 2, 3)]
    steps = 1100
    out = []
    g = None
    rng = np.random.default_rng(9)
    for every in (256, 255):
        b = V.Batch([V.params(**kw) for _ in tubes], [V.Geometry(*t) for t in tubes])
        b.set_adjoint_form(3)
        tr = b.forward_ckpt(steps, every)
        if g is None:
            g = (rng.uniform(0.5, 1.5, tr.shape) * tr).astype(np.float32)
        out.append(b.adjoint(g))
        b.close()
    (ga, za), (gb, zb) = out
    for ta, tb in zip(ga, gb):
        for a, c in zip(ta, tb):
            assert np.array_equal(a, c)
    assert np.array_equal(za, zb)

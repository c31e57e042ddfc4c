"""The device section model (vs_batch_set_sections / vs_batch_section_gradients)
against the torch SectionDepthModel: the same depth maps (the traces of a
forward on them are identical) and the same section gradients through the
adjoint."""
import numpy as np
import pytest
import torch

import vocalsim_b200 as V
from vocalsim_b200 import synthetic as S
from vocalsim_b200.autograd import SectionDepthModel, SectionTrace, TubeTrace, spectral_loss

pytestmark = pytest.mark.gpu

FS = 44100.0 * 15


def _tubes():
    return [S.vowel_tube(5), S.batch_tube(3)[:2]]


def _setup(steps):
    kw = dict(cross_sectional_shape=2, mu3d=0.025, num_steps=steps)
    ps = [V.params(**kw) for _ in range(2)]
    gs = [V.Geometry(L, A) for L, A in _tubes()]
    models = [SectionDepthModel(p, g) for p, g in zip(ps, gs)]
    return ps, gs, models


def _perturbed(models, seed):
    rng = np.random.default_rng(seed)
    ws = [m.width0 * torch.from_numpy(rng.uniform(1.0, 1.2, len(m.width0))) for m in models]
    ds = [m.depth0 * torch.from_numpy(rng.uniform(0.9, 1.2, len(m.depth0))) for m in models]
    zs = torch.tensor([float(m.nominal["dims"]["z_inv_val"]) * 1.3 for m in models], dtype=torch.float64)
    return ws, ds, zs


def test_device_maps_equal_the_torch_model(cuda_ok):
    steps = 600
    ps, gs, models = _setup(steps)
    ws, ds, zs = _perturbed(models, 0)
    a = V.Batch(ps, gs)
    a.set_sections([w.numpy() for w in ws], [d.numpy() for d in ds], zs.numpy())
    tra = a.forward_ckpt(steps, 128)
    b = V.Batch(ps, gs)
    for i, m in enumerate(models):
        with torch.no_grad():
            mp, mx, my = m.maps(ws[i], ds[i])
        b.set_maps(i, mp.numpy().astype(np.float32), mx.numpy().astype(np.float32), my.numpy().astype(np.float32),
                   float(zs[i]))
    trb = b.forward_ckpt(steps, 128)
    assert np.array_equal(tra, trb)


def test_device_section_gradients_equal_the_torch_model(cuda_ok):
    steps = 1500
    ps, gs, models = _setup(steps)
    ws, ds, zs = _perturbed(models, 1)
    target = torch.from_numpy(V.Batch([V.params(cross_sectional_shape=2, mu3d=0.025, num_steps=steps)] * 2,
                                      [V.Geometry(*S.vowel_tube(6))] * 2).run(steps)).double()
    # device path
    wl = [w.clone().requires_grad_(True) for w in ws]
    dl = [d.clone().requires_grad_(True) for d in ds]
    z1 = zs.clone().requires_grad_(True)
    tr = SectionTrace.apply(V.Batch(ps, gs), steps, 256, z1, *wl, *dl)
    spectral_loss(tr, target, FS).backward()
    # torch model + per-cell map gradients
    wt = [w.clone().requires_grad_(True) for w in ws]
    dt = [d.clone().requires_grad_(True) for d in ds]
    z2 = zs.clone().requires_grad_(True)
    maps = []
    for i, m in enumerate(models):
        maps += list(m.maps(wt[i], dt[i]))
    tr2 = TubeTrace.apply(V.Batch(ps, gs), steps, 256, z2, *maps)
    assert torch.equal(tr, tr2)
    spectral_loss(tr2, target, FS).backward()
    for a, b in zip(wl + dl, wt + dt):
        assert torch.count_nonzero(b.grad) > 0
        np.testing.assert_allclose(a.grad.numpy(), b.grad.numpy(), rtol=1e-6, atol=1e-6 * float(b.grad.abs().max()))
    np.testing.assert_allclose(z1.grad.numpy(), z2.grad.numpy(), rtol=1e-6)


def test_device_resident_traces_give_the_same_gradients(cuda_ok):
    """SectionTrace with the traces kept on the GPU (vs_batch_forward_ckpt_device /
    vs_batch_adjoint_device, the spectral loss on the GPU) gives the traces and
    section gradients of the host-trace path."""
    steps = 1500
    ps, gs, models = _setup(steps)
    ws, ds, zs = _perturbed(models, 2)
    dev = torch.device("cuda", torch.cuda.current_device())
    target = torch.from_numpy(V.Batch([V.params(cross_sectional_shape=2, mu3d=0.025, num_steps=steps)] * 2,
                                      [V.Geometry(*S.vowel_tube(6))] * 2).run(steps)).double()
    out = []
    for device in (None, dev):
        b = V.Batch(ps, gs)
        if device is not None:
            b.set_stream(torch.cuda.current_stream(device).cuda_stream)
            b.trace_device = device
        wl = [w.clone().requires_grad_(True) for w in ws]
        dl = [d.clone().requires_grad_(True) for d in ds]
        z = zs.clone().requires_grad_(True)
        tr = SectionTrace.apply(b, steps, 256, z, *wl, *dl)
        spectral_loss(tr, target.to(tr.device), FS).backward()
        out.append((tr.detach().cpu(), [t.grad.clone() for t in wl + dl], z.grad.clone()))
        b.close()
    (ta, ga, za), (tb, gb, zb) = out
    assert torch.equal(ta, tb)
    for a, c in zip(ga, gb):
        np.testing.assert_allclose(a.numpy(), c.numpy(), rtol=1e-9, atol=1e-9 * float(c.abs().max()))
    np.testing.assert_allclose(za.numpy(), zb.numpy(), rtol=1e-9)

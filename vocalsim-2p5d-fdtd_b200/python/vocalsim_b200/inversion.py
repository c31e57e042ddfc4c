"""Batched inversion: fit each tube's section widths, section depths and wall
admittance to a target transfer function.

Every Adam iteration builds the depth maps from the section parameters on the
device (vs_batch_set_sections), runs one batched checkpointed forward
(vs_batch_forward_ckpt) and one batched reverse-time adjoint
(vs_batch_adjoint) for all tubes together, and reduces the map gradients to
section gradients on the device (vs_batch_section_gradients), through the
autograd.Function SectionTrace.  The loss of a tube is the mean squared
difference of log power spectra over 0..5 kHz (the transfer function the
reference plots, results/plt_transfer_function.py:20-24); the optimiser
works on log-multipliers of the nominal parameters, so widths, depths and
z_inv stay positive.

Bounds.  The depth model keeps the wall rows of the nominal rasterisation
(vs_batch_set_sections, autograd.SectionDepthModel).  A section narrower than its rasterised air
band would put the cells next to its walls outside the ellipse, at the 1 mm
depth floor beside deeper faces, where the reference's 2.5D update is
unstable (the FP32 oracle diverges within a few hundred steps for a 5 %
narrowing); so after every Adam step the multipliers are projected onto
width in [1, 1.5], depth in [0.8, 1.5] and z_inv in [0.25, 4] times nominal
-- narrowing is carried by the depth -- a box on which seeded random
multipliers stay stable.  Tubes near the stability limit can still diverge
inside it (a trace that is not finite or exceeds 100 times its target's
amplitude); such a tube is stepped back halfway towards its last parameters
with a good trace, and its later steps are halved (backtracking), while the
other tubes continue.  Each tube's result is the best loss it reached.

    python -m vocalsim_b200.inversion --tubes 64 --srate-mul 30 --ms 20 --iters 100
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from .autograd import SectionTrace, log_power_spectrum, tube_layout
from .abi import VS_ERR_NONFINITE, VsError
from .solver import Batch, Geometry, params


# projection box of the log-multipliers (see the module docstring)
LOG_W_BOUNDS = (0.0, float(np.log(1.5)))
LOG_D_BOUNDS = (float(np.log(0.8)), float(np.log(1.5)))
LOG_Z_BOUNDS = (float(np.log(0.25)), float(np.log(4.0)))


class BatchInversion:
    """Adam over per-tube log-multipliers of (44 widths, 44 depths, z_inv)."""

    def __init__(self, ps, gs, targets, steps: int, ckpt_every: int = 512, lr: float = 0.02,
                 fmax: float = 5000.0):
        if len({int(p.fast_math) for p in ps}) != 1:
            raise ValueError("every tube of a batch needs the same fast_math")
        lays = [tube_layout(p, g) for p, g in zip(ps, gs)]
        self.width0 = [torch.tensor(lay["major"], dtype=torch.float64) for lay in lays]
        self.depth0 = [torch.tensor(lay["minor"], dtype=torch.float64) for lay in lays]
        self.batch = Batch(ps, gs)
        # traces, spectra and the loss live on the GPU, on torch's current
        # stream, which the batch also uses (no host round trip of traces)
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.batch.set_stream(torch.cuda.current_stream(self.device).cuda_stream)
        self.batch.trace_device = self.device
        self.n = len(ps)
        self.steps = steps
        self.ckpt_every = ckpt_every
        self.fs = 44100.0 * ps[0].srate_mul
        self.fmax = fmax
        targets = torch.as_tensor(np.asarray(targets), dtype=torch.float64).reshape(self.n, steps).to(self.device)
        self.target_spec = log_power_spectrum(targets, self.fs, fmax)
        self.amp_limit = 100.0 * targets.abs().amax(dim=1)
        self.best = torch.full((self.n,), float("inf"), dtype=torch.float64)
        ns = [len(w) for w in self.width0]
        self.log_w = torch.zeros(self.n, max(ns), dtype=torch.float64, requires_grad=True)
        self.log_d = torch.zeros(self.n, max(ns), dtype=torch.float64, requires_grad=True)
        self.log_z = torch.zeros(self.n, dtype=torch.float64, requires_grad=True)
        self.z0 = torch.tensor([float(lay["dims"]["z_inv_val"]) for lay in lays], dtype=torch.float64)
        self.opt = torch.optim.Adam([self.log_w, self.log_d, self.log_z], lr=lr)
        self.good = [t.detach().clone() for t in (self.log_w, self.log_d, self.log_z)]
        self.scale = torch.ones(self.n, dtype=torch.float64)

    def loss(self) -> torch.Tensor:
        """Per-tube spectral loss of the current parameters (differentiable); the
        depth maps are built and differentiated on the device (SectionTrace)."""
        ws, ds = [], []
        for i, (w0, d0) in enumerate(zip(self.width0, self.depth0)):
            k = len(w0)
            ws.append(w0 * torch.exp(self.log_w[i, :k]))
            ds.append(d0 * torch.exp(self.log_d[i, :k]))
        z = self.z0 * torch.exp(self.log_z)
        tr = SectionTrace.apply(self.batch, self.steps, self.ckpt_every, z, *ws, *ds)
        d = log_power_spectrum(tr, self.fs, self.fmax) - self.target_spec
        per_tube = (d * d).mean(dim=-1)
        # a diverging trace counts as not finite
        grown = tr.detach().abs().amax(dim=1) > self.amp_limit
        return torch.where(grown, torch.full_like(per_tube, float("nan")), per_tube).cpu()

    def step(self) -> np.ndarray:
        """One Adam iteration; returns each tube's loss before the update (NaN
        for a tube whose forward diverged; it backtracks instead)."""
        params = (self.log_w, self.log_d, self.log_z)
        self.opt.zero_grad()
        t0 = time.perf_counter()
        per_tube = self.loss()
        t1 = time.perf_counter()
        ok = torch.isfinite(per_tube).detach()
        if not ok.any():
            raise RuntimeError("the forward diverged for every tube")
        self.best = torch.where(ok, torch.minimum(self.best, per_tube.detach()), self.best)
        torch.where(ok, per_tube, torch.zeros_like(per_tube)).sum().backward()
        t2 = time.perf_counter()
        rec, rev = self.batch.adjoint_times()
        # wall time of this iteration's parts (s): the forward (depth maps on
        # the device, checkpointed forward, spectral loss), the backward (loss
        # gradient, adjoint, section reverse pass) and, inside the adjoint, the
        # device time of the segment recomputation and of the reverse steps
        self.timings = {"forward_s": t1 - t0, "backward_s": t2 - t1, "recompute_s": rec / 1e3,
                        "reverse_s": rev / 1e3}
        before = [t.detach().clone() for t in params]
        for t in params:
            t.grad.nan_to_num_(0.0)
            t.grad[~ok] = 0.0
        self.opt.step()
        with torch.no_grad():
            self.scale[~ok] *= 0.5
            for t, b, g in zip(params, before, self.good):
                s = self.scale.reshape(-1, *([1] * (t.dim() - 1)))
                stepped = b + s * (t - b)
                back = g + 0.5 * (b - g)
                okr = ok.reshape(-1, *([1] * (t.dim() - 1)))
                t.copy_(torch.where(okr, stepped, back))
                g.copy_(torch.where(okr, b, g))
            self.log_w.clamp_(*LOG_W_BOUNDS)
            self.log_d.clamp_(*LOG_D_BOUNDS)
            self.log_z.clamp_(*LOG_Z_BOUNDS)
        return per_tube.detach().numpy()

    def close(self) -> None:
        self.batch.close()


def synthetic_problem(n_tubes: int, srate_mul: int, steps: int, seed0: int = 0, fast_math: int = 0):
    """n batch tubes (3:1 elliptical sections, Gaussian source) and the traces
    of their targets (synthetic.batch_target_tube), run on the GPU.

    The reference's 2.5D update is not stable for every tube: where a wall
    row's face depth is several times the depth of the air cell beside it
    (depths near the 1 mm floor at fs = 44100 x 30), the effective Courant
    number of that cell exceeds 1 and the field grows without bound -- the
    FP32 oracle (the reference's equations) diverges there too.  Seeds whose
    tube or target trace is not finite over `steps` are skipped; the first
    n_tubes seeds from seed0 on that are stable for both are used.
    Returns (params, geometries, targets, seeds)."""
    from . import synthetic as S
    kw = dict(cross_sectional_shape=2, srate_mul=srate_mul, num_steps=steps, fast_math=fast_math)
    chosen, targets = [], []
    start = seed0
    while len(chosen) < n_tubes:
        cand = list(range(start, start + 2 * (n_tubes - len(chosen)) + 2))
        start = cand[-1] + 1
        ps = [params(**kw) for _ in range(2 * len(cand))]
        gs = [Geometry(*S.batch_tube(s)[:2]) for s in cand] + [Geometry(*S.batch_target_tube(s)[:2]) for s in cand]
        b = Batch(ps, gs)
        tr = torch.zeros((2 * len(cand), steps), dtype=torch.float32, device="cuda")
        try:
            b.run_device(steps, tr.data_ptr())
        except VsError as e:
            # unstable candidates are expected here; their traces are screened below
            if e.status != VS_ERR_NONFINITE:
                raise
        torch.cuda.synchronize()
        b.close()
        ok = torch.isfinite(tr).all(dim=1).cpu().numpy()
        host = tr.cpu().numpy()
        for k, s in enumerate(cand):
            if ok[k] and ok[len(cand) + k] and len(chosen) < n_tubes:
                chosen.append(s)
                targets.append(host[len(cand) + k])
    ps = [params(**kw) for _ in chosen]
    gs = [Geometry(*S.batch_tube(s)[:2]) for s in chosen]
    return ps, gs, np.stack(targets), chosen


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--tubes", type=int, default=64)
    ap.add_argument("--srate-mul", type=int, default=30)
    ap.add_argument("--ms", type=float, default=20.0, help="simulated time per forward")
    ap.add_argument("--iters", type=int, default=100)
    ap.add_argument("--lr", type=float, default=0.02)
    ap.add_argument("--ckpt-every", type=int, default=512)
    ap.add_argument("--fast-math", type=int, default=1, help="1: reciprocal-form arithmetic (quad strips)")
    a = ap.parse_args(argv)
    steps = int(round(a.ms * 1e-3 * 44100 * a.srate_mul))
    ps, gs, targets, seeds = synthetic_problem(a.tubes, a.srate_mul, steps, fast_math=a.fast_math)
    inv = BatchInversion(ps, gs, targets, steps, a.ckpt_every, a.lr)
    print(json.dumps({"tubes": a.tubes, "srate_mul": a.srate_mul, "steps": steps, "seeds": seeds,
                      "interior_cells": inv.batch.interior_cells}), flush=True)
    first = None
    for it in range(a.iters):
        t0 = time.perf_counter()
        loss = inv.step()
        first = loss if first is None else first
        dt = time.perf_counter() - t0
        print(json.dumps({"iter": it, "mean_spectral_error": float(np.nanmean(loss)),
                          "diverged": int(np.isnan(loss).sum()), "s": round(dt, 3)}), flush=True)
    print(json.dumps({"initial_mean_spectral_error": float(first.mean()),
                      "best_mean_spectral_error": float(inv.best.mean())}), flush=True)
    inv.close()


if __name__ == "__main__":
    main()

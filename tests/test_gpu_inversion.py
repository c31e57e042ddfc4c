"""Batched inversion (vocalsim_b200.inversion): Adam over the section widths,
section depths and z_inv of two tubes at once, driven by the batched
checkpointed forward and adjoint, lowers the spectral error to targets from
other seeded tubes."""
import numpy as np
import pytest

from vocalsim_b200.inversion import BatchInversion, synthetic_problem

pytestmark = pytest.mark.gpu


def test_batched_inversion_reduces_spectral_error(cuda_ok):
    steps = 2000
    ps, gs, targets, _ = synthetic_problem(2, 15, steps)
    inv = BatchInversion(ps, gs, targets, steps, ckpt_every=256, lr=0.05)
    losses = [inv.step() for _ in range(6)]
    inv.close()
    first, last = losses[0], losses[-1]
    assert np.all(np.isfinite(losses))   # no tube diverged on this small case
    assert np.all(last < first), (first, last)


def test_inversion_with_fast_math(cuda_ok):
    """The reciprocal-form forward and recomputation (quad strips) drive the
    same inversion."""
    steps = 1500
    ps, gs, targets, _ = synthetic_problem(2, 15, steps, fast_math=1)
    inv = BatchInversion(ps, gs, targets, steps, ckpt_every=256, lr=0.05)
    losses = [inv.step() for _ in range(4)]
    inv.close()
    assert np.all(np.isfinite(losses)) and np.all(losses[-1] < losses[0])

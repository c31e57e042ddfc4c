"""Failure paths, driven without a GPU fault.

* Timeout: a lowered poll limit (vs_batch_set_wait_limit) makes the bounded
  wait for a launch's bulk row copies give up at once; the launch flags
  VS_ERR_TIMEOUT, still waits (with the default limit) for its own copies,
  and exits.  The run reports VS_ERR_TIMEOUT and the next run with the
  default limit is correct again.
* Non-finite: a tube the reference scheme itself makes unstable (batch tube
  4 at fs = 44100 x 30; the FP32 oracle's trace overflows at step 4509) ends
  with VS_ERR_NONFINITE, whether its trace goes to host memory (scanned) or
  stays on the device (the step kernels' watchdog on the listener sample),
  on the graph-replayed strips and on the cluster kernel.
"""
import numpy as np
import pytest

import oracle as O
import vocalsim_b200 as V
from vocalsim_b200 import abi
from vocalsim_b200 import synthetic as S

pytestmark = pytest.mark.gpu

BAND_SHAPE = 12            # band_kernel<4>: one cp.async.bulk per plane per band
CLUSTER = len(V.tile_shapes()) - 1


def _tubes():
    tubes = [S.batch_tube(i)[:2] for i in range(2)]
    return [V.params(cross_sectional_shape=2, source_type=2 if i else 1) for i in range(2)], \
        [V.Geometry(*t) for t in tubes], tubes


# The band kernel waits right after issuing its copies, so one poll cannot see
# them land; the staged quad strips issue several rows ahead before their
# first wait, so a one-poll limit does not reliably run out there.
@pytest.mark.parametrize("shape", [BAND_SHAPE])
def test_wait_that_runs_out_returns_timeout_and_the_next_run_is_clean(cuda_ok, shape):
    ps, gs, tubes = _tubes()
    b = V.Batch(ps, gs)
    b.set_tile(shape)
    b.set_wait_limit(1)
    with pytest.raises(V.VsError) as e:
        b.run(8)
    assert e.value.status == abi.VS_ERR_TIMEOUT
    b.set_wait_limit(0)
    b.reset()
    tr = b.run(300)
    ref = O.run(O.params(cross_sectional_shape=2, source_type=2), O.Geometry(*tubes[1]), 300, "f32")
    assert np.array_equal(tr[1], ref)


UNSTABLE = dict(cross_sectional_shape=2, srate_mul=30)


@pytest.mark.parametrize("on_device", [False, True])
@pytest.mark.parametrize("shape", [7, CLUSTER])
def test_unstable_tube_reports_nonfinite(cuda_ok, on_device, shape):
    import torch
    L, A = S.batch_tube(4)[:2]
    b = V.Batch([V.params(**UNSTABLE)], [V.Geometry(L, A)])
    b.set_tile(shape)
    steps = 5000
    with pytest.raises(V.VsError) as e:
        if on_device:
            buf = torch.empty(steps, dtype=torch.float32, device="cuda")
            b.run_device(steps, buf.data_ptr())
        else:
            b.run(steps)
    assert e.value.status == abi.VS_ERR_NONFINITE
    # a stable run on the same batch afterwards is unaffected
    b.reset()
    tr = b.run(1000)
    assert np.array_equal(tr[0], O.run(O.params(**UNSTABLE), O.Geometry(L, A), 1000, "f32"))

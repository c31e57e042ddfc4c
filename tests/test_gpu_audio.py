"""vs_audio (WAV samples on the device) against the oracle's restatement of
results/generate_audio.py:14-42 on the same traces.  The recursion is the
same double-precision direct form II transposed evaluation; the filter
coefficients may differ from the oracle's in the last bit, so the float32
samples are compared to 2e-7 absolute (they lie in [-1, 1])."""
import numpy as np
import pytest

import audio_oracle as OA
import vocalsim_b200 as V
import vocalsim_b200.audio as VA
from vocalsim_b200 import synthetic as S

pytestmark = pytest.mark.gpu

TOL = 2e-7


@pytest.mark.parametrize("mul", [1, 2, 15, 30])
def test_random_traces_match_oracle(mul, cuda_ok):
    rng = np.random.default_rng(10 + mul)
    x = (rng.standard_normal((3, 5000)) * np.array([[1.0], [30.0], [1e-3]])).astype(np.float32)
    got = VA.audio(x, mul).cpu().numpy()
    assert got.shape == (3, (5000 + mul - 1) // mul)
    for i in range(3):
        assert np.max(np.abs(got[i] - OA.audio(x[i], mul))) <= TOL


def test_simulated_trace_matches_oracle(cuda_ok):
    """A 20 ms config-1 trace (fs = 44100 x 15) through the device audio path."""
    L, A = S.uniform_tube()
    tr = V.Solver(V.params(mu3d=0.005, uniform_depth_m=0.02), V.Geometry(L, A)).run(13230)
    got = VA.audio(tr, 15).cpu().numpy()
    want = OA.audio(tr, 15)
    assert got.shape == want.shape == (882,)
    assert np.max(np.abs(got - want)) <= TOL
    assert np.max(np.abs(got)) > 0.01


def test_zero_trace_gives_nan_like_the_reference(cuda_ok):
    got = VA.audio(np.zeros(100, np.float32), 2).cpu().numpy()
    assert np.all(np.isnan(got))


def test_invalid_arguments(cuda_ok):
    with pytest.raises(V.VsError):
        VA.audio(np.ones(10, np.float32), 0)

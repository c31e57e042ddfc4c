"""vs_formants (cuFFT + scan kernel) against the reference's get_formants_bw:
its golden outputs on seeded signals, and oracle/formants.py on GPU traces."""
from pathlib import Path

import numpy as np
import pytest

import vocalsim_b200 as V
from formants import formants_bw
from vocalsim_b200 import synthetic as S
from vocalsim_b200.spectrum import formants

pytestmark = pytest.mark.gpu

G = np.load(Path(__file__).parent / "golden" / "formants_golden.npz")
FS = 44100.0 * 15


def _close(got, ref):
    # Centre frequencies are bin frequencies: equal.  numpy >= 2 takes the FFT
    # of a float32 signal in single precision (the golden outputs were made
    # so), the device in double: bandwidths agree to 1e-3 Hz, levels to 1e-4 dB.
    assert np.array_equal(got[1], ref[1]), (got[1], ref[1])
    np.testing.assert_allclose(got[0], ref[0], rtol=0, atol=1e-3)
    np.testing.assert_allclose(got[2], ref[2], rtol=0, atol=1e-4)


def test_golden_signals_one_by_one_and_batched(cuda_ok):
    sigs = [G[f"signal_{k}"] for k in range(4)]
    for k, s in enumerate(sigs):
        _close(formants(s, FS, 6), G[f"bw_{k}"])
    same = np.stack([sigs[1], sigs[1] * 0.5])
    res = formants(same, FS, 6)
    _close(res[0], G["bw_1"])


def test_solver_traces_match_the_restatement(cuda_ok):
    b = V.Batch([V.params(cross_sectional_shape=2, num_steps=33075) for _ in range(3)],
                [V.Geometry(*S.batch_tube(i)[:2]) for i in range(3)])
    tr = b.run(33075)
    got = formants(tr, FS, 4)
    for i in range(3):
        _close(got[i], formants_bw(tr[i], FS, 4))

"""Audio output of a listener trace, restating results/generate_audio.py:14-42
of the reference (normalise, clip, Butterworth low-pass, decimate).

TEST INFRASTRUCTURE ONLY (audio parity checks).  The reference script calls
scipy.signal.butter and scipy.signal.lfilter (SciPy, the version installed
with it; 1.18.1 here).  Their published algorithms are restated below and
pinned against SciPy itself by the audio tests:

* butter(2, Wn, 'low'): analog Butterworth prototype poles
  -exp(i pi m / 4), m = -1, 1 (gain 1); pre-warp with fs = 2,
  w = 2 fs tan(pi Wn / fs); scale the poles by w and the gain by w^2;
  bilinear transform with fs2 = 2 fs: poles (fs2 + p) / (fs2 - p), two zeros
  at -1, gain k / prod(fs2 - p) (real part); b = k [1, 2, 1],
  a = real(poly(poles)).
* lfilter(b, a, x): the direct form II transposed recursion
  y[n] = b0 x[n] + z0;  z0 = z1 + b1 x[n] - a1 y[n];  z1 = b2 x[n] - a2 y[n]
  (a normalised so that a0 = 1; zero initial state).

Pipeline (generate_audio.py:14-42): audio = P / max|P|, clipped to [-1, 1];
when srate_mul > 1: fc = 5050 Hz, Wn = fc / (44100 srate_mul / 2), filter,
keep samples 0, srate_mul, 2 srate_mul, ...; the WAV samples are float32.
"""
from __future__ import annotations

import cmath
import math

import numpy as np

FC_HZ = 5050.0          # generate_audio.py:29


def butter2_lowpass(wn: float) -> tuple[np.ndarray, np.ndarray]:
    """(b, a) of the 2nd-order digital Butterworth low-pass at normalised Wn."""
    fs = 2.0
    warped = 2.0 * fs * math.tan(math.pi * wn / fs)
    poles = [-cmath.exp(1j * math.pi * m / 4.0) * warped for m in (-1, 1)]
    k = warped ** 2
    fs2 = 2.0 * fs
    pz = [(fs2 + p) / (fs2 - p) for p in poles]
    kz = k * (1.0 / ((fs2 - poles[0]) * (fs2 - poles[1]))).real
    b = kz * np.array([1.0, 2.0, 1.0])
    a = np.array([1.0, (-(pz[0] + pz[1])).real, (pz[0] * pz[1]).real])
    return b, a


def lfilter_df2t(b, a, x) -> np.ndarray:
    """Direct form II transposed second-order section, zero initial state."""
    b0, b1, b2 = (float(v) / float(a[0]) for v in b)
    a1, a2 = float(a[1]) / float(a[0]), float(a[2]) / float(a[0])
    z0 = z1 = 0.0
    y = np.empty(len(x))
    for i, xi in enumerate(np.asarray(x, dtype=np.float64)):
        yi = z0 + b0 * xi
        z0 = (z1 + xi * b1) - yi * a1
        z1 = xi * b2 - yi * a2
        y[i] = yi
    return y


def audio(trace, srate_mul: int) -> np.ndarray:
    """WAV samples (float32, 44100 Hz) of one pressure trace."""
    p = np.asarray(trace, dtype=np.float64)
    x = np.clip(p / np.max(np.abs(p)), -1.0, 1.0)
    if srate_mul == 1:
        return x.astype(np.float32)
    b, a = butter2_lowpass(FC_HZ / (44100 * srate_mul / 2.0))
    return lfilter_df2t(b, a, x)[::srate_mul].astype(np.float32)

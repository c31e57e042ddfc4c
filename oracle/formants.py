"""Formant / bandwidth extraction, restating results/formants_bandwidths.py:5-80
(get_formants_bw) of the reference.

TEST INFRASTRUCTURE ONLY (F1-F4 parity checks).  Pinned against the
reference's own function by tests/golden/formants_golden.npz.

Algorithm (same steps as the reference): power spectrum in dB of the full
FFT; frequency axis f = 0:df:fs with df = fs/(N-1); scan bins from 1 for a
local maximum; at each peak walk left and right until the level drops 3 dB,
interpolate the two crossing frequencies linearly, and resume the scan at the
right crossing.
"""
from __future__ import annotations

import numpy as np


def formants_bw(signal, fs: float, num_formants: int) -> np.ndarray:
    """Rows: bandwidth (Hz), centre frequency (Hz), peak level (dB)."""
    x = np.asarray(signal)
    n = x.size
    level = 10.0 * np.log10(np.abs(np.fft.fft(x)) ** 2)
    df = fs / (n - 1)
    freq = np.arange(0, fs + df, df)
    out = np.zeros((3, num_formants))
    found = 0
    i = 1
    while found < num_formants and i < n - 1:
        if level[i] > level[i - 1] and level[i] > level[i + 1]:
            peak = level[i]
            cut = peak - 3
            lo = i
            while lo > 0 and level[lo] > cut:
                lo -= 1
            f_lo = np.interp(cut, level[lo:lo + 2], freq[lo:lo + 2])
            hi = i
            while hi < n - 1 and level[hi] > cut:
                hi += 1
            f_hi = np.interp(cut, level[hi - 1:hi + 1], freq[hi - 1:hi + 1])
            out[0, found] = f_hi - f_lo
            out[1, found] = freq[i]
            out[2, found] = peak
            found += 1
            i = hi
        else:
            i += 1
    return out

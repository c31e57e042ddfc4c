"""Seeded synthetic area functions for the benchmark and test tubes.

No public data set is involved: every tube is generated here from a seed with
numpy's PCG64 generator, in the reference's (length cm, area cm^2) per-section
format (TubeGeometry.cu:83-88).

  uniform_tube      straight tube, one section (17.5 cm x 3 cm diameter)
  vowel_area        44 sections of equal length; area = clip(2.2 + sum of five
                    cosine modes with seeded amplitudes/phases, 0.3, 5) cm^2
  batch_tube        vowel_area shape with a seeded length in [12, 20] cm and a
                    seeded maximum width in [2, 4] cm (3:1 elliptical major axis)
  batch_target_tube the inversion target of batch tube `seed`: same length and
                    maximum width, area shape of another seed
"""
from __future__ import annotations

import math

import numpy as np

N_SECTIONS = 44
AREA_MIN, AREA_MAX = 0.3, 5.0


def uniform_tube(length_cm: float = 17.5, diameter_cm: float = 3.0):
    """One section whose circular cross-section has the given diameter."""
    area = math.pi * (diameter_cm / 2.0) ** 2
    return np.array([length_cm], np.float32), np.array([area], np.float32)


def vowel_area(seed: int, n: int = N_SECTIONS) -> np.ndarray:
    """Smooth random area function (cm^2): 2.2 + sum_k a_k cos(pi k x + phi_k), clipped."""
    rng = np.random.default_rng(seed)
    k = np.arange(1, 6)
    amp = rng.uniform(-1.5, 1.5, size=5) / np.sqrt(k)
    phase = rng.uniform(0.0, 2.0 * np.pi, size=5)
    x = (np.arange(n) + 0.5) / n
    a = 2.2 + (amp[None, :] * np.cos(np.pi * k[None, :] * x[:, None] + phase[None, :])).sum(axis=1)
    return np.clip(a, AREA_MIN, AREA_MAX).astype(np.float32)


def vowel_tube(seed: int, length_cm: float = 17.5, n: int = N_SECTIONS):
    """(section lengths cm, areas cm^2) of a config-2 style vowel tube."""
    return np.full(n, length_cm / n, np.float32), vowel_area(seed, n)


def ellipse_area_for_width(width_cm: float) -> float:
    """Area (cm^2) of the 3:1 ellipse whose major axis is width_cm (TubeGeometry.cu:332-364)."""
    return 3.0 * math.pi * (width_cm / 6.0) ** 2


def batch_tube(seed: int, n: int = N_SECTIONS):
    """A tube of the batched workload: length U[12, 20] cm, max width U[2, 4] cm."""
    rng = np.random.default_rng(10_000 + seed)
    length = float(rng.uniform(12.0, 20.0))
    width = float(rng.uniform(2.0, 4.0))
    a = vowel_area(seed, n).astype(np.float64)
    a = a * (ellipse_area_for_width(width) / a.max())
    return np.full(n, length / n, np.float32), a.astype(np.float32), length, width


def batch_target_tube(seed: int, n: int = N_SECTIONS):
    """Target of the batched inversion for batch tube `seed`: the same length and
    maximum width, the area curve of seed 50 000 + seed."""
    L, _, length, width = batch_tube(seed, n)
    a = vowel_area(50_000 + seed, n).astype(np.float64)
    a = a * (ellipse_area_for_width(width) / a.max())
    return L, a.astype(np.float32), length, width

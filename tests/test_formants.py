"""oracle/formants.py against the reference's get_formants_bw (golden outputs)."""
from pathlib import Path

import numpy as np
import pytest

from formants import formants_bw

G = np.load(Path(__file__).parent / "golden" / "formants_golden.npz")


@pytest.mark.parametrize("k", range(4))
def test_formants_match_reference(k):
    got = formants_bw(G[f"signal_{k}"], 44100.0 * 15, 6)
    assert np.array_equal(got, G[f"bw_{k}"])

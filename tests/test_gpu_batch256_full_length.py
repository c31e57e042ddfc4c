"""The 256-tube batch workload at full length (50 ms), in the arithmetic the bench measures.

Eight tubes of the 256-tube batch -- the two shortest, the two longest, the
two narrowest and the two widest (seeds 156, 31, 222, 125, 183, 161, 166,
158) -- run together for all 33 075 steps (50 ms) with fast_math = 1 on the
two-step quad strips of the bench (shape 36, two time steps per launch).
Each FP32 trace must be within relative L2 1e-4 of the FP64 restatement of
the same tube, and its F1-F4 (the reference's get_formants_bw, restated in
oracle/formants.py; ~20 Hz bins at 50 ms, so "within 1 Hz" means the same
peak bin) within 1 Hz of the FP64 trace's.  The FP64 runs go to host
threads (ctypes releases the GIL).
"""
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

import oracle as O
import vocalsim_b200 as V
from formants import formants_bw
from vocalsim_b200 import synthetic as S

pytestmark = pytest.mark.gpu

SEEDS = [156, 31, 222, 125, 183, 161, 166, 158]
STEPS = 33075
BENCH_SHAPE = 36          # quad2_kernel<32, 4, 4, 2>
REL_L2_TOL = 1e-4
FS = 44100.0 * 15


@pytest.fixture(scope="module")
def runs(cuda_ok):
    tubes = [S.batch_tube(s)[:2] for s in SEEDS]
    b = V.Batch([V.params(cross_sectional_shape=2, fast_math=1) for _ in SEEDS], [V.Geometry(*t) for t in tubes])
    assert V.tile_shape_steps(BENCH_SHAPE) == 2
    b.set_tile(BENCH_SHAPE)
    gpu = b.run(STEPS)
    b.close()
    with ThreadPoolExecutor(len(SEEDS)) as ex:
        ref = list(ex.map(lambda t: O.run(O.params(cross_sectional_shape=2), O.Geometry(*t), STEPS, "f64"), tubes))
    return gpu, ref


@pytest.mark.parametrize("i", range(len(SEEDS)), ids=[f"seed{s}" for s in SEEDS])
def test_batch256_tube_rel_l2_vs_double(runs, i):
    gpu, ref = runs
    a, b = gpu[i].astype(np.float64), ref[i]
    err = float(np.linalg.norm(a - b) / np.linalg.norm(b))
    assert err <= REL_L2_TOL, err


@pytest.mark.parametrize("i", range(len(SEEDS)), ids=[f"seed{s}" for s in SEEDS])
def test_batch256_tube_formants_within_1hz(runs, i):
    gpu, ref = runs
    got = formants_bw(gpu[i].astype(np.float64), FS, 4)[1]
    want = formants_bw(ref[i], FS, 4)[1]
    assert np.all(want > 0) and np.all(np.abs(got - want) <= 1.0), (got, want)

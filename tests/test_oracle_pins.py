"""Pin the oracle's restatement against the reference's own compiled code.

The fixtures in tests/golden/reference_pieces.npz were produced by
tests/golden/make_golden.py from oracle/_ref/libvsref.so, i.e. the reference's
TwoMassModel.cpp, GlottalExcitations.cu, SolverParams.cu and
SimulationParams.cu compiled from the reference tree.  Equality is exact.
"""
from pathlib import Path

import numpy as np
import pytest

import oracle as O

G = np.load(Path(__file__).parent / "golden" / "reference_pieces.npz")


@pytest.mark.parametrize("mul", [1, 15, 30])
def test_simulation_params(mul):
    ref = G[f"sim_params_{mul}"]          # c, rho, kappa, dt, ds, max_sigma_dt, layers, cpl, Mw, Bw, Kw, srate
    k = O.consts(mul)                     # c, rho, kappa, dt, ds, max_sigma_dt, K1, K2, Mw, Bw, Kw
    assert np.array_equal(k[:6], ref[:6])
    assert np.array_equal(k[8:11], ref[8:11])
    assert ref[6] == 6 and ref[7] == 0 and ref[11] == 44100 * mul


@pytest.mark.parametrize("mul", [15, 30])
def test_solver_tables(mul):
    b, s, d = O.tables(mul)
    assert np.array_equal(b, G[f"beta_{mul}"])
    assert np.array_equal(s, G[f"sigma_{mul}"])
    assert np.array_equal(d, G[f"dir_{mul}"])


@pytest.mark.parametrize("mul", [15, 30])
def test_step_counts(mul):
    dt = O.consts(mul)[3]
    got = [O.step_count(float(x), float(dt)) for x in G[f"step_durations_{mul}"]]
    assert got == list(G[f"step_counts_{mul}"])


@pytest.mark.parametrize("mul", [15, 30])
@pytest.mark.parametrize("source", [0, 1, 2])
def test_excitation_tables(mul, source):
    p = O.params(source_type=source, srate_mul=mul)
    assert np.array_equal(O.source(p, 4000), G[f"excitation_{source}_{mul}"])


@pytest.mark.parametrize("mul", [15, 30])
def test_two_mass_model_random_pressure(mul):
    ug = O.tmm(686.46, mul, G[f"tmm_p1_{mul}"])
    assert np.array_equal(ug, G[f"tmm_ug_{mul}"])


@pytest.mark.parametrize("mul", [15, 30])
def test_two_mass_model_free_oscillation(mul):
    ug = O.tmm(686.46, mul, np.zeros(20000, np.float32))
    assert np.array_equal(ug, G[f"tmm_ug_zero_p1_{mul}"])
    assert ug.max() > 1e-4          # the folds oscillate and let air through


@pytest.mark.parametrize("mul", [15, 30])
def test_double_model_arrangement_tracks_the_literal_double_model(mul):
    """The tmm_f64 option's arrangement of the double model (per-model
    reciprocals, three divisions a step) against the model's literal
    expressions in double: the same flows to rounding, driven by the golden
    random pressures and in free oscillation over 20 000 steps."""
    for p1 in (G[f"tmm_p1_{mul}"].astype(np.float64), np.zeros(20000)):
        lit = O.tmm(686.46, mul, p1, "f64")
        arr = O.tmm(686.46, mul, p1, "f64r")
        assert np.abs(lit).max() > 1e-4
        assert np.linalg.norm(arr - lit) <= 1e-9 * np.linalg.norm(lit)
        assert np.abs(arr - lit).max() <= 1e-9 * np.abs(lit).max()


def test_double_two_mass_model_tracks_the_fp64_restatement():
    """FP32 fields with the two-mass model in double (tmm_f64) stay within
    1e-4 relative L2 of the all-double run; the reference's float model
    drifts from it by more than 1e-3 over the same 3000 steps."""
    from vocalsim_b200 import synthetic as S
    L, A = S.vowel_tube(0)
    g = O.Geometry(L, A)
    err = {}
    for f64 in (0, 1):
        p = O.params(cross_sectional_shape=2, source_type=2, tmm_ps_pa=800.0, tmm_f64=f64)
        a, b = O.run(p, g, 3000), O.run(p, g, 3000, precision="f64")
        err[f64] = np.linalg.norm(a - b) / np.linalg.norm(b)
    assert err[1] <= 1e-4 and err[0] > 1e-3, err


def test_known_answers():
    """Constants computed by float probes of the reference's own expressions."""
    k15, k30 = O.consts(15), O.consts(30)
    assert k15[3] == np.float32(1.51171582e-06) and k30[3] == np.float32(7.55857911e-07)
    assert k15[4] == np.float32(7.48261169e-04) and k30[4] == np.float32(3.74130585e-04)
    assert k15[2] == np.float32(139650)
    assert abs(k15[6] - 282.13559) < 1e-4 and abs(k30[6] - 282.13559) < 1e-4
    assert k15[7] == np.float32(0.211111113) and k30[7] == np.float32(0.105555557)
    m = O.maps(O.params(mu3d=0.025), O.Geometry([17.5], [np.pi * 1.5 ** 2]))
    assert np.float32(m["dims"]["z_inv_val"]) == np.float32(1.06979205e-04)
    m = O.maps(O.params(mu3d=0.005), O.Geometry([17.5], [np.pi * 1.5 ** 2]))
    assert np.float32(m["dims"]["z_inv_val"]) == np.float32(2.13958047e-05)
    assert m["dims"]["frame_h"] == 57 and m["dims"]["frame_w"] == 253
    assert m["dims"]["interior_cells"] == 13805 and m["dims"]["tube_length_cells"] == 234
    p = O.params()
    assert np.float32(p.gauss_peak_s) == np.float32(6.46000044e-05)
    assert np.float32(p.gauss_width_s) == np.float32(1.87340011e-05)

"""The C++ mirror classes (SimulationParams / TubeGeometry / FDTDSolver /
FDTDEngineB200) compile against the C ABI and reproduce the reference flow."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle as O
from vocalsim_b200 import synthetic as S

PKG = Path(__file__).resolve().parents[1] / "vocalsim-2p5d-fdtd_b200"


@pytest.fixture(scope="module")
def example(tmp_path_factory):
    exe = tmp_path_factory.mktemp("cpp") / "example_engine"
    subprocess.run(["g++", "-std=c++17", "-O2", str(PKG / "cpp" / "example_engine.cpp"), "-I", str(PKG / "cpp"),
                    "-L", str(PKG / "lib"), "-lvocalsim_b200", f"-Wl,-rpath,{PKG / 'lib'}", "-o", str(exe)],
                   check=True)
    return exe


def test_mirror_builds_reference_frame(example):
    out = subprocess.run([str(example), "--maps-only"], check=True, capture_output=True, text=True).stdout
    assert "frame 57 x 253, listener (28, 248), 13229 steps" in out


@pytest.mark.gpu
def test_mirror_engine_record_pressure(example, cuda_ok):
    out = subprocess.run([str(example)], check=True, capture_output=True, text=True).stdout
    L, A = S.uniform_tube()
    ref = O.run(O.params(uniform_depth_m=0.02, mu3d=0.005, audio_dur=0.02), O.Geometry(L, A), 13229, "f32")
    line = [ln for ln in out.splitlines() if ln.startswith("record_pressure")][0]
    energy = float(line.split("energy ")[1].split(",")[0])
    p100 = float(line.split("p[100] ")[1])
    assert abs(energy - float(np.sum(ref.astype(np.float64) ** 2))) <= 1e-6 * energy
    assert np.float32(p100) == ref[100] or abs(p100 - ref[100]) <= 1e-6 * abs(ref[100])

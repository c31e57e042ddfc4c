"""The C++ mirror classes (cpp/vocalsim_b200.hpp: SimulationParams,
TubeGeometry, TubeDepth, GlottalExcitations, FDTDSolver, FDTDEngineCPU,
FDTDEngineEigen) compile against the C ABI and reproduce the reference flow;
the reference's own driver, src/main.cu, builds unchanged against the
reference-named headers in cpp/include and runs on the GPU."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle as O
from vocalsim_b200 import synthetic as S

PKG = Path(__file__).resolve().parents[1] / "vocalsim-2p5d-fdtd_b200"
AF = np.load(Path(__file__).parent / "golden" / "reference_area_functions.npz")


@pytest.fixture(scope="module")
def example(tmp_path_factory):
    exe = tmp_path_factory.mktemp("cpp") / "example_engine"
    subprocess.run(["g++", "-std=c++17", "-O2", str(PKG / "cpp" / "example_engine.cpp"), "-I", str(PKG / "cpp"),
                    "-L", str(PKG / "lib"), "-lvocalsim_b200", f"-Wl,-rpath,{PKG / 'lib'}", "-o", str(exe)],
                   check=True)
    return exe


def write_area(path: Path, name: str) -> None:
    """A reference area-function file: 'length_cm area_cm2' per line."""
    L, A = AF[f"{name}_length_cm"], AF[f"{name}_area_cm2"]
    path.write_text("".join(f"{O._fmt32(l)} {O._fmt32(a)}\n" for l, a in zip(L, A)))


def test_mirror_builds_reference_frame(example):
    out = subprocess.run([str(example), "--maps-only"], check=True, capture_output=True, text=True).stdout
    assert "frame 57 x 253, listener (28, 248), 13229 steps" in out


@pytest.mark.parametrize("vowel,name", [(1, "vocaltract_a"), (2, "vocaltract_i"), (3, "vocaltract_u"),
                                        (7, "cylindrical-tube")])
def test_mirror_reads_the_reference_data_files(example, tmp_path, vowel, name):
    """FDTDSolver without a geometry reads data_dir/<file> chosen by vowel_type
    the way TubeGeometry's constructor does (TubeGeometry.cu:57-88)."""
    write_area(tmp_path / f"{name}.txt", name)
    out = subprocess.run([str(example), "--data-dir", str(tmp_path), str(vowel)], check=True, capture_output=True,
                         text=True).stdout
    m = O.maps(O.params(cross_sectional_shape=1, mouth_radiation_cond=1, pml_flag=0, audio_dur=0.1),
               O.Geometry(AF[f"{name}_length_cm"], AF[f"{name}_area_cm2"]))["dims"]
    steps = O.step_count(0.1, float(O.consts(15)[3]))
    assert f"frame {m['frame_h']} x {m['frame_w']}, listener ({m['listener_y']}, {m['listener_x']}), {steps} steps" in out


@pytest.mark.gpu
def test_mirror_engine_record_pressure(example, cuda_ok, tmp_path):
    """record_pressure of the mirror's engine equals the FP32 oracle's trace, every sample."""
    out_file = tmp_path / "trace.f32"
    subprocess.run([str(example), "--trace", str(out_file)], check=True, capture_output=True, text=True)
    got = np.fromfile(out_file, np.float32)
    L, A = S.uniform_tube()
    ref = O.run(O.params(uniform_depth_m=0.02, mu3d=0.005, audio_dur=0.02), O.Geometry(L, A), 13229, "f32")
    assert got.shape == ref.shape and np.array_equal(got, ref)


@pytest.mark.gpu
@pytest.mark.skipif(not O.MAIN_ON_MIRROR.exists(), reason="oracle/_ref/main_on_mirror not built (needs the reference tree)")
def test_reference_main_runs_unchanged_on_the_mirror(cuda_ok, tmp_path):
    """The reference's main.cu, compiled unchanged against cpp/include: its run
    (vowel /a/, circular, 2.5D, Dirichlet mouth, x15, 100 ms, Gaussian, no PML,
    the Eigen engine) writes ../../results/recorded-pressure.txt; every line
    equals the FP32 oracle's trace (Eigen rounding) printed the same way."""
    (tmp_path / "data" / "tube-geometry").mkdir(parents=True)
    (tmp_path / "results").mkdir()
    (tmp_path / "a" / "b").mkdir(parents=True)
    write_area(tmp_path / "data" / "tube-geometry" / "vocaltract_a.txt", "vocaltract_a")
    r = subprocess.run([str(O.MAIN_ON_MIRROR)], cwd=tmp_path / "a" / "b", capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = (tmp_path / "results" / "recorded-pressure.txt").read_text().split()
    p = O.params(cross_sectional_shape=1, mouth_radiation_cond=1, pml_flag=0, audio_dur=0.1, engine=2)
    n = O.step_count(0.1, float(O.consts(15)[3]))
    ref = O.run(p, O.Geometry(AF["vocaltract_a_length_cm"], AF["vocaltract_a_area_cm2"]), n, "f32")
    assert len(lines) == n
    want = ["%g" % float(v) for v in ref]
    bad = [i for i, (a, b) in enumerate(zip(lines, want)) if a != b]
    assert not bad, f"{len(bad)} lines differ, first at {bad[0]}: {lines[bad[0]]} vs {want[bad[0]]}"

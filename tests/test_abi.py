"""The C-ABI library: loads, exports every declared symbol, struct layout
matches the ctypes mirror, defaults equal the reference's, and device entry
points fail loudly without a GPU.  No GPU compute runs here."""
import ctypes as C
import subprocess
import textwrap

import numpy as np
import pytest

import oracle as O
import vocalsim_b200 as V
from vocalsim_b200 import abi


def test_library_exports_every_header_symbol():
    lib = abi.load_library()
    syms = abi.header_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    assert lib.vs_version() == abi.VS_ABI_VERSION


def test_struct_layout_matches_header(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text(textwrap.dedent(f"""
        #include <stdio.h>
        #include <stddef.h>
        #include "{abi.HEADER_PATH}"
        int main(void) {{
          printf("%zu %zu %zu\\n", sizeof(vs_params), sizeof(vs_geometry), sizeof(vs_dims));
          printf("%zu %zu %zu %zu\\n", offsetof(vs_params, num_steps), offsetof(vs_params, tmm_ps_pa),
                 offsetof(vs_params, listener_y), offsetof(vs_params, reserved));
          printf("%zu %zu\\n", offsetof(vs_dims, num_steps), offsetof(vs_dims, z_inv_val));
          return 0;
        }}"""))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    P, G, D = abi.VsParams, abi.VsGeometry, abi.VsDims
    assert [int(x) for x in out] == [
        C.sizeof(P), C.sizeof(G), C.sizeof(D),
        P.num_steps.offset, P.tmm_ps_pa.offset, P.listener_y.offset, P.reserved.offset,
        D.num_steps.offset, D.z_inv_val.offset]


def test_defaults_equal_reference_configuration():
    assert V.params().as_dict() == O.params().as_dict()


@pytest.mark.parametrize("source", [0, 1, 3])
def test_source_table_matches_oracle(source):
    kw = dict(source_type=source, gauss_peak_s=5e-4, gauss_width_s=1e-4) if source == 3 else dict(source_type=source)
    assert np.array_equal(V.source_table(V.params(**kw), 3000), O.source(O.params(**kw), 3000))


def test_tile_shapes_listed():
    shapes = V.tile_shapes()
    assert len(shapes) >= 4
    *strips, cluster = shapes
    assert all(r > 0 and c % 30 == 0 for r, c in strips)     # strips commit 30 columns per warp
    assert cluster == (0, 0)                                  # the last shape: one tube per cluster
    steps = [V.tile_shape_steps(i) for i in range(len(shapes))]
    assert set(steps[:-1]) == {1, 2} and steps.count(2) >= 8   # single-step and two-step shapes
    assert steps[-1] == 0                                     # the cluster kernel runs a whole run per launch
    assert V.load_library().vs_tile_shape_steps(len(shapes), None) == 1


def test_device_entry_points_fail_loudly_without_gpu():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    from vocalsim_b200 import synthetic as S
    with pytest.raises(V.VsError) as e:
        V.Solver(V.params(), V.Geometry(*S.vowel_tube(0)))
    assert e.value.status == 3          # VS_ERR_CUDA, no CPU fallback


def test_null_arguments_rejected():
    lib = abi.load_library()
    assert lib.vs_params_init(None) == 1
    assert lib.vs_run(None, 10, None, 0) == 1
    assert lib.vs_batch_run(None, 10, None, 0) == 1
    assert lib.vs_batch_create(0, None, None, None) == 1
    assert lib.vs_tile_shape(-1, None, None) == 1
    assert b"" != lib.vs_last_error()

"""vs_run_noalloc: stepping a tube without any device allocation.

Callers that cannot call cudaMalloc when they run the solver (a real-time
audio thread, where an allocation may block; an application whose device
memory another allocator has reserved) hand in buffers they already own.
This test plays such a caller: it places the maps of vs_build_maps and the
table of vs_source_table in device memory it owns, calls vs_run_noalloc
through the C ABI, and compares the trace with what the allocating entry
point vs_run returns for the same tube.  Both run the same FP32 arithmetic,
so the tolerance is the one the other parity tests use: exact equality.
Two different tubes are run back to back (and the first one again) to show
that state left in the shared static array by one call does not leak into
the next.

The file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

import vocalsim_b200 as V
from vocalsim_b200 import abi
from vocalsim_b200 import synthetic as S


def _run_noalloc(torch, p, g, steps):
    """Caller-owned device buffers in, device trace out; returns the host trace."""
    lib = abi.load_library()
    m = V.build_maps(p, g)
    d = abi.VsDims(**{k: v for k, v in m["dims"].items()})
    dev = torch.device("cuda", 0)
    bufs = {k: torch.from_numpy(np.ascontiguousarray(m[k])).to(dev)
            for k in ("cell_type", "depth_p", "depth_x", "depth_y", "z_inv")}
    src = None
    if p.source_type != V.SRC_TMM:
        src = torch.from_numpy(V.source_table(p, steps)).to(dev)
    trace = torch.full((steps,), float("nan"), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    torch.cuda.synchronize()
    rc = lib.vs_run_noalloc(C.byref(p), C.byref(d), C.c_void_p(bufs["cell_type"].data_ptr()),
                            C.c_void_p(bufs["depth_p"].data_ptr()), C.c_void_p(bufs["depth_x"].data_ptr()),
                            C.c_void_p(bufs["depth_y"].data_ptr()), C.c_void_p(bufs["z_inv"].data_ptr()),
                            C.c_void_p(src.data_ptr()) if src is not None else None, steps,
                            C.c_void_p(trace.data_ptr()), C.c_void_p(stream.cuda_stream))
    abi.check(lib, rc, "vs_run_noalloc")
    torch.cuda.synchronize()
    return trace.cpu().numpy()


@pytest.mark.gpu
def test_noalloc_matches_vs_run_on_consecutive_calls(cuda_ok):
    import torch
    steps = 1200
    tube_a = (V.params(cross_sectional_shape=2, source_type=V.SRC_TMM, tmm_ps_pa=800.0), S.vowel_tube(2))
    tube_b = (V.params(mu3d=0.005, uniform_depth_m=0.02, mouth_radiation_cond=1), S.uniform_tube())
    results = []
    for p, (L, A) in (tube_a, tube_b, tube_a):
        g = V.Geometry(L, A)
        got = _run_noalloc(torch, p, g, steps)
        want = V.Solver(p, g).run(steps)
        assert np.array_equal(got, want), f"max |d| = {np.nanmax(np.abs(got - want))}"
        assert np.any(want != 0)
        results.append(got)
    assert np.array_equal(results[0], results[2])


def test_noalloc_rejects_frames_beyond_the_static_scratch():
    lib = abi.load_library()
    p = V.params()
    d = abi.VsDims(frame_h=1200, frame_w=1200, listener_x=5, listener_y=5, excitation_x=3, excitation_y=5)
    dummy = C.c_void_p(16)          # never dereferenced: the size check comes first
    rc = lib.vs_run_noalloc(C.byref(p), C.byref(d), dummy, dummy, dummy, dummy, dummy, dummy, 10, dummy, None)
    assert rc == abi.VS_ERR_INVALID_ARG
    assert b"static scratch" in lib.vs_last_error()


@pytest.mark.parametrize("field,value", [("listener_x", 0), ("listener_x", 252), ("listener_y", 56),
                                         ("excitation_x", -3), ("excitation_y", 0), ("excitation_y", 57)])
def test_noalloc_rejects_cells_outside_the_interior(field, value):
    """Listener and excitation must be interior cells (1..W-2 x 1..H-2), the
    ranges the map builder guarantees; the check comes before any device work."""
    lib = abi.load_library()
    p = V.params()
    dims = dict(frame_h=57, frame_w=253, listener_x=248, listener_y=28, excitation_x=7, excitation_y=28)
    dims[field] = value
    d = abi.VsDims(**dims)
    dummy = C.c_void_p(16)          # never dereferenced: the range check comes first
    rc = lib.vs_run_noalloc(C.byref(p), C.byref(d), dummy, dummy, dummy, dummy, dummy, dummy, 10, dummy, None)
    assert rc == abi.VS_ERR_INVALID_ARG
    assert b"outside the frame" in lib.vs_last_error()


@pytest.mark.gpu
def test_noalloc_invalid_cell_type_gives_a_nan_trace(cuda_ok):
    """A cell type outside 0..12 has no update in the reference; the maps live
    on the device, so the entry point returns a NaN trace instead of reading
    past its coefficient tables, and the next valid call is unaffected."""
    import torch
    lib = abi.load_library()
    p = V.params(mu3d=0.005, uniform_depth_m=0.02)
    g = V.Geometry(*S.uniform_tube())
    m = V.build_maps(p, g)
    d = abi.VsDims(**{k: v for k, v in m["dims"].items()})
    dev = torch.device("cuda", 0)
    bad_types = np.array(m["cell_type"], copy=True)
    bad_types[10, 40] = 13
    bufs = {k: torch.from_numpy(np.ascontiguousarray(m[k])).to(dev)
            for k in ("depth_p", "depth_x", "depth_y", "z_inv")}
    bufs["cell_type"] = torch.from_numpy(bad_types).to(dev)
    steps = 64
    src = torch.from_numpy(V.source_table(p, steps)).to(dev)
    trace = torch.zeros((steps,), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    torch.cuda.synchronize()
    rc = lib.vs_run_noalloc(C.byref(p), C.byref(d), C.c_void_p(bufs["cell_type"].data_ptr()),
                            C.c_void_p(bufs["depth_p"].data_ptr()), C.c_void_p(bufs["depth_x"].data_ptr()),
                            C.c_void_p(bufs["depth_y"].data_ptr()), C.c_void_p(bufs["z_inv"].data_ptr()),
                            C.c_void_p(src.data_ptr()), steps, C.c_void_p(trace.data_ptr()),
                            C.c_void_p(stream.cuda_stream))
    abi.check(lib, rc, "vs_run_noalloc")
    torch.cuda.synchronize()
    assert np.all(np.isnan(trace.cpu().numpy()))
    good = _run_noalloc(torch, p, g, steps)
    assert np.array_equal(good, V.Solver(p, g).run(steps))


"""Formants of listener traces computed on the GPU (vs_formants).

The same quantities as the reference's get_formants_bw
(results/formants_bandwidths.py:5-80), for a batch of traces at once: rows
(bandwidth Hz, centre frequency Hz, peak level dB) per formant.
"""
from __future__ import annotations

import numpy as np

from .abi import check, load_library


def formants(traces, fs: float, num_formants: int = 4) -> np.ndarray:
    """traces: (n,) or (k, n) float32 array (host numpy or a CUDA torch tensor).
    Returns (k, 3, num_formants) float64 (or (3, num_formants) for one trace)."""
    import torch
    single = False
    if isinstance(traces, torch.Tensor):
        t = traces.detach().to(device="cuda", dtype=torch.float32).contiguous()
    else:
        a = np.asarray(traces, dtype=np.float32)
        t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    if t.dim() == 1:
        t = t[None]
        single = True
    k, n = t.shape
    out = torch.zeros((k, 3, num_formants), dtype=torch.float64, device=t.device)
    lib = load_library()
    stream = torch.cuda.current_stream(t.device).cuda_stream
    check(lib, lib.vs_formants(t.data_ptr(), k, n, float(fs), num_formants, out.data_ptr(), stream), "vs_formants")
    res = out.cpu().numpy()
    return res[0] if single else res

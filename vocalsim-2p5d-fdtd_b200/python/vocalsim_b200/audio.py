"""WAV samples of listener traces computed on the GPU (vs_audio).

The same samples as the reference's results/generate_audio.py (lines 14-42)
writes to sound.wav: each trace divided by its largest |P|, clipped to
[-1, 1]; for srate_mul > 1 the 2nd-order Butterworth low-pass at 5050 Hz
(scipy.signal.butter / lfilter, direct form II transposed, in double) and
every srate_mul-th sample kept; float32 at 44100 Hz.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .abi import check, load_library

WAV_RATE = 44100


def audio(traces, srate_mul: int):
    """traces: (n,) or (k, n) float32 (host numpy or a CUDA torch tensor).
    Returns a CUDA float32 tensor (k, ceil(n / srate_mul)) (or (m,) for one trace)."""
    import torch
    if isinstance(traces, torch.Tensor):
        t = traces.detach().to(device="cuda", dtype=torch.float32).contiguous()
    else:
        t = torch.from_numpy(np.ascontiguousarray(np.asarray(traces, dtype=np.float32))).cuda()
    single = t.dim() == 1
    if single:
        t = t[None]
    k, n = t.shape
    m = max(int(srate_mul), 1)          # vs_audio itself rejects srate_mul < 1
    out = torch.empty((k, (n + m - 1) // m), dtype=torch.float32, device=t.device)
    lib = load_library()
    stream = torch.cuda.current_stream(t.device).cuda_stream
    check(lib, lib.vs_audio(t.data_ptr(), k, n, int(srate_mul), out.data_ptr(), stream), "vs_audio")
    return out[0] if single else out


def audio_filter(srate_mul: int) -> tuple[np.ndarray, np.ndarray]:
    """(b, a) of the low-pass vs_audio applies for srate_mul (host only)."""
    lib = load_library()
    b = (C.c_double * 3)()
    a = (C.c_double * 3)()
    check(lib, lib.vs_audio_filter(int(srate_mul), b, a), "vs_audio_filter")
    return np.array(list(b)), np.array(list(a))


def write_wav(path: str, samples) -> None:
    """Write float32 mono samples as the IEEE-float WAV at 44100 Hz that the
    reference's scipy.io.wavfile.write(path, 44100, samples) call writes: RIFF
    header, 18-byte fmt chunk (format 3, cbSize 0), fact chunk (sample
    count), data chunk."""
    import struct
    x = np.asarray(samples.cpu().numpy() if hasattr(samples, "cpu") else samples, dtype="<f4").ravel()
    data = x.tobytes()
    fmt = struct.pack("<HHIIHH", 3, 1, WAV_RATE, WAV_RATE * 4, 4, 32) + b"\x00\x00"
    body = (b"WAVE" + b"fmt " + struct.pack("<I", len(fmt)) + fmt
            + b"fact" + struct.pack("<II", 4, x.size)
            + b"data" + struct.pack("<I", len(data)) + data)
    with open(path, "wb") as f:
        f.write(b"RIFF" + struct.pack("<I", len(body)) + body)

"""Measured modular-multiply peak of the GPU (the compute roofline of the
NTT-bound ct-mult kernels)."""
from __future__ import annotations

import torch

from . import _lib

KINDS = {0: "int64_shoup", 1: "fp64_dword", 2: "mixed"}


def modmul_peak(kind: int = 0, iters: int = 2048, q: int = 35184371884033, w: int = 12345678901234,
                reps: int = 3) -> float:
    """Best modular multiplies per second over `reps` timed launches."""
    dev = torch.device("cuda", torch.cuda.current_device())
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    blocks, threads = sms * 8, 256
    out = torch.empty(blocks * threads, dtype=torch.uint64, device=dev)
    st = torch.cuda.current_stream().cuda_stream
    _lib.call("ckks_modmul_peak", out.data_ptr(), blocks, threads, 64, kind, q, w, st)
    best = 0.0
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        _lib.call("ckks_modmul_peak", out.data_ptr(), blocks, threads, iters, kind, q, w, st)
        e1.record()
        torch.cuda.synchronize()
        s = e0.elapsed_time(e1) / 1000.0
        best = max(best, blocks * threads * iters * 8 / s)
    return best

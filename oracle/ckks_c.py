"""ctypes binding of the native CPU restatement of the RNS ct-mult
(oracle/ckks_cpu.c; test infrastructure: the timed CPU baseline and a
second oracle, pinned bit-exact against oracle.rns_ckks in the CPU tests).

``build()`` compiles it with gcc into oracle/_c/libckks_cpu.so (portable
x86-64 code generation, so the library built here runs on any host)."""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SRC = HERE / "ckks_cpu.c"
LIB = HERE / "_c" / "libckks_cpu.so"

_lib = None


def build(force: bool = False) -> Path:
    if not force and LIB.exists() and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    LIB.parent.mkdir(exist_ok=True)
    cmd = ["gcc", "-O3", "-std=c11", "-fPIC", "-shared", "-Wall", "-Wextra", "-o", str(LIB), str(SRC), "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"gcc failed for {SRC.name}:\n{r.stderr}")
    return LIB


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        lib = C.CDLL(str(LIB))
        lib.cc_create.restype = C.c_void_p
        lib.cc_create.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        lib.cc_destroy.restype = None
        lib.cc_destroy.argtypes = [C.c_void_p]
        lib.cc_ct_mul_relin_rescale.restype = C.c_int
        lib.cc_ct_mul_relin_rescale.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                C.c_longlong, C.c_int, C.c_int]
        _lib = lib
    return _lib


class CpuCtMul:
    """The ct-mult + relin + rescale over one key basis (q_0..q_{L-1}, p),
    the oracle's conventions: ciphertexts [B, 2, l, N] and key
    [L, 2, L + 1, N] in the evaluation domain (bit-reversed order)."""

    def __init__(self, log_n: int, qs, p: int):
        from .modmath import root_2n
        self.n = 1 << log_n
        self.qs = [int(q) for q in qs]
        primes = np.asarray(self.qs + [int(p)], dtype=np.uint64)
        psi = np.asarray([root_2n(int(q), self.n) for q in primes], dtype=np.uint64)
        self._keep = (primes, psi)
        self.h = load().cc_create(log_n, len(self.qs), primes.ctypes.data, psi.ctypes.data)
        if not self.h:
            raise ValueError("cc_create refused the basis")

    def __call__(self, ct_a, ct_b, ksk, threads: int | None = None) -> np.ndarray:
        a = np.ascontiguousarray(ct_a, dtype=np.uint64)
        b = np.ascontiguousarray(ct_b, dtype=np.uint64)
        k = np.ascontiguousarray(ksk, dtype=np.uint64)
        B, _, l, n = a.shape
        assert n == self.n and b.shape == a.shape and k.shape == (len(self.qs), 2, len(self.qs) + 1, n)
        out = np.empty((B, 2, l - 1, n), dtype=np.uint64)
        rc = load().cc_ct_mul_relin_rescale(self.h, out.ctypes.data, a.ctypes.data, b.ctypes.data, k.ctypes.data,
                                            B, l, int(threads or os.cpu_count() or 1))
        if rc:
            raise RuntimeError("cc_ct_mul_relin_rescale failed")
        return out

    def close(self):
        if self.h:
            load().cc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

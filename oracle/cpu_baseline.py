"""Timed CPU baseline of the ct-mult + relin + rescale path (test infrastructure).

Runs the native C restatement of the oracle's RNS ct-mult (oracle/ckks_cpu.c,
pinned bit-exact against oracle.rns_ckks.ct_mul_relin_rescale by
tests/test_oracle_c.py) on every host core, one POSIX thread per core.  Used
only by bench.py's cpu_baseline leg and its ``--impl reference`` arm: the
reference project has no CPU implementation of the RNS path (its goldens are
single-modulus O(N^2) Python loops), so the timed CPU arm is this port.
"""
from __future__ import annotations

import os
import time

import numpy as np


def _primes(levels: int, log_n_max: int = 13):
    from .modmath import find_primes
    pr = find_primes(45, 1 << (log_n_max + 1), levels + 1)
    return pr[1:], pr[0]


class CpuPool:
    """All host cores running the native C ct-mult on one fixed batch."""

    def __init__(self, log_n: int = 12, levels: int = 3, cores: int | None = None, batch: int | None = None):
        from . import ckks_c
        self.log_n, self.levels = log_n, levels
        self.cores = cores or os.cpu_count() or 1
        self.batch = batch or 4 * self.cores
        qs, p = _primes(levels)
        n = 1 << log_n
        rng = np.random.default_rng(1000)

        def rnd(shape, basis):
            x = np.zeros(shape, dtype=np.uint64)
            for i, q in enumerate(basis):
                x[..., i, :] = rng.integers(0, q, size=x[..., i, :].shape, dtype=np.uint64)
            return x

        self.a = rnd((self.batch, 2, levels, n), qs)
        self.b = rnd((self.batch, 2, levels, n), qs)
        self.k = rnd((levels, 2, levels + 1, n), qs + [p])
        self.cm = ckks_c.CpuCtMul(log_n, qs, p)
        self.cm(self.a, self.b, self.k, threads=self.cores)  # warm: pages, tables

    def step(self, seconds: float) -> tuple[int, float]:
        """One timed round of whole-batch calls for ~seconds; returns (done, wall)."""
        done = 0
        t0 = time.perf_counter()
        while True:
            self.cm(self.a, self.b, self.k, threads=self.cores)
            done += self.batch
            if time.perf_counter() - t0 >= seconds:
                break
        return done, time.perf_counter() - t0

    def sample(self, done: int, seconds: float) -> str:
        return (f"{done} ct-mult+relin+rescale (N=2^{self.log_n}, L={self.levels}) in native C "
                f"(oracle/ckks_cpu.c: Shoup / lazy Harvey transforms, floating-point-quotient products) on "
                f"{self.cores} threads, {self.batch} pairs per call, ~{seconds:.1f} s per round")

    def close(self):
        self.cm.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def measure(log_n: int = 12, levels: int = 3, seconds: float = 10.0, cores: int | None = None,
            batch: int | None = None) -> dict:
    """ct-mults per second on `cores` threads (default: all host cores)."""
    with CpuPool(log_n, levels, cores, batch) as pool:
        done, wall = pool.step(seconds)
        return {"value": done / wall, "cores": pool.cores, "done": done, "wall_s": wall,
                "sample": pool.sample(done, seconds)}

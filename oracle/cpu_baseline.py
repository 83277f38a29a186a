"""Timed CPU baseline of the ct-mult + relin + rescale path (test infrastructure).

Runs the oracle's numpy restatement (oracle.rns_ckks.ct_mul_relin_rescale) on
every host core through a spawn-started process pool.  Used only by bench.py's
cpu_baseline leg and its ``--impl reference`` arm: the reference project has
no CPU implementation of the RNS path (its goldens are single-modulus O(N^2)
Python loops), so the timed CPU arm is this port.
"""
from __future__ import annotations

import multiprocessing as mp
import os
import time

import numpy as np


def _primes(levels: int, log_n_max: int = 13):
    from .modmath import find_primes
    pr = find_primes(45, 1 << (log_n_max + 1), levels + 1)
    return pr[1:], pr[0]


def _worker(args):
    log_n, levels, batch, seconds, seed = args
    from . import rns_ckks as R
    qs, p = _primes(levels)
    n = 1 << log_n
    rng = np.random.default_rng(seed)

    def rnd(shape, basis):
        x = np.zeros(shape, dtype=np.uint64)
        for i, q in enumerate(basis):
            x[..., i, :] = rng.integers(0, q, size=x[..., i, :].shape, dtype=np.uint64)
        return x

    a = rnd((batch, 2, levels, n), qs)
    b = rnd((batch, 2, levels, n), qs)
    k = rnd((levels, 2, levels + 1, n), qs + [p])
    R.ct_mul_relin_rescale(a[:1], b[:1], k, qs, p)  # warm tables
    done = 0
    t0 = time.perf_counter()
    while True:
        R.ct_mul_relin_rescale(a, b, k, qs, p)
        done += batch
        if time.perf_counter() - t0 >= seconds:
            break
    return done, time.perf_counter() - t0


class CpuPool:
    """All-core process pool (spawn start) running the oracle ct-mult."""

    def __init__(self, log_n: int = 12, levels: int = 3, cores: int | None = None, batch: int = 4):
        self.log_n, self.levels, self.batch = log_n, levels, batch
        self.cores = cores or os.cpu_count() or 1
        self._pool = mp.get_context("spawn").Pool(self.cores)
        self._pool.map(_worker, [(log_n, levels, 1, 0.0, i) for i in range(self.cores)])
        self._seed = 1000

    def step(self, seconds: float) -> tuple[int, float]:
        """One timed round: every process runs ct-mults for ~seconds; returns (done, wall)."""
        self._seed += self.cores
        t0 = time.perf_counter()
        res = self._pool.map(_worker, [(self.log_n, self.levels, self.batch, seconds, self._seed + i)
                                       for i in range(self.cores)])
        return sum(r[0] for r in res), time.perf_counter() - t0

    def sample(self, done: int, seconds: float) -> str:
        return (f"{done} ct-mult+relin+rescale (N=2^{self.log_n}, L={self.levels}) on {self.cores} "
                f"spawned processes, numpy uint64 restatement, {self.batch} pairs per call, "
                f"~{seconds:.1f} s per process per round")

    def close(self):
        self._pool.close()
        self._pool.join()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def measure(log_n: int = 12, levels: int = 3, seconds: float = 10.0, cores: int | None = None,
            batch: int = 4) -> dict:
    """ct-mults per second on `cores` processes (default: all host cores)."""
    with CpuPool(log_n, levels, cores, batch) as pool:
        done, wall = pool.step(seconds)
        return {"value": done / wall, "cores": pool.cores, "done": done, "wall_s": wall,
                "sample": pool.sample(done, seconds)}

"""Batch-sharded (data-parallel) forms of the hot path, one process per GPU.

Every unit of this path is independent - a ciphertext pair of the ct-mult,
a sample of the encrypted MLP, a noise-monitor trace - so each rank takes a
contiguous shard of the batch (``dist.shard_bounds``), replicates the
context and keys, and computes with no data-path collective.  What remains
is host-side bookkeeping over torch.distributed (NCCL on GPUs, gloo on CPU):

* ``ct_mul_relin_rescale`` - the batched ct-mult of the local shard, outputs
  gathered back in batch order (``dist.gather_rows``) or kept local;
* ``gen_traces``           - each rank generates its share of the gear
  network's training traces with its own seed; the traces are gathered;
* ``fit_loop``             - the data-parallel training loop of the gear
  network: every rank runs the same number of steps on its shard of each
  minibatch and the gradients are averaged by ``dist.allreduce_mean_``
  before the optimiser step, so all ranks hold the same parameters.

Inside one ct-mult the limbs exchange data (basis conversion), but at
N <= 2^13 a pair is far too small to split across GPUs: sharding stops at the
pair.  The reference has no multi-device path (one FPGA,
rtl/m4/e2e_ckks_mult_ctrl_m4.sv:368-482 time-multiplexes its instances).
"""
from __future__ import annotations

from typing import Callable

import numpy as np
import torch

from . import dist as D


def ct_mul_relin_rescale(ctx, ct_a: torch.Tensor, ct_b: torch.Tensor, key_prepared: torch.Tensor,
                         gather: bool = True,
                         compute: Callable[[torch.Tensor, torch.Tensor], torch.Tensor] | None = None
                         ) -> torch.Tensor:
    """ct_a, ct_b [n_ct, 2, level, N], the same full batch on every rank ->
    [n_ct, 2, level - 1, N] on every rank (gather) or this rank's shard of it.
    `compute` replaces the GPU call (the CPU tests pass the oracle)."""
    ws, rank = D.world()
    lo, hi = D.shard_bounds(ct_a.shape[0], ws, rank)
    if compute is None:
        from . import ops

        def compute(a, b):
            return ops.ct_mul_relin_rescale(ctx, a.contiguous(), b.contiguous(), key_prepared)
    out = compute(ct_a[lo:hi], ct_b[lo:hi])
    return D.gather_rows(out) if gather else out


def gen_traces(n_traces: int, seed: int,
               generate: Callable[[int, int], tuple[np.ndarray, np.ndarray]]) -> tuple[np.ndarray, np.ndarray]:
    """This rank's share of n_traces traces, generated by generate(count, seed')
    with a per-rank seed, gathered in rank order on every rank."""
    ws, rank = D.world()
    lo, hi = D.shard_bounds(n_traces, ws, rank)
    X, T = generate(hi - lo, seed * 1_000_003 + rank)
    Xa = D.gather_rows(torch.from_numpy(np.ascontiguousarray(X, dtype=np.float64)))
    Ta = D.gather_rows(torch.from_numpy(np.ascontiguousarray(T, dtype=np.float64)))
    return Xa.numpy(), Ta.numpy()


def fit_loop(n: int, batch: int, epochs: int, rng: np.random.Generator,
             grad_step: Callable[[np.ndarray], tuple[object, int]],
             apply_step: Callable[[object, int, int], None],
             on_epoch: Callable[[int], None] | None = None) -> int:
    """Data-parallel minibatch loop over n training rows, the same on every
    rank.  Each epoch permutes the rows with `rng` (identically seeded on
    every rank), cuts them into minibatches of `batch` rows, and for each
    minibatch gives this rank its contiguous shard: grad_step(rows) returns
    (gradient tensor, row count); the gradients are averaged over ranks
    weighted by row count; apply_step(gradient, step, epoch) updates the
    parameters.  Every rank runs the same steps and collectives in the same
    order.  on_epoch(epoch) runs after each epoch.  Returns the number of
    steps."""
    ws, rank = D.world()
    step = 0
    for ep in range(epochs):
        perm = rng.permutation(n)
        for s in range(0, n - batch + 1, batch):
            rows = perm[s:s + batch]
            lo, hi = D.shard_bounds(batch, ws, rank)
            g, cnt = grad_step(rows[lo:hi])
            D.allreduce_mean_(g, float(cnt))
            step += 1
            apply_step(g, step, ep)
        if on_epoch is not None:
            on_epoch(ep)
    return step

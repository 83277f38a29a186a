"""Multi-process plumbing: one process per GPU over torch.distributed.

The ct-mult path shards by independent units (ciphertext pairs, samples,
traces): each rank takes a contiguous slice of the batch, replicates the
context and keys, and runs with no data-path collective.  The collectives
that remain are host-side bookkeeping:

* ``max_over_ranks``  - step time of a weak-scaling run (the slowest rank);
* ``gather_rows``     - outputs or noise-monitor traces back to every rank
                        (ragged shards padded to the longest);
* ``allreduce_mean_`` - gradient averaging for data-parallel training of the
                        gear network (each rank's traces, one shared model).

The reference has no multi-device path (one FPGA, time-multiplexed instances:
rtl/m4/e2e_ckks_mult_ctrl_m4.sv:368-482).  Works with the ``nccl`` backend on
GPUs and ``gloo`` on CPU.
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def world() -> tuple[int, int]:
    """(world_size, rank); (1, 0) when no process group is initialised."""
    if dist.is_available() and dist.is_initialized():
        return dist.get_world_size(), dist.get_rank()
    return 1, 0


def shard_bounds(n: int, world_size: int, rank: int) -> tuple[int, int]:
    """Contiguous [lo, hi) slice of n units for `rank`; sizes differ by <= 1."""
    if world_size < 1 or not 0 <= rank < world_size or n < 0:
        raise ValueError(f"bad shard request n={n} world={world_size} rank={rank}")
    base, extra = divmod(n, world_size)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def _device() -> torch.device:
    if dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def max_over_ranks(value: float) -> float:
    ws, _ = world()
    if ws == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_rows(x: torch.Tensor) -> torch.Tensor:
    """Concatenate every rank's rows (dim 0) in rank order; shards may differ
    in length."""
    ws, _ = world()
    if ws == 1:
        return x
    dev = _device()
    n = torch.tensor([x.shape[0]], dtype=torch.int64, device=dev)
    sizes = [torch.zeros_like(n) for _ in range(ws)]
    dist.all_gather(sizes, n)
    sizes = [int(s.item()) for s in sizes]
    m = max(sizes)
    pad = torch.zeros((m,) + tuple(x.shape[1:]), dtype=x.dtype, device=dev)
    pad[: x.shape[0]] = x.to(dev)
    parts = [torch.empty_like(pad) for _ in range(ws)]
    dist.all_gather(parts, pad)
    return torch.cat([p[:s] for p, s in zip(parts, sizes)]).to(x.device)


def allreduce_mean_(grad: torch.Tensor, weight: float) -> torch.Tensor:
    """In-place weighted mean over ranks: sum(w_r g_r) / sum(w_r), where w_r
    is e.g. the number of traces behind rank r's gradient."""
    ws, _ = world()
    if ws == 1:
        return grad
    dev = _device()
    buf = torch.cat([(grad.to(dev, torch.float64) * weight).reshape(-1),
                     torch.tensor([float(weight)], dtype=torch.float64, device=dev)])
    dist.all_reduce(buf)
    grad.copy_((buf[:-1] / buf[-1]).reshape(grad.shape).to(grad.device, grad.dtype))
    return grad

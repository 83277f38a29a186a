"""Multi-rank host logic on CPU: two gloo ranks (world size 2) exercise the
sharding, the max-over-ranks step time, the ragged output gather and the
data-parallel gradient average of the gear network (each rank's gradient from
the CPU oracle on its shard must average to the full-batch gradient)."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, errq):
    try:
        sys.path.insert(0, str(ROOT / "cipher-pu_b200"))
        sys.path.insert(0, str(ROOT))
        from ckks_b200 import dist as D
        from oracle import gear_mlp as G
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                                world_size=world)
        assert D.world() == (world, rank)
        # contiguous, disjoint, covering shards
        for n in (0, 1, 5, 256, 4097):
            lo, hi = D.shard_bounds(n, world, rank)
            got = D.gather_rows(torch.tensor([[lo, hi]], dtype=torch.int64))
            spans = got.tolist()
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(spans[i][1] == spans[i + 1][0] for i in range(world - 1))
            assert max(h - l for l, h in spans) - min(h - l for l, h in spans) <= 1
        # slowest rank's time
        assert D.max_over_ranks(1.0 + 1.5 * rank) == 1.0 + 1.5 * (world - 1)
        # ragged gather keeps rank order
        mine = torch.arange(3 * (rank + 2), dtype=torch.float64).reshape(rank + 2, 3) + 100 * rank
        allr = D.gather_rows(mine)
        want = torch.cat([torch.arange(3 * (r + 2), dtype=torch.float64).reshape(r + 2, 3) + 100 * r
                          for r in range(world)])
        assert torch.equal(allr, want)
        # data-parallel gradient of the gear MLP = full-batch gradient
        rng = np.random.default_rng(5)
        p = G.init(3)
        x = rng.standard_normal((37, 16))
        t = rng.standard_normal((37, 4))
        lo, hi = D.shard_bounds(len(x), world, rank)
        g = torch.from_numpy(G.backward(p, x[lo:hi], t[lo:hi]))
        D.allreduce_mean_(g, float(hi - lo))
        assert np.allclose(g.numpy(), G.backward(p, x, t), rtol=1e-12, atol=1e-14)
        dist.barrier()
        dist.destroy_process_group()
    except BaseException as e:  # report to the parent
        errq.put(f"rank {rank}: {type(e).__name__}: {e}")
        raise


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    errq = ctx.SimpleQueue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, errq)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    alive = [p for p in procs if p.is_alive()]
    for p in alive:
        p.kill()
    errs = []
    while not errq.empty():
        errs.append(errq.get())
    assert not alive, "a rank did not finish"
    assert not errs, errs
    assert all(p.exitcode == 0 for p in procs)


def test_shard_bounds_rejects_bad_requests():
    sys.path.insert(0, str(ROOT / "cipher-pu_b200"))
    from ckks_b200.dist import shard_bounds
    with pytest.raises(ValueError):
        shard_bounds(10, 0, 0)
    with pytest.raises(ValueError):
        shard_bounds(10, 2, 2)
    assert shard_bounds(10, 3, 0) == (0, 4) and shard_bounds(10, 3, 2) == (7, 10)

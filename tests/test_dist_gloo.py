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
        _sharded_paths(world, rank)
        dist.barrier()
        dist.destroy_process_group()
    except BaseException as e:  # report to the parent
        errq.put(f"rank {rank}: {type(e).__name__}: {e}")
        raise


def _sharded_paths(world: int, rank: int):
    """The product's sharded paths (ckks_b200.sharded) with the CPU oracle as
    the per-rank compute, against the single-rank result."""
    from ckks_b200 import sharded as S
    from oracle import gear_mlp as G
    from oracle import rns_ckks as R
    from oracle.modmath import find_primes
    # batch-sharded ct-mult + relin + rescale, gathered in batch order
    n, level = 64, 2
    pr = find_primes(40, 2 * n, level + 1)
    special, qs = pr[0], pr[1:]
    rng = np.random.default_rng(11)                      # same batch on every rank

    def rnd(shape, basis):
        x = np.zeros(shape, dtype=np.uint64)
        for i, q in enumerate(basis):
            x[..., i, :] = rng.integers(0, q, size=x[..., i, :].shape, dtype=np.uint64)
        return x
    a = rnd((5, 2, level, n), qs)
    b = rnd((5, 2, level, n), qs)
    ksk = rnd((level, 2, level + 1, n), qs + [special])
    calls = []

    def oracle_compute(x, y):
        calls.append(x.shape[0])
        return torch.from_numpy(R.ct_mul_relin_rescale(x.numpy(), y.numpy(), ksk, qs, special).view(np.int64))
    got = S.ct_mul_relin_rescale(None, torch.from_numpy(a.view(np.int64)), torch.from_numpy(b.view(np.int64)),
                                 None, compute=oracle_compute)
    assert calls == [3 if rank == 0 else 2]              # this rank's shard only
    want = R.ct_mul_relin_rescale(a, b, ksk, qs, special)
    assert np.array_equal(got.numpy().view(np.uint64), want)
    local = S.ct_mul_relin_rescale(None, torch.from_numpy(a.view(np.int64)), torch.from_numpy(b.view(np.int64)),
                                   None, gather=False, compute=oracle_compute)
    lo, hi = (0, 3) if rank == 0 else (3, 5)
    assert np.array_equal(local.numpy().view(np.uint64), want[lo:hi])

    # sharded trace generation: per-rank seeds, gathered in rank order
    def gen(count, seed):
        r = np.random.default_rng(seed)
        return r.standard_normal((count, 16)), r.standard_normal((count, 4))
    X, T = S.gen_traces(9, 4, gen)
    parts = [gen(hi - lo, 4 * 1_000_003 + r) for r, (lo, hi) in
             enumerate([(0, 5), (5, 9)])]
    assert np.array_equal(X, np.concatenate([p[0] for p in parts]))
    assert np.array_equal(T, np.concatenate([p[1] for p in parts]))

    # data-parallel training loop: 2 ranks, gradients averaged per minibatch,
    # against one process taking the whole minibatch
    Xt, Tt = np.random.default_rng(12).standard_normal((70, 16)), np.random.default_rng(13).standard_normal((70, 4))

    def train(distributed: bool):
        p = G.init(2)
        m = np.zeros_like(p)
        v = np.zeros_like(p)

        def grad_step(rows):
            return torch.from_numpy(G.backward(p, Xt[rows], Tt[rows])), len(rows)

        def grad_step_full(rows):
            return torch.from_numpy(G.backward(p, Xt[rows], Tt[rows])), len(rows)

        def apply_step(g, step, ep):
            nonlocal m, v
            g = g.numpy()
            m = 0.9 * m + 0.1 * g
            v = 0.999 * v + 0.001 * g * g
            p[:] = p - 1e-2 * (m / (1 - 0.9 ** step)) / (np.sqrt(v / (1 - 0.999 ** step)) + 1e-8)
        if distributed:
            steps = S.fit_loop(len(Xt), 16, 3, np.random.default_rng(14), grad_step, apply_step)
        else:
            rng = np.random.default_rng(14)
            steps = 0
            for ep in range(3):
                perm = rng.permutation(len(Xt))
                for s0 in range(0, len(Xt) - 16 + 1, 16):
                    g, _ = grad_step_full(perm[s0:s0 + 16])
                    steps += 1
                    apply_step(g, steps, ep)
        return p, steps
    p_dp, steps_dp = train(True)
    p_one, steps_one = train(False)
    assert steps_dp == steps_one == 3 * (70 // 16)
    assert np.allclose(p_dp, p_one, rtol=1e-9, atol=1e-11)


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

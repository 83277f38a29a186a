"""Batched uneven workload (mixed N, levels 2..8, ct x ct and ct x pt) in
one CUDA graph: bit-exact vs the oracle per bucket, graph replay == eager,
autotuned launch shapes give the same results."""
import numpy as np
import pytest

from oracle import rns_ckks as R
from oracle.modmath import mulmod

pytestmark = pytest.mark.gpu


def _np(t):
    import torch
    return t.contiguous().view(torch.int64).cpu().numpy().astype(np.uint64)


def test_ct_mul_plain_rescale_vs_oracle(cuda):
    import torch
    from ckks_b200 import _lib
    from ckks_b200.evaluator import Evaluator
    from ckks_b200.params import CkksParams
    ev = Evaluator(CkksParams.standard(12, 5, seed=1))
    ev.keygen()
    for level, per_ct in ((5, 1), (2, 0)):
        ct = ev.uniform(6, level).reshape(3, 2, level, ev.n)
        pt = ev.uniform(3 if per_ct else 1, level)
        out = torch.empty((3, 2, level - 1, ev.n), dtype=torch.uint64, device="cuda")
        _lib.call("ckks_ct_mul_plain_rescale", ev.ctx.handle, out.data_ptr(), ct.data_ptr(), pt.data_ptr(),
                  per_ct, 3, level, torch.cuda.current_stream().cuda_stream)
        qs = list(ev.params.q[:level])
        a = _np(ct)
        p = _np(pt)
        prod = np.stack([mulmod(a[:, k], (p if per_ct else np.broadcast_to(p, (3,) + p.shape[1:])),
                                np.asarray(qs, dtype=np.uint64)[:, None]) for k in range(2)], axis=1)
        assert np.array_equal(_np(out), R.rescale(prod, qs))


def test_batched_uneven_graph(cuda):
    import torch
    from ckks_b200.batch import BatchExecutor, synthetic_workload
    items = synthetic_workload(96, seed=3)
    ex = BatchExecutor(items, max_level=8)
    ex.run_eager()
    torch.cuda.synchronize()
    eager = [_np(b.out) for b in ex.buckets]
    for b in ex.buckets:
        b.out.zero_()
    ex.capture()
    ex.step()
    torch.cuda.synchronize()
    assert all(np.array_equal(_np(b.out), e) for b, e in zip(ex.buckets, eager))
    # one item of every bucket against the oracle
    for bk, e in zip(ex.buckets, eager):
        ev = ex.evs[bk.shape.log_n]
        qs = list(ev.params.q[:bk.shape.level])
        a = _np(bk.a[:1])
        if bk.shape.op == "ctct":
            ksk = _np(ev.ksk)
            sub = ksk[:bk.shape.level][:, :, list(range(bk.shape.level)) + [ev.params.levels]]
            want = R.ct_mul_relin_rescale(a, _np(bk.b[:1]), sub, qs, ev.params.special)
        else:
            p = _np(bk.b[:1])
            prod = np.stack([mulmod(a[:, k], p, np.asarray(qs, dtype=np.uint64)[:, None]) for k in range(2)], 1)
            want = R.rescale(prod, qs)
        assert np.array_equal(e[:1], want), bk.shape
    # autotuned shapes are result-identical
    ex.autotune(reps=1)
    for b in ex.buckets:
        b.out.zero_()
    ex.step()
    torch.cuda.synchronize()
    assert all(np.array_equal(_np(b.out), e) for b, e in zip(ex.buckets, eager))

"""The persistent batch kernel (ckks_batch_plan_*): one launch drains a work
list of mixed-N, mixed-level ct x ct and ct x pt work units with per-item
dependency counters; N = 2^13 units take a whole 512-thread CTA, N = 2^12
units run in its halves (phased list: each half takes its own units after
the 2^13 phase; paired list: two per slot, side by side).  Both lists' outputs are bit-identical to
the eager per-bucket path (integer results: tolerance zero) under every lag,
for one ring size or both, inside a CUDA graph too; a wait that nothing
satisfies ends at its limit with CKKS_ETIMEOUT and the unfinished items
reported incomplete."""
import numpy as np
import pytest

from oracle import rns_ckks as R
from oracle.modmath import mulmod

pytestmark = pytest.mark.gpu

ETIMEOUT = -2


def _np(t):
    import torch
    return t.contiguous().view(torch.int64).cpu().numpy().astype(np.uint64)


def _executor(n_items, seed, **kw):
    import torch
    from ckks_b200.batch import BatchExecutor, synthetic_workload
    ex = BatchExecutor(synthetic_workload(n_items, seed=seed, **kw), max_level=8)
    ex.run_eager()
    torch.cuda.synchronize()
    return ex, [b.out.clone() for b in ex.buckets]


def _same(ex, ref):
    import torch
    return [bool(torch.equal(b.out, r)) for b, r in zip(ex.buckets, ref)]


def _clear(ex):
    import torch
    for b in ex.buckets:
        b.out.fill_(0xABCD)
    torch.cuda.synchronize()


@pytest.fixture(scope="module")
def mixed(cuda):
    return _executor(160, seed=5)


def test_persistent_equals_eager_and_oracle(mixed):
    import torch
    from ckks_b200 import _lib
    from ckks_b200.batch import PersistentPlan
    ex, ref = mixed
    plan = PersistentPlan(ex.evs, ex.buckets)
    info = plan.info()
    assert info["units"] == sum(b.count * ((2 * b.shape.level + 3) if b.shape.op == "ctct" else 2)
                                for b in ex.buckets)
    units13 = sum(b.count * ((2 * b.shape.level + 3) if b.shape.op == "ctct" else 2)
                  for b in ex.buckets if b.shape.log_n == 13)
    # paired list (the default): every 2^13 unit alone, the 2^12 units two by
    # two (at most one alone); the phased list gives every unit its own slot
    assert info["slots"] - units13 == (info["units"] - units13 + 1) // 2 and info["list"] == "paired"
    assert {b.shape.log_n for b in ex.buckets} == {12, 13}
    for paired in (True, False):
        plan.paired = paired
        _clear(ex)
        plan.run()
        torch.cuda.synchronize()
        assert _lib.load().ckks_device_status() == 0
        assert plan.incomplete() == (0, [True] * len(ex.buckets))
        assert all(_same(ex, ref)), paired
    # the last item of a few buckets against the oracle
    for bk in [b for b in ex.buckets if b.count][::7]:
        ev = ex.evs[bk.shape.log_n]
        L = bk.shape.level
        qs = list(ev.params.q[:L])
        a = _np(bk.a[-1:])
        if bk.shape.op == "ctct":
            ksk = _np(ev.ksk)
            sub = ksk[:L][:, :, list(range(L)) + [ev.params.levels]]
            want = R.ct_mul_relin_rescale(a, _np(bk.b[-1:]), sub, qs, ev.params.special)
        else:
            p = _np(bk.b[-1:])
            prod = np.stack([mulmod(a[:, k], p, np.asarray(qs, dtype=np.uint64)[:, None]) for k in range(2)], 1)
            want = R.rescale(prod, qs)
        assert np.array_equal(_np(bk.out[-1:]), want), bk.shape
    plan.close()


@pytest.mark.parametrize("paired", [False, True])
@pytest.mark.parametrize("lag", [0, 100, 10000])
def test_persistent_any_lag_same_results(mixed, lag, paired):
    """lag 0 lists each dependent stage right after its producers (most
    units wait), 10000 only after every other unit (the work list degenerates
    to stage order): the same bits either way, on either unit list."""
    import torch
    from ckks_b200.batch import PersistentPlan
    ex, ref = mixed
    plan = PersistentPlan(ex.evs, ex.buckets, lag_percent=lag)
    plan.paired = paired
    _clear(ex)
    plan.run()
    torch.cuda.synchronize()
    assert plan.incomplete()[0] == 0
    assert all(_same(ex, ref))
    plan.close()


def test_persistent_graph_replay(mixed):
    """Captured as one memset node and one kernel node; replays reset the
    counters and give the same bits each time."""
    import torch
    ex, ref = mixed
    ex.mode = "persistent"
    try:
        ex.persistent_plan(400)
        _clear(ex)
        ex.capture()
        for _ in range(3):
            ex.step()
        torch.cuda.synchronize()
        assert all(_same(ex, ref))
        assert ex.plan.incomplete()[0] == 0
    finally:
        ex.mode = "streams"


@pytest.mark.parametrize("log_n", [12, 13])
def test_persistent_one_ring_size(cuda, log_n):
    """Plans of one ring size: N = 2^12 only (every slot two half-CTA units,
    the 2^12-only kernel build) and N = 2^13 only (whole-CTA units)."""
    import torch
    from ckks_b200.batch import PersistentPlan
    ex, ref = _executor(64, seed=6 + log_n, log_ns=(log_n,))
    for lag in (0, 400):
        plan = PersistentPlan(ex.evs, ex.buckets, lag_percent=lag)
        for paired in (False, True):
            plan.paired = paired
            _clear(ex)
            plan.run()
            torch.cuda.synchronize()
            assert plan.incomplete()[0] == 0
            assert all(_same(ex, ref)), (lag, paired)
        plan.close()


def test_unmet_wait_times_out_and_reports_incomplete(mixed):
    """The test hook makes the ModUp units of the first ct x ct item wait for
    a tensor unit that does not exist.  The wait ends at its limit (a kernel
    argument, here 2e5 cycles), the launch stops, ckks_device_status reports
    CKKS_ETIMEOUT once, and that item (at least) is reported incomplete.  The
    next normal run is complete and exact."""
    import torch
    from ckks_b200 import _lib
    from ckks_b200.batch import PersistentPlan
    ex, ref = mixed
    lib = _lib.load()
    plan = PersistentPlan(ex.evs, ex.buckets)
    torch.cuda.synchronize()
    assert lib.ckks_device_status() == 0
    _clear(ex)
    plan.run(wait_cycles=200_000, flags=_lib.BATCH_RUN_UNMET_WAIT)
    torch.cuda.synchronize()
    assert lib.ckks_device_status() == ETIMEOUT
    assert lib.ckks_device_status() == 0           # read and cleared
    n_bad, complete = plan.incomplete()
    first_ctct = next(i for i, b in enumerate(ex.buckets) if b.shape.op == "ctct" and b.count)
    assert n_bad >= 1 and not complete[first_ctct]
    # the finished items are exact even in the aborted run
    done = [i for i, c in enumerate(complete) if c]
    same = _same(ex, ref)
    assert all(same[i] for i in done)
    plan.run()
    torch.cuda.synchronize()
    assert lib.ckks_device_status() == 0
    assert plan.incomplete()[0] == 0
    assert all(_same(ex, ref))
    plan.close()


def test_plan_refusals(cuda):
    import ctypes
    from ckks_b200 import _lib
    from ckks_b200._lib import CkksError
    from ckks_b200.context import Context
    from ckks_b200.params import CkksParams
    h = ctypes.c_void_p()
    # empty plan: valid, runs nothing
    _lib.call("ckks_batch_plan_create", None, 0, 200, ctypes.byref(h))
    _lib.call("ckks_batch_plan_run", h, 0, 0, None)
    _lib.raw("ckks_batch_plan_destroy")(h)
    P11 = CkksParams.standard(11, 3)
    ctx11 = Context.get(11, P11.primes, n_special=1)
    arr = (_lib.BatchBucket * 1)()
    arr[0] = _lib.BatchBucket(ctx11.handle, _lib.BATCH_CT_PT, 1, 3, 1, 16, 16, 16, None)
    with pytest.raises(CkksError, match="built for 12 and 13"):
        _lib.call("ckks_batch_plan_create", arr, 1, 200, ctypes.byref(h))
    P12 = CkksParams.standard(12, 3)
    ctx12 = Context.get(12, P12.primes, n_special=1)
    arr[0] = _lib.BatchBucket(ctx12.handle, _lib.BATCH_CT_PT, 1, 4, 1, 16, 16, 16, None)
    with pytest.raises(CkksError, match="level=4"):
        _lib.call("ckks_batch_plan_create", arr, 1, 200, ctypes.byref(h))
    arr[0] = _lib.BatchBucket(ctx12.handle, _lib.BATCH_CT_CT, 1, 3, 0, 16, 16, 16, None)
    with pytest.raises(CkksError, match="NULL"):
        _lib.call("ckks_batch_plan_create", arr, 1, 200, ctypes.byref(h))
    with pytest.raises(CkksError, match="n_buckets"):
        _lib.call("ckks_batch_plan_create", arr, 129, 200, ctypes.byref(h))

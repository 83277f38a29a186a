"""The persistent batch plan's work list, computed on the host
(ckks_batch_schedule, no GPU): every work unit listed exactly once, every
unit after the units it depends on, dependent stages at least `lag` units
after their producers wherever independent work was left to fill the gap,
and the costliest buckets' pairs first."""
import ctypes as C

import numpy as np
import pytest

CT_CT, CT_PT = 0, 1
TENSOR, MODUP, DOWN, CTPT = 0, 1, 2, 3


def _schedule(ops, cts, lvls, costs, lag):
    from ckks_b200 import _lib
    nb = len(ops)
    total = sum(c * (2 * l + 3 if o == CT_CT else 2) for o, c, l in zip(ops, cts, lvls))
    jobs = np.zeros((max(1, total), 2), dtype=np.uint32)
    n = C.c_longlong(total)
    a = lambda v, t: np.ascontiguousarray(np.asarray(v, dtype=t))
    o, c, l, w = a(ops, np.int32), a(cts, np.int32), a(lvls, np.int32), a(costs, np.float64)
    _lib.call("ckks_batch_schedule", nb, o.ctypes.data, c.ctypes.data, l.ctypes.data, w.ctypes.data, lag,
              jobs.ctypes.data, C.byref(n))
    assert n.value == total
    x = jobs[:total, 0].astype(np.int64)
    return np.stack([x >> 8, (x >> 6) & 3, x & 63, jobs[:total, 1].astype(np.int64)], 1)


def _check(ops, cts, lvls, costs, lag):
    J = _schedule(ops, cts, lvls, costs, lag)
    seen = {}
    for pos, (b, st, sub, it) in enumerate(J.tolist()):
        key = (b, st, sub, it)
        assert key not in seen, key
        seen[key] = pos
    # exactly the expected unit set
    want = set()
    for b, (o, c, l) in enumerate(zip(ops, cts, lvls)):
        for it in range(c):
            if o == CT_CT:
                want |= {(b, TENSOR, j, it) for j in range(l)}
                want |= {(b, MODUP, t, it) for t in range(l + 1)}
                want |= {(b, DOWN, k, it) for k in range(2)}
            else:
                want |= {(b, CTPT, k, it) for k in range(2)}
    assert set(seen) == want
    gaps = []
    for b, (o, c, l) in enumerate(zip(ops, cts, lvls)):
        if o != CT_CT:
            continue
        for it in range(c):
            last_t = max(seen[(b, TENSOR, j, it)] for j in range(l))
            first_m = min(seen[(b, MODUP, t, it)] for t in range(l + 1))
            last_m = max(seen[(b, MODUP, t, it)] for t in range(l + 1))
            first_d = min(seen[(b, DOWN, k, it)] for k in range(2))
            assert last_t < first_m and last_m < first_d
            gaps += [first_m - last_t - 1, first_d - last_m - 1]
    return J, seen, gaps


def test_schedule_mixed_workload():
    rng = np.random.default_rng(1)
    ops, cts, lvls, costs = [], [], [], []
    for op in (CT_CT, CT_PT):
        for log_n in (12, 13):
            for lvl in range(2, 9):
                ops.append(op)
                cts.append(int(rng.integers(0, 60)))
                lvls.append(lvl)
                costs.append(float((1 << log_n) * (2 * lvl + 3)))
    lag = 296
    J, seen, gaps = _check(ops, cts, lvls, costs, lag)
    # with ct x pt filler to spare, every dependent stage keeps the full lag
    # except in the tail, where only pending stages remain
    n = len(gaps)
    assert sum(g >= lag for g in gaps) >= 0.9 * n
    # the costliest ct x ct bucket's first pair comes first
    first = J[0]
    cm = [b for b, o in enumerate(ops) if o == CT_CT and cts[b]]
    assert first[0] == max(cm, key=lambda b: (costs[b], -b))


@pytest.mark.parametrize("lag", [0, 1, 7, 10 ** 6])
def test_schedule_lag_extremes(lag):
    _, _, gaps = _check([CT_CT, CT_PT, CT_CT], [5, 3, 4], [3, 2, 8], [1.0, 1.0, 2.0], lag)
    if lag == 0:
        # with no lag every pair's stages follow each other directly
        assert max(gaps) == 0


def test_schedule_empty_and_refusals():
    from ckks_b200 import _lib
    from ckks_b200._lib import CkksError
    n = C.c_longlong(0)
    _lib.call("ckks_batch_schedule", 0, None, None, None, None, 0, None, C.byref(n))
    assert n.value == 0
    _check([CT_CT, CT_PT], [0, 0], [2, 2], [1.0, 1.0], 10)
    o = np.asarray([CT_CT], dtype=np.int32)
    c = np.asarray([4], dtype=np.int32)
    l = np.asarray([3], dtype=np.int32)
    w = np.asarray([1.0])
    jobs = np.zeros((10, 2), dtype=np.uint32)
    n = C.c_longlong(10)
    with pytest.raises(CkksError, match="capacity"):
        _lib.call("ckks_batch_schedule", 1, o.ctypes.data, c.ctypes.data, l.ctypes.data, w.ctypes.data, 0,
                  jobs.ctypes.data, C.byref(n))
    l[0] = 1
    n = C.c_longlong(100)
    with pytest.raises(CkksError, match="level=1"):
        _lib.call("ckks_batch_schedule", 1, o.ctypes.data, c.ctypes.data, l.ctypes.data, w.ctypes.data, 0,
                  jobs.ctypes.data, C.byref(n))

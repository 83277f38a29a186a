"""The persistent batch plan's work list, computed on the host
(ckks_batch_schedule, no GPU): every work unit listed exactly once, every
unit after the units it depends on (or beside it in the same slot),
dependent stages at least `lag` units after their producers wherever
independent work was left to fill the gap, the costliest buckets' pairs
first, and slots of one N = 2^13 unit or two N = 2^12 units."""
import ctypes as C

import numpy as np
import pytest

CT_CT, CT_PT = 0, 1
TENSOR, MODUP, DOWN, CTPT = 0, 1, 2, 3


NONE = 0xFFFFFFFF


def _schedule(ops, cts, lvls, costs, lag, log_ns=None):
    """-> (units [n, 4]: bucket, stage, sub, item in list order; slot index of each unit)."""
    from ckks_b200 import _lib
    nb = len(ops)
    log_ns = log_ns or [12] * nb
    total = sum(c * (2 * l + 3 if o == CT_CT else 2) for o, c, l in zip(ops, cts, lvls))
    slots = np.zeros((max(1, total), 4), dtype=np.uint32)
    n = C.c_longlong(total)
    a = lambda v, t: np.ascontiguousarray(np.asarray(v, dtype=t))
    o, c, l, g, w = (a(ops, np.int32), a(cts, np.int32), a(lvls, np.int32), a(log_ns, np.int32),
                     a(costs, np.float64))
    _lib.call("ckks_batch_schedule", nb, o.ctypes.data, c.ctypes.data, l.ctypes.data, g.ctypes.data,
              w.ctypes.data, lag, slots.ctypes.data, C.byref(n))
    units, where = [], []
    for si, (x0, y0, x1, y1) in enumerate(slots[:n.value].tolist()):
        b0 = x0 >> 8
        if log_ns[b0] == 13:
            assert x1 == NONE                       # a 2^13 unit takes the whole CTA
        for x, y in ((x0, y0), (x1, y1)):
            if x == NONE:
                continue
            assert log_ns[x >> 8] == (13 if log_ns[b0] == 13 else 12)
            units.append((x >> 8, (x >> 6) & 3, x & 63, y))
            where.append(si)
    assert len(units) == total
    return np.asarray(units, dtype=np.int64).reshape(-1, 4), where


def _check(ops, cts, lvls, costs, lag, log_ns=None):
    J, where = _schedule(ops, cts, lvls, costs, lag, log_ns)
    seen, slot = {}, {}
    for pos, (b, st, sub, it) in enumerate(J.tolist()):
        key = (b, st, sub, it)
        assert key not in seen, key
        seen[key] = pos
        slot[key] = where[pos]
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
            # in slot order too: a consumer never in an earlier slot than a producer
            assert max(slot[(b, TENSOR, j, it)] for j in range(l)) <= min(slot[(b, MODUP, t, it)] for t in range(l + 1))
            assert max(slot[(b, MODUP, t, it)] for t in range(l + 1)) <= min(slot[(b, DOWN, k, it)] for k in range(2))
            gaps += [first_m - last_t - 1, first_d - last_m - 1]
    return J, seen, gaps


def test_schedule_mixed_workload():
    rng = np.random.default_rng(1)
    ops, cts, lvls, costs, logs = [], [], [], [], []
    for op in (CT_CT, CT_PT):
        for log_n in (12, 13):
            for lvl in range(2, 9):
                ops.append(op)
                cts.append(int(rng.integers(0, 60)))
                lvls.append(lvl)
                logs.append(log_n)
                costs.append(float((1 << log_n) * (2 * lvl + 3)))
    lag = 296
    J, seen, gaps = _check(ops, cts, lvls, costs, lag, logs)
    # with ct x pt filler to spare, every dependent stage keeps the full lag
    # except in the tail, where only pending stages remain
    n = len(gaps)
    assert sum(g >= lag for g in gaps) >= 0.9 * n
    # the costliest ct x ct bucket's first pair comes first
    first = J[0]
    cm = [b for b, o in enumerate(ops) if o == CT_CT and cts[b]]
    assert first[0] == max(cm, key=lambda b: (costs[b], -b))


@pytest.mark.parametrize("lag", [0, 1, 7, 10 ** 6])
@pytest.mark.parametrize("logs", [[12, 12, 12], [13, 13, 13], [12, 13, 12], [13, 12, 13]])
def test_schedule_lag_extremes(lag, logs):
    _, _, gaps = _check([CT_CT, CT_PT, CT_CT], [5, 3, 4], [3, 2, 8], [1.0, 1.0, 2.0], lag, logs)
    if lag == 0:
        # with no lag every pair's stages follow each other directly (pairs
        # go in two at a time, interleaved: at most the partner's unit between)
        assert max(gaps) <= 1


def test_schedule_empty_and_refusals():
    from ckks_b200 import _lib
    from ckks_b200._lib import CkksError
    n = C.c_longlong(0)
    _lib.call("ckks_batch_schedule", 0, None, None, None, None, None, 0, None, C.byref(n))
    assert n.value == 0
    _check([CT_CT, CT_PT], [0, 0], [2, 2], [1.0, 1.0], 10)
    o = np.asarray([CT_CT], dtype=np.int32)
    c = np.asarray([4], dtype=np.int32)
    l = np.asarray([3], dtype=np.int32)
    g = np.asarray([12], dtype=np.int32)
    w = np.asarray([1.0])
    slots = np.zeros((100, 4), dtype=np.uint32)

    def call(cap):
        n = C.c_longlong(cap)
        _lib.call("ckks_batch_schedule", 1, o.ctypes.data, c.ctypes.data, l.ctypes.data, g.ctypes.data,
                  w.ctypes.data, 0, slots.ctypes.data, C.byref(n))
        return n.value
    with pytest.raises(CkksError, match="capacity"):
        call(10)
    assert call(36) == 18                     # 4 pairs x 9 units, two per slot
    g[0] = 11
    with pytest.raises(CkksError, match="log_n=11"):
        call(100)
    g[0] = 12
    l[0] = 1
    with pytest.raises(CkksError, match="level=1"):
        call(100)


def _phased(ops, cts, lvls, costs, lag, log_ns):
    from ckks_b200 import _lib
    nb = len(ops)
    total = sum(c * (2 * l + 3 if o == CT_CT else 2) for o, c, l in zip(ops, cts, lvls))
    slots = np.zeros((max(1, total), 4), dtype=np.uint32)
    n, whole = C.c_longlong(total), C.c_longlong(-1)
    a = lambda v, t: np.ascontiguousarray(np.asarray(v, dtype=t))
    o, c, l, g, w = (a(ops, np.int32), a(cts, np.int32), a(lvls, np.int32), a(log_ns, np.int32),
                     a(costs, np.float64))
    _lib.call("ckks_batch_schedule_phased", nb, o.ctypes.data, c.ctypes.data, l.ctypes.data, g.ctypes.data,
              w.ctypes.data, lag, slots.ctypes.data, C.byref(n), C.byref(whole))
    return slots[:n.value], whole.value, total


@pytest.mark.parametrize("lag", [0, 5, 296])
def test_phased_schedule(lag):
    """The plan's default list: every unit once in a slot of its own, the
    N = 2^13 units first (whole-CTA slots), then the N = 2^12 units (half
    slots); within each phase every unit after its producers, and with ct x pt
    filler to spare the dependent stages keep `lag` (whole) / 2 lag (half)
    units of distance."""
    rng = np.random.default_rng(2)
    ops, cts, lvls, costs, logs = [], [], [], [], []
    for op in (CT_CT, CT_PT):
        for log_n in (12, 13):
            for lvl in range(2, 9):
                ops.append(op)
                cts.append(int(rng.integers(0, 40)))
                lvls.append(lvl)
                logs.append(log_n)
                costs.append(float((1 << log_n) * (2 * lvl + 3)))
    slots, whole, total = _phased(ops, cts, lvls, costs, lag, logs)
    assert len(slots) == total
    assert all(int(x1) == NONE for x1 in slots[:, 2])
    sizes = [logs[int(x) >> 8] for x in slots[:, 0]]
    assert sizes == [13] * whole + [12] * (total - whole)
    assert whole == sum(c * (2 * l + 3 if o == CT_CT else 2)
                        for o, c, l, g in zip(ops, cts, lvls, logs) if g == 13)
    pos = {}
    for i, (x, y) in enumerate(zip(slots[:, 0].tolist(), slots[:, 1].tolist())):
        key = (x >> 8, (x >> 6) & 3, x & 63, y)
        assert key not in pos
        pos[key] = i
    gaps = []
    for b, (o, c, l, g) in enumerate(zip(ops, cts, lvls, logs)):
        if o != CT_CT:
            continue
        for it in range(c):
            last_t = max(pos[(b, TENSOR, j, it)] for j in range(l))
            mods = [pos[(b, MODUP, t, it)] for t in range(l + 1)]
            downs = [pos[(b, DOWN, k, it)] for k in range(2)]
            assert last_t < min(mods) and max(mods) < min(downs)
            need = lag if g == 13 else 2 * lag
            gaps += [min(mods) - last_t - 1 >= need, min(downs) - max(mods) - 1 >= need]
    if lag:
        assert sum(gaps) >= 0.8 * len(gaps)

"""Every per-thread radix 2^K (K = 2..5) the autotuner can pick gives the
same bit-exact results: the standalone transform against the oracle, ct x ct
+ relin + rescale, ct x pt + rescale and the key-switched rotation against
the default launch shape (itself checked against the oracle)."""
import numpy as np
import pytest

from oracle import galois as GA
from oracle import rns_ckks as R
from oracle.modmath import mulmod

pytestmark = pytest.mark.gpu

# ckks_ctx_set_tuning parameters
CM_K, CM_MINB, CM_SPLIT, NTT_K, CM_UPC, CM_TMA = 0, 1, 2, 3, 4, 5
CM_FUSED = 7  # 0 = fused kernel where built (default), 2 = the three-kernel path these shapes tune
CM_TMEM = 8   # ModUp accumulators: 1 = TMEM (default where built: N = 2^12, K = 4), 2 = shared memory


def _rand(rng, shape, basis):
    x = np.zeros(shape, dtype=np.uint64)
    for i, q in enumerate(basis):
        x[..., i, :] = rng.integers(0, q, size=x[..., i, :].shape, dtype=np.uint64)
    return x


@pytest.fixture(scope="module")
def ck(cuda):
    import ckks_b200.ops as ops
    from ckks_b200 import _lib
    from ckks_b200.context import Context
    return ops, _lib, Context


def _reset(_lib, ctx):
    for p in (CM_K, CM_MINB, CM_SPLIT, NTT_K, CM_UPC, CM_TMA, CM_FUSED, CM_TMEM):
        _lib.call("ckks_ctx_set_tuning", ctx.handle, p, 0)


def _three_kernels(_lib, ctx):
    """Route ct-mults through the three-kernel path, whose launch shapes the
    tests sweep (the default fused kernel has one shape)."""
    _lib.call("ckks_ctx_set_tuning", ctx.handle, CM_FUSED, 2)


@pytest.mark.parametrize("log_n", [6, 10, 12, 13])
def test_ntt_every_radix_matches_oracle(ck, log_n):
    ops, _lib, Context = ck
    from ckks_b200.params import chain_primes
    n = 1 << log_n
    primes = list(chain_primes(3, 14))
    ctx = Context.get(log_n, primes)
    rng = np.random.default_rng(700 + log_n)
    x = np.stack([rng.integers(0, q, size=n, dtype=np.uint64) for q in primes])[None].repeat(2, 0)
    x[1, :, :2] = 0
    want = R.ntt_limbs(x, primes)
    cyc_ref = None
    try:
        for k in (0, 2, 3, 4, 5):
            if k and (n >> k) > 1024:
                continue
            _lib.call("ckks_ctx_set_tuning", ctx.handle, NTT_K, k)
            d = ops.to_device(x)
            ops.ntt(ctx, d)
            assert np.array_equal(ops.to_host(d), want), f"forward K={k}"
            ops.ntt(ctx, d, inverse=True)
            assert np.array_equal(ops.to_host(d), x), f"inverse K={k}"
            c = ops.to_device(x)
            ops.ntt(ctx, c, cyclic=True)
            got_c = ops.to_host(c)
            if cyc_ref is None:
                cyc_ref = got_c
            assert np.array_equal(got_c, cyc_ref), f"cyclic K={k}"
            ops.ntt(ctx, c, cyclic=True, inverse=True)
            assert np.array_equal(ops.to_host(c), x), f"cyclic inverse K={k}"
    finally:
        _reset(_lib, ctx)


def _cm_shapes(log_n):
    from ckks_b200.batch import RADIX_LOG2, cm_shape_built
    return [(k, mb) for k in RADIX_LOG2 for mb in (1, 2) if cm_shape_built(log_n, k, mb)]


@pytest.mark.parametrize("log_n,n_ct", [(12, 40), (13, 6), (10, 9)])
def test_ct_mul_every_launch_shape_identical(ck, log_n, n_ct):
    ops, _lib, Context = ck
    from ckks_b200.params import CkksParams
    P = CkksParams.standard(log_n, 3)
    ctx = Context.get(log_n, P.primes, n_special=1)
    qs = list(P.q)
    n = 1 << log_n
    rng = np.random.default_rng(log_n * 31 + n_ct)
    a = _rand(rng, (n_ct, 2, 3, n), qs)
    b = _rand(rng, (n_ct, 2, 3, n), qs)
    ksk = _rand(rng, (3, 2, 4, n), qs + [P.special])
    key = ops.relin_key_prepare(ctx, ops.to_device(ksk))
    da, db = ops.to_device(a), ops.to_device(b)
    base = ops.to_host(ops.ct_mul_relin_rescale(ctx, da, db, key))
    assert np.array_equal(base[:2], R.ct_mul_relin_rescale(a[:2], b[:2], ksk, qs, P.special))
    shapes = _cm_shapes(log_n)
    assert {k for k, _ in shapes} >= {3, 4, 5}
    try:
        _three_kernels(_lib, ctx)
        for k, mb in shapes:
            _lib.call("ckks_ctx_set_tuning", ctx.handle, CM_K, k)
            _lib.call("ckks_ctx_set_tuning", ctx.handle, CM_MINB, mb)
            got = ops.to_host(ops.ct_mul_relin_rescale(ctx, da, db, key))
            assert np.array_equal(got, base), f"K={k} budget={mb}"
            # level 2 (one limb less) through the same shape
            got2 = ops.to_host(ops.ct_mul_relin_rescale(ctx, da[:, :, :2].contiguous(),
                                                        db[:, :, :2].contiguous(), key))
            if k == shapes[0][0] and mb == shapes[0][1]:
                ref2 = got2
            assert np.array_equal(got2, ref2), f"level 2 K={k} budget={mb}"
    finally:
        _reset(_lib, ctx)
    assert np.array_equal(ref2[:1], R.ct_mul_relin_rescale(a[:1, :, :2], b[:1, :, :2],
                                                          ksk[:2][:, :, [0, 1, 3]], qs[:2], P.special))


def test_rotate_every_launch_shape_identical(ck):
    ops, _lib, Context = ck
    from ckks_b200.params import CkksParams
    P = CkksParams.standard(12, 3)
    ctx = Context.get(12, P.primes, n_special=1)
    qs = list(P.q)
    rng = np.random.default_rng(4242)
    ct = _rand(rng, (5, 2, 3, 4096), qs)
    gk = _rand(rng, (3, 2, 4, 4096), qs + [P.special])
    key = ops.relin_key_prepare(ctx, ops.to_device(gk))
    dct = ops.to_device(ct)
    base = ops.to_host(ops.rotate(ctx, dct, key, 25))
    assert np.array_equal(base[:1], GA.rotate(ct[:1], gk, 25, qs, P.special))
    try:
        for k, mb in _cm_shapes(12):
            _lib.call("ckks_ctx_set_tuning", ctx.handle, CM_K, k)
            _lib.call("ckks_ctx_set_tuning", ctx.handle, CM_MINB, mb)
            assert np.array_equal(ops.to_host(ops.rotate(ctx, dct, key, 25)), base), f"K={k} budget={mb}"
    finally:
        _reset(_lib, ctx)


@pytest.mark.parametrize("log_n", [12, 13])
def test_ct_mul_plain_every_radix_identical(ck, log_n):
    import torch
    ops, _lib, Context = ck
    from ckks_b200.params import CkksParams
    P = CkksParams.standard(log_n, 4)
    ctx = Context.get(log_n, P.primes, n_special=1)
    qs = list(P.q)
    n = 1 << log_n
    rng = np.random.default_rng(log_n + 5)
    ct = _rand(rng, (7, 2, 4, n), qs)
    pt = _rand(rng, (7, 4, n), qs)
    dct, dpt = ops.to_device(ct), ops.to_device(pt)
    st = torch.cuda.current_stream().cuda_stream
    prod = np.stack([mulmod(ct[:, j], pt, np.asarray(qs, dtype=np.uint64)[:, None]) for j in range(2)], axis=1)
    want = R.rescale(prod, qs)
    try:
        for k in (0, 2, 3, 4, 5):
            if k and (n >> k) > 1024:
                continue
            _lib.call("ckks_ctx_set_tuning", ctx.handle, NTT_K, k)
            out = torch.empty((7, 2, 3, n), dtype=torch.uint64, device="cuda")
            _lib.call("ckks_ct_mul_plain_rescale", ctx.handle, out.data_ptr(), dct.data_ptr(), dpt.data_ptr(),
                      1, 7, 4, st)
            assert np.array_equal(ops.to_host(out), want), f"K={k}"
    finally:
        _reset(_lib, ctx)


def test_unbuilt_shapes_refused(ck):
    """Shapes outside the built set return an error (nothing launches)."""
    ops, _lib, Context = ck
    from ckks_b200._lib import CkksError
    from ckks_b200.params import CkksParams
    ctx = Context.get(12, CkksParams.standard(12, 3).primes, n_special=1)
    for bad in (1, 6, -1):
        for param in (CM_K, NTT_K):
            with pytest.raises(CkksError):
                _lib.call("ckks_ctx_set_tuning", ctx.handle, param, bad)
    for bad in (9, -1):
        with pytest.raises(CkksError):
            _lib.call("ckks_ctx_set_tuning", ctx.handle, CM_UPC, bad)
    P = CkksParams.standard(13, 3)
    ctx = Context.get(13, P.primes, n_special=1)
    rng = np.random.default_rng(1)
    a = ops.to_device(_rand(rng, (1, 2, 3, 8192), list(P.q)))
    key = ops.relin_key_prepare(ctx, ops.to_device(_rand(rng, (3, 2, 4, 8192), list(P.q) + [P.special])))
    try:
        _three_kernels(_lib, ctx)
        for k, mb in ((2, 1), (5, 2)):  # K = 2 not built at N = 2^13; K = 5 balanced only
            _lib.call("ckks_ctx_set_tuning", ctx.handle, CM_K, k)
            _lib.call("ckks_ctx_set_tuning", ctx.handle, CM_MINB, mb)
            with pytest.raises(CkksError):
                ops.ct_mul_relin_rescale(ctx, a, a, key)
    finally:
        _reset(_lib, ctx)


def test_units_per_cta_identical(ck):
    """Several work units per CTA (the grid shrinks, a CTA loops) give the
    same ct-mult and rotation results, including a unit count that is not a
    multiple of the units per CTA (37 pairs)."""
    ops, _lib, Context = ck
    from ckks_b200.params import CkksParams
    P = CkksParams.standard(12, 3)
    ctx = Context.get(12, P.primes, n_special=1)
    qs = list(P.q)
    rng = np.random.default_rng(515)
    a = _rand(rng, (37, 2, 3, 4096), qs)
    b = _rand(rng, (37, 2, 3, 4096), qs)
    ksk = _rand(rng, (3, 2, 4, 4096), qs + [P.special])
    key = ops.relin_key_prepare(ctx, ops.to_device(ksk))
    da, db = ops.to_device(a), ops.to_device(b)
    base = ops.to_host(ops.ct_mul_relin_rescale(ctx, da, db, key))
    rot = ops.to_host(ops.rotate(ctx, da, key, 5))
    assert np.array_equal(base[36:], R.ct_mul_relin_rescale(a[36:], b[36:], ksk, qs, P.special))
    try:
        _three_kernels(_lib, ctx)
        for upc in (1, 2, 3, 4, 8):
            _lib.call("ckks_ctx_set_tuning", ctx.handle, CM_UPC, upc)
            for k in (3, 4):
                _lib.call("ckks_ctx_set_tuning", ctx.handle, CM_K, k)
                assert np.array_equal(ops.to_host(ops.ct_mul_relin_rescale(ctx, da, db, key)), base), (upc, k)
            assert np.array_equal(ops.to_host(ops.rotate(ctx, da, key, 5)), rot), upc
    finally:
        _reset(_lib, ctx)


@pytest.mark.parametrize("log_n,n_ct,level", [(12, 300, 3), (12, 7, 2), (13, 5, 4), (10, 33, 3)])
def test_tma_tensor_kernel_identical(ck, log_n, n_ct, level):
    """The persistent TMA-fed tensor kernel (bulk copies into shared memory,
    mbarrier waits) gives the same ct-mult results as one CTA per unit, with
    and without concurrent sub-batches, and no bounded wait expires."""
    ops, _lib, Context = ck
    from ckks_b200.params import CkksParams
    P = CkksParams.standard(log_n, 4)
    ctx = Context.get(log_n, P.primes, n_special=1)
    qs = list(P.q)
    n = 1 << log_n
    rng = np.random.default_rng(log_n * 7 + n_ct)
    a = _rand(rng, (n_ct, 2, level, n), qs[:level])
    b = _rand(rng, (n_ct, 2, level, n), qs[:level])
    ksk = _rand(rng, (4, 2, 5, n), qs + [P.special])
    key = ops.relin_key_prepare(ctx, ops.to_device(ksk))
    da, db = ops.to_device(a), ops.to_device(b)
    try:
        _three_kernels(_lib, ctx)
        _lib.call("ckks_ctx_set_tuning", ctx.handle, CM_TMA, 2)
        base = ops.to_host(ops.ct_mul_relin_rescale(ctx, da, db, key))
        for split in (1, 0):
            _lib.call("ckks_ctx_set_tuning", ctx.handle, CM_SPLIT, split)
            _lib.call("ckks_ctx_set_tuning", ctx.handle, CM_TMA, 1)
            for _ in range(2):
                assert np.array_equal(ops.to_host(ops.ct_mul_relin_rescale(ctx, da, db, key)), base), split
    finally:
        _reset(_lib, ctx)
    assert _lib.raw("ckks_device_status")() == 0
    sub = ksk[:level][:, :, list(range(level)) + [4]]
    assert np.array_equal(base[:1], R.ct_mul_relin_rescale(a[:1], b[:1], sub, qs[:level], P.special))


@pytest.mark.parametrize("level,n_ct,upc", [(2, 33, 1), (3, 300, 1), (5, 17, 2), (8, 9, 4)])
def test_modup_tmem_accumulators_identical(ck, level, n_ct, upc):
    """The ModUp with its key inner-product accumulators in TMEM (three
    256-thread CTAs per SM) against the shared-memory ModUp and the oracle at
    N = 2^12: ragged batches, several levels, several units per CTA."""
    ops, _lib, Context = ck
    from ckks_b200.params import CkksParams
    P = CkksParams.standard(12, 8)
    ctx = Context.get(12, P.primes, n_special=1)
    qs = list(P.q)
    rng = np.random.default_rng(100 + level)
    a = _rand(rng, (n_ct, 2, level, 4096), qs[:level])
    b = _rand(rng, (n_ct, 2, level, 4096), qs[:level])
    a[0, :, :, :] = np.asarray(qs[:level], dtype=np.uint64)[None, :, None] - 1
    ksk = _rand(rng, (8, 2, 9, 4096), qs + [P.special])
    key = ops.relin_key_prepare(ctx, ops.to_device(ksk))
    da, db = ops.to_device(a), ops.to_device(b)
    got = {}
    try:
        _three_kernels(_lib, ctx)
        _lib.call("ckks_ctx_set_tuning", ctx.handle, CM_UPC, upc)
        for tm in (1, 2):
            _lib.call("ckks_ctx_set_tuning", ctx.handle, CM_TMEM, tm)
            got[tm] = ops.to_host(ops.ct_mul_relin_rescale(ctx, da, db, key))
    finally:
        _reset(_lib, ctx)
    assert np.array_equal(got[1], got[2])
    sub = ksk[:level][:, :, list(range(level)) + [8]]
    idx = [0, n_ct - 1]
    assert np.array_equal(got[1][idx], R.ct_mul_relin_rescale(a[idx], b[idx], sub, qs[:level], P.special))
    from ckks_b200._lib import CkksError
    with pytest.raises(CkksError, match="ModUp accumulators"):
        _lib.call("ckks_ctx_set_tuning", ctx.handle, CM_TMEM, 3)

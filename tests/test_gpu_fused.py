"""The fused ct-mult kernel (one thread-block cluster of level + 1 CTAs per
ciphertext pair, intermediates in distributed shared memory and TMEM, no
scratch; selected with CKKS_TUNE_CM_FUSED = 1) is bit-identical to the oracle
and to the three-kernel path.

Integer results: tolerance zero.  CKKS_TUNE_CM_FUSED = 1 makes a call fail
rather than fall back, so these tests know which path ran.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import rns_ckks as R

pytestmark = pytest.mark.gpu

CM_SPLIT, CM_FUSED = 2, 7
STAGE_FUSED = 5


def _rand(rng, shape, basis):
    x = np.zeros(shape, dtype=np.uint64)
    for i, q in enumerate(basis):
        x[..., i, :] = rng.integers(0, q, size=x[..., i, :].shape, dtype=np.uint64)
    return x


@pytest.fixture(scope="module")
def env(cuda):
    import ckks_b200.ops as ops
    from ckks_b200 import _lib
    from ckks_b200.context import Context
    from ckks_b200.params import CkksParams
    return ops, _lib, Context, CkksParams


def _setup(env, log_n, level, n_ct, seed, max_level=None):
    ops, _lib, Context, CkksParams = env
    P = CkksParams.standard(log_n, max_level or level)
    ctx = Context.get(log_n, P.primes, n_special=1)
    qs = list(P.q)
    n = 1 << log_n
    rng = np.random.default_rng(seed)
    a = _rand(rng, (n_ct, 2, level, n), qs[:level])
    b = _rand(rng, (n_ct, 2, level, n), qs[:level])
    big = P.levels
    ksk = _rand(rng, (big, 2, big + 1, n), qs + [P.special])
    key = ops.relin_key_prepare(ctx, ops.to_device(ksk))
    sub = ksk[:level][:, :, list(range(level)) + [big]]
    return P, ctx, qs, a, b, key, sub


@pytest.mark.parametrize("log_n", [10, 11, 12, 13])
@pytest.mark.parametrize("level", [2, 3, 5, 7])
def test_fused_matches_oracle(env, log_n, level):
    ops, _lib, _, _ = env
    P, ctx, qs, a, b, key, sub = _setup(env, log_n, level, 3, 1000 * log_n + level)
    try:
        _lib.call("ckks_ctx_set_tuning", ctx.handle, CM_FUSED, 1)
        assert ops.ct_mul_scratch_bytes(ctx, 3, level) == 0
        got = ops.to_host(ops.ct_mul_relin_rescale(ctx, ops.to_device(a), ops.to_device(b), key))
    finally:
        _lib.call("ckks_ctx_set_tuning", ctx.handle, CM_FUSED, 0)
    assert np.array_equal(got, R.ct_mul_relin_rescale(a, b, sub, qs[:level], P.special))


@pytest.mark.parametrize("log_n,level,n_ct", [(12, 3, 300), (13, 4, 70), (11, 6, 129), (12, 7, 17)])
def test_fused_equals_three_kernels(env, log_n, level, n_ct):
    """Large ragged batches (more clusters than fit at once, counts that are
    not multiples of anything), a context whose key has more digits than the
    ciphertexts' level (level 4 of 7 at N = 2^13), both paths bit-identical."""
    ops, _lib, _, _ = env
    max_level = 7 if log_n == 13 else None
    P, ctx, qs, a, b, key, sub = _setup(env, log_n, level, n_ct, 77 + n_ct, max_level)
    da, db = ops.to_device(a), ops.to_device(b)
    try:
        _lib.call("ckks_ctx_set_tuning", ctx.handle, CM_FUSED, 1)
        fused = ops.to_host(ops.ct_mul_relin_rescale(ctx, da, db, key))
        _lib.call("ckks_ctx_set_tuning", ctx.handle, CM_FUSED, 2)
        assert ops.ct_mul_scratch_bytes(ctx, n_ct, level) == n_ct * (6 * level + 2) * (1 << log_n) * 8
        three = ops.to_host(ops.ct_mul_relin_rescale(ctx, da, db, key))
    finally:
        _lib.call("ckks_ctx_set_tuning", ctx.handle, CM_FUSED, 0)
    assert np.array_equal(fused, three)
    idx = [0, n_ct - 1]
    assert np.array_equal(fused[idx], R.ct_mul_relin_rescale(a[idx], b[idx], sub, qs[:level], P.special))


def test_fused_selection_and_refusal(env):
    """Default: the three kernels (scratch sized for them); with the fused
    kernel selected, no scratch where it is built, and a refusal with a
    message for shapes it is not built for (level 8: a cluster of 9 CTAs
    exceeds the portable 8; N = 2^9)."""
    ops, _lib, Context, CkksParams = env
    from ckks_b200._lib import CkksError
    P = CkksParams.standard(12, 8)
    ctx = Context.get(12, P.primes, n_special=1)
    assert ops.ct_mul_scratch_bytes(ctx, 4, 3) == 4 * 20 * 4096 * 8
    try:
        _lib.call("ckks_ctx_set_tuning", ctx.handle, CM_FUSED, 1)
        assert ops.ct_mul_scratch_bytes(ctx, 4, 3) == 0
        assert ops.ct_mul_scratch_bytes(ctx, 4, 8) == 4 * 50 * 4096 * 8
    finally:
        _lib.call("ckks_ctx_set_tuning", ctx.handle, CM_FUSED, 0)
    rng = np.random.default_rng(9)
    qs = list(P.q)
    a = ops.to_device(_rand(rng, (2, 2, 8, 4096), qs))
    key = ops.relin_key_prepare(ctx, ops.to_device(_rand(rng, (8, 2, 9, 4096), qs + [P.special])))
    try:
        _lib.call("ckks_ctx_set_tuning", ctx.handle, CM_FUSED, 1)
        with pytest.raises(CkksError, match="fused kernel is not built"):
            ops.ct_mul_relin_rescale(ctx, a, a, key, scratch=None)
    finally:
        _lib.call("ckks_ctx_set_tuning", ctx.handle, CM_FUSED, 0)
    P9 = CkksParams.standard(9, 3)
    ctx9 = Context.get(9, P9.primes, n_special=1)
    assert ops.ct_mul_scratch_bytes(ctx9, 2, 3) == 2 * 20 * 512 * 8
    with pytest.raises(CkksError):
        _lib.call("ckks_ctx_set_tuning", ctx.handle, CM_FUSED, 3)


def test_fused_profiled_as_one_launch(env):
    """One fused launch per call, recorded under its own profiler stage."""
    import torch
    ops, _lib, _, _ = env
    P, ctx, qs, a, b, key, sub = _setup(env, 12, 3, 8, 5)
    lib = _lib.load()
    da, db = ops.to_device(a), ops.to_device(b)
    _lib.call("ckks_ctx_set_tuning", ctx.handle, CM_FUSED, 1)
    try:
        ops.ct_mul_relin_rescale(ctx, da, db, key)
        torch.cuda.synchronize()
        lib.ckks_profile_reset()
        lib.ckks_profile_enable(1)
        for _ in range(3):
            ops.ct_mul_relin_rescale(ctx, da, db, key)
        torch.cuda.synchronize()
    finally:
        lib.ckks_profile_enable(0)
        _lib.call("ckks_ctx_set_tuning", ctx.handle, CM_FUSED, 0)
    tot, cnt = C.c_double(), C.c_longlong()
    lib.ckks_profile_read(STAGE_FUSED, C.byref(tot), C.byref(cnt))
    assert cnt.value == 3 and tot.value > 0
    lib.ckks_profile_read(0, C.byref(tot), C.byref(cnt))
    assert cnt.value == 0  # the three-kernel tensor stage did not run

"""The tensor-core transform (ckks_ntt_tc: N = 2^12 as a 64 x 64 four-step
transform whose stages are int8 byte-limb matrix products on tcgen05) is
bit-exact against the oracle's merged negacyclic forward transform
(restating tb/ref/gen_ntt_reference.py:78 ntt with the negacyclic twist) and
against the FP64 engine (ckks_ntt), on the production 45-bit chain, the
config-1 prime, and 46 / 47-bit chains with the patterns that maximise the
byte-limb sums (every residue q - 1, alternating 0 / q - 1, the top 2^20 of
[0, q)).  Integer results: tolerance zero."""
import numpy as np
import pytest

from oracle import rns_ckks as R

pytestmark = pytest.mark.gpu

QC = 35184371884033  # largest 45-bit prime = 1 mod 2^13 (the config-1 prime)
CKKS_ETIMEOUT = -2
TUNE_WAIT_CYCLES = 6


def _fill(rng, shape, basis, pattern):
    x = np.zeros(shape, dtype=np.uint64)
    for i, q in enumerate(basis):
        sl = x[..., i, :]
        if pattern == "random":
            sl[...] = rng.integers(0, q, size=sl.shape, dtype=np.uint64)
        elif pattern == "max":
            sl[...] = q - 1
        elif pattern == "alternating":
            sl[...] = np.where(np.arange(sl.shape[-1]) % 2 == 0, 0, q - 1).astype(np.uint64)
        elif pattern == "zero":
            sl[...] = 0
        else:
            sl[...] = q - 1 - rng.integers(0, 1 << 20, size=sl.shape, dtype=np.uint64)
    return x


@pytest.fixture(scope="module")
def ck(cuda):
    import ckks_b200.ops as ops
    from ckks_b200.context import Context
    return ops, Context


def _check(ops, ctx, basis, x, prime_begin=0):
    d = ops.to_device(x)
    ops.ntt_tc(ctx, d, prime_begin=prime_begin, n_limbs=len(basis))
    got = ops.to_host(d)
    assert np.array_equal(got, R.ntt_limbs(x, basis))
    f = ops.to_device(x)
    ops.ntt(ctx, f, prime_begin=prime_begin, n_limbs=len(basis))
    assert np.array_equal(got, ops.to_host(f))


@pytest.mark.parametrize("n_polys", [1, 3, 37])
def test_ntt_tc_production_chain(ck, n_polys):
    ops, Context = ck
    from ckks_b200.params import CkksParams
    P = CkksParams.standard(12, 3)
    basis = list(P.q) + [P.special]
    ctx = Context.get(12, list(P.q) + [P.special], n_special=1)
    x = _fill(np.random.default_rng(n_polys), (n_polys, len(basis), 4096), basis, "random")
    _check(ops, ctx, basis, x)


def test_ntt_tc_limb_subrange(ck):
    ops, Context = ck
    from ckks_b200.params import CkksParams
    P = CkksParams.standard(12, 3)
    prims = list(P.q) + [P.special]
    ctx = Context.get(12, prims, n_special=1)
    basis = prims[1:3]
    x = _fill(np.random.default_rng(5), (4, 2, 4096), basis, "random")
    _check(ops, ctx, basis, x, prime_begin=1)


@pytest.mark.parametrize("pattern", ["random", "max", "alternating", "top", "zero"])
def test_ntt_tc_config1_prime(ck, pattern):
    ops, Context = ck
    ctx = Context.get(12, [QC])
    x = _fill(np.random.default_rng(7), (2, 1, 4096), [QC], pattern)
    _check(ops, ctx, [QC], x)


@pytest.mark.parametrize("bits", [46, 47])
@pytest.mark.parametrize("pattern", ["random", "max", "alternating", "top"])
def test_ntt_tc_wide_primes(ck, bits, pattern):
    ops, Context = ck
    from ckks_b200.params import chain_primes
    basis = list(chain_primes(3, 13, bits))
    ctx = Context.get(12, basis)
    x = _fill(np.random.default_rng(bits), (2, 3, 4096), basis, pattern)
    _check(ops, ctx, basis, x)


def test_ntt_tc_round_trip_and_argument_checks(ck):
    ops, Context = ck
    from ckks_b200 import _lib
    ctx = Context.get(12, [QC])
    x = _fill(np.random.default_rng(9), (8, 1, 4096), [QC], "random")
    d = ops.to_device(x)
    ops.ntt_tc(ctx, d, n_limbs=1)
    ops.ntt(ctx, d, inverse=True, n_limbs=1)
    assert np.array_equal(ops.to_host(d), x)
    other = Context.get(13, [QC])
    with pytest.raises(RuntimeError, match="N = 2\\^12 only"):
        ops.ntt_tc(other, ops.to_device(np.zeros((1, 1, 8192), dtype=np.uint64)), n_limbs=1)
    with pytest.raises(RuntimeError, match="outside"):
        _lib.call("ckks_ntt_tc", ctx.handle, d.data_ptr(), 1, 0, 2, None)


def test_ntt_tc_wait_expiry_is_reported_and_recoverable(ck):
    """A one-cycle wait limit makes the kernel's first mbarrier wait (the
    matrix image's bulk copy, or the first MMA commit) run out: every CTA
    drains what it issued (bounded), leaves its polynomial unchanged and
    counts the expiry; ckks_device_status reports CKKS_ETIMEOUT once, and
    with the limit restored the same call is bit-exact again."""
    import torch
    from ckks_b200 import _lib
    ops, Context = ck
    lib = _lib.load()
    ctx = Context(12, [QC])  # private context: the tuning change stays local
    x = _fill(np.random.default_rng(11), (16, 1, 4096), [QC], "random")
    torch.cuda.synchronize()
    assert lib.ckks_device_status() == 0, lib.ckks_last_error().decode()
    d = ops.to_device(x)
    try:
        _lib.call("ckks_ctx_set_tuning", ctx.handle, TUNE_WAIT_CYCLES, 1)
        ops.ntt_tc(ctx, d, n_limbs=1)
        torch.cuda.synchronize()
        assert lib.ckks_device_status() == CKKS_ETIMEOUT
        assert lib.ckks_device_status() == 0  # read and cleared
        got = ops.to_host(d)
        exp = R.ntt_limbs(x, [QC])
        # a CTA either finished (correct transform) or gave up (input intact)
        for i in range(x.shape[0]):
            assert np.array_equal(got[i], exp[i]) or np.array_equal(got[i], x[i])
    finally:
        _lib.call("ckks_ctx_set_tuning", ctx.handle, TUNE_WAIT_CYCLES, 0)
    d = ops.to_device(x)
    ops.ntt_tc(ctx, d, n_limbs=1)
    torch.cuda.synchronize()
    assert lib.ckks_device_status() == 0
    assert np.array_equal(ops.to_host(d), R.ntt_limbs(x, [QC]))

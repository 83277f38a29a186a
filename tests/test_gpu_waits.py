"""Bounded device waits run out cleanly and are reported to the host.

Kernels that wait on the GPU (a bulk copy landing in shared memory) spin for
at most CKKS_TUNE_WAIT_CYCLES SM cycles.  These tests shrink that limit to one
cycle so the first wait expires before its copy can land (no fault, no
planted error: every copy is correct and eventually lands), and check that
  - the kernel records the expiry and ckks_device_status returns CKKS_ETIMEOUT,
  - the context stays usable: with the limit restored, the same call runs to
    completion, ckks_device_status returns CKKS_OK, and the results are
    bit-exact against the oracle.
The reference's counterpart is the noise monitor's saturation flag
(rtl/m4/noise_monitor.sv:72-73): a hardware condition surfaced as a status bit.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CKKS_ETIMEOUT = -2
TUNE_TENSOR_TMA = 5
TUNE_WAIT_CYCLES = 6
TUNE_CM_FUSED = 7


def _rand(rng, shape, basis):
    x = np.zeros(shape, dtype=np.uint64)
    for i, q in enumerate(basis):
        x[..., i, :] = rng.integers(0, q, size=x[..., i, :].shape, dtype=np.uint64)
    return x


def test_tma_tensor_wait_expiry_is_reported_and_recoverable(cuda):
    import torch

    import ckks_b200.ops as ops
    from ckks_b200 import _lib
    from ckks_b200.context import Context
    from ckks_b200.params import CkksParams
    from oracle import rns_ckks as R

    lib = _lib.load()
    P = CkksParams.standard(12, 3)
    ctx = Context.get(12, P.primes, n_special=1)
    qs = list(P.q)
    rng = np.random.default_rng(404)
    ksk = _rand(rng, (3, 2, 4, P.n), qs + [P.special])
    key = ops.relin_key_prepare(ctx, ops.to_device(ksk))
    a = _rand(rng, (4, 2, 3, P.n), qs)
    b = _rand(rng, (4, 2, 3, P.n), qs)
    da, db = ops.to_device(a), ops.to_device(b)
    torch.cuda.synchronize()
    assert lib.ckks_device_status() == 0, lib.ckks_last_error().decode()
    try:
        _lib.call("ckks_ctx_set_tuning", ctx.handle, TUNE_CM_FUSED, 2)  # the TMA-fed kernel is on that path
        _lib.call("ckks_ctx_set_tuning", ctx.handle, TUNE_TENSOR_TMA, 1)
        _lib.call("ckks_ctx_set_tuning", ctx.handle, TUNE_WAIT_CYCLES, 1)
        ops.ct_mul_relin_rescale(ctx, da, db, key)
        torch.cuda.synchronize()
        rc = lib.ckks_device_status()
        assert rc == CKKS_ETIMEOUT, rc
        assert b"expired" in lib.ckks_last_error()
        # the status is cleared by the read
        assert lib.ckks_device_status() == 0
        # the context is still usable: default limit, same kernel, exact results
        _lib.call("ckks_ctx_set_tuning", ctx.handle, TUNE_WAIT_CYCLES, 0)
        got = ops.to_host(ops.ct_mul_relin_rescale(ctx, da, db, key))
        torch.cuda.synchronize()
        assert lib.ckks_device_status() == 0, lib.ckks_last_error().decode()
        assert np.array_equal(got, R.ct_mul_relin_rescale(a, b, ksk, qs, P.special))
    finally:
        _lib.call("ckks_ctx_set_tuning", ctx.handle, TUNE_WAIT_CYCLES, 0)
        _lib.call("ckks_ctx_set_tuning", ctx.handle, TUNE_TENSOR_TMA, 0)
        _lib.call("ckks_ctx_set_tuning", ctx.handle, TUNE_CM_FUSED, 0)


def test_wait_limit_rejects_negative(cuda):
    from ckks_b200 import _lib
    from ckks_b200.context import Context
    from ckks_b200.params import CkksParams

    lib = _lib.load()
    P = CkksParams.standard(12, 3)
    ctx = Context.get(12, P.primes, n_special=1)
    assert lib.ckks_ctx_set_tuning(ctx.handle, TUNE_WAIT_CYCLES, -5) == 1
    assert b"wait limit" in lib.ckks_last_error()

"""The allocation-free ct-mult entry point (static device scratch) gives the same
results as the allocating one.

ckks_ct_mul_relin_rescale_noalloc serves callers that are handed only their
input and output buffers and cannot call cudaMalloc (a plugin inside a foreign
runtime whose host owns device memory through its own pool, or a serving loop
whose pool has reserved the GPU).  Its scratch is a fixed 32 MiB static device
array shared by all calls.  This test calls it through the C ABI twice in a
row, with different inputs, and checks each result bit-exactly (integer
results: tolerance zero, as in every other parity test here) against
ckks_ct_mul_relin_rescale with caller scratch; then checks that a batch larger
than the static array is refused before any device work.  The file name makes
pytest collect it last.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rand(rng, shape, basis):
    x = np.zeros(shape, dtype=np.uint64)
    for i, q in enumerate(basis):
        x[..., i, :] = rng.integers(0, q, size=x[..., i, :].shape, dtype=np.uint64)
    return x


def test_noalloc_entry_matches_allocating_entry(cuda):
    import torch

    import ckks_b200.ops as ops
    from ckks_b200 import _lib
    from ckks_b200.context import Context
    from ckks_b200.params import CkksParams

    lib = _lib.load()
    lib.ckks_profile_enable(0)
    P = CkksParams.standard(12, 3)
    ctx = Context.get(12, P.primes, n_special=1)
    qs = list(P.q)
    rng = np.random.default_rng(77)
    ksk = _rand(rng, (3, 2, 4, P.n), qs + [P.special])
    key = ops.relin_key_prepare(ctx, ops.to_device(ksk))
    n_ct, level = 8, 3
    stream = torch.cuda.current_stream().cuda_stream
    noalloc = lib.ckks_ct_mul_relin_rescale_noalloc

    for call in range(2):
        a = ops.to_device(_rand(rng, (n_ct, 2, level, P.n), qs))
        b = ops.to_device(_rand(rng, (n_ct, 2, level, P.n), qs))
        ref = ops.ct_mul_relin_rescale(ctx, a, b, key)      # caller-scratch entry point
        out = torch.zeros_like(ref)
        rc = noalloc(ctx.handle, out.data_ptr(), a.data_ptr(), b.data_ptr(), key.data_ptr(),
                     n_ct, level, stream)
        assert rc == 0, lib.ckks_last_error().decode()
        torch.cuda.synchronize()
        assert np.array_equal(ops.to_host(out), ops.to_host(ref)), f"call {call} differs"

    # one pair more than the static array holds is refused on the host (the
    # entry runs the three-kernel path: (6 level + 2) limbs of scratch per pair)
    per_pair = (6 * level + 2) * P.n * 8
    too_many = (32 * 1024 * 1024) // per_pair + 1
    rc = noalloc(ctx.handle, out.data_ptr(), a.data_ptr(), b.data_ptr(), key.data_ptr(),
                 too_many, level, stream)
    assert rc == 1
    assert b"static" in lib.ckks_last_error()


def test_noalloc_entry_ignores_sub_batch_split(cuda):
    """A batch the allocating entry would fork into concurrent sub-batches
    (N = 2^10, L = 3, 160 pairs; and CKKS_TUNE_CM_SPLIT = 4 set on the
    context) runs as one sub-batch on the caller's stream in the no-alloc
    entry (which creates no stream or event) and still equals the allocating
    entry bit for bit, on two calls in a row."""
    import torch

    import ckks_b200.ops as ops
    from ckks_b200 import _lib
    from ckks_b200.context import Context
    from ckks_b200.params import CkksParams

    lib = _lib.load()
    lib.ckks_profile_enable(0)
    P = CkksParams.standard(10, 3)
    ctx = Context.get(10, P.primes, n_special=1)
    qs = list(P.q)
    rng = np.random.default_rng(78)
    ksk = _rand(rng, (3, 2, 4, P.n), qs + [P.special])
    key = ops.relin_key_prepare(ctx, ops.to_device(ksk))
    n_ct, level = 160, 3
    assert n_ct * (6 * level + 2) * P.n * 8 <= 32 * 1024 * 1024
    stream = torch.cuda.current_stream().cuda_stream
    noalloc = lib.ckks_ct_mul_relin_rescale_noalloc
    try:
        for split in (0, 4):
            _lib.call("ckks_ctx_set_tuning", ctx.handle, 2, split)
            for call in range(2):
                a = ops.to_device(_rand(rng, (n_ct, 2, level, P.n), qs))
                b = ops.to_device(_rand(rng, (n_ct, 2, level, P.n), qs))
                ref = ops.ct_mul_relin_rescale(ctx, a, b, key)
                out = torch.zeros_like(ref)
                rc = noalloc(ctx.handle, out.data_ptr(), a.data_ptr(), b.data_ptr(), key.data_ptr(),
                             n_ct, level, stream)
                assert rc == 0, lib.ckks_last_error().decode()
                torch.cuda.synchronize()
                assert np.array_equal(ops.to_host(out), ops.to_host(ref)), f"split {split} call {call}"
    finally:
        _lib.call("ckks_ctx_set_tuning", ctx.handle, 2, 0)

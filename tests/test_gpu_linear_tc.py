"""The tensor-core encrypted linear layer (tcgen05.mma kind::i8, TMEM
accumulators, byte-limb split) is bit-identical to the oracle and to the
integer-pipe layer (ckks_linear_plain_weights).  Integer results: tolerance
zero."""
import numpy as np
import pytest

from oracle.linear import linear_plain

pytestmark = pytest.mark.gpu

W_MAX = 127 * (1 + 256 + 65536)


def _resid(rng, shape, primes):
    x = np.zeros(shape, dtype=np.uint64)
    for i, q in enumerate(primes):
        x[:, :, i, :] = rng.integers(0, q, size=x[:, :, i, :].shape, dtype=np.uint64)
    return x


def _int_layer(ctx, x, w, bias, keep, level):
    import torch
    from ckks_b200 import _lib
    O, F = w.shape
    out = torch.empty((O, 2, level, x.shape[-1]), dtype=torch.uint64, device="cuda")
    wd = torch.from_numpy(np.ascontiguousarray(w.astype(np.int32))).cuda()
    bd = None if bias is None else torch.from_numpy(np.asarray(bias, dtype=np.int64)).cuda()
    kd = None if keep is None else torch.from_numpy(np.ascontiguousarray(keep.astype(np.uint8))).cuda()
    _lib.call("ckks_linear_plain_weights", ctx.handle, out.data_ptr(), x.data_ptr(), wd.data_ptr(),
              None if bd is None else bd.data_ptr(), None if kd is None else kd.data_ptr(), O, F, level,
              torch.cuda.current_stream().cuda_stream)
    return out


@pytest.mark.parametrize("bits", [45, 47])
@pytest.mark.parametrize("O,F,log_n,level", [(10, 37, 5, 2), (5, 130, 6, 3), (130, 9, 5, 1)])
def test_tc_linear_matches_oracle(cuda, bits, O, F, log_n, level):
    """Small shapes through every edge: fewer outputs than a tile (10, 5) and
    more (130: two tiles), features not a multiple of the 128-feature chunk
    (37, 130, 9), the largest weights three byte limbs hold (+-8355711),
    residues up to q - 1 of 45- and 47-bit primes, a block mask, a bias."""
    import torch
    import ckks_b200.ops as ops
    from ckks_b200.context import Context
    from ckks_b200.params import chain_primes
    primes = list(chain_primes(level, 13, bits))
    ctx = Context.get(log_n, primes)
    rng = np.random.default_rng(O * 1000 + F + bits)
    n = 1 << log_n
    x = _resid(rng, (F, 2, level, n), primes)
    x[0, :, :, :] = np.asarray(primes[:level], dtype=np.uint64)[None, :, None] - 1   # q - 1 everywhere
    w = rng.integers(-W_MAX, W_MAX + 1, size=(O, F), dtype=np.int64)
    w[0, :] = W_MAX
    w[-1, :] = -W_MAX
    keep = (rng.random(((O + 3) // 4, (F + 3) // 4)) < 0.6).astype(np.uint8)
    bias = rng.integers(-(1 << 62), 1 << 62, size=O, dtype=np.int64)
    packed = ops.linear_tc_pack(w, keep)
    dx = ops.to_device(x)
    got = ops.to_host(ops.linear_plain_weights_tc(ctx, dx, packed, O,
                                                  bias=torch.from_numpy(bias).cuda()))
    want = linear_plain(x, w, bias, keep, primes)
    assert np.array_equal(got, want)
    # dense (no mask), no bias
    got2 = ops.to_host(ops.linear_plain_weights_tc(ctx, dx, ops.linear_tc_pack(w), O))
    assert np.array_equal(got2, linear_plain(x, w, None, None, primes))


@pytest.mark.parametrize("O,F,log_n,level", [(128, 784, 13, 4), (1152, 784, 10, 2), (10, 128, 13, 3)])
def test_tc_linear_equals_integer_layer(cuda, O, F, log_n, level):
    """The encrypted MLP's layers (784 -> 128 at N = 2^13, L = 4; 128 -> 10)
    and the CNN's convolution as a 1152 x 784 matrix, with 50 % 4x4 block
    sparsity and weights at the 2^20 scale the MLP uses."""
    import math
    import torch
    import ckks_b200.ops as ops
    from ckks_b200.context import Context
    from ckks_b200.mlp import gear_keep, make_block_sparse
    from ckks_b200.params import CkksParams
    P = CkksParams.standard(log_n, max(level, 2))
    ctx = Context.get(log_n, P.primes, n_special=1)
    rng = np.random.default_rng(O + F)
    W = make_block_sparse(rng.standard_normal((O, F)) / math.sqrt(F), 0.5, 3)
    w = np.round(W * 2 ** 20).astype(np.int64)
    keep = gear_keep(W, 0.25)
    x = _resid(rng, (F, 2, level, 1 << log_n), P.primes[:level])
    bias = rng.integers(-(1 << 60), 1 << 60, size=O, dtype=np.int64)
    dx = ops.to_device(x)
    got = ops.linear_plain_weights_tc(ctx, dx, ops.linear_tc_pack(w, keep), O,
                                      bias=torch.from_numpy(bias).cuda())
    ref = _int_layer(ctx, dx, w, bias, keep, level)
    assert torch.equal(got, ref)
    # a few positions against the oracle
    cols = [0, 1, x.shape[-1] - 1]
    xs = x[:, :, :, cols]
    want = linear_plain(xs, w, bias, keep, P.primes[:level])
    assert np.array_equal(ops.to_host(got)[:, :, :, cols], want)


def test_tc_pack_refuses_large_weights(cuda):
    import ckks_b200.ops as ops
    from ckks_b200._lib import CkksError
    w = np.zeros((4, 8), dtype=np.int64)
    w[2, 3] = W_MAX + 1
    with pytest.raises(CkksError, match="three signed byte limbs"):
        ops.linear_tc_pack(w)
    w[2, 3] = -W_MAX
    ops.linear_tc_pack(w)


def test_tc_linear_short_wait_limit_is_safe(cuda):
    """With a one-cycle limit on the MMA-completion waits, whether a wait
    expires depends on timing (the MMAs often finish while the next are being
    issued).  Either way the call returns, an expiry is reported at most once
    (the status read clears it), and with the limit restored the same call is
    exact: an expired CTA drains its MMAs before it frees its TMEM and leaves."""
    import torch
    import ckks_b200.ops as ops
    from ckks_b200 import _lib
    from ckks_b200.context import Context
    from ckks_b200.params import CkksParams
    lib = _lib.load()
    P = CkksParams.standard(12, 2)
    ctx = Context.get(12, P.primes, n_special=1)
    rng = np.random.default_rng(8)
    x = _resid(rng, (784, 2, 2, 4096), P.primes[:2])
    w = rng.integers(-1000, 1000, size=(128, 784), dtype=np.int64)
    dx = ops.to_device(x)
    packed = ops.linear_tc_pack(w)
    ref = _int_layer(ctx, dx, w, None, None, 2)
    torch.cuda.synchronize()
    assert lib.ckks_device_status() == 0
    try:
        _lib.call("ckks_ctx_set_tuning", ctx.handle, 6, 1)
        for _ in range(4):
            ops.linear_plain_weights_tc(ctx, dx, packed, 128)
        torch.cuda.synchronize()
        assert lib.ckks_device_status() in (0, -2)
        assert lib.ckks_device_status() == 0
    finally:
        _lib.call("ckks_ctx_set_tuning", ctx.handle, 6, 0)
    got = ops.linear_plain_weights_tc(ctx, dx, packed, 128)
    torch.cuda.synchronize()
    assert lib.ckks_device_status() == 0
    assert torch.equal(got, ref)

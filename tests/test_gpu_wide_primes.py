"""Bit-exact parity at the edge of the accepted prime range.

ckks_ctx_create accepts NTT-friendly primes below 2^47; the production chain
is 45-bit.  The FP64 arithmetic's exactness argument (every intermediate an
integer below 2^53, forward-transform values below 2^51) is tightest for the
widest primes, so every hot kernel is checked here on 46-bit and 47-bit
chains (all primes in [2^(b-1), 2^b), so max < 2 min holds) against the
oracle, with random residues and with the adversarial patterns that maximise
the lazy intermediates: every residue q - 1, alternating 0 / q - 1, and
residues in the top 2^20 of [0, q); for the key switch also every key word
q - 1.  Integer results: bit-exact (tolerance zero).
"""
import numpy as np
import pytest

from oracle import galois as GA
from oracle import rns_ckks as R
from oracle.modmath import mulmod
from oracle.ntt import negacyclic_mul_ntt

pytestmark = pytest.mark.gpu

BITS = (46, 47)
PATTERNS = ("random", "max", "alternating", "top")


def _chain(bits: int, count: int, log_n_max: int = 13):
    from ckks_b200.params import chain_primes
    return list(chain_primes(count, log_n_max, bits))


def _fill(rng, shape, basis, pattern):
    """Residues of `shape` [..., len(basis), N] per pattern."""
    x = np.zeros(shape, dtype=np.uint64)
    for i, q in enumerate(basis):
        sl = x[..., i, :]
        if pattern == "random":
            sl[...] = rng.integers(0, q, size=sl.shape, dtype=np.uint64)
        elif pattern == "max":
            sl[...] = q - 1
        elif pattern == "alternating":
            sl[...] = np.where(np.arange(sl.shape[-1]) % 2 == 0, 0, q - 1).astype(np.uint64)
        else:
            sl[...] = q - 1 - rng.integers(0, 1 << 20, size=sl.shape, dtype=np.uint64)
    return x


def test_chains_have_the_requested_width():
    for bits in BITS:
        ch = _chain(bits, 9)
        assert all(q.bit_length() == bits and (q - 1) % (1 << 14) == 0 for q in ch)
        assert max(ch) < 2 * min(ch)


@pytest.mark.parametrize("bits", BITS)
@pytest.mark.parametrize("log_n", [12, 13, 14])
@pytest.mark.parametrize("pattern", PATTERNS)
def test_ntt_wide_primes(cuda, bits, log_n, pattern):
    import ckks_b200.ops as ops
    from ckks_b200.context import Context
    qs = _chain(bits, 3, log_n_max=14)
    ctx = Context.get(log_n, qs)
    rng = np.random.default_rng(bits * 100 + log_n)
    x = _fill(rng, (2, 3, 1 << log_n), qs, pattern)
    d = ops.to_device(x)
    ops.ntt(ctx, d)
    assert np.array_equal(ops.to_host(d), R.ntt_limbs(x, qs))
    ops.ntt(ctx, d, inverse=True)
    assert np.array_equal(ops.to_host(d), x)


@pytest.mark.parametrize("bits", BITS)
@pytest.mark.parametrize("pattern", PATTERNS)
def test_poly_mul_wide_primes(cuda, bits, pattern):
    """The one-kernel NTT -> pointwise -> INTT product at N = 2^12."""
    import ckks_b200.ops as ops
    from ckks_b200.context import Context
    from oracle.modmath import root_2n
    qs = _chain(bits, 2)
    ctx = Context.get(12, qs)
    rng = np.random.default_rng(bits + 7)
    a = _fill(rng, (2, 2, 4096), qs, pattern)
    b = _fill(rng, (2, 2, 4096), qs, "random" if pattern == "alternating" else pattern)
    got = ops.to_host(ops.poly_mul(ctx, ops.to_device(a), ops.to_device(b), n_limbs=2))
    for i, q in enumerate(qs):
        want = negacyclic_mul_ntt(a[:, i], b[:, i], q, root_2n(q, 4096))
        assert np.array_equal(got[:, i], want), (q, i)


@pytest.mark.parametrize("bits", BITS)
@pytest.mark.parametrize("log_n,level", [(12, 3), (12, 8), (13, 3)])
@pytest.mark.parametrize("pattern", PATTERNS)
def test_ct_mult_wide_primes(cuda, bits, log_n, level, pattern):
    import ckks_b200.ops as ops
    from ckks_b200.context import Context
    ch = _chain(bits, level + 1)
    special, qs = ch[0], ch[1:]
    ctx = Context.get(log_n, qs + [special], n_special=1)
    n = 1 << log_n
    rng = np.random.default_rng(bits * 1000 + level * 10 + log_n)
    n_ct = 2
    a = _fill(rng, (n_ct, 2, level, n), qs, pattern)
    b = _fill(rng, (n_ct, 2, level, n), qs, pattern)
    ksk = _fill(rng, (level, 2, level + 1, n), qs + [special], pattern)
    key = ops.relin_key_prepare(ctx, ops.to_device(ksk))
    got = ops.to_host(ops.ct_mul_relin_rescale(ctx, ops.to_device(a), ops.to_device(b), key))
    assert np.array_equal(got, R.ct_mul_relin_rescale(a, b, ksk, qs, special))


@pytest.mark.parametrize("bits", BITS)
@pytest.mark.parametrize("pattern", PATTERNS)
def test_ct_mul_plain_rescale_wide_primes(cuda, bits, pattern):
    import torch
    import ckks_b200.ops as ops
    from ckks_b200 import _lib
    from ckks_b200.context import Context
    level = 3
    ch = _chain(bits, level + 1)
    special, qs = ch[0], ch[1:]
    ctx = Context.get(12, qs + [special], n_special=1)
    rng = np.random.default_rng(bits + 31)
    ct = _fill(rng, (3, 2, level, 4096), qs, pattern)
    pt = _fill(rng, (3, level, 4096), qs, pattern)
    dct, dpt = ops.to_device(ct), ops.to_device(pt)
    out = torch.empty((3, 2, level - 1, 4096), dtype=torch.uint64, device="cuda")
    _lib.call("ckks_ct_mul_plain_rescale", ctx.handle, out.data_ptr(), dct.data_ptr(), dpt.data_ptr(),
              1, 3, level, torch.cuda.current_stream().cuda_stream)
    qv = np.asarray(qs, dtype=np.uint64)[:, None]
    prod = np.stack([mulmod(ct[:, k], pt, qv) for k in range(2)], axis=1)
    assert np.array_equal(ops.to_host(out), R.rescale(prod, qs))


@pytest.mark.parametrize("bits", BITS)
@pytest.mark.parametrize("pattern", PATTERNS)
def test_rotate_wide_primes(cuda, bits, pattern):
    import ckks_b200.ops as ops
    from ckks_b200.context import Context
    level = 3
    ch = _chain(bits, level + 1)
    special, qs = ch[0], ch[1:]
    ctx = Context.get(12, qs + [special], n_special=1)
    rng = np.random.default_rng(bits + 57)
    ct = _fill(rng, (2, 2, level, 4096), qs, pattern)
    gk = _fill(rng, (level, 2, level + 1, 4096), qs + [special], pattern)
    key = ops.relin_key_prepare(ctx, ops.to_device(gk))
    got = ops.to_host(ops.rotate(ctx, ops.to_device(ct), key, 5))
    assert np.array_equal(got, GA.rotate(ct, gk, 5, qs, special))


@pytest.mark.parametrize("bits", BITS)
@pytest.mark.parametrize("pattern", PATTERNS)
def test_mul_plain_multi_wide_primes(cuda, bits, pattern):
    """The conv + GAP product kernel (coefficient-domain ciphertexts times
    evaluation-domain weight polynomials) on one wide prime."""
    import ckks_b200.ops as ops
    from ckks_b200 import convgap as G
    from ckks_b200.context import Context
    from oracle import convgap as OC
    q = _chain(bits, 1, log_n_max=10)[0]
    ctx = Context.get(10, [q])
    rng = np.random.default_rng(bits + 91)
    ct = _fill(rng, (3, 2, 1024), [q] * 2, pattern)
    w = _fill(rng, (2, 1, 1024), [q], pattern).reshape(2, 1024)
    w_hat = ops.to_device(w.reshape(2, 1, 1024))
    ops.ntt(ctx, w_hat, n_limbs=1)
    got = ops.to_host(G.mul_plain_multi(ctx, ops.to_device(ct), w_hat.reshape(2, 1024)))
    for i in range(3):
        for f in range(2):
            assert np.array_equal(got[i, f], OC.mul_plain(ct[i], w[f], q)), (i, f)

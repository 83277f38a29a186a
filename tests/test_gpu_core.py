"""GPU parity of the core kernels against the oracle and the reference's golden
vectors (bit-exact for every integer result)."""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import golden as G
from oracle import ntt as ON
from oracle import rns_ckks as R
from oracle.modmath import bitrev_perm, mulmod, root_2n

pytestmark = pytest.mark.gpu

GD = Path(__file__).resolve().parent / "golden"
META = json.load(open(GD / "golden_core.json"))
ARR = np.load(GD / "golden_core.npz")
QC = 35184371884033


@pytest.fixture(scope="module")
def ck(cuda):
    import ckks_b200.ops as ops
    from ckks_b200.context import Context
    return ops, Context


def test_toy_cyclic_ntt(ck):
    ops, Context = ck
    t = META["toy"]
    ctx = Context.get(4, [t["q"]], omega=[t["omega"]])
    x = ops.to_device(ARR["toy_ntt_in"])
    ops.ntt(ctx, x, cyclic=True, n_limbs=1)
    nat = ops.to_host(ops.bitrev_permute(ctx, x))
    assert np.array_equal(nat, ARR["toy_ntt_out"])
    ops.ntt(ctx, x, cyclic=True, inverse=True, n_limbs=1)
    assert np.array_equal(ops.to_host(x), ARR["toy_ntt_in"])


def test_q3_cyclic_ntt_golden(ck):
    ops, Context = ck
    m = META["q3"]
    ctx = Context.get(12, [m["q"]], omega=[m["omega"]])
    x = ops.to_device(ARR["q3_ntt_in"][None, :])
    ops.ntt(ctx, x, cyclic=True)
    assert np.array_equal(ops.to_host(ops.bitrev_permute(ctx, x))[0], ARR["q3_ntt_out"])


@pytest.mark.parametrize("log_n", [5, 10, 12, 13, 14])
def test_negacyclic_ntt_vs_oracle(ck, log_n):
    ops, Context = ck
    from ckks_b200.params import chain_primes
    n = 1 << log_n
    primes = list(chain_primes(3, 14))
    ctx = Context.get(log_n, primes)
    rng = np.random.default_rng(log_n)
    x = np.stack([rng.integers(0, q, size=n, dtype=np.uint64) for q in primes])[None]
    x[0, 0, :3] = [0, primes[0] - 1, 1]
    d = ops.to_device(x)
    ops.ntt(ctx, d)
    got = ops.to_host(d)
    exp = R.ntt_limbs(x, primes)
    assert np.array_equal(got, exp)
    ops.ntt(ctx, d, inverse=True)
    assert np.array_equal(ops.to_host(d), x)


def test_poly_mul_config1_prime(ck):
    ops, Context = ck
    ctx = Context.get(12, [QC])
    rng = np.random.default_rng(1)
    a = rng.integers(0, QC, size=(3, 1, 4096), dtype=np.uint64)
    b = rng.integers(0, QC, size=(3, 1, 4096), dtype=np.uint64)
    a[2, 0, :] = QC - 1
    got = ops.to_host(ops.poly_mul(ctx, ops.to_device(a), ops.to_device(b)))
    exp = ON.negacyclic_mul_ntt(a, b, QC, root_2n(QC, 4096))
    assert np.array_equal(got, exp)
    # one full schoolbook check (reference poly_mult semantics)
    assert [int(v) for v in got[0, 0]] == G.poly_mult([int(v) for v in a[0, 0]], [int(v) for v in b[0, 0]], QC)


def test_poly_mul_golden_n256(ck):
    ops, Context = ck
    a, b, c = ARR["pmneg256"]
    ctx = Context.get(8, [QC])
    got = ops.to_host(ops.poly_mul(ctx, ops.to_device(a[None]), ops.to_device(b[None])))[0]
    assert np.array_equal(got, c)


def test_poly_mul_cyclic_pm12(ck):
    ops, Context = ck
    m = META["pm12"]
    ctx = Context.get(12, [m["q"]], omega=[m["omega"]])
    for tag in ("rand0", "sparse"):
        a, b, c = ARR[f"pm12_{tag}_a"], ARR[f"pm12_{tag}_b"], ARR[f"pm12_{tag}_c"]
        got = ops.to_host(ops.poly_mul(ctx, ops.to_device(a[None]), ops.to_device(b[None]), cyclic=True))
        assert np.array_equal(got[0], c)


def test_poly_mul_anyq_toy(ck):
    ops, Context = ck
    from ckks_b200.params import chain_primes
    crt = Context.get(4, list(chain_primes(3, 14)))
    a, b, c = ARR["pmneg16_q113"]
    got = ops.to_host(ops.poly_mul_anyq(crt, ops.to_device(a[None]), ops.to_device(b[None]), 113))
    assert np.array_equal(got[0], c)
    # cyclic toy + 45-bit modulus not of NTT form
    rng = np.random.default_rng(3)
    q = (1 << 45) - 55
    x = rng.integers(0, q, size=(4, 16), dtype=np.uint64)
    y = rng.integers(0, q, size=(4, 16), dtype=np.uint64)
    gotc = ops.to_host(ops.poly_mul_anyq(crt, ops.to_device(x), ops.to_device(y), q, cyclic=True))
    gotn = ops.to_host(ops.poly_mul_anyq(crt, ops.to_device(x), ops.to_device(y), q, cyclic=False))
    for i in range(4):
        xi, yi = [int(v) for v in x[i]], [int(v) for v in y[i]]
        assert [int(v) for v in gotc[i]] == G.poly_mult_cyclic(xi, yi, q)
        assert [int(v) for v in gotn[i]] == G.poly_mult(xi, yi, q)


@pytest.mark.parametrize("key,log_n", [("relin16", 4), ("relin64", 6)])
def test_relin_single_golden(ck, key, log_n):
    ops, Context = ck
    q = META["keyswitch"]["q"]
    ctx = Context.get(log_n, [q])
    v = ARR[key]
    d = [ops.to_device(np.ascontiguousarray(v[:, i])) for i in range(5)]
    f0, f1 = ops.relin_single(ctx, *d)
    assert np.array_equal(ops.to_host(f0), v[:, 5])
    assert np.array_equal(ops.to_host(f1), v[:, 6])


def test_rescale_exact_golden(ck):
    ops, _ = ck
    primes = META["rescale"]["primes"]
    for i in range(len(primes) - 1):
        got = ops.to_host(ops.rescale_exact(ops.to_device(ARR[f"rescale_{i}_in"]), primes[i], primes[i + 1]))
        assert np.array_equal(got, ARR[f"rescale_{i}_out"])
    import random
    rng = random.Random(META["rescale"]["poly_seed"])
    poly = [rng.randrange(primes[0]) for _ in range(META["rescale"]["N"])]
    got = ops.to_host(ops.rescale_exact(ops.to_device(poly), primes[0], primes[1]))
    assert np.array_equal(got, ARR["rescale_poly_out"])


def test_rescale_scaled_golden(ck):
    ops, _ = ck
    m = META["e2e"]
    got = ops.to_host(ops.rescale_scaled(ops.to_device(ARR["e2e_rescale_in"]), m["q_in"], m["q_out"], m["scale_bits"]))
    assert np.array_equal(got, ARR["e2e_rescale_out"])


def test_pointwise_fastred_vectors(ck):
    ops, Context = ck
    q = META["fastred"]["q"]
    ctx = Context.get(12, [q])
    got = ops.to_host(ops.pointwise_mul(ctx, ops.to_device(ARR["fastred_b"][None]), ops.to_device(ARR["fastred_w"][None])))
    assert np.array_equal(got[0], ARR["fastred_out"])


def _rand_ct(rng, shape, basis):
    x = np.zeros(shape, dtype=np.uint64)
    for i, q in enumerate(basis):
        x[..., i, :] = rng.integers(0, q, size=x[..., i, :].shape, dtype=np.uint64)
    return x


@pytest.mark.parametrize("log_n,levels,level,n_ct", [(12, 3, 3, 4), (12, 3, 2, 3), (13, 4, 4, 2), (6, 3, 3, 5), (13, 8, 8, 1)])
def test_ct_mul_relin_rescale_vs_oracle(ck, log_n, levels, level, n_ct):
    ops, Context = ck
    from ckks_b200.params import CkksParams
    P = CkksParams.standard(log_n, levels)
    ctx = Context.get(log_n, P.primes, n_special=1)
    n = 1 << log_n
    qs = list(P.q[:level])
    rng = np.random.default_rng(log_n * 100 + level)
    a = _rand_ct(rng, (n_ct, 2, level, n), qs)
    b = _rand_ct(rng, (n_ct, 2, level, n), qs)
    a[0, 0, 0, :4] = [0, qs[0] - 1, 1, qs[0] - 2]
    ksk = _rand_ct(rng, (levels, 2, levels + 1, n), list(P.q) + [P.special])
    key = ops.relin_key_prepare(ctx, ops.to_device(ksk))
    # the prepared key holds, per limb, the N values then their N quotients w / q (doubles)
    kp = ops.to_host(key).view(np.float64).reshape(levels, 2, levels + 1, 2, n)
    assert np.array_equal(kp[:, :, :, 0], ksk.astype(np.float64))
    qq = np.array(list(P.q) + [P.special], dtype=np.float64)
    assert np.array_equal(kp[:, :, :, 1], ksk.astype(np.float64) / qq[None, None, :, None])
    got = ops.to_host(ops.ct_mul_relin_rescale(ctx, ops.to_device(a), ops.to_device(b), key))
    sub_ksk = ksk[:level][:, :, list(range(level)) + [levels]]
    exp = R.ct_mul_relin_rescale(a, b, sub_ksk, qs, P.special)
    assert np.array_equal(got, exp)


def test_rescale_rns_vs_oracle(ck):
    ops, Context = ck
    from ckks_b200.params import CkksParams
    P = CkksParams.standard(12, 3)
    ctx = Context.get(12, P.primes, n_special=1)
    rng = np.random.default_rng(9)
    x = _rand_ct(rng, (3, 2, 3, 4096), list(P.q))
    got = ops.to_host(ops.rescale_rns(ctx, ops.to_device(x)))
    assert np.array_equal(got, R.rescale(x, list(P.q)))


@pytest.mark.parametrize("n,q", [(16, 113), (1024, 998244353), (2048, QC)])
def test_masked_relin_equals_golden_relin(ck, n, q):
    """rtl/m3/keyswitch_pipe_masked.sv semantics: any additive split of the key
    gives the unmasked golden relin (scripts/verify_keyswitch.py:62)."""
    from ckks_b200 import golden_bridge as gb
    rng = np.random.default_rng(n + 7)
    e0, e1, e2, a, b, a1, b1 = ([int(v) for v in rng.integers(0, q, n)] for _ in range(7))
    a2 = [(x - y) % q for x, y in zip(a, a1)]
    b2 = [(x - y) % q for x, y in zip(b, b1)]
    want = G.relin(e0, e1, e2, a, b, q)
    got = gb.relin_masked(e0, e1, e2, a1, b1, a2, b2, q)
    assert list(got[0]) == list(want[0]) and list(got[1]) == list(want[1])


def test_ct_mul_concurrent_sub_batches_identical(ck):
    """A 256-pair call split into 1, 2, 3, 4, 8 or 16 sub-batches (4 internal
    streams joined by events) gives identical results; pairs from every
    sub-batch match the oracle."""
    ops, Context = ck
    import torch
    from ckks_b200 import _lib
    from ckks_b200.params import CkksParams
    P = CkksParams.standard(12, 3)
    ctx = Context.get(12, P.primes, n_special=1)
    qs = list(P.q)
    rng = np.random.default_rng(77)
    a = _rand_ct(rng, (256, 2, 3, 4096), qs)
    b = _rand_ct(rng, (256, 2, 3, 4096), qs)
    ksk = _rand_ct(rng, (3, 2, 4, 4096), qs + [P.special])
    key = ops.relin_key_prepare(ctx, ops.to_device(ksk))
    da, db = ops.to_device(a), ops.to_device(b)
    outs = []
    try:
        _lib.call("ckks_ctx_set_tuning", ctx.handle, 7, 2)  # the three-kernel path (sub-batches apply to it)
        for split in (1, 2, 3, 4, 8, 16, 0):
            _lib.call("ckks_ctx_set_tuning", ctx.handle, 2, split)
            outs.append(ops.to_host(ops.ct_mul_relin_rescale(ctx, da, db, key)))
    finally:
        _lib.call("ckks_ctx_set_tuning", ctx.handle, 2, 0)
        _lib.call("ckks_ctx_set_tuning", ctx.handle, 7, 0)
    outs.append(ops.to_host(ops.ct_mul_relin_rescale(ctx, da, db, key)))  # default: the fused kernel
    assert all(np.array_equal(o, outs[0]) for o in outs[1:])
    idx = [0, 85, 170, 255]
    assert np.array_equal(outs[0][idx], R.ct_mul_relin_rescale(a[idx], b[idx], ksk, qs, P.special))


def test_ct_mul_n16384_rejected_with_a_message(ck):
    """At N = 2^14 the ModUp / ModDown CTAs would need ~400 KB of shared
    memory: the call returns an error naming the limit instead of launching."""
    ops, Context = ck
    from ckks_b200 import _lib
    from ckks_b200.params import CkksParams
    P = CkksParams.standard(14, 3)
    ctx = Context.get(14, P.primes, n_special=1)
    a = ops.to_device(np.zeros((1, 2, 3, 1 << 14), dtype=np.uint64))
    key = ops.to_device(np.zeros((3, 2, 4, 1 << 14, 2), dtype=np.uint64))
    with pytest.raises(_lib.CkksError, match="shared memory"):
        ops.ct_mul_relin_rescale(ctx, a, a, key)

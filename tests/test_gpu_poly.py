"""Ciphertext arithmetic and homomorphic polynomial evaluation: the
elementwise kernels bit-exact against numpy, and a degree-5 activation
approximation of scripts/golden_activation.py (ActivationGoldenModel, one
Chebyshev segment on [-1, 1]) evaluated on encrypted slots: decrypted values
equal the reference's own approximate() outputs within 1e-4 (the tolerance
covers the CKKS noise of three multiplicative levels at scales down to 2^20)."""
import json
from pathlib import Path

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

GD = Path(__file__).resolve().parent / "golden"
ACT = json.load(open(GD / "golden_act.json"))


def _rand(rng, shape, qs):
    x = np.empty(shape, dtype=np.uint64)
    for i, q in enumerate(qs):
        x[..., i, :] = rng.integers(0, q, size=x[..., i, :].shape, dtype=np.uint64)
    return x


def test_elementwise_ciphertext_arithmetic(cuda):
    import ckks_b200.ops as ops
    from ckks_b200.context import Context
    from ckks_b200.params import CkksParams
    P = CkksParams.standard(12, 3)
    ctx = Context.get(12, P.primes, n_special=1)
    qs = np.array(P.q, dtype=object)
    rng = np.random.default_rng(4)
    a = _rand(rng, (3, 2, 3, 4096), list(P.q))
    b = _rand(rng, (3, 2, 3, 4096), list(P.q))
    qv = qs[None, None, :, None]
    A, B = a.astype(object), b.astype(object)
    assert np.array_equal(ops.to_host(ops.ct_add(ctx, ops.to_device(a), ops.to_device(b))),
                          ((A + B) % qv).astype(np.uint64))
    assert np.array_equal(ops.to_host(ops.ct_add(ctx, ops.to_device(a), ops.to_device(b), subtract=True)),
                          ((A - B) % qv).astype(np.uint64))
    for m in (0, 1, -1, 12345678901, -(1 << 61) + 3):
        got = ops.to_host(ops.ct_mul_const(ctx, ops.to_device(a), m))
        assert np.array_equal(got, ((A * m) % qv).astype(np.uint64)), m
    for c in (7, -(1 << 50) - 1):
        got = ops.to_host(ops.ct_add_const(ctx, ops.to_device(a), c))
        want = A.copy()
        want[:, 0] = (A[:, 0] + c) % qv[:, 0]
        assert np.array_equal(got, want.astype(np.uint64)), c


@pytest.mark.parametrize("name", ["sigmoid", "tanh"])
def test_activation_polynomial_matches_reference_approximation(cuda, name):
    from ckks_b200.evaluator import Evaluator
    from ckks_b200.params import CkksParams
    m = ACT["models"]["order5_segments1"][name]
    seg = m["segments"][0]
    assert seg["a"] == -1.0 and seg["b"] == 1.0
    coeffs = seg["poly_coeffs"][::-1]                      # ascending
    ev = Evaluator(CkksParams.standard(12, 6, seed=3))
    ev.keygen()
    xs = np.asarray(m["x"])
    rng = np.random.default_rng(1)
    vals = np.concatenate([xs, rng.uniform(-1, 1, 2048 - len(xs))])
    ct = ev.encrypt_values(torch.from_numpy(vals[None]).to(torch.complex128).cuda())
    r = ev.poly_eval(ct, coeffs)
    assert r.level == 2
    got = ev.decrypt_values(r, 2048).cpu().numpy()[0].real
    assert np.abs(got - np.polyval(seg["poly_coeffs"], vals)).max() < 1e-4
    assert np.abs(got[:len(xs)] - np.asarray(m["approx"])).max() < 1e-4

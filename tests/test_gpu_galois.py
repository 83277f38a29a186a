"""Automorphisms, monomial products and the key-switched rotation on the GPU:
bit-exact against the reference's goldens (coefficient automorphism and
X^nu product, scripts/exp_e24_rotation_bootstrap.py:143,189) and against the
oracle (evaluation-domain permutation, Galois key switch); decrypted slots of
a rotated ciphertext equal the input slots permuted by the Galois map."""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import galois as GA

pytestmark = pytest.mark.gpu

GD = Path(__file__).resolve().parent / "golden"
ROT = np.load(GD / "golden_rot.npz")
CASES = json.load(open(GD / "golden_rot.json"))["cases"]


@pytest.fixture(scope="module")
def ck(cuda):
    import ckks_b200.ops as ops
    from ckks_b200.context import Context
    return ops, Context


def _rand(rng, shape, qs):
    x = np.empty(shape, dtype=np.uint64)
    for i, q in enumerate(qs):
        x[..., i, :] = rng.integers(0, q, size=x[..., i, :].shape, dtype=np.uint64)
    return x


def test_coefficient_automorphism_and_monomial_goldens(ck):
    ops, Context = ck
    for c in CASES:
        if c["kind"] == "automorphism_key_exact":
            continue
        n, q, nu, k = c["n"], c["q"], c["nu"], c["key"]
        ctx = Context.get(n.bit_length() - 1, [q])
        x = ops.to_device(ROT[k + "_in"].reshape(-1, 1, n))
        if c["kind"] == "automorphism_exact":
            got = ops.to_host(ops.automorphism(ctx, x, nu)).reshape(ROT[k + "_out"].shape)
        else:
            got = ops.to_host(ops.mul_monomial(ctx, x, nu)).reshape(ROT[k + "_out"].shape)
        assert np.array_equal(got, ROT[k + "_out"]), c


@pytest.mark.parametrize("nu", [1, 5, 25, 4097, 8191, 6, 0])
def test_multilimb_automorphism_both_domains(ck, nu):
    ops, Context = ck
    from ckks_b200.params import CkksParams
    P = CkksParams.standard(12, 3)
    ctx = Context.get(12, P.primes, n_special=1)
    qs = list(P.primes)
    rng = np.random.default_rng(nu + 11)
    x = _rand(rng, (3, 4, 4096), qs)
    x[0, 0, :3] = [0, qs[0] - 1, 1]
    got = ops.to_host(ops.automorphism(ctx, ops.to_device(x), nu))
    want = np.stack([np.stack([GA.automorphism_coef(x[p, i], nu, q) for i, q in enumerate(qs)])
                     for p in range(3)])
    assert np.array_equal(got, want)
    if nu % 2:
        ge = ops.to_host(ops.automorphism(ctx, ops.to_device(x), nu, eval_domain=True))
        assert np.array_equal(ge, GA.automorphism_eval(x, nu))
    for m in (3, 4096, 4099, 8191):
        gm = ops.to_host(ops.mul_monomial(ctx, ops.to_device(x), m))
        want_m = np.stack([np.stack([GA.mul_monomial(x[p, i], m, q) for i, q in enumerate(qs)])
                           for p in range(3)])
        assert np.array_equal(gm, want_m)


@pytest.mark.parametrize("level,n_ct,nu", [(3, 3, 5), (2, 2, 8191), (3, 1, 25)])
def test_rotate_matches_oracle(ck, level, n_ct, nu):
    ops, Context = ck
    from ckks_b200.params import CkksParams
    P = CkksParams.standard(12, 3)
    ctx = Context.get(12, P.primes, n_special=1)
    qs = list(P.q)
    rng = np.random.default_rng(100 * level + nu)
    ct = _rand(rng, (n_ct, 2, level, 4096), qs[:level])
    gk = _rand(rng, (3, 2, 4, 4096), qs + [P.special])
    key = ops.relin_key_prepare(ctx, ops.to_device(gk))
    got = ops.to_host(ops.rotate(ctx, ops.to_device(ct), key, nu))
    assert np.array_equal(got, GA.rotate(ct, gk, nu, qs[:level], P.special))


def test_rotation_decrypts_to_permuted_slots(cuda):
    import torch
    from ckks_b200.evaluator import Evaluator
    from ckks_b200.params import CkksParams
    ev = Evaluator(CkksParams.standard(12, 3, seed=5))
    ev.keygen()
    rng = np.random.default_rng(3)
    vals = rng.uniform(-1, 1, (2, 2048))
    ct = ev.encrypt_values(torch.from_numpy(vals).to(torch.complex128).cuda())
    for nu in (5, 25, 8191):
        r = ev.rotate(ct, nu)
        src, conj = ev.galois_slot_map(nu)
        got = ev.decrypt_values(r, 2048).cpu().numpy()
        want = vals[:, src]
        assert np.abs(got.real - want).max() < 1e-6, nu
        assert np.abs(got.imag).max() < 1e-6
    # the Galois key equals the oracle's key for the same secret and samples
    L = ev.params.levels
    a = ev.uniform(L, L + 1)
    e = ev.dgauss((L, ev.n))
    raw, _ = ev.galois_key(5, a, e)
    want_gk = GA.galois_key(ev.sk.s_coef.cpu().numpy(), 5, list(ev.params.q), ev.params.special,
                            a.cpu().numpy(), e.cpu().numpy())
    assert np.array_equal(raw.cpu().numpy(), want_gk)


def test_rotation_rejects_even_nu(ck):
    ops, Context = ck
    from ckks_b200 import _lib
    from ckks_b200.params import CkksParams
    P = CkksParams.standard(12, 3)
    ctx = Context.get(12, P.primes, n_special=1)
    x = ops.to_device(np.zeros((1, 2, 3, 4096), dtype=np.uint64))
    key = ops.to_device(np.zeros((3, 2, 4, 4096, 2), dtype=np.uint64))
    with pytest.raises(_lib.CkksError, match="odd"):
        ops.rotate(ctx, x, key, 4)
    with pytest.raises(_lib.CkksError, match="odd"):
        ops.automorphism(ctx, x.reshape(2, 3, 4096), 4, eval_domain=True)

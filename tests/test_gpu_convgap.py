"""Conv + GAP fusion on the GPU (csrc/convgap.cu, ckks_b200/convgap.py) against
the goldens of scripts/exp_e24_rotation_bootstrap.py (golden_convgap.*) and the
oracle: ciphertext x plaintext products and decrypted constant coefficients
bit-exact, inner products identical floats, fused logits within 1e-12."""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import convgap as OC

pytestmark = pytest.mark.gpu

GD = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def g(cuda):
    import ckks_b200.convgap as G
    import ckks_b200.ops as ops
    from ckks_b200.context import Context
    d = np.load(GD / "golden_convgap.npz")
    m = json.load(open(GD / "golden_convgap.json"))
    ctx = Context.get(10, [m["q"]])
    s_res = G.secret_residues(d["s"], m["q"])
    return G, ops, ctx, d, m, s_res


def _hat(ops, ctx, poly):
    p = ops.to_device(np.asarray(poly, dtype=np.uint64).reshape(-1, 1, ctx.n))
    ops.ntt(ctx, p, n_limbs=1)
    return p.reshape(-1, ctx.n)


def test_mul_plain_and_decrypt_golden(g):
    G, ops, ctx, d, m, s_res = g
    out = G.mul_plain_multi(ctx, ops.to_device(d["mp_in"][None]), _hat(ops, ctx, d["sc2_out"]))
    got = ops.to_host(out)[0, 0]
    assert np.array_equal(got, d["mp_out"])
    dec0 = G.decrypt_coef0(ctx, out, s_res).cpu().numpy()
    assert dec0.shape == (1, 1) and dec0[0, 0] == d["mp_dec"][0]


def test_mul_plain_multi_batch_vs_oracle(g):
    """Several ciphertexts x several weight polynomials (one launch), edge
    residues (0, q - 1) included; every product and decryption checked."""
    G, ops, ctx, d, m, s_res = g
    q = m["q"]
    rng = np.random.default_rng(11)
    ct = rng.integers(0, q, (5, 2, ctx.n), dtype=np.uint64)
    ct[0, 0, :] = q - 1
    ct[1, 1, :] = 0
    w = rng.integers(0, q, (3, ctx.n), dtype=np.uint64)
    w[2] = 0
    w[2, 0] = 1  # the identity polynomial
    out = G.mul_plain_multi(ctx, ops.to_device(ct), _hat(ops, ctx, w))
    got = ops.to_host(out)
    dec0 = G.decrypt_coef0(ctx, out, s_res).cpu().numpy()
    for c in range(5):
        for f in range(3):
            want = OC.mul_plain(ct[c], w[f], q)
            assert np.array_equal(got[c, f], want), (c, f)
            assert dec0[c, f] == OC.decrypt(want, d["s"], q)[0]
    assert np.array_equal(got[:, 2], ct)


def test_inner_product_and_coef_sum_golden(g):
    G, ops, ctx, d, m, s_res = g
    q, sc = m["q"], m["scale"]
    for r in m["inner"]:
        ct = ops.to_device(d[r["key"] + "_ct"][None])
        w = d[r["key"] + "_w"]
        ip = G.inner_products(ctx, ct, G.weight_poly_hat(ctx, list(range(len(w))), w, sc), s_res, sc)
        cs = G.inner_products(ctx, ct, G.weight_poly_hat(ctx, list(range(r["dim"])), np.ones(r["dim"]), sc),
                              s_res, sc)
        assert ip[0, 0] == r["inner_product"] and cs[0, 0] == r["coef_sum"], r["key"]


def test_fused_inference_golden(g):
    """Golden images of the reference's encrypted_inference_fused: logits
    within 1e-12 (the plaintext FC sums in another order), same prediction,
    4 ciphertext products per image (one per filter)."""
    G, ops, ctx, d, m, s_res = g
    model = G.ConvGapModel(d["conv_w"], d["conv_b"], d["fc_w"], d["fc_b"])
    keys = [r["key"] for r in m["fused"]]
    ct = ops.to_device(np.stack([d[k + "_ct"] for k in keys]))
    w_hat = G.weight_polys(ctx, model, m["scale"])
    assert w_hat.shape == (4, ctx.n)
    logits = G.fused_inference(ctx, ct, model, s_res, m["scale"], w_hat=w_hat)
    for i, k in enumerate(keys):
        assert np.max(np.abs(logits[i] - d[k + "_logits"])) < 1e-12
        assert np.argmax(logits[i]) == np.argmax(d[k + "_logits"])
        assert np.max(np.abs(logits[i] - d[k + "_plain"])) < 5e-3


def test_fused_inference_batch_encrypted_on_gpu(g):
    """A batch of 300 images encrypted through the library (a s on the GPU):
    logits match the oracle's per-image fused inference and the plain model."""
    G, ops, ctx, d, m, s_res = g
    q, sc = m["q"], m["scale"]
    rng = np.random.default_rng(5)
    x = rng.uniform(0, 1, (300, 784))
    model = G.ConvGapModel.random(3)
    ct = G.encrypt(ctx, x, s_res, sc, seed=9)
    logits = G.fused_inference(ctx, ct, model, s_res, sc)
    host = ops.to_host(ct)
    for i in (0, 151, 299):
        want, mc = OC.fused_inference(host[i], d["s"], q, sc, model.conv_w, model.conv_b, model.fc_w, model.fc_b)
        assert np.max(np.abs(logits[i] - want)) < 1e-12 and mc == 14
    assert np.max(np.abs(logits - model.plain_forward(x))) < 5e-3


def test_general_prime_and_empty(g):
    """A 45-bit prime at N = 2^12 (64-bit products) and empty batches."""
    G, ops, ctx, d, m, s_res = g
    from ckks_b200.context import Context
    q = 35184371884033
    c12 = Context.get(12, [q])
    rng = np.random.default_rng(2)
    ct = rng.integers(0, q, (2, 2, 4096), dtype=np.uint64)
    w = rng.integers(0, q, (2, 4096), dtype=np.uint64)
    s = rng.integers(-1, 2, 4096)
    out = G.mul_plain_multi(c12, ops.to_device(ct), _hat(ops, c12, w))
    got = ops.to_host(out)
    dec0 = G.decrypt_coef0(c12, out, G.secret_residues(s, q)).cpu().numpy()
    for c in range(2):
        for f in range(2):
            want = OC.mul_plain(ct[c], w[f], q)
            assert np.array_equal(got[c, f], want)
            assert dec0[c, f] == OC.decrypt(want, s, q)[0]
    import torch
    empty = torch.empty((0, 2, ctx.n), dtype=torch.uint64, device="cuda")
    assert G.mul_plain_multi(ctx, empty, _hat(ops, ctx, d["sc0_out"])).shape == (0, 1, 2, ctx.n)


@pytest.mark.parametrize("log_n,q", [(4, 97), (5, 193), (13, 998244353)])
def test_small_and_large_rings(g, log_n, q):
    """N = 16 and 32 (fewer coefficients than a warp has lanes in the
    decryption) and N = 8192: products and decrypted constant coefficients
    against the oracle."""
    G, ops, ctx0, d, m, s_res0 = g
    from ckks_b200.context import Context
    n = 1 << log_n
    ctx = Context.get(log_n, [q])
    rng = np.random.default_rng(log_n)
    ct = rng.integers(0, q, (3, 2, n), dtype=np.uint64)
    w = rng.integers(0, q, (2, n), dtype=np.uint64)
    s = rng.integers(-1, 2, n)
    out = G.mul_plain_multi(ctx, ops.to_device(ct), _hat(ops, ctx, w))
    got = ops.to_host(out)
    dec0 = G.decrypt_coef0(ctx, out, G.secret_residues(s, q)).cpu().numpy()
    for c in range(3):
        for f in range(2):
            want = OC.mul_plain(ct[c], w[f], q)
            assert np.array_equal(got[c, f], want), (c, f)
            assert dec0[c, f] == OC.decrypt(want, s, q)[0]

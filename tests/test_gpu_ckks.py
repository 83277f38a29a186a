"""GPU parity of the CKKS layer: sampling, key generation, encode/decode,
encryption, the decrypted ct-mult (config: N = 2^12, L = 3 + 1 special,
Delta = 2^40, ternary secret, sigma = 3.2), DARE, noise monitor, sparsity,
RNS split/merge and the gear controller."""
import ctypes as C
import json
import random
from pathlib import Path

import numpy as np
import pytest

from oracle import encode as OE
from oracle import noise_gear as NG
from oracle import rns_ckks as R

pytestmark = pytest.mark.gpu

GD = Path(__file__).resolve().parent / "golden"
META = json.load(open(GD / "golden_core.json"))
ARR = np.load(GD / "golden_core.npz")


@pytest.fixture(scope="module")
def ev(cuda):
    from ckks_b200.evaluator import Evaluator
    from ckks_b200.params import CkksParams
    e = Evaluator(CkksParams.standard(12, 3, seed=5))
    e.keygen()
    return e


def _np(t):
    return t.cpu().numpy()


def test_sampler_statistics_and_determinism(cuda):
    import ckks_b200.ops as ops
    t = _np(ops.sample_ternary((1 << 20,), 7, 3))
    assert set(np.unique(t)) <= {-1, 0, 1}
    for v in (-1, 0, 1):
        assert abs((t == v).mean() - 1 / 3) < 0.01
    g = _np(ops.sample_dgauss((1 << 20,), 3.2, 7, 4)).astype(np.float64)
    assert abs(g.mean()) < 0.02 and abs(g.std() - 3.2) < 0.02 and np.abs(g).max() <= 39
    assert np.array_equal(_np(ops.sample_dgauss((4096,), 3.2, 7, 4)), g[:4096].astype(np.int64))


def test_keygen_matches_oracle(ev):
    p = ev.params
    a, e = ev._key_samples
    s = _np(ev.sk.s_coef)
    ksk = R.relin_key(s, list(p.q), p.special, _np(a.view(__import__("torch").int64)).astype(np.uint64), _np(e))
    assert np.array_equal(_np(ev.ksk.view(__import__("torch").int64)).astype(np.uint64), ksk)


def test_encode_decode_roundtrip(ev):
    import torch
    rng = np.random.default_rng(1)
    v = rng.uniform(-1, 1, (4, 2048)) + 1j * rng.uniform(-1, 1, (4, 2048))
    pt = ev.encode(v, level=3)
    coef = pt.clone()
    import ckks_b200.ops as ops
    ops.ntt(ev.ctx, coef, inverse=True, n_limbs=3)
    # coefficients agree with the FP64 oracle encoding (to one unit of rounding)
    want = np.stack([OE.ckks_encode(x, 2.0 ** 40, 4096) for x in v])
    got0 = _np(coef.view(torch.int64))[:, 0, :]
    q0 = ev.params.q[0]
    got0 = np.where(got0 > q0 // 2, got0 - q0, got0)
    assert np.abs(got0 - want).max() <= 1
    back = _np(ops.decode(ev.ctx, coef, 2048, 2.0 ** 40))
    assert np.abs(back - v).max() < 1e-9


def test_encrypt_decrypt_matches_oracle(ev):
    import torch
    import ckks_b200.ops as ops
    p = ev.params
    rng = np.random.default_rng(2)
    m = ev.encode(rng.uniform(-1, 1, (2, 2048)), level=3)
    a = ev.uniform(2, 3)
    e = ev.dgauss((2, ev.n))
    ct = ops.encrypt(ev.ctx, m, ev.sk.s_eval, a, e)
    mc = m.clone()
    ops.ntt(ev.ctx, mc, inverse=True, n_limbs=3)
    q0 = p.q[0]
    m_int = _np(mc.view(torch.int64))[:, 0, :]
    m_int = np.where(m_int > q0 // 2, m_int - q0, m_int)
    s = _np(ev.sk.s_coef)
    for c in range(2):
        want = R.encrypt_eval(m_int[c], s, list(p.q), _np(a.view(torch.int64))[c].astype(np.uint64), _np(e)[c])
        assert np.array_equal(_np(ct.view(torch.int64))[c].astype(np.uint64), want)
    dec = _np(ops.decrypt(ev.ctx, ct, ev.sk.s_eval).view(torch.int64)).astype(np.uint64)
    vals = R.crt_centred(dec[0], list(p.q))
    assert max(abs(v - (int(mi) + int(ei))) for v, mi, ei in zip(vals, m_int[0], _np(e)[0])) == 0


def test_config2_ct_mult_decoded_error_and_bit_exact(ev):
    """The ct-mult workload with a real key (N = 2^12, L = 3 + 1 special
    prime, scale 2^40, ternary secret, DG sigma 3.2): 256 pairs of slot
    vectors uniform in [-1, 1] are encrypted, multiplied, relinearised and
    rescaled; the decoded product is compared with the FP64 product x * y
    (the structure of scripts/verify_e2e_mult.py:78-102: encrypt, e2e_mult,
    decrypt, compare with the plaintext product).  Tolerances: max abs slot
    error < 1e-5 and normwise relative error max|z - xy| / max|xy| < 1e-5
    (the noise after rescale is ~2^-27 of the scale); imaginary parts < 1e-5."""
    import torch
    rng = np.random.default_rng(3)
    n_pairs = 256
    x = rng.uniform(-1, 1, (n_pairs, 2048))
    y = rng.uniform(-1, 1, (n_pairs, 2048))
    cx = ev.encrypt_values(x, level=3)
    cy = ev.encrypt_values(y, level=3)
    cz = ev.mul_relin_rescale(cx, cy)
    assert cz.data.shape == (n_pairs, 2, 2, 4096)
    z = _np(ev.decrypt_values(cz, 2048))
    err = np.abs(z.real - x * y)
    assert err.max() < 1e-5, err.max()
    assert err.max() / np.abs(x * y).max() < 1e-5
    assert np.abs(z.imag).max() < 1e-5
    # integers bit-exact against the oracle with the real key
    p = ev.params
    got = _np(cz.data[:2].contiguous().view(torch.int64)).astype(np.uint64)
    ksk = _np(ev.ksk.view(torch.int64)).astype(np.uint64)
    want = R.ct_mul_relin_rescale(_np(cx.data[:2].contiguous().view(torch.int64)).astype(np.uint64),
                                  _np(cy.data[:2].contiguous().view(torch.int64)).astype(np.uint64),
                                  ksk, list(p.q), p.special)
    assert np.array_equal(got, want)


def test_dare_golden_single_modulus(cuda):
    import torch
    import ckks_b200.ops as ops
    from ckks_b200.context import Context
    q = META["dare"]["q"]
    n = META["dare"]["N"]
    ctx = Context.get(10, [q])
    s = ARR["dare_s"].astype(np.int64)
    s_eval = torch.from_numpy(np.mod(s, q).astype(np.int64)).cuda().view(torch.uint64).reshape(1, n).contiguous()
    ops.ntt(ctx, s_eval, n_limbs=1)

    def to_eval(v):
        t = torch.from_numpy(np.mod(np.asarray(v, dtype=np.int64), q)).cuda().view(torch.uint64).reshape(1, 1, n).contiguous()
        ops.ntt(ctx, t, n_limbs=1)
        return t

    c0 = to_eval(ARR["dare_ct_b"])
    c1 = to_eval(-ARR["dare_ct_a"])
    ct = torch.stack([c0[0], c1[0]])[None].contiguous()           # [1, 2, 1, N]
    a_new = to_eval(-ARR["dare_ct2_a"])                            # (b2, a2) -> c1' = -a2
    e_new = torch.from_numpy(ARR["dare_e_new"]).cuda().reshape(1, n).contiguous()
    out = ops.dare_refresh(ctx, ct, s_eval, a_new, e_new, level_out=1)
    o0 = out[:, 0].contiguous()
    ops.ntt(ctx, o0, inverse=True, n_limbs=1)
    assert np.array_equal(_np(o0.view(torch.int64)).reshape(-1), np.mod(ARR["dare_ct2_b"], q))


def test_dare_level_raise_and_shift(ev):
    import torch
    rng = np.random.default_rng(4)
    x = rng.uniform(-1, 1, (3, 2048))
    cx = ev.encrypt_values(x, level=3)
    cz = ev.mul_relin_rescale(cx, cx)                     # level 2, scale ~2^35
    dec_old = R.crt_centred(_np(ev.decrypt_coef(cz)[0].view(torch.int64)).astype(np.uint64), list(ev.params.q[:2]))
    r = ev.dare_refresh(cz, level_out=3, shift_bits=0)
    assert r.level == 3
    dec_new = R.crt_centred(_np(ev.decrypt_coef(r)[0].view(torch.int64)).astype(np.uint64), list(ev.params.q))
    diff = np.array(dec_new, dtype=object) - np.array(dec_old, dtype=object)
    assert max(abs(int(d)) for d in diff) <= 40              # fresh error only (|e| <= 12 sigma)
    r2 = ev.dare_refresh(cz, level_out=3, shift_bits=5)
    z = _np(ev.decrypt_values(r2, 2048))
    assert np.abs(z.real - x * x).max() < 1e-5
    assert np.abs(_np(ev.decrypt_values(r, 2048)).real - x * x).max() < 1e-5


def test_noise_energy_and_snr(cuda):
    import torch
    import ckks_b200.ops as ops
    for c in META["noise"]["cases"]:
        x = ops.to_device(np.array([c["coeffs"]], dtype=np.uint64))
        tot = ops.noise_energy(x, c["q"])[0]
        assert tot / len(c["coeffs"]) == c["E"]
    rng = np.random.default_rng(5)
    ref = torch.from_numpy(rng.standard_normal((3, 1000))).cuda()
    dec = ref + 1e-3 * torch.from_numpy(rng.standard_normal((3, 1000))).cuda()
    s = _np(ops.snr_sums(dec, ref))
    assert np.allclose(s[:, 0], (_np(ref) ** 2).sum(1)) and np.allclose(s[:, 1], ((_np(dec) - _np(ref)) ** 2).sum(1))


def test_block_sparsity_golden_gpu(cuda):
    import torch
    import ckks_b200.ops as ops
    W = torch.from_numpy(ARR["bsm_W"]).cuda()
    for thr in (0.02, 0.05):
        out, keep = ops.block_sparse_mask(W, 4, thr)
        assert np.array_equal(np.packbits(_np(out) != 0), ARR[f"bsm_mask_{thr}"])
        assert int(_np(keep).sum()) == META[f"bsm_{thr}"]["total"] - META[f"bsm_{thr}"]["skip"]
    for rec in META["block_post"]:
        x = ops.to_device(np.array([rec["x"]], dtype=np.uint64))
        out, sk = ops.block_post_process(x, 113, rec["B"], 20)
        assert [int(v) for v in _np(out.view(torch.int64))[0]] == rec["out"]
        assert int(_np(sk)[0]) == rec["skipped"]


def test_rns_split_merge_rtl_primes(cuda):
    import torch
    import ckks_b200.ops as ops
    P = [77309411329, 206158430209, 2061584302081]
    M = P[0] * P[1] * P[2]
    rng = random.Random(6)
    xs = [rng.randrange(M) for _ in range(3000)] + [0, 1, M - 1, M // 2, M // 2 + 1]
    words = np.array([[x & (2 ** 64 - 1), x >> 64] for x in xs], dtype=np.uint64)
    res = ops.rns_split(P, ops.to_device(words))
    h = _np(res.view(torch.int64)).astype(np.uint64)
    for k, p in enumerate(P):
        assert [int(v) for v in h[k]] == [x % p for x in xs]
    back = _np(ops.rns_merge(P, res, 2).view(torch.int64)).astype(np.uint64)
    assert [int(lo) + (int(hi) << 64) for lo, hi in back] == xs
    # centred merge / split of signed values
    ys = [rng.randrange(-(M // 2), M // 2) for _ in range(1000)]
    wy = np.array([[(y % 2 ** 128) & (2 ** 64 - 1), (y % 2 ** 128) >> 64] for y in ys], dtype=np.uint64)
    ry = ops.rns_split(P, ops.to_device(wy), centered=True)
    assert [int(v) for v in _np(ry.view(torch.int64)).astype(np.uint64)[2]] == [y % P[2] for y in ys]
    by = _np(ops.rns_merge(P, ry, 2, centered=True).view(torch.int64)).astype(np.uint64)
    got = [(int(lo) + (int(hi) << 64)) - (2 ** 128 if int(hi) >> 63 else 0) for lo, hi in by]
    assert got == ys


def test_gear_controller_c_matches_rtl_model(cuda):
    from ckks_b200 import _lib
    from ckks_b200.gear import GearCtrl
    rng = random.Random(7)
    g = GearCtrl((500, 200, 50), 3)
    m = NG.GearCtrlRTL(500, 200, 50, 3)
    for _ in range(2000):
        e = rng.choice([rng.randrange(0, 60), rng.randrange(150, 260), rng.randrange(400, 700), 10 ** 30])
        hy = rng.random() < 0.9
        man = rng.random() < 0.05
        mg = rng.randrange(4)
        assert g.flush(e, hysteresis=hy, manual_en=man, manual_gear=mg) == \
            m.flush(e, hysteresis=hy, manual_en=man, manual_gear=mg)

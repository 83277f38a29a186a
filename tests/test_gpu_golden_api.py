"""The drop-in golden-API modules (cipher-pu_b200/scripts/) reproduce the
reference's golden vectors on the GPU, under the reference's own names."""
import json
import random
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
SCRIPTS = ROOT / "cipher-pu_b200" / "scripts"
if str(SCRIPTS) not in sys.path:
    sys.path.insert(0, str(SCRIPTS))

pytestmark = pytest.mark.gpu

GD = Path(__file__).resolve().parent / "golden"
META = json.load(open(GD / "golden_core.json"))
ARR = np.load(GD / "golden_core.npz")


def ints(a):
    return [int(x) for x in a]


def test_gen_omega_tables(cuda):
    import gen_omega_tables as got
    m = META["q3"]
    assert got.generate_table(m["omega"], m["q"], m["N"])[:4] == [1, m["omega"]] + \
        [pow(m["omega"], 2, m["q"]), pow(m["omega"], 3, m["q"])]
    assert got._ntt_dit(ints(ARR["q3_ntt_in"]), m["omega"], m["q"]) == ints(ARR["q3_ntt_out"])
    assert got._intt_dif(ints(ARR["q3_ntt_out"]), m["omega_inv"], m["n_inv"], m["q"]) == ints(ARR["q3_ntt_in"])
    tab = got.generate_table(m["omega"], m["q"], m["N"])
    itab = got.generate_table(m["omega_inv"], m["q"], m["N"])
    assert got.verify(m["N"], m["q"], m["omega"], m["omega_inv"], tab, itab) == []
    assert got.derive_omega(m["q"], m["N"], 11) == m["omega"]
    # the reference's default run crashes; the drop-in's default run verifies q=113, N=16
    assert got.main(["--verify-only"]) == 0


def test_gen_ntt_reference_and_vectors(cuda, tmp_path, monkeypatch):
    import gen_ntt_reference as ref
    t = META["toy"]
    for x, y in zip(ARR["toy_ntt_in"], ARR["toy_ntt_out"]):
        assert ref.ntt(ints(x), t["omega"], 16, t["q"]) == ints(y)
        assert ref.intt(ints(y), t["omega_inv"], 16, t["q"]) == ints(x)
    import gen_ntt_vectors as gv
    monkeypatch.setattr(gv, "SRC_DIR", str(tmp_path / "src"))
    monkeypatch.setattr(gv, "DST_DIR", str(tmp_path / "dst"))
    assert gv.main() == 0
    back = [int(l, 16) for l in open(tmp_path / "dst" / "ntt_in_all.hex") if l.strip()]
    assert back == [int(v) for v in ARR["toy_ntt_in"].reshape(-1)]
    back = [int(l, 16) for l in open(tmp_path / "dst" / "ntt_out_all.hex") if l.strip()]
    assert back == [int(v) for v in ARR["toy_ntt_out"].reshape(-1)]


def test_verify_keyswitch_dropin(cuda):
    import verify_keyswitch as vk
    chain = vk.load_chain()
    for got, want in zip(chain, META["chain4"]):
        for k in ("q", "primitive_root", "omega", "omega_inv", "N", "N_INV"):
            assert got[k] == want[k], k
    q = META["keyswitch"]["q"]
    for key in ("relin16", "relin64"):
        for e0, e1, e2, ka, kb, f0, f1 in ARR[key]:
            g0, g1 = vk.relin(ints(e0), ints(e1), ints(e2), ints(ka), ints(kb), q)
            assert g0 == ints(f0) and g1 == ints(f1)
    a, b, c = ARR["pmneg256"]
    assert vk.poly_mult(ints(a), ints(b), META["keyswitch"]["config_prime"]) == ints(c)
    a, b, c = ARR["pmneg16_q113"]
    assert vk.poly_mult(ints(a), ints(b), 113) == ints(c)
    random.seed(1)
    s = [random.randrange(q) for _ in range(16)]
    assert vk.check_random(q, s, n=200) == []
    assert vk.check_boundary(q, s) == []
    assert vk.main() == 0


def test_verify_rescale_dropin(cuda):
    import verify_rescale as vr
    primes = META["rescale"]["primes"]
    assert [r["q"] for r in vr.load_chain()] == primes
    for i in range(len(primes) - 1):
        got = vr.rescale_poly(ints(ARR[f"rescale_{i}_in"]), primes[i], primes[i + 1])
        assert got == ints(ARR[f"rescale_{i}_out"])
    assert vr.rescale_coeff(int(ARR["rescale_0_in"][7]), primes[0], primes[1]) == int(ARR["rescale_0_out"][7])
    assert vr.main() == 0


def test_verify_e2e_mult_dropin(cuda):
    import verify_e2e_mult as ve
    m = META["e2e"]
    for row in ARR["e2e16"]:
        c = [ints(r) for r in row]
        f0, f1 = ve.e2e_mult(*c[:6], m["q_in"], m["q_out"], m["scale_bits"])
        assert f0 == c[6] and f1 == c[7]
    assert ve.rescale(int(ARR["e2e_rescale_in"][3]), m["q_in"], m["q_out"], m["scale_bits"]) == \
        int(ARR["e2e_rescale_out"][3])
    assert ve.main() == 0


def test_golden_fc_layer_encrypted_forward(cuda):
    """FCLayerGoldenModel.encrypted_forward: the reference's FC1 shape
    (512 -> 128, Xavier-scaled N(0, 2/(in+out)) weights, seed 42;
    scripts/golden_fc_layer.py:28-54) evaluated under CKKS on the GPU (one
    ciphertext per input feature, the batch in the slots, weights quantised to
    2^20 inside the encrypted linear layer) equals the plaintext float
    forward within 1e-3 absolute (weight quantisation bounds the error by
    512 x 2^-21 x max|x| ~ 1e-3; CKKS noise is ~1e-9)."""
    import golden_fc_layer as fc

    m = fc.FCLayerGoldenModel(in_dim=512, out_dim=128, seed=42)
    rng = np.random.default_rng(7)
    x = rng.uniform(-1, 1, (16, 512))
    want = m.forward(x)
    got = m.encrypted_forward(x, log_n=13, levels=3, seed=1)
    assert got.shape == want.shape == (16, 128)
    assert np.abs(got - want).max() < 1e-3, np.abs(got - want).max()

"""Pin the CPU oracle to the reference: golden vectors produced by the
reference's own functions (tests/golden/make_golden.py), its committed twiddle
and modulus-chain fixtures (as digests) and its known-answer constants."""
import hashlib
import json
import random
from pathlib import Path

import numpy as np
import pytest

from oracle import golden as G
from oracle import ntt as ON
from oracle import rns_ckks as R
from oracle.modmath import (bitrev_perm, find_primes, is_prime, mulmod, primitive_root,
                            root_2n)

GD = Path(__file__).resolve().parent / "golden"
META = json.load(open(GD / "golden_core.json"))
ARR = np.load(GD / "golden_core.npz")


def sha(vals):
    h = hashlib.sha256()
    for v in vals:
        h.update(int(v).to_bytes(16, "little", signed=True))
    return h.hexdigest()


def ints(a):
    return [int(x) for x in a]


def test_toy_ntt_known_answers():
    t = META["toy"]
    q, n = t["q"], t["N"]
    assert pow(t["omega"], n, q) == 1 and t["omega"] * t["omega_inv"] % q == 1
    assert n * t["n_inv"] % q == 1
    assert pow(primitive_root(q), (q - 1) // n, q) == t["omega"]   # g=3 -> 40
    for x, y in zip(ARR["toy_ntt_in"], ARR["toy_ntt_out"]):
        assert ON.ntt_dit(ints(x), t["omega"], q) == ints(y)
        assert ON.intt_dit(ints(y), t["omega_inv"], t["n_inv"], q) == ints(x)


def test_q3_ntt_golden():
    m = META["q3"]
    assert m["verify_errors"] == []
    a = ints(ARR["q3_ntt_in"])
    assert ON.ntt_dit(a, m["omega"], m["q"]) == ints(ARR["q3_ntt_out"])
    # merged (GPU-order) cyclic transform == natural transform permuted
    fwd, inv = ON.merged_tables(m["N"], m["q"], None, m["omega"], cyclic=True)
    got = ON.merged_forward(np.array(a, dtype=np.uint64), m["q"], fwd)
    assert np.array_equal(got, ARR["q3_ntt_out"][bitrev_perm(m["N"])])
    back = ON.merged_inverse(got, m["q"], inv, m["n_inv"])
    assert np.array_equal(back, ARR["q3_ntt_in"])


def test_twiddle_fixture_digests():
    m = META["q3"]
    assert sha(G.generate_table(m["omega"], m["q"], m["N"])) == m["tw_sha"]
    assert sha(G.generate_table(m["omega_inv"], m["q"], m["N"])) == m["twinv_sha"]
    for rec in META["chain4"]:
        q, n = rec["q"], rec["N"]
        assert is_prime(q) and (q - 1) % (2 * n) == 0
        assert pow(rec["primitive_root"], (q - 1) // n, q) == rec["omega"]
        assert rec["omega"] * rec["omega_inv"] % q == 1 and n * rec["N_INV"] % q == 1
        assert sha(G.generate_table(rec["omega"], q, n)) == rec["tw_sha"]
        assert sha(G.generate_table(rec["omega_inv"], q, n)) == rec["twinv_sha"]


def test_rns_twiddle_fixture_heads():
    # p1/p2/p3 of rtl/m5/rns_split.sv:40-42 and q3: table starts 1, omega, omega^2 ...
    primes = {"p1": 77309411329, "p2": 206158430209, "p3": 2061584302081, "q3": 17592186175489}
    for key, rec in META["rns_tw"].items():
        kind, tag, nn = key.split("_")
        if tag not in primes:
            continue
        q, n = primes[tag], int(nn[1:])
        w = rec["head"][1]
        assert rec["head"][0] == 1 and pow(w, n, q) == 1 and pow(w, n // 2, q) == q - 1
        assert rec["len"] == n // 2
        if n <= 4096:
            assert sha(G.generate_table(w, q, n)) == rec["sha"]


def test_pm12_cyclic_vectors():
    m = META["pm12"]
    q, n = m["q"], m["N"]
    assert m["psi"] * m["psi"] % q == m["omega"]
    fwd, inv = ON.merged_tables(n, q, None, m["omega"], cyclic=True)
    for tag in ("rand0", "sparse"):
        a, b, c = ARR[f"pm12_{tag}_a"], ARR[f"pm12_{tag}_b"], ARR[f"pm12_{tag}_c"]
        fa = ON.merged_forward(a, q, fwd)
        fb = ON.merged_forward(b, q, fwd)
        got = ON.merged_inverse(mulmod(fa, fb, q), q, inv, m["n_inv"])
        assert np.array_equal(got, c)
        rec = [v for v in m["vectors"] if v["tag"] == tag][0]
        assert sha(c) == rec["c_sha"]


def test_negacyclic_poly_mult_golden():
    qc = META["keyswitch"]["config_prime"]
    a, b, c = ARR["pmneg256"]
    assert G.poly_mult(ints(a), ints(b), qc) == ints(c)
    got = ON.negacyclic_mul_ntt(a, b, qc, root_2n(qc, 256))
    assert np.array_equal(got, c)
    a, b, c = ARR["pmneg16_q113"]
    assert G.poly_mult(ints(a), ints(b), 113) == ints(c)


def test_relin_golden():
    q = META["keyswitch"]["q"]
    for key in ("relin16", "relin64"):
        for e0, e1, e2, ka, kb, f0, f1 in ARR[key]:
            g0, g1 = G.relin(ints(e0), ints(e1), ints(e2), ints(ka), ints(kb), q)
            assert g0 == ints(f0) and g1 == ints(f1)


def test_rescale_golden():
    primes = META["rescale"]["primes"]
    for i in range(len(primes) - 1):
        xin, xout = ARR[f"rescale_{i}_in"], ARR[f"rescale_{i}_out"]
        assert [G.rescale_coeff(int(c), primes[i], primes[i + 1]) for c in xin] == ints(xout)
    rng = random.Random(META["rescale"]["poly_seed"])
    poly = [rng.randrange(primes[0]) for _ in range(META["rescale"]["N"])]
    assert G.rescale_poly(poly, primes[0], primes[1]) == ints(ARR["rescale_poly_out"])


def test_e2e_golden():
    m = META["e2e"]
    for row in ARR["e2e16"]:
        c = [ints(r) for r in row]
        f0, f1 = G.e2e_mult(*c[:6], m["q_in"], m["q_out"], m["scale_bits"])
        assert f0 == c[6] and f1 == c[7]
    xs, ys = ARR["e2e_rescale_in"], ARR["e2e_rescale_out"]
    assert [G.rescale_scaled(int(x), m["q_in"], m["q_out"], m["scale_bits"]) for x in xs] == ints(ys)


def test_fastred_vectors_vs_numpy_mulmod():
    q = META["fastred"]["q"]
    got = mulmod(ARR["fastred_b"], ARR["fastred_w"], q)
    assert np.array_equal(got, ARR["fastred_out"])


def test_config_prime_and_chain():
    qc = 35184371884033
    assert is_prime(qc) and qc.bit_length() == 45 and (qc - 1) % (1 << 13) == 0
    # largest such prime: no prime of the form k*2^13+1 between qc and 2^45
    k = qc >> 13
    assert all(not is_prime(kk * 8192 + 1) for kk in range(k + 1, (1 << 45) >> 13))
    ch = find_primes(45, 1 << 14, 4)
    assert all(p.bit_length() == 45 and (p - 1) % (1 << 14) == 0 for p in ch)


@pytest.mark.parametrize("n,l", [(16, 2), (16, 3), (32, 3)])
def test_rns_oracle_matches_bigint(n, l):
    pr = find_primes(45, 1 << 14, l + 1)
    p, qs = pr[0], pr[1:]
    rng = np.random.default_rng(n * 10 + l)

    def rnd(shape, basis):
        x = np.zeros(shape, dtype=np.uint64)
        for i, q in enumerate(basis):
            x[..., i, :] = rng.integers(0, q, size=x[..., i, :].shape, dtype=np.uint64)
        return x

    a = rnd((1, 2, l, n), qs)
    b = rnd((1, 2, l, n), qs)
    ksk = rnd((l, 2, l + 1, n), qs + [p])
    assert np.array_equal(R.ct_mul_relin_rescale(a, b, ksk, qs, p)[0], R.bigint_ct_mul(a, b, ksk, qs, p))


# ---------------------------------------------------------------- second golden set
from oracle import encode as OE  # noqa: E402
from oracle import noise_gear as NG  # noqa: E402


def test_fc_golden_model_dropin_matches_reference():
    sys_path = str(Path(__file__).resolve().parents[1] / "cipher-pu_b200" / "scripts")
    import sys
    if sys_path not in sys.path:
        sys.path.insert(0, sys_path)
    import golden_fc_layer as fc
    f1, f2 = fc.build_mnist_cnn_model(512, 128, 10)
    assert np.array_equal(f1.weights, ARR["fc1_w"]) and np.array_equal(f2.weights, ARR["fc2_w"])
    y1, y1q = f1.test_forward(num_slots=4)
    assert np.array_equal(np.asarray(y1, dtype=np.float64), ARR["fc1_test_y"])
    assert np.array_equal(np.asarray(y1q, dtype=np.float64), ARR["fc1_test_yq"])
    y2, _ = f2.test_forward(num_slots=4)
    assert np.array_equal(np.asarray(y2, dtype=np.float64), ARR["fc2_test_y"])
    logits = f2.forward(np.maximum(f1.forward(ARR["fc_e2e_x"]), 0))
    assert np.array_equal(np.asarray(logits, dtype=np.float64), ARR["fc_e2e_logits"])


def test_slot_encode_decode_golden():
    m = META["simd"]
    for v, mm, dd in zip(ARR["simd_v"], ARR["simd_m"], ARR["simd_dec"]):
        assert np.allclose(OE.encode(v, m["scale"], m["N"]), mm, atol=1e-12)
        assert np.allclose(OE.decode(OE.encode(v, m["scale"], m["N"]), m["scale"], m["slots"]), dd, atol=1e-12)
    for x, y, z in zip(ARR["negfft_x"], ARR["negfft_y"], ARR["negifft_y"]):
        assert np.allclose(OE.pb_neg_fft(x), y, atol=1e-9)
        assert np.allclose(OE.pb_neg_ifft(x), z, atol=1e-12)
    # the scaled integer codec round-trips uniform [-1, 1] slots to ~1e-12 at Delta = 2^40
    rng = np.random.default_rng(0)
    s = rng.uniform(-1, 1, 2048)
    back = OE.ckks_decode(OE.ckks_encode(s, 2.0 ** 40, 4096), 2.0 ** 40, 2048)
    assert np.abs(back.real - s).max() < 1e-9


def test_noise_monitor_golden():
    for c in META["noise"]["cases"]:
        e, r = NG.noise_energy(c["coeffs"], c["q"])
        assert e == c["E"] and r == c["r_hat"]
        sw, rw = NG.welford(c["coeffs"], c["q"])
        assert abs(sw - c["sigma_w"]) <= 1e-9 * max(1.0, c["sigma_w"]) and abs(rw - c["r_hat_w"]) < 1e-15


def test_gear_controllers_golden():
    g = META["gear"]
    for rec, geo in zip(g["geo"], NG.GEO):
        assert NG.compute_extra(geo)[2] == rec["extra"] and NG.total_growth(geo) == rec["total_growth"]
    assert [NG.select_gear_safe(r) for r in g["r_sweep"]] == g["safe"]
    old, seq = 0, []
    for r in g["seq_r"]:
        old = NG.select_gear_with_hysteresis(NG.select_gear_safe(r), old, r)
        seq.append(old)
    assert seq == g["hyst"]
    assert [NG.gear_config(i) for i in range(6)] == g["gear_config"]
    assert NG.gear_config(2, 1234, True) == g["gear_config_ovr"]
    agc = NG.AgcRhat()
    assert [agc.step(r) for r in [0.05, 0.05, 0.05, 0.3, 0.3, 0.3, 0.15, 0.15, 0.15, 0.6, 0.6, 0.6]] == g["agc_seq"]


def test_rtl_gear_controller_semantics():
    # rtl/m4/adaptive_gear_ctrl.sv: reset gear 3; downgrade at once; upgrade after HYST_CNT
    c = NG.GearCtrlRTL(500, 200, 50, 3)
    assert c.flush(600) == 0            # downgrade immediately
    seq = [c.flush(10) for _ in range(5)]  # candidate 3 must be seen HYST_CNT+1 times
    assert seq == [0, 0, 0, 3, 3]
    assert c.flush(300) == 1
    assert c.flush(10, manual_en=True, manual_gear=2) == 2
    assert c.flush(10, hysteresis=False) == 3


def test_block_sparsity_golden():
    for rec in META["block_post"]:
        out, sk = NG.post_process_block(rec["x"], 20, True, 113, rec["B"])
        assert out == rec["out"] and sk == rec["skipped"]
    W = ARR["bsm_W"]
    for thr in (0.02, 0.05):
        mW, skip, tot, dens = NG.block_sparse_mask(W, thr, 4)
        assert np.array_equal(np.packbits(mW != 0), ARR[f"bsm_mask_{thr}"])
        rec = META[f"bsm_{thr}"]
        assert (skip, tot) == (rec["skip"], rec["total"]) and abs(dens - rec["density"]) < 1e-15


def test_dare_golden_semantics():
    q = META["dare"]["q"]
    s = ARR["dare_s"]
    b, a = ARR["dare_ct_b"], ARR["dare_ct_a"]
    # reference convention (b, a) -> (c0, c1) = (b, -a)
    c0, c1 = [int(x) % q for x in b], [(-int(x)) % q for x in a]
    a2 = ARR["dare_ct2_a"]
    new_c0, new_c1, dec = OE.dare_refresh(c0, c1, s, [(-int(x)) % q for x in a2], ARR["dare_e_new"], q)
    assert dec == [int(x) for x in ARR["dare_dec"]]
    assert new_c0 == [int(x) % q for x in ARR["dare_ct2_b"]]


def test_galois_oracle_matches_reference_goldens():
    """oracle.galois against scripts/exp_e24_rotation_bootstrap.py:143,167,189
    outputs (tests/golden/golden_rot.npz, made by make_golden.py --only rot)."""
    from oracle import galois as GA
    rot = np.load(GD / "golden_rot.npz")
    meta = json.load(open(GD / "golden_rot.json"))
    seen = set()
    for c in meta["cases"]:
        k, q, nu, n = c["key"], c["q"], c["nu"], c["n"]
        if c["kind"] == "automorphism_exact":
            got = GA.automorphism_coef(rot[k + "_in"], nu, q)
        elif c["kind"] == "poly_mul_x_power":
            got = GA.mul_monomial(rot[k + "_in"], nu, q)      # nu < N here: same as the reference
        else:
            s = np.mod(rot[k + "_in"], q).astype(np.uint64)
            got = GA.automorphism_coef(s, nu, q)
        assert np.array_equal(got, rot[k + "_out"]), c
        seen.add(c["kind"])
    assert seen == {"automorphism_exact", "poly_mul_x_power", "automorphism_key_exact"}


def test_activation_golden_fixture_consistent():
    """golden_act.json (scripts/golden_activation.py run by make_golden.py):
    with one segment, approximate(x) is the stored polynomial at x."""
    act = json.load(open(GD / "golden_act.json"))
    for name, m in act["models"]["order5_segments1"].items():
        seg = m["segments"][0]
        got = np.polyval(seg["poly_coeffs"], np.asarray(m["x"]))
        assert np.allclose(got, m["approx"], rtol=0, atol=1e-12), name
    sig = act["models"]["order5_segments1"]["sigmoid"]
    assert np.abs(np.asarray(sig["approx"]) - np.asarray(sig["exact"])).max() < 1e-3


def test_convgap_oracle_matches_reference_goldens():
    """scatter_w, mul_plain_exact, decrypt_exact, inner_product, coef_sum and
    the fused Conv + GAP inference of scripts/exp_e24_rotation_bootstrap.py
    (golden_convgap.*): integers bit-exact, floats identical."""
    from oracle import convgap as C
    d = np.load(GD / "golden_convgap.npz")
    m = json.load(open(GD / "golden_convgap.json"))
    q, n, sc = m["q"], m["N"], m["scale"]
    for k in m["scatter"]:
        assert np.array_equal(C.scatter_w(d[k + "_idx"], d[k + "_w"], sc, q, n), d[k + "_out"]), k
    assert np.array_equal(C.mul_plain(d["mp_in"], d["sc2_out"], q), d["mp_out"])
    assert np.array_equal(C.decrypt(d["mp_out"], d["s"], q), d["mp_dec"])
    for r in m["inner"]:
        ct = d[r["key"] + "_ct"]
        assert C.inner_product(ct, d[r["key"] + "_w"], d["s"], q, sc) == r["inner_product"]
        assert C.coef_sum(ct, r["dim"], d["s"], q, sc) == r["coef_sum"]
        assert abs(r["inner_product"] - r["plain_dot"]) < 0.05
    for r in m["fused"]:
        k = r["key"]
        lg, mc = C.fused_inference(d[k + "_ct"], d["s"], q, sc, d["conv_w"], d["conv_b"], d["fc_w"], d["fc_b"])
        assert np.array_equal(lg, d[k + "_logits"]) and mc == r["mult_count"]
        assert np.max(np.abs(lg - d[k + "_plain"])) < 5e-3

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

"""Drop-in for the reference's scripts/verify_e2e_mult.py (single-modulus ct-mult).

Same names and integer semantics: N, NUM_TESTS, SCALE_BITS, ``load_chain``,
``poly_add``, ``poly_sub``, ``poly_mult``, ``rescale`` (floor((s q_out +
q_in/2) / (q_in 2^scale_bits)) mod q_out), ``e2e_mult`` (tensor product,
single-pair relinearisation, scaled rescale), ``check_output_range``,
``encrypt`` and ``main``.  All polynomial products run as one batched GPU
call per ``e2e_mult``; the rescale runs on the GPU as well.
"""
from __future__ import annotations

import random
import sys

import _bootstrap  # noqa: F401
from ckks_b200 import golden_bridge as gb
from verify_keyswitch import load_chain, poly_add, poly_mult, poly_sub  # noqa: F401

N = 16384
NUM_TESTS = 10
SCALE_BITS = 30


def rescale(s, q_in, q_out, scale_bits):
    return gb.rescale_scaled([s], q_in, q_out, scale_bits)[0]


def e2e_mult(c0_1, c1_1, c0_2, c1_2, a, b, q_in, q_out, scale_bits):
    m0, m1a, m1b, m2 = gb.poly_mult_many([c0_1, c0_1, c1_1, c1_1], [c0_2, c1_2, c0_2, c1_2], q_in)
    m1 = poly_add(m1a, m1b, q_in)
    e2a, e2b = gb.poly_mult_many([m2, m2], [a, b], q_in)
    f0 = poly_add(m0, e2b, q_in)
    f1 = poly_sub(m1, e2a, q_in)
    return (gb.rescale_scaled(f0, q_in, q_out, scale_bits),
            gb.rescale_scaled(f1, q_in, q_out, scale_bits))


def encrypt(m, s, e_noise, q, a_pk, b_pk):
    return poly_add(m, e_noise, q), a_pk


def check_output_range(f0, f1, q_out):
    for i, (x, y) in enumerate(zip(f0, f1)):
        if not (0 <= x < q_out):
            return [f"f0'[{i}]={x} out of range"]
        if not (0 <= y < q_out):
            return [f"f1'[{i}]={y} out of range"]
    return []


def main():
    chain = load_chain()
    q_in, q_out = chain[0]["q"], chain[1]["q"]
    n_toy = 16
    rng = random.Random(42)
    s = [rng.randrange(q_in) for _ in range(n_toy)]
    a_ks = [rng.randrange(q_in) for _ in range(n_toy)]
    e_ks = [rng.randrange(100) for _ in range(n_toy)]
    b_ks = poly_add(poly_mult(a_ks, s, q_in), e_ks, q_in)
    all_pass = True
    print("[1] output range [GPU]")
    for t in range(NUM_TESTS):
        c = [[rng.randrange(q_in) for _ in range(n_toy)] for _ in range(4)]
        f0, f1 = e2e_mult(*c, a_ks, b_ks, q_in, q_out, SCALE_BITS)
        errs = check_output_range(f0, f1, q_out)
        print(f"  [{'FAIL' if errs else 'OK'}]   test {t}")
        all_pass &= not errs
    print("result:", "ALL PASS" if all_pass else "FAIL")
    return 0 if all_pass else 1


if __name__ == "__main__":
    sys.exit(main())

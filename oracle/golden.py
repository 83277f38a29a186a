"""Restatement of the reference's single-modulus golden models (test infrastructure).

* ``poly_mult``       scripts/verify_keyswitch.py:48 (negacyclic schoolbook,
                      identical to scripts/verify_e2e_mult.py:56)
* ``poly_add/sub``    scripts/verify_keyswitch.py:40,44
* ``relin``           scripts/verify_keyswitch.py:62
* ``rescale_coeff``   scripts/verify_rescale.py:38 (round half up)
* ``rescale_scaled``  scripts/verify_e2e_mult.py:70
* ``e2e_mult``        scripts/verify_e2e_mult.py:78
* ``poly_mult_cyclic`` tb/ref/gen_poly_mult_vectors_n12.py:110 (schoolbook cyclic)

Python integers throughout (exact); the schoolbook products are vectorised
with object arrays so N = 4096 checks finish in seconds.
"""
from __future__ import annotations

import numpy as np


def poly_add(a, b, q):
    return [(x + y) % q for x, y in zip(a, b)]


def poly_sub(a, b, q):
    return [(x - y) % q for x, y in zip(a, b)]


def _conv_full(a, b):
    """Exact integer linear convolution (object dtype)."""
    a = np.asarray([int(x) for x in a], dtype=object)
    b = np.asarray([int(x) for x in b], dtype=object)
    n = len(a)
    out = np.zeros(2 * n - 1, dtype=object)
    for i in range(n):
        if a[i]:
            out[i:i + n] += a[i] * b
    return out


def poly_mult(a, b, q):
    """Negacyclic product mod (X^N + 1, q)."""
    n = len(a)
    full = _conv_full(a, b)
    res = full[:n].copy()
    res[:n - 1] -= full[n:]
    return [int(x) % q for x in res]


def poly_mult_cyclic(a, b, q):
    n = len(a)
    full = _conv_full(a, b)
    res = full[:n].copy()
    res[:n - 1] += full[n:]
    return [int(x) % q for x in res]


def relin(e0, e1, e2, a, b, q):
    """f0 = e0 + e2 b, f1 = e1 - e2 a (mod q)."""
    return poly_add(e0, poly_mult(e2, b, q), q), poly_sub(e1, poly_mult(e2, a, q), q)


def rescale_coeff(c, q_in, q_out):
    """round(c q_out / q_in) mod q_out, halves rounded up."""
    t = c * q_out
    r, rem = divmod(t, q_in)
    if 2 * rem >= q_in:
        r += 1
    return r % q_out


def rescale_poly(c, q_in, q_out):
    return [rescale_coeff(x, q_in, q_out) for x in c]


def rescale_scaled(s, q_in, q_out, scale_bits):
    return ((s * q_out + q_in // 2) // (q_in << scale_bits)) % q_out


def e2e_mult(c0_1, c1_1, c0_2, c1_2, a, b, q_in, q_out, scale_bits):
    m0 = poly_mult(c0_1, c0_2, q_in)
    m1 = poly_add(poly_mult(c0_1, c1_2, q_in), poly_mult(c1_1, c0_2, q_in), q_in)
    m2 = poly_mult(c1_1, c1_2, q_in)
    f0 = poly_add(m0, poly_mult(m2, b, q_in), q_in)
    f1 = poly_sub(m1, poly_mult(m2, a, q_in), q_in)
    return ([rescale_scaled(x, q_in, q_out, scale_bits) for x in f0],
            [rescale_scaled(x, q_in, q_out, scale_bits) for x in f1])


def generate_table(omega, q, n):
    """omega^k, k < N/2 (scripts/gen_omega_tables.py:96 generate_table)."""
    t = [1] * (n // 2)
    for k in range(1, n // 2):
        t[k] = t[k - 1] * omega % q
    return t

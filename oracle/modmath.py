"""Scalar and vectorised modular arithmetic for the oracle (test infrastructure).

* ``is_prime`` / ``primitive_root`` restate the reference's parameter generator
  (scripts/gen_omega_tables.py:40 ``is_prime`` — Miller-Rabin with the first
  twelve prime bases — and :63 ``primitive_root``; same algorithm as
  scripts/gen_modulus_chain.py:40,63).
* ``mulmod`` is an exact vectorised 64-bit modular multiply for moduli below
  2^50 on numpy uint64 arrays: the quotient is estimated in float64 and the
  remainder is formed with wrapping uint64 products, then corrected by +-q.
"""
from __future__ import annotations

import numpy as np

U64 = np.uint64
_BASES = (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37)


def is_prime(n: int) -> bool:
    """Miller-Rabin with fixed bases (scripts/gen_omega_tables.py:40-60)."""
    if n < 2:
        return False
    for p in _BASES:
        if n % p == 0:
            return n == p
    d, s = n - 1, 0
    while d % 2 == 0:
        d //= 2
        s += 1
    for a in _BASES:
        x = pow(a, d, n)
        if x == 1 or x == n - 1:
            continue
        for _ in range(s - 1):
            x = x * x % n
            if x == n - 1:
                break
        else:
            return False
    return True


def primitive_root(p: int) -> int:
    """Smallest generator of Z_p^* (scripts/gen_omega_tables.py:63-80)."""
    pm1 = p - 1
    n = pm1
    fset = set()
    d = 2
    while d * d <= n:
        while n % d == 0:
            n //= d
            fset.add(d)
        d += 1
    if n > 1:
        fset.add(n)
    for g in range(2, p):
        if all(pow(g, pm1 // f, p) != 1 for f in fset):
            return g
    raise RuntimeError("no primitive root")


def find_primes(bits: int, modulus_pow2: int, count: int) -> list[int]:
    """``count`` largest primes below 2^bits with q = 1 mod modulus_pow2.

    Same search order as scripts/gen_modulus_chain.py:97 ``find_k_primes``
    (descending k in q = k*M + 1)."""
    out = []
    k = ((1 << bits) - 1) // modulus_pow2
    while len(out) < count and k > 0:
        q = k * modulus_pow2 + 1
        if q < (1 << bits) and is_prime(q):
            out.append(q)
        k -= 1
    return out


def bit_reverse(i: int, bits: int) -> int:
    r = 0
    for _ in range(bits):
        r = (r << 1) | (i & 1)
        i >>= 1
    return r


def bitrev_perm(n: int) -> np.ndarray:
    bits = n.bit_length() - 1
    return np.array([bit_reverse(i, bits) for i in range(n)], dtype=np.int64)


def root_2n(q: int, n: int) -> int:
    """A primitive 2n-th root of unity mod q: g^((q-1)/2n) with g the smallest
    generator (the psi of tb/ref/gen_poly_mult_vectors_n12.py:44)."""
    assert (q - 1) % (2 * n) == 0
    return pow(primitive_root(q), (q - 1) // (2 * n), q)


def root_n(q: int, n: int) -> int:
    """omega = g^((q-1)/n) (scripts/gen_omega_tables.py:85 ``derive_omega``)."""
    assert (q - 1) % n == 0
    return pow(primitive_root(q), (q - 1) // n, q)


# ----------------------------------------------------------------- numpy
def _as_u64(x):
    return np.asarray(x, dtype=np.uint64)


def mulmod(a, b, q):
    """Exact (a*b) mod q elementwise; a, b in [0, 2^50), q < 2^50 (scalar or
    broadcastable array).  Result in [0, q)."""
    a = _as_u64(a)
    b = _as_u64(b)
    qa = _as_u64(q)
    quot = np.floor(a.astype(np.float64) * b.astype(np.float64) / qa.astype(np.float64))
    quot = quot.astype(np.uint64)
    with np.errstate(over="ignore"):
        r = (a * b - quot * qa).view(np.int64)
    qi = qa.astype(np.int64)
    r = np.where(r < 0, r + qi, r)
    r = np.where(r < 0, r + qi, r)
    r = np.where(r >= qi, r - qi, r)
    r = np.where(r >= qi, r - qi, r)
    return r.astype(np.uint64)


def addmod(a, b, q):
    a = _as_u64(a)
    b = _as_u64(b)
    qa = _as_u64(q)
    s = a + b
    return np.where(s >= qa, s - qa, s).astype(np.uint64)


def submod(a, b, q):
    a = _as_u64(a)
    b = _as_u64(b)
    qa = _as_u64(q)
    return np.where(a >= b, a - b, a + qa - b).astype(np.uint64)


def negmod(a, q):
    a = _as_u64(a)
    qa = _as_u64(q)
    return np.where(a == 0, a, qa - a).astype(np.uint64)


def center(a, q):
    """Map [0, q) to the centred representative in (-q/2, q/2] as int64."""
    a = _as_u64(a).astype(np.int64)
    qi = np.asarray(q, dtype=np.int64)
    return np.where(a > qi // 2, a - qi, a)


def reduce_signed(x, q):
    """Signed int64 array -> [0, q) uint64."""
    x = np.asarray(x, dtype=np.int64)
    qi = np.asarray(q, dtype=np.int64)
    return np.mod(x, qi).astype(np.uint64)

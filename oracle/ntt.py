"""NTT restatements for the oracle (test infrastructure).

Two families:

1. The reference's own cyclic NTT (pure Python ints, natural order):
   ``ntt_dit`` restates scripts/gen_omega_tables.py:154 ``_ntt_dit`` (identical
   to tb/ref/gen_ntt_reference.py:78 ``ntt`` and
   tb/ref/gen_poly_mult_vectors_n12.py:68 ``ntt``): bit-reversal permutation,
   then radix-2 Cooley-Tukey DIT with stage base w_len = omega^(N/len) and a
   running ``w *= w_len``.  ``intt_dit`` restates :188 ``_intt_dif`` (same loop
   with omega^-1, then * N^-1).

2. The "merged" negacyclic / cyclic transform the GPU runs, vectorised in numpy:
   natural-order coefficients in, evaluations in bit-reversed order out
   (Cooley-Tukey, twiddle ``tw[m + i]`` for group i of stage m), and the
   Gentleman-Sande inverse.  For the negacyclic ring ``tw[k] = psi^brv(k)``;
   for the cyclic ring ``tw[m+i] = omega^((brv(m+i) - N/(2m))/2)``.  The relation
   to family 1 is pinned in tests: merged_forward(a) == nat[bitrev] where
   nat = ntt_dit(a * psi^j) (negacyclic) or ntt_dit(a) (cyclic).
"""
from __future__ import annotations

import numpy as np

from .modmath import bit_reverse, mulmod, addmod, submod


# ------------------------------------------------------------ reference family
def _bitrev_list(a):
    n = len(a)
    a = list(a)
    j = 0
    for i in range(1, n):
        bit = n >> 1
        while j & bit:
            j ^= bit
            bit >>= 1
        j ^= bit
        if i < j:
            a[i], a[j] = a[j], a[i]
    return a


def ntt_dit(a, omega, q):
    """Cyclic NTT, natural in / natural out (scripts/gen_omega_tables.py:154)."""
    n = len(a)
    a = _bitrev_list(a)
    length = 2
    while length <= n:
        w_len = pow(omega, n // length, q)
        for i in range(0, n, length):
            w = 1
            for k in range(length // 2):
                u = a[i + k]
                v = a[i + k + length // 2] * w % q
                a[i + k] = (u + v) % q
                a[i + k + length // 2] = (u - v) % q
                w = w * w_len % q
        length <<= 1
    return a


def intt_dit(a_hat, omega_inv, n_inv, q):
    """Inverse of ``ntt_dit`` (scripts/gen_omega_tables.py:188 ``_intt_dif``)."""
    return [x * n_inv % q for x in ntt_dit(a_hat, omega_inv, q)]


def cyclic_conv_direct(a, b, q):
    """O(N^2) cyclic convolution (tb/ref/gen_poly_mult_vectors_n12.py:110)."""
    n = len(a)
    return [sum(a[k] * b[(i - k) % n] for k in range(n)) % q for i in range(n)]


# ------------------------------------------------------------ twiddle tables
def merged_tables(n: int, q: int, psi: int | None, omega: int | None, cyclic: bool):
    """(fwd, inv) twiddle tables of length n (index 0 unused) for the merged
    transform.  Negacyclic: fwd[k] = psi^brv(k), inv[k] = psi^-brv(k).
    Cyclic: fwd[m+i] = omega^((brv(m+i) - n/(2m))/2), inv = its inverse."""
    logn = n.bit_length() - 1
    fwd = [0] * n
    inv = [0] * n
    if cyclic:
        oinv = pow(omega, -1, q)
        m = 1
        while m < n:
            for i in range(m):
                e = (bit_reverse(m + i, logn) - n // (2 * m)) // 2
                fwd[m + i] = pow(omega, e, q)
                inv[m + i] = pow(oinv, e, q)
            m <<= 1
    else:
        pinv = pow(psi, -1, q)
        for k in range(1, n):
            e = bit_reverse(k, logn)
            fwd[k] = pow(psi, e, q)
            inv[k] = pow(pinv, e, q)
    return np.array(fwd, dtype=np.uint64), np.array(inv, dtype=np.uint64)


# ------------------------------------------------------------ merged transforms
def merged_forward(x, q, fwd):
    """Batched merged CT forward NTT over the last axis (numpy uint64).
    x values in [0, q); q scalar or array broadcastable to x[..., :1];
    fwd shape (n,) or broadcastable (..., n)."""
    x = np.array(x, dtype=np.uint64, copy=True)
    n = x.shape[-1]
    lead = x.shape[:-1]
    q = np.asarray(q, dtype=np.uint64)
    qb = q.reshape(q.shape + (1, 1)) if q.ndim else q
    t = n
    m = 1
    while m < n:
        t //= 2
        v = x.reshape(lead + (m, 2, t))
        w = np.asarray(fwd)[..., m:2 * m]
        w = w.reshape(w.shape[:-1] + (m, 1))
        u = v[..., 0, :]
        vv = mulmod(v[..., 1, :], w, qb)
        a = addmod(u, vv, qb)
        b = submod(u, vv, qb)
        x = np.stack([a, b], axis=-2).reshape(lead + (n,))
        m *= 2
    return x


def merged_inverse(x, q, inv, n_inv):
    """Batched Gentleman-Sande inverse of ``merged_forward`` (includes N^-1)."""
    x = np.array(x, dtype=np.uint64, copy=True)
    n = x.shape[-1]
    lead = x.shape[:-1]
    q = np.asarray(q, dtype=np.uint64)
    qb = q.reshape(q.shape + (1, 1)) if q.ndim else q
    t = 1
    m = n // 2
    while m >= 1:
        v = x.reshape(lead + (m, 2, t))
        w = np.asarray(inv)[..., m:2 * m]
        w = w.reshape(w.shape[:-1] + (m, 1))
        u = v[..., 0, :]
        vv = v[..., 1, :]
        a = addmod(u, vv, qb)
        b = mulmod(submod(u, vv, qb), w, qb)
        x = np.stack([a, b], axis=-2).reshape(lead + (n,))
        t *= 2
        m //= 2
    qs = q.reshape(q.shape + (1,)) if q.ndim else q
    return mulmod(x, np.asarray(n_inv, dtype=np.uint64).reshape(np.shape(qs)), qs)


def negacyclic_mul_ntt(a, b, q, psi):
    """Negacyclic product via the merged transform (numpy, one prime)."""
    n = np.shape(a)[-1]
    fwd, inv = merged_tables(n, q, psi, None, cyclic=False)
    fa = merged_forward(a, q, fwd)
    fb = merged_forward(b, q, fwd)
    return merged_inverse(mulmod(fa, fb, q), q, inv, pow(n, -1, q))

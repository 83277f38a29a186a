"""FP64 slot encoding and the DARE refresh (test infrastructure).

* ``neg_fft`` / ``neg_ifft`` / ``encode`` / ``decode`` restate
  scripts/verify_multi_slot_simd.py:32,42,75,88: slot k is the evaluation at
  Phi^(2k+1) (Phi = exp(i pi / N)), its conjugate sits at N-1-k, and a real
  coefficient polynomial is obtained from the Hermitian-completed vector.
  The O(N^2) sums are evaluated with np.fft (same values to rounding).
* ``pb_neg_fft`` / ``pb_neg_ifft`` restate the differently defined pair of
  scripts/verify_project_b_mlp_reference.py:60,73 (FFT then per-bin twiddle).
* ``ckks_encode`` / ``ckks_decode``: scale-Delta integer encoding used by the
  GPU path (round(Delta * encode) per coefficient; decode divides by Delta).
* ``dare_refresh`` restates scripts/exp_e24_rotation_bootstrap.py:287
  ``reencrypt`` (decrypt to the centred integer m_int + e_old, re-encrypt it
  with fresh a and small e) in the c0 + c1 s convention used here; a reference
  ciphertext (b, a) with b = a s + e + m maps to (c0, c1) = (b, -a).
"""
from __future__ import annotations

import numpy as np


def neg_fft(m):
    m = np.asarray(m, dtype=np.complex128)
    n = len(m)
    j = np.arange(n)
    phi = np.exp(1j * np.pi * j / n)
    return n * np.fft.ifft(m * phi)


def neg_ifft(V):
    V = np.asarray(V, dtype=np.complex128)
    n = len(V)
    j = np.arange(n)
    return np.fft.fft(V) * np.exp(-1j * np.pi * j / n) / n


def encode(v, scale, n):
    V = np.zeros(n, dtype=np.complex128)
    ns = len(v)
    for k in range(ns):
        V[k] = scale * v[k]
        sk = n - 1 - k
        if sk != k and sk >= ns:
            V[sk] = np.conj(V[k])
    return neg_ifft(V).real


def decode(m, scale, nslot):
    return neg_fft(np.asarray(m, dtype=float)).real[:nslot] / scale


def pb_neg_fft(x):
    x = np.asarray(x, dtype=np.complex128)
    n = len(x)
    k = np.arange(n)
    return np.fft.fft(x) * np.exp(1j * np.pi / n) ** (2 * k + 1)


def pb_neg_ifft(X):
    X = np.asarray(X, dtype=np.complex128)
    n = len(X)
    k = np.arange(n)
    return np.fft.ifft(X * np.exp(1j * np.pi / n) ** (-(2 * k + 1)))


def ckks_encode(slots, delta, n):
    """Complex slots (len <= n/2) -> integer coefficients round(Delta * m)."""
    slots = np.asarray(slots, dtype=np.complex128)
    V = np.zeros(n, dtype=np.complex128)
    ns = len(slots)
    V[:ns] = slots
    V[n - 1 - np.arange(ns)] = np.conj(slots)
    m = neg_ifft(V).real
    return np.round(delta * m).astype(np.int64)


def ckks_decode(coeffs, delta, nslot):
    """Integer (or float) coefficients -> complex slots / Delta."""
    V = neg_fft(np.asarray(coeffs, dtype=np.float64))
    return V[:nslot] / delta


def dare_refresh(c0, c1, s, a_new, e_new, q):
    """Single-modulus DARE in the c0 + c1 s convention (coefficient domain,
    exact integers).  Returns (new_c0, new_c1, dec) with dec the centred
    decryption m_int + e_old."""
    from .golden import poly_mult
    n = len(c0)
    c1s = poly_mult([int(x) % q for x in c1], [int(x) % q for x in s], q)
    dec = [(int(c0[i]) + c1s[i]) % q for i in range(n)]
    dec_c = [d - q if d > q // 2 else d for d in dec]
    a_s = poly_mult([int(x) % q for x in a_new], [int(x) % q for x in s], q)
    new_c0 = [(dec_c[i] + int(e_new[i]) - a_s[i]) % q for i in range(n)]
    return new_c0, [int(x) % q for x in a_new], dec_c

"""Coefficient-encoded inner products and the Conv + GAP fusion (test
infrastructure: the checker of csrc/convgap.cu and ckks_b200/convgap.py).

* ``scatter_w`` restates scripts/exp_e24_rotation_bootstrap.py:241: weight
  w_j of message index m_j goes to coefficient N - m_j of an integer
  polynomial at scale Delta (m_j = 0: coefficient 0, negated), so the
  constant coefficient of (message x weights) in Z_q[X]/(X^N + 1) is
  -Delta * sum_j x_{m_j} w_j.  Repeated indices add up.
* ``mul_plain`` is :136 ``mul_plain_exact``: both ciphertext polynomials
  times the plaintext polynomial, exact negacyclic products mod q.
* ``decrypt`` is :109 ``decrypt_exact``: (b - a s) mod q, centred.
* ``inner_product`` / ``coef_sum`` are :263 / :278: one ciphertext product
  and the constant coefficient of its decryption, -dec_0 / Delta^2.
* ``conv_gap_indices`` / ``fused_inference`` are :615
  ``encrypted_inference_fused``: for each of the 4 filters of a
  Conv(1->4, 3x3, stride 4, pad 1) on a 28 x 28 image, the 49 positions x 9
  taps collapse into one scattered weight polynomial, so conv + global
  average pool is one ciphertext product per filter; the 4 pooled values go
  through the plaintext FC(4 -> 10).
"""
from __future__ import annotations

import numpy as np

from .modmath import root_2n
from .ntt import negacyclic_mul_ntt


def scatter_w(msg_indices, w, scale: int, q: int, n: int) -> np.ndarray:
    m_w = np.zeros(n, dtype=np.int64)
    for j, mi in enumerate(msg_indices):
        val = int(round(scale * float(w[j])))  # Python round: half to even, as the reference
        if mi % n == 0:
            m_w[0] -= val
        else:
            m_w[n - (mi % n)] += val
    return np.mod(m_w, q).astype(np.uint64)


def _negmul(a, b, q: int) -> np.ndarray:
    n = np.shape(a)[-1]
    return negacyclic_mul_ntt(np.asarray(a, dtype=np.uint64) % np.uint64(q),
                              np.asarray(b, dtype=np.uint64) % np.uint64(q), q, root_2n(q, n))


def mul_plain(ct, p, q: int) -> np.ndarray:
    """ct = (b, a) as a [2, N] array -> [2, N] (b p, a p) mod q."""
    ct = np.asarray(ct)
    return np.stack([_negmul(ct[0], p, q), _negmul(ct[1], p, q)])


def decrypt(ct, s, q: int) -> np.ndarray:
    """Centred (b - a s) mod q as int64; s given as integers (any sign)."""
    ct = np.asarray(ct)
    s_q = (np.asarray(s, dtype=np.int64) % q).astype(np.uint64)
    a_s = _negmul(ct[1], s_q, q).astype(np.int64)
    d = (np.asarray(ct[0], dtype=np.int64) % q - a_s) % q
    return np.where(d > q // 2, d - q, d).astype(np.int64)


def inner_product(ct, w, s, q: int, scale: int, msg_indices=None) -> float:
    w = np.asarray(w, dtype=np.float64)
    if msg_indices is None:
        msg_indices = list(range(len(w)))
    m_w = scatter_w(msg_indices, w, scale, q, np.shape(ct)[-1])
    dec = decrypt(mul_plain(ct, m_w, q), s, q)
    return -float(dec[0]) / (scale * scale)


def coef_sum(ct, dim: int, s, q: int, scale: int) -> float:
    return inner_product(ct, np.ones(dim), s, q, scale)


def conv_gap_indices(w_filter) -> tuple[list[int], list[float]]:
    """Message indices and weights of one 3 x 3 filter over the 7 x 7 output
    positions (stride 4, padding 1) of a 28 x 28 image, row-major pixels."""
    idx, vals = [], []
    for i in range(7):
        for j in range(7):
            for ki in range(3):
                for kj in range(3):
                    ii, jj = 4 * i + ki - 1, 4 * j + kj - 1
                    if 0 <= ii < 28 and 0 <= jj < 28:
                        idx.append(ii * 28 + jj)
                        vals.append(float(w_filter[ki, kj]))
    return idx, vals


def fused_inference(ct, s, q: int, scale: int, conv_w, conv_b, fc_w, fc_b):
    """Logits and product count of the fused model on one encrypted image."""
    gap = np.zeros(len(conv_b))
    for f in range(len(conv_b)):
        idx, vals = conv_gap_indices(np.asarray(conv_w)[f, 0])
        # the reference adds its float32 conv bias to a Python float, which
        # NumPy >= 2 evaluates in float32: the pooled value is float32-rounded
        gap[f] = np.float32(inner_product(ct, vals, s, q, scale, msg_indices=idx) / 49.0) + np.float32(conv_b[f])
    fc_w = np.asarray(fc_w, dtype=np.float64)
    logits = np.array([float(np.dot(gap, fc_w[o])) + float(fc_b[o]) for o in range(len(fc_b))])
    return logits, len(conv_b) + len(fc_b)

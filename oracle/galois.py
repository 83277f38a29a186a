"""Automorphisms, monomial products and the Galois key switch (test
infrastructure: the checker of csrc/galois.cu and ckks_rotate).

* ``automorphism_coef`` restates scripts/exp_e24_rotation_bootstrap.py:143
  ``automorphism_exact`` (and :167 ``automorphism_key_exact``): coefficient k
  of f goes to j = nu k mod N with sign (-1)^floor(nu k / N), colliding terms
  are summed mod q (any nu; a signed permutation for odd nu).
* ``mul_monomial`` is f * X^nu in Z_q[X]/(X^N + 1) with nu mod 2N; the
  reference's ``poly_mul_x_power`` (:189) and ``rotate`` (:232) reduce nu mod
  N first, which agrees for nu < N.
* ``automorphism_eval`` is the same map on the bit-reversed evaluation vector
  of the merged negacyclic NTT (slot i = f(psi^(2 brv(i) + 1))): a permutation.
* ``galois_key`` / ``rotate``: the hybrid key switch of ``rns_ckks.keyswitch``
  applied to psi_nu(c1) with a key for psi_nu(s); no rescale.
"""
from __future__ import annotations

import numpy as np

from .modmath import addmod, bitrev_perm, mulmod, negmod
from .rns_ckks import keyswitch, ntt


def automorphism_coef(f, nu: int, q: int) -> np.ndarray:
    f = np.asarray(f, dtype=np.uint64) % np.uint64(q)
    n = f.shape[-1]
    k = np.arange(n, dtype=object)
    p = np.array([(int(nu) * int(x)) for x in k], dtype=object)
    j = np.array([int(x) % n for x in p], dtype=np.int64)
    neg = np.array([(int(x) // n) % 2 == 1 for x in p])
    out = np.zeros(f.shape, dtype=np.uint64)
    flat_in = f.reshape(-1, n)
    flat_out = out.reshape(-1, n)
    for r in range(flat_in.shape[0]):
        acc = [0] * n
        for kk in range(n):
            v = int(flat_in[r, kk])
            acc[j[kk]] += (q - v) % q if neg[kk] else v
        flat_out[r] = np.array([a % q for a in acc], dtype=np.uint64)
    return out


def mul_monomial(f, nu: int, q: int) -> np.ndarray:
    f = np.asarray(f, dtype=np.uint64) % np.uint64(q)
    n = f.shape[-1]
    nu = int(nu) % (2 * n)
    p = (np.arange(n) + nu) % (2 * n)
    j = p % n
    neg = p >= n
    out = np.empty_like(f)
    vals = np.where(neg & (f != 0), np.uint64(q) - f, f)
    out[..., j] = vals
    return out


def automorphism_eval(x, nu: int) -> np.ndarray:
    x = np.asarray(x, dtype=np.uint64)
    n = x.shape[-1]
    log_n = n.bit_length() - 1
    br = bitrev_perm(n)
    i = np.arange(n)
    e = ((2 * br[i] + 1) * (int(nu) % (2 * n))) % (2 * n)
    src = br[(e - 1) // 2]
    assert log_n >= 1
    return x[..., src]


def galois_key(s_coef, nu: int, qs, p, a_eval, e_coef) -> np.ndarray:
    """ksk[j][0] = -a_j s + e_j + delta_ij (p mod q_j) psi_nu(s), ksk[j][1] = a_j,
    evaluation domain over (qs, p)."""
    qs = [int(q) for q in qs]
    basis = qs + [int(p)]
    n = len(s_coef)
    dnum = len(qs)
    s64 = np.asarray(s_coef, dtype=np.int64)
    ksk = np.zeros((dnum, 2, len(basis), n), dtype=np.uint64)
    for r, q in enumerate(basis):
        s_eval = ntt(np.mod(s64, q).astype(np.uint64), q, n)
        ps_eval = automorphism_eval(s_eval, nu)
        for j in range(dnum):
            e = ntt(np.mod(np.asarray(e_coef[j], dtype=np.int64), q).astype(np.uint64), q, n)
            b = addmod(negmod(mulmod(a_eval[j, r], s_eval, q), q), e, q)
            if r == j:
                b = addmod(b, mulmod(ps_eval, np.uint64(int(p) % q), q), q)
            ksk[j, 0, r] = b
            ksk[j, 1, r] = a_eval[j, r]
    return ksk


def rotate(ct, gk, nu: int, qs, p) -> np.ndarray:
    """ct [B, 2, l, N] evaluation domain -> [B, 2, l, N]: (psi(c0) + ks0, ks1)
    with ks the hybrid key switch of psi(c1) under the Galois key gk."""
    qs = [int(q) for q in qs]
    l = ct.shape[2]
    big_l = gk.shape[2] - 1
    c0 = automorphism_eval(ct[:, 0], nu)
    c1 = automorphism_eval(ct[:, 1], nu)
    sub = gk[:l][:, :, list(range(l)) + [big_l]]
    ks = keyswitch(c1, sub, qs, int(p))
    qv = np.asarray(qs, dtype=np.uint64)[:, None]
    return np.stack([addmod(c0, ks[:, 0], qv), ks[:, 1]], axis=1)

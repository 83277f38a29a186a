"""RNS-CKKS restatement for the oracle (test infrastructure).

The reference has no RNS keyswitch or RNS rescale (its keyswitch is one
(a, b) pair over a single modulus, scripts/verify_keyswitch.py:62, and its
rescale is a single-modulus switch, scripts/verify_rescale.py:38).  This
module states, from the CKKS mathematics, the algorithm the GPU path
implements, with numpy over uint64 residues:

  * tensor product  d0 = a0 b0, d1 = a0 b1 + a1 b0, d2 = a1 b1
    (scripts/verify_e2e_mult.py:83-90 structure, per RNS limb);
  * hybrid keyswitch with dnum = level digits (digit j = [d2]_{q_j} taken as
    an integer in [0, q_j)), one special prime p:
       ModUp:   digit_j -> every prime of {q_0..q_{l-1}, p}
       key inner product: acc_k = sum_j digit_j * ksk[j][k]
       ModDown: ks_k = (acc_k - [centred(acc_k mod p)]_{q_i}) * p^-1 mod q_i
    (the single-pair f0 = e0 + e2 b, f1 = e1 - e2 a of
    scripts/verify_keyswitch.py:62 generalised to a gadget decomposition);
  * RNS rescale: out_i = (x_i - [centred(x_t)]_{q_i}) * q_t^-1 mod q_i,
    t = level - 1 (the CRT -> centre -> divide -> re-split of
    rtl/m5/rescale_rns.sv:1-45 expressed per limb).

Arrays: ciphertext [B, 2, level, N] in the evaluation domain, evaluations in
bit-reversed order (oracle.ntt.merged_forward).  ``bigint_ct_mul`` restates
the same map with Python integers over the CRT-composed modulus, as an
independent check of the per-limb formulas.
"""
from __future__ import annotations

from functools import lru_cache

import numpy as np

from .modmath import mulmod, addmod, submod, negmod, center
from .ntt import merged_tables, merged_forward, merged_inverse
from .modmath import root_2n


@lru_cache(maxsize=None)
def tables(q: int, n: int, psi: int | None = None):
    psi = psi or root_2n(q, n)
    fwd, inv = merged_tables(n, q, psi, None, cyclic=False)
    return fwd, inv, pow(n, -1, q), psi


def ntt(x, q, n):
    fwd, _, _, _ = tables(int(q), n)
    return merged_forward(x, np.uint64(q), fwd)


def intt(x, q, n):
    _, inv, ninv, _ = tables(int(q), n)
    return merged_inverse(x, np.uint64(q), inv, ninv)


def ntt_limbs(x, primes):
    """x [..., L, N] coefficient domain -> evaluation domain per limb."""
    n = x.shape[-1]
    out = np.empty_like(x, dtype=np.uint64)
    for i, q in enumerate(primes):
        out[..., i, :] = ntt(x[..., i, :], q, n)
    return out


def intt_limbs(x, primes):
    n = x.shape[-1]
    out = np.empty_like(x, dtype=np.uint64)
    for i, q in enumerate(primes):
        out[..., i, :] = intt(x[..., i, :], q, n)
    return out


def centred_to(x, q_from, q_to):
    """Residues x in [0, q_from) -> centred integer -> residue mod q_to."""
    c = center(x, q_from)
    return np.mod(c, np.int64(q_to)).astype(np.uint64)


def tensor(ct_a, ct_b, qs):
    qv = np.asarray(qs, dtype=np.uint64)[:, None]
    a0, a1 = ct_a[:, 0], ct_a[:, 1]
    b0, b1 = ct_b[:, 0], ct_b[:, 1]
    d0 = mulmod(a0, b0, qv)
    d1 = addmod(mulmod(a0, b1, qv), mulmod(a1, b0, qv), qv)
    d2 = mulmod(a1, b1, qv)
    return d0, d1, d2


def keyswitch(d2, ksk, qs, p):
    """d2 [B, l, N] evaluation domain over qs (len l); ksk [dnum>=l, 2, L+1, N]
    evaluation domain over (q_0..q_{L-1}, p) with the special limb last.
    Returns ks [B, 2, l, N] over qs."""
    B, l, n = d2.shape
    big_l = ksk.shape[2] - 1
    d2c = intt_limbs(d2, qs)                       # digits (coefficient domain)
    targets = list(qs) + [p]
    key_limb = list(range(l)) + [big_l]
    acc = np.zeros((B, 2, l + 1, n), dtype=np.uint64)
    for r, (qr, kl) in enumerate(zip(targets, key_limb)):
        for j in range(l):
            if r == j:
                dj = d2[:, j]                       # digit j at its own prime
            else:
                dj = ntt(np.mod(d2c[:, j], np.uint64(qr)), qr, n)
            for k in range(2):
                acc[:, k, r] = addmod(acc[:, k, r], mulmod(dj, ksk[j, k, kl], qr), qr)
    # ModDown by p
    accp = np.stack([intt(acc[:, k, l], p, n) for k in range(2)], axis=1)  # [B, 2, N]
    ks = np.empty((B, 2, l, n), dtype=np.uint64)
    for i, qi in enumerate(qs):
        pinv = pow(p, -1, qi)
        for k in range(2):
            conv = ntt(centred_to(accp[:, k], p, qi), qi, n)
            ks[:, k, i] = mulmod(submod(acc[:, k, i], conv, qi), pinv, qi)
    return ks


def rescale(x, qs):
    """x [B, P, l, N] evaluation domain over qs -> [B, P, l-1, N]."""
    l = x.shape[2]
    n = x.shape[-1]
    t = l - 1
    qt = qs[t]
    w = intt(x[:, :, t], qt, n)
    out = np.empty(x.shape[:2] + (t, n), dtype=np.uint64)
    for i in range(t):
        qi = qs[i]
        conv = ntt(centred_to(w, qt, qi), qi, n)
        out[:, :, i] = mulmod(submod(x[:, :, i], conv, qi), pow(qt, -1, qi), qi)
    return out


def ct_mul_relin_rescale(ct_a, ct_b, ksk, qs, p):
    """Oracle of the GPU ct-mult path: ct [B, 2, l, N] x2 -> [B, 2, l-1, N]."""
    qs = [int(q) for q in qs]
    d0, d1, d2 = tensor(ct_a, ct_b, qs)
    ks = keyswitch(d2, ksk, qs, int(p))
    qv = np.asarray(qs, dtype=np.uint64)[:, None]
    full = np.stack([addmod(d0, ks[:, 0], qv), addmod(d1, ks[:, 1], qv)], axis=1)
    return rescale(full, qs)


# ------------------------------------------------------------------ keys etc.
def relin_key(s_coef, qs, p, a_eval, e_coef, dnum=None):
    """Hybrid relinearisation key (dnum = len(qs) digits, one special prime).
    s_coef: secret [N] small ints; a_eval [dnum, L+1, N] uniform (evaluation
    domain); e_coef [dnum, L+1, N] small ints (the same error on every limb is
    NOT required; each limb gets its residue of one integer error poly when
    e_coef rows agree).  Returns ksk [dnum, 2, L+1, N]:
        ksk[j][0] = -a_j s + e_j + delta_{ij} (p mod q_j) s^2,  ksk[j][1] = a_j."""
    qs = [int(q) for q in qs]
    basis = qs + [int(p)]
    L1 = len(basis)
    dnum = dnum or len(qs)
    n = len(s_coef)
    s_eval = np.stack([ntt(np.mod(np.asarray(s_coef, dtype=np.int64), q).astype(np.uint64), q, n)
                       for q in basis])
    ksk = np.zeros((dnum, 2, L1, n), dtype=np.uint64)
    for j in range(dnum):
        for r, q in enumerate(basis):
            e = ntt(np.mod(np.asarray(e_coef[j], dtype=np.int64), q).astype(np.uint64), q, n)
            b = addmod(negmod(mulmod(a_eval[j, r], s_eval[r], q), q), e, q)
            if r == j:
                s2 = mulmod(s_eval[r], s_eval[r], q)
                b = addmod(b, mulmod(s2, np.uint64(int(p) % q), q), q)
            ksk[j, 0, r] = b
            ksk[j, 1, r] = a_eval[j, r]
    return ksk


def encrypt_eval(m_coef, s_coef, qs, a_eval, e_coef):
    """c1 = a, c0 = -a s + e + m over qs, evaluation domain; m_coef, e_coef
    integer polynomials.  Returns [2, l, N]."""
    n = len(s_coef)
    out = np.zeros((2, len(qs), n), dtype=np.uint64)
    for i, q in enumerate(qs):
        q = int(q)
        s = ntt(np.mod(np.asarray(s_coef, dtype=np.int64), q).astype(np.uint64), q, n)
        me = np.mod(np.asarray(m_coef, dtype=np.int64) + np.asarray(e_coef, dtype=np.int64), q)
        me = ntt(me.astype(np.uint64), q, n)
        out[0, i] = addmod(negmod(mulmod(a_eval[i], s, q), q), me, q)
        out[1, i] = a_eval[i]
    return out


def decrypt_coef(ct, s_coef, qs):
    """c0 + c1 s per limb -> coefficient domain residues [l, N]."""
    n = ct.shape[-1]
    out = np.zeros((ct.shape[1], n), dtype=np.uint64)
    for i, q in enumerate(qs):
        q = int(q)
        s = ntt(np.mod(np.asarray(s_coef, dtype=np.int64), q).astype(np.uint64), q, n)
        out[i] = intt(addmod(ct[0, i], mulmod(ct[1, i], s, q), q), q, n)
    return out


def crt_centred(res, qs):
    """Residues [l, N] -> Python ints centred mod prod(qs)."""
    Q = 1
    for q in qs:
        Q *= int(q)
    vals = []
    for col in range(res.shape[1]):
        x = 0
        for i, q in enumerate(qs):
            q = int(q)
            Mi = Q // q
            x += int(res[i, col]) * Mi * pow(Mi, -1, q)
        x %= Q
        if x > Q // 2:
            x -= Q
        vals.append(x)
    return vals


# ------------------------------------------------------------------ big-int check
def _negacyclic_int(a, b, n):
    c = [0] * n
    for i in range(n):
        ai = a[i]
        if ai == 0:
            continue
        for j in range(n):
            k = i + j
            if k < n:
                c[k] += ai * b[j]
            else:
                c[k - n] -= ai * b[j]
    return c


def bigint_ct_mul(ct_a, ct_b, ksk, qs, p):
    """Same map as ``ct_mul_relin_rescale`` for ONE ciphertext pair, stated on
    CRT-composed integers: D = tensor over Z_Q, digits, acc over Z_{Qp},
    ks = (acc - centred(acc mod p)) / p, rescale = (x - centred(x mod q_t)) / q_t.
    Returns [2, l-1, N] evaluation-domain residues.  Small N only."""
    qs = [int(q) for q in qs]
    p = int(p)
    l = len(qs)
    n = ct_a.shape[-1]
    Q = 1
    for q in qs:
        Q *= q

    def to_int(res_eval, basis):
        coef = np.stack([intt(res_eval[i], q, n) for i, q in enumerate(basis)])
        M = 1
        for q in basis:
            M *= q
        out = []
        for col in range(n):
            x = 0
            for i, q in enumerate(basis):
                Mi = M // q
                x += int(coef[i, col]) * Mi * pow(Mi, -1, q)
            out.append(x % M)
        return out, M

    a0, _ = to_int(ct_a[0, 0], qs)
    a1, _ = to_int(ct_a[0, 1], qs)
    b0, _ = to_int(ct_b[0, 0], qs)
    b1, _ = to_int(ct_b[0, 1], qs)
    d0 = [x % Q for x in _negacyclic_int(a0, b0, n)]
    d1 = [(x + y) % Q for x, y in zip(_negacyclic_int(a0, b1, n), _negacyclic_int(a1, b0, n))]
    d2 = [x % Q for x in _negacyclic_int(a1, b1, n)]
    basis = qs + [p]
    QP = Q * p
    big_l = ksk.shape[2] - 1
    key_limb = list(range(l)) + [big_l]
    acc = [[0] * n, [0] * n]
    for j in range(l):
        digit = [x % qs[j] for x in d2]
        for k in range(2):
            kv, _ = to_int(ksk[j, k][key_limb], basis)
            prod = _negacyclic_int(digit, kv, n)
            acc[k] = [(u + v) % QP for u, v in zip(acc[k], prod)]

    def div_round(x, m):  # (x - centred(x mod m)) / m
        r = x % m
        if r > m // 2:
            r -= m
        return (x - r) // m

    full = []
    for k, dk in enumerate((d0, d1)):
        ks = [div_round(x, p) % Q for x in acc[k]]
        full.append([(u + v) % Q for u, v in zip(dk, ks)])
    qt = qs[l - 1]
    Qo = Q // qt
    out = np.zeros((2, l - 1, n), dtype=np.uint64)
    for k in range(2):
        res = [div_round(x, qt) % Qo for x in full[k]]
        for i in range(l - 1):
            out[k, i] = ntt(np.array([x % qs[i] for x in res], dtype=np.uint64), qs[i], n)
    return out

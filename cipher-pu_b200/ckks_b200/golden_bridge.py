"""list[int] <-> GPU bridge behind the golden-model drop-in modules.

The reference's golden API (scripts/verify_keyswitch.py, verify_rescale.py,
gen_ntt_vectors.py, tb/ref/gen_ntt_reference.py, scripts/gen_omega_tables.py)
works on Python lists of ints in [0, q).  These helpers move such lists to the
GPU, run the C-ABI kernels and return fresh lists, with the same integer
semantics.  Moduli that are not NTT-friendly for the requested ring go
through the exact three-prime CRT product (ckks_poly_mul_anyq).
"""
from __future__ import annotations

from functools import lru_cache

import numpy as np

from .params import chain_primes, find_ntt_primes, primitive_root

_CRT_PRIMES = None


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("the CKKS core needs a CUDA device (no CPU fallback)")
    return torch


def _ops():
    from . import ops
    return ops


def _log2(n: int) -> int:
    l = n.bit_length() - 1
    if n < 2 or (1 << l) != n:
        raise ValueError(f"N={n} must be a power of two >= 2")
    return l


def _ctx(log_n: int, primes, omega=None, n_special=0):
    from .context import Context
    return Context.get(log_n, primes, n_special=n_special, omega=omega)


def _crt_ctx(log_n: int):
    global _CRT_PRIMES
    if _CRT_PRIMES is None:
        _CRT_PRIMES = list(chain_primes(3, 14))
    return _ctx(log_n, _CRT_PRIMES)


def _dev(vals):
    return _ops().to_device(np.asarray([int(v) for v in vals], dtype=np.uint64))


def _list(t) -> list[int]:
    return [int(v) for v in _ops().to_host(t).reshape(-1)]


def nega_friendly(q: int, n: int) -> bool:
    return q < (1 << 47) and (q - 1) % (2 * n) == 0


# ------------------------------------------------------------------ transforms
def ntt_natural(a, omega: int, q: int) -> list[int]:
    """Cyclic NTT with natural-order output: A[k] = sum_j a_j omega^(jk) mod q."""
    ops = _ops()
    n = len(a)
    ctx = _ctx(_log2(n), [q], omega=[omega])
    x = _dev([v % q for v in a]).reshape(1, n)
    ops.ntt(ctx, x, cyclic=True, n_limbs=1)
    return _list(ops.bitrev_permute(ctx, x))


def intt_natural(a_hat, omega_inv: int, q: int) -> list[int]:
    """Inverse of ``ntt_natural`` given omega^-1 (includes the N^-1 scale)."""
    ops = _ops()
    n = len(a_hat)
    omega = pow(omega_inv, -1, q)
    ctx = _ctx(_log2(n), [q], omega=[omega])
    x = ops.bitrev_permute(ctx, _dev([v % q for v in a_hat]).reshape(1, n))
    ops.ntt(ctx, x, cyclic=True, inverse=True, n_limbs=1)
    return _list(x)


# ------------------------------------------------------------------ products
def poly_mult(a, b, q: int, cyclic: bool = False) -> list[int]:
    """(a * b) mod (X^N + 1, q) (negacyclic) or mod (X^N - 1, q) (cyclic)."""
    return poly_mult_many([a], [b], q, cyclic)[0]


def poly_mult_many(As, Bs, q: int, cyclic: bool = False) -> list[list[int]]:
    ops = _ops()
    n = len(As[0])
    log_n = _log2(n)
    a = _dev([v % q for row in As for v in row]).reshape(len(As), 1, n)
    b = _dev([v % q for row in Bs for v in row]).reshape(len(Bs), 1, n)
    friendly = (q - 1) % n == 0 if cyclic else nega_friendly(q, n)
    if friendly and q < (1 << 47):
        ctx = _ctx(log_n, [q])
        out = ops.poly_mul(ctx, a, b, cyclic=cyclic)
    else:
        if q >= (1 << 45):
            raise ValueError("moduli >= 2^45 must be NTT-friendly for this ring")
        out = ops.poly_mul_anyq(_crt_ctx(log_n), a, b, q, cyclic=cyclic)
    h = ops.to_host(out).reshape(len(As), n)
    return [[int(v) for v in row] for row in h]


def addsub(a, b, q: int, subtract: bool) -> list[int]:
    ops = _ops()
    return _list(ops.vec_addsub(_dev([v % q for v in a]), _dev([v % q for v in b]), q, subtract))


def relin(e0, e1, e2, a, b, q: int):
    """f0 = e0 + e2 b, f1 = e1 - e2 a (mod q, negacyclic)."""
    ops = _ops()
    n = len(e0)
    if nega_friendly(q, n):
        ctx = _ctx(_log2(n), [q])
        d = [_dev([v % q for v in x]).reshape(1, n) for x in (e0, e1, e2, a, b)]
        f0, f1 = ops.relin_single(ctx, *d)
        return _list(f0), _list(f1)
    e2b, e2a = poly_mult_many([e2, e2], [b, a], q)
    return addsub(e0, e2b, q, False), addsub(e1, e2a, q, True)


def relin_masked(e0, e1, e2, a1, b1, a2, b2, q: int):
    """First-order masked relin (rtl/m3/keyswitch_pipe_masked.sv:1-27): key
    shares a = a1 + a2, b = b1 + b2 processed separately; equals relin(e0, e1,
    e2, a, b, q)."""
    ops = _ops()
    n = len(e0)
    if nega_friendly(q, n):
        ctx = _ctx(_log2(n), [q])
        d = [_dev([v % q for v in x]).reshape(1, n) for x in (e0, e1, e2, a1, b1, a2, b2)]
        f0, f1 = ops.relin_single_masked(ctx, *d)
        return _list(f0), _list(f1)
    p_b1, p_b2, p_a1, p_a2 = poly_mult_many([e2] * 4, [b1, b2, a1, a2], q)
    f0 = addsub(addsub(e0, p_b1, q, False), p_b2, q, False)
    f1 = addsub(addsub(e1, p_a1, q, True), p_a2, q, True)
    return f0, f1


# ------------------------------------------------------------------ rescale
def rescale_exact(vals, q_in: int, q_out: int) -> list[int]:
    ops = _ops()
    if len(vals) == 0:
        return []
    return _list(ops.rescale_exact(_dev(vals), q_in, q_out))


def rescale_scaled(vals, q_in: int, q_out: int, scale_bits: int) -> list[int]:
    ops = _ops()
    if len(vals) == 0:
        return []
    return _list(ops.rescale_scaled(_dev(vals), q_in, q_out, scale_bits))


# ------------------------------------------------------------------ parameters
@lru_cache(maxsize=None)
def modulus_chain(k_chain: int = 4, bits: int = 45, n: int = 16384) -> tuple:
    """K-prime modulus chain with the record layout of the reference's
    scripts/gen_modulus_chain.py:97 find_k_primes: candidates q = k*2N + 1 of
    `bits` bits searched upward from 2^(bits-1); the first 3K found are sorted
    by c = q - 2^(bits-1), the K smallest kept and listed with q_0 largest."""
    cond = 2 * n
    base = 1 << (bits - 1)
    found = []
    k = (base + cond - 1) // cond
    from .params import is_prime
    while len(found) < 3 * k_chain:
        q = k * cond + 1
        if q.bit_length() == bits and is_prime(q):
            found.append((q, q - base, k))
        k += 1
    found.sort(key=lambda x: x[1])
    picked = sorted(found[:k_chain], key=lambda x: -x[1])
    out = []
    for q, c, kk in picked:
        g = primitive_root(q)
        omega = pow(g, (q - 1) // n, q)
        omega_inv = pow(omega, -1, q)
        n_inv = pow(n, -1, q)
        out.append({"q": q, "q_bits": q.bit_length(), "c": c, "c_bits": c.bit_length() if c else 0,
                    "k_in_search": kk, "primitive_root": g, "omega": omega, "omega_inv": omega_inv,
                    "N": n, "N_INV": n_inv, "is_prime": True, "cond_satisfied": (q - 1) % cond == 0,
                    "omega_N_mod_q": pow(omega, n, q), "omega_inv_N_mod_q": pow(omega_inv, n, q),
                    "omega_omega_inv_mod_q": omega * omega_inv % q, "N_N_INV_mod_q": n * n_inv % q})
    return tuple(out)


__all__ = ["ntt_natural", "intt_natural", "poly_mult", "poly_mult_many", "addsub", "relin",
           "rescale_exact", "rescale_scaled", "modulus_chain", "nega_friendly", "find_ntt_primes"]

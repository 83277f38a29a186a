"""Parameter generation for the CKKS core (host side).

NTT-friendly prime search (q = 1 mod 2N, Miller-Rabin), primitive roots and
the parameter sets of the workloads.  Mirrors the reference's parameter path
scripts/gen_modulus_chain.py:97 ``find_k_primes`` (descending q = k*M + 1),
:40 ``is_prime``, :63 ``primitive_root`` and scripts/gen_omega_tables.py:85
``derive_omega`` (omega = g^((q-1)/N)).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from functools import lru_cache

_MR_BASES = (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37)


def is_prime(n: int) -> bool:
    """Deterministic Miller-Rabin for n < 3.3e24 (first twelve prime bases)."""
    if n < 2:
        return False
    for p in _MR_BASES:
        if n % p == 0:
            return n == p
    d, s = n - 1, 0
    while not d & 1:
        d >>= 1
        s += 1
    for a in _MR_BASES:
        x = pow(a, d, n)
        if x in (1, n - 1):
            continue
        for _ in range(s - 1):
            x = x * x % n
            if x == n - 1:
                break
        else:
            return False
    return True


def _factor(n: int) -> list[int]:
    fs, d = [], 2
    while d * d <= n:
        if n % d == 0:
            fs.append(d)
            while n % d == 0:
                n //= d
        d += 1 if d == 2 else 2
    if n > 1:
        fs.append(n)
    return fs


@lru_cache(maxsize=None)
def primitive_root(q: int) -> int:
    """Smallest generator of (Z/qZ)^* for prime q."""
    fs = _factor(q - 1)
    g = 2
    while True:
        if all(pow(g, (q - 1) // f, q) != 1 for f in fs):
            return g
        g += 1


def root_of_unity(q: int, order: int) -> int:
    """g^((q-1)/order): a primitive `order`-th root of unity mod q."""
    if (q - 1) % order:
        raise ValueError(f"{order} does not divide q-1 for q={q}")
    return pow(primitive_root(q), (q - 1) // order, q)


def find_ntt_primes(bits: int, modulus: int, count: int, below: int | None = None) -> list[int]:
    """The `count` largest primes q < 2^bits (and < `below`) with q = 1 mod modulus."""
    top = min((1 << bits) - 1, (below - 1) if below else (1 << bits) - 1)
    k = top // modulus
    out = []
    while len(out) < count:
        if k <= 0:
            raise ValueError("ran out of candidates")
        q = k * modulus + 1
        if q.bit_length() == bits and is_prime(q):
            out.append(q)
        k -= 1
    return out


# The largest 45-bit prime = 1 mod 2^13 (plain NTT -> modmul -> INTT workload, N = 2^12).
PRIME_45_N4096 = 35184371884033


@lru_cache(maxsize=None)
def chain_primes(count: int, log_n_max: int = 13, bits: int = 45) -> tuple[int, ...]:
    """`count` 45-bit primes = 1 mod 2^(log_n_max+1), largest first.  The first
    one serves as the special (keyswitch) prime; the rest are q_0, q_1, ..."""
    return tuple(find_ntt_primes(bits, 1 << (log_n_max + 1), count))


@dataclass(frozen=True)
class CkksParams:
    """RNS-CKKS parameter set.

    log_n: ring dimension N = 2^log_n; q: ciphertext primes q_0..q_{L-1};
    special: the keyswitch prime (hybrid key, dnum = L); scale: Delta;
    sigma: discrete-Gaussian error width; h: None = uniform ternary secret."""
    log_n: int
    q: tuple[int, ...]
    special: int
    scale: float = float(2 ** 40)
    sigma: float = 3.2
    seed: int = 0
    extra: dict = field(default_factory=dict, compare=False, hash=False)

    @property
    def n(self) -> int:
        return 1 << self.log_n

    def to_c(self):
        """(ckks_params struct, the primes array it points to): the C mirror of
        this set (all primes with the special one last; roots left to the
        library, which derives them as this module does).  Keep the array
        alive while the struct is used."""
        import ctypes
        from ._lib import CkksParamsC
        arr = (ctypes.c_uint64 * len(self.primes))(*self.primes)
        st = CkksParamsC(self.log_n, len(self.primes), 1, 0, arr, None, None, float(self.scale),
                         float(self.sigma), int(self.seed))
        return st, arr

    @property
    def levels(self) -> int:
        return len(self.q)

    @property
    def primes(self) -> tuple[int, ...]:
        return tuple(self.q) + (self.special,)

    @staticmethod
    def standard(log_n: int, levels: int, scale_bits: int = 40, seed: int = 0,
                 log_n_max: int = 13) -> "CkksParams":
        """45-bit chain with one special prime (the largest), all = 1 mod 2^(log_n_max+1)."""
        pr = chain_primes(levels + 1, max(log_n_max, log_n))
        return CkksParams(log_n=log_n, q=tuple(pr[1:levels + 1]), special=pr[0],
                          scale=float(2 ** scale_bits), seed=seed)

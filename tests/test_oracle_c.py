"""The native CPU restatement of the RNS ct-mult (oracle/ckks_cpu.c, the
timed CPU baseline) is bit-exact against the numpy oracle
(oracle.rns_ckks.ct_mul_relin_rescale, itself pinned by the big-integer
restatement): several ring sizes, levels below and at the key's, residues
up to q - 1, one and several threads.  No GPU."""
import numpy as np
import pytest

from oracle import ckks_c
from oracle import rns_ckks as R
from oracle.modmath import find_primes


def _rand(rng, shape, basis):
    x = np.zeros(shape, dtype=np.uint64)
    for i, q in enumerate(basis):
        x[..., i, :] = rng.integers(0, q, size=x[..., i, :].shape, dtype=np.uint64)
    return x


@pytest.mark.parametrize("log_n,L,level,bits", [(6, 2, 2, 45), (8, 4, 3, 45), (10, 3, 3, 47), (12, 3, 3, 45),
                                                (6, 8, 8, 40)])
def test_c_port_matches_numpy_oracle(log_n, L, level, bits):
    ckks_c.build()
    n = 1 << log_n
    pr = find_primes(bits, 2 * n, L + 1)
    p, qs = pr[0], pr[1:]
    rng = np.random.default_rng(log_n * 100 + L)
    a = _rand(rng, (3, 2, level, n), qs[:level])
    b = _rand(rng, (3, 2, level, n), qs[:level])
    a[0] = np.asarray(qs[:level], dtype=np.uint64)[None, :, None] - 1
    ksk = _rand(rng, (L, 2, L + 1, n), qs + [p])
    sub = ksk[:level][:, :, list(range(level)) + [L]]
    want = R.ct_mul_relin_rescale(a, b, sub, qs[:level], p)
    cm = ckks_c.CpuCtMul(log_n, qs, p)
    for threads in (1, 2):
        assert np.array_equal(cm(a, b, ksk, threads=threads), want)
    cm.close()

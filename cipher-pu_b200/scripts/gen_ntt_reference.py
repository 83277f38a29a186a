"""Drop-in for the reference's tb/ref/gen_ntt_reference.py (NTT reference vectors).

Same constants (LOG_N = 4, N = 16, Q = 113, Q_WIDTH = 7, NUM_VECTORS = 10) and
functions ``find_primitive_root``, ``ntt(a, omega, N, q)`` (bit-reversal +
radix-2 DIT, natural-order result) and ``intt(a, omega_inv, N, q)`` (with the
1/N scale), computed on the GPU.  ``main(output_dir)`` writes the ten
ntt_input_v / ntt_output_v / intt_output_v .mem files (seed 42 + v) that the
reference writes at import time; here nothing runs at import.
"""
from __future__ import annotations

import os
import random
import sys

import _bootstrap  # noqa: F401
from ckks_b200 import golden_bridge as gb
from ckks_b200.params import primitive_root

LOG_N = 4
N = 1 << LOG_N
Q = 113
Q_WIDTH = 7
NUM_VECTORS = 10


def find_primitive_root(q):
    return primitive_root(q)


def ntt(a, omega, N, q):
    assert len(a) == N
    return gb.ntt_natural(list(a), omega, q)


def intt(a, omega_inv, N, q):
    assert len(a) == N
    return gb.intt_natural(list(a), omega_inv, q)


def main(output_dir: str | None = None) -> int:
    output_dir = output_dir or os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref")
    os.makedirs(output_dir, exist_ok=True)
    g = find_primitive_root(Q)
    omega = pow(g, (Q - 1) // N, Q)
    omega_inv = pow(omega, -1, Q)
    for v in range(NUM_VECTORS):
        random.seed(42 + v)
        x = [random.randint(0, Q - 1) for _ in range(N)]
        y = ntt(x, omega, N, Q)
        z = intt(y, omega_inv, N, Q)
        assert z == x, f"INTT round trip failed (vector {v})"
        for name, vals in (("ntt_input", x), ("ntt_output", y), ("intt_output", z)):
            with open(os.path.join(output_dir, f"{name}_{v}.mem"), "w") as f:
                f.writelines(f"{c}\n" for c in vals)
    print(f"omega = {omega}  omega_inv = {omega_inv}  N_inv = {pow(N, -1, Q)}")
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1] if len(sys.argv) > 1 else None))

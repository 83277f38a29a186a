"""Drop-in for the reference's scripts/verify_keyswitch.py (single-pair relin).

Same names and integer semantics: N, NUM_TESTS, CHAIN_FILE, ``load_chain``,
``poly_add``, ``poly_sub``, ``poly_mult`` (negacyclic product mod (X^N+1, q)),
``relin`` (f0 = e0 + e2 b, f1 = e1 - e2 a), ``check_output_range``,
``check_message_preservation``, ``check_boundary``, ``check_random`` and
``main`` (exit code 0 = ALL PASS).  The products run on the GPU (fused
NTT -> pointwise -> INTT kernels, or the exact three-prime CRT product when q
is not NTT-friendly for the ring); the random checks are drawn in the
reference's order and then evaluated as one batch.

``load_chain`` reads CHAIN_FILE when it exists (CKKS_CHAIN_FILE overrides it;
point it at the reference's rtl/m2/modulus_chain_chain4.json) and otherwise
regenerates the same four-prime chain (scripts/gen_modulus_chain.py:97 rules).
"""
from __future__ import annotations

import json
import os
import random
import sys
from pathlib import Path

import _bootstrap  # noqa: F401
from ckks_b200 import golden_bridge as gb

HERE = Path(__file__).resolve().parent
CHAIN_FILE = Path(os.environ.get("CKKS_CHAIN_FILE", HERE.parent / "rtl" / "m2" / "modulus_chain_chain4.json"))

N = 16384
NUM_TESTS = 1000


def load_chain():
    if CHAIN_FILE.exists():
        with open(CHAIN_FILE, "r", encoding="utf-8") as f:
            return json.load(f)
    return [dict(r) for r in gb.modulus_chain(4, 45, 16384)]


def poly_add(a, b, q):
    return gb.addsub(a, b, q, subtract=False)


def poly_sub(a, b, q):
    return gb.addsub(a, b, q, subtract=True)


def poly_mult(a, b, q):
    return gb.poly_mult(a, b, q)


def relin(e0, e1, e2, a, b, q):
    return gb.relin(e0, e1, e2, a, b, q)


def check_output_range(f0, f1, q):
    errs = []
    for i, (x, y) in enumerate(zip(f0, f1)):
        if not (0 <= x < q):
            errs.append(f"f0[{i}]={x} out of range")
            break
        if not (0 <= y < q):
            errs.append(f"f1[{i}]={y} out of range")
            break
    return errs


def check_message_preservation(e0, e1, e2, a, b, s, q, n_toy=16):
    f0, f1 = relin(e0[:n_toy], e1[:n_toy], e2[:n_toy], a[:n_toy], b[:n_toy], q)
    left = poly_add(f0, poly_mult(f1, s[:n_toy], q), q)
    e1s = poly_mult(e1[:n_toy], s[:n_toy], q)
    e2s2 = poly_mult(poly_mult(e2[:n_toy], s[:n_toy], q), s[:n_toy], q)
    right = poly_add(poly_add(e0[:n_toy], e1s, q), e2s2, q)
    errs = []
    for i in range(n_toy):
        if left[i] != right[i]:
            errs.append(f"i={i}: left={left[i]}, right={right[i]}")
            if len(errs) > 5:
                break
    return errs


def check_boundary(q, s):
    n_toy = 16
    e0 = [0] * n_toy
    e1 = [q - 1] * n_toy
    e2 = [1] * n_toy
    a = [random.randrange(q) for _ in range(n_toy)]
    b = poly_add(poly_mult(a, s[:n_toy], q), [1] * n_toy, q)
    f0, f1 = relin(e0, e1, e2, a, b, q)
    return check_output_range(f0, f1, q)


def _relin_batch(cases, q):
    """cases: list of (e0, e1, e2, a, b) of equal length n -> list of (f0, f1)."""
    import numpy as np
    from ckks_b200 import ops
    n = len(cases[0][0])
    if not gb.nega_friendly(q, n):
        return [relin(*c, q) for c in cases]
    from ckks_b200.context import Context
    ctx = Context.get(n.bit_length() - 1, [q])
    cols = [ops.to_device(np.array([[v % q for v in c[i]] for c in cases], dtype=np.uint64))
            for i in range(5)]
    f0, f1 = ops.relin_single(ctx, *cols)
    h0, h1 = ops.to_host(f0), ops.to_host(f1)
    return [([int(v) for v in h0[i]], [int(v) for v in h1[i]]) for i in range(len(cases))]


def check_random(q, s, n=NUM_TESTS):
    n_toy = 16
    drawn = []
    for _ in range(n):
        e0 = [random.randrange(q) for _ in range(n_toy)]
        e1 = [random.randrange(q) for _ in range(n_toy)]
        e2 = [random.randrange(q) for _ in range(n_toy)]
        a = [random.randrange(q) for _ in range(n_toy)]
        e_ks = [random.randrange(100) for _ in range(n_toy)]
        drawn.append((e0, e1, e2, a, e_ks))
    if not drawn:
        return []
    a_s = gb.poly_mult_many([d[3] for d in drawn], [s[:n_toy]] * len(drawn), q)
    cases = [(d[0], d[1], d[2], d[3], [(x + y) % q for x, y in zip(asv, d[4])])
             for d, asv in zip(drawn, a_s)]
    errs = []
    for f0, f1 in _relin_batch(cases, q):
        errs.extend(check_output_range(f0, f1, q))
        if errs:
            break
    return errs


def main():
    print("=" * 70)
    print("M3-c KeySwitch rotation=0 (ReLinearization) equivalence check [GPU]")
    print("=" * 70)
    chain = load_chain()
    q = chain[0]["q"]
    print(f"modulus q = {q} (bits={q.bit_length()}), N = {N}")
    rng = random.Random(42)
    s = [rng.randrange(q) for _ in range(N)]
    all_pass = True
    print("[1] boundary")
    errs = check_boundary(q, s)
    print("  [FAIL]" if errs else "  [OK]   output range")
    all_pass &= not errs
    print("[2] random (1000)")
    errs = check_random(q, s)
    print("  [FAIL]" if errs else "  [OK]   1000 random cases")
    all_pass &= not errs
    print("[3] recomputation (10 samples, N=16)")
    n_toy = 16
    for i in range(10):
        e0 = [rng.randrange(q) for _ in range(n_toy)]
        e1 = [rng.randrange(q) for _ in range(n_toy)]
        e2 = [rng.randrange(q) for _ in range(n_toy)]
        a = [rng.randrange(q) for _ in range(n_toy)]
        e_ks = [rng.randrange(100) for _ in range(n_toy)]
        b = poly_add(poly_mult(a, s[:n_toy], q), e_ks, q)
        f0, f1 = relin(e0, e1, e2, a, b, q)
        ok = f0 == poly_add(e0, poly_mult(e2, b, q), q) and f1 == poly_sub(e1, poly_mult(e2, a, q), q)
        print(f"  [{'OK' if ok else 'FAIL'}]   sample {i}")
        all_pass &= ok
    print("=" * 70)
    print("result:", "ALL PASS" if all_pass else "FAIL")
    print("=" * 70)
    return 0 if all_pass else 1


if __name__ == "__main__":
    sys.exit(main())

"""Drop-in for the reference's scripts/verify_rescale.py (exact modulus switch).

Same names and semantics: N, NUM_RANDOM, CHAIN_FILE, ``load_chain``,
``rescale_coeff`` (round(c q_out / q_in) mod q_out, halves rounded up),
``rescale_poly``, ``check_boundary``, ``check_random``, ``check_roundtrip``,
``check_monotonic``, ``check_poly`` and ``main``.  Rescaling runs on the GPU
(ckks_rescale_exact); the random checks draw their values in the reference's
order and rescale them as one batch.
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
NUM_RANDOM = 100_000


def load_chain():
    if CHAIN_FILE.exists():
        with open(CHAIN_FILE, "r", encoding="utf-8") as f:
            return json.load(f)
    return [dict(r) for r in gb.modulus_chain(4, 45, 16384)]


def rescale_coeff(c, q_in, q_out):
    return gb.rescale_exact([c], q_in, q_out)[0]


def rescale_poly(c, q_in, q_out):
    return gb.rescale_exact(list(c), q_in, q_out)


def check_boundary(q_in, q_out):
    pts = [0, 1, 2, q_in - 3, q_in - 2, q_in - 1, q_out - 1, q_out, q_out + 1]
    pts = sorted({p for p in pts if 0 <= p < q_in})
    return [f"c={c} -> out={o} (out of [0,{q_out}))"
            for c, o in zip(pts, rescale_poly(pts, q_in, q_out)) if not (0 <= o < q_out)]


def check_random(q_in, q_out, n=NUM_RANDOM):
    cs = [random.randrange(q_in) for _ in range(n)]
    errs = []
    for c, o in zip(cs, rescale_poly(cs, q_in, q_out)):
        if not (0 <= o < q_out):
            errs.append(f"c={c} -> out={o}")
            if len(errs) > 20:
                break
    return errs


def check_roundtrip(q_in, q_out, n=1000):
    cs = [random.randrange(q_in) for _ in range(n)]
    errs = []
    for c, co in zip(cs, rescale_poly(cs, q_in, q_out)):
        back = round(co * q_in / q_out)
        if abs(back - c) > 2:
            errs.append(f"c={c} -> c_out={co} -> back={back}")
            if len(errs) > 20:
                break
    return errs


def check_monotonic(q_in, q_out, n=1000):
    pairs = []
    for _ in range(n):
        a = random.randrange(q_in)
        b = random.randrange(q_in)
        pairs.append((a, b) if a <= b else (b, a))
    ra = rescale_poly([p[0] for p in pairs], q_in, q_out)
    rb = rescale_poly([p[1] for p in pairs], q_in, q_out)
    errs = []
    for (a, b), x, y in zip(pairs, ra, rb):
        if x > y:
            errs.append(f"a={a} b={b} -> {x} > {y}")
            if len(errs) > 20:
                break
    return errs


def check_poly(q_in, q_out):
    rng = random.Random(12345)
    poly_in = [rng.randrange(q_in) for _ in range(N)]
    poly_out = rescale_poly(poly_in, q_in, q_out)
    if len(poly_out) != N:
        return [f"len mismatch: {len(poly_out)}"]
    return [f"i={i}: out={b}" for i, b in enumerate(poly_out) if not (0 <= b < q_out)][:21]


def main():
    print("=" * 70)
    print("M3-b Rescale equivalence check [GPU]")
    print("=" * 70)
    primes = [p["q"] for p in load_chain()]
    for i, q in enumerate(primes):
        print(f"  q{i} = {q}  (bits={q.bit_length()})")
    all_pass = True
    for i in range(len(primes) - 1):
        q_in, q_out = primes[i], primes[i + 1]
        print(f"[{i}] q{i} -> q{i + 1}:  {q_in} -> {q_out}")
        for name, fn in (("boundary", check_boundary), ("random 100000", check_random),
                         ("round trip", check_roundtrip), ("monotonic", check_monotonic),
                         ("full polynomial N=16384", check_poly)):
            errs = fn(q_in, q_out)
            print(f"  [{'FAIL' if errs else 'OK'}]   {name}")
            all_pass &= not errs
    print("=" * 70)
    print("result:", "ALL PASS" if all_pass else "FAIL")
    print("=" * 70)
    return 0 if all_pass else 1


if __name__ == "__main__":
    sys.exit(main())

"""Drop-in for the reference's scripts/gen_omega_tables.py (twiddle tables).

Same public names and semantics: ``is_prime``, ``primitive_root``,
``derive_omega`` (omega = g^((q-1)/N)), ``generate_table`` (omega^k, k < N/2),
``verify`` (omega^N = 1, omega * omega_inv = 1 per entry, NTT o INTT = id on
three seeded polynomials), ``_ntt_dit`` / ``_intt_dif`` (cyclic NTT with
natural-order input and output), ``format_hex`` / ``format_sv_header`` and the
``main`` CLI.  The transforms run on the GPU (ckks_ntt + ckks_bitrev_permute);
the tables are host-side precompute as in the reference.

Difference: the reference's default run (no --omega / --primitive-root)
raises TypeError because the ``primitive_root`` argument shadows the
function (scripts/gen_omega_tables.py:91-92); here the default derives g.
"""
from __future__ import annotations

import argparse
import random
import sys
from pathlib import Path

import _bootstrap  # noqa: F401
from ckks_b200 import golden_bridge as gb
from ckks_b200.params import is_prime as _is_prime
from ckks_b200.params import primitive_root as _primitive_root


def is_prime(n: int, rounds=None) -> bool:
    return _is_prime(n)


def primitive_root(p: int) -> int:
    return _primitive_root(p)


def derive_omega(q: int, N: int, primitive_root: int | None) -> int:
    if N & (N - 1):
        raise ValueError(f"N={N} must be a power of two")
    if (q - 1) % N != 0:
        raise ValueError(f"N={N} does not divide q-1={q - 1}")
    g = primitive_root if primitive_root is not None else _primitive_root(q)
    return pow(g, (q - 1) // N, q)


def generate_table(omega: int, q: int, N: int) -> list[int]:
    half = N // 2
    table = [1] * half
    for k in range(1, half):
        table[k] = table[k - 1] * omega % q
    return table


def _ntt_dit(a: list[int], omega: int, q: int) -> list[int]:
    return gb.ntt_natural(a, omega, q)


def _intt_dif(a_hat: list[int], omega_inv: int, N_INV: int, q: int) -> list[int]:
    n = len(a_hat)
    out = gb.intt_natural(a_hat, omega_inv, q)
    if N_INV % q != pow(n, -1, q):  # caller-supplied scale differs from N^-1
        out = [x * pow(n, 1, q) % q * N_INV % q for x in out]
    return out


def verify(n: int, q: int, omega: int, omega_inv: int, omega_table: list[int],
           omega_inv_table: list[int]) -> list[str]:
    errs: list[str] = []
    if n & (n - 1) or n < 2:
        errs.append(f"N={n} is not a power of two")
    if (q - 1) % n != 0:
        errs.append(f"N={n} does not divide q-1={q - 1}")
    if not is_prime(q):
        errs.append(f"q={q} is not prime")
    if errs:
        return errs
    if pow(omega, n, q) != 1:
        errs.append(f"omega^N mod q = {pow(omega, n, q)} != 1")
    if (omega * omega_inv) % q != 1:
        errs.append(f"omega*omega_inv mod q = {(omega * omega_inv) % q} != 1")
    for k, (o, oi) in enumerate(zip(omega_table, omega_inv_table)):
        if (o * oi) % q != 1:
            errs.append(f"table[{k}]: omega^{k} * omega_inv^{k} mod q != 1")
            if len(errs) > 5:
                break
    rng = random.Random(0xC77)
    n_inv = pow(n, -1, q)
    for trial in range(3):
        a = [rng.randint(0, q - 1) for _ in range(n)]
        if _intt_dif(_ntt_dit(a, omega, q), pow(omega, -1, q), n_inv, q) != a:
            errs.append(f"round-trip trial {trial} mismatch")
            break
    return errs


def format_hex(values: list[int], width: int) -> str:
    pad = width // 4 + (1 if width % 4 else 0)
    return "".join(f"{v:0{pad}x}\n" for v in values)


def format_sv_header(tag, Q_WIDTH, q, omega, omega_inv, omega_table, omega_inv_table) -> str:
    n = len(omega_table) * 2
    body = [f"// omega_table_{tag}.sv.h  N={n} q={q} ({Q_WIDTH}-bit)  omega={omega} omega_inv={omega_inv}",
            f"`ifndef OMEGA_TABLE_{tag.upper()}_SV_H", f"`define OMEGA_TABLE_{tag.upper()}_SV_H",
            f"parameter logic [{Q_WIDTH - 1}:0] omega_table [{n // 2 - 1}:0] = '({', '.join(map(str, omega_table))});",
            f"parameter logic [{Q_WIDTH - 1}:0] omega_inv_table [{n // 2 - 1}:0] = '({', '.join(map(str, omega_inv_table))});",
            f"`endif // OMEGA_TABLE_{tag.upper()}_SV_H"]
    return "\n".join(body) + "\n"


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=16)
    ap.add_argument("--q", type=int, default=113)
    ap.add_argument("--omega", type=int, default=None)
    ap.add_argument("--primitive-root", type=int, default=None, dest="primitive_root")
    ap.add_argument("--tag", default="default")
    ap.add_argument("--outdir", default=None)
    ap.add_argument("--verify-only", action="store_true")
    args = ap.parse_args(argv)
    N, q = args.n, args.q
    if N & (N - 1):
        print(f"[FAIL] N={N} must be a power of two", file=sys.stderr)
        return 2
    omega = derive_omega(q, N, args.primitive_root) if args.omega is None else args.omega % q
    omega_inv = pow(omega, -1, q)
    tab = generate_table(omega, q, N)
    itab = generate_table(omega_inv, q, N)
    errs = verify(N, q, omega, omega_inv, tab, itab)
    if errs:
        print("[FAIL] verification failed:", file=sys.stderr)
        for e in errs:
            print(f"  - {e}", file=sys.stderr)
        return 3
    width = q.bit_length()
    print(f"[OK] N={N}  q={q}  ({width}-bit prime)")
    print(f"[OK] omega={omega}   omega_inv={omega_inv}   N_INV={pow(N, -1, q)}")
    print("[OK] (NTT o INTT) = identity  on 3 random polynomials (GPU)")
    if args.verify_only:
        print("[DONE] verify-only mode, no files written")
        return 0
    outdir = Path(args.outdir) if args.outdir else Path("rtl/m2")
    outdir.mkdir(parents=True, exist_ok=True)
    (outdir / f"omega_table_{args.tag}.sv.h").write_text(
        format_sv_header(args.tag, width, q, omega, omega_inv, tab, itab))
    (outdir / f"omega_table_{args.tag}.hex").write_text(format_hex(tab, width))
    (outdir / f"omega_inv_table_{args.tag}.hex").write_text(format_hex(itab, width))
    return 0


if __name__ == "__main__":
    sys.exit(main())

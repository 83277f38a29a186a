"""On-disk formats of the reference's RTL flow, read and written by the GPU core.

* ``$readmemh`` vector files (one hexadecimal word per line, ``//`` comments,
  ``@address`` directives), as written by scripts/gen_ntt_vectors.py
  ``write_hex`` and scripts/gen_omega_tables.py ``format_hex`` and loaded by
  the testbenches (rtl/m1/ntt_unit.sv:99-106 twiddle ROM).
* ``.mem`` decimal vectors of tb/ref/gen_ntt_reference.py.
* Modulus-chain JSON (rtl/m2/modulus_chain_chain4.json, written by
  scripts/gen_modulus_chain.py): a list of records with ``q`` and the cyclic
  ``omega`` of the chain's ring dimension.

``transform_file`` runs the library's NTT on a vector file and writes the
result in the same format, so testbench vectors go through the GPU unchanged.
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import torch

from . import ops
from .context import Context


def read_memh(path) -> np.ndarray:
    """Words of a $readmemh file in file order (addresses from @ directives
    fill a dense array; gaps read as 0)."""
    words: dict[int, int] = {}
    addr = 0
    for raw in Path(path).read_text().splitlines():
        line = raw.split("//", 1)[0].strip()
        if not line:
            continue
        for tok in line.split():
            if tok.startswith("@"):
                addr = int(tok[1:], 16)
                continue
            words[addr] = int(tok.replace("_", ""), 16)
            addr += 1
    out = np.zeros(max(words) + 1 if words else 0, dtype=np.uint64)
    for a, v in words.items():
        out[a] = v
    return out


def write_memh(path, values, width_bits: int | None = None) -> None:
    """One zero-padded hex word per line (width from the largest value when
    not given), readable by read_memh and by $readmemh."""
    vals = [int(v) for v in np.asarray(values, dtype=object).reshape(-1)]
    if width_bits is None:
        width_bits = max(4, max((v.bit_length() for v in vals), default=4))
    digits = (width_bits + 3) // 4
    if any(v < 0 or v.bit_length() > width_bits for v in vals):
        raise ValueError(f"value outside {width_bits} unsigned bits")
    Path(path).write_text("".join(f"{v:0{digits}x}\n" for v in vals))


def read_mem(path) -> np.ndarray:
    """Decimal .mem vector (one integer per line)."""
    return np.array([int(l) for l in Path(path).read_text().split() if l.strip()], dtype=np.uint64)


def load_chain(path) -> list[dict]:
    with open(path, encoding="utf-8") as f:
        return json.load(f)


def context_from_chain(chain: list[dict], log_n: int, n_special: int = 0) -> Context:
    """Context over the chain's primes with its cyclic roots (the records'
    ``omega`` is an N-th root for the chain's N; it is taken to the
    (N_chain / N)-th power for a smaller ring)."""
    primes = [int(r["q"]) for r in chain]
    n = 1 << log_n
    omegas = []
    for r in chain:
        om = int(r.get("omega", 0))
        n_chain = int(r.get("N", n))
        if om and n_chain % n == 0:
            omegas.append(pow(om, n_chain // n, int(r["q"])))
        else:
            omegas.append(0)
    return Context.get(log_n, primes, n_special=n_special, omega=omegas)


def transform_file(ctx: Context, src, dst, prime: int = 0, inverse: bool = False, cyclic: bool = True,
                   natural_order: bool = True) -> np.ndarray:
    """NTT (or INTT) of every N-word vector in `src` (hex, or decimal for .mem)
    modulo primes[prime]; writes `dst` in the same format.  natural_order:
    the cyclic transform with natural-order output (the golden convention of
    tb/ref/gen_ntt_reference.py:78) instead of the bit-reversed evaluation order."""
    src = Path(src)
    vals = read_mem(src) if src.suffix == ".mem" else read_memh(src)
    n = ctx.n
    if vals.size % n:
        raise ValueError(f"{src}: {vals.size} words is not a multiple of N={n}")
    q = ctx.primes[prime]
    x = ops.to_device((vals % np.uint64(q)).reshape(-1, 1, n))
    if inverse and natural_order:
        x = ops.bitrev_permute(ctx, x)
    ops.ntt(ctx, x, prime_begin=prime, inverse=inverse, cyclic=cyclic, n_limbs=1)
    if not inverse and natural_order:
        x = ops.bitrev_permute(ctx, x)
    torch.cuda.synchronize()
    out = ops.to_host(x).reshape(-1)
    dst = Path(dst)
    if dst.suffix == ".mem":
        dst.write_text("".join(f"{int(v)}\n" for v in out))
    else:
        write_memh(dst, out, width_bits=max(4, int(q - 1).bit_length()))
    return out

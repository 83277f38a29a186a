"""Drop-in for the reference's scripts/gen_ntt_vectors.py (NTT test vectors -> hex).

Same names: LOG_N, N, Q, NUM_VECTORS, BASE, SRC_DIR, DST_DIR, ``read_vecs``,
``write_hex`` (row-major hex, one coefficient per line, read back as
$readmemh would and compared) and ``main``.  Differences: the reference
raises NameError at import (``Path`` used without import,
scripts/gen_ntt_vectors.py:20); and when the .mem sources are absent, main()
generates them on the GPU (gen_ntt_reference.main) instead of exiting.  The
NTT outputs read from disk are re-checked against the GPU transform.
SRC_DIR / DST_DIR can be redirected with CKKS_NTT_SRC_DIR / CKKS_NTT_DST_DIR.
"""
from __future__ import annotations

import os
import sys
from pathlib import Path

import _bootstrap  # noqa: F401
import gen_ntt_reference as ref

BASE = str(Path(__file__).resolve().parents[1])
SRC_DIR = os.environ.get("CKKS_NTT_SRC_DIR", os.path.join(BASE, "tb", "ref", "ref"))
DST_DIR = os.environ.get("CKKS_NTT_DST_DIR", os.path.join(BASE, "tb", "ref"))

LOG_N = 4
N = 1 << LOG_N
Q = 113
NUM_VECTORS = 10


def read_vecs(prefix):
    out = []
    for v in range(NUM_VECTORS):
        with open(os.path.join(SRC_DIR, f"{prefix}_{v}.mem")) as f:
            out.append([int(l) for l in f if l.strip()])
    assert len(out) == NUM_VECTORS
    for vec in out:
        assert len(vec) == N, f"vector length {len(vec)} != {N}"
    return out


def write_hex(vecs, path):
    with open(path, "w") as f:
        for vec in vecs:
            for c in vec:
                assert 0 <= c < Q, f"coefficient out of range: {c}"
                f.write(f"{c:02x}\n")
    with open(path) as f:
        back = [int(l, 16) for l in f if l.strip()]
    flat = [c for vec in vecs for c in vec]
    assert back == flat, f"read-back self-check failed: {path}"
    print(f"  wrote {path}  ({len(flat)} lines, hex, read-back OK)")


def main() -> int:
    if not os.path.isdir(SRC_DIR) or not os.path.exists(os.path.join(SRC_DIR, "ntt_input_0.mem")):
        print(f"source vectors missing in {SRC_DIR}: generating them on the GPU")
        ref.main(SRC_DIR)
    os.makedirs(DST_DIR, exist_ok=True)
    print(f"N={N}, LOG_N={LOG_N}, q={Q}, vectors={NUM_VECTORS}")
    inputs = read_vecs("ntt_input")
    ntt_outs = read_vecs("ntt_output")
    intt_outs = read_vecs("intt_output")
    g = 3
    omega = pow(g, (Q - 1) // N, Q)
    omega_inv = pow(omega, -1, Q)
    n_inv = pow(N, -1, Q)
    for v in range(NUM_VECTORS):
        assert inputs[v] == intt_outs[v], f"vector {v}: INTT round trip differs from the input"
        assert ref.ntt(inputs[v], omega, N, Q) == ntt_outs[v], f"vector {v}: GPU NTT differs"
    print(f"[OK] {NUM_VECTORS} INTT round trips == inputs; GPU NTT == stored outputs")
    write_hex(inputs, os.path.join(DST_DIR, "ntt_in_all.hex"))
    write_hex(ntt_outs, os.path.join(DST_DIR, "ntt_out_all.hex"))
    write_hex(intt_outs, os.path.join(DST_DIR, "intt_out_all.hex"))
    assert pow(omega, N, Q) == 1 and omega * omega_inv % Q == 1
    print(f"  Q_VALUE  = {Q}\n  N_INV    = {n_inv}\n  omega    = {omega}\n  omega_inv= {omega_inv}")
    t_omega = [pow(omega, k, Q) for k in range(N // 2)]
    t_omega_inv = [pow(omega_inv, k, Q) for k in range(N // 2)]
    print(f"  omega_table     = {t_omega}\n  omega_inv_table = {t_omega_inv}")
    print("[OK] done")
    return 0


if __name__ == "__main__":
    sys.exit(main())

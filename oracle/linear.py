"""Encrypted linear layer restatement (test infrastructure).

out[o] = sum_f w[o][f] * in[f] (+ bias[o] on component 0) mod q_i with the
4x4 block-keep mask, exact with Python integers (object arrays).  The
reference's encrypted FC layer (scripts/exp_e11_ckks_e2e_real.py:142
encrypted_linear_layer) multiplies one coefficient-encoded ciphertext by a
weight polynomial per output; with slot packing the weights become scalars
and the layer is this modular matrix product.
"""
from __future__ import annotations

import numpy as np


def linear_plain(x: np.ndarray, w: np.ndarray, bias, keep, primes) -> np.ndarray:
    """x [F, 2, L, N] uint64; w [O, F] int; bias [O] int or None; keep [ceil(O/4), ceil(F/4)]."""
    F, two, L, n = x.shape
    O = w.shape[0]
    wm = np.array(w, dtype=object)
    if keep is not None:
        m = np.repeat(np.repeat(np.asarray(keep), 4, axis=0), 4, axis=1)[:O, :F]
        wm = wm * m.astype(object)
    out = np.zeros((O, 2, L, n), dtype=np.uint64)
    for i, q in enumerate(primes[:L]):
        q = int(q)
        for k in range(2):
            xs = x[:, k, i, :].astype(object)          # [F, N]
            y = wm.dot(xs)                             # [O, N] python ints
            if bias is not None and k == 0:
                y = y + np.array([int(b) for b in bias], dtype=object)[:, None]
            out[:, k, i, :] = np.array([[int(v) % q for v in row] for row in y], dtype=np.uint64)
    return out

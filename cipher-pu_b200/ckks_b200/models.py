"""Workload models and the plain-vs-learned gear comparison.

* ``mlp_784_128_10``: 784-128-10 MLP, weights N(0, 1/fan_in) with 50 %
  structured 4x4 block sparsity, square activation (the encrypted MLP
  workload: N = 2^13, L = 4, batch 1024).
* ``mlp_784_128_10_compressible``: the same shape with the weight statistics
  of a trained network: each 4x4 block of the hidden layer scaled by
  exp(N(0, spread^2)) (rows renormalised), so the smallest blocks hold a small
  share of a row's energy and a sparse gear can meet the SNR target.
* ``cnn_28x28``: conv 5x5x8 stride 2 (28x28x1 -> 12x12x8) as a sparse linear
  map, square activation, 2x2 average pool folded into the 288 -> 10 FC
  (the encrypted CNN workload: N = 2^13, L = 5).
* ``run_stream``: a stream of batches through an EncryptedMLP under one gear
  controller; reports samples/s, logit SNR against the FP64 plaintext model,
  top-1 agreement, probes and the gear histogram.
"""
from __future__ import annotations

import math
import time

import numpy as np
import torch

from .mlp import EncryptedMLP, Layer, make_block_sparse


def mlp_784_128_10(seed: int = 0, sparsity: float = 0.5) -> list:
    rng = np.random.default_rng(seed)
    W1 = make_block_sparse(rng.standard_normal((128, 784)) / math.sqrt(784), sparsity, seed + 1)
    W2 = make_block_sparse(rng.standard_normal((10, 128)) / math.sqrt(128), sparsity, seed + 2)
    return [Layer(W1, rng.standard_normal(128) * 0.1, "square"),
            Layer(W2, rng.standard_normal(10) * 0.1, "none")]


def mlp_784_128_10_compressible(seed: int = 0, sparsity: float = 0.5, spread: float = 2.0) -> list:
    rng = np.random.default_rng(seed)
    W1 = rng.standard_normal((128, 784)) / math.sqrt(784)
    scales = np.exp(rng.normal(0.0, spread, (32, 196)))
    W1 = W1 * np.repeat(np.repeat(scales, 4, 0), 4, 1)
    W1 = make_block_sparse(W1 / np.sqrt((W1 ** 2).sum(1, keepdims=True)), sparsity, seed + 1)
    W2 = make_block_sparse(rng.standard_normal((10, 128)) / math.sqrt(128), sparsity, seed + 2)
    return [Layer(W1, rng.standard_normal(128) * 0.1, "square"),
            Layer(W2, rng.standard_normal(10) * 0.1, "none")]


def cnn_28x28(seed: int = 0) -> list:
    rng = np.random.default_rng(seed)
    C, K, S, IN, OUT = 8, 5, 2, 28, 12
    kern = rng.standard_normal((C, K, K)) / math.sqrt(K * K)
    # conv output (c, i, j) is row (i OUT + j) C + c: the C channels of one
    # output pixel are adjacent, so a 4-row weight block shares one 5x5
    # receptive field (dense blocks, few input columns per output tile)
    Wc = np.zeros((C * OUT * OUT, IN * IN))
    for c in range(C):
        for i in range(OUT):
            for j in range(OUT):
                r = (i * OUT + j) * C + c
                for di in range(K):
                    for dj in range(K):
                        Wc[r, (S * i + di) * IN + (S * j + dj)] = kern[c, di, dj]
    bc = np.tile(rng.standard_normal(C) * 0.1, OUT * OUT)
    Wfc = rng.standard_normal((10, C * 6 * 6)) / math.sqrt(C * 36)
    bfc = rng.standard_normal(10) * 0.1
    # fold the 2x2 average pool into the FC: W_eff[o, (i, j, c)] = Wfc[o, (c, i//2, j//2)] / 4
    We = np.zeros((10, C * OUT * OUT))
    for c in range(C):
        for i in range(OUT):
            for j in range(OUT):
                We[:, (i * OUT + j) * C + c] = Wfc[:, (c * 6 + i // 2) * 6 + j // 2] / 4.0
    return [Layer(Wc, bc, "square"), Layer(We, bfc, "none")]


def run_stream(m: EncryptedMLP, ctrl, batches: list, ref_layers: list | None = None,
               calibrate=None, fallback_db: float | None = None) -> dict:
    """Encrypted inference of every batch under `ctrl` (choose / probe_policy /
    on_probe), with recompute at gear 0 when a probe measures less than
    fallback_db.  Client-side input encryption is excluded from the timed
    region."""
    ref_layers = ref_layers or m.layers
    sig = err = 0.0
    agree = total = 0
    gears, attempted = [], []
    recomputed = 0
    t_total = 0.0
    per_batch_snr = []
    max_abs = max_ref = 0.0
    for x in batches:
        X = m.encrypt_inputs(x)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = m.forward(x, ctrl.choose, on_probe=ctrl.on_probe, probe_policy=ctrl.probe_policy, X=X,
                      fallback_db=fallback_db)
        t_total += time.perf_counter() - t0
        ref = EncryptedMLP.plain_forward(ref_layers, x)
        d = r["logits"]
        s, e = float((ref ** 2).sum()), float(((d - ref) ** 2).sum())
        sig += s
        err += e
        per_batch_snr.append(10 * math.log10(s / max(e, 1e-300)))
        max_abs = max(max_abs, float(np.abs(d - ref).max()))
        max_ref = max(max_ref, float(np.abs(ref).max()))
        agree += int((d.argmax(1) == ref.argmax(1)).sum())
        total += len(x)
        gears.append(r["gears"])
        attempted.append(r["attempted_gears"])
        recomputed += r["recomputed"]
        if calibrate:
            calibrate(r)
    return {"samples": total, "seconds": t_total, "samples_per_s": total / t_total,
            "snr_db": 10 * math.log10(sig / max(err, 1e-300)), "top1_agreement": agree / total,
            "probes": getattr(ctrl, "probes", None), "recomputed_layers": recomputed, "gears": gears,
            "attempted_gears": attempted,
            "min_batch_snr_db": min(per_batch_snr),
            # decoded logits against the FP64 plaintext model: max abs error and
            # the normwise relative error max |d - ref| / max |ref|
            "max_abs_err": max_abs, "max_rel_err": max_abs / max(max_ref, 1e-300)}

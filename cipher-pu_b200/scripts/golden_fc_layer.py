"""Drop-in for the reference's scripts/golden_fc_layer.py (plaintext FC model).

Same class and functions: ``FCLayerGoldenModel(in_dim, out_dim, seed)`` with
weights = default_rng(seed).standard_normal((out, in)) * sqrt(2 / (in + out))
and zero bias; ``forward`` (Y = X W^T + b in float32), ``quantize_input`` /
``quantize_weights`` (round(x * scale), clipped to a signed bit width),
``export_weights`` (JSON with the 45-bit two's-complement hex weights at
scale 2^30), ``test_forward``; ``build_mnist_cnn_model`` and ``main``.
This is the FP plaintext oracle of the FC layers, so it stays numpy on the
host exactly as in the reference; ``encrypted_forward`` runs the same layer
under CKKS on the GPU (slot-packed batch, plaintext weights).
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

import _bootstrap  # noqa: F401


class FCLayerGoldenModel:
    def __init__(self, in_dim, out_dim, seed=None):
        self.in_dim = in_dim
        self.out_dim = out_dim
        self.seed = seed if seed is not None else 42
        rng = np.random.default_rng(self.seed)
        scale = np.sqrt(2.0 / (in_dim + out_dim))
        self.weights = rng.standard_normal((out_dim, in_dim)) * scale
        self.bias = np.zeros(out_dim, dtype=np.float32)

    def forward(self, x):
        x = np.asarray(x, dtype=np.float32)
        return x @ self.weights.T + self.bias

    def quantize_input(self, x, bits=10, scale=2 ** 30):
        x_int = np.round(x * scale).astype(np.int64)
        return np.clip(x_int, -(1 << (bits - 1)), (1 << (bits - 1)) - 1)

    def quantize_weights(self, w, bits=8, scale=2 ** 30):
        w_int = np.round(w * scale).astype(np.int64)
        return np.clip(w_int, -(1 << (bits - 1)), (1 << (bits - 1)) - 1)

    def export_weights(self, output_path=None):
        if output_path is None:
            here = os.path.dirname(os.path.abspath(__file__))
            output_path = os.path.join(here, f"fc_weights_{self.in_dim}x{self.out_dim}.json")
        data = {"in_dim": self.in_dim, "out_dim": self.out_dim,
                "weights": self.weights.flatten().tolist(), "bias": self.bias.tolist(),
                "weights_hex": [hex(int(round(v * 2 ** 30)) & ((1 << 45) - 1))
                                for v in self.weights.flatten()]}
        with open(output_path, "w") as f:
            json.dump(data, f, indent=2)
        print(f"weights exported: {output_path}  shape ({self.out_dim}, {self.in_dim})")
        return data

    def test_forward(self, num_slots=4, seed=7):
        rng = np.random.default_rng(seed)
        x = rng.standard_normal((num_slots, self.in_dim))
        y_float = self.forward(x)
        x_q = self.quantize_input(x) / 2 ** 30
        w_q = self.quantize_weights(self.weights) / 2 ** 30
        y_q = x_q @ w_q.T + self.bias
        abs_err = np.abs(y_float - y_q)
        print(f"FC {self.in_dim}x{self.out_dim}: RMSE {np.sqrt(np.mean(abs_err ** 2)):.6f}  "
              f"max {abs_err.max():.6f}  out [{y_float.min():.6f}, {y_float.max():.6f}]")
        return y_float, y_q

    def encrypted_forward(self, x, log_n=13, levels=3, seed=0):
        """Y = X W^T + b under CKKS on the GPU: each input feature is one
        ciphertext whose slots hold the batch (rows of x); returns the decrypted
        [n, out_dim] result (float64)."""
        from ckks_b200.mlp import encrypted_linear_demo
        return encrypted_linear_demo(np.asarray(x, dtype=np.float64), self.weights, self.bias,
                                     log_n=log_n, levels=levels, seed=seed)


def build_mnist_cnn_model(in_dim_fc1=512, mid_dim=128, num_classes=10, seed=42):
    fc1 = FCLayerGoldenModel(in_dim=in_dim_fc1, out_dim=mid_dim, seed=seed)
    fc2 = FCLayerGoldenModel(in_dim=mid_dim, out_dim=num_classes, seed=seed + 1)
    print(f"FC1: {in_dim_fc1} -> {mid_dim}   FC2: {mid_dim} -> {num_classes}")
    return fc1, fc2


def main():
    fc1, fc2 = build_mnist_cnn_model(in_dim_fc1=512, mid_dim=128, num_classes=10)
    fc1.test_forward(num_slots=4)
    fc2.test_forward(num_slots=4)
    rng = np.random.default_rng(99)
    x = rng.standard_normal((4, 512))
    logits = fc2.forward(np.maximum(fc1.forward(x), 0))
    print(f"logits range: [{logits.min():.4f}, {logits.max():.4f}]")
    fc1.export_weights()
    fc2.export_weights()
    return 0


if __name__ == "__main__":
    sys.exit(main())

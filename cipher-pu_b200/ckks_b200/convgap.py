"""Conv + global-average-pool fusion on coefficient-encoded RLWE ciphertexts.

The reference's application A1 (scripts/exp_e24_rotation_bootstrap.py:548-
:700): a Conv(1 -> 4, 3 x 3, stride 4, padding 1) over a 28 x 28 image
followed by a global average pool and FC(4 -> 10).  Without a nonlinearity
between conv and pool, filter f's pooled value is one inner product of the
message with a weight vector (49 positions x 9 taps, repeated pixels adding
up), and an inner product is one ciphertext x plaintext product whose
decryption's constant coefficient is -Delta^2 <x, w> once the weights are
placed at coefficient N - index (``scatter_w``, :241).  So the encrypted part
of the model is one product per filter.

Batched over images on the GPU: ``weight_polys`` scatters and transforms the
filters once; ``mul_plain_multi`` runs every (image, filter) product
(``ckks_mul_plain_multi``: one NTT per ciphertext polynomial, one INTT per
filter); ``decrypt_coef0`` reads the constant coefficient of each product's
decryption (``ckks_decrypt_coef0``).  ``fused_inference`` adds the bias,
pools and applies the plaintext FC as :615 ``encrypted_inference_fused``
does (the pooled values are float32, as the reference's float32 bias makes
them).

Parameters of the reference's run: N = 1024, q = 998244353 (NTT-friendly),
Delta = 1024, ternary secret and error.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import _lib, ops
from .context import Context, _stream

N_REF, Q_REF, SCALE_REF = 1024, 998244353, 1024


def scatter_w(msg_indices, w, scale: int, q: int, n: int) -> np.ndarray:
    """Integer weight polynomial of scripts/exp_e24_rotation_bootstrap.py:241:
    round(scale w_j) at coefficient N - m_j (m_j mod N = 0: at 0, negated)."""
    m_w = np.zeros(n, dtype=np.int64)
    for j, mi in enumerate(msg_indices):
        val = int(round(scale * float(w[j])))
        if mi % n == 0:
            m_w[0] -= val
        else:
            m_w[n - (mi % n)] += val
    return np.mod(m_w, q).astype(np.uint64)


def conv_gap_indices(w_filter) -> tuple[list[int], list[float]]:
    """(pixel index, weight) pairs of one 3 x 3 filter over the 7 x 7 output
    positions (stride 4, padding 1) of a row-major 28 x 28 image."""
    idx, vals = [], []
    for i in range(7):
        for j in range(7):
            for ki in range(3):
                for kj in range(3):
                    ii, jj = 4 * i + ki - 1, 4 * j + kj - 1
                    if 0 <= ii < 28 and 0 <= jj < 28:
                        idx.append(ii * 28 + jj)
                        vals.append(float(w_filter[ki, kj]))
    return idx, vals


@dataclass
class ConvGapModel:
    conv_w: np.ndarray  # [4, 1, 3, 3]
    conv_b: np.ndarray  # [4]
    fc_w: np.ndarray    # [10, 4]
    fc_b: np.ndarray    # [10]

    @staticmethod
    def random(seed: int = 0) -> "ConvGapModel":
        """Uniform initialisation with PyTorch's default bounds
        (1 / sqrt(fan_in)), float32 values."""
        rng = np.random.default_rng(seed)
        f32 = lambda a: np.asarray(a, dtype=np.float32).astype(np.float64)  # noqa: E731
        return ConvGapModel(f32(rng.uniform(-1 / 3, 1 / 3, (4, 1, 3, 3))), f32(rng.uniform(-1 / 3, 1 / 3, 4)),
                            f32(rng.uniform(-0.5, 0.5, (10, 4))), f32(rng.uniform(-0.5, 0.5, 10)))

    def plain_forward(self, images: np.ndarray) -> np.ndarray:
        """Float64 conv + GAP + FC on [B, 784] images (the unencrypted model)."""
        x = np.asarray(images, dtype=np.float64).reshape(-1, 28, 28)
        xp = np.pad(x, ((0, 0), (1, 1), (1, 1)))
        gap = np.zeros((x.shape[0], 4))
        for f in range(4):
            acc = np.zeros((x.shape[0], 7, 7))
            for ki in range(3):
                for kj in range(3):
                    acc += self.conv_w[f, 0, ki, kj] * xp[:, ki:ki + 25:4, kj:kj + 25:4]
            gap[:, f] = acc.mean(axis=(1, 2)) + self.conv_b[f]
        return gap @ self.fc_w.T + self.fc_b


def weight_polys(ctx: Context, model: ConvGapModel, scale: int, prime: int = 0) -> torch.Tensor:
    """The 4 filters' scattered weight polynomials in the evaluation domain
    [4, N] (negacyclic forward NTT mod primes[prime]), prepared once."""
    q = ctx.primes[prime]
    polys = np.stack([scatter_w(*conv_gap_indices(model.conv_w[f, 0]), scale, q, ctx.n)
                      for f in range(model.conv_w.shape[0])])
    w = ops.to_device(polys.reshape(-1, 1, ctx.n))
    ops.ntt(ctx, w, prime_begin=prime, n_limbs=1)
    return w.reshape(-1, ctx.n)


def weight_poly_hat(ctx: Context, msg_indices, w, scale: int, prime: int = 0) -> torch.Tensor:
    """One scattered weight polynomial (any inner product) in the evaluation domain [1, N]."""
    p = ops.to_device(scatter_w(msg_indices, w, scale, ctx.primes[prime], ctx.n).reshape(1, 1, ctx.n))
    ops.ntt(ctx, p, prime_begin=prime, n_limbs=1)
    return p.reshape(1, ctx.n)


def mul_plain_multi(ctx: Context, ct: torch.Tensor, w_hat: torch.Tensor, prime: int = 0,
                    out: torch.Tensor | None = None) -> torch.Tensor:
    """ct [B, 2, N] x w_hat [F, N] -> [B, F, 2, N] (coefficient domain)."""
    n_ct, n_w = ct.shape[0], w_hat.shape[0]
    if ct.shape[1:] != (2, ctx.n) or w_hat.shape[1:] != (ctx.n,):
        raise ValueError("expected ct [B, 2, N] and w_hat [F, N]")
    if out is None:
        out = torch.empty((n_ct, n_w, 2, ctx.n), dtype=ops.U64, device=ct.device)
    _lib.call("ckks_mul_plain_multi", ctx.handle, ops._p(out), ops._p(ct), ops._p(w_hat), n_ct, n_w, prime,
              _stream())
    return out


def decrypt_coef0(ctx: Context, ct: torch.Tensor, s_res: torch.Tensor, prime: int = 0,
                  out: torch.Tensor | None = None) -> torch.Tensor:
    """Centred constant coefficient of (b - a s) for ct [..., 2, N] -> int64 [...]."""
    lead = ct.shape[:-2]
    n_ct = int(np.prod(lead)) if lead else 1
    if out is None:
        out = torch.empty(lead, dtype=torch.int64, device=ct.device)
    _lib.call("ckks_decrypt_coef0", ctx.handle, ops._p(out), ops._p(ct), ops._p(s_res), n_ct, prime, _stream())
    return out


def secret_residues(s, q: int, device=None) -> torch.Tensor:
    """Ternary (or any integer) secret -> its N residues mod q on the device."""
    return ops.to_device((np.asarray(s, dtype=np.int64) % q).astype(np.uint64), device)


def inner_products(ctx: Context, ct: torch.Tensor, w_hat: torch.Tensor, s_res: torch.Tensor, scale: int,
                   prime: int = 0) -> np.ndarray:
    """<x_b, w_f> for every image b and weight f: -dec_0 / Delta^2, [B, F]
    (scripts/exp_e24_rotation_bootstrap.py:263 inner_product, batched)."""
    dec0 = decrypt_coef0(ctx, mul_plain_multi(ctx, ct, w_hat, prime), s_res, prime)
    return -dec0.cpu().numpy().astype(np.float64) / float(scale * scale)


def fused_inference(ctx: Context, ct: torch.Tensor, model: ConvGapModel, s_res: torch.Tensor, scale: int,
                    w_hat: torch.Tensor | None = None, prime: int = 0) -> np.ndarray:
    """Logits [B, 10] of the fused Conv + GAP + FC model on encrypted images
    ct [B, 2, N] (scripts/exp_e24_rotation_bootstrap.py:615, batched): one
    ciphertext product per filter, pooled values float32 as in the reference."""
    if w_hat is None:
        w_hat = weight_polys(ctx, model, scale, prime)
    ip = inner_products(ctx, ct, w_hat, s_res, scale, prime)
    gap = ((ip / 49.0).astype(np.float32) + np.asarray(model.conv_b).astype(np.float32)).astype(np.float64)
    return gap @ np.asarray(model.fc_w, dtype=np.float64).T + np.asarray(model.fc_b, dtype=np.float64)


def encrypt(ctx: Context, msgs: np.ndarray, s_res: torch.Tensor, scale: int, seed: int = 0,
            prime: int = 0) -> torch.Tensor:
    """Coefficient encoding b = a s + e + round(Delta m) mod q, a uniform,
    e ternary (scripts/exp_e24_rotation_bootstrap.py:307 enc_msg) for a batch
    of messages [B, <= N]; the a s products run on the GPU."""
    q = ctx.primes[prime]
    n = ctx.n
    msgs = np.asarray(msgs, dtype=np.float64).reshape(len(msgs), -1)
    bsz = msgs.shape[0]
    rng = np.random.default_rng(seed)
    m = np.zeros((bsz, n), dtype=np.int64)
    m[:, :msgs.shape[1]] = np.round(scale * msgs).astype(np.int64)
    a = rng.integers(0, q, (bsz, n), dtype=np.int64).astype(np.uint64)
    e = rng.integers(-1, 2, (bsz, n)).astype(np.int64)
    da = ops.to_device(a.reshape(bsz, 1, n))
    ds = s_res.reshape(1, 1, n).expand(bsz, 1, n).contiguous()
    a_s = ops.to_host(ops.poly_mul(ctx, da, ds, prime_begin=prime, n_limbs=1)).reshape(bsz, n).astype(np.int64)
    b = ((a_s + e + m) % q).astype(np.uint64)
    return ops.to_device(np.stack([b, a], axis=1))

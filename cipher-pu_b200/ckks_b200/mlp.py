"""Encrypted MLP / CNN inference with sparsity gears, DARE refresh and the
decrypt-based SNR probe.

Packing: SIMD over samples.  Input feature f of a batch of B <= N/2 samples
is one ciphertext whose slot s holds sample s; a linear layer is then a
plaintext-weighted sum of ciphertexts (ckks_linear_plain_weights), with no
rotations.  Pipeline of one layer l (weights W_l, bias b_l):

   X (scale Delta_in) --linear, int weights at 2^wbits--> Y (scale Delta_in 2^wbits)
   --square (ct-mult + relin + rescale)--> Z (scale Y^2 / q_t)
   --DARE (decrypt, divide by 2^shift, re-encrypt at the top level)--> X'
   (scale back near Delta)

The last layer stops after the linear step; its output is decrypted and
decoded.  Gears: gear g keeps the largest (1 - GEAR_SPARSITY[g]) fraction of
the model's nonzero 4x4 weight blocks (by Frobenius norm); gear 0 computes all
of them.  The SNR probe compares a layer's decrypted output with the same
layer evaluated in FP64 on the decrypted layer input with gear-0 weights.

The reference runs its encrypted MLP with coefficient encoding, one
ciphertext per output neuron and decryption between layers
(scripts/exp_e11_ckks_e2e_real.py:142 encrypted_linear_layer, :303
ckks_inference, :361-374 re-encryption); this module keeps that layer /
decrypt-reencrypt structure with slot packing and RNS CKKS.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib, ops
from .evaluator import Ciphertext, Evaluator
from .gear import GEAR_SPARSITY

BLOCK = 4


def block_norms(W: np.ndarray, block: int = BLOCK) -> np.ndarray:
    O, F = W.shape
    Op, Fp = -(-O // block) * block, -(-F // block) * block
    Wp = np.zeros((Op, Fp))
    Wp[:O, :F] = W
    return np.sqrt((Wp.reshape(Op // block, block, Fp // block, block) ** 2).sum(axis=(1, 3)))


def gear_keep(W: np.ndarray, sparsity: float, block: int = BLOCK) -> np.ndarray:
    """uint8 keep mask [ceil(O/4), ceil(F/4)]: the largest (1 - sparsity) share of
    the nonzero blocks, by Frobenius norm (ties broken by position)."""
    nrm = block_norms(W, block)
    nz = np.flatnonzero(nrm.reshape(-1) > 0)
    keep = np.zeros(nrm.size, dtype=np.uint8)
    n_keep = int(round(len(nz) * (1.0 - sparsity)))
    if n_keep > 0:
        order = nz[np.argsort(-nrm.reshape(-1)[nz], kind="stable")]
        keep[order[:n_keep]] = 1
    return keep.reshape(nrm.shape)


def apply_keep(W: np.ndarray, keep: np.ndarray, block: int = BLOCK) -> np.ndarray:
    O, F = W.shape
    m = np.repeat(np.repeat(keep, block, axis=0), block, axis=1)[:O, :F]
    return W * m


def make_block_sparse(W: np.ndarray, sparsity: float, seed: int, block: int = BLOCK) -> np.ndarray:
    """Zero a random `sparsity` share of the 4x4 blocks (the model's structure)."""
    rng = np.random.default_rng(seed)
    O, F = W.shape
    nb = (-(-O // block), -(-F // block))
    kill = rng.permutation(nb[0] * nb[1])[: int(round(sparsity * nb[0] * nb[1]))]
    keep = np.ones(nb[0] * nb[1], dtype=np.uint8)
    keep[kill] = 0
    return apply_keep(W, keep.reshape(nb), block)


@dataclass
class Layer:
    W: np.ndarray                    # float64 [O, F] (model weights, already block-sparse)
    b: np.ndarray                    # float64 [O]
    act: str = "square"              # "square" or "none"
    w_int: torch.Tensor = None       # int32 [O, F] on device (round(W 2^wbits))
    keeps: list = field(default_factory=list)   # per gear: uint8 device masks
    keeps_np: list = field(default_factory=list)
    packed: list = None              # per gear: tensor-core weight images (None: integer pipe)


@dataclass
class ProbeResult:
    layer: int
    gear: int
    snr_db: float
    nsr: float
    input_stats: dict = None   # mean / std / mean square of the layer's decrypted input slots


# largest |w| that three balanced signed byte limbs hold (tensor-core layer)
TC_W_MAX = 127 * (1 + 256 + 65536)


class EncryptedMLP:
    """tensor_cores: run the linear layers on the tensor cores
    (ckks_linear_plain_weights_tc, bit-identical to the integer-pipe layer and
    5x faster on the MLP shape, but dense: a gear's dropped blocks are
    multiplied as zeros); False keeps the integer pipe, whose time shrinks
    with each gear's kept fraction."""

    def __init__(self, ev: Evaluator, layers: list, wbits: int = 20, dare_shift: int | None = None,
                 tensor_cores: bool = True):
        self.ev = ev
        self.wbits = wbits
        self.layers = [l if isinstance(l, Layer) else Layer(*l) for l in layers]
        self.tensor_cores = tensor_cores
        dev = ev.device
        for L in self.layers:
            wq = np.round(L.W * (1 << wbits))
            if np.abs(wq).max() >= 2 ** 24:
                raise ValueError("weights too large for the 24-bit integer path")
            L.w_int = torch.from_numpy(wq.astype(np.int32)).to(dev).contiguous()
            L.keeps_np = [gear_keep(L.W, s) for s in GEAR_SPARSITY]
            L.keeps = [torch.from_numpy(k).to(dev).contiguous() for k in L.keeps_np]
            # the tensor-core layer computes 128 outputs per tile: below 64 outputs
            # the integer pipe is faster (128 -> 10: 0.064 vs 0.12 ms at N = 2^13)
            if tensor_cores and np.abs(wq).max() <= TC_W_MAX and L.W.shape[1] <= 2048 and L.W.shape[0] >= 64:
                L.packed = [ops.linear_tc_pack(wq.astype(np.int64), k, device=dev) for k in L.keeps_np]
        self.dare_shift = dare_shift
        self.timers = {}
        self._bias = {}

    # ---------------------------------------------------------------- plaintext
    @staticmethod
    def plain_forward(layers, x: np.ndarray) -> np.ndarray:
        h = np.asarray(x, dtype=np.float64)
        for L in layers:
            h = h @ L.W.T + L.b
            if L.act == "square":
                h = h * h
        return h

    # ---------------------------------------------------------------- encrypted
    def encrypt_inputs(self, x: np.ndarray) -> Ciphertext:
        """x [B, F] -> F ciphertexts (slot s = sample s) at the top level."""
        xt = torch.from_numpy(np.ascontiguousarray(np.asarray(x, dtype=np.float64).T)).to(self.ev.device)
        return self.ev.encrypt_values(xt.to(torch.complex128))

    def linear(self, X: Ciphertext, li: int, gear: int) -> Ciphertext:
        L = self.layers[li]
        O, F = L.W.shape
        level = X.level
        out = torch.empty((O, 2, level, self.ev.n), dtype=torch.uint64, device=self.ev.device)
        key = (li, X.scale)
        bias = self._bias.get(key)
        if bias is None:   # the integer bias at this input scale, uploaded once
            bias = torch.from_numpy(np.round(L.b * X.scale * (1 << self.wbits)).astype(np.int64)).to(
                self.ev.device).contiguous()
            self._bias[key] = bias
        if L.packed is not None:
            ops.linear_plain_weights_tc(self.ev.ctx, X.data, L.packed[gear], O, bias=bias, out=out)
        else:
            _lib.call("ckks_linear_plain_weights", self.ev.ctx.handle, out.data_ptr(), X.data.data_ptr(),
                      L.w_int.data_ptr(), bias.data_ptr(), L.keeps[gear].data_ptr(), O, F, level,
                      torch.cuda.current_stream().cuda_stream)
        return Ciphertext(out, X.scale * (1 << self.wbits))

    def square(self, Y: Ciphertext) -> Ciphertext:
        return self.ev.mul_relin_rescale(Y, Y)

    def refresh(self, Z: Ciphertext) -> Ciphertext:
        target = self.ev.params.scale
        shift = self.dare_shift if self.dare_shift is not None else max(0, round(math.log2(Z.scale / target)))
        return self.ev.dare_refresh(Z, level_out=self.ev.params.levels, shift_bits=shift)

    def decrypt(self, ct: Ciphertext, n_slots: int) -> np.ndarray:
        return self.ev.decrypt_values(ct, n_slots).real.cpu().numpy()

    # ---------------------------------------------------------------- probe
    def _dev_layer(self, L: Layer):
        if getattr(L, "_Wt", None) is None:
            L._Wt = torch.from_numpy(np.ascontiguousarray(L.W.T)).to(self.ev.device)
            L._b = torch.from_numpy(np.asarray(L.b, dtype=np.float64)).to(self.ev.device)
        return L._Wt, L._b

    def layer_ref(self, li: int, x_in: torch.Tensor) -> torch.Tensor:
        """FP64 gear-0 layer on the device: x_in [B, F] -> [O, B]."""
        L = self.layers[li]
        Wt, b = self._dev_layer(L)
        r = x_in @ Wt + b
        if L.act == "square":
            r = r * r
        return r.T.contiguous()

    def probe(self, li: int, gear: int, out_ct: Ciphertext, x_in: torch.Tensor, B: int) -> tuple:
        """Decrypt the layer output and compare it with the FP64 gear-0 layer
        evaluated on this layer's (decrypted) input; everything stays on the
        device except the two energy sums."""
        dec = self.ev.decrypt_values(out_ct, B).real.contiguous()      # [O, B]
        ref = self.layer_ref(li, x_in)
        st = torch.stack([x_in.mean(), x_in.std(), (x_in * x_in).mean()])
        sums = torch.cat([ops.snr_sums(dec, ref).sum(0), st]).cpu().numpy()   # one host read
        nsr = float(sums[1] / max(sums[0], 1e-300))
        snr = 10 * math.log10(1.0 / max(nsr, 1e-30))
        stats = {"mean": float(sums[2]), "std": float(sums[3]), "ms": float(sums[4])}
        return ProbeResult(li, gear, snr, nsr, stats), dec.T.contiguous()

    # ---------------------------------------------------------------- forward
    def forward(self, x: np.ndarray, choose_gear, on_probe=None, probe_policy=None,
                X: Ciphertext | None = None, fallback_db: float | None = None) -> dict:
        """Run one batch.  choose_gear(layer, info) -> gear; probe_policy(layer,
        gear, info) -> bool decides whether the SNR probe runs (default: always).
        X: the batch already encrypted (else it is encrypted here).
        fallback_db: when a probe measures less than this at a gear > 0, the
        layer is recomputed at gear 0 before its result is used (the probe is
        both the arbiter and the fallback trigger).
        Returns logits [B, O_last] (numpy), the probe records and the number of
        recomputed layers."""
        B = x.shape[0]
        t0 = time.perf_counter()
        if X is None:
            X = self.encrypt_inputs(x)
        x_in = None   # the current layer's input values, for its probe (layer 0: the client's x)
        probes, gears, attempted = [], [], []
        recomputed = 0
        out = None
        for li, L in enumerate(self.layers):
            info = {"layer": li, "level": X.level, "scale": X.scale, "batch": B}
            g = int(choose_gear(li, info))
            gears.append(g)
            attempted.append(g)
            last = li == len(self.layers) - 1
            do_probe = True if probe_policy is None else bool(probe_policy(li, g, info))
            if do_probe and x_in is None:            # the probe needs this layer's input
                x_in = (torch.from_numpy(np.asarray(x, dtype=np.float64)).to(self.ev.device) if li == 0
                        else self.ev.decrypt_values(X, B).real.T.contiguous())
            Y = self.linear(X, li, g)
            if L.act == "square":
                Y = self.square(Y)
            vals = None
            if do_probe:
                pr, vals = self.probe(li, g, Y, x_in, B)
                probes.append(pr)
                if on_probe:
                    on_probe(pr)
                if fallback_db is not None and g > 0 and pr.snr_db < fallback_db:
                    recomputed += 1
                    gears[-1] = 0
                    Y = self.linear(X, li, 0)
                    if L.act == "square":
                        Y = self.square(Y)
                    vals = None
            if last:
                if vals is None:
                    vals = self.ev.decrypt_values(Y, B).real.T
                out = vals.cpu().numpy()
            else:
                X = self.refresh(Y)
                x_in = vals
        torch.cuda.synchronize()
        return {"logits": out, "probes": probes, "gears": gears, "attempted_gears": attempted,
                "recomputed": recomputed, "seconds": time.perf_counter() - t0}


def encrypted_linear_demo(x: np.ndarray, W: np.ndarray, b: np.ndarray, log_n: int = 13, levels: int = 3,
                          seed: int = 0) -> np.ndarray:
    """Y = X W^T + b under CKKS on the GPU (one FC layer, no activation)."""
    from .params import CkksParams
    ev = Evaluator(CkksParams.standard(log_n, levels, seed=seed))
    ev.keygen()
    m = EncryptedMLP(ev, [Layer(np.asarray(W, dtype=np.float64), np.asarray(b, dtype=np.float64), "none")])
    Xc = m.encrypt_inputs(x)
    Y = m.linear(Xc, 0, 0)
    return m.decrypt(Y, x.shape[0]).T

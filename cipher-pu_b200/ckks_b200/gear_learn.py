"""Learned gear controller: features, trace generation, training (on the GPU
with the library's own forward / backward / Adam kernels), checkpointing and
the two controllers compared by the encrypted-inference benchmark.

Trace: one neuron of one encrypted layer evaluation.  Features (16, gear
independent except the per-gear sparsity terms) describe the neuron's
weights, the layer input statistics and the ciphertext level / scale;
targets are the neuron's measured output SNR (dB, FP64 gear-0 layer as the
reference) at each of the four gears.  The network predicts all four at
once; the controller picks the sparsest gear predicted to meet the target and
runs the decrypt-based SNR probe only when the prediction is within the
uncertainty band of the target.

The plain controller is the reference's rule (rtl/m4/adaptive_gear_ctrl.sv:
62-99): downgrade at once when the measured SNR misses the target, upgrade
one gear after HYST_CNT consecutive qualifying measurements, reset to gear 3,
and a probe after every layer of every batch.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .gear import GEAR_SPARSITY
from .mlp import EncryptedMLP, Layer, apply_keep, block_norms, gear_keep, make_block_sparse

N_FEAT = 16
N_GEAR = 4
SCHEMA = 1
SNR_CLIP = (-10.0, 120.0)


# ------------------------------------------------------------------ features
def neuron_features(W: np.ndarray, b: np.ndarray, keeps: list, x_mean: float, x_std: float,
                    x_ms: float, act: str, level: int, scale: float) -> np.ndarray:
    O, F = W.shape
    row_e = (W ** 2).sum(1) + 1e-30
    rb = np.arange(O) // 4
    nz_blocks = (block_norms(W) > 0).sum(1).astype(np.float64) + 1e-9
    feats = np.zeros((O, N_FEAT), dtype=np.float64)
    feats[:, 0] = math.log2(F) / 10.0
    feats[:, 1] = x_mean
    feats[:, 2] = x_std
    feats[:, 3] = math.log10(x_ms + 1e-12) / 4.0
    mu = W @ np.full(F, x_mean) + b
    feats[:, 4] = np.abs(mu) / (np.sqrt(row_e * x_ms) + 1e-12)
    for g, k in enumerate(keeps):
        Wg = apply_keep(W, k)
        dropped = np.clip(1.0 - (Wg ** 2).sum(1) / row_e, 0.0, 1.0)
        feats[:, 5 + g] = np.log10(dropped + 1e-12) / 12.0 + 1.0
        feats[:, 9 + g] = k.sum(1)[rb] / nz_blocks[rb]
    feats[:, 13] = 1.0 if act == "square" else 0.0
    feats[:, 14] = level / 8.0
    feats[:, 15] = math.log2(scale) / 64.0
    return feats


def layer_features(m: EncryptedMLP, li: int, x_in: np.ndarray | None, stats: dict | None, level: int,
                   scale: float) -> np.ndarray:
    L = m.layers[li]
    if stats is None:
        stats = {"mean": float(x_in.mean()), "std": float(x_in.std()), "ms": float((x_in ** 2).mean())}
    return neuron_features(L.W, L.b, L.keeps_np, stats["mean"], stats["std"], stats["ms"], L.act, level,
                           scale)


# ------------------------------------------------------------------ network
class GearNet:
    """The 16 -> 64 -> 64 -> 4 predictor on the GPU (library kernels)."""

    def __init__(self, params: np.ndarray | None = None, seed: int = 0, device=None):
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self.n_params = int(_lib.raw("ckks_gear_mlp_param_count")())
        if params is None:
            from_init = _default_init(seed)
            params = from_init
        self.p = torch.as_tensor(np.asarray(params, dtype=np.float32)).to(self.device).contiguous()
        self.mu = np.zeros(N_FEAT)
        self.sd = np.ones(N_FEAT)

    def _norm(self, X: np.ndarray) -> torch.Tensor:
        Z = (np.asarray(X, dtype=np.float64) - self.mu) / self.sd
        return torch.from_numpy(Z.astype(np.float32)).to(self.device).contiguous()

    def predict(self, X: np.ndarray) -> np.ndarray:
        """features [B, 16] -> predicted SNR dB [B, 4]."""
        x = self._norm(X)
        y = torch.empty((x.shape[0], N_GEAR), dtype=torch.float32, device=self.device)
        _lib.call("ckks_gear_mlp_forward", self.p.data_ptr(), x.data_ptr(), y.data_ptr(), None, x.shape[0],
                  torch.cuda.current_stream().cuda_stream)
        return y.cpu().numpy().astype(np.float64) * 100.0

    def fit(self, X: np.ndarray, T: np.ndarray, epochs: int = 30, batch: int = 1024, lr: float = 2e-3,
            seed: int = 0, val_frac: float = 0.1) -> dict:
        """Adam on the mean squared error (targets in units of 100 dB), cosine
        learning rate.  Under torch.distributed every rank passes the same
        traces (sharded.gen_traces gathers them) and the same seed; each
        minibatch is split over the ranks and the gradients averaged
        (sharded.fit_loop), so every rank ends with the same parameters."""
        from .sharded import fit_loop
        X = np.asarray(X, dtype=np.float64)
        T = np.clip(np.asarray(T, dtype=np.float64), *SNR_CLIP) / 100.0
        self.mu = X.mean(0)
        self.sd = X.std(0) + 1e-6
        rng = np.random.default_rng(seed)
        idx = rng.permutation(len(X))
        nv = int(len(X) * val_frac)
        va, tr = idx[:nv], idx[nv:]
        Xd = self._norm(X)
        Td = torch.from_numpy(T.astype(np.float32)).to(self.device)
        tr_d = torch.from_numpy(tr).to(self.device)
        m = torch.zeros_like(self.p)
        v = torch.zeros_like(self.p)
        grad = torch.empty_like(self.p)
        y = torch.empty((batch, N_GEAR), dtype=torch.float32, device=self.device)
        cache = torch.empty((batch, 128), dtype=torch.float32, device=self.device)
        dcache = torch.empty((batch, 132), dtype=torch.float32, device=self.device)
        st = torch.cuda.current_stream().cuda_stream
        hist = []

        def grad_step(rows):
            b = len(rows)
            bi = tr_d[torch.from_numpy(np.asarray(rows)).to(self.device)]
            xb = Xd[bi].contiguous()
            tb = Td[bi].contiguous()
            _lib.call("ckks_gear_mlp_forward", self.p.data_ptr(), xb.data_ptr(), y.data_ptr(),
                      cache.data_ptr(), b, st)
            _lib.call("ckks_gear_mlp_backward", self.p.data_ptr(), xb.data_ptr(), cache.data_ptr(),
                      y.data_ptr(), tb.data_ptr(), None, grad.data_ptr(), dcache.data_ptr(), b, st)
            return grad, b

        def apply_step(g, step, ep):
            lr_t = lr * 0.5 * (1 + math.cos(math.pi * ep / max(1, epochs)))
            _lib.call("ckks_gear_mlp_adam", self.p.data_ptr(), g.data_ptr(), m.data_ptr(),
                      v.data_ptr(), step, float(lr_t), 0.9, 0.999, 1e-8, st)

        def on_epoch(ep):
            pv = self.predict(X[va])
            hist.append(float(np.sqrt(((pv - T[va] * 100.0) ** 2).mean())))

        steps = fit_loop(len(tr), batch, epochs, rng, grad_step, apply_step, on_epoch)
        return {"val_rmse_db": hist, "train": len(tr), "val": nv, "steps": steps}

    def save(self, path):
        np.savez(path, schema=SCHEMA, params=self.p.cpu().numpy(), mu=self.mu, sd=self.sd)

    @staticmethod
    def load(path, device=None) -> "GearNet":
        z = np.load(path)
        if int(z["schema"]) != SCHEMA:
            raise ValueError("gear network checkpoint schema mismatch")
        g = GearNet(z["params"], device=device)
        g.mu, g.sd = z["mu"], z["sd"]
        return g


def _default_init(seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    parts = [rng.standard_normal((64, 16)) * math.sqrt(2 / 16), np.zeros(64),
             rng.standard_normal((64, 64)) * math.sqrt(2 / 64), np.zeros(64),
             rng.standard_normal((4, 64)) * math.sqrt(1 / 64), np.zeros(4)]
    return np.concatenate([p.reshape(-1) for p in parts]).astype(np.float32)


# ------------------------------------------------------------------ traces
def random_layer(rng, F: int, O: int, act: str, base_sparsity: float, block_spread: float = 0.0) -> Layer:
    """Dense N(0, 1/F) weights with a random base block sparsity; block_spread
    > 0 scales each 4x4 block by exp(N(0, block_spread)) (rows renormalised):
    a compressible layer, whose smallest blocks hold a small share of the
    energy."""
    W = rng.standard_normal((O, F)) / math.sqrt(F)
    if block_spread > 0:
        nb = (-(-O // 4), -(-F // 4))
        s = np.exp(rng.normal(0.0, block_spread, nb))
        W = W * np.repeat(np.repeat(s, 4, 0), 4, 1)[:O, :F]
        W = W / np.sqrt((W ** 2).sum(1, keepdims=True) + 1e-300)   # unit rows, as N(0, 1/F) rows
    W = make_block_sparse(W, base_sparsity, int(rng.integers(1 << 30)))
    b = rng.standard_normal(O) * 0.1
    return Layer(W, b, act)


def random_conv_layer(rng, act: str) -> Layer:
    """A random convolution over a 28 x 28 image as a sparse matrix (channels
    in {4, 8}, kernel 3 or 5, stride 2; the C channels of an output pixel on
    adjacent rows), the structure of the encrypted CNN's first layer."""
    C = int(rng.choice([4, 8]))
    K = int(rng.choice([3, 5]))
    S, IN = 2, 28
    OUT = (IN - K) // S + 1
    kern = rng.standard_normal((C, K, K)) / math.sqrt(K * K)
    W = np.zeros((C * OUT * OUT, IN * IN))
    for c in range(C):
        for i in range(OUT):
            for j in range(OUT):
                r = (i * OUT + j) * C + c
                for di in range(K):
                    W[r, (S * i + di) * IN + S * j:(S * i + di) * IN + S * j + K] = kern[c, di]
    return Layer(W, np.tile(rng.standard_normal(C) * 0.1, OUT * OUT), act)


def gen_traces(ev, n_traces: int, seed: int = 0, batch: int = 256, progress=None) -> tuple:
    """Run random encrypted layers at all four gears; one trace per neuron.
    Three in ten are convolution-structured (random_conv_layer), the rest
    dense block-sparse layers of the MLP family, about a third of those
    compressible (random_layer's block_spread), so the traces cover sparse
    gears that lose almost nothing as well as ones that lose most."""
    rng = np.random.default_rng(seed)
    Xs, Ts = [], []
    total = 0
    while total < n_traces:
        act = "square" if rng.random() < 0.7 else "none"
        if rng.random() < 0.3:
            L = random_conv_layer(rng, act)
        else:
            F = int(rng.choice([128, 256, 512, 784]))
            O = int(rng.choice([16, 32, 64, 128]))
            spread = float(rng.uniform(0.5, 3.0)) if rng.random() < 0.35 else 0.0
            L = random_layer(rng, F, O, act, float(rng.choice([0.25, 0.5, 0.75])), spread)
        O, F = L.W.shape
        m = EncryptedMLP(ev, [L])
        lo, hi = sorted(rng.uniform(0.0, 1.5, 2))
        x = rng.uniform(lo, hi + 0.05, (batch, F))
        X = m.encrypt_inputs(x)
        ref = x @ L.W.T + L.b
        if act == "square":
            ref = ref * ref
        T = np.zeros((O, N_GEAR))
        for g in range(N_GEAR):
            Y = m.linear(X, 0, g)
            if act == "square":
                Y = m.square(Y)
            d = m.decrypt(Y, batch)                       # [O, B]
            err = ((d - ref.T) ** 2).sum(1)
            sig = (ref.T ** 2).sum(1) + 1e-300
            T[:, g] = 10 * np.log10(sig / np.maximum(err, 1e-300))
        feats = layer_features(m, 0, x, None, X.level, X.scale)
        if O > 128:   # a convolution's many neurons: a random 128 of them, so no layer kind dominates
            rows = rng.choice(O, 128, replace=False)
            feats, T = feats[rows], T[rows]
        Xs.append(feats)
        Ts.append(T)
        total += len(T)
        if progress:
            progress(total)
    return np.concatenate(Xs)[:n_traces], np.concatenate(Ts)[:n_traces]


# ------------------------------------------------------------------ controllers
def neuron_signal_weights(W: np.ndarray, b: np.ndarray, stats: dict, act: str) -> np.ndarray:
    """Expected output energy of each neuron from the layer input's mean and
    spread alone: pre-activation y = w.x + b has mean mu = w.1 mean + b and
    variance v = |w|^2 std^2 (independent inputs); E[y^2] = mu^2 + v, and
    for the square activation E[y^4] = mu^4 + 6 mu^2 v + 3 v^2 (Gaussian
    moments).  These weight the per-neuron NSRs into the layer NSR the
    decrypt-based probe measures (total error energy over total signal)."""
    mu = W @ np.full(W.shape[1], stats["mean"]) + b
    v = (W ** 2).sum(1) * stats["std"] ** 2
    if act == "square":
        return mu ** 4 + 6 * mu ** 2 * v + 3 * v ** 2 + 1e-300
    return mu ** 2 + v + 1e-300


def layer_snr_from_neurons(snr_db: np.ndarray, sig_weight: np.ndarray | None = None) -> np.ndarray:
    """[O, G] per-neuron SNR -> [G] layer SNR (signal-weighted NSR average)."""
    nsr = 10.0 ** (-np.clip(np.asarray(snr_db), *SNR_CLIP) / 10.0)
    w = np.ones(nsr.shape[0]) if sig_weight is None else sig_weight
    return -10 * np.log10((w[:, None] * nsr).sum(0) / w.sum())


def nsr_energy(nsr: float) -> int:
    """A probe's noise-to-signal energy ratio as the integer energy the RTL
    controller compares (fixed point, 2^48 = an NSR of 1)."""
    return int(min(max(nsr, 0.0), 2.0 ** 60) * float(1 << 48))


class PlainController:
    """The reference's gear controller, rtl/m4/adaptive_gear_ctrl.sv:43-99,
    run by the library's C state machine (gear.GearCtrl) with one instance per
    layer, fed by the decrypt-based monitor after every layer of every batch
    (the RTL's monitor runs on every flush).  The monitor's noise energy (NSR)
    maps to a raw gear through three thresholds: NSR >= the target's -> gear 0,
    >= target's / 10^(step/10) -> 1, >= target's / 10^(2 step/10) -> 2,
    cleaner -> 3; a lower raw gear takes effect at once, a higher one after
    HYST_CNT agreeing readings; reset gear 3."""

    def __init__(self, n_layers: int, target_db: float, step_db: float = 10.0, hyst: int = 3):
        from .gear import GearCtrl
        self.target = target_db
        th = [nsr_energy(10.0 ** (-(target_db + k * step_db) / 10.0)) for k in range(3)]
        self.ctl = [GearCtrl(thresholds=tuple(th), hyst_cnt=hyst) for _ in range(n_layers)]
        self.probes = 0

    def choose(self, li, info):
        return self.ctl[li].gear

    def probe_policy(self, li, g, info):
        self.probes += 1
        return True

    def on_probe(self, pr):
        self.ctl[pr.layer].flush(nsr_energy(pr.nsr))


class LearnedController:
    """Predict each gear's layer SNR from features; take the sparsest gear
    predicted >= target + margin.  The decrypt-based probe (the plain monitor)
    stays as arbiter and fallback: it runs on the first use of a (layer, gear),
    every `audit_every`-th batch, and whenever the prediction lies within
    `band_db` of the target; a measurement below the target caps the layer's
    gear and triggers the recompute."""

    def __init__(self, m: EncryptedMLP, net: GearNet, target_db: float, margin_db: float = 3.0,
                 band_db: float = 6.0, audit_every: int = 8):
        self.m, self.net = m, net
        self.target, self.margin, self.band, self.audit = target_db, margin_db, band_db, audit_every
        self.cap = [N_GEAR - 1] * len(m.layers)
        self.pred = {}
        self.verified = set()
        self.probes = 0
        self.stats = {}
        self.calls = [0] * len(m.layers)

    # Calibration: until a layer's input statistics are known (the first
    # batch), the controller runs gear 0 and probes every layer; the probes'
    # decrypted layer inputs give the statistics (ProbeResult.input_stats), so
    # the features come from monitor quantities measured inside the stream.
    def calibrated(self, li: int) -> bool:
        return li in self.stats

    def set_input_stats(self, li: int, stats: dict):
        self.stats[li] = stats
        self.pred.pop(li, None)

    def predicted(self, li: int, info) -> np.ndarray:
        key = (info["level"], round(math.log2(info["scale"]), 3))
        hit = self.pred.get(li)
        if hit is None or hit[0] != key:
            st = self.stats[li]
            L = self.m.layers[li]
            feats = layer_features(self.m, li, None, st, info["level"], info["scale"])
            w = neuron_signal_weights(L.W, L.b, st, L.act)
            hit = (key, layer_snr_from_neurons(self.net.predict(feats), w))
            self.pred[li] = hit
        return hit[1]

    def choose(self, li, info):
        if not self.calibrated(li):
            return 0
        p = self.predicted(li, info)
        ok = [g for g in range(N_GEAR) if p[g] >= self.target + self.margin and g <= self.cap[li]]
        return max(ok) if ok else 0

    def probe_policy(self, li, g, info):
        self.calls[li] += 1
        if not self.calibrated(li):
            self.probes += 1
            return True
        p = self.predicted(li, info)
        need = ((li, g) not in self.verified or abs(p[g] - self.target) < self.band
                or (self.audit and self.calls[li] % self.audit == 0))
        if need:
            self.probes += 1
        return need

    def on_probe(self, pr):
        if pr.input_stats is not None and not self.calibrated(pr.layer):
            self.set_input_stats(pr.layer, pr.input_stats)
        if pr.snr_db < self.target:
            self.cap[pr.layer] = max(0, pr.gear - 1)
            self.verified.discard((pr.layer, pr.gear))
        else:
            self.verified.add((pr.layer, pr.gear))

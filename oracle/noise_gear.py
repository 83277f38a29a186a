"""Noise monitor, gear controllers and block sparsity (test infrastructure).

Restatements:
  * ``noise_energy``      rtl/m4/noise_monitor.sv:42-78 / scripts/verify_m4_h_multilayer.py:162
                          (E = sum min(c, q-c)^2 / count, r_hat = sqrt(E) / q); the RTL's
                          integer division is ``noise_energy_int`` (floor, 106-bit sum).
  * ``welford``           scripts/verify_m4_h_multilayer.py:193 layer_sigma_welford
                          (sample std of min(c, q-c)).
  * ``GearCtrlRTL``       rtl/m4/adaptive_gear_ctrl.sv:43-99 (energy thresholds, hysteresis:
                          upgrade after HYST_CNT agreeing candidates, downgrade at once,
                          manual override), reset gear 3.
  * ``GEO`` / ``compute_extra`` / ``total_growth`` / ``select_gear_safe`` /
    ``select_gear_with_hysteresis``  scripts/verify_m4_h_adaptive.py:37-129.
  * ``AgcRhat``           scripts/verify_project_b_mlp_reference.py:279 AdaptiveGearCtrl.
  * ``gear_config``       scripts/verify_m4_a_gear_ctrl.py:41 get_gear_config.
  * ``post_process_block`` scripts/verify_m4_d_approx_mult.py:50.
  * ``block_sparse_mask`` scripts/exp_e10_sparsity_sweep_v2.py:102 apply_block_sparse_mask.
"""
from __future__ import annotations

import math

import numpy as np

# ------------------------------------------------------------------ noise monitor


def noise_energy(coeffs, q):
    total = 0
    n = len(coeffs)
    for c in coeffs:
        a = c if c <= q - c else q - c
        total += a * a
    e = total / n
    return e, math.sqrt(e) / q


def noise_energy_int(coeffs, q, acc_bits=106):
    """(floor(sum / count), count, saturated) as the RTL accumulates it."""
    total = 0
    sat = False
    for c in coeffs:
        a = c if c <= q - c else q - c
        if not sat:
            total += a * a
            if total >= (1 << acc_bits):
                total &= (1 << acc_bits) - 1
                sat = True
    return total // len(coeffs), len(coeffs), sat


def welford(coeffs, q):
    n = 0
    mean = 0.0
    m2 = 0.0
    for c in coeffs:
        x = float(c if c <= q - c else q - c)
        n += 1
        d = x - mean
        mean += d / n
        m2 += d * (x - mean)
    sd = 0.0 if n < 2 else math.sqrt(m2 / (n - 1))
    return sd, (sd / q if q else 0.0)


# ------------------------------------------------------------------ RTL gear controller
class GearCtrlRTL:
    def __init__(self, th1=500, th2=200, th3=50, hyst_cnt=3):
        self.th = (th1, th2, th3)
        self.hyst_cnt = hyst_cnt
        self.gear = 3
        self.counter = 0
        self.candidate = 3

    def raw(self, energy):
        th1, th2, th3 = self.th
        if energy >= th1:
            return 0
        if energy >= th2:
            return 1
        if energy >= th3:
            return 2
        return 3

    def flush(self, energy, hysteresis=True, manual_en=False, manual_gear=0):
        raw = self.raw(energy)
        if manual_en:
            self.gear = manual_gear
            self.counter = 0
        elif hysteresis:
            if raw > self.gear:
                cnt_before = self.counter
                if raw == self.candidate:
                    self.counter += 1
                else:
                    self.candidate = raw
                    self.counter = 1
                if cnt_before >= self.hyst_cnt:
                    self.candidate = self.gear
                    self.gear = raw
                    self.counter = 0
            elif raw < self.gear:
                self.gear = raw
                self.counter = 0
                self.candidate = raw
            else:
                self.counter = 0
                self.candidate = raw
        else:
            self.gear = raw
        return manual_gear if manual_en else self.gear


# ------------------------------------------------------------------ analytic gear model
N_PROD = 2 ** 14
Q_PROD = 2 ** 44 + 131073
R_INIT = 1.0 / (1 << 24)
R_MAX = 0.5
BASE_GROWTH = 1.55
SIGMA_0 = Q_PROD * R_INIT
HYSTERESIS_FRAC = 0.05
GEO = [
    {"threshold": 0, "trunc_bits": 0, "skip_rate": 0.00},
    {"threshold": 4096, "trunc_bits": 0, "skip_rate": 0.15},
    {"threshold": 16384, "trunc_bits": 9, "skip_rate": 0.30},
    {"threshold": 65536, "trunc_bits": 17, "skip_rate": 0.50},
]


def compute_extra(g):
    sigma_skip = math.sqrt(N_PROD * g["skip_rate"]) * g["threshold"] / math.sqrt(12.0)
    sigma_trunc = (2.0 ** g["trunc_bits"]) / math.sqrt(12.0)
    extra = 1.0 + (sigma_skip + sigma_trunc) / (SIGMA_0 * (BASE_GROWTH - 1))
    return sigma_skip, sigma_trunc, extra


def total_growth(g):
    return BASE_GROWTH * compute_extra(g)[2]


def select_gear_safe(r):
    for gi in range(3, -1, -1):
        if r * total_growth(GEO[gi]) < R_MAX:
            return gi
    return 0


def select_gear_with_hysteresis(g_new, g_old, r):
    if g_new < g_old:
        return g_new
    if g_new > g_old:
        if r * total_growth(GEO[g_new]) * (1 + HYSTERESIS_FRAC) < R_MAX:
            return g_new
        return g_old
    return g_new


R_MAX_TABLE = (0.10, 0.20, 0.35, 0.55)


class AgcRhat:
    """Hysteresis on the strictest gear tolerating r_hat (HYST_CNT = 2)."""

    def __init__(self, hyst=2):
        self.gear, self.cnt, self.target, self.hyst = 3, 0, -1, hyst

    def step(self, r):
        target = next((g for g, rm in enumerate(R_MAX_TABLE) if rm >= r), 0)
        if target != self.gear:
            if self.target != target:
                self.target, self.cnt = target, 0
            else:
                self.cnt += 1
            if self.cnt >= self.hyst:
                self.gear, self.cnt, self.target = target, 0, -1
        return self.gear


_GEAR_TABLE = {0: (0, 0, False, False), 1: (4096, 0, False, False),
               2: (16384, 9, True, True), 3: (65536, 17, True, True)}


def gear_config(g, thresh_ovr=0, ovr_en=False):
    th, tb, ap, fr = _GEAR_TABLE.get(g, _GEAR_TABLE[0])
    return {"threshold": thresh_ovr if ovr_en else th, "trunc_bits": tb, "approx_mult": ap,
            "fast_rescale": fr}


# ------------------------------------------------------------------ sparsity
def post_process_block(x, threshold, use_approx, q=113, B=1):
    n = len(x)
    B = max(B, 1)
    blocks = [x] if B > n else [x[i:i + B] for i in range(0, n, B)]
    out, skipped = [], 0
    for blk in blocks:
        if not blk:
            continue
        m = max(min(v, q - v) for v in blk)
        if use_approx and threshold != 0 and m < threshold:
            skipped += 1
            out.extend([0] * len(blk))
        else:
            out.extend(blk)
    return out, skipped


def block_sparse_mask(W, threshold, B):
    """Flat blocks of B consecutive weights whose max |w| < threshold are zeroed."""
    flat = np.asarray(W).reshape(-1).copy()
    nb = len(flat) // B
    blk = np.abs(flat[:nb * B]).reshape(nb, B).max(axis=1)
    kill = blk < threshold
    flat[:nb * B] = np.where(np.repeat(kill, B), 0.0, flat[:nb * B])
    skip = int(kill.sum())
    return flat.reshape(np.shape(W)), skip, nb, (nb - skip) / nb

"""Failure detection, with every fault injected on the HOST (no GPU fault).

The reference's fault model (scripts/gen_e52_fault.py: F1 single-bit flips
in the ciphertext datapath and in the keyswitch key registers, detection by
the noise monitor's energy, rtl/m4/noise_monitor.sv) is exercised here as:
  * a bit flipped in one evaluation-domain word of a ciphertext in host
    memory, or in one word of the relinearisation key, before upload;
  * the corrupted data runs through the ordinary GPU ct-mult;
  * the decrypted limb-0 polynomial goes through the saturating noise monitor
    (ckks_noise_energy_sat), whose window is sized so that a healthy product
    stays far below it: exactly the corrupted pairs are flagged;
  * recovery: recomputing from the intact host copy (or the re-uploaded key)
    gives results bit-identical to the fault-free run.
A key-word flip, any bit, corrupts the whole limb: the ModDown multiplies the
error by p^-1 mod q and the decryption's inverse transform spreads it over
every coefficient as residues of size ~q, far above a message of scale 2^35.
"""
import math

import numpy as np
import pytest

from oracle import noise_gear as NG

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ev(cuda):
    from ckks_b200.evaluator import Evaluator
    from ckks_b200.params import CkksParams
    e = Evaluator(CkksParams.standard(12, 3, seed=21))
    e.keygen()
    return e


def _window_bits(q: int, n: int) -> int:
    """Monitor width: flag once the mean square passes (q / 16)^2, i.e. once
    coefficients look like residues spread over the whole of [0, q)."""
    return int(math.log2(n)) + 2 * (q.bit_length() - 4)


def _limb0_flags(ev, ct):
    """Decrypt, monitor limb 0 of every ciphertext: (sums, saturated)."""
    import ckks_b200.ops as ops
    dec = ops.decrypt(ev.ctx, ct.data, ev.sk.s_eval)           # [C, level, N] coefficient residues
    q0 = ev.params.q[0]
    rows = dec[:, 0, :].contiguous()
    return ops.noise_energy_sat(rows, q0, _window_bits(q0, ev.n))


def test_saturation_flag_matches_rtl_model(cuda):
    """The flag equals the RTL accumulator's (oracle noise_energy_int) for
    every window width; below saturation the sums agree exactly."""
    import ckks_b200.ops as ops
    rng = np.random.default_rng(3)
    q = 35184371884033
    x = np.zeros((6, 4096), dtype=np.uint64)
    x[0] = rng.integers(0, q, 4096, dtype=np.uint64)                   # uniform residues
    x[1] = rng.integers(0, 1 << 20, 4096, dtype=np.uint64)             # small positive
    x[2] = (q - rng.integers(1, 1 << 20, 4096, dtype=np.uint64))       # small negative
    x[3] = q // 2                                                      # the largest |c|
    x[4] = 0
    x[5] = rng.integers(0, 1 << 36, 4096, dtype=np.uint64)
    for bits in (40, 64, 90, 97, 106, 128):
        sums, sat = ops.noise_energy_sat(ops.to_device(x), q, bits)
        exact = ops.noise_energy(ops.to_device(x), q)
        for r in range(6):
            _, _, want_sat = NG.noise_energy_int([int(c) for c in x[r]], q, bits)
            assert sat[r] == want_sat, (bits, r)
            assert sums[r] == (exact[r] if not want_sat else (1 << bits) - 1), (bits, r)


def test_ciphertext_bit_flip_flagged_and_recomputed(ev):
    import torch
    import ckks_b200.ops as ops
    from ckks_b200.evaluator import Ciphertext
    rng = np.random.default_rng(4)
    x = rng.uniform(-1, 1, (8, 2048))
    y = rng.uniform(-1, 1, (8, 2048))
    cx, cy = ev.encrypt_values(x, level=3), ev.encrypt_values(y, level=3)
    clean = ev.mul_relin_rescale(cx, cy)
    ok_dec = ops.to_host(ops.decrypt(ev.ctx, clean.data, ev.sk.s_eval))
    sums, sat = _limb0_flags(ev, clean)
    assert not any(sat), sums
    # F1: one bit of one evaluation-domain word of c0 of pair 3, in host memory
    host = cx.data.cpu().numpy().copy()
    for bit in (0, 20, 44):
        bad = host.copy()
        bad[3, 0, 0, 1234] ^= np.uint64(1 << bit)
        cbad = Ciphertext(torch.from_numpy(bad).to(ev.device), cx.scale)
        out = ev.mul_relin_rescale(cbad, cy)
        sums_b, sat_b = _limb0_flags(ev, out)
        assert sat_b == [i == 3 for i in range(8)], (bit, sat_b)
        # recovery: recompute from the intact host copy
        again = ev.mul_relin_rescale(Ciphertext(torch.from_numpy(host).to(ev.device), cx.scale), cy)
        assert np.array_equal(ops.to_host(ops.decrypt(ev.ctx, again.data, ev.sk.s_eval)), ok_dec)


def test_key_word_flip_flagged_and_reupload_recovers(ev):
    import ckks_b200.ops as ops
    rng = np.random.default_rng(5)
    x = rng.uniform(-1, 1, (4, 2048))
    cx = ev.encrypt_values(x, level=3)
    ok = ops.to_host(ev.mul_relin_rescale(cx, cx).data)
    raw = ev.ksk.cpu().numpy().copy()                  # [dnum, 2, L + 1, N] evaluation domain
    good_rlk = ev.rlk
    try:
        for (j, k, limb, bit) in ((0, 0, 0, 0), (1, 1, 0, 30), (2, 0, 1, 44)):
            bad = raw.copy()
            bad[j, k, limb, 77] ^= np.uint64(1 << bit)
            ev.rlk = ops.relin_key_prepare(ev.ctx, ops.to_device(bad))
            out = ev.mul_relin_rescale(cx, cx)
            dec = ops.decrypt(ev.ctx, out.data, ev.sk.s_eval)
            # the corrupted limb of every pair leaves the monitor's window
            q = ev.params.q[limb]
            _, sat = ops.noise_energy_sat(dec[:, limb, :].contiguous(), q, _window_bits(q, ev.n))
            assert all(sat), (j, k, limb, bit)
    finally:
        ev.rlk = good_rlk
    # recovery: the intact key, re-prepared from the host copy
    ev.rlk = ops.relin_key_prepare(ev.ctx, ops.to_device(raw))
    assert np.array_equal(ops.to_host(ev.mul_relin_rescale(cx, cx).data), ok)


def test_gear_controller_reacts_to_the_monitor(ev):
    """The library's RTL gear controller (ckks_gear_ctrl_*, the policy of
    rtl/m4/adaptive_gear_ctrl.sv:43-99) driven by the monitor on a stream of
    ct-mult results: a corrupted result's saturated window (reported as the
    window's full-scale energy) drops the gear to 0 at once; clean windows
    raise it again only after HYST_CNT + 1 agreeing readings; a recompute from
    the intact copy restores the result exactly."""
    import torch
    import ckks_b200.ops as ops
    from ckks_b200.evaluator import Ciphertext
    from ckks_b200.gear import GearCtrl
    rng = np.random.default_rng(7)
    x = rng.uniform(-1, 1, (2, 2048))
    cx = ev.encrypt_values(x, level=3)
    q0 = ev.params.q[0]
    bits = _window_bits(q0, ev.n)
    full = (1 << bits) - 1
    # thresholds: gear 3 below 1/1024 of the window, gear 0 from half of it
    ctl = GearCtrl(thresholds=(full // 2, full // 64, full // 1024), hyst_cnt=3)
    host = cx.data.cpu().numpy()
    gears, flags = [], []
    for step in range(12):
        data = host.copy()
        if step == 2:
            data[1, 1, 2, 99] ^= np.uint64(1 << 17)      # F1 in c1, limb 2, pair 1
        c = Ciphertext(torch.from_numpy(data).to(ev.device), cx.scale)
        out = ev.mul_relin_rescale(c, c)
        sums, sat = _limb0_flags(ev, out)
        if any(sat):                                      # recover: recompute from the intact copy
            out2 = ev.mul_relin_rescale(Ciphertext(torch.from_numpy(host).to(ev.device), cx.scale),
                                        Ciphertext(torch.from_numpy(host).to(ev.device), cx.scale))
            assert not any(_limb0_flags(ev, out2)[1])
        flags.append(any(sat))
        gears.append(ctl.flush(max(sums)))
    assert flags == [i == 2 for i in range(12)]
    # reset gear 3; the saturated reading forces 0 at once; the clean readings that
    # follow propose 3 again, adopted on the fourth agreeing one (hyst_cnt = 3)
    assert gears[:2] == [3, 3] and gears[2] == 0
    assert gears[3:6] == [0, 0, 0] and gears[6] == 3

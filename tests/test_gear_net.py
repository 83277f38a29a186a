"""Learned gear controller network: CPU oracle gradient check, GPU kernels vs
the oracle, training, and the trained network's gain over the plain
controller."""
from pathlib import Path

import numpy as np
import pytest

from oracle import gear_mlp as GM

ROOT = Path(__file__).resolve().parents[1]
NET = ROOT / "cipher-pu_b200" / "ckks_b200" / "data" / "gear_net.npz"


def test_oracle_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = GM.init(1) + rng.standard_normal(GM.N_PARAMS) * 0.05
    x = rng.standard_normal((32, 16))
    t = rng.standard_normal((32, 4))
    mask = (rng.random((32, 4)) < 0.8).astype(np.float64)
    g = GM.backward(p, x, t, mask)
    idx = rng.choice(GM.N_PARAMS, 200, replace=False)
    ng = GM.numeric_grad(p, x, t, mask, idx)
    assert np.allclose(g[idx], ng[idx], rtol=1e-5, atol=1e-7)


@pytest.mark.gpu
def test_gpu_kernels_match_oracle(cuda):
    import torch
    from ckks_b200 import _lib
    assert _lib.raw("ckks_gear_mlp_param_count")() == GM.N_PARAMS
    rng = np.random.default_rng(2)
    B = 1024
    p = GM.init(3).astype(np.float32)
    x = rng.standard_normal((B, 16)).astype(np.float32)
    t = rng.standard_normal((B, 4)).astype(np.float32)
    dp, dx, dt = (torch.from_numpy(a).cuda() for a in (p, x, t))
    y = torch.empty((B, 4), dtype=torch.float32, device="cuda")
    cache = torch.empty((B, 128), dtype=torch.float32, device="cuda")
    dcache = torch.empty((B, 132), dtype=torch.float32, device="cuda")
    grad = torch.empty(GM.N_PARAMS, dtype=torch.float32, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    _lib.call("ckks_gear_mlp_forward", dp.data_ptr(), dx.data_ptr(), y.data_ptr(), cache.data_ptr(), B, st)
    yo, _ = GM.forward(p.astype(np.float64), x.astype(np.float64))
    assert np.allclose(y.cpu().numpy(), yo, rtol=1e-4, atol=1e-4)
    _lib.call("ckks_gear_mlp_backward", dp.data_ptr(), dx.data_ptr(), cache.data_ptr(), y.data_ptr(),
              dt.data_ptr(), None, grad.data_ptr(), dcache.data_ptr(), B, st)
    go = GM.backward(p.astype(np.float64), x.astype(np.float64), t.astype(np.float64))
    gg = grad.cpu().numpy()
    assert np.abs(gg - go).max() <= 1e-4 * max(1.0, np.abs(go).max())
    # Adam step
    m = torch.zeros_like(dp)
    v = torch.zeros_like(dp)
    _lib.call("ckks_gear_mlp_adam", dp.data_ptr(), grad.data_ptr(), m.data_ptr(), v.data_ptr(), 1, 1e-3,
              0.9, 0.999, 1e-8, st)
    mm = 0.1 * gg
    vv = 0.001 * gg * gg
    want = p - 1e-3 * (mm / 0.1) / (np.sqrt(vv / 0.001) + 1e-8)
    assert np.allclose(dp.cpu().numpy(), want, rtol=1e-5, atol=1e-6)


@pytest.mark.gpu
def test_gpu_training_reduces_loss(cuda):
    from ckks_b200.gear_learn import GearNet
    rng = np.random.default_rng(4)
    X = rng.standard_normal((20000, 16))
    T = np.stack([X[:, :4].sum(1) * 10 + 50, X[:, 4] * 20 + 30, np.abs(X[:, 5]) * 30, X[:, 6] * X[:, 7] * 5 + 10], 1)
    net = GearNet(seed=0)
    before = np.sqrt(((net.predict(X[:2000]) - T[:2000]) ** 2).mean())
    h = net.fit(X, T, epochs=15)
    assert h["val_rmse_db"][-1] < 0.25 * before


@pytest.mark.gpu
def test_learned_controller_gains_over_plain(cuda):
    """The trained predictor lets the controller skip most SNR probes: at least
    1.15x the plain controller's samples/s, SNR no worse than 0.5 dB below, the
    same top-1 agreement, on the encrypted MLP (N = 2^13, L = 4)."""
    if not NET.exists():
        pytest.fail(f"trained gear network missing: {NET}")
    from ckks_b200.train_gear import compare
    r = compare(NET, "mlp", batches=8, batch=1024)
    assert r["learned"]["probes"] < r["plain"]["probes"]
    assert r["learned"]["snr_db"] >= r["plain"]["snr_db"] - 0.5
    assert r["learned"]["top1_agreement"] >= r["plain"]["top1_agreement"]
    assert r["speedup"] >= 1.15, r

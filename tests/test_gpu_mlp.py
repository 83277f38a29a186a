"""Encrypted linear layer (bit-exact vs the oracle) and the encrypted MLP
(784-128-10, square activation, DARE between layers) vs the FP64 plaintext
model: top-1 agreement and logit SNR per gear."""
import numpy as np
import pytest

from oracle.linear import linear_plain

pytestmark = pytest.mark.gpu


def _np(t):
    return t.cpu().numpy()


def test_linear_kernel_bit_exact(cuda):
    import torch
    from ckks_b200 import _lib
    from ckks_b200.context import Context
    from ckks_b200.params import CkksParams
    P = CkksParams.standard(6, 3)
    ctx = Context.get(6, P.primes, n_special=1)
    rng = np.random.default_rng(0)
    F, O, L, n = 22, 13, 3, 64
    x = np.zeros((F, 2, L, n), dtype=np.uint64)
    for i, q in enumerate(P.q):
        x[:, :, i, :] = rng.integers(0, q, size=(F, 2, n), dtype=np.uint64)
    w = rng.integers(-(2 ** 23), 2 ** 23, size=(O, F)).astype(np.int32)
    bias = rng.integers(-(2 ** 62), 2 ** 62, size=O, dtype=np.int64)
    keep = (rng.random((-(-O // 4), -(-F // 4))) < 0.6).astype(np.uint8)
    for kp in (None, keep):
        dx = torch.from_numpy(x.view(np.int64)).cuda().view(torch.uint64).contiguous()
        out = torch.empty((O, 2, L, n), dtype=torch.uint64, device="cuda")
        dw = torch.from_numpy(w).cuda()
        db = torch.from_numpy(bias).cuda()
        dk = torch.from_numpy(kp).cuda() if kp is not None else None
        _lib.call("ckks_linear_plain_weights", ctx.handle, out.data_ptr(), dx.data_ptr(), dw.data_ptr(),
                  db.data_ptr(), dk.data_ptr() if dk is not None else None, O, F, L,
                  torch.cuda.current_stream().cuda_stream)
        got = _np(out.view(torch.int64)).astype(np.uint64)
        assert np.array_equal(got, linear_plain(x, w, bias, kp, P.q))


def _model(seed=0):
    from ckks_b200.mlp import Layer, make_block_sparse
    rng = np.random.default_rng(seed)
    W1 = make_block_sparse(rng.standard_normal((128, 784)) / np.sqrt(784), 0.5, seed + 1)
    W2 = make_block_sparse(rng.standard_normal((10, 128)) / np.sqrt(128), 0.5, seed + 2)
    b1 = rng.standard_normal(128) * 0.1
    b2 = rng.standard_normal(10) * 0.1
    return [Layer(W1, b1, "square"), Layer(W2, b2, "none")]


@pytest.mark.parametrize("log_n", [12, 13])
def test_encrypted_mlp_vs_fp64(cuda, log_n):
    from ckks_b200.evaluator import Evaluator
    from ckks_b200.mlp import EncryptedMLP
    from ckks_b200.params import CkksParams
    ev = Evaluator(CkksParams.standard(log_n, 4, seed=11))
    ev.keygen()
    layers = _model()
    m = EncryptedMLP(ev, layers)
    rng = np.random.default_rng(1)
    B = 256
    x = rng.uniform(0, 1, (B, 784))
    ref = EncryptedMLP.plain_forward(layers, x)
    res = m.forward(x, choose_gear=lambda li, info: 0)
    got = res["logits"]
    nsr = ((got - ref) ** 2).sum() / (ref ** 2).sum()
    snr = 10 * np.log10(1 / nsr)
    assert snr > 60, snr                                   # gear 0: weight rounding + CKKS noise only
    assert (got.argmax(1) == ref.argmax(1)).mean() == 1.0
    assert all(p.snr_db > 60 for p in res["probes"])
    # higher gears drop weight blocks: SNR falls monotonically, still agree mostly
    snrs = []
    for g in (1, 2, 3):
        r = m.forward(x, choose_gear=lambda li, info, g=g: g)
        d = r["logits"]
        snrs.append(10 * np.log10((ref ** 2).sum() / ((d - ref) ** 2).sum()))
    assert snrs[0] > snrs[1] > snrs[2]

"""Host-buffer ct-mult entry: chunked H2D / kernels / D2H pipeline over three
streams must give the device-buffer entry's results bit for bit, for ragged
batches (last chunk short), more chunks than streams (workspace slots reused)
and the empty batch; the first pairs are also checked against the oracle."""
import numpy as np
import pytest
import torch

from oracle import rns_ckks as R

pytestmark = pytest.mark.gpu


def _rand_ct(rng, shape, qs):
    x = np.empty(shape, dtype=np.uint64)
    for i, q in enumerate(qs):
        x[..., i, :] = rng.integers(0, q, size=x[..., i, :].shape, dtype=np.uint64)
    return x


@pytest.mark.parametrize("n_ct,chunk", [(37, 8), (5, 32), (1, 1)])
def test_host_entry_matches_device_entry(cuda, n_ct, chunk):
    import ckks_b200.ops as ops
    from ckks_b200.context import Context
    from ckks_b200.params import CkksParams
    P = CkksParams.standard(12, 3)
    ctx = Context.get(12, P.primes, n_special=1)
    rng = np.random.default_rng(1000 + n_ct)
    qs = list(P.q)
    a = _rand_ct(rng, (n_ct, 2, 3, 4096), qs)
    b = _rand_ct(rng, (n_ct, 2, 3, 4096), qs)
    ksk = _rand_ct(rng, (3, 2, 4, 4096), qs + [P.special])
    key = ops.relin_key_prepare(ctx, ops.to_device(ksk))
    dev = ops.to_host(ops.ct_mul_relin_rescale(ctx, ops.to_device(a), ops.to_device(b), key))
    ha = torch.from_numpy(a.view(np.int64)).view(torch.uint64).pin_memory()
    hb = torch.from_numpy(b.view(np.int64)).view(torch.uint64).pin_memory()
    host = ops.ct_mul_relin_rescale_host(ctx, ha, hb, key, chunk=chunk)
    torch.cuda.synchronize()
    got = host.view(torch.int64).numpy().view(np.uint64)
    assert np.array_equal(got, dev)
    k = min(n_ct, 2)
    assert np.array_equal(got[:k], R.ct_mul_relin_rescale(a[:k], b[:k], ksk, qs, P.special))


def test_host_entry_empty_and_small_workspace(cuda):
    import ckks_b200.ops as ops
    from ckks_b200 import _lib
    from ckks_b200.context import Context
    from ckks_b200.params import CkksParams
    P = CkksParams.standard(12, 3)
    ctx = Context.get(12, P.primes, n_special=1)
    key = torch.zeros((3, 2, 4, 4096, 2), dtype=torch.uint64, device="cuda")
    e = torch.empty((0, 2, 3, 4096), dtype=torch.uint64).pin_memory()
    out = ops.ct_mul_relin_rescale_host(ctx, e, e, key, chunk=4)
    assert out.shape == (0, 2, 2, 4096)
    a = torch.zeros((4, 2, 3, 4096), dtype=torch.uint64).pin_memory()
    need = ops.ct_mul_host_workspace_bytes(ctx, 4, 3)
    ws = torch.empty(need // 8 - 1, dtype=torch.uint64, device="cuda")
    with pytest.raises(_lib.CkksError, match="workspace"):
        _lib.call("ckks_ct_mul_relin_rescale_host", ctx.handle, a.data_ptr(), a.data_ptr(),
                  a.data_ptr(), key.data_ptr(), 4, 3, 4, ws.data_ptr(), ws.numel() * 8,
                  torch.cuda.current_stream().cuda_stream)


@pytest.mark.parametrize("n_ct,chunk", [(37, 8), (3, 64)])
def test_host48_entry_matches_device_entry(cuda, n_ct, chunk):
    """48-bit wire format: packed host inputs -> packed host outputs equal the
    device entry's results."""
    import ckks_b200.ops as ops
    from ckks_b200.context import Context
    from ckks_b200.params import CkksParams
    P = CkksParams.standard(12, 3)
    ctx = Context.get(12, P.primes, n_special=1)
    rng = np.random.default_rng(2000 + n_ct)
    qs = list(P.q)
    a = _rand_ct(rng, (n_ct, 2, 3, 4096), qs)
    b = _rand_ct(rng, (n_ct, 2, 3, 4096), qs)
    ksk = _rand_ct(rng, (3, 2, 4, 4096), qs + [P.special])
    key = ops.relin_key_prepare(ctx, ops.to_device(ksk))
    dev = ops.to_host(ops.ct_mul_relin_rescale(ctx, ops.to_device(a), ops.to_device(b), key))
    ta = torch.from_numpy(a.view(np.int64)).view(torch.uint64)
    tb = torch.from_numpy(b.view(np.int64)).view(torch.uint64)
    a48 = ops.pack48_host(ta).pin_memory()
    b48 = ops.pack48_host(tb).pin_memory()
    out48 = ops.ct_mul_relin_rescale_host48(ctx, a48, b48, key, n_ct, 3, chunk=chunk)
    torch.cuda.synchronize()
    got = ops.unpack48_host(out48, dev.shape).view(torch.int64).numpy().view(np.uint64)
    assert np.array_equal(got, dev)


def test_device_pack48_round_trip(cuda):
    import ckks_b200.ops as ops
    from ckks_b200 import _lib
    rng = np.random.default_rng(9)
    for n in (1, 8, 13, 4096 + 5):
        x = torch.from_numpy(rng.integers(0, 1 << 47, n, dtype=np.int64)).view(torch.uint64).cuda()
        packed = torch.empty(6 * n + 16, dtype=torch.uint8, device="cuda")
        st = torch.cuda.current_stream().cuda_stream
        _lib.call("ckks_pack48", packed.data_ptr(), x.data_ptr(), n, st)
        assert torch.equal(packed[:6 * n].cpu(), ops.pack48_host(x.cpu()))
        back = torch.empty(n + 2, dtype=torch.uint64, device="cuda")
        _lib.call("ckks_unpack48", back.data_ptr(), packed.data_ptr(), n, st)
        assert torch.equal(back[:n].cpu(), x.cpu())


def test_host_async_entry_back_to_back_calls(cuda):
    """Four stream-ordered host-buffer calls on different batches, enqueued
    back to back on one shared workspace (8 chunks over three streams, so
    slots are reused across calls), joined once: every output equals the
    device-buffer entry's; the 48-bit wire-format form likewise."""
    import ckks_b200.ops as ops
    from ckks_b200 import _lib
    from ckks_b200.context import Context
    from ckks_b200.params import CkksParams
    P = CkksParams.standard(12, 3)
    ctx = Context.get(12, P.primes, n_special=1)
    rng = np.random.default_rng(77)
    qs = list(P.q)
    ksk = _rand_ct(rng, (3, 2, 4, 4096), qs + [P.special])
    key = ops.relin_key_prepare(ctx, ops.to_device(ksk))
    chunk, n_ct = 4, (9, 6, 1, 8)
    ws = torch.empty((ops.ct_mul_host_workspace_bytes(ctx, chunk, 3) + 7) // 8, dtype=torch.uint64,
                     device=key.device)
    batches, outs, exps = [], [], []
    for m in n_ct:
        a = _rand_ct(rng, (m, 2, 3, 4096), qs)
        b = _rand_ct(rng, (m, 2, 3, 4096), qs)
        exps.append(ops.to_host(ops.ct_mul_relin_rescale(ctx, ops.to_device(a), ops.to_device(b), key)))
        batches.append((torch.from_numpy(a.view(np.int64)).view(torch.uint64).pin_memory(),
                        torch.from_numpy(b.view(np.int64)).view(torch.uint64).pin_memory()))
        outs.append(torch.zeros((m, 2, 2, 4096), dtype=torch.uint64).pin_memory())
    torch.cuda.synchronize()
    for (ha, hb), o in zip(batches, outs):
        ops.ct_mul_relin_rescale_host_async(ctx, ha, hb, key, o, chunk, ws)
    ops.ct_mul_host_join()
    torch.cuda.synchronize()
    for o, e in zip(outs, exps):
        assert np.array_equal(o.view(torch.int64).numpy().view(np.uint64), e)
    # wire format, stream-ordered (the packed host buffers stay referenced
    # until the join: the copies read them asynchronously)
    ws48 = torch.empty((_lib.raw("ckks_ct_mul_host48_workspace_bytes")(ctx.handle, chunk, 3) + 7) // 8,
                       dtype=torch.uint64, device=key.device)
    keep, outs48 = [], []
    for (ha, hb), m in zip(batches, n_ct):
        a48, b48 = ops.pack48_host(ha).pin_memory(), ops.pack48_host(hb).pin_memory()
        o48 = torch.zeros(6 * m * 2 * 2 * 4096, dtype=torch.uint8).pin_memory()
        keep += [a48, b48]
        outs48.append(o48)
        _lib.call("ckks_ct_mul_relin_rescale_host48_async", ctx.handle, o48.data_ptr(), a48.data_ptr(),
                  b48.data_ptr(), key.data_ptr(), m, 3, chunk, ws48.data_ptr(), ws48.numel() * 8,
                  torch.cuda.current_stream().cuda_stream)
    ops.ct_mul_host_join()
    torch.cuda.synchronize()
    for o48, m, e in zip(outs48, n_ct, exps):
        got = ops.unpack48_host(o48, (m, 2, 2, 4096))
        assert np.array_equal(got.view(torch.int64).numpy().view(np.uint64), e)

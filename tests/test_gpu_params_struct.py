"""The POD parameter struct across the C ABI (ckks_ctx_create_params /
ckks_ctx_get_params): a context created from the struct with the roots left
to the library has the roots the Python side derives (smallest generator of
(Z/qZ)^* raised to (q-1)/2N, resp. (q-1)/N without a 2N-th root), carries
the scheme constants back unchanged, and transforms bit-identically to the
context the Python side creates; malformed structs are refused."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

QC = 35184371884033  # = 1 mod 2^13, not mod 2^14: no negacyclic root at N = 2^13


def _create(st):
    from ckks_b200 import _lib
    h = C.c_void_p()
    _lib.call("ckks_ctx_create_params", C.byref(st), C.byref(h))
    return h


def _read(h):
    from ckks_b200 import _lib
    out = _lib.CkksParamsC()
    _lib.call("ckks_ctx_get_params", h, C.byref(out))
    k = out.n_primes
    return out, [out.primes[i] for i in range(k)], [out.psi[i] for i in range(k)], [out.omega[i] for i in range(k)]


def test_struct_context_matches_python_context(cuda):
    import torch
    import ckks_b200.ops as ops
    from ckks_b200 import _lib
    from ckks_b200.context import Context
    from ckks_b200.params import CkksParams
    P = CkksParams.standard(12, 3, seed=9)
    st, arr = P.to_c()
    h = _create(st)
    try:
        out, primes, psi, omega = _read(h)
        ref = Context.get(12, P.primes, n_special=1)
        assert (out.log_n, out.n_primes, out.n_special) == (12, 4, 1)
        assert primes == list(P.primes) and psi == list(ref.psi) and omega == list(ref.omega)
        assert (out.scale, out.sigma, out.seed) == (P.scale, P.sigma, 9)
        rng = np.random.default_rng(4)
        x = np.stack([rng.integers(0, q, (3, 4096), dtype=np.uint64) for q in P.primes], axis=1)
        a, b = ops.to_device(x), ops.to_device(x)
        st_ = torch.cuda.current_stream().cuda_stream
        _lib.call("ckks_ntt", h, a.data_ptr(), 3, 0, 4, 0, 0, st_)
        ops.ntt(ref, b, n_limbs=4)
        assert torch.equal(a, b)
    finally:
        _lib.raw("ckks_ctx_destroy")(h)


def test_struct_without_negacyclic_root(cuda):
    from ckks_b200 import _lib
    from ckks_b200.context import Context
    arr = (C.c_uint64 * 1)(QC)
    st = _lib.CkksParamsC(13, 1, 0, 0, arr, None, None, 0.0, 0.0, 0)
    h = _create(st)
    try:
        _, _, psi, omega = _read(h)
        ref = Context.get(13, [QC])
        assert psi == [0] and omega == list(ref.omega)
    finally:
        _lib.raw("ckks_ctx_destroy")(h)


def test_struct_refusals(cuda):
    from ckks_b200 import _lib
    from ckks_b200._lib import CkksError
    arr = (C.c_uint64 * 1)(QC)
    with pytest.raises(CkksError, match="reserved"):
        _create(_lib.CkksParamsC(12, 1, 0, 7, arr, None, None, 0.0, 0.0, 0))
    bad = (C.c_uint64 * 1)(QC + 2)
    with pytest.raises(CkksError, match="not a prime"):
        _create(_lib.CkksParamsC(12, 1, 0, 0, bad, None, None, 0.0, 0.0, 0))
    with pytest.raises(CkksError, match="log_n"):
        _create(_lib.CkksParamsC(15, 1, 0, 0, arr, None, None, 0.0, 0.0, 0))

"""Tensor-level wrappers over the C ABI.

Every function takes CUDA tensors of dtype torch.uint64 (contiguous,
limb-major [..., limb, N]) and launches on the current torch stream.  No CPU
fallback: a missing library or a non-CUDA tensor raises.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .context import Context, _stream

U64 = torch.uint64


def _p(t: torch.Tensor) -> int:
    if not t.is_cuda:
        raise ValueError("expected a CUDA tensor")
    if t.dtype not in (torch.uint64, torch.int64):
        raise ValueError(f"expected uint64 data, got {t.dtype}")
    if not t.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return t.data_ptr()


def to_device(x, device=None) -> torch.Tensor:
    """numpy / list of ints -> contiguous CUDA uint64 tensor."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.uint64))
    return torch.from_numpy(a).to(device or torch.device("cuda", torch.cuda.current_device()))


def to_host(t: torch.Tensor) -> np.ndarray:
    return t.cpu().numpy().astype(np.uint64, copy=False)


def empty(shape, device=None) -> torch.Tensor:
    return torch.empty(shape, dtype=U64, device=device or "cuda")


def _polys_limbs(x: torch.Tensor, n: int, n_limbs: int | None):
    if x.shape[-1] != n:
        raise ValueError(f"last dim {x.shape[-1]} != N={n}")
    nl = n_limbs if n_limbs is not None else (x.shape[-2] if x.dim() >= 2 else 1)
    total = x.numel() // n
    if total % nl:
        raise ValueError("tensor size is not a multiple of n_limbs * N")
    return total // nl, nl


def ntt(ctx: Context, x: torch.Tensor, prime_begin: int = 0, inverse: bool = False,
        cyclic: bool = False, n_limbs: int | None = None) -> torch.Tensor:
    """In-place forward/inverse NTT of x [..., n_limbs, N]."""
    npoly, nl = _polys_limbs(x, ctx.n, n_limbs)
    _lib.call("ckks_ntt", ctx.handle, _p(x), npoly, prime_begin, nl, int(inverse), int(cyclic),
              _stream())
    return x


def bitrev_permute(ctx: Context, x: torch.Tensor) -> torch.Tensor:
    out = torch.empty_like(x)
    _lib.call("ckks_bitrev_permute", ctx.handle, _p(out), _p(x), x.numel() // ctx.n, _stream())
    return out


def pointwise_mul(ctx: Context, a: torch.Tensor, b: torch.Tensor, prime_begin: int = 0,
                  n_limbs: int | None = None, out: torch.Tensor | None = None) -> torch.Tensor:
    npoly, nl = _polys_limbs(a, ctx.n, n_limbs)
    out = torch.empty_like(a) if out is None else out
    _lib.call("ckks_pointwise_mul", ctx.handle, _p(out), _p(a), _p(b), npoly, prime_begin, nl,
              _stream())
    return out


def vec_addsub(a: torch.Tensor, b: torch.Tensor, q: int, subtract: bool,
               out: torch.Tensor | None = None) -> torch.Tensor:
    out = torch.empty_like(a) if out is None else out
    _lib.call("ckks_vec_addsub", _p(out), _p(a), _p(b), a.numel(), int(q), int(subtract), _stream())
    return out


def poly_mul(ctx: Context, a: torch.Tensor, b: torch.Tensor, prime_begin: int = 0,
             cyclic: bool = False, n_limbs: int | None = None) -> torch.Tensor:
    npoly, nl = _polys_limbs(a, ctx.n, n_limbs)
    out = torch.empty_like(a)
    _lib.call("ckks_poly_mul", ctx.handle, _p(out), _p(a), _p(b), npoly, prime_begin, nl,
              int(cyclic), _stream())
    return out


def poly_mul_anyq(crt3: Context, a: torch.Tensor, b: torch.Tensor, q: int,
                  cyclic: bool = False) -> torch.Tensor:
    out = torch.empty_like(a)
    _lib.call("ckks_poly_mul_anyq", crt3.handle, _p(out), _p(a), _p(b), a.numel() // crt3.n, int(q),
              int(cyclic), _stream())
    return out


def relin_single(ctx: Context, e0, e1, e2, ka, kb, prime: int = 0):
    f0 = torch.empty_like(e0)
    f1 = torch.empty_like(e1)
    _lib.call("ckks_relin_single", ctx.handle, _p(f0), _p(f1), _p(e0), _p(e1), _p(e2), _p(ka), _p(kb),
              e0.numel() // ctx.n, prime, _stream())
    return f0, f1


def rescale_exact(x: torch.Tensor, q_in: int, q_out: int) -> torch.Tensor:
    out = torch.empty_like(x)
    _lib.call("ckks_rescale_exact", _p(out), _p(x), x.numel(), int(q_in), int(q_out), _stream())
    return out


def rescale_scaled(x: torch.Tensor, q_in: int, q_out: int, scale_bits: int) -> torch.Tensor:
    out = torch.empty_like(x)
    _lib.call("ckks_rescale_scaled", _p(out), _p(x), x.numel(), int(q_in), int(q_out),
              int(scale_bits), _stream())
    return out


def rescale_rns(ctx: Context, x: torch.Tensor) -> torch.Tensor:
    """x [P, level, N] evaluation domain -> [P, level-1, N]."""
    level = x.shape[-2]
    npoly = x.numel() // (level * ctx.n)
    out = torch.empty(x.shape[:-2] + (level - 1, ctx.n), dtype=U64, device=x.device)
    _lib.call("ckks_rescale_rns", ctx.handle, _p(out), _p(x), npoly, level, _stream())
    return out


def relin_key_prepare(ctx: Context, ksk: torch.Tensor) -> torch.Tensor:
    """ksk [n_q, 2, n_q+1, N] -> prepared [n_q, 2, n_q+1, N, 2] (value, Shoup)."""
    out = torch.empty(tuple(ksk.shape) + (2,), dtype=U64, device=ksk.device)
    _lib.call("ckks_relin_key_prepare", ctx.handle, _p(out), _p(ksk), _stream())
    return out


def ct_mul_scratch_bytes(ctx: Context, n_ct: int, level: int) -> int:
    return int(_lib.raw("ckks_ct_mul_scratch_bytes")(ctx.handle, n_ct, level))


def ct_mul_relin_rescale(ctx: Context, ct_a: torch.Tensor, ct_b: torch.Tensor,
                         key_prepared: torch.Tensor, scratch: torch.Tensor | None = None,
                         out: torch.Tensor | None = None) -> torch.Tensor:
    """ct_a, ct_b [n_ct, 2, level, N] -> [n_ct, 2, level-1, N]."""
    n_ct, two, level, n = ct_a.shape
    need = ct_mul_scratch_bytes(ctx, n_ct, level)
    if scratch is None or scratch.numel() * scratch.element_size() < need:
        scratch = torch.empty((need + 7) // 8, dtype=U64, device=ct_a.device)
    if out is None:
        out = torch.empty((n_ct, 2, level - 1, n), dtype=U64, device=ct_a.device)
    _lib.call("ckks_ct_mul_relin_rescale", ctx.handle, _p(out), _p(ct_a), _p(ct_b), _p(key_prepared),
              n_ct, level, _p(scratch), scratch.numel() * scratch.element_size(), _stream())
    return out

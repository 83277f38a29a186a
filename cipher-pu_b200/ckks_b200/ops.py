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


def ntt_tc(ctx: Context, x: torch.Tensor, prime_begin: int = 0, n_limbs: int | None = None) -> torch.Tensor:
    """In-place forward negacyclic NTT of x [..., n_limbs, N] on the tensor
    cores (N = 2^12 only): the same results and order as ``ntt``."""
    npoly, nl = _polys_limbs(x, ctx.n, n_limbs)
    _lib.call("ckks_ntt_tc", ctx.handle, _p(x), npoly, prime_begin, nl, _stream())
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


def relin_single_masked(ctx: Context, e0, e1, e2, a1, b1, a2, b2, prime: int = 0):
    """relin_single with the key as additive shares (a1 + a2, b1 + b2)."""
    f0 = torch.empty_like(e0)
    f1 = torch.empty_like(e1)
    _lib.call("ckks_relin_single_masked", ctx.handle, _p(f0), _p(f1), _p(e0), _p(e1), _p(e2), _p(a1),
              _p(b1), _p(a2), _p(b2), e0.numel() // ctx.n, prime, _stream())
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


def ct_add(ctx: Context, a: torch.Tensor, b: torch.Tensor, subtract: bool = False,
           out: torch.Tensor | None = None) -> torch.Tensor:
    """a +- b for ciphertexts [n_ct, 2, level, N]."""
    out = torch.empty_like(a) if out is None else out
    n_ct, _, level, _ = a.shape
    _lib.call("ckks_ct_add", ctx.handle, _p(out), _p(a), _p(b), n_ct, level, int(subtract), _stream())
    return out


def ct_mul_const(ctx: Context, a: torch.Tensor, m: int, out: torch.Tensor | None = None) -> torch.Tensor:
    out = torch.empty_like(a) if out is None else out
    n_ct, _, level, _ = a.shape
    _lib.call("ckks_ct_mul_const", ctx.handle, _p(out), _p(a), n_ct, level, int(m), _stream())
    return out


def ct_add_const(ctx: Context, a: torch.Tensor, c: int, out: torch.Tensor | None = None) -> torch.Tensor:
    """Adds the (arbitrary-size) integer c to every slot of ciphertexts a."""
    import ctypes as C
    out = torch.empty_like(a) if out is None else out
    n_ct, _, level, _ = a.shape
    res = (C.c_uint64 * level)(*[int(c) % int(q) for q in ctx.primes[:level]])
    _lib.call("ckks_ct_add_const", ctx.handle, _p(out), _p(a), n_ct, level, res, _stream())
    return out


def automorphism(ctx: Context, x: torch.Tensor, nu: int, eval_domain: bool = False,
                 prime_begin: int = 0, n_limbs: int | None = None) -> torch.Tensor:
    """psi_nu(f)(X) = f(X^nu) mod (X^N + 1) of x [..., n_limbs, N]."""
    npoly, nl = _polys_limbs(x, ctx.n, n_limbs)
    out = torch.empty_like(x)
    _lib.call("ckks_automorphism", ctx.handle, _p(out), _p(x), npoly, prime_begin, nl, int(nu),
              int(eval_domain), _stream())
    return out


def mul_monomial(ctx: Context, x: torch.Tensor, nu: int, prime_begin: int = 0,
                 n_limbs: int | None = None) -> torch.Tensor:
    """x * X^nu in the coefficient domain."""
    npoly, nl = _polys_limbs(x, ctx.n, n_limbs)
    out = torch.empty_like(x)
    _lib.call("ckks_mul_monomial", ctx.handle, _p(out), _p(x), npoly, prime_begin, nl, int(nu), _stream())
    return out


def rotate(ctx: Context, ct: torch.Tensor, galois_key_prepared: torch.Tensor, nu: int,
           scratch: torch.Tensor | None = None, out: torch.Tensor | None = None) -> torch.Tensor:
    """Key-switched automorphism of ct [n_ct, 2, level, N] (evaluation domain)."""
    n_ct, two, level, n = ct.shape
    need = int(_lib.raw("ckks_rotate_scratch_bytes")(ctx.handle, n_ct, level))
    if scratch is None or scratch.numel() * scratch.element_size() < need:
        scratch = torch.empty((need + 7) // 8, dtype=U64, device=ct.device)
    if out is None:
        out = torch.empty_like(ct)
    _lib.call("ckks_rotate", ctx.handle, _p(out), _p(ct), _p(galois_key_prepared), n_ct, level, int(nu),
              _p(scratch), scratch.numel() * scratch.element_size(), _stream())
    return out


def ct_mul_host_workspace_bytes(ctx: Context, chunk: int, level: int) -> int:
    return int(_lib.raw("ckks_ct_mul_host_workspace_bytes")(ctx.handle, chunk, level))


def ct_mul_relin_rescale_host(ctx: Context, ct_a: torch.Tensor, ct_b: torch.Tensor,
                              key_prepared: torch.Tensor, out: torch.Tensor | None = None,
                              chunk: int = 32, workspace: torch.Tensor | None = None) -> torch.Tensor:
    """Host (CPU, preferably pinned) ct_a, ct_b [n_ct, 2, level, N] -> host
    [n_ct, 2, level-1, N]; copies and kernels pipelined in chunks."""
    if ct_a.is_cuda or ct_b.is_cuda:
        raise ValueError("ct_mul_relin_rescale_host takes host tensors")
    if not (ct_a.is_contiguous() and ct_b.is_contiguous()) or ct_a.dtype != U64 or ct_b.dtype != U64:
        raise ValueError("expected contiguous uint64 host tensors")
    n_ct, two, level, n = ct_a.shape
    if out is None:
        out = torch.empty((n_ct, 2, level - 1, n), dtype=U64).pin_memory()
    need = ct_mul_host_workspace_bytes(ctx, chunk, level)
    if workspace is None or workspace.numel() * workspace.element_size() < need:
        workspace = torch.empty((need + 7) // 8, dtype=U64, device=key_prepared.device)
    _lib.call("ckks_ct_mul_relin_rescale_host", ctx.handle, out.data_ptr(), ct_a.data_ptr(),
              ct_b.data_ptr(), _p(key_prepared), n_ct, level, chunk, _p(workspace),
              workspace.numel() * workspace.element_size(), _stream())
    return out


def pack48_host(x: torch.Tensor) -> torch.Tensor:
    """uint64 residues (< 2^47, any shape, CPU) -> uint8 [6 * numel] wire format."""
    import numpy as np
    a = x.contiguous().view(torch.int64).numpy().view(np.uint8).reshape(-1, 8)[:, :6]
    return torch.from_numpy(np.ascontiguousarray(a).reshape(-1))


def unpack48_host(b: torch.Tensor, shape) -> torch.Tensor:
    """uint8 wire format -> uint64 tensor of `shape` (CPU)."""
    import numpy as np
    raw = b.contiguous().numpy().reshape(-1, 6)
    w = np.zeros((raw.shape[0], 8), dtype=np.uint8)
    w[:, :6] = raw
    return torch.from_numpy(w.reshape(-1).view(np.int64).copy()).view(U64).reshape(shape)


def ct_mul_relin_rescale_host48(ctx: Context, a48: torch.Tensor, b48: torch.Tensor, key_prepared: torch.Tensor,
                                n_ct: int, level: int, out48: torch.Tensor | None = None, chunk: int = 64,
                                workspace: torch.Tensor | None = None) -> torch.Tensor:
    """Host (pinned) packed ciphertexts -> host packed products (uint8 buffers)."""
    n = ctx.n
    out_bytes = 6 * n_ct * 2 * (level - 1) * n
    if a48.numel() != 6 * n_ct * 2 * level * n or b48.numel() != a48.numel():
        raise ValueError("packed inputs must hold 6 n_ct 2 level N bytes")
    if out48 is None:
        out48 = torch.empty(out_bytes, dtype=torch.uint8).pin_memory()
    need = int(_lib.raw("ckks_ct_mul_host48_workspace_bytes")(ctx.handle, chunk, level))
    if workspace is None or workspace.numel() * workspace.element_size() < need:
        workspace = torch.empty((need + 7) // 8, dtype=U64, device=key_prepared.device)
    _lib.call("ckks_ct_mul_relin_rescale_host48", ctx.handle, out48.data_ptr(), a48.data_ptr(),
              b48.data_ptr(), _p(key_prepared), n_ct, level, chunk, _p(workspace),
              workspace.numel() * workspace.element_size(), _stream())
    return out48


def ct_mul_relin_rescale_host_async(ctx: Context, ct_a: torch.Tensor, ct_b: torch.Tensor,
                                    key_prepared: torch.Tensor, out: torch.Tensor, chunk: int,
                                    workspace: torch.Tensor) -> torch.Tensor:
    """Stream-ordered form of ``ct_mul_relin_rescale_host``: enqueues the
    pipeline and returns at once; ``ct_mul_host_join()`` then orders the
    current stream after every call enqueued so far (synchronise it before
    reading ``out``).  Host tensors and the workspace must stay untouched
    until then."""
    if ct_a.is_cuda or ct_b.is_cuda or out.is_cuda:
        raise ValueError("ct_mul_relin_rescale_host_async takes host tensors")
    if not (ct_a.is_contiguous() and ct_b.is_contiguous() and out.is_contiguous()):
        raise ValueError("expected contiguous host tensors")
    if ct_a.dtype != U64 or ct_b.dtype != U64 or out.dtype != U64:
        raise ValueError("expected uint64 host tensors")
    n_ct, two, level, n = ct_a.shape
    _lib.call("ckks_ct_mul_relin_rescale_host_async", ctx.handle, out.data_ptr(), ct_a.data_ptr(),
              ct_b.data_ptr(), _p(key_prepared), n_ct, level, chunk, _p(workspace),
              workspace.numel() * workspace.element_size(), _stream())
    return out


def ct_mul_host_join() -> None:
    """Order the current stream after every async host-buffer ct-mult enqueued so far."""
    _lib.call("ckks_ct_mul_host_join", _stream())


# ------------------------------------------------------------------ encode / decode
def _f64(t: torch.Tensor) -> int:
    if not t.is_cuda or t.dtype not in (torch.float64, torch.complex128) or not t.is_contiguous():
        raise ValueError("expected a contiguous CUDA float64 / complex128 tensor")
    return t.data_ptr()


def encode(ctx: Context, slots: torch.Tensor, level: int, scale: float) -> torch.Tensor:
    """slots: complex128 [P, n_slots] (CUDA) -> plaintext [P, level, N] (evaluation domain)."""
    slots = slots.to(torch.complex128).contiguous()
    P, ns = slots.shape
    out = torch.empty((P, level, ctx.n), dtype=U64, device=slots.device)
    _lib.call("ckks_encode", ctx.handle, _p(out), _f64(slots), P, ns, level, float(scale), _stream())
    return out


def decode(ctx: Context, coef: torch.Tensor, n_slots: int, scale: float) -> torch.Tensor:
    """coef: [P, level, N] coefficient-domain residues -> complex128 [P, n_slots]."""
    P, level, n = coef.shape
    out = torch.empty((P, n_slots), dtype=torch.complex128, device=coef.device)
    _lib.call("ckks_decode", ctx.handle, _f64(out), _p(coef), P, n_slots, level, float(scale), _stream())
    return out


def decrypt(ctx: Context, ct: torch.Tensor, s_eval: torch.Tensor) -> torch.Tensor:
    """ct [C, 2, level, N] -> coefficient residues [C, level, N] of c0 + c1 s."""
    C_, two, level, n = ct.shape
    out = torch.empty((C_, level, n), dtype=U64, device=ct.device)
    _lib.call("ckks_decrypt", ctx.handle, _p(out), _p(ct), _p(s_eval), C_, level, _stream())
    return out


def encrypt(ctx: Context, m_eval: torch.Tensor | None, s_eval: torch.Tensor, a: torch.Tensor,
            e: torch.Tensor) -> torch.Tensor:
    """a [C, level, N] uniform; e [C, N] int64; m_eval [C, level, N] or None -> ct [C, 2, level, N]."""
    C_, level, n = a.shape
    out = torch.empty((C_, 2, level, n), dtype=U64, device=a.device)
    if e.dtype != torch.int64 or not e.is_contiguous():
        raise ValueError("e must be a contiguous int64 tensor")
    _lib.call("ckks_encrypt", ctx.handle, _p(out), _p(m_eval) if m_eval is not None else None,
              _p(s_eval), _p(a), e.data_ptr(), C_, level, _stream())
    return out


def dare_refresh(ctx: Context, ct: torch.Tensor, s_eval: torch.Tensor, a: torch.Tensor,
                 e: torch.Tensor, level_out: int, shift_bits: int = 0,
                 scratch: torch.Tensor | None = None) -> torch.Tensor:
    C_, two, level_in, n = ct.shape
    need = int(_lib.raw("ckks_dare_scratch_bytes")(ctx.handle, C_, level_in))
    if scratch is None or scratch.numel() * 8 < need:
        scratch = torch.empty((need + 7) // 8, dtype=U64, device=ct.device)
    out = torch.empty((C_, 2, level_out, n), dtype=U64, device=ct.device)
    _lib.call("ckks_dare_refresh", ctx.handle, _p(out), _p(ct), _p(s_eval), _p(a), e.data_ptr(), C_,
              level_in, level_out, int(shift_bits), _p(scratch), scratch.numel() * 8, _stream())
    return out


def noise_energy(x: torch.Tensor, q: int) -> list[int]:
    """Exact sum of min(c, q-c)^2 per row of x [R, L] -> Python ints."""
    R, L = x.shape
    out = torch.empty((R, 2), dtype=U64, device=x.device)
    _lib.call("ckks_noise_energy", _p(out), _p(x), R, L, int(q), _stream())
    h = to_host(out)
    return [int(lo) + (int(hi) << 64) for lo, hi in h]


def noise_energy_sat(x: torch.Tensor, q: int, acc_bits: int = 106) -> tuple[list[int], list[bool]]:
    """The noise monitor with an acc_bits-wide accumulator: per row of x [R, L]
    the sum of min(c, q-c)^2 (clamped to 2^acc_bits - 1) and its saturation flag."""
    R, L = x.shape
    out = torch.empty((R, 2), dtype=U64, device=x.device)
    sat = torch.empty(R, dtype=torch.uint8, device=x.device)
    _lib.call("ckks_noise_energy_sat", _p(out), sat.data_ptr(), _p(x), R, L, int(q), int(acc_bits), _stream())
    h = to_host(out)
    return [int(lo) + (int(hi) << 64) for lo, hi in h], [bool(v) for v in sat.cpu().tolist()]


def snr_sums(dec: torch.Tensor, ref: torch.Tensor) -> torch.Tensor:
    """Per row (signal energy, error energy) of complex or real float64 tensors [R, L]."""
    cplx = dec.is_complex()
    R, L = dec.shape
    out = torch.empty((R, 2), dtype=torch.float64, device=dec.device)
    _lib.call("ckks_snr_sums", out.data_ptr(), dec.contiguous().data_ptr(), ref.contiguous().data_ptr(),
              R, L, int(cplx), _stream())
    return out


def block_sparse_mask(w: torch.Tensor, block: int, threshold: float):
    w = w.to(torch.float64).contiguous()
    out = torch.empty_like(w)
    keep = torch.empty(w.numel() // block, dtype=torch.uint8, device=w.device)
    _lib.call("ckks_block_sparse_mask", out.data_ptr(), keep.data_ptr(), w.data_ptr(), w.numel(), block,
              float(threshold), _stream())
    return out, keep


def block_post_process(x: torch.Tensor, q: int, block: int, threshold: int, use_approx: bool = True):
    R, L = x.shape
    out = torch.empty_like(x)
    skipped = torch.empty(R, dtype=torch.int32, device=x.device)
    _lib.call("ckks_block_post_process", _p(out), skipped.data_ptr(), _p(x), R, L, block, int(q),
              int(threshold), int(use_approx), _stream())
    return out, skipped


def _primes_arr(primes):
    import ctypes as C
    arr = (C.c_uint64 * len(primes))(*[int(p) for p in primes])
    return arr


def rns_split(primes, x_words: torch.Tensor, centered: bool = False) -> torch.Tensor:
    """x_words [n, W] little-endian integers -> residues [k, n]."""
    n, W = x_words.shape
    out = torch.empty((len(primes), n), dtype=U64, device=x_words.device)
    _lib.call("ckks_rns_split", _primes_arr(primes), len(primes), _p(out), _p(x_words), n, W,
              int(centered), _stream())
    return out


def rns_merge(primes, residues: torch.Tensor, words: int, centered: bool = False) -> torch.Tensor:
    k, n = residues.shape
    out = torch.empty((n, words), dtype=U64, device=residues.device)
    _lib.call("ckks_rns_merge", _primes_arr(primes), len(primes), _p(out), _p(residues), n, words,
              int(centered), _stream())
    return out


# ------------------------------------------------------------------ sampling
def sample_uniform(ctx: Context, n_polys: int, n_limbs: int, seed: int, stream_id: int,
                   prime_begin: int = 0, device=None) -> torch.Tensor:
    out = torch.empty((n_polys, n_limbs, ctx.n), dtype=U64, device=device or "cuda")
    _lib.call("ckks_sample_uniform", ctx.handle, _p(out), n_polys, prime_begin, n_limbs,
              int(seed) & (2 ** 64 - 1), int(stream_id) & (2 ** 64 - 1), _stream())
    return out


def sample_ternary(shape, seed: int, stream_id: int, device=None) -> torch.Tensor:
    out = torch.empty(shape, dtype=torch.int64, device=device or "cuda")
    _lib.call("ckks_sample_ternary", out.data_ptr(), out.numel(), int(seed) & (2 ** 64 - 1),
              int(stream_id) & (2 ** 64 - 1), _stream())
    return out


def sample_dgauss(shape, sigma: float, seed: int, stream_id: int, device=None) -> torch.Tensor:
    out = torch.empty(shape, dtype=torch.int64, device=device or "cuda")
    _lib.call("ckks_sample_dgauss", out.data_ptr(), out.numel(), float(sigma), int(seed) & (2 ** 64 - 1),
              int(stream_id) & (2 ** 64 - 1), _stream())
    return out


# ---------------------------------------------------------------- tensor-core linear layer
def linear_tc_pack(w: np.ndarray, keep: np.ndarray | None = None, device=None) -> torch.Tensor:
    """int weights [O, F] (|w| <= 8355711) and an optional 4x4 block-keep mask
    -> the packed byte-limb image on the device (ckks_linear_tc_pack)."""
    import ctypes as C
    w = np.ascontiguousarray(np.asarray(w, dtype=np.int32))
    O, F = w.shape
    nbytes = int(_lib.raw("ckks_linear_tc_packed_bytes")(O, F))
    host = np.zeros(nbytes, dtype=np.uint8)
    k = None if keep is None else np.ascontiguousarray(np.asarray(keep, dtype=np.uint8))
    _lib.call("ckks_linear_tc_pack", host.ctypes.data, nbytes, w.ctypes.data,
              None if k is None else k.ctypes.data, O, F)
    return torch.from_numpy(host).to(device or torch.device("cuda", torch.cuda.current_device()))


def linear_plain_weights_tc(ctx: Context, x: torch.Tensor, packed: torch.Tensor, n_out: int,
                            bias: torch.Tensor | None = None, out: torch.Tensor | None = None) -> torch.Tensor:
    """x [F, 2, level, N] ciphertexts -> [n_out, 2, level, N] on the tensor cores."""
    F, two, level, n = x.shape
    if out is None:
        out = torch.empty((n_out, 2, level, n), dtype=U64, device=x.device)
    _lib.call("ckks_linear_plain_weights_tc", ctx.handle, _p(out), _p(x), packed.data_ptr(),
              None if bias is None else bias.data_ptr(), n_out, F, level, _stream())
    return out

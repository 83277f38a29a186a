"""High-level CKKS evaluator: keys, encryption, homomorphic multiply, DARE.

Conventions: decryption m ~ c0 + c1 s; ciphertexts [C, 2, level, N] in the
evaluation domain over q_0..q_{level-1}; the relinearisation key is hybrid
(dnum = L digits, one special prime P); the scale of every ciphertext is
tracked on the host in float64 (rescaling divides by a 45-bit prime, so the
scale drifts away from Delta; decoding uses the tracked scale).

Randomness comes from the library's Philox sampler: (seed, stream id) pairs
are drawn from a per-evaluator counter, so a run is reproducible per seed.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib, ops
from .context import Context
from .params import CkksParams

U64 = torch.uint64
KEYS_SCHEMA = 1  # version of the key checkpoint written by Evaluator.save_keys


@dataclass
class Ciphertext:
    data: torch.Tensor          # [C, 2, level, N] evaluation domain
    scale: float

    @property
    def level(self) -> int:
        return int(self.data.shape[2])

    @property
    def count(self) -> int:
        return int(self.data.shape[0])


@dataclass
class SecretKey:
    s_coef: torch.Tensor        # [N] int64 ternary
    s_eval: torch.Tensor        # [n_primes, N] evaluation domain over q_0..q_{L-1}, P


class Evaluator:
    def __init__(self, params: CkksParams, device=None):
        self.params = params
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self.ctx = Context.get(params.log_n, params.primes, n_special=1)
        self.n = params.n
        self._stream_id = 1
        self.seed = params.seed
        self.sk: SecretKey | None = None
        self.rlk: torch.Tensor | None = None      # prepared relinearisation key
        self.ksk: torch.Tensor | None = None      # raw [L, 2, L+1, N]
        self._scratch: torch.Tensor | None = None
        self.galois: dict = {}

    # ---------------------------------------------------------------- sampling
    def _sid(self) -> int:
        self._stream_id += 1
        return self._stream_id

    def uniform(self, n_polys: int, n_limbs: int, prime_begin: int = 0) -> torch.Tensor:
        return ops.sample_uniform(self.ctx, n_polys, n_limbs, self.seed, self._sid(), prime_begin,
                                  device=self.device)

    def dgauss(self, shape) -> torch.Tensor:
        return ops.sample_dgauss(shape, self.params.sigma, self.seed, self._sid(), device=self.device)

    # ---------------------------------------------------------------- keys
    def keygen(self, s_coef: torch.Tensor | None = None) -> SecretKey:
        n, k = self.n, len(self.params.primes)
        if s_coef is None:
            s_coef = ops.sample_ternary((n,), self.seed, self._sid(), device=self.device)
        s_coef = s_coef.to(self.device, torch.int64).contiguous()
        s_eval = self._int_poly_to_eval(s_coef, k)
        self.sk = SecretKey(s_coef, s_eval)
        self._make_relin_key()
        return self.sk

    def _int_poly_to_eval(self, x: torch.Tensor, n_limbs: int) -> torch.Tensor:
        """Small signed integer polynomial [N] -> evaluation domain [n_limbs, N]."""
        rows = []
        for i in range(n_limbs):
            q = self.params.primes[i]
            rows.append(torch.remainder(x, q))
        t = torch.stack(rows).contiguous().view(U64)
        ops.ntt(self.ctx, t, prime_begin=0, n_limbs=n_limbs)
        return t

    def _switch_key(self, target_eval: torch.Tensor, a: torch.Tensor | None = None,
                    e: torch.Tensor | None = None) -> tuple:
        """Hybrid key-switching key from `target` (evaluation domain over all
        L + 1 primes) to s: ksk[j] = Enc_s(m_j), m_j[i] = delta_ij (P mod q_j) target."""
        L = self.params.levels
        n = self.n
        s = self.sk.s_eval
        P = self.params.special
        if a is None:
            a = self.uniform(L, L + 1)
        if e is None:
            e = self.dgauss((L, n))
        m = torch.zeros((L, L + 1, n), dtype=U64, device=self.device)
        for j in range(L):
            qj = self.params.q[j]
            c = torch.full((1, n), P % qj, dtype=torch.int64, device=self.device).view(U64)
            m[j, j] = ops.pointwise_mul(self.ctx, target_eval[j:j + 1].contiguous(), c, prime_begin=j,
                                        n_limbs=1)[0]
        ksk = ops.encrypt(self.ctx, m, s, a.contiguous(), e.contiguous())
        return ksk, ops.relin_key_prepare(self.ctx, ksk), (a, e)

    def _make_relin_key(self, a: torch.Tensor | None = None, e: torch.Tensor | None = None):
        """ksk[j] = Enc_s over all L+1 primes of m_j with m_j[i] = delta_ij (P mod q_j) s^2."""
        L = self.params.levels
        s = self.sk.s_eval
        s2 = ops.pointwise_mul(self.ctx, s, s, n_limbs=L + 1)
        self.ksk, self.rlk, self._key_samples = self._switch_key(s2, a, e)
        self.galois = {}

    def galois_key(self, nu: int, a: torch.Tensor | None = None, e: torch.Tensor | None = None):
        """(raw, prepared) Galois key of psi_nu: switches psi_nu(s) to s (cached per nu)."""
        nu = int(nu) % (2 * self.n)
        if nu % 2 == 0:
            raise ValueError("a Galois element must be odd")
        if nu not in self.galois or a is not None:
            ps = ops.automorphism(self.ctx, self.sk.s_eval, nu, eval_domain=True,
                                  n_limbs=self.params.levels + 1)
            ksk, gk, _ = self._switch_key(ps, a, e)
            self.galois[nu] = (ksk, gk)
        return self.galois[nu]

    def rotate(self, ct: Ciphertext, nu: int, out: torch.Tensor | None = None) -> Ciphertext:
        """psi_nu applied to the plaintext of ct, key-switched back to s (same
        level and scale).  Slot k of the result holds slot galois_slot_map(nu)[k]
        of the input (complex-conjugated where the map says so)."""
        _, gk = self.galois_key(nu)
        need = int(_lib.raw("ckks_rotate_scratch_bytes")(self.ctx.handle, ct.count, ct.level))
        if self._scratch is None or self._scratch.numel() * 8 < need:
            self._scratch = torch.empty((need + 7) // 8, dtype=U64, device=self.device)
        r = ops.rotate(self.ctx, ct.data, gk, nu, scratch=self._scratch, out=out)
        return Ciphertext(r, ct.scale)

    # ---------------------------------------------------------------- checkpoint
    def save_keys(self, path) -> None:
        """Write the key material to an .npz (schema KEYS_SCHEMA): the
        parameter set (ring, primes, scale, sigma, seed), the sampler's stream
        counter (so a resumed evaluator draws the same randomness next), the
        ternary secret in the coefficient domain, the raw relinearisation key
        and every raw Galois key.  Twiddle tables are not stored: a context is
        a pure function of (N, primes) and is rebuilt on load."""
        if self.sk is None:
            raise ValueError("no keys to save: call keygen() first")
        host = lambda t: t.contiguous().view(torch.int64).cpu().numpy()
        P = self.params
        rec = {"schema": np.int64(KEYS_SCHEMA), "log_n": np.int64(P.log_n),
               "q": np.asarray(P.q, dtype=np.uint64), "special": np.uint64(P.special),
               "scale": np.float64(P.scale), "sigma": np.float64(P.sigma), "seed": np.int64(P.seed),
               "stream_id": np.int64(self._stream_id), "s_coef": host(self.sk.s_coef),
               "ksk": host(self.ksk), "galois_nu": np.asarray(sorted(self.galois), dtype=np.int64)}
        for nu in sorted(self.galois):
            rec[f"galois_{nu}"] = host(self.galois[nu][0])
        np.savez(path, **rec)

    def load_keys(self, path) -> SecretKey:
        """Restore what save_keys wrote into this evaluator (same parameter
        set required): the secret, the relinearisation key and the Galois
        keys (re-prepared on the device), and the sampler's stream counter."""
        z = np.load(path)
        if int(z["schema"]) != KEYS_SCHEMA:
            raise ValueError(f"key checkpoint schema {int(z['schema'])}, expected {KEYS_SCHEMA}")
        P = self.params
        same = (int(z["log_n"]) == P.log_n and [int(x) for x in z["q"]] == list(P.q)
                and int(z["special"]) == P.special and float(z["scale"]) == P.scale
                and float(z["sigma"]) == P.sigma and int(z["seed"]) == P.seed)
        if not same:
            raise ValueError("key checkpoint was written for another parameter set")
        dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(self.device)
        s_coef = dev(z["s_coef"]).to(torch.int64)
        self.sk = SecretKey(s_coef, self._int_poly_to_eval(s_coef, len(P.primes)))
        self.ksk = dev(z["ksk"]).view(U64).contiguous()
        self.rlk = ops.relin_key_prepare(self.ctx, self.ksk)
        self.galois = {}
        for nu in z["galois_nu"].tolist():
            raw = dev(z[f"galois_{nu}"]).view(U64).contiguous()
            self.galois[int(nu)] = (raw, ops.relin_key_prepare(self.ctx, raw))
        self._stream_id = int(z["stream_id"])
        return self.sk

    # ---------------------------------------------------------------- polynomials
    def drop_to(self, ct: Ciphertext, level: int) -> Ciphertext:
        """The same ciphertext modulo q_0..q_{level-1} (limbs discarded; scale kept)."""
        if level == ct.level:
            return ct
        if not 1 <= level < ct.level:
            raise ValueError(f"cannot drop level {ct.level} to {level}")
        return Ciphertext(ct.data[:, :, :level].contiguous(), ct.scale)

    def lift_scale(self, ct: Ciphertext, target: float) -> Ciphertext:
        """Multiply by the integer floor(target / scale) when that is >= 2: the
        scale grows toward `target` with no level spent and the relative
        precision kept (noise and message scale together)."""
        m = int(target // ct.scale)
        if m < 2:
            return ct
        return Ciphertext(ops.ct_mul_const(self.ctx, ct.data, m), ct.scale * m)

    def mul(self, a: Ciphertext, b: Ciphertext) -> Ciphertext:
        """ct x ct with relinearisation and rescale at the lower of the two
        levels.  Both operands are first lifted to a scale near q_{l-1} / 8
        (messages of magnitude <= 1 keep the product below Q_l / 2 down to
        two limbs), so repeated products do not drift to small scales where
        the key-switching noise would dominate."""
        lv = min(a.level, b.level)
        tgt = self.params.q[lv - 1] / 8.0
        a = self.lift_scale(self.drop_to(a, lv), tgt)
        b = self.lift_scale(self.drop_to(b, lv), tgt)
        return self.mul_relin_rescale(a, b)

    def poly_eval(self, ct: Ciphertext, coeffs, out_scale: float | None = None) -> Ciphertext:
        """sum_k coeffs[k] x^k on every slot (real coefficients, ascending).
        Powers by a doubling tree (depth ceil(log2 d)); each term is brought
        to the deepest level and multiplied by the integer round(c_k T / s_k),
        so all terms share the exact scale T = out_scale q_{l-1} (lowered when
        a term's constant would exceed 2^61); one rescale at the end returns
        scale T / q_{l-1}.  Needs ceil(log2 d) + 2 levels, and |p(x)| T must
        stay below the remaining modulus / 2."""
        coeffs = [float(c) for c in coeffs]
        d = len(coeffs) - 1
        while d > 0 and coeffs[d] == 0.0:
            d -= 1
        out_scale = float(out_scale or ct.scale)
        pw = {1: ct}
        for k in range(2, d + 1):
            hi = 1 << (k.bit_length() - 1)
            pw[k] = self.mul(pw[hi // 2], pw[hi // 2]) if k == hi else self.mul(pw[hi], pw[k - hi])
        terms = [k for k in range(1, d + 1) if coeffs[k] != 0.0]
        lv = min([pw[k].level for k in terms] + [ct.level])
        if lv < 2:
            raise ValueError(f"degree {d} needs more levels than the ciphertext has ({ct.level})")
        T = out_scale * self.params.q[lv - 1]
        # keep every term constant below 2^61 (high powers carry small scales)
        for k in terms:
            T = min(T, 2.0 ** 61 * pw[k].scale / abs(coeffs[k]))
        acc = None
        for k in terms:
            t = self.drop_to(pw[k], lv)
            m = int(round(coeffs[k] * T / t.scale))
            if abs(m) >= 1 << 62:
                raise ValueError("term constant exceeds 62 bits: lower out_scale")
            prod = ops.ct_mul_const(self.ctx, t.data, m)
            acc = prod if acc is None else ops.ct_add(self.ctx, acc, prod, out=acc)
        if acc is None:
            acc = torch.zeros_like(self.drop_to(ct, lv).data)
        c0 = int(round(coeffs[0] * T)) if d >= 0 else 0
        if c0:
            ops.ct_add_const(self.ctx, acc, c0, out=acc)
        return self.rescale(Ciphertext(acc, T))

    def galois_slot_map(self, nu: int) -> tuple[np.ndarray, np.ndarray]:
        """(src, conj) over the N/2 visible slots: after psi_nu, slot k holds
        input slot src[k] (conjugated where conj[k]).  Slot k is the evaluation
        at exp(i pi (2k + 1) / N); conjugates sit at N - 1 - k."""
        n = self.n
        k = np.arange(n // 2)
        e = ((2 * k + 1) * (int(nu) % (2 * n))) % (2 * n)
        kp = (e - 1) // 2
        conj = kp >= n // 2
        return np.where(conj, n - 1 - kp, kp), conj

    # ---------------------------------------------------------------- encode / encrypt
    def encode(self, values, level: int | None = None, scale: float | None = None) -> torch.Tensor:
        """values: [C, n_slots] real or complex (numpy or tensor) -> plaintext [C, level, N]."""
        level = level or self.params.levels
        scale = scale or self.params.scale
        v = torch.as_tensor(np.asarray(values) if not torch.is_tensor(values) else values)
        v = v.to(self.device).to(torch.complex128)
        if v.dim() == 1:
            v = v[None]
        return ops.encode(self.ctx, v.contiguous(), level, scale)

    def encrypt_values(self, values, level: int | None = None, scale: float | None = None) -> Ciphertext:
        level = level or self.params.levels
        scale = scale or self.params.scale
        m = self.encode(values, level, scale)
        C = m.shape[0]
        a = self.uniform(C, level)
        e = self.dgauss((C, self.n))
        return Ciphertext(ops.encrypt(self.ctx, m, self.sk.s_eval, a, e), scale)

    def decrypt_coef(self, ct: Ciphertext) -> torch.Tensor:
        return ops.decrypt(self.ctx, ct.data, self.sk.s_eval)

    def decrypt_values(self, ct: Ciphertext, n_slots: int | None = None) -> torch.Tensor:
        n_slots = n_slots or self.n // 2
        return ops.decode(self.ctx, self.decrypt_coef(ct), n_slots, ct.scale)

    # ---------------------------------------------------------------- evaluation
    def mul_relin_rescale(self, a: Ciphertext, b: Ciphertext, out: torch.Tensor | None = None) -> Ciphertext:
        level = a.level
        need = ops.ct_mul_scratch_bytes(self.ctx, a.count, level)
        if self._scratch is None or self._scratch.numel() * 8 < need:
            self._scratch = torch.empty((need + 7) // 8, dtype=U64, device=self.device)
        r = ops.ct_mul_relin_rescale(self.ctx, a.data, b.data, self.rlk, scratch=self._scratch, out=out)
        return Ciphertext(r, a.scale * b.scale / self.params.q[level - 1])

    def rescale(self, ct: Ciphertext) -> Ciphertext:
        C, two, level, n = ct.data.shape
        r = ops.rescale_rns(self.ctx, ct.data.reshape(C * 2, level, n)).reshape(C, 2, level - 1, n)
        return Ciphertext(r, ct.scale / self.params.q[level - 1])

    def dare_refresh(self, ct: Ciphertext, level_out: int | None = None, shift_bits: int = 0) -> Ciphertext:
        """Decrypt-reencrypt: fresh noise, modulus restored to level_out, scale / 2^shift."""
        level_out = level_out or self.params.levels
        C = ct.count
        a = self.uniform(C, level_out)
        e = self.dgauss((C, self.n))
        r = ops.dare_refresh(self.ctx, ct.data, self.sk.s_eval, a, e, level_out, shift_bits)
        return Ciphertext(r, ct.scale / float(2 ** shift_bits))

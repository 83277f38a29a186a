"""Host-side handle of a ckks_ctx (prime basis + device twiddle tables)."""
from __future__ import annotations

import ctypes as C
import threading

from . import _lib
from .params import root_of_unity

_CACHE: dict = {}
_LOCK = threading.Lock()


def _stream(stream=None) -> int | None:
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


class Context:
    """A prime basis at one ring dimension, resident on the current CUDA device.

    primes: q_0..q_{k-1} (the last `n_special` are special primes).  For each
    prime the negacyclic transform is available when 2N | q-1, the cyclic one
    when N | q-1.  `omega` overrides the cyclic N-th root (default psi^2, or
    g^((q-1)/N) when no 2N-th root exists)."""

    def __init__(self, log_n: int, primes, n_special: int = 0, omega=None):
        import torch
        self.log_n = int(log_n)
        self.n = 1 << self.log_n
        self.primes = tuple(int(q) for q in primes)
        self.n_special = int(n_special)
        self.device = torch.cuda.current_device()
        n = self.n
        psi = []
        om = []
        for i, q in enumerate(self.primes):
            if (q - 1) % (2 * n) == 0:
                ps = root_of_unity(q, 2 * n)
            else:
                ps = 0
            psi.append(ps)
            if omega is not None and omega[i]:
                om.append(int(omega[i]))
            elif ps:
                om.append(ps * ps % q)
            else:
                om.append(root_of_unity(q, n))
        self.psi = tuple(psi)
        self.omega = tuple(om)
        k = len(self.primes)
        arr = C.c_uint64 * k
        h = C.c_void_p()
        _lib.call("ckks_ctx_create", self.log_n, k, self.n_special, arr(*self.primes), arr(*psi),
                  arr(*om), C.byref(h))
        self._h = h

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    @property
    def n_q(self) -> int:
        return len(self.primes) - self.n_special

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.raw("ckks_ctx_destroy")(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def get(log_n: int, primes, n_special: int = 0, omega=None) -> "Context":
        """Cached context for (device, log_n, primes, n_special, omega)."""
        import torch
        key = (torch.cuda.current_device(), int(log_n), tuple(int(q) for q in primes), int(n_special),
               tuple(omega) if omega is not None else None)
        with _LOCK:
            c = _CACHE.get(key)
            if c is None:
                c = Context(log_n, primes, n_special, omega)
                _CACHE[key] = c
            return c

"""B200-native CKKS evaluation core (host side).

Python/PyTorch host code over hand-written sm_100a CUDA kernels reached through
the C ABI of libckks_b200.so (include/ckks_b200.h).  PyTorch provides device
memory and streams only; every arithmetic step runs in the library's kernels.
"""
from .params import CkksParams, PRIME_45_N4096, chain_primes, find_ntt_primes, is_prime, root_of_unity  # noqa: F401
from ._lib import CkksError, LIB_PATH  # noqa: F401

__all__ = ["CkksParams", "PRIME_45_N4096", "chain_primes", "find_ntt_primes", "is_prime",
           "root_of_unity", "CkksError", "LIB_PATH"]

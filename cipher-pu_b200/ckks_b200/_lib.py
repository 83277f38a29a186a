"""ctypes binding of libckks_b200.so (the C ABI declared in include/ckks_b200.h).

The library is built in tree (``python cipher-pu_b200/build.py``).  Loading
fails loudly when it is missing: there is no CPU fallback on the product path.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libckks_b200.so"

_u64p = C.c_void_p  # device pointers are passed as plain addresses
_vp = C.c_void_p
_i32 = C.c_int
_i64 = C.c_int64
_u64 = C.c_uint64
_sz = C.c_size_t



class BatchBucket(C.Structure):
    """ckks_batch_bucket: n_ct same-shape operations of the persistent batch."""
    _fields_ = [("ctx", _vp), ("op", C.c_int32), ("n_ct", C.c_int32), ("level", C.c_int32),
                ("pt_per_ct", C.c_int32), ("a", _vp), ("b", _vp), ("out", _vp), ("key", _vp)]


class CkksParamsC(C.Structure):
    """ckks_params: the parameter set as one POD struct (ckks_ctx_create_params)."""
    _fields_ = [("log_n", C.c_int32), ("n_primes", C.c_int32), ("n_special", C.c_int32),
                ("reserved", C.c_int32), ("primes", C.POINTER(C.c_uint64)), ("psi", C.POINTER(C.c_uint64)),
                ("omega", C.POINTER(C.c_uint64)), ("scale", C.c_double), ("sigma", C.c_double),
                ("seed", C.c_uint64)]


BATCH_CT_CT, BATCH_CT_PT = 0, 1
BATCH_RUN_UNMET_WAIT = 1
BATCH_RUN_PHASED = 2

# name -> (restype, argtypes); must mirror include/ckks_b200.h
SIGNATURES: dict[str, tuple] = {
    "ckks_abi_version": (_i32, []),
    "ckks_last_error": (C.c_char_p, []),
    "ckks_ctx_create_params": (_i32, [C.POINTER(CkksParamsC), C.POINTER(_vp)]),
    "ckks_ctx_get_params": (_i32, [_vp, C.POINTER(CkksParamsC)]),
    "ckks_ctx_create": (_i32, [_i32, _i32, _i32, C.POINTER(_u64), C.POINTER(_u64), C.POINTER(_u64),
                               C.POINTER(_vp)]),
    "ckks_ctx_destroy": (_i32, [_vp]),
    "ckks_ctx_set_tuning": (_i32, [_vp, _i32, _i32]),
    "ckks_device_status": (_i32, []),
    "ckks_ntt": (_i32, [_vp, _u64p, _i32, _i32, _i32, _i32, _i32, _vp]),
    "ckks_ntt_tc": (_i32, [_vp, _u64p, _i32, _i32, _i32, _vp]),
    "ckks_bitrev_permute": (_i32, [_vp, _u64p, _u64p, _i32, _vp]),
    "ckks_pointwise_mul": (_i32, [_vp, _u64p, _u64p, _u64p, _i32, _i32, _i32, _vp]),
    "ckks_vec_addsub": (_i32, [_u64p, _u64p, _u64p, _i64, _u64, _i32, _vp]),
    "ckks_poly_mul": (_i32, [_vp, _u64p, _u64p, _u64p, _i32, _i32, _i32, _i32, _vp]),
    "ckks_poly_mul_anyq": (_i32, [_vp, _u64p, _u64p, _u64p, _i32, _u64, _i32, _vp]),
    "ckks_relin_single": (_i32, [_vp, _u64p, _u64p, _u64p, _u64p, _u64p, _u64p, _u64p, _i32, _i32,
                                 _vp]),
    "ckks_rescale_exact": (_i32, [_u64p, _u64p, _i64, _u64, _u64, _vp]),
    "ckks_rescale_scaled": (_i32, [_u64p, _u64p, _i64, _u64, _u64, _i32, _vp]),
    "ckks_rescale_rns": (_i32, [_vp, _u64p, _u64p, _i32, _i32, _vp]),
    "ckks_relin_key_prepare": (_i32, [_vp, _u64p, _u64p, _vp]),
    "ckks_ct_mul_scratch_bytes": (_sz, [_vp, _i32, _i32]),
    "ckks_ct_mul_relin_rescale": (_i32, [_vp, _u64p, _u64p, _u64p, _u64p, _i32, _i32, _vp, _sz,
                                         _vp]),
    "ckks_ct_mul_host_workspace_bytes": (_sz, [_vp, _i32, _i32]),
    "ckks_ct_mul_relin_rescale_host": (_i32, [_vp, _vp, _vp, _vp, _u64p, _i32, _i32, _i32, _vp, _sz,
                                              _vp]),
    "ckks_unpack48": (_i32, [_u64p, _vp, _i64, _vp]),
    "ckks_pack48": (_i32, [_vp, _u64p, _i64, _vp]),
    "ckks_ct_mul_host48_workspace_bytes": (_sz, [_vp, _i32, _i32]),
    "ckks_ct_mul_relin_rescale_host48": (_i32, [_vp, _vp, _vp, _vp, _u64p, _i32, _i32, _i32, _vp, _sz,
                                                _vp]),
    "ckks_ct_mul_relin_rescale_host_async": (_i32, [_vp, _vp, _vp, _vp, _u64p, _i32, _i32, _i32, _vp, _sz,
                                                    _vp]),
    "ckks_ct_mul_relin_rescale_host48_async": (_i32, [_vp, _vp, _vp, _vp, _u64p, _i32, _i32, _i32, _vp,
                                                      _sz, _vp]),
    "ckks_ct_mul_host_join": (_i32, [_vp]),
    "ckks_ct_mul_relin_rescale_noalloc": (_i32, [_vp, _u64p, _u64p, _u64p, _u64p, _i32, _i32, _vp]),
    "ckks_encode": (_i32, [_vp, _u64p, _vp, _i32, _i32, _i32, C.c_double, _vp]),
    "ckks_decode": (_i32, [_vp, _vp, _u64p, _i32, _i32, _i32, C.c_double, _vp]),
    "ckks_decrypt": (_i32, [_vp, _u64p, _u64p, _u64p, _i32, _i32, _vp]),
    "ckks_encrypt": (_i32, [_vp, _u64p, _u64p, _u64p, _u64p, _vp, _i32, _i32, _vp]),
    "ckks_dare_scratch_bytes": (_sz, [_vp, _i32, _i32]),
    "ckks_dare_refresh": (_i32, [_vp, _u64p, _u64p, _u64p, _u64p, _vp, _i32, _i32, _i32, _i32, _vp,
                                 _sz, _vp]),
    "ckks_noise_energy": (_i32, [_u64p, _u64p, _i32, _i32, _u64, _vp]),
    "ckks_noise_energy_sat": (_i32, [_u64p, _vp, _u64p, _i32, _i32, _u64, _i32, _vp]),
    "ckks_snr_sums": (_i32, [_vp, _vp, _vp, _i32, _i32, _i32, _vp]),
    "ckks_block_sparse_mask": (_i32, [_vp, _vp, _vp, _i64, _i32, C.c_double, _vp]),
    "ckks_block_post_process": (_i32, [_u64p, _vp, _u64p, _i32, _i32, _i32, _u64, _u64, _i32, _vp]),
    "ckks_rns_split": (_i32, [C.POINTER(_u64), _i32, _u64p, _u64p, _i64, _i32, _i32, _vp]),
    "ckks_rns_merge": (_i32, [C.POINTER(_u64), _i32, _u64p, _u64p, _i64, _i32, _i32, _vp]),
    "ckks_linear_plain_weights": (_i32, [_vp, _u64p, _u64p, _vp, _vp, _vp, _i32, _i32, _i32, _vp]),
    "ckks_linear_tc_packed_bytes": (_sz, [_i32, _i32]),
    "ckks_linear_tc_pack": (_i32, [_vp, _sz, _vp, _vp, _i32, _i32]),
    "ckks_linear_plain_weights_tc": (_i32, [_vp, _u64p, _u64p, _vp, _vp, _i32, _i32, _i32, _vp]),
    "ckks_ct_mul_plain_rescale": (_i32, [_vp, _u64p, _u64p, _u64p, _i32, _i32, _i32, _vp]),
    "ckks_relin_single_masked": (_i32, [_vp, _u64p, _u64p, _u64p, _u64p, _u64p, _u64p, _u64p, _u64p,
                                        _u64p, _i32, _i32, _vp]),
    "ckks_ct_add": (_i32, [_vp, _u64p, _u64p, _u64p, _i32, _i32, _i32, _vp]),
    "ckks_ct_mul_const": (_i32, [_vp, _u64p, _u64p, _i32, _i32, _i64, _vp]),
    "ckks_ct_add_const": (_i32, [_vp, _u64p, _u64p, _i32, _i32, C.POINTER(_u64), _vp]),
    "ckks_automorphism": (_i32, [_vp, _u64p, _u64p, _i32, _i32, _i32, _u64, _i32, _vp]),
    "ckks_mul_plain_multi": (_i32, [_vp, _u64p, _u64p, _u64p, _i32, _i32, _i32, _vp]),
    "ckks_decrypt_coef0": (_i32, [_vp, _u64p, _u64p, _u64p, C.c_longlong, _i32, _vp]),
    "ckks_mul_monomial": (_i32, [_vp, _u64p, _u64p, _i32, _i32, _i32, _u64, _vp]),
    "ckks_rotate_scratch_bytes": (_sz, [_vp, _i32, _i32]),
    "ckks_rotate": (_i32, [_vp, _u64p, _u64p, _u64p, _i32, _i32, _u64, _vp, _sz, _vp]),
    "ckks_modmul_peak": (_i32, [_u64p, _i32, _i32, _i32, _i32, _u64, _u64, _vp]),
    "ckks_gear_mlp_param_count": (_i32, []),
    "ckks_gear_mlp_forward": (_i32, [_vp, _vp, _vp, _vp, _i32, _vp]),
    "ckks_gear_mlp_backward": (_i32, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i32, _vp]),
    "ckks_gear_mlp_adam": (_i32, [_vp, _vp, _vp, _vp, _i32, C.c_float, C.c_float, C.c_float, C.c_float,
                                  _vp]),
    "ckks_sample_uniform": (_i32, [_vp, _u64p, _i32, _i32, _i32, _u64, _u64, _vp]),
    "ckks_sample_ternary": (_i32, [_vp, _i64, _u64, _u64, _vp]),
    "ckks_sample_dgauss": (_i32, [_vp, _i64, C.c_double, _u64, _u64, _vp]),
    "ckks_gear_ctrl_init": (_i32, [_vp, C.POINTER(_u64), C.POINTER(_u64), _i32]),
    "ckks_gear_ctrl_raw": (_i32, [_vp, _u64, _u64]),
    "ckks_gear_ctrl_flush": (_i32, [_vp, _u64, _u64, _i32, _i32, _i32]),
    "ckks_batch_plan_create": (_i32, [C.POINTER(BatchBucket), _i32, _i32, C.POINTER(_vp)]),
    "ckks_batch_plan_run": (_i32, [_vp, C.c_longlong, _i32, _vp]),
    "ckks_batch_plan_incomplete": (_i32, [_vp, C.POINTER(_i32), _vp]),
    "ckks_batch_plan_info": (_i32, [_vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong), C.POINTER(_i32),
                                     C.POINTER(_i32), C.POINTER(_sz)]),
    "ckks_batch_plan_destroy": (None, [_vp]),
    "ckks_batch_schedule": (_i32, [_i32, _vp, _vp, _vp, _vp, _vp, C.c_longlong, _vp, C.POINTER(C.c_longlong)]),
    "ckks_batch_schedule_phased": (_i32, [_i32, _vp, _vp, _vp, _vp, _vp, C.c_longlong, _vp,
                                          C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    "ckks_profile_enable": (_i32, [_i32]),
    "ckks_profile_reset": (_i32, []),
    "ckks_profile_read": (_i32, [_i32, C.POINTER(C.c_double), C.POINTER(C.c_longlong)]),
}


class CkksError(RuntimeError):
    def __init__(self, fn: str, code: int, msg: str):
        super().__init__(f"{fn} failed (status {code}): {msg}")
        self.code = code


_lib = None


def load() -> C.CDLL:
    """Load the shared library (once).  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python cipher-pu_b200/build.py` "
            "(the CKKS core has no CPU fallback)")
    lib = C.CDLL(str(LIB_PATH), mode=os.RTLD_LOCAL if hasattr(os, "RTLD_LOCAL") else 0)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def call(name: str, *args) -> int:
    lib = load()
    rc = getattr(lib, name)(*args)
    if rc != 0:
        msg = lib.ckks_last_error().decode(errors="replace")
        raise CkksError(name, rc, msg)
    return rc


def raw(name: str):
    return getattr(load(), name)

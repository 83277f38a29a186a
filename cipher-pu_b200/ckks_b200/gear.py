"""Gear controllers of the adaptive loop.

* ``GearCtrl``: the energy-threshold controller with hysteresis of
  rtl/m4/adaptive_gear_ctrl.sv:43-99, run by the library's C state machine
  (ckks_gear_ctrl_*); energies are exact integers (the RTL's 106-bit
  accumulator, here 128-bit).
* ``GEAR_SPARSITY``: the sparsity gears {0, 25, 50, 75} % of 4x4 weight
  blocks used by the encrypted MLP / CNN; gear 0 is the most precise.
"""
from __future__ import annotations

import ctypes as C

from . import _lib

GEAR_SPARSITY = (0.0, 0.25, 0.50, 0.75)


class _State(C.Structure):
    _fields_ = [("thresh_lo", C.c_uint64 * 3), ("thresh_hi", C.c_uint64 * 3), ("hyst_cnt", C.c_int),
                ("gear", C.c_int), ("counter", C.c_int), ("candidate", C.c_int)]


def _split(v: int):
    v = int(v)
    if v < 0 or v >= 1 << 128:
        raise ValueError("energy outside [0, 2^128)")
    return v & (2 ** 64 - 1), v >> 64


class GearCtrl:
    """energy >= th[0] -> 0, >= th[1] -> 1, >= th[2] -> 2, else 3 (reset gear 3);
    upgrades wait for hyst_cnt agreeing candidates, downgrades are immediate."""

    def __init__(self, thresholds=(500, 200, 50), hyst_cnt: int = 3):
        self._s = _State()
        lo = (C.c_uint64 * 3)(*[_split(t)[0] for t in thresholds])
        hi = (C.c_uint64 * 3)(*[_split(t)[1] for t in thresholds])
        _lib.call("ckks_gear_ctrl_init", C.byref(self._s), lo, hi, int(hyst_cnt))

    @property
    def gear(self) -> int:
        return int(self._s.gear)

    def raw(self, energy: int) -> int:
        lo, hi = _split(energy)
        return int(_lib.raw("ckks_gear_ctrl_raw")(C.byref(self._s), lo, hi))

    def flush(self, energy: int, hysteresis: bool = True, manual_en: bool = False,
              manual_gear: int = 0) -> int:
        lo, hi = _split(energy)
        return int(_lib.raw("ckks_gear_ctrl_flush")(C.byref(self._s), lo, hi, int(hysteresis),
                                                    int(manual_en), int(manual_gear)))

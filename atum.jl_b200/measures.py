"""Measures (src/measures.jl:6-33) as deterministic FP64 device reductions."""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib

__all__ = ["weightednorm", "entropyintegral", "entropyproduct", "check_finite"]


def weightednorm(dg, q, p=2, componentwise: bool = False, stream=None):
    """MJ-weighted p-norm per component, then the p-norm over components (p = 2 or Inf)."""
    ns = dg.law.numberofstates
    comp = np.zeros(ns)
    tot = C.c_double()
    pp = math.inf if p in (math.inf, "Inf", "inf") else float(p)
    _lib.check(_lib.lib().atb_weightednorm(dg.device.h, _lib.field_ptrs(q, ns), pp, _lib.dptr(comp),
                                           C.byref(tot), _lib.stream_ptr(stream)))
    return comp if componentwise else tot.value


def entropyintegral(dg, q, stream=None) -> float:
    out = C.c_double()
    _lib.check(_lib.lib().atb_entropyintegral(dg.device.h, _lib.field_ptrs(q, dg.law.numberofstates),
                                              C.byref(out), _lib.stream_ptr(stream)))
    return out.value


def entropyproduct(dg, p, q, stream=None) -> float:
    ns = dg.law.numberofstates
    out = C.c_double()
    _lib.check(_lib.lib().atb_entropyproduct(dg.device.h, _lib.field_ptrs(p, ns), _lib.field_ptrs(q, ns),
                                             C.byref(out), _lib.stream_ptr(stream)))
    return out.value


def check_finite(dg, q, stream=None):
    """Raises AtbError(ATB_ERR_NONFINITE) if q holds NaN or Inf."""
    _lib.check(_lib.lib().atb_check_finite(dg.device.h, _lib.field_ptrs(q, dg.law.numberofstates),
                                           _lib.stream_ptr(stream)))

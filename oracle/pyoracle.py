"""TEST INFRASTRUCTURE — ctypes wrapper of the CPU oracle (oracle/liboracle.so).

The oracle restates the reference's DGSEM tendency and time stepping on the
CPU (oracle.cpp).  Only tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline leg import this module, as the checker or the timed CPU
baseline; the product path never does.

Fields are numpy float64 arrays of shape (Ns, K, Np) (or anything with that
many elements in that SoA order).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
# void (*)(double ex_time, double im_time, const double* q_stage, void* user)
_STAGE_CB = C.CFUNCTYPE(None, C.c_double, C.c_double, C.POINTER(C.c_double), C.c_void_p)


class _Desc(C.Structure):
    _fields_ = [
        ("law", C.c_int), ("dim", C.c_int), ("N", C.c_int), ("K", C.c_int * 3),
        ("v", C.POINTER(C.c_double) * 3), ("periodic", C.c_int * 3), ("stacked", C.c_int),
        ("volume_form", C.c_int), ("volume_flux", C.c_int), ("fd_kernel", C.c_int),
        ("surface_flux", C.c_int), ("directions", C.c_int),
        ("gamma", C.c_double), ("grav", C.c_double), ("adv_u", C.c_double * 3),
        ("sphere", C.c_int), ("pde_level_balance", C.c_int),
        ("bc_kind", C.c_int), ("bc_state", (C.c_double * 5) * 2),
        ("source_kind", C.c_int), ("omega", C.c_double * 3), ("sw_topography", C.c_int),
        ("naux", C.c_int),
    ]


def build(force: bool = False) -> str:
    so = os.path.join(_HERE, "liboracle.so")
    srcs = [os.path.join(_HERE, f) for f in ("oracle.cpp", "physics.hpp", "oracle.h")]
    if force or not os.path.exists(so) or any(os.path.getmtime(s) > os.path.getmtime(so) for s in srcs):
        subprocess.run(["make", "-C", _HERE, "-s", "liboracle.so"], check=True)
    return so


def lib():
    global _LIB
    if _LIB is None:
        L = C.CDLL(build())
        vp, dp = C.c_void_p, C.POINTER(C.c_double)
        L.orc_op_create.restype = vp
        L.orc_op_create.argtypes = [C.POINTER(_Desc), dp]
        L.orc_op_destroy.argtypes = [vp]
        L.orc_op_apply.argtypes = [vp, dp, dp, C.c_double, C.c_int]
        L.orc_op_set_curved.restype = C.c_int
        L.orc_op_set_curved.argtypes = [vp, dp, dp, dp, dp, C.POINTER(C.c_longlong), C.POINTER(C.c_int), dp]
        L.orc_points.argtypes = [vp, dp]
        L.orc_mj.argtypes = [vp, dp]
        L.orc_solver_create.restype = vp
        L.orc_solver_create.argtypes = [C.c_int, vp, vp, C.c_double, C.c_double, C.c_int, C.c_int]
        L.orc_solver_destroy.argtypes = [vp]
        L.orc_solve.restype = C.c_int
        L.orc_solve.argtypes = [vp, dp, C.c_double, C.c_int]
        L.orc_step.argtypes = [vp, dp, C.c_int]
        for f in ("orc_solver_time", "orc_solver_dt", "orc_solver_gamma"):
            getattr(L, f).restype = C.c_double
            getattr(L, f).argtypes = [vp]
        L.orc_weightednorm.restype = C.c_double
        L.orc_weightednorm.argtypes = [vp, dp, C.c_double, dp]
        L.orc_entropyintegral.restype = C.c_double
        L.orc_entropyintegral.argtypes = [vp, dp]
        L.orc_entropyproduct.restype = C.c_double
        L.orc_entropyproduct.argtypes = [vp, dp, dp]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_count_flops.argtypes = [C.POINTER(_Desc), C.c_int, C.c_int, dp, dp, dp, dp, dp, C.POINTER(C.c_long)]
        L.orc_set_stage_callback.argtypes = [vp, _STAGE_CB, vp]
        _LIB = L
    return _LIB


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def set_threads(n: int):
    lib().orc_set_threads(int(n))


def make_desc(fields: dict):
    """Build the oracle descriptor from the host DGSEM's descriptor fields."""
    d = _Desc()
    keep = []
    for k, v in fields.items():
        if k == "vertices":
            for i, vv in enumerate(v):
                arr = np.ascontiguousarray(vv, dtype=np.float64)
                keep.append(arr)
                d.v[i] = _dp(arr)
        elif k in ("K", "periodic", "adv_u", "omega"):
            arr = getattr(d, k)
            for i, x in enumerate(v):
                arr[i] = x
        elif k == "bc_state":
            for i in range(2):
                for j in range(5):
                    d.bc_state[i][j] = v[i][j]
        elif hasattr(d, k):
            setattr(d, k, v)
    return d, keep


class DGSEM:
    """Oracle twin of a host ``DGSEM`` spec (same law, grid, forms, aux)."""

    def __init__(self, dg):
        self.spec = dg
        fields = dg.descriptor_fields()
        self._desc, self._keep = make_desc(fields)
        aux = np.ascontiguousarray(dg.auxstate_host(), dtype=np.float64)
        self._aux = aux
        self.ns = dg.law.numberofstates
        self.K = len(dg.grid)
        self.Np = dg.grid.cell.Np
        self.dim = dg.grid.dim
        self.h = lib().orc_op_create(C.byref(self._desc), _dp(aux) if aux.size else None)
        geo = getattr(dg.grid, "geometry", None)
        if geo is not None:
            G = geo()
            arrs = [np.ascontiguousarray(G[k], dtype=np.float64) for k in ("g", "MJ", "normals", "faceMJ", "x")]
            nb = np.ascontiguousarray(G["nbr_node"], dtype=np.int64)
            bt = np.ascontiguousarray(G["btag"], dtype=np.int32)
            self._geo = (arrs, nb, bt)
            rc = lib().orc_op_set_curved(self.h, _dp(arrs[0]), _dp(arrs[1]), _dp(arrs[2]), _dp(arrs[3]),
                                         nb.ctypes.data_as(C.POINTER(C.c_longlong)),
                                         bt.ctypes.data_as(C.POINTER(C.c_int)), _dp(arrs[4]))
            if rc != 0:
                raise ValueError("curved geometry rejected by the oracle")

    def __del__(self):
        if getattr(self, "h", None) and _LIB is not None:
            _LIB.orc_op_destroy(self.h)
            self.h = None

    def fieldarray(self):
        return np.zeros((self.ns, self.K, self.Np))

    def __call__(self, dq: np.ndarray, q: np.ndarray, time: float = 0.0, increment: bool = True):
        lib().orc_op_apply(self.h, _dp(dq), _dp(q), float(time), int(bool(increment)))

    def points(self):
        x = np.zeros((self.dim, self.K, self.Np))
        lib().orc_points(self.h, _dp(x))
        return x

    @property
    def MJ(self):
        m = np.zeros((self.K, self.Np))
        lib().orc_mj(self.h, _dp(m))
        return m


_KIND = {"LSRK54": 0, "LSRK144": 1, "RLSRK54": 2, "RLSRK144": 3, "ARK23": 4}


class Solver:
    def __init__(self, kind: str, rhs, dt: float, t0: float = 0.0, linrhs=None, split_rhs: bool = True,
                 paperversion: bool = False):
        self.rhs, self.linrhs = rhs, linrhs
        self.h = lib().orc_solver_create(_KIND[kind], rhs.h if rhs is not None else None,
                                         linrhs.h if linrhs is not None else None, float(dt), float(t0),
                                         int(bool(split_rhs)), int(bool(paperversion)))

    def __del__(self):
        if getattr(self, "h", None) and _LIB is not None:
            _LIB.orc_solver_destroy(self.h)
            self.h = None

    @property
    def time(self):
        return lib().orc_solver_time(self.h)

    @property
    def dt(self):
        return lib().orc_solver_dt(self.h)

    @property
    def gamma(self):
        return lib().orc_solver_gamma(self.h)

    def step(self, q: np.ndarray, nsteps: int = 1):
        lib().orc_step(self.h, _dp(q), int(nsteps))

    def set_after_stage(self, fn):
        """``fn(ex_time, im_time, q_stage)`` after every stage (LSRK / RLSRK)
        or after ARK23 stages 2 and 3, as the reference's ``after_stage``;
        ``q_stage`` is a copy of the stage state.  None clears it."""
        if fn is None:
            self._cb = None
            lib().orc_set_stage_callback(self.h, _STAGE_CB(), None)
            return
        n = self.rhs.ns * self.rhs.K * self.rhs.Np if self.rhs is not None else \
            self.linrhs.ns * self.linrhs.K * self.linrhs.Np

        def cb(ex_t, im_t, qp, user):
            fn(ex_t, im_t, np.ctypeslib.as_array(qp, shape=(n,)).copy())

        self._cb = _STAGE_CB(cb)
        lib().orc_set_stage_callback(self.h, self._cb, None)

    def set_stage_hook(self, fn):
        """``fn(q)`` after every stage with the solver's own state as a
        writable array (no copy): what it writes is what the next stage reads
        (a sharded run's ghost exchange).  None clears it."""
        if fn is None:
            self._cb = None
            lib().orc_set_stage_callback(self.h, _STAGE_CB(), None)
            return
        any_ = self.rhs if self.rhs is not None else self.linrhs
        shape = (any_.ns, any_.K, any_.Np)

        def cb(ex_t, im_t, qp, user):
            fn(np.ctypeslib.as_array(qp, shape=shape))

        self._cb = _STAGE_CB(cb)
        lib().orc_set_stage_callback(self.h, self._cb, None)


def LSRK54(dg, q, dt, t0=0.0):
    return Solver("LSRK54", dg, dt, t0)


def LSRK144(dg, q, dt, t0=0.0):
    return Solver("LSRK144", dg, dt, t0)


def RLSRK54(dg, q, dt, t0=0.0):
    return Solver("RLSRK54", dg, dt, t0)


def RLSRK144(dg, q, dt, t0=0.0):
    return Solver("RLSRK144", dg, dt, t0)


def ARK23(dg, lindg, q, dt, t0=0.0, paperversion=False, split_rhs=True):
    return Solver("ARK23", dg, dt, t0, linrhs=lindg, split_rhs=split_rhs, paperversion=paperversion)


def solve_(q: np.ndarray, timeend: float, solver: Solver, adjust_final: bool = True) -> int:
    """``solve!`` (src/odesolvers.jl:9-26); returns the number of steps."""
    return lib().orc_solve(solver.h, _dp(q), float(timeend), int(bool(adjust_final)))


def weightednorm(dg: DGSEM, q: np.ndarray, p: float = 2, componentwise: bool = False):
    comp = np.zeros(dg.ns)
    tot = lib().orc_weightednorm(dg.h, _dp(np.ascontiguousarray(q)), float(p), _dp(comp))
    return comp if componentwise else tot


def entropyintegral(dg: DGSEM, q: np.ndarray) -> float:
    return lib().orc_entropyintegral(dg.h, _dp(np.ascontiguousarray(q)))


def entropyproduct(dg: DGSEM, p: np.ndarray, q: np.ndarray) -> float:
    return lib().orc_entropyproduct(dg.h, _dp(np.ascontiguousarray(p)), _dp(np.ascontiguousarray(q)))


def count_flops(dg, what: int, kind: int, q1, a1, q2, a2, n):
    """Instrumented-type operation counts for one pointwise call:
    what 0 flux, 1 twopointflux, 2 surfaceflux, 3 wavespeed.
    Returns dict add/mul/div/sqrt/log/pow."""
    d, keep = make_desc(dg.descriptor_fields())
    arrs = []
    for a, n_ in ((q1, 5), (a1, 8), (q2, 5), (a2, 8), (n, 3)):
        x = np.zeros(n_)
        x[: len(a)] = a
        arrs.append(x)
    out = (C.c_long * 6)()
    lib().orc_count_flops(C.byref(d), int(what), int(kind), *[_dp(a) for a in arrs], out)
    return dict(zip(("add", "mul", "div", "sqrt", "log", "pow"), list(out)))

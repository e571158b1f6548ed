"""Time steppers (host side of src/odesolvers.jl) driving the C ABI.

``LSRK54(dg, q, dt)``, ``LSRK144``, ``RLSRK54``, ``RLSRK144`` and
``ARK23(dg, lindg, q, dt; paperversion, split_rhs)`` construct solvers
(src/odesolvers.jl:59-67,138-146,284-309); ``solve_(q, timeend, solver;
after_step, after_stage, adjust_final)`` mirrors ``solve!``
(src/odesolvers.jl:9-26): same step loop, same final-dt adjustment.

Every stage runs on the GPU: LSRK stages are single fused tendency +
write-back kernels, ARK23 stages are tendency kernels plus one batched
vertical banded solve fused with the right-hand-side combination.
"""
from __future__ import annotations

import ctypes as C
from typing import Callable, Optional

from . import _lib

__all__ = ["LSRK54", "LSRK144", "RLSRK54", "RLSRK144", "ARK23", "solve_", "Solver"]

_KINDS = {"LSRK54": 0, "LSRK144": 1, "RLSRK54": 2, "RLSRK144": 3, "ARK23": 4}


class Solver:
    def __init__(self, kind: str, rhs, dt: float, t0: float = 0.0, linrhs=None, split_rhs: bool = True,
                 paperversion: bool = False):
        self.kind = kind
        self.rhs = rhs
        self.linrhs = linrhs
        any_ = rhs if rhs is not None else linrhs
        self.ns = any_.law.numberofstates
        h = C.c_void_p()
        _lib.check(_lib.lib().atb_solver_create(_KINDS[kind], rhs.device.h if rhs is not None else None,
                                                linrhs.device.h if linrhs is not None else None, float(dt),
                                                float(t0), int(bool(split_rhs)), int(bool(paperversion)),
                                                C.byref(h)))
        self.h = h

    def __del__(self):
        h = getattr(self, "h", None)
        if h and _lib._LIB is not None:
            _lib._LIB.atb_solver_destroy(h)
            self.h = None

    def _get(self):
        t, dt, g = C.c_double(), C.c_double(), C.c_double()
        _lib.check(_lib.lib().atb_solver_get(self.h, C.byref(t), C.byref(dt), C.byref(g)))
        return t.value, dt.value, g.value

    @property
    def time(self) -> float:
        return self._get()[0]

    @property
    def dt(self) -> float:
        return self._get()[1]

    @dt.setter
    def dt(self, v: float):
        _lib.check(_lib.lib().atb_solver_set_dt(self.h, float(v)))

    @property
    def gamma(self) -> float:
        return self._get()[2]

    def state(self) -> dict:
        """The solver scalars a checkpoint needs (``atum_b200.checkpoint``)."""
        t, dt, g = self._get()
        return {"kind": self.kind, "time": t, "dt": dt, "gamma": g}

    def set_state(self, time: float, gamma: float = 1.0):
        """Restores the clock and the last relaxation factor of a checkpoint."""
        _lib.check(_lib.lib().atb_solver_set_state(self.h, float(time), float(gamma)))

    def fuse(self, enable: bool = True):
        """ARK23: run the explicit and the linear operator of a stage as one
        kernel (on by default when the operators allow it)."""
        _lib.check(_lib.lib().atb_solver_fuse(self.h, int(bool(enable))))

    def step(self, q, nsteps: int = 1, stream=None):
        """``dostep!`` repeated ``nsteps`` times (no host synchronisation)."""
        _lib.check(_lib.lib().atb_solver_step(self.h, _lib.field_ptrs(q, self.ns), int(nsteps),
                                              _lib.stream_ptr(stream)))


def LSRK54(rhs, q, dt, t0=0.0):
    return Solver("LSRK54", rhs, dt, t0)


def LSRK144(rhs, q, dt, t0=0.0):
    return Solver("LSRK144", rhs, dt, t0)


def RLSRK54(rhs, q, dt, t0=0.0):
    return Solver("RLSRK54", rhs, dt, t0)


def RLSRK144(rhs, q, dt, t0=0.0):
    return Solver("RLSRK144", rhs, dt, t0)


def ARK23(rhs, linrhs, q, dt, t0=0.0, paperversion=False, split_rhs=True):
    return Solver("ARK23", rhs, dt, t0, linrhs=linrhs, split_rhs=split_rhs, paperversion=paperversion)


def solve_(q, timeend: float, solver: Solver, after_step: Optional[Callable] = None,
           after_stage: Optional[Callable] = None, adjust_final: bool = True, stream=None) -> int:
    """``solve!(q, timeend, solver; after_step, after_stage, adjust_final)``.

    Returns the number of steps.  ``after_step(step, time, q)`` runs on the
    host after each step.  ``after_stage`` runs on the host between stages, as
    in the reference (src/odesolvers.jl:54,119,378): LSRK / RLSRK call
    ``after_stage(stagetime, q)`` after every stage with the caller's ``q``
    (changes to it carry into the next stage); ARK23 calls
    ``after_stage((ex_stagetime, im_stagetime), Q)`` after stages 2 and 3 with
    a zero-copy view ``Q`` of the solver's stage state.  The stage's kernels
    are enqueued on the stream when the callback runs; torch operations on the
    same stream are ordered after them.
    """
    if after_stage is None:
        return _solve(q, timeend, solver, after_step, adjust_final, stream)
    err = []
    shape = tuple(q.shape[1:]) if not isinstance(q, (list, tuple)) else tuple(q[0].shape)
    ark = solver.kind == "ARK23"

    def cb(ex_t, im_t, ptrs, user):
        try:
            if ark:
                after_stage((ex_t, im_t), _lib.device_view(ptrs, solver.ns, shape))
            else:
                after_stage(ex_t, q)
            return 0
        except BaseException as e:  # re-raised below; a C callback cannot propagate it
            err.append(e)
            return 1

    fn = _lib.STAGE_CB(cb)
    _lib.check(_lib.lib().atb_solver_set_stage_callback(solver.h, fn, None))
    try:
        return _solve(q, timeend, solver, after_step, adjust_final, stream)
    except _lib.AtbError:
        if err:
            raise err[0]
        raise
    finally:
        _lib.lib().atb_solver_set_stage_callback(solver.h, _lib.STAGE_CB(), None)


def _solve(q, timeend, solver, after_step, adjust_final, stream) -> int:
    if after_step is None:
        steps = C.c_int()
        _lib.check(_lib.lib().atb_solve(solver.h, _lib.field_ptrs(q, solver.ns), float(timeend),
                                        int(bool(adjust_final)), C.byref(steps), _lib.stream_ptr(stream)))
        return steps.value
    step = 0
    while True:
        step += 1
        time, dt, _ = solver._get()
        final = False
        if time + dt >= timeend:
            if adjust_final:
                solver.dt = timeend - time
            final = True
        solver.step(q, 1, stream)
        after_step(step, time, q)
        if final:
            return step

"""Multi-instance batching: many small DGSEM problems advanced by one launch.

The reference builds one ``DGSEM`` per problem (src/dgsem.jl:38-56) and steps
each alone; a small problem (a 32x32 shallow-water basin, a 2-D vortex) fills a
few SMs of a B200.  ``PackedDGSEM(dgs)`` packs instances that share law,
order, forms, fluxes, directions, precision and problem kinds (their grids may
differ) into one operator through ``atb_op_create_batch``: the instances'
elements are concatenated, neighbour indices stay inside each instance, and one
tendency launch advances all of them.  Every instance's result is bitwise the
one it gets alone, because each node sees exactly the same operands in the same
order.

A packed state is a ``(Ns, sum K_i, Np)`` float64 tensor: the instances'
fields concatenated per component (``pack`` / ``unpack``).  ``LSRK54(packed,
q, dt)`` steps it; ``set_instance_dt(solver, dts)`` gives each instance its own
time step.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import _lib
from ._device import make_desc

__all__ = ["PackedDGSEM", "set_instance_dt", "autotune", "set_launch", "set_persistent"]


class _PackedDevice:
    def __init__(self, h, ns):
        self.h = h
        self.ns = ns

    def __del__(self):
        h = getattr(self, "h", None)
        if h and _lib._LIB is not None:
            _lib._LIB.atb_op_destroy(h)
            self.h = None

    def apply(self, dq, q, time=0.0, increment=True, stream=None):
        _lib.check(_lib.lib().atb_op_apply(self.h, _lib.field_ptrs(dq, self.ns), _lib.field_ptrs(q, self.ns),
                                           float(time), int(bool(increment)), _lib.stream_ptr(stream)))


class PackedDGSEM:
    """One operator over ``len(dgs)`` instances (``atb_op_create_batch``)."""

    def __init__(self, dgs: Sequence):
        dgs = list(dgs)
        if not dgs:
            raise ValueError("no instances")
        self.instances = dgs
        self.law = dgs[0].law
        self.ns = self.law.numberofstates
        self.Np = dgs[0].grid.cell.Np
        n = len(dgs)
        descs = (_lib.OpDesc * n)()
        keep = []
        auxs = []
        for i, dg in enumerate(dgs):
            d, k = make_desc(dg)
            descs[i] = d
            keep.append(k)
            auxs.append(np.ascontiguousarray(dg.auxstate_host(), dtype=np.float64).reshape(-1))
        aux_ptrs = (_lib._DP * n)()
        for i, a in enumerate(auxs):
            aux_ptrs[i] = _lib.dptr(a) if a.size else None
        h = C.c_void_p()
        _lib.check(_lib.lib().atb_op_create_batch(descs, n, aux_ptrs, C.byref(h)))
        self._dev = _PackedDevice(h, self.ns)
        nn = C.c_int()
        offs = (C.c_int * (n + 1))()
        _lib.check(_lib.lib().atb_op_instances(h, C.byref(nn), offs))
        self.offsets = [int(offs[i]) for i in range(n + 1)]
        self.K = self.offsets[-1]

    @property
    def device(self):
        return self._dev

    def __len__(self):
        return len(self.instances)

    def __call__(self, dq, q, time: float = 0.0, increment: bool = True):
        self._dev.apply(dq, q, time, increment)

    def pack(self, qs):
        """(Ns, sum K_i, Np) tensor from the instances' (Ns, K_i, Np) fields."""
        import torch

        if len(qs) != len(self.instances):
            raise ValueError("one field per instance")
        return torch.cat([q.reshape(self.ns, -1, self.Np) for q in qs], dim=1).contiguous()

    def unpack(self, q):
        """Views of each instance's (Ns, K_i, Np) part of a packed field."""
        return [q[:, a:b] for a, b in zip(self.offsets[:-1], self.offsets[1:])]

    def autotune(self, q):
        return autotune(self, q)

    def set_launch(self, elements_per_cta: int):
        set_launch(self, elements_per_cta)

    def set_persistent(self, ctas: int):
        set_persistent(self, ctas)


def autotune(dg, q) -> int:
    """Pick the elements-per-CTA launch shape of a ``DGSEM`` or ``PackedDGSEM``
    by timing its tendency on state ``q`` (results do not depend on it)."""
    import torch

    ns = dg.law.numberofstates
    scratch = torch.empty(q.numel(), dtype=torch.float64, device=q.device)
    chosen = C.c_int()
    _lib.check(_lib.lib().atb_op_autotune(dg.device.h, _lib.field_ptrs(q, ns),
                                          C.cast(C.c_void_p(scratch.data_ptr()), _lib._DP),
                                          _lib.stream_ptr(), C.byref(chosen)))
    torch.cuda.current_stream().synchronize()
    return chosen.value


def set_launch(dg, elements_per_cta: int):
    _lib.check(_lib.lib().atb_op_set_launch(dg.device.h, int(elements_per_cta)))


def set_persistent(dg, ctas: int):
    """Persistent tendency launches of at most ``ctas`` CTAs that walk the
    element tiles of every packed instance with a grid stride (0: one CTA per
    tile).  Results do not depend on it."""
    _lib.check(_lib.lib().atb_op_set_persistent(dg.device.h, int(ctas)))


def set_instance_dt(solver, dts):
    """Per-instance time steps of an LSRK solver over a ``PackedDGSEM``
    (``None`` returns to the solver's single dt)."""
    if dts is None:
        _lib.check(_lib.lib().atb_solver_set_instance_dt(solver.h, None))
        return
    arr = np.ascontiguousarray(dts, dtype=np.float64)
    _lib.check(_lib.lib().atb_solver_set_instance_dt(solver.h, _lib.dptr(arr)))

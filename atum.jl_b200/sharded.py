"""One problem sharded over several GPUs by element slabs (no reference
counterpart: the reference runs one problem on one device).

A brick grid is cut along its first dimension into ``world`` slabs of whole
element columns (``numpy.array_split`` of the first-dimension element index,
so the vertical columns of a stacked grid stay whole and ARK23's banded solve
needs no communication).  Each rank holds its slab plus one ghost column of
elements on each side that has a neighbour (periodic wrap included): its
local grid is an ordinary brick grid, non-periodic along the cut dimension,
whose tendency kernels see the ghost elements as neighbours.  Before every
tendency launch that reads a new state (``atb_solver_set_exchange_callback``)
each rank sends the states of its first and last owned columns to its
neighbours and receives their columns into its ghosts; the owned elements'
arithmetic is then exactly that of the unsharded problem (the ghosts' own
updates are overwritten by the next exchange).

* ``slab_layout(grid, rank, world)`` -- the local grid and the element maps;
* ``local_dgsem(dg, layout)`` -- the rank's DGSEM (same law, forms, fluxes,
  directions, precision; aux fields taken from the global ones);
* ``DistExchanger(layout)`` -- the exchange over ``torch.distributed``
  (NCCL on GPUs, gloo on CPUs), batched isend / irecv per exchange;
* ``LocalExchanger(layouts, packed)`` -- every rank's slab packed into one
  operator in one process (``atb_op_create_batch``), the exchange a set of
  device copies (used to test the sharded arithmetic on one GPU);
* ``attach(solver, exchanger)`` -- installs the exchange hook on a solver.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from .cell import BrickGrid, brickgrid

__all__ = ["SlabLayout", "slab_layout", "local_dgsem", "DistExchanger", "LocalExchanger", "attach"]


@dataclass
class SlabLayout:
    rank: int
    world: int
    x0: int                   # first owned column (first-dimension element index) of the global grid
    x1: int                   # one past the last owned column
    ghost_left: bool
    ghost_right: bool
    grid: BrickGrid           # the local grid (ghost columns included)
    local_to_global: np.ndarray  # global element of every local element
    owned: np.ndarray         # local elements that this rank owns, in global order
    left: int                 # rank of the left / right neighbour (-1: none)
    right: int

    def column(self, ix: int) -> np.ndarray:
        """Local elements of local column ix (first-dimension index), in a
        fixed order (the same on every rank for the same global column)."""
        eidx = self.grid.element_indices()
        sel = np.nonzero(eidx[:, 0] == ix)[0]
        order = np.lexsort(tuple(eidx[sel, d] for d in range(self.grid.dim - 1, 0, -1)))
        return sel[order]

    @property
    def nown(self) -> int:
        return self.x1 - self.x0

    def send_left(self):   # first owned column -> the left neighbour's right ghost
        return self.column(1 if self.ghost_left else 0)

    def send_right(self):  # last owned column -> the right neighbour's left ghost
        return self.column((1 if self.ghost_left else 0) + self.nown - 1)

    def recv_left(self):
        return self.column(0)

    def recv_right(self):
        return self.column((1 if self.ghost_left else 0) + self.nown)


def slab_layout(grid: BrickGrid, rank: int, world: int) -> SlabLayout:
    if world < 2:
        raise ValueError("sharding needs world >= 2")
    Kx = grid.Kd[0]
    if Kx < world:
        raise ValueError("fewer element columns than ranks")
    cuts = np.array_split(np.arange(Kx), world)
    x0, x1 = int(cuts[rank][0]), int(cuts[rank][-1]) + 1
    per = grid.periodic[0]
    gl = per or x0 > 0
    gr = per or x1 < Kx
    if per and world == 2 and Kx == 2:
        raise ValueError("a periodic direction needs more than two columns for two ranks")
    v = np.asarray(grid.vertices[0], dtype=np.float64)
    cols = list(range(x0, x1))
    vx = list(v[x0:x1 + 1])
    if gl:
        c = (x0 - 1) % Kx
        vx.insert(0, vx[0] - (v[c + 1] - v[c]))
        cols.insert(0, c)
    if gr:
        c = x1 % Kx
        vx.append(vx[-1] + (v[c + 1] - v[c]))
        cols.append(c)
    verts = (np.array(vx),) + tuple(np.asarray(vv, dtype=np.float64) for vv in grid.vertices[1:])
    lgrid = brickgrid(grid.cell, verts, periodic=(False,) + tuple(grid.periodic[1:]),
                      ordering="stacked" if grid.stacked else "cartesian")
    # local element -> global element through the per-dimension indices
    le = lgrid.element_indices()
    ge = grid.element_indices()
    gindex = {tuple(ix): e for e, ix in enumerate(ge)}
    gidx = le.copy()
    gidx[:, 0] = np.asarray(cols)[le[:, 0]]
    l2g = np.array([gindex[tuple(ix)] for ix in gidx], dtype=np.int64)
    own_lo = 1 if gl else 0
    owned = np.nonzero((le[:, 0] >= own_lo) & (le[:, 0] < own_lo + (x1 - x0)))[0]
    owned = owned[np.argsort(l2g[owned])]
    left = (rank - 1) % world if gl else -1
    right = (rank + 1) % world if gr else -1
    return SlabLayout(rank, world, x0, x1, bool(gl), bool(gr), lgrid, l2g, owned, left, right)


def local_dgsem(dg, layout: SlabLayout):
    """The rank's DGSEM: the global spec on the local grid, its aux fields the
    global ones at the local elements."""
    from .dgsem import DGSEM

    aux = np.ascontiguousarray(dg.auxstate_host()[:, layout.local_to_global, :])
    return DGSEM(law=dg.law, grid=layout.grid, surface_numericalflux=dg.surface_numericalflux,
                 volume_form=dg.volume_form, directions=dg.directions, auxstate=aux, precision=dg.precision)


class DistExchanger:
    """Ghost-column exchange over torch.distributed (any backend with
    point-to-point operations: NCCL, gloo).  ``exchange(q)`` takes the local
    state as an (ns, K, Np) tensor (or a list of ns (K, Np) tensors) and
    fills its ghost columns."""

    def __init__(self, layout: SlabLayout, group=None, device=None):
        import torch

        self.layout, self.group = layout, group
        dev = device if device is not None else "cpu"
        L = layout
        self.idx = {k: torch.as_tensor(getattr(L, k)(), dtype=torch.long, device=dev)
                    for k in ("send_left", "send_right", "recv_left", "recv_right")}

    def exchange(self, q):
        import torch
        import torch.distributed as dist

        L = self.layout
        comps = list(q) if isinstance(q, (list, tuple)) else [q[c] for c in range(q.shape[0])]
        ops, recvs, keep = [], [], []
        # messages going left (a rank's first owned column -> its left
        # neighbour's right ghost, tag 0), then going right (last owned column
        # -> the right neighbour's left ghost, tag 1); every rank posts them in
        # this order, so with two ranks on a periodic cut (both neighbours the
        # same rank) the k-th message between a pair is the same on both sides
        for tag, (to, sk, frm, rk) in enumerate(((L.left, "send_left", L.right, "recv_right"),
                                                 (L.right, "send_right", L.left, "recv_left"))):
            if to >= 0:
                send = torch.stack([c.index_select(0, self.idx[sk]) for c in comps]).contiguous()
                ops.append(dist.P2POp(dist.isend, send, to, group=self.group, tag=tag))
                keep.append(send)
            if frm >= 0:
                n = self.idx[rk].numel()
                recv = torch.empty((len(comps), n) + tuple(comps[0].shape[1:]), dtype=comps[0].dtype,
                                   device=comps[0].device)
                ops.append(dist.P2POp(dist.irecv, recv, frm, group=self.group, tag=tag))
                recvs.append((rk, recv))
        if ops:
            for r in dist.batch_isend_irecv(ops):
                r.wait()
        for rk, recv in recvs:
            for c, comp in enumerate(comps):
                comp.index_copy_(0, self.idx[rk], recv[c])


class LocalExchanger:
    """Every rank's slab in one packed operator (atb_op_create_batch) in one
    process: the exchange copies, on the device, each slab's first and last
    owned columns into its neighbours' ghost columns."""

    def __init__(self, layouts, first_elements, device="cuda"):
        import torch

        self.pairs = []  # (source global-local element rows, destination rows)
        for L in layouts:
            off = int(first_elements[L.rank])
            for peer, sk, rk in ((L.left, "send_left", "recv_right"), (L.right, "send_right", "recv_left")):
                if peer < 0:
                    continue
                src = off + np.asarray(getattr(L, sk)())
                dst = int(first_elements[peer]) + np.asarray(getattr(layouts[peer], rk)())
                self.pairs.append((torch.as_tensor(src, device=device), torch.as_tensor(dst, device=device)))

    def exchange(self, q):
        comps = list(q) if isinstance(q, (list, tuple)) else [q[c] for c in range(q.shape[0])]
        for src, dst in self.pairs:
            for comp in comps:
                comp.index_copy_(0, dst, comp.index_select(0, src))


EXCHANGE_CB = _lib.EXCHANGE_CB


def attach(solver, exchanger, K: int, Np: int):
    """Installs ``exchanger.exchange`` as the solver's exchange hook (state
    views without copies); returns the ctypes callback, which the caller keeps
    alive while the solver steps.  ``attach(solver, None, 0, 0)`` removes it."""
    L = _lib.lib()
    if exchanger is None:
        _lib.check(L.atb_solver_set_exchange_callback(solver.h, EXCHANGE_CB(), None))
        return None
    ns = solver.ns

    def cb(ptrs, user):
        try:
            exchanger.exchange(_lib.device_view(ptrs, ns, (K, Np)))
            return 0
        except Exception:  # noqa: BLE001 -- reported to the caller as ATB_ERR_CALLBACK
            import traceback
            traceback.print_exc()
            return 1

    fn = EXCHANGE_CB(cb)
    _lib.check(L.atb_solver_set_exchange_callback(solver.h, fn, None))
    solver._exchange_cb = fn
    return fn

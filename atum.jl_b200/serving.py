"""Serving loop: a stream of DGSEM problems advanced by shared launches.

No counterpart in the reference (it runs one problem per process).  Requests
arrive over time (``Request``: an instance spec, its initial state, its time
step and step count); the server packs the requests that share an operator
kind -- law, order N, forms, fluxes, precision, problem kinds; element counts
and grids may differ -- into element pools and advances each pool with one
tendency launch per LSRK stage:

* a pool (``_Pool``) is an operator with room for ``capacity`` elements
  (``atb_op_create_pool``); an admitted request takes the next free element
  range, where ``atb_op_place_instance`` writes its metrics, neighbour table and
  aux fields, and its initial state is copied in from pinned host memory;
* admission is continuous: a request joins a pool of its kind with room, or a
  new pool when the HBM budget (bytes of every pool's states, stage buffers,
  aux fields and tables) has room -- idle pools are released for it first --
  otherwise it waits in the queue;
* placed requests stay dense at the front of a pool: when requests finish, the
  later ones move down (state copied on the device, geometry placed again);
  launches cover the used prefix rounded up to ``chunk`` elements, and the
  elements past the last request take a zero time step;
* every element has its own time step (``atb_solver_set_element_dt``, a device
  array refreshed on the pool's stream when membership changes), so requests
  with different dt share a launch;
* each pool runs on its own CUDA stream; a scheduling tick advances a pool by
  ``S`` LSRK steps, ``S`` the largest power of two no larger than the fewest
  steps any of its requests still needs (capped by ``max_tick_steps``), so
  every request takes exactly its own step count; the launches of one tick are
  captured once per (launched prefix, S) into a CUDA graph and replayed;
* a finished request's state is copied to pinned host memory and its latency
  (arrival to result on the host) recorded.

Each request's result is bitwise the one it gets stepped alone: every node of
it sees the same operands in the same order whatever shares its pool.
``Server.run(requests)`` returns the stream's statistics: throughput in
DOF-stage updates per second, p50/p99 latency, peak HBM bytes held by pools.
"""
from __future__ import annotations

import ctypes as C
import math
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np

from . import _lib
from ._device import make_desc

__all__ = ["Request", "Server", "Stats", "kind_key", "pool_bytes_per_element"]

_KIND_STAGES = {"LSRK54": 5, "LSRK144": 14}
_GRID_FIELDS = ("K", "vertices", "periodic", "stacked")


@dataclass
class Request:
    rid: int
    dg: object                 # DGSEM spec of this instance
    q0: np.ndarray             # (Ns, K, Np) float64 initial state
    dt: float
    nsteps: int
    arrival: float = 0.0       # seconds after the stream starts
    # filled by the server
    admitted: float = math.nan
    finished: float = math.nan
    result: Optional[np.ndarray] = None

    @property
    def latency(self) -> float:
        return self.finished - self.arrival

    @property
    def dof(self) -> int:
        return int(np.prod(self.q0.shape))


def kind_key(dg) -> tuple:
    """Requests with equal keys can share a pool (their grids may differ)."""
    f = dg.descriptor_fields()
    parts = []
    for k in sorted(f):
        if k in _GRID_FIELDS:
            continue
        v = f[k]
        if isinstance(v, (list, tuple)):
            v = tuple(tuple(x) if isinstance(x, (list, tuple)) else x for x in v)
        parts.append((k, v))
    return tuple(parts)


def pool_bytes_per_element(dg) -> int:
    """Device bytes one pool element holds: state, LSRK increment and second
    state buffer, aux fields, per-element time step, metrics and neighbours."""
    ns = dg.law.numberofstates
    Np = dg.grid.cell.Np
    naux = dg.descriptor_fields()["naux"]
    return 8 * Np * (3 * ns + max(1, naux)) + (3 * 8 + 8 + 6 * 4 + 8)


class _Placed:
    __slots__ = ("req", "first", "K", "remaining", "desc", "keep", "aux")

    def __init__(self, req, first):
        self.req = req
        self.first = first
        self.K = req.dg.grid.K
        self.remaining = int(req.nsteps)
        self.desc, self.keep = make_desc(req.dg)
        self.aux = np.ascontiguousarray(req.dg.auxstate_host(), dtype=np.float64).reshape(-1)


class _PoolDevice:
    def __init__(self, h, ns):
        self.h = h
        self.ns = ns

    def __del__(self):
        h = getattr(self, "h", None)
        if h and _lib._LIB is not None:
            _lib._LIB.atb_op_destroy(h)
            self.h = None


class _Pool:
    def __init__(self, key, template, capacity: int, chunk: int, kind: str, max_tick_steps: int):
        import torch

        from .odesolvers import Solver

        self.key = key
        self.capacity = int(capacity)
        self.chunk = int(chunk)
        self.kind = kind
        self.max_tick_steps = max_tick_steps
        self.law = template.law
        self.ns = template.law.numberofstates
        self.Np = template.grid.cell.Np
        desc, keep = make_desc(template)
        h = C.c_void_p()
        _lib.check(_lib.lib().atb_op_create_pool(C.byref(desc), self.capacity, C.byref(h)))
        self._dev = _PoolDevice(h, self.ns)
        self.cuda = torch.device("cuda", torch.cuda.current_device())
        self.stream = torch.cuda.Stream(device=self.cuda)
        self.q = torch.zeros((self.ns, self.capacity, self.Np), dtype=torch.float64, device=self.cuda)
        self.solver = Solver(kind, self, 1.0)
        # one time step per element (0 past the last request), a fixed device
        # pointer read by every stage, so captured graphs see updates
        self.dte = torch.zeros(self.capacity, dtype=torch.float64, device=self.cuda)
        self.dte_pinned = torch.zeros(self.capacity, dtype=torch.float64).pin_memory()
        self._dt_event = None
        _lib.check(_lib.lib().atb_solver_set_element_dt(
            self.solver.h, C.cast(C.c_void_p(self.dte.data_ptr()), _lib._DP)))
        self.placed: List[_Placed] = []
        self.used = 0
        self.graphs: Dict[Tuple[int, int], object] = {}
        self.nbytes = self.capacity * pool_bytes_per_element(template)
        self.dof_stage_updates = 0
        self.warm = set()
        self.dirty = True
        self.staging = []

    # a Solver binds to a pool as to an operator
    @property
    def device(self):
        return self._dev

    def close(self):
        import torch

        self.stream.synchronize()
        self.graphs.clear()
        self.solver = None
        self._dev = None
        self.q = self.dte = None
        torch.cuda.empty_cache()

    def room(self) -> int:
        return self.capacity - self.used

    # admission ----------------------------------------------------------
    def _place(self, p: _Placed):
        _lib.check(_lib.lib().atb_op_place_instance(self._dev.h, p.first, C.byref(p.desc),
                                                    _lib.dptr(p.aux) if p.aux.size else None,
                                                    _lib.stream_ptr(self.stream)))

    def admit(self, r: Request, now: float):
        import torch

        p = _Placed(r, self.used)
        K = p.K
        with torch.cuda.stream(self.stream):
            self._place(p)
            src = torch.from_numpy(np.ascontiguousarray(r.q0, dtype=np.float64).reshape(self.ns, K, self.Np))
            stage = src.pin_memory()
            self.q[:, p.first:p.first + K].copy_(stage, non_blocking=True)
            # the pinned staging buffer lives until its copy has run
            self.staging.append((stage, torch.cuda.current_stream().record_event()))
        self.staging = [(s, e) for s, e in self.staging if not e.query()]
        self.placed.append(p)
        self.used += K
        r.admitted = now
        self.dirty = True

    # stepping -----------------------------------------------------------
    def _launched(self) -> int:
        return min(self.capacity, -(-self.used // self.chunk) * self.chunk)

    def tick_steps(self) -> int:
        m = min(p.remaining for p in self.placed)
        s = 1
        while s * 2 <= min(m, self.max_tick_steps):
            s *= 2
        return s

    def _refresh_dt(self):
        import torch

        # the previous transfer out of the pinned buffer must have run
        if self._dt_event is not None:
            self._dt_event.synchronize()
        host = self.dte_pinned.numpy()
        host[:] = 0.0
        for p in self.placed:
            host[p.first:p.first + p.K] = p.req.dt
        self.dte.copy_(self.dte_pinned, non_blocking=True)
        self._dt_event = torch.cuda.current_stream().record_event()
        self.dirty = False

    def tick(self, use_graphs: bool) -> int:
        import torch

        S = self.tick_steps()
        n = self._launched()
        with torch.cuda.stream(self.stream):
            if self.dirty:
                self._refresh_dt()
            _lib.check(_lib.lib().atb_op_set_active_elements(self._dev.h, n))
            key = (n, S)
            g = self.graphs.get(key) if use_graphs else None
            if g is not None:
                g.replay()
            elif not use_graphs or key not in self.warm:
                # direct launches (also the first use of a shape, before capture)
                self.solver.step(self.q, S, stream=self.stream)
                self.warm.add(key)
            else:
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g, stream=self.stream, capture_error_mode="thread_local"):
                    self.solver.step(self.q, S, stream=self.stream)
                self.graphs[key] = g
                g.replay()
        for p in self.placed:
            p.remaining -= S
        self.dof_stage_updates += self.ns * self.used * self.Np * _KIND_STAGES[self.kind] * S
        return S

    def retire(self, now_fn, done: List[Request]):
        """Copy finished requests to the host; move the rest down."""
        import torch

        fin = [p for p in self.placed if p.remaining <= 0]
        if not fin:
            return
        outs = []
        with torch.cuda.stream(self.stream):
            for p in fin:
                h = torch.empty((self.ns, p.K, self.Np), dtype=torch.float64).pin_memory()
                h.copy_(self.q[:, p.first:p.first + p.K], non_blocking=True)
                outs.append((p, h))
        self.stream.synchronize()
        t = now_fn()
        for p, h in outs:
            p.req.result = h.numpy()
            p.req.finished = t
            done.append(p.req)
        keep = [p for p in self.placed if p.remaining > 0]
        first = 0
        with torch.cuda.stream(self.stream):
            for p in keep:
                if p.first != first:
                    src = self.q[:, p.first:p.first + p.K].clone()
                    self.q[:, first:first + p.K].copy_(src)
                    p.first = first
                    self._place(p)
                first += p.K
        self.placed = keep
        self.used = first
        self.dirty = True


@dataclass
class Stats:
    requests: int = 0
    makespan_s: float = 0.0
    dof_stage_per_s: float = 0.0
    p50_latency_s: float = 0.0
    p99_latency_s: float = 0.0
    mean_latency_s: float = 0.0
    peak_pool_bytes: int = 0
    pools: int = 0
    ticks: int = 0
    extra: dict = field(default_factory=dict)


class Server:
    """Continuous-batching server for LSRK time stepping of many problems."""

    def __init__(self, hbm_budget_bytes: float = 150e9, capacity: int = 1 << 16, chunk: int = 256,
                 kind: str = "LSRK54", max_tick_steps: int = 16, use_graphs: bool = True):
        if kind not in _KIND_STAGES:
            raise ValueError("the server steps with LSRK54 or LSRK144")
        self.budget = float(hbm_budget_bytes)
        self.capacity = int(capacity)
        self.chunk = int(chunk)
        self.kind = kind
        self.max_tick_steps = int(max_tick_steps)
        self.use_graphs = use_graphs
        self.pools: Dict[tuple, List[_Pool]] = {}
        self.pool_bytes = 0
        self.peak_bytes = 0
        self.retired_updates = 0
        self.pools_made = 0

    def _release_idle(self, need: int):
        for k in list(self.pools):
            keep = []
            for p in self.pools[k]:
                if not p.placed and self.pool_bytes + need > self.budget:
                    self.pool_bytes -= p.nbytes
                    self.retired_updates += p.dof_stage_updates
                    p.close()
                else:
                    keep.append(p)
            if keep:
                self.pools[k] = keep
            else:
                del self.pools[k]

    def _find_pool(self, r: Request) -> Optional[_Pool]:
        key = kind_key(r.dg)
        K = r.dg.grid.K
        if K > self.capacity:
            raise ValueError(f"request {r.rid} has {K} elements, more than a pool's {self.capacity}")
        for p in self.pools.get(key, []):
            if p.room() >= K:
                return p
        need = self.capacity * pool_bytes_per_element(r.dg)
        if self.pool_bytes + need > self.budget:
            self._release_idle(need)
        if self.pool_bytes + need > self.budget:
            return None
        p = _Pool(key, r.dg, self.capacity, self.chunk, self.kind, self.max_tick_steps)
        self.pools_made += 1
        self.pools.setdefault(key, []).append(p)
        self.pool_bytes += p.nbytes
        self.peak_bytes = max(self.peak_bytes, self.pool_bytes)
        return p

    def run(self, requests: List[Request], realtime: bool = True) -> Stats:
        """Serve ``requests``.  With ``realtime`` a request becomes visible at
        its arrival time on the wall clock; otherwise all arrive at once."""
        import torch

        reqs = sorted(requests, key=lambda r: r.arrival)
        if not realtime:
            for r in reqs:
                r.arrival = 0.0
        queue: List[Request] = []
        done: List[Request] = []
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0  # noqa: E731
        nxt = 0
        ticks = 0
        while len(done) < len(reqs):
            tnow = now()
            while nxt < len(reqs) and reqs[nxt].arrival <= tnow:
                queue.append(reqs[nxt])
                nxt += 1
            waiting = []
            for r in queue:  # FIFO admission
                p = self._find_pool(r)
                if p is None:
                    waiting.append(r)
                else:
                    p.admit(r, now())
            queue = waiting
            busy = [p for ps in self.pools.values() for p in ps if p.placed]
            if not busy:
                if queue:
                    raise RuntimeError("a queued request fits no pool within the HBM budget")
                if nxt < len(reqs):
                    time.sleep(max(0.0, min(reqs[nxt].arrival - now(), 0.001)))
                continue
            for p in busy:
                p.tick(self.use_graphs)
            ticks += 1
            for p in busy:
                p.retire(now, done)
        torch.cuda.synchronize()
        span = now()
        lat = np.array([r.latency for r in done])
        st = Stats()
        st.requests = len(done)
        st.makespan_s = span
        total = self.retired_updates + sum(p.dof_stage_updates for ps in self.pools.values() for p in ps)
        st.dof_stage_per_s = total / span if span > 0 else 0.0
        st.p50_latency_s = float(np.percentile(lat, 50))
        st.p99_latency_s = float(np.percentile(lat, 99))
        st.mean_latency_s = float(lat.mean())
        st.peak_pool_bytes = int(self.peak_bytes)
        st.pools = self.pools_made
        st.ticks = ticks
        st.extra["dof_stage_updates"] = int(total)
        return st

    def close(self):
        for ps in self.pools.values():
            for p in ps:
                p.close()
        self.pools.clear()
        self.pool_bytes = 0

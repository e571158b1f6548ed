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
* a request's inputs may stay on the device: ``make`` builds its initial state
  and aux fields there at admission (on the copy stream), or ``q0`` / ``aux``
  are CUDA tensors; only the small geometry tables cross PCIe;
* a finished request returns what its client asks for: the whole state copied
  to pinned host memory (``result_mode="state"``), or its per-component
  MJ-weighted L2 norms computed on the device (``"norms"``, Ns doubles); its
  latency (arrival to result on the host) is recorded.

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
from typing import Callable, Dict, List, Optional, Tuple

import numpy as np

from . import _lib
from ._device import make_desc

__all__ = ["Request", "Server", "Stats", "kind_key", "pool_bytes_per_element", "pinned_array"]


def pinned_array(a: np.ndarray) -> np.ndarray:
    """A float64 copy of ``a`` in page-locked host memory (numpy view of a
    pinned torch tensor): inputs held this way are admitted by DMA."""
    import torch

    t = torch.empty(a.shape, dtype=torch.float64).pin_memory()
    out = t.numpy()
    out[...] = a
    return out

_KIND_STAGES = {"LSRK54": 5, "LSRK144": 14}
_GRID_FIELDS = ("K", "vertices", "periodic", "stacked")


@dataclass
class Request:
    rid: int
    dg: object                 # DGSEM spec of this instance
    q0: object                 # (Ns, K, Np) float64 initial state: numpy (host) or a CUDA tensor; None with make
    dt: float
    nsteps: int
    arrival: float = 0.0       # seconds after the stream starts
    keep_result: bool = True   # False: the result is copied out, then dropped
    # () -> (q0, aux): CUDA tensors (Ns, K, Np) and (naux, K, Np) or None, built
    # on the device at admission, on the server's copy stream
    make: Optional[Callable] = None
    aux: object = None         # aux fields (host array or CUDA tensor); default: dg.auxstate_host()
    result_mode: str = "state"  # "state": the final state; "norms": its per-component weighted L2 norms
    # filled by the server
    admitted: float = math.nan
    finished: float = math.nan
    result: Optional[np.ndarray] = None

    @property
    def latency(self) -> float:
        return self.finished - self.arrival

    @property
    def dof(self) -> int:
        return int(self.dg.law.numberofstates * self.dg.grid.K * self.dg.grid.cell.Np)


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


def _element_weights(dg, device):
    """Per-element Jacobians J (K) and per-node LGL weights w (Np) of a brick
    grid on the device: MJ = J (x) w (src/dgsem.jl:43-45), cached on the spec."""
    import torch

    jw = getattr(dg, "_serve_jw", None)
    if jw is None or jw[0].device != device:
        g, c = dg.grid, dg.grid.cell
        eidx = g.element_indices()
        J = np.ones(len(g))
        for d in range(g.dim):
            J = J * (np.diff(g.vertices[d])[eidx[:, d]] / 2)
        node = np.arange(c.Np)
        w = np.ones(c.Np)
        for d in range(g.dim):
            w = w * c.weights[(node // c.Nq ** d) % c.Nq]
        jw = (torch.as_tensor(J, device=device), torch.as_tensor(w, device=device))
        dg._serve_jw = jw
    return jw


class _Placed:
    __slots__ = ("req", "first", "K", "remaining", "desc", "keep", "aux")

    def __init__(self, req, first):
        self.req = req
        self.first = first
        self.K = req.dg.grid.K
        self.remaining = int(req.nsteps)
        self.desc, self.keep = make_desc(req.dg)
        if req.make is not None:
            self.aux = None  # built on the device at admission
        elif req.aux is not None:
            self.aux = req.aux
        else:
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


class _Staging:
    """Pinned host buffers for input copies, reused once their copy has run."""

    def __init__(self, limit_bytes: float = 8e9):
        self.bufs = []   # [tensor, event or None]
        self.limit = limit_bytes

    def get(self, n: int):
        import torch

        for b in self.bufs:
            if b[0].numel() >= n and (b[1] is None or b[1].query()):
                return b
        held = sum(b[0].numel() * 8 for b in self.bufs)
        if held + n * 8 > self.limit and self.bufs:
            # wait for the oldest copy, then replace its buffer if too small
            b = self.bufs.pop(0)
            if b[1] is not None:
                b[1].synchronize()
            if b[0].numel() < n:
                b = [torch.empty(n, dtype=torch.float64, pin_memory=True), None]
            self.bufs.append(b)
            return b
        b = [torch.empty(max(n, 1 << 20), dtype=torch.float64, pin_memory=True), None]
        self.bufs.append(b)
        return b


class _ResultArena:
    """One page-locked host arena for result copies, allocated once (page-
    locking costs a few hundred milliseconds per gigabyte, far too much per
    tick); a tick takes a first-fit region and ``poll`` gives it back after
    reading it.  When no region fits, the tick gets a buffer of its own."""

    def __init__(self, nbytes: float = 4e9):
        self.n = int(nbytes) // 8
        self.buf = None
        self.used = []  # sorted (start, end) in doubles
        self.fallbacks = 0

    def get(self, n: int):
        """(tensor view of n doubles, token for ``put``)."""
        import torch

        if self.buf is None and n <= self.n:
            self.buf = torch.empty(self.n, dtype=torch.float64, pin_memory=True)
        if self.buf is not None:
            start = 0
            for k, (a, b) in enumerate(self.used + [(self.n, self.n)]):
                if a - start >= n:
                    self.used.insert(k, (start, start + n))
                    return self.buf[start:start + n], (start, start + n)
                start = b
        self.fallbacks += 1
        return torch.empty(n, dtype=torch.float64, pin_memory=True), None

    def put(self, token):
        if token is not None:
            self.used.remove(token)


class _Pool:
    def __init__(self, key, template, capacity: int, chunk: int, kind: str, max_tick_steps: int,
                 copy_stream=None, staging=None, results=None):
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
        # inputs arrive on a copy stream, so admission never waits for the
        # pool's launches; the pool stream waits for those copies
        self.copy_stream = copy_stream if copy_stream is not None else torch.cuda.Stream(device=self.cuda)
        self.staging = staging if staging is not None else _Staging()
        self.results = results if results is not None else _ResultArena()
        self.pending = []
        self.q = torch.zeros((self.ns, self.capacity, self.Np), dtype=torch.float64, device=self.cuda)
        self.solver = Solver(kind, self, 1.0)
        # one time step per element (0 past the last request), a fixed device
        # pointer read by every stage, so captured graphs see updates
        self.dte = torch.zeros(self.capacity, dtype=torch.float64, device=self.cuda)
        # pinned host copies used in turn, so a refresh rarely waits for an
        # earlier transfer
        self.dte_pinned = [torch.zeros(self.capacity, dtype=torch.float64, pin_memory=True) for _ in range(4)]
        self._dt_events = [None] * 4
        self._dt_turn = 0
        _lib.check(_lib.lib().atb_solver_set_element_dt(
            self.solver.h, C.cast(C.c_void_p(self.dte.data_ptr()), _lib._DP)))
        self.placed: List[_Placed] = []
        self.used = 0
        self.graphs: Dict[Tuple[int, int], object] = {}
        self.nbytes = self.capacity * pool_bytes_per_element(template)
        self.dof_stage_updates = 0
        self.warm = set()
        self.dirty = True
        self.inflight = []       # (event, [(request, pinned view)], buffer) per tick
        self.inflight_prefix = 0
        self.naux = template.descriptor_fields()["naux"]
        self.host = {"dt": 0.0, "launch": 0.0, "results": 0.0, "compact": 0.0, "admit_make": 0.0,
                     "admit_place": 0.0}

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

    def _free_start(self) -> int:
        # past the used prefix and past every launch still in flight
        return max(self._launched(), self.inflight_prefix if self.inflight else 0)

    def room(self) -> int:
        return self.capacity - self._free_start()

    # admission ----------------------------------------------------------
    def _place(self, p: _Placed, stream, aux=None):
        """Geometry and aux fields of a placement; ``aux``: host array or CUDA
        tensor (default: the placement's host aux)."""
        import torch

        a = p.aux if aux is None else aux
        if isinstance(a, torch.Tensor):
            if a.dtype != torch.float64 or not a.is_contiguous():
                raise TypeError("device aux fields must be contiguous float64")
            ptr = C.cast(C.c_void_p(a.data_ptr()), _lib._DP) if a.numel() else None
        else:
            ptr = _lib.dptr(a) if a is not None and a.size else None
        _lib.check(_lib.lib().atb_op_place_instance(self._dev.h, p.first, C.byref(p.desc), ptr,
                                                    _lib.stream_ptr(stream)))

    def admit(self, r: Request, now: float):
        import torch

        # the new range starts past every launch in flight (the launched
        # prefix), so the copy stream writes nothing a running stage touches
        p = _Placed(r, self._free_start())
        K = p.K
        n = self.ns * K * self.Np
        dev_q0 = isinstance(r.q0, torch.Tensor) and r.q0.is_cuda
        if r.make is not None or dev_q0:
            # inputs on the device: built there now (make) or handed over as
            # CUDA tensors; device-to-device copies on the copy stream
            if r.make is None:
                # the caller's tensors were written on its current stream
                self.copy_stream.wait_stream(torch.cuda.current_stream())
            t0 = time.perf_counter()
            with torch.cuda.stream(self.copy_stream):
                if r.make is not None:
                    q0, aux = r.make()
                else:
                    q0 = r.q0
                    aux = r.aux if isinstance(r.aux, torch.Tensor) else None
                t1 = time.perf_counter()
                self._place(p, self.copy_stream, aux=aux.reshape(-1) if aux is not None else None)
                t2 = time.perf_counter()
                self.q[:, p.first:p.first + K].copy_(q0.reshape(self.ns, K, self.Np), non_blocking=True)
                ev = self.copy_stream.record_event()
            self.host["admit_make"] += t1 - t0
            self.host["admit_place"] += t2 - t1
            self.pending.append(ev)
            self.placed.append(p)
            self.used = p.first + K
            r.admitted = now
            self.dirty = True
            return
        src = None
        if isinstance(r.q0, np.ndarray) and r.q0.dtype == np.float64 and r.q0.flags.c_contiguous:
            t = torch.from_numpy(r.q0.reshape(-1))
            if t.is_pinned():
                src = t       # page-locked input: one DMA, no staging copy
        b = None
        if src is None:
            b = self.staging.get(n)
            src = b[0][:n]
            src.numpy()[:] = np.asarray(r.q0, dtype=np.float64).reshape(-1)
        with torch.cuda.stream(self.copy_stream):
            self._place(p, self.copy_stream)
            self.q[:, p.first:p.first + K].copy_(src.view(self.ns, K, self.Np), non_blocking=True)
            ev = self.copy_stream.record_event()
        if b is not None:
            b[1] = ev
        self.pending.append(ev)
        self.placed.append(p)
        self.used = p.first + K
        r.admitted = now
        self.dirty = True

    def _join_copies(self):
        for ev in self.pending:
            self.stream.wait_event(ev)
        self.pending = []

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

        i = self._dt_turn
        self._dt_turn = (i + 1) % len(self.dte_pinned)
        if self._dt_events[i] is not None:
            self._dt_events[i].synchronize()
        host = self.dte_pinned[i].numpy()
        host[:] = 0.0
        for p in self.placed:
            host[p.first:p.first + p.K] = p.req.dt
        self.dte.copy_(self.dte_pinned[i], non_blocking=True)
        self._dt_events[i] = torch.cuda.current_stream().record_event()
        self.dirty = False

    def tick(self, use_graphs: bool) -> int:
        """Launch S steps of every placed request, then (same stream) the
        copies of the requests that finish with them and the moves that
        close their gaps.  Nothing waits here; ``poll`` collects results."""
        import torch

        S = self.tick_steps()
        n = self._launched()
        self._join_copies()
        t0 = time.perf_counter()
        with torch.cuda.stream(self.stream):
            if self.dirty:
                self._refresh_dt()
            t1 = time.perf_counter()
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
                # capture_begin/end directly: the torch.cuda.graph context
                # manager also synchronises, collects garbage and empties the
                # allocator cache on every capture
                g = torch.cuda.CUDAGraph()
                g.capture_begin(capture_error_mode="thread_local")
                try:
                    self.solver.step(self.q, S, stream=self.stream)
                finally:
                    g.capture_end()
                self.graphs[key] = g
                g.replay()
        t2 = time.perf_counter()
        useful = sum(p.K for p in self.placed)
        self.dof_stage_updates += self.ns * useful * self.Np * _KIND_STAGES[self.kind] * S
        for p in self.placed:
            p.remaining -= S
        self.inflight_prefix = max(self.inflight_prefix, n)
        fin = [p for p in self.placed if p.remaining <= 0]
        outs = []
        buf = None
        if fin:
            size = lambda p: self.ns * p.K * self.Np if p.req.result_mode == "state" else self.ns  # noqa: E731
            tot = sum(size(p) for p in fin)
            buf, token = self.results.get(tot)
            o = 0
            with torch.cuda.stream(self.stream):
                for p in fin:
                    m = size(p)
                    if p.req.result_mode == "state":
                        v = buf[o:o + m].view(self.ns, p.K, self.Np)
                        v.copy_(self.q[:, p.first:p.first + p.K], non_blocking=True)
                    else:
                        # per-component sqrt(sum MJ q^2) on the device; Ns doubles to the host
                        J, w = _element_weights(p.req.dg, self.cuda)
                        x = self.q[:, p.first:p.first + p.K]
                        nrm = torch.stack([torch.dot(J, torch.mv(x[c] * x[c], w)) for c in range(self.ns)]).sqrt()
                        v = buf[o:o + m]
                        v.copy_(nrm, non_blocking=True)
                    outs.append((p.req, v))
                    o += m
            t3 = time.perf_counter()
            self._compact()
            self.host["results"] += t3 - t2
            self.host["compact"] += time.perf_counter() - t3
        ev = self.stream.record_event()
        self.host["dt"] += t1 - t0
        self.host["launch"] += t2 - t1
        self.inflight.append((ev, outs, (buf, token) if fin else None))
        return S

    def _compact(self):
        """Move the unfinished requests down over the finished ones (on the
        pool stream, after the result copies)."""
        import torch

        keep = [p for p in self.placed if p.remaining > 0]
        first = 0
        with torch.cuda.stream(self.stream):
            for p in keep:
                if p.first != first:
                    src = self.q[:, p.first:p.first + p.K].clone()
                    self.q[:, first:first + p.K].copy_(src)
                    scratch = None
                    if p.first - first < p.K:
                        nb = p.K * (8 * self.Np * self.naux + 56)
                        scratch = torch.empty(nb, dtype=torch.uint8, device=self.cuda)
                    _lib.check(_lib.lib().atb_op_move_instance(
                        self._dev.h, first, p.first, p.K,
                        C.c_void_p(scratch.data_ptr()) if scratch is not None else None,
                        _lib.stream_ptr(self.stream)))
                    p.first = first
                first += p.K
        self.placed = keep
        self.used = first
        self.dirty = True

    def busy(self) -> bool:
        return bool(self.inflight)

    def poll(self, now_fn, done: List[Request], wait: bool = False) -> int:
        """Collect the ticks that have completed (the oldest one waited for
        when ``wait``); returns how many completed."""
        k = 0
        while self.inflight:
            ev, outs, held = self.inflight[0]
            if not ev.query():
                if not (wait and k == 0):
                    break
                ev.synchronize()
            self.inflight.pop(0)
            t = now_fn()
            for r, v in outs:
                r.result = v.numpy().copy() if r.keep_result else None
                r.finished = t
                done.append(r)
            if held is not None:
                self.results.put(held[1])
            k += 1
        if not self.inflight:
            self.inflight_prefix = 0
        return k


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

    def __init__(self, hbm_budget_bytes: float = 150e9, capacity: Optional[int] = None, chunk: int = 256,
                 kind: str = "LSRK54", max_tick_steps: int = 16, use_graphs: bool = True,
                 pool_bytes: Optional[float] = None, max_pool_elements: int = 1 << 18,
                 result_bytes: float = 2e9):
        """``capacity``: elements per pool (fixed); otherwise a pool holds
        ``pool_bytes`` (default: an eighth of the budget) worth of elements of
        its kind, at most ``max_pool_elements`` and at least the request that
        opens it.  Inputs held in page-locked host memory (``pinned_array``)
        are copied by DMA straight from the caller's buffer, which must stay
        unchanged while the server runs; others go through pinned staging.
        ``result_bytes``: the page-locked host arena that results are copied
        into (allocated at the first result; a tick whose results do not fit
        gets a buffer of its own, which is slow to allocate)."""
        if kind not in _KIND_STAGES:
            raise ValueError("the server steps with LSRK54 or LSRK144")
        self.budget = float(hbm_budget_bytes)
        self.capacity = None if capacity is None else int(capacity)
        self.pool_budget = float(pool_bytes) if pool_bytes is not None else self.budget / 8
        self.max_pool_elements = int(max_pool_elements)
        self._keys = {}
        self.max_inflight = 2
        self._copy_stream = None
        self._staging = _Staging()
        self.result_bytes = float(result_bytes)
        self._results = _ResultArena(self.result_bytes)
        self.timers = {"admit": 0.0, "new_pool": 0.0, "tick": 0.0, "poll": 0.0, "release": 0.0}
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
                if not p.placed and not p.inflight and self.pool_bytes + need > self.budget:
                    self.pool_bytes -= p.nbytes
                    self.retired_updates += p.dof_stage_updates
                    p.close()
                else:
                    keep.append(p)
            if keep:
                self.pools[k] = keep
            else:
                del self.pools[k]

    def _pool_capacity(self, dg) -> int:
        if self.capacity is not None:
            return self.capacity
        fit = int(self.pool_budget // pool_bytes_per_element(dg))
        return max(dg.grid.K, min(self.max_pool_elements, fit))

    def _find_pool(self, r: Request) -> Optional[_Pool]:
        key = self._keys.get(id(r.dg))
        if key is None:
            key = self._keys[id(r.dg)] = kind_key(r.dg)
        K = r.dg.grid.K
        if self.capacity is not None and K > self.capacity:
            raise ValueError(f"request {r.rid} has {K} elements, more than a pool's {self.capacity}")
        for p in self.pools.get(key, []):
            if p.room() >= K:
                return p
        cap = self._pool_capacity(r.dg)
        need = cap * pool_bytes_per_element(r.dg)
        if self.pool_bytes + need > self.budget:
            t = time.perf_counter()
            self._release_idle(need)
            self.timers["release"] += time.perf_counter() - t
        if self.pool_bytes + need > self.budget:
            return None
        t = time.perf_counter()
        import torch

        if self._copy_stream is None:
            self._copy_stream = torch.cuda.Stream()
        p = _Pool(key, r.dg, cap, self.chunk, self.kind, self.max_tick_steps, self._copy_stream, self._staging,
                  self._results)
        self.timers["new_pool"] += time.perf_counter() - t
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
        # statistics cover this run only (pools persist across runs)
        self.retired_updates = 0
        self.timers = {k: 0.0 for k in self.timers}
        self.peak_bytes = self.pool_bytes
        self.pools_made = 0
        for ps in self.pools.values():
            for p in ps:
                p.dof_stage_updates = 0
                p.host = {k: 0.0 for k in p.host}
        queue: List[Request] = []
        done: List[Request] = []
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0  # noqa: E731
        nxt = 0
        ticks = 0
        pools = lambda: [p for ps in self.pools.values() for p in ps]  # noqa: E731
        while len(done) < len(reqs):
            tnow = now()
            while nxt < len(reqs) and reqs[nxt].arrival <= tnow:
                queue.append(reqs[nxt])
                nxt += 1
            waiting = []
            ta = time.perf_counter()
            # FIFO admission; once a request of a kind found no room in this
            # pass, requests of that kind at least as large wait without
            # another search (under overload the queue is long)
            blocked: Dict[tuple, int] = {}
            for r in queue:
                key = self._keys.get(id(r.dg))
                if key is None:
                    key = self._keys[id(r.dg)] = kind_key(r.dg)
                K = r.dg.grid.K
                if key in blocked and K >= blocked[key]:
                    waiting.append(r)
                    continue
                p = self._find_pool(r)
                if p is None:
                    blocked[key] = min(K, blocked.get(key, K))
                    waiting.append(r)
                else:
                    p.admit(r, now())
            self.timers["admit"] += time.perf_counter() - ta
            queue = waiting
            progressed = False
            tt = time.perf_counter()
            for p in pools():
                if p.placed and len(p.inflight) < self.max_inflight:
                    p.tick(self.use_graphs)
                    ticks += 1
                    progressed = True
            tr = time.perf_counter()
            self.timers["tick"] += tr - tt
            for p in pools():
                if p.inflight and p.poll(now, done):
                    progressed = True
            if not progressed:
                busy = [p for p in pools() if p.inflight]
                if busy:
                    busy[0].poll(now, done, wait=True)
                elif queue:
                    raise RuntimeError("a queued request fits no pool within the HBM budget")
                elif nxt < len(reqs):
                    time.sleep(max(0.0, min(reqs[nxt].arrival - now(), 0.001)))
            self.timers["poll"] += time.perf_counter() - tr
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
        st.extra["host_seconds"] = dict(self.timers)
        st.extra["result_arena_fallbacks"] = self._results.fallbacks
        for ps in self.pools.values():
            for p in ps:
                for k, v in p.host.items():
                    st.extra["host_seconds"]["tick_" + k] = st.extra["host_seconds"].get("tick_" + k, 0.0) + v
        return st

    def close(self):
        import torch

        for ps in self.pools.values():
            for p in ps:
                p.close()
        self.pools.clear()
        self.pool_bytes = 0
        torch.cuda.synchronize()
        self._results = _ResultArena(self.result_bytes)

"""Checkpoint / resume: a raw dump of the SoA state plus the solver scalars.

The reference has no checkpoint (its experiments write VTK snapshots only,
experiment/euler_gravity/risingbubble.jl:81-95); this is the raw form a run
needs to stop and continue: the ``Ns`` state components exactly as they sit in
device memory (float64, one contiguous ``K*Np`` array per component, node
fastest; the array's own shape, components first, is kept) and the solver's
clock, time step and last relaxation factor.  A solver rebuilt on the same
operators and time step, given the state back with ``resume``, continues the
run bit for bit.

File layout (little-endian)::

    8 bytes   b"ATBCKPT1"
    8 bytes   uint64 header length H
    H bytes   JSON header: {"shape": [Ns, ...], "ns", "n", "dtype": "float64",
                            "solver": {...} | null, "meta": {...}}
    ns*n*8    the components, one after another

``save`` copies a device state to the host (one synchronous copy per call);
``load`` returns a host array (numpy) or, with ``device``, a torch tensor.
"""
from __future__ import annotations

import json
import os
import struct

import numpy as np

MAGIC = b"ATBCKPT1"

__all__ = ["save", "load", "resume"]


def _host_array(q) -> np.ndarray:
    if isinstance(q, np.ndarray):
        a = q
    else:  # torch tensor (device or host)
        a = q.detach().cpu().numpy()
    a = np.asarray(a)
    if a.dtype != np.float64:
        raise TypeError(f"checkpoint states are float64 (got {a.dtype})")
    if a.ndim < 2:
        raise ValueError(f"expected a state with its components first, got shape {a.shape}")
    return np.ascontiguousarray(a)


def save(path: str, q, solver=None, meta: dict | None = None) -> dict:
    """Writes ``q`` (and ``solver.state()`` when given) to ``path``; the file
    is written to a temporary name first and renamed, so a reader never sees a
    partial checkpoint.  Returns the header."""
    a = _host_array(q)
    header = {"shape": [int(d) for d in a.shape], "ns": int(a.shape[0]), "n": int(a.size // a.shape[0]),
              "dtype": "float64",
              "solver": solver.state() if solver is not None else None, "meta": meta or {}}
    hb = json.dumps(header, sort_keys=True).encode()
    tmp = path + ".tmp"
    with open(tmp, "wb") as f:
        f.write(MAGIC)
        f.write(struct.pack("<Q", len(hb)))
        f.write(hb)
        f.write(a.astype("<f8", copy=False).tobytes())
    os.replace(tmp, path)
    return header


def load(path: str, device=None):
    """Reads a checkpoint: ``(q, header)``.  ``q`` is a numpy array, or a
    torch tensor on ``device`` when one is given."""
    with open(path, "rb") as f:
        magic = f.read(8)
        if magic != MAGIC:
            raise ValueError(f"{path}: not a checkpoint (magic {magic!r})")
        (hl,) = struct.unpack("<Q", f.read(8))
        header = json.loads(f.read(hl).decode())
        if header.get("dtype") != "float64":
            raise ValueError(f"{path}: unsupported dtype {header.get('dtype')}")
        ns, n = int(header["ns"]), int(header["n"])
        raw = f.read(ns * n * 8)
        if len(raw) != ns * n * 8:
            raise ValueError(f"{path}: truncated ({len(raw)} of {ns * n * 8} state bytes)")
    shape = tuple(header.get("shape") or (ns, n))
    q = np.frombuffer(raw, dtype="<f8").reshape(shape).astype(np.float64, copy=True)
    if device is not None:
        import torch
        q = torch.as_tensor(q, device=device).contiguous()
    return q, header


def resume(solver, header: dict):
    """Restores the solver scalars of a checkpoint header into ``solver``
    (built on the same operators).  The time step must match the solver's:
    ARK23 factors its implicit operator for one dt."""
    st = header.get("solver")
    if st is None:
        raise ValueError("the checkpoint holds no solver state")
    if st["kind"] != solver.kind:
        raise ValueError(f"checkpoint of a {st['kind']} solver, resuming a {solver.kind}")
    if st["dt"] != solver.dt:
        solver.dt = st["dt"]
    solver.set_state(st["time"], st["gamma"])

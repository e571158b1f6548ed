"""Helpers shared by the GPU parity tests: seeded smooth states and the
parity metric.

Parity metric (stated once, used everywhere): for every DOF of state
component c,  |gpu - oracle| <= tol * max(|oracle|, floor_c).

* Tendencies and general states: floor_c = max |oracle_c| over the field
  (relative per DOF, with the field's own magnitude as the floor for DOFs
  crossing zero).
* Solver states (``natural_floors``): floor_c is the component's physical
  scale -- max|rho| for mass, max|rho| * max wave speed for momentum (the
  acoustic momentum scale), max|rho e| for energy.  In a hydrostatically
  balanced atmosphere the momentum is a tiny residual of cancelling pressure
  and gravity forces; measured against its own magnitude, the reference's
  three flux-differencing schedules already disagree with each other at
  1e-10 after one step, and a 1-ulp change of the initial state moves the
  linear IMEX solution by 4e-4, so that scale says nothing about parity.
"""
from __future__ import annotations

import numpy as np

import atum_b200 as A


def rel_dof_error(g: np.ndarray, o: np.ndarray, floors=None) -> float:
    g = np.asarray(g, dtype=np.float64).reshape(o.shape[0], -1)
    o = np.asarray(o, dtype=np.float64).reshape(o.shape[0], -1)
    if floors is None:
        scale = np.max(np.abs(o), axis=1, keepdims=True)
    else:
        scale = np.asarray(floors, dtype=np.float64).reshape(-1, 1)
    scale = np.where(scale > 0, scale, 1.0)
    den = np.maximum(np.abs(o), scale)
    return float(np.max(np.abs(g - o) / den))


def natural_floors(dg, o: np.ndarray) -> np.ndarray:
    """Physical per-component scales of a state (see the module docstring)."""
    law = dg.law
    o = np.asarray(o).reshape(o.shape[0], -1)
    ns = o.shape[0]
    fl = np.max(np.abs(o), axis=1)
    if isinstance(law, A.AdvectionLaw):
        return fl
    dim = law.dim
    rho = o[0]
    if isinstance(law, A.ShallowWaterLaw):
        c = np.sqrt(law.grav * np.abs(rho))
    elif isinstance(law, A.LinearEulerGravityLaw):
        aux = dg.auxstate_host().reshape(law.naux, -1)
        c = np.sqrt(law.gamma * aux[dim + 2] / aux[dim + 1])
    else:
        Phi = dg.auxstate_host().reshape(law.naux, -1)[0] if isinstance(law, A.EulerGravityLaw) else 0.0
        ke = sum(o[1 + d] ** 2 for d in range(dim)) / (2 * rho)
        p = (law.gamma - 1) * (o[dim + 1] - ke - rho * Phi)
        c = np.sqrt(law.gamma * np.abs(p / rho))
    u = np.sqrt(sum((o[1 + d] / rho) ** 2 for d in range(dim)))
    mom = np.max(np.abs(rho)) * np.max(c + u)
    for d in range(dim):
        fl[1 + d] = max(fl[1 + d], mom)
    return fl[:ns]


def smooth(x, rng, amp=1.0, modes=3):
    """Sum of a few random periodic-ish sine modes on the node coordinates."""
    dim = x.shape[0]
    out = np.zeros(x.shape[1:])
    for _ in range(modes):
        k = rng.uniform(0.5, 2.0, size=dim)
        ph = rng.uniform(0, 2 * np.pi)
        arg = ph + sum(k[d] * np.pi * x[d] / max(1.0, float(np.ptp(x[d]))) for d in range(dim))
        out += np.sin(arg)
    return amp * out / modes


def random_state(dg, seed=1234):
    rng = np.random.default_rng(seed)
    law = dg.law
    x = dg.grid.points()
    dim = law.dim
    if isinstance(law, A.AdvectionLaw):
        return np.ascontiguousarray(np.stack([2 + smooth(x, rng)]))
    if isinstance(law, A.ShallowWaterLaw):
        h = 2 + 0.3 * smooth(x, rng)
        if law.sw_topography:
            h = h - dg.auxstate_host()[0] * 0.0
        comps = [h] + [h * 0.3 * smooth(x, rng) for _ in range(dim)] + [h * smooth(x, rng)]
        return np.ascontiguousarray(np.stack(comps))
    if isinstance(law, A.LinearEulerGravityLaw):
        aux = dg.auxstate_host()
        rho_ref, p_ref, Phi = aux[dim + 1], aux[dim + 2], aux[0]
        rho = rho_ref * (1 + 0.05 * smooth(x, rng))
        m = [rho * 20.0 * smooth(x, rng) for _ in range(dim)]
        rhoe = law.reference_rhoe(p_ref * (1 + 0.05 * smooth(x, rng)), rho, Phi)
        return np.ascontiguousarray(np.stack([rho] + m + [rhoe]))
    if isinstance(law, A.EulerGravityLaw):
        aux = dg.auxstate_host()
        Phi = aux[0]
        if law.has_reference:
            rho0, p0 = aux[dim + 1], aux[dim + 2]
        else:
            rho0, p0 = 1.0 + 0 * Phi, 1.0 + 0 * Phi
        rho = rho0 * (1 + 0.05 * smooth(x, rng))
        u = [0.3 * smooth(x, rng) for _ in range(dim)]
        p = p0 * (1 + 0.05 * smooth(x, rng))
        m = [rho * ui for ui in u]
        return np.ascontiguousarray(np.stack([rho] + m + [law.energy(rho, m, p, Phi)]))
    # Euler
    rho = 1.5 + 0.3 * smooth(x, rng)
    u = [0.4 * smooth(x, rng) for _ in range(dim)]
    p = 1.2 + 0.2 * smooth(x, rng)
    m = [rho * ui for ui in u]
    return np.ascontiguousarray(np.stack([rho] + m + [law.energy(rho, m, p)]))


def to_dev(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda").contiguous()


def to_host(t):
    return t.detach().cpu().numpy()

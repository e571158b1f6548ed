"""Problem setups of the reference's integration tests, restated on the host
API (numpy initial conditions).  The benchmark configurations (vortex C1,
rising bubble, shallow water) live in the package (``atum_b200.workloads``)
and are re-exported here.

Each builder returns a ``Case``: the DGSEM spec(s), the initial state, dt, end
time, solver kind and the exact solution (when the reference has one).  The
same Case drives the CPU oracle and the GPU library, so parity tests compare
the two on identical inputs.
"""
from __future__ import annotations

import math
import numpy as np

import atum_b200 as A
from atum_b200.workloads import (Case, _vec, _pack, vortex_c1, bubble_3d, sw_fplane,  # noqa: F401
                                 bubble_reference as _bubble_reference)


# ------------------------------------------------------------ advection
def advection_wave(dim, N=4, K=5, form="weak"):
    """test/advection/wave_{1,2,3}d.jl"""
    law = A.AdvectionLaw(dim)
    cell = A.LobattoCell(*([N + 1] * dim))
    v1d = _vec(-1.0, 1.0, K)
    grid = A.brickgrid(cell, (v1d,) * dim, periodic=(True,) * dim)
    vf = A.WeakForm() if form == "weak" else A.FluxDifferencingForm(A.CentralFlux())
    dg = A.DGSEM(law=law, grid=grid, volume_form=vf, surface_numericalflux=A.RusanovFlux())
    cfl = {1: 0.5, 2: 0.25, 3: 0.25}[dim]
    dt = cfl * (v1d[1] - v1d[0]) / N / math.sqrt(dim)

    def wave(x, t):
        return _pack(2 + np.sin(np.pi * (np.sum(x, axis=0) - dim * t)))

    x = grid.points()
    return Case(f"advection_wave_{dim}d_{form}", dg, wave(x, 0.0), dt, 0.7, exact=lambda t: wave(x, t))


# ----------------------------------------------------------------- euler
def euler_wave(dim, N=4, K=5, form="weak", one_step=None):
    """test/euler/wave_{1,2,3}d.jl (3-D: a single LSRK54 step, timeend = dt)"""
    law = A.EulerLaw(dim)
    cell = A.LobattoCell(*([N + 1] * dim))
    v1d = _vec(-1.0, 1.0, K)
    grid = A.brickgrid(cell, (v1d,) * dim, periodic=(True,) * dim)
    vf = A.WeakForm() if form == "weak" else A.FluxDifferencingForm(A.EntropyConservativeFlux())
    dg = A.DGSEM(law=law, grid=grid, volume_form=vf, surface_numericalflux=A.RusanovFlux())
    cfl = 0.5 if dim == 1 else 0.25
    dt = cfl * (v1d[1] - v1d[0]) / N / law.soundspeed(1.0, 1.0)
    timeend = 0.7
    if one_step if one_step is not None else dim == 3:
        timeend = dt

    def wave(x, t):
        rho = 2 + np.sin(np.pi * (np.sum(x, axis=0) - dim * t))
        rhou = [rho * 1.0 for _ in range(dim)]
        rhoe = law.energy(rho, rhou, 1.0)
        return _pack(rho, *rhou, rhoe)

    x = grid.points()
    return Case(f"euler_wave_{dim}d_{form}", dg, wave(x, 0.0), dt, timeend, exact=lambda t: wave(x, t))


def isentropic_vortex(N=4, K=5, form="weak"):
    """test/euler/isentropicvortex.jl: [0,20]x[-5,5], centre (5,0), u0=(1,0)."""
    law = A.EulerLaw(2)
    cell = A.LobattoCell(N + 1, N + 1)
    vx, vy = _vec(0.0, 20.0, K), _vec(-5.0, 5.0, K)
    grid = A.brickgrid(cell, (vx, vy), periodic=(True, True))
    vf = A.WeakForm() if form == "weak" else A.FluxDifferencingForm(A.EntropyConservativeFlux())
    dg = A.DGSEM(law=law, grid=grid, volume_form=vf, surface_numericalflux=A.RusanovFlux())
    dt = 0.25 * (vy[1] - vy[0]) / N
    g = law.gamma

    def vortex(x, t):
        r0 = x[0] - 5.0 - 1.0 * t
        r1 = x[1] - 0.0 - 0.0 * t
        f = 5.0 * np.exp(1 - (r0 * r0 + r1 * r1))
        rho = (1 - (g - 1) * f ** 2 / (16 * g * np.pi ** 2)) ** (1 / (g - 1))
        u0 = 1.0 + f / (2 * np.pi) * (-r1)
        u1 = 0.0 + f / (2 * np.pi) * r0
        rhou = [rho * u0, rho * u1]
        p = rho ** g
        return _pack(rho, *rhou, law.energy(rho, rhou, p))

    x = grid.points()
    return Case(f"isentropic_vortex_{form}_K{K}", dg, vortex(x, 0.0), dt, 5.0, exact=lambda t: vortex(x, t))


# ------------------------------------------------------ entropy conservation
def square_1d(lawname, N=4, K=5):
    """test/{advection,euler,shallow_water}/entropy_conservation_1d.jl"""
    cell = A.LobattoCell(N + 1)
    v1d = _vec(-1.0, 1.0, K)
    grid = A.brickgrid(cell, (v1d,), periodic=(True,))
    x = grid.points()
    rho = np.where(np.abs(x[0]) < 0.5, 2.0, 1.0)
    if lawname == "advection":
        law = A.AdvectionLaw(1)
        flux = A.CentralFlux()
        q0 = _pack(rho)
        dt = 0.25 * A.min_node_distance(grid) / 1.0
    elif lawname == "euler":
        law = A.EulerLaw(1)
        flux = A.EntropyConservativeFlux()
        q0 = _pack(rho, rho * 1.0, law.energy(rho, [rho * 1.0], 1.0))
        dt = 0.5 * A.min_node_distance(grid) / law.soundspeed(1.0, 1.0)
    else:
        law = A.ShallowWaterLaw(1)
        flux = A.EntropyConservativeFlux()
        q0 = _pack(rho, rho * 1.0, np.zeros_like(rho))
        dt = 0.25 * A.min_node_distance(grid) / math.sqrt(law.grav)
    dg = A.DGSEM(law=law, grid=grid, volume_form=A.FluxDifferencingForm(flux), surface_numericalflux=flux)
    return Case(f"entropy_{lawname}_1d", dg, q0, dt, 5.0, solver="RLSRK54")


# ------------------------------------------------------------------- IMEX
def imex_advection_2d(N=4, K=5, form="weak", split_rhs=True):
    """test/advection/imex_wave_2d.jl"""
    u = (1.0, 0.3)
    law = A.AdvectionLaw(2, u, problem=A.InflowZero())
    cell = A.LobattoCell(N + 1, N + 1)
    v1d = _vec(-1.0, 1.0, K)
    grid = A.brickgrid(cell, (v1d, v1d), periodic=(True, False), ordering="stacked")
    vf = A.WeakForm() if form == "weak" else A.FluxDifferencingForm(A.CentralFlux())
    dg = A.DGSEM(law=law, grid=grid, volume_form=vf, surface_numericalflux=A.RusanovFlux(),
                 directions=(1,) if split_rhs else (1, 2))
    lindg = A.DGSEM(law=law, grid=grid, volume_form=vf, surface_numericalflux=A.RusanovFlux(), directions=(2,))
    dt = 0.25 * (v1d[1] - v1d[0]) / N / math.hypot(*u)

    def wave(x, t):
        mu = 1.0 / 5.0
        r = [np.mod(x[d] - u[d] * t + 1, 2) - 1 for d in range(2)]
        return _pack(5 * np.exp(-(r[0] ** 2 + r[1] ** 2) / mu ** 2))

    x = grid.points()
    return Case(f"imex_advection_{form}_{'split' if split_rhs else 'unsplit'}", dg, wave(x, 0.0), dt, 1.0,
                solver="ARK23", lindg=lindg, split_rhs=split_rhs, exact=lambda t: wave(x, t))


def _linear_test_reference(law, x):
    """referencestate of test/euler_gravity/linear.jl:20-43 (constant theta)."""
    z = x[law.dim - 1]
    Phi = law.grav * z
    cv_d = 719.0
    cp_d = law.gamma * cv_d
    R_d = cp_d - cv_d
    theta = 300.0
    p0 = 1e5
    pi_exner = 1 - law.grav / (cp_d * theta) * z
    rho = p0 / (R_d * theta) * pi_exner ** (cv_d / R_d)
    T = theta * pi_exner
    rhoe = rho * (cv_d * T + Phi)
    p = law.pressure(rho, [np.zeros_like(rho)] * law.dim, rhoe, Phi)
    return rho, p


def linear_euler_gravity(N=4, K=5):
    """test/euler_gravity/linear.jl: ARK23(nothing, dg), CFL 100, 5 days."""
    parent = A.EulerGravityLaw(2, problem=A.ReflectiveWall(referencestate=_linear_test_reference))
    law = A.LinearEulerGravityLaw(parent)
    cell = A.LobattoCell(N + 1, N + 1)
    vx, vz = _vec(0.0, 10e3, K), _vec(0.0, 10e3, K)
    grid = A.brickgrid(cell, (vx, vz), periodic=(True, False), ordering="stacked")
    dg_nl = A.DGSEM(law=parent, grid=grid, surface_numericalflux=A.RusanovFlux())
    dg = A.DGSEM(law=law, grid=grid, surface_numericalflux=A.RusanovFlux(), auxstate=dg_nl.auxstate_host(),
                 directions=(2,))
    dz = A.min_node_distance(grid, dims=(2,))
    dt = 100.0 * dz / 330
    aux = dg.auxstate_host()
    rho, p, Phi = aux[3], aux[4], aux[0]
    q0 = _pack(rho, np.zeros_like(rho), np.zeros_like(rho), law.reference_rhoe(p, rho, Phi))
    return Case(f"linear_euler_gravity_K{K}", None, q0, dt, 5 * 24 * 60 * 60.0, solver="ARK23", lindg=dg,
                adjust_final=False, extra={"qref": q0.copy()})


def goldens():
    import json
    import os
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_goldens.json")) as f:
        return json.load(f)


def golden(key, form, level=1):
    for v in goldens()[key]["values"]:
        if v["form"] == form and v["level"] == level:
            return v["value"]
    raise KeyError((key, form, level))



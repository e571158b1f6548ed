"""Problem setups of the reference's integration tests, restated on the host
API (numpy initial conditions), plus the benchmark configurations.

Each builder returns a ``Case``: the DGSEM spec(s), the initial state, dt, end
time, solver kind and the exact solution (when the reference has one).  The
same Case drives the CPU oracle and the GPU library, so parity tests compare
the two on identical inputs.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable, Optional

import numpy as np

import atum_b200 as A


@dataclass
class Case:
    name: str
    dg: object
    q0: np.ndarray
    dt: float
    timeend: float
    solver: str = "LSRK54"
    lindg: object = None
    split_rhs: bool = True
    adjust_final: bool = True
    exact: Optional[Callable] = None
    extra: dict = field(default_factory=dict)


def _vec(lo, hi, K):
    # Julia range(lo, stop=hi, length=K+1): values lo + i*(hi-lo)/K
    return np.array([lo + (hi - lo) * i / K for i in range(K + 1)], dtype=np.float64)


def _pack(*comps):
    return np.ascontiguousarray(np.stack([np.broadcast_to(c, comps[0].shape) for c in comps]))


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


def vortex_c1(N=3, K=8, steps=100, vflux="ec", precision="fp64"):
    """Plain-method config: 2-D Euler isentropic vortex on periodic [-5,5]^2,
    8x8 elements, N=3, rho=1, u=v=1, p=1, gamma=1.4, strength 5 at the origin,
    EC volume flux, Rusanov surface flux, LSRK54, dt = 0.3 dx / N, 100 fixed
    steps; analytic solution wrapped periodically (minimum image)."""
    law = A.EulerLaw(2)
    cell = A.LobattoCell(N + 1, N + 1)
    v = _vec(-5.0, 5.0, K)
    grid = A.brickgrid(cell, (v, v), periodic=(True, True))
    vf = A.FluxDifferencingForm(A.EntropyConservativeFlux() if vflux == "ec" else A.KennedyGruberFlux())
    dg = A.DGSEM(law=law, grid=grid, volume_form=vf, surface_numericalflux=A.RusanovFlux(), precision=precision)
    dx = v[1] - v[0]
    g = law.gamma

    def vortex(x, t):
        r0 = x[0] - 1.0 * t
        r1 = x[1] - 1.0 * t
        r0 = r0 - 10.0 * np.round(r0 / 10.0)
        r1 = r1 - 10.0 * np.round(r1 / 10.0)
        f = 5.0 * np.exp(1 - (r0 * r0 + r1 * r1))
        rho = (1 - (g - 1) * f ** 2 / (16 * g * np.pi ** 2)) ** (1 / (g - 1))
        u0 = 1.0 + f / (2 * np.pi) * (-r1)
        u1 = 1.0 + f / (2 * np.pi) * r0
        rhou = [rho * u0, rho * u1]
        return _pack(rho, *rhou, law.energy(rho, rhou, rho ** g))

    x = grid.points()
    q0 = vortex(x, 0.0)
    # CFL 0.3 in the reference tests' form dt = cfl * dx / N / speed, with the
    # largest wave speed |u| + c of the initial state
    rho, m, E = q0[0], q0[1:3], q0[3]
    p = law.pressure(rho, list(m), E)
    lam = float(np.max(np.sqrt(m[0] ** 2 + m[1] ** 2) / rho + np.sqrt(g * p / rho)))
    dt = 0.3 * dx / N / lam
    return Case("vortex_c1", dg, q0, dt, steps * dt, exact=lambda t: vortex(x, t), extra={"steps": steps})


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


# --------------------------------------------------- 3-D Euler + gravity bubble
def _bubble_reference(law, x):
    """Constant potential temperature (theta0 = 300 K) hydrostatic background."""
    z = x[law.dim - 1]
    cv_d = 719.0
    cp_d = law.gamma * cv_d
    R_d = cp_d - cv_d
    theta = 300.0
    p0 = 1e5
    pi_exner = 1 - law.grav / (cp_d * theta) * z
    rho = p0 / (R_d * theta) * pi_exner ** (cv_d / R_d)
    p = p0 * pi_exner ** (cp_d / R_d)
    return rho, p


def bubble_3d(N=4, K=16, L=10e3, imex=True, steps=200, dt=None, precision="fp64", vflux="ec"):
    """3-D rising warm bubble: box L^3, K^3 hexahedra, order N; constant-theta
    hydrostatic background (theta0 = 300 K, g = 9.81), +2 K Gaussian theta
    perturbation of 2 km radius centred 2 km above ground; periodic laterally,
    reflective walls top/bottom.  IMEX ARK23 (split_rhs = false) with the
    vertical acoustic terms implicit through the banded column solve, or
    explicit LSRK54 at small dt."""
    problem = A.ReflectiveWall(referencestate=_bubble_reference)
    law = A.EulerGravityLaw(3, grav=9.81, problem=problem)
    cell = A.LobattoCell(N + 1, N + 1, N + 1)
    v = _vec(0.0, L, K)
    grid = A.brickgrid(cell, (v, v, v), periodic=(True, True, False), ordering="stacked")
    vf = A.FluxDifferencingForm(A.EntropyConservativeFlux() if vflux == "ec" else A.KennedyGruberFlux())
    dg = A.DGSEM(law=law, grid=grid, volume_form=vf, surface_numericalflux=A.RusanovFlux(), precision=precision)
    x = grid.points()
    aux = dg.auxstate_host()
    Phi = aux[0]
    cv_d = 719.0
    cp_d = law.gamma * cv_d
    R_d = cp_d - cv_d
    r = np.sqrt((x[0] - L / 2) ** 2 + (x[1] - L / 2) ** 2 + (x[2] - 2000.0) ** 2)
    dtheta = 2.0 * np.exp(-(r / 2000.0) ** 2)
    theta = 300.0 + dtheta
    z = x[2]
    # keep the hydrostatic pressure, perturb temperature: rho = p / (R T)
    pi_exner = 1 - law.grav / (cp_d * 300.0) * z
    p = 1e5 * pi_exner ** (cp_d / R_d)
    T = theta * pi_exner
    rho = p / (R_d * T)
    zero = np.zeros_like(rho)
    rhoe = law.energy(rho, [zero] * 3, p, Phi)
    q0 = _pack(rho, zero, zero, zero, rhoe)
    dz = A.min_node_distance(grid, dims=(3,))
    if imex:
        lin = A.LinearEulerGravityLaw(law)
        # the implicit vertical operator and its banded solve stay FP64 in
        # every precision form
        lindg = A.DGSEM(law=lin, grid=grid, surface_numericalflux=A.RusanovFlux(), auxstate=aux, directions=(3,))
        # the box is isotropic: the explicit part's horizontal acoustic CFL sets dt
        dt = dt if dt is not None else 0.25 * dz / 340.0
        return Case("bubble_3d_imex", dg, q0, dt, steps * dt, solver="ARK23", lindg=lindg, split_rhs=False,
                    adjust_final=False, extra={"steps": steps})
    dt = dt if dt is not None else 0.3 * dz / 340.0
    return Case("bubble_3d_lsrk", dg, q0, dt, steps * dt, extra={"steps": steps})


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


# ------------------------------------------------------ shallow water, C3
def sw_fplane(N=4, K=32, L=1.0e6, H=100.0, seed=20261203, lake_at_rest=False, precision="fp64", f=1e-4,
              steps=500):
    """Rotating shallow water (f-plane, g = 9.81) on a periodic square of K x K
    elements, order N; smooth random bottom topography (sum of 8 Gaussians,
    amplitude <= 10% of the mean depth H) and seeded random height
    perturbations (amplitude 1 m, wavelengths 4-16 elements).  EC volume flux
    with the well-balanced bathymetry terms, Rusanov surface flux, LSRK54."""
    rng = np.random.default_rng(seed)
    cell = A.LobattoCell(N + 1, N + 1)
    v = _vec(0.0, L, K)
    grid = A.brickgrid(cell, (v, v), periodic=(True, True))
    g = 9.81
    cx, cy = rng.uniform(0, L, 8), rng.uniform(0, L, 8)
    amp = rng.uniform(-0.1 * H, 0.1 * H, 8) / 2
    wid = rng.uniform(0.05 * L, 0.15 * L, 8)

    def bath(x):
        b = np.zeros(x.shape[1:])
        gx, gy = np.zeros_like(b), np.zeros_like(b)
        for i in range(8):
            dx = (x[0] - cx[i] + L / 2) % L - L / 2
            dy = (x[1] - cy[i] + L / 2) % L - L / 2
            e = amp[i] * np.exp(-(dx * dx + dy * dy) / wid[i] ** 2)
            b += e
            gx += -2 * dx / wid[i] ** 2 * e
            gy += -2 * dy / wid[i] ** 2 * e
        return b, [gx, gy]

    law = A.ShallowWaterLaw(2, grav=g, topography=True, problem=A.Coriolis((0.0, 0.0, f)))
    law.bathymetry = bath
    dg = A.DGSEM(law=law, grid=grid, volume_form=A.FluxDifferencingForm(A.EntropyConservativeFlux()),
                 surface_numericalflux=A.RusanovFlux(), precision=precision)
    x = grid.points()
    b = dg.auxstate_host()[0]
    eta = np.zeros_like(b)
    if not lake_at_rest:
        for _ in range(6):
            wl = rng.uniform(4, 16) * (L / K)
            th = rng.uniform(0, 2 * np.pi)
            kx, ky = 2 * np.pi / wl * np.cos(th), 2 * np.pi / wl * np.sin(th)
            # periodic: round the wavenumber to the box
            kx = 2 * np.pi * np.round(kx * L / (2 * np.pi)) / L
            ky = 2 * np.pi * np.round(ky * L / (2 * np.pi)) / L
            eta += np.sin(kx * x[0] + ky * x[1] + rng.uniform(0, 2 * np.pi))
        eta *= 1.0 / np.max(np.abs(eta))
    h = H - b + eta
    z = np.zeros_like(h)
    q0 = _pack(h, z, z, h * 0.0)
    dx = L / K
    dt = 0.3 * dx / N / (np.sqrt(g * np.max(h)))
    return Case("sw_fplane", dg, q0, dt, steps * dt, extra={"steps": steps})

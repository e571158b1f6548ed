"""Workload builders of the benchmark configurations: seeded synthetic
initial states on brick grids, restated from the reference's test and
experiment setups (test/euler/isentropicvortex.jl:16-32,
test/euler_gravity/linear.jl:20-43, experiment/euler_gravity/risingbubble.jl:10-15).

Each builder returns a ``Case``: the DGSEM spec(s), the initial state, dt, end
time, solver kind and the exact solution (when there is one).  ``bench.py``
times these workloads; the tests drive the same builders through the CUDA
library and the CPU oracle.

* ``vortex_c1``   2-D Euler isentropic vortex, 8x8 elements, N=3, LSRK54
* ``bubble_3d``   3-D Euler-gravity rising bubble, 16^3 elements, N=4, IMEX ARK23
* ``sw_fplane``   rotating shallow water with bathymetry, 32^2 elements, N=4
* ``sphere_acoustic_wave``  3-D Euler-gravity acoustic wave on a cubed-sphere
  shell (experiment/euler_gravity/acousticwave.jl), N=5, KH=10, KV=5, IMEX ARK23
* ``sphere_zonal_flow``     isothermal zonal flow on a small-planet shell
  (experiment/euler_gravity/isothermal_zonal_flow.jl), N=3, KH=KV=5, IMEX ARK23
* ``sphere_baroclinic_wave``  deep-atmosphere baroclinic wave on a rotating
  Earth-radius shell (experiment/euler_gravity/baroclinicwave.jl), N=3, KH=8,
  KV=4, IMEX ARK23
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable, Optional

import numpy as np

from .dgsem import DGSEM
from .laws import (EulerLaw, EulerGravityLaw, LinearEulerGravityLaw, ShallowWaterLaw, ReflectiveWall, Coriolis,
                   RusanovFlux, EntropyConservativeFlux, KennedyGruberFlux, FluxDifferencingForm)
from .cell import LobattoCell, brickgrid, min_node_distance
from .cubedsphere import cubedspheregrid


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



def vortex_c1(N=3, K=8, steps=100, vflux="ec", precision="fp64"):
    """Plain-method config: 2-D Euler isentropic vortex on periodic [-5,5]^2,
    8x8 elements, N=3, rho=1, u=v=1, p=1, gamma=1.4, strength 5 at the origin,
    EC volume flux, Rusanov surface flux, LSRK54, dt = 0.3 dx / N, 100 fixed
    steps; analytic solution wrapped periodically (minimum image)."""
    law = EulerLaw(2)
    cell = LobattoCell(N + 1, N + 1)
    v = _vec(-5.0, 5.0, K)
    grid = brickgrid(cell, (v, v), periodic=(True, True))
    vf = FluxDifferencingForm(EntropyConservativeFlux() if vflux == "ec" else KennedyGruberFlux())
    dg = DGSEM(law=law, grid=grid, volume_form=vf, surface_numericalflux=RusanovFlux(), precision=precision)
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


# --------------------------------------------------- 3-D Euler + gravity bubble
def bubble_reference(law, x):
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


def bubble_3d(N=4, K=16, L=10e3, imex=True, steps=200, dt=None, precision="fp64", vflux="ec",
              fd_kernel="per_dir"):
    """3-D rising warm bubble: box L^3, K^3 hexahedra (K an int) or Kx x Ky x Kz
    (K a 3-tuple), order N; constant-theta
    hydrostatic background (theta0 = 300 K, g = 9.81), +2 K Gaussian theta
    perturbation of 2 km radius centred 2 km above ground; periodic laterally,
    reflective walls top/bottom.  IMEX ARK23 (split_rhs = false) with the
    vertical acoustic terms implicit through the banded column solve, or
    explicit LSRK54 at small dt.  ``fd_kernel`` picks the flux-differencing
    schedule (``per_dir``, ``per_dir_symmetric``, ``naive``)."""
    problem = ReflectiveWall(referencestate=bubble_reference)
    law = EulerGravityLaw(3, grav=9.81, problem=problem)
    cell = LobattoCell(N + 1, N + 1, N + 1)
    Ks = tuple(K) if isinstance(K, (tuple, list)) else (K, K, K)
    grid = brickgrid(cell, tuple(_vec(0.0, L, k) for k in Ks), periodic=(True, True, False), ordering="stacked")
    vf = FluxDifferencingForm(EntropyConservativeFlux() if vflux == "ec" else KennedyGruberFlux(), fd_kernel)
    dg = DGSEM(law=law, grid=grid, volume_form=vf, surface_numericalflux=RusanovFlux(), precision=precision)
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
    dz = min_node_distance(grid, dims=(3,))
    if imex:
        lin = LinearEulerGravityLaw(law)
        # the implicit vertical operator and its banded solve stay FP64 in
        # every precision form
        lindg = DGSEM(law=lin, grid=grid, surface_numericalflux=RusanovFlux(), auxstate=aux, directions=(3,))
        # the box is isotropic: the explicit part's horizontal acoustic CFL sets dt
        dt = dt if dt is not None else 0.25 * dz / 340.0
        return Case("bubble_3d_imex", dg, q0, dt, steps * dt, solver="ARK23", lindg=lindg, split_rhs=False,
                    adjust_final=False, extra={"steps": steps})
    dt = dt if dt is not None else 0.3 * dz / 340.0
    return Case("bubble_3d_lsrk", dg, q0, dt, steps * dt, extra={"steps": steps})


# ------------------------------------------------ cubed-sphere shells
_EARTH_RADIUS = 6.371229e6


def _isothermal_reference(a):
    """Isothermal (T_ref = 300 K) hydrostatic reference state above radius a
    (acousticwave.jl:25-41, isothermal_zonal_flow.jl:42-61)."""
    def ref(law, x):
        r = np.sqrt(np.sum(x * x, axis=0))
        z = r - a
        cv_d = 719.0
        R_d = law.gamma * cv_d - cv_d
        T_ref = 300.0
        delta = law.grav / (R_d * T_ref)
        rho_s = 1e5 / (T_ref * R_d)
        rho = rho_s * np.exp(-delta * z)
        return rho, rho * R_d * T_ref
    return ref


def _sphere_case(name, law, grid, q0, dt, steps, imex, vflux):
    vf = FluxDifferencingForm(EntropyConservativeFlux() if vflux == "ec" else KennedyGruberFlux())
    dg = DGSEM(law=law, grid=grid, volume_form=vf, surface_numericalflux=RusanovFlux())
    if imex:
        lindg = DGSEM(law=LinearEulerGravityLaw(law), grid=grid, surface_numericalflux=RusanovFlux(),
                      auxstate=dg.auxstate_host(), directions=(3,))
        return Case(name, dg, q0(dg), dt, steps * dt, solver="ARK23", lindg=lindg, split_rhs=False,
                    adjust_final=False, extra={"steps": steps})
    return Case(name, dg, q0(dg), dt, steps * dt, adjust_final=False, extra={"steps": steps})


def sphere_acoustic_wave(N=5, KH=10, KV=5, steps=10, imex=True, dt=None, vflux="ec"):
    """Acoustic wave on an Earth-radius shell 10 km deep (cubed sphere, KH x KH
    elements per panel, KV layers, order N): isothermal atmosphere at rest
    with a pressure perturbation of 100 Pa x (1 + cos(pi beta))/2 x sin(pi z/H)
    around (lon, lat) = (0, 0), beta = min(1, 3 * great-circle angle);
    reflective inner and outer spheres; EC volume flux, Rusanov surface flux,
    IMEX ARK23 (split_rhs = false) with dt = 100 (H/KV) / 330 / N^2
    (acousticwave.jl:43-111)."""
    a, H = _EARTH_RADIUS, 10e3
    law = EulerGravityLaw(3, sphere=True, problem=ReflectiveWall(referencestate=_isothermal_reference(a)))
    cell = LobattoCell(N + 1, N + 1, N + 1)
    grid = cubedspheregrid(cell, _vec(a, a + H, KV), KH)

    def q0(dg):
        x = grid.points()
        aux = dg.auxstate_host()
        Phi, p_ref = aux[0], aux[5]
        cv_d = 719.0
        R_d = law.gamma * cv_d - cv_d
        r = np.sqrt(np.sum(x * x, axis=0))
        z = r - a
        lon = np.arctan2(x[1], x[0])
        lat = np.arcsin(x[2] / r)
        beta = np.minimum(1.0, 3.0 * np.arccos(np.cos(lat) * np.cos(lon)))
        p = p_ref + 100.0 * (1 + np.cos(np.pi * beta)) / 2 * np.sin(np.pi * z / H)
        rho = p / (R_d * 300.0)
        zero = np.zeros_like(rho)
        return _pack(rho, zero, zero, zero, rho * (cv_d * 300.0 + Phi))

    dt = dt if dt is not None else 100 * (H / KV) / 330.0 / N ** 2
    return _sphere_case("sphere_acoustic_wave", law, grid, q0, dt, steps, imex, vflux)


def sphere_zonal_flow(N=3, KH=5, KV=5, steps=10, imex=True, dt=None, vflux="ec"):
    """Isothermal zonal flow on a small planet (radius 6.371229e6 / 125, model
    top 10 km): u = 20 (1 + z/a) cos(lat) m/s eastward in the balanced
    isothermal (300 K) state; reflective inner and outer spheres; EC volume
    flux, Rusanov surface flux, IMEX ARK23 (split_rhs = false) with
    dt = 3 dz / 330, dz the smallest radial node distance
    (isothermal_zonal_flow.jl:63-125)."""
    a, top = _EARTH_RADIUS / 125, 10e3
    law = EulerGravityLaw(3, sphere=True, problem=ReflectiveWall(referencestate=_isothermal_reference(a)))
    cell = LobattoCell(N + 1, N + 1, N + 1)
    grid = cubedspheregrid(cell, _vec(a, a + top, KV), KH)

    def q0(dg):
        x = grid.points()
        Phi = dg.auxstate_host()[0]
        cv_d = 719.0
        R_d = law.gamma * cv_d - cv_d
        r = np.sqrt(np.sum(x * x, axis=0))
        z = r - a
        lon = np.arctan2(x[1], x[0])
        lat = np.arcsin(x[2] / r)
        u0, T0, g = 20.0, 300.0, law.grav
        us = u0 * (1 + z / a) * np.cos(lat)  # zonal wind; meridional and radial zero
        u = [-np.sin(lon) * us, np.cos(lon) * us, np.zeros_like(us)]
        f2 = z / a + z ** 2 / (2 * a ** 2)
        prefac = u0 ** 2 / (R_d * T0)
        p = 1e5 * np.exp(prefac * f2 * np.cos(lat) ** 2 - prefac * np.sin(lat) ** 2 / 2 - g * z / (R_d * T0))
        rho = p / (R_d * T0)
        ke = (u[0] ** 2 + u[1] ** 2 + u[2] ** 2) / 2
        return _pack(rho, rho * u[0], rho * u[1], rho * u[2], rho * (cv_d * T0 + ke + Phi))

    dt = dt if dt is not None else 3 * min_node_distance(grid, dims=(3,)) / 330.0
    return _sphere_case("sphere_zonal_flow", law, grid, q0, dt, steps, imex, vflux)


def sphere_baroclinic_wave(N=3, KH=8, KV=4, steps=10, imex=True, dt=None, vflux="ec", perturb=True):
    """Baroclinic wave on a rotating Earth-radius shell 30 km deep
    (baroclinicwave.jl:49-253): the deep-atmosphere balanced state of
    Ullrich, Melvin, Jablonowski and Staniforth (2014) with T_E = 310 K,
    T_P = 240 K, lapse rate 0.005 K/m, k = 3, b = 2, and a zonal-wind
    perturbation of 1 m/s centred at (20 deg E, 40 deg N); g = 9.80616,
    Omega = 7.29212e-5 (the Coriolis source dq[rho u] -= (0, 0, 2 Omega) x rho u),
    reflective inner and outer spheres, isothermal (300 K) reference state;
    EC volume flux, Rusanov surface flux, IMEX ARK23 (split_rhs = false) with
    dt = 3 dz / 330."""
    a, top, Om, grav = _EARTH_RADIUS, 30e3, 7.29212e-5, 9.80616
    problem = Coriolis((0.0, 0.0, 2 * Om), bc=ReflectiveWall().bc, referencestate=_isothermal_reference(a))
    law = EulerGravityLaw(3, sphere=True, grav=grav, problem=problem)
    cell = LobattoCell(N + 1, N + 1, N + 1)
    grid = cubedspheregrid(cell, _vec(a, a + top, KV), KH)

    def q0(dg):
        x = grid.points()
        Phi = dg.auxstate_host()[0]
        cv_d = 719.0
        R_d = law.gamma * cv_d - cv_d
        r = np.sqrt(np.sum(x * x, axis=0))
        z = r - a
        lon = np.arctan2(x[1], x[0])
        lat = np.arcsin(x[2] / r)
        k, T_E, T_P, Gam, b, p_0 = 3.0, 310.0, 240.0, 0.005, 2.0, 1e5
        T_0 = (T_E + T_P) / 2
        A_, B_ = 1 / Gam, (T_0 - T_P) / T_0 / T_P
        C_ = (k + 2) / 2 * (T_E - T_P) / T_E / T_P
        H = R_d * T_0 / grav
        z_t, lon_c, lat_c, d_0, V_p = 15e3, np.pi / 9, 2 * np.pi / 9, a / 6, 1.0
        tz1 = np.exp(Gam * z / T_0)
        tz2 = 1 - 2 * (z / b / H) ** 2
        tz3 = np.exp(-(z / b / H) ** 2)
        tau1 = 1 / T_0 * tz1 + B_ * tz2 * tz3
        tau2 = C_ * tz2 * tz3
        ti1 = A_ * (tz1 - 1) + B_ * z * tz3
        ti2 = C_ * z * tz3
        cz = np.cos(lat) * (1 + z / a)  # deep atmosphere
        I_T = cz ** k - k / (k + 2) * cz ** (k + 2)
        T = 1 / (tau1 - tau2 * I_T)
        p = p_0 * np.exp(-grav / R_d * (ti1 - ti2 * I_T))
        U = grav * k / a * ti2 * T * (cz ** (k - 1) - cz ** (k + 1))
        rc = (a + z) * np.cos(lat)
        u = -Om * rc + np.sqrt((Om * rc) ** 2 + rc * U)
        v = np.zeros_like(u)
        if perturb:
            F_z = np.where(z > z_t, 0.0, 1 - 3 * (z / z_t) ** 2 + 2 * (z / z_t) ** 3)
            cosd = np.sin(lat) * np.sin(lat_c) + np.cos(lat) * np.cos(lat_c) * np.cos(lon - lon_c)
            d = a * np.arccos(np.clip(cosd, -1.0, 1.0))
            inside = (d > 0) & (d < d_0)
            c3 = np.cos(np.pi * d / 2 / d_0) ** 3
            s1 = np.sin(np.pi * d / 2 / d_0)
            sd = np.where(inside, np.sin(d / a), 1.0)
            amp = np.where(inside, 16 * V_p / 3 / np.sqrt(3) * F_z * c3 * s1 / sd, 0.0)
            u = u + amp * -(-np.sin(lat_c) * np.cos(lat) + np.cos(lat_c) * np.sin(lat) * np.cos(lon - lon_c))
            v = v + amp * np.cos(lat_c) * np.sin(lon - lon_c)
        # spherical (east, north, up) to Cartesian components
        uc = -np.sin(lon) * u - np.sin(lat) * np.cos(lon) * v
        vc = np.cos(lon) * u - np.sin(lat) * np.sin(lon) * v
        wc = np.cos(lat) * v
        rho = p / (R_d * T)
        ke = (uc ** 2 + vc ** 2 + wc ** 2) / 2
        return _pack(rho, rho * uc, rho * vc, rho * wc, rho * (cv_d * T + ke + Phi))

    dt = dt if dt is not None else 3 * min_node_distance(grid, dims=(3,)) / 330.0
    return _sphere_case("sphere_baroclinic_wave", law, grid, q0, dt, steps, imex, vflux)


# ------------------------------------------------------ shallow water, C3
def sw_fplane(N=4, K=32, L=1.0e6, H=100.0, seed=20261203, lake_at_rest=False, precision="fp64", f=1e-4,
              steps=500):
    """Rotating shallow water (f-plane, g = 9.81) on a periodic square of K x K
    elements, order N; smooth random bottom topography (sum of 8 Gaussians,
    amplitude <= 10% of the mean depth H) and seeded random height
    perturbations (amplitude 1 m, wavelengths 4-16 elements).  EC volume flux
    with the well-balanced bathymetry terms, Rusanov surface flux, LSRK54."""
    rng = np.random.default_rng(seed)
    cell = LobattoCell(N + 1, N + 1)
    v = _vec(0.0, L, K)
    grid = brickgrid(cell, (v, v), periodic=(True, True))
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

    law = ShallowWaterLaw(2, grav=g, topography=True, problem=Coriolis((0.0, 0.0, f)))
    law.bathymetry = bath
    dg = DGSEM(law=law, grid=grid, volume_form=FluxDifferencingForm(EntropyConservativeFlux()),
                 surface_numericalflux=RusanovFlux(), precision=precision)
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


# --------------------------------------------- device-built initial states
def vortex_c1_device(dg):
    """The vortex of ``vortex_c1`` on ``dg``'s grid, built on the device:
    (q0, aux) CUDA tensors (the Euler law has no aux fields)."""
    import torch
    from .cell import points_device

    x = points_device(dg.grid)
    g = dg.law.gamma
    r0 = x[0] - 10.0 * torch.round(x[0] / 10.0)
    r1 = x[1] - 10.0 * torch.round(x[1] / 10.0)
    f = 5.0 * torch.exp(1 - (r0 * r0 + r1 * r1))
    rho = (1 - (g - 1) * f ** 2 / (16 * g * math.pi ** 2)) ** (1 / (g - 1))
    m0 = rho * (1.0 + f / (2 * math.pi) * (-r1))
    m1 = rho * (1.0 + f / (2 * math.pi) * r0)
    E = rho ** g / (g - 1) + (m0 * m0 + m1 * m1) / (2 * rho)
    return torch.stack([rho, m0, m1, E]).contiguous(), None


def bubble_3d_device(dg, L=10e3):
    """The rising bubble of ``bubble_3d`` on ``dg``'s grid, built on the
    device: (q0, aux) CUDA tensors, aux = [Phi, grad Phi, rho_ref, p_ref] of
    the constant-theta background (src/balancelaws/euler_gravity.jl:38-62)."""
    import torch
    from .cell import points_device

    law = dg.law
    grav = law.grav
    cv = 719.0
    cp = law.gamma * cv
    R = cp - cv
    x = points_device(dg.grid)
    z = x[2]
    pi_ex = 1 - grav / (cp * 300.0) * z
    aux = torch.zeros((law.naux,) + tuple(z.shape), dtype=torch.float64, device=z.device)
    aux[0] = grav * z
    aux[3] = grav
    aux[4] = 1e5 / (R * 300.0) * pi_ex ** (cv / R)
    aux[5] = 1e5 * pi_ex ** (cp / R)
    r = torch.sqrt((x[0] - L / 2) ** 2 + (x[1] - L / 2) ** 2 + (z - 2000.0) ** 2)
    theta = 300.0 + 2.0 * torch.exp(-(r / 2000.0) ** 2)
    p = 1e5 * pi_ex ** (cp / R)
    rho = p / (R * (theta * pi_ex))
    zero = torch.zeros_like(rho)
    rhoe = p / (law.gamma - 1) + rho * aux[0]
    return torch.stack([rho, zero, zero, zero, rhoe]).contiguous(), aux.contiguous()

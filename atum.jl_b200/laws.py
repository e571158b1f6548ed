"""Balance laws, problems, numerical fluxes and volume forms (host side).

Mirrors the reference's physics plugin API:

* ``AbstractBalanceLaw{FT,D,S,C}`` and the concrete laws
  ``AdvectionLaw`` (src/balancelaws/advection.jl:4-14),
  ``EulerLaw`` (src/balancelaws/euler.jl:9-17),
  ``EulerGravityLaw`` (src/balancelaws/euler_gravity.jl:10-23),
  ``LinearEulerGravityLaw`` (src/balancelaws/linear_euler_gravity.jl:1-9),
  ``ShallowWaterLaw`` (src/balancelaws/shallow_water.jl:9-17).
* numerical-flux tags (src/numericalfluxes.jl:25-47) and the volume forms
  ``WeakForm`` / ``FluxDifferencingForm`` (src/dgsem.jl:5-14).
* problems: Julia dispatch on ``AbstractProblem`` subtypes becomes enumerated
  kinds the device can evaluate (reflective wall, inflow-zero, Dirichlet per
  boundary tag, Coriolis source) plus a host callable ``referencestate``
  evaluated once into the aux fields, as the reference does at DGSEM
  construction (src/dgsem.jl:41).

The pointwise state helpers (``energy``, ``pressure``, ``soundspeed``) are
numpy restatements used to build initial conditions, like the reference's
``Euler.energy`` calls in its tests.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable, Optional

import numpy as np

# enumerations shared with include/atum_b200.h
LAW_ADVECTION, LAW_EULER, LAW_EULER_GRAVITY, LAW_LINEAR_EULER_GRAVITY, LAW_SHALLOW_WATER = range(5)
FLUX_CENTRAL, FLUX_RUSANOV, FLUX_EC, FLUX_KG, FLUX_ROE, FLUX_MATRIX = range(6)
BC_COPY, BC_REFLECT, BC_INFLOW_ZERO, BC_DIRICHLET = range(4)
SRC_NONE, SRC_CORIOLIS = range(2)


# ----------------------------------------------------------------- problems
@dataclass
class AbstractProblem:
    """Problem hooks: boundary state kind, source kind, reference state."""

    bc: int = BC_COPY
    bc_state: tuple = ((0.0,) * 5, (0.0,) * 5)
    source: int = SRC_NONE
    omega: tuple = (0.0, 0.0, 0.0)
    referencestate: Optional[Callable] = None  # (law, x: (dim, ...)) -> (rho_ref, p_ref)


def DummyProblem():
    return AbstractProblem()


def ReflectiveWall(**kw):
    """``boundarystate`` mirroring momentum: experiment/euler_gravity/risingbubble.jl:10-15."""
    return AbstractProblem(bc=BC_REFLECT, **kw)


def InflowZero(**kw):
    """Zero state on inflow faces (u.n <= 0): test/advection/imex_wave_2d.jl:19-26."""
    return AbstractProblem(bc=BC_INFLOW_ZERO, **kw)


def DirichletByTag(state_tag1, state_other, **kw):
    """Fixed state per boundary tag (tag 1 vs others): experiment/euler/sod.jl:20-23."""
    s1 = tuple(float(v) for v in state_tag1) + (0.0,) * (5 - len(state_tag1))
    s2 = tuple(float(v) for v in state_other) + (0.0,) * (5 - len(state_other))
    return AbstractProblem(bc=BC_DIRICHLET, bc_state=(s1, s2), **kw)


def Coriolis(omega, bc: int = BC_COPY, **kw):
    """``source!`` dq[mom] -= omega x mom (experiment/euler_gravity/baroclinicwave.jl:27-34);
    in 2-D an f-plane with omega = (0, 0, f)."""
    return AbstractProblem(bc=bc, source=SRC_CORIOLIS, omega=tuple(float(v) for v in omega), **kw)


# --------------------------------------------------------------------- laws
class AbstractBalanceLaw:
    kind: int
    dim: int
    FT = np.float64

    def __init__(self, dim: int, problem: Optional[AbstractProblem] = None):
        if dim not in (1, 2, 3):
            raise ValueError("dim must be 1, 2 or 3")
        self.dim = dim
        self.problem = problem if problem is not None else AbstractProblem()

    @property
    def numberofstates(self) -> int:
        return self.dim + 2

    @property
    def naux(self) -> int:
        return 0

    def auxiliary(self, x: np.ndarray) -> np.ndarray:
        """Aux fields at points ``x`` (dim, K, Np) -> (naux, K, Np)."""
        return np.zeros((0,) + x.shape[1:])

    # descriptor fields shared by the oracle and the device library
    gamma = 1.4
    grav = 9.81
    adv_u = (1.0, 1.0, 1.0)
    sphere = False
    pde_level_balance = False
    sw_topography = False


def numberofstates(law) -> int:
    return law.numberofstates


def constants(law):
    return law


class AdvectionLaw(AbstractBalanceLaw):
    """``AdvectionLaw{FT,D}(u)``: S = 1, flux u q (src/balancelaws/advection.jl)."""

    kind = LAW_ADVECTION

    def __init__(self, dim: int, u=None, problem=None):
        super().__init__(dim, problem)
        u = tuple(float(v) for v in (u if u is not None else (1.0,) * dim))
        if len(u) != dim:
            raise ValueError("advection velocity needs dim components")
        self.u = u
        self.adv_u = u + (0.0,) * (3 - dim)

    @property
    def numberofstates(self) -> int:
        return 1


class EulerLaw(AbstractBalanceLaw):
    """``EulerLaw{FT,D}(; gamma=7//5)``: S = D + 2 (src/balancelaws/euler.jl:9-17)."""

    kind = LAW_EULER

    def __init__(self, dim: int, gamma: float = 7 / 5, problem=None):
        super().__init__(dim, problem)
        self.gamma = float(gamma)

    # src/balancelaws/euler.jl:32-46
    def pressure(self, rho, rhou, rhoe):
        return (self.gamma - 1) * (rhoe - sum(m * m for m in rhou) / (2 * rho))

    def energy(self, rho, rhou, p):
        return p / (self.gamma - 1) + sum(m * m for m in rhou) / (2 * rho)

    def soundspeed(self, rho, p):
        return np.sqrt(self.gamma * p / rho)


class EulerGravityLaw(EulerLaw):
    """``EulerGravityLaw{FT,D}(; gamma, grav=981//100, sphere, pde_level_balance)``.

    aux = [Phi, grad Phi, rho_ref, p_ref] (src/balancelaws/euler_gravity.jl:38-62).
    """

    kind = LAW_EULER_GRAVITY

    def __init__(self, dim: int, gamma: float = 7 / 5, grav: float = 981 / 100, sphere: bool = False,
                 pde_level_balance: bool = False, problem=None):
        super().__init__(dim, gamma, problem)
        self.grav = float(grav)
        self.sphere = bool(sphere)
        self.pde_level_balance = bool(pde_level_balance)

    @property
    def has_reference(self) -> bool:
        return self.problem.referencestate is not None

    @property
    def naux(self) -> int:
        return 1 + self.dim + (2 if self.has_reference else 0)

    def auxiliary(self, x: np.ndarray) -> np.ndarray:
        g = self.grav
        out = np.zeros((self.naux,) + x.shape[1:])
        if self.sphere:
            r = np.sqrt(np.sum(x * x, axis=0))
            out[0] = g * r
            for d in range(self.dim):
                out[1 + d] = g * x[d] / r
        else:
            out[0] = g * x[self.dim - 1]
            out[self.dim] = g
        if self.has_reference:
            rho_ref, p_ref = self.problem.referencestate(self, x)
            out[self.dim + 1] = rho_ref
            out[self.dim + 2] = p_ref
        return out

    def pressure(self, rho, rhou, rhoe, Phi):
        return (self.gamma - 1) * (rhoe - sum(m * m for m in rhou) / (2 * rho) - rho * Phi)

    def energy(self, rho, rhou, p, Phi):
        return p / (self.gamma - 1) + sum(m * m for m in rhou) / (2 * rho) + rho * Phi


class LinearEulerGravityLaw(AbstractBalanceLaw):
    """``LinearEulerGravityLaw(parent)``: linearisation about the aux reference state."""

    kind = LAW_LINEAR_EULER_GRAVITY

    def __init__(self, parent: EulerGravityLaw):
        if not isinstance(parent, EulerGravityLaw):
            raise TypeError("LinearEulerGravityLaw wraps an EulerGravityLaw")
        if not parent.has_reference:
            raise ValueError("the linear law needs a problem with a referencestate")
        super().__init__(parent.dim, parent.problem)
        self.parent = parent
        self.gamma = parent.gamma
        self.grav = parent.grav
        self.sphere = parent.sphere

    @property
    def naux(self) -> int:
        return self.parent.naux

    def auxiliary(self, x):
        return self.parent.auxiliary(x)

    # src/balancelaws/linear_euler_gravity.jl:18-21
    def reference_rhoe(self, p, rho, Phi):
        return p / (self.gamma - 1) + rho * Phi


class ShallowWaterLaw(AbstractBalanceLaw):
    """``ShallowWaterLaw{FT,D}(; grav=10)``: state (h, h u, h theta).

    ``topography=True`` is an extension the reference lacks: aux = [b, grad b]
    with the well-balanced non-conservative term g h grad b in the
    flux-differencing, weak and surface forms.
    """

    kind = LAW_SHALLOW_WATER

    def __init__(self, dim: int, grav: float = 10, topography: bool = False, problem=None):
        super().__init__(dim, problem)
        self.grav = float(grav)
        self.sw_topography = bool(topography)
        self.bathymetry: Optional[Callable] = None  # x -> (b, grad b)

    @property
    def naux(self) -> int:
        return 1 + self.dim if self.sw_topography else 0

    def auxiliary(self, x):
        if not self.sw_topography:
            return np.zeros((0,) + x.shape[1:])
        if self.bathymetry is None:
            raise ValueError("set law.bathymetry = f(x) -> (b, grad_b) for topography")
        b, gb = self.bathymetry(x)
        out = np.zeros((self.naux,) + x.shape[1:])
        out[0] = b
        for d in range(self.dim):
            out[1 + d] = gb[d]
        return out


# ------------------------------------------------------------------- fluxes
class AbstractNumericalFlux:
    kind: int

    def __eq__(self, other):
        return type(self) is type(other)

    def __hash__(self):
        return hash(type(self))

    def __repr__(self):
        return type(self).__name__ + "()"


class CentralFlux(AbstractNumericalFlux):
    kind = FLUX_CENTRAL


class RusanovFlux(AbstractNumericalFlux):
    kind = FLUX_RUSANOV


class EntropyConservativeFlux(AbstractNumericalFlux):
    kind = FLUX_EC


class KennedyGruberFlux(AbstractNumericalFlux):
    kind = FLUX_KG


class RoeFlux(AbstractNumericalFlux):
    kind = FLUX_ROE


class MatrixFlux(AbstractNumericalFlux):
    kind = FLUX_MATRIX


class AbstractVolumeForm:
    pass


class WeakForm(AbstractVolumeForm):
    def __eq__(self, other):
        return isinstance(other, WeakForm)

    def __hash__(self):
        return hash("WeakForm")

    def __repr__(self):
        return "WeakForm()"


_FD_KERNELS = {"naive": 2, "per_dir": 0, "per_dir_symmetric": 1}


class FluxDifferencingForm(AbstractVolumeForm):
    """``FluxDifferencingForm(volume_numericalflux, kernel_type=:per_dir)``."""

    def __init__(self, volume_numericalflux: AbstractNumericalFlux, kernel_type: str = "per_dir"):
        kernel_type = str(kernel_type).lstrip(":")
        if kernel_type not in _FD_KERNELS:
            raise ValueError(f"Unknown kernel type {kernel_type}")
        self.volume_numericalflux = volume_numericalflux
        self.kernel_type = kernel_type

    def __eq__(self, other):
        return (isinstance(other, FluxDifferencingForm) and other.volume_numericalflux == self.volume_numericalflux
                and other.kernel_type == self.kernel_type)

    def __hash__(self):
        return hash(("FD", self.volume_numericalflux, self.kernel_type))

    def __repr__(self):
        return f"FluxDifferencingForm({self.volume_numericalflux!r})"


# which (law, flux) pairs have a two-point flux / surface flux in the reference
_TWOPOINT = {
    LAW_ADVECTION: {FLUX_CENTRAL},
    LAW_EULER: {FLUX_CENTRAL, FLUX_EC, FLUX_KG},
    LAW_EULER_GRAVITY: {FLUX_CENTRAL, FLUX_EC, FLUX_KG},
    LAW_LINEAR_EULER_GRAVITY: {FLUX_CENTRAL},
    LAW_SHALLOW_WATER: {FLUX_CENTRAL, FLUX_EC},
}
_SURFACE_EXTRA = {
    LAW_EULER: {FLUX_RUSANOV, FLUX_ROE, FLUX_MATRIX},
    LAW_EULER_GRAVITY: {FLUX_RUSANOV, FLUX_ROE, FLUX_MATRIX},
    LAW_SHALLOW_WATER: {FLUX_RUSANOV, FLUX_ROE},
    LAW_ADVECTION: {FLUX_RUSANOV},
    LAW_LINEAR_EULER_GRAVITY: {FLUX_RUSANOV},
}


def check_fluxes(law, volume_form, surface_flux):
    """Raise where the reference would raise a MethodError."""
    if isinstance(volume_form, FluxDifferencingForm):
        k = volume_form.volume_numericalflux.kind
        if k not in _TWOPOINT[law.kind]:
            raise NotImplementedError(f"no twopointflux({volume_form.volume_numericalflux!r}, {type(law).__name__})")
    s = surface_flux.kind
    if s not in _TWOPOINT[law.kind] | _SURFACE_EXTRA[law.kind]:
        raise NotImplementedError(f"no surfaceflux({surface_flux!r}, {type(law).__name__})")

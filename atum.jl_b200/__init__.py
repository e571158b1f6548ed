"""atum_b200 — B200-native DGSEM tendency evaluation and time stepping.

A from-scratch sm_100a implementation of the DGSEM hot path of Atum.jl
(balance laws, numerical fluxes, the DGSEM operator call and the LSRK / RLSRK /
ARK23 solvers) behind a C ABI (``include/atum_b200.h``).  This package is the
host-side mirror of the reference's Julia API; the compute runs in the CUDA
library ``csrc/libatumb200.so`` and there is no CPU fallback.

The directory name is not a Python identifier: load it as ``atum_b200`` with
``_load_package()`` from ``__graft_entry__.py`` at the repository root (an
``importlib`` spec over this directory; the tests do the same in conftest).
"""
from .cell import LobattoCell, BrickGrid, brickgrid, min_node_distance, points
from .cubedsphere import CubedSphereGrid, cubedspheregrid
from .laws import (AbstractProblem, DummyProblem, ReflectiveWall, InflowZero, DirichletByTag, Coriolis,
                   AbstractBalanceLaw, AdvectionLaw, EulerLaw, EulerGravityLaw, LinearEulerGravityLaw,
                   ShallowWaterLaw, numberofstates, constants,
                   CentralFlux, RusanovFlux, EntropyConservativeFlux, KennedyGruberFlux, RoeFlux, MatrixFlux,
                   WeakForm, FluxDifferencingForm)
from .dgsem import DGSEM, fieldarray, components

__version__ = "0.1.0"


def __getattr__(name):
    # solvers / measures / serving import torch and the CUDA library lazily
    if name in ("measures", "odesolvers", "serving", "batch", "_lib", "_device", "build", "checkpoint", "vtk",
                "workloads"):
        import importlib
        return importlib.import_module("." + name, __name__)
    if name in ("LSRK54", "LSRK144", "RLSRK54", "RLSRK144", "ARK23", "solve_", "LSRK", "RLSRK", "ARK"):
        from . import odesolvers
        return getattr(odesolvers, name)
    if name in ("weightednorm", "entropyintegral", "entropyproduct"):
        from . import measures
        return getattr(measures, name)
    raise AttributeError(name)

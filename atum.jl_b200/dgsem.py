"""``DGSEM`` operator (host side of src/dgsem.jl).

``DGSEM(law=, grid=, surface_numericalflux=, volume_form=WeakForm(),
directions=1:dim, auxstate=auxiliary.(law, points(grid)))`` builds the spec
(src/dgsem.jl:38-56); calling it, ``dg(dq, q, time, increment=True)``
(src/dgsem.jl:59-98), evaluates the tendency on the GPU through the C ABI
(``atb_op_apply``).  The spec itself needs no GPU, so CPU tests and the oracle
share it.

Fields are torch float64 CUDA tensors of shape (Ns, K, Np): the SoA layout of
the reference's StructArray ``fieldarray`` (each component Np x K,
column-major), node index ``i + Nq*(j + Nq*k)`` fastest.
"""
from __future__ import annotations

from typing import Optional, Sequence

import numpy as np

from .cell import BrickGrid
from .laws import (AbstractBalanceLaw, AbstractNumericalFlux, FluxDifferencingForm, WeakForm, _FD_KERNELS,
                   check_fluxes, LAW_LINEAR_EULER_GRAVITY)

__all__ = ["DGSEM", "fieldarray", "components"]

PRECISIONS = {"fp64": 0, "fp32flux": 1}


class DGSEM:
    def __init__(self, *, law: AbstractBalanceLaw, grid: BrickGrid, surface_numericalflux: AbstractNumericalFlux,
                 volume_form=None, directions: Optional[Sequence[int]] = None, auxstate=None,
                 precision: str = "fp64"):
        self.law = law
        self.grid = grid
        self.surface_numericalflux = surface_numericalflux
        self.volume_form = volume_form if volume_form is not None else WeakForm()
        if law.dim != grid.dim:
            raise ValueError("law and grid dimensions differ")
        dirs = tuple(range(1, law.dim + 1)) if directions is None else tuple(int(d) for d in directions)
        if not dirs or any(d < 1 or d > law.dim for d in dirs) or len(set(dirs)) != len(dirs):
            raise ValueError("directions must be distinct values in 1:dim")
        if list(dirs) != sorted(dirs):
            raise ValueError("directions must be increasing")
        self.directions = dirs
        if isinstance(self.volume_form, FluxDifferencingForm) and self.volume_form.kernel_type == "naive" \
                and dirs != tuple(range(1, law.dim + 1)):
            # src/dgsem.jl:137-138
            raise ValueError("the :naive kernel supports only directions = 1:ndims(law)")
        check_fluxes(law, self.volume_form, surface_numericalflux)
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
        self.precision = precision
        self._aux_dev = None
        if auxstate is not None and getattr(auxstate, "is_cuda", False):
            # aux evaluated on the device (like the reference's
            # auxiliary.(law, points(grid)) on GPU arrays): kept there, uploaded
            # device to device, copied to the host only if a host copy is asked for
            import torch

            want = (self.law.naux, len(self.grid), self.grid.cell.Np)
            if auxstate.numel() != int(np.prod(want)):
                raise ValueError(f"auxstate must have shape {want}")
            self._aux_dev = auxstate.detach().to(dtype=torch.float64).reshape(want).contiguous()
            self._aux = None
        else:
            self._aux = None if auxstate is None else self._as_aux(auxstate)
        self._dev = None

    # ------------------------------------------------------------- host spec
    def _as_aux(self, auxstate):
        if isinstance(auxstate, DGSEM):
            if auxstate._aux_dev is not None and auxstate._aux is None:
                self._aux_dev = auxstate._aux_dev
                return None
            auxstate = auxstate.auxstate_host()
        if hasattr(auxstate, "detach"):
            auxstate = auxstate.detach().cpu().numpy()
        a = np.ascontiguousarray(auxstate, dtype=np.float64)
        want = (self.law.naux, len(self.grid), self.grid.cell.Np)
        if a.size != int(np.prod(want)):
            raise ValueError(f"auxstate must have shape {want}")
        return a.reshape(want)

    def auxstate_host(self) -> np.ndarray:
        if self._aux is None:
            if self._aux_dev is not None:
                self._aux = self._aux_dev.cpu().numpy()
            else:
                self._aux = np.ascontiguousarray(self.law.auxiliary(self.grid.points()), dtype=np.float64)
        return self._aux

    @property
    def auxstate(self):
        return self.auxstate_host()

    @property
    def MJ(self) -> np.ndarray:
        """M * J per node, shape (K, Np) (src/dgsem.jl:43-45)."""
        c, g = self.grid.cell, self.grid
        if hasattr(g, "geometry"):  # curved elements carry their own M J
            return g.geometry()["MJ"]
        node = np.arange(c.Np)
        w = np.ones(c.Np)
        for d in range(g.dim):
            w = w * c.weights[(node // c.Nq ** d) % c.Nq] if d else c.weights[node % c.Nq]
        eidx = g.element_indices()
        J = np.ones(len(g))
        for d in range(g.dim):
            J = J * (np.diff(g.vertices[d])[eidx[:, d]] / 2)
        return w[None, :] * J[:, None]

    def descriptor_fields(self) -> dict:
        law, grid = self.law, self.grid
        vf = self.volume_form
        fd = isinstance(vf, FluxDifferencingForm)
        pr = law.problem
        Kd = list(grid.Kd) + [1] * (3 - grid.dim)
        return dict(
            law=law.kind, dim=law.dim, N=grid.cell.N, K=Kd, vertices=grid.vertices,
            periodic=[int(p) for p in grid.periodic] + [0] * (3 - grid.dim), stacked=int(grid.stacked),
            volume_form=int(fd), volume_flux=vf.volume_numericalflux.kind if fd else 0,
            fd_kernel=_FD_KERNELS[vf.kernel_type] if fd else 0,
            surface_flux=self.surface_numericalflux.kind,
            directions=sum(1 << (d - 1) for d in self.directions),
            gamma=float(law.gamma), grav=float(law.grav), adv_u=list(law.adv_u),
            sphere=int(law.sphere), pde_level_balance=int(law.pde_level_balance),
            bc_kind=pr.bc, bc_state=pr.bc_state, source_kind=pr.source, omega=list(pr.omega),
            sw_topography=int(law.sw_topography), naux=law.naux,
            precision=PRECISIONS[self.precision],
        )

    @property
    def is_linear(self) -> bool:
        return self.law.kind == LAW_LINEAR_EULER_GRAVITY

    def __repr__(self):
        return (f"DGSEM(law={type(self.law).__name__}{self.law.dim}D, N={self.grid.cell.N}, K={self.grid.Kd}, "
                f"volume_form={self.volume_form!r}, surface={self.surface_numericalflux!r}, "
                f"directions={self.directions}, precision={self.precision})")

    # ---------------------------------------------------------- device side
    @property
    def device(self):
        if self._dev is None:
            from ._device import DeviceOp
            self._dev = DeviceOp(self)
        return self._dev

    def __call__(self, dq, q, time: float = 0.0, increment: bool = True):
        self.device.apply(dq, q, time, increment)

    def fieldarray(self, init=None):
        return fieldarray(self.law, self.grid, init)


def fieldarray(law: AbstractBalanceLaw, grid: BrickGrid, init=None, device: str = "cuda"):
    """``fieldarray(init, law, grid)``: (Ns, K, Np) float64 tensor."""
    import torch

    shape = (law.numberofstates, len(grid), grid.cell.Np)
    if init is None:
        return torch.zeros(shape, dtype=torch.float64, device=device)
    t = torch.as_tensor(np.asarray(init, dtype=np.float64).reshape(shape), device=device)
    return t.contiguous()


def components(q):
    return tuple(q[s] for s in range(q.shape[0]))

"""Aux fields evaluated on the device (atb_op_set_aux from device memory, the
way the reference evaluates auxiliary.(law, points(grid)) on GPU arrays) give
the same operator as aux fields uploaded from the host, and device-side grid
points equal the host ones."""
import numpy as np
import pytest

import atum_b200 as A
import parity as PT
import problems as P

pytestmark = pytest.mark.gpu


def test_points_device_equal_host():
    from atum_b200.cell import points_device
    c = P.bubble_3d(N=3, K=3, imex=True)
    assert np.array_equal(points_device(c.dg.grid).cpu().numpy(), c.dg.grid.points())


def test_device_aux_same_tendency_and_ark_step():
    import torch
    c = P.bubble_3d(N=3, K=4, imex=True, steps=2)
    aux_dev = torch.as_tensor(c.dg.auxstate_host(), device="cuda")
    dgd = A.DGSEM(law=c.dg.law, grid=c.dg.grid, volume_form=c.dg.volume_form,
                  surface_numericalflux=c.dg.surface_numericalflux, auxstate=aux_dev)
    lind = A.DGSEM(law=c.lindg.law, grid=c.dg.grid, surface_numericalflux=A.RusanovFlux(), auxstate=aux_dev,
                   directions=(3,))
    q = PT.to_dev(c.q0)
    a, b = torch.zeros_like(q), torch.zeros_like(q)
    c.dg(a, q, 0.0, increment=False)
    dgd(b, q, 0.0, increment=False)
    assert torch.equal(a, b)
    qa, qb = PT.to_dev(c.q0), PT.to_dev(c.q0)
    A.ARK23(c.dg, c.lindg, qa, c.dt, split_rhs=False).step(qa, 2)
    A.ARK23(dgd, lind, qb, c.dt, split_rhs=False).step(qb, 2)
    assert torch.equal(qa, qb)

"""Persistent tendency launches (atb_op_set_persistent): a few CTAs walking
every element tile with a grid stride give the ordinary launch's results bit
for bit -- packed instances of different sizes (LSRK54), the fused ARK23 stage
kernel, and a grid smaller than the tile count by any factor."""
import numpy as np
import pytest
import torch

import atum_b200 as A
import parity as PT
import problems as P

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ctas", [1, 3, 148])
def test_persistent_packed_instances(ctas):
    cases = [P.sw_fplane(N=4, K=k, seed=20 + k, steps=3) for k in (4, 6, 9)]
    packed = A.batch.PackedDGSEM([c.dg for c in cases])
    q0 = packed.pack([torch.as_tensor(c.q0, device="cuda") for c in cases])
    dt = min(c.dt for c in cases)
    qa, qb = q0.clone(), q0.clone()
    A.LSRK54(packed, qa, dt).step(qa, 3)
    packed.set_persistent(ctas)
    A.LSRK54(packed, qb, dt).step(qb, 3)
    packed.set_persistent(0)
    assert torch.equal(qa, qb)


@pytest.mark.parametrize("ctas", [2, 148])
def test_persistent_fused_ark_stage(ctas):
    c = P.bubble_3d(N=4, K=3, imex=True, steps=3)
    qa, qb = PT.to_dev(c.q0), PT.to_dev(c.q0)
    A.ARK23(c.dg, c.lindg, qa, c.dt, split_rhs=False).step(qa, 3)
    A.batch.set_persistent(c.dg, ctas)
    A.ARK23(c.dg, c.lindg, qb, c.dt, split_rhs=False).step(qb, 3)
    A.batch.set_persistent(c.dg, 0)
    assert torch.equal(qa, qb)


def test_persistent_rejects_what_has_no_persistent_kernel():
    g = A.cubedspheregrid(A.LobattoCell(3, 3, 3), [1.0, 2.0], 1)
    dg = A.DGSEM(law=A.EulerLaw(3), grid=g, surface_numericalflux=A.RusanovFlux())
    with pytest.raises(A._lib.AtbError):
        A.batch.set_persistent(dg, 4)
    c = P.vortex_c1()
    with pytest.raises(A._lib.AtbError):
        A.batch.set_persistent(c.dg, -1)
    A.batch.set_persistent(c.dg, 8)  # 2-D Euler EC, Rusanov, N = 3: has one
    A.batch.set_persistent(c.dg, 0)

"""ARK23 stages with the explicit Euler-gravity tendency and the linear
vertical operator in one kernel give the same states as the two-launch path,
and solvers that cannot fuse say so."""
import numpy as np
import pytest

import atum_b200 as A
import parity as PT
import problems as P

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "fp32flux"])
@pytest.mark.parametrize("N,K", [(3, 4), (4, 3)])
def test_fused_equals_two_launches(precision, N, K):
    import torch
    c = P.bubble_3d(N=N, K=K, imex=True, steps=5, precision=precision)
    rng = np.random.default_rng(3)
    q0 = c.q0 * (1 + 1e-4 * rng.standard_normal(c.q0.shape))
    qa, qb = PT.to_dev(q0), PT.to_dev(q0)
    sa = A.ARK23(c.dg, c.lindg, qa, c.dt, split_rhs=False)
    sb = A.ARK23(c.dg, c.lindg, qb, c.dt, split_rhs=False)
    sb.fuse(False)
    sa.step(qa, 5)
    sb.step(qb, 5)
    d = (qa - qb).abs().max().item()
    scale = qb.abs().max().item()
    # FP64: the same operations in the same order; FP32 flux arithmetic may be
    # contracted into FMAs differently by the compiler in the fused kernel, so
    # it agrees to the FP32-flux form's own tolerance
    tol = 1e-14 if precision == "fp64" else 1e-6
    assert d <= tol * scale, d


def test_cannot_fuse_reports():
    c = P.imex_advection_2d(N=3, K=4)
    q = PT.to_dev(c.q0)
    s = A.ARK23(c.dg, c.lindg, q, c.dt)
    with pytest.raises(A._lib.AtbError, match="cannot run as one kernel"):
        s.fuse(True)
    s.fuse(False)

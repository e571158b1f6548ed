"""The tile-sparse warp-owned banded solve (band_solve_warp_kernel) against the
dense-block matrix-unit kernel (band_solve_mma_kernel, selected with
ATB_BAND_DENSE=1 at solver setup): the skipped tiles are exact zeros and each
accumulator adds its tiles in the same order, so whole ARK23 runs agree bit for
bit, for every order the kernels are built for."""
import numpy as np
import pytest

import atum_b200 as A
import parity as PT
import problems as P

pytestmark = pytest.mark.gpu


def _ark_run(case, steps, monkeypatch, dense):
    if dense:
        monkeypatch.setenv("ATB_BAND_DENSE", "1")
    else:
        monkeypatch.delenv("ATB_BAND_DENSE", raising=False)
    q = PT.to_dev(case.q0)
    s = A.ARK23(case.dg, case.lindg, q, case.dt, split_rhs=False)
    s.step(q, steps)
    out = q.cpu().numpy()
    del s
    return out


@pytest.mark.parametrize("N,K", [(1, 3), (2, 4), (3, 4), (4, 5), (5, 3), (6, 3), (7, 2)])
def test_warp_band_solve_bitwise_equals_dense(N, K, monkeypatch):
    case = P.bubble_3d(N=N, K=K, imex=True, steps=3)
    a = _ark_run(case, 3, monkeypatch, dense=False)
    b = _ark_run(case, 3, monkeypatch, dense=True)
    assert np.isfinite(a).all()
    assert np.array_equal(a, b)


def test_warp_band_solve_stacked_columns_vs_oracle(monkeypatch):
    """The warp-owned solve inside the parity metric on a non-cubic grid
    (more columns than a CTA's lines, partial last warp)."""
    import sys, os
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
    import pyoracle
    build = lambda k: P.bubble_3d(N=3, K=3, imex=True, steps=2, fd_kernel=k)  # noqa: E731
    case = build("per_dir")
    monkeypatch.delenv("ATB_BAND_DENSE", raising=False)
    q = PT.to_dev(case.q0)
    s = A.ARK23(case.dg, case.lindg, q, case.dt, split_rhs=False)
    s.step(q, 2)
    (qo,), (spread,) = PT.schedule_spread(pyoracle, build, [2])
    PT.assert_parity("band solve, bubble ARK23 N=3 3^3, 2 steps", q.cpu().numpy(), qo, 1e-12, spread=spread,
                     floors=PT.natural_floors(case.dg, qo))

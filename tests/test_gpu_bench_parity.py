"""Oracle parity of the kernels behind the benchmark numbers.

* The benchmark workload itself (rising bubble, 16^3 hexahedra, N = 4, IMEX
  ARK23 with split_rhs = false), built by the same builder and stepped the same
  way as ``bench.py`` (autotuned launch shapes, the fused ARK23 stage kernel
  ``tendency_kernel<EulerGravity, 3, EC, Nq=5, fused>``): 1 step at 1e-12 and
  100 steps at 1e-10.
* The fused stage kernel at every order N = 1..7 (Nq = 8 is the large
  single-instance workload's kernel) on a 3 x 3 x 4 stacked grid: 1 and 10
  steps.
* The Euler-gravity operator in 3-D at every order (one application).

Reference: src/dgsem.jl:470-561,683-732 (flux-differencing volume and surface
terms), src/balancelaws/euler_gravity.jl:200-236 (EC flux and its gravity
fluctuation), src/odesolvers.jl:312-388 (ARK23 step).  Metric and bounds:
tests/parity.py (plain field-relative per component, against the oracle's own
rounding spread where that is larger).
"""
import numpy as np
import pytest

import atum_b200 as A
import parity as PT
import problems as P
from atum_b200 import _lib
from atum_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _stage_kernel_is_fused(case, q0):
    """One profiled ARK23 step on a copy: no launch of the linear operator's
    own tendency kernel means the stage ran as the fused kernel."""
    L = _lib.lib()
    q = PT.to_dev(q0)
    s = A.ARK23(case.dg, case.lindg, q, case.dt, split_rhs=False)
    _lib.check(L.atb_profile_reset())
    _lib.check(L.atb_profile_enable(1))
    try:
        s.step(q, 1)
        import torch
        torch.cuda.synchronize()
    finally:
        _lib.check(L.atb_profile_enable(0))
    n_t, n_l, ms = _lib.C.c_long(), _lib.C.c_long(), _lib.C.c_double()
    _lib.check(L.atb_profile_read(0, _lib.C.byref(n_t), _lib.C.byref(ms)))
    _lib.check(L.atb_profile_read(1, _lib.C.byref(n_l), _lib.C.byref(ms)))
    return n_t.value == 3 and n_l.value == 0


def _gpu_states(case, counts, tune=True):
    q = PT.to_dev(case.q0)
    if tune:
        A.batch.autotune(case.dg, q)
        A.batch.autotune(case.lindg, q)
    s = A.ARK23(case.dg, case.lindg, q, case.dt, split_rhs=False)
    out, done = [], 0
    for n in counts:
        s.step(q, n - done)
        done = n
        out.append(PT.to_host(q))
    return out


def test_bench_workload_c2(orc):
    """The benchmark's rising bubble (16^3, N = 4), stepped as bench.py steps
    it, against the oracle: 1 step and 100 steps."""
    case = W.bubble_3d(N=4, K=16, imex=True, steps=200)
    assert _stage_kernel_is_fused(case, case.q0)
    counts = [1, 100]
    g = _gpu_states(case, counts)
    o, spread = PT.schedule_spread(orc, lambda k: W.bubble_3d(N=4, K=16, imex=True, steps=200, fd_kernel=k), counts)
    for n, gi, oi, si, tol in zip(counts, g, o, spread, (1e-12, 1e-10)):
        assert np.isfinite(gi).all()
        PT.assert_parity(f"bench workload 16^3 N=4 ARK23, {n} step(s)", gi, oi, tol, spread=si,
                         floors=PT.natural_floors(case.dg, oi))


@pytest.mark.parametrize("N", [1, 2, 3, 4, 5, 6, 7])
def test_fused_stage_kernel_orders(orc, N):
    """The fused ARK23 stage kernel at order N on a 3 x 3 x 4 stacked grid
    (Nq = 8 at N = 7: the large single-instance workload's kernel)."""
    case = W.bubble_3d(N=N, K=(3, 3, 4), imex=True, steps=10)
    assert _stage_kernel_is_fused(case, case.q0)
    counts = [1, 10]
    g = _gpu_states(case, counts, tune=False)
    o, spread = PT.schedule_spread(orc, lambda k: W.bubble_3d(N=N, K=(3, 3, 4), imex=True, steps=10, fd_kernel=k),
                                   counts)
    for n, gi, oi, si, tol in zip(counts, g, o, spread, (1e-12, 1e-11)):
        PT.assert_parity(f"fused ARK23 N={N} 3x3x4, {n} step(s)", gi, oi, tol, spread=si,
                         floors=PT.natural_floors(case.dg, oi))


@pytest.mark.parametrize("N", [1, 2, 3, 4, 5, 6, 7])
@pytest.mark.parametrize("sflux", ["rusanov", "roe", "matrix"])
def test_euler_gravity_3d_orders(orc, N, sflux):
    """One application of the 3-D Euler-gravity EC operator (reflective
    walls) at every order, against the oracle at 1e-12."""
    from test_gpu_parity import make_dg
    dg = make_dg("eg", 3, N, 2, "ec", sflux, "reflect")
    odg = orc.DGSEM(dg)
    q = PT.random_state(dg)
    dq_o = np.zeros_like(q)
    odg(dq_o, q, 0.0, increment=False)
    dqd = PT.to_dev(np.zeros_like(q))
    dg(dqd, PT.to_dev(q), 0.0, increment=False)
    PT.assert_parity(f"Euler-gravity 3-D EC/{sflux} N={N} tendency", PT.to_host(dqd), dq_o, 1e-12)

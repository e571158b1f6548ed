"""after_stage callbacks of solve! (src/odesolvers.jl:10-11,23,54,119,378)
through the C ABI's stage callback: the stage times and stage states the GPU
solvers report equal the oracle's, observing the stages leaves the run
unchanged, and a callback that changes q (LSRK) changes the next stage."""
import math

import numpy as np
import pytest

import atum_b200 as A
import parity as PT
import problems as P

pytestmark = pytest.mark.gpu


def _gpu_record(case, timeend, solver_kind):
    import torch
    q = PT.to_dev(case.q0)
    if solver_kind == "ARK23":
        s = A.ARK23(case.dg, case.lindg, q, case.dt, split_rhs=case.split_rhs)
    else:
        s = getattr(A, solver_kind)(case.dg, q, case.dt)
    seen = []

    def cb(t, qs):
        seen.append((t, qs.clone() if isinstance(qs, torch.Tensor) else torch.stack(qs).clone()))

    n = A.solve_(q, timeend, s, after_stage=cb, adjust_final=case.adjust_final)
    torch.cuda.synchronize()
    return n, PT.to_host(q), [(t, PT.to_host(x)) for t, x in seen]


def _oracle_record(orc, case, timeend, solver_kind):
    odg = orc.DGSEM(case.dg) if case.dg is not None else None
    q = case.q0.copy()
    if solver_kind == "ARK23":
        s = orc.ARK23(odg, orc.DGSEM(case.lindg), q, case.dt, split_rhs=case.split_rhs)
    else:
        s = getattr(orc, solver_kind)(odg, q, case.dt)
    seen = []
    s.set_after_stage(lambda ex, im, qs: seen.append(((ex, im), qs.reshape(case.q0.shape))))
    n = orc.solve_(q, timeend, s, adjust_final=case.adjust_final)
    return n, q, seen


@pytest.mark.parametrize("kind", ["LSRK54", "LSRK144"])
def test_lsrk_after_stage_matches_oracle(orc, kind):
    case = P.vortex_c1()
    T = 2.5 * case.dt  # three steps, the last one shortened by solve!
    n_g, q_g, seen_g = _gpu_record(case, T, kind)
    n_o, q_o, seen_o = _oracle_record(orc, case, T, kind)
    assert n_g == n_o == 3
    assert len(seen_g) == len(seen_o) == 3 * (5 if kind == "LSRK54" else 14)
    for (tg, xg), ((te, ti), xo) in zip(seen_g, seen_o):
        assert tg == te == ti
        PT.assert_parity(f"{kind} stage at t={tg:.4f}", xg, xo, 1e-12)
    # observing the stages changes nothing
    q = PT.to_dev(case.q0)
    s = getattr(A, kind)(case.dg, q, case.dt)
    assert A.solve_(q, T, s) == 3
    assert np.array_equal(PT.to_host(q), q_g)


def test_rlsrk_after_stage_matches_oracle(orc):
    case = P.square_1d("euler")
    T = 2 * case.dt
    n_g, q_g, seen_g = _gpu_record(case, T, "RLSRK54")
    n_o, q_o, seen_o = _oracle_record(orc, case, T, "RLSRK54")
    assert n_g == n_o and len(seen_g) == len(seen_o) == 5 * n_g
    for (tg, xg), ((te, _), xo) in zip(seen_g, seen_o):
        assert tg == te
        PT.assert_parity(f"RLSRK54 stage at t={tg:.4f}", xg, xo, 1e-11)
    PT.assert_parity("RLSRK54 result", q_g, q_o, 1e-11)


@pytest.mark.parametrize("split_rhs", [True, False])
def test_ark23_after_stage_matches_oracle(orc, split_rhs):
    """IMEX advection: the general ARK23 path (split_rhs = true) and the
    accumulated one with the banded solve (split_rhs = false)."""
    case = P.imex_advection_2d(N=3, K=4, split_rhs=split_rhs)
    T = 3 * case.dt
    n_g, q_g, seen_g = _gpu_record(case, T, "ARK23")
    n_o, q_o, seen_o = _oracle_record(orc, case, T, "ARK23")
    assert n_g == n_o and len(seen_g) == len(seen_o) == 2 * n_g
    c2 = 2 - math.sqrt(2)
    for k, ((tg, xg), (to, xo)) in enumerate(zip(seen_g, seen_o)):
        assert tg == to
        step, stage = divmod(k, 2)
        assert tg[0] == pytest.approx((step + (c2 if stage == 0 else 1.0)) * case.dt, rel=1e-14)
        PT.assert_parity(f"ARK23 split_rhs={split_rhs} stage {stage + 2} of step {step + 1}", xg, xo, 1e-12)
    PT.assert_parity(f"ARK23 split_rhs={split_rhs} result", q_g, q_o, 1e-12)


def test_ark23_fused_bubble_after_stage_matches_oracle(orc):
    """The fused ARK23 stage kernel (rising bubble, N = 3): stage states
    against the oracle's, within its schedule spread."""
    build = lambda k: P.bubble_3d(N=3, K=4, imex=True, steps=2, fd_kernel=k)  # noqa: E731
    case = build("per_dir")
    T = 2 * case.dt
    _, q_g, seen_g = _gpu_record(case, T, "ARK23")
    _, q_o, seen_o = _oracle_record(orc, case, T, "ARK23")
    _, _, seen_s = _oracle_record(orc, build("per_dir_symmetric"), T, "ARK23")
    assert len(seen_g) == len(seen_o) == 4
    for (tg, xg), (_, xo), (_, xs) in zip(seen_g, seen_o, seen_s):
        PT.assert_parity(f"fused ARK23 bubble stage at t={tg[0]:.4f}", xg, xo, 1e-12,
                         spread=PT.field_rel_errors(xs, xo))


def test_after_stage_changes_carry_into_the_next_stage():
    """A callback that adds eps to the density after every LSRK stage: on a
    periodic mesh the operator conserves mass, so the total mass grows by
    exactly (stages x eps x sum MJ), up to rounding."""
    import torch
    case = P.vortex_c1()
    q = PT.to_dev(case.q0)
    s = A.LSRK54(case.dg, q, case.dt)
    eps = 1e-6
    mj = PT.to_dev(case.dg.MJ)
    m0 = float((mj * q[0]).sum())

    def bump(t, qq):
        qq[0] += eps

    assert A.solve_(q, 2 * case.dt, s, after_stage=bump) == 2
    m1 = float((mj * q[0]).sum())
    expect = 10 * eps * float(mj.sum())
    assert abs((m1 - m0) - expect) <= 1e-9 * expect


def test_after_stage_exception_stops_the_solve():
    case = P.vortex_c1()
    q = PT.to_dev(case.q0)
    s = A.LSRK54(case.dg, q, case.dt)

    def boom(t, qq):
        raise ValueError("stop here")

    with pytest.raises(ValueError, match="stop here"):
        A.solve_(q, 3 * case.dt, s, after_stage=boom)

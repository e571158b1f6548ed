"""CPU checks of the oracle's after_stage hook (src/odesolvers.jl:54,119,378):
how often and with which stage times it is called, and that observing stages
does not change a run."""
import math

import numpy as np
import pytest

import problems as P


def _record(orc, case, nsteps, kind):
    odg = orc.DGSEM(case.dg) if case.dg is not None else None
    q = case.q0.copy()
    if kind == "ARK23":
        s = orc.ARK23(odg, orc.DGSEM(case.lindg), q, case.dt, split_rhs=case.split_rhs)
    else:
        s = getattr(orc, kind)(odg, q, case.dt)
    seen = []
    s.set_after_stage(lambda ex, im, qs: seen.append((ex, im, qs)))
    s.step(q, nsteps)
    s.set_after_stage(None)
    return q, seen


@pytest.mark.parametrize("kind,nst", [("LSRK54", 5), ("LSRK144", 14)])
def test_lsrk_stage_calls(orc, kind, nst):
    case = P.euler_wave(2, N=2, K=3, form="weak")
    q_plain = case.q0.copy()
    s = getattr(orc, kind)(orc.DGSEM(case.dg), q_plain, case.dt)
    s.step(q_plain, 2)
    q, seen = _record(orc, case, 2, kind)
    assert len(seen) == 2 * nst
    assert np.array_equal(q, q_plain)
    # the last stage's state is the step's result; stage times within [t, t + dt]
    assert np.array_equal(seen[-1][2], q.reshape(-1))
    for i, (ex, im, _) in enumerate(seen):
        assert ex == im
        step = i // nst
        assert step * case.dt - 1e-15 <= ex <= (step + 1) * case.dt + 1e-15
    assert seen[0][0] == 0.0


def test_ark23_stage_calls(orc):
    case = P.imex_advection_2d(N=2, K=3)
    q, seen = _record(orc, case, 3, "ARK23")
    assert len(seen) == 6  # stages 2 and 3 of every step
    c2 = 2 - math.sqrt(2)
    for k in range(3):
        ex2, im2, _ = seen[2 * k]
        ex3, im3, _ = seen[2 * k + 1]
        assert ex2 == pytest.approx((k + c2) * case.dt, rel=1e-15) and im2 == ex2
        assert ex3 == pytest.approx((k + 1) * case.dt, rel=1e-15) and im3 == ex3

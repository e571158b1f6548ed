"""The CPU oracle against the reference's own golden values.

Each case restates one of the reference's integration tests
(test/advection, test/euler, test/shallow_water, test/euler_gravity) and
checks the oracle's result against the value the reference test asserts, with
the reference's tolerance (`≈`, i.e. rtol = sqrt(eps), unless the test states
another).  These pins are what make the oracle trustworthy for GPU parity.
"""
import math

import numpy as np
import pytest

import problems as P

RTOL = math.sqrt(np.finfo(np.float64).eps)


def run_oracle(orc, case):
    dg = orc.DGSEM(case.dg) if case.dg is not None else None
    q = np.ascontiguousarray(case.q0.copy())
    if case.solver == "ARK23":
        lin = orc.DGSEM(case.lindg)
        s = orc.ARK23(dg, lin, q, case.dt, split_rhs=case.split_rhs)
    else:
        s = getattr(orc, case.solver)(dg, q, case.dt)
    steps = orc.solve_(q, case.timeend, s, adjust_final=case.adjust_final)
    return dg, q, steps


def l2_error(orc, dg, q, qe):
    return orc.weightednorm(dg, np.ascontiguousarray(q - qe))


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("form", ["weak", "fd_central"])
def test_advection_wave(orc, dim, form):
    case = P.advection_wave(dim, form=form)
    dg, q, _ = run_oracle(orc, case)
    err = l2_error(orc, dg, q, case.exact(case.timeend))
    assert err == pytest.approx(P.golden(f"advection/wave_{dim}d", form), rel=RTOL)


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("form", ["weak", "fd_ec"])
def test_euler_wave(orc, dim, form):
    case = P.euler_wave(dim, form=form)
    dg, q, steps = run_oracle(orc, case)
    if dim == 3:
        assert steps == 1  # test/euler/wave_3d.jl:53 (timeend = dt)
    err = l2_error(orc, dg, q, case.exact(case.timeend))
    assert err == pytest.approx(P.golden(f"euler/wave_{dim}d", form), rel=RTOL)


@pytest.mark.parametrize("form", ["weak", "fd_ec"])
def test_isentropic_vortex(orc, form):
    case = P.isentropic_vortex(form=form)
    dg, q, steps = run_oracle(orc, case)
    assert steps == 40
    err = l2_error(orc, dg, q, case.exact(case.timeend))
    assert err == pytest.approx(P.golden("euler/isentropicvortex", form), rel=RTOL)


@pytest.mark.parametrize("lawname,key", [("advection", "advection/entropy_conservation_1d"),
                                         ("euler", "euler/entropy_conservation_1d"),
                                         ("shallow_water", "shallow_water/entropy_conservation_1d")])
def test_entropy_conservation(orc, lawname, key):
    case = P.square_1d(lawname)
    dg = orc.DGSEM(case.dg)
    q = case.q0.copy()
    eta0 = orc.entropyintegral(dg, q)
    s = orc.RLSRK54(dg, q, case.dt)
    orc.solve_(q, case.timeend, s)
    etaf = orc.entropyintegral(dg, q)
    tol = P.goldens()[key]["entropy_tol_eps"] * np.finfo(np.float64).eps
    assert abs((etaf - eta0) / abs(eta0)) <= tol


@pytest.mark.parametrize("form", ["weak", "fd_central"])
@pytest.mark.parametrize("split_rhs", [True, False])
def test_imex_advection(orc, form, split_rhs):
    case = P.imex_advection_2d(form=form, split_rhs=split_rhs)
    dg, q, _ = run_oracle(orc, case)
    err = l2_error(orc, dg, q, case.exact(case.timeend))
    assert err == pytest.approx(P.golden("advection/imex_wave_2d", form), rel=RTOL)


@pytest.mark.slow
def test_linear_euler_gravity(orc):
    errs = []
    for level, K in ((1, 5), (2, 10)):
        case = P.linear_euler_gravity(K=K)
        lin = orc.DGSEM(case.lindg)
        q = case.q0.copy()
        s = orc.ARK23(None, lin, q, case.dt, split_rhs=True)
        orc.solve_(q, case.timeend, s, adjust_final=False)
        err = orc.weightednorm(lin, np.ascontiguousarray(q - case.extra["qref"]))
        errs.append(err)
        assert err == pytest.approx(P.golden("euler_gravity/linear", "weak", level), rel=1e-3)
    rate = math.log2(errs[0] / errs[1])
    assert abs(rate - 5) <= 0.1

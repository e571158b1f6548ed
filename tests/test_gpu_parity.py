"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle.

Tolerances (metric in tests/parity.py): one operator application and one
time step <= 1e-12 relative per DOF; 100 steps <= 1e-10.
"""
import math

import numpy as np
import pytest

import atum_b200 as A
import parity as PT
import problems as P

pytestmark = pytest.mark.gpu

FLUX = {"central": A.CentralFlux(), "rusanov": A.RusanovFlux(), "ec": A.EntropyConservativeFlux(),
        "kg": A.KennedyGruberFlux(), "roe": A.RoeFlux(), "matrix": A.MatrixFlux()}


def make_dg(law, dim, N, K, form, sflux, bc="periodic", dirs=None, kernel="per_dir", ordering="cartesian"):
    cell = A.LobattoCell(*([N + 1] * dim))
    if law in ("eg", "leg"):
        L = 1000.0
        verts = [np.linspace(0, L, K + 1)] * dim
    else:
        verts = [np.linspace(-1.0, 1.0, K + 1) ** 1] * dim
        # a non-uniform last dimension exercises per-element metrics
        v = np.linspace(-1.0, 1.0, K + 1)
        verts[-1] = v + 0.1 * np.sin(np.pi * v) / max(K, 1) * (v > -1) * (v < 1)
    periodic = [True] * dim
    if bc != "periodic":
        periodic[-1] = False
    problem = None
    if law == "adv":
        problem = A.InflowZero() if bc == "inflow" else A.DummyProblem()
        lw = A.AdvectionLaw(dim, tuple([1.0, -0.6, 0.3][:dim]), problem=problem)
    elif law == "euler":
        if bc == "dirichlet":
            problem = A.DirichletByTag([1.0] + [0.0] * dim + [2.5], [0.125] + [0.0] * dim + [0.25])
        elif bc == "reflect":
            problem = A.ReflectiveWall()
        lw = A.EulerLaw(dim, problem=problem)
    elif law in ("eg", "leg", "eg_pde", "eg_cor"):
        kw = {}
        if law == "eg_cor":
            kw = dict(omega=(0.0, 0.0, 2 * 7.29212e-5)) if dim == 3 else dict(omega=(0.0, 0.0, 1e-4))
            pr = A.Coriolis(bc=1 if bc == "reflect" else 0, referencestate=P._bubble_reference, **kw)
        elif bc == "reflect":
            pr = A.ReflectiveWall(referencestate=P._bubble_reference)
        else:
            pr = A.AbstractProblem(referencestate=P._bubble_reference)
        lw = A.EulerGravityLaw(dim, grav=9.81, pde_level_balance=(law == "eg_pde"), problem=pr)
        if law == "leg":
            lw = A.LinearEulerGravityLaw(lw)
    elif law in ("sw", "sw_topo", "sw_cor"):
        if law == "sw_cor":
            pr = A.Coriolis((0.0, 0.0, 0.3), bc=1 if bc == "reflect" else 0)
        else:
            pr = A.ReflectiveWall() if bc == "reflect" else A.DummyProblem()
        lw = A.ShallowWaterLaw(dim, grav=9.81, topography=(law == "sw_topo"), problem=pr)
        if law == "sw_topo":
            def bath(x):
                b = 0.2 * np.exp(-np.sum(x * x, axis=0) * 2)
                return b, [-4 * x[d] * b for d in range(dim)]
            lw.bathymetry = bath
    else:
        raise ValueError(law)
    grid = A.brickgrid(cell, verts, periodic=periodic, ordering=ordering)
    if law in ("eg", "leg", "eg_pde", "eg_cor"):
        grid = A.brickgrid(cell, [np.linspace(0, 1000.0, K + 1)] * dim, periodic=periodic, ordering=ordering)
    vf = A.WeakForm() if form == "weak" else A.FluxDifferencingForm(FLUX[form], kernel)
    return A.DGSEM(law=lw, grid=grid, volume_form=vf, surface_numericalflux=FLUX[sflux], directions=dirs)


def _cases():
    out = []
    for dim, N, K in ((1, 4, 5), (2, 3, 3), (3, 2, 2)):
        for form in ("weak", "central"):
            for sf in ("central", "rusanov"):
                out.append(("adv", dim, N, K, form, sf, "periodic"))
        out.append(("adv", dim, N, K, "weak", "rusanov", "inflow"))
        for form in ("weak", "central", "ec", "kg"):
            for sf in ("central", "rusanov", "ec", "kg", "roe", "matrix"):
                out.append(("euler", dim, N, K, form, sf, "periodic"))
        out.append(("euler", dim, N, K, "ec", "rusanov", "reflect"))
        out.append(("euler", dim, N, K, "ec", "rusanov", "dirichlet"))
        for form in ("weak", "central", "ec", "kg"):
            for sf in ("central", "rusanov", "ec", "kg", "roe", "matrix"):
                out.append(("eg", dim, N, K, form, sf, "reflect"))
        out.append(("eg_pde", dim, N, K, "weak", "roe", "reflect"))
        out.append(("eg_pde", dim, N, K, "ec", "rusanov", "reflect"))
        out.append(("eg_cor", dim, N, K, "ec", "rusanov", "reflect"))
        out.append(("eg_cor", dim, N, K, "weak", "rusanov", "reflect"))
        for form in ("weak", "central"):
            for sf in ("central", "rusanov"):
                out.append(("leg", dim, N, K, form, sf, "reflect"))
        for form in ("weak", "central", "ec"):
            for sf in ("central", "rusanov", "ec", "roe"):
                out.append(("sw", dim, N, K, form, sf, "periodic"))
        out.append(("sw", dim, N, K, "ec", "roe", "reflect"))
        out.append(("sw_topo", dim, N, K, "ec", "rusanov", "periodic"))
        out.append(("sw_topo", dim, N, K, "weak", "rusanov", "periodic"))
        out.append(("sw_cor", dim, N, K, "ec", "rusanov", "periodic"))
    return out


@pytest.mark.parametrize("case", _cases(), ids=lambda c: "-".join(map(str, c)))
def test_operator_apply(orc, case):
    law, dim, N, K, form, sf, bc = case
    dg = make_dg(law, dim, N, K, form, sf, bc)
    odg = orc.DGSEM(dg)
    q = PT.random_state(dg)
    rng = np.random.default_rng(7)
    dq0 = rng.standard_normal(q.shape)
    for inc in (False, True):
        dq_o = dq0.copy()
        odg(dq_o, q, 0.0, increment=inc)
        qd, dqd = PT.to_dev(q), PT.to_dev(dq0)
        dg(dqd, qd, 0.0, increment=inc)
        err = PT.rel_dof_error(PT.to_host(dqd), dq_o)
        assert err <= 1e-12, (case, inc, err)


@pytest.mark.parametrize("law,form,sf", [("adv", "weak", "rusanov"), ("euler", "ec", "rusanov"),
                                         ("euler", "kg", "roe"), ("sw", "ec", "rusanov")])
@pytest.mark.parametrize("dim", [1, 2, 3])
def test_single_element_periodic(orc, law, form, sf, dim):
    """K = 1 per dimension: every face's neighbour is the element itself."""
    dg = make_dg(law, dim, 3, 1, form, sf)
    odg = orc.DGSEM(dg)
    q = PT.random_state(dg)
    dq_o = np.zeros_like(q)
    odg(dq_o, q, 0.0, increment=False)
    qd = PT.to_dev(q)
    dqd = PT.to_dev(np.zeros_like(q))
    dg(dqd, qd, 0.0, increment=False)
    assert PT.rel_dof_error(PT.to_host(dqd), dq_o) <= 1e-12


def test_stacked_ordering_matches_cartesian(orc):
    """The stacked element ordering (vertical columns contiguous) gives the
    oracle's operator too."""
    dg = make_dg("euler", 3, 3, 3, "ec", "rusanov", ordering="stacked")
    odg = orc.DGSEM(dg)
    q = PT.random_state(dg)
    dq_o = np.zeros_like(q)
    odg(dq_o, q, 0.0, increment=False)
    qd = PT.to_dev(q)
    dqd = PT.to_dev(np.zeros_like(q))
    dg(dqd, qd, 0.0, increment=False)
    assert PT.rel_dof_error(PT.to_host(dqd), dq_o) <= 1e-12


@pytest.mark.parametrize("kernel", ["per_dir", "per_dir_symmetric", "naive"])
@pytest.mark.parametrize("dim", [2, 3])
def test_fd_kernel_types(orc, kernel, dim):
    dg = make_dg("eg", dim, 3, 2, "ec", "rusanov", "reflect", kernel=kernel)
    odg = orc.DGSEM(dg)
    q = PT.random_state(dg)
    dq_o = np.zeros_like(q)
    odg(dq_o, q, 0.0, increment=False)
    dqd = PT.to_dev(np.zeros_like(q))
    dg(dqd, PT.to_dev(q), 0.0, increment=False)
    assert PT.rel_dof_error(PT.to_host(dqd), dq_o) <= 1e-12


@pytest.mark.parametrize("dirs", [(1,), (2,), (1, 2)])
def test_directions_subsets(orc, dirs):
    for law, form in (("euler", "ec"), ("leg", "weak"), ("adv", "central")):
        dg = make_dg(law, 2, 3, 3, form, "rusanov", "reflect" if law != "adv" else "inflow", dirs=dirs,
                     ordering="stacked")
        odg = orc.DGSEM(dg)
        q = PT.random_state(dg)
        dq_o = np.zeros_like(q)
        odg(dq_o, q, 0.0, increment=False)
        dqd = PT.to_dev(np.zeros_like(q))
        dg(dqd, PT.to_dev(q), 0.0, increment=False)
        assert PT.rel_dof_error(PT.to_host(dqd), dq_o) <= 1e-12, (law, dirs)


@pytest.mark.parametrize("N", [1, 2, 5, 6, 7])
def test_orders(orc, N):
    for dim in (2, 3):
        K = 2 if dim == 3 else 3
        dg = make_dg("euler", dim, N, K, "ec", "rusanov", "periodic")
        odg = orc.DGSEM(dg)
        q = PT.random_state(dg)
        dq_o = np.zeros_like(q)
        odg(dq_o, q, 0.0, increment=False)
        dqd = PT.to_dev(np.zeros_like(q))
        dg(dqd, PT.to_dev(q), 0.0, increment=False)
        assert PT.rel_dof_error(PT.to_host(dqd), dq_o) <= 1e-12, (N, dim)


# ------------------------------------------------------------- solvers
def _run_both(orc, case, nsteps=None, solver=None):
    solver = solver or case.solver
    q_o = case.q0.copy()
    q_d = PT.to_dev(case.q0)
    odg = orc.DGSEM(case.dg) if case.dg is not None else None
    if solver == "ARK23":
        olin = orc.DGSEM(case.lindg)
        so = orc.ARK23(odg, olin, q_o, case.dt, split_rhs=case.split_rhs)
        sd = A.ARK23(case.dg, case.lindg, q_d, case.dt, split_rhs=case.split_rhs)
    else:
        so = getattr(orc, solver)(odg, q_o, case.dt)
        sd = getattr(A, solver)(case.dg, q_d, case.dt)
    if nsteps is None:
        n_o = orc.solve_(q_o, case.timeend, so, adjust_final=case.adjust_final)
        n_d = A.solve_(q_d, case.timeend, sd, adjust_final=case.adjust_final)
        assert n_o == n_d
    else:
        so.step(q_o, nsteps)
        sd.step(q_d, nsteps)
    return q_o, PT.to_host(q_d), odg


@pytest.mark.parametrize("solver", ["LSRK54", "LSRK144"])
def test_one_step(orc, solver):
    for case in (P.euler_wave(3, form="fd_ec"), P.euler_wave(2, form="weak"), P.advection_wave(2, form="weak")):
        q_o, q_d, _ = _run_both(orc, case, nsteps=1, solver=solver)
        assert PT.rel_dof_error(q_d, q_o) <= 1e-12, case.name


def test_vortex_c1_100_steps(orc):
    case = P.vortex_c1()
    q_o, q_d, odg = _run_both(orc, case, nsteps=case.extra["steps"])
    assert np.isfinite(q_o).all()
    err = PT.rel_dof_error(q_d, q_o)  # strict: the field's own magnitude
    assert err <= 1e-10, err


def _gpu_states(case, counts):
    q = PT.to_dev(case.q0)
    if case.solver == "ARK23":
        s = A.ARK23(case.dg, case.lindg, q, case.dt, split_rhs=case.split_rhs)
    else:
        s = getattr(A, case.solver)(case.dg, q, case.dt)
    out, done = [], 0
    for n in counts:
        s.step(q, n - done)
        done = n
        out.append(PT.to_host(q))
    return out


def test_bubble_lsrk_steps(orc):
    build = lambda k: P.bubble_3d(N=3, K=3, imex=False, steps=5, fd_kernel=k)  # noqa: E731
    case = build("per_dir")
    g = _gpu_states(case, [1, 5])
    o, spread = PT.schedule_spread(orc, build, [1, 5])
    for n, gi, oi, si, tol in zip((1, 5), g, o, spread, (1e-12, 1e-11)):
        PT.assert_parity(f"bubble LSRK54 N=3 3^3, {n} step(s)", gi, oi, tol, spread=si,
                         floors=PT.natural_floors(case.dg, oi))


@pytest.mark.parametrize("form", ["weak", "fd_central"])
@pytest.mark.parametrize("split_rhs", [True, False])
def test_imex_advection(orc, form, split_rhs):
    case = P.imex_advection_2d(form=form, split_rhs=split_rhs)
    q_o, q_d, odg = _run_both(orc, case, nsteps=1)
    assert PT.rel_dof_error(q_d, q_o) <= 1e-12
    q_o, q_d, odg = _run_both(orc, case)
    assert PT.rel_dof_error(q_d, q_o) <= 1e-10
    err = orc.weightednorm(odg, np.ascontiguousarray(q_d - case.exact(case.timeend)))
    assert err == pytest.approx(P.golden("advection/imex_wave_2d", form), rel=math.sqrt(2.2e-16))


def test_imex_bubble(orc):
    build = lambda k: P.bubble_3d(N=3, K=4, imex=True, steps=3, fd_kernel=k)  # noqa: E731
    case = build("per_dir")
    g = _gpu_states(case, [1, 3])
    o, spread = PT.schedule_spread(orc, build, [1, 3])
    for n, gi, oi, si, tol in zip((1, 3), g, o, spread, (1e-12, 1e-11)):
        PT.assert_parity(f"bubble ARK23 N=3 4^3, {n} step(s)", gi, oi, tol, spread=si,
                         floors=PT.natural_floors(case.dg, oi))


def test_linear_euler_gravity_short(orc):
    case = P.linear_euler_gravity(K=5)
    lin = case.lindg
    q_o = case.q0.copy()
    q_d = PT.to_dev(case.q0)
    olin = orc.DGSEM(lin)
    so = orc.ARK23(None, olin, q_o, case.dt)
    sd = A.ARK23(None, lin, q_d, case.dt)
    so.step(q_o, 50)
    sd.step(q_d, 50)
    # weak form (no flux-differencing schedule): the oracle's spread is its
    # response to the initial state moved by one ulp
    _, (spread,) = PT.ulp_spread(orc, case, [50])
    PT.assert_parity("linear Euler-gravity IMEX K=5, 50 steps", PT.to_host(q_d), q_o, 1e-10, spread=spread,
                     floors=PT.natural_floors(lin, q_o))


@pytest.mark.parametrize("lawname", ["advection", "euler", "shallow_water"])
def test_rlsrk(orc, lawname):
    case = P.square_1d(lawname)
    q_o, q_d, odg = _run_both(orc, case, nsteps=3)
    assert PT.rel_dof_error(q_d, q_o) <= 1e-11


# ---------------------------------------------- reference tests on the GPU
@pytest.mark.parametrize("form", ["weak", "fd_ec"])
def test_gpu_isentropic_vortex_golden(orc, form):
    case = P.isentropic_vortex(form=form)
    q = PT.to_dev(case.q0)
    s = A.LSRK54(case.dg, q, case.dt)
    assert A.solve_(q, case.timeend, s) == 40
    qe = PT.to_dev(case.exact(case.timeend))
    err = A.weightednorm(case.dg, (q - qe).contiguous())
    assert err == pytest.approx(P.golden("euler/isentropicvortex", form), rel=math.sqrt(2.2e-16))


@pytest.mark.parametrize("form", ["weak", "fd_ec"])
def test_gpu_euler_wave_3d_one_step_golden(form):
    case = P.euler_wave(3, form=form)
    q = PT.to_dev(case.q0)
    s = A.LSRK54(case.dg, q, case.dt)
    assert A.solve_(q, case.timeend, s) == 1
    err = A.weightednorm(case.dg, (q - PT.to_dev(case.exact(case.timeend))).contiguous())
    assert err == pytest.approx(P.golden("euler/wave_3d", form), rel=math.sqrt(2.2e-16))


@pytest.mark.parametrize("lawname,key", [("advection", "advection/entropy_conservation_1d"),
                                         ("euler", "euler/entropy_conservation_1d"),
                                         ("shallow_water", "shallow_water/entropy_conservation_1d")])
def test_gpu_entropy_conservation(lawname, key):
    case = P.square_1d(lawname)
    q = PT.to_dev(case.q0)
    eta0 = A.entropyintegral(case.dg, q)
    s = A.RLSRK54(case.dg, q, case.dt)
    A.solve_(q, case.timeend, s)
    etaf = A.entropyintegral(case.dg, q)
    tol = P.goldens()[key]["entropy_tol_eps"] * np.finfo(np.float64).eps
    assert abs((etaf - eta0) / abs(eta0)) <= tol


# ------------------------------------------------------- invariants
def test_conservation_periodic():
    """Mass and total energy are conserved to round-off on a periodic mesh."""
    case = P.vortex_c1()
    q = PT.to_dev(case.q0)
    mj = PT.to_dev(case.dg.MJ)
    m0 = [float((mj * q[s]).sum()) for s in range(4)]
    s = A.LSRK54(case.dg, q, case.dt)
    s.step(q, 100)
    m1 = [float((mj * q[s]).sum()) for s in range(4)]
    for c in (0, 3):
        assert abs(m1[c] - m0[c]) <= 1e-13 * abs(m0[c]), (c, m0[c], m1[c])


def test_determinism():
    case = P.bubble_3d(N=3, K=3, imex=False, steps=2)
    outs = []
    for _ in range(2):
        q = PT.to_dev(case.q0)
        s = A.LSRK54(case.dg, q, case.dt)
        s.step(q, 2)
        outs.append(PT.to_host(q))
    assert np.array_equal(outs[0], outs[1])


def test_convergence_order():
    """Euler density wave in 2-D: rate between K=5 and K=10 approaches N+1."""
    errs = []
    for K in (5, 10):
        case = P.euler_wave(2, K=K, form="fd_ec")
        q = PT.to_dev(case.q0)
        s = A.LSRK54(case.dg, q, case.dt)
        A.solve_(q, case.timeend, s)
        errs.append(A.weightednorm(case.dg, (q - PT.to_dev(case.exact(case.timeend))).contiguous()))
    assert errs[0] == pytest.approx(P.golden("euler/wave_2d", "fd_ec", 1), rel=1e-8)
    assert errs[1] == pytest.approx(P.golden("euler/wave_2d", "fd_ec", 2), rel=1e-8)
    rate = math.log2(errs[0] / errs[1])
    assert abs(rate - 5) <= 0.4


def test_nonfinite_detection():
    case = P.vortex_c1()
    q = PT.to_dev(case.q0)
    A.measures.check_finite(case.dg, q)
    q[1, 3, 2] = float("nan")
    with pytest.raises(A._lib.AtbError) as ei:
        A.measures.check_finite(case.dg, q)
    assert ei.value.code == -4

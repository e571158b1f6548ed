"""FP32-flux precision form against the FP64 path (both on the GPU; the FP64
path matches the CPU oracle to 1e-12, see test_gpu_parity.py).

The error measure is the reference's own weighted L2 norm (src/measures.jl),
relative: ||q_fp32flux - q_fp64|| / ||q_fp64||, bound 1e-6.  For the rising
bubble the error relative to the bubble's perturbation (q - q_background) is
reported too.
"""
import numpy as np
import pytest

import atum_b200 as A
import parity as PT
import problems as P

pytestmark = pytest.mark.gpu


def _rel(dg, a, b):
    import torch
    return A.weightednorm(dg, (a - b).contiguous()) / A.weightednorm(dg, b)


def test_bubble_imex_fp32flux(capsys):
    import torch
    c64 = P.bubble_3d(N=4, K=6, imex=True, steps=40)
    c32 = P.bubble_3d(N=4, K=6, imex=True, steps=40, precision="fp32flux")
    q64, q32 = PT.to_dev(c64.q0), PT.to_dev(c32.q0)
    s64 = A.ARK23(c64.dg, c64.lindg, q64, c64.dt, split_rhs=False)
    s32 = A.ARK23(c32.dg, c32.lindg, q32, c32.dt, split_rhs=False)
    s64.step(q64, 40)
    s32.step(q32, 40)
    rel = _rel(c64.dg, q32, q64)
    # error relative to the perturbation the bubble made
    qb = PT.to_dev(P.bubble_3d(N=4, K=6, imex=True, steps=1).q0)
    pert = A.weightednorm(c64.dg, (q64 - qb).contiguous())
    rel_pert = A.weightednorm(c64.dg, (q32 - q64).contiguous()) / pert
    with capsys.disabled():
        print(f"\n  bubble 3-D IMEX, 40 steps: rel L2 {rel:.2e}, rel to perturbation {rel_pert:.2e}")
    assert rel <= 1e-6
    assert rel_pert <= 1e-3


def test_vortex_fp32flux():
    c64 = P.vortex_c1()
    c32 = P.vortex_c1(precision="fp32flux")
    q64, q32 = PT.to_dev(c64.q0), PT.to_dev(c32.q0)
    A.LSRK54(c64.dg, q64, c64.dt).step(q64, 100)
    A.LSRK54(c32.dg, q32, c32.dt).step(q32, 100)
    assert _rel(c64.dg, q32, q64) <= 1e-6


def test_vortex_kg_fp32flux():
    """Kennedy-Gruber volume flux in the FP32-flux form (Euler)."""
    c64 = P.vortex_c1(vflux="kg")
    c32 = P.vortex_c1(vflux="kg", precision="fp32flux")
    q64, q32 = PT.to_dev(c64.q0), PT.to_dev(c32.q0)
    A.LSRK54(c64.dg, q64, c64.dt).step(q64, 100)
    A.LSRK54(c32.dg, q32, c32.dt).step(q32, 100)
    assert _rel(c64.dg, q32, q64) <= 1e-6


def test_bubble_imex_kg_fp32flux():
    """Kennedy-Gruber FP32-flux form on the rising bubble (Euler-gravity,
    IMEX): the FP64 pressure average keeps the hydrostatic balance."""
    c64 = P.bubble_3d(N=4, K=6, imex=True, steps=40, vflux="kg")
    c32 = P.bubble_3d(N=4, K=6, imex=True, steps=40, vflux="kg", precision="fp32flux")
    q64, q32 = PT.to_dev(c64.q0), PT.to_dev(c32.q0)
    A.ARK23(c64.dg, c64.lindg, q64, c64.dt, split_rhs=False).step(q64, 40)
    A.ARK23(c32.dg, c32.lindg, q32, c32.dt, split_rhs=False).step(q32, 40)
    assert _rel(c64.dg, q32, q64) <= 1e-6


def test_shallow_water_fp32flux_and_mass():
    import torch
    c64 = P.sw_fplane(K=8, steps=50)
    c32 = P.sw_fplane(K=8, steps=50, precision="fp32flux")
    q64, q32 = PT.to_dev(c64.q0), PT.to_dev(c32.q0)
    A.LSRK54(c64.dg, q64, c64.dt).step(q64, 50)
    A.LSRK54(c32.dg, q32, c32.dt).step(q32, 50)
    assert _rel(c64.dg, q32, q64) <= 1e-6
    mj = PT.to_dev(c32.dg.MJ)
    m0 = float((mj * PT.to_dev(c32.q0)[0]).sum())
    m1 = float((mj * q32[0]).sum())
    assert abs(m1 - m0) <= 1e-13 * abs(m0)


@pytest.mark.parametrize("precision", ["fp64", "fp32flux"])
def test_lake_at_rest(precision):
    """Well-balancedness with bathymetry and Coriolis: h + b = const, u = 0
    stays at rest to round-off."""
    c = P.sw_fplane(K=8, lake_at_rest=True, precision=precision, steps=20)
    q = PT.to_dev(c.q0)
    A.LSRK54(c.dg, q, c.dt).step(q, 20)
    umax = float(q[1:3].abs().max() / q[0].abs().max())
    assert umax <= 1e-12, umax
    assert float((q[0] - PT.to_dev(c.q0)[0]).abs().max()) <= 1e-10


def test_fp32flux_rejected_where_not_built():
    cell = A.LobattoCell(3, 3)
    grid = A.brickgrid(cell, ([0, 1, 2], [0, 1, 2]), periodic=(True, True))
    dg = A.DGSEM(law=A.EulerLaw(2), grid=grid, surface_numericalflux=A.RusanovFlux(), precision="fp32flux")
    with pytest.raises(A._lib.AtbError):
        dg.device


_SFLUX = {"ec": A.EntropyConservativeFlux(), "kg": A.KennedyGruberFlux(), "roe": A.RoeFlux(),
          "matrix": A.MatrixFlux()}


@pytest.mark.parametrize("law,sflux", [("euler", "roe"), ("euler", "matrix"), ("euler", "ec"), ("euler", "kg"),
                                       ("eg", "roe"), ("eg", "matrix"), ("eg", "ec"), ("sw", "roe"),
                                       ("sw", "ec"), ("sw_topo", "roe"), ("sw_topo", "ec")])
def test_fp32flux_surface_fluxes(law, sflux):
    """Every surface flux has an FP32-flux form (src/balancelaws/euler.jl:91-138,
    198-256; euler_gravity.jl:149-198,271-332; shallow_water.jl:68-136): one
    operator application within 1e-6 of FP64 (field-relative per component),
    and not bitwise equal to it (the FP32 arithmetic runs)."""
    from test_gpu_parity import make_dg
    dim = 2
    kw = dict(bc="reflect") if law == "eg" else {}
    d64 = make_dg(law, dim, 3, 3, "ec", sflux, **kw)
    d32 = A.DGSEM(law=d64.law, grid=d64.grid, volume_form=d64.volume_form, surface_numericalflux=_SFLUX[sflux],
                  precision="fp32flux")
    q = PT.random_state(d64)
    a, b = PT.to_dev(np.zeros_like(q)), PT.to_dev(np.zeros_like(q))
    d64(a, PT.to_dev(q), 0.0, increment=False)
    d32(b, PT.to_dev(q), 0.0, increment=False)
    ha, hb = PT.to_host(a), PT.to_host(b)
    err = PT.field_rel_errors(hb, ha)
    assert np.all(err <= 1e-6), err
    assert not np.array_equal(ha, hb)


@pytest.mark.parametrize("sflux", ["roe", "matrix"])
def test_vortex_fp32flux_roe_matrix(sflux):
    """The isentropic vortex (C1) stepped 100 LSRK54 steps with a Roe or
    Matrix surface flux: FP32-flux form within 1e-6 (relative L2) of FP64."""
    c64 = P.vortex_c1()
    d64 = A.DGSEM(law=c64.dg.law, grid=c64.dg.grid, volume_form=c64.dg.volume_form,
                  surface_numericalflux=_SFLUX[sflux])
    d32 = A.DGSEM(law=c64.dg.law, grid=c64.dg.grid, volume_form=c64.dg.volume_form,
                  surface_numericalflux=_SFLUX[sflux], precision="fp32flux")
    q64, q32 = PT.to_dev(c64.q0), PT.to_dev(c64.q0)
    A.LSRK54(d64, q64, c64.dt).step(q64, 100)
    A.LSRK54(d32, q32, c64.dt).step(q32, 100)
    assert _rel(d64, q32, q64) <= 1e-6


def test_lake_at_rest_fp32flux_roe_ec():
    """The well-balanced bathymetry terms stay FP64 in the FP32-flux Roe and
    EC surface fluxes: a lake at rest stays at rest to round-off."""
    import torch
    for sflux in ("roe", "ec"):
        c = P.sw_fplane(K=8, steps=50, precision="fp32flux", lake_at_rest=True)
        dg = A.DGSEM(law=c.dg.law, grid=c.dg.grid, volume_form=c.dg.volume_form,
                     surface_numericalflux=_SFLUX[sflux], precision="fp32flux")
        q = PT.to_dev(c.q0)
        A.LSRK54(dg, q, c.dt).step(q, 50)
        umax = float(q[1:3].abs().max() / q[0].abs().max())
        assert umax <= 1e-12, (sflux, umax)

"""Cubed-sphere shells: geometry, the oracle's curved-element operator, and
the CUDA curved-element kernels (through the C ABI) against the oracle.

CPU: discrete metric identities, shell volume and sphere areas, matching
normals and face masses on both sides of every interior face, the oracle's
free-stream preservation and mass conservation on the sphere, and the
oracle's curved path on a brick's geometry against its brick path.
GPU (marked): tendencies of Euler / Euler-gravity / linear Euler-gravity
operators on the sphere (plain field-relative error per component within
max(1e-12, 10 x the oracle's one-ulp spread)),
the curved kernel on a brick's geometry against the brick kernels, LSRK54 and
IMEX ARK23 steps of the reference's sphere experiments, and the measures.
"""
import ctypes as C

import numpy as np
import pytest

import atum_b200 as A
import parity as PT
from atum_b200 import workloads as W


def _cell(N):
    return A.LobattoCell(N + 1, N + 1, N + 1)


# ---------------------------------------------------------------- geometry
@pytest.mark.parametrize("vr,KH", [([1.0, 1.5, 2.0], 2), (np.linspace(6.371e6, 6.381e6, 3), 3)])
def test_geometry_invariants(vr, KH):
    N = 3
    g = A.cubedspheregrid(_cell(N), vr, KH)
    G = g.geometry()
    K, Np, Nq = g.K, g.cell.Np, g.cell.Nq
    assert K == 6 * KH * KH * (len(vr) - 1)
    x = G["x"]
    r = np.sqrt(np.sum(x * x, axis=0))
    assert np.allclose(r.min(), vr[0], rtol=1e-14) and np.allclose(r.max(), vr[-1], rtol=1e-14)
    # discrete metric identities: sum_i D_i (J a^i) = 0
    from atum_b200.cubedsphere import _dxi
    JA = (G["g"] * G["J"][None, None]).reshape(3, 3, K, Nq, Nq, Nq)
    div = sum(_dxi(JA[i], g.cell.D, i) for i in range(3))
    assert np.abs(div).max() <= 1e-13 * np.abs(JA).max()
    # shell volume and sphere areas converge with the resolution (N = 3, coarse)
    vol = G["MJ"].sum() / (4 / 3 * np.pi * (vr[-1] ** 3 - vr[0] ** 3)) - 1
    assert abs(vol) < 5e-3
    bt = G["btag"]
    assert abs(G["faceMJ"][bt == 5].sum() / (4 * np.pi * vr[0] ** 2) - 1) < 1e-3
    assert abs(G["faceMJ"][bt == 6].sum() / (4 * np.pi * vr[-1] ** 2) - 1) < 1e-3
    # boundary normals point out of the shell (radial up to the polynomial
    # approximation of the sphere by degree-N faces)
    fn = G["face_nodes"]
    for e, f in zip(*np.nonzero(bt)):
        xh = x[:, e, fn[f]] / r[e, fn[f]]
        dot = np.sum(G["normals"][e, f].T * xh, axis=0)
        assert np.allclose(dot, -1.0 if bt[e, f] == 5 else 1.0, atol=2e-3)
    # interior faces: the neighbour's node coincides, normals opposite, face masses equal
    nb = G["nbr_node"]
    e, f, j = np.nonzero(nb >= 0)
    e2, n2 = np.divmod(nb[e, f, j], Np)
    assert np.allclose(x[:, e, fn[f, j]], x[:, e2, n2], rtol=0, atol=1e-9 * vr[-1])
    inv = {}
    for ff in range(6):
        for jj, n in enumerate(fn[ff]):
            inv.setdefault(int(n), []).append((ff, jj))
    for a, b, c, ee, nn in zip(e[::7], f[::7], j[::7], e2[::7], n2[::7]):
        back = [(ff, jj) for ff, jj in inv[int(nn)] if nb[ee, ff, jj] == a * Np + fn[b, c]]
        assert len(back) == 1
        ff, jj = back[0]
        assert np.array_equal(G["normals"][a, b, c], -G["normals"][ee, ff, jj])
        assert G["faceMJ"][a, b, c] == G["faceMJ"][ee, ff, jj]


def test_min_node_distance_radial():
    N, KV, H = 4, 5, 10e3
    g = A.cubedspheregrid(_cell(N), np.linspace(6.371e6, 6.371e6 + H, KV + 1), 2)
    gap = float(np.min(np.diff(g.cell.nodes)))
    assert A.min_node_distance(g, dims=(3,)) == pytest.approx(H / KV / 2 * gap, rel=1e-9)
    assert A.min_node_distance(g) <= A.min_node_distance(g, dims=(3,))


def test_bad_grids_rejected():
    with pytest.raises(ValueError):
        A.cubedspheregrid(A.LobattoCell(3, 3), [1.0, 2.0], 1)
    with pytest.raises(ValueError):
        A.cubedspheregrid(_cell(2), [2.0, 1.0], 1)
    with pytest.raises(ValueError):
        A.cubedspheregrid(_cell(2), [1.0, 2.0], 0)


# ------------------------------------------------------------------ oracle
@pytest.mark.parametrize("vf", ["weak", "ec"])
def test_oracle_free_stream(orc, vf):
    """A uniform flow stays uniform: discrete metric identities and face
    normals consistent with the volume metric (copy boundary state)."""
    g = A.cubedspheregrid(_cell(3), [1.0, 1.3, 1.6, 2.0], 2)
    form = A.WeakForm() if vf == "weak" else A.FluxDifferencingForm(A.EntropyConservativeFlux())
    dg = A.DGSEM(law=A.EulerLaw(3), grid=g, volume_form=form, surface_numericalflux=A.RusanovFlux())
    q = np.zeros((5, g.K, g.cell.Np))
    q[0], q[1], q[2], q[3], q[4] = 1.0, 0.3, -0.2, 0.1, 2.5
    dq = np.zeros_like(q)
    orc.DGSEM(dg)(dq, q, 0.0, False)
    assert np.abs(dq).max() < 1e-11


def test_oracle_conserves_mass(orc):
    case = W.sphere_zonal_flow(N=3, KH=2, KV=2)
    o = orc.DGSEM(case.dg)
    q = case.q0.copy()
    x = case.dg.grid.points()
    q[3] += 0.05 * q[0] * np.sin(x[0] / 1e4)  # radial and meridional flow through the faces
    dq = np.zeros_like(q)
    o(dq, q, 0.0, False)
    MJ = case.dg.MJ
    assert abs(np.sum(MJ * dq[0])) <= 1e-13 * np.sum(MJ * np.abs(dq[0]))


class _BrickAsCurved:
    """A stacked 3-D brick grid presented through the curved-geometry interface."""

    def __init__(self, grid):
        self.__dict__.update(dict(cell=grid.cell, vertices=grid.vertices, periodic=grid.periodic, stacked=True))
        self._g = grid

    dim = 3

    @property
    def Kd(self):
        return self._g.Kd

    @property
    def K(self):
        return self._g.K

    def __len__(self):
        return self._g.K

    def element_indices(self):
        return self._g.element_indices()

    def points(self):
        return self._g.points()

    def geometry(self):
        g, c = self._g, self._g.cell
        K, Np, Nq = g.K, c.Np, c.Nq
        Nfp = Nq * Nq
        eidx = g.element_indices()
        h = np.stack([np.diff(g.vertices[d])[eidx[:, d]] for d in range(3)], axis=1)  # (K, 3)
        node = np.arange(Np)
        ijk = np.stack([node % Nq, (node // Nq) % Nq, node // (Nq * Nq)])
        w = c.weights[ijk[0]] * c.weights[ijk[1]] * c.weights[ijk[2]]
        J = np.prod(h / 2, axis=1)
        gm = np.zeros((3, 3, K, Np))
        for d in range(3):
            gm[d, d] = (2.0 / h[:, d])[:, None]
        fnodes = np.zeros((6, Nfp), dtype=np.int64)
        fw = np.zeros((6, Nfp))
        for k in range(3):
            t = [d for d in range(3) if d != k]
            for side in range(2):
                for j in range(Nfp):
                    a, b = j % Nq, j // Nq
                    idx = [0, 0, 0]
                    idx[k] = Nq - 1 if side else 0
                    idx[t[0]], idx[t[1]] = a, b
                    fnodes[2 * k + side, j] = idx[0] + Nq * (idx[1] + Nq * idx[2])
                    fw[2 * k + side, j] = c.weights[a] * c.weights[b]
        normals = np.zeros((K, 6, Nfp, 3))
        fMJ = np.zeros((K, 6, Nfp))
        nbr = np.full((K, 6, Nfp), -1, dtype=np.int64)
        bt = np.zeros((K, 6), dtype=np.int32)
        where = {tuple(ix): e for e, ix in enumerate(eidx)}
        for e in range(K):
            for k in range(3):
                t = [d for d in range(3) if d != k]
                for side in range(2):
                    f = 2 * k + side
                    normals[e, f, :, k] = 1.0 if side else -1.0
                    fMJ[e, f] = fw[f] * ((h[e, t[0]] / 2) * (h[e, t[1]] / 2))
                    ix = list(eidx[e])
                    ix[k] += 1 if side else -1
                    if 0 <= ix[k] < g.Kd[k] or g.periodic[k]:
                        ix[k] %= g.Kd[k]
                        nbr[e, f] = where[tuple(ix)] * Np + fnodes[f ^ 1]
                    else:
                        bt[e, f] = f + 1
        return {"x": g.points(), "J": np.repeat(J[:, None], Np, 1), "g": gm, "MJ": w[None, :] * J[:, None],
                "face_nodes": fnodes, "normals": normals, "faceMJ": fMJ, "nbr_node": nbr, "btag": bt}


def _bubble_pair(N=3, K=(3, 2, 3), vf="ec", weak=False):
    case = W.bubble_3d(N=N, K=K, imex=True, steps=2, vflux=vf)
    dg = case.dg
    if weak:
        dg = A.DGSEM(law=dg.law, grid=dg.grid, surface_numericalflux=A.RusanovFlux())
    cg = _BrickAsCurved(dg.grid)
    dgc = A.DGSEM(law=dg.law, grid=cg, volume_form=dg.volume_form, surface_numericalflux=dg.surface_numericalflux,
                  auxstate=dg.auxstate_host())
    lin = A.DGSEM(law=case.lindg.law, grid=cg, surface_numericalflux=A.RusanovFlux(), auxstate=dg.auxstate_host(),
                  directions=(3,))
    return case, dg, dgc, lin


def _flowing(q0, x):
    """The bubble state with flow in every direction, so that no tendency
    component is a near-zero residual of cancelling forces."""
    q = q0.copy()
    q[1] += 0.3 * q[0] * np.cos(x[2] / 900.0)
    q[2] -= 0.25 * q[0] * np.sin(x[0] / 800.0)
    q[3] -= 0.2 * q[0] * np.sin(x[0] / 700.0 + x[1] / 600.0)
    return q


@pytest.mark.parametrize("weak", [False, True])
def test_oracle_curved_path_on_brick_geometry(orc, weak):
    """The oracle's curved path, given a brick's geometry, reproduces its brick
    path bit for bit."""
    case, dg, dgc, lin = _bubble_pair(weak=weak)
    q = _flowing(case.q0, dg.grid.points())
    for a, b in ((dg, dgc), (case.lindg, lin)):
        d1, d2 = np.zeros_like(q), np.zeros_like(q)
        orc.DGSEM(a)(d1, q, 0.0, False)
        orc.DGSEM(b)(d2, q, 0.0, False)
        # the same sums in the same order (the off-diagonal metric terms are zeros)
        assert np.array_equal(d1, d2), PT.field_rel_errors(d2, d1)


def test_sphere_vtu_snapshot(tmp_path):
    """VTK snapshots of sphere fields (the experiments' output): the nodes of
    every curved element as points, N^3 linear sub-cells per element."""
    import xml.etree.ElementTree as ET
    from atum_b200 import vtk
    case = W.sphere_acoustic_wave(N=2, KH=1, KV=2)
    g = case.dg.grid
    path = vtk.write_vtu(str(tmp_path / "sphere.vtu"), g, {"rho": case.q0[0]})
    piece = ET.parse(path).getroot().find(".//Piece")
    assert int(piece.get("NumberOfPoints")) == g.K * g.cell.Np
    assert int(piece.get("NumberOfCells")) == g.K * (g.cell.Nq - 1) ** 3


def test_curved_abi_checks_without_gpu():
    from atum_b200 import _lib
    from atum_b200._device import make_desc
    g = A.cubedspheregrid(_cell(2), [1.0, 2.0], 1)
    dg = A.DGSEM(law=A.EulerLaw(3), grid=g, surface_numericalflux=A.RoeFlux())
    desc, keep = make_desc(dg)
    geo = _lib.CurvedGeometry()
    h = C.c_void_p()
    L = _lib.lib()
    assert L.atb_op_create_curved(C.byref(desc), None, None, C.byref(h)) == -1
    G = g.geometry()
    arrs = [np.ascontiguousarray(G[k]) for k in ("g", "MJ", "normals", "faceMJ")]
    nb, bt = np.ascontiguousarray(G["nbr_node"]), np.ascontiguousarray(G["btag"], dtype=np.int32)
    geo = _lib.CurvedGeometry(*[_lib.dptr(a) for a in arrs], nb.ctypes.data_as(C.POINTER(C.c_longlong)),
                              bt.ctypes.data_as(C.POINTER(C.c_int)))
    # an unknown surface flux
    desc.surface_flux = 7
    assert L.atb_op_create_curved(C.byref(desc), None, C.byref(geo), C.byref(h)) == -1
    assert b"surface flux" in L.atb_last_error()
    desc.surface_flux = 1
    desc.dim = 2
    assert L.atb_op_create_curved(C.byref(desc), None, C.byref(geo), C.byref(h)) == -1
    del keep


# --------------------------------------------------------------------- GPU
def _rotating(dg):
    law = dg.law
    pr = A.Coriolis((0.0, 0.0, 2 * 7.29212e-5 * 125), bc=law.problem.bc, referencestate=law.problem.referencestate)
    rot = A.EulerGravityLaw(3, sphere=True, grav=law.grav, problem=pr)
    return A.DGSEM(law=rot, grid=dg.grid, volume_form=dg.volume_form, surface_numericalflux=dg.surface_numericalflux)


def _tendency_cases():
    zon = lambda: W.sphere_zonal_flow(N=3, KH=2, KV=2)  # noqa: E731
    return {
        "eg-ec-rusanov": lambda: (zon().dg, None),
        "eg-kg-ec": lambda: (A.DGSEM(law=zon().dg.law, grid=zon().dg.grid,
                                     volume_form=A.FluxDifferencingForm(A.KennedyGruberFlux()),
                                     surface_numericalflux=A.EntropyConservativeFlux()), None),
        "eg-weak-rusanov": lambda: (A.DGSEM(law=zon().dg.law, grid=zon().dg.grid,
                                            surface_numericalflux=A.RusanovFlux()), None),
        "eg-central-central": lambda: (A.DGSEM(law=zon().dg.law, grid=zon().dg.grid,
                                               volume_form=A.FluxDifferencingForm(A.CentralFlux()),
                                               surface_numericalflux=A.CentralFlux()), None),
        "eg-ec-roe": lambda: (A.DGSEM(law=zon().dg.law, grid=zon().dg.grid,
                                      volume_form=A.FluxDifferencingForm(A.EntropyConservativeFlux()),
                                      surface_numericalflux=A.RoeFlux()), None),
        "eg-ec-matrix": lambda: (A.DGSEM(law=zon().dg.law, grid=zon().dg.grid,
                                         volume_form=A.FluxDifferencingForm(A.EntropyConservativeFlux()),
                                         surface_numericalflux=A.MatrixFlux()), None),
        "leg-weak-z": lambda: (zon().lindg, None),
        # the baroclinic wave's rotating sphere: dq[rho u] -= (0, 0, 2 Omega) x rho u
        # (experiment/euler_gravity/baroclinicwave.jl:27-34)
        "eg-ec-rusanov-coriolis": lambda: (_rotating(zon().dg), None),
        "euler-ec-kg": lambda: (None, "euler"),
    }


@pytest.mark.gpu
@pytest.mark.parametrize("name,N", [(n, N) for N in (2, 3, 5) for n in _tendency_cases()] +
                         [(n, N) for N in (1, 7) for n in ("eg-ec-rusanov", "eg-weak-rusanov", "leg-weak-z")])
def test_curved_tendency_matches_oracle(orc, name, N):
    """Seeded states 5% away from the zonal flow's balanced reference state;
    plain field-relative error per component against max(1e-12, 10 x the
    oracle's one-ulp spread)."""
    dg, other = _tendency_cases()[name]()
    if other == "euler":
        g = A.cubedspheregrid(_cell(N), [1.0, 1.4, 2.0], 2)
        law = A.EulerLaw(3, problem=A.ReflectiveWall())
        dg = A.DGSEM(law=law, grid=g, volume_form=A.FluxDifferencingForm(A.EntropyConservativeFlux()),
                     surface_numericalflux=A.KennedyGruberFlux())
    elif N != 3:
        g = A.cubedspheregrid(_cell(N), dg.grid.vr, dg.grid.KH)
        dg = A.DGSEM(law=dg.law, grid=g, volume_form=dg.volume_form,
                     surface_numericalflux=dg.surface_numericalflux, directions=dg.directions)
    q = PT.random_state(dg)
    rng = np.random.default_rng(5)
    dq0 = rng.standard_normal(q.shape)
    # the oracle's own rounding sensitivity: its tendency from the state moved
    # by one ulp (the momentum of these near-hydrostatic states is a residual of
    # cancelling pressure and gravity terms: about 5e-13 of its field at N = 5)
    od = orc.DGSEM(dg)
    ref, moved = np.zeros_like(q), np.zeros_like(q)
    od(ref, q, 0.0, False)
    od(moved, PT.ulp_perturbed(q), 0.0, False)
    bound = np.maximum(1e-12, PT.SPREAD_FACTOR * PT.field_rel_errors(moved, ref))
    for inc in (False, True):
        d_o = dq0.copy()
        od(d_o, q, 0.0, inc)
        qd, dd = PT.to_dev(q), PT.to_dev(dq0)
        dg(dd, qd, 0.0, increment=inc)
        err = PT.field_rel_errors(PT.to_host(dd), d_o)
        print(f"[parity] sphere tendency {name} N={N} increment={inc}: {err}, bound {bound}")
        assert np.all(err <= bound), (err, bound)


@pytest.mark.gpu
@pytest.mark.parametrize("weak", [False, True])
def test_curved_kernel_on_brick_geometry_matches_brick_kernel(weak):
    case, dg, dgc, lin = _bubble_pair(weak=weak)
    for a, b in ((dg, dgc), (case.lindg, lin)):
        q = PT.random_state(a)
        d1, d2 = PT.to_dev(np.zeros_like(q)), PT.to_dev(np.zeros_like(q))
        qd = PT.to_dev(q)
        a(d1, qd, 0.0, increment=False)
        b(d2, qd, 0.0, increment=False)
        err = PT.field_rel_errors(PT.to_host(d2), PT.to_host(d1))
        assert np.all(err <= 1e-12), err


def _gpu_steps(case, counts):
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


def _oracle_steps(orc, case, counts, q0=None, dt=None):
    q = (case.q0 if q0 is None else q0).copy()
    o = orc.DGSEM(case.dg)
    dt = case.dt if dt is None else dt
    if case.solver == "ARK23":
        s = orc.ARK23(o, orc.DGSEM(case.lindg), q, dt, split_rhs=case.split_rhs)
    else:
        s = getattr(orc, case.solver)(o, q, dt)
    out, done = [], 0
    for n in counts:
        s.step(q, n - done)
        done = n
        out.append(q.copy())
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("build,counts,tol", [
    (lambda: W.sphere_zonal_flow(N=3, KH=2, KV=3, steps=5), (1, 5), (1e-12, 1e-11)),
    (lambda: W.sphere_acoustic_wave(N=3, KH=2, KV=2, steps=3), (1, 3), (1e-12, 1e-11)),
    (lambda: W.sphere_zonal_flow(N=3, KH=2, KV=2, steps=5, imex=False, dt=0.5), (1, 5), (1e-12, 1e-11)),
    (lambda: W.sphere_baroclinic_wave(N=3, KH=2, KV=2, steps=3), (1, 3), (1e-12, 1e-11)),
], ids=["zonal-ark23", "acoustic-ark23", "zonal-lsrk54", "baroclinic-ark23"])
def test_sphere_steps_match_oracle(orc, build, counts, tol):
    """Bound: max(tol, 10 x the oracle's own rounding spread), the spread being
    the larger change of the oracle's result under a one-ulp move of the
    initial state or of dt.  A one-ulp move of dt changes the IMEX step's
    banded factorisation I - dt a L by rounding only, and at the acoustic
    wave's vertical CFL (about 80) that moves the solution by 2e-10 relative:
    the step's own conditioning, which any reordering of the factorisation's
    arithmetic meets as well."""
    case = build()
    g = _gpu_steps(case, counts)
    o = _oracle_steps(orc, case, counts)
    o1 = _oracle_steps(orc, case, counts, q0=PT.ulp_perturbed(case.q0))
    o2 = _oracle_steps(orc, case, counts, dt=np.nextafter(case.dt, np.inf))
    for n, gi, oi, oj, ok, t in zip(counts, g, o, o1, o2, tol):
        assert np.isfinite(gi).all()
        spread = np.maximum(PT.field_rel_errors(oj, oi), PT.field_rel_errors(ok, oi))
        PT.assert_parity(f"{case.name} {case.solver}, {n} step(s)", gi, oi, t, spread=spread)


@pytest.mark.gpu
def test_sphere_measures_match_oracle(orc):
    case = W.sphere_zonal_flow(N=3, KH=2, KV=2)
    o = orc.DGSEM(case.dg)
    qd = PT.to_dev(case.q0)
    for p in (2, np.inf):
        assert A.weightednorm(case.dg, qd, p) == pytest.approx(orc.weightednorm(o, case.q0, p), rel=1e-13)
    assert A.entropyintegral(case.dg, qd) == pytest.approx(orc.entropyintegral(o, case.q0), rel=1e-12)


@pytest.mark.gpu
def test_sphere_line_solve_sparse_equals_dense(monkeypatch):
    """The per-line banded solve that skips the factors' face-coupling zero
    blocks gives the full-band solve's results bit for bit."""
    case = W.sphere_zonal_flow(N=3, KH=2, KV=3, steps=3)
    out = []
    for dense in ("1", "0"):
        monkeypatch.setenv("ATB_BAND_DENSE", dense)
        q = PT.to_dev(case.q0)
        s = A.ARK23(case.dg, case.lindg, q, case.dt, split_rhs=False)
        s.step(q, 3)
        out.append(PT.to_host(q))
        del s
    assert np.array_equal(out[0], out[1])


@pytest.mark.gpu
@pytest.mark.parametrize("vflux", ["ec", "kg"])
def test_sphere_fused_stage_equals_two_launches(orc, vflux):
    """The fused curved ARK23 stage (explicit tendency + radial linear operator
    + accumulation in one launch) gives the two-launch path's states within
    the step's own rounding sensitivity: the two kernels are compiled apart, so
    FMA contraction may differ by an ulp, which the IMEX solve amplifies like a
    one-ulp move of dt (measured on the oracle here)."""
    case = W.sphere_zonal_flow(N=3, KH=2, KV=3, steps=3, vflux=vflux)
    qa, qb = PT.to_dev(case.q0), PT.to_dev(case.q0)
    sa = A.ARK23(case.dg, case.lindg, qa, case.dt, split_rhs=False)
    sb = A.ARK23(case.dg, case.lindg, qb, case.dt, split_rhs=False)
    sb.fuse(False)
    sa.step(qa, 3)
    sb.step(qb, 3)
    err = PT.field_rel_errors(PT.to_host(qa), PT.to_host(qb))
    o = _oracle_steps(orc, case, (3,))[0]
    o2 = _oracle_steps(orc, case, (3,), dt=np.nextafter(case.dt, np.inf))[0]
    bound = np.maximum(1e-12, PT.SPREAD_FACTOR * PT.field_rel_errors(o2, o))
    print(f"[parity] sphere fused vs two launches ({vflux}): {err}, bound {bound}")
    assert np.all(err <= bound), (err, bound)


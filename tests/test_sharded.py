"""One problem sharded by element slabs (atum_b200.sharded).

CPU: the slab layout (owned columns partition the grid, ghosts are the
neighbours' boundary columns, the local grid's coordinates are the global
ones), and two gloo ranks stepping the oracle on their slabs with the ghost
exchange after every stage reproduce the unsharded oracle run bit for bit
(LSRK54; periodic and walled cuts).
GPU: every slab packed into one operator on one device, the exchange device
copies through the solvers' exchange hook: LSRK54 and IMEX ARK23 states equal
the unsharded GPU run bit for bit."""
import os
import socket

import numpy as np
import pytest

import atum_b200 as A
import problems as P
from atum_b200 import sharded as S


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _bubble(periodic_x=True, K=(6, 2, 3)):
    import _sharded_worker as W
    return W.bubble(periodic_x, K)


@pytest.mark.parametrize("world,periodic", [(2, True), (3, True), (2, False), (4, False)])
def test_slab_layout(world, periodic):
    case = _bubble(periodic, K=(7, 2, 3))
    g = case.dg.grid
    owned = []
    for r in range(world):
        L = S.slab_layout(g, r, world)
        assert L.grid.K == len(L.local_to_global)
        owned.append(L.local_to_global[L.owned])
        # local coordinates are the global ones (up to a period for wrapped ghosts)
        xl, xg = L.grid.points(), g.points()[:, L.local_to_global]
        assert np.allclose(xl[1:], xg[1:]) and np.allclose(xl[0][L.owned], xg[0][L.owned])
        for side in ("left", "right"):
            peer = getattr(L, side)
            if peer < 0:
                continue
            Lp = S.slab_layout(g, peer, world)
            mine = L.local_to_global[getattr(L, "recv_" + side)()]
            theirs = Lp.local_to_global[getattr(Lp, "send_" + ("right" if side == "left" else "left"))()]
            assert np.array_equal(mine, theirs)
    allo = np.concatenate(owned)
    assert np.array_equal(np.sort(allo), np.arange(g.K))


@pytest.mark.parametrize("world,periodic", [(2, True), (3, False)])
def test_gloo_ranks_reproduce_unsharded_oracle(orc, world, periodic):
    import torch.multiprocessing as mp
    case = _bubble(periodic)
    ref = case.q0.copy()
    orc.LSRK54(orc.DGSEM(case.dg), ref, case.dt).step(ref, 4)
    ctx = mp.get_context("spawn")
    qu = ctx.Queue()
    port = _free_port()
    import _sharded_worker as W
    procs = [ctx.Process(target=W.rank_main, args=(r, world, port, periodic, qu)) for r in range(world)]
    for p in procs:
        p.start()
    res = [qu.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    got = np.full_like(ref, np.nan)
    for e, v in res[0][1]:
        got[:, e] = v
    assert np.array_equal(got, ref)


def _packed_sharded(case, world):
    """Every slab in one packed operator, the exchange device copies."""
    import torch
    Ls = [S.slab_layout(case.dg.grid, r, world) for r in range(world)]
    dgs = [S.local_dgsem(case.dg, L) for L in Ls]
    packed = A.batch.PackedDGSEM(dgs)
    lins = None
    if case.lindg is not None:
        lins = A.batch.PackedDGSEM([S.local_dgsem(case.lindg, L) for L in Ls])
    q0 = packed.pack([torch.as_tensor(case.q0[:, L.local_to_global], device="cuda") for L in Ls])
    first = packed.offsets
    ex = S.LocalExchanger(Ls, first)
    return Ls, packed, lins, q0, first, ex


@pytest.mark.gpu
@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("scheme", ["lsrk54", "ark23"])
def test_sharded_on_one_gpu_equals_unsharded(world, scheme):
    import torch
    import parity as PT
    if scheme == "lsrk54":
        case = P.bubble_3d(N=3, K=(6, 2, 3), imex=False, steps=3)
    else:
        case = P.bubble_3d(N=3, K=(6, 2, 3), imex=True, steps=3)
    qr = PT.to_dev(case.q0)
    if scheme == "lsrk54":
        A.LSRK54(case.dg, qr, case.dt).step(qr, 3)
    else:
        A.ARK23(case.dg, case.lindg, qr, case.dt, split_rhs=False).step(qr, 3)
    Ls, packed, lins, q, first, ex = _packed_sharded(case, world)
    if scheme == "lsrk54":
        s = A.LSRK54(packed, q, case.dt)
    else:
        s = A.ARK23(packed, lins, q, case.dt, split_rhs=False)
    K, Np = q.shape[1], q.shape[2]
    S.attach(s, ex, K, Np)
    s.step(q, 3)
    S.attach(s, None, 0, 0)
    got = torch.full_like(qr, float("nan"))
    for L in Ls:
        rows = first[L.rank] + torch.as_tensor(L.owned, device="cuda")
        got[:, torch.as_tensor(L.local_to_global[L.owned], device="cuda")] = q[:, rows]
    assert torch.equal(got, qr)

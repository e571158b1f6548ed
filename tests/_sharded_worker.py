"""Worker of tests/test_sharded.py's gloo ranks (a module of its own, so that a
spawned rank imports nothing before it has made the package importable)."""
import os
import sys


def bubble(periodic_x=True, K=(6, 2, 3)):
    import atum_b200 as A
    import problems as P
    case = P.bubble_3d(N=2, K=K, imex=False, steps=4)
    if not periodic_x:
        g = case.dg.grid
        grid = A.brickgrid(g.cell, g.vertices, periodic=(False, True, False), ordering="stacked")
        case.dg = A.DGSEM(law=case.dg.law, grid=grid, volume_form=case.dg.volume_form,
                          surface_numericalflux=case.dg.surface_numericalflux)
    return case


def rank_main(rank, world, port, periodic, out):
    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    sys.path[:0] = [here, root, os.path.join(root, "oracle")]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from __graft_entry__ import _load_package
    _load_package()
    import numpy as np
    import torch
    import torch.distributed as dist
    import atum_b200.sharded as S
    import pyoracle as orc
    dist.init_process_group("gloo", rank=rank, world_size=world)
    orc.set_threads(1)
    case = bubble(periodic)
    L = S.slab_layout(case.dg.grid, rank, world)
    ldg = S.local_dgsem(case.dg, L)
    q = np.ascontiguousarray(case.q0[:, L.local_to_global])
    ex = S.DistExchanger(L)
    ex.exchange(torch.from_numpy(q))
    solver = orc.LSRK54(orc.DGSEM(ldg), q, case.dt)
    solver.set_stage_hook(lambda qs: ex.exchange(torch.from_numpy(qs)))
    solver.step(q, 4)
    solver.set_stage_hook(None)
    mine = (L.local_to_global[L.owned], q[:, L.owned])
    everyone = [None] * world
    dist.all_gather_object(everyone, mine)
    dist.destroy_process_group()
    out.put((rank, everyone))

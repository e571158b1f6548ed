"""The LSRK54 entry point that allocates nothing, against the allocating path.

Some callers cannot allocate device memory around a time step: their device
memory belongs to their own pool allocator, or their loop cannot afford the
synchronisation a cudaMalloc / cudaFree pair can cause.  For them the library
offers atb_lsrk54_step_noalloc, whose scratch is a static array inside the
library.  These tests call it through the C ABI and compare it with the
allocating atb_solver_step path on the same operator, on two calls in a row,
with the parity tolerance used throughout the suite (1e-12 relative per DOF).
The file name makes pytest collect it last; it also passes alone in a fresh
process.
"""
import numpy as np
import pytest

import atum_b200 as A
import parity as PT
import problems as P

pytestmark = pytest.mark.gpu


def test_noalloc_matches_allocating_solver_on_two_consecutive_calls():
    import torch
    from atum_b200 import _lib

    case = P.vortex_c1()  # 2-D Euler vortex, 8x8 elements, N = 3: 4,096 DOFs
    dg = case.dg
    q_alloc = PT.to_dev(case.q0)
    q_noalloc = PT.to_dev(case.q0)
    solver = A.LSRK54(dg, q_alloc, case.dt)
    L = _lib.lib()
    for _ in range(2):
        solver.step(q_alloc, 3)
        _lib.check(L.atb_lsrk54_step_noalloc(dg.device.h, _lib.field_ptrs(q_noalloc, 4), case.dt, 3,
                                             _lib.stream_ptr()))
        torch.cuda.synchronize()
        assert torch.isfinite(q_noalloc).all()
        err = PT.rel_dof_error(PT.to_host(q_noalloc), PT.to_host(q_alloc))
        assert err <= 1e-12, err


def test_noalloc_rejects_states_beyond_its_static_scratch():
    import torch
    from atum_b200 import _lib

    # 3-D Euler, N = 3, 12^3 elements: 552,960 DOFs > ATB_NOALLOC_MAX_DOFS = 524,288
    cell = A.LobattoCell(4, 4, 4)
    v = np.linspace(0.0, 1.0, 13)
    grid = A.brickgrid(cell, (v, v, v), periodic=(True, True, True))
    dg = A.DGSEM(law=A.EulerLaw(3), grid=grid, surface_numericalflux=A.RusanovFlux(),
                 volume_form=A.FluxDifferencingForm(A.EntropyConservativeFlux()))
    q = torch.ones((5, len(grid), cell.Np), dtype=torch.float64, device="cuda")
    q[4] = 2.5
    before = q.clone()
    L = _lib.lib()
    rc = L.atb_lsrk54_step_noalloc(dg.device.h, _lib.field_ptrs(q, 5), 1e-3, 1, _lib.stream_ptr())
    assert rc == -1
    assert b"ATB_NOALLOC_MAX_DOFS" in L.atb_last_error()
    torch.cuda.synchronize()
    assert torch.equal(q, before)

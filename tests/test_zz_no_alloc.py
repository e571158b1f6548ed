"""The LSRK54 entry point that allocates nothing, against the allocating path.

Some callers cannot allocate device memory around a time step: their device
memory belongs to their own pool allocator, or their loop cannot afford the
synchronisation a cudaMalloc / cudaFree pair can cause.  For them the library
offers atb_lsrk54_step_noalloc, whose scratch is a static array inside the
library.  These tests call it through the C ABI and compare it with the
allocating atb_solver_step path on the same operator, on two calls in a row:
bit for bit (the same kernels in the same order), which is within the parity
tolerance used throughout the suite (1e-12 relative per DOF).
The file name makes pytest collect it last; it also passes alone in a fresh
process.
"""
import numpy as np
import pytest

import atum_b200 as A
import parity as PT
import problems as P

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nsteps", [3, 2])
def test_noalloc_matches_allocating_solver_on_two_consecutive_calls(nsteps):
    """Odd step counts end on the scratch buffer (the state is copied back),
    even ones on the caller's buffer: both branches, two calls in a row each.
    Both paths launch the same kernels with the same coefficients in the same
    order on the same operator, so the states agree bit for bit."""
    import torch
    from atum_b200 import _lib

    case = P.vortex_c1()  # 2-D Euler vortex, 8x8 elements, N = 3: 4,096 DOFs
    dg = case.dg
    q_alloc = PT.to_dev(case.q0)
    q_noalloc = PT.to_dev(case.q0)
    solver = A.LSRK54(dg, q_alloc, case.dt)
    L = _lib.lib()
    for _ in range(2):
        solver.step(q_alloc, nsteps)
        _lib.check(L.atb_lsrk54_step_noalloc(dg.device.h, _lib.field_ptrs(q_noalloc, 4), case.dt, nsteps,
                                             _lib.stream_ptr()))
        torch.cuda.synchronize()
        assert torch.isfinite(q_noalloc).all()
        assert torch.equal(q_noalloc, q_alloc)
        assert PT.rel_dof_error(PT.to_host(q_noalloc), PT.to_host(q_alloc)) <= 1e-12


def test_noalloc_zero_steps_and_bad_dt_leave_the_state():
    import torch
    from atum_b200 import _lib

    case = P.vortex_c1()
    q = PT.to_dev(case.q0)
    before = q.clone()
    L = _lib.lib()
    _lib.check(L.atb_lsrk54_step_noalloc(case.dg.device.h, _lib.field_ptrs(q, 4), case.dt, 0, _lib.stream_ptr()))
    for bad in (float("nan"), float("inf")):
        assert L.atb_lsrk54_step_noalloc(case.dg.device.h, _lib.field_ptrs(q, 4), bad, 1, _lib.stream_ptr()) == -1
    torch.cuda.synchronize()
    assert torch.equal(q, before)


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

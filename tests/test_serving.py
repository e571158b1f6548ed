"""Serving loop: requests packed into element pools by operator kind give every
request bitwise the state it gets stepped alone, whatever shares its pool,
with and without CUDA-graph replay, under an HBM budget that makes requests
wait and pools take turns."""
import numpy as np
import pytest

import atum_b200 as A
import parity as PT
import problems as P

pytestmark = pytest.mark.gpu


def _requests(n, seed=7, Ks=(4, 6), rate=None, vortex_every=0):
    rng = np.random.default_rng(seed)
    out = []
    t = 0.0
    for i in range(n):
        K = Ks[i % len(Ks)]
        prec = "fp32flux" if i % 3 == 0 else "fp64"
        if vortex_every and i % vortex_every == 1:
            c = P.vortex_c1(N=3, K=K, precision=prec)
        else:
            c = P.sw_fplane(N=3, K=K, seed=500 + i, precision=prec)
        if rate:
            t += rng.exponential(1.0 / rate)
        out.append(A.serving.Request(rid=i, dg=c.dg, q0=c.q0, dt=c.dt * rng.uniform(0.5, 1.0),
                                     nsteps=int(rng.integers(3, 40)), arrival=t))
    return out


def _alone(r):
    q = PT.to_dev(r.q0)
    s = A.LSRK54(r.dg, q, r.dt)
    s.step(q, r.nsteps)
    return PT.to_host(q)


@pytest.mark.parametrize("graphs", [False, True])
def test_served_equals_alone(graphs):
    reqs = _requests(16, vortex_every=4)
    # 64-element pools: 16- and 36-element requests queue, finish, move down
    srv = A.serving.Server(capacity=64, chunk=16, use_graphs=graphs, max_tick_steps=8)
    st = srv.run(reqs, realtime=False)
    assert st.requests == 16
    # SW and Euler x two precisions: four operator kinds
    assert st.pools >= 4
    for r in reqs:
        assert r.result is not None and np.array_equal(r.result, _alone(r)), r.rid
    assert st.p99_latency_s >= st.p50_latency_s > 0
    assert st.dof_stage_per_s > 0
    srv.close()


def test_budget_makes_pools_take_turns():
    reqs = _requests(6, Ks=(4,))
    one_pool = A.serving.pool_bytes_per_element(reqs[0].dg) * 40
    # room for one 40-element pool: the two precisions take turns and idle
    # pools are released for the other kind
    srv = A.serving.Server(hbm_budget_bytes=one_pool * 1.5, capacity=40, chunk=8)
    st = srv.run(reqs, realtime=False)
    assert st.requests == 6
    assert st.peak_pool_bytes <= one_pool * 1.5
    assert st.pools >= 2
    for r in reqs:
        assert np.array_equal(r.result, _alone(r)), r.rid
    srv.close()


def test_poisson_arrivals_realtime():
    reqs = _requests(10, rate=200.0)
    for r in reqs[::2]:
        r.q0 = A.serving.pinned_array(r.q0)     # DMA admission path
    srv = A.serving.Server(capacity=128, chunk=32)
    st = srv.run(reqs, realtime=True)
    assert st.requests == 10
    for r in reqs:
        assert r.finished >= r.arrival and r.admitted >= r.arrival
        assert np.array_equal(r.result, _alone(r)), r.rid
    srv.close()


def test_many_placements_and_reused_result_buffers():
    """More placements than the pool's ring of geometry staging areas, and more
    finishing ticks than result buffers: every result still equals the
    request stepped alone."""
    base = _requests(6, seed=11)
    reqs = []
    for k in range(4):
        for r in base:
            reqs.append(A.serving.Request(rid=len(reqs), dg=r.dg, q0=r.q0, dt=r.dt, nsteps=r.nsteps + k,
                                          arrival=0.0))
    assert len(reqs) > 8
    srv = A.serving.Server(hbm_budget_bytes=2e9, capacity=4096, chunk=64, use_graphs=True)
    st = srv.run(reqs, realtime=False)
    srv.close()
    assert st.requests == len(reqs) and st.ticks > 8
    for r in reqs:
        assert np.array_equal(r.result, _alone(r))


def test_budget_too_small_raises():
    reqs = _requests(1)
    srv = A.serving.Server(hbm_budget_bytes=1.0, capacity=64)
    with pytest.raises(RuntimeError, match="HBM budget"):
        srv.run(reqs, realtime=False)


def test_request_larger_than_pool_rejected():
    reqs = _requests(1, Ks=(6,))
    srv = A.serving.Server(capacity=16)
    with pytest.raises(ValueError, match="more than a pool"):
        srv.run(reqs, realtime=False)


def test_pool_place_rejects_other_kind_and_overflow():
    import ctypes as C
    from atum_b200 import _lib
    from atum_b200._device import make_desc
    a = P.sw_fplane(N=3, K=4)
    b = P.vortex_c1(N=3, K=4)
    da, ka = make_desc(a.dg)
    db, kb = make_desc(b.dg)
    h = C.c_void_p()
    _lib.check(_lib.lib().atb_op_create_pool(C.byref(da), 20, C.byref(h)))
    try:
        aux = np.ascontiguousarray(a.dg.auxstate_host()).reshape(-1)
        assert _lib.lib().atb_op_place_instance(h, 0, C.byref(da), _lib.dptr(aux), None) == 0
        assert _lib.lib().atb_op_place_instance(h, 8, C.byref(da), _lib.dptr(aux), None) != 0   # 8 + 16 > 20
        assert _lib.lib().atb_op_place_instance(h, 0, C.byref(db), None, None) != 0             # other law
        assert _lib.lib().atb_op_set_active_elements(h, 21) != 0
    finally:
        _lib.lib().atb_op_destroy(h)


@pytest.mark.parametrize("graphs", [False, True])
def test_device_built_inputs_and_norm_results(graphs):
    """Requests whose initial state and aux fields are built on the device at
    admission (``make``), mixed with host-input requests: each served state is
    bitwise the state stepped alone from the same inputs, and a request that
    asks for norms gets the per-component MJ-weighted L2 norms of that state."""
    import torch
    from atum_b200 import workloads as W
    reqs = []
    for i in range(10):
        if i % 2:
            c = P.bubble_3d(N=2, K=3, imex=False, precision="fp32flux" if i % 3 else "fp64")
            make = (lambda dg=c.dg: W.bubble_3d_device(dg))
        else:
            c = P.vortex_c1(N=3, K=4)
            make = (lambda dg=c.dg: W.vortex_c1_device(dg))
        mode = "norms" if i % 4 == 3 else "state"
        reqs.append(A.serving.Request(rid=i, dg=c.dg, q0=None, make=make, dt=c.dt, nsteps=3 + i, arrival=0.0,
                                      result_mode=mode))
    srv = A.serving.Server(capacity=96, chunk=16, use_graphs=graphs, max_tick_steps=4)
    st = srv.run(reqs, realtime=False)
    assert st.requests == 10
    for r in reqs:
        q0, aux = r.make()
        if aux is not None:
            # the device-built aux equals the host-evaluated one
            assert np.allclose(PT.to_host(aux), r.dg.auxstate_host(), rtol=1e-14, atol=1e-12)
        q = q0.clone()
        A.LSRK54(r.dg, q, r.dt).step(q, r.nsteps)
        torch.cuda.synchronize()
        alone = PT.to_host(q)
        if r.result_mode == "state":
            assert np.array_equal(r.result, alone), r.rid
        else:
            mj = r.dg.MJ
            ref = np.sqrt([np.sum(mj * alone[c] ** 2) for c in range(alone.shape[0])])
            assert r.result.shape == ref.shape
            assert np.allclose(r.result, ref, rtol=1e-13, atol=0), r.rid
    srv.close()


def test_device_built_states_match_host_builders():
    """The device builders of the serving workload restate the host ones."""
    from atum_b200 import workloads as W
    for c, fn in ((P.vortex_c1(N=3, K=4), W.vortex_c1_device), (P.bubble_3d(N=3, K=3, imex=False),
                                                                W.bubble_3d_device)):
        q0, _ = fn(c.dg)
        assert np.allclose(PT.to_host(q0), c.q0, rtol=1e-14, atol=1e-12)

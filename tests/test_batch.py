"""Multi-instance batching (atb_op_create_batch): a packed operator gives every
instance bitwise the result that instance gets alone -- tendencies, LSRK steps
with per-instance time steps, ARK23 IMEX steps with the banded column solve --
and the launch-shape autotuner changes no result."""
import numpy as np
import pytest

import atum_b200 as A
import parity as PT
import problems as P

pytestmark = pytest.mark.gpu


def _sw_instances(Ks, precision="fp64"):
    return [P.sw_fplane(N=4, K=k, seed=100 + i, precision=precision) for i, k in enumerate(Ks)]


def test_tendency_packed_equals_alone():
    import torch
    cases = _sw_instances([4, 7, 5])
    packed = A.batch.PackedDGSEM([c.dg for c in cases])
    assert packed.offsets == [0, 16, 65, 90]
    qs = [PT.to_dev(c.q0) for c in cases]
    q = packed.pack(qs)
    dq = torch.zeros_like(q)
    packed(dq, q, 0.0, increment=False)
    for c, qi, part in zip(cases, qs, packed.unpack(dq)):
        alone = torch.zeros_like(qi)
        c.dg(alone, qi, 0.0, increment=False)
        assert torch.equal(part, alone)


def test_tendency_packed_3d_nonperiodic():
    import torch
    cases = [P.bubble_3d(N=3, K=3, imex=False), P.bubble_3d(N=3, K=4, imex=False, L=8e3)]
    packed = A.batch.PackedDGSEM([c.dg for c in cases])
    rng = np.random.default_rng(5)
    qs = [PT.to_dev(c.q0 * (1 + 1e-3 * rng.standard_normal(c.q0.shape))) for c in cases]
    q = packed.pack(qs)
    dq = torch.zeros_like(q)
    packed(dq, q, 0.0, increment=False)
    for c, qi, part in zip(cases, qs, packed.unpack(dq)):
        alone = torch.zeros_like(qi)
        c.dg(alone, qi, 0.0, increment=False)
        assert torch.equal(part, alone)


def test_lsrk_per_instance_dt():
    import torch
    cases = _sw_instances([4, 6, 5], precision="fp32flux")
    packed = A.batch.PackedDGSEM([c.dg for c in cases])
    qs = [PT.to_dev(c.q0) for c in cases]
    q = packed.pack(qs)
    s = A.LSRK54(packed, q, cases[0].dt)
    A.batch.set_instance_dt(s, [c.dt for c in cases])
    s.step(q, 7)
    for c, qi, part in zip(cases, qs, packed.unpack(q)):
        si = A.LSRK54(c.dg, qi, c.dt)
        si.step(qi, 7)
        assert torch.equal(part, qi)
    # back to the single dt
    A.batch.set_instance_dt(s, None)
    s.step(q, 1)
    assert torch.isfinite(q).all()


def test_ark23_packed_equals_alone():
    import torch
    cases = [P.bubble_3d(N=3, K=4, imex=True, steps=3) for _ in range(3)]
    rng = np.random.default_rng(11)
    q0s = [c.q0 * (1 + 1e-4 * rng.standard_normal(c.q0.shape)) for c in cases]
    packed = A.batch.PackedDGSEM([c.dg for c in cases])
    plin = A.batch.PackedDGSEM([c.lindg for c in cases])
    q = packed.pack([PT.to_dev(a) for a in q0s])
    s = A.ARK23(packed, plin, q, cases[0].dt, split_rhs=False)
    s.step(q, 3)
    for c, a, part in zip(cases, q0s, packed.unpack(q)):
        qi = PT.to_dev(a)
        si = A.ARK23(c.dg, c.lindg, qi, c.dt, split_rhs=False)
        si.step(qi, 3)
        assert torch.equal(part, qi)


def test_ark23_ragged_batch_rejected():
    cases = [P.bubble_3d(N=3, K=3, imex=True), P.bubble_3d(N=3, K=4, imex=True)]
    packed = A.batch.PackedDGSEM([c.dg for c in cases])
    plin = A.batch.PackedDGSEM([c.lindg for c in cases])
    q = packed.pack([PT.to_dev(c.q0) for c in cases])
    with pytest.raises(A._lib.AtbError, match="share their element counts"):
        A.ARK23(packed, plin, q, cases[0].dt, split_rhs=False).step(q, 1)


def test_mixed_kinds_rejected():
    a = P.sw_fplane(N=4, K=4)
    b = P.sw_fplane(N=4, K=4, precision="fp32flux")
    with pytest.raises(A._lib.AtbError, match="differs from instance 0"):
        A.batch.PackedDGSEM([a.dg, b.dg])
    c = P.sw_fplane(N=3, K=4)
    with pytest.raises(A._lib.AtbError, match="differs from instance 0"):
        A.batch.PackedDGSEM([a.dg, c.dg])


def test_autotune_keeps_results():
    import torch
    cases = _sw_instances([8] * 6)
    packed = A.batch.PackedDGSEM([c.dg for c in cases])
    q = packed.pack([PT.to_dev(c.q0) for c in cases])
    ref = torch.zeros_like(q)
    packed(ref, q, 0.0, increment=False)
    E = packed.autotune(q)
    assert 1 <= E <= 16
    out = torch.zeros_like(q)
    packed(out, q, 0.0, increment=False)
    assert torch.equal(out, ref)
    for e in (1, 3, 7):
        packed.set_launch(e)
        packed(out, q, 0.0, increment=False)
        assert torch.equal(out, ref)
    with pytest.raises(A._lib.AtbError):
        packed.set_launch(0)

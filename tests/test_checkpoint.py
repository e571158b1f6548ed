"""Checkpoint / resume (atum_b200.checkpoint, atb_solver_set_state).

On the CPU: the raw file format round-trips bit for bit and damaged files are
rejected.  On the GPU: a run stopped after n steps, written to disk, and
continued by a solver rebuilt from scratch ends bit for bit where the
uninterrupted run ends, for LSRK54, RLSRK54 (whose Newton starts from the
last relaxation factor) and ARK23 (banded solve)."""
import os

import numpy as np
import pytest

import atum_b200 as A
import parity as PT
import problems as P
from atum_b200 import checkpoint as CK


class _FakeSolver:
    kind = "LSRK54"

    def state(self):
        return {"kind": self.kind, "time": 0.125, "dt": 1e-3, "gamma": 0.9999999999999998}


def test_format_round_trip(tmp_path):
    rng = np.random.default_rng(7)
    q = rng.standard_normal((5, 40, 25))  # (Ns, K, Np), as the state arrays are
    q[2, 3, 0] = -0.0
    q[4, 7, 1] = 1e-310  # subnormal
    p = str(tmp_path / "run.ckpt")
    h = CK.save(p, q, _FakeSolver(), meta={"step": 40})
    q2, h2 = CK.load(p)
    assert q2.dtype == np.float64 and q2.shape == q.shape
    assert q2.tobytes() == q.tobytes()
    assert h2 == h and h2["solver"]["gamma"] == 0.9999999999999998 and h2["meta"]["step"] == 40
    assert not os.path.exists(p + ".tmp")


def test_damaged_files_rejected(tmp_path):
    q = np.zeros((4, 10))
    p = str(tmp_path / "a.ckpt")
    CK.save(p, q)
    raw = open(p, "rb").read()
    open(p, "wb").write(raw[:-8])
    with pytest.raises(ValueError, match="truncated"):
        CK.load(p)
    open(p, "wb").write(b"NOTACKPT" + raw[8:])
    with pytest.raises(ValueError, match="not a checkpoint"):
        CK.load(p)
    with pytest.raises(TypeError):
        CK.save(p, q.astype(np.float32))
    with pytest.raises(ValueError, match="components first"):
        CK.save(p, np.zeros(10))
    with pytest.raises(ValueError, match="no solver state"):
        CK.resume(_FakeSolver(), {"solver": None})


def _resume_matches(case, make, n, tmp_path):
    # uninterrupted
    qa = PT.to_dev(case.q0)
    sa = make(case, qa)
    sa.step(qa, 2 * n)
    # stopped after n steps, saved, continued by a new solver
    qb = PT.to_dev(case.q0)
    sb = make(case, qb)
    sb.step(qb, n)
    p = str(tmp_path / "mid.ckpt")
    CK.save(p, qb, sb)
    del sb, qb
    qc, h = CK.load(p, device="cuda")
    sc = make(case, qc)
    CK.resume(sc, h)
    sc.step(qc, n)
    assert sc.time == sa.time and sc.gamma == sa.gamma
    assert np.array_equal(qc.cpu().numpy(), qa.cpu().numpy())


@pytest.mark.gpu
def test_resume_lsrk54_bitwise(tmp_path):
    case = P.vortex_c1(N=3, K=8, steps=20)
    _resume_matches(case, lambda c, q: A.LSRK54(c.dg, q, c.dt), 10, tmp_path)


@pytest.mark.gpu
def test_resume_rlsrk54_bitwise(tmp_path):
    case = P.square_1d("euler")
    _resume_matches(case, lambda c, q: A.RLSRK54(c.dg, q, c.dt), 12, tmp_path)


@pytest.mark.gpu
def test_resume_ark23_bitwise(tmp_path):
    case = P.bubble_3d(N=3, K=4, imex=True, steps=8)
    _resume_matches(case, lambda c, q: A.ARK23(c.dg, c.lindg, q, c.dt, split_rhs=False), 4, tmp_path)


@pytest.mark.gpu
def test_set_state_rejects_non_finite():
    case = P.vortex_c1(N=3, K=8, steps=2)
    q = PT.to_dev(case.q0)
    s = A.LSRK54(case.dg, q, case.dt)
    with pytest.raises(Exception):
        s.set_state(float("nan"), 1.0)
    s.set_state(2.5, 1.0)
    assert s.time == 2.5


def test_resume_restores_dt_and_state():
    class S:
        kind = "LSRK54"
        dt = 1e-3
        calls = []

        def set_state(self, time, gamma):
            self.calls.append((time, gamma))

    s = S()
    CK.resume(s, {"solver": {"kind": "LSRK54", "time": 2.5, "dt": 2e-3, "gamma": 0.75}})
    assert s.dt == 2e-3 and s.calls == [(2.5, 0.75)]
    with pytest.raises(ValueError, match="RLSRK54"):
        CK.resume(s, {"solver": {"kind": "RLSRK54", "time": 0.0, "dt": 2e-3, "gamma": 1.0}})

"""Programmatic dependent launch changes when kernels start, not what they
compute.

The tendency kernels (flat and curved) and the banded solves are launched with
programmatic stream serialization unless ATB_PDL=0 is set (read once per
process, so each setting runs in a fresh process).  Every such kernel waits for
the previous grid's completion before its first dependent read, so the states
after whole time steps must agree bit for bit: IMEX ARK23 on the rising bubble
(fused stage kernel + shared-factor banded solve), LSRK54 on the same bubble
(five tendency launches per step), and ARK23 on a small cubed-sphere shell
(curved stage kernel + per-line banded solve).
"""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import bench
A = bench.load_pkg()
import torch
from atum_b200 import workloads as W

out = []
case = W.bubble_3d(N=3, K=(4, 4, 6), imex=True, steps=3)
q = torch.as_tensor(case.q0, device="cuda").contiguous()
s = A.ARK23(case.dg, case.lindg, q, case.dt, split_rhs=False)
s.step(q, 3)
out.append(q.cpu().numpy().ravel())
case = W.bubble_3d(N=3, K=(4, 4, 6), imex=False, steps=3)
q = torch.as_tensor(case.q0, device="cuda").contiguous()
s = A.LSRK54(case.dg, q, case.dt)
s.step(q, 3)
out.append(q.cpu().numpy().ravel())
case = W.sphere_acoustic_wave(N=2, KH=3, KV=3, steps=2)
q = torch.as_tensor(case.q0, device="cuda").contiguous()
s = A.ARK23(case.dg, case.lindg, q, case.dt, split_rhs=False)
s.step(q, 2)
out.append(q.cpu().numpy().ravel())
torch.cuda.synchronize()
np.save(sys.argv[2], np.concatenate(out))
"""


def _run(tmp_path, pdl):
    env = dict(os.environ)
    env["ATB_PDL"] = "1" if pdl else "0"
    out = str(tmp_path / f"pdl{int(pdl)}.npy")
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT, out], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-4000:]
    return np.load(out)


def test_pdl_launches_leave_results_bitwise_unchanged(tmp_path):
    a = _run(tmp_path, True)
    b = _run(tmp_path, False)
    assert np.isfinite(a).all()
    assert np.array_equal(a, b)

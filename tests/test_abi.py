"""C-ABI checks that need no GPU: the library loads and exports every entry
point ``include/atum_b200.h`` declares; argument validation fails loudly."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import atum_b200 as A

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "atum_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(atb_\w+)\s*\(", src, re.M)))


def test_header_declares_entry_points():
    names = _declared()
    assert "atb_op_create" in names and "atb_solve" in names and len(names) >= 15


def test_library_exports_every_declared_symbol():
    from atum_b200 import _lib
    L = _lib.lib()
    for n in _declared():
        assert hasattr(L, n), n
    assert L.atb_version() >= 1


def test_python_binding_covers_header():
    from atum_b200 import _lib
    for n in _declared():
        assert n in _lib.SIGNATURES or n == "atb_last_error", n


def test_invalid_descriptor_rejected_without_gpu():
    from atum_b200 import _lib, _device
    dg = A.DGSEM(law=A.EulerLaw(2), grid=A.brickgrid(A.LobattoCell(3, 3), ([0, 1], [0, 1])),
                 surface_numericalflux=A.RusanovFlux())
    d, keep = _device.make_desc(dg)
    d.N = 9  # beyond the supported orders: rejected before any device call
    h = C.c_void_p()
    rc = _lib.lib().atb_op_create(C.byref(d), None, C.byref(h))
    assert rc == -1
    assert b"order" in _lib.lib().atb_last_error()


def test_host_spec_validation():
    with pytest.raises(NotImplementedError):
        A.DGSEM(law=A.AdvectionLaw(2), grid=A.brickgrid(A.LobattoCell(3, 3), ([0, 1], [0, 1])),
                surface_numericalflux=A.RoeFlux())
    with pytest.raises(ValueError):
        A.FluxDifferencingForm(A.EntropyConservativeFlux(), "bogus")
    with pytest.raises(ValueError):
        A.DGSEM(law=A.EulerLaw(2), grid=A.brickgrid(A.LobattoCell(3, 3), ([0, 1], [0, 1])),
                surface_numericalflux=A.RusanovFlux(), directions=(3,))


def test_lgl_tables_match_oracle(orc):
    for N in range(1, 8):
        c = A.LobattoCell(N + 1)
        # D annihilates constants and differentiates x exactly
        assert np.allclose(c.D @ np.ones(N + 1), 0, atol=1e-13)
        assert np.allclose(c.D @ c.nodes, 1, atol=1e-12)
        assert abs(c.weights.sum() - 2) < 1e-14


@pytest.mark.parametrize("dt", [0.0, -1e-3, float("nan"), float("inf")])
def test_solver_rejects_unusable_dt_without_gpu(dt):
    """A dt that is not finite and positive would make solve! loop forever;
    the constructor rejects it before touching the operators or the device."""
    from atum_b200 import _lib
    h = C.c_void_p()
    L = _lib.lib()
    rc = L.atb_solver_create(0, None, None, dt, 0.0, 1, 0, C.byref(h))
    assert rc == -1
    assert b"dt must be finite and positive" in L.atb_last_error()
    assert not h.value

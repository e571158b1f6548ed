"""ctypes binding of the C ABI in ``include/atum_b200.h``.

Loads ``csrc/libatumb200.so`` from this package directory.  There is no
fallback: if the library is missing or fails to load, every device call
raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "csrc", "libatumb200.so")

ATB_OK = 0
ERRORS = {-1: "invalid argument", -2: "CUDA error", -3: "out of device memory", -4: "non-finite state",
          -5: "HBM budget exceeded", -6: "device wait timed out", -7: "stage callback failed"}


class AtbError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"atum_b200 error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


class OpDesc(C.Structure):
    _fields_ = [
        ("law", C.c_int), ("dim", C.c_int), ("N", C.c_int), ("K", C.c_int * 3),
        ("vertices", C.POINTER(C.c_double) * 3), ("periodic", C.c_int * 3), ("stacked", C.c_int),
        ("volume_form", C.c_int), ("volume_flux", C.c_int), ("fd_kernel", C.c_int), ("surface_flux", C.c_int),
        ("directions", C.c_int), ("gamma", C.c_double), ("grav", C.c_double), ("adv_u", C.c_double * 3),
        ("sphere", C.c_int), ("pde_level_balance", C.c_int), ("bc_kind", C.c_int),
        ("bc_state", (C.c_double * 5) * 2), ("source_kind", C.c_int), ("omega", C.c_double * 3),
        ("sw_topography", C.c_int), ("naux", C.c_int), ("precision", C.c_int),
        ("lgl_nodes", C.POINTER(C.c_double)), ("lgl_weights", C.POINTER(C.c_double)),
        ("lgl_D", C.POINTER(C.c_double)),
    ]


PtrArr = C.c_void_p * 5
_LIB = None
# int (*)(double ex_time, double im_time, double* const* q_stage, void* user)
STAGE_CB = C.CFUNCTYPE(C.c_int, C.c_double, C.c_double, C.POINTER(C.c_void_p), C.c_void_p)
# int (*)(double* const* state, void* user): atb_solver_set_exchange_callback
EXCHANGE_CB = C.CFUNCTYPE(C.c_int, C.POINTER(C.c_void_p), C.c_void_p)

# exported entry points and their argtypes (every one returns int status)
_VP, _DP, _IP = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int)
class CurvedGeometry(C.Structure):
    """``atb_curved_geometry``: per-node metric terms and M J, per face node
    normals, face masses and neighbour nodes, per face boundary tags."""
    _fields_ = [
        ("metric", C.POINTER(C.c_double)), ("mj", C.POINTER(C.c_double)), ("normals", C.POINTER(C.c_double)),
        ("face_mj", C.POINTER(C.c_double)), ("nbr_node", C.POINTER(C.c_longlong)), ("btag", C.POINTER(C.c_int)),
    ]


SIGNATURES = {
    "atb_version": [],
    "atb_device_count": [_IP],
    "atb_op_create": [C.POINTER(OpDesc), _DP, C.POINTER(C.c_void_p)],
    "atb_op_destroy": [_VP],
    "atb_op_dims": [_VP, _IP, _IP, _IP],
    "atb_op_set_aux": [_VP, _DP, _VP],
    "atb_op_create_curved": [C.POINTER(OpDesc), _DP, C.POINTER(CurvedGeometry), C.POINTER(C.c_void_p)],
    "atb_op_create_batch": [C.POINTER(OpDesc), C.c_int, C.POINTER(_DP), C.POINTER(C.c_void_p)],
    "atb_op_instances": [_VP, _IP, _IP],
    "atb_op_autotune": [_VP, PtrArr, _DP, _VP, _IP],
    "atb_op_set_launch": [_VP, C.c_int],
    "atb_op_set_persistent": [_VP, C.c_int],
    "atb_op_set_active": [_VP, C.c_int],
    "atb_op_create_pool": [C.POINTER(OpDesc), C.c_int, C.POINTER(C.c_void_p)],
    "atb_op_place_instance": [_VP, C.c_int, C.POINTER(OpDesc), _DP, _VP],
    "atb_op_set_active_elements": [_VP, C.c_int],
    "atb_op_move_instance": [_VP, C.c_int, C.c_int, C.c_int, _VP, _VP],
    "atb_op_set_instance_aux": [_VP, C.c_int, _DP, _VP],
    "atb_op_copy_instance_aux": [_VP, C.c_int, C.c_int, _VP],
    "atb_op_apply": [_VP, PtrArr, PtrArr, C.c_double, C.c_int, _VP],
    "atb_solver_create": [C.c_int, _VP, _VP, C.c_double, C.c_double, C.c_int, C.c_int, C.POINTER(C.c_void_p)],
    "atb_solver_destroy": [_VP],
    "atb_solver_step": [_VP, PtrArr, C.c_int, _VP],
    "atb_solve": [_VP, PtrArr, C.c_double, C.c_int, _IP, _VP],
    "atb_solver_get": [_VP, _DP, _DP, _DP],
    "atb_solver_set_dt": [_VP, C.c_double],
    "atb_solver_set_state": [_VP, C.c_double, C.c_double],
    "atb_solver_set_instance_dt": [_VP, _DP],
    "atb_solver_set_element_dt": [_VP, _DP],
    "atb_solver_fuse": [_VP, C.c_int],
    "atb_weightednorm": [_VP, PtrArr, C.c_double, _DP, _DP, _VP],
    "atb_entropyintegral": [_VP, PtrArr, _DP, _VP],
    "atb_entropyproduct": [_VP, PtrArr, PtrArr, _DP, _VP],
    "atb_check_finite": [_VP, PtrArr, _VP],
    "atb_probe_fp64_peak": [_DP, _VP],
    "atb_profile_enable": [C.c_int],
    "atb_profile_reset": [],
    "atb_profile_read": [C.c_int, C.POINTER(C.c_long), _DP],
    "atb_launch_count": [C.POINTER(C.c_long)],
    "atb_lsrk54_step_noalloc": [_VP, PtrArr, C.c_double, C.c_int, _VP],
    "atb_solver_set_stage_callback": [_VP, STAGE_CB, _VP],
    "atb_solver_set_exchange_callback": [_VP, EXCHANGE_CB, _VP],
}


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIBPATH):
            raise AtbError(-1, f"{LIBPATH} is not built: run atum_b200 build (python atum.jl_b200/build.py)")
        L = C.CDLL(LIBPATH)
        for name, args in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        L.atb_last_error.restype = C.c_char_p
        L.atb_last_error.argtypes = []
        _LIB = L
    return _LIB


def check(rc: int):
    if rc != ATB_OK:
        raise AtbError(rc, lib().atb_last_error().decode(errors="replace"))


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def field_ptrs(t, ns: int) -> PtrArr:
    """Pointer array for a (Ns, K, Np) float64 CUDA tensor (or a list of component tensors)."""
    import torch

    if isinstance(t, (list, tuple)):
        comps = list(t)
    else:
        if not isinstance(t, torch.Tensor):
            raise TypeError("fields are torch float64 CUDA tensors")
        comps = [t[s] for s in range(t.shape[0])]
    if len(comps) != ns:
        raise ValueError(f"expected {ns} state components, got {len(comps)}")
    arr = PtrArr()
    for s, c in enumerate(comps):
        if c.dtype != torch.float64 or not c.is_cuda or not c.is_contiguous():
            raise TypeError("state components must be contiguous float64 CUDA tensors")
        arr[s] = c.data_ptr()
    for s in range(len(comps), 5):
        arr[s] = arr[0]
    return arr


class _DeviceBlock:
    """A device array given by its address, for zero-copy torch views
    (``__cuda_array_interface__``)."""

    def __init__(self, ptr: int, shape):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<f8", "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def device_view(ptrs, ns: int, shape):
    """Torch view (no copy) of a state held as ``ns`` device component
    pointers: one (ns, *shape) tensor when the components are consecutive,
    else a list of component tensors."""
    import torch

    n = int(np.prod(shape))
    p = [int(ptrs[c] or 0) for c in range(ns)]
    if all(p[c] == p[0] + 8 * n * c for c in range(ns)):
        return torch.as_tensor(_DeviceBlock(p[0], (ns,) + tuple(shape)), device="cuda")
    return [torch.as_tensor(_DeviceBlock(p[c], tuple(shape)), device="cuda") for c in range(ns)]


def stream_ptr(stream=None):
    import torch

    if stream is None:
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream)

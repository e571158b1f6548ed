"""Device handle of a DGSEM spec: owns the ``atb_op`` created through the C ABI."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib


def make_desc(dg) -> tuple:
    f = dg.descriptor_fields()
    d = _lib.OpDesc()
    keep = []
    for k, v in f.items():
        if k == "vertices":
            for i, vv in enumerate(v):
                arr = np.ascontiguousarray(vv, dtype=np.float64)
                keep.append(arr)
                d.vertices[i] = _lib.dptr(arr)
        elif k in ("K", "periodic", "adv_u", "omega"):
            arr = getattr(d, k)
            for i, x in enumerate(v):
                arr[i] = x
        elif k == "bc_state":
            for i in range(2):
                for j in range(5):
                    d.bc_state[i][j] = v[i][j]
        else:
            setattr(d, k, v)
    cell = dg.grid.cell
    for name, arr in (("lgl_nodes", cell.nodes), ("lgl_weights", cell.weights), ("lgl_D", cell.D)):
        a = np.ascontiguousarray(arr, dtype=np.float64).reshape(-1)
        keep.append(a)
        setattr(d, name, _lib.dptr(a))
    return d, keep


class DeviceOp:
    def __init__(self, dg):
        self.dg = dg
        self.ns = dg.law.numberofstates
        desc, keep = make_desc(dg)
        h = C.c_void_p()
        dev_aux = getattr(dg, "_aux_dev", None)
        if hasattr(dg.grid, "geometry"):
            # curved elements: the grid's metric terms, face normals / masses and face map
            G = dg.grid.geometry()
            arrs = [np.ascontiguousarray(G[k], dtype=np.float64) for k in ("g", "MJ", "normals", "faceMJ")]
            nb = np.ascontiguousarray(G["nbr_node"], dtype=np.int64)
            bt = np.ascontiguousarray(G["btag"], dtype=np.int32)
            geo = _lib.CurvedGeometry(_lib.dptr(arrs[0]), _lib.dptr(arrs[1]), _lib.dptr(arrs[2]), _lib.dptr(arrs[3]),
                                      nb.ctypes.data_as(C.POINTER(C.c_longlong)),
                                      bt.ctypes.data_as(C.POINTER(C.c_int)))
            aux = None if dev_aux is not None else np.ascontiguousarray(dg.auxstate_host(), dtype=np.float64)
            _lib.check(_lib.lib().atb_op_create_curved(C.byref(desc), _lib.dptr(aux) if aux is not None and aux.size
                                                       else None, C.byref(geo), C.byref(h)))
            self.h = h
            if dev_aux is not None:
                _lib.check(_lib.lib().atb_op_set_aux(h, C.cast(C.c_void_p(dev_aux.data_ptr()), _lib._DP),
                                                     _lib.stream_ptr()))
                import torch
                torch.cuda.current_stream().synchronize()
        elif dev_aux is not None:
            # aux evaluated on the device: create with zeros, then copy device to device
            _lib.check(_lib.lib().atb_op_create(C.byref(desc), None, C.byref(h)))
            self.h = h
            _lib.check(_lib.lib().atb_op_set_aux(h, C.cast(C.c_void_p(dev_aux.data_ptr()), _lib._DP),
                                                 _lib.stream_ptr()))
            import torch
            torch.cuda.current_stream().synchronize()
        else:
            aux = np.ascontiguousarray(dg.auxstate_host(), dtype=np.float64)
            _lib.check(_lib.lib().atb_op_create(C.byref(desc), _lib.dptr(aux) if aux.size else None, C.byref(h)))
            self.h = h
        self._keep = keep

    def __del__(self):
        h = getattr(self, "h", None)
        if h and _lib._LIB is not None:
            _lib._LIB.atb_op_destroy(h)
            self.h = None

    def apply(self, dq, q, time=0.0, increment=True, stream=None):
        L = _lib.lib()
        _lib.check(L.atb_op_apply(self.h, _lib.field_ptrs(dq, self.ns), _lib.field_ptrs(q, self.ns),
                                  float(time), int(bool(increment)), _lib.stream_ptr(stream)))

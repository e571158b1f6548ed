"""VTK output of nodal fields: XML unstructured grids (.vtu) and ParaView
time collections (.pvd).

The reference's experiments write snapshots with WriteVTK through Bennu
(``vtk_grid(file, grid)``, fields interpolated to equispaced nodes for
Lagrange cells, experiment/euler_gravity/risingbubble.jl:75-101).  Here every
element is written as the linear sub-cells between its neighbouring LGL nodes
(N^dim lines / quadrilaterals / hexahedra per element), so the points are the
nodes themselves and the values are the nodal values exactly, with no
interpolation.  Fields are host arrays (or torch tensors) shaped like one
state component: (K, Np), node index i + Nq (j + Nq k) fastest.

``write_vtu(path, grid, fields)`` writes one snapshot; ``write_pvd(path,
entries)`` a collection of (time, file) snapshots, which ParaView opens as a
time series (WriteVTK's ``paraview_collection``).
"""
from __future__ import annotations

import base64
import os
from typing import Dict, Iterable, Tuple

import numpy as np

__all__ = ["write_vtu", "write_pvd", "subcell_connectivity"]

# VTK cell type ids of the linear cells
_VTK_LINE, _VTK_QUAD, _VTK_HEXAHEDRON = 3, 9, 12


def subcell_connectivity(dim: int, Nq: int) -> np.ndarray:
    """Corner nodes of the (Nq-1)^dim linear sub-cells of one element, in VTK
    order (counter-clockwise in each i-j layer, the k = 0 layer first); shape
    (cells, 2^dim), node numbers i + Nq (j + Nq k)."""
    n = Nq - 1
    node = lambda i, j=0, k=0: i + Nq * (j + Nq * k)  # noqa: E731
    cells = []
    if dim == 1:
        for i in range(n):
            cells.append([node(i), node(i + 1)])
    elif dim == 2:
        for j in range(n):
            for i in range(n):
                cells.append([node(i, j), node(i + 1, j), node(i + 1, j + 1), node(i, j + 1)])
    elif dim == 3:
        for k in range(n):
            for j in range(n):
                for i in range(n):
                    lo = [node(i, j, k), node(i + 1, j, k), node(i + 1, j + 1, k), node(i, j + 1, k)]
                    hi = [node(i, j, k + 1), node(i + 1, j, k + 1), node(i + 1, j + 1, k + 1), node(i, j + 1, k + 1)]
                    cells.append(lo + hi)
    else:
        raise ValueError(f"dim must be 1, 2 or 3 (got {dim})")
    return np.asarray(cells, dtype=np.int64)


def _host(a) -> np.ndarray:
    if not isinstance(a, np.ndarray):
        a = a.detach().cpu().numpy()
    return np.ascontiguousarray(a)


def _data_array(name: str, a: np.ndarray, ncomp: int, binary: bool) -> str:
    vt = {np.dtype(np.float64): "Float64", np.dtype(np.int64): "Int64", np.dtype(np.uint8): "UInt8"}[a.dtype]
    attrs = f'type="{vt}" Name="{name}" NumberOfComponents="{ncomp}"'
    if binary:
        # inline base64 of a UInt64 byte count followed by the raw
        # little-endian values (uncompressed)
        raw = a.astype(a.dtype.newbyteorder("<"), copy=False).tobytes()
        payload = base64.b64encode(np.uint64(len(raw)).tobytes() + raw).decode("ascii")
        return f'<DataArray {attrs} format="binary">{payload}</DataArray>'
    if a.dtype.kind == "f":
        body = " ".join(repr(float(v)) for v in a.reshape(-1))
    else:
        body = " ".join(str(int(v)) for v in a.reshape(-1))
    return f'<DataArray {attrs} format="ascii">{body}</DataArray>'


def write_vtu(path: str, grid, fields: Dict[str, object], binary: bool = False) -> str:
    """Writes ``fields`` (name -> nodal array shaped (K, Np) or with K*Np
    values) on ``grid`` to ``path`` (".vtu" appended when missing); returns
    the file name.  ``binary`` stores the arrays base64-encoded inline
    instead of as text."""
    if not path.endswith(".vtu"):
        path += ".vtu"
    dim, K, Np, Nq = grid.dim, grid.K, grid.cell.Np, grid.cell.Nq
    x = np.asarray(grid.points(), dtype=np.float64).reshape(dim, K * Np)
    pts = np.zeros((K * Np, 3))
    pts[:, :dim] = x.T
    local = subcell_connectivity(dim, Nq)
    conn = (local[None, :, :] + (np.arange(K, dtype=np.int64) * Np)[:, None, None]).reshape(-1)
    ncell = K * local.shape[0]
    nv = local.shape[1]
    offsets = np.arange(1, ncell + 1, dtype=np.int64) * nv
    ctype = {1: _VTK_LINE, 2: _VTK_QUAD, 3: _VTK_HEXAHEDRON}[dim]
    types = np.full(ncell, ctype, dtype=np.uint8)
    data = []
    for name, v in fields.items():
        a = _host(v).astype(np.float64, copy=False).reshape(-1)
        if a.size != K * Np:
            raise ValueError(f"field {name!r} has {a.size} values, the grid {K * Np} nodes")
        data.append(_data_array(name, a, 1, binary))
    parts = [
        '<?xml version="1.0"?>',
        '<VTKFile type="UnstructuredGrid" version="1.0" byte_order="LittleEndian" header_type="UInt64">',
        "<UnstructuredGrid>",
        f'<Piece NumberOfPoints="{K * Np}" NumberOfCells="{ncell}">',
        "<Points>", _data_array("Points", pts.reshape(-1), 3, binary), "</Points>",
        "<Cells>",
        _data_array("connectivity", conn, 1, binary),
        _data_array("offsets", offsets, 1, binary),
        _data_array("types", types, 1, binary),
        "</Cells>",
        "<PointData>", *data, "</PointData>",
        "</Piece>", "</UnstructuredGrid>", "</VTKFile>", "",
    ]
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        f.write("\n".join(parts))
    os.replace(tmp, path)
    return path


def write_pvd(path: str, entries: Iterable[Tuple[float, str]]) -> str:
    """A ParaView collection of ``(time, vtu file)`` snapshots; the files are
    referenced relative to the collection's directory."""
    if not path.endswith(".pvd"):
        path += ".pvd"
    base = os.path.dirname(os.path.abspath(path))
    rows = []
    for t, f in entries:
        rel = os.path.relpath(os.path.abspath(f), base)
        rows.append(f'<DataSet timestep="{float(t)!r}" group="" part="0" file="{rel}"/>')
    text = "\n".join(['<?xml version="1.0"?>',
                      '<VTKFile type="Collection" version="1.0" byte_order="LittleEndian">',
                      "<Collection>", *rows, "</Collection>", "</VTKFile>", ""])
    with open(path, "w") as f:
        f.write(text)
    return path

"""VTK output (atum_b200.vtk): the written unstructured grid has the grid's
nodes as points, N^dim linear sub-cells per element that tile every element
exactly once, and the fields' nodal values; ASCII and inline-binary files
decode to the same arrays; the .pvd collection lists the snapshots."""
import base64
import os
import xml.etree.ElementTree as ET

import numpy as np
import pytest

import atum_b200 as A
from atum_b200 import vtk


def _decode(da, header=np.uint64):
    dt = {"Float64": np.float64, "Int64": np.int64, "UInt8": np.uint8}[da.get("type")]
    if da.get("format") == "ascii":
        return np.array(da.text.split(), dtype=dt)
    raw = base64.b64decode(da.text)
    n = int(np.frombuffer(raw[:8], dtype=header)[0])
    assert n == len(raw) - 8
    return np.frombuffer(raw[8:], dtype=dt)


def _read(path):
    root = ET.parse(path).getroot()
    piece = root.find("UnstructuredGrid/Piece")
    arrays = {da.get("Name"): _decode(da) for da in piece.iter("DataArray")}
    return root, piece, arrays


def _grid(dim, N=3):
    cell = A.LobattoCell(*([N + 1] * dim))
    verts = [np.linspace(0.0, 1.0, 3), np.linspace(-1.0, 2.0, 4), np.array([0.0, 0.5, 2.0])][:dim]
    return A.brickgrid(cell, tuple(verts))


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("binary", [False, True])
def test_vtu_points_cells_fields(tmp_path, dim, binary):
    g = _grid(dim)
    x = g.points()
    rho = np.sin(3 * x[0]) + (x[-1] ** 2 if dim > 1 else 0)
    mom = np.arange(g.K * g.cell.Np, dtype=np.float64).reshape(g.K, g.cell.Np)
    p = vtk.write_vtu(str(tmp_path / "snap"), g, {"rho": rho, "rhou": mom}, binary=binary)
    assert p.endswith(".vtu")
    root, piece, arr = _read(p)
    assert root.get("type") == "UnstructuredGrid"
    npts, ncell = int(piece.get("NumberOfPoints")), int(piece.get("NumberOfCells"))
    N, Np, K = g.cell.N, g.cell.Np, g.K
    assert npts == K * Np and ncell == K * N ** dim
    pts = arr["Points"].reshape(npts, 3)
    assert np.array_equal(pts[:, :dim], x.reshape(dim, -1).T)
    assert np.all(pts[:, dim:] == 0.0)
    nv = 2 ** dim
    conn = arr["connectivity"].reshape(ncell, nv)
    assert np.array_equal(arr["offsets"], np.arange(1, ncell + 1) * nv)
    assert set(arr["types"].tolist()) == {{1: 3, 2: 9, 3: 12}[dim]}
    # every cell lies in one element and spans one node spacing per direction
    assert np.all(conn // Np == conn[:, :1] // Np)
    lo, hi = pts[conn].min(axis=1), pts[conn].max(axis=1)
    assert np.all(hi[:, :dim] > lo[:, :dim])
    # the sub-cells tile each element: their volumes add up to the element's
    vol = np.prod(hi[:, :dim] - lo[:, :dim], axis=1)
    elem = conn[:, 0] // Np
    ev = np.bincount(elem, weights=vol)
    ext = pts.reshape(K, Np, 3)
    want = np.prod(ext[:, :, :dim].max(axis=1) - ext[:, :, :dim].min(axis=1), axis=1)
    assert np.allclose(ev, want, rtol=1e-13)
    assert np.array_equal(arr["rho"], rho.reshape(-1))
    assert np.array_equal(arr["rhou"], mom.reshape(-1))


def test_hexahedron_corner_order():
    # VTK hexahedron: bottom face counter-clockwise, then the top face above it
    c = vtk.subcell_connectivity(3, 2)[0]
    Nq = 2
    ijk = [(n % Nq, (n // Nq) % Nq, n // (Nq * Nq)) for n in c]
    assert ijk == [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]


def test_field_size_checked(tmp_path):
    g = _grid(2)
    with pytest.raises(ValueError, match="nodes"):
        vtk.write_vtu(str(tmp_path / "bad"), g, {"rho": np.zeros(3)})


def test_pvd_collection(tmp_path):
    g = _grid(2)
    files = []
    for k in range(3):
        files.append((0.5 * k, vtk.write_vtu(str(tmp_path / f"step{k:06d}"), g,
                                             {"rho": np.full((g.K, g.cell.Np), float(k))})))
    p = vtk.write_pvd(str(tmp_path / "timesteps"), files)
    root = ET.parse(p).getroot()
    ds = root.findall("Collection/DataSet")
    assert [float(d.get("timestep")) for d in ds] == [0.0, 0.5, 1.0]
    assert [d.get("file") for d in ds] == ["step000000.vtu", "step000001.vtu", "step000002.vtu"]
    for d in ds:
        assert os.path.exists(os.path.join(tmp_path, d.get("file")))

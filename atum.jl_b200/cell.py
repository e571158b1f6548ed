"""Lobatto reference cell and affine brick grid (host side).

Restates the Bennu 0.3 pieces Atum.jl calls on this path (Bennu is an
un-vendored dependency of the reference, `Project.toml:7`, version unpinned):

* ``LobattoCell{FT,A}(Nq, ...)`` -- Legendre-Gauss-Lobatto nodes and weights
  (Newton iteration on ``q = L_{N+1} - L_{N-1}``) and the 1-D derivative matrix
  ``derivatives_1d(cell)[1]`` (barycentric form, negative-sum diagonal);
  used at ``src/dgsem.jl:42-51,111``.
* ``brickgrid(cell, vertices; periodic, ordering)`` -- axis-aligned brick with
  per-dimension vertex vectors, Cartesian or stacked element ordering
  (``test/euler_gravity/linear.jl:63-64``), node coordinates ``points(grid)``
  and ``min_node_distance(grid; dims)``.

The 1-D tables computed here are what the C ABI receives: a Julia caller would
pass Bennu's own ``derivatives_1d`` and weights instead.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

__all__ = ["LobattoCell", "BrickGrid", "brickgrid", "min_node_distance", "points"]


def _lgl(N: int):
    """LGL nodes (ascending) and weights for order N."""
    if N < 1:
        raise ValueError("polynomial order must be >= 1")
    x = np.zeros(N + 1)
    w = np.zeros(N + 1)

    def qeval(xx):
        Lm2, Lm1, dLm2, dLm1 = 1.0, xx, 0.0, 1.0
        for k in range(2, N + 1):
            L = (2.0 * k - 1.0) / k * xx * Lm1 - (k - 1.0) / k * Lm2
            dL = dLm2 + (2.0 * k - 1.0) * Lm1
            Lm2, Lm1, dLm2, dLm1 = Lm1, L, dLm1, dL
        LN1 = (2.0 * N + 1.0) / (N + 1.0) * xx * Lm1 - N / (N + 1.0) * Lm2
        dLN1 = dLm2 + (2.0 * N + 1.0) * Lm1
        return LN1 - Lm2, dLN1 - dLm2, Lm1

    if N == 1:
        return np.array([-1.0, 1.0]), np.array([1.0, 1.0])
    x[0], x[N] = -1.0, 1.0
    w[0] = w[N] = 2.0 / (N * (N + 1.0))
    for j in range(1, (N + 1) // 2):
        xx = -math.cos((j + 0.25) * math.pi / N - 3.0 / (8.0 * N * math.pi * (j + 0.25)))
        for _ in range(100):
            q, dq, _LN = qeval(xx)
            delta = -q / dq
            xx += delta
            if abs(delta) <= 4 * 2.220446049250313e-16 * abs(xx):
                break
        _q, _dq, LN = qeval(xx)
        x[j], x[N - j] = xx, -xx
        w[j] = w[N - j] = 2.0 / (N * (N + 1.0) * LN * LN)
    if N % 2 == 0:
        _q, _dq, LN = qeval(0.0)
        x[N // 2] = 0.0
        w[N // 2] = 2.0 / (N * (N + 1.0) * LN * LN)
    return x, w


def _derivative_matrix(x):
    n = len(x)
    bw = np.ones(n)
    for j in range(n):
        for k in range(n):
            if k != j:
                bw[j] *= x[j] - x[k]
    bw = 1.0 / bw
    D = np.zeros((n, n))
    for i in range(n):
        s = 0.0
        for j in range(n):
            if i == j:
                continue
            D[i, j] = (bw[j] / bw[i]) / (x[i] - x[j])
            s += D[i, j]
        D[i, i] = -s
    return D


class LobattoCell:
    """``LobattoCell{Float64}(Nq, Nq[, Nq])``: tensor-product LGL cell."""

    def __init__(self, *Nqs: int):
        if not 1 <= len(Nqs) <= 3 or any(n != Nqs[0] for n in Nqs):
            raise ValueError("LobattoCell needs 1-3 equal node counts (all(size(cell) .== Nq))")
        self.dim = len(Nqs)
        self.Nq = int(Nqs[0])
        self.N = self.Nq - 1
        self.nodes, self.weights = _lgl(self.N)
        self.D = _derivative_matrix(self.nodes)

    @property
    def Np(self) -> int:
        return self.Nq ** self.dim

    def __repr__(self):
        return f"LobattoCell({', '.join([str(self.Nq)] * self.dim)})"


@dataclass
class BrickGrid:
    cell: LobattoCell
    vertices: tuple
    periodic: tuple
    stacked: bool = False
    _points: np.ndarray | None = field(default=None, repr=False)

    @property
    def dim(self) -> int:
        return self.cell.dim

    @property
    def Kd(self) -> tuple:
        return tuple(len(v) - 1 for v in self.vertices)

    @property
    def K(self) -> int:
        return int(np.prod(self.Kd))

    def __len__(self):
        return self.K

    def element_indices(self):
        """Per-dimension element indices, shape (K, dim), in storage order."""
        Kd = self.Kd
        dim = self.dim
        idx = np.zeros((self.K, dim), dtype=np.int64)
        grids = np.meshgrid(*[np.arange(k) for k in Kd], indexing="ij")
        flat = [g.reshape(-1) for g in grids]
        if self.stacked:
            ev = flat[dim - 1]
            eh = np.zeros_like(ev)
            m = 1
            for d in range(dim - 1):
                eh += flat[d] * m
                m *= Kd[d]
            e = eh * Kd[dim - 1] + ev
        else:
            e = np.zeros_like(flat[0])
            m = 1
            for d in range(dim):
                e += flat[d] * m
                m *= Kd[d]
        for d in range(dim):
            idx[e, d] = flat[d]
        return idx

    def points(self) -> np.ndarray:
        """Node coordinates, shape (dim, K, Np)."""
        if self._points is None:
            c = self.cell
            dim, Nq, Np, K = self.dim, c.Nq, c.Np, self.K
            eidx = self.element_indices()
            node = np.arange(Np)
            ijk = [(node // Nq ** d) % Nq for d in range(dim)]
            x = np.zeros((dim, K, Np))
            for d in range(dim):
                v = np.asarray(self.vertices[d], dtype=np.float64)
                v0 = v[eidx[:, d]][:, None]
                v1 = v[eidx[:, d] + 1][:, None]
                xi = c.nodes[ijk[d]][None, :]
                x[d] = (v0 * (1 - xi) + v1 * (1 + xi)) / 2
            self._points = x
        return self._points


def points_device(grid: "BrickGrid", device="cuda"):
    """Node coordinates as a (dim, K, Np) float64 torch tensor computed on the
    device, in the same storage order and with the same arithmetic as
    ``grid.points()`` (for grids too large to build on the host)."""
    import torch

    c = grid.cell
    dim, Nq, Np, K, Kd = grid.dim, c.Nq, c.Np, grid.K, grid.Kd
    # the node and vertex tables are copied to the device once per grid (a
    # copy from pageable host memory makes the host wait for the stream)
    dev = torch.device(device)
    if dev.type == "cuda" and dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    cache = grid.__dict__.setdefault("_device_tables", {})
    if dev not in cache:
        cache[dev] = (torch.as_tensor(np.asarray(c.nodes, dtype=np.float64), device=dev),
                      [torch.as_tensor(np.asarray(grid.vertices[d], dtype=np.float64), device=dev)
                       for d in range(dim)])
    nodes, verts = cache[dev]
    e = torch.arange(K, device=device, dtype=torch.int64)
    idx = [None] * dim
    if grid.stacked:
        idx[dim - 1] = e % Kd[dim - 1]
        r = e // Kd[dim - 1]
        for d in range(dim - 1):
            idx[d] = r % Kd[d]
            r = r // Kd[d]
    else:
        r = e
        for d in range(dim):
            idx[d] = r % Kd[d]
            r = r // Kd[d]
    node = torch.arange(Np, device=device, dtype=torch.int64)
    x = torch.empty((dim, K, Np), dtype=torch.float64, device=device)
    for d in range(dim):
        v = verts[d]
        v0 = v[idx[d]][:, None]
        v1 = v[idx[d] + 1][:, None]
        xi = nodes[(node // Nq ** d) % Nq][None, :]
        x[d] = (v0 * (1 - xi) + v1 * (1 + xi)) / 2
    return x


def brickgrid(cell: LobattoCell, vertices, periodic=None, ordering: str = "cartesian") -> BrickGrid:
    """``brickgrid(cell, (vx, vy, ...); periodic, ordering)``.

    ``ordering="stacked"`` is ``StackedOrdering{CartesianOrdering}()``: the
    elements of each vertical (last-dimension) column are contiguous, which
    the vertical banded solve of the IMEX stepper needs.
    """
    vertices = tuple(np.asarray(v, dtype=np.float64) for v in vertices)
    if len(vertices) != cell.dim:
        raise ValueError("one vertex vector per cell dimension")
    for v in vertices:
        if len(v) < 2 or not np.all(np.diff(v) > 0):
            raise ValueError("vertex vectors must be strictly increasing with >= 2 entries")
    if periodic is None:
        periodic = (False,) * cell.dim
    if ordering not in ("cartesian", "stacked"):
        raise ValueError("ordering must be 'cartesian' or 'stacked'")
    return BrickGrid(cell, vertices, tuple(bool(p) for p in periodic), ordering == "stacked")


def points(grid: BrickGrid) -> np.ndarray:
    return grid.points()


def min_node_distance(grid: BrickGrid, dims=None) -> float:
    """Smallest distance between neighbouring nodes along ``dims`` (1-based)."""
    if dims is None:
        dims = range(1, grid.dim + 1)
    if hasattr(grid, "min_node_distance"):  # curved grids measure their node coordinates
        return grid.min_node_distance(dims)
    gap = float(np.min(np.diff(grid.cell.nodes)))
    best = math.inf
    for d in dims:
        h = np.diff(grid.vertices[d - 1])
        best = min(best, float(np.min(h)) / 2 * gap)
    return best

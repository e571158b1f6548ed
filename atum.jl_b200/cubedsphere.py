"""Cubed-sphere shell grid and curved-element geometry (host side).

Restates the grid the reference's sphere experiments build with Bennu's
``cubedspheregrid(cell, vr, KH)`` (experiment/euler_gravity/acousticwave.jl:90-92):
six panels of KH x KH elements on the equiangular gnomonic projection of a
cube onto spheres, and KV = len(vr) - 1 layers between the radii ``vr``.  The
elements of each radial column are contiguous (the stacked ordering, which the
vertical banded solve of the IMEX stepper needs), the radial direction is the
third reference direction.  Bennu is not vendored and its version is
unpinned (Project.toml:7): the panel orientation, the node placement (linear
in the equiangular angles and in the radius) and the metric terms are this
module's own restatement.

Geometry, the quantities the reference's DGSEM reads (src/dgsem.jl:38-56
``metrics(grid)``, ``facemetrics(grid)``; 470-561 ``l_g = MJ g[dir, d]``;
683-732 ``faceix``, ``facenormal``, ``faceMJ``):

* node coordinates ``x`` (3, K, Np);
* the contravariant vectors ``J a^i`` per node in Kopriva's conservative curl
  form (D. A. Kopriva, "Metric identities and the discontinuous spectral
  element method on curvilinear meshes", J. Sci. Comput. 26, 2006) with LGL
  spectral differentiation, so the discrete metric identities hold and a
  uniform state stays uniform; the Jacobian ``J`` = det(dx/dxi); the metric
  terms ``g[i, c] = (J a^i)_c / J``;
* per face node: the outward unit normal ``n = +-J a^i / |J a^i|``, ``faceMJ``
  = the face's LGL weights times ``|J a^i|``, and the global node index of the
  matching node of the neighbouring element (found by coordinates), or a
  boundary tag on the inner (tag 5) and the outer (tag 6) sphere.
"""
from __future__ import annotations

import math

import numpy as np

from .cell import LobattoCell

__all__ = ["CubedSphereGrid", "cubedspheregrid"]

# panel p maps the equiangular coordinates (X, Y) = (tan a, tan b) to a cube
# point; every panel's (a, b, r) frame is right-handed with r outwards
_PANELS = (
    lambda X, Y: (np.ones_like(X), X, Y),     # +x
    lambda X, Y: (-X, np.ones_like(X), Y),    # +y
    lambda X, Y: (-np.ones_like(X), -X, Y),   # -x
    lambda X, Y: (X, -np.ones_like(X), Y),    # -y
    lambda X, Y: (-Y, X, np.ones_like(X)),    # +z
    lambda X, Y: (Y, X, -np.ones_like(X)),    # -z
)


def _dxi(f, D, axis):
    """Spectral derivative of nodal values f[..., k, j, i] along reference
    direction ``axis`` (0: i, 1: j, 2: k)."""
    if axis == 0:
        return np.einsum("ab,...kjb->...kja", D, f)
    if axis == 1:
        return np.einsum("ab,...kbi->...kai", D, f)
    return np.einsum("ab,...bji->...aji", D, f)


class CubedSphereGrid:
    """A cubed-sphere shell of 6 x KH x KH x KV curved hexahedra (stacked:
    element e = (panel * KH^2 + j * KH + i) * KV + layer)."""

    dim = 3
    stacked = True
    periodic = (False, False, False)

    def __init__(self, cell: LobattoCell, vr, KH: int):
        if cell.dim != 3:
            raise ValueError("the cubed-sphere grid needs a 3-D cell")
        vr = np.asarray(vr, dtype=np.float64)
        if vr.ndim != 1 or len(vr) < 2 or np.any(np.diff(vr) <= 0) or vr[0] <= 0:
            raise ValueError("vr: increasing positive radii")
        if KH < 1:
            raise ValueError("KH >= 1")
        self.cell = cell
        self.vr = vr
        self.KH = int(KH)
        self.KV = len(vr) - 1
        self.Kd = (6 * self.KH, self.KH, self.KV)  # horizontal columns x layers (used for the stacked layout)
        self._geo = None

    @property
    def K(self) -> int:
        return 6 * self.KH * self.KH * self.KV

    def __len__(self):
        return self.K

    @property
    def vertices(self):
        return (np.arange(6 * self.KH + 1, dtype=np.float64), np.arange(self.KH + 1, dtype=np.float64), self.vr)

    def element_indices(self):
        """(K, 4): panel, i, j, layer of every element in storage order."""
        KH, KV = self.KH, self.KV
        e = np.arange(self.K)
        layer = e % KV
        eh = e // KV
        i = eh % KH
        j = (eh // KH) % KH
        p = eh // (KH * KH)
        return np.stack([p, i, j, layer], axis=1)

    def points(self) -> np.ndarray:
        return self.geometry()["x"]

    def geometry(self) -> dict:
        if self._geo is None:
            self._geo = _build_geometry(self)
        return self._geo

    def min_node_distance(self, dims=None) -> float:
        """Smallest distance between neighbouring nodes along reference
        directions ``dims`` (1-based), measured on the node coordinates."""
        if dims is None:
            dims = (1, 2, 3)
        Nq, K = self.cell.Nq, self.K
        x = self.geometry()["x"].reshape(3, K, Nq, Nq, Nq)  # [c, e, k, j, i]
        best = math.inf
        for d in dims:
            ax = 4 - (d - 1)  # direction 1 -> i (last axis)
            step = np.diff(x, axis=ax)
            best = min(best, float(np.sqrt(np.sum(step * step, axis=0)).min()))
        return best


def cubedspheregrid(cell: LobattoCell, vr, KH: int) -> CubedSphereGrid:
    """``cubedspheregrid(cell, vr, KH)`` (Bennu; experiment/euler_gravity/acousticwave.jl:90-92)."""
    return CubedSphereGrid(cell, vr, KH)


def _build_geometry(g: CubedSphereGrid) -> dict:
    c = g.cell
    Nq, Np, K, KH = c.Nq, c.Np, g.K, g.KH
    xi = c.nodes
    eidx = g.element_indices()
    da = (math.pi / 2) / KH
    # node (k, j, i) of element e: a from xi_1 (i), b from xi_2 (j), r from xi_3 (k)
    a = (-math.pi / 4 + (eidx[:, 1, None] + (xi[None, :] + 1) / 2) * da)         # (K, Nq)
    b = (-math.pi / 4 + (eidx[:, 2, None] + (xi[None, :] + 1) / 2) * da)
    r0, r1 = g.vr[eidx[:, 3]], g.vr[eidx[:, 3] + 1]
    r = (r0[:, None] * (1 - xi[None, :]) + r1[:, None] * (1 + xi[None, :])) / 2  # (K, Nq)
    X = np.tan(a)[:, None, None, :] * np.ones((1, Nq, Nq, 1))                  # [e, k, j, i]
    Y = np.tan(b)[:, None, :, None] * np.ones((1, Nq, 1, Nq))
    R = r[:, :, None, None] * np.ones((1, 1, Nq, Nq))
    x = np.zeros((3, K, Nq, Nq, Nq))
    for p in range(6):
        sel = eidx[:, 0] == p
        cx, cy, cz = _PANELS[p](X[sel], Y[sel])
        nrm = np.sqrt(cx * cx + cy * cy + cz * cz)
        x[0, sel], x[1, sel], x[2, sel] = R[sel] * cx / nrm, R[sel] * cy / nrm, R[sel] * cz / nrm
    D = c.D
    # covariant derivatives dx_n / dxi_j: d[j][n] (K, Nq, Nq, Nq)
    d = [[_dxi(x[n], D, j) for n in range(3)] for j in range(3)]
    J = (d[0][0] * (d[1][1] * d[2][2] - d[1][2] * d[2][1]) - d[0][1] * (d[1][0] * d[2][2] - d[1][2] * d[2][0])
         + d[0][2] * (d[1][0] * d[2][1] - d[1][1] * d[2][0]))
    # J a^i_n = - xhat_i . curl_xi (X_l grad_xi X_m), (n, m, l) cyclic; X_l
    # relative to the element's centroid (the curl of c grad X_m vanishes, so
    # the origin only changes the rounding, which it keeps at the element's
    # size instead of the sphere's radius)
    xc = x - x.mean(axis=(2, 3, 4), keepdims=True)
    JA = np.zeros((3, 3, K, Nq, Nq, Nq))  # [i][n]
    for n in range(3):
        m, l = (n + 1) % 3, (n + 2) % 3
        V = [xc[l] * d[j][m] for j in range(3)]  # V_j = X_l dX_m/dxi_j
        curl = [_dxi(V[2], D, 1) - _dxi(V[1], D, 2),
                _dxi(V[0], D, 2) - _dxi(V[2], D, 0),
                _dxi(V[1], D, 0) - _dxi(V[0], D, 1)]
        for i in range(3):
            JA[i, n] = -curl[i]
    if np.any(J <= 0):
        raise RuntimeError("non-positive Jacobian in the cubed-sphere geometry")
    gm = JA / J[None, None]                              # g[i, n] = d xi_i / d x_n
    w1 = c.weights
    M = (w1[None, :, None, None] * w1[None, None, :, None] * w1[None, None, None, :])[0]  # (k, j, i)
    MJ = M[None] * J
    # faces 2*dir + side: the node index sets, outward normals, faceMJ
    node = np.arange(Np).reshape(Nq, Nq, Nq)  # [k, j, i]
    fnodes = [node[:, :, 0], node[:, :, -1], node[:, 0, :], node[:, -1, :], node[0, :, :], node[-1, :, :]]
    fw = np.outer(w1, w1).reshape(-1)      # face weights in the (row-major) order of fnodes
    Nfp = Nq * Nq
    JAf = JA.reshape(3, 3, K, Np)
    normals = np.zeros((K, 6, Nfp, 3))
    fMJ = np.zeros((K, 6, Nfp))
    for f in range(6):
        dr, side = f // 2, f % 2
        nodes_f = fnodes[f].reshape(-1)
        v = JAf[dr][:, :, nodes_f]               # (3, K, Nfp)
        mag = np.sqrt(np.sum(v * v, axis=0))
        normals[:, f] = (np.moveaxis(v / mag, 0, -1)) * (1.0 if side else -1.0)
        fMJ[:, f] = fw[None, :] * mag
    xf = x.reshape(3, K, Np)
    # neighbours: faces matched by their centres, then nodes by coordinates
    fn_all = np.stack([fn.reshape(-1) for fn in fnodes])          # (6, Nfp)
    fx = xf[:, :, fn_all]                                           # (3, K, 6, Nfp)
    scale = float(g.vr[-1])
    keys = np.round(fx.mean(axis=3) / scale * 1e9).astype(np.int64)  # (3, K, 6)
    centre = {}
    for e in range(K):
        for f in range(6):
            centre.setdefault((keys[0, e, f], keys[1, e, f], keys[2, e, f]), []).append((e, f))
    nbr_node = np.full((K, 6, Nfp), -1, dtype=np.int64)
    partner = np.full((K, 6, Nfp), -1, dtype=np.int64)  # (e2*6 + f2)*Nfp + j2 of the matching face node
    btag = np.zeros((K, 6), dtype=np.int32)
    for e in range(K):
        for f in range(6):
            cands = [c for c in centre[(keys[0, e, f], keys[1, e, f], keys[2, e, f])] if c[0] != e]
            if not cands:
                layer = eidx[e, 3]
                if f == 4 and layer == 0:
                    btag[e, f] = 5
                elif f == 5 and layer == g.KV - 1:
                    btag[e, f] = 6
                else:
                    raise RuntimeError("unmatched interior face in the cubed-sphere grid")
                continue
            e2, f2 = cands[0]
            d2 = np.sum((fx[:, e, f, :, None] - fx[:, e2, f2, None, :]) ** 2, axis=0)  # (Nfp, Nfp)
            jj = np.argmin(d2, axis=1)
            if np.max(d2[np.arange(Nfp), jj]) > (1e-9 * scale) ** 2:
                raise RuntimeError("face nodes of neighbouring elements do not coincide")
            nbr_node[e, f] = e2 * Np + fn_all[f2, jj]
            partner[e, f] = (e2 * 6 + f2) * Nfp + jj
    # the two sides of an interior face share one normal (up to sign) and one
    # face mass, so the surface fluxes cancel exactly (conservation)
    pf = partner.reshape(-1)
    nflat, mflat = normals.reshape(-1, 3), fMJ.reshape(-1)
    a = np.nonzero((pf >= 0) & (np.arange(pf.size) < pf))[0]
    b = pf[a]
    if not np.array_equal(pf[b], a):
        raise RuntimeError("the face map of the cubed-sphere grid is not symmetric")
    nrm = nflat[a] - nflat[b]
    nrm = nrm / np.sqrt(np.sum(nrm * nrm, axis=1, keepdims=True))
    nflat[a], nflat[b] = nrm, -nrm
    m = (mflat[a] + mflat[b]) / 2
    mflat[a] = m
    mflat[b] = m
    return {
        "x": xf, "J": J.reshape(K, Np), "g": gm.reshape(3, 3, K, Np), "MJ": MJ.reshape(K, Np),
        "face_nodes": np.stack([fn.reshape(-1) for fn in fnodes]).astype(np.int32),
        "normals": normals, "faceMJ": fMJ, "nbr_node": nbr_node, "btag": btag,
    }

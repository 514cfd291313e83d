"""Structured unit-cube meshes in Elmer's mesh conventions.

These generate the same kind of input ElmerGrid writes for ``mesh.{nodes,elements,boundary}``:
1-based node indices, bulk elements with Elmer element type codes, and boundary
elements tagged by boundary-condition id.

Node order inside an element follows Elmer's reference elements:

* ``808`` (trilinear hexahedron), ``fem/src/elements.def:606-643``: nodes 1-4 are the
  w=-1 face counter-clockwise from (u,v)=(-1,-1), nodes 5-8 the w=+1 face.
* ``504`` (linear tetrahedron), ``fem/src/elements.def:365-404``: (0,0,0),(1,0,0),(0,1,0),(0,0,1).
* ``303`` (linear triangle), ``fem/src/elements.def:155-185``.

Global node numbering is lexicographic with x fastest:
``node(i,j,k) = 1 + i + (nx+1)*(j + (ny+1)*k)``; elements are numbered the same way
over cells.  Boundary-condition ids: 1 x=0, 2 x=1, 3 y=0, 4 y=1, 5 z=0, 6 z=1.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Mesh:
    """A bulk mesh plus its boundary elements (all index arrays 1-based, int32)."""

    coords: np.ndarray            # (nnodes, 3) float64
    elem_code: int                # 808, 504, 303
    elements: np.ndarray          # (nelem, nen) int32, 1-based node ids
    bnd_code: int                 # 404, 303, 202
    bnd_elements: np.ndarray      # (nbnd, nben) int32, 1-based node ids
    bnd_ids: np.ndarray           # (nbnd,) int32 boundary-condition id
    dims: tuple = field(default_factory=tuple)

    @property
    def nnodes(self) -> int:
        return int(self.coords.shape[0])

    @property
    def nelem(self) -> int:
        return int(self.elements.shape[0])

    def boundary_nodes(self, ids) -> np.ndarray:
        """Sorted unique 1-based node ids on the boundaries whose id is in ``ids``."""
        ids = np.asarray(list(ids), dtype=np.int32)
        sel = np.isin(self.bnd_ids, ids)
        nodes = np.unique(self.bnd_elements[sel].ravel())
        return nodes[nodes > 0].astype(np.int32)


def _node_id(nx, ny, i, j, k):
    return 1 + i + (nx + 1) * (j + (ny + 1) * k)


def hex_cube(nx: int, ny: int | None = None, nz: int | None = None) -> Mesh:
    """Unit cube split into nx*ny*nz trilinear 808 hexahedra."""
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    xs = np.arange(nx + 1, dtype=np.float64) / nx
    ys = np.arange(ny + 1, dtype=np.float64) / ny
    zs = np.arange(nz + 1, dtype=np.float64) / nz
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    coords = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)

    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    n = lambda a, b, c: _node_id(nx, ny, a, b, c)
    elements = np.stack([
        n(i, j, k), n(i + 1, j, k), n(i + 1, j + 1, k), n(i, j + 1, k),
        n(i, j, k + 1), n(i + 1, j, k + 1), n(i + 1, j + 1, k + 1), n(i, j + 1, k + 1),
    ], axis=1).astype(np.int32)

    bnd, ids = _hex_boundary_quads(nx, ny, nz)
    return Mesh(coords, 808, elements, 404, bnd, ids, (nx, ny, nz))


def _hex_boundary_quads(nx, ny, nz):
    faces, ids = [], []
    n = lambda a, b, c: _node_id(nx, ny, a, b, c)
    # x = 0 / x = 1
    for bid, ii in ((1, 0), (2, nx)):
        kk, jj = np.meshgrid(np.arange(nz), np.arange(ny), indexing="ij")
        kk, jj = kk.ravel(), jj.ravel()
        faces.append(np.stack([n(ii, jj, kk), n(ii, jj + 1, kk), n(ii, jj + 1, kk + 1), n(ii, jj, kk + 1)], 1))
        ids.append(np.full(kk.size, bid))
    for bid, jj in ((3, 0), (4, ny)):
        kk, ii = np.meshgrid(np.arange(nz), np.arange(nx), indexing="ij")
        kk, ii = kk.ravel(), ii.ravel()
        faces.append(np.stack([n(ii, jj, kk), n(ii + 1, jj, kk), n(ii + 1, jj, kk + 1), n(ii, jj, kk + 1)], 1))
        ids.append(np.full(kk.size, bid))
    for bid, kk in ((5, 0), (6, nz)):
        jj, ii = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
        jj, ii = jj.ravel(), ii.ravel()
        faces.append(np.stack([n(ii, jj, kk), n(ii + 1, jj, kk), n(ii + 1, jj + 1, kk), n(ii, jj + 1, kk)], 1))
        ids.append(np.full(jj.size, bid))
    return (np.concatenate(faces).astype(np.int32), np.concatenate(ids).astype(np.int32))


# Kuhn split of the unit cube into 6 tetrahedra sharing the (0,0,0)-(1,1,1) diagonal.
# Corner numbering c = a + 2b + 4c over (a,b,c) in {0,1}^3.
_KUHN = (
    (0, 1, 3, 7), (0, 1, 5, 7), (0, 2, 3, 7),
    (0, 2, 6, 7), (0, 4, 5, 7), (0, 4, 6, 7),
)


def tet_cube(nx: int, ny: int | None = None, nz: int | None = None) -> Mesh:
    """Unit cube with every hex cell split into 6 linear 504 tetrahedra (Kuhn split)."""
    h = hex_cube(nx, ny, nz)
    nx, ny, nz = h.dims
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    corner = [_node_id(nx, ny, i + (c & 1), j + ((c >> 1) & 1), k + ((c >> 2) & 1)) for c in range(8)]
    tets = np.stack([np.stack([corner[a] for a in t], axis=1) for t in _KUHN], axis=1)
    tets = tets.reshape(-1, 4).astype(np.int32)
    # boundary triangles: split every boundary quad along the diagonal consistent with the Kuhn split
    q, ids = h.bnd_elements, h.bnd_ids
    tri = np.concatenate([q[:, [0, 1, 2]], q[:, [0, 2, 3]]], axis=0)
    tids = np.concatenate([ids, ids])
    return Mesh(h.coords, 504, tets, 303, tri.astype(np.int32), tids.astype(np.int32), (nx, ny, nz))


def lognormal_conductivity(nelem: int, sigma: float, seed: int, mu: float = 0.0) -> np.ndarray:
    """Per-element conductivity k ~ logN(mu, sigma), drawn in element order from a seeded PCG64."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.exp(rng.normal(mu, sigma, size=nelem)).astype(np.float64)


def sine_source(coords: np.ndarray) -> np.ndarray:
    """Nodal f(x,y,z) = sin(pi x) sin(pi y) sin(pi z)."""
    x, y, z = coords[:, 0], coords[:, 1], coords[:, 2]
    return np.sin(np.pi * x) * np.sin(np.pi * y) * np.sin(np.pi * z)


def read_elmer_mesh(dirname: str) -> Mesh:
    """Read an Elmer ``mesh.{header,nodes,elements,boundary}`` directory (one bulk element type)."""
    import os

    nodes = np.loadtxt(os.path.join(dirname, "mesh.nodes"), ndmin=2)
    order = np.argsort(nodes[:, 0])
    nodes = nodes[order]
    ids = nodes[:, 0].astype(np.int64)
    if not np.array_equal(ids, np.arange(1, ids.size + 1)):
        raise ValueError("mesh.nodes ids must be 1..n")
    coords = nodes[:, 2:5].astype(np.float64)
    rows = [l.split() for l in open(os.path.join(dirname, "mesh.elements")) if l.strip()]
    codes = {int(r[2]) for r in rows}
    if len(codes) != 1:
        raise ValueError(f"mixed bulk element types {codes}")
    code = codes.pop()
    rows.sort(key=lambda r: int(r[0]))
    elements = np.array([[int(v) for v in r[3:]] for r in rows], dtype=np.int32)
    brows = [l.split() for l in open(os.path.join(dirname, "mesh.boundary")) if l.strip()]
    bcodes = {int(r[4]) for r in brows}
    bcode = bcodes.pop() if len(bcodes) == 1 else 0
    width = max(len(r) - 5 for r in brows)
    bnd = np.zeros((len(brows), width), dtype=np.int32)  # mixed boundary types: 0-padded
    for i, r in enumerate(brows):
        bnd[i, : len(r) - 5] = [int(v) for v in r[5:]]
    bids = np.array([int(r[1]) for r in brows], dtype=np.int32)
    return Mesh(coords, code, elements, bcode, bnd, bids, ())

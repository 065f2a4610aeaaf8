"""Seeded synthetic meshes written in the Gmsh v1 ``$NOD/$ELM`` format.

DG-Parallel reads meshes only through ``mImportExport::importGmshFile``
(``mImportExport.cc:77-170``): node lines ``id x y z`` and element lines
``elm-number elm-type phys-tag elem-tag n-nodes node-list``.  The third column is
the physical tag, which becomes the classification id that the boundary
conditions dispatch on (``DGCell.cc:687-705``: 20000 curved wall, 510/610
periodic, anything else goes to ``boundaryFlux``).  The solver and the oracle
read the same file, so coordinates are written with 17 significant digits and
round-trip exactly.

Meshes:

* :func:`tri_square` -- an ``nx x ny`` grid of a rectangle, each cell split into
  two counter-clockwise triangles along the (i,j)-(i+1,j+1) diagonal, interior
  vertices jittered by a seeded uniform offset of +-``jitter*h`` per axis.
* :func:`tri_graded` -- the same triangulation with node lines spaced
  geometrically (ratio ``ratio`` between neighbouring spacings, per axis), so
  that cell sizes span several factors of two (local time stepping bins).
* :func:`tet_graded` -- the same tets with node planes spaced geometrically.
* :func:`tet_cube` -- an ``n^3`` grid of a box, each cube split into the six
  Kuhn tetrahedra around its main diagonal (conforming across cubes), interior
  vertices jittered the same way.

Boundary edges/faces are emitted as line (type 1) or triangle (type 2)
elements carrying ``boundary_tag``; cells carry ``domain_tag``.
"""
from __future__ import annotations

import itertools
from dataclasses import dataclass

import numpy as np


@dataclass
class Mesh:
    """Vertices and cells of a simplex mesh with tagged boundary facets.

    ``cells`` and ``bfaces`` hold 0-based vertex indices; the file writes them
    1-based.  ``dim`` is 2 (triangles) or 3 (tetrahedra).
    """
    dim: int
    vertices: np.ndarray       # (nv, 3) float64
    cells: np.ndarray          # (E, dim+1) int64
    bfaces: np.ndarray         # (B, dim) int64
    btags: np.ndarray          # (B,) int64
    domain_tag: int = 100

    @property
    def num_cells(self) -> int:
        return int(self.cells.shape[0])


def _jitter(coords: np.ndarray, interior: np.ndarray, h: np.ndarray, jitter: float,
            seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    off = rng.uniform(-1.0, 1.0, size=coords.shape) * (jitter * h)
    out = coords.copy()
    out[interior] += off[interior]
    return out


def tri_square(nx: int, ny: int, x0: float = 0.0, x1: float = 1.0, y0: float = 0.0,
               y1: float = 1.0, jitter: float = 0.15, seed: int = 1,
               boundary_tag: int = 1, domain_tag: int = 100, side_tags=None) -> Mesh:
    """Structured ``nx x ny`` rectangle grid cut into ``2*nx*ny`` jittered triangles.

    ``side_tags`` = (bottom, right, top, left) classification ids overrides
    ``boundary_tag`` per side; DG-Parallel pairs sides tagged 510 (left/right)
    and 610 (bottom/top) as periodic (``mMesh::setPeriodicBC``, mMesh.cc:457-524).
    """
    ii, jj = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), indexing="xy")
    hx = (x1 - x0) / nx
    hy = (y1 - y0) / ny
    xs = x0 + ii.ravel() * hx
    ys = y0 + jj.ravel() * hy
    coords = np.stack([xs, ys], axis=1)
    interior = ((ii.ravel() > 0) & (ii.ravel() < nx) & (jj.ravel() > 0) & (jj.ravel() < ny))
    coords = _jitter(coords, interior, np.array([hx, hy]), jitter, seed)
    verts = np.zeros((coords.shape[0], 3))
    verts[:, :2] = coords

    def vid(i, j):
        return j * (nx + 1) + i

    ci, cj = np.meshgrid(np.arange(nx), np.arange(ny), indexing="xy")
    ci = ci.ravel()
    cj = cj.ravel()
    v00 = vid(ci, cj)
    v10 = vid(ci + 1, cj)
    v11 = vid(ci + 1, cj + 1)
    v01 = vid(ci, cj + 1)
    t1 = np.stack([v00, v10, v11], axis=1)
    t2 = np.stack([v00, v11, v01], axis=1)
    cells = np.empty((2 * nx * ny, 3), dtype=np.int64)
    cells[0::2] = t1
    cells[1::2] = t2

    st = side_tags if side_tags is not None else (boundary_tag,) * 4
    b, t = [], []
    for i in range(nx):
        b.append((vid(i, 0), vid(i + 1, 0)))
        t.append(st[0])
        b.append((vid(i + 1, ny), vid(i, ny)))
        t.append(st[2])
    for j in range(ny):
        b.append((vid(nx, j), vid(nx, j + 1)))
        t.append(st[1])
        b.append((vid(0, j + 1), vid(0, j)))
        t.append(st[3])
    bfaces = np.array(b, dtype=np.int64)
    btags = np.array(t, dtype=np.int64)
    return Mesh(2, verts, cells, bfaces, btags, domain_tag)


def tri_graded(nx: int, ny: int, ratio: float = 1.08, x0: float = 0.0, x1: float = 1.0,
               y0: float = 0.0, y1: float = 1.0, boundary_tag: int = 1, domain_tag: int = 100,
               side_tags=None) -> Mesh:
    """``tri_square`` (no jitter) with node line i at
    ``x0 + (x1 - x0) (ratio^i - 1) / (ratio^nx - 1)`` (and likewise in y): the
    cells shrink geometrically towards the (x0, y0) corner."""
    m = tri_square(nx, ny, 0.0, 1.0, 0.0, 1.0, jitter=0.0, boundary_tag=boundary_tag,
                   domain_tag=domain_tag, side_tags=side_tags)

    def grade(u, n, lo, hi):
        i = np.rint(u * n)
        return lo + (hi - lo) * (ratio ** i - 1.0) / (ratio ** n - 1.0)

    v = m.vertices.copy()
    v[:, 0] = grade(v[:, 0], nx, x0, x1)
    v[:, 1] = grade(v[:, 1], ny, y0, y1)
    return Mesh(2, v, m.cells, m.bfaces, m.btags, domain_tag)


def _kuhn_cube_tets() -> list[tuple[int, int, int, int]]:
    """Six tets of the unit cube around the (0,0,0)-(1,1,1) diagonal, corner ids i+2j+4k."""
    tets = []
    for perm in itertools.permutations(range(3)):
        p = [0, 0, 0]
        corners = [0]
        for axis in perm:
            p[axis] = 1
            corners.append(p[0] + 2 * p[1] + 4 * p[2])
        tets.append(tuple(corners))
    return tets


def tet_cube(n: int, x0: float = 0.0, x1: float = 1.0, jitter: float = 0.1, seed: int = 3,
             boundary_tag: int = 1, domain_tag: int = 100) -> Mesh:
    """``n^3`` cube grid of a box, each cube split into 6 Kuhn tets (``6*n^3`` cells)."""
    h = (x1 - x0) / n
    idx = np.arange(n + 1)
    kk, jj, ii = np.meshgrid(idx, idx, idx, indexing="ij")
    ii = ii.ravel()
    jj = jj.ravel()
    kk = kk.ravel()
    coords = np.stack([x0 + ii * h, x0 + jj * h, x0 + kk * h], axis=1)
    interior = ((ii > 0) & (ii < n) & (jj > 0) & (jj < n) & (kk > 0) & (kk < n))
    coords = _jitter(coords, interior, np.array([h, h, h]), jitter, seed)

    def vid(i, j, k):
        return (k * (n + 1) + j) * (n + 1) + i

    ci, cj, ck = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    ci = ci.ravel()
    cj = cj.ravel()
    ck = ck.ravel()
    corner = np.stack([vid(ci + (c & 1), cj + ((c >> 1) & 1), ck + ((c >> 2) & 1))
                       for c in range(8)], axis=1)
    cells = []
    for t in _kuhn_cube_tets():
        cells.append(corner[:, list(t)])
    cells = np.stack(cells, axis=1).reshape(-1, 4)
    # orient every tet with a positive Jacobian
    p = coords[cells]
    vol = np.einsum("ij,ij->i", np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]), p[:, 3] - p[:, 0])
    neg = vol < 0
    cells[neg, 1], cells[neg, 2] = cells[neg, 2].copy(), cells[neg, 1].copy()

    faces = np.concatenate([cells[:, [0, 1, 2]], cells[:, [0, 1, 3]],
                            cells[:, [0, 2, 3]], cells[:, [1, 2, 3]]])
    key = np.sort(faces, axis=1)
    _, inv, counts = np.unique(key, axis=0, return_inverse=True, return_counts=True)
    bfaces = faces[counts[inv.ravel()] == 1]
    btags = np.full(len(bfaces), boundary_tag, dtype=np.int64)
    return Mesh(3, coords, cells.astype(np.int64), bfaces.astype(np.int64), btags, domain_tag)


def tet_graded(n: int, ratio: float = 1.2, x0: float = 0.0, x1: float = 1.0, boundary_tag: int = 1,
               domain_tag: int = 100) -> Mesh:
    """``tet_cube`` (no jitter) with node plane i at
    ``x0 + (x1 - x0) (ratio^i - 1) / (ratio^n - 1)`` on every axis: the boxes,
    and their six Kuhn tets, shrink geometrically towards the (x0, x0, x0)
    corner (the monotone per-axis map keeps every tet's orientation)."""
    m = tet_cube(n, 0.0, 1.0, jitter=0.0, boundary_tag=boundary_tag, domain_tag=domain_tag)
    v = m.vertices.copy()
    i = np.rint(v * n)
    v = x0 + (x1 - x0) * (ratio ** i - 1.0) / (ratio ** n - 1.0)
    return Mesh(3, v, m.cells, m.bfaces, m.btags, domain_tag)


def write_msh_v1(mesh: Mesh, path: str) -> None:
    """Write ``mesh`` as a Gmsh v1 file readable by ``mImportExport::importGmshFile``."""
    nv = mesh.vertices.shape[0]
    cell_type = 2 if mesh.dim == 2 else 4
    face_type = 1 if mesh.dim == 2 else 2
    lines = ["$NOD", str(nv)]
    ids = np.arange(1, nv + 1)
    lines.extend("%d %.17g %.17g %.17g" % (i, x, y, z)
                 for i, (x, y, z) in zip(ids, mesh.vertices))
    lines.append("$ENDNOD")
    lines.append("$ELM")
    nb = mesh.bfaces.shape[0]
    ne = mesh.cells.shape[0]
    lines.append(str(nb + ne))
    num = 1
    for f, tag in zip(mesh.bfaces + 1, mesh.btags):
        lines.append("%d %d %d %d %d %s" % (num, face_type, tag, tag, len(f),
                                            " ".join(map(str, f))))
        num += 1
    ncv = mesh.dim + 1
    tag = mesh.domain_tag
    cells1 = mesh.cells + 1
    for c in cells1:
        lines.append("%d %d %d %d %d %s" % (num, cell_type, tag, tag, ncv, " ".join(map(str, c))))
        num += 1
    lines.append("$ENDELM")
    with open(path, "w") as fh:
        fh.write("\n".join(lines))
        fh.write("\n")

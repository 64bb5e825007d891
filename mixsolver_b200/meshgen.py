"""Seeded synthetic unstructured meshes in the reference's face-list layout.

Every generator returns a :class:`FaceMesh`: node coordinates plus a Fluent-style
face list (nodes of each face, owner ``c0``, neighbour ``c1`` with 0 meaning a
boundary face, face zone id). This is the same information the reference's
``.cas`` reader stores in ``mesh_t`` (``src/unstructured/mod_uns_mesh.f90:17-54``);
indices are 1-based exactly as there, so the arrays can be handed to the
reference's Fortran types or written out as a ``.cas`` file unchanged.

Generators:
  * :func:`cavity2d`   -- N x N x 1 hex cavity with the face/zone layout of the
    reference's ``cases/natconv/gen_cas.py`` (zone 3 interior, 4 symmetry z-planes,
    5 walls).
  * :func:`box_hex`    -- nx x ny x nz hex box with seeded node jitter.
  * :func:`box_tet`    -- every hex of an n^3 box split into 6 tetrahedra
    (Kuhn split along the main diagonal, conforming between cubes).
Helpers renumber cells (:func:`permute_cells`) and sort faces by owner
(:func:`sort_faces`).
"""
from __future__ import annotations

import dataclasses

import numpy as np


@dataclasses.dataclass
class FaceMesh:
    x: np.ndarray          # (nnodes, 3) float64 node coordinates
    fnode_ptr: np.ndarray  # (nfaces+1,) int32 offsets into fnodes
    fnodes: np.ndarray     # int32 node ids, 1-based
    c0: np.ndarray         # (nfaces,) int32 owner cell, 1-based
    c1: np.ndarray         # (nfaces,) int32 neighbour cell, 1-based, 0 = boundary
    zone: np.ndarray       # (nfaces,) int32 face zone id
    ncells: int
    zone_names: dict       # zone id -> condition name (fluent style)

    @property
    def nfaces(self) -> int:
        return int(self.c0.shape[0])

    @property
    def nnodes(self) -> int:
        return int(self.x.shape[0])

    def n_interior(self) -> int:
        return int(np.count_nonzero(self.c1 > 0))

    def copy(self) -> "FaceMesh":
        return dataclasses.replace(
            self, x=self.x.copy(), fnode_ptr=self.fnode_ptr.copy(),
            fnodes=self.fnodes.copy(), c0=self.c0.copy(), c1=self.c1.copy(),
            zone=self.zone.copy(), zone_names=dict(self.zone_names))


def _uniform_faces(nodes: np.ndarray, c0, c1, zone) -> tuple:
    nodes = np.ascontiguousarray(nodes, dtype=np.int32)
    nf, nn = nodes.shape
    ptr = (np.arange(nf + 1, dtype=np.int64) * nn).astype(np.int32)
    return (ptr, nodes.reshape(-1), np.asarray(c0, np.int32),
            np.asarray(c1, np.int32), np.asarray(zone, np.int32))


def _concat(parts):
    ptrs, fns, c0s, c1s, zs = [], [], [], [], []
    off = 0
    for ptr, fn, c0, c1, z in parts:
        ptrs.append(ptr[:-1] + off)
        off += int(ptr[-1])
        fns.append(fn); c0s.append(c0); c1s.append(c1); zs.append(z)
    ptr = np.concatenate(ptrs + [np.array([off], np.int32)]).astype(np.int32)
    return (ptr, np.concatenate(fns), np.concatenate(c0s),
            np.concatenate(c1s), np.concatenate(zs))


def cavity2d(n: int) -> FaceMesh:
    """N x N x 1 hex cavity on [0,1]^2 x [0,1], face order of gen_cas.py.

    Face blocks in order: interior y-normal faces (rows j-1|j), interior x-normal
    faces, symmetry z=0 then z=1 faces (zone 4), walls y=0, y=1, x=0, x=1 (zone 5).
    """
    m1 = n + 1
    npl = m1 * m1
    i = np.arange(m1)
    xs, ys = np.meshgrid(i / n, i / n, indexing="xy")          # node (i,j) at [j,i]
    bot = np.stack([xs.ravel(), ys.ravel(), np.zeros(npl)], 1)
    top = np.stack([xs.ravel(), ys.ravel(), np.ones(npl)], 1)
    x = np.concatenate([bot, top]).astype(np.float64)

    def bn(ii, jj):
        return 1 + ii + jj * m1

    def tn(ii, jj):
        return bn(ii, jj) + npl

    def cell(ii, jj):
        return 1 + ii + jj * n

    parts = []
    # interior faces with normal in y: between rows j-1 and j
    jj, ii = np.meshgrid(np.arange(1, n), np.arange(n), indexing="ij")
    jj, ii = jj.ravel(), ii.ravel()
    nodes = np.stack([bn(ii, jj), tn(ii, jj), tn(ii + 1, jj), bn(ii + 1, jj)], 1)
    parts.append(_uniform_faces(nodes, cell(ii, jj - 1), cell(ii, jj), np.full(ii.size, 3)))
    # interior faces with normal in x: between columns i-1 and i
    ii, jj = np.meshgrid(np.arange(1, n), np.arange(n), indexing="ij")
    ii, jj = ii.ravel(), jj.ravel()
    nodes = np.stack([bn(ii, jj), tn(ii, jj), tn(ii, jj + 1), bn(ii, jj + 1)], 1)
    parts.append(_uniform_faces(nodes, cell(ii - 1, jj), cell(ii, jj), np.full(ii.size, 3)))
    # symmetry: z=0 plane then z=1 plane
    jj, ii = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    jj, ii = jj.ravel(), ii.ravel()
    z0 = np.zeros(ii.size, np.int32)
    nodes = np.stack([bn(ii, jj), bn(ii + 1, jj), bn(ii + 1, jj + 1), bn(ii, jj + 1)], 1)
    parts.append(_uniform_faces(nodes, cell(ii, jj), z0, np.full(ii.size, 4)))
    nodes = np.stack([tn(ii, jj), tn(ii + 1, jj), tn(ii + 1, jj + 1), tn(ii, jj + 1)], 1)
    parts.append(_uniform_faces(nodes, cell(ii, jj), z0, np.full(ii.size, 4)))
    # walls: y=0, y=N, x=0, x=N
    a = np.arange(n)
    zn = np.zeros(n, np.int32)
    w = np.full(n, 5)
    parts.append(_uniform_faces(np.stack([bn(a, 0), tn(a, 0), tn(a + 1, 0), bn(a + 1, 0)], 1), cell(a, 0), zn, w))
    parts.append(_uniform_faces(np.stack([bn(a, n), tn(a, n), tn(a + 1, n), bn(a + 1, n)], 1), cell(a, n - 1), zn, w))
    parts.append(_uniform_faces(np.stack([bn(0, a), tn(0, a), tn(0, a + 1), bn(0, a + 1)], 1), cell(0, a), zn, w))
    parts.append(_uniform_faces(np.stack([bn(n, a), tn(n, a), tn(n, a + 1), bn(n, a + 1)], 1), cell(n - 1, a), zn, w))
    ptr, fn, c0, c1, z = _concat(parts)
    return FaceMesh(x, ptr, fn, c0, c1, z, n * n,
                    {3: "interior", 4: "symmetry", 5: "wall"})


def _box_nodes(nx, ny, nz, lx, ly, lz, jitter, seed):
    xs = np.linspace(0.0, lx, nx + 1)
    ys = np.linspace(0.0, ly, ny + 1)
    zs = np.linspace(0.0, lz, nz + 1)
    # node (i,j,k) -> id 1 + i + (nx+1)*(j + (ny+1)*k)
    zz, yy, xx = np.meshgrid(zs, ys, xs, indexing="ij")
    x = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], 1).astype(np.float64)
    if jitter > 0.0:
        rng = np.random.default_rng(seed)
        k, j, i = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
        interior = ((i > 0) & (i < nx) & (j > 0) & (j < ny) & (k > 0) & (k < nz)).ravel()
        h = np.array([lx / nx, ly / ny, lz / nz])
        d = rng.uniform(-jitter, jitter, size=x.shape) * h
        x[interior] += d[interior]
    return x


def box_hex(nx: int, ny: int, nz: int, lx=1.0, ly=1.0, lz=1.0, jitter=0.0,
            seed=0, zones=None) -> FaceMesh:
    """Hex box [0,lx]x[0,ly]x[0,lz]; interior nodes jittered by U(+-jitter) x local
    spacing (seeded). Face order: interior x-, y-, z-normal faces (zone 3), then
    boundary faces x=0, x=lx, y=0, y=ly, z=0, z=lz with zone ids from ``zones``
    (default 4, 5, 6, 6, 6, 6)."""
    if zones is None:
        zones = (4, 5, 6, 6, 6, 6)
    x = _box_nodes(nx, ny, nz, lx, ly, lz, jitter, seed)

    def nid(i, j, k):
        return 1 + i + (nx + 1) * (j + (ny + 1) * k)

    def cid(i, j, k):
        return 1 + i + nx * (j + ny * k)

    parts = []
    # x-normal interior faces at i = 1..nx-1
    k, j, i = [a.ravel() for a in np.meshgrid(np.arange(nz), np.arange(ny), np.arange(1, nx), indexing="ij")]
    nodes = np.stack([nid(i, j, k), nid(i, j + 1, k), nid(i, j + 1, k + 1), nid(i, j, k + 1)], 1)
    parts.append(_uniform_faces(nodes, cid(i - 1, j, k), cid(i, j, k), np.full(i.size, 3)))
    k, j, i = [a.ravel() for a in np.meshgrid(np.arange(nz), np.arange(1, ny), np.arange(nx), indexing="ij")]
    nodes = np.stack([nid(i, j, k), nid(i, j, k + 1), nid(i + 1, j, k + 1), nid(i + 1, j, k)], 1)
    parts.append(_uniform_faces(nodes, cid(i, j - 1, k), cid(i, j, k), np.full(i.size, 3)))
    k, j, i = [a.ravel() for a in np.meshgrid(np.arange(1, nz), np.arange(ny), np.arange(nx), indexing="ij")]
    nodes = np.stack([nid(i, j, k), nid(i + 1, j, k), nid(i + 1, j + 1, k), nid(i, j + 1, k)], 1)
    parts.append(_uniform_faces(nodes, cid(i, j, k - 1), cid(i, j, k), np.full(i.size, 3)))
    # boundary faces
    for side, zid in zip(range(6), zones):
        axis, hi = divmod(side, 2)
        if axis == 0:
            k, j = [a.ravel() for a in np.meshgrid(np.arange(nz), np.arange(ny), indexing="ij")]
            i = np.full(j.size, nx if hi else 0)
            nodes = np.stack([nid(i, j, k), nid(i, j + 1, k), nid(i, j + 1, k + 1), nid(i, j, k + 1)], 1)
            cells = cid(np.minimum(i, nx - 1), j, k)
        elif axis == 1:
            k, i = [a.ravel() for a in np.meshgrid(np.arange(nz), np.arange(nx), indexing="ij")]
            j = np.full(i.size, ny if hi else 0)
            nodes = np.stack([nid(i, j, k), nid(i, j, k + 1), nid(i + 1, j, k + 1), nid(i + 1, j, k)], 1)
            cells = cid(i, np.minimum(j, ny - 1), k)
        else:
            j, i = [a.ravel() for a in np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")]
            k = np.full(i.size, nz if hi else 0)
            nodes = np.stack([nid(i, j, k), nid(i + 1, j, k), nid(i + 1, j + 1, k), nid(i, j + 1, k)], 1)
            cells = cid(i, j, np.minimum(k, nz - 1))
        parts.append(_uniform_faces(nodes, cells, np.zeros(cells.size, np.int32), np.full(cells.size, zid)))
    ptr, fn, c0, c1, z = _concat(parts)
    names = {3: "interior"}
    for zid in zones:
        names.setdefault(int(zid), f"zone{zid}")
    return FaceMesh(x, ptr, fn, c0, c1, z, nx * ny * nz, names)


# Kuhn split: the 6 tetrahedra of a unit cube along the 0 -> 7 diagonal; corner c
# has bits (x, y, z) = (c & 1, c >> 1 & 1, c >> 2 & 1).
_KUHN = [(0, 1, 3, 7), (0, 1, 5, 7), (0, 2, 3, 7), (0, 2, 6, 7), (0, 4, 5, 7), (0, 4, 6, 7)]


def box_tet(n: int, length=1.0, jitter=0.0, seed=0, wall_zone=4) -> FaceMesh:
    """n^3 cubes on [0,length]^3, each split into 6 tets (6 n^3 cells).

    Faces are the unique node triplets: interior faces (zone 3) in order of first
    appearance, then boundary faces (zone ``wall_zone``) in order of appearance.
    """
    x = _box_nodes(n, n, n, length, length, length, jitter, seed)
    k, j, i = [a.ravel() for a in np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")]

    def nid(ii, jj, kk):
        return 1 + ii + (n + 1) * (jj + (n + 1) * kk)

    corners = np.stack([nid(i + (c & 1), j + (c >> 1 & 1), k + (c >> 2 & 1)) for c in range(8)], 1)
    tets = np.concatenate([corners[:, list(t)][:, None, :] for t in _KUHN], axis=1).reshape(-1, 4)
    ncell = tets.shape[0]
    # 4 faces per tet (drop one vertex each)
    fl = np.stack([tets[:, [1, 2, 3]], tets[:, [0, 2, 3]], tets[:, [0, 1, 3]], tets[:, [0, 1, 2]]], 1).reshape(-1, 3)
    owner = np.repeat(np.arange(1, ncell + 1, dtype=np.int64), 4)
    srt = np.sort(fl, axis=1).astype(np.int64)
    key = srt[:, 0] | (srt[:, 1] << 21) | (srt[:, 2] << 42)
    uniq, first, inv, cnt = np.unique(key, return_index=True, return_inverse=True, return_counts=True)
    order = np.argsort(first, kind="stable")          # faces in order of first appearance
    rank = np.empty_like(order)
    rank[order] = np.arange(order.size)
    fid = rank[inv]                                   # face id (0-based) per tet face
    nface = uniq.size
    c0 = np.zeros(nface, np.int64)
    c1 = np.zeros(nface, np.int64)
    # first occurrence -> owner, second -> neighbour
    occ_first = np.zeros(fl.shape[0], bool)
    occ_first[first] = True
    c0[fid[occ_first]] = owner[occ_first]
    c1[fid[~occ_first]] = owner[~occ_first]
    fnodes = fl[first[order]]
    interior = c1 > 0
    perm = np.concatenate([np.nonzero(interior)[0], np.nonzero(~interior)[0]])
    zone = np.where(interior, 3, wall_zone)[perm]
    ptr, fn, c0a, c1a, za = _uniform_faces(fnodes[perm], c0[perm], c1[perm], zone)
    return FaceMesh(x, ptr, fn, c0a, c1a, za, ncell, {3: "interior", int(wall_zone): "wall"})


def permute_cells(m: FaceMesh, new_of_old: np.ndarray) -> FaceMesh:
    """Renumber cells: cell ``c`` (1-based) becomes ``new_of_old[c-1]`` (1-based)."""
    new_of_old = np.asarray(new_of_old, np.int64)
    lut = np.concatenate([[0], new_of_old]).astype(np.int32)
    out = m.copy()
    out.c0 = lut[m.c0]
    out.c1 = lut[m.c1]
    return out


def shuffle_cells(m: FaceMesh, seed: int) -> FaceMesh:
    """Seeded random cell renumbering (a permutation of 1..ncells)."""
    rng = np.random.default_rng(seed)
    return permute_cells(m, rng.permutation(m.ncells) + 1)


def sort_faces(m: FaceMesh) -> FaceMesh:
    """Owner/neighbour-sorted face order: interior faces first with c0 < c1 and
    sorted by (c0, c1), then boundary faces sorted by (zone order of appearance,
    c0). Swapping c0/c1 of a face only flips its area vector, which the
    reference's geometry orients from c0 anyway."""
    out = m.copy()
    c0 = m.c0.astype(np.int64)
    c1 = m.c1.astype(np.int64)
    interior = c1 > 0
    swap = interior & (c1 < c0)
    a = np.where(swap, c1, c0)
    b = np.where(swap, c0, c1)
    zorder = {z: r for r, z in enumerate(dict.fromkeys(m.zone[~interior].tolist()))}
    zrank = np.array([zorder.get(int(z), 0) for z in m.zone]) if (~interior).any() else np.zeros(m.nfaces, np.int64)
    key_b = np.where(interior, 0, 1)
    order = np.lexsort((b, a, np.where(interior, 0, zrank), key_b))
    ptr = m.fnode_ptr.astype(np.int64)
    counts = (ptr[1:] - ptr[:-1])[order]
    starts = ptr[:-1][order]
    new_ptr = np.zeros(m.nfaces + 1, np.int64)
    np.cumsum(counts, out=new_ptr[1:])
    idx = np.repeat(starts - new_ptr[:-1], counts) + np.arange(new_ptr[-1])
    out.fnodes = m.fnodes[idx].astype(np.int32)
    out.fnode_ptr = new_ptr.astype(np.int32)
    out.c0 = a[order].astype(np.int32)
    out.c1 = b[order].astype(np.int32)
    out.zone = m.zone[order].astype(np.int32)
    return out


def taylor_green(xc: np.ndarray, amplitude=1.0, noise=0.01, seed=0) -> np.ndarray:
    """Divergence-free Taylor-Green field on the unit box, sampled at cell centres
    ``xc`` (ncells, 3): u = A sin(2 pi x) cos(2 pi y) cos(2 pi z),
    v = -A cos(2 pi x) sin(2 pi y) cos(2 pi z), w = 0, plus seeded U(+-noise*A)."""
    k = 2.0 * np.pi
    x, y, z = xc[:, 0], xc[:, 1], xc[:, 2]
    u = np.stack([amplitude * np.sin(k * x) * np.cos(k * y) * np.cos(k * z),
                  -amplitude * np.cos(k * x) * np.sin(k * y) * np.cos(k * z),
                  np.zeros_like(x)], 1)
    rng = np.random.default_rng(seed)
    u += rng.uniform(-noise * amplitude, noise * amplitude, size=u.shape)
    return np.ascontiguousarray(u)

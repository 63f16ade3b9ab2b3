"""Synthetic triangular meshes and the reference's five-file mesh format.

Triangle convention (the reference's, ``src/triangleinfo.cpp:174-189`` and
``src/unstructuredgrid.cpp:193-229`` of multi_gpuRkdg):

* vertices are counter-clockwise;
* edge k is the edge opposite vertex k, i.e. edge 0 = v1->v2, edge 1 = v2->v0,
  edge 2 = v0->v1;
* ``neighbours[t, k]`` is the triangle across edge k, or -1 on a boundary;
* ``bc[t, k]`` tags boundary edges with the reference's cell tags
  (``inc/defines.h:48-54``): 1 far field (given state), 2 outflow (copy),
  3 reflection (slip wall); 0 on interior edges.

Periodic meshes keep every triangle's own, unwrapped vertex coordinates
(vertices on the periodic seam are duplicated) while ``neighbours`` wraps
around the torus, so a solver that pairs edges by topology, as the reference
flux kernel does (``src/kernelfunctions.cu:545-549``), runs periodically with
no ghost cells.

All generators are seeded and deterministic.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np

BC_INTERIOR = 0
BC_FARFIELD = 1
BC_OUTFLOW = 2
BC_REFLECTION = 3


@dataclass
class Mesh:
    vertices: np.ndarray  # (V, 2) float64
    tris: np.ndarray  # (T, 3) int32, counter-clockwise
    neighbours: np.ndarray  # (T, 3) int32
    bc: np.ndarray  # (T, 3) int8
    periodic: bool = False
    name: str = "mesh"
    extent: tuple = (0.0, 0.0, 1.0, 1.0)  # (x0, y0, x1, y1) of the domain
    meta: dict = field(default_factory=dict)

    @property
    def ntri(self) -> int:
        return int(self.tris.shape[0])

    def coords(self) -> np.ndarray:
        """(T, 3, 2) vertex coordinates of every triangle."""
        return self.vertices[self.tris]

    def areas(self) -> np.ndarray:
        c = self.coords()
        a = c[:, 1] - c[:, 0]
        b = c[:, 2] - c[:, 0]
        return 0.5 * (a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0])

    def check(self) -> None:
        """Validates orientation and the symmetry of the neighbour relation."""
        if np.any(self.areas() <= 0):
            raise ValueError(f"{self.name}: non-positive triangle area")
        T = self.ntri
        nb = self.neighbours
        for k in range(3):
            m = nb[:, k] >= 0
            t = np.nonzero(m)[0]
            n = nb[t, k]
            back = (nb[n] == t[:, None]).sum(axis=1)
            if np.any(back == 0):
                raise ValueError(f"{self.name}: neighbour relation not symmetric")
        bnd = nb < 0
        if np.any((self.bc[bnd] == 0)):
            raise ValueError(f"{self.name}: untagged boundary edge")
        if np.any(self.bc[~bnd] != 0):
            raise ValueError(f"{self.name}: tagged interior edge")
        if T == 0:
            raise ValueError("empty mesh")


def _orient_ccw(verts: np.ndarray, tris: np.ndarray) -> np.ndarray:
    c = verts[tris]
    a = c[:, 1] - c[:, 0]
    b = c[:, 2] - c[:, 0]
    det = a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]
    tris = tris.copy()
    flip = det < 0
    tris[flip, 1], tris[flip, 2] = tris[flip, 2].copy(), tris[flip, 1].copy()
    return tris


def connect(canon_tris: np.ndarray) -> np.ndarray:
    """Neighbour table from canonical vertex ids by edge matching (O(T log T)).

    Edge k of triangle t joins canonical vertices (k+1)%3 and (k+2)%3.
    Returns (T, 3) int32 with -1 where an edge has no partner.  Raises if an
    edge is shared by more than two triangles.
    """
    T = canon_tris.shape[0]
    a = canon_tris[:, [1, 2, 0]].reshape(-1).astype(np.int64)
    b = canon_tris[:, [2, 0, 1]].reshape(-1).astype(np.int64)
    lo = np.minimum(a, b)
    hi = np.maximum(a, b)
    key = lo * (int(canon_tris.max()) + 1) + hi
    order = np.argsort(key, kind="stable")
    ks = key[order]
    nb = np.full(3 * T, -1, dtype=np.int64)
    same = ks[1:] == ks[:-1]
    if np.any(same[1:] & same[:-1]):
        raise ValueError("non-manifold mesh: edge shared by more than two triangles")
    i = np.nonzero(same)[0]
    e0 = order[i]
    e1 = order[i + 1]
    nb[e0] = e1 // 3
    nb[e1] = e0 // 3
    return nb.reshape(T, 3).astype(np.int32)


def periodic_structured(nx: int, ny: int, L: float = 10.0, jitter: float = 0.0, seed: int = 0,
                        name: str | None = None) -> Mesh:
    """nx x ny squares on [0, L]^2, each split along its rising diagonal, periodic.

    ``jitter`` moves every lattice vertex (and all its periodic images) by
    U(-jitter*h, jitter*h) per coordinate.
    """
    hx, hy = L / nx, L / ny
    ii, jj = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), indexing="ij")
    ii = ii.reshape(-1)
    jj = jj.reshape(-1)
    canon = (ii % nx) + nx * (jj % ny)
    rng = np.random.default_rng(seed)
    d = rng.uniform(-jitter, jitter, size=(nx * ny, 2)) if jitter > 0 else np.zeros((nx * ny, 2))
    verts = np.stack([(ii + d[canon, 0]) * hx, (jj + d[canon, 1]) * hy], axis=1)

    def vid(i, j):
        return i * (ny + 1) + j

    I, J = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    I = I.reshape(-1)
    J = J.reshape(-1)
    t1 = np.stack([vid(I, J), vid(I + 1, J), vid(I + 1, J + 1)], axis=1)
    t2 = np.stack([vid(I, J), vid(I + 1, J + 1), vid(I, J + 1)], axis=1)
    tris = np.empty((2 * nx * ny, 3), dtype=np.int64)
    tris[0::2] = t1
    tris[1::2] = t2
    nb = connect(canon[tris])
    m = Mesh(verts, tris.astype(np.int32), nb, np.zeros_like(nb, dtype=np.int8), periodic=True,
             name=name or f"periodic_{nx}x{ny}", extent=(0.0, 0.0, L, L))
    m.check()
    return m


def periodic_delaunay(n: int, L: float = 10.0, jitter: float = 0.3, seed: int = 2,
                      name: str | None = None) -> Mesh:
    """Delaunay triangulation of an n x n lattice on the [0, L)^2 torus with
    every vertex jittered by U(-jitter*h, jitter*h) per coordinate.

    The lattice is padded by three periodic layers, triangulated with
    scipy's Qhull Delaunay, and each periodic triangle is kept once: the copy
    whose centroid lies in [0, L)^2.  For the torus T = 2 n^2 exactly.
    """
    from scipy.spatial import Delaunay

    h = L / n
    rng = np.random.default_rng(seed)
    d = rng.uniform(-jitter * h, jitter * h, size=(n * n, 2))
    ii, jj = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    base = np.stack([ii.reshape(-1) * h, jj.reshape(-1) * h], axis=1) + d
    pad = 3
    sx, sy = np.meshgrid(np.arange(-1, 2), np.arange(-1, 2), indexing="ij")
    pts = []
    cid = []
    for ox, oy in zip(sx.reshape(-1), sy.reshape(-1)):
        p = base + np.array([ox * L, oy * L])
        keep = ((p[:, 0] > -pad * h) & (p[:, 0] < L + pad * h) & (p[:, 1] > -pad * h)
                & (p[:, 1] < L + pad * h))
        pts.append(p[keep])
        cid.append(np.nonzero(keep)[0])
    pts = np.concatenate(pts)
    cid = np.concatenate(cid)
    tri = Delaunay(pts).simplices
    cen = pts[tri].mean(axis=1)
    keep = (cen[:, 0] >= 0) & (cen[:, 0] < L) & (cen[:, 1] >= 0) & (cen[:, 1] < L)
    tri = tri[keep]
    used, inv = np.unique(tri.reshape(-1), return_inverse=True)
    verts = pts[used]
    tris = inv.reshape(-1, 3)
    tris = _orient_ccw(verts, tris)
    canon = cid[used]
    nb = connect(canon[tris])
    if np.any(nb < 0) or tris.shape[0] != 2 * n * n:
        raise ValueError("periodic Delaunay construction failed (padding too thin?)")
    m = Mesh(verts, tris.astype(np.int32), nb, np.zeros_like(nb, dtype=np.int8), periodic=True,
             name=name or f"periodic_delaunay_{n}", extent=(0.0, 0.0, L, L),
             meta={"seed": seed, "jitter": jitter, "lattice": n})
    m.check()
    return m


def _tag_boundary(verts: np.ndarray, tris: np.ndarray, nb: np.ndarray, tagger) -> np.ndarray:
    bc = np.zeros(nb.shape, dtype=np.int8)
    c = verts[tris]
    for k in range(3):
        t = np.nonzero(nb[:, k] < 0)[0]
        if t.size == 0:
            continue
        p = c[t, (k + 1) % 3]
        q = c[t, (k + 2) % 3]
        bc[t, k] = tagger(0.5 * (p + q), p, q)
    return bc


def box_with_obstacle(n: int = 16, half: float = 20.0, hole: int = 1, jitter: float = 0.2,
                      seed: int = 7, name: str | None = None) -> Mesh:
    """[-half, half]^2 split into n x n squares (n even) with the central
    (2*hole) x (2*hole) block of squares removed.

    Outer edges are far field, the hole's edges are slip walls -- the same
    tags the reference assigns by ghost-cell barycentre against |x|,|y| > 15
    (src/unstructuredgrid.cpp:729-760) when half > 15 and the hole lies well
    inside that box.  Every square at a corner of the box is split through
    the corner vertex so that no triangle has two boundary edges (the
    reference creates at most one ghost cell per triangle,
    src/unstructuredgrid.cpp:527-641).  Interior vertices are jittered.
    """
    assert n % 2 == 0
    h = 2 * half / n
    rng = np.random.default_rng(seed)
    ii, jj = np.meshgrid(np.arange(n + 1), np.arange(n + 1), indexing="ij")
    x = -half + ii * h
    y = -half + jj * h
    interior = (ii > 0) & (ii < n) & (jj > 0) & (jj < n)
    c = n // 2
    on_hole = (np.abs(ii - c) <= hole) & (np.abs(jj - c) <= hole)
    movable = interior & ~on_hole
    dx = rng.uniform(-jitter * h, jitter * h, size=x.shape) * movable
    dy = rng.uniform(-jitter * h, jitter * h, size=y.shape) * movable
    verts = np.stack([(x + dx).reshape(-1), (y + dy).reshape(-1)], axis=1)

    def vid(i, j):
        return i * (n + 1) + j

    tris = []
    for i in range(n):
        for j in range(n):
            if c - hole <= i < c + hole and c - hole <= j < c + hole:
                continue
            a, b, cc, d = vid(i, j), vid(i + 1, j), vid(i + 1, j + 1), vid(i, j + 1)
            falling = (i == n - 1 and j == 0) or (i == 0 and j == n - 1)
            if falling:  # diagonal through (i+1, j) / (i, j+1)
                tris.append((a, b, d))
                tris.append((b, cc, d))
            else:
                tris.append((a, b, cc))
                tris.append((a, cc, d))
    tris = np.array(tris, dtype=np.int64)
    nb = connect(tris)

    def tagger(mid, p, q):
        outer = (np.abs(mid[:, 0]) > half - 1e-9) | (np.abs(mid[:, 1]) > half - 1e-9)
        return np.where(outer, BC_FARFIELD, BC_REFLECTION).astype(np.int8)

    bc = _tag_boundary(verts, tris, nb, tagger)
    m = Mesh(verts, tris.astype(np.int32), nb, bc, periodic=False,
             name=name or f"box_obstacle_{n}", extent=(-half, -half, half, half))
    m.check()
    if np.any((nb < 0).sum(axis=1) > 1):
        raise ValueError("a triangle has two boundary edges")
    return m


def channel(nx: int = 24, ny: int = 8, lx: float = 3.0, ly: float = 1.0, jitter: float = 0.2,
            seed: int = 11, name: str | None = None) -> Mesh:
    """Structured jittered channel [0,lx]x[0,ly]: inflow (far-field state) at
    x=0, outflow at x=lx, slip walls at y=0 and y=ly."""
    hx, hy = lx / nx, ly / ny
    rng = np.random.default_rng(seed)
    ii, jj = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), indexing="ij")
    interior = (ii > 0) & (ii < nx) & (jj > 0) & (jj < ny)
    dx = rng.uniform(-jitter * hx, jitter * hx, size=ii.shape) * interior
    dy = rng.uniform(-jitter * hy, jitter * hy, size=jj.shape) * interior
    verts = np.stack([(ii * hx + dx).reshape(-1), (jj * hy + dy).reshape(-1)], axis=1)

    def vid(i, j):
        return i * (ny + 1) + j

    tris = []
    for i in range(nx):
        for j in range(ny):
            a, b, cc, d = vid(i, j), vid(i + 1, j), vid(i + 1, j + 1), vid(i, j + 1)
            falling = (i == nx - 1 and j == 0) or (i == 0 and j == ny - 1)
            if falling:
                tris.append((a, b, d))
                tris.append((b, cc, d))
            else:
                tris.append((a, b, cc))
                tris.append((a, cc, d))
    tris = np.array(tris, dtype=np.int64)
    nb = connect(tris)

    def tagger(mid, p, q):
        tag = np.full(mid.shape[0], BC_REFLECTION, dtype=np.int8)
        tag[mid[:, 0] < 1e-9] = BC_FARFIELD
        tag[mid[:, 0] > lx - 1e-9] = BC_OUTFLOW
        return tag

    bc = _tag_boundary(verts, tris, nb, tagger)
    m = Mesh(verts, tris.astype(np.int32), nb, bc, name=name or f"channel_{nx}x{ny}",
             extent=(0.0, 0.0, lx, ly))
    m.check()
    return m


def forward_step(h: float = 1.0 / 400, jitter: float = 0.3, seed: int = 3,
                 name: str | None = None) -> Mesh:
    """Mach-3 wind-tunnel step: [0,3]x[0,1] minus [0.6,3]x[0,0.2].

    Vertices: a lattice of spacing h (boundary vertices on the boundary,
    interior ones jittered by U(-jitter*h, jitter*h)), triangulated by
    scipy's Delaunay; triangles with centroid inside the step are dropped.
    Tags: x=0 inflow (far-field state), x=3 outflow, all walls (y=0, y=1,
    step faces) slip walls.
    """
    from scipy.spatial import Delaunay

    nx = int(round(3.0 / h))
    ny = int(round(1.0 / h))
    sx = int(round(0.6 / h))
    sy = int(round(0.2 / h))
    ii, jj = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), indexing="ij")
    ii = ii.reshape(-1)
    jj = jj.reshape(-1)
    inside_step = (ii > sx) & (jj < sy)
    keep = ~inside_step
    ii = ii[keep]
    jj = jj[keep]
    on_bnd = (ii == 0) | (ii == nx) | (jj == 0) | (jj == ny) | ((ii == sx) & (jj <= sy)) | (
        (jj == sy) & (ii >= sx))
    rng = np.random.default_rng(seed)
    d = rng.uniform(-jitter * h, jitter * h, size=(ii.size, 2))
    d[on_bnd] = 0.0
    pts = np.stack([ii * h, jj * h], axis=1) + d
    tri = Delaunay(pts).simplices
    cen = pts[tri].mean(axis=1)
    eps = 1e-12
    good = ~((cen[:, 0] > 0.6 + eps) & (cen[:, 1] < 0.2 - eps))
    tri = tri[good]
    # drop degenerate slivers Qhull may leave on collinear boundary points
    c = pts[tri]
    det = ((c[:, 1, 0] - c[:, 0, 0]) * (c[:, 2, 1] - c[:, 0, 1])
           - (c[:, 1, 1] - c[:, 0, 1]) * (c[:, 2, 0] - c[:, 0, 0]))
    tri = tri[np.abs(det) > 1e-6 * h * h]
    used, inv = np.unique(tri.reshape(-1), return_inverse=True)
    verts = pts[used]
    tris = _orient_ccw(verts, inv.reshape(-1, 3))
    nb = connect(tris)

    def tagger(mid, p, q):
        tag = np.full(mid.shape[0], BC_REFLECTION, dtype=np.int8)
        tag[mid[:, 0] < 1e-9] = BC_FARFIELD
        tag[mid[:, 0] > 3.0 - 1e-9] = BC_OUTFLOW
        return tag

    bc = _tag_boundary(verts, tris, nb, tagger)
    # every boundary edge must lie on the domain boundary
    cc = verts[tris]
    for k in range(3):
        t = np.nonzero(nb[:, k] < 0)[0]
        mid = 0.5 * (cc[t, (k + 1) % 3] + cc[t, (k + 2) % 3])
        on = ((np.abs(mid[:, 0]) < 1e-9) | (np.abs(mid[:, 0] - 3) < 1e-9)
              | (np.abs(mid[:, 1]) < 1e-9) | (np.abs(mid[:, 1] - 1) < 1e-9)
              | ((np.abs(mid[:, 0] - 0.6) < 1e-9) & (mid[:, 1] <= 0.2 + 1e-9))
              | ((np.abs(mid[:, 1] - 0.2) < 1e-9) & (mid[:, 0] >= 0.6 - 1e-9)))
        if not np.all(on):
            raise ValueError("forward_step: boundary edge off the domain boundary")
    m = Mesh(verts, tris.astype(np.int32), nb, bc, name=name or f"forward_step_{nx}",
             extent=(0.0, 0.0, 3.0, 1.0), meta={"seed": seed, "h": h})
    m.check()
    return m


def locality_order(mesh: Mesh, bits: int = 16) -> np.ndarray:
    """Morton (Z-order) permutation of the triangles by centroid.

    This is the single-device stand-in for the reference's partition file:
    the partition's only role left on one GPU is to keep neighbours close in
    memory so that neighbour reads hit L2.
    """
    c = mesh.coords().mean(axis=1)
    lo = c.min(axis=0)
    span = np.maximum(c.max(axis=0) - lo, 1e-300)
    q = np.minimum(((c - lo) / span * (2 ** bits - 1)).astype(np.uint64), 2 ** bits - 1)

    def spread(v):
        v = v & np.uint64(0x0000FFFF)
        v = (v | (v << np.uint64(8))) & np.uint64(0x00FF00FF)
        v = (v | (v << np.uint64(4))) & np.uint64(0x0F0F0F0F)
        v = (v | (v << np.uint64(2))) & np.uint64(0x33333333)
        v = (v | (v << np.uint64(1))) & np.uint64(0x55555555)
        return v

    code = spread(q[:, 0]) | (spread(q[:, 1]) << np.uint64(1))
    return np.argsort(code, kind="stable")


def permute(mesh: Mesh, order: np.ndarray) -> Mesh:
    """Renumbers triangles so that new triangle i is old triangle order[i]."""
    inv = np.empty_like(order)
    inv[order] = np.arange(order.size)
    nb = mesh.neighbours[order]
    nb = np.where(nb >= 0, inv[np.maximum(nb, 0)], -1).astype(np.int32)
    return Mesh(mesh.vertices, mesh.tris[order], nb, mesh.bc[order], mesh.periodic,
                mesh.name, mesh.extent, dict(mesh.meta))


def shared_edges(mesh: Mesh) -> np.ndarray:
    """(T, 3) local edge index, in the neighbour, of the edge shared with it
    (the reference's sharedEdge, src/unstructuredgrid.cpp:934-976); -1 on
    boundary edges."""
    nb = mesh.neighbours
    T = mesh.ntri
    se = np.full((T, 3), -1, dtype=np.int32)
    t = np.arange(T)
    for k in range(3):
        n = nb[:, k]
        m = n >= 0
        back = nb[np.maximum(n, 0)] == t[:, None]
        idx = np.argmax(back, axis=1)
        se[m, k] = idx[m]
    return se


def write_reference_format(mesh: Mesh, workdir: str) -> str:
    """Writes the mesh in the reference's input layout (src/unstructuredgrid.cpp:14-60,
    193-305) below ``workdir`` and returns the mesh-configuration path
    relative to ``workdir``.

    Files: input/mesh.conf, input/Vertice.dat, input/ElemVertice.dat,
    input/ElemNeigh.dat (written WITHOUT a header line, since the reference's
    reader does not skip one, src/unstructuredgrid.cpp:219-220),
    input/ElemEdge.dat, input/EdgeVertice.dat and input/ElemDepart.dat (one
    partition, all zeros).  Edge ids are shared by the two triangles of an
    edge, periodic seams included, which is how the reference finds
    sharedEdge.
    """
    os.makedirs(os.path.join(workdir, "input"), exist_ok=True)
    T = mesh.ntri
    nb = mesh.neighbours
    se = shared_edges(mesh)
    eid = np.full((T, 3), -1, dtype=np.int64)
    nxt = 0
    for t in range(T):
        for k in range(3):
            if eid[t, k] >= 0:
                continue
            eid[t, k] = nxt
            n = nb[t, k]
            if n >= 0:
                eid[n, se[t, k]] = nxt
            nxt += 1
    ev = np.zeros((nxt, 2), dtype=np.int64)
    for t in range(T):
        for k in range(3):
            ev[eid[t, k]] = (mesh.tris[t, (k + 1) % 3], mesh.tris[t, (k + 2) % 3])
    inp = os.path.join(workdir, "input")
    with open(os.path.join(inp, "Vertice.dat"), "w") as f:
        f.write("#vertice data\n")
        for x, y in mesh.vertices:
            f.write(f"{x:.17g} {y:.17g}\n")
    with open(os.path.join(inp, "ElemVertice.dat"), "w") as f:
        f.write("#ElemVertex data\n")
        for a, b, c in mesh.tris:
            f.write(f"{a} {b} {c}\n")
    with open(os.path.join(inp, "ElemNeigh.dat"), "w") as f:
        for a, b, c in nb:
            f.write(f"{a} {b} {c}\n")
    with open(os.path.join(inp, "ElemEdge.dat"), "w") as f:
        f.write("#Elemside data\n")
        for a, b, c in eid:
            f.write(f"{a} {b} {c}\n")
    with open(os.path.join(inp, "EdgeVertice.dat"), "w") as f:
        f.write("#Sidelist data\n")
        for a, b in ev:
            f.write(f"{a} {b}\n")
    with open(os.path.join(inp, "ElemDepart.dat"), "w") as f:
        f.write("0\n" * T)
    with open(os.path.join(inp, "mesh.conf"), "w") as f:
        f.write(f"trianglenum {T}\nverticenum {mesh.vertices.shape[0]}\nedgenum {nxt}\n")
        f.write("trivertice_filename input/ElemVertice.dat\n")
        f.write("trineigh_filename input/ElemNeigh.dat\n")
        f.write("triedge_filename input/ElemEdge.dat\n")
        f.write("vertice_filename input/Vertice.dat\n")
        f.write("edgevertice_filename input/EdgeVertice.dat\n")
        f.write("output_filename output/mesh.plt\n")
    return "input/mesh.conf"

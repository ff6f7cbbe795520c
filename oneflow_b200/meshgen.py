"""Seeded synthetic meshes for the benchmark configurations.

No dataset is involved: every mesh is generated from a formula and a seed
(numpy PCG64), so the GPU solver and the reference CPU solver read the same
grid.  Face numbering follows the reference's convention (boundary faces
first, normal pointing from lCells to rCells).
"""
from __future__ import annotations

import numpy as np

from .meshio import Mesh

SOLID, SYM, FAR, OUT = 2, 3, 4, 6


def _faces_from_cells_2d(cells, bc_of_edge):
    """Edges of a list of CCW polygons (tuples of node ids).  The first cell
    that lists an edge owns it (lc) and keeps its direction, so the normal
    (y2-y1, x1-x2) points from lc to rc.  Boundary edges come first, in the
    order their owning cells list them; interior edges follow in order of
    first appearance.  bc_of_edge(a, b) -> BC code of a boundary edge."""
    seen = {}
    order = []
    for ci, cell in enumerate(cells):
        n = len(cell)
        for k in range(n):
            a, b = int(cell[k]), int(cell[(k + 1) % n])
            key = (a, b) if a < b else (b, a)
            if key in seen:
                seen[key][2] = ci
            else:
                seen[key] = [a, b, -1, ci]
                order.append(key)
    bnd = [seen[k] for k in order if seen[k][2] < 0]
    inn = [seen[k] for k in order if seen[k][2] >= 0]
    faces = bnd + inn
    nodes = np.array([[f[0], f[1]] for f in faces], np.int64)
    lc = np.array([f[3] for f in faces], np.int64)
    rc = np.array([f[2] for f in faces], np.int64)
    bct = np.array([bc_of_edge(f[0], f[1]) for f in bnd], np.int32)
    return nodes, lc, rc, len(bnd), bct


def bump_channel(ni: int = 256, nj: int = 128, thickness: float = 0.10, jitter: float = 0.2,
                 seed: int = 20261203) -> Mesh:
    """2-D channel [0,3]x[0,1] with a circular-arc bump of the given
    thickness on the lower wall over x in [1,2]; ni x nj quads, each split in
    two triangles with an alternating diagonal (2*ni*nj cells); interior nodes
    jittered by U(-jitter*h, jitter*h).  Walls are SOLID_SURFACE, inlet and
    outlet FARFIELD."""
    rng = np.random.default_rng(seed)
    xs = np.linspace(0.0, 3.0, ni + 1)
    # circular arc through (1,0), (1.5,t), (2,0)
    t = thickness
    radius = (0.25 + t * t) / (2.0 * t)
    yb = np.where((xs > 1.0) & (xs < 2.0), np.sqrt(np.maximum(radius ** 2 - (xs - 1.5) ** 2, 0.0)) - (radius - t), 0.0)
    eta = np.linspace(0.0, 1.0, nj + 1)
    X = np.repeat(xs[:, None], nj + 1, axis=1)
    Y = yb[:, None] + (1.0 - yb[:, None]) * eta[None, :]
    hx = 3.0 / ni
    hy = (1.0 - yb[:, None]) / nj
    jx = rng.uniform(-jitter, jitter, X.shape) * hx
    jy = rng.uniform(-jitter, jitter, X.shape) * hy
    interior = np.zeros(X.shape, bool)
    interior[1:-1, 1:-1] = True
    X = X + np.where(interior, jx, 0.0)
    Y = Y + np.where(interior, jy, 0.0)
    nid = lambda i, j: i * (nj + 1) + j
    tris = []
    for i in range(ni):
        for j in range(nj):
            a, b, c, d = nid(i, j), nid(i + 1, j), nid(i + 1, j + 1), nid(i, j + 1)
            if (i + j) % 2 == 0:
                tris.append((a, b, c)); tris.append((a, c, d))
            else:
                tris.append((a, b, d)); tris.append((b, c, d))
    x = X.ravel(); y = Y.ravel()

    def bc(a, b):
        ia, ja = divmod(a, nj + 1)
        ib, jb = divmod(b, nj + 1)
        if ia == ib and ia in (0, ni):
            return FAR
        return SOLID

    nodes, lc, rc, nb, bct = _faces_from_cells_2d(tris, bc)
    nf = nodes.shape[0]
    return Mesh(2, x, y, np.zeros_like(x), np.full(nf, 2, np.int32), nodes.ravel().astype(np.int32),
                lc.astype(np.int32), rc.astype(np.int32), len(tris), nb, bct,
                meta=dict(kind="bump_channel", ni=ni, nj=nj, seed=seed, jitter=jitter))


def plate_2d(ni: int = 48, nj: int = 32, ratio: float = 1.15, y1: float = 2.0e-4, x_lead: float = 0.5,
             length: float = 1.0, jitter: float = 0.1, seed: int = 20261205) -> Mesh:
    """2-D flat plate of quadrilaterals: wall (SOLID_SURFACE) on y = 0 for
    x in [0, length], symmetry plane upstream, FARFIELD inlet and top,
    OUTFLOW at the exit.  Wall-normal spacing grows geometrically from y1;
    interior nodes jittered in x by U(-jitter*h, jitter*h) (seeded)."""
    rng = np.random.default_rng(seed)
    n_up = max(ni // 6, 2)
    xu = -x_lead * (1.0 - np.linspace(0.0, 1.0, n_up + 1)) ** 1.5
    xp = length * np.linspace(0.0, 1.0, ni - n_up + 1) ** 1.3
    xs = np.concatenate([xu[:-1], xp])
    ys = np.concatenate([[0.0], y1 * np.cumsum(ratio ** np.arange(nj))])
    X, Y = np.meshgrid(xs, ys, indexing="ij")
    hx = np.gradient(xs)[:, None] * np.ones_like(X)
    interior = np.zeros(X.shape, bool)
    interior[1:-1, 1:-1] = True
    X = X + np.where(interior, rng.uniform(-jitter, jitter, X.shape) * hx, 0.0)
    nid = lambda i, j: i * (nj + 1) + j
    quads = [(nid(i, j), nid(i + 1, j), nid(i + 1, j + 1), nid(i, j + 1)) for i in range(ni) for j in range(nj)]
    x, y = X.ravel(), Y.ravel()

    def bc(a, b):
        ia, ja = divmod(a, nj + 1)
        ib, jb = divmod(b, nj + 1)
        if ja == 0 and jb == 0:
            return SOLID if min(xs[ia], xs[ib]) >= -1e-12 else SYM
        if ia == ib == ni:
            return OUT
        return FAR

    nodes, lc, rc, nb, bct = _faces_from_cells_2d(quads, bc)
    nf = nodes.shape[0]
    return Mesh(2, x, y, np.zeros_like(x), np.full(nf, 2, np.int32), nodes.ravel().astype(np.int32),
                lc.astype(np.int32), rc.astype(np.int32), len(quads), nb, bct,
                meta=dict(kind="plate_2d", ni=ni, nj=nj, seed=seed))


# ------------------------------------------------------------------------
# 3-D flat plate: hexahedral lattice split into 6 tetrahedra per hex
# ------------------------------------------------------------------------
# Kuhn split of the unit cube along the diagonal v0 -> v6; vertex ids
# 0:(0,0,0) 1:(1,0,0) 2:(1,1,0) 3:(0,1,0) 4:(0,0,1) 5:(1,0,1) 6:(1,1,1) 7:(0,1,1).
# Every tet is a monotone path 0 -> ... -> 6, so shared quad faces of
# neighbouring hexes get the same diagonal and the tets conform.
_KUHN = np.array([[0, 1, 2, 6], [0, 2, 3, 6], [0, 3, 7, 6], [0, 7, 4, 6], [0, 4, 5, 6], [0, 5, 1, 6]], np.int64)
_CORNER = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], np.int64)


def flat_plate_tets(nx: int = 200, ny: int = 100, nz: int = 50, ratio: float = 1.15, reynolds: float = 5.0e6,
                    yplus: float = 1.0, x_lead: float = 0.5, length: float = 1.0, span: float = 0.5,
                    jitter: float = 0.1, seed: int = 20261204) -> Mesh:
    """Flat plate on y = 0, x in [0, length], preceded by a symmetry plane over
    [-x_lead, 0).  Wall-normal spacing grows geometrically (ratio) from a
    first cell at the requested y+ (turbulent skin-friction estimate
    cf = 0.0592 Re^-0.2 at x = length).  Each of nx*ny*nz hexes is split into 6
    tets (6*nx*ny*nz cells).  Interior nodes are jittered in x and z by
    U(-jitter*h, jitter*h) (seeded).  BCs: wall SOLID_SURFACE, upstream floor
    and both span planes SYMMETRY, inlet/top/outlet FARFIELD."""
    rng = np.random.default_rng(seed)
    cf = 0.0592 * reynolds ** -0.2
    utau = np.sqrt(0.5 * cf)
    y1 = yplus / (utau * reynolds)
    ys = np.concatenate([[0.0], y1 * np.cumsum(ratio ** np.arange(ny))])
    # x: cluster at the leading edge, uniform-ish on the plate
    n_up = max(nx // 8, 2)
    xu = -x_lead * (1.0 - np.linspace(0.0, 1.0, n_up + 1)) ** 1.5
    xp = length * np.linspace(0.0, 1.0, nx - n_up + 1) ** 1.2
    xs = np.concatenate([xu[:-1], xp])
    zs = np.linspace(0.0, span, nz + 1)
    X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
    hx = np.gradient(xs)[:, None, None] * np.ones_like(X)
    hz = (span / nz) * np.ones_like(X)
    interior = np.zeros(X.shape, bool)
    interior[1:-1, 1:-1, 1:-1] = True
    X = X + np.where(interior, rng.uniform(-jitter, jitter, X.shape) * hx, 0.0)
    Z = Z + np.where(interior, rng.uniform(-jitter, jitter, X.shape) * hz, 0.0)
    NX, NY, NZ = nx + 1, ny + 1, nz + 1
    x, y, z = X.ravel(), Y.ravel(), Z.ravel()
    nid = lambda i, j, k: (i * NY + j) * NZ + k

    # hex cells in natural (k fastest, then j, then i) order, 6 tets each
    ii, jj, kk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    ii, jj, kk = ii.ravel(), jj.ravel(), kk.ravel()
    corner = np.stack([nid(ii + c[0], jj + c[1], kk + c[2]) for c in _CORNER], axis=1)  # [nhex, 8]
    tets = corner[:, _KUHN].reshape(-1, 4)                                           # [6*nhex, 4]
    nc = tets.shape[0]
    # tet faces (opposite each vertex), oriented outward
    lf = np.array([[1, 2, 3], [0, 3, 2], [0, 1, 3], [0, 2, 1]], np.int64)
    tri = tets[:, lf].reshape(-1, 3)
    owner = np.repeat(np.arange(nc), 4)
    # orient outward: normal . (face centroid - cell centroid) > 0
    P = np.stack([x, y, z], 1)
    cc = P[tets].mean(1)
    a, b, c = P[tri[:, 0]], P[tri[:, 1]], P[tri[:, 2]]
    nrm = np.cross(b - a, c - a)
    out = np.einsum("ij,ij->i", nrm, (a + b + c) / 3.0 - cc[owner]) > 0
    tri[~out] = tri[~out][:, [0, 2, 1]]
    del a, b, c, nrm, out, cc
    s = np.sort(tri, axis=1)
    key = (s[:, 0] * (len(x)) + s[:, 1]) * len(x) + s[:, 2]
    del s
    order = np.argsort(key, kind="stable")
    ks = key[order]
    del key
    new = np.ones(ks.shape[0], bool)
    new[1:] = ks[1:] != ks[:-1]
    grp = np.cumsum(new) - 1
    nf = int(grp[-1]) + 1
    first = order[new]
    cnt = np.bincount(grp, minlength=nf)
    # for interior faces the second entry of the group is the other cell
    pos2 = np.flatnonzero(new) + 1
    has2 = cnt == 2
    lc = owner[first]
    rc = np.full(nf, -1, np.int64)
    rc[has2] = owner[order[pos2[has2]]]
    nodes = tri[first]
    # the face keeps the lower cell as lc (its outward orientation)
    swap = has2 & (rc < lc)
    lc2 = np.where(swap, rc, lc)
    rc2 = np.where(swap, lc, rc)
    second_nodes = tri[order[np.minimum(pos2, len(order) - 1)]]
    nodes = np.where(swap[:, None], second_nodes, nodes)
    lc, rc = lc2, rc2
    del order, ks, grp, new, second_nodes
    isb = rc < 0
    # boundary classification from the face centroid position
    fcx = x[nodes].mean(1); fcy = y[nodes].mean(1); fcz = z[nodes].mean(1)
    tol = 1e-12
    bct_all = np.full(nf, FAR, np.int32)
    floor = fcy < y1 * 1e-6
    bct_all[floor & (fcx >= -tol)] = SOLID
    bct_all[floor & (fcx < -tol)] = SYM
    sidez = (np.abs(fcz) < tol) | (np.abs(fcz - span) < tol)
    bct_all[sidez & ~floor] = SYM
    # order: boundary faces first (by owning cell), interior faces by (lc, rc)
    forder = np.lexsort((rc, lc, ~isb))
    lc, rc, nodes, bct_all = lc[forder], rc[forder], nodes[forder], bct_all[forder]
    nb = int(isb.sum())
    mesh = Mesh(3, x, y, z, np.full(nf, 3, np.int32), nodes.ravel().astype(np.int32), lc.astype(np.int32),
                rc.astype(np.int32), nc, nb, bct_all[:nb].copy(),
                meta=dict(kind="flat_plate_tets", nx=nx, ny=ny, nz=nz, ratio=ratio, y1=y1, seed=seed))
    return mesh


# the six quad faces of a hex (corner order of _CORNER), each outward-oriented
_HEX_FACES = np.array([[0, 3, 2, 1], [4, 5, 6, 7], [0, 1, 5, 4], [3, 7, 6, 2], [0, 4, 7, 3], [1, 2, 6, 5]], np.int64)


def bump_box_hexes(nx: int = 12, ny: int = 8, nz: int = 10, height: float = 0.15, jitter: float = 0.15,
                   seed: int = 20261203) -> Mesh:
    """Hexahedral box [0,1] x [0,1] x [0,1] over a Gaussian bump on its floor
    (y_floor = height * exp(-((x-.5)^2 + (z-.5)^2) / 0.05)); the layers above
    follow the floor, fading out towards the top.  Interior nodes jittered
    (seeded), so the quad faces are warped.  BCs: floor SOLID_SURFACE, the
    other five sides FARFIELD.  A mesh with non-planar quadrilateral walls,
    for metrics and wall-distance tests."""
    rng = np.random.default_rng(seed)
    xs, ys, zs = np.linspace(0, 1, nx + 1), np.linspace(0, 1, ny + 1), np.linspace(0, 1, nz + 1)
    X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
    floor = height * np.exp(-((X - 0.5) ** 2 + (Z - 0.5) ** 2) / 0.05)
    Y = Y + floor * (1.0 - Y)
    interior = np.zeros(X.shape, bool)
    interior[1:-1, 1:-1, 1:-1] = True
    h = np.array([1.0 / nx, 1.0 / ny, 1.0 / nz])
    for A, hh in ((X, h[0]), (Y, h[1]), (Z, h[2])):
        A += np.where(interior, rng.uniform(-jitter, jitter, A.shape) * hh, 0.0)
    NY, NZ = ny + 1, nz + 1
    x, y, z = X.ravel(), Y.ravel(), Z.ravel()
    nid = lambda i, j, k: (i * NY + j) * NZ + k
    ii, jj, kk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    ii, jj, kk = ii.ravel(), jj.ravel(), kk.ravel()
    corner = np.stack([nid(ii + c[0], jj + c[1], kk + c[2]) for c in _CORNER], axis=1)   # [nc, 8]
    nc = corner.shape[0]
    quad = corner[:, _HEX_FACES].reshape(-1, 4)
    owner = np.repeat(np.arange(nc), 6)
    # the left-handed corner order of _CORNER makes these faces inward: flip
    P = np.stack([x, y, z], 1)
    cc = P[corner].mean(1)
    fc = P[quad].mean(1)
    nrm = np.cross(P[quad[:, 2]] - P[quad[:, 0]], P[quad[:, 3]] - P[quad[:, 1]])
    inward = np.einsum("ij,ij->i", nrm, fc - cc[owner]) < 0
    quad[inward] = quad[inward][:, ::-1]
    s = np.sort(quad, axis=1)
    key = ((s[:, 0] * len(x) + s[:, 1]) * len(x) + s[:, 2]) * len(x) + s[:, 3]
    order = np.argsort(key, kind="stable")
    ks = key[order]
    new = np.ones(ks.shape[0], bool)
    new[1:] = ks[1:] != ks[:-1]
    grp = np.cumsum(new) - 1
    nf = int(grp[-1]) + 1
    first = order[new]
    cnt = np.bincount(grp, minlength=nf)
    pos2 = np.flatnonzero(new) + 1
    has2 = cnt == 2
    lc = owner[first]
    rc = np.full(nf, -1, np.int64)
    rc[has2] = owner[order[pos2[has2]]]
    nodes = quad[first]
    swap = has2 & (rc < lc)
    second = quad[order[np.minimum(pos2, len(order) - 1)]]
    nodes = np.where(swap[:, None], second, nodes)
    lc, rc = np.where(swap, rc, lc), np.where(swap, lc, rc)
    isb = rc < 0
    bct_all = np.full(nf, FAR, np.int32)
    floor_nodes = nid(*np.meshgrid(np.arange(nx + 1), [0], np.arange(nz + 1), indexing="ij")).ravel()
    bct_all[isb & np.all(np.isin(nodes, floor_nodes), axis=1)] = SOLID
    forder = np.lexsort((rc, lc, ~isb))
    lc, rc, nodes, bct_all = lc[forder], rc[forder], nodes[forder], bct_all[forder]
    nb = int(isb.sum())
    return Mesh(3, x, y, z, np.full(nf, 4, np.int32), nodes.ravel().astype(np.int32), lc.astype(np.int32),
                rc.astype(np.int32), nc, nb, bct_all[:nb].copy(),
                meta=dict(kind="bump_box_hexes", nx=nx, ny=ny, nz=nz, seed=seed))


def _faces_from_polygons_2d(poly: np.ndarray, counts: np.ndarray, n_nodes: int):
    """Vectorised edge extraction for CCW polygons given as a padded node
    array poly[nc, kmax] with counts[nc] valid entries: returns (nodes[nf,2],
    lc, rc) with boundary edges (rc = -1) first, each edge directed as its
    owner (the lower-numbered cell) lists it, so (y2-y1, x1-x2) points from lc
    to rc."""
    nc, kmax = poly.shape
    k = np.arange(kmax)[None, :]
    valid = k < counts[:, None]
    nxt = np.where(k + 1 < counts[:, None], np.roll(poly, -1, axis=1), poly[:, :1])
    a, b = poly[valid], nxt[valid]
    owner = np.repeat(np.arange(nc), counts)
    key = np.minimum(a, b).astype(np.int64) * n_nodes + np.maximum(a, b)
    order = np.lexsort((owner, key))
    ks = key[order]
    new = np.ones(ks.shape[0], bool)
    new[1:] = ks[1:] != ks[:-1]
    grp = np.cumsum(new) - 1
    nf = int(grp[-1]) + 1
    first = order[new]
    cnt = np.bincount(grp, minlength=nf)
    pos2 = np.flatnonzero(new) + 1
    lc = owner[first]
    rc = np.full(nf, -1, np.int64)
    has2 = cnt == 2
    rc[has2] = owner[order[pos2[has2]]]
    nodes = np.stack([a[first], b[first]], 1)
    isb = rc < 0
    forder = np.lexsort((rc, lc, ~isb))
    return nodes[forder], lc[forder], rc[forder], int(isb.sum())


def naca4_parts(m: float, p: float, t: float, x: np.ndarray):
    """NACA 4-digit section at chord stations x (chord 1): half thickness yt
    (closed-trailing-edge coefficient -0.1036), camber line yc and its angle"""
    x = np.asarray(x, np.float64)
    yt = 5.0 * t * (0.2969 * np.sqrt(x) - 0.1260 * x - 0.3516 * x ** 2 + 0.2843 * x ** 3 - 0.1036 * x ** 4)
    if m > 0.0:
        fore = x < p
        yc = np.where(fore, m / p ** 2 * (2 * p * x - x ** 2), m / (1 - p) ** 2 * ((1 - 2 * p) + 2 * p * x - x ** 2))
        dyc = np.where(fore, 2 * m / p ** 2 * (p - x), 2 * m / (1 - p) ** 2 * (p - x))
    else:
        yc = np.zeros_like(x); dyc = np.zeros_like(x)
    return yt, yc, np.arctan(dyc)


def naca4_surface(m: float, p: float, t: float, n_half: int) -> np.ndarray:
    """Closed NACA 4-digit section (max camber m, its position p, thickness t,
    chord 1), cosine-spaced: 2 n_half points from the trailing edge along the
    lower surface to the leading edge and back along the upper surface."""
    beta = np.linspace(0.0, np.pi, n_half + 1)
    x = 0.5 * (1.0 - np.cos(beta))
    yt, yc, th = naca4_parts(m, p, t, x)
    xu, yu = x - yt * np.sin(th), yc + yt * np.cos(th)
    xl, yl = x + yt * np.sin(th), yc - yt * np.cos(th)
    lower = np.stack([xl[::-1], yl[::-1]], 1)          # TE -> LE
    upper = np.stack([xu[1:-1], yu[1:-1]], 1)          # after LE -> before TE
    return np.concatenate([lower, upper])


def naca_ogrid(m: float = 0.02, p: float = 0.4, t: float = 0.12, n_surface: int = 200, n_layers: int = 100,
               n_quad_layers: int = None, y1: float = 1.0e-5, radius: float = 20.0) -> Mesh:
    """Hybrid O-grid around a NACA 4-digit section: n_surface points on the
    section, n_layers layers out to a circle of the given radius (chords)
    about mid-chord, the layer spacing growing geometrically from y1 at the
    wall.  The inner n_quad_layers layers are quadrilaterals (the boundary
    layer), the rest split into triangles (alternating diagonals).  Layers
    leave the wall along its normals (the bisector at the trailing edge) and
    then run straight to the circle point at the same arc-length fraction of
    the offset curve where they turn.
    BCs: section SOLID_SURFACE, circle FARFIELD."""
    if n_quad_layers is None:
        n_quad_layers = n_layers // 2
    S = naca4_surface(m, p, t, n_surface // 2)
    n = S.shape[0]
    # layer fractions: first step y1/radius, geometric growth to 1
    d0 = y1 / radius
    lo, hi = 1.0 + 1e-12, 2.0
    for _ in range(200):
        r = 0.5 * (lo + hi)
        if d0 * (r ** n_layers - 1.0) / (r - 1.0) > 1.0:
            hi = r
        else:
            lo = r
    f = np.concatenate([[0.0], np.cumsum(d0 * r ** np.arange(n_layers))])
    f /= f[-1]
    # within `reach` of the wall the layers follow the section's normals (the
    # bisector at the trailing edge), so the boundary-layer cells are
    # wall-normal; beyond it straight lines run on to the circle
    tng = np.roll(S, -1, 0) - np.roll(S, 1, 0)
    nrm = np.stack([-tng[:, 1], tng[:, 0]], 1)          # outward for the section's clockwise loop
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    reach = 0.05
    d = (f * radius)[:, None, None]
    E = S + reach * nrm
    # the outer lines run straight from the offset curve E to the circle point
    # at the same arc-length fraction of E (matched by the section's own arc
    # length instead, the clustered trailing-edge points went to nearly one
    # circle point and the grid folded where the lines turned)
    seg = np.linalg.norm(np.roll(E, -1, 0) - E, axis=1)
    s = np.concatenate([[0.0], np.cumsum(seg)[:-1]]) / seg.sum()
    ang = -2.0 * np.pi * s                              # same turning sense as the section loop
    Cc = np.stack([0.5 + radius * np.cos(ang), radius * np.sin(ang)], 1)
    near = S[None] + np.minimum(d, reach) * nrm[None]
    far = E[None] + np.clip((d - reach) / (radius - reach), 0.0, 1.0) * (Cc - E)[None]
    P = np.where(d <= reach, near, far)                                 # [K+1, n, 2]
    x, y = P[..., 0].ravel(), P[..., 1].ravel()
    nid = lambda k, i: k * n + (i % n)
    kk, ii = np.meshgrid(np.arange(n_layers), np.arange(n), indexing="ij")
    a, b, c, d = nid(kk, ii), nid(kk, ii + 1), nid(kk + 1, ii + 1), nid(kk + 1, ii)
    quad = kk < n_quad_layers
    qa = np.stack([a[quad], b[quad], c[quad], d[quad]], 1)
    tk, ti = kk[~quad], ii[~quad]
    alt = (tk + ti) % 2 == 0
    A, B, Cn, D = a[~quad], b[~quad], c[~quad], d[~quad]
    t1 = np.where(alt[:, None], np.stack([A, B, Cn], 1), np.stack([A, B, D], 1))
    t2 = np.where(alt[:, None], np.stack([A, Cn, D], 1), np.stack([B, Cn, D], 1))
    tri = np.stack([t1, t2], 1).reshape(-1, 3)
    poly = np.full((qa.shape[0] + tri.shape[0], 4), -1, np.int64)
    poly[:qa.shape[0]] = qa
    poly[qa.shape[0]:, :3] = tri
    counts = np.concatenate([np.full(qa.shape[0], 4), np.full(tri.shape[0], 3)])
    # counter-clockwise cells (shoelace area > 0)
    idx = np.where(poly < 0, poly[:, :1], poly)
    px, py = x[idx], y[idx]
    kx = np.arange(4)[None, :] < counts[:, None]
    nx_ = np.where(np.arange(4)[None, :] + 1 < counts[:, None], np.roll(px, -1, 1), px[:, :1])
    ny_ = np.where(np.arange(4)[None, :] + 1 < counts[:, None], np.roll(py, -1, 1), py[:, :1])
    area2 = np.where(kx, px * ny_ - nx_ * py, 0.0).sum(1)
    cw = area2 < 0
    for cnt in (3, 4):
        sel = cw & (counts == cnt)
        poly[sel, :cnt] = poly[sel, :cnt][:, ::-1]
    nodes, lc, rc, nb = _faces_from_polygons_2d(poly, counts, x.shape[0])
    wall = nodes[:nb].max(1) < n
    bct = np.where(wall, SOLID, FAR).astype(np.int32)
    nf = nodes.shape[0]
    return Mesh(2, x, y, np.zeros_like(x), np.full(nf, 2, np.int32), nodes.ravel().astype(np.int32),
                lc.astype(np.int32), rc.astype(np.int32), poly.shape[0], nb, bct,
                meta=dict(kind="naca_ogrid", m=m, p=p, t=t, n_surface=n, n_layers=n_layers))


def airfoil_cases(n_cases: int = 64, seed: int = 20261205, min_cells: int = 20000, max_cells: int = 400000):
    """Seeded batch of 2-D RANS-SA airfoil solves: NACA 4-digit sections
    (camber 0-6 % at 40 % chord, thickness 8-18 %), hybrid O-grids whose cell
    counts are log-uniform in [min_cells, max_cells], Mach U(0.3, 0.8), AoA
    U(-2, 8) degrees, Re log-uniform in [1e6, 1e7]; first-cell height for
    y+ ~ 1.  Returns [(mesh, dict(mach, aoa, reynolds))]; the meshes carry no
    wall distance (an SA solve computes it on the GPU)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_cases):
        m, t = rng.uniform(0.0, 0.06), rng.uniform(0.08, 0.18)
        cells = float(np.exp(rng.uniform(np.log(min_cells), np.log(max_cells))))
        mach, aoa = rng.uniform(0.3, 0.8), rng.uniform(-2.0, 8.0)
        re = float(np.exp(rng.uniform(np.log(1e6), np.log(1e7))))
        # quads in the inner half of the layers, two triangles per cell outside:
        # cells = n_s * 1.5 * n_layers with n_layers = n_s / 2
        ns = int(round(np.sqrt(cells / 0.75) / 2.0)) * 2
        nl = max(ns // 2, 8)
        utau = np.sqrt(0.5 * 0.0592 * re ** -0.2)
        mesh = naca_ogrid(m, 0.4, t, ns, nl, y1=1.0 / (utau * re))
        out.append((mesh, dict(mach=mach, aoa=aoa, reynolds=re)))
    return out


def _faces_3d(faces_list, owners, n_nodes):
    """Shared-face extraction for 3-D cells: faces_list is a list of node
    arrays [m, k] (k = 3 or 4, each face listed outward from its owner) with
    owners [m].  Returns (face node lists, counts, lc, rc) with boundary faces
    first (ordered by owner), interior faces ordered by (lc, rc); each face
    keeps the node order of its lower-numbered cell, so its normal points
    from lc to rc."""
    keys, nodes, cnts, own = [], [], [], []
    for F, O in zip(faces_list, owners):
        k = F.shape[1]
        s = np.sort(F, axis=1).astype(np.int64)
        key = np.zeros(F.shape[0], np.int64) + k
        for c in range(k):
            key = key * n_nodes + s[:, c]
        if k == 3:
            key = key * n_nodes + n_nodes - 1      # distinct from any quad key
        keys.append(key)
        pad = np.full((F.shape[0], 4), -1, np.int64)
        pad[:, :k] = F
        nodes.append(pad); cnts.append(np.full(F.shape[0], k)); own.append(O)
    key = np.concatenate(keys); nodes = np.concatenate(nodes); cnt = np.concatenate(cnts)
    owner = np.concatenate(own)
    order = np.lexsort((owner, key))
    ks = key[order]
    new = np.ones(ks.shape[0], bool)
    new[1:] = ks[1:] != ks[:-1]
    grp = np.cumsum(new) - 1
    nf = int(grp[-1]) + 1
    first = order[new]
    num = np.bincount(grp, minlength=nf)
    pos2 = np.flatnonzero(new) + 1
    lc = owner[first]
    rc = np.full(nf, -1, np.int64)
    has2 = num == 2
    rc[has2] = owner[order[pos2[has2]]]
    fn, fc = nodes[first], cnt[first]
    isb = rc < 0
    forder = np.lexsort((rc, lc, ~isb))
    return fn[forder], fc[forder], lc[forder], rc[forder], int(isb.sum())


def bump_box_mixed(nx: int = 12, ny: int = 8, nz: int = 10, height: float = 0.15, jitter: float = 0.15,
                   prism_from: int = None, seed: int = 20261203) -> Mesh:
    """The bump box of bump_box_hexes with the columns i >= prism_from (default
    nx/2) split into two triangular prisms each (through the diagonal of the
    column's x-z quad), so hexahedra and prisms share quadrilateral side faces
    and the floor carries quadrilateral and triangular wall faces.  BCs: floor
    SOLID_SURFACE, the other sides FARFIELD."""
    if prism_from is None:
        prism_from = nx // 2
    rng = np.random.default_rng(seed)
    xs, ys, zs = np.linspace(0, 1, nx + 1), np.linspace(0, 1, ny + 1), np.linspace(0, 1, nz + 1)
    X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
    Y = Y + height * np.exp(-((X - 0.5) ** 2 + (Z - 0.5) ** 2) / 0.05) * (1.0 - Y)
    interior = np.zeros(X.shape, bool)
    interior[1:-1, 1:-1, 1:-1] = True
    h = np.array([1.0 / nx, 1.0 / ny, 1.0 / nz])
    for A, hh in ((X, h[0]), (Y, h[1]), (Z, h[2])):
        A += np.where(interior, rng.uniform(-jitter, jitter, A.shape) * hh, 0.0)
    NY, NZ = ny + 1, nz + 1
    x, y, z = X.ravel(), Y.ravel(), Z.ravel()
    P = np.stack([x, y, z], 1)
    nid = lambda i, j, k: (i * NY + j) * NZ + k
    ii, jj, kk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    ii, jj, kk = ii.ravel(), jj.ravel(), kk.ravel()
    corner = np.stack([nid(ii + c[0], jj + c[1], kk + c[2]) for c in _CORNER], axis=1)
    hexm = ii < prism_from
    H = corner[hexm]
    Pc = corner[~hexm]
    # prism A: (c0 c1 c5 | c3 c2 c6), prism B: (c0 c5 c4 | c3 c6 c7), cells of a column adjacent
    pa = Pc[:, [0, 1, 5, 3, 2, 6]]
    pb = Pc[:, [0, 5, 4, 3, 6, 7]]
    prisms = np.stack([pa, pb], 1).reshape(-1, 6)
    nh, npr = H.shape[0], prisms.shape[0]
    nc = nh + npr
    # faces of each cell (any orientation; made outward below)
    hq = H[:, _HEX_FACES].reshape(-1, 4); hq_own = np.repeat(np.arange(nh), 6)
    tri_idx = np.array([[0, 1, 2], [3, 4, 5]]); quad_idx = np.array([[0, 1, 4, 3], [1, 2, 5, 4], [2, 0, 3, 5]])
    pt = prisms[:, tri_idx].reshape(-1, 3); pt_own = nh + np.repeat(np.arange(npr), 2)
    pq = prisms[:, quad_idx].reshape(-1, 4); pq_own = nh + np.repeat(np.arange(npr), 3)
    cc = np.concatenate([P[H].mean(1), P[prisms].mean(1)])

    def outward(F, own):
        fcn = P[F].mean(1)
        if F.shape[1] == 3:
            n = np.cross(P[F[:, 1]] - P[F[:, 0]], P[F[:, 2]] - P[F[:, 0]])
        else:
            n = np.cross(P[F[:, 2]] - P[F[:, 0]], P[F[:, 3]] - P[F[:, 1]])
        inward = np.einsum("ij,ij->i", n, fcn - cc[own]) < 0
        F = F.copy()
        F[inward] = F[inward][:, ::-1]
        return F

    fn, fc, lc, rc, nb = _faces_3d([outward(hq, hq_own), outward(pt, pt_own), outward(pq, pq_own)],
                                   [hq_own, pt_own, pq_own], len(x))
    floor_nodes = nid(*np.meshgrid(np.arange(nx + 1), [0], np.arange(nz + 1), indexing="ij")).ravel()
    fb = fn[:nb]
    on_floor = np.all(np.isin(np.where(fb < 0, floor_nodes[0], fb), floor_nodes), axis=1)
    bct = np.where(on_floor, SOLID, FAR).astype(np.int32)
    flat = fn[np.arange(4)[None, :] < fc[:, None]]          # row by row: each face's nodes in order
    return Mesh(3, x, y, z, fc.astype(np.int32), flat.astype(np.int32), lc.astype(np.int32), rc.astype(np.int32),
                nc, nb, bct, meta=dict(kind="bump_box_mixed", nx=nx, ny=ny, nz=nz, prism_from=prism_from, seed=seed))


# ------------------------------------------------------------------------
# 3-D swept wing: hexahedral boundary layer + tetrahedral far field
# ------------------------------------------------------------------------
def _dedupe_faces(F: np.ndarray, owner: np.ndarray):
    """Shared faces of one face kind (all rows k nodes, listed outward from
    their owner): returns (nodes, lc, rc) with rc = -1 on boundary faces and
    each face in the orientation of its lower-numbered cell (lc < rc).  Rows
    are matched on their sorted node tuples (no combined integer key, so any
    node count works)."""
    s = np.sort(F, axis=1)
    order = np.lexsort(tuple(s[:, c] for c in range(s.shape[1] - 1, -1, -1)) + ())
    ss = s[order]
    new = np.ones(len(order), bool)
    new[1:] = np.any(ss[1:] != ss[:-1], axis=1)
    del s, ss
    grp = np.cumsum(new) - 1
    nf = int(grp[-1]) + 1
    cnt = np.bincount(grp, minlength=nf)
    if cnt.max() > 2:
        raise ValueError("a face is shared by more than two cells")
    first = order[new]
    pos2 = np.minimum(np.flatnonzero(new) + 1, len(order) - 1)
    second = order[pos2]
    has2 = cnt == 2
    lc = owner[first].copy()
    rc = np.where(has2, owner[second], -1)
    nodes = F[first].copy()
    swap = has2 & (rc < lc)
    lc[swap], rc[swap] = rc[swap], owner[first][swap]
    nodes[swap] = F[second[swap]]
    return nodes, lc, rc


def swept_wing_hybrid(n_around: int = 256, n_hex: int = 30, hex_ratio: float = 1.2, n_tet: int = 44,
                      nz_wing: int = 76, nz_tip: int = 30, t: float = 0.12, aspect_ratio: float = 4.0,
                      sweep_deg: float = 30.0, radius: float = 20.0, reynolds: float = 1.2e7,
                      yplus: float = 1.0) -> Mesh:
    """Hybrid mesh around a swept NACA 00xx wing (half model, chord 1, root on
    the symmetry plane z = 0, semi-span aspect_ratio / 2, leading edge swept
    back by sweep_deg; the whole grid is sheared with it).  Cross-section: an
    O-grid of n_around points around the section; its first n_hex layers grow
    from a first cell at the requested y+ (flat-plate skin-friction estimate
    at the wing's Reynolds number) by hex_ratio and are hexahedra, the next
    n_tet layers grow geometrically to a cylinder of the given radius and each
    hexahedral cell there is split into six tetrahedra (the Kuhn split along
    the cell's (i, k, z) diagonal, so neighbouring splits conform; the last
    hexahedral layer carries the two triangles of its outer neighbour's split
    in place of that quadrilateral face).  Spanwise: nz_wing slabs over the
    wing (clustered at the tip) and nz_tip slabs beyond it to the far-field
    plane, where the section's interior is filled by a ladder of cells between
    matching lower- and upper-surface points (quadrilaterals, triangles at the
    leading and trailing edges), closed at the tip by a wall.
    BCs: wing and tip SOLID_SURFACE, root plane SYMMETRY, cylinder and the
    outer plane FARFIELD.  About 8.0 M cells at the defaults."""
    nh = n_around // 2
    S = naca4_surface(0.0, 0.4, t, nh)                   # [n] TE -> lower -> LE -> upper
    n = S.shape[0]
    K = n_hex + n_tet
    cf = 0.0592 * reynolds ** -0.2
    y1 = yplus / (np.sqrt(0.5 * cf) * reynolds)
    dh = y1 * hex_ratio ** np.arange(n_hex)              # hexahedral layer thicknesses
    reach = dh.sum()
    # tet layers: geometric growth from the last hex layer's thickness to the cylinder
    lo, hi = 1.0 + 1e-9, 3.0
    d_last = dh[-1]
    for _ in range(200):
        r = 0.5 * (lo + hi)
        if d_last * r * (r ** n_tet - 1.0) / (r - 1.0) > radius - reach:
            hi = r
        else:
            lo = r
    dt = d_last * r ** np.arange(1, n_tet + 1)
    dt *= (radius - reach) / dt.sum()
    dist = np.concatenate([[0.0], np.cumsum(np.concatenate([dh, dt]))])    # [K+1]
    seg = np.linalg.norm(np.roll(S, -1, 0) - S, axis=1)
    sarc = np.concatenate([[0.0], np.cumsum(seg)[:-1]]) / seg.sum()
    ang = -2.0 * np.pi * sarc
    Cc = np.stack([0.5 + radius * np.cos(ang), radius * np.sin(ang)], 1)
    tng = np.roll(S, -1, 0) - np.roll(S, 1, 0)
    nrm = np.stack([-tng[:, 1], tng[:, 0]], 1)
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    d = dist[:, None, None]
    E = S + reach * nrm
    near = S[None] + np.minimum(d, reach) * nrm[None]
    far = E[None] + np.clip((d - reach) / (radius - reach), 0.0, 1.0) * (Cc - E)[None]
    P2 = np.where(d <= reach, near, far)                 # [K+1, n, 2]
    semi = 0.5 * aspect_ratio
    zt = semi * (1.0 - np.cos(np.linspace(0.0, 0.5 * np.pi, nz_wing + 1)))     # clustered at the tip
    ze = semi + (radius - semi) * np.linspace(0.0, 1.0, nz_tip + 1)[1:] ** 1.5
    zs = np.concatenate([zt, ze])
    nz = len(zs) - 1
    tan = np.tan(np.radians(sweep_deg))
    # nodes (s, k, i): index (s * (K + 1) + k) * n + i
    X = P2[None, :, :, 0] + tan * zs[:, None, None]
    Y = np.broadcast_to(P2[None, :, :, 1], X.shape)
    Z = np.broadcast_to(zs[:, None, None], X.shape)
    x, y, z = X.ravel().copy(), Y.ravel().copy(), Z.ravel().copy()
    nid = lambda s, k, i: (s * (K + 1) + k) * n + (i % n)
    # ring cells (s, k, i) in natural order (i fastest, then k, then s)
    ss, kk, ii = np.meshgrid(np.arange(nz), np.arange(K), np.arange(n), indexing="ij")
    ss, kk, ii = ss.ravel(), kk.ravel(), ii.ravel()
    # corners in _CORNER order over local axes (i, k, s)
    corner = np.stack([nid(ss + c[2], kk + c[1], ii + c[0]) for c in _CORNER], axis=1)
    hexm = kk < n_hex
    Hc, Tc = corner[hexm], corner[~hexm]
    H_k = kk[hexm]
    n_h, n_t = Hc.shape[0], Tc.shape[0] * 6
    tets = Tc[:, _KUHN].reshape(-1, 4)
    # ladder cells beyond the tip: lower point j with upper point n - j
    js = np.arange(nh)
    lad_q = js[(js >= 1) & (js <= nh - 2)]
    s_ext = np.arange(nz_wing, nz)
    lad_cells = []
    for s in s_ext:
        a0, a1 = nid(s, 0, 0), nid(s + 1, 0, 0)
        # prism at the trailing edge (0, 1, n-1), hexahedra (j, j+1, n-j-1, n-j), prism at the leading edge
        lad_cells.append(("prism", np.array([[a0 + 0, a0 + 1, a0 + n - 1, a1 + 0, a1 + 1, a1 + n - 1]])))
        q = np.stack([lad_q, lad_q + 1, n - lad_q - 1, n - lad_q], 1)
        lad_cells.append(("hex", np.concatenate([a0 + q, a1 + q], 1)))
        lad_cells.append(("prism", np.array([[a0 + nh - 1, a0 + nh, a0 + nh + 1, a1 + nh - 1, a1 + nh, a1 + nh + 1]])))
    LH = np.concatenate([c for kind, c in lad_cells if kind == "hex"])       # [m, 8]: 4 bottom + 4 top
    LP = np.concatenate([c for kind, c in lad_cells if kind == "prism"])     # [m, 6]: 3 bottom + 3 top
    # cell numbering: ring cells in (s, k, i) order with each outer hexahedron's
    # six tetrahedra in place, then the ladder cells
    ring_id = np.empty(len(kk), np.int64)
    per = np.where(hexm, 1, 6)
    start = np.concatenate([[0], np.cumsum(per)[:-1]])
    ring_id[:] = start
    n_ring = int(per.sum())
    hex_id = ring_id[hexm]
    tet_id = (ring_id[~hexm][:, None] + np.arange(6)[None, :]).ravel()
    lh_id = n_ring + np.arange(LH.shape[0])
    lp_id = n_ring + LH.shape[0] + np.arange(LP.shape[0])
    nc = n_ring + LH.shape[0] + LP.shape[0]
    Pn = np.stack([x, y, z], 1)

    def outward(F, own_centre):
        Fc = Pn[F].mean(1)
        if F.shape[1] == 3:
            nv = np.cross(Pn[F[:, 1]] - Pn[F[:, 0]], Pn[F[:, 2]] - Pn[F[:, 0]])
        else:
            nv = np.cross(Pn[F[:, 2]] - Pn[F[:, 0]], Pn[F[:, 3]] - Pn[F[:, 1]])
        inward = np.einsum("ij,ij->i", nv, Fc - own_centre) < 0
        F = F.copy()
        F[inward] = F[inward][:, ::-1]
        return F

    tri_l, tri_o, quad_l, quad_o = [], [], [], []
    # tetrahedra
    lf = np.array([[1, 2, 3], [0, 3, 2], [0, 1, 3], [0, 2, 1]], np.int64)
    tt = tets[:, lf].reshape(-1, 3)
    to = np.repeat(tet_id, 4)
    tri_l.append(outward(tt, Pn[tets].mean(1)[np.repeat(np.arange(len(tets)), 4)])); tri_o.append(to)
    # ring hexahedra: 6 quads, the outer one (k + 1 side) of the last hex layer split in two
    hcc = Pn[Hc].mean(1)
    hq = Hc[:, _HEX_FACES]                                   # [n_h, 6, 4]
    outer = H_k == n_hex - 1
    # _HEX_FACES[3] = [3, 7, 6, 2] is the k + 1 face (corners with local k = 1)
    keep = np.ones((n_h, 6), bool)
    keep[outer, 3] = False
    quad_l.append(outward(hq[keep], hcc[np.nonzero(keep)[0]])); quad_o.append(hex_id[np.nonzero(keep)[0]])
    # the split k + 1 face: triangles of the Kuhn split of the tetrahedral cell
    # above, whose k-face is (c0 c1 c5 c4) with diagonal c0 -> c5; in this
    # hexahedron's corners those are (3, 2, 6, 7) with diagonal 3 -> 6
    Ho = Hc[outer]
    t1 = Ho[:, [3, 2, 6]]; t2 = Ho[:, [3, 6, 7]]
    own = hex_id[outer]
    tri_l.append(outward(np.concatenate([t1, t2]), np.concatenate([hcc[outer], hcc[outer]]))); tri_o.append(np.concatenate([own, own]))
    # ladder hexahedra: corners (bottom j, j+1, n-j-1, n-j, then top) -> hex faces
    lcc = Pn[LH].mean(1)
    lhf = np.array([[0, 1, 2, 3], [4, 5, 6, 7], [0, 1, 5, 4], [1, 2, 6, 5], [2, 3, 7, 6], [3, 0, 4, 7]], np.int64)
    lq = LH[:, lhf].reshape(-1, 4)
    quad_l.append(outward(lq, lcc[np.repeat(np.arange(len(LH)), 6)])); quad_o.append(np.repeat(lh_id, 6))
    pcc = Pn[LP].mean(1)
    pt = LP[:, [[0, 1, 2], [3, 4, 5]]].reshape(-1, 3)
    pq = LP[:, [[0, 1, 4, 3], [1, 2, 5, 4], [2, 0, 3, 5]]].reshape(-1, 4)
    tri_l.append(outward(pt, pcc[np.repeat(np.arange(len(LP)), 2)])); tri_o.append(np.repeat(lp_id, 2))
    quad_l.append(outward(pq, pcc[np.repeat(np.arange(len(LP)), 3)])); quad_o.append(np.repeat(lp_id, 3))
    Tn, tl, tr = _dedupe_faces(np.concatenate(tri_l), np.concatenate(tri_o))
    Qn, ql_, qr_ = _dedupe_faces(np.concatenate(quad_l), np.concatenate(quad_o))
    nodes = np.full((len(Tn) + len(Qn), 4), -1, np.int64)
    nodes[:len(Tn), :3] = Tn
    nodes[len(Tn):] = Qn
    cnt = np.concatenate([np.full(len(Tn), 3), np.full(len(Qn), 4)])
    lc = np.concatenate([tl, ql_]); rc = np.concatenate([tr, qr_])
    isb = rc < 0
    forder = np.lexsort((rc, lc, ~isb))
    nodes, cnt, lc, rc = nodes[forder], cnt[forder], lc[forder], rc[forder]
    nb = int(isb.sum())
    # boundary codes from the node indices: root plane, outer plane, cylinder, wall
    fb = nodes[:nb]
    valid = fb >= 0
    fbs = np.where(valid, fb, fb[:, :1])
    s_of = fbs // ((K + 1) * n); k_of = (fbs // n) % (K + 1)
    bct = np.full(nb, FAR, np.int32)
    bct[np.all(s_of == 0, axis=1)] = SYM
    wall = np.all(k_of == 0, axis=1) & np.all(s_of <= nz_wing, axis=1)
    bct[wall] = SOLID
    flat = nodes[np.arange(4)[None, :] < cnt[:, None]]
    return Mesh(3, x, y, z, cnt.astype(np.int32), flat.astype(np.int32), lc.astype(np.int32), rc.astype(np.int32),
                nc, nb, bct, meta=dict(kind="swept_wing_hybrid", n_around=n, n_hex=n_hex, n_tet=n_tet,
                                       nz_wing=nz_wing, nz_tip=nz_tip, sweep_deg=sweep_deg, y1=y1,
                                       semi_span=semi))


# ------------------------------------------------------------------------
# lid-driven cavities for the incompressible solver
# ------------------------------------------------------------------------
def lid_cavity_2d(n: int = 64, jitter: float = 0.0, triangles: bool = False, seed: int = 20261206) -> Mesh:
    """Unit square cavity of n x n quadrilaterals (or 2 n^2 triangles with an
    alternating diagonal), interior nodes jittered by U(-jitter*h, jitter*h).
    Every boundary face is SOLID_SURFACE; the lid (y = 1) faces carry
    bc_name_id 1, the other walls 0 -- the region the wall-velocity data of
    the incompressible solver refers to (lid_velocity)."""
    rng = np.random.default_rng(seed)
    xs = np.linspace(0.0, 1.0, n + 1)
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    interior = np.zeros(X.shape, bool)
    interior[1:-1, 1:-1] = True
    h = 1.0 / n
    X = X + np.where(interior, rng.uniform(-jitter, jitter, X.shape) * h, 0.0)
    Y = Y + np.where(interior, rng.uniform(-jitter, jitter, X.shape) * h, 0.0)
    nid = lambda i, j: i * (n + 1) + j
    cells = []
    for i in range(n):
        for j in range(n):
            a, b, c, d = nid(i, j), nid(i + 1, j), nid(i + 1, j + 1), nid(i, j + 1)
            if not triangles:
                cells.append((a, b, c, d))
            elif (i + j) % 2 == 0:
                cells.append((a, b, c)); cells.append((a, c, d))
            else:
                cells.append((a, b, d)); cells.append((b, c, d))
    x, y = X.ravel(), Y.ravel()
    nodes, lc, rc, nb, bct = _faces_from_cells_2d(cells, lambda a, b: SOLID)
    lid = ((y[nodes[:nb, 0]] > 1.0 - 1e-12) & (y[nodes[:nb, 1]] > 1.0 - 1e-12)).astype(np.int32)
    nf = nodes.shape[0]
    return Mesh(2, x, y, np.zeros_like(x), np.full(nf, 2, np.int32), nodes.ravel().astype(np.int32),
                lc.astype(np.int32), rc.astype(np.int32), len(cells), nb, bct, bc_name_id=lid,
                meta=dict(kind="lid_cavity_2d", n=n, jitter=jitter, triangles=triangles, seed=seed))


def lid_cavity_3d(n: int = 24, jitter: float = 0.1, prisms: bool = False, seed: int = 20261206) -> Mesh:
    """Unit cube cavity of n^3 hexahedra (interior nodes jittered, so faces
    are warped), every boundary face SOLID_SURFACE; the lid (y = 1) faces
    carry bc_name_id 1, the other walls 0.  prisms: the columns of the upper
    half in x split into two triangular prisms each (bump_box_mixed)."""
    if prisms:
        m = bump_box_mixed(n, n, n, height=0.0, jitter=jitter, seed=seed)
    else:
        m = bump_box_hexes(n, n, n, height=0.0, jitter=jitter, seed=seed)
    nb = m.n_bfaces
    off = np.concatenate([[0], np.cumsum(m.face_node_count)])
    lid = np.array([np.all(m.y[m.face_nodes[off[f]:off[f + 1]]] > 1.0 - 1e-12) for f in range(nb)], np.int32)
    m.bc_type = np.full(nb, SOLID, np.int32)
    m.bc_name_id = lid
    m.meta = dict(kind="lid_cavity_3d", n=n, jitter=jitter, prisms=prisms, seed=seed)
    return m


def lid_velocity(mesh: Mesh, u_lid: float = 1.0) -> np.ndarray:
    """Per boundary face wall velocity [nBFaces, 3]: (u_lid, 0, 0) on the lid
    (bc_name_id 1), zero elsewhere."""
    w = np.zeros((mesh.n_bfaces, 3), np.float64)
    w[np.asarray(mesh.bc_name_id) == 1, 0] = u_lid
    return w

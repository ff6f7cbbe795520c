"""Wall distance of cell centres (needed by the SA source term).

The reference computes, for every cell centre, the minimum squared distance
to every SOLID_SURFACE boundary face (segments in 2-D, triangles in 3-D,
polygons split about their centroid) and takes the square root
(CalcWallDist / CalcPoint2FaceDist, codes/geometry/src/WallDist.cpp:136-330).
This is the same exact point-to-face distance, vectorised over chunks of
cells with numpy."""
from __future__ import annotations

import numpy as np

from .meshio import Mesh

SOLID = 2


def _seg_d2(P, A, B):
    """squared distance from points P[n,3] to segments A[m,3]-B[m,3] -> [n,m]"""
    AB = B - A                                        # [m,3]
    L2 = np.einsum("ij,ij->i", AB, AB)                # [m]
    AP = P[:, None, :] - A[None, :, :]                # [n,m,3]
    t = np.einsum("nmk,mk->nm", AP, AB) / np.where(L2 > 0, L2, 1.0)
    t = np.clip(t, 0.0, 1.0)
    C = A[None] + t[..., None] * AB[None]
    D = P[:, None, :] - C
    return np.einsum("nmk,nmk->nm", D, D)


def _tri_d2(P, A, B, C):
    """squared distance from points P[n,3] to triangles (A,B,C)[m,3] -> [n,m]"""
    AB, AC = B - A, C - A
    N = np.cross(AB, AC)
    N2 = np.einsum("ij,ij->i", N, N)
    AP = P[:, None, :] - A[None]
    # barycentric coordinates of the projection
    d00 = np.einsum("ij,ij->i", AB, AB); d01 = np.einsum("ij,ij->i", AB, AC); d11 = np.einsum("ij,ij->i", AC, AC)
    d20 = np.einsum("nmk,mk->nm", AP, AB); d21 = np.einsum("nmk,mk->nm", AP, AC)
    den = d00 * d11 - d01 * d01
    den = np.where(den != 0, den, 1.0)
    v = (d11 * d20 - d01 * d21) / den
    w = (d00 * d21 - d01 * d20) / den
    inside = (v >= 0) & (w >= 0) & (v + w <= 1)
    h = np.einsum("nmk,mk->nm", AP, N)
    plane = h * h / np.where(N2 > 0, N2, 1.0)
    e = np.minimum(np.minimum(_seg_d2(P, A, B), _seg_d2(P, B, C)), _seg_d2(P, C, A))
    return np.where(inside, plane, e)


def wall_distance(mesh: Mesh, chunk: int = 4096) -> np.ndarray:
    """Exact distance from every cell centre to the nearest SOLID_SURFACE
    face.  Cell centres follow the reference's metrics (computed here the same
    way from the face list).  O(nCells x nWallFaces): for test-sized meshes."""
    from .solver import load_library  # noqa: F401  (keeps the import graph simple)
    cc = cell_centres(mesh)
    off = np.concatenate([[0], np.cumsum(mesh.face_node_count)])
    walls = [f for f in range(mesh.n_bfaces) if mesh.bc_type[f] == SOLID]
    X = np.stack([mesh.x, mesh.y, mesh.z], 1)
    segs, tris = [], []
    for f in walls:
        nodes = mesh.face_nodes[off[f]:off[f + 1]]
        if len(nodes) <= 2:
            segs.append((nodes[0], nodes[1]))
        elif len(nodes) == 3:
            tris.append((X[nodes[0]], X[nodes[1]], X[nodes[2]]))
        else:
            ctr = X[nodes].mean(0)
            for k in range(len(nodes)):
                tris.append((X[nodes[k]], X[nodes[(k + 1) % len(nodes)]], ctr))
    out = np.full(mesh.n_cells, np.inf)
    for s in range(0, mesh.n_cells, chunk):
        P = cc[s:s + chunk]
        d2 = np.full(P.shape[0], np.inf)
        if segs:
            S = np.array(segs)
            d2 = np.minimum(d2, _seg_d2(P, X[S[:, 0]], X[S[:, 1]]).min(1))
        if tris:
            T = np.array(tris)
            d2 = np.minimum(d2, _tri_d2(P, T[:, 0], T[:, 1], T[:, 2]).min(1))
        out[s:s + chunk] = np.sqrt(d2)
    return out


def plate_wall_distance(mesh: Mesh, length: float = 1.0) -> np.ndarray:
    """Wall distance for meshes whose SOLID_SURFACE faces tile the planar
    rectangle y = 0, 0 <= x <= length (the flat-plate generators): the exact
    point-to-face minimum equals the distance to that rectangle, computed in
    closed form for every cell centre (O(nCells))."""
    cc = cell_centres(mesh)
    dx = np.maximum(np.maximum(-cc[:, 0], cc[:, 0] - length), 0.0)
    return np.sqrt(dx * dx + cc[:, 1] * cc[:, 1])


def cell_centres(mesh: Mesh) -> np.ndarray:
    """Cell centres with the reference's formulas (UnsGrid::CalcCellCenterVol2D/3D)."""
    import ctypes as C
    from .solver import load_library
    L = load_library()
    nc = mesh.n_cells
    out = np.zeros((nc, 3), np.float64)
    a = mesh.as_arrays()
    L.ofg_cell_centres.argtypes = [C.c_int, C.c_int, np.ctypeslib.ndpointer(np.float64), np.ctypeslib.ndpointer(np.float64),
                                   np.ctypeslib.ndpointer(np.float64), C.c_int, np.ctypeslib.ndpointer(np.int32),
                                   np.ctypeslib.ndpointer(np.int32), np.ctypeslib.ndpointer(np.int32),
                                   np.ctypeslib.ndpointer(np.int32), C.c_int, C.c_int,
                                   np.ctypeslib.ndpointer(np.float64)]
    rc = L.ofg_cell_centres(mesh.dim, mesh.n_nodes, a["x"], a["y"], a["z"], mesh.n_faces, a["fnc"], a["fn"], a["lc"],
                            a["rc"], nc, mesh.n_bfaces, out)
    if rc != 0:
        raise RuntimeError(f"ofg_cell_centres failed ({rc})")
    return out

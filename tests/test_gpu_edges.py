"""Malformed meshes at the C ABI on a device: an empty mesh, sizes that do not
fit, node and cell indices out of range, a degenerate face, an interior face
whose two sides are one cell, an unsupported boundary code.  Each is refused
with OFG_E_ARG and a message before any kernel runs (the checks the reference
makes on grid input, UnsGrid::ReadGridFaceTopology / NormalizeBc,
codes/geometry/src/UnsGrid.cpp:90-201, and its supported boundary codes,
codes/geometry/src/Boundary.cpp:35-54); a context whose re-upload was refused
runs nothing on the previous mesh (OFG_E_STATE), and a good mesh uploaded
afterwards steps bitwise like a fresh context."""
import ctypes as C

import numpy as np
import pytest

from oneflow_b200 import meshgen, params as P
from oneflow_b200.solver import Solver

pytestmark = pytest.mark.gpu
E_ARG, E_STATE = -1, -4


def _upload(s, mesh, sizes=None, **over):
    a = dict(s._keep)
    a.update({k: np.ascontiguousarray(v) for k, v in over.items()})
    n = dict(nn=mesh.n_nodes, nf=mesh.n_faces, nc=mesh.n_cells, nb=mesh.n_bfaces)
    n.update(sizes or {})
    return s.L.ofg_upload_mesh(s.h, n["nn"], a["x"], a["y"], a["z"], n["nf"], a["fnc"], a["fn"], a["lc"], a["rc"],
                               n["nc"], n["nb"], a["bct"], None)


def _bad_cases(mesh, a):
    nb = mesh.n_bfaces
    fn = a["fn"].copy(); fn[5] = mesh.n_nodes
    fnc = a["fnc"].copy(); fnc[nb] = 1
    lc = a["lc"].copy(); lc[nb] = mesh.n_cells
    rc = a["rc"].copy(); rc[nb] = a["lc"][nb]
    bct = a["bct"].copy(); bct[0] = 7
    return {
        "empty": dict(sizes=dict(nc=0)),
        "no faces": dict(sizes=dict(nf=0)),
        "more boundary faces than faces": dict(sizes=dict(nb=mesh.n_faces + 1)),
        "node index out of range": dict(fn=fn),
        "face with one node": dict(fnc=fnc),
        "left cell out of range": dict(lc=lc),
        "interior face with one cell on both sides": dict(rc=rc),
        "unsupported boundary code": dict(bct=bct),
    }


def test_malformed_meshes_are_refused_and_the_context_recovers():
    mesh = meshgen.bump_channel(16, 8)
    prm = P.euler_bump()
    s = Solver(mesh, prm)
    s.init_flowfield()
    s.step(2)
    for what, kw in _bad_cases(mesh, s._keep).items():
        assert _upload(s, mesh, **kw) == E_ARG, what
        assert s.L.ofg_last_error(s.h), what
        # nothing runs on the previous mesh's buffers until an upload succeeds
        assert s.L.ofg_step(s.h, 1) == E_STATE, what
        assert s.L.ofg_init_flowfield(s.h) == E_STATE, what
    assert _upload(s, mesh) == 0
    s.init_flowfield()
    s.step(5)
    ref = Solver(mesh, prm)
    ref.init_flowfield()
    ref.step(5)
    assert np.array_equal(s.state(), ref.state())

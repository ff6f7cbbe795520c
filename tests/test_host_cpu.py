"""Host-side tests that need no GPU: the C ABI library loads and exports
every entry point of include/oneflow_b200.h, refuses to run without a device
(no CPU fallback), and its host utilities (metrics, colouring) agree with
the oracle; mesh file round trips; the replica aggregation of bench.py over
two gloo ranks."""
import ctypes as C
import os
import re
import socket
import tempfile

import numpy as np
import pytest

from oneflow_b200 import colour_order, load_library, meshgen, params as P
from oneflow_b200.meshio import read_ofl, write_ofl
from oneflow_b200.walldist import cell_centres
from oracle_lib import Oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    src = open(os.path.join(ROOT, "include", "oneflow_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ofg_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = load_library()
    syms = header_symbols()
    assert len(syms) >= 25
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


def test_params_struct_matches_c_layout():
    L = load_library()
    L.ofg_params_size.restype = C.c_int
    assert L.ofg_params_size() == C.sizeof(P.OfgParams)
    d = P.OfgParams()
    L.ofg_default_params(C.byref(d))
    ours = P.defaults()
    for k in ("ischeme", "ilim", "ncfl", "visSRModel", "cfled", "max_time_ratio", "gama_ref", "prl", "ref_sa"):
        assert getattr(d, k) == pytest.approx(getattr(ours, k)), k


def test_no_cpu_fallback_without_a_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    L = load_library()
    h = C.c_void_p()
    prm = P.euler_bump()
    assert L.ofg_create(C.byref(prm), C.byref(h)) == -2   # OFG_E_CUDA


def test_bad_arguments_are_rejected():
    L = load_library()
    h = C.c_void_p()
    assert L.ofg_create(None, C.byref(h)) == -1
    prm = P.euler_bump(ischeme=7)          # not implemented scheme
    assert L.ofg_create(C.byref(prm), C.byref(h)) == -1
    prm = P.euler_bump(sweep_order=5)
    assert L.ofg_create(C.byref(prm), C.byref(h)) == -1
    prm = P.euler_bump(ivischeme=5)        # viscous face-gradient schemes are 0-4
    assert L.ofg_create(C.byref(prm), C.byref(h)) == -1


@pytest.mark.parametrize("dim", [2, 3])
def test_host_metrics_match_oracle(dim):
    mesh = meshgen.bump_channel(16, 8) if dim == 2 else meshgen.flat_plate_tets(4, 3, 2)
    prm = P.euler_bump() if dim == 2 else P.defaults(dimension=3, vismodel=0)
    o = Oracle(mesh, prm)
    cc = cell_centres(mesh)
    N = mesh.n_cells
    assert np.array_equal(cc[:, 0], o.field("xcc")[:N])
    assert np.array_equal(cc[:, 1], o.field("ycc")[:N])
    assert np.array_equal(cc[:, 2], o.field("zcc")[:N])


@pytest.mark.parametrize("name", ["plate2d_sa_roe", "plate3d_sa_roe", "hexbox_sa"])
def test_host_wall_distance_matches_the_reference(name):
    # the numpy restatement of CALC_WALL_DIST (used to write the distance files
    # the reference reads) against the distances the reference computed itself
    from golden_cases import build_walldist
    from oneflow_b200.walldist import wall_distance
    mesh, _ = build_walldist(name)
    ref = np.load(os.path.join(ROOT, "tests", "golden", f"walldist_{name}.npz"))["walldist"]
    assert np.abs(wall_distance(mesh) / ref - 1.0).max() < 1e-14


def test_colour_order_is_a_proper_colouring():
    mesh = meshgen.flat_plate_tets(6, 5, 4)
    perm, ncol = colour_order(mesh)
    nb = mesh.n_bfaces
    l, r = mesh.lc[nb:], mesh.rc[nb:]
    # greedy colouring in natural order, restated
    adj = [[] for _ in range(mesh.n_cells)]
    for a, b in zip(l, r):
        adj[a].append(b); adj[b].append(a)
    col = np.full(mesh.n_cells, -1)
    for i in range(mesh.n_cells):
        used = {col[j] for j in adj[i] if col[j] >= 0}
        col[i] = min(set(range(len(used) + 1)) - used)
    assert ncol == col.max() + 1 <= 8
    assert np.all(col[l] != col[r])                          # a proper colouring
    expect = np.concatenate([np.flatnonzero(col == k) for k in range(ncol)])
    assert np.array_equal(perm, expect)                      # colour-major, ids ascending


def test_ofl_round_trip():
    mesh = meshgen.plate_2d(8, 6)
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "m.ofl")
        write_ofl(mesh, p)
        m2 = read_ofl(p, dim=2)
    for k in ("x", "y", "z", "face_node_count", "face_nodes", "lc", "rc", "bc_type"):
        assert np.array_equal(getattr(mesh, k), getattr(m2, k)), k
    assert (m2.n_cells, m2.n_bfaces) == (mesh.n_cells, mesh.n_bfaces)


def _replica_worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms = [120.0, 150.0][rank]                      # per-rank device time of the timed steps
    total_ms, value = bench.replica_aggregate(ms, cells=1000, steps=10, world=world, dist=dist)
    out[rank] = (total_ms, value)
    dist.barrier()
    dist.destroy_process_group()


def test_replica_aggregation_two_gloo_ranks():
    import sys
    import torch.multiprocessing as mp
    sys.path.insert(0, ROOT)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_replica_worker, args=(2, port, out), nprocs=2, join=True)
    # max over ranks, whole-job throughput = all ranks' cell-iterations / that time
    for r in (0, 1):
        assert out[r][0] == 150.0
        assert out[r][1] == pytest.approx(2 * 1000 * 10 / 0.150)


def test_rcm_order_is_a_permutation_and_restores_locality():
    # a randomly shuffled bump mesh: reverse Cuthill-McKee brings the largest
    # cell-id gap across an interior face back below the generator's own
    import numpy as np
    from oneflow_b200 import meshgen, rcm_order
    m = meshgen.bump_channel(64, 32)
    shuffled = m.renumber_cells(np.random.default_rng(7).permutation(m.n_cells))

    def bandwidth(mm):
        nb = mm.n_bfaces
        return int(np.abs(mm.lc[nb:] - mm.rc[nb:]).max())

    p = rcm_order(shuffled)
    assert sorted(p.tolist()) == list(range(m.n_cells))
    assert np.array_equal(p, rcm_order(shuffled))          # deterministic
    r = shuffled.renumber_cells(p).sort_faces()
    assert bandwidth(shuffled) > 50 * bandwidth(r)
    assert bandwidth(r) <= bandwidth(m)
    # sort_faces keeps every face with its nodes and cells, boundary faces first
    assert r.n_bfaces == m.n_bfaces and sorted(r.bc_type.tolist()) == sorted(m.bc_type.tolist())
    assert np.all(r.rc[:r.n_bfaces] < 0) and np.all(r.rc[r.n_bfaces:] >= 0)


def test_rcm_order_rejects_bad_arguments():
    import ctypes as C
    import numpy as np
    from oneflow_b200.solver import load_library
    L = load_library()
    lc = np.array([0, 0, 1], np.int32); rc = np.array([-1, 1, 5], np.int32); perm = np.zeros(2, np.int32)
    assert L.ofg_rcm_order(2, 3, -1, lc, rc, perm) == -1      # negative boundary-face count
    assert L.ofg_rcm_order(2, 3, 1, lc, rc, perm) == -1       # interior face to a cell out of range
    assert L.ofg_colour_order(2, 3, -1, lc, rc, perm) == -1


def test_swept_wing_mesh_is_closed_and_classified():
    # every cell's outward face-area vectors sum to zero, every volume is
    # positive, and the boundary faces are wall (wing and tip), symmetry (root)
    # and far field, in the counts the construction gives
    import numpy as np
    from oneflow_b200 import meshgen
    m = meshgen.swept_wing_hybrid(n_around=32, n_hex=4, n_tet=4, nz_wing=6, nz_tip=3)
    P3 = np.stack([m.x, m.y, m.z], 1)
    off = np.concatenate([[0], np.cumsum(m.face_node_count)])
    A = np.zeros((m.n_faces, 3)); C = np.zeros((m.n_faces, 3))
    for k in (3, 4):
        sel = np.nonzero(m.face_node_count == k)[0]
        pts = P3[m.face_nodes[off[sel][:, None] + np.arange(k)[None, :]]]
        c = pts.mean(1)
        A[sel] = sum(0.5 * np.cross(pts[:, j] - c, pts[:, (j + 1) % k] - c) for j in range(k))
        C[sel] = c
    inn = m.rc >= 0
    acc = np.zeros((m.n_cells, 3)); vol = np.zeros(m.n_cells)
    np.add.at(acc, m.lc, A); np.add.at(acc, m.rc[inn], -A[inn])
    fv = np.einsum("ij,ij->i", C, A) / 3.0
    np.add.at(vol, m.lc, fv); np.add.at(vol, m.rc[inn], -fv[inn])
    assert np.abs(acc).max() < 1e-12 and vol.min() > 0.0
    assert np.all(m.rc[:m.n_bfaces] < 0) and np.all(m.rc[m.n_bfaces:] >= 0)
    counts = np.bincount(m.bc_type, minlength=7)
    n = 32
    # the root plane: the hexahedra's quadrilaterals and two triangles per split hexahedron
    assert counts[3] == n * 4 + n * 4 * 2
    # wall faces: the wing's quadrilaterals (n per slab) and the tip cap (n / 2 cells)
    assert counts[2] == n * 6 + (n // 2)
    assert counts[4] > 0 and counts[1] == counts[5] == counts[6] == 0


@pytest.mark.parametrize("m,t,y1,quads", [(0.06, 0.08, 2e-3, 0), (0.0, 0.18, 2e-3, 0), (0.06, 0.08, 8.6e-6, 24),
                                          (0.03, 0.12, 1e-5, 24)])
def test_naca_ogrid_has_no_folded_cells(m, t, y1, quads):
    # node k * n + i is point i of layer k: every grid quadrilateral between
    # two layers keeps the orientation of the section loop (a fold behind the
    # trailing edge of thin cambered sections inverted some, and the cells
    # there overlapped), and the cells tile the ring between section and circle
    n, K = 96, 48
    msh = meshgen.naca_ogrid(m, 0.4, t, n, K, n_quad_layers=quads, y1=y1, radius=20.0)
    x, y = msh.x.reshape(K + 1, n), msh.y.reshape(K + 1, n)
    xa, ya, xd, yd = x[:-1], y[:-1], x[1:], y[1:]
    xb, yb, xc, yc = np.roll(xa, -1, 1), np.roll(ya, -1, 1), np.roll(xd, -1, 1), np.roll(yd, -1, 1)
    area = 0.5 * ((xa * yb - xb * ya) + (xb * yc - xc * yb) + (xc * yd - xd * yc) + (xd * ya - xa * yd))
    assert np.all(area < 0) or np.all(area > 0)
    ring = lambda k: 0.5 * abs(np.sum(x[k] * np.roll(y[k], -1) - np.roll(x[k], -1) * y[k]))
    assert abs(np.abs(area).sum() - (ring(K) - ring(0))) < 1e-9 * ring(K)


def test_airfoil_shape_features():
    # the 16 shape inputs of the airfoil warm-start family: upper and lower
    # surface heights at eight chord stations; symmetric sections give
    # mirror-image ordinates equal to the thickness polynomial, camber shifts
    # both by the camber line, and they lie on the mesh generator's section
    from oneflow_b200 import warmstart
    xs = np.array(warmstart.AIRFOIL_STATIONS)
    o = warmstart.naca4_ordinates(0.0, 0.4, 0.12, xs)
    yt = 5 * 0.12 * (0.2969 * np.sqrt(xs) - 0.1260 * xs - 0.3516 * xs ** 2 + 0.2843 * xs ** 3 - 0.1036 * xs ** 4)
    assert o.shape == (16,) and np.allclose(o[:8], yt, rtol=0, atol=1e-15) and np.allclose(o[8:], -yt, atol=1e-15)
    c = warmstart.naca4_ordinates(0.04, 0.4, 0.12, xs)
    assert np.all(c[:8] > c[8:]) and abs(c[4] + c[12] - 2 * 0.04) < 1e-12   # camber line at p = 0.4 is m
    S = meshgen.naca4_surface(0.0, 0.4, 0.12, 200)
    up = S[S[:, 1] > 0]
    i = np.argsort(up[:, 0])
    assert np.allclose(np.interp(xs, up[i, 0], up[i, 1]), o[:8], atol=2e-4)
    assert len(warmstart.AirfoilFamily.feature_names) == 22

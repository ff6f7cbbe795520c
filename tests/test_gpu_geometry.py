"""Mesh metrics and wall distance computed on the GPU at ofg_upload_mesh /
ofg_calc_wall_dist: metrics bitwise equal to the oracle's restatement of
UnsGrid::CalcMetrics (which the reference pins); wall distance against the
distances the reference computed itself (CALC_WALL_DIST, ireadwdst = 0;
tests/golden/walldist_*.npz)."""
import os

import numpy as np
import pytest

from oneflow_b200 import meshgen, params as P
from oneflow_b200.solver import TURB_SOLVER, Solver
from oneflow_b200.walldist import plate_wall_distance
from golden_cases import WALLDIST_CASES, build, build_walldist
from oracle_lib import Oracle

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))

CELL_FIELDS = ("xcc", "ycc", "zcc", "vol")
FACE_FIELDS = ("area", "xfn", "yfn", "zfn", "xfc", "yfc", "zfc")


def meshes():
    return {
        "bump_triangles": (meshgen.bump_channel(32, 16), P.euler_bump()),
        "plate_quads": (meshgen.plate_2d(24, 16), P.defaults(ischeme=12, ilim=0, vismodel=1)),
        "plate_tets": (meshgen.flat_plate_tets(8, 6, 4, ratio=1.3), P.defaults(dimension=3)),
        "bump_box_hexes": (meshgen.bump_box_hexes(), P.defaults(dimension=3)),
    }


@pytest.mark.parametrize("name", list(meshes()))
def test_gpu_metrics_bitwise(name):
    mesh, prm = meshes()[name]
    g = Solver(mesh, prm)
    g.init_flowfield()
    o = Oracle(mesh, prm)
    nT, nF = mesh.n_cells + mesh.n_bfaces, mesh.n_faces
    for f in CELL_FIELDS:
        assert np.array_equal(g.field(f)[:nT], o.field(f)[:nT]), f
    for f in FACE_FIELDS:
        assert np.array_equal(g.field(f)[:nF], o.field(f)[:nF]), f


@pytest.mark.parametrize("name", WALLDIST_CASES)
def test_gpu_wall_distance_matches_the_reference(name):
    mesh, prm = build_walldist(name)      # no wall distance supplied: computed on the GPU
    g = Solver(mesh, prm)
    g.init_flowfield()
    N = mesh.n_cells
    wd = g.field("walldist")[:N]
    ref = np.load(os.path.join(HERE, "golden", f"walldist_{name}.npz"))["walldist"]
    # the same exact point-face distance, evaluated in another order: a few ulps
    assert np.abs(wd / ref - 1.0).max() < 1e-14
    # recomputing it on the GPU gives the same bits
    g.calc_wall_dist()
    assert np.array_equal(g.field("walldist")[:N], wd)


def test_wall_distance_of_a_larger_plate_matches_the_closed_form():
    # 28,800 tets, 2,560 wall triangles: the tile ordering prunes most of them
    mesh = meshgen.flat_plate_tets(40, 12, 10)
    N = mesh.n_cells
    g = Solver(mesh, P.defaults(dimension=3, vismodel=3, ischeme=1, ilim=0))
    g.init_flowfield()
    wd = g.field("walldist")[:N]
    cf = plate_wall_distance(mesh)
    assert np.abs(wd - cf).max() <= 1e-12 * cf.max()


def test_sa_solve_with_the_gpu_wall_distance():
    # the SA plate golden case (reference run with a supplied distance, which
    # equals the reference's own to the bit on this mesh) solved with the
    # distance computed on the GPU
    mesh, prm, steps = build("plate2d_sa_roe")
    mesh.wall_dist = None
    g = Solver(mesh, prm)
    g.init_flowfield()
    g.step(steps)
    gold = np.load(os.path.join(HERE, "golden", "plate2d_sa_roe.npz"))
    N = mesh.n_cells
    q = g.state()
    assert np.abs(q[:, :N] - gold["q"][:, :N]).max() / np.abs(gold["q"][:, :N]).max() < 1e-9
    t = g.state(TURB_SOLVER)[:N]
    assert np.linalg.norm(t - gold["turbq"][:N]) / np.linalg.norm(gold["turbq"][:N]) < 1e-5

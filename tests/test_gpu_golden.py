"""The GPU path against the reference's own results (tests/golden/*.npz, made
by running the reference built from its sources on the same seeded meshes):
every golden case -- 2-D and 3-D, triangles, quadrilaterals, tetrahedra and a
hexahedron/prism mesh; Roe and SLAU2; first order, Barth, Venkatakrishnan;
Euler, laminar and SA -- run through the C ABI on the FP64 path."""
import os

import numpy as np
import pytest

from oneflow_b200 import params as P
from oneflow_b200.solver import TURB_SOLVER, Solver
from golden_cases import CASES, build
from oracle_lib import Oracle

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("name", list(CASES))
def test_gpu_matches_the_reference_fixture(name):
    mesh, prm, steps = build(name)
    g = Solver(mesh, prm)
    g.init_flowfield()
    g.step(steps)
    gold = np.load(os.path.join(HERE, "golden", f"{name}.npz"))
    N = mesh.n_cells
    sa = "turbq" in gold
    q, qg = g.state(), gold["q"]
    # FP64 path: round-off (SA: the reference's far-field nu~ flip carries
    # round-off into the state)
    assert np.abs(q[:, :N] - qg[:, :N]).max() / np.abs(qg[:, :N]).max() < (1e-9 if sa else 1e-12)
    # residual history as the reference printed it (6 significant digits)
    h, hg = g.res_history(), gold["reshist"]
    assert np.all(np.abs(h - hg) <= 5.01e-6 * np.abs(hg) + 1e-12)
    if sa:
        t, tg = g.state(TURB_SOLVER)[:N], gold["turbq"][:N]
        assert np.linalg.norm(t - tg) / np.linalg.norm(tg) < 1e-5


@pytest.mark.parametrize("name", ["mixed3d_slau2_gg_barth_sa", "plate2d_laminar_roe_inflow_extrap",
                                  "plate2d_sa_roe_inflow_extrap", "plate2d_laminar_roe_isowall"])
def test_iteration_by_iteration_against_the_oracle(name):
    # hexahedra + prisms, SLAU2, Green-Gauss, Barth, SA; and the inflow,
    # extrapolation and isothermal-wall boundary conditions: the state, time
    # step and residual of each of the first iterations against the oracle
    mesh, prm, _ = build(name)
    g = Solver(mesh, prm)
    g.init_flowfield()
    o = Oracle(mesh, prm)
    o.init()
    N = mesh.n_cells
    for it in range(3):
        g.step(1)
        o.step(1)
        q, qo = g.state(), o.q()
        assert np.abs(q - qo).max() / np.abs(qo).max() < 1e-12, it
        nT = N + mesh.n_bfaces
        # the time step and the residual of the iteration (interior cells of
        # each equation); the limiter itself is not compared: on a nearly
        # uniform start it is a discontinuous function of round-off-sized
        # gradients, and the iterates above agree all the same
        for f in ("timestep", "res"):
            a, b = g.field(f).reshape(-1, nT)[:, :N], o.field(f).reshape(-1, nT)[:, :N]
            assert np.abs(a - b).max() <= 1e-10 * max(np.abs(b).max(), 1e-30), (it, f)


# the FP32 face path (its own viscous face-gradient code) against FP64
@pytest.mark.parametrize("name", ["mixed3d_slau2_gg_barth_sa", "plate2d_laminar_roe_vistest",
                                  "plate2d_laminar_roe_visnew1", "plate2d_laminar_roe_visnew2",
                                  "mixed3d_laminar_vistest"])
def test_fp32_face_path_tracks_fp64(name):
    mesh, prm, steps = build(name)
    a = Solver(mesh, prm); a.init_flowfield(); a.step(steps)
    prm1 = P.defaults(**{**P.to_dict(prm), "precision": 1})
    b = Solver(mesh, prm1); b.init_flowfield(); b.step(steps)
    qa, qb = a.state(), b.state()
    assert np.abs(qb - qa).max() / np.abs(qa).max() < 1e-4


def test_multi_stage_task_by_task_equals_the_fused_iteration():
    # TimeIntegral::RungeKutta through the task entry points, stage by stage,
    # against ofg_step's captured iteration: bitwise
    mesh, prm, _ = build("bump_euler_rk3")
    a = Solver(mesh, prm); a.init_flowfield(); a.step(4)
    b = Solver(mesh, prm); b.init_flowfield()
    for it in range(4):
        b.set_outer_step(it + 1)
        b.task("CALC_TIME_STEP")
        for k in range(prm.rk_stage):
            b.task("LOAD_RESIDUALS")
            b.task("UPDATE_RESIDUALS")
            b.calc_lhs(1.0 / (k + 1))
            b.task("UPDATE_FLOWFIELD_LUSGS")
            b.task("CALC_BOUNDARY")
    assert np.array_equal(a.state(), b.state())


@pytest.mark.parametrize("name", ["bump_euler_roe_venkat", "plate2d_sa_roe"])
def test_residual_max_and_its_cell(name):
    # ResidualTask's resmax record: the largest |res| per equation and the
    # first cell (in cell order) that holds it
    mesh, prm, _ = build(name)
    g = Solver(mesh, prm)
    g.init_flowfield()
    g.step(3)
    N, nT = mesh.n_cells, mesh.n_cells + mesh.n_bfaces
    r = np.abs(g.field("res").reshape(5, -1)[:, :N])
    v, i = g.residual_max()
    assert np.array_equal(v, r.max(1)) and np.array_equal(i, r.argmax(1))
    if prm.vismodel >= 3:
        t = np.abs(g.field("turbres", TURB_SOLVER)[:N])
        v, i = g.residual_max(TURB_SOLVER)
        assert v[0] == t.max() and i[0] == t.argmax()

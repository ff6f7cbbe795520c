"""GPU parity of the Spalart-Allmaras solver (TURB_SOLVER tasks) against the
CPU oracle on a seeded 2-D turbulent flat plate.  FP64 path: round-off
agreement (relative tolerances written per check)."""
import numpy as np
import pytest

from oneflow_b200 import meshgen, params as P
from oneflow_b200.solver import LUSGS_SEQUENCE, TURB_SOLVER, Solver
from oneflow_b200.walldist import wall_distance
from oracle_lib import Oracle

pytestmark = pytest.mark.gpu


def rel(a, b, floor=1e-300):
    a = np.asarray(a); b = np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), floor))


def sa_case(**kw):
    m = meshgen.plate_2d(32, 24, y1=1e-5, ratio=1.25)
    m.wall_dist = wall_distance(m)
    base = dict(ischeme=1, ilim=0, mach_ref=0.2, reynolds=5e6, vismodel=3)
    base.update(kw)
    return m, P.defaults(**base)


@pytest.mark.parametrize("kw", [dict(), dict(ischeme=12, ilim=2, vencat_coef=0.05)])
def test_sa_task_by_task_fp64(kw):
    mesh, prm = sa_case(**kw)
    N = mesh.n_cells
    o = Oracle(mesh, prm); o.init()
    g = Solver(mesh, prm); g.init_flowfield()
    assert rel(g.state(TURB_SOLVER), o.field("turbq")) < 1e-15
    for it in range(3):
        o.task("NEXT_STEP")
        g.set_outer_step(it + 1)
        for t in LUSGS_SEQUENCE:
            o.task(t); g.task(t)
        assert rel(g.state(), o.q()) < 1e-12, (it, "ns q")
        for t in LUSGS_SEQUENCE:
            o.task("TURB:" + t); g.task(t, TURB_SOLVER)
            if t == "UPDATE_RESIDUALS":
                assert rel(g.field("turbres")[:N], o.field("turbres")[:N], 1e-30) < 1e-10, (it, "turbres")
                assert rel(g.field("turbimpsr")[:N], o.field("turbimpsr")[:N]) < 1e-12, (it, "turbimpsr")
            if t.startswith("LUSGS"):
                assert rel(g.field("turbdq")[:N], o.field("turbdq")[:N], 1e-30) < 1e-10, (it, t)
        assert rel(g.state(TURB_SOLVER), o.field("turbq")) < 1e-12, (it, "nut")
        assert rel(g.field("vist")[:N], o.field("vist")[:N], 1e-30) < 1e-12, (it, "vist")


def test_sa_fused_steps_fp64():
    mesh, prm = sa_case()
    o = Oracle(mesh, prm); o.init(); o.step(30)
    g = Solver(mesh, prm); g.init_flowfield(); g.step(30)
    assert rel(g.state(), o.q()) < 1e-10
    assert rel(g.state(TURB_SOLVER), o.field("turbq")) < 1e-8
    ht, ho = g.field("turbreshist"), o.field("turbreshist")
    assert ht.shape == ho.shape and np.abs(ht - ho).max() / ho.max() < 1e-6


def test_sa_mixed_precision_tracks_fp64():
    mesh, prm = sa_case()
    prm32 = P.defaults(**{**P.to_dict(prm), "precision": 1})
    a = Solver(mesh, prm); a.init_flowfield(); a.step(30)
    b = Solver(mesh, prm32); b.init_flowfield(); b.step(30)
    assert rel(b.state(), a.state()) < 1e-4
    assert rel(b.state(TURB_SOLVER), a.state(TURB_SOLVER)) < 1e-2


def test_sa_residual_norm_matches_the_residual_field():
    m, prm = sa_case()
    g = Solver(m, prm); g.init_flowfield(); g.step(3)
    g.task("UPDATE_RESIDUALS", TURB_SOLVER)
    N = m.n_cells
    r = g.field("turbres", TURB_SOLVER)[:N]
    assert np.allclose(g.residual_norms(TURB_SOLVER), [np.sqrt((r * r).mean())], rtol=1e-12, atol=0)

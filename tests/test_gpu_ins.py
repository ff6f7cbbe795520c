"""GPU tests of the incompressible solver (ofg_ins_*, oneflow_b200/csrc/ofg_ins.cu)
against the oracle (oracle/src/oracle_ins.h, bitwise the reference) and the
reference's own cavity runs (tests/golden/ins_*.npz).

Tolerance: everything but the GMRES inner products runs the reference's
operations in its order; the inner products are summed in blocks, so the
Krylov coefficients differ from the reference's in the last bits and the
fields by round-off amplified by the solves -- held to 1e-9 of each field's
magnitude after the cases' inner iterations, with the same GMRES iteration
counts."""
import os

import numpy as np
import pytest

from oneflow_b200 import meshgen, params as P
from oneflow_b200.solver import Incompressible, OfgError
from golden_cases import INS_CASES, build_ins
from oracle_lib import InsOracle

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
TOL = 1e-9


def _close(a, b, what):
    scale = max(np.abs(b).max(), 1e-300)
    err = np.abs(a - b).max() / scale
    assert err < TOL, (what, err)


@pytest.mark.parametrize("name", list(INS_CASES))
def test_gpu_ins_matches_the_reference_fixture(name):
    mesh, prm, wall, steps = build_ins(name)
    g = Incompressible(mesh, prm, wall)
    assert g.run(steps) == steps
    gold = np.load(os.path.join(HERE, "golden", f"ins_{name}.npz"))
    q = g.q()
    for e in range(5):
        _close(q[e], gold["q"][e], f"q[{e}]")
    gx = g.field("dqdx").reshape(5, -1)
    for e in range(1, 5):
        _close(gx[e], gold["dqdx"][e], f"dqdx[{e}]")
    st = g.stats()
    printed = gold["remax_printed"][-1]
    for k in range(4):
        assert abs(st["remax"][k] - printed[k]) <= 5e-6 * max(abs(printed[k]), 1e-30) + 1e-12, (k, st["remax"])


@pytest.mark.parametrize("name", list(INS_CASES))
def test_gpu_ins_tracks_the_oracle_step_by_step(name):
    mesh, prm, wall, steps = build_ins(name)
    g = Incompressible(mesh, prm, wall)
    o = InsOracle(mesh, prm, wall)
    for it in range(steps):
        g.update_residuals()
        o.run(it + 1)
        sg, so = g.stats(), o.stats()
        # same Krylov dimensions in every solve
        assert list(sg["gmres_iters"]) == list(so["gmres_iters"]), (it, sg, so)
        qg, qo = g.q(), o.q()
        for e in range(5):
            _close(qg[e], qo[e], f"step {it} q[{e}]")
        for k in ("pp", "uc", "vc", "spc"):
            _close(g.field(k), o.field(k), f"step {it} {k}")
        np.testing.assert_allclose(sg["remax"], so["remax"], rtol=1e-8, atol=1e-14)


def test_gpu_ins_first_step_assembly_is_bitwise_the_oracle():
    # before any solve result enters them, the assembled coefficients round
    # exactly like the reference's: the momentum diagonal and the first
    # Green-Gauss gradients
    mesh, prm, wall, _ = build_ins("cavity2d_tri_jitter")
    g = Incompressible(mesh, prm, wall)
    o = InsOracle(mesh, prm, wall)
    g.update_residuals()
    o.run(1)
    for k in ("dqdx", "dqdy"):
        a, b = g.field(k).reshape(5, -1), o.field(k).reshape(5, -1)
        np.testing.assert_array_equal(a, b)


def test_gpu_ins_run_stops_at_the_inner_limit():
    mesh, prm, wall, _ = build_ins("cavity2d_quad")
    g = Incompressible(mesh, prm, wall)
    assert g.run(2) == 2
    assert g.run(2) == 0
    assert g.run(4) == 2
    assert g.stats()["inner"] == 4
    t = g.timing()
    assert t["ms"] > 0 and t["gmres_iters"] > 0
    g.init_flowfield()
    assert g.stats()["inner"] == 0 and g.run(1) == 1


def test_gpu_ins_refuses_meshes_outside_the_reference_scope():
    with pytest.raises(OfgError):
        Incompressible(meshgen.bump_channel(8, 4), P.defaults(vismodel=1))
    cav = meshgen.lid_cavity_2d(4)
    with pytest.raises(OfgError):
        Incompressible(cav, P.defaults(vismodel=0), meshgen.lid_velocity(cav))


def test_gpu_ins_larger_cavity_keeps_the_oracle_to_round_off():
    # a 64 x 64 cavity: pressure solves of a few hundred Krylov steps
    mesh = meshgen.lid_cavity_2d(64, jitter=0.1)
    prm = P.defaults(vismodel=1, reynolds=1000.0, mach_ref=0.1)
    wall = meshgen.lid_velocity(mesh)
    g = Incompressible(mesh, prm, wall)
    o = InsOracle(mesh, prm, wall)
    g.run(3)
    o.run(3)
    assert list(g.stats()["gmres_iters"]) == list(o.stats()["gmres_iters"])
    qg, qo = g.q(), o.q()
    for e in range(5):
        _close(qg[e], qo[e], f"q[{e}]")

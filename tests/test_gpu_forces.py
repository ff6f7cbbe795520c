"""GPU aerodynamic forces (ofg_forces) against the CPU oracle and against the
reference's own force routine (the golden fixtures): FP64 path to round-off;
the FP32-face path against the FP64 path on converged solutions."""
import json
import os

import numpy as np
import pytest

from oneflow_b200 import meshgen, params as P
from oneflow_b200.solver import Solver
from golden_cases import CASES, build
from oracle_lib import Oracle

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("name", [n for n in CASES if "colour" not in n])
def test_gpu_forces_match_oracle_and_reference(name):
    mesh, prm, steps = build(name)
    o = Oracle(mesh, prm); o.init(); o.step(steps)
    g = Solver(mesh, prm); g.init_flowfield(); g.step(steps)
    fo, fg = o.forces(1.0), g.forces(1.0)
    ref = np.load(os.path.join(HERE, "golden", f"{name}.npz"))["forces"]
    sa = prm.vismodel >= 3
    # FP64 path against the oracle: the same arithmetic, summed in another order
    assert rel(fg, fo) < (1e-7 if sa else 1e-11)
    # against the reference's own force routine on its own final state
    assert rel(fg, ref) < (1e-6 if sa else 1e-10)


def test_forces_are_zero_without_walls():
    mesh = meshgen.bump_channel(16, 8)
    prm = P.euler_bump()
    bct = mesh.bc_type.copy()
    mesh.bc_type[:] = np.where(bct == 2, 3, bct)   # walls -> symmetry planes
    g = Solver(mesh, prm); g.init_flowfield(); g.step(2)
    assert np.array_equal(g.forces(1.0), np.zeros(13))


@pytest.mark.parametrize("kw,steps", [({}, 3000), (dict(ilim=2, vencat_coef=0.05), 4000)],
                         ids=["first_order", "venkat"])
def test_converged_forces_fp64_and_fp32_face_paths(kw, steps):
    # 2-D Euler bump, Roe, CFL 5, run to convergence on both paths.  The FP64
    # path converges to round-off.  The FP32-face path forms its face states,
    # central flux and gradient differences in FP64, so no FP32 rounding of the
    # large pressure terms sets a floor: it reaches a 1e-8 drop of the density
    # residual (measured 1.2e-8 / 1.8e-8 after 3000 / 4000 steps; an all-FP32
    # face flux stalls near 6e-6).  Its geometry is face-local (FP32 offsets
    # formed in FP64, FP64 normals in the central flux), so its converged state
    # solves the same discrete equations as the FP64 path's up to FP32 rounding
    # of the small terms (measured: fields 5e-10 - 1e-9 relative L2, forces
    # 2.5e-8 / 8.9e-8 relative; the tolerance is the 1e-6 force target).
    mesh = meshgen.bump_channel(32, 16)
    a = Solver(mesh, P.euler_bump(**kw)); a.init_flowfield(); a.step(steps)
    b = Solver(mesh, P.euler_bump(precision=1, **kw)); b.init_flowfield(); b.step(steps)
    ha, hb = a.res_history(), b.res_history()
    assert ha[-1, 0] / ha[0, 0] < 1e-12
    assert hb[-1, 0] / hb[0, 0] < 5e-8
    fa, fb = a.forces(1.0), b.forces(1.0)
    assert rel(fb[[0, 1, 9, 10]], fa[[0, 1, 9, 10]]) < 1e-6, (fa, fb)
    qa, qb = a.state(), b.state()
    for e in (0, 4):   # density and pressure fields, well inside the 1e-5 field-L2 tolerance
        assert np.linalg.norm(qb[e] - qa[e]) / np.linalg.norm(qa[e]) < 1e-7

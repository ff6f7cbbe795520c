"""The positivity fix of UPDATE_FLOWFIELD (NsUpdate::CalcFlowField's
WeekSolutionFix and the neighbour average of SolutionFix,
codes/ns/src/NsUpdate.cpp:40-67,192-217) forced on the GPU: a state whose
velocities are perturbed at random (seeded) makes the update drive density
or pressure negative in some tens of cells per iteration, and the GPU's FP64
path must repair them exactly as the oracle does (k_solution_fix replays the
reference's in-place order)."""
import numpy as np
import pytest

from oneflow_b200 import meshgen, params as P
from oneflow_b200.solver import Solver
from oracle_lib import Oracle

pytestmark = pytest.mark.gpu


def _violent_state(mesh, o):
    q = o.q().copy()
    rng = np.random.default_rng(7)
    n = mesh.n_cells
    q[1:4, :n] += rng.normal(0.0, 1.0, (3, n))
    q[4, :n] *= rng.uniform(0.001, 1.0, n)
    return q


@pytest.mark.parametrize("ilim", [-1, 2])
def test_gpu_repairs_negative_states_like_the_oracle(ilim):
    mesh = meshgen.bump_channel(32, 16)
    prm = P.euler_bump(cflst=5.0, cfled=5.0, ilim=ilim)
    o = Oracle(mesh, prm)
    o.init()
    q0 = _violent_state(mesh, o)
    o.set_q(q0)
    g = Solver(mesh, prm)
    g.init_flowfield()
    g.upload_state(q0)
    for it in range(3):
        o.step(1)
        g.step(1)
        qo, qg = o.q(), g.state()
        err = np.abs(qg - qo).max() / np.abs(qo).max()
        assert err < 1e-10, (it, err)
    assert o.field("nfixes")[0] > 10   # the fix did run, in the oracle and so on the GPU

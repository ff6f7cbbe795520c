"""The least-squares gradient on the GPU (igrad = 2, no reference
implementation) pinned analytically: a linear state's gradient is reproduced
exactly in every cell whose faces are all interior -- to round-off on the
FP64 path, to FP32 rounding on the mixed path (its gradients are FP32, formed
from FP64 neighbour differences)."""
import numpy as np
import pytest

from oneflow_b200 import meshgen, params as P
from oneflow_b200.solver import Solver

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,tol", [(0, 1e-12), (1, 1e-5)])
@pytest.mark.parametrize("name", ["tri2d", "mixed3d"])
def test_least_squares_gradient_is_exact_for_linear_fields(name, precision, tol):
    m, dim = (meshgen.bump_channel(32, 16), 2) if name == "tri2d" else (meshgen.bump_box_mixed(8, 6, 4), 3)
    s = Solver(m, P.defaults(dimension=dim, ischeme=1, igrad=2, ilim=0, vismodel=0, mach_ref=0.5,
                             precision=precision))
    s.init_flowfield()
    N, nT = m.n_cells, m.n_cells + m.n_bfaces
    X = np.stack([s.field("xcc"), s.field("ycc"), s.field("zcc")])
    g = np.array([[0.01, -0.02, 0.03], [0.1, 0.05, -0.02], [-0.04, 0.02, 0.01], [0.02, -0.01, 0.03], [0.3, -0.1, 0.2]])
    if dim == 2:
        g[:, 2] = 0.0
        g[3] = 0.0
    base = np.array([1.0, 0.5, 0.1, 0.0, 1.0 / (1.4 * 0.25)])
    s.upload_state(base[:, None] + g @ X)
    s.task("UPDATE_RESIDUALS")
    G = np.stack([s.field(f).reshape(5, nT)[:, :N] for f in ("dqdx", "dqdy", "dqdz")], 2)
    inner = np.ones(N, bool)
    inner[m.lc[:m.n_bfaces]] = False
    assert inner.sum() > N // 4
    err = np.abs(G[:, inner] - g[:, None, :]).max() / np.abs(g).max()
    assert err < tol, err
    s.close()

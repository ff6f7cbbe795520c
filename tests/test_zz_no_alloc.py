"""GPU test of ofg_residual_rms_noalloc, the allocation-free residual RMS
(static device scratch): two calls in a row must agree with the context's
ofg_residual_norms and with each other, and oversized requests are refused
with OFG_E_SIZE.  Kept in its own file, collected last, so it runs both
alone and after every other test of the session."""
import ctypes as C

import numpy as np
import pytest

from oneflow_b200 import meshgen, params as P
from oneflow_b200.solver import Solver, load_library

pytestmark = pytest.mark.gpu

OFG_E_ARG, OFG_E_SIZE = -1, -7


def _bind():
    L = load_library()
    f = L.ofg_residual_rms_noalloc
    f.argtypes = [C.c_void_p, C.c_int64, C.c_int, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return f


def test_noalloc_rms_matches_residual_norms_on_two_calls():
    import torch
    f = _bind()
    mesh = meshgen.bump_channel(64, 32)
    prm = P.euler_bump(ilim=2, vencat_coef=0.05)
    s = Solver(mesh, prm)
    s.init_flowfield()
    s.step(4)
    want = s.residual_norms()
    N = mesh.n_cells
    res = s.field("res").reshape(5, -1)[:, :N]                  # [5][N] host copy of the device residual
    d_res = torch.tensor(np.ascontiguousarray(res.T), dtype=torch.float64, device="cuda")   # [N][5]
    outs = [torch.full((5,), -1.0, dtype=torch.float64, device="cuda") for _ in range(2)]
    stream = torch.cuda.current_stream().cuda_stream
    for o in outs:   # two calls in a row: the second finds the scratch re-armed by the first
        assert f(d_res.data_ptr(), N, 5, o.data_ptr(), stream) == 0
    torch.cuda.synchronize()
    a, b = outs[0].cpu().numpy(), outs[1].cpu().numpy()
    assert np.array_equal(a, b)
    assert np.allclose(a, want, rtol=1e-12, atol=0.0)


def test_noalloc_rms_refuses_requests_beyond_its_scratch():
    import torch
    f = _bind()
    x = torch.zeros((16, 9), dtype=torch.float64, device="cuda")
    o = torch.zeros(9, dtype=torch.float64, device="cuda")
    assert f(x.data_ptr(), 16, 9, o.data_ptr(), None) == OFG_E_SIZE   # 9 equations > OFG_NOALLOC_MAX_EQ
    assert f(None, 16, 5, o.data_ptr(), None) == OFG_E_ARG
    assert f(x.data_ptr(), 0, 5, o.data_ptr(), None) == OFG_E_ARG
    # a valid call still works after the refusals (nothing was left half-done)
    assert f(x.data_ptr(), 16, 8, o.data_ptr(), None) == 0
    torch.cuda.synchronize()
    assert np.array_equal(o.cpu().numpy()[:8], np.zeros(8))


@pytest.mark.parametrize("n,neq", [(1_000_003, 5), (300_001, 8), (77, 3)])
def test_noalloc_rms_matches_numpy_on_random_data(n, neq):
    # Large enough that the grid is capped (296 blocks) and every block strides
    # over more than its 256 threads; odd sizes leave a ragged last range; the
    # 8-equation case fills every partial-sum slot with nonzero values.
    import torch
    f = _bind()
    rng = np.random.default_rng(n + neq)
    x = rng.standard_normal((n, neq)) * rng.uniform(0.1, 10.0, size=neq)
    want = np.sqrt(np.mean(x * x, axis=0))
    d = torch.tensor(x, dtype=torch.float64, device="cuda")
    outs = [torch.full((neq,), -1.0, dtype=torch.float64, device="cuda") for _ in range(2)]
    stream = torch.cuda.current_stream().cuda_stream
    for o in outs:   # two full-size calls in a row on the shared scratch
        assert f(d.data_ptr(), n, neq, o.data_ptr(), stream) == 0
    torch.cuda.synchronize()
    a, b = outs[0].cpu().numpy(), outs[1].cpu().numpy()
    assert np.array_equal(a, b)
    assert np.allclose(a, want, rtol=1e-12, atol=0.0)

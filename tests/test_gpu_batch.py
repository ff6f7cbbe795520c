"""Batched solves (ofg_batch_*): independent contexts of different meshes,
models and precisions advanced by one graph launch per outer iteration give
bitwise the states and residual histories of stepping each on its own."""
import numpy as np
import pytest

from oneflow_b200 import meshgen, params as P
from oneflow_b200.solver import TURB_SOLVER, Batch, OfgError, Solver
from oneflow_b200.walldist import plate_wall_distance, wall_distance

pytestmark = pytest.mark.gpu


def cases():
    plate = meshgen.plate_2d(24, 16, y1=1e-5, ratio=1.25)
    plate.wall_dist = wall_distance(plate)
    tets = meshgen.flat_plate_tets(6, 5, 3, ratio=1.3)
    tets.wall_dist = plate_wall_distance(tets)
    out = [(meshgen.bump_channel(32, 16), P.euler_bump(ilim=2, vencat_coef=0.05)),
           (plate, P.defaults(ischeme=1, ilim=0, mach_ref=0.2, reynolds=5e6, vismodel=3, precision=1)),
           (tets, P.defaults(dimension=3, ischeme=1, ilim=0, vismodel=3, mach_ref=0.2, reynolds=5e6))]
    for mesh, fs in meshgen.airfoil_cases(2, min_cells=2000, max_cells=6000):
        out.append((mesh, P.rans_airfoil(**fs)))
    return out


def fresh(cs):
    ss = []
    for mesh, prm in cs:
        s = Solver(mesh, prm)
        s.init_flowfield()
        ss.append(s)
    return ss


def same(a, b):
    assert np.array_equal(a.state(), b.state())
    assert np.array_equal(a.res_history(), b.res_history())
    if a.params.vismodel >= 3:
        assert np.array_equal(a.state(TURB_SOLVER), b.state(TURB_SOLVER))


def test_batch_equals_separate_solves():
    cs = cases()
    solo, batched = fresh(cs), fresh(cs)
    for s in solo:
        s.step(10)
    b = Batch(batched)
    with pytest.raises(OfgError):
        b.device_ms()                    # no step timed yet
    b.step(6)
    ms6 = b.device_ms()
    b.step(4)
    assert 0.0 < b.device_ms() and 0.0 < ms6
    for x, y in zip(solo, batched):
        same(x, y)
    b.close()


def test_batch_after_a_context_moved_on_alone():
    # one context steps on its own between batch steps (its parity no longer
    # matches the others'): the batch rebuilds its graph and stays exact
    cs = cases()[:3]
    solo, batched = fresh(cs), fresh(cs)
    b = Batch(batched)
    b.step(3)
    batched[1].step(2)
    b.step(3)
    for k, s in enumerate(solo):
        s.step(8 if k == 1 else 6)
    for x, y in zip(solo, batched):
        same(x, y)
    b.close()


def test_batch_rejects_a_repeated_context():
    mesh, prm = cases()[0]
    s = Solver(mesh, prm)
    s.init_flowfield()
    with pytest.raises(OfgError):
        Batch([s, s])

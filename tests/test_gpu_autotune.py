"""The autotuner (ofg_autotune): candidate launch shapes of the mixed path's
face pass, gradient/limiter kernel and LU-SGS level kernels timed on the
context's own mesh; the choice is a valid compiled shape, no slower than the
context's starting shape, cached per mesh, and does not change the results
beyond FP32 rounding."""
import numpy as np
import pytest

from oneflow_b200 import meshgen, params as P
from oneflow_b200.solver import OfgError, Solver, TURB_SOLVER
from oneflow_b200.walldist import plate_wall_distance

pytestmark = pytest.mark.gpu

VALID = {"face_min_blocks": {2, 3, 4, 5}, "face_block": {64, 128}, "grad_min_blocks": {4, 6, 8}, "grad_block": {64, 128},
         "sweep_min_blocks": {6, 8, 10}, "sweep_block": {64, 128}}


def plate():
    m = meshgen.flat_plate_tets(24, 12, 8)
    m.wall_dist = plate_wall_distance(m)
    return m


def test_autotune_picks_a_valid_shape_and_caches_it():
    m = plate()
    prm = P.rans_plate(sweep_order=1)
    a = Solver(m, prm); a.init_flowfield(); a.step(3)
    t = a.autotune(reps=3)
    for k, allowed in VALID.items():
        assert t[k] in allowed, (k, t[k])
    assert 0.0 < t["ms_tuned"] <= t["ms_default"]
    b = Solver(m, prm); b.init_flowfield()
    tb = b.autotune()            # same mesh and options: the cached choice, no timing
    assert {k: tb[k] for k in VALID} == {k: t[k] for k in VALID}


def test_tuned_shapes_give_the_same_solution():
    m = plate()
    prm = P.rans_plate(sweep_order=1)
    a = Solver(m, prm); a.init_flowfield(); a.step(2)
    b = Solver(m, prm); b.init_flowfield(); b.step(2)
    # every non-default shape at once
    b.set_tuning(face_min_blocks=5, face_block=64, grad_min_blocks=8, grad_block=64, sweep_min_blocks=10,
                 sweep_block=64)
    a.step(10); b.step(10)
    qa, qb = a.state(), b.state()
    assert np.abs(qb - qa).max() / np.abs(qa).max() < 1e-6
    ta, tb = a.state(TURB_SOLVER), b.state(TURB_SOLVER)
    assert np.linalg.norm(tb - ta) / np.linalg.norm(ta) < 1e-5


def test_gradient_block_size_gives_the_same_bits():
    # the gradient kernel's cells do not depend on the block size, and the
    # zone-wide Venkatakrishnan eps reduces exact minima and maxima per block
    m = meshgen.bump_channel(32, 16)
    prm = P.euler_bump(ilim=2, vencat_coef=0.05, precision=1)
    a = Solver(m, prm); a.init_flowfield()
    b = Solver(m, prm); b.init_flowfield()
    b.set_tuning(grad_block=64)
    a.step(20); b.step(20)
    assert np.array_equal(a.state(), b.state())


def test_set_tuning_rejects_shapes_that_are_not_compiled():
    s = Solver(meshgen.bump_channel(16, 8), P.euler_bump(precision=1))
    with pytest.raises(OfgError):
        s.set_tuning(face_min_blocks=7)
    with pytest.raises(OfgError):
        s.set_tuning(sweep_block=256)
    with pytest.raises(OfgError):
        s.set_tuning(grad_block=32)


def test_fp64_path_keeps_its_fixed_shapes_and_tunes_its_sweep_schedule():
    # the FP64 path's gathers keep their fixed shapes; only the sweep schedule
    # (level launches or one persistent block per sweep) is timed, and on the
    # natural order of a bump channel (dozens of small levels) the persistent
    # form is not slower by construction of the choice
    s = Solver(meshgen.bump_channel(32, 16), P.euler_bump())
    s.init_flowfield()
    t = s.autotune()
    assert (t["face_min_blocks"], t["face_block"], t["grad_min_blocks"], t["sweep_min_blocks"],
            t["sweep_block"]) == (3, 128, 6, 8, 128)
    assert t["sweep_persistent"] in (0, 1)
    assert 0.0 < t["ms_tuned"] <= t["ms_default"]


@pytest.mark.parametrize("case", ["bump_fp64_natural", "sa_plate_mixed_natural", "sa_plate_mixed_colour"])
def test_persistent_sweep_gives_the_same_bits(case):
    # one launch per sweep (a single block running every level with a block
    # barrier between levels) against one launch per level: the same
    # per-cell arithmetic in the same dependency order, so the same bits
    if case == "bump_fp64_natural":
        m, prm = meshgen.bump_channel(32, 16), P.euler_bump(ilim=2, vencat_coef=0.05)
    else:
        m = meshgen.plate_2d(32, 24, y1=1e-5, ratio=1.25)
        from oneflow_b200.walldist import wall_distance
        m.wall_dist = wall_distance(m)
        prm = P.defaults(ischeme=1, ilim=0, mach_ref=0.2, reynolds=5e6, vismodel=3, precision=1,
                         sweep_order=1 if case.endswith("colour") else 0)
    a = Solver(m, prm); a.init_flowfield()
    b = Solver(m, prm); b.init_flowfield()
    b.set_tuning(sweep_persistent=1)
    a.step(15); b.step(15)
    assert np.array_equal(a.state(), b.state())
    assert np.array_equal(a.res_history(), b.res_history())
    if prm.vismodel >= 3:
        assert np.array_equal(a.state(TURB_SOLVER), b.state(TURB_SOLVER))

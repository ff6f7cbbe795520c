"""CPU tests (no GPU) of the incompressible solver's oracle: the sequential
restatement (oracle/src/oracle_ins.h) against the reference's own runs of
its INsSolver on lid-driven cavities (tests/golden/ins_*.npz, made by
tests/golden/make_golden.py --ins-only) -- bitwise -- and its scope checks."""
import json
import os

import numpy as np
import pytest

from oneflow_b200 import meshgen, params as P
from golden_cases import INS_CASES, build_ins
from oracle_lib import InsOracle, Oracle, lib

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("name", list(INS_CASES))
def test_ins_oracle_is_bitwise_the_reference(name):
    mesh, prm, wall, steps = build_ins(name)
    gold = np.load(os.path.join(HERE, "golden", f"ins_{name}.npz"))
    assert json.loads(str(gold["params"])) == P.to_dict(prm)
    o = InsOracle(mesh, prm, wall)
    assert o.run(steps) == steps
    # same operations in the same order as the reference: equal to the last bit
    np.testing.assert_array_equal(o.q(), gold["q"])
    np.testing.assert_array_equal(o.field("dqdx").reshape(5, -1), gold["dqdx"])
    np.testing.assert_array_equal(o.field("dqdy").reshape(5, -1), gold["dqdy"])
    # the residual maxima the reference printed (6 significant digits)
    st = o.stats()
    printed = gold["remax_printed"][-1]
    for k in range(4):
        assert abs(st["remax"][k] - printed[k]) <= 5e-6 * max(abs(printed[k]), 1e-30), (k, st["remax"], printed)


def test_ins_oracle_refuses_meshes_outside_the_reference_scope():
    # a boundary type other than SOLID_SURFACE: the reference's MomPre and
    # UpdateSpeed boundary loops index past their region there
    mesh = meshgen.bump_channel(8, 4)
    o = Oracle(mesh, P.defaults(vismodel=1))
    assert not lib().oro_ins_create(o.h)
    # an inviscid model: the reference never forms the gradients its source term reads
    cav = meshgen.lid_cavity_2d(4)
    o2 = Oracle(cav, P.defaults(vismodel=0))
    assert not lib().oro_ins_create(o2.h)


def test_ins_oracle_stops_on_the_inner_step_limit_and_keeps_counting():
    mesh, prm, wall, _ = build_ins("cavity2d_quad")
    o = InsOracle(mesh, prm, wall)
    assert o.run(2) == 2
    assert o.run(2) == 0          # the limit counts every inner step since init
    assert o.run(5) == 3
    assert o.stats()["inner"] == 5


def test_lid_cavity_meshes_are_closed_and_flagged():
    for m in (meshgen.lid_cavity_2d(8), meshgen.lid_cavity_2d(8, jitter=0.2, triangles=True),
              meshgen.lid_cavity_3d(4)):
        assert np.all(m.bc_type == 2)
        nb = m.n_bfaces
        lid = m.bc_name_id == 1
        per_side = nb // (4 if m.dim == 2 else 6)
        assert lid.sum() == per_side
        w = meshgen.lid_velocity(m, 2.5)
        assert np.all(w[lid, 0] == 2.5) and np.all(w[~lid] == 0.0) and np.all(w[:, 1:] == 0.0)

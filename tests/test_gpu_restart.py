"""READ_RESTART / DUMP_RESTART through the C ABI (ofg_read_restart,
ofg_write_restart) against the restart files the reference itself wrote
(tests/golden/restart_*.npz rebuild them byte for byte): the GPU continues a
solve from the reference's file and reaches the reference's uninterrupted
solution; the file the GPU writes carries the reference's record."""
import os

import numpy as np
import pytest

from oneflow_b200 import meshio, params as P
from oneflow_b200.solver import NS_SOLVER, TURB_SOLVER, OfgError, Solver
from golden_cases import RESTART_CASES, build

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / np.abs(b).max())


def l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def reference_files(name, d):
    f = np.load(os.path.join(HERE, "golden", f"restart_{name}.npz"))
    out = {}
    for key, fname in (("ns", "flow.dat"), ("turb", "turbflow.dat")):
        if f"{key}_q1" in f:
            out[key] = os.path.join(d, fname)
            meshio.write_flow_dat(out[key], f[f"{key}_q1"], int(f["step"]), float(f["time"]), q2=f[f"{key}_q2"])
    return f, out


@pytest.mark.parametrize("name", list(RESTART_CASES))
def test_gpu_continues_from_the_reference_restart_files(name, tmp_path):
    mesh, prm, steps = build(name)
    at = RESTART_CASES[name]
    f, files = reference_files(name, str(tmp_path))
    g = Solver(mesh, prm)
    step, t = g.read_restart(files["ns"], NS_SOLVER)
    assert (step, t) == (at, float(f["time"]))
    if "turb" in files:
        assert g.read_restart(files["turb"], TURB_SOLVER)[0] == at
    g.step(steps - at)
    gold = np.load(os.path.join(HERE, "golden", f"{name}.npz"))
    N = mesh.n_cells
    sa = "turbq" in gold
    # the reference's uninterrupted run to the same step (FP64 path: round-off;
    # SA: the far-field nu~ flip of the reference carries round-off into the state)
    assert rel(g.state()[:, :N], gold["q"][:, :N]) < (1e-9 if sa else 1e-12)
    if sa:
        assert l2(g.state(TURB_SOLVER)[:N], gold["turbq"][:N]) < 1e-5
    # the residual history continues at the file's step, as res.dat does
    h = g.res_history()
    assert h.shape[0] == steps
    assert np.all(np.abs(h[at:] - gold["reshist"][at:]) <= 5.01e-6 * np.abs(gold["reshist"][at:]) + 1e-12)


@pytest.mark.parametrize("name", list(RESTART_CASES))
def test_gpu_writes_the_reference_record(name, tmp_path):
    mesh, prm, _ = build(name)
    at = RESTART_CASES[name]
    f, _ = reference_files(name, str(tmp_path))
    g = Solver(mesh, prm)
    g.init_flowfield()
    g.step(at)
    nt = mesh.n_cells + mesh.n_bfaces
    path = str(tmp_path / "gpu_flow.dat")
    g.write_restart(path, NS_SOLVER, curr_time=float(f["time"]))
    rec = meshio.read_flow_dat(path, 5, nt)
    assert rec["step"] == at and rec["time"] == float(f["time"])
    sa = "turb_q1" in f
    tol = 1e-9 if sa else 1e-12
    assert rel(rec["q1"], f["ns_q1"]) < tol       # the state after step `at`
    assert rel(rec["q2"], f["ns_q2"]) < tol       # and one outer step earlier
    assert not rec["res1"].any() and not rec["res2"].any()
    assert os.path.getsize(path) == 8 + 4 + 8 + 4 * 5 * nt * 8
    if sa:
        tpath = str(tmp_path / "gpu_turbflow.dat")
        g.write_restart(tpath, TURB_SOLVER, curr_time=float(f["time"]))
        trec = meshio.read_flow_dat(tpath, 1, nt)
        assert trec["step"] == at
        assert l2(trec["q1"][0, :mesh.n_cells], f["turb_q1"][0, :mesh.n_cells]) < 1e-5
        assert np.array_equal(trec["q2"], trec["q1"])   # SA keeps no earlier state


def test_restart_round_trip_on_both_paths(tmp_path):
    # a GPU-written file read back by another context continues bitwise like
    # the context that wrote it
    mesh, prm, _ = build("bump_euler_roe_venkat")
    for prec in (0, 1):
        prm = P.euler_bump(ilim=2, vencat_coef=0.05, precision=prec)
        a = Solver(mesh, prm); a.init_flowfield(); a.step(7)
        path = str(tmp_path / f"rt{prec}.dat")
        a.write_restart(path)
        b = Solver(mesh, prm)
        assert b.read_restart(path) == (7, 0.0)
        a.step(5); b.step(5)
        assert np.array_equal(a.state(), b.state())
        assert np.array_equal(a.res_history()[7:], b.res_history()[7:])


def test_restart_errors(tmp_path):
    mesh, prm, _ = build("bump_euler_roe_venkat")
    g = Solver(mesh, prm)
    with pytest.raises(OfgError, match="error -8"):
        g.read_restart(str(tmp_path / "missing.dat"))
    other = str(tmp_path / "other.dat")
    meshio.write_flow_dat(other, np.ones((5, 10)), 3)       # a record of another mesh
    with pytest.raises(OfgError, match="error -1"):
        g.read_restart(other)
    with pytest.raises(OfgError, match="error -4"):
        g.write_restart(str(tmp_path / "nothing.dat"))     # no state yet

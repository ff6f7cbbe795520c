"""Restart files in the reference's layout, host side: the reader/writer of
oneflow_b200.meshio against the files the reference wrote (fixtures made by
tests/golden/make_golden.py), and -- where the reference build is present --
the reference continuing a solve from a file this writer made."""
import os
import tempfile

import numpy as np
import pytest

from oneflow_b200 import meshio
from golden_cases import RESTART_CASES, build
from oracle_lib import REF_ROOT, ref_available, run_ref

HERE = os.path.dirname(os.path.abspath(__file__))


def fixture(name):
    return np.load(os.path.join(HERE, "golden", f"restart_{name}.npz"))


@pytest.mark.parametrize("name", list(RESTART_CASES))
def test_writer_reproduces_the_record_layout(name, tmp_path):
    mesh, prm, _ = build(name)
    nt = mesh.n_cells + mesh.n_bfaces
    f = fixture(name)
    assert int(f["step"]) == RESTART_CASES[name]
    for key, ne in (("ns", 5), ("turb", 1)):
        if f"{key}_q1" not in f:
            continue
        path = str(tmp_path / f"{key}.dat")
        meshio.write_flow_dat(path, f[f"{key}_q1"], int(f["step"]), float(f["time"]), q2=f[f"{key}_q2"])
        raw = open(path, "rb").read()
        # int64 byte count, int32 step, f64 time, 4 x [ne][nT] f64
        assert len(raw) == 8 + 4 + 8 + 4 * ne * nt * 8
        assert int(np.frombuffer(raw, "<i8", 1)[0]) == len(raw) - 8
        rec = meshio.read_flow_dat(path, ne, nt)
        assert rec["step"] == int(f["step"]) and rec["time"] == float(f["time"])
        assert np.array_equal(rec["q1"], f[f"{key}_q1"]) and np.array_equal(rec["q2"], f[f"{key}_q2"])
        assert not rec["res1"].any() and not rec["res2"].any()
        with pytest.raises(ValueError):
            meshio.read_flow_dat(path, ne, nt + 1)   # another mesh


def test_reader_on_the_reference_s_own_restart_file():
    # the restart file shipped with the reference's plateuns2dslau2_continue case
    base = os.path.join(REF_ROOT, "test", "plateuns2dslau2_continue")
    if not os.path.isdir(base):
        pytest.skip("reference tree not present")
    mesh = meshio.read_ofl(os.path.join(base, "grid", "plate20182d.ofl"))
    rec = meshio.read_flow_dat(os.path.join(base, "restart", "flow.dat"), 5, mesh.n_cells + mesh.n_bfaces)
    assert rec["step"] == 34950 and abs(rec["time"] - 34.95) < 1e-9
    assert not rec["res1"].any() and not rec["res2"].any()
    rho, p = rec["q1"][0, :mesh.n_cells], rec["q1"][4, :mesh.n_cells]
    assert rho.min() > 0.5 and p.min() > 0.0
    assert 0 < np.abs(rec["q2"] - rec["q1"]).max() < 1e-4   # one outer step earlier


@pytest.mark.skipif(not ref_available(), reason="reference build (oracle/_ref) absent")
@pytest.mark.parametrize("name", list(RESTART_CASES))
def test_reference_continues_from_files_this_writer_made(name):
    mesh, prm, steps = build(name)
    f = fixture(name)
    files = {}
    with tempfile.TemporaryDirectory() as d:
        for key, fname in (("ns", "flow.dat"), ("turb", "turbflow.dat")):
            if f"{key}_q1" in f:
                path = os.path.join(d, fname)
                meshio.write_flow_dat(path, f[f"{key}_q1"], int(f["step"]), float(f["time"]), q2=f[f"{key}_q2"])
                files[fname] = open(path, "rb").read()
    dump, rows = run_ref(mesh, prm, steps, restart_in=files)
    g = np.load(os.path.join(HERE, "golden", f"{name}.npz"))
    # bitwise the uninterrupted run
    assert np.array_equal(dump["q"], g["q"])
    assert rows[0, 0] == RESTART_CASES[name] + 1 and rows.shape[0] == steps - RESTART_CASES[name]

"""Regenerates the golden fixtures of this folder by running the reference
CPU solver (built from its sources into oracle/_ref by oracle/Makefile) on
seeded meshes, with the full-precision dump hook of oracle/refbuild.

    python tests/golden/make_golden.py

Each fixture <case>.npz holds the case parameters, the final primitive state
q [5][nCells+nBFaces], nu~ for SA cases, the aerodynamic forces of the final
state (total, pressure, viscous x y z, CL, CD, CD_pres, CD_vis) and the
residual history the reference printed (res.dat / turbres.dat rows).  The meshes are regenerated
from their seeds by the tests, so only the outputs are stored.

restart_<case>.npz holds the restart files the reference wrote at outer step
RESTART_CASES[case] of the same case (restart/flow.dat, and restart/turbflow.dat
for SA), as the arrays of their single-zone record: step, time, q1, q2 (the
residual records are zero in a steady run).  oneflow_b200.meshio.write_flow_dat
rebuilds the files byte for byte from them; the reference continued from those
files reaches the same state as its uninterrupted run (<case>.npz) bitwise.

walldist_<name>.npz holds the wall distance the reference computed itself
(CALC_WALL_DIST, ireadwdst = 0) on the meshes of WALLDIST_CASES.

bump2d_c1.npz is the 2-D Euler bump at its benchmark size (65,536 triangles,
first-order Roe, LU-SGS, CFL 5, 2,000 outer iterations) as the reference ran
it: every 16th interior cell of the final state, the per-equation sum and sum
of squares of the whole interior state, the forces and the residual history
(the whole state would be 2.6 MB).  bump2d_c1_converged.npz: the same case run for
40,000 iterations, to a 4.6e-10 drop of its density residual (every 16th cell, forces,
every 100th residual row, the final drop).

    python tests/golden/make_golden.py --restart-only   # only the restart fixtures
    python tests/golden/make_golden.py --walldist-only  # only the wall-distance fixtures
    python tests/golden/make_golden.py --c1-only        # only the benchmark-size bump (about 2 CPU minutes)
    python tests/golden/make_golden.py --c1-converged-only  # the same bump run for 40,000 iterations
                                                        # (about 45 CPU minutes)
    python tests/golden/make_golden.py --case=<name>    # one case fixture
    python tests/golden/make_golden.py --ins-only       # only the incompressible cavity fixtures

ins_<case>.npz (INS_CASES): the incompressible solver on a lid-driven cavity,
the reference's state q [5][nCells+nBFaces] and gradients after the case's
inner iterations, and the remax_up/vp/wp/pp it printed per step (6 digits)."""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oneflow_b200 import meshio, params as P  # noqa: E402
from golden_cases import C1_STEPS, C1_STRIDE, CASES, INS_CASES, RESTART_CASES, WALLDIST_CASES, build, build_c1, \
    build_ins, build_walldist  # noqa: E402
from oracle_lib import run_ref, run_ref_ins  # noqa: E402


def restart_fixtures():
    import tempfile
    for name, at in RESTART_CASES.items():
        mesh, prm, steps = build(name)
        files = {}
        run_ref(mesh, prm, at, restart_out=files)
        nt = mesh.n_cells + mesh.n_bfaces
        out = {}
        for fname, key, ne in (("flow.dat", "ns", 5), ("turbflow.dat", "turb", 1)):
            if fname not in files:
                continue
            with tempfile.NamedTemporaryFile(suffix=".dat") as tmp:
                tmp.write(files[fname]); tmp.flush()
                rec = meshio.read_flow_dat(tmp.name, ne, nt)
                meshio.write_flow_dat(tmp.name + ".chk", rec["q1"], rec["step"], rec["time"], q2=rec["q2"])
                same = open(tmp.name + ".chk", "rb").read() == files[fname]
                os.remove(tmp.name + ".chk")
            assert same and not rec["res1"].any() and not rec["res2"].any(), fname
            out.update({f"{key}_q1": rec["q1"], f"{key}_q2": rec["q2"], "step": rec["step"], "time": rec["time"]})
        np.savez_compressed(os.path.join(HERE, f"restart_{name}.npz"), **out)
        print("restart", name, "at step", at, sorted(files))


def walldist_fixtures():
    for name in WALLDIST_CASES:
        mesh, prm = build_walldist(name)
        dump, _ = run_ref(mesh, prm, 1)
        wd = dump["walldist"][0, :mesh.n_cells]
        np.savez_compressed(os.path.join(HERE, f"walldist_{name}.npz"), walldist=wd)
        print("walldist", name, mesh.n_cells, "cells", float(wd.min()), float(wd.max()))


def c1_fixture():
    mesh, prm = build_c1()
    dump, rows = run_ref(mesh, prm, C1_STEPS)
    q = dump["q"][:, :mesh.n_cells]
    np.savez_compressed(os.path.join(HERE, "bump2d_c1.npz"), q_sub=q[:, ::C1_STRIDE], q_sum=q.sum(axis=1),
                        q_sumsq=(q * q).sum(axis=1), forces=dump["forces"].ravel()[:13], reshist=rows[:, 2:7],
                        steps=C1_STEPS, params=json.dumps(P.to_dict(prm)))
    print("bump2d_c1", mesh.n_cells, "cells", C1_STEPS, "steps")


def c1_converged_fixture(steps: int = 40000):
    mesh, prm = build_c1()
    dump, rows = run_ref(mesh, prm, steps)
    q = dump["q"][:, :mesh.n_cells]
    h = rows[:, 2]
    np.savez_compressed(os.path.join(HERE, "bump2d_c1_converged.npz"), q_sub=q[:, ::C1_STRIDE],
                        forces=dump["forces"].ravel()[:13], reshist_every_100=rows[::100, 2:7],
                        final_drop=float(h[-1] / h[0]), steps=steps, params=json.dumps(P.to_dict(prm)))
    print("bump2d_c1_converged", mesh.n_cells, "cells", steps, "steps, drop", h[-1] / h[0])


def ins_fixtures():
    for name in INS_CASES:
        mesh, prm, wall, steps = build_ins(name)
        dump, rem = run_ref_ins(mesh, prm, 1.0, steps)
        np.savez_compressed(os.path.join(HERE, f"ins_{name}.npz"), q=dump["q"], dqdx=dump["dqdx"], dqdy=dump["dqdy"],
                            remax_printed=rem, steps=steps, params=json.dumps(P.to_dict(prm)))
        print("ins", name, mesh.n_cells, "cells", steps, "inner steps")


def main():
    if "--ins-only" in sys.argv:
        ins_fixtures()
        return
    if "--c1-only" in sys.argv:
        c1_fixture()
        return
    if "--c1-converged-only" in sys.argv:
        c1_converged_fixture()
        return
    if "--walldist-only" in sys.argv:
        walldist_fixtures()
        return
    if not any(a.startswith("--case=") for a in sys.argv):
        restart_fixtures()
    if "--restart-only" in sys.argv:
        return
    if not any(a.startswith("--case=") for a in sys.argv):
        walldist_fixtures()
    only = [a.split("=", 1)[1] for a in sys.argv[1:] if a.startswith("--case=")]
    for name, spec in CASES.items():
        if only and name not in only:
            continue
        mesh, prm, steps = build(name)
        dump, rows = run_ref(mesh, prm, steps)
        out = {"q": dump["q"], "reshist": rows[:, 2:7], "params": json.dumps(P.to_dict(prm)), "steps": steps}
        if "turbq" in dump:
            out["turbq"] = dump["turbq"][0]
        if "forces" in dump:   # the reference's own force routine, full precision
            out["forces"] = dump["forces"].ravel()[:13]
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(name, mesh.n_cells, "cells", steps, "steps")


if __name__ == "__main__":
    main()

"""Regenerates the golden fixtures of this folder by running the reference
CPU solver (built from its sources into oracle/_ref by oracle/Makefile) on
seeded meshes, with the full-precision dump hook of oracle/refbuild.

    python tests/golden/make_golden.py

Each fixture <case>.npz holds the case parameters, the final primitive state
q [5][nCells+nBFaces], nu~ for SA cases, the aerodynamic forces of the final
state (total, pressure, viscous x y z, CL, CD, CD_pres, CD_vis) and the
residual history the reference printed (res.dat / turbres.dat rows).  The meshes are regenerated
from their seeds by the tests, so only the outputs are stored."""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oneflow_b200 import params as P  # noqa: E402
from golden_cases import CASES, build  # noqa: E402
from oracle_lib import run_ref  # noqa: E402


def main():
    for name, spec in CASES.items():
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

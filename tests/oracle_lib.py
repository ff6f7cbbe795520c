"""ctypes access to the CPU oracle (oracle/liboforacle.so) and a runner for
the reference-built oracle (oracle/_ref/oneflow_ref).  Test infrastructure."""
from __future__ import annotations

import ctypes as C
import os
import shutil
import subprocess
import tempfile

import numpy as np

from oneflow_b200 import params as P
from oneflow_b200.meshio import Mesh, read_ref_dump, read_res_dat, write_case

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "liboforacle.so")
REF_EXE = os.path.join(ROOT, "oracle", "_ref", "oneflow_ref")
# the reference's source tree (its regression cases are read from there): the
# ONEFLOW_REF environment variable, as in oracle/Makefile
REF_ROOT = os.environ.get("ONEFLOW_REF", "/root/reference")

_dp = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


def _load():
    if not os.path.exists(ORACLE_SO):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "liboforacle.so"], check=True,
                       stdout=subprocess.DEVNULL)
    lib = C.CDLL(ORACLE_SO)
    lib.oro_create.restype = C.c_void_p
    lib.oro_create.argtypes = [C.POINTER(P.OfgParams)]
    lib.oro_destroy.argtypes = [C.c_void_p]
    lib.oro_set_mesh.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp, C.c_int, _ip, _ip, _ip, _ip, C.c_int, C.c_int,
                                 _ip, C.c_void_p]
    lib.oro_init_flowfield.argtypes = [C.c_void_p]
    lib.oro_step.argtypes = [C.c_void_p, C.c_int]
    lib.oro_task.argtypes = [C.c_void_p, C.c_char_p]
    lib.oro_field.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p]
    lib.oro_field.restype = C.c_int64
    lib.oro_set_q.argtypes = [C.c_void_p, _dp]
    lib.oro_outer_steps.argtypes = [C.c_void_p]
    lib.oro_outer_steps.restype = C.c_long
    lib.oro_forces.argtypes = [C.c_void_p, C.c_double, C.c_void_p]
    lib.oro_ins_create.restype = C.c_void_p
    lib.oro_ins_create.argtypes = [C.c_void_p]
    lib.oro_ins_destroy.argtypes = [C.c_void_p]
    lib.oro_ins_set_wall.argtypes = [C.c_void_p, _dp]
    lib.oro_ins_init.argtypes = [C.c_void_p]
    lib.oro_ins_run.argtypes = [C.c_void_p, C.c_int]
    lib.oro_ins_stats.argtypes = [C.c_void_p, _dp]
    lib.oro_ins_field.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p]
    lib.oro_ins_field.restype = C.c_int64
    return lib


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        _LIB = _load()
    return _LIB


class Oracle:
    """One CPU solve: mirrors the reference's task sequence in FP64."""

    def __init__(self, mesh: Mesh, params: P.OfgParams):
        self.L = lib()
        self.mesh = mesh
        self.params = params
        self.h = self.L.oro_create(C.byref(params))
        a = mesh.as_arrays()
        wd = None if a["wd"] is None else a["wd"].ctypes.data_as(C.c_void_p)
        self._wd = a["wd"]
        rc = self.L.oro_set_mesh(self.h, mesh.n_nodes, a["x"], a["y"], a["z"], mesh.n_faces, a["fnc"], a["fn"],
                                 a["lc"], a["rc"], mesh.n_cells, mesh.n_bfaces, a["bct"], wd)
        assert rc == 0
        self.nT = mesh.n_cells + mesh.n_bfaces

    def __del__(self):
        try:
            self.L.oro_destroy(self.h)
        except Exception:
            pass

    def init(self):
        self.L.oro_init_flowfield(self.h)

    def step(self, n=1):
        return self.L.oro_step(self.h, n)

    def task(self, name):
        rc = self.L.oro_task(self.h, name.encode())
        assert rc == 0, name

    def field(self, name):
        n = self.L.oro_field(self.h, name.encode(), None)
        assert n >= 0, name
        out = np.empty(n, np.float64)
        self.L.oro_field(self.h, name.encode(), out.ctypes.data_as(C.c_void_p))
        return out

    def q(self):
        return self.field("q").reshape(5, self.nT)

    def res_history(self):
        return self.field("reshist").reshape(-1, 5)

    def set_q(self, q):
        self.L.oro_set_q(self.h, np.ascontiguousarray(q, np.float64).ravel())

    def forces(self, aref=1.0):
        """[13]: total, pressure and viscous force (x y z each), CL, CD, CD_pres, CD_vis."""
        out = np.zeros(13, np.float64)
        assert self.L.oro_forces(self.h, aref, out.ctypes.data_as(C.c_void_p)) == 0
        return out


def ref_available() -> bool:
    return os.path.exists(REF_EXE)


def run_ref(mesh: Mesh, params: P.OfgParams, steps: int, workdir: str = None, keep: bool = False,
            restart_in: dict = None, restart_out: dict = None):
    """Run the reference CPU solver on ``mesh`` up to outer iteration ``steps``.
    Returns (dump dict, res.dat rows).  ``restart_in`` ({"flow.dat": bytes,
    "turbflow.dat": bytes}) starts it from those restart files (startStrategy 1);
    with ``restart_out`` (a dict) it writes restart files at its last step
    (nFieldSave = steps), which are put there by name."""
    tmp = workdir or tempfile.mkdtemp(prefix="ofgref_")
    case = os.path.join(tmp, "case")
    write_case(case, mesh, P.to_dict(params), steps, start_strategy=1 if restart_in else 0,
               field_save=steps if restart_out is not None else 10 ** 8)
    for name, data in (restart_in or {}).items():
        with open(os.path.join(case, "restart", name), "wb") as fh:
            fh.write(data)
    dump = os.path.join(tmp, "dump.bin")
    env = dict(os.environ, OFG_REF_DUMP=dump)
    r = subprocess.run([REF_EXE, "0", "case"], cwd=tmp, env=env, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                       timeout=3600)
    if r.returncode != 0:
        raise RuntimeError(r.stdout.decode(errors="replace")[-3000:])
    out = read_ref_dump(dump), read_res_dat(os.path.join(case, "results", "res.dat"))
    if restart_out is not None:
        for name in ("flow.dat", "turbflow.dat"):
            fn = os.path.join(case, "restart", name)
            if os.path.exists(fn):
                restart_out[name] = open(fn, "rb").read()
    if not keep and workdir is None:
        shutil.rmtree(tmp, ignore_errors=True)
    return out


class InsOracle:
    """The incompressible SIMPLE solve of the reference (oracle_ins.h) on one
    mesh whose boundary is all solid wall; ``wall`` [nBFaces, 3] is the wall
    velocity of each boundary face."""

    def __init__(self, mesh: Mesh, params: P.OfgParams, wall: np.ndarray):
        self.base = Oracle(mesh, params)
        self.L = self.base.L
        self.nT = self.base.nT
        self.h = self.L.oro_ins_create(self.base.h)
        assert self.h, "mesh not supported by the incompressible oracle"
        self.L.oro_ins_set_wall(self.h, np.ascontiguousarray(wall, np.float64).ravel())
        self.L.oro_ins_init(self.h)

    def __del__(self):
        try:
            self.L.oro_ins_destroy(self.h)
        except Exception:
            pass

    def run(self, max_inner: int) -> int:
        return self.L.oro_ins_run(self.h, max_inner)

    def stats(self) -> dict:
        o = np.zeros(13, np.float64)
        self.L.oro_ins_stats(self.h, o)
        return dict(remax=o[:4].copy(), gmres_iters=o[4:8].astype(int), gmres_res=o[8:12].copy(), inner=int(o[12]))

    def field(self, name):
        n = self.L.oro_ins_field(self.h, name.encode(), None)
        assert n >= 0, name
        out = np.empty(n, np.float64)
        self.L.oro_ins_field(self.h, name.encode(), out.ctypes.data_as(C.c_void_p))
        return out

    def q(self):
        return self.field("q").reshape(5, self.nT)


def run_ref_ins(mesh: Mesh, params: P.OfgParams, u_lid: float, steps: int, workdir: str = None, exe: str = None,
                output: list = None):
    """Run the reference's incompressible solver (INsSolver, startStrategy 2,
    time_integral 3) for ``steps`` inner iterations on a cavity whose
    bc_name_id 1 faces move at (u_lid, 0, 0) (grid/ins_bc.txt).  Returns the
    dump dict and the printed remax lines (one [up, vp, wp, pp] per step).
    ``exe``: another build of the reference (the drop-in); ``output``: a list
    that receives the run's printed output."""
    tmp = workdir or tempfile.mkdtemp(prefix="ofgins_")
    case = os.path.join(tmp, "case")
    d = P.to_dict(params)
    d["time_integral"] = 3
    write_case(case, mesh, d, steps, start_strategy=2)
    with open(os.path.join(case, "script", "solver.txt"), "w") as fh:
        fh.write("INsSolver\n")
    with open(os.path.join(case, "script", "cfd.txt"), "a") as fh:
        fh.write(f"int maxIterSteps = {steps};\n")
    with open(os.path.join(case, "grid", "ins_bc.txt"), "w") as fh:
        fh.write(f"1 5 1.0 {u_lid!r} 0.0 0.0 0.0\n")
    dump = os.path.join(tmp, "dump.bin")
    env = dict(os.environ, OFG_REF_DUMP=dump)
    r = subprocess.run([exe or REF_EXE, "0", "case"], cwd=tmp, env=env, stdout=subprocess.PIPE,
                       stderr=subprocess.STDOUT, timeout=3600)
    out = r.stdout.decode(errors="replace")
    if output is not None:
        output.append(out)
    if r.returncode != 0:
        raise RuntimeError(out[-3000:])
    rem, cur = [], {}
    for line in out.splitlines():
        if line.startswith("iinv.remax_"):
            k, v = line[len("iinv.remax_"):].split(":")
            cur[k] = float(v)
            if k == "pp":
                rem.append([cur.get("up"), cur.get("vp"), cur.get("wp"), cur.get("pp")])
                cur = {}
    res = read_ref_dump(dump), np.array(rem)
    if workdir is None:
        shutil.rmtree(tmp, ignore_errors=True)
    return res

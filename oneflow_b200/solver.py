"""Python face of the C ABI: one ``Solver`` per context, with one method per
reference task (the names of system/ns/function/funcMap.txt) and the fused
outer iteration.  The CUDA library is required: there is no CPU path."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import params as P
from .meshio import Mesh

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libofg.so")

NS_SOLVER, TURB_SOLVER = 0, 1
_dp = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


class OfgError(RuntimeError):
    pass


class OfgTuning(C.Structure):
    """ctypes mirror of ofg_tuning (include/oneflow_b200.h)."""
    _fields_ = [("face_min_blocks", C.c_int), ("face_block", C.c_int), ("grad_min_blocks", C.c_int),
                ("sweep_min_blocks", C.c_int), ("sweep_block", C.c_int), ("sweep_persistent", C.c_int),
                ("grad_block", C.c_int), ("reserved", C.c_int * 1),
                ("ms_default", C.c_double), ("ms_tuned", C.c_double)]

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_ if n != "reserved"}


_LIB = None


def load_library() -> C.CDLL:
    """Load oneflow_b200/libofg.so (built by ``__graft_entry__.build()`` or
    ``make -C oneflow_b200/csrc``).  Raises if it is missing."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise OfgError(f"CUDA library not built: {LIB_PATH} (run make -C oneflow_b200/csrc)")
    L = C.CDLL(LIB_PATH)
    L.ofg_default_params.argtypes = [C.POINTER(P.OfgParams)]
    L.ofg_create.argtypes = [C.POINTER(P.OfgParams), C.POINTER(C.c_void_p)]
    L.ofg_destroy.argtypes = [C.c_void_p]
    L.ofg_last_error.argtypes = [C.c_void_p]
    L.ofg_last_error.restype = C.c_char_p
    L.ofg_upload_mesh.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp, C.c_int, _ip, _ip, _ip, _ip, C.c_int, C.c_int,
                                  _ip, C.c_void_p]
    for name in ("ofg_init_flowfield",):
        getattr(L, name).argtypes = [C.c_void_p]
    L.ofg_upload_state.argtypes = [C.c_void_p, C.c_int, _dp]
    L.ofg_download_state.argtypes = [C.c_void_p, C.c_int, _dp]
    L.ofg_calc_wall_dist.argtypes = [C.c_void_p]
    L.ofg_calc_lhs.argtypes = [C.c_void_p, C.c_int, C.c_double]
    L.ofg_batch_create.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_void_p)]
    L.ofg_batch_step.argtypes = [C.c_void_p, C.c_int]
    L.ofg_batch_destroy.argtypes = [C.c_void_p]
    L.ofg_batch_last_error.argtypes = [C.c_void_p]
    L.ofg_batch_last_error.restype = C.c_char_p
    L.ofg_batch_device_ms.argtypes = [C.c_void_p, C.POINTER(C.c_float)]
    L.ofg_write_restart.argtypes = [C.c_void_p, C.c_int, C.c_char_p, C.c_double]
    L.ofg_read_restart.argtypes = [C.c_void_p, C.c_int, C.c_char_p, C.POINTER(C.c_int64), C.POINTER(C.c_double)]
    for name in ("ofg_zero_dq", "ofg_calc_time_step", "ofg_load_residuals", "ofg_update_residuals", "ofg_init_lusgs",
                 "ofg_lusgs_lower", "ofg_lusgs_upper", "ofg_update_flowfield", "ofg_calc_boundary"):
        getattr(L, name).argtypes = [C.c_void_p, C.c_int]
    L.ofg_step.argtypes = [C.c_void_p, C.c_int]
    L.ofg_residual_norms.argtypes = [C.c_void_p, C.c_int, _dp]
    L.ofg_residual_max.argtypes = [C.c_void_p, C.c_int, _dp, np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")]
    L.ofg_forces.argtypes = [C.c_void_p, C.c_double, C.c_void_p]
    L.ofg_download_field.argtypes = [C.c_void_p, C.c_int, C.c_char_p, C.c_void_p, C.c_int64, C.POINTER(C.c_int64)]
    L.ofg_get_counters.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    L.ofg_set_outer_step.argtypes = [C.c_void_p, C.c_int64]
    L.ofg_set_stream.argtypes = [C.c_void_p, C.c_void_p]
    L.ofg_sweep_levels.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.ofg_profile_step.argtypes = [C.c_void_p, _dp, np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")]
    L.ofg_colour_order.argtypes = [C.c_int, C.c_int, C.c_int, _ip, _ip, _ip]
    L.ofg_rcm_order.argtypes = [C.c_int, C.c_int, C.c_int, _ip, _ip, _ip]
    L.ofg_autotune.argtypes = [C.c_void_p, C.c_int, C.POINTER(OfgTuning)]
    L.ofg_get_tuning.argtypes = [C.c_void_p, C.POINTER(OfgTuning)]
    L.ofg_set_tuning.argtypes = [C.c_void_p, C.POINTER(OfgTuning)]
    L.ofg_version.restype = C.c_int
    L.ofg_ins_create.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p)]
    L.ofg_ins_destroy.argtypes = [C.c_void_p]
    L.ofg_ins_destroy.restype = None
    for name in ("ofg_ins_init_flowfield", "ofg_ins_update_residuals"):
        getattr(L, name).argtypes = [C.c_void_p]
    L.ofg_ins_run.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int)]
    L.ofg_ins_upload_state.argtypes = [C.c_void_p, _dp]
    L.ofg_ins_stats.argtypes = [C.c_void_p, _dp]
    L.ofg_ins_timing.argtypes = [C.c_void_p, _dp]
    L.ofg_ins_get_field.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p, C.c_int64]
    _LIB = L
    return L


# reference task name -> C entry point (funcMap.txt / TimeIntegral::Lusgs)
TASKS = {
    "ZERO_DQ_FIELD": "ofg_zero_dq",
    "CALC_TIME_STEP": "ofg_calc_time_step",
    "LOAD_RESIDUALS": "ofg_load_residuals",
    "UPDATE_RESIDUALS": "ofg_update_residuals",
    "INIT_LUSGS": "ofg_init_lusgs",
    "LUSGS_LOWER_SWEEP": "ofg_lusgs_lower",
    "LUSGS_UPPER_SWEEP": "ofg_lusgs_upper",
    "UPDATE_FLOWFIELD_LUSGS": "ofg_update_flowfield",
    "CALC_BOUNDARY": "ofg_calc_boundary",
}
LUSGS_SEQUENCE = ["ZERO_DQ_FIELD", "CALC_TIME_STEP", "LOAD_RESIDUALS", "UPDATE_RESIDUALS", "INIT_LUSGS",
                  "LUSGS_LOWER_SWEEP", "LUSGS_UPPER_SWEEP", "UPDATE_FLOWFIELD_LUSGS", "CALC_BOUNDARY"]


class Solver:
    """One steady solve on one GPU."""

    def __init__(self, mesh: Mesh, params: P.OfgParams):
        self.L = load_library()
        self.mesh = mesh
        self.params = params
        h = C.c_void_p()
        rc = self.L.ofg_create(C.byref(params), C.byref(h))
        if rc != 0:
            raise OfgError(f"ofg_create failed ({rc})")
        self.h = h
        self.nT = mesh.n_cells + mesh.n_bfaces
        a = mesh.as_arrays()
        self._keep = a
        wd = None if a["wd"] is None else a["wd"].ctypes.data_as(C.c_void_p)
        self._check(self.L.ofg_upload_mesh(self.h, mesh.n_nodes, a["x"], a["y"], a["z"], mesh.n_faces, a["fnc"],
                                           a["fn"], a["lc"], a["rc"], mesh.n_cells, mesh.n_bfaces, a["bct"], wd))

    def _check(self, rc):
        if rc != 0:
            msg = self.L.ofg_last_error(self.h)
            raise OfgError(f"error {rc}: {msg.decode() if msg else ''}")

    def close(self):
        if getattr(self, "h", None):
            self.L.ofg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- lifecycle ----
    def init_flowfield(self):
        self._check(self.L.ofg_init_flowfield(self.h))

    def upload_state(self, q: np.ndarray, tid: int = NS_SOLVER):
        self._check(self.L.ofg_upload_state(self.h, tid, np.ascontiguousarray(q, np.float64).ravel()))

    def state(self, tid: int = NS_SOLVER, out: np.ndarray = None) -> np.ndarray:
        """[5][nCells+nBFaces] primitive NS state, or [nCells+nBFaces] nu~ for tid 1.
        ``out``: a C-contiguous float64 array of that size to fill (e.g. a view
        of pinned host memory, which makes the copy a direct DMA)."""
        ne = 5 if tid == NS_SOLVER else 1
        if out is None:
            out = np.empty(ne * self.nT, np.float64)
        elif out.dtype != np.float64 or not out.flags.c_contiguous or out.size != ne * self.nT:
            raise ValueError("out must be a C-contiguous float64 array of the state's size")
        flat = out.reshape(-1)
        self._check(self.L.ofg_download_state(self.h, tid, flat))
        return out.reshape(5, self.nT) if ne == 5 else out.reshape(-1)

    def calc_wall_dist(self):
        """CALC_WALL_DIST on the GPU (ofg_calc_wall_dist); the SA source uses it
        from then on.  The distances: field("walldist")."""
        self._check(self.L.ofg_calc_wall_dist(self.h))

    def write_restart(self, path: str, tid: int = NS_SOLVER, curr_time: float = 0.0):
        """DUMP_RESTART: the solver's restart record in the reference's file
        layout (ofg_write_restart; "flowFile" for NS, "turbflowFile" for SA)."""
        self._check(self.L.ofg_write_restart(self.h, tid, os.fsencode(path), C.c_double(curr_time)))

    def read_restart(self, path: str, tid: int = NS_SOLVER):
        """READ_RESTART from a file in the reference's layout (ofg_read_restart):
        the state becomes the file's q1; for NS the outer step counter follows
        the file.  Returns (outer step, time) of the file."""
        step, t = C.c_int64(), C.c_double()
        self._check(self.L.ofg_read_restart(self.h, tid, os.fsencode(path), C.byref(step), C.byref(t)))
        return step.value, t.value

    # ---- tasks ----
    def task(self, name: str, tid: int = NS_SOLVER):
        self._check(getattr(self.L, TASKS[name])(self.h, tid))

    def calc_lhs(self, lhscoef: float, tid: int = NS_SOLVER):
        """CALC_LHS of the multi-stage scheme (ofg_calc_lhs): res *= dt/vol * lhscoef."""
        self._check(self.L.ofg_calc_lhs(self.h, tid, C.c_double(lhscoef)))

    def set_outer_step(self, n: int):
        """Iteration::outerSteps as seen by the next CALC_TIME_STEP (task API)."""
        self._check(self.L.ofg_set_outer_step(self.h, n))

    def step(self, n: int = 1):
        self._check(self.L.ofg_step(self.h, n))

    def set_stream(self, stream_ptr: int):
        """Launch on the caller's CUDA stream (e.g. torch.cuda.current_stream().cuda_stream)."""
        self._check(self.L.ofg_set_stream(self.h, C.c_void_p(stream_ptr) if stream_ptr else None))

    PROFILE_GROUPS = ("cfl", "gradlim", "residual", "residual_sum", "clip", "lusgs_lower", "lusgs_upper", "update",
                      "boundary", "norm", "sa_grad", "sa_residual", "sa_lower", "sa_upper", "sa_update", "sa_boundary",
                      "sa_norm")

    def profile_step(self):
        """One iteration task by task with CUDA events: ({group: ms}, {group: launches}).
        "residual" is the flux + time-step pass alone (the FP64 path's per-cell
        gather, the mixed path's face pass), "residual_sum" the mixed path's
        per-cell sum of the face results (empty on the FP64 path); "gradlim"
        the gradient+limiter kernel(s) before them, "clip" the time-step clip
        after them."""
        ms = np.zeros(17, np.float64)
        nl = np.zeros(17, np.int32)
        self._check(self.L.ofg_profile_step(self.h, ms, nl))
        n = 17 if self.params.vismodel >= 3 else 10
        names = self.PROFILE_GROUPS[:n]
        return dict(zip(names, ms[:n].tolist())), dict(zip(names, nl[:n].tolist()))

    def autotune(self, reps: int = 5) -> dict:
        """ofg_autotune: time the candidate launch shapes on this mesh and keep
        the fastest (cached per mesh); returns the choice and its timings."""
        t = OfgTuning()
        self._check(self.L.ofg_autotune(self.h, reps, C.byref(t)))
        return t.as_dict()

    def tuning(self) -> dict:
        t = OfgTuning()
        self._check(self.L.ofg_get_tuning(self.h, C.byref(t)))
        return t.as_dict()

    def set_tuning(self, **kw):
        t = OfgTuning()
        self._check(self.L.ofg_get_tuning(self.h, C.byref(t)))
        for k, v in kw.items():
            setattr(t, k, v)
        self._check(self.L.ofg_set_tuning(self.h, C.byref(t)))

    FORCE_NAMES = ("Fx", "Fy", "Fz", "Fpx", "Fpy", "Fpz", "Fvx", "Fvy", "Fvz", "CL", "CD", "CD_pres", "CD_vis")

    def forces(self, aref: float = 1.0) -> np.ndarray:
        """Aerodynamic forces of the current state on the solid walls (ofg_forces):
        [13] = total, pressure and viscous force (x y z each), CL, CD, CD_pres, CD_vis."""
        out = np.zeros(13, np.float64)
        self._check(self.L.ofg_forces(self.h, C.c_double(aref), out.ctypes.data_as(C.c_void_p)))
        return out

    def residual_norms(self, tid: int = NS_SOLVER) -> np.ndarray:
        """RMS residual of the solver's last UPDATE_RESIDUALS: 5 values (NS) or 1 (SA)."""
        out = np.zeros(5, np.float64)
        self._check(self.L.ofg_residual_norms(self.h, tid, out))
        return out if tid == NS_SOLVER else out[:1]

    def residual_max(self, tid: int = NS_SOLVER):
        """(largest |residual| per equation, first cell holding it) of the last
        UPDATE_RESIDUALS: 5 entries (NS) or 1 (SA)."""
        v = np.zeros(5, np.float64)
        i = np.zeros(5, np.int64)
        self._check(self.L.ofg_residual_max(self.h, tid, v, i))
        n = 5 if tid == NS_SOLVER else 1
        return v[:n], i[:n]

    def field(self, name: str, tid: int = NS_SOLVER) -> np.ndarray:
        need = C.c_int64()
        self._check(self.L.ofg_download_field(self.h, tid, name.encode(), None, 0, C.byref(need)))
        out = np.empty(need.value, np.float64)
        self._check(self.L.ofg_download_field(self.h, tid, name.encode(), out.ctypes.data_as(C.c_void_p),
                                              need.value, C.byref(need)))
        return out

    def res_history(self) -> np.ndarray:
        return self.field("reshist").reshape(-1, 5)

    def sweep_levels(self):
        """(lower, upper) number of LU-SGS dependency levels of this numbering."""
        a, b = C.c_int(), C.c_int()
        self._check(self.L.ofg_sweep_levels(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def counters(self):
        a, b = C.c_int64(), C.c_int64()
        self._check(self.L.ofg_get_counters(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value


def colour_order(mesh: Mesh):
    """(perm, ncolours): the colour-major cell order of ofg_colour_order."""
    L = load_library()
    perm = np.empty(mesh.n_cells, np.int32)
    a = mesh.as_arrays()
    n = L.ofg_colour_order(mesh.n_cells, mesh.n_faces, mesh.n_bfaces, a["lc"], a["rc"], perm)
    if n < 0:
        raise OfgError(f"ofg_colour_order failed ({n})")
    return perm, n


class Batch:
    """Independent solves advanced together (ofg_batch_*): one CUDA-graph
    launch per outer iteration for all of them, bitwise the same as
    ``Solver.step`` on each.  Close the batch before its solvers."""

    def __init__(self, solvers):
        self.L = load_library()
        self.solvers = list(solvers)
        arr = (C.c_void_p * len(self.solvers))(*[s.h.value for s in self.solvers])
        h = C.c_void_p()
        rc = self.L.ofg_batch_create(arr, len(self.solvers), C.byref(h))
        if rc != 0:
            raise OfgError(f"ofg_batch_create failed ({rc})")
        self.h = h

    def step(self, n: int = 1):
        rc = self.L.ofg_batch_step(self.h, n)
        if rc != 0:
            msg = self.L.ofg_batch_last_error(self.h)
            raise OfgError(f"error {rc}: {msg.decode() if msg else ''}")

    def device_ms(self) -> float:
        """Device time of the last ``step`` call (CUDA events around its graph launches)."""
        ms = C.c_float()
        rc = self.L.ofg_batch_device_ms(self.h, C.byref(ms))
        if rc != 0:
            raise OfgError(f"ofg_batch_device_ms failed ({rc})")
        return ms.value

    def close(self):
        if getattr(self, "h", None):
            self.L.ofg_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def rcm_order(mesh: Mesh) -> np.ndarray:
    """perm[new] = old: the reverse Cuthill-McKee cell order of ofg_rcm_order."""
    L = load_library()
    a = mesh.as_arrays()
    perm = np.zeros(mesh.n_cells, np.int32)
    rc = L.ofg_rcm_order(mesh.n_cells, mesh.n_faces, mesh.n_bfaces, a["lc"], a["rc"], perm)
    if rc != 0:
        raise OfgError(f"ofg_rcm_order failed ({rc})")
    return perm


class Incompressible:
    """The reference's incompressible solver (INsSolver with startStrategy 2
    and the SIMPLE time integral) on one GPU: one inner iteration per
    ``update_residuals`` (its UPDATE_RESIDUALS task), ``run`` for MG::Run's
    inner loop.  ``params`` gives reynolds, mach_ref, the flow angles,
    global_dt and the dimension; every boundary face must be a solid wall,
    ``wall`` [nBFaces, 3] is the velocity of each (None: still walls)."""

    def __init__(self, mesh: Mesh, params: P.OfgParams, wall: np.ndarray = None):
        self.base = Solver(mesh, params)
        self.L = self.base.L
        self.mesh = mesh
        self.nT = mesh.n_cells + mesh.n_bfaces
        self._wall = None if wall is None else np.ascontiguousarray(wall, np.float64).reshape(mesh.n_bfaces, 3)
        h = C.c_void_p()
        wp = None if self._wall is None else self._wall.ctypes.data_as(C.c_void_p)
        self.base._check(self.L.ofg_ins_create(self.base.h, wp, C.byref(h)))
        self.h = h
        self.init_flowfield()

    def _check(self, rc):
        self.base._check(rc)

    def close(self):
        if getattr(self, "h", None):
            self.L.ofg_ins_destroy(self.h)
            self.h = None
        self.base.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init_flowfield(self):
        self._check(self.L.ofg_ins_init_flowfield(self.h))

    def upload_state(self, q: np.ndarray):
        self._check(self.L.ofg_ins_upload_state(self.h, np.ascontiguousarray(q, np.float64).reshape(-1)))

    def update_residuals(self):
        self._check(self.L.ofg_ins_update_residuals(self.h))

    def run(self, max_inner: int) -> int:
        n = C.c_int()
        self._check(self.L.ofg_ins_run(self.h, max_inner, C.byref(n)))
        return n.value

    def stats(self) -> dict:
        o = np.zeros(13, np.float64)
        self._check(self.L.ofg_ins_stats(self.h, o))
        return dict(remax=o[:4].copy(), gmres_iters=o[4:8].astype(int), gmres_res=o[8:12].copy(), inner=int(o[12]))

    def timing(self) -> dict:
        o = np.zeros(4, np.float64)
        self._check(self.L.ofg_ins_timing(self.h, o))
        return dict(ms=float(o[0]), gmres_iters=int(o[1]), gmres_ms=float(o[2]), gmres_bytes=float(o[3]))

    def field(self, name: str) -> np.ndarray:
        n = 5 * self.nT if name in ("q", "dqdx", "dqdy", "dqdz") else (
            self.mesh.n_faces if name in ("fq", "ajp") else self.nT)
        out = np.empty(n, np.float64)
        self._check(self.L.ofg_ins_get_field(self.h, name.encode(), out.ctypes.data_as(C.c_void_p), n))
        return out

    def q(self) -> np.ndarray:
        return self.field("q").reshape(5, self.nT)

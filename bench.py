"""Benchmark of the unstructured residual + LU-SGS iteration on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config NAME] [--impl ofg|reference]

One JSON line on rank 0.  A step is one outer iteration of the steady solve
(TimeIntegral::Lusgs for every solver) over the whole mesh.  ``value`` is
cell-iterations/s with the state resident in HBM (CUDA events on the
library's stream, max over ranks); ``e2e`` is the same metric through the
C ABI with the state copied host->device and back every step.  Multi-GPU runs
are independent replicas (one solve per GPU, no collective on the data path).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from oneflow_b200 import meshgen, params as P  # noqa: E402
from oneflow_b200.meshio import Mesh, write_case  # noqa: E402

L2_BYTES = 126 * 2 ** 20


# ---------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------
def make_workload(name: str):
    from oneflow_b200.walldist import plate_wall_distance
    if name in ("plate3d", "plate3d_small", "plate3d_sample"):
        dims = {"plate3d": (200, 100, 50), "plate3d_small": (40, 20, 10), "plate3d_sample": (200, 100, 5)}[name]
        mesh = meshgen.flat_plate_tets(*dims)
        mesh.wall_dist = plate_wall_distance(mesh)
        prm = P.rans_plate()
        nx, ny, nz = dims
        desc = dict(workload=f"3-D RANS-SA flat plate: {nx}x{ny}x{nz} hexes split into 6 tets "
                             f"({6 * nx * ny * nz:,} cells), wall-normal ratio 1.15, first cell y+~1 at Re 5e6, "
                             "Mach 0.2, Roe 2nd order, least-squares gradients, Venkatakrishnan eps^2=(K h)^3 K=5, "
                             "SA, LU-SGS; FP32 face terms, FP64 accumulation/update/norms",
                    lattice=list(dims))
        return mesh, prm, desc
    if name in ("wing3d", "wing3d_sample"):
        kw = {} if name == "wing3d" else dict(n_around=128, n_tet=20, nz_wing=30, nz_tip=10)
        mesh = meshgen.swept_wing_hybrid(**kw)
        prm = P.transonic_wing()
        m = mesh.meta
        desc = dict(workload=f"3-D transonic swept wing: NACA0012 section, aspect ratio 4, sweep 30 deg, half model; "
                             f"{m['n_hex']} hexahedral layers (ratio 1.2, y+~1) + tetrahedral far field "
                             f"({mesh.n_cells:,} cells); Mach 0.84, AoA 3.06, Re 1.2e7, SLAU2, Green-Gauss + Barth, "
                             "SA, LU-SGS; FP32 face terms, FP64 accumulation/update/norms")
        return mesh, prm, desc
    if name == "bump2d":
        mesh = meshgen.bump_channel(256, 128)
        prm = P.euler_bump()
        desc = dict(workload="2-D Euler bump channel, 256x128 quads split into 65,536 jittered triangles, "
                             "Mach 0.5, first-order Roe, LU-SGS, CFL 5, FP64")
    elif name == "bump2d_small":
        mesh = meshgen.bump_channel(64, 32)
        prm = P.euler_bump()
        desc = dict(workload="2-D Euler bump channel 64x32 (4,096 triangles), first-order Roe, LU-SGS, FP64")
    else:
        raise SystemExit(f"unknown config {name}")
    return mesh, prm, desc


_SAMPLE = {"plate3d": "plate3d_sample"}


def _ref_procs(mesh) -> int:
    """Concurrent reference processes: all host cores, bounded by memory
    (the reference holds about 1.7 kB per cell of a tetrahedral RANS-SA mesh,
    measured: 80 MB peak for 48,000 cells; 2 kB is budgeted) and by 64."""
    n = os.cpu_count() or 1
    try:
        import psutil
        avail = psutil.virtual_memory().available
        n = min(n, max(1, int(avail * 0.6 // (mesh.n_cells * 2000 + 1))))
    except Exception:
        pass
    return max(1, min(n, 64))


KERNEL_OF_GROUP = {"gradlim": "k_gradlim", "residual": "k_face_pass<0> (face fluxes + spectral radii, mixed path)",
                   "residual_sum": "k_face_sum<0> (per-cell sum of the face results, time step)",
                   "clip": "k_timestep_clip", "lusgs_lower": "k_lusgs_lower", "lusgs_upper": "k_lusgs_upper",
                   "update": "k_update", "sa_residual": "k_turb_rhs", "sa_grad": "k_turb_grad"}

# DRAM bytes (read + write) per cell of one step's launches of a profile
# group, from `ncu --section MemoryWorkloadAnalysis` of the 600,000-cell plate
# sample (plate3d_sample: same kernels, layout and sweep levels); the kernels
# stream their arrays once per launch, so the traffic scales with the cell
# count.
NCU_TRAFFIC_PER_CELL = {
    ("plate3d", "residual"): 334.7, ("plate3d", "gradlim"): 241.3, ("plate3d", "clip"): 40.0,
    ("plate3d", "lusgs_lower"): 445.4, ("plate3d", "lusgs_upper"): 356.9, ("plate3d", "update"): 109.7,
    ("plate3d", "sa_grad"): 63.5, ("plate3d", "sa_residual"): 398.9,
}


def bench_config(desc: dict, st: dict, ordering: str, world: int, flush: bool) -> dict:
    """The `config` object of the JSON line (the same for both arms)."""
    return dict(desc, cells=st["N"], faces=st["F"], ordering=ordering,
                l2="flushed between timed steps" if flush else "working set larger than L2",
                parallelism=f"replicas x{world}")


# Algorithmic bytes per cell-iteration of the agreed measurement contract
# (every array of a phase counted once at its stored size, perfect neighbour
# reuse; FP32 shadow state, gradients, limiter and geometry, FP64 residual,
# increments and master state): tetrahedral RANS-SA plate with least-squares
# gradients and Venkatakrishnan, F/N = 2.  The count in alg_bytes below is this
# implementation's own (its FP64 state reads and face records included).
CONTRACT_BYTES = {"plate3d": 1296, "plate3d_small": 1296, "plate3d_sample": 1296}


def mesh_stats(mesh: Mesh):
    N, B, F = mesh.n_cells, mesh.n_bfaces, mesh.n_faces
    return dict(N=N, B=B, F=F, E=2 * F - B)


def alg_bytes(st, prm) -> dict:
    """Algorithmic bytes of each profile group of one outer iteration: every
    array a kernel of the group reads or writes counted once per kernel, at its
    stored size, neighbour gathers counted once (perfect reuse).  Data layout of
    the CUDA path (g = 8 B FP64 path, 4 B mixed):
      state record (rho u v w p T mu_l mu_t): FP64 master 64 B, read by the
        gradient and residual kernels (both paths: the mixed path forms its face
        states and gradient differences in FP64); the sweeps and the SA kernels
        read the copy at the face precision (8g B)
      face record 8g B (normal, area, centre), cell record 4g B (centre, volume)
      gradient+limiter record 24g B, neighbour list entry 8 B (face|side, cell)
      residual, dq 40 B; dt, inviscid and viscous radii 8 B each."""
    N, B, F, E = st["N"], st["B"], st["F"], st["E"]
    NT = N + B
    FI = F - B
    g = 8 if prm.precision == 0 else 4
    mixed = prm.precision != 0
    vis = prm.vismodel > 0
    sa = prm.vismodel >= 3
    need_grad = prm.ilim != -1 or vis
    lsq = prm.igrad == 2
    qs = NT * 8 * g                            # state records at the face precision
    qm = NT * 64                               # FP64 master records
    cg = NT * 4 * g
    fg = F * 8 * g
    nbl = E * 8 + (N + 1) * 4
    half_lists = FI * 8 + (N + 1) * 4          # lower (or upper) lists: each interior face once
    gl = N * 24 * g
    out = {"cfl": 0}
    gradlim = 0
    if need_grad:
        # k_gradlim: states + centres of the cell and its neighbours, list,
        # face records (Green-Gauss weights or the limiter's face centres);
        # the mixed path reads the face-local offsets instead of the centres
        gradlim += qm + cg + nbl + fg + gl + (F * 32 if mixed else 0)
        if prm.ilim == 2 and not prm.venkat_kh3:
            gradlim += N * 10 * g + (gl + N * 10 * g + cg + nbl + fg + N * 5 * g)   # min/max, global eps pass
    out["gradlim"] = gradlim
    blocks = (N + 127) // 128
    if mixed:
        # k_face_pass: per face its two cells, FP64 normal and area, face-local
        # offsets, the FP64 state records and gradient records of both cells
        # (each read once: perfect reuse), wall states of the boundary faces;
        # writes the 48-B face record.  k_face_sum: the neighbour lists, the
        # face records, the volumes; writes res, dt and the two radii, and the
        # per-block norm sums
        out["residual"] = F * 8 + F * 32 + F * 32 + qm + (gl if need_grad else 0) + B * 44 + F * 48
        out["residual_sum"] = nbl + F * 48 + N * 4 + N * 40 + N * 24 + blocks * 40
    else:
        # k_residual: states, centres, face records, list, gradient records of the
        # cell and its neighbours, wall states; writes res, dt and the two radii,
        # and the per-block norm sums
        out["residual"] = qm + cg + fg + nbl + (gl if need_grad else 0) + B * 44 + N * 40 + N * 24 + blocks * 40
        out["residual_sum"] = 0
    out["clip"] = N * 24 + N * g + N * 16                        # dt, radii, vol -> dt, diagonal
    dq = N * 8 * g                                               # increment records
    sweep = qs + cg + F * 4 * g + half_lists + dq + dq + N * 8 + N * 4   # neighbour dq, own dq write, diagonal, order
    out["lusgs_lower"] = sweep + N * 40                          # + res
    out["lusgs_upper"] = sweep + dq                              # + own dq read before the write
    out["update"] = N * 64 + dq + N * 64 + (N * 8 * g if mixed else 0)
    out["boundary"] = B * (4 + 4 + 8 * g + 64 + 8 + 64 + 40) + (B * 8 * g if mixed else 0)
    out["norm"] = ((N + 127) // 128) * 40                        # per-block sums left by the residual kernel
    if sa:
        # the mixed path reads the face-local offsets in place of cell centres
        # (least squares, Green-Gauss weights)
        grad_nut = NT * 8 + nbl + cg + (0 if lsq else fg) + N * 4 * g + (F * 32 if mixed else 0)
        # k_turb_rhs: state records, centres, face records, lists, nu~, grad
        # nu~, velocity gradients, dt, wall distance, wall states; writes the
        # sweep coefficients, diagonal and residual (the mixed path also reads
        # the face-local offsets of the diffusion term)
        rhs = qs + cg + fg + nbl + NT * 8 + N * 4 * g + N * 12 * g + N * 16 + N * 8 + N * 8 + B * 44 \
            + F * 16 + N * 16 + (F * 32 if mixed else 0)
        out["sa_grad"] = B * 24 + grad_nut
        out["sa_residual"] = rhs
        sa_sweep = half_lists + FI * 16 + N * 8 + N * 8 + N * 8 + N * 8 + N * 4
        out["sa_lower"] = sa_sweep
        out["sa_upper"] = sa_sweep
        # nu~ and its increment read, nu~ written; rho and mu_l read; the
        # master record's last sector and the FP32 copy rewritten whole
        out["sa_update"] = N * 24 + N * 8 + N * 32 + N * 32 + (N * 8 * g if mixed else 0)
        out["sa_boundary"] = B * (4 + 4 + 8 * g + 24 + 8 + 16)
        out["sa_norm"] = ((N + 127) // 128) * 8
    return out


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run_nvml(self):
        # NVML reads take well under a millisecond, so a timed region of a
        # fraction of a second still gets tens of samples (read-only queries)
        import pynvml as nv
        nv.nvmlInit()
        try:
            h = nv.nvmlDeviceGetHandleByIndex(self.index)
            mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            bits = (nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                    nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap)
            while not self._stop.is_set():
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                pw = nv.nvmlDeviceGetPowerUsage(h) / 1000.0
                self.rows.append([str(self.index), str(sm), str(mx), f"{pw:.1f}", hex(rs)] +
                                 ["Active" if rs & b else "Not Active" for b in bits])
                self._stop.wait(0.02)
        finally:
            nv.nvmlShutdown()

    def _run(self):
        try:
            self._run_nvml()
            return
        except Exception:
            pass
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                for line in out.stdout.strip().splitlines():
                    self.rows.append([v.strip() for v in line.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ---------------------------------------------------------------------------
# CPU baselines (the reference built from its sources, or the oracle port)
# ---------------------------------------------------------------------------
REF_EXE = os.path.join(ROOT, "oracle", "_ref", "oneflow_ref")
ORACLE_SO = os.path.join(ROOT, "oracle", "liboforacle.so")


def reference_colour_order(mesh: Mesh):
    """The colour-major renumbering (perm[new] = old) from the oracle
    library, so that a reference run loads none of the product's code."""
    import ctypes as C
    L = C.CDLL(ORACLE_SO)
    ip = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
    L.oro_colour_order.argtypes = [C.c_int, C.c_int, C.c_int, ip, ip, ip]
    perm = np.zeros(mesh.n_cells, np.int32)
    n = L.oro_colour_order(mesh.n_cells, mesh.n_faces, mesh.n_bfaces, np.ascontiguousarray(mesh.lc, np.int32),
                           np.ascontiguousarray(mesh.rc, np.int32), perm)
    if n < 1:
        raise RuntimeError("oro_colour_order failed")
    return perm


def _run_dirs(mesh, prm, steps, n, dump=False):
    """One reference project written once (grid, scripts), and n run
    directories whose case shares its grid and scripts; returns (base, dirs)."""
    import shutil
    base = tempfile.mkdtemp(prefix="ofgref_")
    write_case(os.path.join(base, "case"), mesh, P.to_dict(prm), steps)
    dirs = []
    for i in range(n):
        case = os.path.join(base, f"run{i}", "case")
        os.makedirs(case)
        shutil.copytree(os.path.join(base, "case", "script"), os.path.join(case, "script"))
        os.symlink(os.path.join(base, "case", "grid"), os.path.join(case, "grid"))
        for sub in ("results", "restart", "visual", "log"):
            os.makedirs(os.path.join(case, sub))
        dirs.append(os.path.dirname(case))
    return base, dirs


def reference_timed(mesh, prm, warm: int, timed: int, nproc: int, dump: bool = False):
    """The reference CPU solver (built from its own sources) on `mesh`:
    nproc concurrent single-rank solves of warm + timed outer iterations.
    Each iteration's wall time is read from when its last residual line
    appears on the process's line-buffered stdout (the reference prints one
    line per solver per iteration), so set-up is excluded without a second
    run.  Returns (aggregate cell-iter/s, seconds per iteration (median over
    the processes), wall seconds of the whole run, the full-precision dump of
    process 0 or None)."""
    import shutil
    base, dirs = _run_dirs(mesh, prm, warm + timed, nproc)
    cmd = ([shutil.which("stdbuf"), "-oL"] if shutil.which("stdbuf") else []) + [REF_EXE, "0", "case"]
    stamps = [dict() for _ in dirs]
    t0 = time.perf_counter()
    procs = []
    for i, d in enumerate(dirs):
        env = dict(os.environ)
        if dump and i == 0:
            env["OFG_REF_DUMP"] = os.path.join(d, "dump.bin")
        procs.append(subprocess.Popen(cmd, cwd=d, env=env, stdout=subprocess.PIPE, stderr=subprocess.STDOUT))

    def reader(p, st):
        for line in p.stdout:
            f = line.split()
            if len(f) >= 3 and f[0].isdigit() and f[1].isdigit():
                st[int(f[0])] = time.perf_counter()

    ths = [threading.Thread(target=reader, args=(p, st), daemon=True) for p, st in zip(procs, stamps)]
    for t in ths:
        t.start()
    rcs = [p.wait() for p in procs]
    for t in ths:
        t.join(timeout=10)
    wall = time.perf_counter() - t0
    if any(rcs):
        shutil.rmtree(base, ignore_errors=True)
        raise RuntimeError(f"reference run failed: {rcs}")
    per = []
    for st in stamps:
        if warm in st and warm + timed in st:
            per.append((st[warm + timed] - st[warm]) / timed)
    if len(per) != len(dirs):
        shutil.rmtree(base, ignore_errors=True)
        raise RuntimeError("reference iterations not seen on stdout")
    out = None
    if dump:
        from oneflow_b200.meshio import read_ref_dump
        out = read_ref_dump(os.path.join(dirs[0], "dump.bin"))
    shutil.rmtree(base, ignore_errors=True)
    return sum(mesh.n_cells / t for t in per), statistics.median(per), wall, out


def reference_options(prm):
    """The reference's closest options to a configuration: it has only the
    Green-Gauss gradient and its own Venkatakrishnan eps (vencat_coef *
    max(qmax - qmin, 1)), so least squares and eps^2 = (K h)^3 fall back to
    those; precision is its FP64.  Returns (params, note or None)."""
    q = P.defaults(**P.to_dict(prm))
    q.precision = 0
    notes = []
    if q.igrad == 2:
        q.igrad = 0
        notes.append("Green-Gauss gradients in place of least squares")
    if q.ilim == 2 and q.venkat_kh3:
        q.venkat_kh3 = 0
        notes.append("the reference's Venkatakrishnan eps in place of eps^2=(K h)^3")
    return q, ("; ".join(notes) + " (the reference has no such option)") if notes else None


def oracle_port_throughput(mesh, prm, n1, n2):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_lib import Oracle
    o = Oracle(mesh, prm)
    o.init()
    t0 = time.perf_counter(); o.step(n1); t1 = time.perf_counter(); o.step(n2 - n1); t2 = time.perf_counter()
    return mesh.n_cells / ((t2 - t1) / (n2 - n1)), (t2 - t1) / (n2 - n1)


# ---------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--config", default="plate3d")
    ap.add_argument("--impl", default="ofg", choices=["ofg", "reference"])
    ap.add_argument("--ordering", default="colour", choices=["natural", "colour"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-converge", action="store_true", help="skip the time-to-1e-8-drop runs")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched airfoil runs")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned warm-start experiment")
    ap.add_argument("--no-pinned", action="store_true", help="skip the reference-options variant of the workload")
    ap.add_argument("--no-c1", action="store_true", help="skip the benchmark-size 2-D bump")
    ap.add_argument("--no-tune", action="store_true", help="keep the default launch shapes (no autotuner)")
    ap.add_argument("--no-wing", action="store_true", help="skip the 8M-cell transonic swept wing")
    ap.add_argument("--no-uins", action="store_true", help="skip the incompressible cavity")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    if args.impl == "reference":
        if rank != 0:
            return
        if not os.path.exists(REF_EXE):
            print(json.dumps({"impl": "reference", "unavailable": "reference CPU solver not built (oracle/_ref)"}))
            return
        # the reference solver on the workload itself (its own mesh, renumbered
        # as the GPU sweeps it): nproc concurrent single-rank solves, as many as
        # host memory holds; one untimed iteration, then a few timed ones (each
        # takes tens of seconds on one core at 6M cells)
        mesh, prm, desc = make_workload(args.config)
        st = mesh_stats(mesh)
        prm_ref, note = reference_options(prm)
        if args.ordering == "colour":
            mesh = mesh.renumber_cells(reference_colour_order(mesh))
        nproc = _ref_procs(mesh)
        warm, timed = 1, max(1, min(args.steps, 3))
        thr, per_iter, wall, _ = reference_timed(mesh, prm_ref, warm, timed, nproc)
        sample = (f"{nproc} concurrent single-rank solves of the reference CPU solver (built from its sources) on "
                  f"the workload's {mesh.n_cells:,}-cell mesh, {warm} untimed + {timed} timed outer iterations each; "
                  f"wall time per iteration from the processes' line-buffered residual output (median over the "
                  f"processes); precomputed wall distance" + (f"; {note}" if note else ""))
        line = {"metric": "cell-iters/s", "value": thr, "unit": "cell-iter/s", "impl": "reference",
                "n_gpus": args.gpus, "steps": timed, "warmup": warm,
                "ms_per_step": per_iter * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64", "data": "synthetic (seeded mesh generator)",
                "config": bench_config(desc, st, args.ordering, world,
                                       sum(alg_bytes(st, prm).values()) < 2 * L2_BYTES),
                "cpu_baseline": {"value": thr, "unit": "cell-iter/s", "cores": nproc, "kind": "reference",
                                 "sample": sample, "run_wall_s": wall},
                "e2e": {"value": thr, "unit": "cell-iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    mesh, prm, desc = make_workload(args.config)

    import torch
    from oneflow_b200 import Solver, colour_order
    dev = local if world > 1 else 0
    torch.cuda.set_device(dev)
    # colour ordering: the LU-SGS sweeps run in colour-major order (identical to
    # the reference solving the mesh renumbered by ofg_colour_order) while the
    # cells stay stored in the generator's spatial order
    prm.sweep_order = 1 if args.ordering == "colour" else 0
    st = mesh_stats(mesh)
    stream = torch.cuda.current_stream()
    s = Solver(mesh, prm)
    s.set_stream(stream.cuda_stream)
    s.init_flowfield()
    # CALC_WALL_DIST on the GPU (exact point-to-wall-face distance of every
    # cell centre), timed once; it replaces the closed-form plate distance the
    # mesh came with, and the timed steps use it
    t0 = time.perf_counter()
    s.calc_wall_dist()
    wall_s = time.perf_counter() - t0
    wall_err = None
    if mesh.wall_dist is not None:
        wd = s.field("walldist")[:st["N"]]
        wall_err = float(np.abs(wd - mesh.wall_dist).max() / np.abs(mesh.wall_dist).max())
    for _ in range(args.warmup):
        s.step(1)
    # launch shapes of the gather kernels picked by the autotuner on this mesh
    tuning = s.autotune() if not args.no_tune else s.tuning()
    s.step(1)
    torch.cuda.synchronize()
    abytes = alg_bytes(st, prm)
    working = sum(abytes.values())
    flush = working < 2 * L2_BYTES
    scratch = torch.empty(int(2 * L2_BYTES // 4), dtype=torch.float32, device="cuda") if flush else None
    _, l0 = s.counters()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev = []
    with ClockSampler(dev) as clk:
        if flush:
            total_ms = 0.0
            for _ in range(args.steps):
                scratch.fill_(1.0)          # write > L2 between timed steps
                a = torch.cuda.Event(enable_timing=True); b = torch.cuda.Event(enable_timing=True)
                a.record(stream); s.step(1); b.record(stream)
                ev.append((a, b))
            torch.cuda.synchronize()
            total_ms = sum(a.elapsed_time(b) for a, b in ev)
        else:
            a = torch.cuda.Event(enable_timing=True); b = torch.cuda.Event(enable_timing=True)
            a.record(stream); s.step(args.steps); b.record(stream)
            torch.cuda.synchronize()
            total_ms = a.elapsed_time(b)
    _, l1 = s.counters()
    torch.cuda.synchronize()
    total_ms, value = replica_aggregate(total_ms, st["N"], args.steps, world, dist)

    # per-group device times (task-by-task launch with events) for the roofline
    prof = []
    for _ in range(3):
        if flush:
            scratch.fill_(1.0)
        prof.append(s.profile_step())
    grp_ms = {k: statistics.median(p[0][k] for p in prof) for k in prof[0][0]}
    grp_n = prof[0][1]
    top = max((k for k in grp_ms if k != "cfl"), key=lambda k: grp_ms[k])
    hbm = _peak_hbm()
    per_launch_ms = grp_ms[top] / max(grp_n[top], 1)
    achieved = abytes[top] / (grp_ms[top] * 1e-3) / 1e9   # GB/s over the group's launches
    tpc = NCU_TRAFFIC_PER_CELL.get((args.config, top))
    traffic = tpc * st["N"] / max(grp_n[top], 1) if tpc else None
    roofline = {"bound": "hbm", "kernel": KERNEL_OF_GROUP.get(top, top), "group": top, "achieved": achieved,
                "peak": hbm["value"], "unit": "GB/s", "frac": achieved / hbm["value"], "traffic": traffic,
                "traffic_source": "ncu dram bytes per cell on the 600k-cell sample, scaled by cells" if tpc else None,
                "peak_source": hbm["source"],
                "alg_bytes_per_step": abytes[top], "launches_per_step": grp_n[top],
                "avg_launch_ms": per_launch_ms,
                "whole_step_achieved_gbs": working / (total_ms / args.steps * 1e-3) / 1e9,
                "whole_step_frac": working / (total_ms / args.steps * 1e-3) / 1e9 / hbm["value"],
                "contract_bytes_per_cell": CONTRACT_BYTES.get(args.config),
                "whole_step_frac_contract": (CONTRACT_BYTES[args.config] * st["N"] /
                                                    (total_ms / args.steps * 1e-3) / 1e9 / hbm["value"])
                if args.config in CONTRACT_BYTES else None,
                "group_ms": grp_ms, "group_alg_bytes": abytes}

    # end to end through the C ABI with host buffers: every step uploads the
    # state q[5][nCells+nBFaces] from pinned host memory (the reference's field
    # layout), runs one outer iteration and reads the new state back
    e2e_steps = max(3, min(args.steps, 10))
    qh = torch.empty((5, s.nT), dtype=torch.float64, pin_memory=True).numpy()
    s.state(out=qh)
    h2d = qh.nbytes
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        s.upload_state(qh)
        s.step(1)
        s.state(out=qh)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_val = st["N"] * e2e_steps * world / e2e_s
    if dist:
        t = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_val = st["N"] * e2e_steps * world / float(t.item())

    cpu = parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu, parity = parity_and_cpu_baseline(args.config, args.ordering, stream)
    pinned = None
    if rank == 0 and world == 1 and not args.no_pinned and args.config in _SAMPLE:
        pinned = pinned_variant(mesh, prm, stream, min(args.steps, 50), args.warmup)
    c1 = None
    if rank == 0 and world == 1 and not args.no_c1:
        c1 = config1_throughput(stream)
    wing = None
    if rank == 0 and world == 1 and not args.no_wing:
        wing = config3_wing(stream, args.ordering)
    uins = None
    if rank == 0 and world == 1 and not args.no_uins:
        uins = uins_cavity()
    conv = None
    if rank == 0 and world == 1 and not args.no_converge:
        conv = time_to_drop("bump2d_small", 1e-8, stream)
    batched = None
    if rank == 0 and world == 1 and not args.no_batched:
        batched = batched_throughput()
    learned = learned_af = None
    if rank == 0 and world == 1 and not args.no_learned:
        from oneflow_b200 import warmstart
        learned = warmstart.run_experiment()
        learned_af = warmstart.run_experiment(family="airfoil")

    clocks = clk.summary()
    if rank == 0:
        line = {"metric": "cell-iters/s", "value": value, "unit": "cell-iter/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64" if prm.precision == 0 else "f32/f64",
                "data": "synthetic (seeded mesh generator)",
                "config": bench_config(desc, st, args.ordering, world, flush),
                "sweep_levels": list(s.sweep_levels()), "tuning": tuning,
                "roofline": roofline, "cpu_baseline": cpu, "parity": parity, "pinned_variant": pinned,
                "config1_bump2d": c1, "config3_wing": wing, "uins_cavity": uins,
                "e2e": {"value": e2e_val, "unit": "cell-iter/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d},
                "gpu_launches": int(l1 - l0), "clocks": clocks, "time_to_1e-8": conv,
                "setup": {"calc_wall_dist_s": wall_s, "wall_dist_vs_closed_form": wall_err},
                "batched": batched, "learned_warm_start": learned,
                "learned_warm_start_airfoils": learned_af}
        print(json.dumps(line))
    if dist:
        dist.barrier()
        s.close()
        dist.destroy_process_group()


def replica_aggregate(total_ms, cells, steps, world, dist):
    """Independent replicas (one solve per GPU, no data-path collective): the
    job time is the slowest rank's device time, and the whole-job throughput
    counts every rank's cell-iterations.  Returns (max ms, cell-iter/s)."""
    if dist is not None and world > 1:
        import torch
        dev = "cuda" if torch.cuda.is_available() and dist.get_backend() == "nccl" else "cpu"
        t = torch.tensor([float(total_ms)], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        dist.barrier()
    return total_ms, cells * steps * world / (total_ms * 1e-3)


def batched_throughput(n_cases: int = 64, steps: int = 100, warmup: int = 3, reps: int = 5):
    """The batched configuration: 64 seeded 2-D RANS-SA airfoil solves of
    uneven sizes (20k-400k cells, 7.9M in all), advanced (a) one after
    another, each by its own graph launches, and (b) together by one batch
    graph launch per iteration.  Device time with CUDA events: (a) the sum over
    the solves of the events around each one's iterations on one stream, (b)
    the batch's own events around its graph launches.  The `steps` timed
    iterations are taken as `reps` runs of steps / reps, each from the free
    stream after `warmup` untimed iterations: the second-order airfoil cases do
    not converge, and a few of the 64 blow up within about a hundred
    iterations."""
    import torch
    from oneflow_b200 import Batch, Solver
    cases = meshgen.airfoil_cases(n_cases)
    stream = torch.cuda.Stream()
    ss = []
    for mesh, fs in cases:
        s = Solver(mesh, P.rans_airfoil(**fs))
        s.set_stream(stream.cuda_stream)
        s.init_flowfield()
        ss.append(s)
    cells = sum(m.n_cells for m, _ in cases)
    tunes = []
    for s in ss:
        s.step(warmup)
        tunes.append(s.autotune())   # per mesh: launch shapes timed on its own cells
    torch.cuda.synchronize()
    per = steps // reps
    seq_ms = 0.0
    for _ in range(reps):
        for s in ss:
            s.init_flowfield()
            s.step(warmup)
        for s in ss:
            a = torch.cuda.Event(enable_timing=True); e = torch.cuda.Event(enable_timing=True)
            a.record(stream); s.step(per); e.record(stream)
            e.synchronize()
            seq_ms += a.elapsed_time(e)
    b = Batch(ss)
    bat_ms = 0.0
    for _ in range(reps):
        for s in ss:
            s.init_flowfield()
        b.step(warmup)
        b.step(per)
        bat_ms += b.device_ms()
    b.close()
    for s in ss:
        s.close()
    timed = per * reps
    return {"workload": f"{n_cases} 2-D RANS-SA NACA 4-digit airfoils, hybrid O-grids of "
                        f"{min(m.n_cells for m, _ in cases):,}-{max(m.n_cells for m, _ in cases):,} cells, "
                        "Mach 0.3-0.8, AoA -2..8 deg, Re 1e6-1e7 (seeded); Roe 2nd order Green-Gauss + Venkatakrishnan, "
                        "SA, LU-SGS, FP32 faces",
            "cells": cells, "steps": timed, "runs": reps, "warmup_per_run": warmup, "unit": "cell-iter/s",
            "sequential": cells * timed / (seq_ms * 1e-3), "batched": cells * timed / (bat_ms * 1e-3),
            "sequential_ms_per_step": seq_ms / timed, "batched_ms_per_step": bat_ms / timed,
            "autotuner": {"tuned_ms_sum": sum(t["ms_tuned"] for t in tunes),
                          "default_ms_sum": sum(t["ms_default"] for t in tunes),
                          "choices": {k: {str(v): sum(1 for t in tunes if t[k] == v) for v in sorted({t[k] for t in tunes})}
                                      for k in ("face_min_blocks", "face_block", "grad_min_blocks", "grad_block",
                                                "sweep_min_blocks", "sweep_block", "sweep_persistent")}},
            "timing": "CUDA events on the launching stream: sequential = sum over the solves, batched = around the "
                      f"batch's graph launches; {reps} runs of {per} iterations, each from the free stream after "
                      f"{warmup} untimed iterations"}


def time_to_drop(config: str, target: float, stream, chunk: int = 200, max_iters: int = 40000):
    """Device time for the RMS density residual to fall by `target` relative
    to the first iteration, from a cold (free-stream) start, on the FP64 and
    the FP32-face paths: steps in chunks of `chunk` iterations (CUDA events
    around each chunk), the crossing iteration read from the residual history;
    the time of the last chunk is prorated to that iteration."""
    import torch
    from oneflow_b200 import Solver
    mesh, prm0, desc = make_workload(config)
    out = {"workload": desc["workload"], "cells": mesh.n_cells, "target_drop": target}
    for key, prec in (("f64", 0), ("f32_faces", 1)):
        prm = make_workload(config)[1]
        prm.precision = prec
        prm.sweep_order = 1          # colour-major sweeps, as in the throughput runs
        s = Solver(mesh, prm)
        s.set_stream(stream.cuda_stream)
        s.init_flowfield()
        total, done, hit = 0.0, 0, None
        while done < max_iters and hit is None:
            a = torch.cuda.Event(enable_timing=True); b = torch.cuda.Event(enable_timing=True)
            a.record(stream); s.step(chunk); b.record(stream)
            torch.cuda.synchronize()
            ms = a.elapsed_time(b)
            h = s.res_history()[:, 0]
            below = np.nonzero(h[done:done + chunk] / h[0] <= target)[0]
            if below.size:
                hit = done + int(below[0]) + 1
                total += ms * (below[0] + 1) / chunk
            else:
                total += ms
            done += chunk
        h = s.res_history()[:, 0]
        out[key] = {"iterations": hit, "seconds": total * 1e-3 if hit else None,
                    "final_drop": float(h[-1] / h[0]), "iterations_run": done}
        s.close()
    return out


def _rel_l2(a, b) -> float:
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


FORCE_KEYS = [0, 1, 2, 9, 10]   # Fx Fy Fz CL CD of Solver.forces / the reference's dump


def _force_err(f, fr) -> float:
    f, fr = np.asarray(f)[FORCE_KEYS], np.asarray(fr)[FORCE_KEYS]
    return float(np.abs(f - fr).max() / max(np.abs(fr).max(), 1e-300))


def parity_and_cpu_baseline(config: str, ordering: str, stream, steps: int = 12):
    """Parity of the benchmarked path against the reference, and the CPU
    baseline, from one run of the reference solver (built from its sources,
    one process on one core) on the 600,000-cell sample of the workload with
    the reference's own gradient and limiter options (Green-Gauss, its
    Venkatakrishnan eps: the options whose parity the reference pins).  The
    GPU runs the same mesh and options for the same number of iterations on
    both paths; the reference sweeps the mesh renumbered in the colour-major
    order, which is what the GPU's colour-major sweep computes, and its fields
    are mapped back to the storage order.  Returns (cpu_baseline, parity)."""
    from oneflow_b200 import Solver
    from oneflow_b200.solver import TURB_SOLVER
    sample = _SAMPLE.get(config, config)
    mesh, prm, desc = make_workload(sample)
    prm_ref, note = reference_options(prm)
    N = mesh.n_cells
    if not os.path.exists(REF_EXE):
        thr, per_iter = oracle_port_throughput(mesh, prm_ref, 2, 4)
        return ({"value": thr, "unit": "cell-iter/s", "cores": 1, "kind": "port",
                 "sample": f"CPU restatement, 1 thread, {N:,}-cell sample, 2 iterations (reference build absent)"},
                None)
    perm = reference_colour_order(mesh) if ordering == "colour" else np.arange(N)
    rmesh = mesh.renumber_cells(perm) if ordering == "colour" else mesh
    thr, per_iter, wall, dump = reference_timed(rmesh, prm_ref, 1, steps - 1, 1, dump=True)
    cpu = {"value": thr, "unit": "cell-iter/s", "cores": 1, "kind": "reference",
           "sample": f"reference CPU solver (built from its sources), 1 process on 1 core, the {N:,}-cell sample of "
                     f"the workload ({desc['workload'].split(':')[0]}), iterations 2-{steps} timed from its "
                     f"line-buffered residual output" + (f"; {note}" if note else "")}

    def ref_field(name, e=0):
        out = np.empty(N)
        out[perm] = dump[name][e, :N]
        return out

    ref = {"rho": ref_field("q", 0), "p": ref_field("q", 4), "forces": dump["forces"].ravel()[:13]}
    sa = prm.vismodel >= 3
    if sa:
        ref["nut"] = ref_field("turbq")
        ref["vist"] = ref_field("vist")
    out = {"workload": f"{N:,}-cell sample of the workload, the reference's options: "
                       + (note or "as configured"), "steps": steps,
           "tolerance": {"forces_rel": 1e-6, "field_rel_l2": 1e-5},
           "reference_forces": {"CL": float(ref["forces"][9]), "CD": float(ref["forces"][10])}}
    got = {}
    for key, prec in (("fp64", 0), ("mixed", 1)):
        q = P.defaults(**P.to_dict(prm_ref))
        q.precision = prec
        q.sweep_order = 1 if ordering == "colour" else 0
        s = Solver(mesh, q)
        s.set_stream(stream.cuda_stream)
        s.init_flowfield()
        s.step(steps)
        st = s.state()
        g = {"rho": st[0, :N], "p": st[4, :N], "forces": s.forces(1.0)}
        if sa:
            g["nut"] = s.state(TURB_SOLVER)[:N]
            g["vist"] = s.field("vist")[:N]
        got[key] = g
        r = {"rho_l2": _rel_l2(g["rho"], ref["rho"]), "p_l2": _rel_l2(g["p"], ref["p"]),
             "forces_rel": _force_err(g["forces"], ref["forces"]),
             "CL": float(g["forces"][9]), "CD": float(g["forces"][10])}
        if sa:
            r["nut_l2"] = _rel_l2(g["nut"], ref["nut"])
            r["mu_t_l2"] = _rel_l2(g["vist"], ref["vist"])
        out[f"{key}_vs_reference"] = r
        s.close()
    a, b = got["mixed"], got["fp64"]
    out["mixed_vs_fp64"] = {"rho_l2": _rel_l2(a["rho"], b["rho"]), "p_l2": _rel_l2(a["p"], b["p"]),
                            "forces_rel": _force_err(a["forces"], b["forces"])}
    if sa:
        out["mixed_vs_fp64"]["nut_l2"] = _rel_l2(a["nut"], b["nut"])
        out["mixed_vs_fp64"]["mu_t_l2"] = _rel_l2(a["vist"], b["vist"])
    return cpu, out


def _timed_steps(s, stream, steps: int, flush_buf=None) -> float:
    """Device ms of `steps` outer iterations on the solver's stream (CUDA
    events); with flush_buf, a write larger than L2 before every step, each
    step timed alone."""
    import torch
    if flush_buf is None:
        a = torch.cuda.Event(enable_timing=True); b = torch.cuda.Event(enable_timing=True)
        a.record(stream); s.step(steps); b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b)
    ev = []
    for _ in range(steps):
        flush_buf.fill_(1.0)
        a = torch.cuda.Event(enable_timing=True); b = torch.cuda.Event(enable_timing=True)
        a.record(stream); s.step(1); b.record(stream)
        ev.append((a, b))
    torch.cuda.synchronize()
    return sum(a.elapsed_time(b) for a, b in ev)


def pinned_variant(mesh, prm, stream, steps: int, warmup: int):
    """The workload's mesh on the benchmarked (mixed) path with the reference's
    own gradient and limiter options -- the variant `parity` pins against the
    reference -- timed like the main line."""
    from oneflow_b200 import Solver
    q, note = reference_options(prm)
    q.precision = prm.precision
    q.sweep_order = prm.sweep_order
    s = Solver(mesh, q)
    s.set_stream(stream.cuda_stream)
    s.init_flowfield()
    s.step(warmup)
    ms = _timed_steps(s, stream, steps)
    s.close()
    return {"options": note, "value": mesh.n_cells * steps / (ms * 1e-3), "unit": "cell-iter/s",
            "ms_per_step": ms / steps, "steps": steps, "warmup": warmup}


def config3_wing(stream, ordering: str, steps: int = 20, warmup: int = 5, parity_steps: int = 3):
    """The transonic swept-wing configuration: the 8.0M-cell hybrid mesh
    (hexahedral boundary layer, tetrahedral far field) on the mixed path --
    cell-iter/s, the per-kernel profile and the dominant kernel's roofline --
    and parity on its 0.8M-cell sample (the same generator, coarser) against
    the reference solver run for parity_steps iterations on the same mesh, with
    the wall distance computed on the GPU and passed to it."""
    import torch
    from oneflow_b200 import Solver
    from oneflow_b200.solver import TURB_SOLVER
    mesh, prm, desc = make_workload("wing3d")
    prm.sweep_order = 1 if ordering == "colour" else 0
    st = mesh_stats(mesh)
    s = Solver(mesh, prm)
    s.set_stream(stream.cuda_stream)
    s.init_flowfield()
    s.step(warmup)
    tuning = s.autotune()
    ms = _timed_steps(s, stream, steps)
    prof = s.profile_step()
    grp_ms, grp_n = prof
    ab = alg_bytes(st, prm)
    top = max((k for k in grp_ms if k != "cfl"), key=lambda k: grp_ms[k])
    hbm = _peak_hbm()
    achieved = ab[top] / (grp_ms[top] * 1e-3) / 1e9
    out = {"workload": desc["workload"], "cells": st["N"], "faces": st["F"], "steps": steps, "warmup": warmup,
           "value": st["N"] * steps / (ms * 1e-3), "unit": "cell-iter/s", "ms_per_step": ms / steps,
           "sweep_levels": list(s.sweep_levels()), "tuning": tuning,
           "roofline": {"bound": "hbm", "kernel": KERNEL_OF_GROUP.get(top, top), "achieved": achieved,
                        "peak": hbm["value"], "unit": "GB/s", "frac": achieved / hbm["value"],
                        "whole_step_frac": sum(ab.values()) / (ms / steps * 1e-3) / 1e9 / hbm["value"],
                        "group_ms": grp_ms}}
    s.close()
    # parity on the sample: FP64 and mixed paths against the reference
    smesh, sprm, sdesc = make_workload("wing3d_sample")
    g = Solver(smesh, P.defaults(**{**P.to_dict(sprm), "precision": 0, "sweep_order": 0}))
    g.init_flowfield()
    smesh.wall_dist = g.field("walldist")[:smesh.n_cells].copy()    # CALC_WALL_DIST on the GPU
    g.close()
    N = smesh.n_cells
    par = {"sample_cells": N, "steps": parity_steps, "tolerance": {"forces_rel": 1e-6, "field_rel_l2": 1e-5}}
    if os.path.exists(REF_EXE):
        rprm = P.defaults(**{**P.to_dict(sprm), "precision": 0, "sweep_order": 0})
        thr, per_iter, wall, dump = reference_timed(smesh, rprm, 1, parity_steps - 1, 1, dump=True)
        ref = {"rho": dump["q"][0, :N], "p": dump["q"][4, :N], "nut": dump["turbq"][0, :N],
               "forces": dump["forces"].ravel()[:13]}
        par["reference_cell_iter_s_1core"] = thr
        for key, prec in (("fp64", 0), ("mixed", 1)):
            q = P.defaults(**{**P.to_dict(sprm), "precision": prec, "sweep_order": 0})
            gs = Solver(smesh, q)
            gs.set_stream(stream.cuda_stream)
            gs.init_flowfield()
            gs.step(parity_steps)
            stt = gs.state()
            f = gs.forces(1.0)
            par[f"{key}_vs_reference"] = {"rho_l2": _rel_l2(stt[0, :N], ref["rho"]), "p_l2": _rel_l2(stt[4, :N], ref["p"]),
                                          "nut_l2": _rel_l2(gs.state(TURB_SOLVER)[:N], ref["nut"]),
                                          "forces_rel": _force_err(f, ref["forces"]),
                                          "CL": float(f[9]), "CD": float(f[10])}
            gs.close()
        par["reference_forces"] = {"CL": float(ref["forces"][9]), "CD": float(ref["forces"][10])}
    out["parity"] = par
    return out


def config1_throughput(stream, steps: int = 200, warmup: int = 5):
    """The 2-D Euler bump at its benchmark size (65,536 triangles, first-order
    Roe, LU-SGS, CFL 5): cell-iter/s on the FP64 path sweeping in the
    reference's cell order, and on the mixed path with colour-major sweeps.
    Its working set (about 40 MB) fits L2, so L2 is flushed before every
    timed step."""
    import torch
    from oneflow_b200 import Solver
    mesh, prm0, desc = make_workload("bump2d")
    flush = torch.empty(int(2 * L2_BYTES // 4), dtype=torch.float32, device="cuda")
    out = {"workload": desc["workload"], "cells": mesh.n_cells, "steps": steps,
           "l2": "flushed before every timed step"}
    for key, prec, order in (("fp64_reference_order", 0, 0), ("mixed_colour_order", 1, 1)):
        q = P.defaults(**P.to_dict(prm0))
        q.precision = prec
        q.sweep_order = order
        s = Solver(mesh, q)
        s.set_stream(stream.cuda_stream)
        s.init_flowfield()
        s.step(warmup)
        tuning = s.autotune()     # the sweep schedule (persistent or level launches), and the mixed shapes
        ms = _timed_steps(s, stream, steps, flush)
        out[key] = {"value": mesh.n_cells * steps / (ms * 1e-3), "ms_per_step": ms / steps,
                    "sweep_levels": list(s.sweep_levels()), "tuning": tuning}
        s.close()
    # parity at the config's own length: 2,000 iterations in the reference's
    # cell order against the reference's run of the same case (the committed
    # fixture tests/golden/bump2d_c1.npz: every 16th cell, forces)
    gold = np.load(os.path.join(ROOT, "tests", "golden", "bump2d_c1.npz"))
    stride, n_it = 16, int(gold["steps"])
    par = {"iterations": n_it, "against": "the reference CPU solver's run of the same mesh (every 16th cell, forces)"}
    for key, prec in (("fp64", 0), ("mixed", 1)):
        q = P.defaults(**P.to_dict(prm0))
        q.precision = prec
        q.sweep_order = 0
        s = Solver(mesh, q)
        s.set_stream(stream.cuda_stream)
        s.init_flowfield()
        s.step(n_it)
        st = s.state()[:, :mesh.n_cells][:, ::stride]
        f = s.forces(1.0)
        par[key] = {"rho_l2": _rel_l2(st[0], gold["q_sub"][0]), "p_l2": _rel_l2(st[4], gold["q_sub"][4]),
                    "forces_rel": _force_err(f, gold["forces"])}
        s.close()
    out["parity"] = par
    return out


def uins_cavity(n: int = 512, inner: int = 4, sample_n: int = 128, parity_n: int = 64, parity_inner: int = 3):
    """The incompressible solver (the reference's INsSolver with the SIMPLE
    time integral: momentum and pressure-correction GMRES solves, Krylov
    dimension 500) on a lid-driven cavity (unit square, jittered quads, lid
    at u = 1, Re 1000, dt 0.001).  GPU: inner iterations of an n x n cavity
    from the initial state (device time by CUDA events, GMRES steps and their
    roofline).  Same-mesh comparison on a sample_n x sample_n cavity: the GPU
    against the reference CPU solver (oracle/_ref, one core; per inner
    iteration = the difference of a 1- and a 2-iteration run).  Parity: the
    GPU against the CPU restatement (bitwise the reference) after
    parity_inner iterations of a parity_n x parity_n cavity."""
    from oneflow_b200 import Incompressible
    prm = P.defaults(vismodel=1, reynolds=1000.0, mach_ref=0.1)
    out = {"workload": f"lid-driven cavity {n}x{n} quads (jitter 0.1), Re 1000, dt 0.001, FP64"}

    def gpu_run(m, k):
        g = Incompressible(m, prm, meshgen.lid_velocity(m))
        g.run(2)                      # warm (first-step initialisation, allocations)
        g.init_flowfield()
        its = []
        for _ in range(k):
            g.update_residuals()
            its.append([int(v) for v in g.stats()["gmres_iters"]])
        t = g.timing()
        return g, t, its

    mesh = meshgen.lid_cavity_2d(n, jitter=0.1)
    g, t, its = gpu_run(mesh, inner)
    hbm = _peak_hbm()
    gbs = t["gmres_bytes"] / (t["gmres_ms"] * 1e-3) / 1e9
    out.update({"cells": mesh.n_cells, "inner_iterations": inner, "ms_per_inner": t["ms"] / inner,
                "value": mesh.n_cells * inner / (t["ms"] * 1e-3), "unit": "cell-iter/s",
                "gmres_iters_per_inner": its, "gmres_share_of_time": t["gmres_ms"] / t["ms"],
                "krylov_steps_per_s": t["gmres_iters"] / (t["gmres_ms"] * 1e-3),
                "roofline": {"bound": "hbm", "kernel": "k_gm_spmv_dots + k_gm_orth (GMRES)", "achieved": gbs,
                             "peak": hbm["value"], "unit": "GB/s", "frac": gbs / hbm["value"],
                             "peak_source": hbm["source"], "alg_bytes": t["gmres_bytes"]}})
    g.close()
    # same mesh, GPU and the reference CPU solver
    sm = meshgen.lid_cavity_2d(sample_n, jitter=0.1)
    gs, ts, _ = gpu_run(sm, 2)
    gs.close()
    cmp = {"mesh": f"{sample_n}x{sample_n} quads", "cells": sm.n_cells, "gpu_ms_per_inner": ts["ms"] / 2}
    if os.path.exists(REF_EXE):
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from oracle_lib import run_ref_ins
        wall = []
        for k in (1, 2):
            t0 = time.perf_counter()
            run_ref_ins(sm, prm, 1.0, k)
            wall.append(time.perf_counter() - t0)
        cpu_s = wall[1] - wall[0]
        cmp.update({"reference_cpu_s_per_inner": cpu_s, "cores": 1, "kind": "reference",
                    "gpu_speedup": cpu_s / (ts["ms"] / 2 * 1e-3)})
    out["same_mesh_vs_reference"] = cmp
    # parity against the restatement
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_lib import InsOracle
    pm = meshgen.lid_cavity_2d(parity_n, jitter=0.1)
    w = meshgen.lid_velocity(pm)
    gp = Incompressible(pm, prm, w)
    gp.run(parity_inner)
    o = InsOracle(pm, prm, w)
    o.run(parity_inner)
    qg, qo = gp.q(), o.q()
    out["parity"] = {"mesh": f"{parity_n}x{parity_n}", "inner": parity_inner,
                     "q_max_rel_err": max(float(np.abs(qg[e] - qo[e]).max() / max(np.abs(qo[e]).max(), 1e-300))
                                          for e in range(5)),
                     "gmres_iters_equal": list(gp.stats()["gmres_iters"]) == list(o.stats()["gmres_iters"])}
    gp.close()
    return out


def _peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return {"value": float(json.load(fh)["hbm_gbs"]), "source": "measured"}
    except Exception:
        return {"value": 6650.0, "source": "fallback"}


if __name__ == "__main__":
    main()

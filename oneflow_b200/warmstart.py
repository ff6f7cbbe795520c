"""Learned warm start of steady solves: a coordinate MLP (BF16 tensor-core
kernels, oneflow_b200.mlp) trained on converged solutions this solver
produced, predicting the initial flow field of a new case.  The cold-started
solve stays the fallback and the arbiter: a warm-started case counts as
converged only when its RMS density residual falls below the same absolute
threshold as the cold start's (the cold start's first residual x 1e-8).

Two case families, each case with its own mesh, so the network sees the
geometry through its inputs:
* BumpFamily: 2-D Euler bump channels (circular-arc bumps of thickness
  4-10 % in a 3 x 1 channel, jittered triangles, Mach 0.3-0.6);
* AirfoilFamily: 2-D Euler flow past NACA 4-digit sections drawn from the
  batched configuration's shape distribution (camber 0-6 % at 40 % chord,
  thickness 8-18 %) on triangle O-grids, Mach 0.3-0.6, AoA -2..6 degrees; 22
  inputs, 16 of them shape features of the section, the others polar
  coordinates about mid-chord, the wall distance and the flow parameters.
Both solve first-order Roe, LU-SGS, colour-major sweeps, FP64."""
from __future__ import annotations

import time

import numpy as np

from . import meshgen, params as P
from .solver import Batch, Solver

GAMMA = 1.4
FEATURES = ("x", "y", "wall_distance", "mach", "thickness", "bump_height_at_x", "y_over_channel", "mach^2")


def bump_cases(n: int, seed: int, ni: int = 64, nj: int = 32):
    """n seeded cases: (mesh, mach, thickness)"""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        t, mach = rng.uniform(0.04, 0.10), rng.uniform(0.3, 0.6)
        mesh = meshgen.bump_channel(ni, nj, thickness=t, seed=int(rng.integers(1 << 31)))
        out.append((mesh, mach, t))
    return out


def case_params(mach: float):
    return P.euler_bump(mach_ref=mach, sweep_order=1)


def features(solver: Solver, mach: float, t: float) -> np.ndarray:
    """[nCells][8] inputs of the network for one case (cell centres, the wall
    distance computed on the GPU, the case parameters, the local bump height)"""
    N = solver.mesh.n_cells
    x, y = solver.field("xcc")[:N], solver.field("ycc")[:N]
    solver.calc_wall_dist()
    d = solver.field("walldist")[:N]
    r = (0.25 + t * t) / (2.0 * t)
    yb = np.where((x > 1.0) & (x < 2.0), np.sqrt(np.maximum(r * r - (x - 1.5) ** 2, 0.0)) - (r - t), 0.0)
    eta = (y - yb) / (1.0 - yb)
    return np.stack([x, y, d, np.full(N, mach), np.full(N, t), yb, eta, np.full(N, mach * mach)], 1)


def targets(q: np.ndarray, mach: float, n_cells: int) -> np.ndarray:
    """[nCells][4] outputs: rho, u, v and p scaled by the free-stream pressure 1/(gamma M^2)"""
    return np.stack([q[0, :n_cells], q[1, :n_cells], q[2, :n_cells], q[4, :n_cells] * GAMMA * mach * mach], 1)


def state_from_prediction(pred: np.ndarray, mach: float, n_t: int) -> np.ndarray:
    """primitive state [5][nT] from a prediction of the interior cells (ghost
    entries start at a valid state and are reset by CALC_BOUNDARY)"""
    n = pred.shape[0]
    q = np.zeros((5, n_t))
    q[0, :n], q[1, :n], q[2, :n] = pred[:, 0], pred[:, 1], pred[:, 2]
    q[4, :n] = pred[:, 3] / (GAMMA * mach * mach)
    q[0] = np.maximum(q[0], 1e-3)
    q[4] = np.maximum(q[4], 1e-3 / (GAMMA * mach * mach))
    q[:, n:] = q[:, :1]
    return q


class BumpFamily:
    """The bump channels: a case is (mesh, mach, thickness)."""
    name = "bump"
    train_steps = 20000
    description = ("2-D Euler bump channels, 64x32 quads -> 4,096 jittered triangles each, bump thickness 4-10 %, "
                   "Mach 0.3-0.6, first-order Roe, LU-SGS, CFL 5, colour-major sweeps, FP64")
    feature_names = FEATURES

    def cases(self, n: int, seed: int):
        return bump_cases(n, seed)

    def params(self, case):
        return case_params(case[1])

    def features(self, solver: Solver, case) -> np.ndarray:
        return features(solver, case[1], case[2])

    def targets(self, q: np.ndarray, case) -> np.ndarray:
        return targets(q, case[1], case[0].n_cells)

    def state(self, pred: np.ndarray, case, n_t: int) -> np.ndarray:
        return state_from_prediction(pred, case[1], n_t)


AIRFOIL_STATIONS = (0.05, 0.1, 0.2, 0.3, 0.4, 0.6, 0.8, 0.95)


def naca4_ordinates(m: float, p: float, t: float, xs) -> np.ndarray:
    """upper and lower surface heights of a NACA 4-digit section at the chord
    stations xs (taken on the camber line): [2 len(xs)] = upper..., lower..."""
    yt, yc, th = meshgen.naca4_parts(m, p, t, xs)
    return np.concatenate([yc + yt * np.cos(th), yc - yt * np.cos(th)])


class AirfoilFamily:
    """Inviscid flow past NACA 4-digit sections on triangle O-grids (96 points
    on the section, 48 layers to a circle of 20 chords, 9,216 cells): a case is
    a dict(mesh, m, t, mach, aoa).  Inputs (22): the log of the distance r from
    mid-chord, the cosine and sine of the polar angle about mid-chord, the log
    of the wall distance, Mach, the angle of attack and 16 shape features --
    the upper and lower surface heights at eight chord stations (polar inputs
    resolve the near field of a domain 40 chords wide better than x and y);
    outputs rho, u, v and p scaled by the free-stream pressure."""
    name = "airfoil"
    description = ("2-D Euler NACA 4-digit sections (camber 0-6 % at 40 % chord, thickness 8-18 %), triangle O-grids "
                   "of 9,216 cells (far field at 20 chords), Mach 0.3-0.6, AoA -2..6 deg, first-order Roe, LU-SGS, "
                   "CFL 20, colour-major sweeps, FP64")
    feature_names = (("log_r", "cos_theta", "sin_theta", "log_wall_distance", "mach", "aoa_deg")
                     + tuple(f"y_upper_{x:g}" for x in AIRFOIL_STATIONS)
                     + tuple(f"y_lower_{x:g}" for x in AIRFOIL_STATIONS))
    train_steps = 20000

    def __init__(self, n_surface: int = 96, n_layers: int = 48):
        self.n_surface, self.n_layers = n_surface, n_layers

    def cases(self, n: int, seed: int):
        rng = np.random.default_rng(seed)
        out = []
        for _ in range(n):
            m, t = rng.uniform(0.0, 0.06), rng.uniform(0.08, 0.18)
            mach, aoa = rng.uniform(0.3, 0.6), rng.uniform(-2.0, 6.0)
            mesh = meshgen.naca_ogrid(m, 0.4, t, self.n_surface, self.n_layers, n_quad_layers=0, y1=2e-3,
                                      radius=20.0)
            out.append(dict(mesh=mesh, m=m, t=t, mach=mach, aoa=aoa))
        return out

    def params(self, case):
        return P.euler_bump(mach_ref=case["mach"], aoa_degree=case["aoa"], cflst=20.0, cfled=20.0, sweep_order=1)

    def features(self, solver: Solver, case) -> np.ndarray:
        N = solver.mesh.n_cells
        dx, dy = solver.field("xcc")[:N] - 0.5, solver.field("ycc")[:N]
        solver.calc_wall_dist()
        d = solver.field("walldist")[:N]
        r = np.sqrt(dx * dx + dy * dy)
        shape = naca4_ordinates(case["m"], 0.4, case["t"], AIRFOIL_STATIONS)
        cols = [np.log(r), dx / r, dy / r, np.log(d + 1e-3), np.full(N, case["mach"]), np.full(N, case["aoa"])]
        cols += [np.full(N, v) for v in shape]
        return np.stack(cols, 1)

    def targets(self, q: np.ndarray, case) -> np.ndarray:
        return targets(q, case["mach"], case["mesh"].n_cells)

    def state(self, pred: np.ndarray, case, n_t: int) -> np.ndarray:
        return state_from_prediction(pred, case["mach"], n_t)


FAMILIES = {"bump": BumpFamily, "airfoil": AirfoilFamily}


def case_mesh(case):
    return case["mesh"] if isinstance(case, dict) else case[0]


def solve_to(solvers, threshold, batch: bool, chunk: int = 200, max_iters: int = 40000):
    """Iterate the solvers until each one's RMS density residual is below its
    threshold.  batch: one Batch for all (every case advances until the last
    converges); else one after another.  Returns (iterations per case, None
    where the limit came first; wall seconds) -- host wall clock around
    synchronous calls."""
    iters = [None] * len(solvers)

    def check(k, s):
        h = s.res_history()[:, 0]
        hit = np.nonzero(h <= threshold[k])[0]
        if hit.size:
            iters[k] = int(hit[0]) + 1

    t0 = time.perf_counter()
    if batch:
        b = Batch(solvers)
        done = 0
        while done < max_iters and any(i is None for i in iters):
            b.step(chunk)
            done += chunk
            for k, s in enumerate(solvers):
                if iters[k] is None:
                    check(k, s)
        b.close()
    else:
        for k, s in enumerate(solvers):
            done = 0
            while done < max_iters and iters[k] is None:
                s.step(chunk)
                done += chunk
                check(k, s)
    return iters, time.perf_counter() - t0


def build_dataset(family, cases, drop: float = 1e-8):
    """Converge every case (batched, cold start) and return the network's
    inputs and outputs over all interior cells of the cases that reached the
    threshold, and the iteration counts (None: not converged, left out)"""
    solvers = []
    for case in cases:
        s = Solver(case_mesh(case), family.params(case))
        s.init_flowfield()
        solvers.append(s)
    first = []
    for s in solvers:   # the first residual of a cold start sets each case's threshold
        s.step(1)
        first.append(s.res_history()[0, 0])
    iters, _ = solve_to(solvers, [f * drop for f in first], batch=True)
    X, Y = [], []
    for case, s, it in zip(cases, solvers, iters):
        if it is not None:
            X.append(family.features(s, case))
            Y.append(family.targets(s.state(), case))
        s.close()
    return np.concatenate(X), np.concatenate(Y), iters


class Normaliser:
    def __init__(self, a: np.ndarray):
        self.mean = a.mean(0)
        self.std = np.maximum(a.std(0), 1e-6)

    def fwd(self, a):
        return (a - self.mean) / self.std

    def inv(self, a):
        return a * self.std + self.mean


def run_experiment(n_train: int = 192, n_test: int = 32, width: int = 256, depth: int = 6, train_steps: int = None,
                   batch: int = 8192, lr: float = 1e-3, seed: int = 20261206, drop: float = 1e-8,
                   family: str = "bump", max_iters: int = 40000, polish_drop: float = 1e-11):
    """Train on n_train converged cases of the family, then solve n_test
    held-out cases to the same absolute threshold four ways: cold one after
    another (the plain solve), cold batched, warm one after another, warm
    batched.  Returns a dict of iterations, wall seconds, the training summary
    and the largest difference of the lift and drag, warm against cold
    (relative to the cold value, or to 1e-3 where that is smaller): at the
    threshold, and after both solves went on (untimed) to the first residual x
    polish_drop, where each has converged to its own steady state."""
    import torch
    from .mlp import MLP
    fam = FAMILIES[family]()
    if train_steps is None:
        train_steps = fam.train_steps
    t0 = time.perf_counter()
    X, Y, train_iters = build_dataset(fam, fam.cases(n_train, seed), drop)
    t_data = time.perf_counter() - t0
    nx, ny = Normaliser(X), Normaliser(Y)
    xd = torch.tensor(nx.fwd(X), dtype=torch.float32, device="cuda").contiguous()
    yd = torch.tensor(ny.fwd(Y), dtype=torch.float32, device="cuda").contiguous()
    net = MLP(X.shape[1], width, depth, Y.shape[1], seed=seed)
    t0 = time.perf_counter()
    losses = net.train(xd, yd, steps=train_steps, batch=batch, lr=lr, seed=seed)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0

    test = fam.cases(n_test, seed + 1)

    def cold():
        ss = []
        for case in test:
            s = Solver(case_mesh(case), fam.params(case))
            s.init_flowfield()
            ss.append(s)
        return ss

    # thresholds from the cold starts' first residuals
    thr = []
    for s in cold():
        s.step(1)
        thr.append(s.res_history()[0, 0] * drop)
        s.close()

    def warm():
        t0 = time.perf_counter()
        ss = []
        for case in test:
            s = Solver(case_mesh(case), fam.params(case))
            s.init_flowfield()
            f = torch.tensor(nx.fwd(fam.features(s, case)), dtype=torch.float32, device="cuda").contiguous()
            pred = ny.inv(net.predict(f).cpu().numpy().astype(np.float64))
            s.upload_state(fam.state(pred, case, s.nT))
            ss.append(s)
        return ss, time.perf_counter() - t0

    out = {"family": fam.description,
           "features": list(fam.feature_names),
           "network": f"{X.shape[1]}->{depth}x{width} GELU->{Y.shape[1]}, BF16 tcgen05.mma GEMMs",
           "train_cases": n_train, "train_cases_converged": int(sum(i is not None for i in train_iters)),
           "test_cases": n_test, "train_samples": int(X.shape[0]),
           "train_steps": train_steps, "batch": batch, "lr": lr,
           "loss_first": float(losses[0]), "loss_last": float(np.mean(losses[-50:])),
           "data_s": t_data, "train_s": t_train, "threshold": f"cold first residual x {drop:g}"}
    forces = {}
    for name, is_warm, batched in (("plain", False, False), ("cold_batched", False, True),
                                   ("warm", True, False), ("warm_batched", True, True)):
        if is_warm:
            ss, t_pred = warm()
        else:
            ss, t_pred = cold(), 0.0
        it, t = solve_to(ss, thr, batch=batched, max_iters=max_iters)
        out[name] = {"iterations_mean": float(np.mean([i if i is not None else np.nan for i in it])),
                     "converged": int(sum(i is not None for i in it)), "seconds": t + t_pred,
                     "predict_s": t_pred}
        if name in ("plain", "warm"):
            ok = [i is not None for i in it]
            forces[name] = [(s.forces()[9:11] if k else None) for s, k in zip(ss, ok)]
            # untimed: on to the tighter threshold, every case in one batch
            sub = [s for s, k in zip(ss, ok) if k]
            tight = [tr / drop * polish_drop for tr, k in zip(thr, ok) if k]
            it2, _ = solve_to(sub, tight, batch=True, max_iters=max_iters)
            fp = iter([(s.forces()[9:11] if i is not None else None) for s, i in zip(sub, it2)])
            forces[name + "_polished"] = [next(fp) if k else None for k in ok]
        for s in ss:
            s.close()

    def compare(a, b):
        errs = [np.abs(w - c) / np.maximum(np.abs(c), 1e-3) for c, w in zip(forces[a], forces[b])
                if c is not None and w is not None]
        return {"cases": len(errs), "cl_rel_max": float(max(e[0] for e in errs)) if errs else None,
                "cd_rel_max": float(max(e[1] for e in errs)) if errs else None}

    out["forces_warm_vs_cold"] = {"at_threshold": compare("plain", "warm"),
                                  f"at_{polish_drop:g}": compare("plain_polished", "warm_polished")}
    out["speedup_warm_batched_vs_plain"] = out["plain"]["seconds"] / out["warm_batched"]["seconds"]
    net.close()
    return out

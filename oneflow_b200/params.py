"""ctypes mirror of ``ofg_params`` (include/oneflow_b200.h) and helpers.

Field names are the reference's script keys (``GetDataValue<T>("key")`` in
codes/ns/src/NsCom.cpp:45-94, codes/global/src/Ctrl.cpp:40-113,
codes/turb/src/TurbCom.cpp:110-350)."""
from __future__ import annotations

import ctypes as C

_INT = ["dimension", "ischeme", "ilim", "igrad", "ieigenfix", "timestepModel", "ncfl", "visSRModel",
        "visTimeStepModel", "vismodel", "ivischeme", "isowallbc", "iprod_sa", "ft2_flag", "turb_ilim",
        "precision", "venkat_kh3", "sweep_order", "time_integral", "rk_stage"]
_DBL = ["vencat_coef", "centropy1", "centropy2", "cflst", "cfled", "max_time_ratio", "global_dt", "mach_ref",
        "aoa_degree", "sideslip_degree", "reynolds", "gama_ref", "prl", "prt", "tref_dim", "twall_dim",
        "inflow_viscosity", "rprod", "turb_cfl_ratio", "ref_sa", "max_vis_ratio"]


class OfgParams(C.Structure):
    _fields_ = ([(n, C.c_int) for n in _INT] + [("reserved_i", C.c_int * 4)] +
                [(n, C.c_double) for n in _DBL] + [("reserved_d", C.c_double * 6)])


def defaults(**kw) -> OfgParams:
    """The reference regression cases' settings (test/*/script/cfd.txt,
    inflow.txt, turb.txt): Roe, second order unlimited, local time step with
    the CFL ramp 0.1 -> 10 over 100 steps, LU-SGS, laminar."""
    p = OfgParams()
    p.dimension = 2
    p.ischeme = 1
    p.ilim = 0
    p.igrad = 0
    p.ieigenfix = 1
    p.timestepModel = 0
    p.ncfl = 100
    p.visSRModel = 2
    p.visTimeStepModel = 1
    p.vismodel = 1
    p.ivischeme = 0
    p.isowallbc = 0
    p.iprod_sa = 2
    p.ft2_flag = 0
    p.turb_ilim = -1
    p.precision = 0
    p.venkat_kh3 = 0
    p.time_integral = 2
    p.rk_stage = 1
    p.vencat_coef = 0.0001
    p.centropy1 = 0.0001
    p.centropy2 = 0.0001
    p.cflst = 0.1
    p.cfled = 10.0
    p.max_time_ratio = 1.0e10
    p.global_dt = 0.001
    p.mach_ref = 0.2
    p.aoa_degree = 0.0
    p.sideslip_degree = 0.0
    p.reynolds = 1.0e6
    p.gama_ref = 1.4
    p.prl = 0.72
    p.prt = 0.90
    p.tref_dim = 300.0
    p.twall_dim = 300.0
    p.inflow_viscosity = 0.01
    p.rprod = 1.0
    p.turb_cfl_ratio = 1.0
    p.ref_sa = 0.1
    p.max_vis_ratio = 1.0e6
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


def to_dict(p: OfgParams) -> dict:
    return {n: getattr(p, n) for n in _INT + _DBL}


def euler_bump(**kw) -> OfgParams:
    """2-D inviscid Euler, first-order Roe, LU-SGS, fixed CFL 5, FP64 (the
    reference-runnable bump configuration)."""
    base = dict(dimension=2, ischeme=1, ilim=-1, vismodel=0, cflst=5.0, cfled=5.0, ncfl=1, mach_ref=0.5,
                aoa_degree=0.0, precision=0)
    base.update(kw)
    return defaults(**base)


def rans_plate(**kw) -> OfgParams:
    """3-D RANS-SA flat plate: Roe, second order with least-squares gradients
    and the Venkatakrishnan limiter, LU-SGS, mixed precision."""
    base = dict(dimension=3, ischeme=1, ilim=2, igrad=2, vencat_coef=5.0, venkat_kh3=1, vismodel=3, mach_ref=0.2,
                reynolds=5.0e6, cflst=5.0, cfled=50.0, ncfl=200, precision=1)
    base.update(kw)
    return defaults(**base)


def rans_airfoil(mach: float, aoa: float, reynolds: float, **kw) -> OfgParams:
    """2-D RANS-SA airfoil (the batched cases): Roe, second order with
    Green-Gauss gradients and the Venkatakrishnan limiter, LU-SGS,
    colour-major sweeps, mixed precision.  (Least-squares gradients on the
    curved, high-aspect-ratio O-grid cells near the wall drove the SA
    production unstable within twenty iterations, in the oracle as well.)"""
    base = dict(dimension=2, ischeme=1, ilim=2, igrad=0, vencat_coef=5.0, venkat_kh3=1, vismodel=3, mach_ref=mach,
                aoa_degree=aoa, reynolds=reynolds, cflst=1.0, cfled=20.0, ncfl=200, precision=1, sweep_order=1)
    base.update(kw)
    return defaults(**base)


def transonic_wing(**kw) -> OfgParams:
    """3-D transonic swept wing, RANS-SA: SLAU2, Green-Gauss gradients with the
    Barth limiter, LU-SGS with the reference regression cases' CFL ramp
    (0.1 -> 10 over 100 steps), Mach 0.84, AoA 3.06 degrees, Re 1.2e7, mixed
    precision."""
    base = dict(dimension=3, ischeme=12, ilim=1, igrad=0, vismodel=3, mach_ref=0.84, aoa_degree=3.06,
                reynolds=1.2e7, cflst=0.1, cfled=10.0, ncfl=100, precision=1)
    base.update(kw)
    return defaults(**base)

"""Seeded cases of the golden fixtures (tests/golden/*.npz): the mesh and the
parameters of each, regenerated from their seeds."""
import numpy as np

from oneflow_b200 import colour_order, meshgen, params as P
from oneflow_b200.walldist import plate_wall_distance, wall_distance

CASES = {
    "bump_euler_roe1": dict(steps=50),
    "bump_euler_roe_venkat": dict(steps=30),
    "bump_euler_roe_barth": dict(steps=30),
    "plate2d_laminar_slau2": dict(steps=30),
    "plate2d_sa_roe": dict(steps=30),
    "plate3d_sa_roe": dict(steps=10),
    "plate3d_sa_roe_colour_renumbered": dict(steps=10),
    "mixed3d_slau2_gg_barth_sa": dict(steps=10),
    "bump_euler_rk3": dict(steps=30),
    "plate2d_laminar_roe_rk2": dict(steps=30),
    "plate2d_laminar_roe_visaver": dict(steps=30),
    "plate2d_laminar_roe_vistest": dict(steps=30),
    "plate2d_laminar_roe_visnew1": dict(steps=30),
    "plate2d_laminar_roe_visnew2": dict(steps=30),
    "mixed3d_laminar_vistest": dict(steps=10),
    # boundary conditions no other case uses: INFLOW (5) and EXTRAPOLATION (1)
    # on a laminar and an SA plate, and the isothermal no-slip wall (isowallbc 1)
    "plate2d_laminar_roe_inflow_extrap": dict(steps=30),
    "plate2d_sa_roe_inflow_extrap": dict(steps=30),
    "plate2d_laminar_roe_isowall": dict(steps=30),
    # a small swept-wing hybrid mesh: hexahedral layers whose outer face is
    # split into two triangles, tetrahedra, the tip's prisms and hexahedra;
    # SLAU2 + Green-Gauss + Barth + SA at the transonic wing condition
    "wing3d_small_slau2_barth_sa": dict(steps=10),
}
# the 2-D Euler bump at its benchmark size: 256x128 quads split into 65,536
# jittered triangles, first-order Roe, LU-SGS, CFL 5, run for 2,000 outer
# iterations (tests/golden/bump2d_c1.npz keeps every C1_STRIDE-th cell)
C1_STEPS, C1_STRIDE = 2000, 16


def build_c1():
    return meshgen.bump_channel(256, 128), P.euler_bump()


# the incompressible solver (INsSolver, startStrategy 2, SIMPLE) on lid-driven
# cavities (every boundary face a solid wall, the lid moving at u = 1):
# tests/golden/ins_<name>.npz holds the reference's state after the given
# number of inner iterations and the remax values it printed
INS_CASES = {
    "cavity2d_quad": dict(steps=10),
    "cavity2d_tri_jitter": dict(steps=8),
    "cavity3d_hex": dict(steps=4),
    "cavity3d_hex_prism": dict(steps=3),
}


def build_ins(name):
    """(mesh, params, wall velocity [nBFaces, 3], inner steps) of an incompressible case"""
    if name == "cavity2d_quad":
        mesh = meshgen.lid_cavity_2d(16)
        prm = P.defaults(vismodel=1, reynolds=100.0, mach_ref=0.1)
    elif name == "cavity2d_tri_jitter":
        mesh = meshgen.lid_cavity_2d(12, jitter=0.2, triangles=True)
        prm = P.defaults(vismodel=1, reynolds=400.0, mach_ref=0.1)
    elif name == "cavity3d_hex":
        mesh = meshgen.lid_cavity_3d(6, jitter=0.1)
        prm = P.defaults(dimension=3, vismodel=1, reynolds=100.0, mach_ref=0.1)
    elif name == "cavity3d_hex_prism":
        mesh = meshgen.lid_cavity_3d(6, jitter=0.1, prisms=True)
        prm = P.defaults(dimension=3, vismodel=1, reynolds=200.0, mach_ref=0.1)
    else:
        raise KeyError(name)
    return mesh, prm, meshgen.lid_velocity(mesh, 1.0), INS_CASES[name]["steps"]


# meshes whose wall distance the reference computed itself (ireadwdst = 0):
# tests/golden/walldist_<name>.npz
WALLDIST_CASES = ("plate2d_sa_roe", "plate3d_sa_roe", "hexbox_sa")


def build_walldist(name):
    """mesh (without a wall distance) and SA parameters of a wall-distance case"""
    if name == "hexbox_sa":
        mesh = meshgen.bump_box_hexes()
        prm = P.defaults(dimension=3, ischeme=1, ilim=0, vismodel=3, mach_ref=0.2, reynolds=5e6)
    else:
        mesh, prm, _ = build(name)
    mesh.wall_dist = None
    return mesh, prm


# cases whose restart files (written by the reference at this outer step) are fixtures too
RESTART_CASES = {"bump_euler_roe_venkat": 20, "plate2d_sa_roe": 20}


def inflow_extrap(mesh):
    """The plate with its upstream far-field faces (x at the inlet) made
    INFLOW and its OUTFLOW exit made EXTRAPOLATION."""
    fnc = mesh.face_node_count[:mesh.n_bfaces]
    off = np.concatenate([[0], np.cumsum(mesh.face_node_count)])
    xf = np.array([mesh.x[mesh.face_nodes[off[f]:off[f] + fnc[f]]].mean() for f in range(mesh.n_bfaces)])
    bct = mesh.bc_type.copy()
    bct[(bct == 4) & (xf <= mesh.x.min() + 1e-12)] = 5
    bct[bct == 6] = 1
    assert (bct == 5).any() and (bct == 1).any()
    mesh.bc_type = bct.astype(np.int32)
    return mesh


def small_wing():
    m = meshgen.swept_wing_hybrid(n_around=32, n_hex=4, n_tet=4, nz_wing=6, nz_tip=3)
    m.wall_dist = wall_distance(m)
    return m


def build(name):
    steps = CASES[name]["steps"]
    if name == "wing3d_small_slau2_barth_sa":
        return small_wing(), P.transonic_wing(precision=0), steps
    if name == "plate2d_laminar_roe_inflow_extrap":
        return inflow_extrap(meshgen.plate_2d(24, 16)), P.defaults(ischeme=1, ilim=0, mach_ref=0.2, reynolds=1e5,
                                                                    vismodel=1), steps
    if name == "plate2d_sa_roe_inflow_extrap":
        mesh = inflow_extrap(meshgen.plate_2d(32, 24, y1=1e-5, ratio=1.25))
        mesh.wall_dist = wall_distance(mesh)
        return mesh, P.defaults(ischeme=1, ilim=0, mach_ref=0.2, reynolds=5e6, vismodel=3), steps
    if name == "plate2d_laminar_roe_isowall":
        # a wall 20 % hotter than the free stream
        return meshgen.plate_2d(24, 16), P.defaults(ischeme=1, ilim=0, mach_ref=0.2, reynolds=1e5, vismodel=1,
                                                     isowallbc=1, twall_dim=360.0), steps
    if name == "bump_euler_rk3":
        # the multi-stage scheme (TimeIntegral::RungeKutta), 3 stages, CFL 0.8
        return meshgen.bump_channel(32, 16), P.euler_bump(time_integral=1, rk_stage=3, cflst=0.8, cfled=0.8), steps
    if name == "plate2d_laminar_roe_rk2":
        return meshgen.plate_2d(24, 16), P.defaults(ischeme=1, ilim=0, mach_ref=0.2, reynolds=1e5, vismodel=1,
                                                     time_integral=1, rk_stage=2, cflst=0.5, cfled=0.5), steps
    if name.startswith("plate2d_laminar_roe_vis"):
        # the viscous face-gradient schemes: VIS_AVER, VIS_TEST, VIS_NEW1, VIS_NEW2
        iv = {"visaver": 1, "vistest": 2, "visnew1": 3, "visnew2": 4}[name.rsplit("_", 1)[1]]
        return meshgen.plate_2d(24, 16), P.defaults(ischeme=1, ilim=0, mach_ref=0.2, reynolds=1e5, vismodel=1,
                                                     ivischeme=iv), steps
    if name == "mixed3d_laminar_vistest":
        return meshgen.bump_box_mixed(), P.defaults(dimension=3, ischeme=1, ilim=0, vismodel=1, mach_ref=0.3,
                                                    reynolds=1e4, ivischeme=2), steps
    if name.startswith("bump"):
        mesh = meshgen.bump_channel(32, 16)
        kw = {"bump_euler_roe1": {}, "bump_euler_roe_venkat": dict(ilim=2, vencat_coef=0.05),
              "bump_euler_roe_barth": dict(ilim=1)}[name]
        return mesh, P.euler_bump(**kw), steps
    if name == "plate2d_laminar_slau2":
        return meshgen.plate_2d(24, 16), P.defaults(ischeme=12, ilim=0, mach_ref=0.2, reynolds=1e5, vismodel=1), steps
    if name == "plate2d_sa_roe":
        mesh = meshgen.plate_2d(32, 24, y1=1e-5, ratio=1.25)
        mesh.wall_dist = wall_distance(mesh)
        return mesh, P.defaults(ischeme=1, ilim=0, mach_ref=0.2, reynolds=5e6, vismodel=3), steps
    if name == "mixed3d_slau2_gg_barth_sa":
        # hexahedra and prisms over a bump: SLAU2, Green-Gauss, Barth, SA at
        # the transonic swept-wing condition (Mach 0.84, AoA 3.06, Re 1.2e7)
        mesh = meshgen.bump_box_mixed()
        mesh.wall_dist = wall_distance(mesh)
        return mesh, P.defaults(dimension=3, ischeme=12, ilim=1, igrad=0, vismodel=3, mach_ref=0.84,
                                aoa_degree=3.06, reynolds=1.2e7), steps
    mesh = meshgen.flat_plate_tets(8, 6, 4, ratio=1.3)
    mesh.wall_dist = plate_wall_distance(mesh)
    if name == "plate3d_sa_roe_colour_renumbered":
        perm, _ = colour_order(mesh)
        mesh = mesh.renumber_cells(perm)
    return mesh, P.defaults(dimension=3, ischeme=1, ilim=0, vismodel=3, mach_ref=0.2, reynolds=5e6), steps

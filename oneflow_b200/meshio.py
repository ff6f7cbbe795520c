"""Unstructured mesh container and the reference's grid / case file formats.

The ``.ofl`` grid layout follows the reference's reader:
``codes/zone/src/GridGroup.cpp:67-138`` (zone header: int32 nZones,
int32 pid[nZones], int32 zoneType[nZones]; per zone an int64 byte length
followed by the zone's DataBook bytes) and ``codes/geometry/src/UnsGrid.cpp:90-201``
(int32 nNodes, nFaces, nCells; double xN[], yN[], zN[]; int32 volBcType;
int32 numFaceNode[nFaces]; the face->node list; int32 lCells[nFaces],
rCells[nFaces]; int32 nBFaces; int32 bcType[nBFaces], bcNameId[nBFaces];
int32 nIFaces).  Boundary faces come first and carry rCells = -1.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np

BC_NAMES = {1: "BCExtrapolate", 2: "BCWall", 3: "BCSymmetryPlane", 4: "BCFarfield", 5: "BCInflow",
            6: "BCOutflow"}


@dataclass
class Mesh:
    """One zone in the reference's numbering (boundary faces first)."""
    dim: int
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    face_node_count: np.ndarray   # int32 [nFaces]
    face_nodes: np.ndarray        # int32 [sum(face_node_count)]
    lc: np.ndarray                # int32 [nFaces]
    rc: np.ndarray                # int32 [nFaces], -1 on boundary faces
    n_cells: int
    n_bfaces: int
    bc_type: np.ndarray           # int32 [nBFaces]
    bc_name_id: np.ndarray = None  # int32 [nBFaces]
    wall_dist: np.ndarray = None  # float64 [nCells] (SA only)
    meta: dict = field(default_factory=dict)

    @property
    def n_nodes(self) -> int:
        return int(self.x.shape[0])

    @property
    def n_faces(self) -> int:
        return int(self.lc.shape[0])

    def as_arrays(self):
        """Contiguous arrays with the dtypes the C ABI expects."""
        c = np.ascontiguousarray
        return dict(x=c(self.x, np.float64), y=c(self.y, np.float64), z=c(self.z, np.float64),
                    fnc=c(self.face_node_count, np.int32), fn=c(self.face_nodes, np.int32),
                    lc=c(self.lc, np.int32), rc=c(self.rc, np.int32), bct=c(self.bc_type, np.int32),
                    wd=None if self.wall_dist is None else c(self.wall_dist, np.float64))

    def sort_faces(self) -> "Mesh":
        """Return the mesh with its faces reordered by their cells: boundary
        faces (still first) by their left cell, interior faces by (smaller,
        larger) cell id -- after a cell renumbering, the face order that
        walks the cells in order.  Each face keeps its nodes and cells."""
        nb = self.n_bfaces
        lo, hi = np.minimum(self.lc, np.where(self.rc >= 0, self.rc, self.lc)), np.maximum(self.lc, self.rc)
        fb = np.argsort(self.lc[:nb], kind="stable")
        fi = nb + np.lexsort((hi[nb:], lo[nb:]))
        order = np.concatenate([fb, fi])
        off = np.concatenate([[0], np.cumsum(self.face_node_count)])
        fn = np.concatenate([self.face_nodes[off[f]:off[f + 1]] for f in order]) if len(order) else self.face_nodes
        bcn = None if self.bc_name_id is None else self.bc_name_id[fb]
        return Mesh(self.dim, self.x, self.y, self.z, self.face_node_count[order], fn.astype(np.int32),
                    self.lc[order], self.rc[order], self.n_cells, nb, self.bc_type[fb], bcn, self.wall_dist,
                    dict(self.meta))

    def renumber_cells(self, perm: np.ndarray) -> "Mesh":
        """Return the mesh with interior cell ``perm[new] = old`` renumbered.

        Faces keep their order (boundary faces first); a face whose left cell
        would get a larger id than its right cell is left as it is, so the
        geometry (normal from lc to rc) is unchanged."""
        perm = np.asarray(perm, np.int64)
        inv = np.empty(self.n_cells, np.int64)
        inv[perm] = np.arange(self.n_cells)
        lc = inv[self.lc].astype(np.int32)
        rc = self.rc.copy()
        m = rc >= 0
        rc[m] = inv[rc[m]].astype(np.int32)
        wd = None if self.wall_dist is None else self.wall_dist[perm].copy()
        return Mesh(self.dim, self.x, self.y, self.z, self.face_node_count, self.face_nodes, lc, rc,
                    self.n_cells, self.n_bfaces, self.bc_type, self.bc_name_id, wd, dict(self.meta))


def read_ofl(path: str, dim: int = 2) -> Mesh:
    buf = open(path, "rb").read()
    off = 0

    def rd(dt, n):
        nonlocal off
        a = np.frombuffer(buf, dtype=dt, count=n, offset=off)
        off += a.nbytes
        return a.copy()

    nz = int(rd("<i4", 1)[0])
    rd("<i4", nz)
    rd("<i4", nz)
    if nz != 1:
        raise ValueError("only single-zone grids are supported")
    rd("<i8", 1)
    nn, nf, nc = (int(v) for v in rd("<i4", 3))
    x, y, z = rd("<f8", nn), rd("<f8", nn), rd("<f8", nn)
    rd("<i4", 1)
    fnc = rd("<i4", nf)
    fn = rd("<i4", int(fnc.sum()))
    lc, rc = rd("<i4", nf), rd("<i4", nf)
    nb = int(rd("<i4", 1)[0])
    bct, bcn = rd("<i4", nb), rd("<i4", nb)
    return Mesh(dim, x, y, z, fnc, fn, lc, rc, nc, nb, bct, bcn)


def write_ofl(mesh: Mesh, path: str) -> None:
    nb = mesh.n_bfaces
    bcn = mesh.bc_name_id if mesh.bc_name_id is not None else _region_ids(mesh.bc_type)
    body = b"".join([
        np.array([mesh.n_nodes, mesh.n_faces, mesh.n_cells], "<i4").tobytes(),
        np.asarray(mesh.x, "<f8").tobytes(), np.asarray(mesh.y, "<f8").tobytes(),
        np.asarray(mesh.z, "<f8").tobytes(),
        np.array([-1], "<i4").tobytes(),
        np.asarray(mesh.face_node_count, "<i4").tobytes(), np.asarray(mesh.face_nodes, "<i4").tobytes(),
        np.asarray(mesh.lc, "<i4").tobytes(), np.asarray(mesh.rc, "<i4").tobytes(),
        np.array([nb], "<i4").tobytes(), np.asarray(mesh.bc_type, "<i4").tobytes(),
        np.asarray(bcn, "<i4").tobytes(), np.array([0], "<i4").tobytes(),
    ])
    with open(path, "wb") as fh:
        fh.write(np.array([1, 0, 0], "<i4").tobytes())
        fh.write(np.array([len(body)], "<i8").tobytes())
        fh.write(body)


def _region_ids(bc_type: np.ndarray) -> np.ndarray:
    """One boundary region per distinct BC code, numbered in code order."""
    codes = sorted(set(int(v) for v in bc_type))
    lut = {c: i for i, c in enumerate(codes)}
    return np.array([lut[int(v)] for v in bc_type], np.int32)


def write_case(case_dir: str, mesh: Mesh, params: dict, max_steps: int, start_strategy: int = 0,
               field_save: int = 10 ** 8) -> None:
    """Write a reference project directory (script/, grid/, results/, ...)
    that runs ``mesh`` with ``params`` up to outer iteration ``max_steps``.

    ``params`` holds the reference's script keys (see ofg_params).  The file
    set mirrors the reference's regression cases (test/*/script).
    ``start_strategy`` 1 starts from restart/flow.dat (and restart/turbflow.dat
    for SA), which the caller places there (codes/restart/src/RestartTaskReg.cpp:141-163); the
    reference writes those files whenever the outer step is a multiple of
    ``field_save`` (nFieldSave, codes/ns/src/NsSolverImp.cpp:154-157)."""
    for sub in ("script", "grid", "results", "restart", "visual", "log"):
        os.makedirs(os.path.join(case_dir, sub), exist_ok=True)
    write_ofl(mesh, os.path.join(case_dir, "grid", "mesh.ofl"))
    bcn = mesh.bc_name_id if mesh.bc_name_id is not None else _region_ids(mesh.bc_type)
    regions = {}
    for t, n in zip(mesh.bc_type, bcn):
        regions[int(n)] = int(t)
    with open(os.path.join(case_dir, "grid", "bcRegionMap.txt"), "w") as fh:
        fh.write(f"{len(regions)}\n")
        for rid in sorted(regions):
            fh.write(f"{rid} {BC_NAMES.get(regions[rid], 'BCGeneral')}{rid}\n")
    open(os.path.join(case_dir, "grid", "ns_bc.txt"), "w").close()
    open(os.path.join(case_dir, "grid", "turb_bc.txt"), "w").close()
    turb = params.get("vismodel", 0) >= 3
    wdfile = "grid/walldist.dat"
    if turb and mesh.wall_dist is not None:
        _write_walldist(os.path.join(case_dir, wdfile), mesh.wall_dist)
    p = dict(params)
    files = {
        "simu.txt": [("string", "simutask", '"Solve"')],
        "dimension.txt": [("int", "dimension", mesh.dim)],
        "tolerence.txt": [("Real", "ptTol", 1.0e-10)],
        "cfd.txt": [
            ("int", "startStrategy", start_strategy), ("int", "iexitflag", 0), ("int", "maxSteps", max_steps),
            ("Real", "maxTime", 0.2), ("int", "nFieldSave", field_save), ("int", "nForceSave", 1),
            ("int", "nResSave", 1), ("int", "nVisualSave", 10 ** 8), ("int", "addVisualizationSteps", 0),
            ("string", "gridFileName", '"grid/mesh.ofl"'), ("string", "aeroFile", '"results/aero.dat"'),
            ("string", "resFile", '"results/res.dat"'), ("string", "wallaeroFile", '"results/wallaero.dat"'),
            ("string", "heatfluxFile", '"results/heatflux.dat"'), ("string", "visualFile", '"visual/visual.dat"'),
            ("string", "flowFile", '"restart/flow.dat"'), ("int", "showfield", 0),
            ("int", "nTEqu", 5), ("int", "nEqu", 5), ("int", "nTModel", 1),
            ("int", "timestepModel", p["timestepModel"]), ("Real", "global_dt", p["global_dt"]),
            ("Real", "cflst", p["cflst"]), ("Real", "cfled", p["cfled"]), ("int", "ncfl", p["ncfl"]),
            ("Real", "max_time_ratio", p["max_time_ratio"]), ("int", "visSRModel", p["visSRModel"]),
            ("int", "visTimeStepModel", p["visTimeStepModel"]), ("int", "chemModel", 0),
            ("int", "idualtime", 0), ("int", "time_integral", p.get("time_integral", 2) or 2),
            ("int", "rk_stage", p.get("rk_stage", 1)),
            ("int", "linearTwoStepMethods", 1), ("int", "ischeme", p["ischeme"]),
            ("int", "ivischeme", p["ivischeme"]), ("int", "ieigenfix", p["ieigenfix"]),
            ("Real", "centropy1", p["centropy1"]), ("Real", "centropy2", p["centropy2"]),
            ("int", "idump", 0), ("int", "ilim", p["ilim"]), ("Real", "vencat_coef", p["vencat_coef"]),
        ],
        "vismodel.txt": [("int", "vismodel", p["vismodel"]),
                         ("string", "visname", {0: '"euler"', 1: '"laminar"'}.get(p["vismodel"], '"1eq-sa"'))],
        "multigrid.txt": [("int", "nmg", 1), ("int", "nmgSmoothingSteps", 1), ("int", "nmgPreSmoothingSteps", 1),
                          ("int", "nmgPostSmoothingSteps", 1), ("int", "mgCycleType", 1), ("int", "mgIterMode", 1),
                          ("int", "mgLaminarViscosity", 1), ("int", "mgTurbulentViscosity", 0),
                          ("int", "mgProlongationMethod", 2), ("Real", "mgFactor", 0.5), ("Real", "mgTurbFactor", 0.5)],
        "inflow.txt": [
            ("int", "inflowType", 0), ("Real", "mach_ref", p["mach_ref"]), ("Real", "aoa_degree", p["aoa_degree"]),
            ("Real", "sideslip_degree", p["sideslip_degree"]), ("Real", "reynolds", p["reynolds"]),
            ("Real", "lref", 1.0), ("Real", "aref", 1.0), ("Real", "xref", 0.0), ("Real", "yref", 0.0),
            ("Real", "zref", 0.0), ("int", "gasInfoStrategy", 2), ("int", "machStrategy", 0),
            ("Real", "elevation", 61.0), ("Real", "tref_dim", p["tref_dim"]), ("Real", "pref_dim", 101325.0),
            ("Real", "dref_dim", 1.225), ("Real", "vref_dim", 34.0294), ("Real", "reylref_dim", 1.0),
            ("Real", "gama_ref", p["gama_ref"]), ("Real", "prl", p["prl"]), ("Real", "prt", p["prt"]),
            ("Real", "schmidtl", 0.5), ("Real", "schmidtt", 0.5), ("string", "gasModelFile", '"gasmodel/air5s11r.dat"'),
            ("int", "isowallbc", p["isowallbc"]), ("Real", "twall_dim", p["twall_dim"]),
        ],
        "turb.txt": [
            ("int", "transition_model", 0), ("Real", "inflow_intensity", 0.5),
            ("Real", "inflow_viscosity", p["inflow_viscosity"]), ("int", "des_model", 0),
            ("Real", "coefficientOfSaDes", 0.65), ("Real", "coefficientOfSstDesKe", 0.61),
            ("Real", "coefficientOfSstDesKw", 0.78), ("int", "easm_model", -3),
            ("int", "numberOfAnisotropicStress", 5), ("int", "modifyTurbulentResidualStrategy", 0),
            ("int", "turbulentResidualSmoothOrNot", 0), ("int", "turbulentSourceModel", 0),
            ("int", "ft2_flag", p["ft2_flag"]), ("int", "turb_ilim", -1), ("int", "tns_ilim", -1),
            ("Real", "turbulentRelaxationCoefficient", 1.0), ("Real", "coefficientOfMinimumTurbulentQuantity", 1.0e-5),
            ("Real", "ref_sa", p["ref_sa"]), ("Real", "ref_sst", 0.001), ("int", "iturb_visflux", 2),
            ("int", "iprod_sa", p["iprod_sa"]), ("int", "iprod_sst", 1), ("Real", "max_vis_ratio", p["max_vis_ratio"]),
            ("Real", "rprod", p["rprod"]), ("int", "monitorMaximumTurbulentViscosityCoefficient", 0),
            ("int", "numberOfAbnormalTurbulentCellsLimit", 1), ("Real", "turb_cfl_ratio", p["turb_cfl_ratio"]),
            ("string", "turbresFile", '"results/turbres.dat"'), ("string", "turbflowFile", '"restart/turbflow.dat"'),
        ],
        "walldist.txt": [("string", "walldist_file", f'"{wdfile}"'),
                         ("int", "ireadwdst", 1 if (turb and mesh.wall_dist is not None) else 0)],
    }
    for name, items in files.items():
        with open(os.path.join(case_dir, "script", name), "w") as fh:
            for typ, key, val in items:
                if isinstance(val, float):
                    val = repr(val)
                fh.write(f"{typ} {key} = {val};\n")
    with open(os.path.join(case_dir, "script", "solver.txt"), "w") as fh:
        fh.write("NsSolver\n" + ("TurbSolver\n" if turb else ""))
    with open(os.path.join(case_dir, "script", "control.txt"), "w") as fh:
        for name in ("simu.txt", "dimension.txt", "tolerence.txt", "cfd.txt", "vismodel.txt", "multigrid.txt",
                     "inflow.txt", "turb.txt", "walldist.txt"):
            fh.write(f'"{name}";\n')


def _write_walldist(path: str, wd: np.ndarray) -> None:
    """Wall distance in the layout the reference reads when ireadwdst = 1
    (one DataBook: int64 byte length, then double dist[nCells];
    codes/geometry/src/CellMesh.cpp:73-77, codes/database/src/DataBook.cpp:283-299)."""
    with open(path, "wb") as fh:
        fh.write(np.array([wd.shape[0] * 8], "<i8").tobytes())
        fh.write(np.asarray(wd, "<f8").tobytes())


def read_ref_dump(path: str) -> dict:
    """Read the full-precision field dump written by the reference oracle's
    dump hook: {name: array [nEqu, nTCell]} plus 'nCells'."""
    buf = open(path, "rb").read()
    nc, nt, nfld = np.frombuffer(buf, "<i4", 3)
    off = 12
    out = {"nCells": int(nc)}
    for _ in range(int(nfld)):
        name = buf[off:off + 16].split(b"\0")[0].decode()
        off += 16
        ne = int(np.frombuffer(buf, "<i4", 1, off)[0])
        off += 4
        a = np.frombuffer(buf, "<f8", ne * int(nt), off).reshape(ne, int(nt)).copy()
        off += a.nbytes
        out[name] = a
    return out


def read_res_dat(path: str) -> np.ndarray:
    """The reference's res.dat / turbres.dat: rows of iter, sub-iter, res..."""
    rows = []
    for line in open(path, encoding="latin-1"):
        tok = line.split()
        if tok and tok[0].lstrip("-").isdigit():
            rows.append([float(t) for t in tok])
    return np.array(rows)


def read_flow_dat(path: str, n_eq: int, n_t: int) -> dict:
    """A restart file in the reference's layout (Restart::Dump through
    DataBook::WriteFile, codes/restart/src/Restart.cpp:155-164,190-194,99-120,
    codes/database/src/DataBook.cpp:301-316), one zone: int64 byte count,
    int32 outer step, f64 time, then q1, q2, res1, res2 as [n_eq][n_t] f64.
    Returns {"step", "time", "q1", "q2", "res1", "res2"}."""
    buf = open(path, "rb").read()
    nbytes = int(np.frombuffer(buf, "<i8", 1, 0)[0])
    need = 4 + 8 + 4 * n_eq * n_t * 8
    if nbytes != need or len(buf) != 8 + nbytes:
        raise ValueError(f"{path}: record of {nbytes} bytes in a {len(buf)}-byte file; "
                         f"{n_eq} equations x {n_t} cells need {need}")
    out = {"step": int(np.frombuffer(buf, "<i4", 1, 8)[0]), "time": float(np.frombuffer(buf, "<f8", 1, 12)[0])}
    a = np.frombuffer(buf, "<f8", 4 * n_eq * n_t, 20).reshape(4, n_eq, n_t)
    for k, name in enumerate(("q1", "q2", "res1", "res2")):
        out[name] = a[k].copy()
    return out


def write_flow_dat(path: str, q1: np.ndarray, step: int, time: float = 0.0, q2: np.ndarray = None,
                   res1: np.ndarray = None, res2: np.ndarray = None) -> None:
    """Write the same single-zone restart record (q2 defaults to q1, the
    residuals to zero)."""
    q1 = np.atleast_2d(np.asarray(q1, "<f8"))
    z = np.zeros_like(q1)
    parts = [q1, q1 if q2 is None else q2, z if res1 is None else res1, z if res2 is None else res2]
    body = np.concatenate([np.asarray(p, "<f8").reshape(q1.shape).ravel() for p in parts])
    with open(path, "wb") as fh:
        fh.write(np.array([4 + 8 + body.nbytes], "<i8").tobytes())
        fh.write(np.array([step], "<i4").tobytes())
        fh.write(np.array([time], "<f8").tobytes())
        fh.write(body.tobytes())

// CPU restatement of OneFLOW's unstructured residual + LU-SGS iteration.
//
// TEST INFRASTRUCTURE ONLY: this file is the oracle that the CUDA path is
// checked against (tests/, __graft_entry__.smoke(), bench.py's CPU
// baseline).  Nothing in the product imports, links or calls it.
//
// It restates, in plain sequential FP64 C++, the algorithms of the reference
// (eric2003/OneFLOW) in the same summation order as the reference's serial
// loops; each function cites the reference file:line it follows.  The
// oracle is pinned against the reference itself: oracle/refbuild builds the
// reference CPU solver into oracle/_ref and the tests compare the two on
// the reference's own regression cases and on the seeded meshes.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace {

const double SMALL = 1.0e-40;   // codes/basic/include/HXTypeBasic.h:34
const double LARGE = 1.0e40;    // codes/basic/include/HXTypeBasic.h:33
const double half = 0.5, two3rd = 2.0 / 3.0, third = 1.0 / 3.0, fourth = 0.25;
const double PI = 3.141592653589793;

inline double SQR3(double a, double b, double c) { return a * a + b * b + c * c; }
inline double DIST3(double a, double b, double c) { return std::sqrt(SQR3(a, b, c)); }
inline double MAXd(double a, double b) { return a > b ? a : b; }
inline double MINd(double a, double b) { return a < b ? a : b; }

enum { IR = 0, IU = 1, IV = 2, IW = 3, IP = 4 };
const int NEQ = 5;

}  // namespace

// Greedy colouring of the cell graph (interior faces), cells visited in
// natural order, each taking the smallest colour no earlier neighbour holds;
// order[k] = the k-th cell of the colour-major order (colours ascending, ids
// ascending inside a colour).  Returns the number of colours.
static int colourMajor(int nCells, int nBFaces, const std::vector<std::vector<int>> &c2f,
                       const std::vector<int> &lc, const std::vector<int> &rc, int *order) {
    std::vector<int> col(nCells, -1);
    int ncol = 0;
    for (int i = 0; i < nCells; ++i) {
        std::vector<char> used(ncol + 1, 0);
        for (int f : c2f[i]) {
            if (f < nBFaces) continue;
            int nb = lc[f] == i ? rc[f] : lc[f];
            if (col[nb] >= 0) used[col[nb]] = 1;
        }
        int cc = 0;
        while (cc < (int)used.size() && used[cc]) ++cc;
        col[i] = cc;
        ncol = std::max(ncol, cc + 1);
    }
    std::vector<int> start(ncol + 1, 0);
    for (int i = 0; i < nCells; ++i) start[col[i] + 1]++;
    for (int k = 0; k < ncol; ++k) start[k + 1] += start[k];
    for (int i = 0; i < nCells; ++i) order[start[col[i]]++] = i;
    return ncol;
}

struct Oracle {
    ofg_params p;
    // ---------------- mesh ----------------
    int nNodes = 0, nFaces = 0, nCells = 0, nBFaces = 0, nT = 0;
    std::vector<double> xN, yN, zN;
    std::vector<std::vector<int>> f2n;
    std::vector<int> lc, rc, bcType;
    std::vector<double> xfn, yfn, zfn, area, xfc, yfc, zfc;
    std::vector<double> xcc, ycc, zcc, vol;
    std::vector<std::vector<int>> c2f;
    std::vector<double> walldist;
    // ---------------- fields (reference layout [eq][nT]) ----------------
    std::vector<double> q[NEQ], dq[NEQ], res[NEQ];
    std::vector<double> dqdx[NEQ], dqdy[NEQ], dqdz[NEQ], limiter[NEQ];
    std::vector<double> bc_q[NEQ];
    std::vector<double> tempr, dtdx, dtdy, dtdz, visl, vist;
    std::vector<double> timestep, invsr, vissr, impsr;
    // turbulence (SA), reference layout
    std::vector<double> nut, dnut, resT, dtT, impsrT, invsrT, vissrT, dnutdx, dnutdy, dnutdz;
    // ---------------- reference state ----------------
    double statecoef = 0, pref = 0, inflow[NEQ] = {0}, oreynolds = 0, const_cp = 0, oprl = 0, oprt = 0;
    double sutherland_ts = 0;
    double cfl = 0;
    long outerSteps = 0;
    std::vector<double> resHist;      // per outer step: 5 NS RMS
    std::vector<double> turbHist;     // per outer step: SA RMS
    std::string err;

    // ======================= mesh & metrics =======================
    // codes/geometry/src/UnsGrid.cpp:131-176 (face reversal), :123-129 (ghost ids)
    int setMesh(int nn, const double *x, const double *y, const double *z, int nf, const int *fnc,
                const int *fn, const int *l, const int *r, int nc, int nb, const int *bct, const double *wd) {
        nNodes = nn; nFaces = nf; nCells = nc; nBFaces = nb; nT = nc + nb;
        xN.assign(x, x + nn); yN.assign(y, y + nn); zN.assign(z, z + nn);
        f2n.assign(nf, {});
        size_t pos = 0;
        for (int f = 0; f < nf; ++f) { f2n[f].assign(fn + pos, fn + pos + fnc[f]); pos += fnc[f]; }
        lc.assign(l, l + nf); rc.assign(r, r + nf);
        for (int f = 0; f < nf; ++f)
            if (lc[f] < 0) { std::reverse(f2n[f].begin(), f2n[f].end()); std::swap(lc[f], rc[f]); }
        for (int f = 0; f < nb; ++f) rc[f] = f + nc;  // UnsGrid::NormalizeBc
        bcType.assign(bct, bct + nb);
        walldist.assign(nT, 0.0);
        if (wd) for (int c = 0; c < nc; ++c) walldist[c] = wd[c];
        calcMetrics();
        // CellTopo::CalcC2f, codes/geometry/src/CellTopo.cpp:95-119
        c2f.assign(nT, {});
        for (int f = 0; f < nb; ++f) c2f[lc[f]].push_back(f);
        for (int f = nb; f < nf; ++f) { c2f[lc[f]].push_back(f); c2f[rc[f]].push_back(f); }
        buildKey();
        alloc();
        return 0;
    }

    // Sweep order.  sweep_order 0: the cell numbering (the reference).
    // sweep_order 1: colour-major (greedy colouring in natural order, colours
    // ascending, ids ascending inside a colour) -- the order in which the
    // reference would sweep the mesh renumbered that way.  Ghosts come last.
    std::vector<int> key, keyOrder;
    void buildKey() {
        keyOrder.resize(nCells);
        if (p.sweep_order == 1) {
            colourMajor(nCells, nBFaces, c2f, lc, rc, keyOrder.data());
        } else {
            for (int i = 0; i < nCells; ++i) keyOrder[i] = i;
        }
        key.assign(nT, 0);
        for (int k = 0; k < nCells; ++k) key[keyOrder[k]] = k;
        for (int f = 0; f < nBFaces; ++f) key[nCells + f] = nCells + f;
    }

    void calcMetrics() {
        xfn.assign(nFaces, 0); yfn.assign(nFaces, 0); zfn.assign(nFaces, 0); area.assign(nFaces, 0);
        xfc.assign(nFaces, 0); yfc.assign(nFaces, 0); zfc.assign(nFaces, 0);
        xcc.assign(nT, 0); ycc.assign(nT, 0); zcc.assign(nT, 0); vol.assign(nT, 0);
        if (p.dimension == 2) {
            // FaceMesh::CalcFaceNormal2D / CalcFaceCenter2D, codes/geometry/src/FaceMesh.cpp:112-160
            for (int f = 0; f < nFaces; ++f) {
                int p1 = f2n[f][0], p2 = f2n[f][1];
                xfn[f] = yN[p2] - yN[p1];
                yfn[f] = xN[p1] - xN[p2];
                zfn[f] = 0.0;
                area[f] = DIST3(xfn[f], yfn[f], zfn[f]);
            }
            for (int f = 0; f < nFaces; ++f) {
                double oa = 1.0 / (area[f] + SMALL);
                xfn[f] *= oa; yfn[f] *= oa; zfn[f] *= oa;
            }
            for (int f = 0; f < nFaces; ++f) {
                int p1 = f2n[f][0], p2 = f2n[f][1];
                xfc[f] = half * (xN[p1] + xN[p2]);
                yfc[f] = half * (yN[p1] + yN[p2]);
                zfc[f] = half * (zN[p1] + zN[p2]);
            }
            // UnsGrid::CalcCellCenterVol2D, codes/geometry/src/UnsGrid.cpp:630-741
            for (int f = 0; f < nBFaces; ++f) {
                int l = lc[f];
                double dot = (xfc[f] * xfn[f] + yfc[f] * yfn[f] + zfc[f] * zfn[f]) * area[f];
                xcc[l] += xfc[f] * dot; ycc[l] += yfc[f] * dot; zcc[l] += zfc[f] * dot; vol[l] += dot;
            }
            for (int f = nBFaces; f < nFaces; ++f) {
                int l = lc[f], r = rc[f];
                double dot = (xfc[f] * xfn[f] + yfc[f] * yfn[f] + zfc[f] * zfn[f]) * area[f];
                xcc[l] += xfc[f] * dot; ycc[l] += yfc[f] * dot; zcc[l] += zfc[f] * dot; vol[l] += dot;
                xcc[r] -= xfc[f] * dot; ycc[r] -= yfc[f] * dot; zcc[r] -= zfc[f] * dot; vol[r] -= dot;
            }
            for (int c = 0; c < nCells; ++c) {
                double tmp = 1.0 / (1.5 * vol[c] + SMALL);
                xcc[c] *= tmp; ycc[c] *= tmp; zcc[c] *= tmp;
                vol[c] *= half;
                if (vol[c] <= 0.0) vol[c] = -vol[c];
            }
        } else {
            // FaceMesh::CalcFaceNormal3D, codes/geometry/src/FaceMesh.cpp:162-208
            for (int f = 0; f < nFaces; ++f) {
                const std::vector<int> &fi = f2n[f];
                size_t n = fi.size();
                for (size_t i = 0; i < n; ++i) {
                    int p1 = fi[i], p2 = fi[(i + 1) % n];
                    double dx1 = xN[p1], dy1 = yN[p1], dz1 = zN[p1];
                    double dx2 = xN[p2], dy2 = yN[p2], dz2 = zN[p2];
                    xfn[f] += half * (dy1 * dz2 - dy2 * dz1);
                    yfn[f] += half * (dz1 * dx2 - dz2 * dx1);
                    zfn[f] += half * (dx1 * dy2 - dx2 * dy1);
                }
                area[f] = DIST3(xfn[f], yfn[f], zfn[f]);
            }
            for (int f = 0; f < nFaces; ++f) {
                double oa = 1.0 / (area[f] + SMALL);
                xfn[f] *= oa; yfn[f] *= oa; zfn[f] *= oa;
            }
            // FaceMesh::CalcFaceCenter3D, codes/geometry/src/FaceMesh.cpp:210-286
            for (int f = 0; f < nFaces; ++f) {
                const std::vector<int> &fi = f2n[f];
                size_t n = fi.size();
                double x0 = 0, y0 = 0, z0 = 0;
                for (size_t i = 0; i < n; ++i) { x0 += xN[fi[i]]; y0 += yN[fi[i]]; z0 += zN[fi[i]]; }
                double factor = 1.0 / n;
                x0 *= factor; y0 *= factor; z0 *= factor;
                double sx = 0, sy = 0, sz = 0, sarea = 0;
                for (size_t i = 0; i < n; ++i) {
                    int p1 = fi[i], p2 = fi[(i + 1) % n];
                    double dx1 = xN[p1] - x0, dy1 = yN[p1] - y0, dz1 = zN[p1] - z0;
                    double dx2 = xN[p2] - x0, dy2 = yN[p2] - y0, dz2 = zN[p2] - z0;
                    double x00 = third * (xN[p1] + xN[p2] + x0);
                    double y00 = third * (yN[p1] + yN[p2] + y0);
                    double z00 = third * (zN[p1] + zN[p2] + z0);
                    double anx = dy1 * dz2 - dy2 * dz1;
                    double any = dz1 * dx2 - dz2 * dx1;
                    double anz = dx1 * dy2 - dx2 * dy1;
                    double fa = half * DIST3(anx, any, anz);
                    double nrm = anx * xfn[f] + any * yfn[f] + anz * zfn[f];
                    if (nrm < 0.0) fa = -fa;
                    sarea += fa;
                    sx += fa * x00; sy += fa * y00; sz += fa * z00;
                }
                double os = 1.0 / (sarea + SMALL);
                xfc[f] = sx * os; yfc[f] = sy * os; zfc[f] = sz * os;
            }
            // UnsGrid::CalcCellCenterVol3D, codes/geometry/src/UnsGrid.cpp:743-886
            for (int f = 0; f < nFaces; ++f) {
                int l = lc[f], r = rc[f];
                const std::vector<int> &fi = f2n[f];
                size_t n = fi.size();
                for (size_t i = 0; i < n; ++i) {
                    int p2 = fi[i], p3 = fi[(i + 1) % n];
                    double x21 = xN[p2] - xfc[f], y21 = yN[p2] - yfc[f], z21 = zN[p2] - zfc[f];
                    double x31 = xN[p3] - xfc[f], y31 = yN[p3] - yfc[f], z31 = zN[p3] - zfc[f];
                    double nx = y21 * z31 - y31 * z21;
                    double ny = z21 * x31 - z31 * x21;
                    double nz = x21 * y31 - x31 * y21;
                    double trix = xfc[f] + xN[p2] + xN[p3];
                    double triy = yfc[f] + yN[p2] + yN[p3];
                    double triz = zfc[f] + zN[p2] + zN[p3];
                    double tmp = nx * trix + ny * triy + nz * triz;
                    trix *= tmp; triy *= tmp; triz *= tmp;
                    xcc[l] += trix; ycc[l] += triy; zcc[l] += triz; vol[l] += tmp;
                    xcc[r] -= trix; ycc[r] -= triy; zcc[r] -= triz; vol[r] -= tmp;
                }
            }
            for (int c = 0; c < nCells; ++c) {
                double tmp = 1.0 / (4.0 * vol[c] + SMALL);
                xcc[c] *= tmp; ycc[c] *= tmp; zcc[c] *= tmp;
                vol[c] /= 18.0;
                if (vol[c] <= 0.0) vol[c] = -vol[c];
            }
        }
        // ghost cells (mirror of the interior centre through the face)
        for (int f = 0; f < nBFaces; ++f) {
            int l = lc[f], r = f + nCells;
            if (area[f] > SMALL) {
                double tmp = 2.0 * ((xcc[l] - xfc[f]) * xfn[f] + (ycc[l] - yfc[f]) * yfn[f] +
                                    (zcc[l] - zfc[f]) * zfn[f]);
                xcc[r] = xcc[l] - xfn[f] * tmp;
                ycc[r] = ycc[l] - yfn[f] * tmp;
                zcc[r] = zcc[l] - zfn[f] * tmp;
            } else {
                xcc[r] = -xcc[l] + 2.0 * xfc[f];
                ycc[r] = -ycc[l] + 2.0 * yfc[f];
                zcc[r] = -zcc[l] + 2.0 * zfc[f];
            }
            vol[r] = vol[l];
        }
    }

    void alloc() {
        for (int e = 0; e < NEQ; ++e) {
            q[e].assign(nT, 0); dq[e].assign(nT, 0); res[e].assign(nT, 0);
            dqdx[e].assign(nT, 0); dqdy[e].assign(nT, 0); dqdz[e].assign(nT, 0);
            limiter[e].assign(nT, 1.0); bc_q[e].assign(nBFaces, 0);
        }
        tempr.assign(nT, 0); dtdx.assign(nT, 0); dtdy.assign(nT, 0); dtdz.assign(nT, 0);
        visl.assign(nT, 0); vist.assign(nT, 0);
        timestep.assign(nT, 0); invsr.assign(nT, 0); vissr.assign(nT, 0); impsr.assign(nT, 0);
        nut.assign(nT, 0); dnut.assign(nT, 0); resT.assign(nT, 0); dtT.assign(nT, 0);
        impsrT.assign(nT, 0); invsrT.assign(nT, 0); vissrT.assign(nT, 0);
        dnutdx.assign(nT, 0); dnutdy.assign(nT, 0); dnutdz.assign(nT, 0);
    }

    // ======================= reference state =======================
    // codes/chemical/src/Chemical.cpp:280-325, codes/ns/src/NsCom.cpp:45-94
    void initReference() {
        statecoef = 1.0 / (p.gama_ref * (p.mach_ref * p.mach_ref));   // gama_ref * SQR(mach_ref)
        pref = statecoef * 1.0 * 1.0 / 1.0;
        double aoa = p.aoa_degree * PI / 180.0, aos = p.sideslip_degree * PI / 180.0;
        inflow[IR] = 1.0;
        inflow[IU] = 1.0 * std::cos(aoa) * std::cos(aos);
        inflow[IV] = 1.0 * std::sin(aoa) * std::cos(aos);
        inflow[IW] = 1.0 * std::sin(aos);
        inflow[IP] = pref;
        oreynolds = 1.0 / p.reynolds;
        oprl = 1.0 / p.prl;
        oprt = 1.0 / p.prt;
        const_cp = 1.0 / ((p.gama_ref - 1.0) * (p.mach_ref * p.mach_ref));
        sutherland_ts = 110.4 / p.tref_dim;  // codes/model/src/Sutherland.cpp:47-53
    }

    // codes/model/src/Sutherland.cpp:62-66
    double sutherland(double t) const {
        double t3 = t * t * t;
        return std::sqrt(t3) * (1 + sutherland_ts) / (t + sutherland_ts);
    }

    // ======================= CALC_BOUNDARY =======================
    // NsCalcGamaT (codes/ns/src/NsRhs.cpp:71-95) on [ist, ied)
    void calcT(int ist, int ied) {
        for (int c = ist; c < ied; ++c) tempr[c] = q[IP][c] / (statecoef * q[IR][c] * 1.0);
    }
    // CalcLaminarViscosity, codes/uns/src/UNsVisFlux.cpp:442-459
    void calcVisl(int ist, int ied) {
        for (int c = ist; c < ied; ++c) visl[c] = MAXd(0.0, sutherland(tempr[c]));
    }

    // NsBcSolver face BCs, codes/ns/src/NsBcSolver.cpp:51-440 via
    // UNsBcSolver::CalcBc, codes/uns/src/UNsBcSolver.cpp:55-166
    void calcBc() {
        double gama = p.gama_ref;
        for (int f = 0; f < nBFaces; ++f) {
            int bt = bcType[f];
            int l = lc[f], r = rc[f];
            double s[NEQ], t[NEQ], pr[NEQ];
            bool havePrim = false;
            for (int e = 0; e < NEQ; ++e) s[e] = q[e][l];
            double xn = xfn[f], yn = yfn[f], zn = zfn[f], vfn = 0.0;
            if (bt == OFG_BC_SYMMETRY || (bt == OFG_BC_SOLID_SURFACE && p.vismodel == 0)) {
                // SymmetryBc, :396-430
                double vn = xn * s[IU] + yn * s[IV] + zn * s[IW] - vfn;
                for (int e = 0; e < NEQ; ++e) t[e] = s[e];
                t[IU] = s[IU] - 2.0 * xn * vn;
                t[IV] = s[IV] - 2.0 * yn * vn;
                t[IW] = s[IW] - 2.0 * zn * vn;
                for (int e = 0; e < NEQ; ++e) pr[e] = half * (s[e] + t[e]);
                havePrim = true;
            } else if (bt == OFG_BC_SOLID_SURFACE && p.isowallbc == 0) {
                // AdiabaticVisWallBc + VelocityBc (vfx = 0), :357-394
                for (int e = 0; e < NEQ; ++e) t[e] = s[e];
                t[IU] = -t[IU] + 2.0 * 0.0;
                t[IV] = -t[IV] + 2.0 * 0.0;
                t[IW] = -t[IW] + 2.0 * 0.0;
                pr[IR] = s[IR]; pr[IU] = 0.0; pr[IV] = 0.0; pr[IW] = 0.0; pr[IP] = s[IP];
                havePrim = true;
            } else if (bt == OFG_BC_SOLID_SURFACE) {
                // IsothermalVisWallBc, :278-340
                for (int e = 0; e < NEQ; ++e) t[e] = s[e];
                t[IU] = -t[IU]; t[IV] = -t[IV]; t[IW] = -t[IW];
                double twall = p.twall_dim / p.tref_dim;
                double tlim = 0.1 * twall;
                double rm = s[IR], pm = s[IP], temperature = tempr[l];
                double rw_face = pm / (statecoef * twall * 1.0);
                pr[IR] = rw_face; pr[IU] = 0; pr[IV] = 0; pr[IW] = 0; pr[IP] = pm;
                double pg1 = pm, tg1 = 2.0 * twall - temperature;
                if (tg1 < tlim) tg1 = tlim;
                double rw = pg1 / (statecoef * twall * 1.0);
                double rg1 = 2.0 * rw - rm;
                rg1 = MAXd(0.5 * rw, rg1);
                t[IR] = rg1; t[IP] = pg1;
                (void)tg1;
                havePrim = true;
            } else if (bt == OFG_BC_FARFIELD) {
                // FarFieldBc, :171-276
                for (int e = 0; e < NEQ; ++e) t[e] = s[e];
                double rin = s[IR], uin = s[IU], vin = s[IV], win = s[IW], pin = s[IP];
                double rref = inflow[IR], uref = inflow[IU], vref = inflow[IV], wref = inflow[IW], pref_ = inflow[IP];
                double vnref = xn * uref + yn * vref + zn * wref - vfn;
                double vnin = xn * uin + yn * vin + zn * win - vfn;
                double cref = std::sqrt(std::fabs(p.gama_ref * pref_ / rref));
                double cin = std::sqrt(std::fabs(gama * pin / rin));
                double gamm1 = gama - 1.0;
                double velin = DIST3(uin, vin, win);
                if (velin > cin) {
                    if (vnin >= 0.0) {
                        for (int e = 0; e < NEQ; ++e) t[e] = s[e];
                    } else {
                        for (int e = 0; e < NEQ; ++e) t[e] = inflow[e];
                    }
                } else {
                    double riemp = vnin + 2.0 * cin / gamm1;
                    double riemm = vnref - 2.0 * cref / gamm1;
                    double vnb = half * (riemp + riemm);
                    double cb = fourth * (riemp - riemm) * gamm1;
                    double vtx, vty, vtz, entr;
                    if (vnb >= 0.0) {
                        entr = pin / std::pow(rin, gama);
                        vtx = uin - xn * vnin; vty = vin - yn * vnin; vtz = win - zn * vnin;
                    } else {
                        entr = pref_ / std::pow(rref, gama);
                        vtx = uref - xn * vnref; vty = vref - yn * vnref; vtz = wref - zn * vnref;
                    }
                    double rb = std::pow((cb * cb / (entr * gama)), 1.0 / gamm1);
                    double ub = vtx + xn * vnb, vb = vty + yn * vnb, wb = vtz + zn * vnb;
                    double pb = cb * cb * rb / gama;
                    t[IR] = rb; t[IU] = ub; t[IV] = vb; t[IW] = wb; t[IP] = pb;
                }
            } else if (bt == OFG_BC_INFLOW) {
                for (int e = 0; e < NEQ; ++e) t[e] = inflow[e];
            } else {  // OUTFLOW, EXTRAPOLATION, POLE: copy interior
                for (int e = 0; e < NEQ; ++e) t[e] = s[e];
            }
            for (int e = 0; e < NEQ; ++e) q[e][r] = t[e];
            if (havePrim) for (int e = 0; e < NEQ; ++e) bc_q[e][f] = pr[e];
        }
    }

    // NsCalcBoundary, codes/ns/src/NsSolverImp.cpp:90-97
    void calcBoundary() {
        calcT(0, nCells);
        calcVisl(0, nCells);
        calcBc();
        calcT(nCells, nT);
        calcVisl(nCells, nT);
    }

    void initFlowfield() {
        initReference();
        outerSteps = 0;
        for (int e = 0; e < NEQ; ++e) std::fill(q[e].begin(), q[e].end(), inflow[e]);
        calcBoundary();
        if (turb()) {   // UTurbRestart::InitRestart + TurbInitFinal
            std::fill(nut.begin(), nut.end(), p.ref_sa);
            turbBoundary();
        }
    }

    // ======================= CALC_TIME_STEP =======================
    // TimeStep::CalcCfl, codes/ns/src/TimeStep.cpp:43-59
    void calcCfl(long iter) {
        cfl = p.cfled;
        if (iter < p.ncfl) {
            double delta = (p.cfled - p.cflst) / p.ncfl;
            cfl = p.cflst + delta * iter;
        }
    }
    // TimeStep::CalcFaceInvSpec, codes/ns/src/TimeStep.cpp:61-88
    double faceInvSpec(int f) const {
        int l = lc[f], r = rc[f];
        double g1 = p.gama_ref, g2 = p.gama_ref;
        double rl = q[IR][l], ul = q[IU][l], vl = q[IV][l], wl = q[IW][l], pl = q[IP][l];
        double rr = q[IR][r], ur = q[IU][r], vr = q[IV][r], wr = q[IW][r], pr = q[IP][r];
        double vnl = xfn[f] * ul + yfn[f] * vl + zfn[f] * wl - 0.0;
        double vnr = xfn[f] * ur + yfn[f] * vr + zfn[f] * wr - 0.0;
        double gama = half * (g1 + g2);
        double pm = half * (pl + pr), rm = half * (rl + rr);
        double cm = std::sqrt(gama * pm / rm);
        double vn = half * (vnl + vnr);
        return half * area[f] * (std::fabs(vn) + cm);
    }
    // TimeStep::CalcFaceVisSpec, codes/ns/src/TimeStep.cpp:90-122
    double faceVisSpec(int f) const {
        int l = lc[f], r = rc[f];
        double vl_ = half * (visl[l] + visl[r]), vt_ = half * (vist[l] + vist[r]);
        double gama = half * (p.gama_ref + p.gama_ref);
        if (p.visSRModel == 1) {
            double density = half * (q[IR][l] + q[IR][r]);
            double c1 = 4.0 / 3.0 * (vl_ + vt_);
            double c2 = gama * (vl_ * oprl + vt_ * oprt);
            double c3 = 2.0 * MAXd(c1, c2) / (p.reynolds * density);
            return area[f] * area[f] * c3;
        } else if (p.visSRModel == 2) {
            double dist = std::fabs(xfn[f] * (xcc[r] - xcc[l]) + yfn[f] * (ycc[r] - ycc[l]) + zfn[f] * (zcc[r] - zcc[l]));
            double viscosity = vl_ + vt_;
            double density = half * (q[IR][l] + q[IR][r]);
            double c1 = 2.0 * viscosity / (density * dist * p.reynolds + SMALL);
            return half * c1 * area[f];
        } else if (p.visSRModel == 3) {
            double density = half * (q[IR][l] + q[IR][r]);
            return area[f] * area[f] / (p.reynolds * density + SMALL);
        }
        return 0.0;
    }
    // UTimeStep::CalcTimeStep, codes/uns/src/UTimeStep.cpp:190-416
    void calcTimeStep() {
        calcCfl(outerSteps);
        std::fill(invsr.begin(), invsr.begin() + nCells, 0.0);
        for (int f = 0; f < nFaces; ++f) {
            double s = faceInvSpec(f);
            invsr[lc[f]] += s; invsr[rc[f]] += s;
        }
        std::fill(vissr.begin(), vissr.begin() + nCells, 0.0);
        if (p.vismodel > 0) {
            for (int f = 0; f < nFaces; ++f) {
                double s = faceVisSpec(f);
                vissr[lc[f]] += s; vissr[rc[f]] += s;
            }
        }
        if (p.timestepModel == 1) {
            for (int c = 0; c < nCells; ++c) timestep[c] = p.global_dt;
            return;
        }
        for (int c = 0; c < nCells; ++c) timestep[c] = cfl * vol[c] / invsr[c];
        if (p.vismodel > 0 && p.visTimeStepModel > 0) {
            for (int c = 0; c < nCells; ++c) {
                double vts = cfl * vol[c] / vissr[c];
                timestep[c] *= vts / (timestep[c] + vts);
            }
        }
        double minTs = LARGE;
        for (int c = 0; c < nCells; ++c) minTs = MINd(timestep[c], minTs);
        if (p.max_time_ratio > 0) {
            double mx = p.max_time_ratio * minTs;
            for (int c = 0; c < nCells; ++c) timestep[c] = MINd(timestep[c], mx);
        }
        if (p.timestepModel == 2) {
            for (int c = 0; c < nCells; ++c) timestep[c] = minTs;
        }
    }

    // ======================= gradients =======================
    // CalcGradGGCellWeight, codes/usolver/src/UGrad.cpp:88-149
    void gradGG(const std::vector<double> &v, std::vector<double> &gx, std::vector<double> &gy, std::vector<double> &gz) {
        std::fill(gx.begin(), gx.end(), 0.0); std::fill(gy.begin(), gy.end(), 0.0); std::fill(gz.begin(), gz.end(), 0.0);
        for (int f = 0; f < nFaces; ++f) {
            int l = lc[f], r = rc[f];
            double value;
            if (p.igrad == 1) {
                value = half * (v[l] + v[r]);   // CalcGrad, UGrad.cpp:40-86
            } else {
                double dxl = xfc[f] - xcc[l], dyl = yfc[f] - ycc[l], dzl = zfc[f] - zcc[l];
                double dxr = xfc[f] - xcc[r], dyr = yfc[f] - ycc[r], dzr = zfc[f] - zcc[r];
                double delt1 = DIST3(dxl, dyl, dzl), delt2 = DIST3(dxr, dyr, dzr);
                double delta = 1.0 / (delt1 + delt2 + SMALL);
                double cl = delt2 * delta, cr = delt1 * delta;
                value = cl * v[l] + cr * v[r];
            }
            double fnxa = xfn[f] * area[f], fnya = yfn[f] * area[f], fnza = zfn[f] * area[f];
            gx[l] += fnxa * value; gy[l] += fnya * value; gz[l] += fnza * value;
            if (f < nBFaces) continue;
            gx[r] -= fnxa * value; gy[r] -= fnya * value; gz[r] -= fnza * value;
        }
        for (int c = 0; c < nCells; ++c) {
            double ov = 1.0 / vol[c];
            gx[c] *= ov; gy[c] *= ov; gz[c] *= ov;
        }
        for (int f = 0; f < nBFaces; ++f) {
            int l = lc[f], r = rc[f];
            gx[r] = gx[l]; gy[r] = gy[l]; gz[r] = gz[l];
        }
    }

    // Weighted least squares (new: no reference implementation).  Weights
    // 1/|d|^2 over the face neighbours (ghosts included), solved per cell with
    // the 3x3 normal equations (2x2 in 2D).
    void gradLSQ(const std::vector<double> &v, std::vector<double> &gx, std::vector<double> &gy, std::vector<double> &gz) {
        for (int c = 0; c < nCells; ++c) {
            double a11 = 0, a12 = 0, a13 = 0, a22 = 0, a23 = 0, a33 = 0, b1 = 0, b2 = 0, b3 = 0;
            for (int f : c2f[c]) {
                int nb = lc[f] == c ? rc[f] : lc[f];
                double dx = xcc[nb] - xcc[c], dy = ycc[nb] - ycc[c], dz = zcc[nb] - zcc[c];
                double w = 1.0 / (dx * dx + dy * dy + dz * dz);
                double dv = v[nb] - v[c];
                a11 += w * dx * dx; a12 += w * dx * dy; a13 += w * dx * dz;
                a22 += w * dy * dy; a23 += w * dy * dz; a33 += w * dz * dz;
                b1 += w * dx * dv; b2 += w * dy * dv; b3 += w * dz * dv;
            }
            if (p.dimension == 2) {
                double det = a11 * a22 - a12 * a12;
                double id = 1.0 / det;
                gx[c] = (a22 * b1 - a12 * b2) * id;
                gy[c] = (a11 * b2 - a12 * b1) * id;
                gz[c] = 0.0;
            } else {
                double c11 = a22 * a33 - a23 * a23, c12 = a13 * a23 - a12 * a33, c13 = a12 * a23 - a13 * a22;
                double c22 = a11 * a33 - a13 * a13, c23 = a12 * a13 - a11 * a23, c33 = a11 * a22 - a12 * a12;
                double det = a11 * c11 + a12 * c12 + a13 * c13;
                double id = 1.0 / det;
                gx[c] = (c11 * b1 + c12 * b2 + c13 * b3) * id;
                gy[c] = (c12 * b1 + c22 * b2 + c23 * b3) * id;
                gz[c] = (c13 * b1 + c23 * b2 + c33 * b3) * id;
            }
        }
        for (int f = 0; f < nBFaces; ++f) {
            int l = lc[f], r = rc[f];
            gx[r] = gx[l]; gy[r] = gy[l]; gz[r] = gz[l];
        }
    }

    void grad(const std::vector<double> &v, std::vector<double> &gx, std::vector<double> &gy, std::vector<double> &gz) {
        if (p.igrad == 2) gradLSQ(v, gx, gy, gz); else gradGG(v, gx, gy, gz);
    }

    // ======================= limiter =======================
    // codes/usolver/src/ULimiter.cpp:35-97 (functions), :377-644 (drivers)
    static double barthFunction(double dqv, double minv, double maxv, double dot) {
        if (dot < 0.0) return 0.0;
        else if (dqv > maxv) return maxv / dqv;
        else if (dqv < minv) return minv / dqv;
        return 1.0;
    }
    static double vencat(double x, double y, double eps) {
        double x2 = x * x, xy = x * y, y2 = y * y, cc = 2.0;
        return ((x2 + eps + cc * xy) / (x2 + cc * y2 + xy + eps));
    }
    static double vencatFunction(double dqv, double minv, double maxv, double eps) {
        if (dqv > SMALL) return vencat(maxv, dqv, eps);
        else if (dqv < -SMALL) return vencat(minv, dqv, eps);
        return 1.0;
    }
    void calcLimiter(int e) {
        std::vector<double> &lim = limiter[e];
        const std::vector<double> &v = q[e];
        std::fill(lim.begin(), lim.end(), 1.0);
        if (p.ilim == -1) {
            for (int f = 0; f < nFaces; ++f) { lim[lc[f]] = 0.0; lim[rc[f]] = 0.0; }
            return;
        }
        if (p.ilim == 0) return;  // the no-limiter loop writes 1.0 everywhere
        std::vector<double> minv(nT, 0.0), maxv(nT, 0.0);
        for (int c = 0; c < nCells; ++c) { minv[c] = v[c]; maxv[c] = v[c]; }
        for (int f = nBFaces; f < nFaces; ++f) {
            int l = lc[f], r = rc[f];
            minv[l] = MINd(minv[l], v[r]); maxv[l] = MAXd(maxv[l], v[r]);
            minv[r] = MINd(minv[r], v[l]); maxv[r] = MAXd(maxv[r], v[l]);
        }
        for (int c = 0; c < nCells; ++c) { minv[c] -= v[c]; maxv[c] -= v[c]; }
        double qmin = LARGE, qmax = -LARGE;
        for (int c = 0; c < nCells; ++c) { qmin = MINd(qmin, minv[c]); qmax = MAXd(qmax, maxv[c]); }
        double eps = p.vencat_coef * MAXd(qmax - qmin, 1.0);
        double epsg = eps * eps + SMALL;
        for (int f = 0; f < nFaces; ++f) {
            int l = lc[f], r = rc[f];
            double dx1 = xfc[f] - xcc[l], dy1 = yfc[f] - ycc[l], dz1 = zfc[f] - zcc[l];
            double dq1 = dqdx[e][l] * dx1 + dqdy[e][l] * dy1 + dqdz[e][l] * dz1;
            double dx2 = xfc[f] - xcc[r], dy2 = yfc[f] - ycc[r], dz2 = zfc[f] - zcc[r];
            double dq2 = dqdx[e][r] * dx2 + dqdy[e][r] * dy2 + dqdz[e][r] * dz2;
            double l1, l2;
            if (p.ilim == 1) {
                double ds1 = DIST3(dx1, dy1, dz1);
                double dot1 = (xfn[f] * dx1 + yfn[f] * dy1 + zfn[f] * dz1) / (ds1 + SMALL);
                l1 = barthFunction(dq1, minv[l], maxv[l], dot1);
                double ds2 = DIST3(dx2, dy2, dz2);
                double dot2 = -(xfn[f] * dx2 + yfn[f] * dy2 + zfn[f] * dz2) / (ds2 + SMALL);
                l2 = barthFunction(dq2, minv[r], maxv[r], dot2);
            } else {
                double e1 = epsg, e2 = epsg;
                if (p.venkat_kh3) {
                    // eps^2 = (K h)^3, h = cell size (new option; no reference form)
                    double h1 = p.dimension == 2 ? std::sqrt(vol[l]) : std::cbrt(vol[l]);
                    double h2 = p.dimension == 2 ? std::sqrt(vol[r]) : std::cbrt(vol[r]);
                    double k1 = p.vencat_coef * h1, k2 = p.vencat_coef * h2;
                    e1 = k1 * k1 * k1 + SMALL; e2 = k2 * k2 * k2 + SMALL;
                }
                l1 = vencatFunction(dq1, minv[l], maxv[l], e1);
                l2 = vencatFunction(dq2, minv[r], maxv[r], e2);
            }
            lim[l] = MINd(lim[l], l1);
            lim[r] = MINd(lim[r], l2);
        }
    }

    // ======================= inviscid flux =======================
    // NsInvFlux::Roe, codes/ns/src/NsInvFlux.cpp:186-308
    void roe(const double *p1, const double *p2, double xn, double yn, double zn, double *flux) const {
        const double vfn = 0.0, g1 = p.gama_ref, g2 = p.gama_ref;
        double rl = p1[IR], ul = p1[IU], vl = p1[IV], wl = p1[IW], pl = p1[IP];
        double rr = p2[IR], ur = p2[IU], vr = p2[IV], wr = p2[IW], pr = p2[IP];
        double v2l = SQR3(ul, vl, wl), v2r = SQR3(ur, vr, wr);
        double hl = (g1 / (g1 - 1.0)) * (pl / rl) + half * v2l;
        double hr = (g2 / (g2 - 1.0)) * (pr / rr) + half * v2r;
        double vnl = xn * ul + yn * vl + zn * wl - vfn;
        double vnr = xn * ur + yn * vr + zn * wr - vfn;
        double rvnl = rl * vnl, rvnr = rr * vnr;
        double ratio = std::sqrt(rr / rl);
        double coef = 1.0 / (1.0 + ratio);
        double rm = std::sqrt(rl * rr);
        double um = (ul + ur * ratio) * coef;
        double vm = (vl + vr * ratio) * coef;
        double wm = (wl + wr * ratio) * coef;
        double hm = (hl + hr * ratio) * coef;
        double pm = (pl + pr * ratio) * coef;
        double gama = (g1 + g2 * ratio) * coef;
        double v2 = SQR3(um, vm, wm);
        double vnflow = xn * um + yn * vm + zn * wm;
        double vnrel = vnflow - vfn;
        double gamm1 = gama - 1.0;
        double c2 = gamm1 * (hm - half * v2);
        double cm = std::sqrt(std::fabs(c2));
        double aeig1 = std::fabs(vnrel), aeig2 = std::fabs(vnrel + cm), aeig3 = std::fabs(vnrel - cm);
        double f1[NEQ], f2[NEQ];
        f1[0] = rvnl; f1[1] = rvnl * ul + xn * pl; f1[2] = rvnl * vl + yn * pl; f1[3] = rvnl * wl + zn * pl; f1[4] = rvnl * hl + vfn * pl;
        f2[0] = rvnr; f2[1] = rvnr * ur + xn * pr; f2[2] = rvnr * vr + yn * pr; f2[3] = rvnr * wr + zn * pr; f2[4] = rvnr * hr + vfn * pr;
        for (int e = 0; e < NEQ; ++e) flux[e] = f1[e] + f2[e];
        double q1[NEQ], q2[NEQ], dqv[NEQ];
        primToQ(p1, g1, q1); primToQ(p2, g2, q2);
        for (int e = 0; e < NEQ; ++e) dqv[e] = q2[e] - q1[e];
        double meig1 = aeig1, meig2 = aeig2, meig3 = aeig3;
        if (p.ieigenfix == 1) {  // ModifyAbsoluteEigenvalue, :167-184
            double mx = MAXd(aeig2, aeig3);
            double m1 = mx * p.centropy1, m2 = mx * p.centropy2;
            meig1 = MAXd(m1, aeig1); meig2 = MAXd(m2, aeig2); meig3 = MAXd(m2, aeig3);
        }
        double xi1 = (2.0 * meig1 - meig2 - meig3) / (2.0 * c2);
        double xi2 = (meig2 - meig3) / (2.0 * cm);
        double dc = vnflow * dqv[0] - xn * dqv[1] - yn * dqv[2] - zn * dqv[3];
        double c2dc = c2 * dc;
        // CalcTotalEnthalpyChange, :1334-1353
        double ae = gama - 1.0, af = half * ae * v2;
        double dh = -ae * (um * dqv[1] + vm * dqv[2] + wm * dqv[3] - dqv[4]);
        dh += af * dqv[0];
        double term1 = dh * xi1 + dc * xi2;
        double term2 = c2dc * xi1 + dh * xi2;
        flux[0] -= (meig1 * dqv[0] - term1);
        flux[1] -= (meig1 * dqv[1] - um * term1 + xn * term2);
        flux[2] -= (meig1 * dqv[2] - vm * term1 + yn * term2);
        flux[3] -= (meig1 * dqv[3] - wm * term1 + zn * term2);
        flux[4] -= (meig1 * dqv[4] - hm * term1 + vnflow * term2);
        for (int e = 0; e < NEQ; ++e) flux[e] *= half;
        (void)rm; (void)pm;
    }
    static void primToQ(const double *pr, double gama, double *qq) {
        double v2 = SQR3(pr[IU], pr[IV], pr[IW]);
        double em = (pr[IP] / pr[IR]) / (gama - 1.0) + half * v2;
        qq[0] = pr[IR]; qq[1] = pr[IR] * pr[IU]; qq[2] = pr[IR] * pr[IV]; qq[3] = pr[IR] * pr[IW]; qq[4] = pr[IR] * em;
    }
    static double fmSplit2(double mach, double ipn) { return ipn * fourth * (mach + ipn) * (mach + ipn); }
    static double fpSplit5(double mach, double alpha, double ipn) {
        double macha = std::fabs(mach);
        if (macha >= 1.0) return half * (1.0 + ipn * mach / (macha + SMALL));
        return fmSplit2(mach, ipn) * ((2.0 * ipn - mach) - ipn * 16.0 * alpha * mach * fmSplit2(mach, -ipn));
    }
    // NsInvFlux::Slau2, codes/ns/src/NsInvFlux.cpp:1246-1314
    void slau2(const double *p1, const double *p2, double xn, double yn, double zn, double *flux) const {
        const double vfn = 0.0, g1 = p.gama_ref, g2 = p.gama_ref;
        double rl = p1[IR], ul = p1[IU], vl = p1[IV], wl = p1[IW], pl = p1[IP];
        double rr = p2[IR], ur = p2[IU], vr = p2[IV], wr = p2[IW], pr = p2[IP];
        double v2l = SQR3(ul, vl, wl), v2r = SQR3(ur, vr, wr);
        double hl = (g1 / (g1 - 1.0)) * (pl / rl) + half * v2l;
        double hr = (g2 / (g2 - 1.0)) * (pr / rr) + half * v2r;
        double vnl = xn * ul + yn * vl + zn * wl - vfn;
        double vnr = xn * ur + yn * vr + zn * wr - vfn;
        double orl = 1.0 / (rl + SMALL), orr = 1.0 / (rr + SMALL);
        double c2l = g1 * pl * orl, c2r = g2 * pr * orr;
        double cl = std::sqrt(c2l), cr = std::sqrt(c2r);
        double cm = half * (cl + cr);
        double t = rr / rl;
        double vna = (std::fabs(vnl) + t * std::fabs(vnr)) / (1 + t);
        double ml = vnl / cm, mr = vnr / cm;
        double g = -MAXd(MINd(ml, 0.0), -1.0) * MINd(MAXd(mr, 0.0), 1.0);
        double vnp = (1 - g) * vna + g * std::fabs(vnl);
        double vnn = (1 - g) * vna + g * std::fabs(vnr);
        double va = std::sqrt(half * (v2l + v2r));
        double m12 = MINd(1.0, va / cm);
        double ka = (1 - m12) * (1 - m12);
        double ms = half * (rl * (vnl + vnp) + rr * (vnr - vnn) - ka * (pr - pl) / cm);
        double fp5ml = fpSplit5(ml, 0.0, 1.0);
        double fp5mr = fpSplit5(mr, 0.0, -1.0);
        double ps = 0;
        ps += half * (pl + pr);
        ps += half * (fp5ml - fp5mr) * (pl - pr);
        ps += va * (fp5ml + fp5mr - 1) * std::sqrt(rl * rr) * cm;
        double mp = half * (ms + std::fabs(ms)), mn = half * (ms - std::fabs(ms));
        flux[0] = (mp + mn);
        flux[1] = (mp * ul + mn * ur) + xn * ps;
        flux[2] = (mp * vl + mn * vr) + yn * ps;
        flux[3] = (mp * wl + mn * wr) + zn * ps;
        flux[4] = (mp * hl + mn * hr) + vfn * ps;
    }

    // UNsInvFlux::CalcFlux, codes/uns/src/UNsInvFlux.cpp:123-215
    void invFlux() {
        bool second = p.ilim != -1;
        if (second) {
            for (int e = 0; e < NEQ; ++e) grad(q[e], dqdx[e], dqdy[e], dqdz[e]);
            for (int e = 0; e < NEQ; ++e) calcLimiter(e);
        } else {
            // first order: gradients are still computed by the reference, but the
            // zero limiter multiplies them away exactly; keep them for downloads
            for (int e = 0; e < NEQ; ++e) grad(q[e], dqdx[e], dqdy[e], dqdz[e]);
            for (int e = 0; e < NEQ; ++e) calcLimiter(e);
        }
        std::vector<double> qf1(NEQ * (size_t)nFaces), qf2(NEQ * (size_t)nFaces);
        // GetQlQr + CalcFaceValue, codes/usolver/src/ULimiter.cpp:131-256
        for (int f = 0; f < nFaces; ++f) {
            int l = lc[f], r = rc[f];
            double t1[NEQ], t2[NEQ];
            double dx = xfc[f] - xcc[l], dy = yfc[f] - ycc[l], dz = zfc[f] - zcc[l];
            for (int e = 0; e < NEQ; ++e) {
                double phi = MINd(limiter[e][l], limiter[e][r]);
                t1[e] = q[e][l] + phi * (dqdx[e][l] * dx + dqdy[e][l] * dy + dqdz[e][l] * dz);
            }
            bool ok1 = !(t1[IR] <= 0.0 || t1[IP] <= 0.0);
            dx = xfc[f] - xcc[r]; dy = yfc[f] - ycc[r]; dz = zfc[f] - zcc[r];
            for (int e = 0; e < NEQ; ++e) {
                double phi = MINd(limiter[e][r], limiter[e][l]);
                t2[e] = q[e][r] + phi * (dqdx[e][r] * dx + dqdy[e][r] * dy + dqdz[e][r] * dz);
            }
            bool ok2 = !(t2[IR] <= 0.0 || t2[IP] <= 0.0);
            for (int e = 0; e < NEQ; ++e) {
                qf1[e * (size_t)nFaces + f] = ok1 ? t1[e] : q[e][l];
                qf2[e * (size_t)nFaces + f] = ok2 ? t2[e] : q[e][r];
            }
        }
        // NsLimField::BcQlQrFix, codes/uns/src/UNsLimiter.cpp:67-101
        for (int f = 0; f < nBFaces; ++f) {
            int l = lc[f], r = rc[f];
            for (int e = 0; e < NEQ; ++e) {
                double tmp = half * (q[e][l] + q[e][r]);
                qf1[e * (size_t)nFaces + f] = tmp; qf2[e * (size_t)nFaces + f] = tmp;
            }
            if (bcType[f] == OFG_BC_SOLID_SURFACE)
                for (int e = 0; e < NEQ; ++e) { qf1[e * (size_t)nFaces + f] = bc_q[e][f]; qf2[e * (size_t)nFaces + f] = bc_q[e][f]; }
        }
        // CalcInvFlux + AddInvFlux (AddF2CField, codes/usolver/src/UCom.cpp:144-171)
        for (int f = 0; f < nFaces; ++f) {
            double p1[NEQ], p2[NEQ], fl[NEQ];
            for (int e = 0; e < NEQ; ++e) { p1[e] = qf1[e * (size_t)nFaces + f]; p2[e] = qf2[e * (size_t)nFaces + f]; }
            if (p.ischeme == 12) slau2(p1, p2, xfn[f], yfn[f], zfn[f], fl);
            else roe(p1, p2, xfn[f], yfn[f], zfn[f], fl);
            for (int e = 0; e < NEQ; ++e) {
                double v = area[f] * fl[e];
                res[e][lc[f]] -= v;
                if (f >= nBFaces) res[e][rc[f]] += v;
            }
        }
    }

    // ======================= viscous flux (STD) =======================
    // UNsVisFlux::CalcFlux (codes/uns/src/UNsVisFlux.cpp:90-440) with the
    // VIS_STD face gradient (codes/usolver/src/VisGrad.cpp:150-175,356-366)
    // Face gradients of the VIS_TEST / VIS_NEW1 / VIS_NEW2 schemes for one
    // variable: VisGrad::CalcTestMethod, CalcNew1Method, CalcNew2Method and
    // ModifyFaceGrad (codes/usolver/src/VisGrad.cpp:268-353) with the geometry of
    // VisGradGeom::CalcFaceWeight / PrepareCellGeom (:44-97) and the face
    // tangents of GCom::CalcTangent (codes/global/src/Com.cpp:74-121).
    struct VisGeom {
        double fw1, fw2, d1, d2, dxnl, dynl, dznl, dxnr, dynr, dznr, angle1, angle2, t1[3], t2[3];
    };
    static double visAngle(double dx, double dy, double dz, double dist) {
        double result = dist / (DIST3(dx, dy, dz) + SMALL);
        if (result > 1.0) result = 1.0;
        if (result < -1.0) result = -1.0;
        return std::asin(result) * 180.0 / 3.141592653589793;
    }
    VisGeom visGeom(int f, int l, int r) const {
        VisGeom G;
        double xn = xfn[f], yn = yfn[f], zn = zfn[f];
        double ax = xfc[f] - xcc[l], ay = yfc[f] - ycc[l], az = zfc[f] - zcc[l];
        double bx = xfc[f] - xcc[r], by = yfc[f] - ycc[r], bz = zfc[f] - zcc[r];
        double delt1 = DIST3(ax, ay, az), delt2 = DIST3(bx, by, bz);
        double delta = 1.0 / (delt1 + delt2 + SMALL);
        G.fw1 = delt2 * delta;
        G.fw2 = delt1 * delta;
        double dxl = xcc[l] - xfc[f], dyl = ycc[l] - yfc[f], dzl = zcc[l] - zfc[f];
        double dxr = xcc[r] - xfc[f], dyr = ycc[r] - yfc[f], dzr = zcc[r] - zfc[f];
        G.d1 = xn * dxl + yn * dyl + zn * dzl;
        G.d2 = xn * dxr + yn * dyr + zn * dzr;
        G.dxnl = xn * G.d1 - dxl; G.dynl = yn * G.d1 - dyl; G.dznl = zn * G.d1 - dzl;
        G.dxnr = xn * G.d2 - dxr; G.dynr = yn * G.d2 - dyr; G.dznr = zn * G.d2 - dzr;
        G.angle1 = visAngle(dxl, dyl, dzl, -G.d1);
        G.angle2 = visAngle(dxr, dyr, dzr, G.d2);
        double *t1 = G.t1, *t2 = G.t2;
        if (xn != 0.0) { t1[0] = yn; t1[1] = -xn; t1[2] = 0.0; }
        else if (yn != 0.0) { t1[0] = -yn; t1[1] = xn; t1[2] = 0.0; }
        else if (zn != 0.0) { t1[0] = 0.0; t1[1] = -zn; t1[2] = yn; }
        else { for (int k = 0; k < 3; ++k) t1[k] = t2[k] = 0.0; return G; }
        double dtmp = 1.0 / DIST3(t1[0], t1[1], t1[2]);
        t1[0] *= dtmp; t1[1] *= dtmp; t1[2] *= dtmp;
        t2[0] = yn * t1[2] - zn * t1[1];
        t2[1] = zn * t1[0] - xn * t1[2];
        t2[2] = xn * t1[1] - yn * t1[0];
        return G;
    }
    void visVariant(const VisGeom &G, bool bface, double xn, double yn, double zn, double q1, double q2,
                    const double *g1, const double *g2, double *grad, double &dqdn) const {
        const int scheme = p.ivischeme;
        double q = half * (q1 + q2), q11 = q1, q22 = q2;
        dqdn = 0.0;
        auto side = [&]() {   // AccurateSideValue
            q11 += g1[0] * G.dxnl + g1[1] * G.dynl + g1[2] * G.dznl;
            q22 += g2[0] * G.dxnr + g2[1] * G.dynr + g2[2] * G.dznr;
        };
        if (scheme == 2) {
            if (G.angle1 > 20.0 && G.angle2 > 20.0) { side(); q = half * (q1 + q2); }
            if (G.angle1 > 0.0 && G.angle2 > 0.0 && std::fabs(G.d1) > SMALL && std::fabs(G.d2) > SMALL) {
                double dtmp = G.d1 * G.d1 + G.d2 * G.d2;
                double c1 = G.d1 * G.d1 / dtmp, c2 = 1.0 - c1;
                if (bface) { c1 = 1.0; c2 = 0.0; }
                double dqdn1 = (q11 - q) / G.d1, dqdn2 = (q22 - q) / G.d2;
                dqdn = c1 * dqdn1 + c2 * dqdn2;
            }
        } else if (scheme == 3) {
            if (G.d1 * G.d2 < 0.0 && std::fabs(G.d1) > SMALL && std::fabs(G.d2) > SMALL) {
                double d = -2.0 * G.d1 * G.d2 / (G.d1 * G.d1 + G.d2 * G.d2 + SMALL);
                double od = d / (G.d2 - G.d1);
                side();
                dqdn = (q22 - q11) * od;
            }
        } else {
            double d = -2.0 * G.d1 * G.d2 / (G.d1 * G.d1 + G.d2 * G.d2 + SMALL);
            if (d > 0.1) {
                side();
                double dqdn1 = (q11 - q) / G.d1, dqdn2 = (q22 - q) / G.d2;
                if (dqdn1 * dqdn2 > 0.0) dqdn = 2.0 * dqdn1 * dqdn2 / (dqdn1 + dqdn2);
            }
        }
        double gx = G.fw1 * g1[0] + G.fw2 * g2[0];
        double gy = G.fw1 * g1[1] + G.fw2 * g2[1];
        double gz = G.fw1 * g1[2] + G.fw2 * g2[2];
        double dqdt1 = G.t1[0] * gx + G.t1[1] * gy + G.t1[2] * gz;
        double dqdt2 = G.t2[0] * gx + G.t2[1] * gy + G.t2[2] * gz;
        grad[0] = xn * dqdn + G.t1[0] * dqdt1 + G.t2[0] * dqdt2;
        grad[1] = yn * dqdn + G.t1[1] * dqdt1 + G.t2[1] * dqdt2;
        grad[2] = zn * dqdn + G.t1[2] * dqdt1 + G.t2[2] * dqdt2;
    }

    void visFlux() {
        if (p.vismodel == 0) return;
        grad(tempr, dtdx, dtdy, dtdz);   // UTGrad: the reference's GG cell-weighted for igrad 0
        for (int f = 0; f < nFaces; ++f) {
            int l = lc[f], r = rc[f];
            double vl1 = visl[l], vl2 = visl[r], vt1 = vist[l], vt2 = vist[r];
            double vlm = half * (vl1 + vl2), vtm = half * (vt1 + vt2);
            double vis = vlm + vtm;
            double dx = xcc[r] - xcc[l], dy = ycc[r] - ycc[l], dz = zcc[r] - zcc[l];
            double ods = 1.0 / DIST3(dx, dy, dz);
            dx *= ods; dy *= ods; dz *= ods;
            double gx[6], gy[6], gz[6], qm[6];
            for (int e = 0; e < 6; ++e) {
                double q1 = e < NEQ ? q[e][l] : tempr[l];
                double q2 = e < NEQ ? q[e][r] : tempr[r];
                double ax1 = e < NEQ ? dqdx[e][l] : dtdx[l], ay1 = e < NEQ ? dqdy[e][l] : dtdy[l], az1 = e < NEQ ? dqdz[e][l] : dtdz[l];
                double ax2 = e < NEQ ? dqdx[e][r] : dtdx[r], ay2 = e < NEQ ? dqdy[e][r] : dtdy[r], az2 = e < NEQ ? dqdz[e][r] : dtdz[r];
                qm[e] = half * (q1 + q2);
                gx[e] = half * (ax1 + ax2); gy[e] = half * (ay1 + ay2); gz[e] = half * (az1 + az2);
                // CorrectGrad, VisGrad.cpp:356-366 (VIS_STD); VIS_AVER keeps the
                // average (UNsVisFlux::AverMethod, codes/uns/src/UNsVisFlux.cpp:357-366)
                if (p.ivischeme != 1) {
                    double fOld = gx[e] * dx + gy[e] * dy + gz[e] * dz;
                    double fnew = (q2 - q1) * ods;
                    double df = fnew - fOld;
                    gx[e] += df * dx; gy[e] += df * dy; gz[e] += df * dz;
                }
            }
            double xn = xfn[f], yn = yfn[f], zn = zfn[f];
            double dtdn = xn * gx[5] + yn * gy[5] + zn * gz[5];
            if (p.ivischeme >= 2) {   // TEST / NEW1 / NEW2: the face gradients above are replaced
                VisGeom G = visGeom(f, l, r);
                for (int e = 0; e < 6; ++e) {
                    double q1 = e < NEQ ? q[e][l] : tempr[l];
                    double q2 = e < NEQ ? q[e][r] : tempr[r];
                    double g1[3] = {e < NEQ ? dqdx[e][l] : dtdx[l], e < NEQ ? dqdy[e][l] : dtdy[l], e < NEQ ? dqdz[e][l] : dtdz[l]};
                    double g2[3] = {e < NEQ ? dqdx[e][r] : dtdx[r], e < NEQ ? dqdy[e][r] : dtdy[r], e < NEQ ? dqdz[e][r] : dtdz[r]};
                    double gr[3], dn;
                    visVariant(G, f < nBFaces, xn, yn, zn, q1, q2, g1, g2, gr, dn);
                    gx[e] = gr[0]; gy[e] = gr[1]; gz[e] = gr[2];
                    if (e == 5) dtdn = dn;   // SaveFacePara: the heat flux takes the scheme's dT/dn
                }
            }
            double kcp = (vlm * oprl + vtm * oprt) * const_cp;
            double qNormal = 0.0;
            qNormal += xn * 0.0 + yn * 0.0 + zn * 0.0;
            qNormal += kcp * dtdn;
            double dudx = gx[IU], dudy = gy[IU], dudz = gz[IU];
            double dvdx = gx[IV], dvdy = gy[IV], dvdz = gz[IV];
            double dwdx = gx[IW], dwdy = gy[IW], dwdz = gz[IW];
            double divv2p3 = two3rd * (dudx + dvdy + dwdz);
            double txx = vis * (2.0 * dudx - divv2p3);
            double tyy = vis * (2.0 * dvdy - divv2p3);
            double tzz = vis * (2.0 * dwdz - divv2p3);
            double txy = vis * (dudy + dvdx);
            double txz = vis * (dudz + dwdx);
            double tyz = vis * (dvdz + dwdy);
            double fv[NEQ];
            fv[0] = 0.0;
            fv[1] = xn * txx + yn * txy + zn * txz;
            fv[2] = xn * txy + yn * tyy + zn * tyz;
            fv[3] = xn * txz + yn * tyz + zn * tzz;
            fv[4] = qm[IU] * fv[1] + qm[IV] * fv[2] + qm[IW] * fv[3] + qNormal;
            double coeff = -oreynolds * area[f];
            for (int e = 0; e < NEQ; ++e) {
                double v = coeff * fv[e];
                res[e][l] -= v;
                if (f >= nBFaces) res[e][r] += v;
            }
        }
    }

    void loadResiduals() {  // LoadResiduals: res = -rhs, rhs = 0
        for (int e = 0; e < NEQ; ++e) std::fill(res[e].begin(), res[e].end(), -0.0);
    }
    void updateResiduals() { invFlux(); visFlux(); }

    // ======================= LU-SGS =======================
    // UNsSpectrum::CalcImplicitSpectrum, codes/uns/src/UNsSpectrum.cpp:52-94
    void calcImplicitSpectrum() {
        for (int c = 0; c < nCells; ++c) impsr[c] = (1.0 / timestep[c]) * vol[c];
        for (int c = 0; c < nCells; ++c) impsr[c] += invsr[c];
        for (int c = 0; c < nCells; ++c) impsr[c] += vissr[c];
    }

    // per-face increment: UNsLusgs::Solve (codes/uns/src/UNsLusgs.cpp:193-208),
    // PrepareDataFacePrim (:251-293), NsLusgs::GetStandardFluxIncrement
    // (codes/ns/src/NsLusgs.cpp:121-202), UNsLusgs::CalcViscousTerm (:295-330).
    // ci = the cell being solved, f its face; adds into rhs0.
    void faceIncrement(int ci, int f, double *rhs0) const {
        int l = lc[f], r = rc[f];
        double xn = xfn[f], yn = yfn[f], zn = zfn[f], vfn = 0.0, fa = area[f];
        if (r == ci) { std::swap(l, r); xn = -xn; yn = -yn; zn = -zn; vfn = -vfn; }
        double gl = p.gama_ref, gr = p.gama_ref;
        double rl = q[IR][l], ul = q[IU][l], vl = q[IV][l], wl = q[IW][l], pl = q[IP][l];
        double rr = q[IR][r], ur = q[IU][r], vr = q[IV][r], wr = q[IW][r], pr = q[IP][r];
        double hl = gl / (gl - 1.0) * pl / rl + half * SQR3(ul, vl, wl);
        double hr = gr / (gr - 1.0) * pr / rr + half * SQR3(ur, vr, wr);
        double tmp0 = std::sqrt(rr / rl);
        double tmp1 = 1.0 / (1.0 + tmp0);
        double rm = std::sqrt(rr * rl);
        double um = (ul + ur * tmp0) * tmp1;
        double vm = (vl + vr * tmp0) * tmp1;
        double wm = (wl + wr * tmp0) * tmp1;
        double hm = (hl + hr * tmp0) * tmp1;
        double pm = rm * (hm - half * SQR3(um, vm, wm)) * (gl - 1.0) / gl;
        double gama = gr;
        // CalcFaceEigenValue (primF)
        double c2f_ = std::fabs(gama * pm / rm);
        double cmf = std::sqrt(c2f_);
        double vnf = xn * um + yn * vm + zn * wm;
        double maxEig = std::fabs(vnf - vfn) + cmf;
        // neighbour state
        double dqj[NEQ];
        for (int e = 0; e < NEQ; ++e) dqj[e] = dq[e][r];
        double rj = q[IR][r], uj = q[IU][r], vj = q[IV][r], wj = q[IW][r], pj = q[IP][r];
        double c2 = std::fabs(gama * pj / rj);
        double cm = std::sqrt(c2);
        double vn_fluid = xn * uj + yn * vj + zn * wj;
        double vn_rel = vn_fluid - vfn;
        double lmd1 = vn_rel, lmd2 = vn_rel + cm, lmd3 = vn_rel - cm;
        lmd1 = half * (lmd1 + (-1) * maxEig);
        lmd2 = half * (lmd2 + (-1) * maxEig);
        lmd3 = half * (lmd3 + (-1) * maxEig);
        double x1 = (lmd1 + lmd1 - lmd2 - lmd3) / (c2 + c2);
        double x2 = (lmd2 - lmd3) / (cm + cm);
        double dc = vn_fluid * dqj[0] - xn * dqj[1] - yn * dqj[2] - zn * dqj[3];
        double c2dc = c2 * dc;
        // CalcDH, codes/ns/src/NsLusgs.cpp:348-366
        double v2 = SQR3(uj, vj, wj);
        double ae = gama - 1.0, af = half * ae * v2;
        double dh = -ae * (uj * dqj[1] + vj * dqj[2] + wj * dqj[3] - dqj[4]);
        double enthalpy = (gama / (gama - 1.0)) * (pj / rj);
        dh += af * dqj[0];
        double htot = enthalpy + half * v2;
        double term1 = dh * x1 + dc * x2;
        double term2 = c2dc * x1 + dh * x2;
        double dfj[NEQ];
        dfj[0] = lmd1 * dqj[0] - term1;
        dfj[1] = lmd1 * dqj[1] - uj * term1 + xn * term2;
        dfj[2] = lmd1 * dqj[2] - vj * term1 + yn * term2;
        dfj[3] = lmd1 * dqj[3] - wj * term1 + zn * term2;
        dfj[4] = lmd1 * dqj[4] - htot * term1 + vn_fluid * term2;
        for (int e = 0; e < NEQ; ++e) dfj[e] *= fa;
        if (p.vismodel > 0) {
            double visrad;
            double vl_ = visl[r], vt_ = vist[r];
            if (p.visSRModel == 1) {
                double density = half * (q[IR][l] + q[IR][r]);
                double c1 = 4.0 / 3.0 * (vl_ + vt_);
                double cc2 = p.gama_ref * (vl_ * oprl + vt_ * oprt);
                double c3 = 2.0 * MAXd(c1, cc2) / (p.reynolds * density);
                visrad = fa * fa * c3 / vol[r];
            } else {
                double dist = std::fabs(xn * (xcc[r] - xcc[l]) + yn * (ycc[r] - ycc[l]) + zn * (zcc[r] - zcc[l]));
                double viscosity = vl_ + vt_;
                double density = half * (q[IR][l] + q[IR][r]);
                double c1 = 2.0 * viscosity / (density * dist * p.reynolds + SMALL);
                visrad = half * c1 * fa;
            }
            for (int e = 0; e < NEQ; ++e) rhs0[e] -= visrad * dqj[e];
        }
        for (int e = 0; e < NEQ; ++e) rhs0[e] += dfj[e];
    }

    // UNsLusgs::LowerSweep, codes/uns/src/UNsLusgs.cpp:75-108; NsLusgs::CalcLowerChange (:230-277)
    void lusgsLower() {
        calcImplicitSpectrum();
        for (int k = 0; k < nCells; ++k) {
            int c = keyOrder[k];
            double rhs0[NEQ] = {0, 0, 0, 0, 0};
            for (int f : c2f[c]) {
                if (key[lc[f]] > key[c] || key[rc[f]] > key[c]) continue;
                faceIncrement(c, f, rhs0);
            }
            for (int e = 0; e < NEQ; ++e) dq[e][c] = (res[e][c] - rhs0[e]) / impsr[c];
        }
    }
    // UNsLusgs::UpperSweep, codes/uns/src/UNsLusgs.cpp:110-138; NsLusgs::CalcUpperChange (:279-326)
    void lusgsUpper() {
        calcImplicitSpectrum();
        for (int k = nCells - 1; k >= 0; --k) {
            int c = keyOrder[k];
            double rhs0[NEQ] = {0, 0, 0, 0, 0};
            for (int f : c2f[c]) {
                if (key[lc[f]] < key[c] || key[rc[f]] < key[c]) continue;
                faceIncrement(c, f, rhs0);
            }
            for (int e = 0; e < NEQ; ++e) dq[e][c] += (-rhs0[e]) / impsr[c];
        }
    }

    // ======================= update =======================
    // UNsUpdate::UpdateFlowField (codes/uns/src/UNsUpdate.cpp:46-146),
    // NsUpdate::CalcFlowField / WeekSolutionFix (codes/ns/src/NsUpdate.cpp:40-67,192-217)
    long nFixes = 0;
    void updateFlowfield() {
        double gama = p.gama_ref;
        for (int kk = 0; kk < nCells; ++kk) {
            int c = keyOrder[kk];   // in place, in sweep order (SolutionFix reads updated neighbours)
            double prim0[NEQ], q0[NEQ], qq[NEQ], pr[NEQ], d[NEQ];
            for (int e = 0; e < NEQ; ++e) { prim0[e] = q[e][c]; d[e] = dq[e][c]; }
            primToQ(prim0, gama, q0);
            for (int e = 0; e < NEQ; ++e) qq[e] = q0[e] + d[e];
            // QToPrim, codes/ns/src/NsInvFlux.cpp:1377-1399
            double density = std::fabs(qq[0]);
            double rd = 1.0 / density;
            double um = qq[1] * rd, vm = qq[2] * rd, wm = qq[3] * rd, rem = qq[4];
            double v2 = SQR3(um, vm, wm);
            double reint = rem - half * density * v2;
            pr[0] = density; pr[1] = um; pr[2] = vm; pr[3] = wm; pr[4] = (gama - 1.0) * reint;
            if (pr[IR] <= 0.0 || pr[IP] <= 0.0) {
                ++nFixes;
                bool ok = false;
                const double coefs[3] = {0.5, 0.1, 0.01};
                for (int k = 0; k < 3 && !ok; ++k) {
                    for (int e = 0; e < NEQ; ++e) pr[e] += coefs[k] * d[e];
                    if (!(pr[IR] < 0.0 || pr[IP] < 0.0)) ok = true;
                }
                if (!ok) {  // SolutionFix: neighbour average (in-place, natural order)
                    double sumV = 0.0;
                    for (int e = 0; e < NEQ; ++e) pr[e] = 0.0;
                    for (int f : c2f[c]) {
                        int nb = lc[f] == c ? rc[f] : lc[f];
                        sumV += 1.0;
                        for (int e = 0; e < NEQ; ++e) {
                            double v = q[e][nb];
                            if (e == IR || e == IP) v = std::fabs(v);
                            pr[e] += v * 1.0;
                        }
                    }
                    double rv = 1.0 / sumV;
                    for (int e = 0; e < NEQ; ++e) pr[e] *= rv;
                }
            }
            for (int e = 0; e < NEQ; ++e) q[e][c] = pr[e];
        }
    }

    // ======================= residual norm =======================
    void residualRms(double *rms, bool *nan) const {
        *nan = false;
        for (int e = 0; e < NEQ; ++e) {
            double s = 0.0;
            for (int c = 0; c < nCells; ++c) {
                double r = res[e][c];
                if (std::isnan(r)) *nan = true;
                s += r * r;
            }
            rms[e] = std::sqrt(s / nCells);
        }
    }

    // ======================= Spalart-Allmaras solver =======================
    // constants: TurbCom::InitConst (codes/turb/src/TurbCom.cpp:110-350)
    struct SaConst {
        double karm = 0.41, karm2, okarm2, cb1 = 0.1355, cb2 = 0.622, cv1 = 7.1, cv13, cw2 = 0.3, cw3 = 2.0, cw36;
        double ct3 = 1.2, ct4 = 0.5, sigma = 2.0 / 3.0, osigma, cw1, sac2 = 0.7, sac3 = 0.9, cb2s, cw1k;
        SaConst() {
            karm2 = karm * karm; okarm2 = 1.0 / karm2; cv13 = cv1 * cv1 * cv1; cw36 = std::pow(cw3, 6);
            osigma = 1.0 / sigma; cw1 = cb1 * okarm2 + (1.0 + cb2) / sigma; cb2s = osigma * cb2; cw1k = cw1 * karm2;
        }
    } sa;
    std::vector<double> matL, matR;
    bool turb() const { return p.vismodel >= 3; }

    // CalcTurbulentViscosity -> UTurbSrcFlux::CalcVist (codes/uturb/src/UTurbSrcFlux.cpp:101-243),
    // TurbSrcFlux::CalcCellVist1Equ (codes/turb/src/TurbSrcFlux.cpp:279-290)
    void calcVist() {
        for (int c = 0; c < nCells; ++c) {
            double rho = q[IR][c], nuet = nut[c], vl = visl[c];
            double olam = rho / (vl + SMALL);
            double xsi = nuet * olam;
            double xsi3 = xsi * xsi * xsi;
            double fv1 = xsi3 / (xsi3 + sa.cv13);
            double v = fv1 * rho * nuet;
            vist[c] = MINd(vl * p.max_vis_ratio, v);
        }
        for (int f = 0; f < nBFaces; ++f) vist[rc[f]] = vist[lc[f]];
    }
    // TurbBcSolver (codes/turb/src/TurbBcSolver.cpp:51-262) via UTurbBcSolver::CalcBc
    void turbBc() {
        for (int f = 0; f < nBFaces; ++f) {
            int bt = bcType[f], l = lc[f], r = rc[f];
            double s = nut[l], t = s;
            if (bt == OFG_BC_SOLID_SURFACE) t = -s;
            else if (bt == OFG_BC_INFLOW) t = p.ref_sa;
            else if (bt == OFG_BC_FARFIELD) {
                // the normal is scaled by gcom.faceOuterNormal, a member of a
                // global object that is never assigned (zero-initialised), so
                // the turbulent far-field decision sees a zero normal velocity
                // (codes/turb/src/TurbBcSolver.cpp:154-156, codes/global/include/Com.h:38)
                double xn = xfn[f] * 0, yn = yfn[f] * 0, zn = zfn[f] * 0;
                double rin = q[IR][l], uin = q[IU][l], vin = q[IV][l], win = q[IW][l], pin = q[IP][l];
                double vnref = xn * inflow[IU] + yn * inflow[IV] + zn * inflow[IW] - 0.0;
                double vnin = xn * uin + yn * vin + zn * win - 0.0;
                double cref = std::sqrt(std::fabs(p.gama_ref * inflow[IP] / inflow[IR]));
                double cin = std::sqrt(std::fabs(p.gama_ref * pin / rin));
                double velin = DIST3(uin, vin, win);
                if (velin > cin) {
                    t = vnin >= 0.0 ? s : p.ref_sa;
                } else {
                    double gamm1 = p.gama_ref - 1.0;
                    double riemp = vnin + 2.0 * cin / gamm1;
                    double riemm = vnref - 2.0 * cref / gamm1;
                    double vnb = half * (riemp + riemm);
                    t = vnb >= 0.0 ? s : p.ref_sa;
                }
            }
            nut[r] = t;
        }
    }
    void turbBoundary() { calcVist(); turbBc(); }

    // UTurbSpectrum::CalcSpectrum1Equ + TurbSpectrum::CalcFaceSpectrum1Equ
    // (codes/uturb/src/UTurbSpectrum.cpp:132-240, codes/turb/src/TurbSpectrum.cpp:75-134)
    void turbSpectrum() {
        std::fill(impsrT.begin(), impsrT.end(), 0.0);
        matL.assign(nFaces, 0.0); matR.assign(nFaces, 0.0);
        for (int c = 0; c < nCells; ++c) {
            double ts = timestep[c] * p.turb_cfl_ratio;
            impsrT[c] += (1.0 / ts) * vol[c];
        }
        for (int f = 0; f < nFaces; ++f) {
            int l = lc[f], r = rc[f];
            double r1 = 0, r2 = 0, m1 = 0, m2 = 0;
            double vnl = xfn[f] * q[IU][l] + yfn[f] * q[IV][l] + zfn[f] * q[IW][l] - 0.0;
            double vnr = xfn[f] * q[IU][r] + yfn[f] * q[IV][r] + zfn[f] * q[IW][r] - 0.0;
            double vnRel = half * (vnl + vnr);
            double absVn = std::fabs(vnRel);
            r1 += area[f] * half * absVn;
            r2 += area[f] * half * absVn;
            m1 += area[f] * half * (-vnl - absVn);
            m2 += area[f] * half * (vnr - absVn);
            double orl = 1.0 / (q[IR][l] + SMALL), orr = 1.0 / (q[IR][r] + SMALL);
            double nuet1 = visl[l] * orl + nut[l], nuet2 = visl[r] * orr + nut[r];
            double nueff = std::fabs(half * (nuet1 + nuet2));
            double cv = half * (vol[l] + vol[r]);
            double ovol = 1.0 / cv;
            double areaS2 = area[f] * area[f];
            r1 += oreynolds * ovol * (sa.osigma * nueff * areaS2);
            r2 += oreynolds * ovol * (sa.osigma * nueff * areaS2);
            m1 += -oreynolds * ovol * (sa.osigma * nueff * areaS2);
            m2 += -oreynolds * ovol * (sa.osigma * nueff * areaS2);
            impsrT[l] += r1; impsrT[r] += r2;
            matL[f] += m1; matR[f] += m2;
        }
    }

    // TurbCom::CalcSrcSa (codes/turb/src/TurbCom.cpp:771-881) per cell, added as
    // UTurbSrcFlux::Update1Equ does (codes/uturb/src/UTurbSrcFlux.cpp:315-319)
    void turbSource() {
        grad(nut, dnutdx, dnutdy, dnutdz);   // uturb_grad (GG cell-weighted for igrad 0)
        for (int c = 0; c < nCells; ++c) {
            double dudx = dqdx[IU][c], dudy = dqdy[IU][c], dudz = dqdz[IU][c];
            double dvdx = dqdx[IV][c], dvdy = dqdy[IV][c], dvdz = dqdz[IV][c];
            double dwdx = dqdx[IW][c], dwdy = dqdy[IW][c], dwdz = dqdz[IW][c];
            double rho = q[IR][c], nuet = nut[c], vl = visl[c];
            double olam = rho / (vl + SMALL);
            double ls = walldist[c];
            double d2 = ls * ls, od2 = 1.0 / d2;
            // CalcWorkVar / CalcSaProd, TurbCom.cpp:429-466
            double work1 = dudx + dvdy + dwdz;
            double work2 = SQR3(dudx, dudy, dudz);
            double work3 = SQR3(dudy + dvdx, dvdz + dwdy, dwdx + dudz);
            double work4 = DIST3(dwdy - dvdz, dudz - dwdx, dvdx - dudy);
            if (p.iprod_sa == 1) {
                double stp = 2.0 * work2 + work3 - two3rd * work1 * work1;
                work4 = std::sqrt(std::fabs(stp));
            } else if (p.iprod_sa == 4) {
                double stp = 2.0 * work2 + work3 - two3rd * work1 * work1;
                double str = work4;
                work4 = str - 2.0 * MAXd(0.0, str - std::sqrt(std::fabs(stp)));
            } else if (p.iprod_sa == 5) {
                double stp = 2.0 * work2 + work3 - two3rd * work1 * work1;
                double str = work4;
                stp = std::fabs(stp);
                work4 = str * (1.0 - MAXd(0.0, (str * str - stp) / (str * str + stp + SMALL)));
            }
            double str = work4;
            double xsi = nuet * olam + SMALL;
            double xsi3 = xsi * xsi * xsi;
            double fv1 = xsi3 / (xsi3 + sa.cv13);
            double fv2 = 1.0 - xsi / (1.0 + xsi * fv1);
            double rs = nuet * sa.okarm2 * od2 * oreynolds;
            double nuetRs = nuet * rs;
            double sBar = rs * fv2;
            double omega = str;
            double std_;
            if (sBar >= -sa.sac2 * omega) {
                std_ = omega + sBar;
            } else {
                double term1 = (sa.sac2 * sa.sac2 * omega + sa.sac3 * sBar);
                double term2 = (sa.sac3 - 2 * sa.sac2) * omega - sBar;
                std_ = omega + omega * term1 / term2;
            }
            double ostd = 1.0 / (std_ + SMALL);
            double r = rs * ostd;
            r = MINd(r, 10.0);
            double r5 = std::pow(r, 5);
            double g = r + sa.cw2 * (r5 * r - r);
            double g6 = std::pow(g, 6);
            double or6 = 1.0 / 6.0;
            double fw = g * std::pow((1.0 + sa.cw36) / (g6 + sa.cw36), or6);
            double xsi2 = xsi * xsi;
            double ft2 = 0.0;
            if (p.ft2_flag) ft2 = sa.ct3 * std::exp(-sa.ct4 * xsi2) * 1.0;
            double grd2 = SQR3(dnutdx[c], dnutdy[c], dnutdz[c]);
            double prod = sa.cb1 * (1.0 - ft2) * std_ * nuet;
            double diff = sa.cb2s * grd2 * oreynolds;
            double dest = (sa.cw1k * fw - sa.cb1 * ft2) * nuetRs;
            diff = MINd(p.rprod * prod, diff);
            double srcTerm = prod - dest;
            srcTerm += diff;
            double dfv2dk = (3.0 * sa.cv13 * std::pow(fv1 / (xsi + SMALL), 2) - 1.0) / std::pow(1.0 + xsi * fv1, 2);
            double dsdnu = oreynolds * sa.okarm2 * od2 * (fv2 + xsi * dfv2dk);
            double dfwdg = fw / (g + SMALL) * (1.0 - g6 / (g6 + sa.cw36));
            double dgdr = 1.0 + sa.cw2 * (6.0 * r5 - 1.0);
            double drdnu = oreynolds * sa.okarm2 * od2 * ostd * (1.0 - nuet * ostd * dsdnu);
            double dfwdnu = dfwdg * dgdr * drdnu;
            double prod0 = sa.cb1 * (1.0 - ft2) * std_;
            double dest0 = (sa.cw1 * fw - sa.cb1 * ft2 * sa.okarm2) * nuet * od2 * oreynolds;
            double prodp = sa.cb1 * ((1.0 - ft2) * dsdnu);
            double destp = (sa.cw1 * (fw + dfwdnu * nuet) - sa.cb1 * ft2 * sa.okarm2) * od2 * oreynolds;
            double prde0 = prod0 - dest0, prdep = prodp - destp;
            double part1 = -half * (prde0 - std::fabs(prde0));
            double part2 = -half * (prdep - std::fabs(prdep)) * nuet;
            double spec = part1 + part2;
            impsrT[c] += spec * vol[c];
            resT[c] += srcTerm * vol[c];
        }
    }

    // UTurbInvFlux (codes/uturb/src/UTurbInvFlux.cpp:55-202) with the first
    // order turbulent and NS face states (turb_ilim = tns_ilim = -1) and
    // TurbInvFlux::RoeFlux (codes/turb/src/TurbInvFlux.cpp:78-98), rho_coef = 1
    void turbInvFlux() {
        for (int f = 0; f < nFaces; ++f) {
            int l = lc[f], r = rc[f];
            double t1 = nut[l], t2 = nut[r];
            double u1 = q[IU][l], v1 = q[IV][l], w1 = q[IW][l], u2 = q[IU][r], v2 = q[IV][r], w2 = q[IW][r];
            if (f < nBFaces) {
                double tm = half * (nut[l] + nut[r]);
                t1 = t2 = tm;
                if (bcType[f] == OFG_BC_SOLID_SURFACE) {
                    u1 = u2 = bc_q[IU][f]; v1 = v2 = bc_q[IV][f]; w1 = w2 = bc_q[IW][f];
                } else {
                    u1 = u2 = half * (q[IU][l] + q[IU][r]);
                    v1 = v2 = half * (q[IV][l] + q[IV][r]);
                    w1 = w2 = half * (q[IW][l] + q[IW][r]);
                }
            }
            double vnl = xfn[f] * u1 + yfn[f] * v1 + zfn[f] * w1 - 0.0;
            double vnr = xfn[f] * u2 + yfn[f] * v2 + zfn[f] * w2 - 0.0;
            double vnl_p = half * (vnl + std::fabs(vnl));
            double vnr_n = half * (vnr - std::fabs(vnr));
            double coef_l = vnl_p * (1.0 * 1.0 + (1.0 - 1.0) * 0.0);
            double coef_r = vnr_n * (1.0 * 1.0 + (1.0 - 1.0) * 0.0);
            double flux = coef_l * t1 + coef_r * t2;
            double v = area[f] * flux;
            resT[l] -= v;
            if (f >= nBFaces) resT[r] += v;
        }
    }

    static double calcAngle(double dx, double dy, double dz, double dist) {
        double result = dist / (DIST3(dx, dy, dz) + SMALL);
        if (result > 1.0) result = 1.0;
        if (result < -1.0) result = -1.0;
        return std::asin(result) * 180.0 / PI;
    }
    // UTurbVisFlux::CalcVisFlux1Equ with the VIS_TEST face gradient
    // (codes/uturb/src/UTurbVisFlux.cpp:64-407, codes/usolver/src/VisGrad.cpp:60-120,248-290)
    void turbVisFlux() {
        for (int f = 0; f < nFaces; ++f) {
            int l = lc[f], r = rc[f];
            double xn = xfn[f], yn = yfn[f], zn = zfn[f];
            double q1 = nut[l], q2 = nut[r];
            double q11 = q1, q22 = q2;
            double qf = half * (q1 + q2);
            double dxl = xcc[l] - xfc[f], dyl = ycc[l] - yfc[f], dzl = zcc[l] - zfc[f];
            double dxr = xcc[r] - xfc[f], dyr = ycc[r] - yfc[f], dzr = zcc[r] - zfc[f];
            double d1 = xn * dxl + yn * dyl + zn * dzl;
            double d2 = xn * dxr + yn * dyr + zn * dzr;
            double dxnl = xn * d1 - dxl, dynl = yn * d1 - dyl, dznl = zn * d1 - dzl;
            double dxnr = xn * d2 - dxr, dynr = yn * d2 - dyr, dznr = zn * d2 - dzr;
            double angle1 = calcAngle(dxl, dyl, dzl, -d1);
            double angle2 = calcAngle(dxr, dyr, dzr, d2);
            double dqdn = 0.0;
            if (angle1 > 20.0 && angle2 > 20.0) {
                q11 += dnutdx[l] * dxnl + dnutdy[l] * dynl + dnutdz[l] * dznl;
                q22 += dnutdx[r] * dxnr + dnutdy[r] * dynr + dnutdz[r] * dznr;
                qf = half * (q1 + q2);
            }
            if (angle1 > 0.0 && angle2 > 0.0 && std::fabs(d1) > SMALL && std::fabs(d2) > SMALL) {
                double dtmp = d1 * d1 + d2 * d2;
                double c1 = d1 * d1 / dtmp, c2 = 1.0 - c1;
                if (f < nBFaces) { c1 = 1.0; c2 = 0.0; }
                double dqdn1 = (q11 - qf) / d1;
                double dqdn2 = (q22 - qf) / d2;
                dqdn = c1 * dqdn1 + c2 * dqdn2;
            }
            double orl = 1.0 / (q[IR][l] + SMALL), orr = 1.0 / (q[IR][r] + SMALL);
            double visl_nv = half * (visl[l] * orl + visl[r] * orr);
            double vist_nv = half * (q1 + q2);
            double comVis = (visl_nv + vist_nv) * sa.osigma;
            double flux = -oreynolds * comVis * dqdn * area[f];
            resT[l] -= flux;
            if (f >= nBFaces) resT[r] += flux;
        }
    }

    // UTurbLusgs sweeps (codes/uturb/src/UTurbLusgs.cpp:90-300) with
    // TurbLusgs::GetStandardFluxIncrement (codes/turb/src/TurbLusgs.cpp:123-129)
    void turbLower() {
        for (int k = 0; k < nCells; ++k) {
            int c = keyOrder[k];
            double rhs0 = 0.0;
            for (int f : c2f[c]) {
                if (key[lc[f]] > key[c] || key[rc[f]] > key[c]) continue;
                bool swap = rc[f] == c;
                int nb = swap ? lc[f] : rc[f];
                double m = swap ? matL[f] : matR[f];
                rhs0 += m * dnut[nb];
            }
            dnut[c] = (resT[c] - rhs0) / impsrT[c];
        }
    }
    void turbUpper() {
        for (int k = nCells - 1; k >= 0; --k) {
            int c = keyOrder[k];
            double rhs0 = 0.0;
            for (int f : c2f[c]) {
                if (key[lc[f]] < key[c] || key[rc[f]] < key[c]) continue;
                bool swap = rc[f] == c;
                int nb = swap ? lc[f] : rc[f];
                double m = swap ? matL[f] : matR[f];
                rhs0 += m * dnut[nb];
            }
            dnut[c] += (-rhs0) / impsrT[c];
        }
    }
    // UTurbUpdate::UpdateFlowField1EquStd / TurbUpdate::CalcFlowField1Equ (crelax = 1)
    void turbUpdate() {
        for (int c = 0; c < nCells; ++c) {
            double qOld = nut[c], qNew = qOld + dnut[c];
            nut[c] = (1.0 - 1.0) * qOld + 1.0 * qNew;
        }
    }
    void turbRelax() {
        std::fill(dnut.begin(), dnut.end(), 0.0);
        std::fill(resT.begin(), resT.end(), -0.0);
        // TurbCalcRHS, codes/turb/src/TurbRhs.cpp:57-70
        turbBc();
        turbSpectrum();
        turbSource();
        turbInvFlux();
        turbVisFlux();
        turbLower();
        turbUpper();
        turbUpdate();
        turbBoundary();
    }

    // ======================= one outer iteration =======================
    // TimeIntegral::Lusgs (codes/solver/src/TimeIntegral.cpp:113-130)
    void nsRelax() {
        for (int e = 0; e < NEQ; ++e) std::fill(dq[e].begin(), dq[e].end(), 0.0);
        calcTimeStep();
        loadResiduals();
        updateResiduals();
        lusgsLower();
        lusgsUpper();
        updateFlowfield();
        calcBoundary();
    }

    // CALC_LHS, ULhs::CalcLHS (codes/usolver/src/ULhs.cpp:47-65): res *= (dt/vol)
    // * lhscoef; under MULTI_STAGE the update's increment field is the residual
    // itself (UNsField::Init, codes/uns/src/UNsCom.cpp:85-88)
    void calcLhs(double lhscoef) {
        for (int e = 0; e < NEQ; ++e)
            for (int c = 0; c < nCells; ++c) {
                res[e][c] *= (timestep[c] / vol[c]) * lhscoef;
                dq[e][c] = res[e][c];
            }
    }
    // TimeIntegral::RungeKutta (codes/solver/src/TimeIntegral.cpp:81-111) on the
    // finest grid: the time step once, then per stage the residual, CALC_LHS
    // with lhscoef = rk_coef[stage] = 1/(stage+1) (Ctrl::Init,
    // codes/global/src/Ctrl.cpp:72-77), UPDATE_FLOWFIELD from the current state
    // and CALC_BOUNDARY.  LOAD_Q stores q in a field that UPDATE_FLOWFIELD does
    // not read (GetUpdateField, codes/update/src/Update.cpp:64-86, assigns its
    // pointer parameters by value), so it changes nothing here.
    void nsRelaxMultiStage() {
        calcTimeStep();
        for (int k = 0; k < p.rk_stage; ++k) {
            loadResiduals();
            updateResiduals();
            calcLhs(1.0 / (k + 1));
            updateFlowfield();
            calcBoundary();
        }
    }

    int step(int n) {
        for (int it = 0; it < n; ++it) {
            ++outerSteps;
            // MG::StrongIter: NS relaxation, then the turbulence solver
            if (p.time_integral == 1) nsRelaxMultiStage();
            else nsRelax();
            if (turb()) turbRelax();
            double rms[NEQ]; bool nan;
            residualRms(rms, &nan);
            for (int e = 0; e < NEQ; ++e) resHist.push_back(rms[e]);
            if (turb()) {
                double s = 0.0;
                for (int c = 0; c < nCells; ++c) { s += resT[c] * resT[c]; if (std::isnan(resT[c])) nan = true; }
                turbHist.push_back(std::sqrt(s / nCells));
            }
            if (nan) { err = "NotANumber in residual"; return OFG_E_NAN; }
        }
        return 0;
    }

    // ======================= aerodynamic forces =======================
    // CalcAeroForce (codes/force/src/AeroForceTask.cpp:186-451, the
    // compressible branch): over the solid-wall faces, in face order, the
    // pressure force (wall pressure extrapolated with the interior cell's
    // gradient, cp = 2 (p_w - p_inf)) and, with a viscous model, the viscous
    // force from the interior cell's velocity gradient corrected along the
    // cell-to-ghost line (CorrectGrad, codes/usolver/src/VisGrad.cpp:355-365)
    // and the stress of Stress::CalcForce (codes/solver/src/Stress.cpp:40-64)
    // with the interior laminar viscosity.  Sums as AeroForce::AddForce
    // (codes/force/src/Force.cpp:202-208), coefficients as
    // AeroForceInfo::CalcCoef (:254-269).  out[13]: total force x y z,
    // pressure part x y z, viscous part x y z, CL, CD, CD_pres, CD_vis.
    void forces(double aref, double *out) {
        double tot[3] = {0, 0, 0}, pr[3] = {0, 0, 0}, vs[3] = {0, 0, 0};
        for (int f = 0; f < nBFaces; ++f) {
            if (bcType[f] != OFG_BC_SOLID_SURFACE) continue;
            int l = lc[f], r = rc[f];
            double fanx = xfn[f] * area[f], fany = yfn[f] * area[f], fanz = zfn[f] * area[f];
            double dx = xfc[f] - xcc[l], dy = yfc[f] - ycc[l], dz = zfc[f] - zcc[l];
            double wp = q[IP][l] + dqdx[IP][l] * dx + dqdy[IP][l] * dy + dqdz[IP][l] * dz;
            if (wp < 0.0) wp = q[IP][l];
            double cp = 2.0 * (wp - inflow[IP]);
            double fp[3] = {fanx * cp, fany * cp, fanz * cp};
            double fv[3] = {0.0, 0.0, 0.0};
            if (p.vismodel > 0) {
                double g[3][3];   // [u v w][x y z]
                for (int e = 0; e < 3; ++e) { g[e][0] = dqdx[IU + e][l]; g[e][1] = dqdy[IU + e][l]; g[e][2] = dqdz[IU + e][l]; }
                dx = xcc[r] - xcc[l]; dy = ycc[r] - ycc[l]; dz = zcc[r] - zcc[l];
                double ods = 1.0 / DIST3(dx, dy, dz);
                dx *= ods; dy *= ods; dz *= ods;
                for (int e = 0; e < 3; ++e) {
                    double fOld = g[e][0] * dx + g[e][1] * dy + g[e][2] * dz;
                    double fnew = (q[IU + e][r] - q[IU + e][l]) * ods;
                    double df = fnew - fOld;
                    g[e][0] += df * dx; g[e][1] += df * dy; g[e][2] += df * dz;
                }
                double vis = visl[l];
                double divv2p3 = two3rd * (g[0][0] + g[1][1] + g[2][2]);
                double txx = vis * (2.0 * g[0][0] - divv2p3);
                double tyy = vis * (2.0 * g[1][1] - divv2p3);
                double tzz = vis * (2.0 * g[2][2] - divv2p3);
                double txy = vis * (g[0][1] + g[1][0]);
                double txz = vis * (g[0][2] + g[2][0]);
                double tyz = vis * (g[1][2] + g[2][1]);
                double coef = -2.0 * area[f] * oreynolds;
                fv[0] = coef * (xfn[f] * txx + yfn[f] * txy + zfn[f] * txz);
                fv[1] = coef * (xfn[f] * txy + yfn[f] * tyy + zfn[f] * tyz);
                fv[2] = coef * (xfn[f] * txz + yfn[f] * tyz + zfn[f] * tzz);
            }
            for (int k = 0; k < 3; ++k) {
                tot[k] += fp[k] + fv[k];
                pr[k] += fp[k];
                vs[k] += fv[k];
            }
        }
        for (int k = 0; k < 3; ++k) { out[k] = tot[k]; out[3 + k] = pr[k]; out[6 + k] = vs[k]; }
        double aoa = p.aoa_degree * PI / 180.0, aos = p.sideslip_degree * PI / 180.0;
        double sina = std::sin(aoa), cosa = std::cos(aoa), sinb = std::sin(aos), cosb = std::cos(aos);
        double cf[3], cpres[3];
        for (int k = 0; k < 3; ++k) { cf[k] = tot[k] / aref; cpres[k] = pr[k] / aref; }
        out[9] = -sina * cf[0] + cosa * cf[1];
        out[10] = cosa * cosb * cf[0] + sina * cosb * cf[1] + sinb * cf[2];
        out[11] = cosa * cosb * cpres[0] + sina * cosb * cpres[1] + sinb * cpres[2];
        out[12] = out[10] - out[11];
    }
};

#include "oracle_ins.h"

// ============================ C interface ============================
extern "C" {

// The colour-major renumbering of a mesh (perm[new] = old), for running the
// reference itself in the order the GPU path sweeps; returns the colour count.
int oro_colour_order(int nCells, int nFaces, int nBFaces, const int *lCells, const int *rCells, int *perm) {
    if (nCells <= 0 || nBFaces < 0 || nFaces < nBFaces || !lCells || !rCells || !perm) return -1;
    std::vector<int> lc(lCells, lCells + nFaces), rc(rCells, rCells + nFaces);
    std::vector<std::vector<int>> c2f(nCells);
    for (int f = nBFaces; f < nFaces; ++f) {
        if (lc[f] < 0 || rc[f] < 0 || lc[f] >= nCells || rc[f] >= nCells) return -1;
        c2f[lc[f]].push_back(f); c2f[rc[f]].push_back(f);
    }
    return colourMajor(nCells, nBFaces, c2f, lc, rc, perm);
}

void *oro_create(const ofg_params *p) {
    Oracle *o = new Oracle();
    o->p = *p;
    return o;
}
void oro_destroy(void *h) { delete (Oracle *)h; }

int oro_set_mesh(void *h, int nn, const double *x, const double *y, const double *z, int nf, const int *fnc,
                 const int *fn, const int *l, const int *r, int nc, int nb, const int *bct, const double *wd) {
    return ((Oracle *)h)->setMesh(nn, x, y, z, nf, fnc, fn, l, r, nc, nb, bct, wd);
}
int oro_init_flowfield(void *h) { ((Oracle *)h)->initFlowfield(); return 0; }
int oro_step(void *h, int n) { return ((Oracle *)h)->step(n); }

// individual tasks (for per-kernel parity tests)
int oro_task(void *h, const char *name) {
    Oracle *o = (Oracle *)h;
    std::string s(name);
    if (s == "ZERO_DQ_FIELD") { for (int e = 0; e < NEQ; ++e) std::fill(o->dq[e].begin(), o->dq[e].end(), 0.0); }
    else if (s == "CALC_TIME_STEP") o->calcTimeStep();
    else if (s == "LOAD_RESIDUALS") o->loadResiduals();
    else if (s == "UPDATE_RESIDUALS") o->updateResiduals();
    else if (s == "LUSGS_LOWER_SWEEP") o->lusgsLower();
    else if (s == "LUSGS_UPPER_SWEEP") o->lusgsUpper();
    else if (s == "UPDATE_FLOWFIELD_LUSGS") o->updateFlowfield();
    else if (s == "CALC_BOUNDARY") o->calcBoundary();
    else if (s == "INIT_LUSGS") {}   // CLusgsInit: no-op (codes/implicit/src/ImplicitTaskReg.cpp:69-72)
    // the turbulence solver's tasks (tid TURB_SOLVER)
    else if (s == "TURB:ZERO_DQ_FIELD") std::fill(o->dnut.begin(), o->dnut.end(), 0.0);
    else if (s == "TURB:CALC_TIME_STEP" || s == "TURB:LOAD_RESIDUALS" || s == "TURB:INIT_LUSGS") {
        if (s == "TURB:LOAD_RESIDUALS") std::fill(o->resT.begin(), o->resT.end(), -0.0);
    }
    else if (s == "TURB:UPDATE_RESIDUALS") { o->turbBc(); o->turbSpectrum(); o->turbSource(); o->turbInvFlux(); o->turbVisFlux(); }
    else if (s == "TURB:LUSGS_LOWER_SWEEP") o->turbLower();
    else if (s == "TURB:LUSGS_UPPER_SWEEP") o->turbUpper();
    else if (s == "TURB:UPDATE_FLOWFIELD_LUSGS") o->turbUpdate();
    else if (s == "TURB:CALC_BOUNDARY") o->turbBoundary();
    else if (s == "NEXT_STEP") ++o->outerSteps;
    else return OFG_E_ARG;
    return 0;
}

// field access, reference layout
int64_t oro_field(void *h, const char *name, double *out) {
    Oracle *o = (Oracle *)h;
    std::string s(name);
    auto put = [&](const std::vector<double> *v, int ne, int64_t n) -> int64_t {
        if (out) for (int e = 0; e < ne; ++e) std::copy(v[e].begin(), v[e].begin() + n, out + e * n);
        return ne * n;
    };
    int64_t nT = o->nT, nF = o->nFaces;
    if (s == "q") return put(o->q, NEQ, nT);
    if (s == "dq") return put(o->dq, NEQ, nT);
    if (s == "res") return put(o->res, NEQ, nT);
    if (s == "dqdx") return put(o->dqdx, NEQ, nT);
    if (s == "dqdy") return put(o->dqdy, NEQ, nT);
    if (s == "dqdz") return put(o->dqdz, NEQ, nT);
    if (s == "limiter") return put(o->limiter, NEQ, nT);
    if (s == "timestep") return put(&o->timestep, 1, nT);
    if (s == "invsr") return put(&o->invsr, 1, nT);
    if (s == "vissr") return put(&o->vissr, 1, nT);
    if (s == "impsr") return put(&o->impsr, 1, nT);
    if (s == "tempr") return put(&o->tempr, 1, nT);
    if (s == "visl") return put(&o->visl, 1, nT);
    if (s == "vist") return put(&o->vist, 1, nT);
    if (s == "vol") return put(&o->vol, 1, nT);
    if (s == "xcc") return put(&o->xcc, 1, nT);
    if (s == "ycc") return put(&o->ycc, 1, nT);
    if (s == "zcc") return put(&o->zcc, 1, nT);
    if (s == "area") return put(&o->area, 1, nF);
    if (s == "xfn") return put(&o->xfn, 1, nF);
    if (s == "yfn") return put(&o->yfn, 1, nF);
    if (s == "zfn") return put(&o->zfn, 1, nF);
    if (s == "xfc") return put(&o->xfc, 1, nF);
    if (s == "yfc") return put(&o->yfc, 1, nF);
    if (s == "zfc") return put(&o->zfc, 1, nF);
    if (s == "reshist") { if (out) std::copy(o->resHist.begin(), o->resHist.end(), out); return (int64_t)o->resHist.size(); }
    if (s == "turbreshist") { if (out) std::copy(o->turbHist.begin(), o->turbHist.end(), out); return (int64_t)o->turbHist.size(); }
    if (s == "turbq") return put(&o->nut, 1, nT);
    if (s == "turbres") return put(&o->resT, 1, nT);
    if (s == "turbdq") return put(&o->dnut, 1, nT);
    if (s == "turbimpsr") return put(&o->impsrT, 1, nT);
    if (s == "walldist") return put(&o->walldist, 1, nT);
    if (s == "nfixes") { if (out) out[0] = double(o->nFixes); return 1; }
    return -1;
}
int oro_set_q(void *h, const double *qin) {
    Oracle *o = (Oracle *)h;
    for (int e = 0; e < NEQ; ++e) std::copy(qin + e * (int64_t)o->nT, qin + (e + 1) * (int64_t)o->nT, o->q[e].begin());
    o->initReference();
    o->calcBoundary();
    return 0;
}
long oro_outer_steps(void *h) { return ((Oracle *)h)->outerSteps; }

// ---- the incompressible solver on an oracle's mesh (oracle_ins.h) ----
void *oro_ins_create(void *h) {
    Oracle *o = (Oracle *)h;
    InsOracle *s = new InsOracle(*o);
    std::string why;
    if (!s->supported(why)) { o->err = why; delete s; return nullptr; }
    return s;
}
void oro_ins_destroy(void *s) { delete (InsOracle *)s; }
// per boundary face u v w of the wall (the reference's ins_bc data)
int oro_ins_set_wall(void *s, const double *uvw) {
    InsOracle *n = (InsOracle *)s;
    for (int f = 0; f < n->nB; ++f) { n->wu[f] = uvw[3 * f]; n->wv[f] = uvw[3 * f + 1]; n->ww[f] = uvw[3 * f + 2]; }
    return 0;
}
int oro_ins_init(void *s) { ((InsOracle *)s)->init(); return 0; }
// maxIter > 0: MG::Run's loop up to inner step maxIter; returns the steps run
int oro_ins_run(void *s, int maxIter) { return ((InsOracle *)s)->run(maxIter); }
// remax_up vp wp pp, then per solve (u v w p) GMRES iterations and residual
int oro_ins_stats(void *s, double *out) {
    InsOracle *n = (InsOracle *)s;
    for (int k = 0; k < 4; ++k) { out[k] = n->remax[k]; out[4 + k] = n->linIts[k]; out[8 + k] = n->linRes[k]; }
    out[12] = (double)n->innerSteps;
    return 0;
}
int64_t oro_ins_field(void *s, const char *name, double *out) {
    InsOracle *n = (InsOracle *)s;
    std::string k(name);
    const std::vector<double> *v = nullptr;
    if (k == "uc") v = &n->uc; else if (k == "vc") v = &n->vc; else if (k == "wc") v = &n->wc;
    else if (k == "pp") v = &n->pp; else if (k == "spc") v = &n->spc; else if (k == "spp") v = &n->spp;
    else if (k == "bp") v = &n->bp; else if (k == "buc") v = &n->buc; else if (k == "bvc") v = &n->bvc;
    else if (k == "fq") v = &n->fq; else if (k == "ajp") v = &n->ajp; else if (k == "ai0") v = &n->ai0;
    else if (k == "ai1") v = &n->ai1; else if (k == "Fn") v = &n->Fn; else if (k == "dqqdx") v = &n->dqqdx;
    else if (k == "uf") v = &n->uf; else if (k == "vf") v = &n->vf;
    else return oro_field(&n->m, name, out);
    if (out) std::copy(v->begin(), v->end(), out);
    return (int64_t)v->size();
}
int oro_forces(void *h, double aref, double *out) {
    if (!h || !out || !(aref > 0.0)) return OFG_E_ARG;
    ((Oracle *)h)->forces(aref, out);
    return 0;
}

}  // extern "C"

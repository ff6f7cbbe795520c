// C ABI (include/oneflow_b200.h): context lifecycle, mesh preprocessing
// (metrics, CSR cell->face lists, LU-SGS level schedules), state transfer,
// one entry point per reference task, and the graph-captured outer iteration.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "ofg_ctx.h"

using namespace ofg;

namespace {

const double SMALL = 1.0e-40;
const double PI = 3.141592653589793;

#define CK(call)                                                                           \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return c->fail(e_ == cudaErrorMemoryAllocation ? OFG_E_NOMEM : OFG_E_CUDA,     \
                           std::string(#call) + ": " + cudaGetErrorString(e_));            \
    } while (0)

int launch(ofg_ctx *c, int task) {
    int rc = c->p.precision == OFG_PREC_MIXED ? launch_task_f32(c, task, c->stream) : launch_task_f64(c, task, c->stream);
    if (rc) return rc;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return c->fail(OFG_E_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    return OFG_OK;
}

int sync(ofg_ctx *c) {
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return c->fail(OFG_E_CUDA, std::string("stream: ") + cudaGetErrorString(e));
    return OFG_OK;
}

// ---------------------------------------------------------------------------
// Metrics: UnsGrid::CalcMetrics (codes/geometry/src/UnsGrid.cpp:469-900) with
// FaceMesh::CalcFaceNormal2D/3D and CalcFaceCenter2D/3D
// (codes/geometry/src/FaceMesh.cpp:112-286).
// ---------------------------------------------------------------------------
void compute_metrics(ofg_ctx *c, int dim, const std::vector<double> &xN, const std::vector<double> &yN,
                     const std::vector<double> &zN, const std::vector<int> &fOff, const std::vector<int> &fNod) {
    int nF = c->nFaces, nC = c->nCells, nB = c->nBFaces, nT = c->nT;
    c->xfn.assign(nF, 0); c->yfn.assign(nF, 0); c->zfn.assign(nF, 0); c->area.assign(nF, 0);
    c->xfc.assign(nF, 0); c->yfc.assign(nF, 0); c->zfc.assign(nF, 0);
    c->xcc.assign(nT, 0); c->ycc.assign(nT, 0); c->zcc.assign(nT, 0); c->vol.assign(nT, 0);
    auto &xfn = c->xfn, &yfn = c->yfn, &zfn = c->zfn, &area = c->area, &xfc = c->xfc, &yfc = c->yfc, &zfc = c->zfc;
    auto &xcc = c->xcc, &ycc = c->ycc, &zcc = c->zcc, &vol = c->vol;
    const auto &lc = c->lc, &rc = c->rc;
    if (dim == 2) {
        for (int f = 0; f < nF; ++f) {
            int p1 = fNod[fOff[f]], p2 = fNod[fOff[f] + 1];
            xfn[f] = yN[p2] - yN[p1];
            yfn[f] = xN[p1] - xN[p2];
            zfn[f] = 0.0;
            area[f] = std::sqrt(xfn[f] * xfn[f] + yfn[f] * yfn[f] + zfn[f] * zfn[f]);
        }
        for (int f = 0; f < nF; ++f) {
            double oa = 1.0 / (area[f] + SMALL);
            xfn[f] *= oa; yfn[f] *= oa; zfn[f] *= oa;
        }
        for (int f = 0; f < nF; ++f) {
            int p1 = fNod[fOff[f]], p2 = fNod[fOff[f] + 1];
            xfc[f] = 0.5 * (xN[p1] + xN[p2]);
            yfc[f] = 0.5 * (yN[p1] + yN[p2]);
            zfc[f] = 0.5 * (zN[p1] + zN[p2]);
        }
        for (int f = 0; f < nF; ++f) {
            int l = lc[f], r = rc[f];
            double dot = (xfc[f] * xfn[f] + yfc[f] * yfn[f] + zfc[f] * zfn[f]) * area[f];
            xcc[l] += xfc[f] * dot; ycc[l] += yfc[f] * dot; zcc[l] += zfc[f] * dot; vol[l] += dot;
            if (f >= nB) { xcc[r] -= xfc[f] * dot; ycc[r] -= yfc[f] * dot; zcc[r] -= zfc[f] * dot; vol[r] -= dot; }
        }
        for (int i = 0; i < nC; ++i) {
            double tmp = 1.0 / (1.5 * vol[i] + SMALL);
            xcc[i] *= tmp; ycc[i] *= tmp; zcc[i] *= tmp;
            vol[i] *= 0.5;
            if (vol[i] <= 0.0) vol[i] = -vol[i];
        }
    } else {
        for (int f = 0; f < nF; ++f) {
            int n = fOff[f + 1] - fOff[f];
            const int *fi = &fNod[fOff[f]];
            for (int i = 0; i < n; ++i) {
                int p1 = fi[i], p2 = fi[(i + 1) % n];
                double dx1 = xN[p1], dy1 = yN[p1], dz1 = zN[p1], dx2 = xN[p2], dy2 = yN[p2], dz2 = zN[p2];
                xfn[f] += 0.5 * (dy1 * dz2 - dy2 * dz1);
                yfn[f] += 0.5 * (dz1 * dx2 - dz2 * dx1);
                zfn[f] += 0.5 * (dx1 * dy2 - dx2 * dy1);
            }
            area[f] = std::sqrt(xfn[f] * xfn[f] + yfn[f] * yfn[f] + zfn[f] * zfn[f]);
        }
        for (int f = 0; f < nF; ++f) {
            double oa = 1.0 / (area[f] + SMALL);
            xfn[f] *= oa; yfn[f] *= oa; zfn[f] *= oa;
        }
        const double third = 1.0 / 3.0;
        for (int f = 0; f < nF; ++f) {
            int n = fOff[f + 1] - fOff[f];
            const int *fi = &fNod[fOff[f]];
            double x0 = 0, y0 = 0, z0 = 0;
            for (int i = 0; i < n; ++i) { x0 += xN[fi[i]]; y0 += yN[fi[i]]; z0 += zN[fi[i]]; }
            double factor = 1.0 / n;
            x0 *= factor; y0 *= factor; z0 *= factor;
            double sx = 0, sy = 0, sz = 0, sarea = 0;
            for (int i = 0; i < n; ++i) {
                int p1 = fi[i], p2 = fi[(i + 1) % n];
                double dx1 = xN[p1] - x0, dy1 = yN[p1] - y0, dz1 = zN[p1] - z0;
                double dx2 = xN[p2] - x0, dy2 = yN[p2] - y0, dz2 = zN[p2] - z0;
                double x00 = third * (xN[p1] + xN[p2] + x0);
                double y00 = third * (yN[p1] + yN[p2] + y0);
                double z00 = third * (zN[p1] + zN[p2] + z0);
                double anx = dy1 * dz2 - dy2 * dz1, any = dz1 * dx2 - dz2 * dx1, anz = dx1 * dy2 - dx2 * dy1;
                double fa = 0.5 * std::sqrt(anx * anx + any * any + anz * anz);
                if (anx * xfn[f] + any * yfn[f] + anz * zfn[f] < 0.0) fa = -fa;
                sarea += fa;
                sx += fa * x00; sy += fa * y00; sz += fa * z00;
            }
            double os = 1.0 / (sarea + SMALL);
            xfc[f] = sx * os; yfc[f] = sy * os; zfc[f] = sz * os;
        }
        for (int f = 0; f < nF; ++f) {
            int l = lc[f], r = rc[f];
            int n = fOff[f + 1] - fOff[f];
            const int *fi = &fNod[fOff[f]];
            for (int i = 0; i < n; ++i) {
                int p2 = fi[i], p3 = fi[(i + 1) % n];
                double x21 = xN[p2] - xfc[f], y21 = yN[p2] - yfc[f], z21 = zN[p2] - zfc[f];
                double x31 = xN[p3] - xfc[f], y31 = yN[p3] - yfc[f], z31 = zN[p3] - zfc[f];
                double nx = y21 * z31 - y31 * z21, ny = z21 * x31 - z31 * x21, nz = x21 * y31 - x31 * y21;
                double trix = xfc[f] + xN[p2] + xN[p3];
                double triy = yfc[f] + yN[p2] + yN[p3];
                double triz = zfc[f] + zN[p2] + zN[p3];
                double tmp = nx * trix + ny * triy + nz * triz;
                trix *= tmp; triy *= tmp; triz *= tmp;
                xcc[l] += trix; ycc[l] += triy; zcc[l] += triz; vol[l] += tmp;
                xcc[r] -= trix; ycc[r] -= triy; zcc[r] -= triz; vol[r] -= tmp;
            }
        }
        for (int i = 0; i < nC; ++i) {
            double tmp = 1.0 / (4.0 * vol[i] + SMALL);
            xcc[i] *= tmp; ycc[i] *= tmp; zcc[i] *= tmp;
            vol[i] /= 18.0;
            if (vol[i] <= 0.0) vol[i] = -vol[i];
        }
    }
    for (int f = 0; f < nB; ++f) {
        int l = lc[f], r = f + nC;
        if (area[f] > SMALL) {
            double tmp = 2.0 * ((xcc[l] - xfc[f]) * xfn[f] + (ycc[l] - yfc[f]) * yfn[f] + (zcc[l] - zfc[f]) * zfn[f]);
            xcc[r] = xcc[l] - xfn[f] * tmp; ycc[r] = ycc[l] - yfn[f] * tmp; zcc[r] = zcc[l] - zfn[f] * tmp;
        } else {
            xcc[r] = -xcc[l] + 2.0 * xfc[f]; ycc[r] = -ycc[l] + 2.0 * yfc[f]; zcc[r] = -zcc[l] + 2.0 * zfc[f];
        }
        vol[r] = vol[l];
    }
}

// Greedy colouring of the cell graph (interior faces) in natural order and
// the colour-major order: colours ascending, ids ascending inside a colour.
// Returns the number of colours, fills perm[position] = cell.
int colour_major_order(int nCells, int nFaces, int nBFaces, const int *lCells, const int *rCells, int *perm) {
    std::vector<int> deg(nCells + 1, 0);
    for (int f = nBFaces; f < nFaces; ++f) {
        int l = lCells[f], r = rCells[f];
        if (l < 0 || r < 0 || l >= nCells || r >= nCells) return OFG_E_ARG;
        deg[l + 1]++; deg[r + 1]++;
    }
    for (int i = 0; i < nCells; ++i) deg[i + 1] += deg[i];
    std::vector<int> adj(deg[nCells]);
    std::vector<int> pos(deg.begin(), deg.end() - 1);
    for (int f = nBFaces; f < nFaces; ++f) {
        int l = lCells[f], r = rCells[f];
        adj[pos[l]++] = r; adj[pos[r]++] = l;
    }
    std::vector<int> col(nCells, -1);
    int ncol = 0;
    std::vector<int> mark(64, -1);
    for (int i = 0; i < nCells; ++i) {
        for (int k = deg[i]; k < deg[i + 1]; ++k) {
            int cc = col[adj[k]];
            if (cc >= 0) { if (cc >= (int)mark.size()) mark.resize(cc + 1, -1); mark[cc] = i; }
        }
        int cc = 0;
        while (cc < (int)mark.size() && mark[cc] == i) ++cc;
        col[i] = cc;
        ncol = std::max(ncol, cc + 1);
    }
    std::vector<int> cnt(ncol + 1, 0);
    for (int i = 0; i < nCells; ++i) cnt[col[i] + 1]++;
    for (int k = 0; k < ncol; ++k) cnt[k + 1] += cnt[k];
    for (int i = 0; i < nCells; ++i) perm[cnt[col[i]]++] = i;
    return ncol;
}

// Sweep key: the position of every cell in the LU-SGS order (ghosts after
// every interior cell, as their ids nCells + f are in the reference).
void build_sweep_key(ofg_ctx *c) {
    int N = c->nCells;
    c->keyOrder.resize(N);
    if (c->p.sweep_order == 1) {
        colour_major_order(N, c->nFaces, c->nBFaces, c->lc.data(), c->rc.data(), c->keyOrder.data());
    } else {
        for (int i = 0; i < N; ++i) c->keyOrder[i] = i;
    }
    c->key.assign(c->nT, 0);
    for (int k = 0; k < N; ++k) c->key[c->keyOrder[k]] = k;
    for (int f = 0; f < c->nBFaces; ++f) c->key[N + f] = N + f;
}

// Level schedule of a sequential sweep: a cell's level is one more than the
// deepest level among the neighbours it reads (lower: smaller key; upper:
// larger key).
void build_levels(ofg_ctx *c, bool lower, std::vector<int> &order, std::vector<int> &off) {
    int N = c->nCells;
    const std::vector<int> &key = c->key;
    std::vector<int> lev(N, 0);
    int maxl = 0;
    auto visit = [&](int i) {
        int L = 0;
        for (int k = c->c2f_off[i]; k < c->c2f_off[i + 1]; ++k) {
            int f = c->c2f[k];
            if (f < c->nBFaces) continue;
            int nb = c->lc[f] == i ? c->rc[f] : c->lc[f];
            if (lower ? key[nb] < key[i] : key[nb] > key[i]) L = std::max(L, lev[nb] + 1);
        }
        lev[i] = L;
        maxl = std::max(maxl, L);
    };
    if (lower) for (int k = 0; k < N; ++k) visit(c->keyOrder[k]);
    else for (int k = N - 1; k >= 0; --k) visit(c->keyOrder[k]);
    off.assign(maxl + 2, 0);
    for (int i = 0; i < N; ++i) off[lev[i] + 1]++;
    for (int l = 0; l <= maxl; ++l) off[l + 1] += off[l];
    order.assign(N, 0);
    std::vector<int> pos(off.begin(), off.end() - 1);
    // inside a level the cells are independent; both sweeps list them in
    // ascending sweep order
    for (int k = 0; k < N; ++k) { int i = c->keyOrder[k]; order[pos[lev[i]]++] = i; }
}

// Per-cell neighbour lists in ascending face id (the c2f order), one int2 per
// face: {face | side << 31, neighbour}, side = 1 where the cell is the face's
// right cell.  Full lists for the residual and gradient gathers; for the
// sweeps, the interior faces to cells earlier (lower) and later (upper) in
// the sweep order.
struct NbLists {
    std::vector<int> nbOff, nbl, loOff, lol, upOff, upl;
};

void build_lists(const ofg_ctx *c, NbLists &L) {
    int N = c->nCells;
    L.nbOff.assign(N + 1, 0); L.loOff.assign(N + 1, 0); L.upOff.assign(N + 1, 0);
    L.nbl.clear(); L.lol.clear(); L.upl.clear();
    L.nbl.reserve(2 * c->c2f.size());
    for (int i = 0; i < N; ++i) {
        int ki = c->key[i];
        for (int k = c->c2f_off[i]; k < c->c2f_off[i + 1]; ++k) {
            int f = c->c2f[k];
            bool right = c->rc[f] == i && f >= c->nBFaces;
            int nb = right ? c->lc[f] : c->rc[f];
            int tag = int(unsigned(f) | (right ? 0x80000000u : 0u));
            L.nbl.push_back(tag); L.nbl.push_back(nb);
            if (f < c->nBFaces) continue;
            if (c->key[nb] < ki) { L.lol.push_back(tag); L.lol.push_back(nb); }
            else { L.upl.push_back(tag); L.upl.push_back(nb); }
        }
        L.nbOff[i + 1] = int(L.nbl.size() / 2);
        L.loOff[i + 1] = int(L.lol.size() / 2);
        L.upOff[i + 1] = int(L.upl.size() / 2);
    }
}

// face records [F][8] (nx ny nz area xfc yfc zfc dist) and cell records [nT][4]
// (xcc ycc zcc vol) at the face precision
template <typename R>
void pack_geometry(const ofg_ctx *c, std::vector<R> &fg, std::vector<R> &cg) {
    fg.assign((size_t)c->nFaces * 8, R(0));
    for (int f = 0; f < c->nFaces; ++f) {
        R *o = &fg[(size_t)f * 8];
        o[0] = R(c->xfn[f]); o[1] = R(c->yfn[f]); o[2] = R(c->zfn[f]); o[3] = R(c->area[f]);
        o[4] = R(c->xfc[f]); o[5] = R(c->yfc[f]); o[6] = R(c->zfc[f]);
        // normal distance between the two cell centres, for the LU-SGS viscous
        // radius (UNsLusgs::CalcViscousTerm): the same value, bit for bit, as
        // the sweep computes from either side (both signs flip there)
        int l = c->lc[f], r = c->rc[f];
        o[7] = R(std::fabs(c->xfn[f] * (c->xcc[r] - c->xcc[l]) + c->yfn[f] * (c->ycc[r] - c->ycc[l]) +
                           c->zfn[f] * (c->zcc[r] - c->zcc[l])));
    }
    cg.assign((size_t)c->nT * 4, R(0));
    for (int i = 0; i < c->nT; ++i) {
        R *o = &cg[(size_t)i * 4];
        o[0] = R(c->xcc[i]); o[1] = R(c->ycc[i]); o[2] = R(c->zcc[i]); o[3] = R(c->vol[i]);
    }
}

template <typename T>
int upload(ofg_ctx *c, T **d, const T *h, size_t n) {
    if (*d) { cudaFree(*d); *d = nullptr; }
    if (n == 0) n = 1;
    CK(cudaMalloc((void **)d, n * sizeof(T)));
    if (h) CK(cudaMemcpy(*d, h, n * sizeof(T), cudaMemcpyHostToDevice));
    return OFG_OK;
}

int upload_bytes(ofg_ctx *c, void **d, const void *h, size_t bytes) {
    if (*d) { cudaFree(*d); *d = nullptr; }
    if (bytes == 0) bytes = 16;
    CK(cudaMalloc(d, bytes));
    if (h) CK(cudaMemcpy(*d, h, bytes, cudaMemcpyHostToDevice));
    else CK(cudaMemset(*d, 0, bytes));
    return OFG_OK;
}

void derive_params(ofg_ctx *c) {
    const ofg_params &p = c->p;
    DevParams &d = c->dp;
    d.ischeme = p.ischeme; d.ilim = p.ilim; d.vismodel = p.vismodel; d.visSRModel = p.visSRModel;
    d.visTimeStepModel = p.visTimeStepModel; d.ieigenfix = p.ieigenfix; d.timestepModel = p.timestepModel;
    d.isowallbc = p.isowallbc; d.dim = p.dimension; d.precision = p.precision; d.venkat_kh3 = p.venkat_kh3;
    d.igrad = p.igrad;
    d.ivischeme = p.ivischeme;
    d.gama = p.gama_ref; d.centropy1 = p.centropy1; d.centropy2 = p.centropy2; d.vencat_coef = p.vencat_coef;
    d.reynolds = p.reynolds; d.oreynolds = 1.0 / p.reynolds; d.oprl = 1.0 / p.prl; d.oprt = 1.0 / p.prt;
    d.const_cp = 1.0 / ((p.gama_ref - 1.0) * (p.mach_ref * p.mach_ref));
    d.statecoef = 1.0 / (p.gama_ref * (p.mach_ref * p.mach_ref));   // Chemical::CalcStateCoefNs
    double aoa = p.aoa_degree * PI / 180.0, aos = p.sideslip_degree * PI / 180.0;
    d.inflow[IR] = 1.0;
    d.inflow[IU] = 1.0 * std::cos(aoa) * std::cos(aos);
    d.inflow[IV] = 1.0 * std::sin(aoa) * std::cos(aos);
    d.inflow[IW] = 1.0 * std::sin(aos);
    d.inflow[IP] = d.statecoef * 1.0 * 1.0 / 1.0;
    d.twall = p.twall_dim / p.tref_dim;
    d.sutherland_ts = 110.4 / p.tref_dim;
    d.max_time_ratio = p.max_time_ratio;
    d.global_dt = p.global_dt;
    d.nut_inf = p.ref_sa;   // TurbCom::InitInflow: inflow[ISA] = ref_sa for the SA model
    d.max_vis_ratio = p.max_vis_ratio;
    d.turb_cfl_ratio = p.turb_cfl_ratio;
    d.rprod = p.rprod;
    d.iprod_sa = p.iprod_sa;
    d.ft2_flag = p.ft2_flag;
    {
        double karm = 0.41, karm2 = karm * karm, okarm2 = 1.0 / karm2, cb1 = 0.1355, cb2 = 0.622, cv1 = 7.1;
        double sigma = 2.0 / 3.0, osigma = 1.0 / sigma, cw1 = cb1 * okarm2 + (1.0 + cb2) / sigma;
        d.sa_cb1 = cb1; d.sa_cv13 = cv1 * cv1 * cv1; d.sa_cw2 = 0.3; d.sa_cw36 = std::pow(2.0, 6);
        d.sa_ct3 = 1.2; d.sa_ct4 = 0.5; d.sa_osigma = osigma; d.sa_cw1 = cw1; d.sa_sac2 = 0.7; d.sa_sac3 = 0.9;
        d.sa_cb2s = osigma * cb2; d.sa_cw1k = cw1 * karm2; d.sa_okarm2 = okarm2;
    }
}

double host_sutherland(const DevParams &P, double t) {
    double t3 = t * t * t;
    return std::sqrt(t3) * (1 + P.sutherland_ts) / (t + P.sutherland_ts);
}

bool has_turb(const ofg_ctx *c) { return c->p.vismodel >= 3; }
bool multi_stage(const ofg_ctx *c) { return c->p.time_integral == 1; }

int check_tid(ofg_ctx *c, int tid) {
    if (!c) return OFG_E_ARG;
    if (tid != OFG_NS_SOLVER && !(tid == OFG_TURB_SOLVER && has_turb(c)))
        return c->fail(OFG_E_ARG, "no such solver in this context (tid 1 needs vismodel 3)");
    if (!c->haveMesh) return c->fail(OFG_E_STATE, "no mesh uploaded");
    if (!c->haveState) return c->fail(OFG_E_STATE, "no flow field: call ofg_init_flowfield or ofg_upload_state");
    return OFG_OK;
}

void destroy_graphs(ofg_ctx *c) {
    for (int i = 0; i < 2; ++i) {
        if (c->graph[i]) { cudaGraphExecDestroy(c->graph[i]); c->graph[i] = nullptr; }
        if (c->graphT[i]) { cudaGraphDestroy(c->graphT[i]); c->graphT[i] = nullptr; }
    }
    c->graphGen++;
}

}  // namespace

extern "C" {

int ofg_version(void) { return 1; }

int ofg_params_size(void) { return int(sizeof(ofg_params)); }

void ofg_default_params(ofg_params *p) {
    std::memset(p, 0, sizeof(*p));
    p->dimension = 2; p->ischeme = 1; p->ilim = 0; p->igrad = 0; p->ieigenfix = 1; p->timestepModel = 0;
    p->ncfl = 100; p->visSRModel = 2; p->visTimeStepModel = 1; p->vismodel = 1; p->ivischeme = 0;
    p->isowallbc = 0; p->iprod_sa = 2; p->ft2_flag = 0; p->turb_ilim = -1; p->precision = OFG_PREC_FP64;
    p->vencat_coef = 1.0e-4; p->centropy1 = 1.0e-4; p->centropy2 = 1.0e-4; p->cflst = 0.1; p->cfled = 10.0;
    p->max_time_ratio = 1.0e10; p->global_dt = 1.0e-3; p->mach_ref = 0.2; p->reynolds = 1.0e6;
    p->gama_ref = 1.4; p->prl = 0.72; p->prt = 0.9; p->tref_dim = 300.0; p->twall_dim = 300.0;
    p->inflow_viscosity = 0.01; p->rprod = 1.0; p->turb_cfl_ratio = 1.0; p->ref_sa = 0.1; p->max_vis_ratio = 1.0e6;
    p->time_integral = 2; p->rk_stage = 1;
}

int ofg_create(const ofg_params *p, ofg_ctx **out) {
    if (!p || !out) return OFG_E_ARG;
    *out = nullptr;
    if (p->dimension != 2 && p->dimension != 3) return OFG_E_ARG;
    if (p->ischeme != 1 && p->ischeme != 12) return OFG_E_ARG;
    if (p->ilim < -1 || p->ilim > 2) return OFG_E_ARG;
    if (p->igrad < 0 || p->igrad > 2) return OFG_E_ARG;
    if (p->precision != OFG_PREC_FP64 && p->precision != OFG_PREC_MIXED) return OFG_E_ARG;
    if (p->sweep_order != 0 && p->sweep_order != 1) return OFG_E_ARG;
    if (p->vismodel != 0 && p->vismodel != 1 && p->vismodel != 3) return OFG_E_ARG;   // Euler, laminar, SA
    if (p->vismodel == 3 && p->turb_ilim != -1) return OFG_E_ARG;   // first-order SA convection only
    if (p->ivischeme < 0 || p->ivischeme > 4) return OFG_E_ARG;   // VIS_STD, AVER, TEST, NEW1, NEW2
    if (p->time_integral < 0 || p->time_integral > 2) return OFG_E_ARG;
    // the multi-stage scheme: NS solver only, 1..16 stages
    if (p->time_integral == 1 && (p->rk_stage < 1 || p->rk_stage > 16 || p->vismodel == 3)) return OFG_E_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return OFG_E_CUDA;
    ofg_ctx *c = new ofg_ctx();
    c->p = *p;
    derive_params(c);
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) { delete c; return OFG_E_CUDA; }
    *out = c;
    return OFG_OK;
}

void ofg_destroy(ofg_ctx *c) {
    if (!c) return;
    cudaStreamSynchronize(c->stream);
    destroy_graphs(c);
    void *ptrs[] = {c->d_lcb, c->d_bct, c->d_nb_off, c->d_nbl, c->d_lo_off, c->d_lol, c->d_up_off, c->d_upl,
                    c->d_lowOrder, c->d_upOrder, c->d_key, c->d_fgeo, c->d_cgeo, c->d_wdist, c->d_wall, c->d_wallG,
                    c->d_fgeoD, c->d_fofs, c->d_lr, c->d_fout, c->d_lowOff, c->d_upOff,
                    c->d_q[0], c->d_q[1], c->d_qs[0], c->d_qs[1], c->d_res, c->d_dq, c->d_dt, c->d_invsr, c->d_vissr, c->d_rad,
                    c->d_bcq, c->d_partial, c->d_npart, c->d_tpart, c->d_red, c->d_redCount, c->d_stage, c->d_scal, c->d_hist, c->d_gl, c->d_mm, c->d_fix,
                    c->d_nut, c->d_dnut, c->d_resT, c->d_impsrT, c->d_matL, c->d_matR, c->d_thist, c->d_gnut};
    for (void *v : ptrs) if (v) cudaFree(v);
    cudaStreamDestroy(c->ownStream ? c->ownStream : c->stream);
    delete c;
}

const char *ofg_last_error(const ofg_ctx *c) { return c ? c->err.c_str() : "null context"; }

int ofg_upload_mesh(ofg_ctx *c, int nNodes, const double *xN, const double *yN, const double *zN, int nFaces,
                    const int *faceNodeCount, const int *faceNodes, const int *lCells, const int *rCells, int nCells,
                    int nBFaces, const int *bcType, const double *wall_dist) {
    if (!c) return OFG_E_ARG;
    // the context's sizes change before the arrays are checked: after a
    // refused upload no call runs kernels until an upload succeeds
    c->haveMesh = false;
    c->haveState = false;
    if (nNodes <= 0 || nFaces <= 0 || nCells <= 0 || nBFaces < 0 || nBFaces > nFaces)
        return c->fail(OFG_E_ARG, "bad mesh sizes");
    if (!xN || !yN || !zN || !faceNodeCount || !faceNodes || !lCells || !rCells || (nBFaces && !bcType))
        return c->fail(OFG_E_ARG, "null mesh array");
    destroy_graphs(c);
    c->nCells = nCells; c->nBFaces = nBFaces; c->nFaces = nFaces; c->nT = nCells + nBFaces;
    std::vector<double> X(xN, xN + nNodes), Y(yN, yN + nNodes), Z(zN, zN + nNodes);
    std::vector<int> fOff(nFaces + 1, 0);
    for (int f = 0; f < nFaces; ++f) {
        int n = faceNodeCount[f];
        if (n < 2 || (c->p.dimension == 3 && n < 3)) return c->fail(OFG_E_ARG, "face with too few nodes");
        fOff[f + 1] = fOff[f] + n;
    }
    std::vector<int> fNod(faceNodes, faceNodes + fOff[nFaces]);
    for (int v : fNod) if (v < 0 || v >= nNodes) return c->fail(OFG_E_ARG, "face node index out of range");
    c->lc.assign(lCells, lCells + nFaces);
    c->rc.assign(rCells, rCells + nFaces);
    // UnsGrid::ReadGridFaceTopology: a negative left cell means the face is reversed
    for (int f = 0; f < nFaces; ++f)
        if (c->lc[f] < 0) {
            std::reverse(fNod.begin() + fOff[f], fNod.begin() + fOff[f + 1]);
            std::swap(c->lc[f], c->rc[f]);
        }
    for (int f = 0; f < nBFaces; ++f) c->rc[f] = f + nCells;   // UnsGrid::NormalizeBc
    for (int f = 0; f < nFaces; ++f) {
        if (c->lc[f] < 0 || c->lc[f] >= nCells) return c->fail(OFG_E_ARG, "left cell out of range");
        if (f >= nBFaces && (c->rc[f] < 0 || c->rc[f] >= nCells || c->rc[f] == c->lc[f]))
            return c->fail(OFG_E_ARG, "interior face with a bad right cell");
    }
    c->bct.assign(bcType, bcType + nBFaces);
    for (int t : c->bct)
        if (t < 1 || t > 6)
            return c->fail(OFG_E_ARG, "unsupported boundary type (codes 1-6; interface, overset, periodic and pole "
                                      "faces belong to multi-zone or structured cases)");
    // CSR cell->face in ascending face id (CellTopo::CalcC2f)
    c->c2f_off.assign(nCells + 1, 0);
    for (int f = 0; f < nFaces; ++f) {
        c->c2f_off[c->lc[f] + 1]++;
        if (f >= nBFaces) c->c2f_off[c->rc[f] + 1]++;
    }
    for (int i = 0; i < nCells; ++i) c->c2f_off[i + 1] += c->c2f_off[i];
    c->c2f.assign(c->c2f_off[nCells], 0);
    std::vector<int> pos(c->c2f_off.begin(), c->c2f_off.end() - 1);
    for (int f = 0; f < nFaces; ++f) {
        c->c2f[pos[c->lc[f]]++] = f;
        if (f >= nBFaces) c->c2f[pos[c->rc[f]]++] = f;
    }
    {   // FNV-1a of the face->cell lists: the autotuner's cache key for this mesh
        unsigned long long h = 1469598103934665603ull;
        auto mix = [&](unsigned v) { for (int b = 0; b < 4; ++b) { h ^= (v >> (8 * b)) & 0xffu; h *= 1099511628211ull; } };
        mix(unsigned(nCells)); mix(unsigned(nFaces)); mix(unsigned(nBFaces));
        for (int f = 0; f < nFaces; ++f) { mix(unsigned(c->lc[f])); mix(unsigned(c->rc[f])); }
        c->meshHash = h;
    }
    build_sweep_key(c);
    build_levels(c, true, c->lowOrder, c->lowOff);
    build_levels(c, false, c->upOrder, c->upOff);

    // ---- device copies ----
    int rc;
    const bool mixed = c->p.precision == OFG_PREC_MIXED;
    {
        NbLists L;
        build_lists(c, L);
        std::vector<int> lcb(c->lc.begin(), c->lc.begin() + nBFaces);
        if ((rc = upload(c, &c->d_lcb, lcb.data(), nBFaces))) return rc;
        if ((rc = upload(c, &c->d_nb_off, L.nbOff.data(), L.nbOff.size()))) return rc;
        if ((rc = upload(c, &c->d_nbl, L.nbl.data(), L.nbl.size()))) return rc;
        if ((rc = upload(c, &c->d_lo_off, L.loOff.data(), L.loOff.size()))) return rc;
        if ((rc = upload(c, &c->d_lol, L.lol.data(), L.lol.size()))) return rc;
        if ((rc = upload(c, &c->d_up_off, L.upOff.data(), L.upOff.size()))) return rc;
        if ((rc = upload(c, &c->d_upl, L.upl.data(), L.upl.size()))) return rc;
    }
    // metrics on the GPU (UnsGrid::CalcMetrics); for an SA solve without a
    // caller-supplied wall distance, CALC_WALL_DIST on the GPU as well
    c->xN = std::move(X); c->yN = std::move(Y); c->zN = std::move(Z);
    c->fOff = std::move(fOff); c->fNod = std::move(fNod);
    const bool needWall = has_turb(c) && !wall_dist;
    c->wdist.assign(nCells, 0.0);
    if (wall_dist) std::copy(wall_dist, wall_dist + nCells, c->wdist.begin());
    if ((rc = gpu_geometry(c, c->xN, c->yN, c->zN, c->fOff, c->fNod, true, needWall))) return rc;
    for (int i = 0; i < nCells; ++i)
        if (!(c->vol[i] > 0.0)) return c->fail(OFG_E_ARG, "degenerate cell volume");
    if ((rc = upload(c, &c->d_bct, c->bct.data(), nBFaces))) return rc;
    if ((rc = upload(c, &c->d_lowOrder, c->lowOrder.data(), nCells))) return rc;
    if ((rc = upload(c, &c->d_upOrder, c->upOrder.data(), nCells))) return rc;
    if ((rc = upload(c, &c->d_lowOff, c->lowOff.data(), c->lowOff.size()))) return rc;
    if ((rc = upload(c, &c->d_upOff, c->upOff.data(), c->upOff.size()))) return rc;
    if ((rc = upload(c, &c->d_key, c->key.data(), c->nT))) return rc;
    if ((rc = upload(c, &c->d_wdist, c->wdist.data(), nCells))) return rc;
    {
        // solid-wall faces and their FP64 geometry for the force integration
        // (the quantities CalcAeroForce forms per face, AeroForceTask.cpp:262-330)
        std::vector<int> wall;
        std::vector<double> wg;
        for (int f = 0; f < nBFaces; ++f) {
            if (c->bct[f] != OFG_BC_SOLID_SURFACE) continue;
            int l = c->lc[f], r = c->rc[f];
            wall.push_back(f); wall.push_back(l);
            double dx = c->xcc[r] - c->xcc[l], dy = c->ycc[r] - c->ycc[l], dz = c->zcc[r] - c->zcc[l];
            double ods = 1.0 / std::sqrt(dx * dx + dy * dy + dz * dz);
            double g[16] = {c->xfn[f] * c->area[f], c->yfn[f] * c->area[f], c->zfn[f] * c->area[f],
                            c->xfn[f], c->yfn[f], c->zfn[f], c->area[f],
                            c->xfc[f] - c->xcc[l], c->yfc[f] - c->ycc[l], c->zfc[f] - c->zcc[l],
                            dx * ods, dy * ods, dz * ods, ods, 0.0, 0.0};
            wg.insert(wg.end(), g, g + 16);
        }
        c->nWall = int(wall.size() / 2);
        if ((rc = upload(c, &c->d_wall, wall.data(), wall.size()))) return rc;
        if ((rc = upload(c, &c->d_wallG, wg.data(), wg.size()))) return rc;
    }
    if (mixed) {
        std::vector<float> fg, cg;
        pack_geometry(c, fg, cg);
        if ((rc = upload_bytes(c, &c->d_fgeo, fg.data(), fg.size() * sizeof(float)))) return rc;
        if ((rc = upload_bytes(c, &c->d_cgeo, cg.data(), cg.size() * sizeof(float)))) return rc;
        // the face pass's inputs: FP64 face records, face-local offsets
        // (x_f - x_L, x_f - x_R formed in FP64 and rounded once, and their
        // lengths) and the two cells of each face; and its output records
        std::vector<double> fgd, cgd;
        pack_geometry(c, fgd, cgd);
        if ((rc = upload(c, &c->d_fgeoD, fgd.data(), fgd.size()))) return rc;
        std::vector<float> fo((size_t)nFaces * FOFS);
        std::vector<int> lr((size_t)nFaces * 2);
        for (int f = 0; f < nFaces; ++f) {
            int l = c->lc[f], r = c->rc[f];
            double a[3] = {c->xfc[f] - c->xcc[l], c->yfc[f] - c->ycc[l], c->zfc[f] - c->zcc[l]};
            double b[3] = {c->xfc[f] - c->xcc[r], c->yfc[f] - c->ycc[r], c->zfc[f] - c->zcc[r]};
            float *o = &fo[(size_t)f * FOFS];
            for (int k = 0; k < 3; ++k) { o[k] = float(a[k]); o[3 + k] = float(b[k]); }
            o[6] = float(std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]));
            o[7] = float(std::sqrt(b[0] * b[0] + b[1] * b[1] + b[2] * b[2]));
            lr[2 * (size_t)f] = l; lr[2 * (size_t)f + 1] = r;
        }
        if ((rc = upload(c, &c->d_fofs, fo.data(), fo.size()))) return rc;
        if ((rc = upload(c, &c->d_lr, lr.data(), lr.size()))) return rc;
        if ((rc = upload<double>(c, &c->d_fout, nullptr, (size_t)nFaces * FOR))) return rc;
    } else {
        std::vector<double> fg, cg;
        pack_geometry(c, fg, cg);
        if ((rc = upload_bytes(c, &c->d_fgeo, fg.data(), fg.size() * sizeof(double)))) return rc;
        if ((rc = upload_bytes(c, &c->d_cgeo, cg.data(), cg.size() * sizeof(double)))) return rc;
        for (void **v : {(void **)&c->d_fgeoD, (void **)&c->d_fofs, (void **)&c->d_lr, (void **)&c->d_fout})
            if (*v) { cudaFree(*v); *v = nullptr; }
    }
    size_t nT = c->nT, N = nCells;
    if ((rc = upload<double>(c, &c->d_q[0], nullptr, nT * REC))) return rc;
    if ((rc = upload<double>(c, &c->d_q[1], nullptr, nT * REC))) return rc;
    for (int i = 0; i < 2; ++i) {
        if (c->d_qs[i]) { cudaFree(c->d_qs[i]); c->d_qs[i] = nullptr; }
        if (mixed) CK(cudaMalloc(&c->d_qs[i], nT * REC * sizeof(float)));
    }
    size_t rs = mixed ? sizeof(float) : sizeof(double);
    if (c->d_stage) { cudaFree(c->d_stage); c->d_stage = nullptr; }   // sized by nT: re-made on first use
    if ((rc = upload<double>(c, &c->d_res, nullptr, N * NEQ))) return rc;
    if ((rc = upload_bytes(c, &c->d_dq, nullptr, N * DQR * rs))) return rc;
    if ((rc = upload<double>(c, &c->d_dt, nullptr, N))) return rc;
    if ((rc = upload<double>(c, &c->d_invsr, nullptr, N))) return rc;
    if ((rc = upload<double>(c, &c->d_vissr, nullptr, N))) return rc;
    if ((rc = upload<double>(c, &c->d_rad, nullptr, N))) return rc;
    if ((rc = upload<double>(c, &c->d_bcq, nullptr, (size_t)std::max(nBFaces, 1) * NEQ))) return rc;
    // (the gradient kernel's limiter extremes: 10 per block, blocks of 64 threads at the smallest)
    c->nPartialMax = std::max<size_t>((N + 63) / 64 * 10, 2 * 148 * NEQ) + 16;
    if ((rc = upload<double>(c, &c->d_partial, nullptr, c->nPartialMax))) return rc;
    size_t nb128 = (N + 127) / 128;
    if ((rc = upload<double>(c, &c->d_npart, nullptr, nb128 * NEQ))) return rc;
    if ((rc = upload<double>(c, &c->d_tpart, nullptr, nb128))) return rc;
    CK(cudaMemset(c->d_npart, 0, nb128 * NEQ * sizeof(double)));
    CK(cudaMemset(c->d_tpart, 0, nb128 * sizeof(double)));
    if ((rc = upload<double>(c, &c->d_red, nullptr, (size_t)kRedBlocks * NEQ))) return rc;
    if ((rc = upload<unsigned int>(c, &c->d_redCount, nullptr, 1))) return rc;
    CK(cudaMemset(c->d_redCount, 0, sizeof(unsigned int)));
    if ((rc = upload<double>(c, &c->d_scal, nullptr, 32))) return rc;
    c->histCap = 1 << 16;
    if ((rc = upload<double>(c, &c->d_hist, nullptr, (size_t)c->histCap * NEQ))) return rc;
    if ((rc = upload<int>(c, &c->d_fix, nullptr, 1 + c->fixcap))) return rc;
    if ((rc = upload_bytes(c, &c->d_gl, nullptr, N * GLR * rs))) return rc;
    bool venkatGlobal = c->p.ilim == 2 && !c->p.venkat_kh3;
    if ((rc = upload_bytes(c, &c->d_mm, nullptr, venkatGlobal ? N * MMR * rs : 0))) return rc;
    CK(cudaMemset(c->d_bcq, 0, (size_t)std::max(nBFaces, 1) * NEQ * sizeof(double)));
    CK(cudaMemset(c->d_scal, 0, 32 * sizeof(double)));
    CK(cudaMemset(c->d_fix, 0, (1 + c->fixcap) * sizeof(int)));
    if (has_turb(c)) {
        for (int i = 0; i < nCells; ++i)   // supplied, or computed on the GPU above
            if (!(c->wdist[i] > 0.0)) return c->fail(OFG_E_ARG, "wall distance must be positive");
        if ((rc = upload<double>(c, &c->d_nut, nullptr, nT))) return rc;
        if ((rc = upload<double>(c, &c->d_dnut, nullptr, nT))) return rc;
        if ((rc = upload<double>(c, &c->d_resT, nullptr, N))) return rc;
        if ((rc = upload<double>(c, &c->d_impsrT, nullptr, N))) return rc;
        if ((rc = upload<double>(c, &c->d_matL, nullptr, nFaces))) return rc;
        if ((rc = upload<double>(c, &c->d_matR, nullptr, nFaces))) return rc;
        if ((rc = upload<double>(c, &c->d_thist, nullptr, c->histCap))) return rc;
        if ((rc = upload_bytes(c, &c->d_gnut, nullptr, N * 4 * rs))) return rc;
        CK(cudaMemset(c->d_dnut, 0, nT * sizeof(double)));
    }
    c->haveMesh = true;
    c->haveState = false;
    c->outerSteps = 0;
    c->hist.clear();
    c->thist.clear();
    return OFG_OK;
}

int ofg_init_flowfield(ofg_ctx *c) {
    if (!c) return OFG_E_ARG;
    if (!c->haveMesh) return c->fail(OFG_E_STATE, "no mesh uploaded");
    destroy_graphs(c);
    // UNsRestart::InitRestart: q = inflow everywhere (ghosts included)
    std::vector<double> rec((size_t)c->nT * REC, 0.0);
    const DevParams &P = c->dp;
    double t = P.inflow[IP] / (P.statecoef * P.inflow[IR] * 1.0);
    double ml = std::max(0.0, host_sutherland(P, t));
    for (int i = 0; i < c->nT; ++i) {
        double *o = &rec[(size_t)i * REC];
        for (int e = 0; e < NEQ; ++e) o[e] = P.inflow[e];
        o[ITT] = t; o[IML] = ml; o[IMT] = 0.0;
    }
    c->cur = 0;
    CK(cudaMemcpy(c->d_q[0], rec.data(), rec.size() * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->d_q[1], rec.data(), rec.size() * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemset(c->d_scal, 0, 32 * sizeof(double)));
    c->outerSteps = 0;
    c->hist.clear();
    c->thist.clear();
    c->haveState = true;
    c->lastResBuf = -1;
    c->pendingNext = false;
    int rc = launch(c, T_BOUNDARY_CUR);   // NsInitFinal -> NsCalcBoundary
    if (rc) return rc;
    if (has_turb(c)) {
        // UTurbRestart::InitRestart (nu~ = ref_sa everywhere) + TurbInitFinal
        std::vector<double> nut(c->nT, P.nut_inf);
        CK(cudaMemcpyAsync(c->d_nut, nut.data(), nut.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        if ((rc = launch(c, T_TURB_BOUNDARY_CUR))) return rc;
    }
    return sync(c);
}

// staging buffer for state transfers: [5][nT] FP64, allocated on first use
static int ensure_stage(ofg_ctx *c) {
    if (c->d_stage) return OFG_OK;
    CK(cudaMalloc(&c->d_stage, (size_t)NEQ * c->nT * sizeof(double)));
    return OFG_OK;
}

int ofg_upload_state(ofg_ctx *c, int tid, const double *q) {
    if (!c || !q) return OFG_E_ARG;
    if (tid != OFG_NS_SOLVER && !(tid == OFG_TURB_SOLVER && has_turb(c)))
        return c->fail(OFG_E_ARG, "no such solver in this context");
    if (!c->haveMesh) return c->fail(OFG_E_STATE, "no mesh uploaded");
    if (c->pendingNext) return c->fail(OFG_E_STATE, "UPDATE_FLOWFIELD without CALC_BOUNDARY");
    int rc;
    if (tid == OFG_TURB_SOLVER) {
        if (!c->haveState) return c->fail(OFG_E_STATE, "upload the NS state first");
        CK(cudaMemcpyAsync(c->d_nut, q, (size_t)c->nT * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        if ((rc = launch(c, T_TURB_BOUNDARY_CUR))) return rc;
        return sync(c);
    }
    // host [5][nT] -> staging -> the records of the current buffer (the eddy
    // viscosity, a field of its own in the reference, is kept); then
    // temperature, laminar viscosity and the ghost states as after a restart
    if ((rc = ensure_stage(c))) return rc;
    CK(cudaMemcpyAsync(c->d_stage, q, (size_t)NEQ * c->nT * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    if (!c->haveState) {   // first state: start the records from zero (no eddy viscosity yet)
        CK(cudaMemsetAsync(c->d_q[c->cur], 0, (size_t)c->nT * REC * sizeof(double), c->stream));
    }
    if ((rc = launch(c, T_PACK_STATE))) return rc;
    c->haveState = true;
    c->lastResBuf = -1;
    c->pendingNext = false;
    if ((rc = launch(c, T_BOUNDARY_CUR))) return rc;
    return sync(c);
}

int ofg_download_state(ofg_ctx *c, int tid, double *q) {
    int rc = check_tid(c, tid);
    if (rc) return rc;
    if (!q) return c->fail(OFG_E_ARG, "null output");
    if (tid == OFG_TURB_SOLVER) {
        CK(cudaMemcpyAsync(q, c->d_nut, (size_t)c->nT * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        return sync(c);
    }
    if ((rc = ensure_stage(c))) return rc;
    if ((rc = launch(c, T_UNPACK_STATE))) return rc;
    CK(cudaMemcpyAsync(q, c->d_stage, (size_t)NEQ * c->nT * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    return sync(c);
}

int ofg_calc_wall_dist(ofg_ctx *c) {
    if (!c) return OFG_E_ARG;
    if (!c->haveMesh) return c->fail(OFG_E_STATE, "no mesh uploaded");
    int rc = gpu_geometry(c, c->xN, c->yN, c->zN, c->fOff, c->fNod, false, true);
    if (rc) return rc;
    CK(cudaMemcpy(c->d_wdist, c->wdist.data(), (size_t)c->nCells * sizeof(double), cudaMemcpyHostToDevice));
    return OFG_OK;
}

// ---------------------------------------------------------------------------
// Restart files: the single-zone record Restart::Dump writes through
// DataBook::WriteFile (codes/restart/src/Restart.cpp:155-164,190-194,99-120,
// codes/database/src/DataBook.cpp:301-316): int64 byte count, int32 outer
// step, f64 time, then q1, q2, res1, res2 as [n][nT] f64.
// ---------------------------------------------------------------------------
static int64_t restart_bytes(const ofg_ctx *c, int n) {
    return int64_t(sizeof(int32_t) + sizeof(double)) + 4 * int64_t(n) * c->nT * int64_t(sizeof(double));
}

int ofg_write_restart(ofg_ctx *c, int tid, const char *path, double curr_time) {
    int rc = check_tid(c, tid);
    if (rc) return rc;
    if (!path) return c->fail(OFG_E_ARG, "null path");
    if (!c->haveState) return c->fail(OFG_E_STATE, "no state to write");
    if (c->pendingNext || c->pendingTurb) return c->fail(OFG_E_STATE, "UPDATE_FLOWFIELD without CALC_BOUNDARY");
    if (c->outerSteps > INT32_MAX) return c->fail(OFG_E_ARG, "outer step does not fit the file's int32");
    const int n = tid == OFG_TURB_SOLVER ? 1 : NEQ;
    const size_t block = size_t(n) * c->nT;
    std::vector<double> rec(4 * block, 0.0);   // q1, q2, res1 = res2 = 0
    if ((rc = ofg_download_state(c, tid, rec.data()))) return rc;
    // the other NS state buffer holds the state one outer iteration earlier
    // once an iteration has completed from it
    if (tid == OFG_NS_SOLVER && c->lastResBuf == (c->cur ^ 1) && !(multi_stage(c) && c->p.rk_stage > 1)) {
        c->cur ^= 1;
        rc = ofg_download_state(c, tid, rec.data() + block);
        c->cur ^= 1;
        if (rc) return rc;
    } else {
        std::copy(rec.begin(), rec.begin() + block, rec.begin() + block);
    }
    int64_t bytes = restart_bytes(c, n);
    int32_t step = int32_t(c->outerSteps);
    std::FILE *f = std::fopen(path, "wb");
    if (!f) return c->fail(OFG_E_IO, std::string("cannot create ") + path);
    bool ok = std::fwrite(&bytes, sizeof bytes, 1, f) == 1 && std::fwrite(&step, sizeof step, 1, f) == 1 &&
              std::fwrite(&curr_time, sizeof curr_time, 1, f) == 1 &&
              std::fwrite(rec.data(), sizeof(double), rec.size(), f) == rec.size();
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) return c->fail(OFG_E_IO, std::string("write failed: ") + path);
    return OFG_OK;
}

int ofg_read_restart(ofg_ctx *c, int tid, const char *path, int64_t *outer_step, double *curr_time) {
    if (!c) return OFG_E_ARG;
    if (tid != OFG_NS_SOLVER && !(tid == OFG_TURB_SOLVER && has_turb(c)))
        return c->fail(OFG_E_ARG, "no such solver in this context (tid 1 needs vismodel 3)");
    if (!path) return c->fail(OFG_E_ARG, "null path");
    if (!c->haveMesh) return c->fail(OFG_E_STATE, "no mesh uploaded");
    if (tid == OFG_TURB_SOLVER && !c->haveState) return c->fail(OFG_E_STATE, "read the NS restart first");
    int rc;
    const int n = tid == OFG_TURB_SOLVER ? 1 : NEQ;
    const size_t block = size_t(n) * c->nT;
    std::FILE *f = std::fopen(path, "rb");
    if (!f) return c->fail(OFG_E_IO, std::string("cannot open ") + path);
    int64_t bytes = 0;
    int32_t step = 0;
    double t = 0.0;
    std::vector<double> q1(block);
    bool ok = std::fread(&bytes, sizeof bytes, 1, f) == 1;
    if (ok && bytes != restart_bytes(c, n)) {
        std::fclose(f);
        return c->fail(OFG_E_ARG, "restart record of " + std::to_string(bytes) + " bytes; this mesh and solver need " +
                                      std::to_string(restart_bytes(c, n)) + " (one zone, " + std::to_string(n) +
                                      " equations, " + std::to_string(c->nT) + " cells with ghosts)");
    }
    ok = ok && std::fread(&step, sizeof step, 1, f) == 1 && std::fread(&t, sizeof t, 1, f) == 1 &&
         std::fread(q1.data(), sizeof(double), block, f) == block;
    // q2, res1, res2 follow; anything after them is another zone's record
    long size = -1;
    if (ok && std::fseek(f, 0, SEEK_END) == 0) size = std::ftell(f);
    std::fclose(f);
    if (!ok || size < long(sizeof bytes) + long(bytes))
        return c->fail(OFG_E_IO, std::string("short or unreadable restart file: ") + path);
    if (size > long(sizeof bytes) + long(bytes)) return c->fail(OFG_E_ARG, std::string("more than one zone in ") + path);
    if ((rc = ofg_upload_state(c, tid, q1.data()))) return rc;
    if (tid == OFG_NS_SOLVER) c->outerSteps = step;
    if (outer_step) *outer_step = step;
    if (curr_time) *curr_time = t;
    return OFG_OK;
}

int ofg_calc_lhs(ofg_ctx *c, int tid, double lhscoef) {
    int rc = check_tid(c, tid);
    if (rc) return rc;
    if (tid != OFG_NS_SOLVER) return c->fail(OFG_E_ARG, "CALC_LHS is built for the NS solver");
    if (c->lastResBuf != c->cur) return c->fail(OFG_E_STATE, "CALC_LHS needs UPDATE_RESIDUALS of the current state");
    c->lhsCoef = lhscoef;
    return launch(c, T_CALC_LHS);
}

int ofg_zero_dq(ofg_ctx *c, int tid) {
    int rc = check_tid(c, tid);
    if (rc) return rc;
    if (tid == OFG_TURB_SOLVER)
        CK(cudaMemsetAsync(c->d_dnut, 0, (size_t)c->nT * sizeof(double), c->stream));
    else
        CK(cudaMemsetAsync(c->d_dq, 0,
                           (size_t)c->nCells * DQR * (c->p.precision == OFG_PREC_MIXED ? sizeof(float) : sizeof(double)),
                           c->stream));
    return OFG_OK;
}

int ofg_calc_time_step(ofg_ctx *c, int tid) {
    int rc = check_tid(c, tid);
    if (rc) return rc;
    if (tid == OFG_TURB_SOLVER) return OFG_OK;   // no CALC_TIME_STEP in system/turb/function/funcMap.txt
    if ((rc = launch(c, T_CFL))) return rc;
    return launch(c, T_TIMESTEP);
}

int ofg_load_residuals(ofg_ctx *c, int tid) {
    // res = -rhs with rhs = 0 on a single grid: folded into UPDATE_RESIDUALS,
    // which starts every cell's accumulation from -0.0
    return check_tid(c, tid);
}

int ofg_update_residuals(ofg_ctx *c, int tid) {
    int rc = check_tid(c, tid);
    if (rc) return rc;
    if (tid == OFG_TURB_SOLVER && c->pendingNext) return c->fail(OFG_E_STATE, "NS update without CALC_BOUNDARY");
    if (tid == OFG_NS_SOLVER) c->lastResBuf = c->cur;
    return launch(c, tid == OFG_TURB_SOLVER ? T_TURB_RHS : T_RESIDUAL);
}

int ofg_init_lusgs(ofg_ctx *c, int tid) { return check_tid(c, tid); }

int ofg_lusgs_lower(ofg_ctx *c, int tid) {
    int rc = check_tid(c, tid);
    if (rc) return rc;
    return launch(c, tid == OFG_TURB_SOLVER ? T_TURB_LOWER : T_LOWER);
}

int ofg_lusgs_upper(ofg_ctx *c, int tid) {
    int rc = check_tid(c, tid);
    if (rc) return rc;
    return launch(c, tid == OFG_TURB_SOLVER ? T_TURB_UPPER : T_UPPER);
}

int ofg_update_flowfield(ofg_ctx *c, int tid) {
    int rc = check_tid(c, tid);
    if (rc) return rc;
    if (tid == OFG_TURB_SOLVER) {
        if ((rc = launch(c, T_TURB_UPDATE))) return rc;   // nu~ update + interior eddy viscosity
        c->pendingTurb = true;
        return OFG_OK;
    }
    if ((rc = launch(c, T_UPDATE))) return rc;
    c->pendingNext = true;
    return OFG_OK;
}

int ofg_calc_boundary(ofg_ctx *c, int tid) {
    int rc = check_tid(c, tid);
    if (rc) return rc;
    if (tid == OFG_TURB_SOLVER) {
        // TurbCalcBoundary: CalcTurbulentViscosity + TurbCalcBc
        rc = launch(c, c->pendingTurb ? T_TURB_BOUNDARY : T_TURB_BOUNDARY_CUR);
        c->pendingTurb = false;
        return rc;
    }
    if (c->pendingNext) {
        if ((rc = launch(c, T_BOUNDARY_NEXT))) return rc;
        c->cur ^= 1;
        c->pendingNext = false;
        return OFG_OK;
    }
    return launch(c, T_BOUNDARY_CUR);
}

// tasks of one outer iteration (MG::StrongIter: NS relaxation, then SA), with
// the state-buffer flip between the two solvers.  CALC_TIME_STEP,
// LOAD_RESIDUALS and UPDATE_RESIDUALS share one gather (T_TS_RES).
// (Measured on the 6M-cell plate: fusing UPDATE_FLOWFIELD into the upper
// sweep's level launches was slower than the separate streaming pass.)
static const int kNsTasks[] = {T_ADVANCE, T_TS_RES, T_LOWER, T_UPPER, T_UPDATE, T_BOUNDARY_NEXT, T_NORM};
static const int kTurbTasks[] = {T_TURB_RHS, T_TURB_LOWER, T_TURB_UPPER, T_TURB_UPDATE, T_TURB_BOUNDARY, T_TURB_NORM};

static int sync_history(ofg_ctx *c) {
    size_t have = c->hist.size() / NEQ;
    size_t want = (size_t)c->outerSteps;
    if (want > have) {
        std::vector<double> tmp((want - have) * NEQ);
        CK(cudaMemcpy(tmp.data(), c->d_hist + have * NEQ, tmp.size() * sizeof(double), cudaMemcpyDeviceToHost));
        c->hist.insert(c->hist.end(), tmp.begin(), tmp.end());
        for (double v : tmp)
            if (std::isnan(v)) return c->fail(OFG_E_NAN, "NotANumber in the NS residual");
        if (has_turb(c)) {
            std::vector<double> tt(want - have);
            CK(cudaMemcpy(tt.data(), c->d_thist + have, tt.size() * sizeof(double), cudaMemcpyDeviceToHost));
            c->thist.insert(c->thist.end(), tt.begin(), tt.end());
            for (double v : tt)
                if (std::isnan(v)) return c->fail(OFG_E_NAN, "NotANumber in the SA residual");
        }
    }
    return OFG_OK;
}

// checks before n fused outer iterations; the device step counter and history
// indices follow the host counters (queued on the context's stream)
static int prepare_steps(ofg_ctx *c, int nsteps) {
    int rc = check_tid(c, OFG_NS_SOLVER);
    if (rc) return rc;
    if (nsteps < 0) return c->fail(OFG_E_ARG, "negative step count");
    if (c->pendingNext || c->pendingTurb) return c->fail(OFG_E_STATE, "UPDATE_FLOWFIELD without CALC_BOUNDARY");
    if (c->outerSteps + nsteps > c->histCap) return c->fail(OFG_E_ARG, "residual history capacity exceeded");
    double sc[4] = {double(c->outerSteps), double(c->outerSteps), 0.0, double(c->outerSteps)};
    CK(cudaMemcpyAsync(c->d_scal + S_STEP, sc, 2 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->d_scal + S_THISTN, sc + 3, sizeof(double), cudaMemcpyHostToDevice, c->stream));
    return sync(c);
}

// one outer iteration per state-buffer parity, captured once (ZERO_DQ_FIELD
// is not needed: no kernel reads an increment it did not write this iteration)
static int ensure_graphs(ofg_ctx *c) {
    if (c->graph[0]) return OFG_OK;
    int rc, saveCur = c->cur;
    for (int g = 0; g < 2; ++g) {
        long long before = c->launches;
        cudaGraph_t graph;
        CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        c->cur = g;
        auto run = [&](int t) {
            return c->p.precision == OFG_PREC_MIXED ? launch_task_f32(c, t, c->stream) : launch_task_f64(c, t, c->stream);
        };
        if (multi_stage(c)) {
            // TimeIntegral::RungeKutta (codes/solver/src/TimeIntegral.cpp:81-111): the
            // time step once, then per stage the residual, CALC_LHS with
            // lhscoef = 1/(stage+1), UPDATE_FLOWFIELD and CALC_BOUNDARY, each
            // stage reading the buffer the previous one wrote.  (LOAD_Q copies q
            // to a field UPDATE_FLOWFIELD never reads -- GetUpdateField,
            // codes/update/src/Update.cpp:64-86, sets its pointer arguments by
            // value -- so it has no effect on the iterates and is not run.)
            const int st[] = {T_ADVANCE, T_TIMESTEP};
            for (int t : st)
                if ((rc = run(t))) { cudaStreamEndCapture(c->stream, &graph); c->cur = saveCur; return rc; }
            for (int k = 0; k < c->p.rk_stage; ++k) {
                c->cur = g ^ (k & 1);
                c->lhsCoef = 1.0 / (k + 1);
                const int stage[] = {T_RESIDUAL, T_CALC_LHS, T_UPDATE, T_BOUNDARY_NEXT};
                for (int t : stage)
                    if ((rc = run(t))) { cudaStreamEndCapture(c->stream, &graph); c->cur = saveCur; return rc; }
            }
            if ((rc = run(T_NORM))) { cudaStreamEndCapture(c->stream, &graph); c->cur = saveCur; return rc; }
        } else {
            for (int t : kNsTasks) {
                if ((rc = run(t))) { cudaStreamEndCapture(c->stream, &graph); c->cur = saveCur; return rc; }
            }
        }
        c->cur = g ^ 1;
        if (has_turb(c))
            for (int t : kTurbTasks) {
                rc = c->p.precision == OFG_PREC_MIXED ? launch_task_f32(c, t, c->stream) : launch_task_f64(c, t, c->stream);
                if (rc) { cudaStreamEndCapture(c->stream, &graph); c->cur = saveCur; return rc; }
            }
        CK(cudaStreamEndCapture(c->stream, &graph));
        CK(cudaGraphInstantiate(&c->graph[g], graph, 0));
        c->graphT[g] = graph;   // kept: a batch embeds it as a child graph
        c->graphKernels[g] = c->launches - before;
        c->launches = before;
    }
    c->cur = saveCur;
    return OFG_OK;
}

// host bookkeeping of one outer iteration launched from parity c->cur (the
// multi-stage scheme moves between the two state buffers once per stage)
static void account_step(ofg_ctx *c) {
    c->launches += c->graphKernels[c->cur];
    int flips = multi_stage(c) ? c->p.rk_stage : 1;
    c->lastResBuf = c->cur ^ ((flips - 1) & 1);   // the buffer the last residual pass read
    c->cur ^= flips & 1;
    c->outerSteps++;
}

int ofg_step(ofg_ctx *c, int nsteps) {
    int rc = prepare_steps(c, nsteps);
    if (rc) return rc;
    if ((rc = ensure_graphs(c))) return rc;
    for (int it = 0; it < nsteps; ++it) {
        CK(cudaGraphLaunch(c->graph[c->cur], c->stream));
        account_step(c);
    }
    if ((rc = sync(c))) return rc;
    return sync_history(c);
}

// ---------------------------------------------------------------------------
// Batched solves: independent contexts advanced by one graph launch per outer
// iteration, whose branches are the contexts' own iteration graphs.
// ---------------------------------------------------------------------------
struct ofg_batch {
    std::vector<ofg_ctx *> ctx;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};         // around the graph launches of one ofg_batch_step
    float lastMs = -1.f;                            // their device time, after a successful step
    cudaGraphExec_t exec[2] = {nullptr, nullptr};   // [k]: each context at parity built[i] ^ k
    std::vector<int> built;                          // the contexts' parities when the execs were built
    std::vector<unsigned> gen;                       // and their graph generations
    std::string err;
    int fail(int code, const std::string &m) { err = m; return code; }
};

static void batch_release(ofg_batch *b) {
    for (auto &e : b->exec)
        if (e) { cudaGraphExecDestroy(e); e = nullptr; }
}

int ofg_batch_create(ofg_ctx *const *ctxs, int n, ofg_batch **out) {
    if (!ctxs || n <= 0 || !out) return OFG_E_ARG;
    auto *b = new ofg_batch();
    for (int i = 0; i < n; ++i) {
        if (!ctxs[i]) { delete b; return OFG_E_ARG; }
        for (int j = 0; j < i; ++j)
            if (ctxs[j] == ctxs[i]) { delete b; return OFG_E_ARG; }   // each context once
        b->ctx.push_back(ctxs[i]);
    }
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) { delete b; return OFG_E_CUDA; }
    if (cudaEventCreate(&b->ev[0]) != cudaSuccess || cudaEventCreate(&b->ev[1]) != cudaSuccess) {
        for (auto &e : b->ev)
            if (e) cudaEventDestroy(e);
        cudaStreamDestroy(b->stream);
        delete b;
        return OFG_E_CUDA;
    }
    *out = b;
    return OFG_OK;
}

void ofg_batch_destroy(ofg_batch *b) {
    if (!b) return;
    cudaStreamSynchronize(b->stream);
    batch_release(b);
    for (auto &e : b->ev) cudaEventDestroy(e);
    cudaStreamDestroy(b->stream);
    delete b;
}

const char *ofg_batch_last_error(const ofg_batch *b) { return b ? b->err.c_str() : "null batch"; }

int ofg_batch_device_ms(const ofg_batch *b, float *ms) {
    if (!b || !ms || b->lastMs < 0.f) return OFG_E_ARG;
    *ms = b->lastMs;
    return OFG_OK;
}

int ofg_batch_step(ofg_batch *b, int nsteps) {
    if (!b) return OFG_E_ARG;
    const int n = int(b->ctx.size());
    for (int i = 0; i < n; ++i) {
        ofg_ctx *c = b->ctx[i];
        int rc = prepare_steps(c, nsteps);
        if (!rc) rc = ensure_graphs(c);
        if (rc) return b->fail(rc, "context " + std::to_string(i) + ": " + c->err);
    }
    // the two batch graphs stay valid while every context keeps the graphs
    // they were built from and all contexts have flipped parity together
    bool valid = b->exec[0] && int(b->built.size()) == n;
    int flip = valid ? (b->ctx[0]->cur ^ b->built[0]) : 0;
    for (int i = 0; valid && i < n; ++i)
        valid = b->gen[i] == b->ctx[i]->graphGen && (b->ctx[i]->cur ^ b->built[i]) == flip;
    if (!valid) {
        batch_release(b);
        b->built.assign(n, 0); b->gen.assign(n, 0);
        for (int i = 0; i < n; ++i) { b->built[i] = b->ctx[i]->cur; b->gen[i] = b->ctx[i]->graphGen; }
        for (int k = 0; k < 2; ++k) {
            cudaGraph_t g;
            if (cudaGraphCreate(&g, 0) != cudaSuccess) return b->fail(OFG_E_CUDA, "cudaGraphCreate");
            for (int i = 0; i < n; ++i) {
                cudaGraphNode_t node;
                if (cudaGraphAddChildGraphNode(&node, g, nullptr, 0, b->ctx[i]->graphT[b->built[i] ^ k]) != cudaSuccess) {
                    cudaGraphDestroy(g);
                    return b->fail(OFG_E_CUDA, "cudaGraphAddChildGraphNode");
                }
            }
            cudaError_t e = cudaGraphInstantiate(&b->exec[k], g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return b->fail(OFG_E_CUDA, std::string("batch graph: ") + cudaGetErrorString(e));
        }
        flip = 0;
    }
    b->lastMs = -1.f;
    if (cudaEventRecord(b->ev[0], b->stream) != cudaSuccess) return b->fail(OFG_E_CUDA, "cudaEventRecord");
    for (int it = 0; it < nsteps; ++it) {
        if (cudaGraphLaunch(b->exec[flip], b->stream) != cudaSuccess) return b->fail(OFG_E_CUDA, "cudaGraphLaunch");
        for (ofg_ctx *c : b->ctx) account_step(c);
        flip ^= 1;
    }
    if (cudaEventRecord(b->ev[1], b->stream) != cudaSuccess) return b->fail(OFG_E_CUDA, "cudaEventRecord");
    cudaError_t e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return b->fail(OFG_E_CUDA, cudaGetErrorString(e));
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, b->ev[0], b->ev[1]) != cudaSuccess) return b->fail(OFG_E_CUDA, "cudaEventElapsedTime");
    for (int i = 0; i < n; ++i) {
        int rc = sync_history(b->ctx[i]);
        if (rc) return b->fail(rc, "context " + std::to_string(i) + ": " + b->ctx[i]->err);
    }
    b->lastMs = ms;
    return OFG_OK;
}

// ---------------------------------------------------------------------------
// Largest |residual| per equation and the first cell holding it
// (ResidualTask::CalcRes, codes/residual/src/ResidualTask.cpp:91-107: a strict
// comparison in ascending cell order keeps the first).  Per 128-cell block:
// out[block][e] = the block's maximum, out[block][neq + e] = its lowest cell
// index (as a double, exact), combined on the host in block order.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_res_max(const double *res, int n, int neq, double *out) {
    __shared__ double sv[128];
    __shared__ int si[128];
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    for (int e = 0; e < neq; ++e) {
        sv[threadIdx.x] = c < n ? fabs(res[(size_t)c * neq + e]) : -1.0;
        si[threadIdx.x] = c;
        __syncthreads();
        for (int w = 64; w > 0; w >>= 1) {
            if (threadIdx.x < w) {
                double a = sv[threadIdx.x], b = sv[threadIdx.x + w];
                if (b > a || (b == a && si[threadIdx.x + w] < si[threadIdx.x])) {
                    sv[threadIdx.x] = b;
                    si[threadIdx.x] = si[threadIdx.x + w];
                }
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            out[(size_t)blockIdx.x * 2 * neq + e] = sv[0];
            out[(size_t)blockIdx.x * 2 * neq + neq + e] = double(si[0]);
        }
        __syncthreads();
    }
}

int ofg_residual_max(ofg_ctx *c, int tid, double *resmax, int64_t *cell) {
    int rc = check_tid(c, tid);
    if (rc) return rc;
    if (!resmax || !cell) return c->fail(OFG_E_ARG, "null output");
    bool turb = tid == OFG_TURB_SOLVER;
    const int neq = turb ? 1 : NEQ, n = c->nCells, nb = (n + 127) / 128;
    if ((size_t)nb * 2 * neq > c->nPartialMax) return c->fail(OFG_E_ARG, "partials buffer too small");
    k_res_max<<<nb, 128, 0, c->stream>>>(turb ? c->d_resT : c->d_res, n, neq, c->d_partial);
    CK(cudaGetLastError());
    c->launches++;
    std::vector<double> part((size_t)nb * 2 * neq);
    CK(cudaMemcpyAsync(part.data(), c->d_partial, part.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if ((rc = sync(c))) return rc;
    for (int e = 0; e < neq; ++e) {
        double m = -1.0;
        int64_t at = 0;
        for (int b = 0; b < nb; ++b) {   // ascending blocks: the first cell wins ties
            double v = part[(size_t)b * 2 * neq + e];
            if (v > m) { m = v; at = int64_t(part[(size_t)b * 2 * neq + neq + e]); }
        }
        resmax[e] = m;
        cell[e] = at;
    }
    return OFG_OK;
}

int ofg_residual_norms(ofg_ctx *c, int tid, double *rms) {
    int rc = check_tid(c, tid);
    if (rc) return rc;
    if (!rms) return c->fail(OFG_E_ARG, "null output");
    // from the per-block sums the residual kernels leave (per-task callers get them too)
    bool turb = tid == OFG_TURB_SOLVER;
    if ((rc = launch(c, turb ? T_TURB_NORM_ONLY : T_NORM_ONLY))) return rc;
    if ((rc = sync(c))) return rc;
    CK(cudaMemcpy(rms, c->d_scal + (turb ? S_TNORM : S_NORM), (turb ? 1 : NEQ) * sizeof(double),
                  cudaMemcpyDeviceToHost));
    return OFG_OK;
}

int ofg_forces(ofg_ctx *c, double aref, double *out) {
    int rc = check_tid(c, OFG_NS_SOLVER);
    if (rc) return rc;
    if (!out || !(aref > 0.0)) return c->fail(OFG_E_ARG, "null output or non-positive reference area");
    double f[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (c->nWall > 0) {
        if (c->p.ilim == -1 && c->p.vismodel == 0) {
            // first-order inviscid runs keep no gradients, but the reference
            // computes them in every residual pass and extrapolates the wall
            // pressure with them: the gradients of the state that pass read
            // (still in the other buffer), or none before any pass
            if (c->lastResBuf < 0) {
                size_t rs = c->p.precision == OFG_PREC_MIXED ? sizeof(float) : sizeof(double);
                CK(cudaMemsetAsync(c->d_gl, 0, (size_t)c->nCells * GLR * rs, c->stream));
            } else {
                int save = c->cur;
                c->cur = c->lastResBuf;
                rc = launch(c, T_GRAD_ONLY);
                c->cur = save;
                if (rc) return rc;
            }
        }
        if ((rc = launch(c, T_FORCES))) return rc;
        if ((rc = sync(c))) return rc;
        CK(cudaMemcpy(f, c->d_scal + S_FORCE, sizeof(f), cudaMemcpyDeviceToHost));
    }
    for (int k = 0; k < 9; ++k) out[k] = f[k];
    // AeroForceInfo::CalcCoef, codes/force/src/Force.cpp:254-269 (AeroCom::CalcCL/CalcCD :148-158)
    double aoa = c->p.aoa_degree * PI / 180.0, aos = c->p.sideslip_degree * PI / 180.0;
    double sina = std::sin(aoa), cosa = std::cos(aoa), sinb = std::sin(aos), cosb = std::cos(aos);
    double cf[3], cpres[3];
    for (int k = 0; k < 3; ++k) { cf[k] = f[k] / aref; cpres[k] = f[3 + k] / aref; }
    out[9] = -sina * cf[0] + cosa * cf[1];
    out[10] = cosa * cosb * cf[0] + sina * cosb * cf[1] + sinb * cf[2];
    out[11] = cosa * cosb * cpres[0] + sina * cosb * cpres[1] + sinb * cpres[2];
    out[12] = out[10] - out[11];
    return OFG_OK;
}

int ofg_download_field(ofg_ctx *c, int tid, const char *name, double *out, int64_t n_out, int64_t *n_needed) {
    int rc = check_tid(c, tid);
    if (rc) return rc;
    if (!name) return c->fail(OFG_E_ARG, "null name");
    if ((rc = sync(c))) return rc;
    std::string s(name);
    int64_t nT = c->nT, N = c->nCells;
    std::vector<double> buf;
    auto rec_field = [&](int comp) {
        std::vector<double> rec((size_t)nT * REC);
        cudaMemcpy(rec.data(), c->d_q[c->cur], rec.size() * sizeof(double), cudaMemcpyDeviceToHost);
        buf.resize(nT);
        for (int64_t i = 0; i < nT; ++i) buf[i] = rec[(size_t)i * REC + comp];
    };
    auto aos_field = [&](const double *d, int ne, int64_t nrow, int64_t ntot) {
        std::vector<double> tmp((size_t)nrow * ne);
        cudaMemcpy(tmp.data(), d, tmp.size() * sizeof(double), cudaMemcpyDeviceToHost);
        buf.assign((size_t)ne * ntot, 0.0);
        for (int e = 0; e < ne; ++e)
            for (int64_t i = 0; i < nrow; ++i) buf[(size_t)e * ntot + i] = tmp[(size_t)i * ne + e];
    };
    // gradient+limiter records (R-typed [N][GLR]): component e at off + e * step
    auto gl_field = [&](int off, int step) {
        buf.assign((size_t)NEQ * nT, 0.0);
        if (c->p.precision == OFG_PREC_MIXED) {
            std::vector<float> tmp((size_t)N * GLR);
            cudaMemcpy(tmp.data(), c->d_gl, tmp.size() * sizeof(float), cudaMemcpyDeviceToHost);
            for (int e = 0; e < NEQ; ++e) for (int64_t i = 0; i < N; ++i) buf[(size_t)e * nT + i] = tmp[(size_t)i * GLR + off + e * step];
        } else {
            std::vector<double> tmp((size_t)N * GLR);
            cudaMemcpy(tmp.data(), c->d_gl, tmp.size() * sizeof(double), cudaMemcpyDeviceToHost);
            for (int e = 0; e < NEQ; ++e) for (int64_t i = 0; i < N; ++i) buf[(size_t)e * nT + i] = tmp[(size_t)i * GLR + off + e * step];
        }
    };
    auto host_vec = [&](const std::vector<double> &v) { buf = v; };
    if (s == "res") aos_field(c->d_res, NEQ, N, nT);
    else if (s == "dq") {   // [nCells][DQR] records at the face precision; ghosts 0
        buf.assign((size_t)NEQ * nT, 0.0);
        if (c->p.precision == OFG_PREC_MIXED) {
            std::vector<float> tmp((size_t)N * DQR);
            cudaMemcpy(tmp.data(), c->d_dq, tmp.size() * sizeof(float), cudaMemcpyDeviceToHost);
            for (int e = 0; e < NEQ; ++e) for (int64_t i = 0; i < N; ++i) buf[(size_t)e * nT + i] = tmp[(size_t)i * DQR + e];
        } else {
            std::vector<double> tmp((size_t)N * DQR);
            cudaMemcpy(tmp.data(), c->d_dq, tmp.size() * sizeof(double), cudaMemcpyDeviceToHost);
            for (int e = 0; e < NEQ; ++e) for (int64_t i = 0; i < N; ++i) buf[(size_t)e * nT + i] = tmp[(size_t)i * DQR + e];
        }
    }
    else if (s == "timestep") aos_field(c->d_dt, 1, N, nT);
    else if (s == "invsr") aos_field(c->d_invsr, 1, N, nT);
    else if (s == "vissr") aos_field(c->d_vissr, 1, N, nT);
    else if (s == "impsr") {
        std::vector<double> dt(N), iv(N), vs(N);
        cudaMemcpy(dt.data(), c->d_dt, N * 8, cudaMemcpyDeviceToHost);
        cudaMemcpy(iv.data(), c->d_invsr, N * 8, cudaMemcpyDeviceToHost);
        cudaMemcpy(vs.data(), c->d_vissr, N * 8, cudaMemcpyDeviceToHost);
        buf.assign(nT, 0.0);
        for (int64_t i = 0; i < N; ++i) { double v = (1.0 / dt[i]) * c->vol[i]; v += iv[i]; v += vs[i]; buf[i] = v; }
    }
    else if (s == "tempr") rec_field(ITT);
    else if (s == "visl") rec_field(IML);
    else if (s == "vist") rec_field(IMT);
    else if (s == "limiter") gl_field(18, 1);
    else if (s == "dqdx") gl_field(0, 3);
    else if (s == "dqdy") gl_field(1, 3);
    else if (s == "dqdz") gl_field(2, 3);
    else if (s == "vol") host_vec(c->vol);
    else if (s == "xcc") host_vec(c->xcc);
    else if (s == "ycc") host_vec(c->ycc);
    else if (s == "zcc") host_vec(c->zcc);
    else if (s == "area") host_vec(c->area);
    else if (s == "xfn") host_vec(c->xfn);
    else if (s == "yfn") host_vec(c->yfn);
    else if (s == "zfn") host_vec(c->zfn);
    else if (s == "xfc") host_vec(c->xfc);
    else if (s == "yfc") host_vec(c->yfc);
    else if (s == "zfc") host_vec(c->zfc);
    else if (s == "reshist") host_vec(tid == OFG_TURB_SOLVER ? c->thist : c->hist);
    else if (s == "turbreshist") host_vec(c->thist);
    else if (has_turb(c) && (s == "turbq" || s == "turbdq")) aos_field(s == "turbq" ? c->d_nut : c->d_dnut, 1, nT, nT);
    else if (has_turb(c) && s == "turbres") aos_field(c->d_resT, 1, N, nT);
    else if (has_turb(c) && s == "turbimpsr") aos_field(c->d_impsrT, 1, N, nT);
    else if (s == "walldist") { buf.assign(nT, 0.0); std::copy(c->wdist.begin(), c->wdist.end(), buf.begin()); }
    else return c->fail(OFG_E_ARG, "unknown field " + s);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return c->fail(OFG_E_CUDA, cudaGetErrorString(e));
    if (n_needed) *n_needed = (int64_t)buf.size();
    if (out) {
        if (n_out < (int64_t)buf.size()) return c->fail(OFG_E_ARG, "output buffer too small");
        std::copy(buf.begin(), buf.end(), out);
    }
    return OFG_OK;
}

int ofg_set_stream(ofg_ctx *c, void *stream) {
    if (!c) return OFG_E_ARG;
    int rc = sync(c);
    if (rc) return rc;
    destroy_graphs(c);
    if (!c->ownStream) c->ownStream = c->stream;
    c->stream = stream ? (cudaStream_t)stream : c->ownStream;
    return OFG_OK;
}

int ofg_profile_step(ofg_ctx *c, double *ms, int *launches) {
    int rc = check_tid(c, OFG_NS_SOLVER);
    if (rc) return rc;
    if (!ms) return c->fail(OFG_E_ARG, "null output");
    if (c->pendingNext || c->pendingTurb) return c->fail(OFG_E_STATE, "UPDATE_FLOWFIELD without CALC_BOUNDARY");
    double sc[2] = {double(c->outerSteps), double(c->outerSteps)};
    CK(cudaMemcpyAsync(c->d_scal + S_STEP, sc, 2 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->d_scal + S_THISTN, sc, sizeof(double), cudaMemcpyHostToDevice, c->stream));
    // groups: the 10 NS groups (cfl; gradients+limiter, flux/time-step pass,
    // face-result sum, time-step clip; lower, upper, update, boundary, norm),
    // then the 7 SA groups (nu~ boundary+gradient, rhs gather, lower, upper,
    // update, boundary, norm): the kernels of one ofg_step in the same order
    static const int kNsProf[] = {T_ADVANCE, T_P_GRADLIM, T_P_FLUX, T_P_FSUM, T_P_CLIP, T_LOWER, T_UPPER, T_UPDATE,
                                  T_BOUNDARY_NEXT, T_NORM};
    static const int kTurbProf[] = {T_P_TURB_GRAD, T_P_TURB_FLUX, T_TURB_LOWER, T_TURB_UPPER, T_TURB_UPDATE,
                                    T_TURB_BOUNDARY, T_TURB_NORM};
    const int nns = 10, nt = has_turb(c) ? 7 : 0, n = nns + nt;
    cudaEvent_t ev[18];
    for (int i = 0; i <= n; ++i) CK(cudaEventCreate(&ev[i]));
    CK(cudaEventRecord(ev[0], c->stream));
    for (int i = 0; i < n; ++i) {
        long long before = c->launches;
        if (i == nns) c->cur ^= 1;   // the SA solver reads the relaxed NS state
        if ((rc = launch(c, i < nns ? kNsProf[i] : kTurbProf[i - nns]))) return rc;
        if (launches) launches[i] = int(c->launches - before);
        CK(cudaEventRecord(ev[i + 1], c->stream));
    }
    if (nt == 0) c->cur ^= 1;
    c->lastResBuf = c->cur ^ 1;
    CK(cudaEventSynchronize(ev[n]));
    for (int i = 0; i < n; ++i) {
        float t = 0.f;
        CK(cudaEventElapsedTime(&t, ev[i], ev[i + 1]));
        ms[i] = t;
    }
    for (int i = 0; i <= n; ++i) cudaEventDestroy(ev[i]);
    c->outerSteps++;
    return sync_history(c);
}

int ofg_sweep_levels(ofg_ctx *c, int *lower_levels, int *upper_levels) {
    if (!c) return OFG_E_ARG;
    if (!c->haveMesh) return c->fail(OFG_E_STATE, "no mesh uploaded");
    if (lower_levels) *lower_levels = int(c->lowOff.size()) - 1;
    if (upper_levels) *upper_levels = int(c->upOff.size()) - 1;
    return OFG_OK;
}

int ofg_set_outer_step(ofg_ctx *c, int64_t outer_steps) {
    if (!c || outer_steps < 0) return OFG_E_ARG;
    c->outerSteps = outer_steps;
    return OFG_OK;
}

int ofg_get_counters(ofg_ctx *c, int64_t *outer_steps, int64_t *kernel_launches) {
    if (!c) return OFG_E_ARG;
    if (outer_steps) *outer_steps = c->outerSteps;
    if (kernel_launches) *kernel_launches = c->launches;
    return OFG_OK;
}

int ofg_cell_centres(int dim, int nNodes, const double *xN, const double *yN, const double *zN, int nFaces,
                     const int *faceNodeCount, const int *faceNodes, const int *lCells, const int *rCells, int nCells,
                     int nBFaces, double *out) {
    if (nNodes <= 0 || nFaces <= 0 || nCells <= 0 || nBFaces < 0 || !out) return OFG_E_ARG;
    ofg_ctx tmp;
    tmp.nCells = nCells; tmp.nBFaces = nBFaces; tmp.nFaces = nFaces; tmp.nT = nCells + nBFaces;
    std::vector<int> fOff(nFaces + 1, 0);
    for (int f = 0; f < nFaces; ++f) fOff[f + 1] = fOff[f] + faceNodeCount[f];
    std::vector<int> fNod(faceNodes, faceNodes + fOff[nFaces]);
    tmp.lc.assign(lCells, lCells + nFaces);
    tmp.rc.assign(rCells, rCells + nFaces);
    for (int f = 0; f < nFaces; ++f)
        if (tmp.lc[f] < 0) {
            std::reverse(fNod.begin() + fOff[f], fNod.begin() + fOff[f + 1]);
            std::swap(tmp.lc[f], tmp.rc[f]);
        }
    for (int f = 0; f < nBFaces; ++f) tmp.rc[f] = f + nCells;
    for (int f = 0; f < nFaces; ++f)
        if (tmp.lc[f] < 0 || tmp.lc[f] >= nCells || tmp.rc[f] < 0 || tmp.rc[f] >= tmp.nT) return OFG_E_ARG;
    std::vector<double> X(xN, xN + nNodes), Y(yN, yN + nNodes), Z(zN, zN + nNodes);
    compute_metrics(&tmp, dim, X, Y, Z, fOff, fNod);
    for (int i = 0; i < nCells; ++i) {
        out[3 * (size_t)i] = tmp.xcc[i]; out[3 * (size_t)i + 1] = tmp.ycc[i]; out[3 * (size_t)i + 2] = tmp.zcc[i];
    }
    return OFG_OK;
}

// Reverse Cuthill-McKee order of the cell graph (cells joined by interior
// faces): per connected component, a breadth-first search from a
// pseudo-peripheral cell (the last cell reached by repeated searches from a
// cell of least degree, while the search depth grows), each cell's unvisited
// neighbours taken in ascending degree (ties: ascending id); the concatenated
// order is reversed.  Keeps every cell's neighbours close in the numbering, so
// the gathers of neighbour records touch few distinct cache lines.
int ofg_rcm_order(int nCells, int nFaces, int nBFaces, const int *lCells, const int *rCells, int *perm) {
    if (nCells <= 0 || nBFaces < 0 || nFaces < nBFaces || !lCells || !rCells || !perm) return OFG_E_ARG;
    std::vector<int> off(nCells + 1, 0);
    for (int f = nBFaces; f < nFaces; ++f) {
        int l = lCells[f], r = rCells[f];
        if (l < 0 || r < 0 || l >= nCells || r >= nCells) return OFG_E_ARG;
        off[l + 1]++; off[r + 1]++;
    }
    for (int i = 0; i < nCells; ++i) off[i + 1] += off[i];
    std::vector<int> adj(off[nCells]);
    {
        std::vector<int> pos(off.begin(), off.end() - 1);
        for (int f = nBFaces; f < nFaces; ++f) {
            int l = lCells[f], r = rCells[f];
            adj[pos[l]++] = r; adj[pos[r]++] = l;
        }
    }
    auto deg = [&](int i) { return off[i + 1] - off[i]; };
    for (int i = 0; i < nCells; ++i)   // neighbours by ascending degree, then id
        std::sort(adj.begin() + off[i], adj.begin() + off[i + 1], [&](int a, int b) {
            return deg(a) != deg(b) ? deg(a) < deg(b) : a < b;
        });
    std::vector<int> level(nCells, -1), order;
    order.reserve(nCells);
    std::vector<char> done(nCells, 0);
    // breadth-first levels from s over the unfinished cells; returns the depth
    // and the cell of least degree in the last level
    std::vector<int> q;
    auto bfs = [&](int s, int &far) {
        q.assign(1, s);
        level[s] = 0;
        int depth = 0;
        for (size_t h = 0; h < q.size(); ++h) {
            int c = q[h];
            for (int k = off[c]; k < off[c + 1]; ++k) {
                int n = adj[k];
                if (level[n] < 0 && !done[n]) { level[n] = level[c] + 1; q.push_back(n); }
            }
        }
        depth = level[q.back()];
        far = q.back();
        for (int c : q) if (level[c] == depth && deg(c) < deg(far)) far = c;
        for (int c : q) level[c] = -1;
        return depth;
    };
    for (int seed = 0; seed < nCells; ++seed) {
        if (done[seed]) continue;
        int s = seed, far = seed;
        // least-degree cell of this component as the first start
        {
            int dummy;
            bfs(s, dummy);
            for (int c : q) if (deg(c) < deg(s) || (deg(c) == deg(s) && c < s)) s = c;
        }
        int depth = bfs(s, far);
        for (int it = 0; it < 8; ++it) {   // pseudo-peripheral cell
            int far2, d2 = bfs(far, far2);
            if (d2 <= depth) break;
            s = far; depth = d2; far = far2;
        }
        // Cuthill-McKee from s
        size_t h0 = order.size();
        order.push_back(s);
        done[s] = 1;
        for (size_t h = h0; h < order.size(); ++h) {
            int c = order[h];
            for (int k = off[c]; k < off[c + 1]; ++k) {
                int n = adj[k];
                if (!done[n]) { done[n] = 1; order.push_back(n); }
            }
        }
    }
    for (int k = 0; k < nCells; ++k) perm[k] = order[nCells - 1 - k];
    return OFG_OK;
}

// ---------------------------------------------------------------------------
// Launch shapes and the autotuner
// ---------------------------------------------------------------------------
static bool valid_tuning(const ofg_tuning &t) {
    auto in = [](int v, std::initializer_list<int> l) { for (int x : l) if (x == v) return true; return false; };
    return in(t.face_min_blocks, {2, 3, 4, 5}) && in(t.face_block, {64, 128}) && in(t.grad_min_blocks, {4, 6, 8}) &&
           in(t.sweep_min_blocks, {6, 8, 10}) && in(t.sweep_block, {64, 128}) && in(t.sweep_persistent, {0, 1}) &&
           in(t.grad_block, {0, 64, 128});
}

int ofg_get_tuning(ofg_ctx *c, ofg_tuning *out) {
    if (!c || !out) return OFG_E_ARG;
    *out = c->tune;
    return OFG_OK;
}

int ofg_set_tuning(ofg_ctx *c, const ofg_tuning *t) {
    if (!c || !t) return OFG_E_ARG;
    if (!valid_tuning(*t)) return c->fail(OFG_E_ARG, "launch shape outside the compiled set");
    int rc = sync(c);
    if (rc) return rc;
    ofg_tuning n = *t;
    n.ms_default = c->tune.ms_default; n.ms_tuned = c->tune.ms_tuned;
    c->tune = n;
    destroy_graphs(c);   // recaptured with the new kernels at the next ofg_step
    return OFG_OK;
}

namespace {
std::mutex g_tuneMutex;
std::map<std::string, ofg_tuning> g_tuneCache;   // mesh + options -> chosen shapes

std::string tune_key(const ofg_ctx *c) {
    char k[256];
    std::snprintf(k, sizeof k, "%llx:%d:%d:%d:%d:%d:%d:%d:%d:%d", c->meshHash, c->nCells, c->nFaces, c->p.precision,
                  c->p.vismodel, c->p.ilim, c->p.igrad, c->p.ischeme, c->p.ivischeme, c->p.sweep_order);
    return k;
}
}  // namespace

int ofg_autotune(ofg_ctx *c, int reps, ofg_tuning *out) {
    int rc = check_tid(c, OFG_NS_SOLVER);
    if (rc) return rc;
    if (c->pendingNext || c->pendingTurb) return c->fail(OFG_E_STATE, "UPDATE_FLOWFIELD without CALC_BOUNDARY");
    if (multi_stage(c)) {   // no sweeps, fixed shapes
        c->tune.ms_default = c->tune.ms_tuned = 0.0;
        if (out) *out = c->tune;
        return OFG_OK;
    }
    const bool mixed = c->p.precision == OFG_PREC_MIXED;
    if (reps < 1) reps = 5;
    const std::string key = tune_key(c);
    {
        std::lock_guard<std::mutex> g(g_tuneMutex);
        auto it = g_tuneCache.find(key);
        if (it != g_tuneCache.end()) {
            if ((rc = ofg_set_tuning(c, &it->second))) return rc;
            c->tune.ms_default = it->second.ms_default; c->tune.ms_tuned = it->second.ms_tuned;
            if (out) *out = c->tune;
            return OFG_OK;
        }
    }
    if ((rc = sync(c))) return rc;
    destroy_graphs(c);
    // fill every input of the timed groups once: CFL, gradients, fluxes, residual, diagonal
    if ((rc = launch(c, T_CFL))) return rc;
    if ((rc = launch(c, T_TS_RES))) return rc;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    // median device time of one group (a list of tasks) over reps runs
    auto time_group = [&](std::initializer_list<int> tasks, double &ms) -> int {
        std::vector<float> t(reps);
        for (int r = 0; r < reps; ++r) {
            CK(cudaEventRecord(e0, c->stream));
            for (int task : tasks) { int q = launch(c, task); if (q) return q; }
            CK(cudaEventRecord(e1, c->stream));
            CK(cudaEventSynchronize(e1));
            CK(cudaEventElapsedTime(&t[r], e0, e1));
        }
        std::sort(t.begin(), t.end());
        ms = t[reps / 2];
        return OFG_OK;
    };
    const ofg_tuning start = c->tune;
    double msDefault = 0.0, msTuned = 0.0;
    // groups in turn, each over its own candidates, the others at their current choice
    struct Cand { int *a; int *b; std::vector<std::pair<int, int>> values; std::vector<int> tasks; };
    ofg_tuning &T = c->tune;
    std::vector<Cand> groups;
    if (mixed) {
        groups.push_back({&T.face_min_blocks, &T.face_block,
                          {{2, 128}, {3, 128}, {4, 128}, {5, 128}, {2, 64}, {3, 64}, {4, 64}, {5, 64}}, {T_P_FLUX}});
        groups.push_back({&T.grad_min_blocks, &T.grad_block,
                          {{4, 128}, {6, 128}, {8, 128}, {4, 64}, {6, 64}, {8, 64}}, {T_P_GRADLIM}});
        groups.push_back({&T.sweep_min_blocks, &T.sweep_block,
                          {{6, 128}, {8, 128}, {10, 128}, {6, 64}, {8, 64}, {10, 64}}, {T_LOWER, T_UPPER}});
    }
    // the sweep schedule: level launches or the persistent single-block form
    // (not tried when the levels average more than 16 passes of the block:
    // one block cannot keep up with a full-width level launch there)
    const int nlev = std::max<int>(1, int(c->lowOff.size()) - 1);
    if (c->nCells / nlev <= 16 * kSeqThreads)
        groups.push_back({&T.sweep_persistent, nullptr, {{0, 0}, {1, 0}}, {T_LOWER, T_UPPER}});
    for (Cand &g : groups) {
        const int a0 = *g.a, b0 = g.b ? *g.b : 0;
        double best = 1e30, first = 0.0;
        int ba = a0, bb = b0;
        for (size_t k = 0; k < g.values.size(); ++k) {
            *g.a = g.values[k].first;
            if (g.b) *g.b = g.values[k].second;
            double ms = 0.0;
            std::vector<int> tl(g.tasks);
            int q;
            if (tl.size() == 1) q = time_group({tl[0]}, ms);
            else q = time_group({tl[0], tl[1]}, ms);
            if (q) { cudaEventDestroy(e0); cudaEventDestroy(e1); c->tune = start; return q; }
            if (*g.a == a0 && (!g.b || *g.b == b0)) first = ms;   // the shape the context came with
            if (ms < best) { best = ms; ba = *g.a; bb = g.b ? *g.b : 0; }
        }
        *g.a = ba;
        if (g.b) *g.b = bb;
        msDefault += first;
        msTuned += best;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    T.ms_default = msDefault;
    T.ms_tuned = msTuned;
    destroy_graphs(c);
    {
        std::lock_guard<std::mutex> g(g_tuneMutex);
        g_tuneCache[key] = T;
    }
    if (out) *out = T;
    return sync(c);
}

int ofg_colour_order(int nCells, int nFaces, int nBFaces, const int *lCells, const int *rCells, int *perm) {
    if (nCells <= 0 || nBFaces < 0 || nFaces < nBFaces || !lCells || !rCells || !perm) return OFG_E_ARG;
    return colour_major_order(nCells, nFaces, nBFaces, lCells, rCells, perm);
}

}  // extern "C"

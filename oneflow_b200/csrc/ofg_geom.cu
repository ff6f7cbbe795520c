// Mesh metrics and wall distance on the GPU (compiled without FMA
// contraction, like the FP64 path, so the metrics round like the reference's
// serial code).
//
// Metrics: UnsGrid::CalcMetrics (codes/geometry/src/UnsGrid.cpp:469-900):
// face normals and areas (CalcFaceNormal2D/3D), face centres (CalcFaceCenter
// 2D/3D), cell centres and volumes (CalcCellCenterVol2D/3D), ghost cells
// mirrored across their boundary face.  One thread per face, then one thread
// per cell gathering its faces in ascending face id -- the order in which the
// reference's face loop adds them -- so the sums are bitwise the reference's.
//
// Wall distance: CalcWallDist / CalcPoint2FaceDist
// (codes/geometry/src/WallDist.cpp:136-330): for every cell centre the minimum
// squared distance to the SOLID_SURFACE faces (segments in 2-D; triangles in
// 3-D, faces of more than three nodes split about their node average), then
// the square root.  The reference evaluates every (cell, face) pair; here the
// wall primitives are grouped into spatially sorted tiles with bounding boxes,
// and a block of cells visits the tiles nearest to its own bounding box first,
// stopping when no remaining tile can hold a closer primitive: the minimum is
// the same (every skipped tile's lower bound is at least the current minimum).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <numeric>
#include <string>
#include <vector>

#include "ofg_ctx.h"

namespace ofg {

namespace {

constexpr double GSMALL = 1.0e-40;   // SMALL, codes/basic/include/HXTypeBasic.h
constexpr double GLARGE = 1.0e40;    // LARGE, the initial wall distance of CalcWallDist
constexpr int MT = 256;              // threads per block of the metric kernels
constexpr int WT = 128;              // cells per block of the wall-distance kernel
constexpr int TILE = 128;            // wall primitives per tile
constexpr int MAXTILES = 8192;       // tiles ordered per block (shared memory)

#define GCK(call)                                                                          \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) return c->fail(OFG_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

__global__ void __launch_bounds__(MT) k_face_metrics(int dim, int nF, const double *__restrict__ x,
                                                     const double *__restrict__ y, const double *__restrict__ z,
                                                     const int *__restrict__ fOff, const int *__restrict__ fNod,
                                                     double *xfn, double *yfn, double *zfn, double *area,
                                                     double *xfc, double *yfc, double *zfc) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nF) return;
    const int *fi = fNod + fOff[f];
    int n = fOff[f + 1] - fOff[f];
    double nx = 0.0, ny = 0.0, nz = 0.0, cx, cy, cz;
    if (dim == 2) {
        // UnsGrid::CalcFaceNormal2D / CalcFaceCenter2D
        int p1 = fi[0], p2 = fi[1];
        nx = y[p2] - y[p1];
        ny = x[p1] - x[p2];
        nz = 0.0;
        cx = 0.5 * (x[p1] + x[p2]);
        cy = 0.5 * (y[p1] + y[p2]);
        cz = 0.5 * (z[p1] + z[p2]);
    } else {
        // UnsGrid::CalcFaceNormal3D: half the sum of the edge cross products
        for (int i = 0; i < n; ++i) {
            int p1 = fi[i], p2 = fi[(i + 1) % n];
            double dx1 = x[p1], dy1 = y[p1], dz1 = z[p1], dx2 = x[p2], dy2 = y[p2], dz2 = z[p2];
            nx += 0.5 * (dy1 * dz2 - dy2 * dz1);
            ny += 0.5 * (dz1 * dx2 - dz2 * dx1);
            nz += 0.5 * (dx1 * dy2 - dx2 * dy1);
        }
    }
    double a = sqrt(nx * nx + ny * ny + nz * nz);
    double oa = 1.0 / (a + GSMALL);
    nx *= oa; ny *= oa; nz *= oa;
    if (dim != 2) {
        // UnsGrid::CalcFaceCenter3D: area-weighted centroids of the triangles
        // fanned from the node average (signed by the face normal)
        const double third = 1.0 / 3.0;
        double x0 = 0.0, y0 = 0.0, z0 = 0.0;
        for (int i = 0; i < n; ++i) { x0 += x[fi[i]]; y0 += y[fi[i]]; z0 += z[fi[i]]; }
        double factor = 1.0 / n;
        x0 *= factor; y0 *= factor; z0 *= factor;
        double sx = 0.0, sy = 0.0, sz = 0.0, sarea = 0.0;
        for (int i = 0; i < n; ++i) {
            int p1 = fi[i], p2 = fi[(i + 1) % n];
            double dx1 = x[p1] - x0, dy1 = y[p1] - y0, dz1 = z[p1] - z0;
            double dx2 = x[p2] - x0, dy2 = y[p2] - y0, dz2 = z[p2] - z0;
            double x00 = third * (x[p1] + x[p2] + x0);
            double y00 = third * (y[p1] + y[p2] + y0);
            double z00 = third * (z[p1] + z[p2] + z0);
            double anx = dy1 * dz2 - dy2 * dz1, any = dz1 * dx2 - dz2 * dx1, anz = dx1 * dy2 - dx2 * dy1;
            double fa = 0.5 * sqrt(anx * anx + any * any + anz * anz);
            if (anx * nx + any * ny + anz * nz < 0.0) fa = -fa;
            sarea += fa;
            sx += fa * x00; sy += fa * y00; sz += fa * z00;
        }
        double os = 1.0 / (sarea + GSMALL);
        cx = sx * os; cy = sy * os; cz = sz * os;
    }
    xfn[f] = nx; yfn[f] = ny; zfn[f] = nz; area[f] = a;
    xfc[f] = cx; yfc[f] = cy; zfc[f] = cz;
}

// UnsGrid::CalcCellCenterVol2D/3D as a gather: the cell's faces in ascending
// face id (the neighbour list), + where the cell is the face's left cell,
// - where it is the right cell.
__global__ void __launch_bounds__(MT) k_cell_metrics(int dim, int nC, const int *__restrict__ nbOff,
                                                     const int2 *__restrict__ nbl, const int *__restrict__ fOff,
                                                     const int *__restrict__ fNod, const double *__restrict__ x,
                                                     const double *__restrict__ y, const double *__restrict__ z,
                                                     const double *__restrict__ xfn, const double *__restrict__ yfn,
                                                     const double *__restrict__ zfn, const double *__restrict__ area,
                                                     const double *__restrict__ xfc, const double *__restrict__ yfc,
                                                     const double *__restrict__ zfc, double *xcc, double *ycc,
                                                     double *zcc, double *vol) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    double sx = 0.0, sy = 0.0, sz = 0.0, sv = 0.0;
    for (int k = nbOff[c]; k < nbOff[c + 1]; ++k) {
        int2 e = nbl[k];
        int f = e.x & 0x7fffffff;
        bool right = e.x < 0;
        if (dim == 2) {
            double dot = (xfc[f] * xfn[f] + yfc[f] * yfn[f] + zfc[f] * zfn[f]) * area[f];
            if (!right) { sx += xfc[f] * dot; sy += yfc[f] * dot; sz += zfc[f] * dot; sv += dot; }
            else        { sx -= xfc[f] * dot; sy -= yfc[f] * dot; sz -= zfc[f] * dot; sv -= dot; }
        } else {
            const int *fi = fNod + fOff[f];
            int n = fOff[f + 1] - fOff[f];
            double fx = xfc[f], fy = yfc[f], fz = zfc[f];
            for (int i = 0; i < n; ++i) {
                int p2 = fi[i], p3 = fi[(i + 1) % n];
                double x21 = x[p2] - fx, y21 = y[p2] - fy, z21 = z[p2] - fz;
                double x31 = x[p3] - fx, y31 = y[p3] - fy, z31 = z[p3] - fz;
                double nx = y21 * z31 - y31 * z21, ny = z21 * x31 - z31 * x21, nz = x21 * y31 - x31 * y21;
                double trix = fx + x[p2] + x[p3];
                double triy = fy + y[p2] + y[p3];
                double triz = fz + z[p2] + z[p3];
                double tmp = nx * trix + ny * triy + nz * triz;
                trix *= tmp; triy *= tmp; triz *= tmp;
                if (!right) { sx += trix; sy += triy; sz += triz; sv += tmp; }
                else        { sx -= trix; sy -= triy; sz -= triz; sv -= tmp; }
            }
        }
    }
    double v;
    if (dim == 2) {
        double tmp = 1.0 / (1.5 * sv + GSMALL);
        sx *= tmp; sy *= tmp; sz *= tmp;
        v = sv * 0.5;
    } else {
        double tmp = 1.0 / (4.0 * sv + GSMALL);
        sx *= tmp; sy *= tmp; sz *= tmp;
        v = sv / 18.0;
    }
    if (v <= 0.0) v = -v;
    xcc[c] = sx; ycc[c] = sy; zcc[c] = sz; vol[c] = v;
}

// ghost cell of boundary face f: the interior centre mirrored across the face
__global__ void __launch_bounds__(MT) k_ghost_metrics(int nC, int nB, const int *__restrict__ lcb,
                                                      const double *__restrict__ xfn, const double *__restrict__ yfn,
                                                      const double *__restrict__ zfn, const double *__restrict__ area,
                                                      const double *__restrict__ xfc, const double *__restrict__ yfc,
                                                      const double *__restrict__ zfc, double *xcc, double *ycc,
                                                      double *zcc, double *vol) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nB) return;
    int l = lcb[f], r = f + nC;
    if (area[f] > GSMALL) {
        double tmp = 2.0 * ((xcc[l] - xfc[f]) * xfn[f] + (ycc[l] - yfc[f]) * yfn[f] + (zcc[l] - zfc[f]) * zfn[f]);
        xcc[r] = xcc[l] - xfn[f] * tmp; ycc[r] = ycc[l] - yfn[f] * tmp; zcc[r] = zcc[l] - zfn[f] * tmp;
    } else {
        xcc[r] = -xcc[l] + 2.0 * xfc[f]; ycc[r] = -ycc[l] + 2.0 * yfc[f]; zcc[r] = -zcc[l] + 2.0 * zfc[f];
    }
    vol[r] = vol[l];
}

// ---- wall distance ----
// Squared distance from p to the segment ab: the projection parameter of p on
// the line, clamped to the segment.
__device__ __forceinline__ double seg_d2(double px, double py, double pz, const double *s) {
    double dx = s[3] - s[0], dy = s[4] - s[1], dz = s[5] - s[2];
    double ex = px - s[0], ey = py - s[1], ez = pz - s[2];
    double t = dx * ex + dy * ey + dz * ez;
    double qx = s[0], qy = s[1], qz = s[2];
    if (t > 0.0) {
        double L = dx * dx + dy * dy + dz * dz;
        if (t >= L) { qx = s[3]; qy = s[4]; qz = s[5]; }
        else { double u = t / L; qx += u * dx; qy += u * dy; qz += u * dz; }
    }
    double rx = px - qx, ry = py - qy, rz = pz - qz;
    return rx * rx + ry * ry + rz * rz;
}

// Squared distance from p to the triangle abc: the closest point found by the
// Voronoi-region tests of C. Ericson, "Real-Time Collision Detection" (2005),
// section 5.1.5 (vertex regions, edge regions, then the face interior).
__device__ __forceinline__ double tri_d2(double px, double py, double pz, const double *t) {
    double ax = t[0], ay = t[1], az = t[2];
    double abx = t[3] - ax, aby = t[4] - ay, abz = t[5] - az;
    double acx = t[6] - ax, acy = t[7] - ay, acz = t[8] - az;
    double apx = px - ax, apy = py - ay, apz = pz - az;
    double qx, qy, qz;
    double d1 = abx * apx + aby * apy + abz * apz, d2 = acx * apx + acy * apy + acz * apz;
    double bpx = px - t[3], bpy = py - t[4], bpz = pz - t[5];
    double d3 = abx * bpx + aby * bpy + abz * bpz, d4 = acx * bpx + acy * bpy + acz * bpz;
    double cpx = px - t[6], cpy = py - t[7], cpz = pz - t[8];
    double d5 = abx * cpx + aby * cpy + abz * cpz, d6 = acx * cpx + acy * cpy + acz * cpz;
    double vc = d1 * d4 - d3 * d2, vb = d5 * d2 - d1 * d6, va = d3 * d6 - d5 * d4;
    if (d1 <= 0.0 && d2 <= 0.0) {                                  // vertex a
        qx = ax; qy = ay; qz = az;
    } else if (d3 >= 0.0 && d4 <= d3) {                            // vertex b
        qx = t[3]; qy = t[4]; qz = t[5];
    } else if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {              // edge ab
        double v = d1 / (d1 - d3);
        qx = ax + v * abx; qy = ay + v * aby; qz = az + v * abz;
    } else if (d6 >= 0.0 && d5 <= d6) {                            // vertex c
        qx = t[6]; qy = t[7]; qz = t[8];
    } else if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {              // edge ac
        double w = d2 / (d2 - d6);
        qx = ax + w * acx; qy = ay + w * acy; qz = az + w * acz;
    } else if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0) {  // edge bc
        double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        qx = t[3] + w * (t[6] - t[3]); qy = t[4] + w * (t[7] - t[4]); qz = t[5] + w * (t[8] - t[5]);
    } else {
        double s = va + vb + vc;
        if (!(s > 0.0)) {   // degenerate triangle: the nearest of its edges
            double e0[6] = {t[0], t[1], t[2], t[3], t[4], t[5]}, e1[6] = {t[3], t[4], t[5], t[6], t[7], t[8]},
                   e2[6] = {t[6], t[7], t[8], t[0], t[1], t[2]};
            return fmin(seg_d2(px, py, pz, e0), fmin(seg_d2(px, py, pz, e1), seg_d2(px, py, pz, e2)));
        }
        double denom = 1.0 / s, v = vb * denom, w = vc * denom;
        qx = ax + abx * v + acx * w; qy = ay + aby * v + acy * w; qz = az + abz * v + acz * w;
    }
    double rx = px - qx, ry = py - qy, rz = pz - qz;
    return rx * rx + ry * ry + rz * rz;
}

__device__ __forceinline__ double box_gap2(const double *lo, const double *hi, const double *tb) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double g = fmax(0.0, fmax(tb[k] - hi[k], lo[k] - tb[3 + k]));
        s += g * g;
    }
    return s;
}

// block-wide (min value, its index) and max; every thread gets the results
__device__ __forceinline__ void block_argmin(double v, int i, double *sv, int *si, double &outv, int &outi) {
    for (int o = 16; o > 0; o >>= 1) {
        double v2 = __shfl_down_sync(0xffffffffu, v, o);
        int i2 = __shfl_down_sync(0xffffffffu, i, o);
        if (v2 < v || (v2 == v && i2 < i)) { v = v2; i = i2; }
    }
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { sv[w] = v; si[w] = i; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < int(blockDim.x >> 5); ++k)
            if (sv[k] < sv[0] || (sv[k] == sv[0] && si[k] < si[0])) { sv[0] = sv[k]; si[0] = si[k]; }
    }
    __syncthreads();
    outv = sv[0]; outi = si[0];
    __syncthreads();
}

__device__ __forceinline__ double block_max(double v, double *sv) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sv[w] = v;
    __syncthreads();
    if (threadIdx.x == 0)
        for (int k = 1; k < int(blockDim.x >> 5); ++k) sv[0] = fmax(sv[0], sv[k]);
    __syncthreads();
    double r = sv[0];
    __syncthreads();
    return r;
}

// prim: [nPrim][9] (segments use the first 6), tiles of TILE consecutive
// primitives with bounding boxes tbox[nTiles][6] (lo xyz, hi xyz)
__global__ void __launch_bounds__(WT) k_wall_dist(int nC, int kind, const double *__restrict__ xcc,
                                                  const double *__restrict__ ycc, const double *__restrict__ zcc,
                                                  int nPrim, const double *__restrict__ prim, int nTiles,
                                                  const double *__restrict__ tbox, double *dist) {
    extern __shared__ double smem[];
    double *sp = smem;                     // [TILE][9]
    double *lb = sp + TILE * 9;            // [nTiles] lower bounds of the block's distance to each tile
    __shared__ double red[WT / 32];
    __shared__ int redi[WT / 32];
    __shared__ double bbox[6];
    int c = blockIdx.x * WT + threadIdx.x;
    bool act = c < nC;
    double px = act ? xcc[c] : 0.0, py = act ? ycc[c] : 0.0, pz = act ? zcc[c] : 0.0;
    // the block's bounding box of cell centres
    {
        double lo[3] = {act ? px : GLARGE, act ? py : GLARGE, act ? pz : GLARGE};
        double hi[3] = {act ? px : -GLARGE, act ? py : -GLARGE, act ? pz : -GLARGE};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            double m = -block_max(-lo[k], red);
            double M = block_max(hi[k], red);
            if (threadIdx.x == 0) { bbox[k] = m; bbox[3 + k] = M; }
        }
        __syncthreads();
    }
    for (int t = threadIdx.x; t < nTiles; t += WT) lb[t] = box_gap2(bbox, bbox + 3, tbox + 6 * t);
    __syncthreads();
    double best = GLARGE;
    for (int it = 0; it < nTiles; ++it) {
        // the unvisited tile nearest to the block
        double v = GLARGE * 10.0;
        int vi = nTiles;
        for (int t = threadIdx.x; t < nTiles; t += WT)
            if (lb[t] < v) { v = lb[t]; vi = t; }
        double lbmin;
        int tmin;
        block_argmin(v, vi, red, redi, lbmin, tmin);
        double worst = block_max(act ? best : -1.0, red);
        // a tile whose lower bound reaches the block's largest current minimum
        // cannot lower any of them (the bound is shrunk by a relative 1e-12 so
        // that its rounding never skips a tile holding a minimum)
        if (tmin >= nTiles || lbmin * (1.0 - 1.0e-12) >= worst) break;
        if (threadIdx.x == 0) lb[tmin] = GLARGE * 10.0;
        int base = tmin * TILE, cnt = min(TILE, nPrim - base);
        for (int k = threadIdx.x; k < cnt * 9; k += WT) sp[k] = prim[(size_t)base * 9 + k];
        __syncthreads();
        if (act) {
            if (kind == 2)
                for (int j = 0; j < cnt; ++j) best = fmin(best, seg_d2(px, py, pz, sp + 9 * j));
            else
                for (int j = 0; j < cnt; ++j) best = fmin(best, tri_d2(px, py, pz, sp + 9 * j));
        }
        __syncthreads();
    }
    if (act) dist[c] = sqrt(best);
}

}  // namespace

// Metrics of the uploaded topology (c->lc/rc after the read-time swaps, the
// device neighbour lists and boundary left cells already uploaded) into the
// host vectors c->xfn ... c->vol; with wallDist, also the wall distance into
// c->wdist (from the metrics just computed, or from c->xcc.. when metrics is
// false).  The caller moves c->wdist to the device.
int gpu_geometry(ofg_ctx *c, const std::vector<double> &X, const std::vector<double> &Y,
                 const std::vector<double> &Z, const std::vector<int> &fOff, const std::vector<int> &fNod,
                 bool metrics, bool wallDist) {
    const int nF = c->nFaces, nC = c->nCells, nB = c->nBFaces, nT = c->nT, dim = c->p.dimension;
    const size_t nN = X.size();
    // temporaries, freed on every return
    struct Tmp {
        void *p[10] = {};
        ~Tmp() { for (void *q : p) cudaFree(q); }
    } tmp;
    double *&dX = reinterpret_cast<double *&>(tmp.p[0]), *&dY = reinterpret_cast<double *&>(tmp.p[1]),
           *&dZ = reinterpret_cast<double *&>(tmp.p[2]), *&dF = reinterpret_cast<double *&>(tmp.p[3]),
           *&dC = reinterpret_cast<double *&>(tmp.p[4]);
    int *&dOff = reinterpret_cast<int *&>(tmp.p[5]), *&dNod = reinterpret_cast<int *&>(tmp.p[6]);
    GCK(cudaMalloc(&dX, nN * 8)); GCK(cudaMalloc(&dY, nN * 8)); GCK(cudaMalloc(&dZ, nN * 8));
    GCK(cudaMalloc(&dOff, (nF + 1) * sizeof(int))); GCK(cudaMalloc(&dNod, fNod.size() * sizeof(int)));
    GCK(cudaMalloc(&dF, (size_t)7 * nF * 8)); GCK(cudaMalloc(&dC, (size_t)4 * nT * 8));
    cudaStream_t s = c->stream;
    GCK(cudaMemcpyAsync(dX, X.data(), nN * 8, cudaMemcpyHostToDevice, s));
    GCK(cudaMemcpyAsync(dY, Y.data(), nN * 8, cudaMemcpyHostToDevice, s));
    GCK(cudaMemcpyAsync(dZ, Z.data(), nN * 8, cudaMemcpyHostToDevice, s));
    GCK(cudaMemcpyAsync(dOff, fOff.data(), (nF + 1) * sizeof(int), cudaMemcpyHostToDevice, s));
    GCK(cudaMemcpyAsync(dNod, fNod.data(), fNod.size() * sizeof(int), cudaMemcpyHostToDevice, s));
    double *xfn = dF, *yfn = dF + nF, *zfn = dF + 2 * (size_t)nF, *area = dF + 3 * (size_t)nF,
           *xfc = dF + 4 * (size_t)nF, *yfc = dF + 5 * (size_t)nF, *zfc = dF + 6 * (size_t)nF;
    double *xcc = dC, *ycc = dC + nT, *zcc = dC + 2 * (size_t)nT, *vol = dC + 3 * (size_t)nT;
    if (metrics) {
        k_face_metrics<<<(nF + MT - 1) / MT, MT, 0, s>>>(dim, nF, dX, dY, dZ, dOff, dNod, xfn, yfn, zfn, area, xfc,
                                                         yfc, zfc);
        k_cell_metrics<<<(nC + MT - 1) / MT, MT, 0, s>>>(dim, nC, c->d_nb_off, reinterpret_cast<const int2 *>(c->d_nbl),
                                                         dOff, dNod, dX, dY, dZ, xfn, yfn, zfn, area, xfc, yfc, zfc,
                                                         xcc, ycc, zcc, vol);
        if (nB > 0)
            k_ghost_metrics<<<(nB + MT - 1) / MT, MT, 0, s>>>(nC, nB, c->d_lcb, xfn, yfn, zfn, area, xfc, yfc, zfc,
                                                              xcc, ycc, zcc, vol);
        GCK(cudaGetLastError());
        c->launches += 2 + (nB > 0);
        std::vector<double> *fv[7] = {&c->xfn, &c->yfn, &c->zfn, &c->area, &c->xfc, &c->yfc, &c->zfc};
        for (int k = 0; k < 7; ++k) {
            fv[k]->resize(nF);
            GCK(cudaMemcpyAsync(fv[k]->data(), dF + (size_t)k * nF, (size_t)nF * 8, cudaMemcpyDeviceToHost, s));
        }
        std::vector<double> *cv[4] = {&c->xcc, &c->ycc, &c->zcc, &c->vol};
        for (int k = 0; k < 4; ++k) {
            cv[k]->resize(nT);
            GCK(cudaMemcpyAsync(cv[k]->data(), dC + (size_t)k * nT, (size_t)nT * 8, cudaMemcpyDeviceToHost, s));
        }
        GCK(cudaStreamSynchronize(s));
    } else {
        std::vector<double> *cv[4] = {&c->xcc, &c->ycc, &c->zcc, &c->vol};
        for (int k = 0; k < 4; ++k)
            GCK(cudaMemcpyAsync(dC + (size_t)k * nT, cv[k]->data(), (size_t)nT * 8, cudaMemcpyHostToDevice, s));
    }
    if (!wallDist) return OFG_OK;

    // wall primitives (FillWallStruct order; faces of more than three nodes
    // fanned about their node average as in CalcPoint2FaceDist)
    std::vector<double> prim;
    int kind = dim == 2 ? 2 : 3;
    for (int f = 0; f < nB; ++f) {
        if (c->bct[f] != OFG_BC_SOLID_SURFACE) continue;
        const int *fi = &fNod[fOff[f]];
        int n = fOff[f + 1] - fOff[f];
        if (kind == 2) {
            double p[9] = {X[fi[0]], Y[fi[0]], Z[fi[0]], X[fi[1]], Y[fi[1]], Z[fi[1]], 0.0, 0.0, 0.0};
            prim.insert(prim.end(), p, p + 9);
        } else if (n == 3) {
            double p[9] = {X[fi[0]], Y[fi[0]], Z[fi[0]], X[fi[1]], Y[fi[1]], Z[fi[1]], X[fi[2]], Y[fi[2]], Z[fi[2]]};
            prim.insert(prim.end(), p, p + 9);
        } else {
            double xc = 0.0, yc = 0.0, zc = 0.0;
            for (int i = 0; i < n; ++i) { xc += X[fi[i]]; yc += Y[fi[i]]; zc += Z[fi[i]]; }
            double coef = 1.0 / n;
            xc *= coef; yc *= coef; zc *= coef;
            for (int i = 0; i < n; ++i) {
                int a = fi[i], b = fi[(i + 1) % n];
                double p[9] = {X[a], Y[a], Z[a], X[b], Y[b], Z[b], xc, yc, zc};
                prim.insert(prim.end(), p, p + 9);
            }
        }
    }
    int nPrim = int(prim.size() / 9);
    c->wdist.assign(nC, 0.0);
    if (nPrim == 0) {
        // no wall: the reference leaves sqrt(LARGE)
        std::fill(c->wdist.begin(), c->wdist.end(), std::sqrt(GLARGE));
    } else {
        // spatial order of the primitives (Morton code of the centroid in the
        // wall's bounding box), then tiles and their boxes
        double lo[3] = {GLARGE, GLARGE, GLARGE}, hi[3] = {-GLARGE, -GLARGE, -GLARGE};
        int nv = kind == 2 ? 2 : 3;
        std::vector<double> cen((size_t)nPrim * 3);
        for (int p = 0; p < nPrim; ++p)
            for (int k = 0; k < 3; ++k) {
                double m = 0.0;
                for (int v = 0; v < nv; ++v) m += prim[(size_t)p * 9 + 3 * v + k];
                cen[(size_t)p * 3 + k] = m / nv;
                lo[k] = std::min(lo[k], cen[(size_t)p * 3 + k]); hi[k] = std::max(hi[k], cen[(size_t)p * 3 + k]);
            }
        auto spread = [](uint64_t v) {
            v &= 0x1fffff;
            v = (v | v << 32) & 0x1f00000000ffffULL; v = (v | v << 16) & 0x1f0000ff0000ffULL;
            v = (v | v << 8) & 0x100f00f00f00f00fULL; v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
            v = (v | v << 2) & 0x1249249249249249ULL;
            return v;
        };
        std::vector<uint64_t> code(nPrim);
        for (int p = 0; p < nPrim; ++p) {
            uint64_t q[3];
            for (int k = 0; k < 3; ++k) {
                double ext = hi[k] - lo[k];
                double u = ext > 0.0 ? (cen[(size_t)p * 3 + k] - lo[k]) / ext : 0.0;
                q[k] = uint64_t(std::min(std::max(u, 0.0), 1.0) * 2097151.0);
            }
            code[p] = spread(q[0]) | spread(q[1]) << 1 | spread(q[2]) << 2;
        }
        std::vector<int> order(nPrim);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return code[a] < code[b]; });
        std::vector<double> sorted((size_t)nPrim * 9);
        for (int p = 0; p < nPrim; ++p)
            std::copy(&prim[(size_t)order[p] * 9], &prim[(size_t)order[p] * 9 + 9], &sorted[(size_t)p * 9]);
        int nTiles = (nPrim + TILE - 1) / TILE;
        if (nTiles > MAXTILES)
            return c->fail(OFG_E_SIZE, "wall distance: more than " + std::to_string(MAXTILES * TILE) +
                                           " wall primitives");
        std::vector<double> tbox((size_t)nTiles * 6);
        for (int t = 0; t < nTiles; ++t) {
            double b[6] = {GLARGE, GLARGE, GLARGE, -GLARGE, -GLARGE, -GLARGE};
            for (int p = t * TILE; p < std::min(nPrim, (t + 1) * TILE); ++p)
                for (int v = 0; v < nv; ++v)
                    for (int k = 0; k < 3; ++k) {
                        double x = sorted[(size_t)p * 9 + 3 * v + k];
                        b[k] = std::min(b[k], x); b[3 + k] = std::max(b[3 + k], x);
                    }
            std::copy(b, b + 6, &tbox[(size_t)t * 6]);
        }
        double *&dP = reinterpret_cast<double *&>(tmp.p[7]), *&dB = reinterpret_cast<double *&>(tmp.p[8]),
               *&dD = reinterpret_cast<double *&>(tmp.p[9]);
        GCK(cudaMalloc(&dP, sorted.size() * 8)); GCK(cudaMalloc(&dB, tbox.size() * 8)); GCK(cudaMalloc(&dD, (size_t)nC * 8));
        GCK(cudaMemcpyAsync(dP, sorted.data(), sorted.size() * 8, cudaMemcpyHostToDevice, s));
        GCK(cudaMemcpyAsync(dB, tbox.data(), tbox.size() * 8, cudaMemcpyHostToDevice, s));
        size_t shm = ((size_t)TILE * 9 + nTiles) * sizeof(double);
        if (shm > 48 * 1024) GCK(cudaFuncSetAttribute(k_wall_dist, cudaFuncAttributeMaxDynamicSharedMemorySize, int(shm)));
        k_wall_dist<<<(nC + WT - 1) / WT, WT, shm, s>>>(nC, kind, xcc, ycc, zcc, nPrim, dP, nTiles, dB, dD);
        GCK(cudaGetLastError());
        c->launches += 1;
        GCK(cudaMemcpyAsync(c->wdist.data(), dD, (size_t)nC * 8, cudaMemcpyDeviceToHost, s));
        GCK(cudaStreamSynchronize(s));
    }
    return OFG_OK;
}

}  // namespace ofg

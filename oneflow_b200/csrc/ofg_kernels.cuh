// Kernels of the NS residual + LU-SGS iteration, templated on the face
// arithmetic type R (double: the all-FP64 path; float: FP32 face terms with
// FP64 accumulation, update and norms).
//
// Every kernel is a cell-centred gather over a precomputed per-cell
// neighbour list in ascending face id -- the order in which the reference's
// serial face loops scatter into a cell -- so the FP64 accumulations round
// like the reference's and no atomics are used.  Data is packed for 128-bit
// loads: the state record (rho,u,v,w,p,T,mu_l,mu_t), the gradient+limiter
// record, the face record (normal, area, centre) and the cell record
// (centre, volume).
#pragma once
#include "ofg_device.cuh"

namespace ofg {

// Kernel arguments shared by all kernels of one context.
template <typename R>
struct KArgs {
    DevParams P;
    int nCells, nBFaces, nFaces, nT;
    const int *nb_off; const int2 *nbl;    // all faces of a cell {face | side<<31, neighbour}
    const int *lo_off; const int2 *lol;    // faces to earlier cells of the sweep order
    const int *up_off; const int2 *upl;    // faces to later cells of the sweep order (interior only)
    const int *bcType;                     // [nBFaces]
    const int *key;                        // [nT] sweep position
    const double *walldist;                // [nCells]
    const R *fgeo;                         // [nFaces][FGR]
    const R *cgeo;                         // [nT][CGR]
    const double *fgeoD;                   // [nFaces][FGR] the face records in FP64 (== fgeo on the FP64 path)
    // mixed path only: face-local geometry and the face pass of the residual
    const float *fofs;                     // [nFaces][8] x_f - x_L, x_f - x_R (formed in FP64), |x_f - x_L|, |x_f - x_R|
    const int2 *lr;                        // [nFaces] left cell, right cell (ghost nCells + f on boundary faces)
    double *fout;                          // [nFaces][FOR] face results of the face pass
    const double *q;  double *qn;          // master state records [nT][REC], current / next
    const R *qs;      R *qsn;              // state records read by face kernels (== master in FP64)
    double *res, *dt, *invsr, *vissr, *rad, *bcq;   // rad: LU-SGS diagonal
    R *dq;                                 // [nCells][DQR] LU-SGS increments (whole sectors per cell)
    R *gl;                                 // [nCells][GLR]
    R *mm;                                 // [nCells][MMR]
    double *partial, *scal;
    double *npart, *tpart;                 // per-block sums of squares of res / resT (128-cell blocks)
    double *red; unsigned int *redCount;   // block sums and ticket of the grid reductions
    int *fixlist; int fixcap;
    // Spalart-Allmaras
    double *nut, *dnut, *resT, *impsrT, *matL, *matR;
    R *gnut;                               // [nCells][4]
};

// ---------------------------------------------------------------------------
// vector loads
// ---------------------------------------------------------------------------
__device__ __forceinline__ void ld4(const float *p, float *o) {
    float4 a = __ldg(reinterpret_cast<const float4 *>(p));
    o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
}
__device__ __forceinline__ void ld4(const double *p, double *o) {
    double2 a = __ldg(reinterpret_cast<const double2 *>(p)), b = __ldg(reinterpret_cast<const double2 *>(p) + 1);
    o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
}
template <typename T> __device__ __forceinline__ void ld8(const T *p, T *o) { ld4(p, o); ld4(p + 4, o + 4); }
// plain (coherent) vector loads, for a record the same launch writes afterwards
__device__ __forceinline__ void ldp8(const float *p, float *o) {
    float4 a = reinterpret_cast<const float4 *>(p)[0], b = reinterpret_cast<const float4 *>(p)[1];
    o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w; o[4] = b.x; o[5] = b.y; o[6] = b.z; o[7] = b.w;
}
__device__ __forceinline__ void ldp8(const double *p, double *o) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        double2 a = reinterpret_cast<const double2 *>(p)[i];
        o[2 * i] = a.x; o[2 * i + 1] = a.y;
    }
}

__device__ __forceinline__ void st4(float *p, const float *v) {
    *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void st4(double *p, const double *v) {
    reinterpret_cast<double2 *>(p)[0] = make_double2(v[0], v[1]);
    reinterpret_cast<double2 *>(p)[1] = make_double2(v[2], v[3]);
}

// Block reductions for 1-D blocks of up to 1024 threads (a multiple of 32),
// in a fixed shuffle/tree order (run-to-run deterministic).  Every thread of
// the block must call them.
template <int N>
__device__ __forceinline__ void block_sum_to(const double *v, double *out) {
    __shared__ double s[32][N];
    int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
#pragma unroll
    for (int e = 0; e < N; ++e) {
        double x = v[e];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (l == 0) s[w][e] = x;
    }
    __syncthreads();
    if (w == 0) {
#pragma unroll
        for (int e = 0; e < N; ++e) {
            double y = l < nw ? s[l][e] : 0.0;
            for (int o = 16; o > 0; o >>= 1) y += __shfl_down_sync(0xffffffffu, y, o);
            if (l == 0) out[e] = y;
        }
    }
}

// Deterministic sum over the grid of n records of N doubles (in[i*N+e]):
// every block adds a contiguous chunk in a fixed order and leaves its sum in
// red[block]; the last block to finish (ticket on *counter) adds the block
// sums in block order into out[] (valid in that block's thread 0 only) and
// re-arms the counter.  Returns true in the block that produced out[].
template <int N>
__device__ __forceinline__ bool grid_sum_last(const double *in, int n, double *red, unsigned int *counter,
                                              double *out) {
    int G = gridDim.x;
    int per = (n + G - 1) / G;
    int b0 = blockIdx.x * per, b1 = min(n, b0 + per);
    double acc[N];
#pragma unroll
    for (int e = 0; e < N; ++e) acc[e] = 0.0;
    for (int i = b0 + threadIdx.x; i < b1; i += blockDim.x)
#pragma unroll
        for (int e = 0; e < N; ++e) acc[e] += in[(size_t)i * N + e];
    __shared__ double tot[N];
    __shared__ bool last;
    block_sum_to<N>(acc, tot);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int e = 0; e < N; ++e) red[(size_t)blockIdx.x * N + e] = tot[e];
        __threadfence();
        last = atomicAdd(counter, 1u) == unsigned(G - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
#pragma unroll
    for (int e = 0; e < N; ++e) acc[e] = 0.0;
    for (int i = threadIdx.x; i < G; i += blockDim.x)
#pragma unroll
        for (int e = 0; e < N; ++e) acc[e] += __ldcg(red + (size_t)i * N + e);
    block_sum_to<N>(acc, out);
    if (threadIdx.x == 0) *counter = 0u;
    return true;
}

__device__ __forceinline__ double block_min(double x) {
    __shared__ double s[32];
    __shared__ double r;
    int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int o = 16; o > 0; o >>= 1) x = fmin(x, __shfl_down_sync(0xffffffffu, x, o));
    if (l == 0) s[w] = x;
    __syncthreads();
    if (w == 0) {
        double y = l < nw ? s[l] : 1.0e300;
        for (int o = 16; o > 0; o >>= 1) y = fmin(y, __shfl_down_sync(0xffffffffu, y, o));
        if (l == 0) r = y;
    }
    __syncthreads();
    return r;
}

__device__ __forceinline__ int nb_face(int2 e) { return e.x & 0x7fffffff; }
__device__ __forceinline__ bool nb_right(int2 e) { return e.x < 0; }   // the cell is the face's right cell

// ---------------------------------------------------------------------------
// CALC_TIME_STEP face radii: TimeStep::CalcFaceInvSpec / CalcFaceVisSpec
// (codes/ns/src/TimeStep.cpp:61-122), as seen from the face's own left/right
// ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ double face_inv_spec(const DevParams &P, const R *ql, const R *qr, const R *fg) {
    R xn = fg[0], yn = fg[1], zn = fg[2], ar = fg[3];
    R gama = R(P.gama);
    R vnl = xn * ql[IU] + yn * ql[IV] + zn * ql[IW] - R(0);
    R vnr = xn * qr[IU] + yn * qr[IV] + zn * qr[IW] - R(0);
    R g = R(0.5) * (gama + gama);
    R pm = R(0.5) * (ql[IP] + qr[IP]), rm = R(0.5) * (ql[IR] + qr[IR]);
    R cm = Rsqrt(g * pm / rm);
    R vn = R(0.5) * (vnl + vnr);
    return double(R(0.5) * ar * (Rabs(vn) + cm));
}

template <typename R>
__device__ __forceinline__ double face_vis_spec(const DevParams &P, const R *ql, const R *qr, const R *fg,
                                                const R *cgl, const R *cgr) {
    R ar = fg[3];
    R vl = R(0.5) * (ql[IML] + qr[IML]);
    R vt = R(0.5) * (ql[IMT] + qr[IMT]);
    R density = R(0.5) * (ql[IR] + qr[IR]);
    if (P.visSRModel == 1) {
        R c1 = R(4.0) / R(3.0) * (vl + vt);
        R c2 = R(P.gama) * (vl * R(P.oprl) + vt * R(P.oprt));
        R c3 = R(2.0) * Rmax(c1, c2) / (R(P.reynolds) * density);
        return double(ar * ar * c3);
    } else if (P.visSRModel == 2) {
        R dist = Rabs(fg[0] * (cgr[0] - cgl[0]) + fg[1] * (cgr[1] - cgl[1]) + fg[2] * (cgr[2] - cgl[2]));
        R viscosity = vl + vt;
        R c1 = R(2.0) * viscosity / (density * dist * R(P.reynolds) + small_v<R>());
        return double(R(0.5) * c1 * ar);
    } else if (P.visSRModel == 3) {
        return double(ar * ar / (R(P.reynolds) * density + small_v<R>()));
    }
    return 0.0;
}

// UTimeStep::ModifyTimeStep / CalcLgTimeStep, then the diagonal of the
// LU-SGS system for the sweeps: UNsSpectrum::CalcImplicitSpectrum
// (sp2 = 1 for a steady solve), rad = (1/dt) vol + inviscid + viscous radius
template <typename R>
__global__ void __launch_bounds__(256) k_timestep_clip(KArgs<R> A) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= A.nCells) return;
    double ts = A.dt[c];
    if (A.P.timestepModel != 1) {
        double mn = A.scal[S_MINDT];
        if (A.P.timestepModel == 2) { ts = mn; A.dt[c] = ts; }
        else if (A.P.max_time_ratio > 0) { ts = fmin(ts, A.P.max_time_ratio * mn); A.dt[c] = ts; }
    }
    double s = (1.0 / ts) * double(A.cgeo[(size_t)c * CGR + 3]);
    s += A.invsr[c];
    s += A.vissr[c];
    A.rad[c] = s;
}

// x + (-y) / d without the division when it adds nothing: y = +0.0 and d > 0
// give -0.0, and v + (-0.0) == v bit for bit.  (Measured: without the test,
// the first upper-sweep level, whose cells have no later neighbours and so
// y = +0.0, executed three times the instructions of the first lower level.)
__device__ __forceinline__ double add_neg_quot(double x, double y, double d) {
    if (y == 0.0 && !signbit(y) && d > 0.0) return x;
    return x + (-y) / d;
}

// ---------------------------------------------------------------------------
// Gradients + limiter in one gather.  Gradients: CalcGradGGCellWeight
// (codes/usolver/src/UGrad.cpp:88-149), the face-average Green-Gauss
// (:40-86) or weighted least squares (new).  var 0-4: q, var 5: temperature
// (UTGrad, codes/uns/src/UNsGrad.cpp:81-101).  Limiter: Limiter::CalcMinMaxDiff
// + CalcBarthLimiter / CalcVencatLimiter (codes/usolver/src/ULimiter.cpp:377-644).
// limMode: 0 gradients only (limiter preset), 1 local limiter (Barth, or
// Venkatakrishnan with eps^2 = (K h)^3), 2 min/max and block extremes for the
// zone-wide Venkatakrishnan eps (limiter in k_limiter_global).
// ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ R barth_fn(R dqv, R minv, R maxv, R dot) {
    if (dot < R(0)) return R(0);
    else if (dqv > maxv) return maxv / dqv;
    else if (dqv < minv) return minv / dqv;
    return R(1);
}
template <typename R>
__device__ __forceinline__ R venkat(R x, R y, R eps) {
    R x2 = x * x, xy = x * y, y2 = y * y, cc = R(2);
    return ((x2 + eps + cc * xy) / (x2 + cc * y2 + xy + eps));
}
template <typename R>
__device__ __forceinline__ R venkat_fn(R dqv, R minv, R maxv, R eps) {
    if (dqv > small_v<R>()) return venkat(maxv, dqv, eps);
    else if (dqv < -small_v<R>()) return venkat(minv, dqv, eps);
    return R(1);
}

// limiter value of cell c over its faces (gradient g, neighbour min/max mn/mx)
template <typename R>
__device__ __forceinline__ void cell_limiter(const KArgs<R> &A, int c, const R *cgc, const R *g, const R *mn,
                                             const R *mx, const R *eps, R *lim) {
#pragma unroll
    for (int e = 0; e < NEQ; ++e) lim[e] = R(1);
    for (int k = A.nb_off[c]; k < A.nb_off[c + 1]; ++k) {
        int2 en = __ldg(&A.nbl[k]);
        int f = nb_face(en);
        R fg[FGR];
        R dx, dy, dz;
        if constexpr (sizeof(R) == 4) {
            // x_f - x_c from the face's offsets (formed in FP64); the normal
            // only for Barth
            float fo[FOFS];
            ld8(A.fofs + (size_t)f * FOFS, fo);
            const bool rt = nb_right(en);
            dx = rt ? fo[3] : fo[0]; dy = rt ? fo[4] : fo[1]; dz = rt ? fo[5] : fo[2];
            if (A.P.ilim == 1) ld4(A.fgeo + (size_t)f * FGR, fg);
        } else {
            ld8(A.fgeo + (size_t)f * FGR, fg);
            dx = fg[4] - cgc[0]; dy = fg[5] - cgc[1]; dz = fg[6] - cgc[2];
        }
        R dot = R(0);
        if (A.P.ilim == 1) {
            R ds = Rsqrt(SQR3(dx, dy, dz));
            R nd = fg[0] * dx + fg[1] * dy + fg[2] * dz;
            dot = nb_right(en) ? -nd / (ds + small_v<R>()) : nd / (ds + small_v<R>());
        }
#pragma unroll
        for (int e = 0; e < NEQ; ++e) {
            R dqf = g[e * 3 + 0] * dx + g[e * 3 + 1] * dy + g[e * 3 + 2] * dz;
            R v = (A.P.ilim == 1) ? barth_fn(dqf, mn[e], mx[e], dot) : venkat_fn(dqf, mn[e], mx[e], eps[e]);
            lim[e] = Rmin(lim[e], v);
        }
    }
}

// MINB: resident 128-thread blocks per SM asked of the compiler (its register
// cap is 65536 / (128 MINB)); the default is the measured choice for the 6M
// plate, other values are instantiated for the autotuner (ofg_autotune).
template <typename R, int MINB = MinBlocks<R>::gl>
__global__ void __launch_bounds__(128, MINB) k_gradlim(KArgs<R> A, int nvar, int limMode) {
    __shared__ double sred[2 * NEQ][128];
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    bool active = c < A.nCells;
    R mn[NEQ], mx[NEQ];
    // The FP32 path forms every neighbour difference in FP64 from the FP64
    // records (a difference of two FP32-rounded pressures would carry the
    // rounding of p itself) and sums differences, not values, over the faces;
    // its geometric differences come from the face offsets x_f - x_L,
    // x_f - x_R (formed in FP64, rounded once), never from FP32 coordinates.
    constexpr bool mixed = sizeof(R) == 4;
    if (active) {
        R qc[REC], cgc[CGR];
        if constexpr (!mixed) ld8(A.qs + (size_t)c * REC, qc);
        ld4(A.cgeo + (size_t)c * CGR, cgc);
        R gx[6], gy[6], gz[6];
#pragma unroll
        for (int v = 0; v < 6; ++v) gx[v] = gy[v] = gz[v] = R(0);
#pragma unroll
        for (int e = 0; e < NEQ; ++e) mn[e] = mx[e] = mixed ? R(0) : qc[e];
        int b = A.nb_off[c], en = A.nb_off[c + 1];
        if (A.P.igrad == 2) {
            // weighted least squares over face neighbours (ghosts included), w = 1/|d|^2
            R a11 = 0, a12 = 0, a13 = 0, a22 = 0, a23 = 0, a33 = 0, bb[6][3];
#pragma unroll
            for (int v = 0; v < 6; ++v) bb[v][0] = bb[v][1] = bb[v][2] = R(0);
            for (int k = b; k < en; ++k) {
                int2 e2 = __ldg(&A.nbl[k]);
                int nb = e2.y;
                R qn[REC], cgn[CGR], dn[6];
                R dx, dy, dz;
                if constexpr (mixed) {
                    double t[REC];
                    ld8(A.q + (size_t)nb * REC, t);
#pragma unroll
                    for (int v = 0; v < 6; ++v)   // the cell's own values re-read (L1 hits), not held
                        dn[v] = R(t[v < 5 ? v : ITT] - __ldg(A.q + (size_t)c * REC + (v < 5 ? v : ITT)));
                    // x_nb - x_c = (x_f - x_c) - (x_f - x_nb), from the face's offsets
                    float fo[FOFS];
                    ld8(A.fofs + (size_t)nb_face(e2) * FOFS, fo);
                    const float sg = nb_right(e2) ? -1.0f : 1.0f;
                    dx = sg * (fo[0] - fo[3]); dy = sg * (fo[1] - fo[4]); dz = sg * (fo[2] - fo[5]);
                } else {
                    ld8(A.qs + (size_t)nb * REC, qn);
#pragma unroll
                    for (int v = 0; v < 6; ++v) dn[v] = qn[v < 5 ? v : ITT] - qc[v < 5 ? v : ITT];
                    ld4(A.cgeo + (size_t)nb * CGR, cgn);
                    dx = cgn[0] - cgc[0]; dy = cgn[1] - cgc[1]; dz = cgn[2] - cgc[2];
                }
                R w = R(1) / (dx * dx + dy * dy + dz * dz);
                a11 += w * dx * dx; a12 += w * dx * dy; a13 += w * dx * dz;
                a22 += w * dy * dy; a23 += w * dy * dz; a33 += w * dz * dz;
#pragma unroll
                for (int v = 0; v < 6; ++v) {
                    if (v >= nvar) break;
                    R dv = dn[v];
                    bb[v][0] += w * dx * dv; bb[v][1] += w * dy * dv; bb[v][2] += w * dz * dv;
                }
                if (nb < A.nCells) {
#pragma unroll
                    for (int e = 0; e < NEQ; ++e) {
                        R m = mixed ? dn[e] : qn[e];
                        mn[e] = Rmin(mn[e], m); mx[e] = Rmax(mx[e], m);
                    }
                }
            }
            if (A.P.dim == 2) {
                R id = R(1) / (a11 * a22 - a12 * a12);
#pragma unroll
                for (int v = 0; v < 6; ++v) {
                    gx[v] = (a22 * bb[v][0] - a12 * bb[v][1]) * id;
                    gy[v] = (a11 * bb[v][1] - a12 * bb[v][0]) * id;
                    gz[v] = R(0);
                }
            } else {
                R c11 = a22 * a33 - a23 * a23, c12 = a13 * a23 - a12 * a33, c13 = a12 * a23 - a13 * a22;
                R c22 = a11 * a33 - a13 * a13, c23 = a12 * a13 - a11 * a23, c33 = a11 * a22 - a12 * a12;
                R id = R(1) / (a11 * c11 + a12 * c12 + a13 * c13);
#pragma unroll
                for (int v = 0; v < 6; ++v) {
                    gx[v] = (c11 * bb[v][0] + c12 * bb[v][1] + c13 * bb[v][2]) * id;
                    gy[v] = (c12 * bb[v][0] + c22 * bb[v][1] + c23 * bb[v][2]) * id;
                    gz[v] = (c13 * bb[v][0] + c23 * bb[v][1] + c33 * bb[v][2]) * id;
                }
            }
        } else {
            for (int k = b; k < en; ++k) {
                int2 e2 = __ldg(&A.nbl[k]);
                int f = nb_face(e2), nb = e2.y;
                bool right = nb_right(e2);
                R qn[REC], cgn[CGR], fg[FGR], dn[6];
                R cl, cr;
                if constexpr (mixed) {
                    double t[REC];
                    ld8(A.q + (size_t)nb * REC, t);
#pragma unroll
                    for (int v = 0; v < 6; ++v)   // the cell's own values re-read (L1 hits), not held
                        dn[v] = R(t[v < 5 ? v : ITT] - __ldg(A.q + (size_t)c * REC + (v < 5 ? v : ITT)));
                    ld4(A.fgeo + (size_t)f * FGR, fg);   // normal and area
                    if (A.P.igrad == 1) {
                        cl = R(0.5); cr = R(0.5);
                    } else {   // |x_f - x_L|, |x_f - x_R| formed in FP64
                        float2 dd = __ldg(reinterpret_cast<const float2 *>(A.fofs + (size_t)f * FOFS + 6));
                        R delta = R(1) / (dd.x + dd.y + small_v<R>());
                        cl = dd.y * delta; cr = dd.x * delta;
                    }
                } else {
                    ld8(A.qs + (size_t)nb * REC, qn);
                    ld4(A.cgeo + (size_t)nb * CGR, cgn);
                    ld8(A.fgeo + (size_t)f * FGR, fg);
                    const R *cl_ = right ? cgn : cgc, *cr_ = right ? cgc : cgn;
                    if (A.P.igrad == 1) {
                        cl = R(0.5); cr = R(0.5);
                    } else {
                        R dxl = fg[4] - cl_[0], dyl = fg[5] - cl_[1], dzl = fg[6] - cl_[2];
                        R dxr = fg[4] - cr_[0], dyr = fg[5] - cr_[1], dzr = fg[6] - cr_[2];
                        R delt1 = Rsqrt(SQR3(dxl, dyl, dzl)), delt2 = Rsqrt(SQR3(dxr, dyr, dzr));
                        R delta = R(1) / (delt1 + delt2 + small_v<R>());
                        cl = delt2 * delta; cr = delt1 * delta;
                    }
                }
                const R *ql = right ? qn : qc, *qr = right ? qc : qn;
                R ar = fg[3];
                R fnxa = fg[0] * ar, fnya = fg[1] * ar, fnza = fg[2] * ar;
                // FP32 path: face value minus the cell value (the cell's own
                // term sums to zero over the closed cell surface)
                R wn = right ? cl : cr;
#pragma unroll
                for (int v = 0; v < 6; ++v) {
                    if (v >= nvar) break;
                    int iv = v < 5 ? v : ITT;
                    R value;
                    if constexpr (mixed) value = wn * dn[v];
                    else value = (A.P.igrad == 1) ? R(0.5) * (ql[iv] + qr[iv]) : cl * ql[iv] + cr * qr[iv];
                    if (!right) { gx[v] += fnxa * value; gy[v] += fnya * value; gz[v] += fnza * value; }
                    else        { gx[v] -= fnxa * value; gy[v] -= fnya * value; gz[v] -= fnza * value; }
                }
                if (nb < A.nCells) {
#pragma unroll
                    for (int e = 0; e < NEQ; ++e) {
                        R m = mixed ? dn[e] : qn[e];
                        mn[e] = Rmin(mn[e], m); mx[e] = Rmax(mx[e], m);
                    }
                }
            }
            R ovol = R(1) / cgc[3];
#pragma unroll
            for (int v = 0; v < 6; ++v) { gx[v] *= ovol; gy[v] *= ovol; gz[v] *= ovol; }
        }
        R rec[GLR];
#pragma unroll
        for (int v = 0; v < 6; ++v) { rec[v * 3] = gx[v]; rec[v * 3 + 1] = gy[v]; rec[v * 3 + 2] = gz[v]; }
        if constexpr (!mixed) {
#pragma unroll
            for (int e = 0; e < NEQ; ++e) { mn[e] -= qc[e]; mx[e] -= qc[e]; }
        }
        R lim[NEQ];
        if (limMode == 1) {
            R eps[NEQ];
            R h = A.P.dim == 2 ? Rsqrt(cgc[3]) : R(cbrt(double(cgc[3])));
            R kk = R(A.P.vencat_coef) * h;
            R epsc = kk * kk * kk + small_v<R>();
#pragma unroll
            for (int e = 0; e < NEQ; ++e) eps[e] = epsc;
            cell_limiter(A, c, cgc, rec, mn, mx, eps, lim);
        } else {
            R pre = (A.P.ilim == 0) ? R(1) : R(0);   // CalcNoLimiter / CalcZeroLimiter
#pragma unroll
            for (int e = 0; e < NEQ; ++e) lim[e] = pre;
        }
#pragma unroll
        for (int e = 0; e < NEQ; ++e) rec[18 + e] = lim[e];
        rec[23] = R(0);
        R *o = A.gl + (size_t)c * GLR;
#pragma unroll
        for (int i = 0; i < GLR; i += 4) st4(o + i, rec + i);
        if (limMode == 2) {
            R *m = A.mm + (size_t)c * MMR;
#pragma unroll
            for (int e = 0; e < NEQ; ++e) { m[e] = mn[e]; m[5 + e] = mx[e]; }
        }
    }
    if (limMode == 2) {   // block extremes for the zone-wide eps (ULimiter.cpp:571-593)
#pragma unroll
        for (int e = 0; e < NEQ; ++e) {
            sred[e][threadIdx.x] = active ? double(mn[e]) : 1.0e40;
            sred[NEQ + e][threadIdx.x] = active ? double(mx[e]) : -1.0e40;
        }
        __syncthreads();
        for (int s = blockDim.x / 2; s > 0; s >>= 1) {
            if (threadIdx.x < s) {
#pragma unroll
                for (int e = 0; e < NEQ; ++e) {
                    sred[e][threadIdx.x] = fmin(sred[e][threadIdx.x], sred[e][threadIdx.x + s]);
                    sred[NEQ + e][threadIdx.x] = fmax(sred[NEQ + e][threadIdx.x], sred[NEQ + e][threadIdx.x + s]);
                }
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
#pragma unroll
            for (int e = 0; e < 2 * NEQ; ++e) A.partial[(size_t)blockIdx.x * 10 + e] = sred[e][0];
        }
    }
}

// zone-wide eps per equation, ULimiter.cpp:571-593 (single block; min/max exact)
template <typename R>
__global__ void __launch_bounds__(256) k_limiter_eps(KArgs<R> A, int nPartial) {
    __shared__ double smn[NEQ][256], smx[NEQ][256];
    double lmin[NEQ], lmax[NEQ];
#pragma unroll
    for (int e = 0; e < NEQ; ++e) { lmin[e] = 1.0e40; lmax[e] = -1.0e40; }
    for (int i = threadIdx.x; i < nPartial; i += blockDim.x)
#pragma unroll
        for (int e = 0; e < NEQ; ++e) {
            lmin[e] = fmin(lmin[e], A.partial[(size_t)i * 10 + e]);
            lmax[e] = fmax(lmax[e], A.partial[(size_t)i * 10 + 5 + e]);
        }
#pragma unroll
    for (int e = 0; e < NEQ; ++e) { smn[e][threadIdx.x] = lmin[e]; smx[e][threadIdx.x] = lmax[e]; }
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
#pragma unroll
            for (int e = 0; e < NEQ; ++e) {
                smn[e][threadIdx.x] = fmin(smn[e][threadIdx.x], smn[e][threadIdx.x + s]);
                smx[e][threadIdx.x] = fmax(smx[e][threadIdx.x], smx[e][threadIdx.x + s]);
            }
        __syncthreads();
    }
    if (threadIdx.x == 0)
#pragma unroll
        for (int e = 0; e < NEQ; ++e) {
            double eps = A.P.vencat_coef * fmax(smx[e][0] - smn[e][0], 1.0);
            A.scal[S_EPS + e] = eps * eps + SMALLD;
        }
}

template <typename R>
__global__ void __launch_bounds__(128) k_limiter_global(KArgs<R> A) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= A.nCells) return;
    R cgc[CGR], rec[GLR];
    ld4(A.cgeo + (size_t)c * CGR, cgc);
    R *o = A.gl + (size_t)c * GLR;
#pragma unroll
    for (int i = 0; i < GLR; i += 4) ld4(o + i, rec + i);
    const R *m = A.mm + (size_t)c * MMR;
    R mn[NEQ], mx[NEQ], eps[NEQ], lim[NEQ];
#pragma unroll
    for (int e = 0; e < NEQ; ++e) { mn[e] = m[e]; mx[e] = m[5 + e]; eps[e] = R(A.scal[S_EPS + e]); }
    cell_limiter(A, c, cgc, rec, mn, mx, eps, lim);
#pragma unroll
    for (int e = 0; e < NEQ; ++e) o[18 + e] = lim[e];
}

// ---------------------------------------------------------------------------
// UPDATE_RESIDUALS: UNsInvFlux::CalcFlux (codes/uns/src/UNsInvFlux.cpp:123-215)
// + UNsVisFlux::CalcFlux (codes/uns/src/UNsVisFlux.cpp:90-440), per cell in
// ascending face order (AddF2CField, codes/usolver/src/UCom.cpp:144-171),
// fused with the spectral radii and local time step of CALC_TIME_STEP.
// ---------------------------------------------------------------------------
// face states qL/qR of face f (left l, right r): NsLimField::BcQlQrFix
// (codes/uns/src/UNsLimiter.cpp:67-101) on boundary faces, LimField::CalcFaceValue
// (codes/usolver/src/ULimiter.cpp:188-256) + NsCheckFunction inside
template <typename R>
__device__ __forceinline__ void face_states(const KArgs<R> &A, int f, const R *ql, const R *qr, const R *fg,
                                            const R *cgl, const R *cgr, const R *gll, const R *glr, R *t1, R *t2) {
    if (f < A.nBFaces) {
        if (A.bcType[f] == BC_SOLID) {
            const double *b = A.bcq + (size_t)f * NEQ;
#pragma unroll
            for (int e = 0; e < NEQ; ++e) t1[e] = t2[e] = R(b[e]);
        } else {
#pragma unroll
            for (int e = 0; e < NEQ; ++e) t1[e] = t2[e] = R(0.5) * (ql[e] + qr[e]);
        }
        return;
    }
#pragma unroll
    for (int e = 0; e < NEQ; ++e) { t1[e] = ql[e]; t2[e] = qr[e]; }
    if (A.P.ilim == -1) return;   // first order: the zero limiter keeps the cell values
    R u1[NEQ], u2[NEQ];
    R dx = fg[4] - cgl[0], dy = fg[5] - cgl[1], dz = fg[6] - cgl[2];
#pragma unroll
    for (int e = 0; e < NEQ; ++e) {
        R phi = Rmin(gll[18 + e], glr[18 + e]);
        u1[e] = t1[e] + phi * (gll[e * 3] * dx + gll[e * 3 + 1] * dy + gll[e * 3 + 2] * dz);
    }
    dx = fg[4] - cgr[0]; dy = fg[5] - cgr[1]; dz = fg[6] - cgr[2];
#pragma unroll
    for (int e = 0; e < NEQ; ++e) {
        R phi = Rmin(glr[18 + e], gll[18 + e]);
        u2[e] = t2[e] + phi * (glr[e * 3] * dx + glr[e * 3 + 1] * dy + glr[e * 3 + 2] * dz);
    }
    if (!(u1[IR] <= R(0) || u1[IP] <= R(0)))
#pragma unroll
        for (int e = 0; e < NEQ; ++e) t1[e] = u1[e];
    if (!(u2[IR] <= R(0) || u2[IP] <= R(0)))
#pragma unroll
        for (int e = 0; e < NEQ; ++e) t2[e] = u2[e];
}

// The same face states for the FP32-face path, formed in FP64 (t1, t2) from
// the FP64 cell values (qlD, qrD) plus the FP32 limited gradient corrections,
// so that they carry no FP32 rounding of the (large) cell values; s1, s2 are
// their FP32 counterparts from the FP32 copies (qlf, qrf) of the cell values.
__device__ __forceinline__ void face_states_mixed(const KArgs<float> &A, int f, const double *qlD, const double *qrD,
                                                  const float *qlf, const float *qrf, const float *fg,
                                                  const float *cgl, const float *cgr, const float *gll,
                                                  const float *glr, double *t1, double *t2, float *s1, float *s2) {
    if (f < A.nBFaces) {
        if (A.bcType[f] == BC_SOLID) {
            const double *b = A.bcq + (size_t)f * NEQ;
#pragma unroll
            for (int e = 0; e < NEQ; ++e) { t1[e] = t2[e] = b[e]; s1[e] = s2[e] = float(b[e]); }
        } else {
#pragma unroll
            for (int e = 0; e < NEQ; ++e) {
                t1[e] = t2[e] = 0.5 * (qlD[e] + qrD[e]);
                s1[e] = s2[e] = 0.5f * (qlf[e] + qrf[e]);
            }
        }
        return;
    }
#pragma unroll
    for (int e = 0; e < NEQ; ++e) { t1[e] = qlD[e]; t2[e] = qrD[e]; s1[e] = qlf[e]; s2[e] = qrf[e]; }
    if (A.P.ilim == -1) return;
    float c1[NEQ], c2[NEQ];
    float dx = fg[4] - cgl[0], dy = fg[5] - cgl[1], dz = fg[6] - cgl[2];
#pragma unroll
    for (int e = 0; e < NEQ; ++e)
        c1[e] = fminf(gll[18 + e], glr[18 + e]) * (gll[e * 3] * dx + gll[e * 3 + 1] * dy + gll[e * 3 + 2] * dz);
    dx = fg[4] - cgr[0]; dy = fg[5] - cgr[1]; dz = fg[6] - cgr[2];
#pragma unroll
    for (int e = 0; e < NEQ; ++e)
        c2[e] = fminf(glr[18 + e], gll[18 + e]) * (glr[e * 3] * dx + glr[e * 3 + 1] * dy + glr[e * 3 + 2] * dz);
    double r1 = t1[IR] + double(c1[IR]), p1 = t1[IP] + double(c1[IP]);
    double r2 = t2[IR] + double(c2[IR]), p2 = t2[IP] + double(c2[IP]);
    if (!(r1 <= 0.0 || p1 <= 0.0)) {
#pragma unroll
        for (int e = 0; e < NEQ; ++e) { t1[e] += double(c1[e]); s1[e] += c1[e]; }
    }
    if (!(r2 <= 0.0 || p2 <= 0.0)) {
#pragma unroll
        for (int e = 0; e < NEQ; ++e) { t2[e] += double(c2[e]); s2[e] += c2[e]; }
    }
}

// Face geometry of the VIS_TEST / VIS_NEW1 / VIS_NEW2 face gradients: the
// distance weights and normal offsets of VisGradGeom::CalcFaceWeight /
// PrepareCellGeom (codes/usolver/src/VisGrad.cpp:44-97) and the face tangents
// of GCom::CalcTangent (codes/global/src/Com.cpp:74-121).
template <typename R> struct VisGeomD {
    R fw1, fw2, d1, d2, dxnl, dynl, dznl, dxnr, dynr, dznr, angle1, angle2, t1[3], t2[3];
};

template <typename R> __device__ __forceinline__ R vis_angle(R dx, R dy, R dz, R dist) {
    R r = dist / (Rsqrt(SQR3(dx, dy, dz)) + small_v<R>());
    if (r > R(1)) r = R(1);
    if (r < R(-1)) r = R(-1);
    return asin(r) * R(180) / R(3.141592653589793);
}

template <typename R>
__device__ __forceinline__ void vis_geom(const R *fg, const R *cgl, const R *cgr, VisGeomD<R> &G) {
    R xn = fg[0], yn = fg[1], zn = fg[2];
    R ax = fg[4] - cgl[0], ay = fg[5] - cgl[1], az = fg[6] - cgl[2];
    R bx = fg[4] - cgr[0], by = fg[5] - cgr[1], bz = fg[6] - cgr[2];
    R delt1 = Rsqrt(SQR3(ax, ay, az)), delt2 = Rsqrt(SQR3(bx, by, bz));
    R delta = R(1) / (delt1 + delt2 + small_v<R>());
    G.fw1 = delt2 * delta;
    G.fw2 = delt1 * delta;
    R dxl = cgl[0] - fg[4], dyl = cgl[1] - fg[5], dzl = cgl[2] - fg[6];
    R dxr = cgr[0] - fg[4], dyr = cgr[1] - fg[5], dzr = cgr[2] - fg[6];
    G.d1 = xn * dxl + yn * dyl + zn * dzl;
    G.d2 = xn * dxr + yn * dyr + zn * dzr;
    G.dxnl = xn * G.d1 - dxl; G.dynl = yn * G.d1 - dyl; G.dznl = zn * G.d1 - dzl;
    G.dxnr = xn * G.d2 - dxr; G.dynr = yn * G.d2 - dyr; G.dznr = zn * G.d2 - dzr;
    G.angle1 = vis_angle(dxl, dyl, dzl, -G.d1);
    G.angle2 = vis_angle(dxr, dyr, dzr, G.d2);
    R *t1 = G.t1, *t2 = G.t2;
    if (xn != R(0)) { t1[0] = yn; t1[1] = -xn; t1[2] = R(0); }
    else if (yn != R(0)) { t1[0] = -yn; t1[1] = xn; t1[2] = R(0); }
    else if (zn != R(0)) { t1[0] = R(0); t1[1] = -zn; t1[2] = yn; }
    else {
#pragma unroll
        for (int k = 0; k < 3; ++k) t1[k] = t2[k] = R(0);
        return;
    }
    R dtmp = R(1) / Rsqrt(SQR3(t1[0], t1[1], t1[2]));
    t1[0] *= dtmp; t1[1] *= dtmp; t1[2] *= dtmp;
    t2[0] = yn * t1[2] - zn * t1[1];
    t2[1] = zn * t1[0] - xn * t1[2];
    t2[2] = xn * t1[1] - yn * t1[0];
}

// One variable's face gradient and normal derivative under VIS_TEST (2),
// VIS_NEW1 (3) or VIS_NEW2 (4): VisGrad::CalcTestMethod / CalcNew1Method /
// CalcNew2Method followed by ModifyFaceGrad (codes/usolver/src/VisGrad.cpp:268-353).
// g1, g2: the left and right cell gradients; a boundary face weights the
// left side only in VIS_TEST.
template <typename R>
__device__ __forceinline__ void vis_variant(int scheme, const VisGeomD<R> &G, bool bface, R xn, R yn, R zn, R q1,
                                            R q2, const R *g1, const R *g2, R *grad, R &dqdn) {
    const R sm = small_v<R>();
    R q = R(0.5) * (q1 + q2), q11 = q1, q22 = q2;
    dqdn = R(0);
    if (scheme == 2) {
        if (G.angle1 > R(20) && G.angle2 > R(20)) {
            q11 += g1[0] * G.dxnl + g1[1] * G.dynl + g1[2] * G.dznl;
            q22 += g2[0] * G.dxnr + g2[1] * G.dynr + g2[2] * G.dznr;
        }
        if (G.angle1 > R(0) && G.angle2 > R(0) && Rabs(G.d1) > sm && Rabs(G.d2) > sm) {
            R dtmp = G.d1 * G.d1 + G.d2 * G.d2;
            R c1 = G.d1 * G.d1 / dtmp, c2 = R(1) - c1;
            if (bface) { c1 = R(1); c2 = R(0); }
            R dqdn1 = (q11 - q) / G.d1, dqdn2 = (q22 - q) / G.d2;
            dqdn = c1 * dqdn1 + c2 * dqdn2;
        }
    } else if (scheme == 3) {
        if (G.d1 * G.d2 < R(0) && Rabs(G.d1) > sm && Rabs(G.d2) > sm) {
            R d = R(-2) * G.d1 * G.d2 / (G.d1 * G.d1 + G.d2 * G.d2 + sm);
            R od = d / (G.d2 - G.d1);
            q11 += g1[0] * G.dxnl + g1[1] * G.dynl + g1[2] * G.dznl;
            q22 += g2[0] * G.dxnr + g2[1] * G.dynr + g2[2] * G.dznr;
            dqdn = (q22 - q11) * od;
        }
    } else {
        R d = R(-2) * G.d1 * G.d2 / (G.d1 * G.d1 + G.d2 * G.d2 + sm);
        if (d > R(0.1)) {
            q11 += g1[0] * G.dxnl + g1[1] * G.dynl + g1[2] * G.dznl;
            q22 += g2[0] * G.dxnr + g2[1] * G.dynr + g2[2] * G.dznr;
            R dqdn1 = (q11 - q) / G.d1, dqdn2 = (q22 - q) / G.d2;
            if (dqdn1 * dqdn2 > R(0)) dqdn = R(2) * dqdn1 * dqdn2 / (dqdn1 + dqdn2);
        }
    }
    R gx = G.fw1 * g1[0] + G.fw2 * g2[0];
    R gy = G.fw1 * g1[1] + G.fw2 * g2[1];
    R gz = G.fw1 * g1[2] + G.fw2 * g2[2];
    R dqdt1 = G.t1[0] * gx + G.t1[1] * gy + G.t1[2] * gz;
    R dqdt2 = G.t2[0] * gx + G.t2[1] * gy + G.t2[2] * gz;
    grad[0] = xn * dqdn + G.t1[0] * dqdt1 + G.t2[0] * dqdt2;
    grad[1] = yn * dqdn + G.t1[1] * dqdt1 + G.t2[1] * dqdt2;
    grad[2] = zn * dqdn + G.t1[2] * dqdt1 + G.t2[2] * dqdt2;
}

// The six face gradients of VIS_TEST / NEW1 / NEW2 and the scheme's dT/dn,
// which the heat flux takes.  Compiled only into the k_residual instances for
// these schemes (VV): even an untaken call costs the common path registers.
template <typename R>
__device__ __forceinline__ void vis_variant_grads(int scheme, const R *fg, const R *cgl, const R *cgr, const R *ql,
                                               const R *qr, const R *gl, const R *gr, bool bface, R *gx, R *gy,
                                               R *gz, R &dtdn) {
    VisGeomD<R> G;
    vis_geom(fg, cgl, cgr, G);
#pragma unroll
    for (int v = 0; v < 6; ++v) {
        int iv = v < 5 ? v : ITT;
        R gr3[3], dn;
        vis_variant(scheme, G, bface, fg[0], fg[1], fg[2], ql[iv], qr[iv], gl + v * 3, gr + v * 3, gr3, dn);
        gx[v] = gr3[0]; gy[v] = gr3[1]; gz[v] = gr3[2];
        if (v == 5) dtdn = dn;
    }
}

// viscous face flux with the VIS_STD face gradient (VIS_AVER: the average of
// the cell gradients, UNsVisFlux::AverMethod, codes/uns/src/UNsVisFlux.cpp:357-366;
// VIS_TEST / NEW1 / NEW2: vis_variant above), before the -S/Re factor
// (UNsVisFlux::PrepareFaceValue/StdMethod/CalcStress/CalcNsVisFlux,
// codes/usolver/src/VisGrad.cpp:150-175,356-366)
// dlr: qr - ql of the six gradient variables (rho, u, v, w, p, T)
template <typename R, bool VV>
__device__ __forceinline__ void face_vis_flux(const DevParams &P, const R *ql, const R *qr, const R *dlr, const R *fg,
                                              const R *cgl, const R *cgr, const R *gl, const R *gr, bool bface,
                                              R *fv) {
    R half = R(0.5);
    R vlm = half * (ql[IML] + qr[IML]), vtm = half * (ql[IMT] + qr[IMT]);
    R vis = vlm + vtm;
    R dx = cgr[0] - cgl[0], dy = cgr[1] - cgl[1], dz = cgr[2] - cgl[2];
    R ods = R(1) / Rsqrt(SQR3(dx, dy, dz));
    dx *= ods; dy *= ods; dz *= ods;
    R gx[6], gy[6], gz[6], qm[6];
#pragma unroll
    for (int v = 0; v < 6; ++v) {
        int iv = v < 5 ? v : ITT;
        R q1 = ql[iv], q2 = qr[iv];
        qm[v] = half * (q1 + q2);
        gx[v] = half * (gl[v * 3] + gr[v * 3]);
        gy[v] = half * (gl[v * 3 + 1] + gr[v * 3 + 1]);
        gz[v] = half * (gl[v * 3 + 2] + gr[v * 3 + 2]);
        if (P.ivischeme == 0) {   // VIS_STD's CorrectGrad; VIS_AVER keeps the average
            R fOld = gx[v] * dx + gy[v] * dy + gz[v] * dz;
            R fnew = dlr[v] * ods;
            R df = fnew - fOld;
            gx[v] += df * dx; gy[v] += df * dy; gz[v] += df * dz;
        }
    }
    R xn = fg[0], yn = fg[1], zn = fg[2];
    R dtdn = xn * gx[5] + yn * gy[5] + zn * gz[5];
    if constexpr (VV)   // TEST / NEW1 / NEW2 replace the face gradients
        vis_variant_grads(P.ivischeme, fg, cgl, cgr, ql, qr, gl, gr, bface, gx, gy, gz, dtdn);
    R kcp = (vlm * R(P.oprl) + vtm * R(P.oprt)) * R(P.const_cp);
    R qNormal = R(0);
    qNormal += xn * R(0) + yn * R(0) + zn * R(0);
    qNormal += kcp * dtdn;
    R divv2p3 = R(2.0 / 3.0) * (gx[IU] + gy[IV] + gz[IW]);
    R txx = vis * (R(2) * gx[IU] - divv2p3);
    R tyy = vis * (R(2) * gy[IV] - divv2p3);
    R tzz = vis * (R(2) * gz[IW] - divv2p3);
    R txy = vis * (gy[IU] + gx[IV]);
    R txz = vis * (gz[IU] + gx[IW]);
    R tyz = vis * (gz[IV] + gy[IW]);
    fv[0] = R(0);
    fv[1] = xn * txx + yn * txy + zn * txz;
    fv[2] = xn * txy + yn * tyy + zn * tyz;
    fv[3] = xn * txz + yn * tyz + zn * tzz;
    fv[4] = qm[IU] * fv[1] + qm[IV] * fv[2] + qm[IW] * fv[3] + qNormal;
}

template <typename R, bool VV>
__device__ __forceinline__ void face_vis_flux(const DevParams &P, const R *ql, const R *qr, const R *fg, const R *cgl,
                                              const R *cgr, const R *gl, const R *gr, bool bface, R *fv) {
    R dlr[6];
#pragma unroll
    for (int v = 0; v < 6; ++v) {
        int iv = v < 5 ? v : ITT;
        dlr[v] = qr[iv] - ql[iv];
    }
    face_vis_flux<R, VV>(P, ql, qr, dlr, fg, cgl, cgr, gl, gr, bface, fv);
}

// The end of the residual pass of one cell: its residual and block sums of
// squares (for the norms), and the local time step from the summed face
// radii (UTimeStep::CalcInvTimeStep / CalcVisTimeStep) with the zone-wide
// minimum.  The block epilogue sums the squares in a fixed order
// (deterministic) and lowers the minimum time step by an atomic minimum on
// the bit pattern (non-negative doubles order like their bits).  Every thread
// of the block calls it; `active` is false past the last cell.
template <bool doRes, bool doDt>
__device__ __forceinline__ void residual_epilogue(const DevParams &P, double *res, double *dt, double *invsr,
                                                  double *vissr, double *npart, double *scal, int c, bool active,
                                                  const double *acc, double inv, double vis, double vol) {
    double mydt = 1.0e40;
    double sq[NEQ] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (active) {
        if (doRes) {
            double *o = res + (size_t)c * NEQ;
#pragma unroll
            for (int e = 0; e < NEQ; ++e) { o[e] = acc[e]; sq[e] = acc[e] * acc[e]; }
        }
        if (doDt) {
            double cfl = scal[S_CFL];
            double ts;
            if (P.timestepModel == 1) {
                ts = P.global_dt;
            } else {
                ts = cfl * vol / inv;
                if (P.vismodel > 0 && P.visTimeStepModel > 0) {
                    double vts = cfl * vol / vis;
                    ts *= vts / (ts + vts);
                }
            }
            invsr[c] = inv;
            vissr[c] = vis;
            dt[c] = ts;
            mydt = ts;
        }
    }
    if (doRes) block_sum_to<NEQ>(sq, npart + (size_t)blockIdx.x * NEQ);
    if (doDt) {
        double m = block_min(mydt);
        if (threadIdx.x == 0)
            atomicMin(reinterpret_cast<unsigned long long *>(scal + S_MINDT), (unsigned long long)__double_as_longlong(m));
    }
}

// The FP64 path's residual: one gather pass per cell -- face radii + time
// step, inviscid residual, then the viscous residual in a second loop over the
// same faces, as the reference's two scatter passes add them (every sum in
// the reference's order, so the path rounds like the reference).
// MODE 0: residual and time step (one outer iteration), 1: time step only
// (the CALC_TIME_STEP task), 2: residual only (the UPDATE_RESIDUALS task).
template <typename R, int MODE, bool VV = false>
__global__ void __launch_bounds__(128, MinBlocks<R>::res) k_residual(KArgs<R> A) {
    static_assert(sizeof(R) == 8, "the mixed path runs k_face_pass + k_face_sum");
    constexpr bool doRes = MODE != 1, doDt = MODE != 2;
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    bool active = c < A.nCells;
    double acc[NEQ];
#pragma unroll
    for (int e = 0; e < NEQ; ++e) acc[e] = -0.0;   // LoadResiduals: res = -rhs, rhs = 0
    double inv = 0.0, vis = 0.0, vol = 0.0;
    if (active) {
        const DevParams &P = A.P;
        R qc[REC], cgc[CGR], glc[GLR];
        ld8(A.qs + (size_t)c * REC, qc);
        ld4(A.cgeo + (size_t)c * CGR, cgc);
        vol = double(cgc[3]);
        bool needGl = doRes && (P.ilim != -1 || P.vismodel > 0);
        if (needGl) {
#pragma unroll
            for (int i = 0; i < GLR; i += 4) ld4(A.gl + (size_t)c * GLR + i, glc + i);
        }
        R gam = R(P.gama), ce1 = R(P.centropy1), ce2 = R(P.centropy2), orey = R(P.oreynolds);
        int b = A.nb_off[c], en = A.nb_off[c + 1];
        // the next neighbour-list entry is loaded one face ahead, so that the
        // loads of a face's records do not wait on its list entry
        int2 e2n = b < en ? __ldg(&A.nbl[b]) : make_int2(0, 0);
        for (int k = b; k < en; ++k) {
            int2 e2 = e2n;
            if (k + 1 < en) e2n = __ldg(&A.nbl[k + 1]);
            int f = nb_face(e2), nb = e2.y;
            bool right = nb_right(e2);
            R qn[REC], cgn[CGR], fg[FGR], gln[GLR];
            ld8(A.qs + (size_t)nb * REC, qn);
            ld8(A.fgeo + (size_t)f * FGR, fg);
            ld4(A.cgeo + (size_t)nb * CGR, cgn);
            bool ghost = nb >= A.nCells;
            if (needGl && !ghost) {
#pragma unroll
                for (int i = 0; i < GLR; i += 4) ld4(A.gl + (size_t)nb * GLR + i, gln + i);
            }
            const R *ql = right ? qn : qc, *qr = right ? qc : qn;
            const R *cgl = right ? cgn : cgc, *cgr = right ? cgc : cgn;
            // ghost cells carry their interior cell's gradient (UGrad.cpp:140-148)
            const R *gll = right ? gln : glc, *glr = (right || ghost) ? glc : gln;
            if (doDt) {
                inv += face_inv_spec(P, ql, qr, fg);
                if (P.vismodel > 0) vis += face_vis_spec(P, ql, qr, fg, cgl, cgr);
            }
            if (!doRes) continue;
            R t1[NEQ], t2[NEQ], fl[NEQ];
            face_states(A, f, ql, qr, fg, cgl, cgr, gll, glr, t1, t2);
            if (P.ischeme == 12) slau2Flux(t1, t2, fg[0], fg[1], fg[2], gam, fl);
            else roeFlux(t1, t2, fg[0], fg[1], fg[2], gam, P.ieigenfix, ce1, ce2, fl);
            R ar = fg[3];
#pragma unroll
            for (int e = 0; e < NEQ; ++e) {
                double v = double(ar * fl[e]);
                if (!right) acc[e] -= v; else acc[e] += v;
            }
        }
        if (doRes && P.vismodel > 0) {
            int2 e2n = b < en ? __ldg(&A.nbl[b]) : make_int2(0, 0);   // list entry one face ahead
            for (int k = b; k < en; ++k) {
                int2 e2 = e2n;
                if (k + 1 < en) e2n = __ldg(&A.nbl[k + 1]);
                int f = nb_face(e2), nb = e2.y;
                bool right = nb_right(e2);
                R qn[REC], cgn[CGR], fg[FGR], gln[GLR];
                ld8(A.qs + (size_t)nb * REC, qn);
                ld8(A.fgeo + (size_t)f * FGR, fg);
                ld4(A.cgeo + (size_t)nb * CGR, cgn);
                bool ghost = nb >= A.nCells;
                if (!ghost) {
#pragma unroll
                    for (int i = 0; i < GLR; i += 4) ld4(A.gl + (size_t)nb * GLR + i, gln + i);
                }
                const R *ql = right ? qn : qc, *qr = right ? qc : qn;
                const R *cgl = right ? cgn : cgc, *cgr = right ? cgc : cgn;
                const R *gll = right ? gln : glc, *glr = (right || ghost) ? glc : gln;
                R fv[NEQ];
                face_vis_flux<R, VV>(P, ql, qr, fg, cgl, cgr, gll, glr, ghost, fv);
                R coeff = -orey * fg[3];
#pragma unroll
                for (int e = 0; e < NEQ; ++e) {
                    double v = double(coeff * fv[e]);
                    if (!right) acc[e] -= v; else acc[e] += v;
                }
            }
        }
    }
    residual_epilogue<doRes, doDt>(A.P, A.res, A.dt, A.invsr, A.vissr, A.npart, A.scal, c, active, acc, inv, vis,
                                   vol);
}

// ---------------------------------------------------------------------------
// The mixed path's UPDATE_RESIDUALS + CALC_TIME_STEP in two passes.
//
// k_face_pass: one thread per face, in face order (the face arrays are read
// coalesced, each face's flux is evaluated once): the face's spectral radii,
// its MUSCL face states, Roe or SLAU2 flux and viscous flux, written to the
// face record fout[f] = {flux[5] (left to right, FP64), {inviscid, viscous
// radius} (FP32)}.  Its geometry is local to the face: the offsets from the
// face centre to the two cell centres, formed in FP64 from the reference's
// metrics and rounded once to FP32 (so no FP32 rounding of an absolute
// coordinate enters a difference), and the FP64 unit normal and area for the
// FP64 central part of the Roe flux (so that in a uniform state the pressure
// terms of a cell's faces cancel to FP64 round-off, as the reference's do).
//
// k_face_sum: one thread per cell adds its faces' records in ascending face
// id -- the order of the reference's serial scatter (AddF2CField,
// codes/usolver/src/UCom.cpp:144-171) -- into its residual and radii.  Both
// cells of a face add the same FP64 value, so the sum over the mesh telescopes
// exactly.  MODE as in k_residual.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void store_face_out(double *o, const double *v, float si, float sv) {
    double packed = __hiloint2double(__float_as_int(sv), __float_as_int(si));
    reinterpret_cast<double2 *>(o)[0] = make_double2(v[0], v[1]);
    reinterpret_cast<double2 *>(o)[1] = make_double2(v[2], v[3]);
    reinterpret_cast<double2 *>(o)[2] = make_double2(v[4], packed);
}

template <int MODE, bool VV = false, int MINB = MinBlocks<float>::fp>
__global__ void __launch_bounds__(128, MINB) k_face_pass(KArgs<float> A) {
    constexpr bool doRes = MODE != 1, doDt = MODE != 2;
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= A.nFaces) return;
    const DevParams &P = A.P;
    const int2 lr = __ldg(A.lr + f);
    const bool bface = f < A.nBFaces;
    double nD[4];   // unit normal and area, FP64
    ld4(A.fgeoD + (size_t)f * FGR, nD);
    float fo[FOFS];
    ld8(A.fofs + (size_t)f * FOFS, fo);
    // the face's own frame: face centre at the origin, cell centres at
    // -(x_f - x_L) and -(x_f - x_R); every kernel function below only forms
    // differences of these positions
    const float fg[FGR] = {float(nD[0]), float(nD[1]), float(nD[2]), float(nD[3]), 0.0f, 0.0f, 0.0f, 0.0f};
    const float cgl[CGR] = {-fo[0], -fo[1], -fo[2], 0.0f}, cgr[CGR] = {-fo[3], -fo[4], -fo[5], 0.0f};
    double tl[REC], tr[REC];
    ld8(A.q + (size_t)lr.x * REC, tl);
    ld8(A.q + (size_t)lr.y * REC, tr);
    float ql[REC], qr[REC];
#pragma unroll
    for (int i = 0; i < REC; ++i) { ql[i] = float(tl[i]); qr[i] = float(tr[i]); }
    float si = 0.0f, sv = 0.0f;
    if (doDt) {
        si = float(face_inv_spec(P, ql, qr, fg));
        if (P.vismodel > 0) sv = float(face_vis_spec(P, ql, qr, fg, cgl, cgr));
    }
    double v[NEQ] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (doRes) {
        float gll[GLR], glr[GLR];
        if (P.ilim != -1 || P.vismodel > 0) {
#pragma unroll
            for (int i = 0; i < GLR; i += 4) ld4(A.gl + (size_t)lr.x * GLR + i, gll + i);
            // a ghost cell carries its interior cell's gradient (UGrad.cpp:140-148)
            if (bface) {
#pragma unroll
                for (int i = 0; i < GLR; ++i) glr[i] = gll[i];
            } else {
#pragma unroll
                for (int i = 0; i < GLR; i += 4) ld4(A.gl + (size_t)lr.y * GLR + i, glr + i);
            }
        }
        const float gam = float(P.gama), ce1 = float(P.centropy1), ce2 = float(P.centropy2);
        float fvs[NEQ];   // viscous term, formed first while fewer values are live
        if (P.vismodel > 0) {
            float fv[NEQ];
            face_vis_flux<float, VV>(P, ql, qr, fg, cgl, cgr, gll, glr, bface, fv);
            float coeff = -float(P.oreynolds) * fg[3];
#pragma unroll
            for (int e = 0; e < NEQ; ++e) fvs[e] = coeff * fv[e];
        } else {
#pragma unroll
            for (int e = 0; e < NEQ; ++e) fvs[e] = 0.0f;
        }
        double t1[NEQ], t2[NEQ];
        float s1[NEQ], s2[NEQ];
        face_states_mixed(A, f, tl, tr, ql, qr, fg, cgl, cgr, gll, glr, t1, t2, s1, s2);
        double fc[NEQ];
        float d[NEQ];
        double ard;   // the flux is ard * fc - (arf * d - fvs)
        float arf;
        if (P.ischeme == 12) {
            slau2FluxMixed(t1, t2, s1, s2, nD[0], nD[1], nD[2], fg[0], fg[1], fg[2], gam, fc, d);
            ard = nD[3]; arf = fg[3];
        } else {
            const double og1 = 1.0 / (P.gama - 1.0);
            roeFluxMixed(t1, t2, s1, s2, nD[0], nD[1], nD[2], fg[0], fg[1], fg[2], gam, og1, P.ieigenfix, ce1, ce2,
                         fc, d);
            ard = 0.5 * nD[3]; arf = 0.5f * fg[3];
        }
#pragma unroll
        for (int e = 0; e < NEQ; ++e) v[e] = ard * fc[e] - double(arf * d[e] - fvs[e]);
    }
    store_face_out(A.fout + (size_t)f * FOR, v, si, sv);
}

template <int MODE>
__global__ void __launch_bounds__(128) k_face_sum(KArgs<float> A) {
    constexpr bool doRes = MODE != 1, doDt = MODE != 2;
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    bool active = c < A.nCells;
    double acc[NEQ];
#pragma unroll
    for (int e = 0; e < NEQ; ++e) acc[e] = -0.0;   // LoadResiduals: res = -rhs, rhs = 0
    double inv = 0.0, vis = 0.0, vol = 0.0;
    if (active) {
        vol = double(__ldg(A.cgeo + (size_t)c * CGR + 3));
        int b = A.nb_off[c], en = A.nb_off[c + 1];
        int2 e2n = b < en ? __ldg(&A.nbl[b]) : make_int2(0, 0);   // list entry one face ahead
        for (int k = b; k < en; ++k) {
            int2 e2 = e2n;
            if (k + 1 < en) e2n = __ldg(&A.nbl[k + 1]);
            const double2 *o = reinterpret_cast<const double2 *>(A.fout + (size_t)nb_face(e2) * FOR);
            double2 a = __ldg(o), bb = __ldg(o + 1), cc = __ldg(o + 2);
            if (doDt) {
                int2 sp = make_int2(__double2loint(cc.y), __double2hiint(cc.y));
                inv += double(__int_as_float(sp.x));
                vis += double(__int_as_float(sp.y));
            }
            if (doRes) {
                double v[NEQ] = {a.x, a.y, bb.x, bb.y, cc.x};
                if (!nb_right(e2)) {
#pragma unroll
                    for (int e = 0; e < NEQ; ++e) acc[e] -= v[e];
                } else {
#pragma unroll
                    for (int e = 0; e < NEQ; ++e) acc[e] += v[e];
                }
            }
        }
    }
    residual_epilogue<doRes, doDt>(A.P, A.res, A.dt, A.invsr, A.vissr, A.npart, A.scal, c, active, acc, inv, vis,
                                   vol);
}

// ---------------------------------------------------------------------------
// LU-SGS: UNsLusgs::{LowerSweep,UpperSweep} (codes/uns/src/UNsLusgs.cpp:75-138),
// face increment NsLusgs::GetStandardFluxIncrement (codes/ns/src/NsLusgs.cpp:121-202)
// with the Roe-averaged face radius (UNsLusgs::PrepareDataFacePrim :251-293)
// and the viscous radius (UNsLusgs::CalcViscousTerm :295-330).  Level-scheduled:
// every cell of a level only reads increments of cells in earlier levels.
// ---------------------------------------------------------------------------
// qa: the cell being solved (left after GCom::SetGeometry's swap), qb: neighbour;
// dist = |n . (x_b - x_a)| (the face record's eighth slot, the same from both
// sides), volb the neighbour's volume (read only for visSRModel 1)
template <typename R>
__device__ __forceinline__ void face_increment(const DevParams &P, const R *qa, const R *qb, const R *dqj, R xn,
                                               R yn, R zn, R fa, R dist, R volb, double *rhs0) {
    R vfn = R(0);
    R half = R(0.5), one = R(1), gl = R(P.gama), gr = gl;
    R rl = qa[IR], ul = qa[IU], vl = qa[IV], wl = qa[IW], pl = qa[IP];
    R rr = qb[IR], ur = qb[IU], vr = qb[IV], wr = qb[IW], pr = qb[IP];
    R hl = gl / (gl - one) * pl / rl + half * SQR3(ul, vl, wl);
    R hr = gr / (gr - one) * pr / rr + half * SQR3(ur, vr, wr);
    R tmp0 = Rsqrt(rr / rl);
    R tmp1 = one / (one + tmp0);
    R rm = Rsqrt(rr * rl);
    R um = (ul + ur * tmp0) * tmp1;
    R vm = (vl + vr * tmp0) * tmp1;
    R wm = (wl + wr * tmp0) * tmp1;
    R hm = (hl + hr * tmp0) * tmp1;
    R pm = rm * (hm - half * SQR3(um, vm, wm)) * (gl - one) / gl;
    R gama = gr;
    R c2f_ = Rabs(gama * pm / rm);
    R cmf = Rsqrt(c2f_);
    R vnf = xn * um + yn * vm + zn * wm;
    R maxEig = Rabs(vnf - vfn) + cmf;
    R d0 = R(dqj[0]), d1 = R(dqj[1]), d2 = R(dqj[2]), d3 = R(dqj[3]), d4 = R(dqj[4]);
    R rj = rr, uj = ur, vj = vr, wj = wr, pj = pr;
    R c2 = Rabs(gama * pj / rj);
    R cm = Rsqrt(c2);
    R vn_fluid = xn * uj + yn * vj + zn * wj;
    R vn_rel = vn_fluid - vfn;
    R lmd1 = vn_rel, lmd2 = vn_rel + cm, lmd3 = vn_rel - cm;
    lmd1 = half * (lmd1 + (-maxEig));
    lmd2 = half * (lmd2 + (-maxEig));
    lmd3 = half * (lmd3 + (-maxEig));
    R x1 = (lmd1 + lmd1 - lmd2 - lmd3) / (c2 + c2);
    R x2 = (lmd2 - lmd3) / (cm + cm);
    R dc = vn_fluid * d0 - xn * d1 - yn * d2 - zn * d3;
    R c2dc = c2 * dc;
    R v2 = SQR3(uj, vj, wj);
    R ae = gama - one, af = half * ae * v2;
    R dh = -ae * (uj * d1 + vj * d2 + wj * d3 - d4);
    R enthalpy = (gama / (gama - one)) * (pj / rj);
    dh += af * d0;
    R htot = enthalpy + half * v2;
    R term1 = dh * x1 + dc * x2;
    R term2 = c2dc * x1 + dh * x2;
    R df[NEQ];
    df[0] = lmd1 * d0 - term1;
    df[1] = lmd1 * d1 - uj * term1 + xn * term2;
    df[2] = lmd1 * d2 - vj * term1 + yn * term2;
    df[3] = lmd1 * d3 - wj * term1 + zn * term2;
    df[4] = lmd1 * d4 - htot * term1 + vn_fluid * term2;
#pragma unroll
    for (int e = 0; e < NEQ; ++e) df[e] *= fa;
    if (P.vismodel > 0) {
        R vl_ = qb[IML], vt_ = qb[IMT];
        R visrad;
        R density = half * (rl + rr);
        if (P.visSRModel == 1) {
            R c1 = R(4.0) / R(3.0) * (vl_ + vt_);
            R cc2 = R(P.gama) * (vl_ * R(P.oprl) + vt_ * R(P.oprt));
            R c3 = R(2) * Rmax(c1, cc2) / (R(P.reynolds) * density);
            visrad = fa * fa * c3 / volb;
        } else {
            R viscosity = vl_ + vt_;
            R c1 = R(2) * viscosity / (density * dist * R(P.reynolds) + small_v<R>());
            visrad = half * c1 * fa;
        }
        rhs0[0] -= double(visrad * d0); rhs0[1] -= double(visrad * d1); rhs0[2] -= double(visrad * d2);
        rhs0[3] -= double(visrad * d3); rhs0[4] -= double(visrad * d4);
    }
#pragma unroll
    for (int e = 0; e < NEQ; ++e) rhs0[e] += double(df[e]);
}

// COH: the neighbours' increments are read with coherent loads, for a kernel
// that itself wrote them earlier (the persistent sweep); otherwise through the
// read-only path
template <typename R, bool COH = false>
__device__ __forceinline__ void sweep_rhs0(const KArgs<R> &A, int c, const int *off, const int2 *list, double *rhs0) {
    R qc[REC];
    ld8(A.qs + (size_t)c * REC, qc);
    const int kb = off[c], ke = off[c + 1];
    int2 e2n = kb < ke ? __ldg(&list[kb]) : make_int2(0, 0);   // list entry one face ahead
    for (int k = kb; k < ke; ++k) {
        int2 e2 = e2n;
        if (k + 1 < ke) e2n = __ldg(&list[k + 1]);
        int f = nb_face(e2), nb = e2.y;
        R qn[REC], fg[FGR], dqj[DQR];
        ld8(A.qs + (size_t)nb * REC, qn);
        ld8(A.fgeo + (size_t)f * FGR, fg);
        // the neighbour's increment was written by an earlier level (an earlier
        // launch, or an earlier pass of the persistent sweep)
        if constexpr (COH) ldp8(A.dq + (size_t)nb * DQR, dqj);
        else ld8(A.dq + (size_t)nb * DQR, dqj);
        R volb = A.P.visSRModel == 1 ? A.cgeo[(size_t)nb * CGR + 3] : R(1);
        R xn = fg[0], yn = fg[1], zn = fg[2];
        if (nb_right(e2)) { xn = -xn; yn = -yn; zn = -zn; }   // GCom::SetGeometry
        face_increment(A.P, qc, qn, dqj, xn, yn, zn, fg[3], fg[7], volb, rhs0);
    }
}

template <typename R, bool COH>
__device__ __forceinline__ void lusgs_lower_cell(const KArgs<R> &A, int c) {
    double rhs0[NEQ] = {0.0, 0.0, 0.0, 0.0, 0.0};
    sweep_rhs0<R, COH>(A, c, A.lo_off, A.lol, rhs0);
    double rad = A.rad[c];
    const double *rs = A.res + (size_t)c * NEQ;
    R o[DQR];
#pragma unroll
    for (int e = 0; e < NEQ; ++e) o[e] = R((rs[e] - rhs0[e]) / rad);
    o[5] = o[6] = o[7] = R(0);
    st4(A.dq + (size_t)c * DQR, o);
    st4(A.dq + (size_t)c * DQR + 4, o + 4);
}

template <typename R, bool COH>
__device__ __forceinline__ void lusgs_upper_cell(const KArgs<R> &A, int c) {
    double rhs0[NEQ] = {0.0, 0.0, 0.0, 0.0, 0.0};
    sweep_rhs0<R, COH>(A, c, A.up_off, A.upl, rhs0);   // ghost increments are zero: boundary faces not listed
    double rad = A.rad[c];
    R o[DQR];
    ldp8(A.dq + (size_t)c * DQR, o);   // its own lower-sweep increment, rewritten below
#pragma unroll
    for (int e = 0; e < NEQ; ++e) o[e] = R(add_neg_quot(double(o[e]), rhs0[e], rad));
    st4(A.dq + (size_t)c * DQR, o);
    st4(A.dq + (size_t)c * DQR + 4, o + 4);
}

// one level of a sweep per launch (cells order[start .. start+count))
template <typename R, int MINB = MinBlocks<R>::sw>
__global__ void __launch_bounds__(128, MINB) k_lusgs_lower(KArgs<R> A, const int *order, int start, int count) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < count) lusgs_lower_cell<R, false>(A, order[start + t]);
}

template <typename R, int MINB = MinBlocks<R>::sw>
__global__ void __launch_bounds__(128, MINB) k_lusgs_upper(KArgs<R> A, const int *order, int start, int count) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < count) lusgs_upper_cell<R, false>(A, order[start + t]);
}

// The persistent form: one block of kSeqThreads runs every level of the sweep
// in order, with a block barrier between levels (a barrier also orders the
// block's global writes before its later reads, so each level sees the
// increments of the levels before it).  The same per-cell arithmetic as the
// level launches, so the same bits; it replaces nlev launches by one, which
// pays off when the levels are many and small (natural-order sweeps of
// structured-like meshes: hundreds of levels of tens to hundreds of cells).
template <typename R>
__global__ void __launch_bounds__(kSeqThreads, 1) k_lusgs_lower_seq(KArgs<R> A, const int *order, const int *loff,
                                                                 int nlev) {
    for (int l = 0; l < nlev; ++l) {
        const int st = loff[l], en = loff[l + 1];
        for (int k = st + threadIdx.x; k < en; k += blockDim.x) lusgs_lower_cell<R, true>(A, order[k]);
        __syncthreads();
    }
}

template <typename R>
__global__ void __launch_bounds__(kSeqThreads, 1) k_lusgs_upper_seq(KArgs<R> A, const int *order, const int *loff,
                                                                 int nlev) {
    for (int l = 0; l < nlev; ++l) {
        const int st = loff[l], en = loff[l + 1];
        for (int k = st + threadIdx.x; k < en; k += blockDim.x) lusgs_upper_cell<R, true>(A, order[k]);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// CALC_LHS of the multi-stage scheme: ULhs::CalcLHS (codes/usolver/src/ULhs.cpp:47-65),
// res *= (dt / vol) * lhscoef in place.  Under MULTI_STAGE the update's
// increment field is the residual itself (UNsField::Init,
// codes/uns/src/UNsCom.cpp:85-88), so the scaled values also go to the
// increment records UPDATE_FLOWFIELD adds; and the residual history of the
// iteration is the norm of this scaled residual (ResidualTask::CalcRes reads
// the residual field after the last stage), so the per-block sums of squares
// are written again here.
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(128) k_calc_lhs(KArgs<R> A, double coef) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    double sq[NEQ] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (c < A.nCells) {
        double f = (A.dt[c] / double(A.cgeo[(size_t)c * CGR + 3])) * coef;
        double *r = A.res + (size_t)c * NEQ;
        R d[DQR];
#pragma unroll
        for (int e = 0; e < NEQ; ++e) {
            double v = r[e] * f;
            r[e] = v;
            sq[e] = v * v;
            d[e] = R(v);
        }
#pragma unroll
        for (int e = NEQ; e < DQR; ++e) d[e] = R(0);
        st4(A.dq + (size_t)c * DQR, d);
        st4(A.dq + (size_t)c * DQR + 4, d + 4);
    }
    block_sum_to<NEQ>(sq, A.npart + (size_t)blockIdx.x * NEQ);
}

// ---------------------------------------------------------------------------
// UPDATE_FLOWFIELD_LUSGS: NsUpdate::CalcFlowField + WeekSolutionFix
// (codes/ns/src/NsUpdate.cpp:40-67,192-217), QToPrim (codes/ns/src/NsInvFlux.cpp:1377-1399);
// then the interior half of CALC_BOUNDARY: NsCalcGamaT + CalcLaminarViscosity.
// Writes the next state buffer (and its FP32 copy); cells that still fail go
// to a list for the neighbour-average fix (UNsUpdate::SolutionFix).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double sutherland(const DevParams &P, double t) {
    // codes/model/src/Sutherland.cpp:62-66
    double t3 = t * t * t;
    return sqrt(t3) * (1 + P.sutherland_ts) / (t + P.sutherland_ts);
}

template <typename R>
__device__ __forceinline__ void store_state(const KArgs<R> &A, int i, const double *rec) {
    double *o = A.qn + (size_t)i * REC;
    st4(o, rec);
    st4(o + 4, rec + 4);
    if (sizeof(R) == 4) {
        R s[REC];
#pragma unroll
        for (int e = 0; e < REC; ++e) s[e] = R(rec[e]);
        st4(A.qsn + (size_t)i * REC, s);
        st4(A.qsn + (size_t)i * REC + 4, s + 4);
    }
}

// state transfer between the reference's field layout q[5][nCells+nBFaces]
// (staged in device memory) and the records of the current buffer
template <typename R>
__global__ void __launch_bounds__(256) k_pack_state(KArgs<R> A, const double *stage) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.nT) return;
    double *o = A.qn + (size_t)i * REC;
#pragma unroll
    for (int e = 0; e < NEQ; ++e) o[e] = stage[(size_t)e * A.nT + i];
}

template <typename R>
__global__ void __launch_bounds__(256) k_unpack_state(KArgs<R> A, double *stage) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.nT) return;
    const double *o = A.q + (size_t)i * REC;
#pragma unroll
    for (int e = 0; e < NEQ; ++e) stage[(size_t)e * A.nT + i] = o[e];
}

// NsCalcGamaT(F_INNER) + CalcLaminarViscosity(F_INNER) on the current buffer
// (after a state upload or the initial field); refreshes the FP32 copy too
template <typename R>
__global__ void __launch_bounds__(256) k_interior_tvisl(KArgs<R> A) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= A.nCells) return;
    const double *qc = A.q + (size_t)c * REC;
    double rec[REC];
#pragma unroll
    for (int e = 0; e < REC; ++e) rec[e] = qc[e];
    double t = rec[IP] / (A.P.statecoef * rec[IR] * 1.0);
    rec[ITT] = t;
    rec[IML] = fmax(0.0, sutherland(A.P, t));
    store_state(A, c, rec);
}

template <typename R>
__device__ __forceinline__ void update_cell(const KArgs<R> &A, int c, const double *dd) {
    const double *qc = A.q + (size_t)c * REC;
    double gama = A.P.gama;
    double prim0[NEQ], q0[NEQ], qq[NEQ], pr[NEQ];
#pragma unroll
    for (int e = 0; e < NEQ; ++e) prim0[e] = qc[e];
    primToQ(prim0, gama, q0);
#pragma unroll
    for (int e = 0; e < NEQ; ++e) qq[e] = q0[e] + dd[e];
    double density = fabs(qq[0]);
    double rd = 1.0 / density;
    double um = qq[1] * rd, vm = qq[2] * rd, wm = qq[3] * rd, rem = qq[4];
    double v2 = SQR3(um, vm, wm);
    double reint = rem - 0.5 * density * v2;
    pr[0] = density; pr[1] = um; pr[2] = vm; pr[3] = wm; pr[4] = (gama - 1.0) * reint;
    bool needFix = false;
    if (pr[IR] <= 0.0 || pr[IP] <= 0.0) {
        bool ok = false;
        const double coefs[3] = {0.5, 0.1, 0.01};
        for (int k = 0; k < 3 && !ok; ++k) {
#pragma unroll
            for (int e = 0; e < NEQ; ++e) pr[e] += coefs[k] * dd[e];
            if (!(pr[IR] < 0.0 || pr[IP] < 0.0)) ok = true;
        }
        if (!ok) {
            needFix = true;
            int slot = atomicAdd(A.fixlist, 1);
            if (slot < A.fixcap) A.fixlist[1 + slot] = c;
        }
    }
    double rec[REC];
#pragma unroll
    for (int e = 0; e < NEQ; ++e) rec[e] = pr[e];
    rec[ITT] = 0.0; rec[IML] = 0.0;
    if (!needFix) {
        double t = pr[IP] / (A.P.statecoef * pr[IR] * 1.0);
        rec[ITT] = t;
        rec[IML] = fmax(0.0, sutherland(A.P, t));
    }
    rec[IMT] = qc[IMT];
    store_state(A, c, rec);
}

template <typename R>
__global__ void __launch_bounds__(256) k_update(KArgs<R> A) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= A.nCells) return;
    R d[DQR];
    ld8(A.dq + (size_t)c * DQR, d);
    double dd[NEQ];
#pragma unroll
    for (int e = 0; e < NEQ; ++e) dd[e] = double(d[e]);
    update_cell(A, c, dd);
}

// UNsUpdate::SolutionFix (codes/uns/src/UNsUpdate.cpp:94-133) for the cells
// that failed every positivity retry.  The reference updates in place in its
// sweep order, so a neighbour earlier in that order contributes its new value
// and a later one its old value; one thread replays that order.
template <typename R>
__global__ void k_solution_fix(KArgs<R> A) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    int n = A.fixlist[0];
    if (n <= 0) return;
    if (n > A.fixcap) n = A.fixcap;
    int *ids = A.fixlist + 1;
    for (int i = 1; i < n; ++i) {   // insertion sort by sweep position (the list is short)
        int v = ids[i], j = i - 1;
        while (j >= 0 && A.key[ids[j]] > A.key[v]) { ids[j + 1] = ids[j]; --j; }
        ids[j + 1] = v;
    }
    for (int i = 0; i < n; ++i) {
        int c = ids[i];
        double pr[NEQ] = {0, 0, 0, 0, 0}, sumV = 0.0;
        for (int k = A.nb_off[c]; k < A.nb_off[c + 1]; ++k) {
            int nb = A.nbl[k].y;
            bool done = nb < A.nCells && A.key[nb] < A.key[c];
            const double *src = done ? A.qn + (size_t)nb * REC : A.q + (size_t)nb * REC;
            sumV += 1.0;
            for (int e = 0; e < NEQ; ++e) {
                double v = src[e];
                if (e == IR || e == IP) v = fabs(v);
                pr[e] += v * 1.0;
            }
        }
        double rv = 1.0 / sumV;
        double rec[REC];
        for (int e = 0; e < NEQ; ++e) rec[e] = pr[e] * rv;
        double t = rec[IP] / (A.P.statecoef * rec[IR] * 1.0);
        rec[ITT] = t;
        rec[IML] = fmax(0.0, sutherland(A.P, t));
        rec[IMT] = A.q[(size_t)c * REC + IMT];
        store_state(A, c, rec);
    }
    A.fixlist[0] = 0;
}

// ---------------------------------------------------------------------------
// CALC_BOUNDARY, ghost half: UNsBcSolver::CalcBc (codes/uns/src/UNsBcSolver.cpp:55-166)
// with NsBcSolver's face BCs (codes/ns/src/NsBcSolver.cpp:51-440), then
// NsCalcGamaT + CalcLaminarViscosity on the ghost cells.  Operates on qn
// (interior cells already final), ghost records written to qn.
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(256) k_boundary(KArgs<R> A, const int *lcb) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= A.nBFaces) return;
    int bt = A.bcType[f];
    int l = lcb[f];
    const double *s = A.qn + (size_t)l * REC;
    int g = A.nCells + f;
    double t[NEQ], pr[NEQ];
    bool havePrim = false;
    const double *fg = A.fgeoD + (size_t)f * FGR;   // FP64 normal on both paths
    double xn = fg[0], yn = fg[1], zn = fg[2], vfn = 0.0;
    double gama = A.P.gama;
    if (bt == BC_SYM || (bt == BC_SOLID && A.P.vismodel == 0)) {
        double vn = xn * s[IU] + yn * s[IV] + zn * s[IW] - vfn;
#pragma unroll
        for (int e = 0; e < NEQ; ++e) t[e] = s[e];
        t[IU] = s[IU] - 2.0 * xn * vn;
        t[IV] = s[IV] - 2.0 * yn * vn;
        t[IW] = s[IW] - 2.0 * zn * vn;
#pragma unroll
        for (int e = 0; e < NEQ; ++e) pr[e] = 0.5 * (s[e] + t[e]);
        havePrim = true;
    } else if (bt == BC_SOLID && A.P.isowallbc == 0) {
#pragma unroll
        for (int e = 0; e < NEQ; ++e) t[e] = s[e];
        t[IU] = -t[IU] + 2.0 * 0.0;
        t[IV] = -t[IV] + 2.0 * 0.0;
        t[IW] = -t[IW] + 2.0 * 0.0;
        pr[IR] = s[IR]; pr[IU] = 0.0; pr[IV] = 0.0; pr[IW] = 0.0; pr[IP] = s[IP];
        havePrim = true;
    } else if (bt == BC_SOLID) {
#pragma unroll
        for (int e = 0; e < NEQ; ++e) t[e] = s[e];
        t[IU] = -t[IU] + 2.0 * 0.0; t[IV] = -t[IV] + 2.0 * 0.0; t[IW] = -t[IW] + 2.0 * 0.0;
        double twall = A.P.twall, tlim = 0.1 * twall;
        double rm = s[IR], pm = s[IP], temperature = s[ITT];
        double rw_face = pm / (A.P.statecoef * twall * 1.0);
        pr[IR] = rw_face; pr[IU] = 0; pr[IV] = 0; pr[IW] = 0; pr[IP] = pm;
        double pg1 = pm, tg1 = 2.0 * twall - temperature;
        if (tg1 < tlim) tg1 = tlim;
        double rw = pg1 / (A.P.statecoef * twall * 1.0);
        double rg1 = 2.0 * rw - rm;
        rg1 = fmax(0.5 * rw, rg1);
        t[IR] = rg1; t[IP] = pg1;
        havePrim = true;
    } else if (bt == BC_FAR) {
        const double *inf = A.P.inflow;
#pragma unroll
        for (int e = 0; e < NEQ; ++e) t[e] = s[e];
        double rin = s[IR], uin = s[IU], vin = s[IV], win = s[IW], pin = s[IP];
        double rref = inf[IR], uref = inf[IU], vref = inf[IV], wref = inf[IW], pref = inf[IP];
        double vnref = xn * uref + yn * vref + zn * wref - vfn;
        double vnin = xn * uin + yn * vin + zn * win - vfn;
        double cref = sqrt(fabs(gama * pref / rref));
        double cin = sqrt(fabs(gama * pin / rin));
        double gamm1 = gama - 1.0;
        double velin = sqrt(SQR3(uin, vin, win));
        if (velin > cin) {
            if (vnin >= 0.0) {
#pragma unroll
                for (int e = 0; e < NEQ; ++e) t[e] = s[e];
            } else {
#pragma unroll
                for (int e = 0; e < NEQ; ++e) t[e] = inf[e];
            }
        } else {
            double riemp = vnin + 2.0 * cin / gamm1;
            double riemm = vnref - 2.0 * cref / gamm1;
            double vnb = 0.5 * (riemp + riemm);
            double cb = 0.25 * (riemp - riemm) * gamm1;
            double vtx, vty, vtz, entr;
            if (vnb >= 0.0) {
                entr = pin / pow(rin, gama);
                vtx = uin - xn * vnin; vty = vin - yn * vnin; vtz = win - zn * vnin;
            } else {
                entr = pref / pow(rref, gama);
                vtx = uref - xn * vnref; vty = vref - yn * vnref; vtz = wref - zn * vnref;
            }
            double rb = pow((cb * cb / (entr * gama)), 1.0 / gamm1);
            t[IR] = rb;
            t[IU] = vtx + xn * vnb; t[IV] = vty + yn * vnb; t[IW] = vtz + zn * vnb;
            t[IP] = cb * cb * rb / gama;
        }
    } else if (bt == BC_INFLOW) {
#pragma unroll
        for (int e = 0; e < NEQ; ++e) t[e] = A.P.inflow[e];
    } else {
#pragma unroll
        for (int e = 0; e < NEQ; ++e) t[e] = s[e];
    }
    double rec[REC];
#pragma unroll
    for (int e = 0; e < NEQ; ++e) rec[e] = t[e];
    double tt = t[IP] / (A.P.statecoef * t[IR] * 1.0);
    rec[ITT] = tt;
    rec[IML] = fmax(0.0, sutherland(A.P, tt));
    rec[IMT] = A.q[(size_t)g * REC + IMT];   // ghost eddy viscosity is set by the SA solver
    store_state(A, g, rec);
    if (havePrim) {
        double *b = A.bcq + (size_t)f * NEQ;
#pragma unroll
        for (int e = 0; e < NEQ; ++e) b[e] = pr[e];
    }
}

// ---------------------------------------------------------------------------
// Residual norms: ResidualTask::CalcRes + ResAver::CalcAver
// (codes/residual/src/ResidualTask.cpp:75-126, codes/residual/src/Residual.cpp:52-72).
// Aerodynamic forces: CalcAeroForce (codes/force/src/AeroForceTask.cpp:186-451,
// the compressible branch) over the solid-wall faces.  Wall geometry comes in
// FP64 from the host (wg[w][16]: n*area, n, area, face centre - cell centre,
// unit cell-to-ghost vector, 1/distance), so both paths integrate with the
// reference's geometry; the gradients are the last residual pass's records.
// Sums in a fixed order; out[9] = total, pressure, viscous force.
template <typename R>
__global__ void __launch_bounds__(256) k_forces(KArgs<R> A, const int2 *wall, const double *wg, int nWall,
                                                double *out) {
    double acc[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) acc[k] = 0.0;
    const DevParams &P = A.P;
    for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < nWall; w += gridDim.x * blockDim.x) {
        int f = wall[w].x, l = wall[w].y, r = A.nCells + f;
        const double *g = wg + (size_t)w * 16;
        const double *ql = A.q + (size_t)l * REC, *qr = A.q + (size_t)r * REC;
        const R *gr = A.gl + (size_t)l * GLR;
        double wp = ql[IP] + double(gr[IP * 3]) * g[7] + double(gr[IP * 3 + 1]) * g[8] + double(gr[IP * 3 + 2]) * g[9];
        if (wp < 0.0) wp = ql[IP];
        double cp = 2.0 * (wp - P.inflow[IP]);
        double fp[3] = {g[0] * cp, g[1] * cp, g[2] * cp};
        double fv[3] = {0.0, 0.0, 0.0};
        if (P.vismodel > 0) {
            double d[3][3];   // [u v w][x y z]
#pragma unroll
            for (int e = 0; e < 3; ++e)
#pragma unroll
                for (int k = 0; k < 3; ++k) d[e][k] = double(gr[(IU + e) * 3 + k]);
            double dx = g[10], dy = g[11], dz = g[12], ods = g[13];
#pragma unroll
            for (int e = 0; e < 3; ++e) {   // CorrectGrad, codes/usolver/src/VisGrad.cpp:355-365
                double fOld = d[e][0] * dx + d[e][1] * dy + d[e][2] * dz;
                double fnew = (qr[IU + e] - ql[IU + e]) * ods;
                double df = fnew - fOld;
                d[e][0] += df * dx; d[e][1] += df * dy; d[e][2] += df * dz;
            }
            double vis = ql[IML];   // Stress::CalcForce, codes/solver/src/Stress.cpp:40-64
            double divv2p3 = (2.0 / 3.0) * (d[0][0] + d[1][1] + d[2][2]);
            double txx = vis * (2.0 * d[0][0] - divv2p3);
            double tyy = vis * (2.0 * d[1][1] - divv2p3);
            double tzz = vis * (2.0 * d[2][2] - divv2p3);
            double txy = vis * (d[0][1] + d[1][0]);
            double txz = vis * (d[0][2] + d[2][0]);
            double tyz = vis * (d[1][2] + d[2][1]);
            double coef = -2.0 * g[6] * P.oreynolds;
            fv[0] = coef * (g[3] * txx + g[4] * txy + g[5] * txz);
            fv[1] = coef * (g[3] * txy + g[4] * tyy + g[5] * tyz);
            fv[2] = coef * (g[3] * txz + g[4] * tyz + g[5] * tzz);
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            acc[k] += fp[k] + fv[k];
            acc[3 + k] += fp[k];
            acc[6 + k] += fv[k];
        }
    }
    // per-thread sums -> one record per thread for the grid reduction
    __shared__ double tot[9];
    __shared__ bool last;
    block_sum_to<9>(acc, tot);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < 9; ++k) A.red[(size_t)blockIdx.x * 9 + k] = tot[k];
        __threadfence();
        last = atomicAdd(A.redCount, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    for (int k = 0; k < 9; ++k) {
        double s = 0.0;
        for (unsigned int b = 0; b < gridDim.x; ++b) s += __ldcg(A.red + (size_t)b * 9 + k);
        out[k] = s;
    }
    *A.redCount = 0u;
}

// The residual kernel leaves per-block sums of squares; they are added in a
// fixed order (FP64, deterministic run to run) by a grid of blocks whose last
// block to finish produces the norms.
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(256) k_norm_final(KArgs<R> A, int nPartial) {
    __shared__ double tot[NEQ];
    if (grid_sum_last<NEQ>(A.npart, nPartial, A.red, A.redCount, tot) && threadIdx.x == 0)
        for (int e = 0; e < NEQ; ++e) A.scal[S_NORM + e] = sqrt(tot[e] / A.nCells);
}

}  // namespace ofg

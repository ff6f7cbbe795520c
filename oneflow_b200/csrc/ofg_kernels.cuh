// Kernels of the NS residual + LU-SGS iteration (templated on the face
// arithmetic type R).  Every kernel is a cell-centred gather over the CSR
// cell->face list in ascending face id, which is the order in which the
// reference's serial face loops scatter into a cell, so the FP64
// accumulations round exactly as the reference's do and no atomics are used.
#pragma once
#include "ofg_device.cuh"

namespace ofg {

// Kernel arguments shared by all kernels of one context.
template <typename R>
struct KArgs {
    DevParams P;
    DevMesh M;
    DevGeom<R> G;
    const double *q;      // current state records [nT][REC]
    double *qn;           // next state records    [nT][REC]
    double *res;          // [nCells][NEQ]
    double *dq;           // [nT][NEQ]
    double *dt, *invsr, *vissr;   // [nCells]
    double *bcq;          // [nBFaces][NEQ]
    R *grad;              // [nCells][18]: (var*3 + dir), var 0-4 = q, 5 = T
    R *lim;               // [nCells][NEQ]
    double *partial;      // per-block partials
    double *scal;         // small device scalars (cfl, eps, min dt, norms)
    int *fixlist;         // [1 + cap]: count, cell ids
    int fixcap;
    // Spalart-Allmaras solver
    double *nut;          // [nT] nu~ (ghosts at nCells + f)
    double *dnut;         // [nT]
    double *resT;         // [nCells]
    double *impsrT;       // [nCells]
    double *matL, *matR;  // [nFaces] sweep coefficients
    R *gnut;              // [nCells][3]
};


__device__ __forceinline__ int other_cell(int l, int r, int c) { return l == c ? r : l; }

// ---------------------------------------------------------------------------
// CALC_TIME_STEP: UTimeStep::CalcTimeStep, codes/uns/src/UTimeStep.cpp:190-416,
// face radii TimeStep::CalcFaceInvSpec/CalcFaceVisSpec, codes/ns/src/TimeStep.cpp:61-122
// ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ double face_inv_spec(const KArgs<R> &A, int f) {
    int l = A.M.lc[f], r = A.M.rc[f];
    const double *ql = A.q + (size_t)l * REC, *qr = A.q + (size_t)r * REC;
    R xn = A.G.xfn[f], yn = A.G.yfn[f], zn = A.G.zfn[f], ar = A.G.area[f];
    R gama = R(A.P.gama);
    R rl = R(ql[IR]), ul = R(ql[IU]), vl = R(ql[IV]), wl = R(ql[IW]), pl = R(ql[IP]);
    R rr = R(qr[IR]), ur = R(qr[IU]), vr = R(qr[IV]), wr = R(qr[IW]), pr = R(qr[IP]);
    R vnl = xn * ul + yn * vl + zn * wl - R(0);
    R vnr = xn * ur + yn * vr + zn * wr - R(0);
    R g = R(0.5) * (gama + gama);
    R pm = R(0.5) * (pl + pr), rm = R(0.5) * (rl + rr);
    R cm = Rsqrt(g * pm / rm);
    R vn = R(0.5) * (vnl + vnr);
    return double(R(0.5) * ar * (Rabs(vn) + cm));
}

template <typename R>
__device__ __forceinline__ double face_vis_spec(const KArgs<R> &A, int f) {
    int l = A.M.lc[f], r = A.M.rc[f];
    const double *ql = A.q + (size_t)l * REC, *qr = A.q + (size_t)r * REC;
    R ar = A.G.area[f];
    R vl = R(0.5) * (R(ql[IML]) + R(qr[IML]));
    R vt = R(0.5) * (R(ql[IMT]) + R(qr[IMT]));
    R density = R(0.5) * (R(ql[IR]) + R(qr[IR]));
    if (A.P.visSRModel == 1) {
        R c1 = R(4.0) / R(3.0) * (vl + vt);
        R c2 = R(A.P.gama) * (vl * R(A.P.oprl) + vt * R(A.P.oprt));
        R c3 = R(2.0) * Rmax(c1, c2) / (R(A.P.reynolds) * density);
        return double(ar * ar * c3);
    } else if (A.P.visSRModel == 2) {
        R dist = Rabs(A.G.xfn[f] * (A.G.xcc[r] - A.G.xcc[l]) + A.G.yfn[f] * (A.G.ycc[r] - A.G.ycc[l]) +
                      A.G.zfn[f] * (A.G.zcc[r] - A.G.zcc[l]));
        R viscosity = vl + vt;
        R c1 = R(2.0) * viscosity / (density * dist * R(A.P.reynolds) + small_v<R>());
        return double(R(0.5) * c1 * ar);
    } else if (A.P.visSRModel == 3) {
        return double(ar * ar / (R(A.P.reynolds) * density + small_v<R>()));
    }
    return 0.0;
}

template <typename R>
__global__ void __launch_bounds__(256) k_timestep(KArgs<R> A) {
    __shared__ double smin[256];
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    double mydt = 1.0e40;
    if (c < A.M.nCells) {
        double cfl = A.scal[S_CFL];
        int b = A.M.c2f_off[c], e = A.M.c2f_off[c + 1];
        double inv = 0.0;
        for (int k = b; k < e; ++k) inv += face_inv_spec(A, A.M.c2f[k]);
        double vis = 0.0;
        if (A.P.vismodel > 0)
            for (int k = b; k < e; ++k) vis += face_vis_spec(A, A.M.c2f[k]);
        double vol = double(A.G.vol[c]);
        double ts;
        if (A.P.timestepModel == 1) {
            ts = A.P.global_dt;
        } else {
            ts = cfl * vol / inv;
            if (A.P.vismodel > 0 && A.P.visTimeStepModel > 0) {
                double vts = cfl * vol / vis;
                ts *= vts / (ts + vts);
            }
        }
        A.invsr[c] = inv;
        A.vissr[c] = vis;
        A.dt[c] = ts;
        mydt = ts;
    }
    smin[threadIdx.x] = mydt;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) smin[threadIdx.x] = fmin(smin[threadIdx.x], smin[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) A.partial[blockIdx.x] = smin[0];
}

// UTimeStep::CalcMinTimeStep: zone-wide minimum of the local steps (single
// block over the per-block partials; min is exact in any order)
template <typename R>
__global__ void __launch_bounds__(256) k_timestep_min(KArgs<R> A, int nPartial) {
    __shared__ double smin[256];
    double m = 1.0e40;
    for (int i = threadIdx.x; i < nPartial; i += blockDim.x) m = fmin(m, A.partial[i]);
    smin[threadIdx.x] = m;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) smin[threadIdx.x] = fmin(smin[threadIdx.x], smin[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) A.scal[S_MINDT] = smin[0];
}

// UTimeStep::ModifyTimeStep / CalcLgTimeStep
template <typename R>
__global__ void __launch_bounds__(256) k_timestep_clip(KArgs<R> A) {
    if (A.P.timestepModel == 1) return;
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= A.M.nCells) return;
    double mn = A.scal[S_MINDT];
    if (A.P.timestepModel == 2) { A.dt[c] = mn; return; }
    if (A.P.max_time_ratio > 0) A.dt[c] = fmin(A.dt[c], A.P.max_time_ratio * mn);
}

// ---------------------------------------------------------------------------
// Gradients: CalcGradGGCellWeight (codes/usolver/src/UGrad.cpp:88-149) or the
// face-average Green-Gauss (:40-86); weighted least squares is new.
// var 0-4: q (rho,u,v,w,p), var 5: temperature (UTGrad, codes/uns/src/UNsGrad.cpp:81-101)
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(128) k_gradient(KArgs<R> A, int nvar) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= A.M.nCells) return;
    R gx[6], gy[6], gz[6];
#pragma unroll
    for (int v = 0; v < 6; ++v) gx[v] = gy[v] = gz[v] = R(0);
    int b = A.M.c2f_off[c], e = A.M.c2f_off[c + 1];
    if (A.P.igrad == 2) {
        // weighted least squares over face neighbours (ghosts included), w = 1/|d|^2
        R a11 = 0, a12 = 0, a13 = 0, a22 = 0, a23 = 0, a33 = 0, bb[6][3];
#pragma unroll
        for (int v = 0; v < 6; ++v) bb[v][0] = bb[v][1] = bb[v][2] = R(0);
        const double *qc = A.q + (size_t)c * REC;
        for (int k = b; k < e; ++k) {
            int f = A.M.c2f[k];
            int nb = other_cell(A.M.lc[f], A.M.rc[f], c);
            R dx = A.G.xcc[nb] - A.G.xcc[c], dy = A.G.ycc[nb] - A.G.ycc[c], dz = A.G.zcc[nb] - A.G.zcc[c];
            R w = R(1) / (dx * dx + dy * dy + dz * dz);
            a11 += w * dx * dx; a12 += w * dx * dy; a13 += w * dx * dz;
            a22 += w * dy * dy; a23 += w * dy * dz; a33 += w * dz * dz;
            const double *qn = A.q + (size_t)nb * REC;
            for (int v = 0; v < nvar; ++v) {
                int iv = v < 5 ? v : ITT;
                R dv = R(qn[iv]) - R(qc[iv]);
                bb[v][0] += w * dx * dv; bb[v][1] += w * dy * dv; bb[v][2] += w * dz * dv;
            }
        }
        if (A.P.dim == 2) {
            R id = R(1) / (a11 * a22 - a12 * a12);
            for (int v = 0; v < nvar; ++v) {
                gx[v] = (a22 * bb[v][0] - a12 * bb[v][1]) * id;
                gy[v] = (a11 * bb[v][1] - a12 * bb[v][0]) * id;
                gz[v] = R(0);
            }
        } else {
            R c11 = a22 * a33 - a23 * a23, c12 = a13 * a23 - a12 * a33, c13 = a12 * a23 - a13 * a22;
            R c22 = a11 * a33 - a13 * a13, c23 = a12 * a13 - a11 * a23, c33 = a11 * a22 - a12 * a12;
            R id = R(1) / (a11 * c11 + a12 * c12 + a13 * c13);
            for (int v = 0; v < nvar; ++v) {
                gx[v] = (c11 * bb[v][0] + c12 * bb[v][1] + c13 * bb[v][2]) * id;
                gy[v] = (c12 * bb[v][0] + c22 * bb[v][1] + c23 * bb[v][2]) * id;
                gz[v] = (c13 * bb[v][0] + c23 * bb[v][1] + c33 * bb[v][2]) * id;
            }
        }
    } else {
        for (int k = b; k < e; ++k) {
            int f = A.M.c2f[k];
            int l = A.M.lc[f], r = A.M.rc[f];
            R cl, cr;
            if (A.P.igrad == 1) {
                cl = R(0.5); cr = R(0.5);
            } else {
                R dxl = A.G.xfc[f] - A.G.xcc[l], dyl = A.G.yfc[f] - A.G.ycc[l], dzl = A.G.zfc[f] - A.G.zcc[l];
                R dxr = A.G.xfc[f] - A.G.xcc[r], dyr = A.G.yfc[f] - A.G.ycc[r], dzr = A.G.zfc[f] - A.G.zcc[r];
                R delt1 = Rsqrt(SQR3(dxl, dyl, dzl)), delt2 = Rsqrt(SQR3(dxr, dyr, dzr));
                R delta = R(1) / (delt1 + delt2 + small_v<R>());
                cl = delt2 * delta; cr = delt1 * delta;
            }
            R ar = A.G.area[f];
            R fnxa = A.G.xfn[f] * ar, fnya = A.G.yfn[f] * ar, fnza = A.G.zfn[f] * ar;
            const double *ql = A.q + (size_t)l * REC, *qr = A.q + (size_t)r * REC;
            bool left = (l == c);
            for (int v = 0; v < nvar; ++v) {
                int iv = v < 5 ? v : ITT;
                R value = (A.P.igrad == 1) ? R(0.5) * (R(ql[iv]) + R(qr[iv])) : cl * R(ql[iv]) + cr * R(qr[iv]);
                if (left) { gx[v] += fnxa * value; gy[v] += fnya * value; gz[v] += fnza * value; }
                else      { gx[v] -= fnxa * value; gy[v] -= fnya * value; gz[v] -= fnza * value; }
            }
        }
        R ovol = R(1) / A.G.vol[c];
        for (int v = 0; v < nvar; ++v) { gx[v] *= ovol; gy[v] *= ovol; gz[v] *= ovol; }
    }
    R *g = A.grad + (size_t)c * 18;
    for (int v = 0; v < nvar; ++v) { g[v * 3 + 0] = gx[v]; g[v * 3 + 1] = gy[v]; g[v * 3 + 2] = gz[v]; }
}

// gradient of a (possibly ghost) cell: ghosts carry their interior cell's
// gradient (UGrad.cpp:140-148)
__device__ __forceinline__ int grad_cell(const DevMesh &M, int c) {
    return c < M.nCells ? c : M.lc[c - M.nCells];
}

// ---------------------------------------------------------------------------
// Limiter: Limiter::CalcMinMaxDiff + CalcBarthLimiter/CalcVencatLimiter,
// codes/usolver/src/ULimiter.cpp:377-644.  Pass 1: neighbour min/max
// differences per cell and the zone-wide extremes (block partials).
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(256) k_limiter_minmax(KArgs<R> A, R *mm /* [nCells][10] */) {
    __shared__ double smn[NEQ][256], smx[NEQ][256];
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    double lmin[NEQ], lmax[NEQ];
#pragma unroll
    for (int e = 0; e < NEQ; ++e) { lmin[e] = 1.0e40; lmax[e] = -1.0e40; }
    if (c < A.M.nCells) {
        const double *qc = A.q + (size_t)c * REC;
        R mn[NEQ], mx[NEQ];
#pragma unroll
        for (int e = 0; e < NEQ; ++e) mn[e] = mx[e] = R(qc[e]);
        int b = A.M.c2f_off[c], en = A.M.c2f_off[c + 1];
        for (int k = b; k < en; ++k) {
            int f = A.M.c2f[k];
            if (f < A.M.nBFaces) continue;   // only interface boundaries count
            int nb = other_cell(A.M.lc[f], A.M.rc[f], c);
            const double *qn = A.q + (size_t)nb * REC;
#pragma unroll
            for (int e = 0; e < NEQ; ++e) { mn[e] = Rmin(mn[e], R(qn[e])); mx[e] = Rmax(mx[e], R(qn[e])); }
        }
        R *o = mm + (size_t)c * 10;
#pragma unroll
        for (int e = 0; e < NEQ; ++e) {
            mn[e] -= R(qc[e]); mx[e] -= R(qc[e]);
            o[e] = mn[e]; o[5 + e] = mx[e];
            lmin[e] = double(mn[e]); lmax[e] = double(mx[e]);
        }
    }
#pragma unroll
    for (int e = 0; e < NEQ; ++e) { smn[e][threadIdx.x] = lmin[e]; smx[e][threadIdx.x] = lmax[e]; }
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
#pragma unroll
            for (int e = 0; e < NEQ; ++e) {
                smn[e][threadIdx.x] = fmin(smn[e][threadIdx.x], smn[e][threadIdx.x + s]);
                smx[e][threadIdx.x] = fmax(smx[e][threadIdx.x], smx[e][threadIdx.x + s]);
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
#pragma unroll
        for (int e = 0; e < NEQ; ++e) {
            A.partial[(size_t)blockIdx.x * 10 + e] = smn[e][0];
            A.partial[(size_t)blockIdx.x * 10 + 5 + e] = smx[e][0];
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

// pass 2: per cell, min over its faces of the face limiter value on its side
template <typename R>
__global__ void __launch_bounds__(128) k_limiter(KArgs<R> A, const R *mm) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= A.M.nCells) return;
    R lim[NEQ];
#pragma unroll
    for (int e = 0; e < NEQ; ++e) lim[e] = R(1);
    const R *g = A.grad + (size_t)c * 18;
    const R *m = mm + (size_t)c * 10;
    R eps[NEQ];
    R epsc = R(0);
    if (A.P.venkat_kh3) {
        R h = A.P.dim == 2 ? Rsqrt(A.G.vol[c]) : R(cbrt(double(A.G.vol[c])));
        R k = R(A.P.vencat_coef) * h;
        epsc = k * k * k + small_v<R>();
    }
#pragma unroll
    for (int e = 0; e < NEQ; ++e) eps[e] = A.P.venkat_kh3 ? epsc : R(A.scal[S_EPS + e]);
    int b = A.M.c2f_off[c], en = A.M.c2f_off[c + 1];
    for (int k = b; k < en; ++k) {
        int f = A.M.c2f[k];
        R dx = A.G.xfc[f] - A.G.xcc[c], dy = A.G.yfc[f] - A.G.ycc[c], dz = A.G.zfc[f] - A.G.zcc[c];
        R dot = R(0);
        if (A.P.ilim == 1) {
            R ds = Rsqrt(SQR3(dx, dy, dz));
            R nd = A.G.xfn[f] * dx + A.G.yfn[f] * dy + A.G.zfn[f] * dz;
            dot = (A.M.lc[f] == c) ? nd / (ds + small_v<R>()) : -nd / (ds + small_v<R>());
        }
#pragma unroll
        for (int e = 0; e < NEQ; ++e) {
            R dqf = g[e * 3 + 0] * dx + g[e * 3 + 1] * dy + g[e * 3 + 2] * dz;
            R v = (A.P.ilim == 1) ? barth_fn(dqf, m[e], m[5 + e], dot) : venkat_fn(dqf, m[e], m[5 + e], eps[e]);
            lim[e] = Rmin(lim[e], v);
        }
    }
    R *o = A.lim + (size_t)c * NEQ;
#pragma unroll
    for (int e = 0; e < NEQ; ++e) o[e] = lim[e];
}

// ---------------------------------------------------------------------------
// UPDATE_RESIDUALS: UNsInvFlux::CalcFlux (codes/uns/src/UNsInvFlux.cpp:123-215)
// + UNsVisFlux::CalcFlux (codes/uns/src/UNsVisFlux.cpp:90-440), accumulated
// per cell in ascending face order (AddF2CField, codes/usolver/src/UCom.cpp:144-171).
// ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ void face_states(const KArgs<R> &A, int f, R *t1, R *t2) {
    int l = A.M.lc[f], r = A.M.rc[f];
    const double *ql = A.q + (size_t)l * REC, *qr = A.q + (size_t)r * REC;
    if (f < A.M.nBFaces) {
        // NsLimField::BcQlQrFix, codes/uns/src/UNsLimiter.cpp:67-101
        if (A.M.bcType[f] == BC_SOLID) {
            const double *b = A.bcq + (size_t)f * NEQ;
#pragma unroll
            for (int e = 0; e < NEQ; ++e) t1[e] = t2[e] = R(b[e]);
        } else {
#pragma unroll
            for (int e = 0; e < NEQ; ++e) t1[e] = t2[e] = R(0.5) * (R(ql[e]) + R(qr[e]));
        }
        return;
    }
#pragma unroll
    for (int e = 0; e < NEQ; ++e) { t1[e] = R(ql[e]); t2[e] = R(qr[e]); }
    if (A.P.ilim == -1) return;   // first order: the zero limiter keeps the cell values
    // LimField::CalcFaceValue, codes/usolver/src/ULimiter.cpp:188-256
    R u1[NEQ], u2[NEQ];
    const R *gl = A.grad + (size_t)l * 18, *gr = A.grad + (size_t)r * 18;
    const R *ll = A.lim + (size_t)l * NEQ, *lr = A.lim + (size_t)r * NEQ;
    R dx = A.G.xfc[f] - A.G.xcc[l], dy = A.G.yfc[f] - A.G.ycc[l], dz = A.G.zfc[f] - A.G.zcc[l];
#pragma unroll
    for (int e = 0; e < NEQ; ++e) {
        R phi = Rmin(ll[e], lr[e]);
        u1[e] = t1[e] + phi * (gl[e * 3] * dx + gl[e * 3 + 1] * dy + gl[e * 3 + 2] * dz);
    }
    dx = A.G.xfc[f] - A.G.xcc[r]; dy = A.G.yfc[f] - A.G.ycc[r]; dz = A.G.zfc[f] - A.G.zcc[r];
#pragma unroll
    for (int e = 0; e < NEQ; ++e) {
        R phi = Rmin(lr[e], ll[e]);
        u2[e] = t2[e] + phi * (gr[e * 3] * dx + gr[e * 3 + 1] * dy + gr[e * 3 + 2] * dz);
    }
    // NsCheckFunction, codes/ns/src/NsCom.cpp:133-137
    if (!(u1[IR] <= R(0) || u1[IP] <= R(0)))
#pragma unroll
        for (int e = 0; e < NEQ; ++e) t1[e] = u1[e];
    if (!(u2[IR] <= R(0) || u2[IP] <= R(0)))
#pragma unroll
        for (int e = 0; e < NEQ; ++e) t2[e] = u2[e];
}

// viscous face flux (VIS_STD face gradient), returns fv[NEQ] before the
// -S/Re factor; UNsVisFlux::PrepareFaceValue/StdMethod/CalcStress/CalcNsVisFlux
template <typename R>
__device__ __forceinline__ void face_vis_flux(const KArgs<R> &A, int f, R *fv) {
    int l = A.M.lc[f], r = A.M.rc[f];
    const double *ql = A.q + (size_t)l * REC, *qr = A.q + (size_t)r * REC;
    const R *gl = A.grad + (size_t)l * 18, *gr = A.grad + (size_t)grad_cell(A.M, r) * 18;
    R half = R(0.5);
    R vlm = half * (R(ql[IML]) + R(qr[IML])), vtm = half * (R(ql[IMT]) + R(qr[IMT]));
    R vis = vlm + vtm;
    R dx = A.G.xcc[r] - A.G.xcc[l], dy = A.G.ycc[r] - A.G.ycc[l], dz = A.G.zcc[r] - A.G.zcc[l];
    R ods = R(1) / Rsqrt(SQR3(dx, dy, dz));
    dx *= ods; dy *= ods; dz *= ods;
    R gx[6], gy[6], gz[6], qm[6];
#pragma unroll
    for (int v = 0; v < 6; ++v) {
        int iv = v < 5 ? v : ITT;
        R q1 = R(ql[iv]), q2 = R(qr[iv]);
        qm[v] = half * (q1 + q2);
        gx[v] = half * (gl[v * 3] + gr[v * 3]);
        gy[v] = half * (gl[v * 3 + 1] + gr[v * 3 + 1]);
        gz[v] = half * (gl[v * 3 + 2] + gr[v * 3 + 2]);
        // CorrectGrad, codes/usolver/src/VisGrad.cpp:356-366
        R fOld = gx[v] * dx + gy[v] * dy + gz[v] * dz;
        R fnew = (q2 - q1) * ods;
        R df = fnew - fOld;
        gx[v] += df * dx; gy[v] += df * dy; gz[v] += df * dz;
    }
    R xn = A.G.xfn[f], yn = A.G.yfn[f], zn = A.G.zfn[f];
    R dtdn = xn * gx[5] + yn * gy[5] + zn * gz[5];
    R kcp = (vlm * R(A.P.oprl) + vtm * R(A.P.oprt)) * R(A.P.const_cp);
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

template <typename R>
__global__ void __launch_bounds__(128) k_residual(KArgs<R> A) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= A.M.nCells) return;
    double acc[NEQ];
#pragma unroll
    for (int e = 0; e < NEQ; ++e) acc[e] = -0.0;   // LoadResiduals: res = -rhs, rhs = 0
    int b = A.M.c2f_off[c], en = A.M.c2f_off[c + 1];
    R gam = R(A.P.gama), ce1 = R(A.P.centropy1), ce2 = R(A.P.centropy2);
    for (int k = b; k < en; ++k) {
        int f = A.M.c2f[k];
        R t1[NEQ], t2[NEQ], fl[NEQ];
        face_states(A, f, t1, t2);
        R xn = A.G.xfn[f], yn = A.G.yfn[f], zn = A.G.zfn[f], ar = A.G.area[f];
        if (A.P.ischeme == 12) slau2Flux(t1, t2, xn, yn, zn, gam, fl);
        else roeFlux(t1, t2, xn, yn, zn, gam, A.P.ieigenfix, ce1, ce2, fl);
        bool left = A.M.lc[f] == c;
#pragma unroll
        for (int e = 0; e < NEQ; ++e) {
            double v = double(ar * fl[e]);
            if (left) acc[e] -= v; else acc[e] += v;
        }
    }
    if (A.P.vismodel > 0) {
        R orey = R(A.P.oreynolds);
        for (int k = b; k < en; ++k) {
            int f = A.M.c2f[k];
            R fv[NEQ];
            face_vis_flux(A, f, fv);
            R coeff = -orey * A.G.area[f];
            bool left = A.M.lc[f] == c;
#pragma unroll
            for (int e = 0; e < NEQ; ++e) {
                double v = double(coeff * fv[e]);
                if (left) acc[e] -= v; else acc[e] += v;
            }
        }
    }
    double *o = A.res + (size_t)c * NEQ;
#pragma unroll
    for (int e = 0; e < NEQ; ++e) o[e] = acc[e];
}

// ---------------------------------------------------------------------------
// LU-SGS: UNsLusgs::{LowerSweep,UpperSweep} (codes/uns/src/UNsLusgs.cpp:75-138),
// face increment NsLusgs::GetStandardFluxIncrement (codes/ns/src/NsLusgs.cpp:121-202)
// with the Roe-averaged face radius (UNsLusgs::PrepareDataFacePrim :251-293)
// and the viscous radius (UNsLusgs::CalcViscousTerm :295-330).  Level-scheduled:
// every cell of a level only reads dq of cells in earlier levels.
// ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ void face_increment(const KArgs<R> &A, int ci, int f, double *rhs0) {
    int l = A.M.lc[f], r = A.M.rc[f];
    R xn = A.G.xfn[f], yn = A.G.yfn[f], zn = A.G.zfn[f], fa = A.G.area[f], vfn = R(0);
    if (r == ci) { r = l; l = ci; xn = -xn; yn = -yn; zn = -zn; vfn = -vfn; }
    const double *qa = A.q + (size_t)l * REC, *qb = A.q + (size_t)r * REC;
    R half = R(0.5), one = R(1), gl = R(A.P.gama), gr = gl;
    R rl = R(qa[IR]), ul = R(qa[IU]), vl = R(qa[IV]), wl = R(qa[IW]), pl = R(qa[IP]);
    R rr = R(qb[IR]), ur = R(qb[IU]), vr = R(qb[IV]), wr = R(qb[IW]), pr = R(qb[IP]);
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
    const double *dqj = A.dq + (size_t)r * NEQ;
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
    if (A.P.vismodel > 0) {
        R vl_ = R(qb[IML]), vt_ = R(qb[IMT]);
        R visrad;
        R density = half * (rl + rr);
        if (A.P.visSRModel == 1) {
            R c1 = R(4.0) / R(3.0) * (vl_ + vt_);
            R cc2 = R(A.P.gama) * (vl_ * R(A.P.oprl) + vt_ * R(A.P.oprt));
            R c3 = R(2) * Rmax(c1, cc2) / (R(A.P.reynolds) * density);
            visrad = fa * fa * c3 / A.G.vol[r];
        } else {
            R dist = Rabs(xn * (A.G.xcc[r] - A.G.xcc[l]) + yn * (A.G.ycc[r] - A.G.ycc[l]) + zn * (A.G.zcc[r] - A.G.zcc[l]));
            R viscosity = vl_ + vt_;
            R c1 = R(2) * viscosity / (density * dist * R(A.P.reynolds) + small_v<R>());
            visrad = half * c1 * fa;
        }
        rhs0[0] -= double(visrad * d0); rhs0[1] -= double(visrad * d1); rhs0[2] -= double(visrad * d2);
        rhs0[3] -= double(visrad * d3); rhs0[4] -= double(visrad * d4);
    }
#pragma unroll
    for (int e = 0; e < NEQ; ++e) rhs0[e] += double(df[e]);
}

template <typename R>
__device__ __forceinline__ double implicit_radius(const KArgs<R> &A, int c) {
    // UNsSpectrum::CalcImplicitSpectrum (sp2 = 1 for a steady solve)
    double s = (1.0 / A.dt[c]) * double(A.G.vol[c]);
    s += A.invsr[c];
    s += A.vissr[c];
    return s;
}

template <typename R>
__global__ void __launch_bounds__(128) k_lusgs_lower(KArgs<R> A, const int *order, int start, int count) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    int c = order[start + t];
    double rhs0[NEQ] = {0.0, 0.0, 0.0, 0.0, 0.0};
    int b = A.M.c2f_off[c], en = A.M.c2f_off[c + 1];
    int kc = A.M.key[c];
    for (int k = b; k < en; ++k) {
        int f = A.M.c2f[k];
        if (A.M.key[A.M.lc[f]] > kc || A.M.key[A.M.rc[f]] > kc) continue;   // UNsLusgs::CanNotLowerSolve
        face_increment(A, c, f, rhs0);
    }
    double rad = implicit_radius(A, c);
    const double *rs = A.res + (size_t)c * NEQ;
    double *d = A.dq + (size_t)c * NEQ;
#pragma unroll
    for (int e = 0; e < NEQ; ++e) d[e] = (rs[e] - rhs0[e]) / rad;
}

template <typename R>
__global__ void __launch_bounds__(128) k_lusgs_upper(KArgs<R> A, const int *order, int start, int count) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    int c = order[start + t];
    double rhs0[NEQ] = {0.0, 0.0, 0.0, 0.0, 0.0};
    int b = A.M.c2f_off[c], en = A.M.c2f_off[c + 1];
    int kc = A.M.key[c];
    for (int k = b; k < en; ++k) {
        int f = A.M.c2f[k];
        if (f < A.M.nBFaces) continue;   // ghost dq is zero: no contribution
        if (A.M.key[A.M.lc[f]] < kc || A.M.key[A.M.rc[f]] < kc) continue;   // UNsLusgs::CanNotUpperSolve
        face_increment(A, c, f, rhs0);
    }
    double rad = implicit_radius(A, c);
    double *d = A.dq + (size_t)c * NEQ;
#pragma unroll
    for (int e = 0; e < NEQ; ++e) d[e] += (-rhs0[e]) / rad;
}

// ---------------------------------------------------------------------------
// UPDATE_FLOWFIELD_LUSGS: NsUpdate::CalcFlowField + WeekSolutionFix
// (codes/ns/src/NsUpdate.cpp:40-67,192-217), QToPrim (codes/ns/src/NsInvFlux.cpp:1377-1399);
// then the interior half of CALC_BOUNDARY: NsCalcGamaT + CalcLaminarViscosity.
// Writes the next state buffer; cells that still fail go to a list for the
// sequential neighbour-average fix (UNsUpdate::SolutionFix).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double sutherland(const DevParams &P, double t) {
    // codes/model/src/Sutherland.cpp:62-66
    double t3 = t * t * t;
    return sqrt(t3) * (1 + P.sutherland_ts) / (t + P.sutherland_ts);
}

template <typename R>
__global__ void __launch_bounds__(256) k_update(KArgs<R> A) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= A.M.nCells) return;
    const double *qc = A.q + (size_t)c * REC;
    const double *d = A.dq + (size_t)c * NEQ;
    double gama = A.P.gama;
    double prim0[NEQ], q0[NEQ], qq[NEQ], pr[NEQ], dd[NEQ];
#pragma unroll
    for (int e = 0; e < NEQ; ++e) { prim0[e] = qc[e]; dd[e] = d[e]; }
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
    double *o = A.qn + (size_t)c * REC;
#pragma unroll
    for (int e = 0; e < NEQ; ++e) o[e] = pr[e];
    if (!needFix) {
        double t = pr[IP] / (A.P.statecoef * pr[IR] * 1.0);
        o[ITT] = t;
        o[IML] = fmax(0.0, sutherland(A.P, t));
    }
    o[IMT] = qc[IMT];
}

// UNsUpdate::SolutionFix (codes/uns/src/UNsUpdate.cpp:94-133) for the cells
// that failed every positivity retry.  The reference updates in place in
// natural order, so a neighbour with a lower id contributes its new value and
// one with a higher id its old value; one thread replays that order.
template <typename R>
__global__ void k_solution_fix(KArgs<R> A) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    int n = A.fixlist[0];
    if (n <= 0) return;
    if (n > A.fixcap) n = A.fixcap;
    int *ids = A.fixlist + 1;
    for (int i = 1; i < n; ++i) {   // insertion sort (the list is short)
        int v = ids[i], j = i - 1;
        while (j >= 0 && A.M.key[ids[j]] > A.M.key[v]) { ids[j + 1] = ids[j]; --j; }
        ids[j + 1] = v;
    }
    for (int i = 0; i < n; ++i) {
        int c = ids[i];
        double pr[NEQ] = {0, 0, 0, 0, 0}, sumV = 0.0;
        for (int k = A.M.c2f_off[c]; k < A.M.c2f_off[c + 1]; ++k) {
            int f = A.M.c2f[k];
            int nb = other_cell(A.M.lc[f], A.M.rc[f], c);
            bool done = nb < A.M.nCells && A.M.key[nb] < A.M.key[c];   // already updated in sweep order
            const double *src = done ? A.qn + (size_t)nb * REC : A.q + (size_t)nb * REC;
            sumV += 1.0;
            for (int e = 0; e < NEQ; ++e) {
                double v = src[e];
                if (e == IR || e == IP) v = fabs(v);
                pr[e] += v * 1.0;
            }
        }
        double rv = 1.0 / sumV;
        double *o = A.qn + (size_t)c * REC;
        for (int e = 0; e < NEQ; ++e) o[e] = pr[e] * rv;
        double t = o[IP] / (A.P.statecoef * o[IR] * 1.0);
        o[ITT] = t;
        o[IML] = fmax(0.0, sutherland(A.P, t));
    }
    A.fixlist[0] = 0;
}

// ---------------------------------------------------------------------------
// CALC_BOUNDARY, ghost half: UNsBcSolver::CalcBc (codes/uns/src/UNsBcSolver.cpp:55-166)
// with NsBcSolver's face BCs (codes/ns/src/NsBcSolver.cpp:51-440), then
// NsCalcGamaT + CalcLaminarViscosity on the ghost cells.  Operates on qn.
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(256) k_boundary(KArgs<R> A) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= A.M.nBFaces) return;
    int bt = A.M.bcType[f];
    int l = A.M.lc[f];
    const double *s = A.qn + (size_t)l * REC;
    double *g = A.qn + (size_t)(A.M.nCells + f) * REC;
    double t[NEQ], pr[NEQ];
    bool havePrim = false;
    double xn = double(A.G.xfn[f]), yn = double(A.G.yfn[f]), zn = double(A.G.zfn[f]), vfn = 0.0;
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
#pragma unroll
    for (int e = 0; e < NEQ; ++e) g[e] = t[e];
    double tt = t[IP] / (A.P.statecoef * t[IR] * 1.0);
    g[ITT] = tt;
    g[IML] = fmax(0.0, sutherland(A.P, tt));
    g[IMT] = A.q[(size_t)(A.M.nCells + f) * REC + IMT];   // ghost eddy viscosity is set by the SA solver
    if (havePrim) {
        double *b = A.bcq + (size_t)f * NEQ;
#pragma unroll
        for (int e = 0; e < NEQ; ++e) b[e] = pr[e];
    }
}

// ---------------------------------------------------------------------------
// Residual norms: ResidualTask::CalcRes + ResAver::CalcAver
// (codes/residual/src/ResidualTask.cpp:75-126, codes/residual/src/Residual.cpp:52-72).
// Two-stage fixed-shape reduction in FP64: deterministic run to run.
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(256) k_norm_partial(KArgs<R> A) {
    __shared__ double s[NEQ][256];
    double acc[NEQ] = {0, 0, 0, 0, 0};
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < A.M.nCells; c += gridDim.x * blockDim.x) {
        const double *r = A.res + (size_t)c * NEQ;
#pragma unroll
        for (int e = 0; e < NEQ; ++e) acc[e] += r[e] * r[e];
    }
#pragma unroll
    for (int e = 0; e < NEQ; ++e) s[e][threadIdx.x] = acc[e];
    __syncthreads();
    for (int st = blockDim.x / 2; st > 0; st >>= 1) {
        if (threadIdx.x < st)
#pragma unroll
            for (int e = 0; e < NEQ; ++e) s[e][threadIdx.x] += s[e][threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x == 0)
#pragma unroll
        for (int e = 0; e < NEQ; ++e) A.partial[(size_t)blockIdx.x * NEQ + e] = s[e][0];
}

template <typename R>
__global__ void __launch_bounds__(256) k_norm_final(KArgs<R> A, int nPartial, double *hist) {
    __shared__ double s[NEQ][256];
    double acc[NEQ] = {0, 0, 0, 0, 0};
    for (int i = threadIdx.x; i < nPartial; i += blockDim.x)
#pragma unroll
        for (int e = 0; e < NEQ; ++e) acc[e] += A.partial[(size_t)i * NEQ + e];
#pragma unroll
    for (int e = 0; e < NEQ; ++e) s[e][threadIdx.x] = acc[e];
    __syncthreads();
    for (int st = blockDim.x / 2; st > 0; st >>= 1) {
        if (threadIdx.x < st)
#pragma unroll
            for (int e = 0; e < NEQ; ++e) s[e][threadIdx.x] += s[e][threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        for (int e = 0; e < NEQ; ++e) {
            double rms = sqrt(s[e][0] / A.M.nCells);
            A.scal[S_NORM + e] = rms;
            if (hist) hist[e] = rms;
        }
    }
}

}  // namespace ofg

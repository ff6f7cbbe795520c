// Incompressible solver of the reference (INsSolver, startStrategy 2,
// time_integral 3): one SIMPLE inner iteration per UPDATE_RESIDUALS
// (INsCalcRHS, codes/ins/src/INsRhs.cpp:105-132) in FP64 on the device.
//
// Layout: every per-cell field is one FP64 array over the nTCell cells
// (interior cells, then the ghost cell of each boundary face, as in the
// reference); every per-face field one array over the faces; q is [5][nT]
// (rho u v w p), the reference's layout.  Geometry that the reference forms
// per face on every iteration from the metrics alone (distance weights,
// n . (x_R - x_L), the viscous coefficient vis*S/dist) is formed once at
// creation on the host with the same expressions and stored as a 24-double
// face record.
//
// Each face loop of the reference that accumulates into cells becomes a
// per-cell gather over the cell's faces in ascending face id -- the order in
// which the reference's face loop reaches the cell -- so those sums round
// exactly like the reference's; face loops that write per-face values are
// one thread per face.  The linear solves are the reference's GMRES
// (codes/bgmres/include/GMRES.h: classical Gram-Schmidt, Givens rotations,
// Krylov dimension 500, no restart, identity preconditioner, stop when the
// rotated residual drops below 1e-8 times the right-hand side's norm) with
// the same update formulas; only its inner products are summed in a
// different (blocked, deterministic) order.
//
// GMRES on the device: per Krylov step two kernels.  k_gm_spmv_dots scales
// the previous unnormalised vector on read, stores the new basis vector,
// forms w = A v and, per 256-row chunk, the chunk's share of every inner
// product V[r] . w (one warp per r), summed per block in shared memory; the
// last block to finish (ticket counter, no waiting) sums the blocks' shares
// into column j of the Hessenberg matrix.  k_gm_orth subtracts the projections row by row in the reference's
// order and sums |w|^2; its last block applies the earlier rotations and the
// new one to column j, updates the rotated residual and decides convergence.
// The host launches the steps in chunks and reads one flag per chunk; a step
// launched after convergence returns at once.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "ofg_ctx.h"

namespace {

constexpr int IR = 0, IU = 1, IV = 2, IW = 3, IP = 4;
constexpr double kSmall = 1.0e-40;   // SMALL of codes/basic/include/HXTypeBasic.h
constexpr int kKrylov = 500;         // krylovDimension of SolveMRhs::BGMRES
constexpr double kTol = 1.0e-8;      // its tolerance
constexpr int kThreads = 256;
constexpr int kChunk = kThreads;     // rows per block of k_gm_spmv_dots (one per thread)
constexpr int kStepsPerSync = 8;     // Krylov steps launched between flag reads

// face record [nFaces][kFR]
enum : int {
    F_XN = 0, F_YN, F_ZN, F_AREA, F_DIST, F_LX, F_LY, F_LZ, F_DX1, F_DY1, F_DZ1, F_DX2, F_DY2, F_DZ2,
    F_W1, F_W2, F_G1, F_G2, F_FN, F_NXA, F_NYA, F_NZA, kFR = 24
};

__device__ __forceinline__ double max0(double v) { return 0.0 > v ? 0.0 : v; }   // MAX(0, v), HXMath.h:158-161

// GMRES scalars shared by the kernels of one solve
struct GmState {
    int j;          // current Krylov step
    int done;       // 1 once converged or out of steps
    int dim;        // dimension of the update (the step that converged, or kKrylov - 1)
    int iters;      // steps counted as the reference returns them
    double normRHS, rho, inv, res;
    unsigned int ticket;
};

struct Dev {
    int nF, nB, nC, nT;
    double dt, vis;
    const int *lc, *rc;           // [nF]
    const double *fr;             // [nF][kFR]
    const double *vol;            // [nT]
    const int *cOff, *cFace;      // per cell (ghosts: their one face) faces ascending, side in bit 0
    const int *rOff;              // matrix rows of the solves: row c holds the reference's c2f entries + diagonal
    const int *JA;                // column of each matrix entry
    const double *wall;           // [nB][3]
    double *q;                    // [5][nT]
    double *gx, *gy, *gz;         // [5][nT] gradients (rho row zero)
    double *rf, *uf, *vf, *wf, *fq, *ai0, *ai1, *bi;   // bi: [6][nF] biu0 biu1 biv0 biv1 biw0 biw1
    double *Vdv, *ajp;
    double *spt, *bt;             // bt: [3][nT] but bvt bwt
    double *up, *spc, *bm;        // up: [3][nT] up vp wp; bm: [3][nT] buc bvc bwc
    double *uc;                   // [3][nT] uc vc wc
    double *spp, *bp, *pp, *VdU, *gq;   // gq: [3][nT] dqqdx dqqdy dqqdz
    double *mu;                   // [3][nC] mu mv mw (kept across inner steps)
    double *Am, *Ap;              // matrix values of the momentum and pressure solves
    double *part;                 // [nPart][4] residual partial sums
    double *red;                  // [4] remax
    unsigned int *ticket;
};

// ---------------------------------------------------------------- kernels
// UINsInvterm::INsPreflux (first inner step), UINsInvterm.cpp:138-178;
// INsInvterm::CalcINsinvFlux / CalcINsBcinvFlux, codes/ins/src/INsInvterm.cpp:89-140
__global__ void k_ins_preflux(Dev D) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= D.nF) return;
    const double *q = D.q;
    const int nT = D.nT, l = D.lc[f], r = D.rc[f];
    const double *g = D.fr + (size_t)f * kFR;
    double rf = (q[IR * nT + l] + q[IR * nT + r]) * 0.5;
    double uf = (q[IU * nT + l] + q[IU * nT + r]) * 0.5;
    double vf = (q[IV * nT + l] + q[IV * nT + r]) * 0.5;
    double wf = (q[IW * nT + l] + q[IW * nT + r]) * 0.5;
    double vn = g[F_XN] * uf + g[F_YN] * vf + g[F_ZN] * wf - 0.0;
    D.rf[f] = rf; D.uf[f] = uf; D.vf[f] = vf; D.wf[f] = wf;
    D.fq[f] = f < D.nB ? 0.0 : rf * vn * g[F_AREA];
}

// Green-Gauss gradient with distance-weighted face values (UINsVisterm::
// CalcPreandVisGrad, UINsVisterm.cpp:98-228; UINsInvterm::CalcPreGrad,
// UINsInvterm.cpp:1984-2059): NV fields v[k] (stride nT) -> g*[k]; a ghost
// takes its interior cell's gradient (computed again here).  wsel 0: the
// weights of the viscous gradient, 1: those with SMALL.
template <int NV>
__global__ void k_ins_grad(Dev D, const double *v, double *gx, double *gy, double *gz, int wsel) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= D.nT) return;
    const int nT = D.nT;
    const int cell = c < D.nC ? c : D.lc[c - D.nC];
    double ax[NV], ay[NV], az[NV];
#pragma unroll
    for (int i = 0; i < NV; ++i) ax[i] = ay[i] = az[i] = 0.0;
    for (int k = D.cOff[cell]; k < D.cOff[cell + 1]; ++k) {
        const int e = D.cFace[k], f = e >> 1;
        const double *g = D.fr + (size_t)f * kFR;
        const int l = D.lc[f], r = D.rc[f];
        const double cl = g[wsel ? F_G1 : F_W1], cr = g[wsel ? F_G2 : F_W2];
        const double nxa = g[F_NXA], nya = g[F_NYA], nza = g[F_NZA];
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            double val = cl * v[i * nT + l] + cr * v[i * nT + r];
            if (!(e & 1)) { ax[i] += nxa * val; ay[i] += nya * val; az[i] += nza * val; }
            else { ax[i] += -nxa * val; ay[i] += -nya * val; az[i] += -nza * val; }
        }
    }
    const double ovol = 1.0 / D.vol[cell];
#pragma unroll
    for (int i = 0; i < NV; ++i) {
        gx[i * nT + c] = ax[i] * ovol; gy[i * nT + c] = ay[i] * ovol; gz[i * nT + c] = az[i] * ovol;
    }
}

// CalcInvMassFlux (INsInvterm::CalcINsinvTerm, INsInvterm.cpp:142-154) and
// UINsVisterm::CalcFaceVisterm (UINsVisterm.cpp:281-394), every face
__global__ void k_ins_face_coef(Dev D) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= D.nF) return;
    const int nT = D.nT, nF = D.nF, l = D.lc[f], r = D.rc[f];
    const double *g = D.fr + (size_t)f * kFR;
    const double clr = max0(D.fq[f]);
    double a0 = clr, a1 = clr - D.fq[f];
    a0 += g[F_FN];
    a1 += g[F_FN];
    D.ai0[f] = a0; D.ai1[f] = a1;
    const double w1 = g[F_W1], w2 = g[F_W2], dist = g[F_DIST], area = g[F_AREA], vis = D.vis;
    for (int k = 0; k < 3; ++k) {
        const int e = (IU + k) * nT;
        double gxf = w1 * D.gx[e + l] + w2 * D.gx[e + r];
        double gyf = w1 * D.gy[e + l] + w2 * D.gy[e + r];
        double gzf = w1 * D.gz[e + l] + w2 * D.gz[e + r];
        double Pf = gxf * g[F_XN] + gyf * g[F_YN] + gzf * g[F_ZN];
        double Pd = -(gxf * g[F_LX] + gyf * g[F_LY] + gzf * g[F_LZ]) / dist;
        double F1 = Pf * area * vis, F2 = Pd * area * vis;
        D.bi[(2 * k) * nF + f] = F1 + F2;
        D.bi[(2 * k + 1) * nF + f] = -F1 - F2;
    }
}

// UINsVisterm::CalcUnsteadcoff (UINsVisterm.cpp:479-562) and CalcINsSrc
// (UINsVisterm.cpp:564-632), one cell; then its row of the momentum matrix
// (MomPre, UINsInvterm.cpp:446-478: -ai of each c2f face, spc last)
__global__ void k_ins_momentum_rows(Dev D, int first) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= D.nT) return;
    const int nT = D.nT, nF = D.nF;
    const double rho = D.q[IR * nT + c], vol = D.vol[c];
    const double spt = vol * rho / D.dt;
    D.spt[c] = spt;
    double bt[3];
    for (int k = 0; k < 3; ++k) {
        if (first) D.up[k * nT + c] = D.q[(IU + k) * nT + c];
        bt[k] = vol * rho * D.up[k * nT + c] / D.dt;
        D.bt[k * nT + c] = bt[k];
    }
    double spc = 0.0, b[3] = {0.0, 0.0, 0.0};
    if (c < D.nC) {
        for (int k = D.cOff[c]; k < D.cOff[c + 1]; ++k) {
            const int e = D.cFace[k], f = e >> 1, s = e & 1;
            spc += s ? D.ai1[f] : D.ai0[f];
            for (int i = 0; i < 3; ++i) b[i] += D.bi[(2 * i + s) * nF + f];
        }
    } else {
        const int f = c - D.nC;   // the ghost is the right cell of its face
        spc += D.ai1[f];
        for (int i = 0; i < 3; ++i) b[i] += D.bi[(2 * i + 1) * nF + f];
    }
    spc += spt;
    const double gp[3] = {D.gx[IP * nT + c], D.gy[IP * nT + c], D.gz[IP * nT + c]};
    for (int i = 0; i < 3; ++i) { b[i] += bt[i] - vol * gp[i]; D.bm[i * nT + c] = b[i]; }
    D.spc[c] = spc;
    const int n = D.rOff[c];
    const int nf = c < D.nC ? D.cOff[c + 1] - D.cOff[c] : 0;
    for (int k = 0; k < nf; ++k) {
        const int e = D.cFace[D.cOff[c] + k], f = e >> 1;
        D.Am[n + k] = (e & 1) ? -D.ai1[f] : -D.ai0[f];
    }
    D.Am[n + nf] = spc;
}

// ghost velocity of a solid wall: -v_interior + 2 v_wall
// (MomPre, UINsInvterm.cpp:617-700)
__global__ void k_ins_wall_uc(Dev D) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= D.nB) return;
    const int nT = D.nT, l = D.lc[f], r = D.rc[f];
    for (int k = 0; k < 3; ++k) D.uc[k * nT + r] = -D.uc[k * nT + l] + 2 * D.wall[3 * f + k];
}

// UINsInvterm::CalcFaceflux (UINsInvterm.cpp:866-908) with the face states
// of PrepareProFaceValue (UINsInvterm.cpp:338-362; the right state's w is
// vc of the right cell there); INsInvterm::CalcINsFaceflux / CalcINsBcFaceflux
// (codes/ins/src/INsInvterm.cpp:170-271)
__global__ void k_ins_face_flux(Dev D) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= D.nF) return;
    const int nT = D.nT, l = D.lc[f], r = D.rc[f];
    const double *q = D.q, *uc = D.uc, *vc = D.uc + nT, *wc = D.uc + 2 * nT;
    double fq, rf, uf, vf, wf;
    if (f >= D.nB) {
        const double *g = D.fr + (size_t)f * kFR;
        const double rl = q[IR * nT + l], ul = uc[l], vl = vc[l], wl = wc[l], pl = q[IP * nT + l];
        const double rr = q[IR * nT + r], ur = uc[r], vr = vc[r], wr = vc[r], pr = q[IP * nT + r];
        const double xn = g[F_XN], yn = g[F_YN], zn = g[F_ZN], w1 = g[F_W1], w2 = g[F_W2];
        const double vl_ = D.vol[l], vr_ = D.vol[r], sl = D.spc[l], sr = D.spc[r];
        double Vau = w1 * (vl_ * xn / sl) + w2 * (vr_ * xn / sr);
        double Vav = w1 * (vl_ * yn / sl) + w2 * (vr_ * yn / sr);
        double Vaw = w1 * (vl_ * zn / sl) + w2 * (vr_ * zn / sr);
        const double dist = g[F_DIST];
        double Deun = Vau / dist, Devn = Vav / dist, Dewn = Vaw / dist;
        const double *gx = D.gx + IP * nT, *gy = D.gy + IP * nT, *gz = D.gz + IP * nT;
        double Bpe = gx[l] * (g[F_DX1]) + gy[l] * (g[F_DY1]) + gz[l] * (g[F_DZ1]) + gx[r] * (g[F_DX2]) +
                     gy[r] * (g[F_DY2]) + gz[r] * (g[F_DZ2]) - (pr - pl);
        rf = 0.5 * (rl + rr);
        uf = (w1 * ul + w2 * ur) + Deun * Bpe;
        vf = (w1 * vl + w2 * vr) + Devn * Bpe;
        wf = (w1 * wl + w2 * wr) + Dewn * Bpe;
        double vn = xn * uf + yn * vf + zn * wf;
        fq = rf * vn * g[F_AREA];
    } else {
        rf = (q[IR * nT + l] + q[IR * nT + r]) * 0.5;
        uf = (uc[l] + uc[r]) * 0.5;
        vf = (vc[l] + vc[r]) * 0.5;
        wf = (wc[l] + vc[r]) * 0.5;
        fq = 0;   // SOLID_SURFACE
    }
    D.rf[f] = rf; D.uf[f] = uf; D.vf[f] = vf; D.wf[f] = wf; D.fq[f] = fq;
    const double clr = max0(fq);
    D.ai0[f] = clr;
    D.ai1[f] = clr - fq;
}

// UINsInvterm::CalcNewMomCoe (UINsInvterm.cpp:1184-1213) and the unit
// correction coefficient VdU (UINsInvterm.cpp:1082-1091)
__global__ void k_ins_new_spc(Dev D) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= D.nT) return;
    double spc = 0.0;
    if (c < D.nC) {
        for (int k = D.cOff[c]; k < D.cOff[c + 1]; ++k) {
            const int e = D.cFace[k], f = e >> 1;
            spc += ((e & 1) ? D.ai1[f] : D.ai0[f]) + D.fr[(size_t)f * kFR + F_FN];
        }
    } else {
        const int f = c - D.nC;
        spc += D.ai1[f] + D.fr[(size_t)f * kFR + F_FN];
    }
    spc += D.spt[c];
    D.spc[c] = spc;
    D.VdU[c] = -D.vol[c] / ((1 + 1) * spc);
}

// INsInvterm::CalcINsFaceCorrectPresscoef / CalcINsBcFaceCorrectPresscoef
// (codes/ins/src/INsInvterm.cpp:273-334)
__global__ void k_ins_face_pcoef(Dev D) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= D.nF) return;
    if (f < D.nB) { D.Vdv[f] = 0; D.ajp[f] = 0; return; }
    const int l = D.lc[f], r = D.rc[f];
    const double *g = D.fr + (size_t)f * kFR;
    const double a = g[F_W1] * (D.vol[l] / (D.spc[l])) + g[F_W2] * (D.vol[r] / (D.spc[r]));
    D.Vdv[f] = a;
    const double xn = g[F_XN], yn = g[F_YN], zn = g[F_ZN];
    D.ajp[f] = D.rf[f] * (a * xn * xn + a * yn * yn + a * zn * zn) * g[F_AREA] / g[F_DIST];
}

// spp and bp (UINsInvterm.cpp:1060-1080) and the pressure-correction matrix
// row (UINsInvterm.cpp:1272-1306: -ajp off the diagonal, spp on it)
__global__ void k_ins_pressure_rows(Dev D) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= D.nT) return;
    double spp = 0.0, bp = 0.0;
    const int n = D.rOff[c];
    if (c < D.nC) {
        const int b = D.cOff[c], nf = D.cOff[c + 1] - b;
        for (int k = 0; k < nf; ++k) {
            const int e = D.cFace[b + k], f = e >> 1;
            const double a = D.ajp[f];
            spp += a;
            bp += (e & 1) ? D.fq[f] : -D.fq[f];
            D.Ap[n + k] = -a;
        }
        D.Ap[n + nf] = spp;
    } else {
        const int f = c - D.nC;
        spp = 1;   // a boundary face sets its ghost's coefficient to one
        bp += D.fq[f];
        D.Ap[n] = spp;
    }
    D.spp[c] = spp;
    D.bp[c] = bp;
}

// pressure update (UINsInvterm.cpp:1318-1338): the interior cells take
// 0.8 pp; each ghost copies its interior cell's pp
__global__ void k_ins_p_update(Dev D) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= D.nT) return;
    if (c < D.nC) D.q[IP * D.nT + c] = D.q[IP * D.nT + c] + 0.8 * D.pp[c];
    else D.pp[c] = D.pp[D.lc[c - D.nC]];
}

// UINsInvterm::UpdateSpeed (UINsInvterm.cpp:1607-1840): velocity correction
// and the solid-wall ghosts; a ghost also takes its interior cell's pressure
// (UINsInvterm.cpp:1346-1349)
__global__ void k_ins_speed(Dev D) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= D.nT) return;
    const int nT = D.nT;
    if (c < D.nC) {
        for (int k = 0; k < 3; ++k) {
            double u = D.uc[k * nT + c] + D.VdU[c] * D.gq[k * nT + c] * 0.8;
            D.up[k * nT + c] = u;
            D.q[(IU + k) * nT + c] = u;
        }
    } else {
        const int f = c - D.nC, l = D.lc[f];
        for (int k = 0; k < 3; ++k) {
            double ul = D.uc[k * nT + l] + D.VdU[l] * D.gq[k * nT + l] * 0.8;
            double u = -ul + 2 * D.wall[3 * f + k];
            D.up[k * nT + c] = u;
            D.q[(IU + k) * nT + c] = u;
        }
        D.q[IP * nT + c] = D.q[IP * nT + l];
    }
}

// UINsInvterm::UpdateFaceflux, interior faces (UINsInvterm.cpp:1589-1605);
// on the boundary faces the correction is zero
__global__ void k_ins_face_update(Dev D) {
    int f = D.nB + blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= D.nF) return;
    const int l = D.lc[f], r = D.rc[f];
    const double *g = D.fr + (size_t)f * kFR;
    const double xn = g[F_XN], yn = g[F_YN], zn = g[F_ZN], dist = g[F_DIST], a = D.Vdv[f];
    const double dp = D.pp[l] - D.pp[r];
    double uuj = a * dp * xn / dist, vvj = a * dp * yn / dist, wwj = a * dp * zn / dist;
    D.uf[f] = D.uf[f] + uuj; D.vf[f] = D.vf[f] + vvj; D.wf[f] = D.wf[f] + wwj;
    double fux = D.rf[f] * (xn * uuj + yn * vvj + zn * wwj) * g[F_AREA];
    D.fq[f] = D.fq[f] + fux;
}

// UINsInvterm::UpdateINsRes (UINsInvterm.cpp:1842-1982): bp collects the
// corrected mass fluxes, mu mv mw the off-diagonal sums (kept across inner
// steps, as there); per-block sums of the squared residuals, the last block
// to finish adds them (block order) and takes the square roots
__global__ void k_ins_residuals(Dev D) {
    __shared__ double sh[4][kThreads / 32];
    __shared__ bool last;
    const int nT = D.nT;
    double s[4] = {0, 0, 0, 0};
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < D.nT) {
        double bp = D.bp[c];
        if (c < D.nC) {
            double m[3] = {D.mu[c], D.mu[D.nC + c], D.mu[2 * D.nC + c]};
            for (int k = D.cOff[c]; k < D.cOff[c + 1]; ++k) {
                const int e = D.cFace[k], f = e >> 1, l = D.lc[f], r = D.rc[f];
                const double fq = D.fq[f];
                bp += (e & 1) ? fq : -fq;
                const int o = (e & 1) ? l : r;
                const double a = (e & 1) ? D.ai1[f] : D.ai0[f];
                for (int i = 0; i < 3; ++i) m[i] += -a * (D.up[i * nT + o] - D.uc[i * nT + o]);
            }
            for (int i = 0; i < 3; ++i) {
                D.mu[i * D.nC + c] = m[i];
                double ma = D.spc[c] * (D.up[i * nT + c] - D.uc[i * nT + c]) + m[i];
                s[i] = ma * ma;
            }
            s[3] = bp * bp;
        } else {
            bp += D.fq[c - D.nC];
        }
        D.bp[c] = bp;
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int i = 0; i < 4; ++i) {
        double v = s[i];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sh[i][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double v = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) v += sh[threadIdx.x][w];
        D.part[(size_t)blockIdx.x * 4 + threadIdx.x] = v;
        __threadfence();
    }
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(D.ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (wid < 4) {   // warp i adds quantity i over the blocks (lanes strided, then the warp tree)
        double v = 0.0;
        for (unsigned b = lane; b < gridDim.x; b += 32) v += ((volatile double *)D.part)[(size_t)b * 4 + wid];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) D.red[wid] = sqrt(v);
    }
    if (threadIdx.x == 0) *D.ticket = 0;
}

// ------------------------------------------------------------------ GMRES
struct Gm {
    int nT;
    const int *rOff, *JA;
    const double *A;
    const double *b;   // right-hand side
    double *x;         // solution
    double *V;         // [kKrylov + 1][nT] normalised basis
    double *W;         // [nT] unnormalised next vector
    double *Y;         // [nT] A v_j
    double *H;         // [(kKrylov + 1) * kKrylov] row-major (i, j) -> i * kKrylov + j
    double *gc, *gs, *s;
    double *part;      // [nBlk][kKrylov + 1] per-chunk inner products, then [nBlk] norms
    GmState *st;
};

__device__ __forceinline__ double block_sum(double v, double *sh) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
    return t;   // valid in thread 0
}

// sum of n partial sums (stride `stride`) by the whole block, in a fixed
// order (thread t adds t, t + blockDim, ...; then the block tree): the
// result is valid in thread 0.  Only for the last block of a ticket
// reduction: the partials are read through volatile loads.
__device__ __forceinline__ double last_block_sum(const double *part, int n, int stride, double *sh) {
    double v = 0.0;
    for (int b = threadIdx.x; b < n; b += blockDim.x) v += ((volatile const double *)part)[(size_t)b * stride];
    return block_sum(v, sh);
}

// |b|^2 per block (the initial residual is b: x starts at zero)
__global__ void k_gm_init(Gm G) {
    __shared__ double sh[32];
    __shared__ bool last;
    double v = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < G.nT; i += gridDim.x * blockDim.x) {
        const double r = G.b[i];
        G.W[i] = r;
        G.x[i] = 0.0;
        v += r * r;
    }
    double t = block_sum(v, sh);
    if (threadIdx.x == 0) {
        G.part[blockIdx.x] = t;
        __threadfence();
        last = atomicAdd(&G.st->ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    const double sum = last_block_sum(G.part, gridDim.x, 1, sh);
    if (threadIdx.x != 0) return;
    GmState *S = G.st;
    const double normr1 = sqrt(sum);
    double normRHS = normr1;
    S->rho = normr1;
    S->res = normr1;
    if (normRHS < 1.0e-5) normRHS = 1.0;
    S->normRHS = normRHS;
    S->j = 0;
    S->iters = 0;
    S->dim = -1;
    S->ticket = 0;
    if (!(normr1 > kTol * normRHS)) { S->done = 1; return; }
    S->done = 0;
    G.s[0] = normr1;
    S->inv = 1.0 / normr1;
}

// one Krylov step, first half: v_j = W / |W| (stored), Y = A v_j, and the
// inner products V[r] . Y, r <= j, into column j of H.  Each block walks its
// 256-row chunks (grid stride), forms the chunk's rows of A v_j in shared
// memory and adds the chunk's share of each product to its own sum in shared
// memory (warp r % 8 owns r); its sums go out r-major, and the last block
// (ticket counter, no waiting) adds the blocks' sums for each r with a warp
// over the blocks -- a fixed order throughout.
__global__ void __launch_bounds__(kThreads) k_gm_spmv_dots(Gm G) {
    __shared__ double ys[kChunk];
    __shared__ double acc[kKrylov + 1];
    __shared__ bool last;
    GmState *S = G.st;
    if (((volatile int *)&S->done)[0]) return;
    const int j = S->j;
    const double inv = S->inv;
    const int nT = G.nT;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double *Vj = G.V + (size_t)j * nT;
    for (int r = threadIdx.x; r <= j; r += blockDim.x) acc[r] = 0.0;
    const int nChunks = (nT + kChunk - 1) / kChunk;
    for (int ch = blockIdx.x; ch < nChunks; ch += gridDim.x) {
        const int r0 = ch * kChunk;
        __syncthreads();   // ys of the previous chunk consumed
        {
            const int t = threadIdx.x, i = r0 + t;
            double y = 0.0;
            if (i < nT) {
                Vj[i] = G.W[i] * inv;
                for (int k = G.rOff[i]; k < G.rOff[i + 1]; ++k) y += G.A[k] * (G.W[G.JA[k]] * inv);
                G.Y[i] = y;
            }
            ys[t] = y;
        }
        __syncthreads();
        const int rows = min(kChunk, nT - r0);
        // this lane's rows of the chunk: lane, lane + 32, ... (kChunk / 32 of them)
        constexpr int KR = kChunk / 32;
        double yv[KR];
#pragma unroll
        for (int k = 0; k < KR; ++k) yv[k] = ys[lane + 32 * k];
        // v_j = W * inv for the lane's rows (this step's vector, not stored yet)
        double wv[KR];
#pragma unroll
        for (int k = 0; k < KR; ++k) wv[k] = lane + 32 * k < rows ? G.W[r0 + lane + 32 * k] * inv : 0.0;
        // the stored basis vectors r < j, four per pass of the warp (32 loads
        // in flight per lane), each summed over the lane's rows in ascending
        // order, then over the warp; warp w owns r with (r / 4) % 8 == w
        for (int rb = 4 * wid; rb < j; rb += 4 * nw) {
            const double *V0 = G.V + (size_t)rb * nT + r0;
            double d0 = 0.0, d1 = 0.0, d2 = 0.0, d3 = 0.0;
            if (rows == kChunk && rb + 4 <= j) {   // the common case: no guards
                double a[KR], b[KR], c[KR], e[KR];
#pragma unroll
                for (int k = 0; k < KR; ++k) {
                    const int t = lane + 32 * k;
                    a[k] = __ldg(V0 + t);
                    b[k] = __ldg(V0 + nT + t);
                    c[k] = __ldg(V0 + 2 * (size_t)nT + t);
                    e[k] = __ldg(V0 + 3 * (size_t)nT + t);
                }
#pragma unroll
                for (int k = 0; k < KR; ++k) {
                    d0 += yv[k] * a[k]; d1 += yv[k] * b[k]; d2 += yv[k] * c[k]; d3 += yv[k] * e[k];
                }
            } else {
#pragma unroll
                for (int k = 0; k < KR; ++k) {
                    const int t = lane + 32 * k;
                    if (t < rows) {
                        d0 += yv[k] * __ldg(V0 + t);
                        if (rb + 1 < j) d1 += yv[k] * __ldg(V0 + nT + t);
                        if (rb + 2 < j) d2 += yv[k] * __ldg(V0 + 2 * (size_t)nT + t);
                        if (rb + 3 < j) d3 += yv[k] * __ldg(V0 + 3 * (size_t)nT + t);
                    }
                }
            }
            for (int o = 16; o > 0; o >>= 1) {
                d0 += __shfl_down_sync(0xffffffffu, d0, o);
                d1 += __shfl_down_sync(0xffffffffu, d1, o);
                d2 += __shfl_down_sync(0xffffffffu, d2, o);
                d3 += __shfl_down_sync(0xffffffffu, d3, o);
            }
            if (lane == 0) {
                acc[rb] += d0;
                if (rb + 1 < j) acc[rb + 1] += d1;
                if (rb + 2 < j) acc[rb + 2] += d2;
                if (rb + 3 < j) acc[rb + 3] += d3;
            }
        }
        // r = j, by the warp that owns it
        if (((j / 4) % nw) == wid) {
            double d = 0.0;
#pragma unroll
            for (int k = 0; k < KR; ++k)
                if (lane + 32 * k < rows) d += yv[k] * wv[k];
            for (int o = 16; o > 0; o >>= 1) d += __shfl_down_sync(0xffffffffu, d, o);
            if (lane == 0) acc[j] += d;
        }
    }
    __syncthreads();
    const int nb = gridDim.x;
    for (int r = threadIdx.x; r <= j; r += blockDim.x) G.part[(size_t)r * nb + blockIdx.x] = acc[r];
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(&S->ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    // column j of H: per r, the lanes over the blocks' sums (fixed order) and
    // a warp reduction; a warp takes four r per pass (four loads in flight)
    for (int rq = 4 * wid; rq <= j; rq += 4 * nw) {
        double h[4] = {0.0, 0.0, 0.0, 0.0};
        const double *P = G.part + (size_t)rq * nb;
        for (int b = lane; b < nb; b += 32) {
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (rq + q <= j) h[q] += __ldcg(P + (size_t)q * nb + b);
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            for (int o = 16; o > 0; o >>= 1) h[q] += __shfl_down_sync(0xffffffffu, h[q], o);
            if (lane == 0 && rq + q <= j) G.H[(size_t)(rq + q) * kKrylov + j] = h[q];
        }
    }
    if (threadIdx.x == 0) S->ticket = 0;
}

// one Krylov step, second half: W = Y - sum_r V[r] H[r][j] (subtracted in
// order r = 0..j, as the reference), |W|^2, then (last block) H[j+1][j],
// the Givens rotations of column j, the rotated residual and the decision
__global__ void __launch_bounds__(kThreads) k_gm_orth(Gm G) {
    __shared__ double sh[32];
    __shared__ double hcol[kKrylov + 1];
    __shared__ double rc[kKrylov], rs[kKrylov];   // the last block's copy of the earlier rotations
    __shared__ bool last;
    GmState *S = G.st;
    if (((volatile int *)&S->done)[0]) return;
    const int j = S->j;
    const int nT = G.nT;
    for (int r = threadIdx.x; r <= j; r += blockDim.x) hcol[r] = G.H[(size_t)r * kKrylov + j];
    __syncthreads();
    double v = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nT; i += gridDim.x * blockDim.x) {
        double w = G.Y[i];
        // in the reference's order r = 0..j; the basis entries of 16 steps
        // are loaded together ahead of their subtractions
        int r = 0;
        for (; r + 16 <= j + 1; r += 16) {
            double vv[16];
#pragma unroll
            for (int q = 0; q < 16; ++q) vv[q] = __ldg(G.V + (size_t)(r + q) * nT + i);
#pragma unroll
            for (int q = 0; q < 16; ++q) w = w - vv[q] * hcol[r + q];
        }
        for (; r <= j; ++r) w = w - __ldg(G.V + (size_t)r * nT + i) * hcol[r];
        G.W[i] = w;
        v += w * w;
    }
    double t = block_sum(v, sh);
    if (threadIdx.x == 0) {
        G.part[blockIdx.x] = t;
        __threadfence();
        last = atomicAdd(&S->ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    const double sum = last_block_sum(G.part, gridDim.x, 1, sh);
    for (int r = threadIdx.x; r < j; r += blockDim.x) { rc[r] = G.gc[r]; rs[r] = G.gs[r]; }
    __syncthreads();
    if (threadIdx.x != 0) return;
    const double normr2 = sqrt(sum);
    double *H = G.H;
    auto h = [&](int a, int b) -> double & { return H[(size_t)a * kKrylov + b]; };
    const int col = j;
    // the earlier rotations down column j (hcol holds it as the products left
    // it): the running entry h(row, col) stays in a register, the rotated
    // entries go out as they are final
    double hr = hcol[0];
    for (int row = 0; row < col; ++row) {
        const double hn = hcol[row + 1], c = rc[row], sn = rs[row];
        double tmp = c * hr + sn * hn;
        hr = -sn * hr + c * hn;
        h(row, col) = tmp;
    }
    double hcc = hr, hc1 = normr2;   // h(col, col), h(col + 1, col)
    if (hc1 == 0.0) {
        G.gc[col] = 1.0; G.gs[col] = 0.0;
    } else if (fabs(hc1) > fabs(hcc)) {
        double tmp = hcc / hc1;
        G.gs[col] = 1.0 / sqrt(1.0 + tmp * tmp);
        G.gc[col] = tmp * G.gs[col];
    } else {
        double tmp = hc1 / hcc;
        G.gc[col] = 1.0 / sqrt(1.0 + tmp * tmp);
        G.gs[col] = tmp * G.gc[col];
    }
    {
        const double c = G.gc[col], sn = G.gs[col];
        double tmp = c * hcc + sn * hc1;
        hc1 = -sn * hcc + c * hc1;
        hcc = tmp;
    }
    if (hc1 < 1e-10) hc1 = 0;
    h(col, col) = hcc;
    h(col + 1, col) = hc1;
    const double st = G.gc[col] * G.s[col] + G.gs[col] * G.s[col + 1];
    G.s[col + 1] = -G.gs[col] * G.s[col] + G.gc[col] * G.s[col + 1];
    G.s[col] = st;
    const double Sv = G.s[j + 1];
    S->rho = sqrt(Sv * Sv);
    S->inv = 1.0 / normr2;
    S->ticket = 0;
    if (S->rho < kTol * S->normRHS) {
        S->dim = j; S->iters = j; S->done = 1;
    } else if (j + 1 == kKrylov) {
        S->dim = kKrylov - 1; S->iters = kKrylov; S->done = 1;
    } else {
        S->j = j + 1;
    }
}

// Update (GMRES.h:20-61), first part: back substitution of s in place
__global__ void k_gm_backsub(Gm G) {
    GmState *S = G.st;
    const int dim = S->dim;
    for (int l = dim; l >= 0; --l) {
        if (threadIdx.x == 0) G.s[l] = G.s[l] / G.H[(size_t)l * kKrylov + l];
        __syncthreads();
        const double sl = G.s[l];
        for (int i = threadIdx.x; i < l; i += blockDim.x) G.s[i] -= sl * G.H[(size_t)i * kKrylov + l];
        __syncthreads();
    }
}

// x += V s, basis vectors from the last (GMRES.h:47-60)
__global__ void k_gm_update_x(Gm G) {
    const int dim = G.st->dim;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < G.nT; i += gridDim.x * blockDim.x) {
        double x = G.x[i];
        for (int m = dim; m >= 0; --m) x += G.V[(size_t)m * G.nT + i] * G.s[m];
        G.x[i] = x;
    }
}

// Rank.residual after an update: |A x - b|
__global__ void k_gm_residual(Gm G) {
    __shared__ double sh[32];
    __shared__ bool last;
    double v = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < G.nT; i += gridDim.x * blockDim.x) {
        double y = 0.0;
        for (int k = G.rOff[i]; k < G.rOff[i + 1]; ++k) y += G.A[k] * G.x[G.JA[k]];
        const double r = y - G.b[i];
        v += r * r;
    }
    double t = block_sum(v, sh);
    if (threadIdx.x == 0) {
        G.part[blockIdx.x] = t;
        __threadfence();
        last = atomicAdd(&G.st->ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    const double sum = last_block_sum(G.part, gridDim.x, 1, sh);
    if (threadIdx.x != 0) return;
    G.st->res = sqrt(sum);
    G.st->ticket = 0;
}

}  // namespace

// ------------------------------------------------------------------ host
struct ofg_ins {
    ofg_ctx *c = nullptr;
    Dev D{};
    std::vector<void *> allocs;
    // GMRES workspace
    double *V = nullptr, *W = nullptr, *Y = nullptr, *H = nullptr, *gc = nullptr, *gs = nullptr, *s = nullptr,
           *gpart = nullptr;
    GmState *st = nullptr;
    GmState *hst = nullptr;           // pinned host copy of the GMRES scalars
    double *hred = nullptr;           // pinned host copy of remax
    int nPart = 0, nChunkBlk = 0, nGrid = 0;
    long long nnz = 0;
    long innerSteps = 0;
    double remax[4] = {1, 1, 1, 1};
    int linIts[4] = {0, 0, 0, 0};
    double linRes[4] = {0, 0, 0, 0};
    double ms = 0.0, gmresMs = 0.0;
    long gmresTotal = 0;
    double gmresBytes = 0.0;   // algorithmic bytes of the Krylov steps run (see gmres())
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, eg0 = nullptr, eg1 = nullptr;

    int fail(int code, const std::string &m) { c->err = "ins: " + m; return code; }
    template <typename T> int alloc(T **p, size_t n) {
        if (cudaMalloc((void **)p, (n ? n : 1) * sizeof(T)) != cudaSuccess) { *p = nullptr; return OFG_E_NOMEM; }
        allocs.push_back((void *)*p);
        return OFG_OK;
    }
};

#define INS_CK(call)                                                                        \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess) return s->fail(OFG_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

namespace {

int blocks(int n) { return (n + kThreads - 1) / kThreads; }

// one GMRES solve of A x = b on the context's stream; returns OFG_OK and the
// iteration count / residual in *its, *res
int gmres(ofg_ins *s, const double *A, const double *b, double *x, int *its, double *res) {
    cudaStream_t st = s->c->stream;
    Gm G{};
    G.nT = s->D.nT; G.rOff = s->D.rOff; G.JA = s->D.JA; G.A = A; G.b = b; G.x = x;
    G.V = s->V; G.W = s->W; G.Y = s->Y; G.H = s->H; G.gc = s->gc; G.gs = s->gs; G.s = s->s; G.part = s->gpart;
    G.st = s->st;
    INS_CK(cudaEventRecord(s->eg0, st));
    INS_CK(cudaMemsetAsync(s->H, 0, sizeof(double) * (size_t)(kKrylov + 1) * kKrylov, st));
    INS_CK(cudaMemsetAsync(s->s, 0, sizeof(double) * (kKrylov + 1), st));
    INS_CK(cudaMemsetAsync(&s->st->ticket, 0, sizeof(unsigned int), st));
    k_gm_init<<<s->nGrid, kThreads, 0, st>>>(G);
    for (int step = 0; step < kKrylov;) {
        for (int k = 0; k < kStepsPerSync && step < kKrylov; ++k, ++step) {
            k_gm_spmv_dots<<<s->nChunkBlk, kThreads, 0, st>>>(G);
            k_gm_orth<<<s->nGrid, kThreads, 0, st>>>(G);
        }
        INS_CK(cudaGetLastError());
        INS_CK(cudaMemcpyAsync(s->hst, s->st, sizeof(GmState), cudaMemcpyDeviceToHost, st));
        INS_CK(cudaStreamSynchronize(st));
        if (s->hst->done) break;
    }
    if (!s->hst->done) return s->fail(OFG_E_STATE, "GMRES did not finish");
    if (s->hst->dim >= 0) {
        k_gm_backsub<<<1, kThreads, 0, st>>>(G);
        k_gm_update_x<<<s->nGrid, kThreads, 0, st>>>(G);
        k_gm_residual<<<s->nGrid, kThreads, 0, st>>>(G);
        INS_CK(cudaGetLastError());
        INS_CK(cudaMemcpyAsync(s->hst, s->st, sizeof(GmState), cudaMemcpyDeviceToHost, st));
        INS_CK(cudaStreamSynchronize(st));
    }
    INS_CK(cudaEventRecord(s->eg1, st));
    INS_CK(cudaEventSynchronize(s->eg1));
    float ms = 0.f;
    INS_CK(cudaEventElapsedTime(&ms, s->eg0, s->eg1));
    s->gmresMs += ms;
    *its = s->hst->dim >= 0 ? s->hst->iters : 0;
    *res = s->hst->res;
    s->gmresTotal += *its;
    // algorithmic bytes: Krylov step j reads the matrix (values, columns,
    // row offsets), the previous vector, the j earlier basis vectors twice
    // (products, subtraction) and writes v_j, A v_j and the next vector; the
    // update reads dim + 1 basis vectors and writes x
    const double T = (double)s->D.nT, nnz = (double)s->nnz;
    const int steps = s->hst->dim >= 0 ? s->hst->dim + 1 : 0;
    for (int j = 0; j < steps; ++j) s->gmresBytes += nnz * 12.0 + T * 4.0 + T * 8.0 * (2.0 * j + 6.0);
    if (steps) s->gmresBytes += T * 8.0 * (steps + 1);
    return OFG_OK;
}

// one inner iteration (INsCalcRHS)
int inner(ofg_ins *s) {
    cudaStream_t st = s->c->stream;
    Dev &D = s->D;
    const bool first = s->innerSteps == 0;
    const int bF = blocks(D.nF), bT = blocks(D.nT), bB = blocks(D.nB > 0 ? D.nB : 1);
    if (first) k_ins_preflux<<<bF, kThreads, 0, st>>>(D);
    k_ins_grad<4><<<bT, kThreads, 0, st>>>(D, D.q + IU * D.nT, D.gx + IU * D.nT, D.gy + IU * D.nT, D.gz + IU * D.nT, 0);
    k_ins_face_coef<<<bF, kThreads, 0, st>>>(D);
    k_ins_momentum_rows<<<bT, kThreads, 0, st>>>(D, first ? 1 : 0);
    INS_CK(cudaGetLastError());
    int rc;
    for (int k = 0; k < 3; ++k)
        if ((rc = gmres(s, D.Am, D.bm + (size_t)k * D.nT, D.uc + (size_t)k * D.nT, &s->linIts[k], &s->linRes[k])))
            return rc;
    if (D.nB > 0) k_ins_wall_uc<<<bB, kThreads, 0, st>>>(D);
    k_ins_face_flux<<<bF, kThreads, 0, st>>>(D);
    k_ins_new_spc<<<bT, kThreads, 0, st>>>(D);
    k_ins_face_pcoef<<<bF, kThreads, 0, st>>>(D);
    k_ins_pressure_rows<<<bT, kThreads, 0, st>>>(D);
    INS_CK(cudaGetLastError());
    if ((rc = gmres(s, D.Ap, D.bp, D.pp, &s->linIts[3], &s->linRes[3]))) return rc;
    k_ins_p_update<<<bT, kThreads, 0, st>>>(D);
    k_ins_grad<1><<<bT, kThreads, 0, st>>>(D, D.pp, D.gq, D.gq + D.nT, D.gq + 2 * D.nT, 1);
    k_ins_speed<<<bT, kThreads, 0, st>>>(D);
    if (D.nF > D.nB) k_ins_face_update<<<blocks(D.nF - D.nB), kThreads, 0, st>>>(D);
    k_ins_residuals<<<bT, kThreads, 0, st>>>(D);
    INS_CK(cudaGetLastError());
    INS_CK(cudaMemcpyAsync(s->hred, D.red, 4 * sizeof(double), cudaMemcpyDeviceToHost, st));
    INS_CK(cudaStreamSynchronize(st));
    for (int k = 0; k < 4; ++k) s->remax[k] = s->hred[k];
    ++s->innerSteps;
    return OFG_OK;
}

void release(ofg_ins *s) {
    for (void *p : s->allocs) cudaFree(p);
    s->allocs.clear();
    if (s->hst) cudaFreeHost(s->hst);
    if (s->hred) cudaFreeHost(s->hred);
    for (cudaEvent_t e : {s->ev0, s->ev1, s->eg0, s->eg1})
        if (e) cudaEventDestroy(e);
}

}  // namespace

extern "C" {

int ofg_ins_create(ofg_ctx *c, const double *wall_uvw, ofg_ins **out) {
    if (!out) return OFG_E_ARG;
    *out = nullptr;
    if (!c) return OFG_E_ARG;
    if (!c->haveMesh) return c->fail(OFG_E_STATE, "ins: no mesh");
    const int nC = c->nCells, nB = c->nBFaces, nF = c->nFaces, nT = c->nT;
    for (int f = 0; f < nB; ++f)
        if (c->bct[f] != OFG_BC_SOLID_SURFACE)
            return c->fail(OFG_E_ARG, "ins: every boundary face must be SOLID_SURFACE");
    if (c->p.vismodel < 1) return c->fail(OFG_E_ARG, "ins: a viscous model is required");
    if (!(c->p.global_dt > 0.0) || !(c->p.reynolds > 0.0)) return c->fail(OFG_E_ARG, "ins: global_dt, reynolds");
    ofg_ins *s = new ofg_ins();
    s->c = c;
    Dev &D = s->D;
    D.nF = nF; D.nB = nB; D.nC = nC; D.nT = nT;
    D.dt = c->p.global_dt;
    D.vis = 1 / c->p.reynolds;
    // face records (the per-face geometry of CalcFaceVisterm, CalcPreandVisGrad,
    // CalcPreGrad and CalcINsFaceflux, formed with their expressions)
    std::vector<double> fr((size_t)nF * kFR, 0.0);
    for (int f = 0; f < nF; ++f) {
        const int l = c->lc[f], r = c->rc[f];
        double *g = &fr[(size_t)f * kFR];
        const double xn = c->xfn[f], yn = c->yfn[f], zn = c->zfn[f], area = c->area[f];
        g[F_XN] = xn; g[F_YN] = yn; g[F_ZN] = zn; g[F_AREA] = area;
        g[F_DIST] = xn * (c->xcc[r] - c->xcc[l]) + yn * (c->ycc[r] - c->ycc[l]) + zn * (c->zcc[r] - c->zcc[l]);
        g[F_LX] = c->xcc[r] - c->xcc[l]; g[F_LY] = c->ycc[r] - c->ycc[l]; g[F_LZ] = c->zcc[r] - c->zcc[l];
        const double dx1 = c->xfc[f] - c->xcc[l], dy1 = c->yfc[f] - c->ycc[l], dz1 = c->zfc[f] - c->zcc[l];
        const double dx2 = c->xfc[f] - c->xcc[r], dy2 = c->yfc[f] - c->ycc[r], dz2 = c->zfc[f] - c->zcc[r];
        g[F_DX1] = dx1; g[F_DY1] = dy1; g[F_DZ1] = dz1;
        g[F_DX2] = c->xcc[r] - c->xfc[f]; g[F_DY2] = c->ycc[r] - c->yfc[f]; g[F_DZ2] = c->zcc[r] - c->zfc[f];
        const double d1 = std::sqrt(dx1 * dx1 + dy1 * dy1 + dz1 * dz1);
        const double d2 = std::sqrt(dx2 * dx2 + dy2 * dy2 + dz2 * dz2);
        const double de = 1.0 / (d1 + d2);
        g[F_W1] = d2 * de; g[F_W2] = d1 * de;
        const double de2 = 1.0 / (d1 + d2 + kSmall);
        g[F_G1] = d2 * de2; g[F_G2] = d1 * de2;
        g[F_FN] = D.vis * area / g[F_DIST];
        g[F_NXA] = xn * area; g[F_NYA] = yn * area; g[F_NZA] = zn * area;
    }
    // per-cell faces in ascending id (CellTopo::CalcC2f, codes/geometry/src/CellTopo.cpp:95-119),
    // side in bit 0; matrix rows: those entries and the diagonal (ghost rows: diagonal only)
    std::vector<int> cnt(nC + 1, 0), cOff(nC + 1, 0);
    for (int f = 0; f < nB; ++f) ++cnt[c->lc[f]];
    for (int f = nB; f < nF; ++f) { ++cnt[c->lc[f]]; ++cnt[c->rc[f]]; }
    for (int i = 0; i < nC; ++i) cOff[i + 1] = cOff[i] + cnt[i];
    std::vector<int> cFace(cOff[nC]), pos(cOff.begin(), cOff.end() - 1);
    for (int f = 0; f < nB; ++f) cFace[pos[c->lc[f]]++] = f << 1;
    for (int f = nB; f < nF; ++f) { cFace[pos[c->lc[f]]++] = f << 1; cFace[pos[c->rc[f]]++] = (f << 1) | 1; }
    std::vector<int> rOff(nT + 1, 0), JA;
    for (int i = 0; i < nT; ++i) rOff[i + 1] = rOff[i] + (i < nC ? cnt[i] : 0) + 1;
    JA.resize(rOff[nT]);
    for (int i = 0; i < nT; ++i) {
        int n = rOff[i], k = 0;
        if (i < nC)
            for (int e = cOff[i]; e < cOff[i + 1]; ++e, ++k) {
                const int f = cFace[e] >> 1;
                JA[n + k] = (cFace[e] & 1) ? c->lc[f] : c->rc[f];
            }
        JA[n + k] = i;
    }
    std::vector<double> wall((size_t)nB * 3, 0.0);
    if (wall_uvw) std::memcpy(wall.data(), wall_uvw, wall.size() * sizeof(double));
    int rc = OFG_OK;
    auto up_i = [&](const int **d, const std::vector<int> &h) {
        int *p = nullptr;
        if (!rc) rc = s->alloc(&p, h.size());
        if (!rc && !h.empty() && cudaMemcpy(p, h.data(), h.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
            rc = OFG_E_CUDA;
        *d = p;
    };
    auto up_d = [&](const double **d, const std::vector<double> &h) {
        double *p = nullptr;
        if (!rc) rc = s->alloc(&p, h.size());
        if (!rc && !h.empty() && cudaMemcpy(p, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
            rc = OFG_E_CUDA;
        *d = p;
    };
    std::vector<int> lcv(c->lc.begin(), c->lc.begin() + nF), rcv(c->rc.begin(), c->rc.begin() + nF);
    up_i(&D.lc, lcv); up_i(&D.rc, rcv);
    up_d(&D.fr, fr);
    std::vector<double> volv(c->vol.begin(), c->vol.begin() + nT);
    up_d(&D.vol, volv);
    up_i(&D.cOff, cOff); up_i(&D.cFace, cFace); up_i(&D.rOff, rOff); up_i(&D.JA, JA);
    up_d(&D.wall, wall);
    const size_t T = nT, F = nF;
    auto z = [&](double **p, size_t n) { if (!rc) rc = s->alloc(p, n); };
    z(&D.q, 5 * T); z(&D.gx, 5 * T); z(&D.gy, 5 * T); z(&D.gz, 5 * T);
    z(&D.rf, F); z(&D.uf, F); z(&D.vf, F); z(&D.wf, F); z(&D.fq, F); z(&D.ai0, F); z(&D.ai1, F); z(&D.bi, 6 * F);
    z(&D.Vdv, F); z(&D.ajp, F);
    z(&D.spt, T); z(&D.bt, 3 * T); z(&D.up, 3 * T); z(&D.spc, T); z(&D.bm, 3 * T); z(&D.uc, 3 * T);
    z(&D.spp, T); z(&D.bp, T); z(&D.pp, T); z(&D.VdU, T); z(&D.gq, 3 * T); z(&D.mu, 3 * (size_t)nC);
    z(&D.Am, rOff[nT]); z(&D.Ap, rOff[nT]);
    z(&D.part, 4 * (size_t)blocks(nT)); z(&D.red, 4);
    if (!rc) rc = s->alloc(&D.ticket, 1);
    // blocks of k_gm_spmv_dots: at most one resident wave (three per SM) taking
    // the 256-row chunks in grid stride, as few as give every block the same
    // number of chunks (a last round of a few blocks leaves most SMs idle)
    {
        const int nChunks = (nT + kChunk - 1) / kChunk, slots = 148 * 3;
        const int rounds = (nChunks + slots - 1) / slots;
        s->nChunkBlk = (nChunks + rounds - 1) / rounds;
    }
    s->nGrid = std::min(blocks(nT), 148 * 8);
    s->nPart = std::max(s->nChunkBlk * (kKrylov + 1), s->nGrid);
    z(&s->V, (size_t)(kKrylov + 1) * T); z(&s->W, T); z(&s->Y, T);
    z(&s->H, (size_t)(kKrylov + 1) * kKrylov); z(&s->gc, kKrylov); z(&s->gs, kKrylov); z(&s->s, kKrylov + 1);
    z(&s->gpart, (size_t)s->nPart);
    if (!rc) rc = s->alloc(&s->st, 1);
    if (!rc && cudaMallocHost((void **)&s->hst, sizeof(GmState)) != cudaSuccess) rc = OFG_E_NOMEM;
    if (!rc && cudaMallocHost((void **)&s->hred, 4 * sizeof(double)) != cudaSuccess) rc = OFG_E_NOMEM;
    if (!rc && (cudaEventCreate(&s->ev0) != cudaSuccess || cudaEventCreate(&s->ev1) != cudaSuccess ||
                cudaEventCreate(&s->eg0) != cudaSuccess || cudaEventCreate(&s->eg1) != cudaSuccess))
        rc = OFG_E_CUDA;
    s->nnz = rOff[nT];
    if (!rc && (cudaMemset(D.ticket, 0, sizeof(unsigned)) != cudaSuccess ||
                cudaMemset(s->st, 0, sizeof(GmState)) != cudaSuccess ||
                cudaMemset(D.mu, 0, 3 * (size_t)nC * sizeof(double)) != cudaSuccess))
        rc = OFG_E_CUDA;
    if (rc) {
        release(s);
        delete s;
        return c->fail(rc, "ins: device allocation or upload failed");
    }
    *out = s;
    return OFG_OK;
}

void ofg_ins_destroy(ofg_ins *s) {
    if (!s) return;
    cudaStreamSynchronize(s->c->stream);
    release(s);
    delete s;
}

int ofg_ins_init_flowfield(ofg_ins *s) {
    if (!s) return OFG_E_ARG;
    ofg_ctx *c = s->c;
    const int nT = s->D.nT, nB = s->D.nB;
    // the reference state (codes/chemical/src/Chemical.cpp:280-325)
    const double statecoef = 1.0 / (c->p.gama_ref * (c->p.mach_ref * c->p.mach_ref));
    const double pi = 3.141592653589793;
    const double aoa = c->p.aoa_degree * pi / 180.0, aos = c->p.sideslip_degree * pi / 180.0;
    const double inflow[5] = {1.0, 1.0 * std::cos(aoa) * std::cos(aos), 1.0 * std::sin(aoa) * std::cos(aos),
                              1.0 * std::sin(aos), statecoef * 1.0 * 1.0 / 1.0};
    std::vector<double> q((size_t)5 * nT);
    for (int e = 0; e < 5; ++e) std::fill(q.begin() + (size_t)e * nT, q.begin() + (size_t)(e + 1) * nT, inflow[e]);
    std::vector<double> wall((size_t)nB * 3);
    INS_CK(cudaMemcpy(wall.data(), s->D.wall, wall.size() * sizeof(double), cudaMemcpyDeviceToHost));
    for (int f = 0; f < nB; ++f) {   // AdiabaticVisWallBc / VelocityBc (codes/ins/src/INsBcSolver.cpp:329-367)
        const int l = c->lc[f], r = c->rc[f];
        for (int e = 0; e < 5; ++e) q[(size_t)e * nT + r] = q[(size_t)e * nT + l];
        for (int k = 0; k < 3; ++k)
            q[(size_t)(IU + k) * nT + r] = -q[(size_t)(IU + k) * nT + r] + 2.0 * wall[3 * f + k];
    }
    return ofg_ins_upload_state(s, q.data());
}

int ofg_ins_upload_state(ofg_ins *s, const double *q) {
    if (!s || !q) return OFG_E_ARG;
    const int nT = s->D.nT;
    INS_CK(cudaStreamSynchronize(s->c->stream));
    INS_CK(cudaMemcpy(s->D.q, q, (size_t)5 * nT * sizeof(double), cudaMemcpyHostToDevice));
    INS_CK(cudaMemset(s->D.mu, 0, 3 * (size_t)s->D.nC * sizeof(double)));
    INS_CK(cudaMemset(s->D.gx, 0, 5 * (size_t)nT * sizeof(double)));
    INS_CK(cudaMemset(s->D.gy, 0, 5 * (size_t)nT * sizeof(double)));
    INS_CK(cudaMemset(s->D.gz, 0, 5 * (size_t)nT * sizeof(double)));
    s->innerSteps = 0;
    s->ms = 0.0;
    s->gmresMs = 0.0;
    s->gmresBytes = 0.0;
    s->gmresTotal = 0;
    for (int k = 0; k < 4; ++k) { s->remax[k] = 1; s->linIts[k] = 0; s->linRes[k] = 0; }
    return OFG_OK;
}

int ofg_ins_update_residuals(ofg_ins *s) {
    if (!s) return OFG_E_ARG;
    cudaStream_t st = s->c->stream;
    INS_CK(cudaEventRecord(s->ev0, st));
    int rc = inner(s);
    if (rc) return rc;
    INS_CK(cudaEventRecord(s->ev1, st));
    INS_CK(cudaEventSynchronize(s->ev1));
    float ms = 0.f;
    INS_CK(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
    s->ms += ms;
    return OFG_OK;
}

int ofg_ins_run(ofg_ins *s, int max_inner, int *ran) {
    if (!s) return OFG_E_ARG;
    int n = 0, rc = OFG_OK;
    while ((s->remax[0] > 1e-8 || s->remax[1] > 1e-8 || s->remax[2] > 1e-8) && s->innerSteps < max_inner) {
        if ((rc = ofg_ins_update_residuals(s))) break;
        ++n;
    }
    if (ran) *ran = n;
    return rc;
}

int ofg_ins_stats(ofg_ins *s, double *out) {
    if (!s || !out) return OFG_E_ARG;
    for (int k = 0; k < 4; ++k) { out[k] = s->remax[k]; out[4 + k] = s->linIts[k]; out[8 + k] = s->linRes[k]; }
    out[12] = (double)s->innerSteps;
    return OFG_OK;
}

int ofg_ins_timing(ofg_ins *s, double *out) {
    if (!s || !out) return OFG_E_ARG;
    out[0] = s->ms;
    out[1] = (double)s->gmresTotal;
    out[2] = s->gmresMs;
    out[3] = s->gmresBytes;
    return OFG_OK;
}

int ofg_ins_get_field(ofg_ins *s, const char *name, double *out, int64_t n) {
    if (!s || !name || !out) return OFG_E_ARG;
    const Dev &D = s->D;
    const size_t T = D.nT, F = D.nF;
    const double *src = nullptr;
    size_t cnt = 0;
    std::string k(name);
    if (k == "q") { src = D.q; cnt = 5 * T; }
    else if (k == "dqdx") { src = D.gx; cnt = 5 * T; }
    else if (k == "dqdy") { src = D.gy; cnt = 5 * T; }
    else if (k == "dqdz") { src = D.gz; cnt = 5 * T; }
    else if (k == "pp") { src = D.pp; cnt = T; }
    else if (k == "uc") { src = D.uc; cnt = T; }
    else if (k == "vc") { src = D.uc + T; cnt = T; }
    else if (k == "wc") { src = D.uc + 2 * T; cnt = T; }
    else if (k == "spc") { src = D.spc; cnt = T; }
    else if (k == "bp") { src = D.bp; cnt = T; }
    else if (k == "fq") { src = D.fq; cnt = F; }
    else if (k == "ajp") { src = D.ajp; cnt = F; }
    else return s->fail(OFG_E_ARG, "unknown field " + k);
    if (n < (int64_t)cnt) return OFG_E_SIZE;
    INS_CK(cudaStreamSynchronize(s->c->stream));
    INS_CK(cudaMemcpy(out, src, cnt * sizeof(double), cudaMemcpyDeviceToHost));
    return OFG_OK;
}

}  // extern "C"

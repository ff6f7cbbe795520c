// Spalart-Allmaras solver kernels (TURB_SOLVER tasks).  Same gather structure
// as the NS kernels: one thread per cell over its neighbour list in ascending
// face id, so every per-cell accumulation follows the reference's face-loop
// order.  They read the NS state of the current buffer (already relaxed in
// this outer iteration, as in the reference's StrongIter order).
#pragma once
#include "ofg_kernels.cuh"

namespace ofg {

// CalcTurbulentViscosity: UTurbSrcFlux::CalcVist1Equ + TurbSrcFlux::CalcCellVist1Equ
// (codes/uturb/src/UTurbSrcFlux.cpp:220-241, codes/turb/src/TurbSrcFlux.cpp:279-290)
__device__ __forceinline__ double sa_vist(const DevParams &P, double rho, double nuet, double vl) {
    double olam = rho / (vl + SMALLD);
    double xsi = nuet * olam;
    double xsi3 = xsi * xsi * xsi;
    double fv1 = xsi3 / (xsi3 + P.sa_cv13);
    double v = fv1 * rho * nuet;
    return fmin(vl * P.max_vis_ratio, v);
}

// write the eddy viscosity of cell i into the master record and its FP32
// copy, rewriting whole 32-byte sectors (p T mu_l mu_t of the master, the
// whole copy) rather than single words
template <typename R>
__device__ __forceinline__ void put_vist(const KArgs<R> &A, int i, double v) {
    double2 *m = reinterpret_cast<double2 *>(const_cast<double *>(A.q) + (size_t)i * REC);
    double2 a = m[2], b = m[3];
    b.y = v;
    m[2] = a;
    m[3] = b;
    if (sizeof(R) == 4) {
        float4 *s = reinterpret_cast<float4 *>(const_cast<R *>(A.qs) + (size_t)i * REC);
        float4 s0 = s[0], s1 = s[1];
        s1.w = float(v);
        s[0] = s0;
        s[1] = s1;
    }
}

// TurbBcSolver face rules (codes/turb/src/TurbBcSolver.cpp:51-262); the
// far-field normal is scaled by GCom::faceOuterNormal, which the reference
// never assigns (zero-initialised global), so only the sound speeds decide.
template <typename R>
__global__ void __launch_bounds__(256) k_turb_bc(KArgs<R> A, const int *lcb, int withVist) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= A.nBFaces) return;
    int bt = A.bcType[f], l = lcb[f];
    int g = A.nCells + f;
    double s = A.nut[l], t = s;
    if (bt == BC_SOLID) t = -s;
    else if (bt == BC_INFLOW) t = A.P.nut_inf;
    else if (bt == BC_FAR) {
        const double *ql = A.q + (size_t)l * REC;
        const R *fg = A.fgeo + (size_t)f * FGR;
        double xn = double(fg[0]) * 0, yn = double(fg[1]) * 0, zn = double(fg[2]) * 0;
        const double *inf = A.P.inflow;
        double vnref = xn * inf[IU] + yn * inf[IV] + zn * inf[IW] - 0.0;
        double vnin = xn * ql[IU] + yn * ql[IV] + zn * ql[IW] - 0.0;
        double cref = sqrt(fabs(A.P.gama * inf[IP] / inf[IR]));
        double cin = sqrt(fabs(A.P.gama * ql[IP] / ql[IR]));
        double velin = sqrt(SQR3(ql[IU], ql[IV], ql[IW]));
        if (velin > cin) {
            t = vnin >= 0.0 ? s : A.P.nut_inf;
        } else {
            double gamm1 = A.P.gama - 1.0;
            double riemp = vnin + 2.0 * cin / gamm1;
            double riemm = vnref - 2.0 * cref / gamm1;
            double vnb = 0.5 * (riemp + riemm);
            t = vnb >= 0.0 ? s : A.P.nut_inf;
        }
    }
    A.nut[g] = t;
    if (withVist) put_vist(A, g, A.q[(size_t)l * REC + IMT]);   // UTurbSrcFlux::SetGhostCellVist
}

// gradient of nu~ (uturb_grad: Green-Gauss cell-weighted for igrad 0, or the
// option chosen for the NS gradients); ghosts carry the interior gradient
template <typename R>
__global__ void __launch_bounds__(128) k_turb_grad(KArgs<R> A) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= A.nCells) return;
    R cgc[CGR];
    ld4(A.cgeo + (size_t)c * CGR, cgc);
    R gx = 0, gy = 0, gz = 0;
    int b = A.nb_off[c], e = A.nb_off[c + 1];
    R vc = R(A.nut[c]);
    if constexpr (sizeof(R) == 4) {
        // mixed path: the differences nu~_nb - nu~_c formed in FP64 and the
        // face-local geometry (distances and least-squares terms formed in
        // FP64 at upload), as the NS gradient of this path; absolute FP32
        // coordinates lose the thin near-wall cells' offsets
        const double nc = A.nut[c];
        if (A.P.igrad == 2) {
            R a11 = 0, a12 = 0, a13 = 0, a22 = 0, a23 = 0, a33 = 0, b1 = 0, b2 = 0, b3 = 0;
            for (int k = b; k < e; ++k) {
                const int2 e2 = __ldg(&A.nbl[k]);
                const R dv = R(A.nut[e2.y] - nc);
                // x_nb - x_c = (x_f - x_c) - (x_f - x_nb), from the face's offsets
                float fo[FOFS];
                ld8(A.fofs + (size_t)nb_face(e2) * FOFS, fo);
                const R sg = nb_right(e2) ? R(-1) : R(1);
                const R dx = sg * (fo[0] - fo[3]), dy = sg * (fo[1] - fo[4]), dz = sg * (fo[2] - fo[5]);
                const R w = R(1) / (dx * dx + dy * dy + dz * dz);
                a11 += w * dx * dx; a12 += w * dx * dy; a13 += w * dx * dz;
                a22 += w * dy * dy; a23 += w * dy * dz; a33 += w * dz * dz;
                b1 += w * dx * dv; b2 += w * dy * dv; b3 += w * dz * dv;
            }
            if (A.P.dim == 2) {
                R id = R(1) / (a11 * a22 - a12 * a12);
                gx = (a22 * b1 - a12 * b2) * id; gy = (a11 * b2 - a12 * b1) * id; gz = R(0);
            } else {
                R c11 = a22 * a33 - a23 * a23, c12 = a13 * a23 - a12 * a33, c13 = a12 * a23 - a13 * a22;
                R c22 = a11 * a33 - a13 * a13, c23 = a12 * a13 - a11 * a23, c33 = a11 * a22 - a12 * a12;
                R id = R(1) / (a11 * c11 + a12 * c12 + a13 * c13);
                gx = (c11 * b1 + c12 * b2 + c13 * b3) * id;
                gy = (c12 * b1 + c22 * b2 + c23 * b3) * id;
                gz = (c13 * b1 + c23 * b2 + c33 * b3) * id;
            }
        } else {
            for (int k = b; k < e; ++k) {
                const int2 e2 = __ldg(&A.nbl[k]);
                const int f = nb_face(e2);
                const bool right = nb_right(e2);
                R fg[4];
                ld4(A.fgeo + (size_t)f * FGR, fg);   // normal and area
                R wn;
                if (A.P.igrad == 1) {
                    wn = R(0.5);
                } else {   // |x_f - x_L|, |x_f - x_R| formed in FP64
                    const float2 dd = __ldg(reinterpret_cast<const float2 *>(A.fofs + (size_t)f * FOFS + 6));
                    const R delta = R(1) / (dd.x + dd.y + small_v<R>());
                    wn = right ? dd.y * delta : dd.x * delta;
                }
                // the face value less the cell's own (which sums to zero over
                // the closed cell surface)
                const R value = wn * R(A.nut[e2.y] - nc);
                const R ar = fg[3];
                const R fx = fg[0] * ar, fy = fg[1] * ar, fz = fg[2] * ar;
                if (!right) { gx += fx * value; gy += fy * value; gz += fz * value; }
                else        { gx -= fx * value; gy -= fy * value; gz -= fz * value; }
            }
            const R ovol = R(1) / cgc[3];
            gx *= ovol; gy *= ovol; gz *= ovol;
        }
    } else if (A.P.igrad == 2) {
        R a11 = 0, a12 = 0, a13 = 0, a22 = 0, a23 = 0, a33 = 0, b1 = 0, b2 = 0, b3 = 0;
        for (int k = b; k < e; ++k) {
            int nb = __ldg(&A.nbl[k]).y;
            R cgn[CGR];
            ld4(A.cgeo + (size_t)nb * CGR, cgn);
            R dx = cgn[0] - cgc[0], dy = cgn[1] - cgc[1], dz = cgn[2] - cgc[2];
            R w = R(1) / (dx * dx + dy * dy + dz * dz);
            R dv = R(A.nut[nb]) - vc;
            a11 += w * dx * dx; a12 += w * dx * dy; a13 += w * dx * dz;
            a22 += w * dy * dy; a23 += w * dy * dz; a33 += w * dz * dz;
            b1 += w * dx * dv; b2 += w * dy * dv; b3 += w * dz * dv;
        }
        if (A.P.dim == 2) {
            R id = R(1) / (a11 * a22 - a12 * a12);
            gx = (a22 * b1 - a12 * b2) * id; gy = (a11 * b2 - a12 * b1) * id; gz = R(0);
        } else {
            R c11 = a22 * a33 - a23 * a23, c12 = a13 * a23 - a12 * a33, c13 = a12 * a23 - a13 * a22;
            R c22 = a11 * a33 - a13 * a13, c23 = a12 * a13 - a11 * a23, c33 = a11 * a22 - a12 * a12;
            R id = R(1) / (a11 * c11 + a12 * c12 + a13 * c13);
            gx = (c11 * b1 + c12 * b2 + c13 * b3) * id;
            gy = (c12 * b1 + c22 * b2 + c23 * b3) * id;
            gz = (c13 * b1 + c23 * b2 + c33 * b3) * id;
        }
    } else {
        for (int k = b; k < e; ++k) {
            int2 e2 = __ldg(&A.nbl[k]);
            int f = nb_face(e2), nb = e2.y;
            bool right = nb_right(e2);
            R cgn[CGR], fg[FGR];
            ld4(A.cgeo + (size_t)nb * CGR, cgn);
            ld8(A.fgeo + (size_t)f * FGR, fg);
            R vn = R(A.nut[nb]);
            R vl = right ? vn : vc, vr = right ? vc : vn;
            const R *cl_ = right ? cgn : cgc, *cr_ = right ? cgc : cgn;
            R cl, cr;
            if (A.P.igrad == 1) { cl = R(0.5); cr = R(0.5); }
            else {
                R dxl = fg[4] - cl_[0], dyl = fg[5] - cl_[1], dzl = fg[6] - cl_[2];
                R dxr = fg[4] - cr_[0], dyr = fg[5] - cr_[1], dzr = fg[6] - cr_[2];
                R delt1 = Rsqrt(SQR3(dxl, dyl, dzl)), delt2 = Rsqrt(SQR3(dxr, dyr, dzr));
                R delta = R(1) / (delt1 + delt2 + small_v<R>());
                cl = delt2 * delta; cr = delt1 * delta;
            }
            R value = (A.P.igrad == 1) ? R(0.5) * (vl + vr) : cl * vl + cr * vr;
            R ar = fg[3];
            R fx = fg[0] * ar, fy = fg[1] * ar, fz = fg[2] * ar;
            if (!right) { gx += fx * value; gy += fy * value; gz += fz * value; }
            else        { gx -= fx * value; gy -= fy * value; gz -= fz * value; }
        }
        R ovol = R(1) / cgc[3];
        gx *= ovol; gy *= ovol; gz *= ovol;
    }
    R o[4] = {gx, gy, gz, R(0)};
    st4(A.gnut + (size_t)c * 4, o);
}

template <typename R>
__device__ __forceinline__ R calc_angle(R dx, R dy, R dz, R dist) {
    // VisGradGeom::CalcAngle, codes/usolver/src/VisGrad.cpp:62-68
    R result = dist / (Rsqrt(SQR3(dx, dy, dz)) + small_v<R>());
    if (result > R(1)) result = R(1);
    if (result < R(-1)) result = R(-1);
    if (sizeof(R) == 4) return R(asinf(float(result)) * 57.29577951f);
    return R(asin(double(result)) * 180.0 / 3.141592653589793);
}

// UPDATE_RESIDUALS for SA: TurbCalcRHS (codes/turb/src/TurbRhs.cpp:57-70):
// spectrum (UTurbSpectrum::CalcSpectrum1Equ + TurbSpectrum::CalcFaceSpectrum1Equ,
// codes/uturb/src/UTurbSpectrum.cpp:132-240, codes/turb/src/TurbSpectrum.cpp:75-134),
// source (TurbCom::CalcSrcSa, codes/turb/src/TurbCom.cpp:771-881), first-order
// convection (TurbInvFlux::RoeFlux, codes/turb/src/TurbInvFlux.cpp:78-98) and
// diffusion with the VIS_TEST face gradient (UTurbVisFlux, codes/uturb/src/UTurbVisFlux.cpp:64-407).
// The FP64 path keeps the reference's three face passes (spectrum, convection,
// diffusion) in order; the FP32 path fuses them into one pass with separate
// FP64 accumulators that are added in the reference's order at the end.
// The SA source of cell c (TurbCom::CalcSrcSa, codes/turb/src/TurbCom.cpp:771-881)
// and its implicit part: adds the source x volume to acc and its linearised
// part x volume to imp (gnc: the cell's gradient of nu~).
template <typename R>
__device__ __forceinline__ void sa_source(const KArgs<R> &A, int c, double nutc, double vol, const R *gnc,
                                          double &imp, double &acc) {
    const DevParams &P = A.P;
    const double half = 0.5;
    double dudx, dudy, dudz, dvdx, dvdy, dvdz, dwdx, dwdy, dwdz;
    {
        R gq[GLR];
#pragma unroll
        for (int i = 0; i < 12; i += 4) ld4(A.gl + (size_t)c * GLR + i, gq + i);
        dudx = gq[IU * 3]; dudy = gq[IU * 3 + 1]; dudz = gq[IU * 3 + 2];
        dvdx = gq[IV * 3]; dvdy = gq[IV * 3 + 1]; dvdz = gq[IV * 3 + 2];
        dwdx = gq[IW * 3]; dwdy = gq[IW * 3 + 1]; dwdz = gq[IW * 3 + 2];
    }
    double rho = A.q[(size_t)c * REC + IR], nuet = nutc, vlc = A.q[(size_t)c * REC + IML];
    double olam = rho / (vlc + SMALLD);
    double ls = A.walldist[c];
    double od2 = 1.0 / (ls * ls);
    double work1 = dudx + dvdy + dwdz;
    double work2 = SQR3(dudx, dudy, dudz);
    double work3 = SQR3(dudy + dvdx, dvdz + dwdy, dwdx + dudz);
    double work4 = sqrt(SQR3(dwdy - dvdz, dudz - dwdx, dvdx - dudy));
    if (P.iprod_sa == 1) {
        double stp = 2.0 * work2 + work3 - (2.0 / 3.0) * work1 * work1;
        work4 = sqrt(fabs(stp));
    } else if (P.iprod_sa == 4) {
        double stp = 2.0 * work2 + work3 - (2.0 / 3.0) * work1 * work1;
        double str = work4;
        work4 = str - 2.0 * fmax(0.0, str - sqrt(fabs(stp)));
    } else if (P.iprod_sa == 5) {
        double stp = fabs(2.0 * work2 + work3 - (2.0 / 3.0) * work1 * work1);
        double str = work4;
        work4 = str * (1.0 - fmax(0.0, (str * str - stp) / (str * str + stp + SMALLD)));
    }
    double str = work4;
    double xsi = nuet * olam + SMALLD;
    double xsi3 = xsi * xsi * xsi;
    double fv1 = xsi3 / (xsi3 + P.sa_cv13);
    double fv2 = 1.0 - xsi / (1.0 + xsi * fv1);
    double rs = nuet * P.sa_okarm2 * od2 * P.oreynolds;
    double nuetRs = nuet * rs;
    double sBar = rs * fv2;
    double omega = str;
    double stdv;
    if (sBar >= -P.sa_sac2 * omega) stdv = omega + sBar;
    else {
        double term1 = (P.sa_sac2 * P.sa_sac2 * omega + P.sa_sac3 * sBar);
        double term2 = (P.sa_sac3 - 2 * P.sa_sac2) * omega - sBar;
        stdv = omega + omega * term1 / term2;
    }
    double ostd = 1.0 / (stdv + SMALLD);
    double rr = fmin(rs * ostd, 10.0);
    double r5 = pow(rr, 5.0);
    double g = rr + P.sa_cw2 * (r5 * rr - rr);
    double g6 = pow(g, 6.0);
    double fw = g * pow((1.0 + P.sa_cw36) / (g6 + P.sa_cw36), 1.0 / 6.0);
    double xsi2 = xsi * xsi;
    double ft2 = P.ft2_flag ? P.sa_ct3 * exp(-P.sa_ct4 * xsi2) * 1.0 : 0.0;
    double grd2 = SQR3(double(gnc[0]), double(gnc[1]), double(gnc[2]));
    double prod = P.sa_cb1 * (1.0 - ft2) * stdv * nuet;
    double diff = P.sa_cb2s * grd2 * P.oreynolds;
    double dest = (P.sa_cw1k * fw - P.sa_cb1 * ft2) * nuetRs;
    diff = fmin(P.rprod * prod, diff);
    double srcTerm = prod - dest;
    srcTerm += diff;
    double q1x = fv1 / (xsi + SMALLD), q1y = 1.0 + xsi * fv1;
    double dfv2dk = (3.0 * P.sa_cv13 * (q1x * q1x) - 1.0) / (q1y * q1y);
    double dsdnu = P.oreynolds * P.sa_okarm2 * od2 * (fv2 + xsi * dfv2dk);
    double dfwdg = fw / (g + SMALLD) * (1.0 - g6 / (g6 + P.sa_cw36));
    double dgdr = 1.0 + P.sa_cw2 * (6.0 * r5 - 1.0);
    double drdnu = P.oreynolds * P.sa_okarm2 * od2 * ostd * (1.0 - nuet * ostd * dsdnu);
    double dfwdnu = dfwdg * dgdr * drdnu;
    double prod0 = P.sa_cb1 * (1.0 - ft2) * stdv;
    double dest0 = (P.sa_cw1 * fw - P.sa_cb1 * ft2 * P.sa_okarm2) * nuet * od2 * P.oreynolds;
    double prodp = P.sa_cb1 * ((1.0 - ft2) * dsdnu);
    double destp = (P.sa_cw1 * (fw + dfwdnu * nuet) - P.sa_cb1 * ft2 * P.sa_okarm2) * od2 * P.oreynolds;
    double prde0 = prod0 - dest0, prdep = prodp - destp;
    double part1 = -half * (prde0 - fabs(prde0));
    double part2 = -half * (prdep - fabs(prdep)) * nuet;
    imp += (part1 + part2) * vol;
    acc += srcTerm * vol;
}

template <typename R>
__device__ __forceinline__ double turb_rhs_cell(const KArgs<R> &A, int c) {
    constexpr bool exactOrder = sizeof(R) == 8;
    const DevParams &P = A.P;
    int b = A.nb_off[c], en = A.nb_off[c + 1];
    R qc[REC], cgc[CGR], gnc[4];
    ld8(A.qs + (size_t)c * REC, qc);
    ld4(A.cgeo + (size_t)c * CGR, cgc);
    ld4(A.gnut + (size_t)c * 4, gnc);
    double nutc = A.nut[c];
    double vol = double(cgc[3]);
    double imp = 0.0;
    imp += (1.0 / (A.dt[c] * P.turb_cfl_ratio)) * vol;
    double conv = 0.0, diffu = 0.0;   // FP32 path: per-pass accumulators
    double acc = -0.0;
    // FP64: pass 0 spectrum, then the source, pass 1 convection, pass 2
    // diffusion (the TurbCalcRHS order)
    for (int pass = 0; pass < (exactOrder ? 3 : 1); ++pass) {
        int2 e2n = b < en ? __ldg(&A.nbl[b]) : make_int2(0, 0);   // list entry one face ahead
        for (int k = b; k < en; ++k) {
            int2 e2 = e2n;
            if (k + 1 < en) e2n = __ldg(&A.nbl[k + 1]);
            int f = nb_face(e2), nb = e2.y;
            bool right = nb_right(e2);
            R qn[REC], cgn[CGR], fg[FGR];
            ld8(A.qs + (size_t)nb * REC, qn);
            ld8(A.fgeo + (size_t)f * FGR, fg);
            ld4(A.cgeo + (size_t)nb * CGR, cgn);
            const R *ql = right ? qn : qc, *qr = right ? qc : qn;
            const R *cgl = right ? cgn : cgc, *cgr = right ? cgc : cgn;
            // face terms at the face precision (FP64 path: the reference's
            // arithmetic), accumulated in FP64
            R nutn = R(A.nut[nb]), nutcR = R(nutc);
            R nl = right ? nutn : nutcR, nr = right ? nutcR : nutn;
            R xn = fg[0], yn = fg[1], zn = fg[2], ar = fg[3];
            const R hf = R(0.5);
            if (!exactOrder || pass == 0) {
                // ---- spectral radius and sweep coefficients ----
                R vnl = xn * ql[IU] + yn * ql[IV] + zn * ql[IW] - R(0);
                R vnr = xn * qr[IU] + yn * qr[IV] + zn * qr[IW] - R(0);
                R absVn = Rabs(hf * (vnl + vnr));
                R r1 = R(0), m1 = R(0), m2 = R(0);
                r1 += ar * hf * absVn;
                m1 += ar * hf * (-vnl - absVn);
                m2 += ar * hf * (vnr - absVn);
                R orl = R(1) / (ql[IR] + small_v<R>()), orr = R(1) / (qr[IR] + small_v<R>());
                R nuet1 = ql[IML] * orl + nl, nuet2 = qr[IML] * orr + nr;
                R nueff = Rabs(hf * (nuet1 + nuet2));
                R ovol = R(1) / (hf * (cgl[3] + cgr[3]));
                R d = R(P.oreynolds) * ovol * (R(P.sa_osigma) * nueff * (ar * ar));
                r1 += d;
                m1 += -d;
                m2 += -d;
                imp += double(r1);
                if (!right) { A.matL[f] = double(m1); A.matR[f] = double(m2); }
            }
            if (!exactOrder || pass == 1) {
                // ---- first-order convection with the NS face states ----
                R t1 = nl, t2 = nr;
                R u1 = ql[IU], v1 = ql[IV], w1 = ql[IW], u2 = qr[IU], v2 = qr[IV], w2 = qr[IW];
                if (f < A.nBFaces) {
                    R tm = hf * (nl + nr);
                    t1 = t2 = tm;
                    if (A.bcType[f] == BC_SOLID) {
                        const double *bq = A.bcq + (size_t)f * NEQ;
                        u1 = u2 = R(bq[IU]); v1 = v2 = R(bq[IV]); w1 = w2 = R(bq[IW]);
                    } else {
                        u1 = u2 = hf * (ql[IU] + qr[IU]);
                        v1 = v2 = hf * (ql[IV] + qr[IV]);
                        w1 = w2 = hf * (ql[IW] + qr[IW]);
                    }
                }
                R vnl = xn * u1 + yn * v1 + zn * w1 - R(0);
                R vnr = xn * u2 + yn * v2 + zn * w2 - R(0);
                R coef_l = hf * (vnl + Rabs(vnl)) * R(1);
                R coef_r = hf * (vnr - Rabs(vnr)) * R(1);
                double v = double(ar * (coef_l * t1 + coef_r * t2));
                if (exactOrder) { if (!right) acc -= v; else acc += v; }
                else { if (!right) conv -= v; else conv += v; }
            }
            if (!exactOrder || pass == 2) {
                // ---- diffusion (VIS_TEST face gradient) ----
                R fxn = fg[0], fyn = fg[1], fzn = fg[2];
                R q1 = nl, q2 = nr;
                R q11 = q1, q22 = q2, qf = R(0.5) * (q1 + q2);
                R dxl, dyl, dzl, dxr, dyr, dzr;
                R e1, e2;   // FP32 path: q11 - qf and q22 - qf
                if constexpr (exactOrder) {
                    dxl = cgl[0] - fg[4]; dyl = cgl[1] - fg[5]; dzl = cgl[2] - fg[6];
                    dxr = cgr[0] - fg[4]; dyr = cgr[1] - fg[5]; dzr = cgr[2] - fg[6];
                } else {
                    // the cell centres seen from the face centre, formed in FP64
                    // (absolute FP32 coordinates lose thin cells' offsets), and
                    // q - qf from the FP64 difference of nu~ (its FP32 values
                    // would cancel where nu~ varies little)
                    float fo[FOFS];
                    ld8(A.fofs + (size_t)f * FOFS, fo);
                    dxl = -fo[0]; dyl = -fo[1]; dzl = -fo[2];
                    dxr = -fo[3]; dyr = -fo[4]; dzr = -fo[5];
                    const double nlD = right ? A.nut[nb] : nutc, nrD = right ? nutc : A.nut[nb];
                    e1 = R(0.5 * (nlD - nrD));
                    e2 = -e1;
                }
                R d1 = fxn * dxl + fyn * dyl + fzn * dzl;
                R d2 = fxn * dxr + fyn * dyr + fzn * dzr;
                R angle1 = calc_angle(dxl, dyl, dzl, -d1);
                R angle2 = calc_angle(dxr, dyr, dzr, d2);
                R dqdn = R(0);
                if (angle1 > R(20) && angle2 > R(20)) {
                    R gn[4];
                    bool ghost = nb >= A.nCells;
                    if (!ghost) ld4(A.gnut + (size_t)nb * 4, gn);
                    const R *g1 = right ? gn : gnc;
                    const R *g2 = (right || ghost) ? gnc : gn;
                    const R c1x = g1[0] * (fxn * d1 - dxl) + g1[1] * (fyn * d1 - dyl) + g1[2] * (fzn * d1 - dzl);
                    const R c2x = g2[0] * (fxn * d2 - dxr) + g2[1] * (fyn * d2 - dyr) + g2[2] * (fzn * d2 - dzr);
                    if constexpr (exactOrder) {
                        q11 += c1x;
                        q22 += c2x;
                        qf = R(0.5) * (q1 + q2);
                    } else {
                        e1 += c1x;
                        e2 += c2x;
                    }
                }
                if (angle1 > R(0) && angle2 > R(0) && Rabs(d1) > small_v<R>() && Rabs(d2) > small_v<R>()) {
                    R dtmp = d1 * d1 + d2 * d2;
                    R c1 = d1 * d1 / dtmp, c2 = R(1) - c1;
                    if (f < A.nBFaces) { c1 = R(1); c2 = R(0); }
                    if constexpr (exactOrder) dqdn = c1 * ((q11 - qf) / d1) + c2 * ((q22 - qf) / d2);
                    else dqdn = c1 * (e1 / d1) + c2 * (e2 / d2);
                }
                R orl = R(1) / (ql[IR] + small_v<R>()), orr = R(1) / (qr[IR] + small_v<R>());
                R visl_nv = hf * (ql[IML] * orl + qr[IML] * orr);
                R vist_nv = hf * (nl + nr);
                R comVis = (visl_nv + vist_nv) * R(P.sa_osigma);
                double flux = double(-R(P.oreynolds) * comVis * dqdn * ar);
                if (exactOrder) { if (!right) acc -= flux; else acc += flux; }
                else { if (!right) diffu -= flux; else diffu += flux; }
            }
        }
        if (pass == 0 || !exactOrder) sa_source(A, c, nutc, vol, gnc, imp, acc);   // per cell, after the spectrum
    }
    if (!exactOrder) { acc += conv; acc += diffu; }
    A.impsrT[c] = imp;
    A.resT[c] = acc;
    return acc;
}

// one thread per cell; the block leaves the sum of squares of its residuals
// for the norm
template <typename R>
__global__ void __launch_bounds__(128, MinBlocks<R>::tr) k_turb_rhs(KArgs<R> A) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    double sq = 0.0;
    if (c < A.nCells) {
        double r = turb_rhs_cell(A, c);
        sq = r * r;
    }
    block_sum_to<1>(&sq, A.tpart + blockIdx.x);
}


// LU-SGS sweeps of the SA equation (codes/uturb/src/UTurbLusgs.cpp:90-300,
// codes/turb/src/TurbLusgs.cpp:123-260): dfj = matrix * dq_j
template <typename R>
__device__ __forceinline__ void turb_lower_cell(const KArgs<R> &A, int c) {
    double rhs0 = 0.0;
    for (int k = A.lo_off[c]; k < A.lo_off[c + 1]; ++k) {
        int2 e2 = __ldg(&A.lol[k]);
        int f = nb_face(e2);
        rhs0 += (nb_right(e2) ? A.matL[f] : A.matR[f]) * A.dnut[e2.y];
    }
    A.dnut[c] = (A.resT[c] - rhs0) / A.impsrT[c];
}

template <typename R>
__device__ __forceinline__ void turb_upper_cell(const KArgs<R> &A, int c) {
    double rhs0 = 0.0;
    for (int k = A.up_off[c]; k < A.up_off[c + 1]; ++k) {   // ghost increments are zero: not listed
        int2 e2 = __ldg(&A.upl[k]);
        int f = nb_face(e2);
        rhs0 += (nb_right(e2) ? A.matL[f] : A.matR[f]) * A.dnut[e2.y];
    }
    A.dnut[c] = add_neg_quot(A.dnut[c], rhs0, A.impsrT[c]);
}

template <typename R>
__global__ void __launch_bounds__(128) k_turb_lower(KArgs<R> A, const int *order, int start, int count) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < count) turb_lower_cell(A, order[start + t]);
}

// the persistent forms (one block, every level, a barrier between levels; the
// increments are read with plain, coherent loads)
template <typename R>
__global__ void __launch_bounds__(kSeqThreads, 1) k_turb_lower_seq(KArgs<R> A, const int *order, const int *loff,
                                                                int nlev) {
    for (int l = 0; l < nlev; ++l) {
        const int st = loff[l], en = loff[l + 1];
        for (int k = st + threadIdx.x; k < en; k += blockDim.x) turb_lower_cell(A, order[k]);
        __syncthreads();
    }
}

template <typename R>
__global__ void __launch_bounds__(kSeqThreads, 1) k_turb_upper_seq(KArgs<R> A, const int *order, const int *loff,
                                                                int nlev) {
    for (int l = 0; l < nlev; ++l) {
        const int st = loff[l], en = loff[l + 1];
        for (int k = st + threadIdx.x; k < en; k += blockDim.x) turb_upper_cell(A, order[k]);
        __syncthreads();
    }
}

// UPDATE_FLOWFIELD (TurbUpdate::CalcFlowField1Equ, crelax = 1) fused with the
// interior half of CALC_BOUNDARY (the eddy viscosity of the new nu~)
template <typename R>
__device__ __forceinline__ void turb_update_cell(const KArgs<R> &A, int c, double dn, int withVist) {
    double qOld = A.nut[c], qNew = qOld + dn;
    double v = (1.0 - 1.0) * qOld + 1.0 * qNew;
    A.nut[c] = v;
    if (withVist) {
        const double *qc = A.q + (size_t)c * REC;
        put_vist(A, c, sa_vist(A.P, qc[IR], v, qc[IML]));
    }
}

template <typename R>
__global__ void __launch_bounds__(128) k_turb_upper(KArgs<R> A, const int *order, int start, int count) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < count) turb_upper_cell(A, order[start + t]);
}

template <typename R>
__global__ void __launch_bounds__(256) k_turb_update(KArgs<R> A, int withVist) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= A.nCells) return;
    turb_update_cell(A, c, A.dnut[c], withVist);
}

// interior eddy viscosity only (CALC_BOUNDARY without an update)
template <typename R>
__global__ void __launch_bounds__(256) k_turb_vist(KArgs<R> A) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= A.nCells) return;
    const double *qc = A.q + (size_t)c * REC;
    put_vist(A, c, sa_vist(A.P, qc[IR], A.nut[c], qc[IML]));
}

template <typename R>
__global__ void __launch_bounds__(256) k_turb_norm_final(KArgs<R> A, int nPartial, double *hist, int cap) {
    __shared__ double tot;
    if (grid_sum_last<1>(A.tpart, nPartial, A.red, A.redCount, &tot) && threadIdx.x == 0) {
        double rms = sqrt(tot / A.nCells);
        A.scal[S_TNORM] = rms;
        if (hist) {   // one more entry of the SA residual history
            int n = int(A.scal[S_THISTN]);
            if (n < cap) hist[n] = rms;
            A.scal[S_THISTN] = double(n + 1);
        }
    }
}

}  // namespace ofg

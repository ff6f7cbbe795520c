// Device-side data model and the per-face physics of the residual + LU-SGS
// path, for sm_100a.  Every function restates one reference routine (cited)
// with the same operation order as the reference's serial code, so that the
// FP64 build (compiled without FMA contraction) rounds like the reference.
// The arithmetic type R is double (FP64 path) or float (mixed path: face
// terms in FP32, accumulation in FP64 by the callers; the face states, the
// central part of the Roe flux and the gradient differences are formed in FP64
// from the FP64 state records, so that the FP32 rounding of the large
// low-Mach pressure and enthalpy terms sets no floor under the residual).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ofg {

constexpr double SMALLD = 1.0e-40;   // codes/basic/include/HXTypeBasic.h:34
constexpr int NEQ = 5;
constexpr int REC = 8;               // state record: rho u v w p T mul mut
enum { IR = 0, IU = 1, IV = 2, IW = 3, IP = 4, ITT = 5, IML = 6, IMT = 7 };
// Minimum resident 128-thread blocks per SM asked of the compiler for the
// FP32 gather kernels; caps their registers at 65536 / (128 n).  Chosen by
// timing the 6M-cell plate (no spills at these caps).  The FP64 kernels keep
// the compiler's choice.
#ifndef OFG_MINB_RES
#define OFG_MINB_RES 3
#endif
#ifndef OFG_MINB_GL
#define OFG_MINB_GL 6
#endif
#ifndef OFG_MINB_SW
#define OFG_MINB_SW 8
#endif
#ifndef OFG_MINB_TR
#define OFG_MINB_TR 8
#endif
#ifndef OFG_MINB_FP
#define OFG_MINB_FP 3
#endif
template <typename R> struct MinBlocks { enum { res = 1, gl = 1, sw = 1, tr = 1, fp = 1 }; };
template <> struct MinBlocks<float> {
    enum { res = OFG_MINB_RES, gl = OFG_MINB_GL, sw = OFG_MINB_SW, tr = OFG_MINB_TR, fp = OFG_MINB_FP };
};

constexpr int kRedBlocks = 148;   // blocks of the grid reductions (one per SM)
constexpr int kSeqThreads = 512;  // threads of the one block of a persistent (single-block) sweep

constexpr int GLR = 24;   // gradient+limiter record: [var*3+dir] for 6 vars (q, T), limiter at 18..22
constexpr int FGR = 8;    // face record: nx ny nz area xfc yfc zfc dist (|n . (x_r - x_l)|)
constexpr int CGR = 4;    // cell record: xcc ycc zcc vol
constexpr int DQR = 8;    // increment record: dq[5] + 3 zero slots (64 B FP64, 32 B FP32: whole sectors)
constexpr int MMR = 10;   // neighbour min/max differences per cell (Venkatakrishnan with the zone-wide eps)
constexpr int FOR = 6;    // face-pass record (mixed path): flux[5] FP64, then the inviscid and viscous
                          // spectral radii as two FP32 values in the sixth slot (48 B, three 16-B words)
constexpr int FOFS = 8;   // face-local offsets record (mixed path), FP32

// slots of the small device scalar array (cfl, min dt, limiter eps, norms,
// outer-step counter, residual-history length)
enum { S_CFL = 0, S_MINDT = 1, S_EPS = 2 /* 5 slots */, S_NORM = 8 /* 5 slots */, S_STEP = 14, S_HISTN = 15,
       S_TNORM = 16, S_THISTN = 17, S_FORCE = 20 /* 9 slots: total, pressure, viscous force */, S_NSCAL = 29 };

enum BcCode { BC_EXTRAP = 1, BC_SOLID = 2, BC_SYM = 3, BC_FAR = 4, BC_INFLOW = 5, BC_OUTFLOW = 6 };

template <typename R> __device__ __forceinline__ R small_v();
template <> __device__ __forceinline__ double small_v<double>() { return 1.0e-40; }
// 1e-40 is subnormal in FP32; the guard only has to keep a zero denominator
// away, so the FP32 path uses the smallest normal value instead.
template <> __device__ __forceinline__ float small_v<float>() { return 1.17549435e-38f; }

template <typename R> __device__ __forceinline__ R Rsqrt(R x);
template <> __device__ __forceinline__ double Rsqrt<double>(double x) { return sqrt(x); }
template <> __device__ __forceinline__ float Rsqrt<float>(float x) { return sqrtf(x); }
template <typename R> __device__ __forceinline__ R Rabs(R x);   // std::abs: clears the sign of -0.0 too
template <> __device__ __forceinline__ double Rabs<double>(double x) { return fabs(x); }
template <> __device__ __forceinline__ float Rabs<float>(float x) { return fabsf(x); }
template <typename R> __device__ __forceinline__ R Rmax(R a, R b) { return a > b ? a : b; }
template <typename R> __device__ __forceinline__ R Rmin(R a, R b) { return a < b ? a : b; }
template <typename R> __device__ __forceinline__ R SQR3(R a, R b, R c) { return a * a + b * b + c * c; }

// Constant parameters of one solve (reference script keys + derived state,
// codes/chemical/src/Chemical.cpp:280-340, codes/ns/src/NsCom.cpp:45-94).
struct DevParams {
    int ischeme, ilim, vismodel, visSRModel, visTimeStepModel, ieigenfix, timestepModel, isowallbc;
    int dim, precision, venkat_kh3, igrad, ivischeme;
    double gama, centropy1, centropy2, vencat_coef, reynolds, oreynolds, oprl, oprt, const_cp, statecoef;
    double inflow[NEQ];
    double twall, sutherland_ts, max_time_ratio, global_dt;
    // SA (TurbCom::InitConst, codes/turb/src/TurbCom.cpp:110-350)
    double nut_inf, max_vis_ratio, turb_cfl_ratio, rprod;
    int iprod_sa, ft2_flag;
    double sa_cb1, sa_cv13, sa_cw2, sa_cw36, sa_ct3, sa_ct4, sa_osigma, sa_cw1, sa_sac2, sa_sac3, sa_cb2s, sa_cw1k,
        sa_okarm2;
};

// Primitive -> conservative, NsInvFlux.cpp:1355-1375 (CalcInternalEnergy :1400-1412)
template <typename R>
__device__ __forceinline__ void primToQ(const R *pr, R gama, R *qq) {
    R v2 = SQR3(pr[IU], pr[IV], pr[IW]);
    R em = (pr[IP] / pr[IR]) / (gama - R(1)) + R(0.5) * v2;
    qq[0] = pr[IR]; qq[1] = pr[IR] * pr[IU]; qq[2] = pr[IR] * pr[IV]; qq[3] = pr[IR] * pr[IW]; qq[4] = pr[IR] * em;
}

// NsInvFlux::Roe + ModifyAbsoluteEigenvalue, codes/ns/src/NsInvFlux.cpp:167-308
template <typename R>
__device__ __forceinline__ void roeFlux(const R *p1, const R *p2, R xn, R yn, R zn, R gam, int ieigenfix, R ce1, R ce2,
                                        R *flux) {
    const R half = R(0.5), one = R(1), two = R(2), vfn = R(0);
    R rl = p1[IR], ul = p1[IU], vl = p1[IV], wl = p1[IW], pl = p1[IP];
    R rr = p2[IR], ur = p2[IU], vr = p2[IV], wr = p2[IW], pr = p2[IP];
    R v2l = SQR3(ul, vl, wl), v2r = SQR3(ur, vr, wr);
    R hl = (gam / (gam - one)) * (pl / rl) + half * v2l;
    R hr = (gam / (gam - one)) * (pr / rr) + half * v2r;
    R vnl = xn * ul + yn * vl + zn * wl - vfn;
    R vnr = xn * ur + yn * vr + zn * wr - vfn;
    R rvnl = rl * vnl, rvnr = rr * vnr;
    R ratio = Rsqrt(rr / rl);
    R coef = one / (one + ratio);
    R um = (ul + ur * ratio) * coef;
    R vm = (vl + vr * ratio) * coef;
    R wm = (wl + wr * ratio) * coef;
    R hm = (hl + hr * ratio) * coef;
    R gama = (gam + gam * ratio) * coef;
    R v2 = SQR3(um, vm, wm);
    R vnflow = xn * um + yn * vm + zn * wm;
    R vnrel = vnflow - vfn;
    R gamm1 = gama - one;
    R c2 = gamm1 * (hm - half * v2);
    R cm = Rsqrt(Rabs(c2));
    R aeig1 = Rabs(vnrel), aeig2 = Rabs(vnrel + cm), aeig3 = Rabs(vnrel - cm);
    flux[0] = rvnl + rvnr;
    flux[1] = (rvnl * ul + xn * pl) + (rvnr * ur + xn * pr);
    flux[2] = (rvnl * vl + yn * pl) + (rvnr * vr + yn * pr);
    flux[3] = (rvnl * wl + zn * pl) + (rvnr * wr + zn * pr);
    flux[4] = (rvnl * hl + vfn * pl) + (rvnr * hr + vfn * pr);
    R q1[NEQ], q2[NEQ], dqv[NEQ];
    primToQ(p1, gam, q1);
    primToQ(p2, gam, q2);
#pragma unroll
    for (int e = 0; e < NEQ; ++e) dqv[e] = q2[e] - q1[e];
    R meig1 = aeig1, meig2 = aeig2, meig3 = aeig3;
    if (ieigenfix == 1) {
        R mx = Rmax(aeig2, aeig3);
        R m1 = mx * ce1, m2 = mx * ce2;
        meig1 = Rmax(m1, aeig1); meig2 = Rmax(m2, aeig2); meig3 = Rmax(m2, aeig3);
    }
    R xi1 = (two * meig1 - meig2 - meig3) / (two * c2);
    R xi2 = (meig2 - meig3) / (two * cm);
    R dc = vnflow * dqv[0] - xn * dqv[1] - yn * dqv[2] - zn * dqv[3];
    R c2dc = c2 * dc;
    R ae = gama - one, af = half * ae * v2;
    R dh = -ae * (um * dqv[1] + vm * dqv[2] + wm * dqv[3] - dqv[4]);
    dh += af * dqv[0];
    R term1 = dh * xi1 + dc * xi2;
    R term2 = c2dc * xi1 + dh * xi2;
    flux[0] -= (meig1 * dqv[0] - term1);
    flux[1] -= (meig1 * dqv[1] - um * term1 + xn * term2);
    flux[2] -= (meig1 * dqv[2] - vm * term1 + yn * term2);
    flux[3] -= (meig1 * dqv[3] - wm * term1 + zn * term2);
    flux[4] -= (meig1 * dqv[4] - hm * term1 + vnflow * term2);
#pragma unroll
    for (int e = 0; e < NEQ; ++e) flux[e] *= half;
}

// The same Roe flux for the FP32-face path, split by magnitude.  The central
// part fc = F(qL) + F(qR) and the jump qR - qL of the conservative variables
// are formed in FP64 from the FP64 face states p1/p2: at low Mach numbers they
// carry the large pressure and enthalpy terms (p ~ 1/(gamma M^2)), whose FP32
// rounding would set the floor of the converged residual.  The Roe averages,
// eigenvalues and the dissipation d = |A| (qR - qL), a small correction near
// convergence, are FP32, from the FP32 copies f1/f2 of the same states.  The
// face flux is (fc - d) / 2.  og1 = 1/(gamma-1); the FP64 part has no division.
// The central part takes the FP64 unit normal (xn, yn, zn), so that the
// pressure terms of a cell's faces cancel to FP64 round-off in a uniform
// state; the dissipation takes its FP32 rounding (xnf, ynf, znf).
__device__ __forceinline__ void roeFluxMixed(const double *p1, const double *p2, const float *f1, const float *f2,
                                             double xn, double yn, double zn, float xnf, float ynf, float znf,
                                             float gam, double og1, int ieigenfix, float ce1, float ce2, double *fc,
                                             float *d) {
    double rl = p1[IR], ul = p1[IU], vl = p1[IV], wl = p1[IW], pl = p1[IP];
    double rr = p2[IR], ur = p2[IU], vr = p2[IV], wr = p2[IW], pr = p2[IP];
    double el = pl * og1 + 0.5 * rl * SQR3(ul, vl, wl);   // total energy per volume
    double er = pr * og1 + 0.5 * rr * SQR3(ur, vr, wr);
    double vnl = xn * ul + yn * vl + zn * wl, vnr = xn * ur + yn * vr + zn * wr;
    double rvnl = rl * vnl, rvnr = rr * vnr;
    fc[0] = rvnl + rvnr;
    fc[1] = (rvnl * ul + xn * pl) + (rvnr * ur + xn * pr);
    fc[2] = (rvnl * vl + yn * pl) + (rvnr * vr + yn * pr);
    fc[3] = (rvnl * wl + zn * pl) + (rvnr * wr + zn * pr);
    fc[4] = vnl * (el + pl) + vnr * (er + pr);
    float dqv[NEQ];
    dqv[0] = float(rr - rl);
    dqv[1] = float(rr * ur - rl * ul);
    dqv[2] = float(rr * vr - rl * vl);
    dqv[3] = float(rr * wr - rl * wl);
    dqv[4] = float(er - el);
    const float half = 0.5f, one = 1.0f, two = 2.0f;
    float rlf = f1[IR], rrf = f2[IR];
    float gg1 = gam / (gam - one);
    float hl = gg1 * (f1[IP] / rlf) + half * SQR3(f1[IU], f1[IV], f1[IW]);
    float hr = gg1 * (f2[IP] / rrf) + half * SQR3(f2[IU], f2[IV], f2[IW]);
    float ratio = sqrtf(rrf / rlf);
    float coef = one / (one + ratio);
    float um = (f1[IU] + f2[IU] * ratio) * coef;
    float vm = (f1[IV] + f2[IV] * ratio) * coef;
    float wm = (f1[IW] + f2[IW] * ratio) * coef;
    float hm = (hl + hr * ratio) * coef;
    float gama = (gam + gam * ratio) * coef;
    float v2 = SQR3(um, vm, wm);
    float vnflow = xnf * um + ynf * vm + znf * wm;
    float gamm1 = gama - one;
    float c2 = gamm1 * (hm - half * v2);
    float cm = sqrtf(fabsf(c2));
    float aeig1 = fabsf(vnflow), aeig2 = fabsf(vnflow + cm), aeig3 = fabsf(vnflow - cm);
    float meig1 = aeig1, meig2 = aeig2, meig3 = aeig3;
    if (ieigenfix == 1) {
        float mx = fmaxf(aeig2, aeig3);
        float m1 = mx * ce1, m2 = mx * ce2;
        meig1 = fmaxf(m1, aeig1); meig2 = fmaxf(m2, aeig2); meig3 = fmaxf(m2, aeig3);
    }
    float xi1 = (two * meig1 - meig2 - meig3) / (two * c2);
    float xi2 = (meig2 - meig3) / (two * cm);
    float dc = vnflow * dqv[0] - xnf * dqv[1] - ynf * dqv[2] - znf * dqv[3];
    float c2dc = c2 * dc;
    float ae = gama - one, af = half * ae * v2;
    float dh = -ae * (um * dqv[1] + vm * dqv[2] + wm * dqv[3] - dqv[4]);
    dh += af * dqv[0];
    float term1 = dh * xi1 + dc * xi2;
    float term2 = c2dc * xi1 + dh * xi2;
    d[0] = meig1 * dqv[0] - term1;
    d[1] = meig1 * dqv[1] - um * term1 + xnf * term2;
    d[2] = meig1 * dqv[2] - vm * term1 + ynf * term2;
    d[3] = meig1 * dqv[3] - wm * term1 + znf * term2;
    d[4] = meig1 * dqv[4] - hm * term1 + vnflow * term2;
}

template <typename R>
__device__ __forceinline__ R fmSplit2(R mach, R ipn) { return ipn * R(0.25) * (mach + ipn) * (mach + ipn); }
// FPSplit5, codes/ns/src/NsInvFlux.cpp:56-65 (alpha = 0 on this path)
template <typename R>
__device__ __forceinline__ R fpSplit5(R mach, R alpha, R ipn) {
    R macha = Rabs(mach);
    if (macha >= R(1)) return R(0.5) * (R(1) + ipn * mach / (macha + small_v<R>()));
    return fmSplit2(mach, ipn) * ((R(2) * ipn - mach) - ipn * R(16) * alpha * mach * fmSplit2(mach, -ipn));
}

// NsInvFlux::Slau2, codes/ns/src/NsInvFlux.cpp:1246-1314
template <typename R>
__device__ __forceinline__ void slau2Flux(const R *p1, const R *p2, R xn, R yn, R zn, R gam, R *flux) {
    const R half = R(0.5), one = R(1), vfn = R(0);
    R rl = p1[IR], ul = p1[IU], vl = p1[IV], wl = p1[IW], pl = p1[IP];
    R rr = p2[IR], ur = p2[IU], vr = p2[IV], wr = p2[IW], pr = p2[IP];
    R v2l = SQR3(ul, vl, wl), v2r = SQR3(ur, vr, wr);
    R hl = (gam / (gam - one)) * (pl / rl) + half * v2l;
    R hr = (gam / (gam - one)) * (pr / rr) + half * v2r;
    R vnl = xn * ul + yn * vl + zn * wl - vfn;
    R vnr = xn * ur + yn * vr + zn * wr - vfn;
    R orl = one / (rl + small_v<R>()), orr = one / (rr + small_v<R>());
    R c2l = gam * pl * orl, c2r = gam * pr * orr;
    R cl = Rsqrt(c2l), cr = Rsqrt(c2r);
    R cm = half * (cl + cr);
    R t = rr / rl;
    R vna = (Rabs(vnl) + t * Rabs(vnr)) / (one + t);
    R ml = vnl / cm, mr = vnr / cm;
    R g = -Rmax(Rmin(ml, R(0)), R(-1)) * Rmin(Rmax(mr, R(0)), R(1));
    R vnp = (one - g) * vna + g * Rabs(vnl);
    R vnn = (one - g) * vna + g * Rabs(vnr);
    R va = Rsqrt(half * (v2l + v2r));
    R m12 = Rmin(one, va / cm);
    R ka = (one - m12) * (one - m12);
    R ms = half * (rl * (vnl + vnp) + rr * (vnr - vnn) - ka * (pr - pl) / cm);
    R fp5ml = fpSplit5(ml, R(0), one);
    R fp5mr = fpSplit5(mr, R(0), -one);
    R ps = R(0);
    ps += half * (pl + pr);
    ps += half * (fp5ml - fp5mr) * (pl - pr);
    ps += va * (fp5ml + fp5mr - one) * Rsqrt(rl * rr) * cm;
    R mp = half * (ms + Rabs(ms)), mn = half * (ms - Rabs(ms));
    flux[0] = (mp + mn);
    flux[1] = (mp * ul + mn * ur) + xn * ps;
    flux[2] = (mp * vl + mn * vr) + yn * ps;
    flux[3] = (mp * wl + mn * wr) + zn * ps;
    flux[4] = (mp * hl + mn * hr) + vfn * ps;
}

// The same SLAU2 flux for the FP32-face path, split by magnitude like the
// mixed Roe flux.  With mp psi_L + mn psi_R = ms/2 (psi_L + psi_R) -
// |ms|/2 (psi_R - psi_L), psi = (1, u, v, w, h), the face flux is fc - d with
//   fc = ms/2 (psi_L + psi_R) + n p_c,   p_c = (p_L + p_R)/2          (FP64)
//   d  = |ms|/2 (psi_R - psi_L) - n p_d                                (FP32)
// where p_d = ps - p_c holds the pressure-split and low-Mach terms of ps.
// The enthalpies, the pressure average and the jumps psi_R - psi_L, p_R - p_L
// are formed in FP64 from the FP64 face states p1/p2 (at low Mach numbers p
// and h carry the large 1/(gamma M^2) terms), and so are the O(1) parts of
// the mass flux ms (rho vn and the averaged normal speed); the Mach splits,
// the switch g, the low-Mach factor ka, the pressure-diffusion term of ms and
// p_d are FP32 from the FP32 copies f1/f2 and the FP32 jumps.  The central
// pressure term takes the FP64 normal (xn, yn, zn); d takes its FP32 rounding
// (xnf, ynf, znf).
__device__ __forceinline__ void slau2FluxMixed(const double *p1, const double *p2, const float *f1, const float *f2,
                                               double xn, double yn, double zn, float xnf, float ynf, float znf,
                                               float gam, double *fc, float *d) {
    const float half = 0.5f, one = 1.0f;
    const double gg = double(gam) / (double(gam) - 1.0);
    double hlD = gg * (p1[IP] / p1[IR]) + 0.5 * SQR3(p1[IU], p1[IV], p1[IW]);
    double hrD = gg * (p2[IP] / p2[IR]) + 0.5 * SQR3(p2[IU], p2[IV], p2[IW]);
    float rl = f1[IR], ul = f1[IU], vl = f1[IV], wl = f1[IW], pl = f1[IP];
    float rr = f2[IR], ur = f2[IU], vr = f2[IV], wr = f2[IW], pr = f2[IP];
    float dp = float(p2[IP] - p1[IP]);   // p_R - p_L
    float v2l = SQR3(ul, vl, wl), v2r = SQR3(ur, vr, wr);
    const double vnlD = xn * p1[IU] + yn * p1[IV] + zn * p1[IW];
    const double vnrD = xn * p2[IU] + yn * p2[IV] + zn * p2[IW];
    float vnl = float(vnlD), vnr = float(vnrD);
    float orl = one / (rl + small_v<float>()), orr = one / (rr + small_v<float>());
    float c2l = gam * pl * orl, c2r = gam * pr * orr;
    float cl = sqrtf(c2l), cr = sqrtf(c2r);
    float cm = half * (cl + cr);
    const double tD = p2[IR] / p1[IR];
    const double vnaD = (fabs(vnlD) + tD * fabs(vnrD)) / (1.0 + tD);
    float ml = vnl / cm, mr = vnr / cm;
    float g = -fmaxf(fminf(ml, 0.0f), -1.0f) * fminf(fmaxf(mr, 0.0f), 1.0f);
    const double gD = g;
    const double vnpD = (1.0 - gD) * vnaD + gD * fabs(vnlD);
    const double vnnD = (1.0 - gD) * vnaD + gD * fabs(vnrD);
    float va = sqrtf(half * (v2l + v2r));
    float m12 = fminf(one, va / cm);
    float ka = (one - m12) * (one - m12);
    const double msD = 0.5 * (p1[IR] * (vnlD + vnpD) + p2[IR] * (vnrD - vnnD)) - double(half * ka * dp / cm);
    const float ms = float(msD);
    float fp5ml = fpSplit5(ml, 0.0f, one);
    float fp5mr = fpSplit5(mr, 0.0f, -one);
    float pd = half * (fp5ml - fp5mr) * (-dp) + va * (fp5ml + fp5mr - one) * sqrtf(rl * rr) * cm;
    const double pc = 0.5 * (p1[IP] + p2[IP]);
    fc[0] = msD;
    fc[1] = 0.5 * msD * (p1[IU] + p2[IU]) + xn * pc;
    fc[2] = 0.5 * msD * (p1[IV] + p2[IV]) + yn * pc;
    fc[3] = 0.5 * msD * (p1[IW] + p2[IW]) + zn * pc;
    fc[4] = 0.5 * msD * (hlD + hrD);
    const float am = half * fabsf(ms);
    d[0] = 0.0f;
    d[1] = am * float(p2[IU] - p1[IU]) - xnf * pd;
    d[2] = am * float(p2[IV] - p1[IV]) - ynf * pd;
    d[3] = am * float(p2[IW] - p1[IW]) - znf * pd;
    d[4] = am * float(hrD - hlD);
}

}  // namespace ofg

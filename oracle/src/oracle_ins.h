// Test infrastructure: sequential CPU restatement of the reference's
// unstructured incompressible solver (INsSolver, startStrategy 2,
// time_integral 3 = TimeIntegral::Simple), the checker for the GPU
// pressure-correction path.  Included by oracle.cpp after the Oracle struct
// (it reuses its mesh, metrics and inflow state).
//
// One inner iteration is INsCalcRHS (codes/ins/src/INsRhs.cpp:105-132):
// mass-flux upwind coefficients, Green-Gauss gradients of u v w p, the
// viscous face coefficients, the unsteady and source terms, three momentum
// solves and one pressure-correction solve by the reference's GMRES
// (codes/bgmres/include/GMRES.h, identity preconditioner, Krylov dimension
// 500, no restart, tolerance 1e-8), the Rhie-Chow face fluxes, the pressure
// and velocity corrections (under-relaxation 0.8) and the residual maxima.
// Every loop keeps the reference's order and every expression its operand
// order, so that this restatement rounds like the reference.
//
// Scope, as the reference runs it: the boundary loops of MomPre and
// UpdateSpeed (codes/uins/src/UINsInvterm.cpp:617-700, 1622-1780) walk the
// boundary faces through bcInfo->bcFace[ir] of the last boundary-condition
// region, so the reference reads in bounds only when every boundary face has
// one type; the type they apply (ug.bctype) is also the last region's.  The
// restatement therefore covers meshes whose boundary is all SOLID_SURFACE
// (closed cavities, lids moving through per-face wall velocities -- the
// reference's ins_bc.txt data) with a viscous model (vismodel >= 1; with
// vismodel 0 the reference never forms the gradients the source term uses).
#pragma once

struct InsOracle {
    Oracle &m;
    int nF, nB, nC, nT;
    double dt = 1.0e-3;            // iinv.timestep = global_dt (UINsInvterm.cpp:114-117)
    double vis = 0;                // iinv.vis = 1 / reynolds (UINsVisterm.cpp:290)
    std::vector<double> wu, wv, ww;            // per boundary face: wall velocity (ins_bc data, else grid velocity 0)
    // face arrays (iinv.*, sized nFaces)
    std::vector<double> f1, f2, rf, uf, vf, wf, fq, Fn, ai0, ai1, biu0, biu1, biv0, biv1, biw0, biw1;
    std::vector<double> Vdvu, Vdvv, Vdvw, ajp;
    // cell arrays (sized nTCell)
    std::vector<double> spt, but, bvt, bwt, up, vp, wp, spc, buc, bvc, bwc, uc, vc, wc;
    std::vector<double> spp, bp, pp, VdU, VdV, VdW, dqqdx, dqqdy, dqqdz, mu, mv, mw;
    double remax[4] = {1, 1, 1, 1};   // remax_up, remax_vp, remax_wp, remax_pp
    double linRes[4] = {0, 0, 0, 0};  // GMRES residual of the u, v, w and pressure solves
    int linIts[4] = {0, 0, 0, 0};     // GMRES iterations of the same solves
    long innerSteps = 0;
    // CSR of the solves (MomPre, UINsInvterm.cpp:446-478): row = cell (ghosts
    // included), entries in c2f order, the diagonal last
    std::vector<int> IA, JA;

    explicit InsOracle(Oracle &o) : m(o) {
        nF = m.nFaces; nB = m.nBFaces; nC = m.nCells; nT = m.nT;
        wu.assign(nB, 0.0); wv.assign(nB, 0.0); ww.assign(nB, 0.0);
        for (auto *v : {&f1, &f2, &rf, &uf, &vf, &wf, &fq, &Fn, &ai0, &ai1, &biu0, &biu1, &biv0, &biv1, &biw0, &biw1,
                        &Vdvu, &Vdvv, &Vdvw, &ajp})
            v->assign(nF, 0.0);
        for (auto *v : {&spt, &but, &bvt, &bwt, &up, &vp, &wp, &spc, &buc, &bvc, &bwc, &uc, &vc, &wc, &spp, &bp, &pp,
                        &VdU, &VdV, &VdW, &dqqdx, &dqqdy, &dqqdz})
            v->assign(nT, 0.0);
        mu.assign(nC, 0.0); mv.assign(nC, 0.0); mw.assign(nC, 0.0);
        IA.assign(nT + 1, 0);
        for (int c = 0; c < nT; ++c) IA[c + 1] = IA[c] + int(m.c2f[c].size()) + 1;
        JA.assign(IA[nT], 0);
        for (int c = 0; c < nT; ++c) {
            int n = IA[c], fn = int(m.c2f[c].size());
            for (int k = 0; k < fn; ++k) {
                int f = m.c2f[c][k];
                JA[n + k] = c == m.lc[f] ? m.rc[f] : m.lc[f];
            }
            JA[n + fn] = c;
        }
    }

    bool supported(std::string &why) const {
        for (int f = 0; f < nB; ++f)
            if (m.bcType[f] != OFG_BC_SOLID_SURFACE) { why = "boundary faces other than SOLID_SURFACE"; return false; }
        if (m.p.vismodel < 1) { why = "inviscid model"; return false; }
        return true;
    }

    // INsInitFinal (codes/ins/src/INsSolverImp.cpp:58-77): q = inflow in every
    // cell (UINsRestart::InitinsRestart, codes/uins/src/UINsRestart.cpp:50-62),
    // then the ghost states of the adiabatic viscous wall: the interior state
    // with the velocity mirrored about the wall velocity
    // (INsBcSolver::AdiabaticVisWallBc / VelocityBc, codes/ins/src/INsBcSolver.cpp:329-367).
    void init() {
        m.initReference();
        m.outerSteps = 0;
        innerSteps = 0;
        dt = m.p.global_dt;
        vis = 1 / m.p.reynolds;
        for (int e = 0; e < NEQ; ++e) std::fill(m.q[e].begin(), m.q[e].end(), m.inflow[e]);
        for (int f = 0; f < nB; ++f) {
            int l = m.lc[f], r = m.rc[f];
            for (int e = 0; e < NEQ; ++e) m.q[e][r] = m.q[e][l];
            m.q[IU][r] = -m.q[IU][r] + 2.0 * wu[f];
            m.q[IV][r] = -m.q[IV][r] + 2.0 * wv[f];
            m.q[IW][r] = -m.q[IW][r] + 2.0 * ww[f];
        }
        std::fill(mu.begin(), mu.end(), 0.0); std::fill(mv.begin(), mv.end(), 0.0); std::fill(mw.begin(), mw.end(), 0.0);
        for (double &r : remax) r = 1;
    }

    // -------- UINsInvterm::INsPreflux (first inner step), UINsInvterm.cpp:138-178,
    // INsInvterm::CalcINsinvFlux / CalcINsBcinvFlux, codes/ins/src/INsInvterm.cpp:89-140
    void preflux() {
        auto face = [&](int f, bool bnd) {
            int l = m.lc[f], r = m.rc[f];
            rf[f] = (m.q[IR][l] + m.q[IR][r]) * half;
            uf[f] = (m.q[IU][l] + m.q[IU][r]) * half;
            vf[f] = (m.q[IV][l] + m.q[IV][r]) * half;
            wf[f] = (m.q[IW][l] + m.q[IW][r]) * half;
            double vn = m.xfn[f] * uf[f] + m.yfn[f] * vf[f] + m.zfn[f] * wf[f] - 0.0;
            fq[f] = bnd ? 0.0 : rf[f] * vn * m.area[f];   // every boundary face is a solid wall here
        };
        for (int f = nB; f < nF; ++f) face(f, false);
        for (int f = 0; f < nB; ++f) face(f, true);
    }

    // -------- CalcInvMassFlux: INsInvterm::CalcINsinvTerm, INsInvterm.cpp:142-154
    static double max0(double v) { return 0.0 > v ? 0.0 : v; }   // MAX(0, v) of HXMath.h:158-161
    void invCoef() {
        for (int f = 0; f < nF; ++f) {
            double clr = max0(fq[f]);
            ai0[f] = clr;
            ai1[f] = clr - fq[f];
        }
    }

    // -------- Green-Gauss gradient with distance-weighted face values:
    // UINsVisterm::CalcPreandVisGrad (UINsVisterm.cpp:98-228, eps 0) and
    // UINsInvterm::CalcPreGrad (UINsInvterm.cpp:1984-2059, eps SMALL)
    void ggrad(const std::vector<double> *const *v, int nv, std::vector<double> *const *gx,
               std::vector<double> *const *gy, std::vector<double> *const *gz, double eps) {
        for (int k = 0; k < nv; ++k) {
            std::fill(gx[k]->begin(), gx[k]->end(), 0.0);
            std::fill(gy[k]->begin(), gy[k]->end(), 0.0);
            std::fill(gz[k]->begin(), gz[k]->end(), 0.0);
        }
        for (int f = 0; f < nF; ++f) {
            int l = m.lc[f], r = m.rc[f];
            double dxl = m.xfc[f] - m.xcc[l], dyl = m.yfc[f] - m.ycc[l], dzl = m.zfc[f] - m.zcc[l];
            double dxr = m.xfc[f] - m.xcc[r], dyr = m.yfc[f] - m.ycc[r], dzr = m.zfc[f] - m.zcc[r];
            double d1 = std::sqrt(dxl * dxl + dyl * dyl + dzl * dzl);
            double d2 = std::sqrt(dxr * dxr + dyr * dyr + dzr * dzr);
            double delta = eps == 0.0 ? 1.0 / (d1 + d2) : 1.0 / (d1 + d2 + eps);
            double cl = d2 * delta, cr = d1 * delta;
            double fnxa = m.xfn[f] * m.area[f], fnya = m.yfn[f] * m.area[f], fnza = m.zfn[f] * m.area[f];
            for (int k = 0; k < nv; ++k) {
                double val = cl * (*v[k])[l] + cr * (*v[k])[r];
                (*gx[k])[l] += fnxa * val; (*gy[k])[l] += fnya * val; (*gz[k])[l] += fnza * val;
                if (f < nB) continue;
                (*gx[k])[r] += -fnxa * val; (*gy[k])[r] += -fnya * val; (*gz[k])[r] += -fnza * val;
            }
        }
        for (int c = 0; c < nC; ++c) {
            double ovol = 1.0 / m.vol[c];
            for (int k = 0; k < nv; ++k) { (*gx[k])[c] *= ovol; (*gy[k])[c] *= ovol; (*gz[k])[c] *= ovol; }
        }
        for (int f = 0; f < nB; ++f) {
            int l = m.lc[f], r = m.rc[f];
            for (int k = 0; k < nv; ++k) { (*gx[k])[r] = (*gx[k])[l]; (*gy[k])[r] = (*gy[k])[l]; (*gz[k])[r] = (*gz[k])[l]; }
        }
    }
    void velPresGrad() {
        std::fill(m.dqdx[IR].begin(), m.dqdx[IR].end(), 0.0);
        std::fill(m.dqdy[IR].begin(), m.dqdy[IR].end(), 0.0);
        std::fill(m.dqdz[IR].begin(), m.dqdz[IR].end(), 0.0);
        const std::vector<double> *v[4] = {&m.q[IU], &m.q[IV], &m.q[IW], &m.q[IP]};
        std::vector<double> *gx[4] = {&m.dqdx[IU], &m.dqdx[IV], &m.dqdx[IW], &m.dqdx[IP]};
        std::vector<double> *gy[4] = {&m.dqdy[IU], &m.dqdy[IV], &m.dqdy[IW], &m.dqdy[IP]};
        std::vector<double> *gz[4] = {&m.dqdz[IU], &m.dqdz[IV], &m.dqdz[IW], &m.dqdz[IP]};
        ggrad(v, 4, gx, gy, gz, 0.0);
    }

    // -------- UINsVisterm::CalcFaceVisterm, UINsVisterm.cpp:281-394 (every face)
    void visCoef() {
        for (int f = 0; f < nF; ++f) {
            int l = m.lc[f], r = m.rc[f];
            double lx = m.xcc[r] - m.xcc[l], ly = m.ycc[r] - m.ycc[l], lz = m.zcc[r] - m.zcc[l];
            double dist = m.xfn[f] * (m.xcc[r] - m.xcc[l]) + m.yfn[f] * (m.ycc[r] - m.ycc[l]) +
                          m.zfn[f] * (m.zcc[r] - m.zcc[l]);
            Fn[f] = vis * m.area[f] / dist;
            double dx1 = m.xfc[f] - m.xcc[l], dy1 = m.yfc[f] - m.ycc[l], dz1 = m.zfc[f] - m.zcc[l];
            double dx2 = m.xfc[f] - m.xcc[r], dy2 = m.yfc[f] - m.ycc[r], dz2 = m.zfc[f] - m.zcc[r];
            double de1 = std::sqrt(dx1 * dx1 + dy1 * dy1 + dz1 * dz1);
            double de2 = std::sqrt(dx2 * dx2 + dy2 * dy2 + dz2 * dz2);
            double de = 1.0 / (de1 + de2);
            f1[f] = de2 * de;
            f2[f] = de1 * de;
            double a = f1[f], b = f2[f];
            double Ft[3][2];
            for (int k = 0; k < 3; ++k) {
                int e = IU + k;
                double gxf = a * m.dqdx[e][l] + b * m.dqdx[e][r];
                double gyf = a * m.dqdy[e][l] + b * m.dqdy[e][r];
                double gzf = a * m.dqdz[e][l] + b * m.dqdz[e][r];
                double Pf = gxf * m.xfn[f] + gyf * m.yfn[f] + gzf * m.zfn[f];
                double Pd = -(gxf * lx + gyf * ly + gzf * lz) / dist;
                Ft[k][0] = Pf * m.area[f] * vis;
                Ft[k][1] = Pd * m.area[f] * vis;
            }
            ai0[f] += Fn[f];
            ai1[f] += Fn[f];
            biu0[f] = Ft[0][0] + Ft[0][1]; biu1[f] = -Ft[0][0] - Ft[0][1];
            biv0[f] = Ft[1][0] + Ft[1][1]; biv1[f] = -Ft[1][0] - Ft[1][1];
            biw0[f] = Ft[2][0] + Ft[2][1]; biw1[f] = -Ft[2][0] - Ft[2][1];
        }
    }

    // -------- UINsVisterm::CalcUnsteadcoff, UINsVisterm.cpp:479-562 (interior
    // cells, then ghosts: the same formula); the previous-time velocity is
    // taken from q on the first inner step
    void unsteadyCoef(bool first) {
        for (int c = 0; c < nT; ++c) {
            double rho = m.q[IR][c], vol = m.vol[c];
            spt[c] = vol * rho / dt;
            if (first) { up[c] = m.q[IU][c]; vp[c] = m.q[IV][c]; wp[c] = m.q[IW][c]; }
            but[c] = vol * rho * up[c] / dt;
            bvt[c] = vol * rho * vp[c] / dt;
            bwt[c] = vol * rho * wp[c] / dt;
        }
    }

    // -------- UINsVisterm::CalcINsSrc, UINsVisterm.cpp:564-632
    void source() {
        std::fill(spc.begin(), spc.end(), 0.0);
        std::fill(buc.begin(), buc.end(), 0.0);
        std::fill(bvc.begin(), bvc.end(), 0.0);
        std::fill(bwc.begin(), bwc.end(), 0.0);
        for (int f = 0; f < nF; ++f) {
            int l = m.lc[f], r = m.rc[f];
            spc[l] += ai0[f]; spc[r] += ai1[f];
            buc[l] += biu0[f]; buc[r] += biu1[f];
            bvc[l] += biv0[f]; bvc[r] += biv1[f];
            bwc[l] += biw0[f]; bwc[r] += biw1[f];
        }
        for (int c = 0; c < nT; ++c) {
            spc[c] += spt[c];
            buc[c] += but[c] - m.vol[c] * m.dqdx[IP][c];
            bvc[c] += bvt[c] - m.vol[c] * m.dqdy[IP][c];
            bwc[c] += bwt[c] - m.vol[c] * m.dqdz[IP][c];
        }
    }

    // -------- the momentum matrix (MomPre, UINsInvterm.cpp:446-478): row c,
    // entry per face of c2f[c]: -ai[f][0] when c is the left cell, -ai[f][1]
    // when c is the right cell; the diagonal spc[c] last
    void momentumMatrix(std::vector<double> &A) const {
        A.assign(IA[nT], 0.0);
        for (int c = 0; c < nT; ++c) {
            int n = IA[c], fn = int(m.c2f[c].size());
            for (int k = 0; k < fn; ++k) {
                int f = m.c2f[c][k];
                A[n + k] = c == m.lc[f] ? -ai0[f] : -ai1[f];
            }
            A[n + fn] = spc[c];
        }
    }
    // pressure-correction matrix (UINsInvterm.cpp:1272-1306): -ajp off the
    // diagonal, spp on it
    void pressureMatrix(std::vector<double> &A) const {
        A.assign(IA[nT], 0.0);
        for (int c = 0; c < nT; ++c) {
            int n = IA[c], fn = int(m.c2f[c].size());
            for (int k = 0; k < fn; ++k) A[n + k] = -ajp[m.c2f[c][k]];
            A[n + fn] = spp[c];
        }
    }

    // Poisson::operator*, codes/bgmres/src/poisson.cpp:53-78
    void spmv(const std::vector<double> &A, const std::vector<double> &x, std::vector<double> &y) const {
        for (int i = 0; i < nT; ++i) {
            double t = 0.0;
            for (int k = IA[i]; k < IA[i + 1]; ++k) t += A[k] * x[JA[k]];
            y[i] = t;
        }
    }
    // Solution::norm, codes/bgmres/src/solution.cpp:383-395 (rows in reverse)
    static double normRev(const std::vector<double> &v) {
        double s = 0.0;
        for (int i = int(v.size()) - 1; i >= 0; --i) s += v[i] * v[i];
        return std::sqrt(s);
    }

    // GMRES of codes/bgmres/include/GMRES.h:72-405 with one right-hand side,
    // Krylov dimension 500, no restart, tolerance 1e-8, identity
    // preconditioner (Preconditioner::solve2); x starts at zero
    // (SolveMRhs::BGMRES, codes/bgmres/src/systemSolver.cpp:43-74).
    // Returns the iterations used; *res = Rank.residual.
    int gmres(const std::vector<double> &A, const std::vector<double> &b, std::vector<double> &x, double *res) const {
        const int K = 500;
        const double tol = 1.0e-8;
        const int N = nT;
        x.assign(N, 0.0);
        std::vector<double> r(N), ax(N);
        spmv(A, x, ax);
        for (int i = N - 1; i >= 0; --i) r[i] = b[i] - ax[i];
        double t = 0.0;
        for (int i = 0; i < N; ++i) t += r[i] * r[i];
        double normr1 = std::sqrt(t);
        double normRHS = normRev(b);
        double rho = normRev(r);
        *res = rho;
        if (normRHS < 1.0e-5) normRHS = 1.0;
        if (!(rho > tol * normRHS)) return 0;
        std::vector<std::vector<double>> V;
        V.emplace_back(N);
        for (int i = 0; i < N; ++i) V[0][i] = r[i] * (1.0 / normr1);
        std::vector<double> H((size_t)(K + 1) * K, 0.0), gc(K, 0.0), gs(K, 0.0), s(K + 1, 0.0);
        auto h = [&](int i, int j) -> double & { return H[(size_t)i * K + j]; };
        s[0] = normr1;
        int it = 0;
        for (it = 0; it < K; ++it) {
            V.emplace_back(N);
            std::vector<double> &w = V[it + 1];
            spmv(A, V[it], w);
            for (int row = 0; row <= it; ++row) {
                double d = 0.0;
                for (int n = 0; n < N; ++n) d += w[n] * V[row][n];
                h(row, it) = d;
            }
            for (int row = 0; row <= it; ++row)
                for (int n = 0; n < N; ++n) w[n] = w[n] - V[row][n] * h(row, it);
            double tt = 0.0;
            for (int n = 0; n < N; ++n) tt += w[n] * w[n];
            double normr2 = std::sqrt(tt);
            for (int n = 0; n < N; ++n) w[n] = w[n] * (1.0 / normr2);
            h(it + 1, it) = normr2;
            const int col = it;
            for (int row = 0; row < col; ++row) {
                double tmp = gc[row] * h(row, col) + gs[row] * h(row + 1, col);
                h(row + 1, col) = -gs[row] * h(row, col) + gc[row] * h(row + 1, col);
                h(row, col) = tmp;
            }
            if (h(col + 1, col) == 0.0) {
                gc[col] = 1.0; gs[col] = 0.0;
            } else if (std::fabs(h(col + 1, col)) > std::fabs(h(col, col))) {
                double tmp = h(col, col) / h(col + 1, col);
                gs[col] = 1.0 / std::sqrt(1.0 + tmp * tmp);
                gc[col] = tmp * gs[col];
            } else {
                double tmp = h(col + 1, col) / h(col, col);
                gc[col] = 1.0 / std::sqrt(1.0 + tmp * tmp);
                gs[col] = tmp * gc[col];
            }
            double tmp = gc[col] * h(col, col) + gs[col] * h(col + 1, col);
            h(col + 1, col) = -gs[col] * h(col, col) + gc[col] * h(col + 1, col);
            h(col, col) = tmp;
            if (h(col + 1, col) < 1e-10) h(col + 1, col) = 0;
            tmp = gc[col] * s[col] + gs[col] * s[col + 1];
            s[col + 1] = -gs[col] * s[col] + gc[col] * s[col + 1];
            s[col] = tmp;
            double S = s[it + 1];
            rho = std::sqrt(S * S);
            if (rho < tol * normRHS) {
                update(H, K, x, s, V, it);
                spmv(A, x, ax);
                for (int i = N - 1; i >= 0; --i) r[i] = ax[i] - b[i];
                *res = normRev(r);
                return it;
            }
        }
        update(H, K, x, s, V, it - 1);
        spmv(A, x, ax);
        for (int i = N - 1; i >= 0; --i) r[i] = ax[i] - b[i];
        *res = normRev(r);
        return K;
    }
    // Update, GMRES.h:20-61: back substitution in place, then x += V s with
    // rows in reverse and basis vectors from the last
    static void update(const std::vector<double> &H, int K, std::vector<double> &x, std::vector<double> &s,
                       const std::vector<std::vector<double>> &V, int dim) {
        for (int l = dim; l >= 0; --l) {
            s[l] = s[l] / H[(size_t)l * K + l];
            for (int i = l - 1; i >= 0; --i) s[i] -= s[l] * H[(size_t)i * K + l];
        }
        for (int row = int(x.size()) - 1; row >= 0; --row)
            for (int mm = dim; mm >= 0; --mm) x[row] += V[mm][row] * s[mm];
    }

    // ghost velocity of a solid wall: -v_interior + 2 v_wall
    // (UINsInvterm.cpp:638-648, 1637-1647)
    void wallGhosts(std::vector<double> &u, std::vector<double> &v, std::vector<double> &w) const {
        for (int f = 0; f < nB; ++f) {
            int l = m.lc[f], r = m.rc[f];
            u[r] = -u[l] + 2 * wu[f];
            v[r] = -v[l] + 2 * wv[f];
            w[r] = -w[l] + 2 * ww[f];
        }
    }

    // -------- UINsInvterm::MomPre, UINsInvterm.cpp:369-864
    void momentum() {
        std::vector<double> A;
        momentumMatrix(A);
        linIts[0] = gmres(A, buc, uc, &linRes[0]);
        linIts[1] = gmres(A, bvc, vc, &linRes[1]);
        linIts[2] = gmres(A, bwc, wc, &linRes[2]);
        wallGhosts(uc, vc, wc);
    }

    // -------- UINsInvterm::CalcFaceflux, UINsInvterm.cpp:866-908, with the face
    // states of PrepareProFaceValue (UINsInvterm.cpp:338-362: the right state's
    // w is vc[rc], as there); INsInvterm::CalcINsFaceflux / CalcINsBcFaceflux,
    // codes/ins/src/INsInvterm.cpp:170-271
    void faceFlux() {
        for (int f = nB; f < nF; ++f) {
            int l = m.lc[f], r = m.rc[f];
            double rl = m.q[IR][l], ul = uc[l], vl = vc[l], wl = wc[l], pl = m.q[IP][l];
            double rr = m.q[IR][r], ur = uc[r], vr = vc[r], wr = vc[r], pr = m.q[IP][r];
            double xn = m.xfn[f], yn = m.yfn[f], zn = m.zfn[f];
            double Vau = f1[f] * (m.vol[l] * xn / spc[l]) + f2[f] * (m.vol[r] * xn / spc[r]);
            double Vav = f1[f] * (m.vol[l] * yn / spc[l]) + f2[f] * (m.vol[r] * yn / spc[r]);
            double Vaw = f1[f] * (m.vol[l] * zn / spc[l]) + f2[f] * (m.vol[r] * zn / spc[r]);
            double dist = xn * (m.xcc[r] - m.xcc[l]) + yn * (m.ycc[r] - m.ycc[l]) + zn * (m.zcc[r] - m.zcc[l]);
            double Deun = Vau / dist, Devn = Vav / dist, Dewn = Vaw / dist;
            double dx1 = m.xfc[f] - m.xcc[l], dy1 = m.yfc[f] - m.ycc[l], dz1 = m.zfc[f] - m.zcc[l];
            double dx2 = m.xcc[r] - m.xfc[f], dy2 = m.ycc[r] - m.yfc[f], dz2 = m.zcc[r] - m.zfc[f];
            double Bpe = m.dqdx[IP][l] * (dx1) + m.dqdy[IP][l] * (dy1) + m.dqdz[IP][l] * (dz1) +
                         m.dqdx[IP][r] * (dx2) + m.dqdy[IP][r] * (dy2) + m.dqdz[IP][r] * (dz2) - (pr - pl);
            rf[f] = half * (rl + rr);
            uf[f] = (f1[f] * ul + f2[f] * ur) + Deun * Bpe;
            vf[f] = (f1[f] * vl + f2[f] * vr) + Devn * Bpe;
            wf[f] = (f1[f] * wl + f2[f] * wr) + Dewn * Bpe;
            double vn = xn * uf[f] + yn * vf[f] + zn * wf[f];
            fq[f] = rf[f] * vn * m.area[f];
            double clr = max0(fq[f]);
            ai0[f] = clr;
            ai1[f] = clr - fq[f];
        }
        for (int f = 0; f < nB; ++f) {
            int l = m.lc[f], r = m.rc[f];
            rf[f] = (m.q[IR][l] + m.q[IR][r]) * half;
            uf[f] = (uc[l] + uc[r]) * half;
            vf[f] = (vc[l] + vc[r]) * half;
            wf[f] = (wc[l] + vc[r]) * half;
            fq[f] = 0;   // SOLID_SURFACE
            double clr = max0(fq[f]);
            ai0[f] = clr;
            ai1[f] = clr - fq[f];
        }
    }

    // -------- UINsInvterm::CalcCorrectPresscoef + CalcNewMomCoe,
    // UINsInvterm.cpp:1027-1213; INsInvterm::CalcINsFaceCorrectPresscoef /
    // CalcINsBcFaceCorrectPresscoef, codes/ins/src/INsInvterm.cpp:273-334
    void pressureCoef() {
        std::fill(spc.begin(), spc.end(), 0.0);
        for (int f = 0; f < nF; ++f) {
            int l = m.lc[f], r = m.rc[f];
            spc[l] += ai0[f] + Fn[f];
            spc[r] += ai1[f] + Fn[f];
        }
        for (int c = 0; c < nT; ++c) spc[c] += spt[c];
        for (int f = nB; f < nF; ++f) {
            int l = m.lc[f], r = m.rc[f];
            double xn = m.xfn[f], yn = m.yfn[f], zn = m.zfn[f];
            double a = f1[f] * (m.vol[l] / (spc[l])) + f2[f] * (m.vol[r] / (spc[r]));
            Vdvu[f] = a; Vdvv[f] = a; Vdvw[f] = a;
            double dist = xn * (m.xcc[r] - m.xcc[l]) + yn * (m.ycc[r] - m.ycc[l]) + zn * (m.zcc[r] - m.zcc[l]);
            ajp[f] = rf[f] * (Vdvu[f] * xn * xn + Vdvv[f] * yn * yn + Vdvw[f] * zn * zn) * m.area[f] / dist;
        }
        for (int f = 0; f < nB; ++f) { Vdvu[f] = 0; Vdvv[f] = 0; Vdvw[f] = 0; ajp[f] = 0; }
        std::fill(spp.begin(), spp.end(), 0.0);
        std::fill(bp.begin(), bp.end(), 0.0);
        for (int f = 0; f < nF; ++f) {
            int l = m.lc[f], r = m.rc[f];
            spp[l] += ajp[f];
            spp[r] += ajp[f];
            bp[l] += -fq[f];
            bp[r] += fq[f];
            if (f < nB) spp[r] = 1;
        }
        for (int c = 0; c < nT; ++c) {
            VdU[c] = -m.vol[c] / ((1 + 1) * spc[c]);
            VdV[c] = -m.vol[c] / ((1 + 1) * spc[c]);
            VdW[c] = -m.vol[c] / ((1 + 1) * spc[c]);
        }
    }

    // -------- UINsInvterm::CalcPressCorrectEqu, UINsInvterm.cpp:1215-1502
    void pressureCorrection() {
        std::vector<double> A;
        pressureMatrix(A);
        linIts[3] = gmres(A, bp, pp, &linRes[3]);
        for (int f = 0; f < nB; ++f) pp[m.rc[f]] = pp[m.lc[f]];
        for (int c = 0; c < nC; ++c) m.q[IP][c] = m.q[IP][c] + 0.8 * pp[c];
        for (int f = 0; f < nB; ++f) m.q[IP][m.rc[f]] = m.q[IP][m.lc[f]];   // SOLID_SURFACE
    }

    // -------- UINsInvterm::UpdateSpeed, UINsInvterm.cpp:1607-1840
    void updateSpeed() {
        const std::vector<double> *v[1] = {&pp};
        std::vector<double> *gx[1] = {&dqqdx}, *gy[1] = {&dqqdy}, *gz[1] = {&dqqdz};
        ggrad(v, 1, gx, gy, gz, SMALL);
        for (int c = 0; c < nC; ++c) {
            double uu = VdU[c] * dqqdx[c] * 0.8, vv = VdV[c] * dqqdy[c] * 0.8, ww_ = VdW[c] * dqqdz[c] * 0.8;
            up[c] = uc[c] + uu; vp[c] = vc[c] + vv; wp[c] = wc[c] + ww_;
            m.q[IU][c] = up[c]; m.q[IV][c] = vp[c]; m.q[IW][c] = wp[c];
        }
        wallGhosts(up, vp, wp);
        for (int f = 0; f < nB; ++f) {
            int r = m.rc[f];
            m.q[IU][r] = up[r]; m.q[IV][r] = vp[r]; m.q[IW][r] = wp[r];
        }
    }

    // -------- UINsInvterm::UpdateFaceflux, UINsInvterm.cpp:1530-1605
    void updateFaceFlux() {
        for (int f = nB; f < nF; ++f) {
            int l = m.lc[f], r = m.rc[f];
            double xn = m.xfn[f], yn = m.yfn[f], zn = m.zfn[f];
            double dist = xn * (m.xcc[r] - m.xcc[l]) + yn * (m.ycc[r] - m.ycc[l]) + zn * (m.zcc[r] - m.zcc[l]);
            double uuj = Vdvu[f] * (pp[l] - pp[r]) * xn / dist;
            double vvj = Vdvv[f] * (pp[l] - pp[r]) * yn / dist;
            double wwj = Vdvw[f] * (pp[l] - pp[r]) * zn / dist;
            uf[f] = uf[f] + uuj; vf[f] = vf[f] + vvj; wf[f] = wf[f] + wwj;
            double fux = rf[f] * (xn * uuj + yn * vvj + zn * wwj) * m.area[f];
            fq[f] = fq[f] + fux;
        }
        for (int f = 0; f < nB; ++f) {   // zero face corrections
            double fux = rf[f] * (m.xfn[f] * 0.0 + m.yfn[f] * 0.0 + m.zfn[f] * 0.0) * m.area[f];
            fq[f] = fq[f] + fux;
        }
    }

    // -------- UINsInvterm::UpdateINsRes, UINsInvterm.cpp:1842-1982 (the
    // off-diagonal sums mu mv mw persist across inner steps, as there)
    void residuals() {
        double s[4] = {0, 0, 0, 0};
        for (int f = 0; f < nF; ++f) {
            int l = m.lc[f], r = m.rc[f];
            bp[l] += -fq[f];
            bp[r] += fq[f];
        }
        for (int c = 0; c < nC; ++c) {
            for (int f : m.c2f[c]) {
                int l = m.lc[f], r = m.rc[f];
                if (c == l) {
                    mu[c] += -ai0[f] * (up[r] - uc[r]);
                    mv[c] += -ai0[f] * (vp[r] - vc[r]);
                    mw[c] += -ai0[f] * (wp[r] - wc[r]);
                } else {
                    mu[c] += -ai1[f] * (up[l] - uc[l]);
                    mv[c] += -ai1[f] * (vp[l] - vc[l]);
                    mw[c] += -ai1[f] * (wp[l] - wc[l]);
                }
            }
            double mua = spc[c] * (up[c] - uc[c]) + mu[c];
            double mva = spc[c] * (vp[c] - vc[c]) + mv[c];
            double mwa = spc[c] * (wp[c] - wc[c]) + mw[c];
            s[0] += mua * mua; s[1] += mva * mva; s[2] += mwa * mwa; s[3] += bp[c] * bp[c];
        }
        for (int k = 0; k < 4; ++k) remax[k] = std::sqrt(s[k]);
    }

    // one inner iteration: INsCalcRHS, codes/ins/src/INsRhs.cpp:105-132
    void inner() {
        bool first = innerSteps == 0;
        ++innerSteps;
        ++m.outerSteps;
        if (first) preflux();
        invCoef();
        velPresGrad();
        visCoef();
        unsteadyCoef(first);
        source();
        momentum();
        faceFlux();
        pressureCoef();
        pressureCorrection();
        updateSpeed();
        updateFaceFlux();
        residuals();
    }

    // MG::Run with startStrategy 2 (codes/multigrid/src/Multigrid.cpp:111-147):
    // inner steps while any momentum residual exceeds 1e-8, at most maxIter
    int run(int maxIter) {
        int n = 0;
        while ((remax[0] > 1e-8 || remax[1] > 1e-8 || remax[2] > 1e-8) && innerSteps < maxIter) { inner(); ++n; }
        return n;
    }
};

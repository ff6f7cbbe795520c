// Launch sequences of the tasks, templated on the face arithmetic type.
// Included by one translation unit per precision (ofg_k64.cu is compiled
// without FMA contraction so that the FP64 path rounds like the reference).
#pragma once
#include "ofg_ctx.h"
#include "ofg_kernels.cuh"
#include "ofg_turb.cuh"

namespace ofg {

// CFL ramp (TimeStep::CalcCfl, codes/ns/src/TimeStep.cpp:43-59).  step < 0:
// advance the device-side outer-step counter first (graph path).  Also resets
// the zone-wide minimum time step that the residual kernel's blocks lower.
static __global__ void k_cfl(double *scal, double step, double cflst, double cfled, int ncfl) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    scal[S_MINDT] = 1.0e40;
    double it = step;
    if (step < 0) { scal[S_STEP] += 1.0; it = scal[S_STEP]; } else { scal[S_STEP] = step; }
    double cfl = cfled;
    if (it < ncfl) {
        double delta = (cfled - cflst) / ncfl;
        cfl = cflst + delta * it;
    }
    scal[S_CFL] = cfl;
}

static __global__ void k_norm_hist(double *scal, double *hist, int cap) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int n = int(scal[S_HISTN]);
    if (n < cap)
        for (int e = 0; e < NEQ; ++e) hist[(size_t)n * NEQ + e] = scal[S_NORM + e];
    scal[S_HISTN] = double(n + 1);
}

template <typename R>
KArgs<R> make_args(ofg_ctx *c, bool onCurrent) {
    KArgs<R> A;
    A.P = c->dp;
    A.nCells = c->nCells; A.nBFaces = c->nBFaces; A.nFaces = c->nFaces; A.nT = c->nT;
    A.nb_off = c->d_nb_off; A.nbl = reinterpret_cast<const int2 *>(c->d_nbl);
    A.lo_off = c->d_lo_off; A.lol = reinterpret_cast<const int2 *>(c->d_lol);
    A.up_off = c->d_up_off; A.upl = reinterpret_cast<const int2 *>(c->d_upl);
    A.bcType = c->d_bct; A.key = c->d_key; A.walldist = c->d_wdist;
    A.fgeo = static_cast<const R *>(c->d_fgeo); A.cgeo = static_cast<const R *>(c->d_cgeo);
    A.fgeoD = sizeof(R) == 8 ? static_cast<const double *>(c->d_fgeo) : c->d_fgeoD;
    A.fofs = c->d_fofs; A.lr = reinterpret_cast<const int2 *>(c->d_lr); A.fout = c->d_fout;
    int nx = onCurrent ? c->cur : c->cur ^ 1;
    A.q = c->d_q[c->cur];
    A.qn = c->d_q[nx];
    if (sizeof(R) == 4) {
        A.qs = reinterpret_cast<const R *>(c->d_qs[c->cur]);
        A.qsn = reinterpret_cast<R *>(c->d_qs[nx]);
    } else {
        A.qs = reinterpret_cast<const R *>(A.q);
        A.qsn = reinterpret_cast<R *>(A.qn);
    }
    A.res = c->d_res; A.dq = static_cast<R *>(c->d_dq); A.dt = c->d_dt; A.invsr = c->d_invsr; A.vissr = c->d_vissr;
    A.rad = c->d_rad;
    A.bcq = c->d_bcq; A.gl = static_cast<R *>(c->d_gl); A.mm = static_cast<R *>(c->d_mm);
    A.partial = c->d_partial; A.scal = c->d_scal; A.fixlist = c->d_fix; A.fixcap = c->fixcap;
    A.npart = c->d_npart; A.tpart = c->d_tpart; A.red = c->d_red; A.redCount = c->d_redCount;
    A.nut = c->d_nut; A.dnut = c->d_dnut; A.resT = c->d_resT; A.impsrT = c->d_impsrT;
    A.matL = c->d_matL; A.matR = c->d_matR; A.gnut = static_cast<R *>(c->d_gnut);
    return A;
}

inline int nblk(long long n, int b) { return int((n + b - 1) / b); }

#define OFG_LAUNCH(kern, grid, block, stream, ...)                         \
    do {                                                                   \
        kern<<<(grid), (block), 0, (stream)>>>(__VA_ARGS__);               \
        ++c->launches;                                                     \
    } while (0)

// gradients and limiter of the current state (UPDATE_RESIDUALS' first half)
template <typename R>
void launch_gradlim(ofg_ctx *c, const KArgs<R> &A, cudaStream_t s) {
    const int N = c->nCells;
    bool needGrad = c->p.ilim != -1 || c->p.vismodel > 0;
    if (!needGrad) return;
    int nvar = c->p.vismodel > 0 ? 6 : 5;
    bool venkatGlobal = c->p.ilim == 2 && !c->p.venkat_kh3;
    int limMode = (c->p.ilim == 1 || c->p.ilim == 2) ? (venkatGlobal ? 2 : 1) : 0;
    int nb = nblk(N, 128);
    if constexpr (sizeof(R) == 4) {
        const int gb = c->tune.grad_block == 64 ? 64 : 128;   // the limiter's block extremes are exact either way
        nb = nblk(N, gb);
        switch (c->tune.grad_min_blocks) {
        case 4: OFG_LAUNCH((k_gradlim<R, 4>), nb, gb, s, A, nvar, limMode); break;
        case 8: OFG_LAUNCH((k_gradlim<R, 8>), nb, gb, s, A, nvar, limMode); break;
        default: OFG_LAUNCH((k_gradlim<R, 6>), nb, gb, s, A, nvar, limMode); break;
        }
    } else {
        OFG_LAUNCH(k_gradlim<R>, nb, 128, s, A, nvar, limMode);
    }
    if (limMode == 2) {
        OFG_LAUNCH(k_limiter_eps<R>, 1, 256, s, A, nb);
        OFG_LAUNCH(k_limiter_global<R>, nb, 128, s, A);
    }
}

// The flux / time-step pass of MODE (as k_residual): the FP64 path's
// per-cell gather, or the mixed path's face pass followed by the per-cell sum
// of the face results (part: 1 the first kernel only, 2 the second only, 3 both).
template <typename R, int MODE>
void launch_flux(ofg_ctx *c, const KArgs<R> &A, cudaStream_t s, int part = 3) {
    const int N = c->nCells;
    const bool vv = c->p.ivischeme >= 2;   // the TEST / NEW1 / NEW2 viscous face gradients
    if constexpr (sizeof(R) == 8) {
        if (!(part & 1)) return;
        if (vv) OFG_LAUNCH((k_residual<R, MODE, true>), nblk(N, 128), 128, s, A);
        else OFG_LAUNCH((k_residual<R, MODE>), nblk(N, 128), 128, s, A);
    } else {
        if (part & 1) {
            const int F = c->nFaces, bs = c->tune.face_block;
            if (vv) {
                OFG_LAUNCH((k_face_pass<MODE, true>), nblk(F, 128), 128, s, A);
            } else if constexpr (MODE == 0) {   // the iteration's pass: the tuned shape
                switch (c->tune.face_min_blocks) {
                case 2: OFG_LAUNCH((k_face_pass<0, false, 2>), nblk(F, bs), bs, s, A); break;
                case 4: OFG_LAUNCH((k_face_pass<0, false, 4>), nblk(F, bs), bs, s, A); break;
                case 5: OFG_LAUNCH((k_face_pass<0, false, 5>), nblk(F, bs), bs, s, A); break;
                default: OFG_LAUNCH((k_face_pass<0, false, 3>), nblk(F, bs), bs, s, A); break;
                }
            } else {
                OFG_LAUNCH((k_face_pass<MODE>), nblk(F, 128), 128, s, A);
            }
        }
        if (part & 2) OFG_LAUNCH((k_face_sum<MODE>), nblk(N, 128), 128, s, A);
    }
}

template <typename R>
int launch_task(ofg_ctx *c, int task, cudaStream_t s) {
    const int N = c->nCells;
    switch (task) {
    case T_CFL: {
        OFG_LAUNCH(k_cfl, 1, 32, s, c->d_scal, double(c->outerSteps), c->p.cflst, c->p.cfled, c->p.ncfl);
        break;
    }
    case T_ADVANCE: {
        OFG_LAUNCH(k_cfl, 1, 32, s, c->d_scal, -1.0, c->p.cflst, c->p.cfled, c->p.ncfl);
        break;
    }
    case T_TIMESTEP: {   // CALC_TIME_STEP alone (after T_CFL, which resets the minimum)
        KArgs<R> A = make_args<R>(c, false);
        launch_flux<R, 1>(c, A, s);
        OFG_LAUNCH(k_timestep_clip<R>, nblk(N, 256), 256, s, A);
        break;
    }
    case T_RESIDUAL: {   // UPDATE_RESIDUALS alone
        KArgs<R> A = make_args<R>(c, false);
        launch_gradlim<R>(c, A, s);
        launch_flux<R, 2>(c, A, s);
        break;
    }
    case T_TS_RES:       // CALC_TIME_STEP + LOAD_RESIDUALS + UPDATE_RESIDUALS in one gather
    case T_P_GRADLIM:    // (its three parts, launched separately by the profiler)
    case T_P_FLUX:
    case T_P_FSUM:
    case T_P_CLIP: {
        KArgs<R> A = make_args<R>(c, false);
        if (task == T_TS_RES || task == T_P_GRADLIM) launch_gradlim<R>(c, A, s);
        if (task == T_TS_RES) launch_flux<R, 0>(c, A, s);
        if (task == T_P_FLUX) launch_flux<R, 0>(c, A, s, 1);
        if (task == T_P_FSUM) launch_flux<R, 0>(c, A, s, 2);
        if (task == T_TS_RES || task == T_P_CLIP) OFG_LAUNCH(k_timestep_clip<R>, nblk(N, 256), 256, s, A);
        break;
    }
    case T_CALC_LHS: {   // CALC_LHS of the multi-stage scheme (same 128-cell blocks as the norm partials)
        KArgs<R> A = make_args<R>(c, false);
        OFG_LAUNCH(k_calc_lhs<R>, nblk(N, 128), 128, s, A, c->lhsCoef);
        break;
    }
    case T_LOWER: {
        KArgs<R> A = make_args<R>(c, false);
        int nl = int(c->lowOff.size()) - 1;
        if (c->tune.sweep_persistent) {
            OFG_LAUNCH(k_lusgs_lower_seq<R>, 1, kSeqThreads, s, A, (const int *)c->d_lowOrder, (const int *)c->d_lowOff, nl);
            break;
        }
        for (int l = 0; l < nl; ++l) {
            int st = c->lowOff[l], cnt = c->lowOff[l + 1] - st;
            const int *ord = (const int *)c->d_lowOrder;
            if constexpr (sizeof(R) == 4) {
                const int bs = c->tune.sweep_block;
                switch (c->tune.sweep_min_blocks) {
                case 6: OFG_LAUNCH((k_lusgs_lower<R, 6>), nblk(cnt, bs), bs, s, A, ord, st, cnt); break;
                case 10: OFG_LAUNCH((k_lusgs_lower<R, 10>), nblk(cnt, bs), bs, s, A, ord, st, cnt); break;
                default: OFG_LAUNCH((k_lusgs_lower<R, 8>), nblk(cnt, bs), bs, s, A, ord, st, cnt); break;
                }
            } else {
                OFG_LAUNCH(k_lusgs_lower<R>, nblk(cnt, 128), 128, s, A, ord, st, cnt);
            }
        }
        break;
    }
    case T_UPPER: {
        // level 0 of the upper sweep holds the cells without later
        // neighbours: their increment gains -(+0)/rad, which leaves it
        // unchanged bit for bit (add_neg_quot), so that level is not launched
        KArgs<R> A = make_args<R>(c, false);
        int nl = int(c->upOff.size()) - 1;
        if (c->tune.sweep_persistent) {
            OFG_LAUNCH(k_lusgs_upper_seq<R>, 1, kSeqThreads, s, A, (const int *)c->d_upOrder, (const int *)c->d_upOff + 1,
                       nl - 1);
            break;
        }
        for (int l = 1; l < nl; ++l) {
            int st = c->upOff[l], cnt = c->upOff[l + 1] - st;
            const int *ord = (const int *)c->d_upOrder;
            if constexpr (sizeof(R) == 4) {
                const int bs = c->tune.sweep_block;
                switch (c->tune.sweep_min_blocks) {
                case 6: OFG_LAUNCH((k_lusgs_upper<R, 6>), nblk(cnt, bs), bs, s, A, ord, st, cnt); break;
                case 10: OFG_LAUNCH((k_lusgs_upper<R, 10>), nblk(cnt, bs), bs, s, A, ord, st, cnt); break;
                default: OFG_LAUNCH((k_lusgs_upper<R, 8>), nblk(cnt, bs), bs, s, A, ord, st, cnt); break;
                }
            } else {
                OFG_LAUNCH(k_lusgs_upper<R>, nblk(cnt, 128), 128, s, A, ord, st, cnt);
            }
        }
        break;
    }
    case T_UPDATE: {
        KArgs<R> A = make_args<R>(c, false);
        OFG_LAUNCH(k_update<R>, nblk(N, 256), 256, s, A);
        OFG_LAUNCH(k_solution_fix<R>, 1, 32, s, A);
        break;
    }
    case T_BOUNDARY_NEXT: {
        KArgs<R> A = make_args<R>(c, false);
        if (c->nBFaces > 0) OFG_LAUNCH(k_boundary<R>, nblk(c->nBFaces, 256), 256, s, A, (const int *)c->d_lcb);
        break;
    }
    case T_BOUNDARY_CUR: {
        KArgs<R> A = make_args<R>(c, true);
        OFG_LAUNCH(k_interior_tvisl<R>, nblk(N, 256), 256, s, A);
        if (c->nBFaces > 0) OFG_LAUNCH(k_boundary<R>, nblk(c->nBFaces, 256), 256, s, A, (const int *)c->d_lcb);
        break;
    }
    case T_PACK_STATE: {
        KArgs<R> A = make_args<R>(c, true);
        OFG_LAUNCH(k_pack_state<R>, nblk(c->nT, 256), 256, s, A, (const double *)c->d_stage);
        break;
    }
    case T_UNPACK_STATE: {
        KArgs<R> A = make_args<R>(c, true);
        OFG_LAUNCH(k_unpack_state<R>, nblk(c->nT, 256), 256, s, A, c->d_stage);
        break;
    }
    case T_GRAD_ONLY: {   // gradients of the current buffer (no limiter), for a path that keeps none
        KArgs<R> A = make_args<R>(c, true);
        OFG_LAUNCH(k_gradlim<R>, nblk(N, 128), 128, s, A, 5, 0);
        break;
    }
    case T_FORCES: {
        KArgs<R> A = make_args<R>(c, true);
        if (c->nWall == 0) break;
        int nb = nblk(c->nWall, 256);
        if (nb > 64) nb = 64;   // the block sums fit the reduction buffer
        OFG_LAUNCH(k_forces<R>, nb, 256, s, A, reinterpret_cast<const int2 *>(c->d_wall), (const double *)c->d_wallG,
                   c->nWall, c->d_scal + S_FORCE);
        break;
    }
    case T_NORM:         // norms of the last residual, appended to the history
    case T_NORM_ONLY: {  // the same without the history entry
        KArgs<R> A = make_args<R>(c, false);
        OFG_LAUNCH(k_norm_final<R>, kRedBlocks, 256, s, A, nblk(N, 128));
        if (task == T_NORM) OFG_LAUNCH(k_norm_hist, 1, 32, s, c->d_scal, c->d_hist, c->histCap);
        break;
    }
    case T_TURB_RHS:
    case T_P_TURB_GRAD:  // (its parts, launched separately by the profiler)
    case T_P_TURB_FLUX: {
        KArgs<R> A = make_args<R>(c, true);
        if (task != T_P_TURB_FLUX) {
            if (c->nBFaces > 0) OFG_LAUNCH(k_turb_bc<R>, nblk(c->nBFaces, 256), 256, s, A, (const int *)c->d_lcb, 0);
            OFG_LAUNCH(k_turb_grad<R>, nblk(N, 128), 128, s, A);
        }
        if (task != T_P_TURB_GRAD) OFG_LAUNCH(k_turb_rhs<R>, nblk(N, 128), 128, s, A);
        break;
    }
    case T_TURB_LOWER: {
        KArgs<R> A = make_args<R>(c, true);
        int nl = int(c->lowOff.size()) - 1;
        if (c->tune.sweep_persistent) {
            OFG_LAUNCH(k_turb_lower_seq<R>, 1, kSeqThreads, s, A, (const int *)c->d_lowOrder, (const int *)c->d_lowOff, nl);
            break;
        }
        for (int l = 0; l < nl; ++l) {
            int st = c->lowOff[l], cnt = c->lowOff[l + 1] - st;
            OFG_LAUNCH(k_turb_lower<R>, nblk(cnt, 128), 128, s, A, (const int *)c->d_lowOrder, st, cnt);
        }
        break;
    }
    case T_TURB_UPPER: {   // level 0 skipped, as in T_UPPER
        KArgs<R> A = make_args<R>(c, true);
        int nl = int(c->upOff.size()) - 1;
        if (c->tune.sweep_persistent) {
            OFG_LAUNCH(k_turb_upper_seq<R>, 1, kSeqThreads, s, A, (const int *)c->d_upOrder, (const int *)c->d_upOff + 1,
                       nl - 1);
            break;
        }
        for (int l = 1; l < nl; ++l) {
            int st = c->upOff[l], cnt = c->upOff[l + 1] - st;
            OFG_LAUNCH(k_turb_upper<R>, nblk(cnt, 128), 128, s, A, (const int *)c->d_upOrder, st, cnt);
        }
        break;
    }
    case T_TURB_UPDATE: {
        KArgs<R> A = make_args<R>(c, true);
        OFG_LAUNCH(k_turb_update<R>, nblk(N, 256), 256, s, A, 1);
        break;
    }
    case T_TURB_BOUNDARY: {
        KArgs<R> A = make_args<R>(c, true);
        if (c->nBFaces > 0) OFG_LAUNCH(k_turb_bc<R>, nblk(c->nBFaces, 256), 256, s, A, (const int *)c->d_lcb, 1);
        break;
    }
    case T_TURB_BOUNDARY_CUR: {
        KArgs<R> A = make_args<R>(c, true);
        OFG_LAUNCH(k_turb_vist<R>, nblk(N, 256), 256, s, A);
        if (c->nBFaces > 0) OFG_LAUNCH(k_turb_bc<R>, nblk(c->nBFaces, 256), 256, s, A, (const int *)c->d_lcb, 1);
        break;
    }
    case T_TURB_NORM:
    case T_TURB_NORM_ONLY: {
        KArgs<R> A = make_args<R>(c, true);
        OFG_LAUNCH(k_turb_norm_final<R>, kRedBlocks, 256, s, A, nblk(N, 128),
                   task == T_TURB_NORM ? c->d_thist : (double *)nullptr, c->histCap);
        break;
    }
    default:
        return c->fail(OFG_E_ARG, "unknown task");
    }
    return OFG_OK;
}

}  // namespace ofg

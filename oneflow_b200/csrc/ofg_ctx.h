// Host-side context of one solve: mesh, parameters, device buffers and the
// captured CUDA graphs of one outer iteration.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/oneflow_b200.h"
#include "ofg_device.cuh"

struct ofg_ctx {
    ofg_params p{};
    ofg::DevParams dp{};
    std::string err;
    ofg_tuning tune{3, 128, 6, 8, 128, 0, 128, {0}, 0.0, 0.0};   // launch shapes of the gathers and sweeps
    unsigned long long meshHash = 0;                         // of the face->cell lists (autotuner cache key)

    // ---- mesh (host copies, reference numbering) ----
    int nCells = 0, nBFaces = 0, nFaces = 0, nT = 0;
    std::vector<int> lc, rc, bct, c2f_off, c2f;
    std::vector<double> xfn, yfn, zfn, area, xfc, yfc, zfc, xcc, ycc, zcc, vol, wdist;
    std::vector<double> xN, yN, zN;                      // nodes, and the face->node lists (CSR, reversed
    std::vector<int> fOff, fNod;                         // faces turned) the metrics were computed from
    std::vector<int> lowOrder, lowOff, upOrder, upOff;   // LU-SGS level schedules
    std::vector<int> key, keyOrder;                      // sweep position of each cell, and its inverse
    bool haveMesh = false, haveState = false;

    // ---- device ----
    cudaStream_t stream = nullptr;      // stream every launch goes to
    cudaStream_t ownStream = nullptr;   // the context's own stream (set when a caller's stream is in use)
    int *d_lcb = nullptr, *d_bct = nullptr;                 // left cell and BC code of each boundary face
    int *d_nb_off = nullptr, *d_nbl = nullptr;              // per-cell neighbour lists (int2 pairs)
    int *d_lo_off = nullptr, *d_lol = nullptr, *d_up_off = nullptr, *d_upl = nullptr;
    int *d_lowOrder = nullptr, *d_upOrder = nullptr, *d_key = nullptr;
    int *d_lowOff = nullptr, *d_upOff = nullptr;           // level offsets of the sweeps (persistent form)
    void *d_fgeo = nullptr, *d_cgeo = nullptr;              // face / cell records at the face precision
    double *d_fgeoD = nullptr;                              // mixed path: FP64 face records
    float *d_fofs = nullptr;                                // mixed path: face-local offsets [F][FOFS]
    int *d_lr = nullptr;                                    // mixed path: {left, right} cell of each face
    double *d_fout = nullptr;                               // mixed path: face-pass results [F][FOR]
    double *d_wdist = nullptr;
    int nWall = 0;
    int *d_wall = nullptr;                                  // solid-wall faces {face, interior cell} (int2)
    double *d_wallG = nullptr;                              // their FP64 geometry [nWall][16] (k_forces)
    double *d_q[2] = {nullptr, nullptr};
    float *d_qs[2] = {nullptr, nullptr};                    // FP32 copies of the state records (mixed path)
    int cur = 0;
    double lhsCoef = 1.0;       // lhscoef of the next CALC_LHS (multi-stage scheme)
    int lastResBuf = -1;        // state buffer of the last residual pass (-1: none since the state was set)
    bool pendingNext = false;   // UPDATE_FLOWFIELD wrote d_q[cur^1], CALC_BOUNDARY not yet run
    bool pendingTurb = false;   // SA UPDATE_FLOWFIELD ran, its CALC_BOUNDARY not yet
    double *d_res = nullptr, *d_dt = nullptr, *d_invsr = nullptr, *d_vissr = nullptr, *d_rad = nullptr;
    void *d_dq = nullptr;                                   // [nCells][DQR] at the face precision
    double *d_stage = nullptr;                              // [5][nT] state transfer staging (on first use)
    double *d_bcq = nullptr, *d_partial = nullptr, *d_scal = nullptr, *d_hist = nullptr;
    double *d_npart = nullptr, *d_tpart = nullptr;          // per-block sums of squares of the residuals
    double *d_red = nullptr;                                // [kRedBlocks][5] block sums of the grid reductions
    unsigned int *d_redCount = nullptr;                     // their ticket counter (0 between launches)
    void *d_gl = nullptr, *d_mm = nullptr;                  // gradient+limiter records, min/max differences
    int *d_fix = nullptr;
    // SA solver
    double *d_nut = nullptr, *d_dnut = nullptr, *d_resT = nullptr, *d_impsrT = nullptr, *d_matL = nullptr,
           *d_matR = nullptr, *d_thist = nullptr;
    void *d_gnut = nullptr;
    std::vector<double> thist;         // host copy of the SA residual history
    int fixcap = 4096;
    int histCap = 0;
    size_t nPartialMax = 0;

    // ---- iteration state ----
    long long outerSteps = 0;
    long long launches = 0;
    std::vector<double> hist;          // host copy of residual history
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    cudaGraph_t graphT[2] = {nullptr, nullptr};   // their templates (child graphs of a batch)
    unsigned graphGen = 0;                         // bumped whenever the graphs are dropped
    long long graphKernels[2] = {0, 0};

    int fail(int code, const std::string &msg) {
        err = msg;
        return code;
    }
};

namespace ofg {
// tasks executed by the precision-specific launchers
enum Task {
    T_CFL = 0, T_TIMESTEP, T_RESIDUAL, T_LOWER, T_UPPER, T_UPDATE, T_BOUNDARY_NEXT, T_BOUNDARY_CUR,
    T_NORM, T_ADVANCE, T_TS_RES, T_NORM_ONLY, T_PACK_STATE, T_UNPACK_STATE,
    T_TURB_RHS, T_TURB_LOWER, T_TURB_UPPER, T_TURB_UPDATE, T_TURB_BOUNDARY, T_TURB_BOUNDARY_CUR, T_TURB_NORM,
    T_TURB_NORM_ONLY,
    // parts of T_TS_RES / T_TURB_RHS, timed separately by ofg_profile_step
    T_P_GRADLIM, T_P_FLUX, T_P_CLIP, T_P_TURB_GRAD, T_P_TURB_FLUX, T_P_FSUM,
    T_FORCES, T_GRAD_ONLY, T_CALC_LHS
};
int launch_task_f64(ofg_ctx *c, int task, cudaStream_t s);
int launch_task_f32(ofg_ctx *c, int task, cudaStream_t s);
// ofg_geom.cu: metrics (metrics = true) and/or the wall distance on the GPU
int gpu_geometry(ofg_ctx *c, const std::vector<double> &X, const std::vector<double> &Y,
                 const std::vector<double> &Z, const std::vector<int> &fOff, const std::vector<int> &fNod,
                 bool metrics, bool wallDist);
}  // namespace ofg

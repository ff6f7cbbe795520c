/*
 * oneflow_b200.h -- C ABI of the B200 implementation of OneFLOW's
 * unstructured finite-volume residual + LU-SGS update path.
 *
 * The reference dispatches one iteration of a steady solve as string tasks
 * (codes/solver/src/TimeIntegral.cpp:113-130, names mapped to classes in
 * system/ns/function/funcMap.txt) operating on fields owned by UnsGrid.  Each
 * task below replaces one of those tasks for one solver (tid 0 = NS_SOLVER,
 * tid 1 = TURB_SOLVER); the context owns the device copies of every field.
 *
 * All functions return 0 on success and a negative OFG_E* code on failure;
 * ofg_last_error() gives the message.  Nothing aborts the process (the
 * reference's Stop() at codes/project/src/Stop.cpp:27-40 is replaced by
 * status codes).  Host pointers are borrowed for the duration of the call.
 * Arrays use the reference's numbering and its structure-of-arrays layout:
 * a per-equation field is [nEqu][nCells + nBFaces] (ghost cell of boundary
 * face f at index nCells + f), matching MRField in
 * codes/array/include/Marray.h:29-60.
 */
#ifndef ONEFLOW_B200_H
#define ONEFLOW_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define OFG_OK            0
#define OFG_E_ARG        -1   /* bad argument / size                         */
#define OFG_E_CUDA       -2   /* CUDA runtime error                          */
#define OFG_E_NAN        -3   /* NaN in a residual (reference: Stop("NotANumber"),
                                 codes/residual/src/ResidualTask.cpp:95-100)   */
#define OFG_E_STATE      -4   /* call out of order (no mesh, no state, ...)  */
#define OFG_E_TIMEOUT    -5   /* a bounded device wait gave up               */
#define OFG_E_NOMEM      -6   /* device allocation failed                    */
#define OFG_E_SIZE       -7   /* request larger than a fixed scratch allows  */
#define OFG_E_IO         -8   /* file could not be opened, read or written   */

/* solver ids: the reference's SolverState::tid less one (its NS_SOLVER = 1,
   TURB_SOLVER = 2, codes/global/include/SolverDef.h:31-32) */
#define OFG_NS_SOLVER     0
#define OFG_TURB_SOLVER   1

/* boundary codes (reference BC::*, codes/geometry/src/Boundary.cpp:35-54) */
#define OFG_BC_EXTRAPOLATION 1
#define OFG_BC_SOLID_SURFACE 2
#define OFG_BC_SYMMETRY      3
#define OFG_BC_FARFIELD      4
#define OFG_BC_INFLOW        5
#define OFG_BC_OUTFLOW       6

/* arithmetic of the face terms */
#define OFG_PREC_FP64     0   /* every step in FP64 (the all-FP64 oracle path) */
#define OFG_PREC_MIXED    1   /* FP32 fluxes/gradients/limiters/SA source; FP64
                                 residual accumulation, update and norms        */

/*
 * Solver parameters: the script keys the reference reads with
 * GetDataValue<T>("key") on this path (codes/ns/src/NsCom.cpp:45-94,
 * codes/global/src/Ctrl.cpp:40-113, codes/turb/src/TurbCom.cpp:110-350).
 * ofg_default_params() fills the reference's test-case defaults.
 */
typedef struct ofg_params {
    int    dimension;        /* 2 or 3                                         */
    int    ischeme;          /* 1 Roe, 12 SLAU2                                */
    int    ilim;             /* -1 first order, 0 none, 1 Barth, 2 Venkat      */
    int    igrad;            /* 0 GG cell-weighted (reference), 1 GG face
                                average, 2 weighted least squares (new)        */
    int    ieigenfix;
    int    timestepModel;    /* 0 local, 1 global, 2 local->min                */
    int    ncfl;
    int    visSRModel;       /* 1,2,3                                          */
    int    visTimeStepModel;
    int    vismodel;         /* 0 Euler, 1 laminar, 3 SA                       */
    int    ivischeme;        /* 0 std, 1 aver, 2 test, 3 new1, 4 new2         */
    int    isowallbc;        /* 0 adiabatic, 1 isothermal                      */
    int    iprod_sa;         /* SA production form                             */
    int    ft2_flag;
    int    turb_ilim;        /* only -1 (first order SA convection) supported  */
    int    precision;        /* OFG_PREC_*                                     */
    int    venkat_kh3;       /* 0: eps = vencat_coef*max(qmax-qmin,1) (reference);
                                1: eps^2 = (K h)^3 with K = vencat_coef (new)  */
    int    sweep_order;      /* LU-SGS sweep order: 0 the cell numbering (reference);
                                1 colour-major: a greedy colouring of the cell
                                graph in natural order, colours ascending, cell
                                ids ascending inside a colour.  Identical to the
                                reference run on the mesh renumbered that way
                                (ofg_colour_order), with storage left in place. */
    int    time_integral;    /* 2 LU-SGS (TimeIntegral::Lusgs; 0 means 2), 1 the
                                multi-stage scheme (TimeIntegral::RungeKutta) */
    int    rk_stage;         /* stages of the multi-stage scheme (stage i scales
                                its update by 1/(i+1), codes/global/src/Ctrl.cpp:72-77) */
    int    reserved_i[4];
    double vencat_coef;
    double centropy1, centropy2;
    double cflst, cfled;
    double max_time_ratio;
    double global_dt;
    double mach_ref, aoa_degree, sideslip_degree, reynolds;
    double gama_ref, prl, prt, tref_dim, twall_dim;
    double inflow_viscosity;  /* SA nu~ of the freestream                      */
    double rprod;
    double turb_cfl_ratio;
    double ref_sa;            /* SA nu~ of the freestream (TurbCom::InitInflow)  */
    double max_vis_ratio;     /* cap of mu_t / mu_l                              */
    double reserved_d[6];
} ofg_params;

typedef struct ofg_ctx ofg_ctx;

void        ofg_default_params(ofg_params *p);
int         ofg_params_size(void);   /* sizeof(ofg_params), for binding checks */
int         ofg_create(const ofg_params *p, ofg_ctx **out);
void        ofg_destroy(ofg_ctx *ctx);
const char *ofg_last_error(const ofg_ctx *ctx);
int         ofg_version(void);

/*
 * Mesh upload: the content of one .ofl zone (codes/geometry/src/UnsGrid.cpp:90-201).
 * lCells may be negative for a boundary face, in which case the face is
 * reversed (UnsGrid::ReadGridFaceTopology, :157-175).  Boundary faces are
 * [0, nBFaces).  Metrics (UnsGrid::CalcMetrics, :469-900) are computed here,
 * on the GPU.  wall_dist is per interior cell; NULL makes an SA solve compute
 * it (ofg_calc_wall_dist) and is ignored otherwise.  Malformed input (no
 * cells or faces, indices out of range, a face of fewer than 2 (2-D) or 3
 * (3-D) nodes, an interior face with one cell on both sides, a boundary code
 * outside 1-6) returns OFG_E_ARG; after any refused upload the context holds
 * no mesh (calls that run kernels return OFG_E_STATE) until one succeeds.
 */
int ofg_upload_mesh(ofg_ctx *ctx, int nNodes, const double *xN, const double *yN, const double *zN,
                    int nFaces, const int *faceNodeCount, const int *faceNodes,
                    const int *lCells, const int *rCells, int nCells, int nBFaces,
                    const int *bcType, const double *wall_dist);

/* CALC_WALL_DIST (CalcWallDist + CalcPoint2FaceDist, codes/geometry/src/WallDist.cpp:136-330):
   the distance from every cell centre to the nearest SOLID_SURFACE face
   (segments in 2-D; triangles in 3-D, faces of more than three nodes fanned
   about their node average), computed on the GPU and used by the SA source
   from then on.  ofg_upload_mesh runs it by itself for an SA solve whose
   wall_dist is NULL (the reference's ireadwdst = 0); the result is readable
   as the field "walldist". */
int ofg_calc_wall_dist(ofg_ctx *ctx);

/* INIT_FLOWFIELD with startStrategy 0: freestream + CALC_BOUNDARY
   (codes/uns/src/UNsRestart.cpp:48-60, codes/ns/src/NsSolverImp.cpp:61-73). */
int ofg_init_flowfield(ofg_ctx *ctx);

/* state transfer, reference layout [nEqu][nCells+nBFaces] (primitive q for
   NS: rho,u,v,w,p; nu~ for SA).  Upload runs CALC_BOUNDARY for that solver. */
int ofg_upload_state(ofg_ctx *ctx, int tid, const double *q);
int ofg_download_state(ofg_ctx *ctx, int tid, double *q);

/* Restart files in the reference's layout (READ_RESTART / DUMP_RESTART:
   Restart::Read / Restart::Dump, codes/restart/src/Restart.cpp:144-164, with
   ReadRestartHeader / DumpRestartHeader :178-182,190-194 and ReadUnsteady /
   DumpUnsteady :74-120, written per zone by DataBook::WriteFile,
   codes/database/src/DataBook.cpp:283-316).  One single-zone record:
     int64 byte count of what follows, int32 outer step, f64 current time,
     q1[n][nT], q2[n][nT], res1[n][nT], res2[n][nT]   (f64, n = 5 for NS
     "flowFile", 1 for SA "turbflowFile", nT = nCells + nBFaces)
   Write: q1 = the current state; q2 = the state one outer iteration earlier
   (Unsteady::UpdateUnsteady, codes/unsteady/src/Unsteady.cpp:44-58, shifts q1
   into q2 after every outer step; here the NS solver's other state buffer,
   or q1 when no iteration has completed since the state was set; always q1
   for SA, whose update is in place);
   res1 = res2 = 0 (a steady run never sets them).  The outer step written is
   the context's counter.
   Read: the state becomes q1 (as Restart::ReadUnsteady sets q = q1), CALC_BOUNDARY
   runs as after ofg_upload_state, and for the NS solver the context's outer
   step counter is set from the file (the CFL ramp continues from it).  The
   file's step and time are returned through the optional pointers.  A record
   of another size (another mesh, interface data of a multi-zone grid) is
   rejected with OFG_E_ARG; file errors return OFG_E_IO. */
int ofg_write_restart(ofg_ctx *ctx, int tid, const char *path, double curr_time);
int ofg_read_restart(ofg_ctx *ctx, int tid, const char *path, int64_t *outer_step, double *curr_time);

/* CALC_LHS of the multi-stage scheme (ULhs::CalcLHS, codes/usolver/src/ULhs.cpp:47-65):
   res *= (dt / vol) * lhscoef, which is also the increment the next
   UPDATE_FLOWFIELD adds (UNsField::Init makes dq the residual field under
   MULTI_STAGE, codes/uns/src/UNsCom.cpp:85-88).  TimeIntegral::RungeKutta
   (codes/solver/src/TimeIntegral.cpp:81-111) calls it once per stage with
   lhscoef = 1/(stage+1).  NS solver only. */
int ofg_calc_lhs(ofg_ctx *ctx, int tid, double lhscoef);

/* One task each (system/ns/function/funcMap.txt, codes/turb/src/TurbSolverImp.cpp:33-42). */
int ofg_zero_dq(ofg_ctx *ctx, int tid);             /* ZERO_DQ_FIELD          */
int ofg_calc_time_step(ofg_ctx *ctx, int tid);      /* CALC_TIME_STEP         */
int ofg_load_residuals(ofg_ctx *ctx, int tid);      /* LOAD_RESIDUALS         */
int ofg_update_residuals(ofg_ctx *ctx, int tid);    /* UPDATE_RESIDUALS       */
int ofg_init_lusgs(ofg_ctx *ctx, int tid);          /* INIT_LUSGS (no-op)     */
int ofg_lusgs_lower(ofg_ctx *ctx, int tid);         /* LUSGS_LOWER_SWEEP      */
int ofg_lusgs_upper(ofg_ctx *ctx, int tid);         /* LUSGS_UPPER_SWEEP      */
int ofg_update_flowfield(ofg_ctx *ctx, int tid);    /* UPDATE_FLOWFIELD_LUSGS */
int ofg_calc_boundary(ofg_ctx *ctx, int tid);       /* CALC_BOUNDARY          */

/* The whole TimeIntegral::Lusgs sequence for every solver, nsteps outer
   iterations (MG::Run with StrongIter, codes/multigrid/src/Multigrid.cpp:111-169,
   :349-360), with the RMS residual of every iteration appended to the history. */
int ofg_step(ofg_ctx *ctx, int nsteps);

/* Batched solves: n independent contexts (each its own mesh, parameters and
   state) advanced together, as if ofg_step(ctx, nsteps) ran on each: one
   CUDA-graph launch per outer iteration whose branches are the contexts'
   own iteration graphs, so that many small solves share the GPU at once.
   The reference runs one case per process (MG::Run); this replaces a set of
   such runs.  Results are bitwise those of ofg_step on each context.  The
   contexts stay usable on their own between batch steps (the batch rebuilds
   its graph when one of them changed).  Errors name the context. */
typedef struct ofg_batch ofg_batch;
int         ofg_batch_create(ofg_ctx *const *ctxs, int n, ofg_batch **out);
int         ofg_batch_step(ofg_batch *batch, int nsteps);
void        ofg_batch_destroy(ofg_batch *batch);
const char *ofg_batch_last_error(const ofg_batch *batch);
/* Device time of the last successful ofg_batch_step, in milliseconds: CUDA
   events on the batch's stream before its first and after its last graph
   launch.  OFG_E_ARG before the first step. */
int         ofg_batch_device_ms(const ofg_batch *batch, float *ms);

/* Coordinate MLP for warm starts (no counterpart in the reference): n_in
   inputs -> depth hidden layers of `width` (a multiple of 16) with GELU ->
   n_out outputs; BF16 weights and activations on the tensor cores with FP32
   accumulation, FP32 master weights, Adam (beta 0.9 / 0.999, eps 1e-8), mean
   squared error.  Weights start U(-1/sqrt(fan_in), 1/sqrt(fan_in)) from
   `seed`, biases 0.  x, y are device arrays [n][n_in], [n][n_out] (FP32).
   Parameters as one host array: per layer W[fan_in][fan_out], then b. */
typedef struct ofg_mlp ofg_mlp;
int         ofg_mlp_create(int n_in, int width, int depth, int n_out, uint64_t seed, ofg_mlp **out);
void        ofg_mlp_destroy(ofg_mlp *mlp);
const char *ofg_mlp_last_error(const ofg_mlp *mlp);
int64_t     ofg_mlp_num_params(const ofg_mlp *mlp);
int         ofg_mlp_get_params(ofg_mlp *mlp, float *out);
int         ofg_mlp_set_params(ofg_mlp *mlp, const float *in);     /* also resets the Adam moments */
int         ofg_mlp_predict(ofg_mlp *mlp, const float *x, int64_t n, float *y);
/* loss and gradient (host, parameter layout) of one batch, n a multiple of
   64 up to 65,536; no update */
int         ofg_mlp_loss_grad(ofg_mlp *mlp, const float *x, const float *y, int64_t n, float *loss, float *grad);
/* `steps` Adam steps at rate lr on minibatches of `batch` rows (a multiple of
   64 up to 65,536) drawn by a seeded hash; loss_out[steps] (host, may be
   NULL) gets each minibatch's loss */
int         ofg_mlp_train(ofg_mlp *mlp, const float *x, const float *y, int64_t n, int batch, int steps, float lr,
                          uint64_t seed, float *loss_out);

/* RMS residual per equation of the solver's last UPDATE_RESIDUALS
   (ResidualTask::CalcRes + ResAver::CalcAver,
   codes/residual/src/ResidualTask.cpp:75-126, codes/residual/src/Residual.cpp:52-72):
   rms[0..4] for the NS solver, rms[0] for the SA solver.  The residual
   history is not touched. */
int ofg_residual_norms(ofg_ctx *ctx, int tid, double *rms);

/* Largest |residual| per equation of the solver's last UPDATE_RESIDUALS and
   the first cell (lowest index) that holds it -- the resmax record of
   ResidualTask::CalcRes (codes/residual/src/ResidualTask.cpp:91-123; its
   centre and volume are the fields "xcc".."vol" at that index).  resmax and
   cell get 5 entries (NS) or 1 (SA). */
int ofg_residual_max(ofg_ctx *ctx, int tid, double *resmax, int64_t *cell);

/* Named device field -> host, reference layout:
   "res","dq","timestep","invsr","vissr","impsr","limiter","dqdx","dqdy","dqdz",
   "tempr","visl","vist","vol","xcc","ycc","zcc","area","xfn","yfn","zfn",
   "xfc","yfc","zfc","walldist".
   n_out = capacity in doubles; the size needed is returned in *n_needed. */
int ofg_download_field(ofg_ctx *ctx, int tid, const char *name, double *out, int64_t n_out,
                       int64_t *n_needed);

/* Aerodynamic forces of the current state on the solid-wall faces
   (AerodynamicForceTask: CalcAeroForce, codes/force/src/AeroForceTask.cpp:186-451,
   compressible branch; AeroForceInfo::CalcCoef, codes/force/src/Force.cpp:254-269):
   wall pressure extrapolated with the interior cell's gradient of the last
   UPDATE_RESIDUALS, viscous stress from its velocity gradient corrected
   along the cell-to-ghost line.  out[13]: total force x y z, pressure part
   x y z, viscous part x y z (sums over the wall faces, nondimensional as in
   the reference), CL, CD, CD_pres, CD_vis with reference area aref.
   (The reference does not accumulate moments, so none are returned.) */
int ofg_forces(ofg_ctx *ctx, double aref, double *out);

/* Run every later launch of this context on the caller's CUDA stream
   (a cudaStream_t passed as void*; NULL restores the context's own stream).
   Captured graphs are rebuilt on the next ofg_step. */
int ofg_set_stream(ofg_ctx *ctx, void *stream);

/* One outer iteration launched task by task (no graph) with CUDA events
   between the groups; ms[] receives the device time of: CFL advance;
   CALC_TIME_STEP + UPDATE_RESIDUALS as its parts (gradients + limiter;
   the flux/time-step pass -- the FP64 path's per-cell gather, the mixed
   path's face pass; the mixed path's per-cell sum of the face results, an
   empty group on the FP64 path; time-step clip); LUSGS_LOWER_SWEEP,
   LUSGS_UPPER_SWEEP, UPDATE_FLOWFIELD, CALC_BOUNDARY, residual norm; and
   with the SA model seven more (nu~ boundary + gradient, its rhs gather,
   lower, upper, update, boundary, norm);
   launches[] the number of kernel launches of each group.  Both arrays
   must hold 17 entries. */
int ofg_profile_step(ofg_ctx *ctx, double *ms, int *launches);

/* Number of dependency levels of the lower and upper LU-SGS sweeps in the
   uploaded cell numbering (each level is one parallel launch). */
int ofg_sweep_levels(ofg_ctx *ctx, int *lower_levels, int *upper_levels);

/* Iteration::outerSteps for the task-level API (the CFL ramp of the next
   CALC_TIME_STEP reads it); ofg_step advances it itself. */
int ofg_set_outer_step(ofg_ctx *ctx, int64_t outer_steps);

/* Outer-iteration counter (Iteration::outerSteps) and a counter of every
   CUDA kernel launch this context issued (for reporting). */
int ofg_get_counters(ofg_ctx *ctx, int64_t *outer_steps, int64_t *kernel_launches);

/* Cell centres [nCells][3] of a mesh with the reference's metrics (host
   only, no device needed): used to build wall distances and probes. */
int ofg_cell_centres(int dimension, int nNodes, const double *xN, const double *yN, const double *zN, int nFaces,
                     const int *faceNodeCount, const int *faceNodes, const int *lCells, const int *rCells,
                     int nCells, int nBFaces, double *out);

/* Cell renumbering for the GPU sweeps: a greedy colouring of the cell graph
   (interior faces, cells visited in natural order), colours ascending and cell
   ids ascending inside a colour.  Writes perm[newId] = oldId for interior
   cells and returns the number of colours (>= 1).  Pure host function; apply
   it to the mesh arrays before ofg_upload_mesh.  Returns OFG_E_ARG for
   nCells < 1, nBFaces < 0, nFaces < nBFaces, a null pointer or an interior
   face whose cells are out of range; perm is undefined after an error. */
int ofg_colour_order(int nCells, int nFaces, int nBFaces, const int *lCells, const int *rCells,
                     int *perm);

/* Cell renumbering for locality: reverse Cuthill-McKee of the cell graph
   (cells joined by interior faces; per connected component from a
   pseudo-peripheral cell, neighbours visited in ascending degree).  Writes
   perm[newId] = oldId for interior cells.  No counterpart in the reference,
   which keeps the file's cell order (codes/geometry/src/UnsGrid.cpp:123-129);
   pure host function, applied to the mesh arrays before ofg_upload_mesh (the
   reference itself gives the same results on the renumbered mesh).  Returns
   OFG_OK, or OFG_E_ARG for the arguments ofg_colour_order rejects; perm is
   undefined after an error. */
int ofg_rcm_order(int nCells, int nFaces, int nBFaces, const int *lCells, const int *rCells, int *perm);

/* ---- launch shapes and the autotuner (no counterpart in the reference) ----
   The mixed path's heaviest gathers each exist in several compiled shapes:
   min_blocks = resident 128-thread blocks per SM asked of the compiler, i.e.
   a register cap of 65536 / (128 min_blocks) per thread (more blocks: more
   warps in flight, fewer registers, possibly spills); block = threads per
   block.  The defaults were chosen by timing the 6M-cell plate; the best
   shape depends on the mesh (cell types, size, ordering). */
typedef struct ofg_tuning {
    int    face_min_blocks;   /* face pass: 2, 3 (default), 4 or 5                 */
    int    face_block;        /* face pass threads per block: 64 or 128 (default)  */
    int    grad_min_blocks;   /* gradients + limiter: 4, 6 (default) or 8          */
    int    sweep_min_blocks;  /* LU-SGS level kernels: 6, 8 (default) or 10        */
    int    sweep_block;       /* LU-SGS level kernels: 64 or 128 (default)         */
    int    sweep_persistent;  /* 0: one launch per level (default); 1: one launch
                                 per sweep, a single block running every level
                                 with a block barrier between levels (the same
                                 bits; for many small levels).  Both paths.   */
    int    grad_block;        /* gradients + limiter threads per block: 64 or 128
                                 (default; 0 also means 128)                  */
    int    reserved[1];
    double ms_default;        /* device ms per iteration of these kernels, default shapes */
    double ms_tuned;          /* the same with the shapes chosen                   */
} ofg_tuning;

/* Times every candidate shape of the tunable kernels on this context's own
   mesh and state (each kernel group `reps` times per candidate, CUDA events,
   the median kept; one group after another, the others at their current
   choice), keeps the fastest and reports them in *out.  The groups timed are
   repeatable on a fixed state (gradients, face fluxes and residual, both
   sweeps), so the solve itself is not advanced; the captured graphs are
   rebuilt at the next ofg_step.  The result is cached per mesh (cell, face and
   boundary-face counts and a hash of the face->cell lists) and parameter set:
   a later context with the same mesh takes the cached shapes without timing.
   On the FP64 path only sweep_persistent is timed (its kernels keep their
   fixed shapes).  Needs a state (after ofg_init_flowfield / upload / a step). */
int ofg_autotune(ofg_ctx *ctx, int reps, ofg_tuning *out);
int ofg_get_tuning(ofg_ctx *ctx, ofg_tuning *out);
/* Sets the shapes (values outside the lists above return OFG_E_ARG). */
int ofg_set_tuning(ofg_ctx *ctx, const ofg_tuning *t);

/* ---- allocation-free entry point (no counterpart in the reference: OneFLOW
   computes its residual norms on the host, ResidualTask::CalcRes) ---- */

#define OFG_NOALLOC_MAX_EQ 8   /* equations per cell the fixed scratch holds */

/* RMS per equation, sqrt(sum_i res[i][e]^2 / n_cells), of a residual array
   res[n_cells][n_eq] (FP64, row per cell, e.g. the solver's own "res" layout)
   that the caller keeps in device memory; writes rms_out[n_eq] in device
   memory, stream-ordered on `stream` (a cudaStream_t, NULL = legacy default
   stream).  Same quantity as ofg_residual_norms, without a context.

   It allocates nothing: no device or host allocation, no allocating library
   routine.  It is meant for callers that must not allocate at this point --
   a host that has given the device memory to its own pool, or a convergence
   monitor running between the iterations of a solve that cannot take the
   implicit device synchronisation a cudaMalloc/cudaFree may cause.  Its
   scratch is a fixed static device array of this library (18,952 bytes per
   device: 296 blocks x 8 partial sums + a ticket), so:
     - n_eq above OFG_NOALLOC_MAX_EQ returns OFG_E_SIZE (devices with an
       ordinal of 64 or more too); n_cells may be any positive count;
     - every call first clears the scratch's ticket on `stream` (a 4-byte
       cudaMemsetAsync, which allocates nothing), then runs one kernel; the
       partial sums are rewritten by every call before they are read;
     - calls that overlap in time on the same device race on the scratch:
       serialise them (one stream, or an event between streams);
     - the first call on each device (made with that device current) looks up
       the scratch address with cudaGetSymbolAddress and loads the module;
       make that first call before capturing any stream;
     - the looked-up address is kept for the life of the process: after a
       cudaDeviceReset of a device this entry point must not be called on
       that device again (the kept address would be stale).
   Returns OFG_OK, OFG_E_ARG (null pointer, n_cells < 1, n_eq < 1), OFG_E_SIZE
   or OFG_E_CUDA. */
int ofg_residual_rms_noalloc(const double *res, int64_t n_cells, int n_eq, double *rms_out, void *stream);

/* ------------------------------------------------------------------------
   Incompressible solver: the reference's INsSolver run with startStrategy 2
   and time_integral 3 (TimeIntegral::Simple, codes/solver/src/TimeIntegral.cpp:132-138),
   whose one task UPDATE_RESIDUALS (CINsUpdateResiduals -> INsCalcRHS,
   codes/ins/src/INsRhs.cpp:105-132) is one SIMPLE inner iteration: upwind
   mass-flux and viscous face coefficients, three momentum solves and one
   pressure-correction solve by GMRES (codes/bgmres: Krylov dimension 500,
   no restart, relative tolerance 1e-8, identity preconditioner), Rhie-Chow
   face fluxes, pressure and velocity corrections (relaxation 0.8), and the
   residual maxima remax_up/vp/wp/pp.  All arithmetic is FP64.

   Scope (the reference's own): every boundary face SOLID_SURFACE -- its
   MomPre and UpdateSpeed boundary loops index the last boundary-condition
   region by boundary face id, in bounds only with a single boundary type
   (codes/uins/src/UINsInvterm.cpp:617-626, 1622-1631) -- and a viscous model
   (vismodel >= 1).  Wall velocities come per boundary face (the values its
   region carries in the reference's grid/ins_bc.txt; zero without data).
   The reference initialises its arrays on the inner step where
   currTime == 0.001, i.e. with global_dt = 0.001 only; here the first inner
   step after ofg_ins_init_flowfield does it for any global_dt.
   ------------------------------------------------------------------------ */
typedef struct ofg_ins ofg_ins;

/* Creates the solver on a context that holds a mesh (ofg_upload_mesh; its
   parameters give reynolds, mach_ref, aoa/sideslip and global_dt).
   wall_uvw: [nBFaces][3] wall velocity of each boundary face, or NULL for
   still walls.  Allocates (Krylov dimension + 2) x nTCell doubles of Krylov
   basis besides the fields.  Returns OFG_E_ARG (and *out = NULL) when the
   mesh or model is outside the scope above, OFG_E_STATE without a mesh,
   OFG_E_NOMEM. */
int ofg_ins_create(ofg_ctx *ctx, const double *wall_uvw, ofg_ins **out);
/* Destroy the solver before its context (it runs on the context's stream). */
void ofg_ins_destroy(ofg_ins *s);

/* INIT_INSRESTART + INIT_FINAL (UINsRestart::InitinsRestart,
   codes/uins/src/UINsRestart.cpp:50-62; INsInitFinal,
   codes/ins/src/INsSolverImp.cpp:58-77): q = inflow in every cell, ghost
   states of the adiabatic walls; resets the inner-step count. */
int ofg_ins_init_flowfield(ofg_ins *s);

/* Sets the state from host memory, q [5][nTCell] in the reference's layout
   (ghost cells included, as its INIT_FINAL leaves them), and resets the
   inner-step count as ofg_ins_init_flowfield does: the next inner step
   takes its previous-time velocity and initial face fluxes from this q. */
int ofg_ins_upload_state(ofg_ins *s, const double *q);

/* UPDATE_RESIDUALS of the incompressible solver: one inner iteration. */
int ofg_ins_update_residuals(ofg_ins *s);

/* MG::Run with startStrategy 2 (codes/multigrid/src/Multigrid.cpp:111-147):
   inner iterations while remax_up, remax_vp or remax_wp exceeds 1e-8 and
   fewer than max_inner have run since ofg_ins_init_flowfield; *ran (may be
   NULL) receives the number run by this call. */
int ofg_ins_run(ofg_ins *s, int max_inner, int *ran);

/* out[13]: remax_up, remax_vp, remax_wp, remax_pp of the last inner step;
   GMRES iterations of its u, v, w and pressure solves; their final residual
   norms (Rank.residual); the inner-step count. */
int ofg_ins_stats(ofg_ins *s, double *out);

/* Copies a field to host memory, reference layout: "q" [5][nTCell]
   (rho u v w p), "dqdx" "dqdy" "dqdz" [5][nTCell] (Green-Gauss gradients
   of u v w p; rho row zero), "pp" "uc" "vc" "wc" "spc" "bp" [nTCell],
   "fq" "ajp" [nFaces].  n is the capacity of out in doubles; returns
   OFG_E_SIZE when too small, OFG_E_ARG for an unknown name. */
int ofg_ins_get_field(ofg_ins *s, const char *name, double *out, int64_t n);

/* out[4]: device time (ms, CUDA events on the context's stream) of the
   inner iterations run since ofg_ins_init_flowfield, the GMRES iterations
   they took in total, the device time of those GMRES solves (ms), and the
   solves' algorithmic bytes (per Krylov step j: matrix values, columns and
   row offsets, the previous vector, the j earlier basis vectors read twice,
   three vector writes; per update: the basis vectors read, x written). */
int ofg_ins_timing(ofg_ins *s, double *out);

#ifdef __cplusplus
}
#endif
#endif

/*
 * samrai_fac_b200.h -- C ABI of the B200-native FAC Poisson hot path.
 *
 * Plain C: opaque context, plain pointers and sizes, int status returns
 * (0 = success; see fac_status).  No CUDA or C++ types cross this boundary.
 *
 * Each entry point replaces one piece of SAMRAI's cell-centred FAC path
 * (paths relative to the SAMRAI source tree):
 *   solv/CellPoissonFACSolver.{h,C}   solver wrapper      -> fac_solve*
 *   solv/FACPreconditioner.{h,C}      FAC cycling         -> fac_fac_cycle
 *   solv/CellPoissonFACOps.{h,C}      level operators     -> fac_smooth,
 *                                     fac_comp_residual, fac_restrict,
 *                                     fac_prolong_correct, fac_rms_norm ...
 *   xfer/RefineSchedule::fillData     ghost fill          -> fac_ghost_fill
 * The reference reaches its numerical kernels through the F77 ABI
 * (SAMRAI_F77_FUNC, every argument by pointer, no return value); this ABI
 * instead works one level of the whole hierarchy per call.
 *
 * One context holds a batch of independent problems ("problems") that share
 * the dimension and the number of levels; every level operation acts on
 * that level of every active problem at once.
 *
 * Cell data use SAMRAI's ArrayData layout (pdat/ArrayData.C:79-127):
 * column-major over the ghosted box, i fastest.  Host buffers passed to the
 * upload/download calls hold one level of one problem: the patches' ghosted
 * arrays concatenated in patch order.  Side data (D): per patch, axis
 * 0..dim-1, the side box (upper+1 along the axis), ghost width 0.
 */
#ifndef SAMRAI_FAC_B200_H
#define SAMRAI_FAC_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fac_ctx fac_ctx;

enum fac_status {
   FAC_OK = 0,
   FAC_ERR_ARG = 1,        /* bad argument (reference: TBOX_ERROR/TBOX_ASSERT) */
   FAC_ERR_STATE = 2,      /* call out of order (e.g. before fac_initialize) */
   FAC_ERR_CUDA = 3,       /* a CUDA runtime call failed */
   FAC_ERR_NESTING = 4,    /* hierarchy not properly nested */
   FAC_ERR_NOMEM = 5,      /* device allocation failed */
   FAC_ERR_DEVICE = 6      /* device-side error flag was set */
};

/* Cell field ids (ghost width): the vectors of FACPreconditioner and the
 * Poisson C coefficient. */
enum fac_field {
   FAC_U = 0,   /* solution u            (1) */
   FAC_F = 1,   /* right-hand side f     (0) */
   FAC_E = 2,   /* error e               (1) */
   FAC_R = 3,   /* residual r            (0) */
   FAC_TR = 4,  /* coarser-level residual (0) */
   FAC_W = 5,   /* control volume weight (0) */
   FAC_C = 6    /* Poisson C field       (0) */
};

/* Last error message of this thread (never NULL). */
const char *fac_last_error(void);

/* ---- context and hierarchy (CellPoissonFACSolver ctor,
 *      FACPreconditioner::initializeSolverState FACPreconditioner.C:158-229) */

/* Create an empty context of dimension dim (2 or 3) on CUDA device `device`.
 * device = -1 makes a host-only context: fac_initialize builds and checks
 * every device table without touching a GPU; operations then fail with
 * FAC_ERR_STATE. */
int fac_ctx_create(fac_ctx **ctx, int dim, int device);
int fac_ctx_destroy(fac_ctx *ctx);

/* Add one problem.  n0: level-0 cells per axis (physical domain is the
 * box [0,n0-1]); xlo/xup: physical extent; ratio: nlev x 3 refinement
 * ratios to the next coarser level, 1 .. 16 per axis (level 0: 1 1 1);
 * npatch: patches per level; boxes: lo0 lo1 lo2 hi0 hi1 hi2 per patch in
 * level order.
 * Returns the problem index through *problem. */
int fac_add_problem(fac_ctx *ctx, const int *n0, const double *xlo,
                    const double *xup, int nlev, const int *ratio,
                    const int *npatch, const int *boxes, int *problem);

/* Multigrid coarsest-level solve (no counterpart in the reference, whose
 * equivalent is its hypre coarse solver, CellPoissonFACOps.C:1741-1781):
 * every problem added after this call gets `levels` extra levels below its
 * level 0, each one patch covering the domain at half the previous
 * resolution, so the FAC cycle continues as a multigrid V-cycle whose
 * coarsest solve is small.  The added cells are all covered, so the
 * composite problem, its weights and norms are unchanged.  Requires a level
 * 0 that covers the domain with n0 divisible by 2^levels; call before
 * fac_add_problem.  Level numbers in every other call count the added
 * levels: the caller's level l is level l + levels, and the host tables of
 * fac_solve_host hold the caller's levels only.  D (and C) on the added
 * levels derive from the caller's level 0 (face means; C, f and u zero);
 * solves redo that after D or C of that level was uploaded, and
 * fac_extend_coefficients does it on demand. */
int fac_set_coarse_extension(fac_ctx *ctx, int levels);
int fac_extend_coefficients(fac_ctx *ctx);

/* PoissonSpecifications (solv/PoissonSpecifications.h:51-345):
 * div(D grad u) + C u = f.  d_variable: D is side data (fac_upload_side);
 * c_kind 0 = zero, 1 = constant c_const, 2 = cell field FAC_C. */
int fac_set_poisson(fac_ctx *ctx, int d_variable, double d_const,
                    int c_kind, double c_const);

/* Robin boundary coefficients a u + b du/dn = g per location index
 * 0..2*dim-1 (solv/RobinBcCoefStrategy.h; Dirichlet a=1,b=0 as
 * SimpleCellRobinBcCoefs::setBcCoefs, SimpleCellRobinBcCoefs.C:283-290).
 * May be called again after fac_initialize; later operations use the new
 * coefficients.  Once coefficients are set (here or by fac_set_bc_faces)
 * the solves leave the physical-boundary ghost cells of u as their last
 * fill leaves them, as CellPoissonFACSolver does with a caller's
 * RobinBcCoefStrategy; without them (the solver's own Dirichlet object) the
 * solves put back the ghost values u had (cacheDirichletData /
 * restoreDirichletData, CellPoissonFACSolver.C:327-349). */
int fac_set_bc(fac_ctx *ctx, const double *a, const double *b,
               const double *g);
/* Robin coefficients that vary along the boundary, as a
 * RobinBcCoefStrategy::setBcCoefs fills them per boundary face
 * (solv/RobinBcCoefStrategy.h:138-145): for one problem, level and
 * location index, abg holds (a, b, g) triples over that level's whole
 * domain face on that side (the lowest tangential axis fastest); sides
 * without them keep the constants of fac_set_bc.  The coefficients of the
 * coarse interpolation array of prolongation come from the coarser level's
 * arrays, by position, as the reference's coefficient object evaluates
 * them there.  While any are set, smoothing takes the fill-based colour
 * passes (the fused and staged ones apply side constants).  After
 * fac_initialize. */
int fac_set_bc_faces(fac_ctx *ctx, int problem, int ln, int location,
                     const double *abg);

/* Input keys of FACPreconditioner (FACPreconditioner.C:80-114) and
 * CellPoissonFACOps (CellPoissonFACOps.C:692-739).  ewing: 1 selects
 * cf_discretization "Ewing" (0 is rejected: only Ewing is implemented). */
int fac_set_params(fac_ctx *ctx, int max_cycles, double residual_tol,
                   double relative_residual_tol, int pre_sweeps,
                   int post_sweeps, double coarse_tol, int coarse_max_it,
                   int ewing);

/* 1 (default): red-black colour passes read the value across a patch face
 * from the neighbour patch's interior (or the physical-boundary formula, or
 * the Ewing flux at a coarse-fine face) instead of from ghost cells, so the
 * same-level ghost fills around every colour pass are skipped; one fill
 * after the last sweep leaves the ghost cells as the reference leaves them.
 * Results are bit-identical to 0 (fills as in CellPoissonFACOps.C:
 * 1392-1495).  Used on a level only when its colouring is consistent across
 * patches (always in 3-D). */
int fac_set_fused(fac_ctx *ctx, int on);

/* 1 (default): on levels where the fused pass is used, sweeps with a fixed
 * count (every sweep except the coarsest-level solve to a tolerance) run on
 * shared-memory staged units: TMA bulk copies bring a run of slices of one
 * patch into shared memory, the colour pass runs there and the new values
 * go back to HBM.  The composite residuals inside the solves run staged the
 * same way (fluxes and residual from the staged slices, then the cells on
 * coarse-fine faces and next to finer-level faces redone by a fix-up pass).
 * Results are bit-identical to 0. */
int fac_set_staged(fac_ctx *ctx, int on);

/* 1: the composite residual forms the face fluxes while it sums
 * them (computeFluxOnPatch and the residual loop of
 * CellPoissonFACOps.C:1792-1956 in one kernel), taking the coarsened finer
 * fluxes where the flux coarsening stored them.  Bit-identical to 0.
 * fac_comp_residual itself always stores the face fluxes (fac_download_flux);
 * the setting applies to the residuals inside fac_solve / fac_fac_cycle.
 * on = 1: every level, 0: none, -1 (the default): the levels whose patches
 * average at least 8192 cells, where on B200 the one pass is faster (on
 * levels of 8^3..16^3 patches the two kernels are). */
int fac_set_fused_residual(fac_ctx *ctx, int on);

/* Shared-memory bytes of one stage (one work unit) of the staged pass,
 * 4096 .. 116,160 (default 32,768): patches are cut into units of as many
 * slices as fit.  Rebuilds the unit tables when the context is
 * initialised; a level whose largest unit does not fit depth stages in
 * 227 KiB of shared memory runs the unstaged pass.  fac_autotune picks it
 * by timing. */
int fac_set_stage_budget(fac_ctx *ctx, int bytes);
/* Stages a CTA of the staged pass cycles through, 2 .. 4 (default 2): more
 * stages keep more copies in flight per CTA, fewer leave room for more
 * CTAs per SM.  Rebuilds the unit tables like fac_set_stage_budget. */
int fac_set_stage_depth(fac_ctx *ctx, int depth);

/* Autotuner: times one red-black sweep of every smoothed level for stage
 * sizes of 12, 16, 24, 32 and 48 KiB at depths 2 and 3 (best of three, CUDA
 * events) and keeps the fastest; ms_per_candidate (10 entries, depth 2
 * then depth 3, sizes ascending) and the chosen outputs may be NULL.  Uses
 * the smoothing fields as scratch: call it before fac_solve. */
int fac_autotune(fac_ctx *ctx, int *chosen_bytes, int *chosen_depth, double *ms_per_candidate);

/* FGMRES(restart) with one FAC cycle (FP32 in the mixed precision) as the
 * flexible right preconditioner, every problem with its own Krylov space.
 * Inner products are the weighted sums of fac_rms_norm, the stopping rule
 * that of fac_solve (weighted RMS composite residual <= max(residual_tol,
 * relative_residual_tol * ||f||)); max_cycles bounds the preconditioner
 * applications, which iterations reports.  Same outputs as fac_solve.
 * Holds 2*restart+1 composite vectors per context.  No counterpart in the
 * reference (FACPreconditioner is the stationary iteration). */
int fac_solve_fgmres(fac_ctx *ctx, int restart, int *converged, int *iterations,
                     double *residual);
/* restart > 0: fac_solve and fac_solve_host run fac_solve_fgmres(restart);
 * 0 (default): the reference's stationary FAC iteration. */
int fac_set_krylov(fac_ctx *ctx, int restart);

/* 1 (default): fac_solve captures one FAC cycle (V-cycle, correction,
 * restriction, composite residual, norm kernels) into a CUDA graph on first
 * use and replays it every cycle; converged problems are skipped on the
 * device, and one host synchronisation per cycle reads the norms.  0: the
 * same launches issued one by one.  Profiling and tracing use the latter. */
int fac_set_graph(fac_ctx *ctx, int on);

/* Precision of the FAC cycle (call before fac_initialize).  0: all FP64, the
 * reference's arithmetic.  1: mixed -- red-black smoothing, prolongation
 * and the error vector in FP32; composite residual with its coarse-fine
 * flux sums, residual restriction, coarsest-level solve and the outer
 * defect-correction loop in FP64.  No reference counterpart (the reference
 * is FP64 throughout). */
int fac_set_precision(fac_ctx *ctx, int mixed);

/* Build device tables and allocate device state
 * (CellPoissonFACOps::initializeOperatorState, CellPoissonFACOps.C:751-1106). */
int fac_initialize(fac_ctx *ctx);

/* Sizes (doubles) of one level of one problem in the host layout. */
int fac_field_size(fac_ctx *ctx, int fid, int problem, int ln, size_t *n);
int fac_side_size(fac_ctx *ctx, int problem, int ln, size_t *n);
int fac_oside_size(fac_ctx *ctx, int problem, int ln, size_t *n);

/* Host <-> device copies of one level of one problem (host layout above).
 * Synchronous with respect to the context's stream. */
int fac_upload_field(fac_ctx *ctx, int fid, int problem, int ln,
                     const double *host);
int fac_download_field(fac_ctx *ctx, int fid, int problem, int ln,
                       double *host);
int fac_upload_side(fac_ctx *ctx, int problem, int ln, const double *host);
int fac_download_side(fac_ctx *ctx, int problem, int ln, double *host);
/* Flux scratch (side layout) as left by the last fac_comp_residual on ln:
 * D grad u with the Ewing fix and the coarsened finer-level flux. */
int fac_download_flux(fac_ctx *ctx, int problem, int ln, double *host);
/* Saved outer-side flux of a refined level (CellPoissonFACOps.C:1933-1948):
 * per patch, axis, lower then upper side. */
int fac_download_oside(fac_ctx *ctx, int problem, int ln, double *host);

/* ---- level operators (FACOperatorStrategy, FACOperatorStrategy.h:83-364) */

/* xeqScheduleGhostFill (with_coarse=1) / xeqScheduleGhostFillNoCoarse
 * (CellPoissonFACOps.C:2861-2900). */
int fac_ghost_fill(fac_ctx *ctx, int fid, int ln, int with_coarse,
                   int homogeneous);
/* The copies a ghost fill of level ln makes (the transactions of the
 * reference's RefineSchedule, RefineSchedule.C:4821-4866, element by
 * element), for splitting a hierarchy over ranks as tbox::Schedule splits
 * transactions into local, send and receive sets (tbox/Schedule.C:98-175):
 * element q copies into dst[q] (an index of the level's ghost-1 cell array)
 * from src[q] >= 0 (the same level) or, with_coarse, from -src[q]-1 of the
 * next coarser level's ghost-1 array (constant refine).  Physical-boundary
 * ghost cells are not in the table (each patch fills its own).  cap = 0
 * returns the count in *n only.  Works on host-only contexts. */
int fac_fill_table(fac_ctx *ctx, int ln, int with_coarse, long long *dst,
                   long long *src, size_t cap, size_t *n);
/* smoothErrorByRedBlack (CellPoissonFACOps.C:1339-1514): nsweeps red-black
 * Gauss-Seidel sweeps of field fid_e against right-hand side fid_r; tol < 0
 * disables the convergence test.  sweeps (optional, one int per problem)
 * receives the sweeps taken. */
int fac_smooth(fac_ctx *ctx, int fid_e, int fid_r, int ln, int nsweeps,
               double tol, int *sweeps);
/* computeCompositeResidualOnLevel (CellPoissonFACOps.C:1792-1956). */
int fac_comp_residual(fac_ctx *ctx, int fid_r, int fid_u, int fid_f, int ln,
                      int error_equation);
/* restrictResidual / restrictSolution without the ghost fill
 * (CellPoissonFACOps.C:1197-1242): volume-weighted average of level
 * dest_ln+1 into level dest_ln. */
int fac_restrict(fac_ctx *ctx, int fid_src, int fid_dst, int dest_ln);
/* restrictSolution (CellPoissonFACOps.C:1197-1220). */
int fac_restrict_solution(fac_ctx *ctx, int fid, int dest_ln);
/* prolongErrorAndCorrect (CellPoissonFACOps.C:1254-1304). */
int fac_prolong_correct(fac_ctx *ctx, int fid_src, int fid_dst, int dest_ln);
/* computeVectorWeights (CellPoissonFACOps.C:2005-2102) into FAC_W. */
int fac_compute_weights(fac_ctx *ctx);
/* SAMRAIVectorReal::RMSNorm (SAMRAIVectorReal.C:821-840) over all levels;
 * norms: one double per problem. */
int fac_rms_norm(fac_ctx *ctx, int fid, double *norms);
/* solveCoarsestLevel (CellPoissonFACOps.C:1681-1730). */
int fac_solve_coarsest(fac_ctx *ctx, int *sweeps);
/* One FACPreconditioner::facCycle_Recursive V-cycle (FACPreconditioner.C:
 * 462-518) on e = FAC_E, r = FAC_R. */
int fac_fac_cycle(fac_ctx *ctx);

/* ---- solver (CellPoissonFACSolver::solveSystem, CellPoissonFACSolver.C:
 *      310-352, over FACPreconditioner::solveSystem FACPreconditioner.C:
 *      277-452).  u (FAC_U) and f (FAC_F) must be resident.
 * converged, iterations, residual: one entry per problem (may be NULL). */
int fac_solve(fac_ctx *ctx, int *converged, int *iterations,
              double *residual);

/* Solve from host memory: uploads f (and u0, when not NULL) for every
 * problem and level, solves, and downloads u.  Array k of f_host/u_host
 * holds level (k % nlev) of problem (k / nlev) in the host layout (nlev:
 * the caller's levels, without those of fac_set_coarse_extension). */
int fac_solve_host(fac_ctx *ctx, const double *const *f_host,
                   const double *const *u0_host, double *const *u_host,
                   int *converged, int *iterations, double *residual);

/* Set a cell field to zero on every level of every problem (ghosts
 * included), e.g. u before a solve from a zero initial guess. */
int fac_zero_field(fac_ctx *ctx, int fid);

/* Per-cycle residual norms of the last fac_solve for one problem:
 * hist[0] = before the first cycle, hist[k] after cycle k; *n entries. */
int fac_residual_history(fac_ctx *ctx, int problem, double *hist, int cap,
                         int *n);

/* Red-black sweeps taken by coarsest-level solves since the last reset,
 * per problem (long long each). */
int fac_coarse_sweeps(fac_ctx *ctx, long long *sweeps);
int fac_reset_stats(fac_ctx *ctx);

/* Synchronise the context's stream. */
int fac_synchronize(fac_ctx *ctx);

/* ---- instrumentation (the reference's tbox::Timer around each FAC op,
 *      CellPoissonFACOps.C:626-639, as CUDA events on the context stream). */

/* Per-operation wall-clock totals with a stream synchronisation around each
 * operation (tbox::Timer::barrierAndStart semantics); fac_trace_read writes
 * a JSON object {"op@Lln": [calls, ms], ...}. */
int fac_trace_enable(fac_ctx *ctx, int on);
int fac_trace_read(fac_ctx *ctx, char *buf, int cap, int *len);
/* Kernels launched by this process so far, over all contexts. */
int fac_kernel_launches(long long *n);
/* Record CUDA events around every red-black colour pass (kind 0 FP64,
 * kind 2 FP32), ghost fill (kind 1 FP64, kind 3 FP32) and FGMRES vector
 * operation (kind 4 multi-dot, kind 5 linear combination; per level) from
 * now on; clears earlier records.  Bytes count only problems still
 * iterating. */
int fac_profile_enable(fac_ctx *ctx, int on);
/* Totals over the records of one kind: launches, device milliseconds and
 * algorithmic bytes (colour pass: 8*(ghosted cells + cells) + 8*dim*cells
 * when D is variable; ghost fill: 16 bytes per ghost cell written; vector
 * operations on K vectors: 8*(K+2) bytes per cell). */
int fac_profile_read(fac_ctx *ctx, int kind, long long *launches, double *ms,
                     double *bytes);
int fac_profile_reset(fac_ctx *ctx);
/* Device timer on the context stream: stop = 0 records the start event;
 * stop = 1 records the end event, waits for it and returns milliseconds. */
int fac_timer(fac_ctx *ctx, int stop, double *ms);

/* ---- learned coarse-correction network.  No counterpart in the reference.
 *
 * Four 3x3x3 convolutions 1 -> 16 -> 16 -> 16 -> 1 channels, ReLU after the
 * first three, no biases, zero padding; BF16 weights and activations, FP32
 * accumulation (16 -> 16 layers on the tensor cores).  A sample is a patch
 * plus a one-cell halo, zero-padded to FAC_CNN_BOX^3 cells, i fastest.
 * Weights (FP32 masters, host arrays): w1 [27][16] (tap, out), w2, w3
 * [27][16][16] (tap, in, out), w4 [27][16] (tap, in); tap = (dz+1)*9 +
 * (dy+1)*3 + (dx+1).  x, y, target and mask are FP32 device arrays of
 * nsamp*FAC_CNN_BOX^3 values. */
#define FAC_CNN_BOX 18
typedef struct fac_cnn fac_cnn;
const char *fac_cnn_last_error(void);
int fac_cnn_create(fac_cnn **net, int device, int max_batch, unsigned long long seed);
int fac_cnn_destroy(fac_cnn *net);
int fac_cnn_set_weights(fac_cnn *net, const float *w1, const float *w2,
                        const float *w3, const float *w4);
int fac_cnn_get_weights(fac_cnn *net, float *w1, float *w2, float *w3,
                        float *w4);
int fac_cnn_forward(fac_cnn *net, const float *x, long long nsamp, float *y);
/* Masked mean squared error of the prediction and its weight gradients
 * (host arrays; any may be NULL). */
int fac_cnn_gradients(fac_cnn *net, const float *x, const float *target,
                      const float *mask, long long nsamp, double *loss,
                      float *g1, float *g2, float *g3, float *g4);
/* One Adam step (beta 0.9/0.999) on the masked MSE; mask_sum = sum(mask). */
int fac_cnn_train_step(fac_cnn *net, const float *x, const float *target,
                       const float *mask, long long nsamp, double mask_sum,
                       float lr, double *loss);

/* Learned correction inside fac_solve (NULL disables it).  After every
 * cycle the network predicts, from the composite residual on each patch of
 * `level` (patch plus one-cell halo, scaled by the patch's RMS residual),
 * the error on that patch (times the patch RMS residual and dx^2).  The
 * prediction e is applied as u += alpha e with the per-problem
 * minimal-residual step alpha = <r, A e> / <A e, A e> (weighted by the
 * control volumes), and alpha = 0 whenever it would not lower the residual,
 * so the FAC residual never grows.  Under FGMRES (fac_set_krylov > 0) the
 * network is instead the second stage of the preconditioner: for the
 * residual s = v - A z that the FAC cycle's correction z leaves, its
 * prediction e of the error goes into z += alpha e with the same
 * minimal-residual alpha for s.  Patches of `level` must have at most
 * FAC_CNN_BOX-2 cells per side and the network a batch of at least the
 * level's patch count. */
int fac_set_learned(fac_ctx *ctx, fac_cnn *net, int level);
/* The network's inputs for the current residual FAC_R of `level`: one
 * FAC_CNN_BOX^3 FP32 sample per patch into the device array x, and the
 * patch scales (RMS of r) into the host array scale (may be NULL).  Uses
 * FAC_E of that level as scratch. */
int fac_learned_samples(fac_ctx *ctx, int level, float *x, double *scale);

/* ---- other centerings: time interpolation and index boxes (no part of the
 *      FAC path; the reference's RefineSchedule applies them to any patch
 *      data: xfer/RefineSchedule.C:2037 fillData with time interpolation,
 *      pdat/CellDoubleLinearTimeInterpolateOp.C:86 and its side, face, node
 *      and edge twins over pdat_m4lintimeintops{2,3}d.i). */
enum fac_centering {
   FAC_CELL = 0,
   FAC_SIDE = 1,   /* SideGeometry::toSideBox: upper+1 along the axis */
   FAC_FACE = 2,   /* FaceGeometry::toFaceBox: axis first, upper+1 along it */
   FAC_NODE = 3,   /* NodeGeometry::toNodeBox: upper+1 along every axis */
   FAC_EDGE = 4    /* EdgeGeometry::toEdgeBox: upper+1 along the other axes */
};
/* The index box of centering (and axis, for side, face and edge data) of the
 * cell box lo..hi, in the storage order of that data. */
int fac_centered_box(int dim, int centering, int axis, const int *lo, const int *hi,
                     int *out_lo, int *out_hi);
/* One box of a time interpolation: device arrays (one component, column-
 * major over their boxes, first index fastest), each box in the data's own
 * index space (fac_centered_box), where inside all three. */
typedef struct fac_time_box {
   const double *old_data;
   const double *new_data;
   double *dst_data;
   int where_lo[3], where_hi[3];
   int old_lo[3], old_hi[3];
   int new_lo[3], new_hi[3];
   int dst_lo[3], dst_hi[3];
} fac_time_box;
/* dst = old (1 - t) + new t over every box, t = (dst_time - old_time) /
 * (new_time - old_time) (0 when the times coincide), the arithmetic of the
 * reference's LinearTimeInterpolateOps; queued on stream (a cudaStream_t,
 * NULL: legacy default), nothing allocated.  A where box outside an array's
 * box returns FAC_ERR_ARG before anything runs. */
int fac_time_interpolate(int dim, const fac_time_box *boxes, int nboxes,
                         double old_time, double new_time, double dst_time,
                         void *stream);

/* ---- bounded device waits (no counterpart in the reference).
 * The staged colour pass's consumer warps wait for each unit's copies at
 * most limit_cycles SM clock cycles (default 4e9, about 2 s) and then set
 * the context's device error flag, which the next norm or solve reports as
 * FAC_ERR_CUDA; every copy a block issued lands before the block exits, so
 * the context stays usable.  never = 1 makes that wait be for a phase no
 * copy completes: a test of the bound that ends with the error.
 * fac_clear_device_error resets the flag. */
int fac_set_wait_test(fac_ctx *ctx, long long limit_cycles, int never);
int fac_clear_device_error(fac_ctx *ctx);

/* ---- composite-vector operations (solv/SAMRAIVectorReal.C: dot :889,
 *      RMSNorm :821, L2Norm, maxNorm, linearSum), for Krylov and nonlinear
 *      solvers that call FAC as a preconditioner
 *      (source/test/nonlinear/ModifiedBratuProblem.C:2283-2352).
 * A vector is one cell field over every level of a problem; the inner
 * products carry the control-volume weights FAC_W (zero under finer
 * levels), as SAMRAIVectorReal's do when made with those weights.  Interior
 * cells only; one result per problem, every problem of the context. */
/* dots[p] = sum w x y */
int fac_vec_dot(fac_ctx *ctx, int fid_x, int fid_y, double *dots);
/* norms[p] = sqrt(sum w x^2) */
int fac_vec_l2_norm(fac_ctx *ctx, int fid, double *norms);
/* norms[p] = max |x| over cells with w > 0 */
int fac_vec_max_norm(fac_ctx *ctx, int fid, double *norms);
/* z = a[p] x + b[p] y (host arrays a, b of one scalar per problem; z may be
 * x or y).  RMS norm: fac_rms_norm. */
int fac_vec_linear_sum(fac_ctx *ctx, int fid_z, const double *a, int fid_x,
                       const double *b, int fid_y);

/* ---- regrid step: tagging and Berger-Rigoutsos clustering (the step
 *      before FAC in an adaptive run: mesh/GriddingAlgorithm.C's tagging
 *      and box generation).
 * fac_tag_gradient tags the cells of level ln of every problem where the
 * adaption estimate of the ghosted FP64 field fid (FAC_U or FAC_E) exceeds
 * threshold: the estimate of source/test/FAC_adaptive/AdaptivePoisson.C:
 * 622-720 (largest |u(+) + u(-) - 2u| along the axes, half of it along the
 * face diagonals; ghost cells read as they are, so fill them first) and
 * its threshold test (applyGradientDetector, :517-527).  ntagged (host,
 * one per problem, may be NULL) gets the counts.  The tags stay on the
 * device (fac_download_tags: one byte per cell, ghost-0 layout). */
int fac_tag_gradient(fac_ctx *ctx, int fid, int ln, double threshold, long long *ntagged);
int fac_download_tags(fac_ctx *ctx, int problem, int ln, unsigned char *host);
/* Boxes covering the tags of level ln of one problem inside each of the
 * nbound bound boxes (lo0 lo1 lo2 hi0 hi1 hi2 in the level's index space),
 * as mesh::BergerRigoutsos::findBoxesContainingTags
 * (mesh/BergerRigoutsos.C:251-420, BergerRigoutsosNode.C) forms them on one
 * process: tag histograms per node (on the device, one launch per tree
 * depth), the tags' bounding box, acceptance when the tagged fraction
 * reaches efficiency (efficiency_tolerance) or no direction can be cut
 * without a side below min_box, else a cut at the zero swath nearest the
 * middle or at the strongest inflection of the histogram, and recombination
 * of two accepted children whose cells are at least combine (combine_
 * efficiency) of their parent's.  max_box (0 per axis: none) is
 * max_box_size; the other input keys at the reference's defaults.  The
 * product of two histogram Laplacians is formed in 64 bits (the reference
 * uses int, which overflows only for planes of more than ~11,600 tags).
 * Up to cap boxes go to boxes (6 ints each) in depth-first order; nboxes
 * gets their number. */
int fac_cluster_tags(fac_ctx *ctx, int problem, int ln, int nbound, const int *bound,
                     const int *min_box, const int *max_box, double efficiency,
                     double combine, int cap, int *boxes, int *nboxes);
/* fac_cluster_tags for every problem of the context at once: problem p
 * clusters inside its nbound[p] (>= 1) bound boxes, which follow problem
 * p - 1's in bound.  The problems' trees are walked together, one histogram
 * launch per depth for all of them, with the same decisions and boxes as
 * fac_cluster_tags problem by problem.  The boxes go to boxes problem after
 * problem (up to cap in all); counts[p] (host, one per problem) gets
 * problem p's number, whether written or not. */
int fac_cluster_tags_all(fac_ctx *ctx, int ln, const int *nbound, const int *bound,
                         const int *min_box, const int *max_box, double efficiency,
                         double combine, int cap, int *boxes, int *counts);

/* ---- allocation-free norm.  No counterpart in the reference.
 *
 * For callers that cannot allocate device memory when they need a norm:
 * codes that hand all device memory to a pool allocator up front (as
 * SAMRAI does with Umpire pools), so a cudaMalloc would fail or take memory
 * the pool was promised, and codes whose time step may not call cudaMalloc
 * because it synchronises the device and stalls their other streams.
 *
 * Weighted RMS norm per segment: norms[s] = sqrt(sum w x^2) / sqrt(sum w)
 * over elements seg_offsets[s] .. seg_offsets[s+1]-1 of the device arrays
 * x and w (the reduction of fac_rms_norm).  x, w and norms are device
 * pointers owned by the caller; seg_offsets is a host array of nseg+1
 * ascending offsets; stream is a cudaStream_t (NULL: legacy default
 * stream) and the call returns without waiting for the result.
 *
 * Partial sums live in a static device array of FAC_NOALLOC_MAX_SEGMENTS x
 * 64 double2 (256 KiB) that every GPU loading this library holds until the
 * process exits; nothing is allocated or freed per call.  nseg above
 * FAC_NOALLOC_MAX_SEGMENTS returns FAC_ERR_ARG.  The first call on each
 * device looks up that device's address of the array (cudaGetSymbolAddress,
 * with the device current).
 * All calls share the array: calls whose work can overlap on the GPU (two
 * streams, or two host threads) race and must be serialised by the caller.
 * Every partial sum a call reads it first writes, so no clearing is needed.
 * The looked-up address is kept for the life of the process: do not use
 * this entry point on a device after cudaDeviceReset.  An error already
 * pending on the calling thread when the call starts (left by earlier,
 * unrelated work) is reported as FAC_ERR_CUDA and left in place for its
 * owner; the call then launches nothing.  An empty segment's norm is 0.
 * Each segment is reduced by 64 blocks, so a call with few large segments
 * runs below memory bandwidth. */
#define FAC_NOALLOC_MAX_SEGMENTS 256
int fac_rms_norm_noalloc(const double *x, const double *w,
                         const long long *seg_offsets, int nseg, double *norms,
                         void *stream);

#ifdef __cplusplus
}
#endif
#endif

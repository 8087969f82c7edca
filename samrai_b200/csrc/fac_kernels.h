// Launchers of the FP64 FAC kernels (fac_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "fac_internal.h"

namespace samrai_b200 {

// Kernels launched by this process so far (all contexts).
long long kernel_launch_count();
// Adjust the count: kernels of other files, kernels captured into a CUDA
// graph (removed at capture, added per replay).
void add_kernel_launches(long long n);

// Staged colour pass (fac_stage.cu): units {patch, first copy, copies,
// header} of the compacted list (active problems only) with their copy
// lists and headers; stage_bytes is the largest StagePlan::bytes of the
// units and depth (2 .. kStageDepthMax) the stages a CTA cycles through;
// pushmap gives per face cell where its new value goes (>= 0 a
// neighbour's ghost cell, -1 physical boundary, -2 coarse-fine face); err is
// set to 1 when a bounded wait runs out.  The field's face ghost cells must
// be filled before the first pass.
template <class T>
void launch_rb_staged(cudaStream_t s, int dim, const PoissonSpec &spec, int nunits,
                      int stage_bytes, int depth, const Chunk *units, const UnitCopy *copies,
                      const unsigned char *headers, T *u, const T *f, const T *dside,
                      const T *cfield, const T *cfflux, int offset, const int *pushmap,
                      const BcCoefs &bc, int *err, const WaitTest &wt = WaitTest());

// Staged composite residual over a level's residual units (fac_stage.cu):
// res = f - div flux - C u on every cell of the units, outer-side fluxes of
// the patch faces when oflux is not null; u FP64 or FP32, the rest FP64.
template <class TU>
void launch_res_staged(cudaStream_t s, int dim, const PoissonSpec &spec, int nunits,
                       int stage_bytes, int depth, const Chunk *units, const UnitCopy *copies,
                       const unsigned char *headers, const TU *u, const double *f,
                       const double *dside, const double *cfield, double *res, double *oflux,
                       int *err, const WaitTest &wt = WaitTest());
// The residual (and outer-side fluxes) of listed cells as the one-pass
// kernel forms them, Ewing fix and coarsened finer fluxes included: the
// fix-up after the staged residual.
template <class TU>
void launch_residual_cells(cudaStream_t s, int dim, const PoissonSpec &spec, int ncells,
                           const CellRef *cells, const PatchDesc *patches, const TU *u,
                           const double *dside, const unsigned char *cfmask,
                           const double *tranwt, const double *longwt,
                           const int *ratio_to_coarser, const unsigned char *fcmask,
                           const double *fcflux, const double *f, const double *cfield,
                           double *res, double *oflux, const int *run);

// Regrid step (fac_regrid.cu): tags (ghost-0 bytes) where the adaption
// estimate of u (ghost-1, FP64) exceeds threshold, counts[prob] += tags;
// one problem's tags into a dense array over [lo, lo + n); the tag
// histograms of Berger-Rigoutsos node boxes (each node names its problem's
// dense array).
void launch_adaption_tags(cudaStream_t s, int dim, int nchunks, const PatchDesc *patches,
                          const Chunk *chunks, const double *u, double threshold,
                          unsigned char *tags, unsigned long long *counts, const int *run);
void launch_tags_dense(cudaStream_t s, int dim, int nchunks, const PatchDesc *patches,
                       const Chunk *chunks, const unsigned char *tags, int prob, const int *lo,
                       const int *n, unsigned char *dense);
void launch_br_histogram(cudaStream_t s, int nitems, const BrItem *items, const BrNode *nodes,
                         const unsigned char *dense, int *hist);

// Krylov vector operations on composite vectors: ghost-0 level arrays, one
// vector every vstride elements; per-problem coefficients; chunks are runs
// of one problem's cells {problem, first cell, cells, chunk index} (partial
// is nchunks x K).
// out[p*KT+i] += sum_w x V_i over problem p's chunks of this level, KT = K
// (+1 with self_dot: entry K is <x, x>, the same sum as taking x as V_K).
void launch_multidot(cudaStream_t s, int nchunks, const Chunk *chunks, const double *w,
                     const double *x, const double *V, long long vstride, int K,
                     double *partial, const int *prob_chunk_begin, int nprob, const int *active,
                     double *out, bool self_dot = false);
// x = a[p] xin + sum_i coef[p*K+i] V_i (xin null: x itself), also written
// to x2 when it is not null
void launch_combine(cudaStream_t s, int nchunks, const Chunk *chunks, double *x, const double *a,
                    const double *V, long long vstride, int K, const double *coef,
                    const double *xin = nullptr, double *x2 = nullptr);
// The same (without x2), and out[p] += <x, x> (weighted, the new x) over
// problem p's chunks of this level, equal to launch_multidot(x, x, K = 1).
void launch_combine_norm(cudaStream_t s, int nchunks, const Chunk *chunks, double *x,
                         const double *a, const double *V, long long vstride, int K,
                         const double *coef, const double *w, double *partial,
                         const int *prob_chunk_begin, int nprob, const int *active, double *out,
                         const double *xin = nullptr);
// Largest K of launch_combine_dots.
constexpr int kCombineDotsMax = 24;
// x = a[p] xin + sum_i coef[p*K+i] V_i as launch_combine, and out[p*(K+1)+i]
// += <x, V_i> for i < K, out[p*(K+1)+K] += <x, x> (weighted, the new x) over
// problem p's chunks of this level: the numbers of launch_multidot(x, V, K,
// self_dot) after the combination, from the same pass.  Returns false
// (nothing launched) unless 1 <= K <= kCombineDotsMax.
bool launch_combine_dots(cudaStream_t s, int nchunks, const Chunk *chunks, double *x,
                         const double *a, const double *V, long long vstride, int K,
                         const double *coef, const double *w, double *partial,
                         const int *prob_chunk_begin, int nprob, const int *active, double *out,
                         const double *xin = nullptr);
// dst (ghost-0) = interior of src (ghost-1), converted to FP64, times
// scale[problem] when scale is given (with add: dst += it); with dst1 (a
// ghost-1 FP64 field, not src) the same values also go to its interior
template <class TS>
void launch_g1_to_g0(cudaStream_t s, int dim, int nchunks, const PatchDesc *patches,
                     const Chunk *chunks, const TS *src, double *dst, bool add = false,
                     const double *scale = nullptr, double *dst1 = nullptr);
// u interior += sum_i y[p*K+i] Z_i
void launch_add_combination(cudaStream_t s, int dim, int nchunks, const PatchDesc *patches,
                            const Chunk *chunks, double *u, const double *Z, long long zstride,
                            int K, const double *y);

// Rebuild every registered work list for the current active flags.
void launch_compact(cudaStream_t s, const WorkReg *regs, int nregs, const int *active, int nprob);

template <class T>
void launch_fill(cudaStream_t s, const FillItem *items, const Chunk *chunks, int nchunks,
                 const int *prefix, T *dst, const T *src_same, const T *src_coarse, int homogeneous,
                 const BcCoefs &bc, const int *active);
// Red-black smoothing to a tolerance, all sweeps in one launch, of a level
// without a coarser level and with one patch per problem (patch b of
// problem patches[b].prob); run, sweeps and the per-patch red / black
// residual maxima as the per-pass launches and the sweep check leave them.
// smem > 0: every patch's arrays fit that many bytes of shared memory and
// the face table has no same-level neighbour; the sweeps run on shared
// copies (same bits).
// Let the shared-memory form of the one-launch solve (FP64) take up to
// `bytes` of dynamic shared memory on the current device; false if refused.
bool allow_solve_smem(int bytes);
template <class T>
void launch_rbgs_solve(cudaStream_t s, int dim, const PoissonSpec &spec, int npatch,
                       const PatchDesc *patches, T *u, const T *f, const T *dside,
                       const T *cfield, const long long *facemap, const BcCoefs &bc,
                       int nsweeps, double tol, int *run, long long *sweeps,
                       unsigned long long *maxres_red, unsigned long long *maxres_blk,
                       int smem = 0);
// Ghost fill from a gather list of n elements (copies and constant refines,
// see k_fill_gather) plus the physical-boundary items of the same fill.
template <class T>
void launch_fill_gather(cudaStream_t s, long long n, const unsigned *to, const int *from,
                        const unsigned short *prob, const FillItem *bc_items,
                        const Chunk *bc_chunks, int nbc, const int *bc_prefix, T *dst,
                        const T *src_same, const T *src_coarse, int homogeneous,
                        const BcCoefs &bc, const int *active);

template <class T>
void launch_cf_flux(cudaStream_t s, const CfFace *faces, int nfaces, const PatchDesc *patches,
                    const T *u, const T *dside, int dvar, double dconst, const double *tranwt,
                    const double *longwt, T *cfflux, const int *run);

// facemap != NULL: fused colour pass (no ghost cells read, see fac_kernels.cu)
template <class T>
void launch_rbgs(cudaStream_t s, int dim, const PoissonSpec &spec, int nchunks,
                 const PatchDesc *patches, const Chunk *chunks, T *u, const T *f,
                 const T *dside, const T *cfield, const T *cfflux,
                 const unsigned char *cfmask, int offset, unsigned long long *maxres,
                 const int *run, const long long *facemap, const BcCoefs &bc);

// Fluxes and residual are always FP64; the unknown may be FP32 (mixed).
template <class TU>
void launch_flux(cudaStream_t s, int dim, const PoissonSpec &spec, int nchunks,
                 const PatchDesc *patches, const Chunk *chunks, const TU *u,
                 const double *dside, const unsigned char *cfmask, const double *tranwt,
                 const double *longwt, const int *ratio_dev, double *flux, const int *run);

template <class TU>
void launch_residual(cudaStream_t s, int dim, const PoissonSpec &spec, int nchunks,
                     const PatchDesc *patches, const Chunk *chunks, const TU *u,
                     const double *f, const double *flux, const double *cfield,
                     double *res, double *oflux, const int *run);

// Ewing fix of the stored fluxes on the level's coarse-fine faces.
template <class TU>
void launch_ewing_fix(cudaStream_t s, const CfFace *faces, int nfaces, const PatchDesc *patches,
                      const TU *u, const double *dside, int dvar, double dconst,
                      const double *tranwt, const double *longwt, double *flux, const int *run);

// All face fluxes of a level from its cell chunks (one decode per cell);
// the coarse-fine faces need launch_ewing_fix afterwards.
template <class TU>
void launch_flux_cells(cudaStream_t s, int dim, const PoissonSpec &spec, int nchunks,
                       const PatchDesc *patches, const Chunk *cell_chunks, const TU *u,
                       const double *dside, const unsigned char *cfmask, const double *tranwt,
                       const double *longwt, const int *ratio_dev, double *flux, const int *run);

// Fluxes on the fly + residual (+ outer-side fluxes): k_flux and k_residual
// in one pass; fcmask marks faces whose flux is the coarsened finer-level
// flux already stored in fcflux (NULL when the level has no finer level).
template <class TU>
void launch_residual_fused(cudaStream_t s, int dim, const PoissonSpec &spec, int nchunks,
                           const PatchDesc *patches, const Chunk *chunks, const TU *u,
                           const double *dside, const unsigned char *cfmask,
                           const double *tranwt, const double *longwt, const int *ratio_dev,
                           const unsigned char *fcmask, const double *fcflux, const double *f,
                           const double *cfield, double *res, double *oflux, const int *run);

// Transaction-list launchers take the list's item prefix sums (packed
// chunks, see Chunk).
void launch_flux_coarsen(cudaStream_t s, const FluxCoarsenItem *items, const Chunk *chunks,
                         int nchunks, const int *prefix, const PatchDesc *fine,
                         const PatchDesc *coarse, const double *oflux_fine, double *flux_coarse,
                         const int *run);

void launch_restrict(cudaStream_t s, int dim, const RestrictItem *items, const Chunk *chunks,
                     int nchunks, const int *prefix, const PatchDesc *fine,
                     const PatchDesc *coarse, const double *src, int src_g, double *dst,
                     int dst_g, const int *run);

template <class T>
void launch_prolong_add(cudaStream_t s, int dim, const ProlongItem *items, const Chunk *chunks,
                        int nchunks, const int *prefix, const PatchDesc *fine, const T *tmp,
                        const double *dxc_prob, const int *ratio, T *e, const int *run);
// the same for ratio 2 on every axis, over the coarse cells of the fine
// patches (items counted in coarse cells): same bits, one load of each
// interpolation value per coarse cell
template <class T>
void launch_prolong_add_r2(cudaStream_t s, int dim, const ProlongItem *items,
                           const Chunk *chunks, int nchunks, const int *prefix,
                           const PatchDesc *fine, const T *tmp, const double *dxc_prob, T *e,
                           const int *run);

template <class T>
void launch_add_interior(cudaStream_t s, int dim, int nchunks, const PatchDesc *patches,
                         const Chunk *chunks, double *u, const T *e, const int *run);

template <class S, class D>
void launch_convert(cudaStream_t s, const S *src, D *dst, long long n);

void launch_norm(cudaStream_t s, int dim, int nchunks, const PatchDesc *patches,
                 const Chunk *chunks, const double *x, int xg, const double *w,
                 double2 *partial, const int *prob_chunk_begin, int nprob, double2 *acc);

// Composite-vector reductions over interior cells, per problem added into
// acc: mode 0 acc += (sum w x y, sum w); mode 1 acc.x = max(acc.x, max |x|
// where w > 0).
void launch_vec_reduce(cudaStream_t s, int dim, int mode, int nchunks, const PatchDesc *patches,
                       const Chunk *chunks, const double *x, int xg, const double *y, int yg,
                       const double *w, double2 *partial, const int *prob_chunk_begin,
                       int nprob, double2 *acc);
// z = a[prob] x + b[prob] y on interior cells
void launch_vec_lincomb(cudaStream_t s, int dim, int nchunks, const PatchDesc *patches,
                        const Chunk *chunks, double *z, int zg, const double *x, int xg,
                        const double *y, int yg, const double *a, const double *b);

void launch_sweep_check(cudaStream_t s, const unsigned long long *red,
                        const unsigned long long *blk, const int *last_patch, int nprob,
                        double tol, int *run, long long *sweeps);

void launch_accumulate(cudaStream_t s, const long long *src, long long *dst, int n);

// learned correction
void launch_g0_to_g1(cudaStream_t s, int dim, int nchunks, const PatchDesc *patches,
                     const Chunk *chunks, const double *src, double *dst);
void launch_patch_rms(cudaStream_t s, int dim, int npatch, const PatchDesc *patches,
                      const double *x, double *rms);
void launch_gather_samples(cudaStream_t s, int dim, int npatch, const PatchDesc *patches,
                           const double *x, const double *scale, float *out, int S);
void launch_scatter_samples(cudaStream_t s, int dim, int nchunks, const PatchDesc *patches,
                            const Chunk *chunks, const float *y, const double *scale, int S,
                            double *dst);
void launch_dot_pair(cudaStream_t s, int dim, int nchunks, const PatchDesc *patches,
                     const Chunk *chunks, const double *r, const double *r2, const double *w,
                     double2 *partial, const int *prob_chunk_begin, int nprob, double2 *acc);
void launch_alpha(cudaStream_t s, const double2 *acc, const int *active, int nprob,
                  double *alpha);
void launch_apply_alpha(cudaStream_t s, int dim, int nchunks, const PatchDesc *patches,
                        const Chunk *chunks, const double *alpha, double *u, const double *e,
                        double *r, const double *r2);
void launch_gather(cudaStream_t s, const long long *idx, long long n, const double *src,
                   double *dst);
void launch_scatter(cudaStream_t s, const long long *idx, long long n, const double *src,
                    double *dst);

}  // namespace samrai_b200

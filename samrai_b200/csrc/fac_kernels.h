// Launchers of the FP64 FAC kernels (fac_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "fac_internal.h"

namespace samrai_b200 {

// Kernels launched by this process so far (all contexts).
long long kernel_launch_count();

void launch_fill(cudaStream_t s, const FillItem *items, const Chunk *chunks, int nchunks,
                 double *dst, const double *src_same, const double *src_coarse,
                 int homogeneous, const BcCoefs &bc, const int *active);

void launch_cf_flux(cudaStream_t s, const CfFace *faces, int nfaces, const PatchDesc *patches,
                    const double *u, const double *dside, int dvar, double dconst,
                    const double *tranwt, const double *longwt, double *cfflux,
                    const int *run);

void launch_rbgs(cudaStream_t s, int dim, const PoissonSpec &spec, int nchunks,
                 const PatchDesc *patches, const Chunk *chunks, double *u, const double *f,
                 const double *dside, const double *cfield, const double *cfflux,
                 const unsigned char *cfmask, int offset, unsigned long long *maxres,
                 const int *run);

void launch_flux(cudaStream_t s, int dim, const PoissonSpec &spec, int nchunks,
                 const PatchDesc *patches, const Chunk *chunks, const double *u,
                 const double *dside, const unsigned char *cfmask, const double *tranwt,
                 const double *longwt, const int *ratio_dev, double *flux, const int *run);

void launch_residual(cudaStream_t s, int dim, const PoissonSpec &spec, int nchunks,
                     const PatchDesc *patches, const Chunk *chunks, const double *u,
                     const double *f, const double *flux, const double *cfield,
                     double *res, double *oflux, const int *run);

void launch_flux_coarsen(cudaStream_t s, const FluxCoarsenItem *items, const Chunk *chunks,
                         int nchunks, const PatchDesc *fine, const PatchDesc *coarse,
                         const double *oflux_fine, double *flux_coarse, const int *run);

void launch_restrict(cudaStream_t s, int dim, const RestrictItem *items, const Chunk *chunks,
                     int nchunks, const PatchDesc *fine, const PatchDesc *coarse,
                     const double *src, int src_g, double *dst, int dst_g, const int *run);

void launch_prolong_add(cudaStream_t s, int dim, const ProlongItem *items, const Chunk *chunks,
                        int nchunks, const PatchDesc *fine, const double *tmp,
                        const double *dxc_prob, const int *ratio, double *e, const int *run);

void launch_add_interior(cudaStream_t s, int dim, int nchunks, const PatchDesc *patches,
                         const Chunk *chunks, double *u, const double *e, const int *run);

void launch_norm(cudaStream_t s, int dim, int nchunks, const PatchDesc *patches,
                 const Chunk *chunks, const double *x, int xg, const double *w,
                 double2 *partial, const int *prob_chunk_begin, int nprob, double2 *acc);

void launch_sweep_check(cudaStream_t s, const unsigned long long *red,
                        const unsigned long long *blk, const int *last_patch, int nprob,
                        double tol, int *run, long long *sweeps);

void launch_gather(cudaStream_t s, const long long *idx, long long n, const double *src,
                   double *dst);
void launch_scatter(cudaStream_t s, const long long *idx, long long n, const double *src,
                    double *dst);

}  // namespace samrai_b200

// The regrid step on the device: tagging by the FAC_adaptive adaption
// estimate and the tag histograms (signatures) of Berger-Rigoutsos
// clustering.  The clustering's decisions (bounding box, efficiency,
// zero-swath and inflection cuts, recombination) are host logic over the
// histograms, in fac_host.cu (fac_cluster_tags).
#include <cuda_runtime.h>

#include "fac_device.h"
#include "fac_internal.h"
#include "fac_kernels.h"

namespace samrai_b200 {

namespace {

using namespace dev;

// AdaptivePoisson::computeAdaptionEstimate (source/test/FAC_adaptive/
// AdaptivePoisson.C:622-720) and the threshold test of
// applyGradientDetector (:517-527): the largest |(u(+) + u(-)) - 2 u(0)|
// along the axes and half of it along the face diagonals; tag where it
// exceeds the threshold.  The maxima are taken in the reference's order
// (max is exact, the order only matters for NaN).
template <int DIM>
__global__ void __launch_bounds__(kThreads)
k_adaption_tags(const PatchDesc *__restrict__ patches, const Chunk *__restrict__ chunks,
                int nwork, const double *__restrict__ u, double threshold,
                unsigned char *__restrict__ tags, unsigned long long *__restrict__ counts,
                const int *__restrict__ run)
{
   __shared__ unsigned cnt[kThreads / 32];
   WORK_LOOP(ch) {
      const PatchDesc &p = patches[ch.patch];
      if (run && !run[p.prob]) continue;
      const int nx = p.hi[0] - p.lo[0] + 1;
      const int ny = p.hi[1] - p.lo[1] + 1;
      const int gx = nx + 2, gxy = (nx + 2) * (ny + 2);
      const double *up = u + p.off1;
      unsigned mine = 0;
      for (int t = threadIdx.x; t < ch.count; t += blockDim.x) {
         const int lin = ch.begin + t;
         int li, lj, lk;
         patch_cell(p, lin, nx, ny, li, lj, lk);
         const int c = (li + 1) + gx * (lj + 1) + (DIM == 3 ? gxy * (lk + 1) : 0);
         const double u0 = up[c];
         auto d2 = [&](int o) { return fabs((up[c + o] + up[c - o]) - 2 * u0); };
         double est;
         if (DIM == 2) {
            const double est0 = d2(1);
            const double est1 = d2(gx);
            const double est2 = 0.5 * d2(1 + gx);
            const double est3 = 0.5 * fabs((up[c + 1 - gx] + up[c - 1 + gx]) - 2 * u0);
            est = fmax(fmax(est0, est1), fmax(est2, est3));
         } else {
            const double est0 = d2(1);
            const double est1 = d2(gx);
            const double est2 = d2(gxy);
            const double est3 = 0.5 * d2(gx + gxy);
            const double est4 = 0.5 * fabs((up[c + gx - gxy] + up[c - gx + gxy]) - 2 * u0);
            const double est5 = 0.5 * d2(1 + gxy);
            const double est6 = 0.5 * fabs((up[c + 1 - gxy] + up[c - 1 + gxy]) - 2 * u0);
            const double est7 = 0.5 * d2(1 + gx);
            const double est8 = 0.5 * fabs((up[c + 1 - gx] + up[c - 1 + gx]) - 2 * u0);
            const double esta = fmax(est0, est1), estb = fmax(est2, est3);
            const double estc = fmax(est4, est5), estd = fmax(est6, est7);
            est = fmax(fmax(fmax(esta, estb), fmax(estc, estd)), est8);
         }
         const bool tag = est > threshold;
         tags[p.off0 + lin] = tag ? 1 : 0;
         mine += tag ? 1u : 0u;
      }
      for (int o = 16; o > 0; o >>= 1) mine += __shfl_down_sync(0xffffffffu, mine, o);
      if ((threadIdx.x & 31) == 0) cnt[threadIdx.x >> 5] = mine;
      __syncthreads();
      if (threadIdx.x == 0) {
         unsigned long long s = 0;
         for (int w = 0; w < kThreads / 32; ++w) s += cnt[w];
         if (s) atomicAdd(counts + p.prob, s);
      }
      __syncthreads();
   }
}

// The tags of one problem's patches of a level placed into a dense array
// over the box [lo, lo + n) (x fastest); the array is zeroed before.
template <int DIM>
__global__ void __launch_bounds__(kThreads)
k_tags_dense(const PatchDesc *__restrict__ patches, const Chunk *__restrict__ chunks, int nwork,
             const unsigned char *__restrict__ tags, int prob, int3 lo, int3 n,
             unsigned char *__restrict__ dense)
{
   WORK_LOOP(ch) {
      const PatchDesc &p = patches[ch.patch];
      if (p.prob != prob) continue;
      const int nx = p.hi[0] - p.lo[0] + 1;
      const int ny = p.hi[1] - p.lo[1] + 1;
      for (int t = threadIdx.x; t < ch.count; t += blockDim.x) {
         const int lin = ch.begin + t;
         int li, lj, lk;
         patch_cell(p, lin, nx, ny, li, lj, lk);
         const long long x = p.lo[0] + li - lo.x, y = p.lo[1] + lj - lo.y;
         const long long z = DIM == 3 ? p.lo[2] + lk - lo.z : 0;
         dense[x + (long long)n.x * (y + (long long)n.y * z)] = tags[p.off0 + lin];
      }
   }
}

// Tag histograms of Berger-Rigoutsos nodes (makeLocalTagHistogram,
// mesh/BergerRigoutsosNode.C:1186-1241): per node, the number of tags in
// each index plane normal to each axis.  One block per work item (a run of
// rows of one node box; a row runs along x): a thread keeps the count of
// its x positions over the rows, each row's total goes to the node's y and
// z counts with one atomic.  Integer atomics: the result does not depend
// on the order.
__global__ void __launch_bounds__(kBrThreads)
k_br_histogram(const BrItem *__restrict__ items, const BrNode *__restrict__ nodes,
               const unsigned char *__restrict__ dense_all, int *__restrict__ hist)
{
   __shared__ int wsum[kBrThreads / 32];
   const BrItem it = items[blockIdx.x];
   const BrNode nd = nodes[it.node];
   const unsigned char *dense = dense_all + nd.doff;
   const int3 lo = make_int3(nd.dlo[0], nd.dlo[1], nd.dlo[2]);
   const int3 n = make_int3(nd.dn[0], nd.dn[1], nd.dn[2]);
   const int ex = nd.hi[0] - nd.lo[0] + 1, ey = nd.hi[1] - nd.lo[1] + 1;
   int *hx = hist + nd.hoff, *hy = hx + ex, *hz = hy + ey;
   const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
   // x positions of this thread: threadIdx.x + k kBrThreads, k < kBrMaxXPerThread
   int xc[kBrMaxXPerThread];
#pragma unroll
   for (int k = 0; k < kBrMaxXPerThread; ++k) xc[k] = 0;
   for (int r = it.row0; r < it.row0 + it.nrows; ++r) {
      const int ry = r % ey, rz = r / ey;
      const long long y = nd.lo[1] + ry - lo.y, z = nd.lo[2] + rz - lo.z;
      const unsigned char *row = dense + (nd.lo[0] - lo.x) + (long long)n.x * (y + (long long)n.y * z);
      int rc = 0;
#pragma unroll
      for (int k = 0; k < kBrMaxXPerThread; ++k) {
         const int x = threadIdx.x + k * kBrThreads;
         const int v = x < ex ? row[x] : 0;
         xc[k] += v;
         rc += v;
      }
      for (int o = 16; o > 0; o >>= 1) rc += __shfl_down_sync(0xffffffffu, rc, o);
      if (lane == 0) wsum[wid] = rc;
      __syncthreads();
      if (threadIdx.x == 0) {
         int s = 0;
         for (int w = 0; w < kBrThreads / 32; ++w) s += wsum[w];
         if (s) {
            atomicAdd(hy + ry, s);
            atomicAdd(hz + rz, s);
         }
      }
      __syncthreads();
   }
#pragma unroll
   for (int k = 0; k < kBrMaxXPerThread; ++k) {
      const int x = threadIdx.x + k * kBrThreads;
      if (x < ex && xc[k]) atomicAdd(hx + x, xc[k]);
   }
}

}  // namespace

void launch_adaption_tags(cudaStream_t s, int dim, int nchunks, const PatchDesc *patches,
                          const Chunk *chunks, const double *u, double threshold,
                          unsigned char *tags, unsigned long long *counts, const int *run)
{
   if (nchunks <= 0) return;
   add_kernel_launches(1);
   if (dim == 2)
      k_adaption_tags<2><<<work_grid(k_adaption_tags<2>, nchunks), kThreads, 0, s>>>(
         patches, chunks, nchunks, u, threshold, tags, counts, run);
   else
      k_adaption_tags<3><<<work_grid(k_adaption_tags<3>, nchunks), kThreads, 0, s>>>(
         patches, chunks, nchunks, u, threshold, tags, counts, run);
}

void launch_tags_dense(cudaStream_t s, int dim, int nchunks, const PatchDesc *patches,
                       const Chunk *chunks, const unsigned char *tags, int prob, const int *lo,
                       const int *n, unsigned char *dense)
{
   if (nchunks <= 0) return;
   add_kernel_launches(1);
   const int3 l = make_int3(lo[0], lo[1], lo[2]), e = make_int3(n[0], n[1], n[2]);
   if (dim == 2)
      k_tags_dense<2><<<work_grid(k_tags_dense<2>, nchunks), kThreads, 0, s>>>(
         patches, chunks, nchunks, tags, prob, l, e, dense);
   else
      k_tags_dense<3><<<work_grid(k_tags_dense<3>, nchunks), kThreads, 0, s>>>(
         patches, chunks, nchunks, tags, prob, l, e, dense);
}

void launch_br_histogram(cudaStream_t s, int nitems, const BrItem *items, const BrNode *nodes,
                         const unsigned char *dense, int *hist)
{
   if (nitems <= 0) return;
   add_kernel_launches(1);
   k_br_histogram<<<nitems, kBrThreads, 0, s>>>(items, nodes, dense, hist);
}

}  // namespace samrai_b200

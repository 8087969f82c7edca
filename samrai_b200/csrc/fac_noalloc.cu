// Allocation-free segmented weighted RMS norm.
//
// fac_rms_norm (fac_host.cu) reduces through per-chunk partial sums kept in
// device memory that fac_initialize allocates.  Some callers cannot allocate
// device memory at the point where they need a norm: a code whose device
// memory is all handed to a pool allocator up front (SAMRAI places patch
// data in Umpire pools, tbox/AllocatorDatabase.C:66-110), where a cudaMalloc
// would fail or take memory the pool was promised, or a code whose time step
// may not call cudaMalloc because it synchronises the device and stalls the
// code's other streams.  fac_rms_norm_noalloc computes the same
// norm with its partial sums in a fixed array of static device memory that
// the CUDA module reserves when the library is loaded.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "../../include/samrai_fac_b200.h"

namespace {

constexpr int kMaxSegments = FAC_NOALLOC_MAX_SEGMENTS;
constexpr int kBlocksPerSegment = 64;
constexpr int kThreads = 256;
constexpr int kMaxDevices = 64;

// Partial sums (sum w x^2, sum w) of every (segment, block) pair: 256 x 64
// x 16 bytes = 256 KiB, held by every GPU that loads the library until the
// process exits.  In host code this name is only a stand-in for the device
// symbol: kernels receive the address cudaGetSymbolAddress returns.
static __device__ __align__(256) double2 g_norm_scratch[kMaxSegments * kBlocksPerSegment];

struct SegmentOffsets {
   long long off[kMaxSegments + 1];
};

std::mutex g_setup_mutex;
double2 *g_scratch_ptr[kMaxDevices] = {nullptr};

// Block (b, s) sums segment s with a stride of the segment's blocks and
// writes its own scratch slot; every slot the reduction reads is written
// first in the same call, so nothing needs clearing between calls.
__global__ void __launch_bounds__(kThreads)
k_segment_partial(const double *__restrict__ x, const double *__restrict__ w,
                  SegmentOffsets seg, double2 *__restrict__ scratch)
{
   const int s = blockIdx.y;
   const long long b = seg.off[s], e = seg.off[s + 1];
   double sd = 0.0, sv = 0.0;
   for (long long i = b + (long long)blockIdx.x * kThreads + threadIdx.x; i < e;
        i += (long long)gridDim.x * kThreads) {
      const double xv = x[i], wv = w[i];
      sd += xv * xv * wv;
      sv += wv;
   }
   __shared__ double rs[kThreads], rv[kThreads];
   rs[threadIdx.x] = sd;
   rv[threadIdx.x] = sv;
   __syncthreads();
   for (int o = kThreads / 2; o > 0; o >>= 1) {
      if ((int)threadIdx.x < o) {
         rs[threadIdx.x] += rs[threadIdx.x + o];
         rv[threadIdx.x] += rv[threadIdx.x + o];
      }
      __syncthreads();
   }
   if (threadIdx.x == 0)
      scratch[s * kBlocksPerSegment + blockIdx.x] = make_double2(rs[0], rv[0]);
}

__global__ void k_segment_finish(const double2 *__restrict__ scratch, double *__restrict__ norms)
{
   const int s = blockIdx.x;
   __shared__ double rs[kBlocksPerSegment], rv[kBlocksPerSegment];
   const double2 v = scratch[s * kBlocksPerSegment + threadIdx.x];
   rs[threadIdx.x] = v.x;
   rv[threadIdx.x] = v.y;
   __syncthreads();
   for (int o = kBlocksPerSegment / 2; o > 0; o >>= 1) {
      if ((int)threadIdx.x < o) {
         rs[threadIdx.x] += rs[threadIdx.x + o];
         rv[threadIdx.x] += rv[threadIdx.x + o];
      }
      __syncthreads();
   }
   if (threadIdx.x == 0) norms[s] = rv[0] > 0.0 ? sqrt(rs[0]) / sqrt(rv[0]) : 0.0;
}

}  // namespace

extern "C" int fac_rms_norm_noalloc(const double *x, const double *w,
                                    const long long *seg_offsets, int nseg, double *norms,
                                    void *stream)
{
   if (nseg < 1 || nseg > kMaxSegments) {
      return FAC_ERR_ARG;
   }
   if (!x || !w || !seg_offsets || !norms) {
      return FAC_ERR_ARG;
   }
   SegmentOffsets seg;
   for (int s = 0; s <= nseg; ++s) {
      seg.off[s] = seg_offsets[s];
      if (seg.off[s] < 0 || (s > 0 && seg.off[s] < seg.off[s - 1])) {
         return FAC_ERR_ARG;
      }
   }
   // an error left pending by earlier work belongs to its owner: report it
   // without consuming it, so that any error after the launches is ours
   if (cudaPeekAtLastError() != cudaSuccess) {
      return FAC_ERR_CUDA;
   }
   int dev = 0;
   if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
      return FAC_ERR_CUDA;
   }
   double2 *scratch = nullptr;
   {
      // One-time set-up per device, with that device current: the address
      // of this device's copy of the static scratch array.
      std::lock_guard<std::mutex> lock(g_setup_mutex);
      if (!g_scratch_ptr[dev]) {
         void *p = nullptr;
         if (cudaGetSymbolAddress(&p, g_norm_scratch) != cudaSuccess || !p) {
            return FAC_ERR_CUDA;
         }
         g_scratch_ptr[dev] = static_cast<double2 *>(p);
      }
      scratch = g_scratch_ptr[dev];
   }
   cudaStream_t s = static_cast<cudaStream_t>(stream);
   k_segment_partial<<<dim3(kBlocksPerSegment, nseg), kThreads, 0, s>>>(x, w, seg, scratch);
   k_segment_finish<<<nseg, kBlocksPerSegment, 0, s>>>(scratch, norms);
   if (cudaGetLastError() != cudaSuccess) {
      return FAC_ERR_CUDA;
   }
   return FAC_OK;
}

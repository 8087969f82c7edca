// Transfer operators of the reference's other patch-data centerings, on the
// device: linear time interpolation of cell, side, face, node and edge data
// (pdat/*DoubleLinearTimeInterpolateOp.C over pdat_m4lintimeintops{2,3}d.i)
// and the index boxes of each centering (pdat/{Side,Face,Node,Edge}
// Geometry::to*Box), for codes that run RefineSchedules with time
// interpolation on data other than the FAC path's cell data.
//
// One launch interpolates a batch of up to kTimeBatch boxes whose
// descriptors travel as the kernel's parameter, so the call needs no device
// memory of its own; every element of the batch is one thread of a grid
// stride loop, boxes found by a binary search of their element prefix.
#include <cuda_runtime.h>

#include <cfloat>
#include <vector>

#include "../../include/samrai_fac_b200.h"
#include "fac_kernels.h"

namespace {

constexpr int kTimeBatch = 192;
constexpr int kThreads = 256;

struct TimeDesc {
   const double *old_data, *new_data;
   double *dst_data;
   int lo[3], n[3];                       // where box: lower corner, extents
   int ooff[3], noff[3], doff[3];         // where lower minus each array's lower
   int on[2], nn[2], dn[2];               // extents of the arrays' first two axes
};

struct TimeBatch {
   TimeDesc d[kTimeBatch];
   long long prefix[kTimeBatch + 1];
   int count;
};

static_assert(sizeof(TimeBatch) < 30000, "kernel parameter space");

__device__ __forceinline__ long long at(const int off[3], const int ext[2], int i, int j, int k)
{
   return (long long)(off[0] + i) +
          (long long)ext[0] * ((long long)(off[1] + j) + (long long)ext[1] * (off[2] + k));
}

// dst = old (1 - t) + new t, as lin_time_int_body_{2,3}d
// (pdat_m4lintimeintops2d.i: oldfrac = one - tfrac; arraydst = arrayold *
// oldfrac + arraynew * tfrac)
__global__ void __launch_bounds__(kThreads) k_time_interp(const TimeBatch b, double tfrac)
{
   const double oldfrac = 1.0 - tfrac;
   const long long total = b.prefix[b.count];
   for (long long e = (long long)blockIdx.x * kThreads + threadIdx.x; e < total;
        e += (long long)gridDim.x * kThreads) {
      int lo = 0, hi = b.count - 1;
      while (lo < hi) {
         const int mid = (lo + hi + 1) >> 1;
         if (b.prefix[mid] <= e) lo = mid;
         else hi = mid - 1;
      }
      const TimeDesc &d = b.d[lo];
      long long r = e - b.prefix[lo];
      const int i = (int)(r % d.n[0]);
      r /= d.n[0];
      const int j = (int)(r % d.n[1]);
      const int k = (int)(r / d.n[1]);
      const double vo = d.old_data[at(d.ooff, d.on, i, j, k)];
      const double vn = d.new_data[at(d.noff, d.nn, i, j, k)];
      d.dst_data[at(d.doff, d.dn, i, j, k)] = vo * oldfrac + vn * tfrac;
   }
}

bool inside(int dim, const int *lo, const int *hi, const int *blo, const int *bhi)
{
   for (int a = 0; a < dim; ++a)
      if (lo[a] < blo[a] || hi[a] > bhi[a]) return false;
   return true;
}

}  // namespace

extern "C" int fac_centered_box(int dim, int centering, int axis, const int *lo, const int *hi,
                                int *out_lo, int *out_hi)
{
   if (dim < 1 || dim > 3 || !lo || !hi || !out_lo || !out_hi) return FAC_ERR_ARG;
   if (centering != FAC_CELL && (axis < 0 || axis >= dim)) return FAC_ERR_ARG;
   for (int a = 0; a < 3; ++a) {
      out_lo[a] = a < dim ? lo[a] : 0;
      out_hi[a] = a < dim ? hi[a] : 0;
   }
   switch (centering) {
      case FAC_CELL:
         break;
      case FAC_SIDE:  // SideGeometry::toSideBox: upper + 1 along the axis
         out_hi[axis] += 1;
         break;
      case FAC_NODE:  // NodeGeometry::toNodeBox: upper + 1 along every axis
         for (int a = 0; a < dim; ++a) out_hi[a] += 1;
         break;
      case FAC_EDGE:  // EdgeGeometry::toEdgeBox: upper + 1 along the others
         for (int a = 0; a < dim; ++a)
            if (a != axis) out_hi[a] += 1;
         break;
      case FAC_FACE:  // FaceGeometry::toFaceBox: the axis first, the others
                      // in cyclic order, upper + 1 along the axis
         for (int q = 0; q < dim; ++q) {
            const int y = (axis + q) % dim;
            out_lo[q] = lo[y];
            out_hi[q] = hi[y] + (q == 0 ? 1 : 0);
         }
         break;
      default:
         return FAC_ERR_ARG;
   }
   return FAC_OK;
}

extern "C" int fac_time_interpolate(int dim, const fac_time_box *boxes, int nboxes,
                                    double old_time, double new_time, double dst_time,
                                    void *stream)
{
   if (dim < 1 || dim > 3 || nboxes < 0 || (nboxes > 0 && !boxes)) return FAC_ERR_ARG;
   if (cudaPeekAtLastError() != cudaSuccess) return FAC_ERR_CUDA;
   // CellDoubleLinearTimeInterpolateOp::timeInterpolate: the fraction of
   // the way from the old to the new time, 0 when the two coincide
   double tfrac = dst_time - old_time;
   const double denom = new_time - old_time;
   if (denom > DBL_MIN) tfrac /= denom;
   else tfrac = 0.0;
   cudaStream_t s = static_cast<cudaStream_t>(stream);
   TimeBatch b;
   int q = 0;
   while (q < nboxes) {
      b.count = 0;
      b.prefix[0] = 0;
      for (; q < nboxes && b.count < kTimeBatch; ++q) {
         const fac_time_box &x = boxes[q];
         if (!x.old_data || !x.new_data || !x.dst_data) return FAC_ERR_ARG;
         bool empty = false;
         for (int a = 0; a < dim; ++a) empty = empty || x.where_hi[a] < x.where_lo[a];
         if (empty) continue;
         if (!inside(dim, x.where_lo, x.where_hi, x.old_lo, x.old_hi) ||
             !inside(dim, x.where_lo, x.where_hi, x.new_lo, x.new_hi) ||
             !inside(dim, x.where_lo, x.where_hi, x.dst_lo, x.dst_hi))
            return FAC_ERR_ARG;
         TimeDesc &d = b.d[b.count];
         d.old_data = x.old_data;
         d.new_data = x.new_data;
         d.dst_data = x.dst_data;
         long long cells = 1;
         for (int a = 0; a < 3; ++a) {
            const bool on = a < dim;
            d.lo[a] = on ? x.where_lo[a] : 0;
            d.n[a] = on ? x.where_hi[a] - x.where_lo[a] + 1 : 1;
            d.ooff[a] = on ? x.where_lo[a] - x.old_lo[a] : 0;
            d.noff[a] = on ? x.where_lo[a] - x.new_lo[a] : 0;
            d.doff[a] = on ? x.where_lo[a] - x.dst_lo[a] : 0;
            if (a < 2) {
               d.on[a] = on ? x.old_hi[a] - x.old_lo[a] + 1 : 1;
               d.nn[a] = on ? x.new_hi[a] - x.new_lo[a] + 1 : 1;
               d.dn[a] = on ? x.dst_hi[a] - x.dst_lo[a] + 1 : 1;
            }
            cells *= d.n[a];
         }
         b.prefix[b.count + 1] = b.prefix[b.count] + cells;
         ++b.count;
      }
      if (b.count == 0) continue;
      const long long total = b.prefix[b.count];
      const long long blocks = (total + kThreads - 1) / kThreads;
      const int grid = (int)(blocks < 148 * 8 ? blocks : 148 * 8);
      samrai_b200::add_kernel_launches(1);
      k_time_interp<<<grid, kThreads, 0, s>>>(b, tfrac);
      if (cudaGetLastError() != cudaSuccess) return FAC_ERR_CUDA;
   }
   return FAC_OK;
}

// Device-side helpers shared by the FAC kernel files: index maps of the
// level buffers, the work-list loop and the Robin boundary formula.
#pragma once

#include <cuda_runtime.h>

#include "fac_internal.h"

namespace samrai_b200 {
namespace dev {

constexpr int kThreads = 256;
// Blocks of a chunk kernel when the occupancy query fails: enough to fill
// the GPU; each block walks the work list with a grid stride.
constexpr int kGridCap = 148 * 8;

// Blocks of kernel fn (kThreads threads, no dynamic shared memory) that fit
// on the device at once: the SMs times the resident blocks per SM, queried
// once per kernel.
int resident_blocks(const void *fn);

// Grid of a chunk kernel: one wave of resident blocks at most, so that no
// block of a second partial wave is left to run alone at the end.
template <class F>
inline int work_grid(F *fn, int nchunks)
{
   const int cap = resident_blocks(reinterpret_cast<const void *>(fn));
   return nchunks < cap ? nchunks : cap;
}

// Grid-stride walk over a work list of nwork entries.  The list is compacted
// on the device whenever the set of iterating problems changes: the chunks of
// those problems come first and a chunk with patch < 0 ends the list.
#define WORK_LOOP(ch)                                      \
   for (int w_ = blockIdx.x; w_ < nwork; w_ += gridDim.x) \
      if (const Chunk ch = chunks[w_]; ch.patch < 0)       \
         break;                                            \
      else

// Item and cell (within the item) of element t of a transaction-list chunk:
// a chunk of one item covers its cells [begin, begin + count); a packed
// chunk covers its aux items back to back (prefix: first cell of each item).
__device__ __forceinline__ int chunk_item(const Chunk &ch, const int *__restrict__ prefix, int t,
                                          int &lin)
{
   if (ch.aux <= 1) {
      lin = ch.begin + t;
      return ch.patch;
   }
   const int g = prefix[ch.patch] + t;
   int lo = ch.patch, hi = ch.patch + ch.aux - 1;
   while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (prefix[mid] <= g) lo = mid;
      else hi = mid - 1;
   }
   lin = g - prefix[lo];
   return lo;
}

__device__ __forceinline__ long long aidx(const ArrDesc &A, int i, int j, int k)
{
   return A.base + (long long)(i - A.lo[0]) +
          (long long)A.n[0] * ((long long)(j - A.lo[1]) +
                               (long long)A.n[1] * (long long)(k - A.lo[2]));
}

// Index of cell (i,j,k) in a patch's array with ghost width g.
template <int DIM>
__device__ __forceinline__ long long cidx(const PatchDesc &p, long long off,
                                          int g, int i, int j, int k)
{
   const int gz = DIM == 3 ? g : 0;
   const long long nx = p.hi[0] - p.lo[0] + 1 + 2 * g;
   const long long ny = p.hi[1] - p.lo[1] + 1 + 2 * g;
   return off + (i - p.lo[0] + g) + nx * ((j - p.lo[1] + g) + ny * (k - p.lo[2] + gz));
}

// Index of face (i,j,k) of axis a in a patch's side array (ghost 0).
__device__ __forceinline__ long long sidx(const PatchDesc &p, int a, int i, int j,
                                          int k)
{
   const long long nx = p.hi[0] - p.lo[0] + 1 + (a == 0);
   const long long ny = p.hi[1] - p.lo[1] + 1 + (a == 1);
   return p.offs[a] + (i - p.lo[0]) + nx * ((j - p.lo[1]) + ny * (k - p.lo[2]));
}

// Index of the tangential position of cell (i,j,k) in a face array of axis a.
__device__ __forceinline__ long long oidx(const PatchDesc &p, int a, int s, int i,
                                          int j, int k)
{
   const long long nx = p.hi[0] - p.lo[0] + 1;
   const long long ny = p.hi[1] - p.lo[1] + 1;
   long long t;
   if (a == 0) t = (j - p.lo[1]) + ny * (k - p.lo[2]);
   else if (a == 1) t = (i - p.lo[0]) + nx * (k - p.lo[2]);
   else t = (i - p.lo[0]) + nx * (j - p.lo[1]);
   return p.offo[a][s] + t;
}

// Cell (li, lj, lk) of linear index lin (x fastest) of a patch's cells:
// quotients by reciprocal multiplication when the patch carries its
// divisors (q / d = umulhi(q, ceil(2^32 / d)) for q d < 2^32).
__device__ __forceinline__ void patch_cell(const PatchDesc &p, int lin, int nx, int ny, int &li,
                                           int &lj, int &lk)
{
   if (p.mx) {
      const int r = (int)__umulhi((unsigned)lin, p.mx);
      li = lin - r * nx;
      lk = (int)__umulhi((unsigned)r, p.my);
      lj = r - lk * ny;
   } else {
      li = lin % nx;
      const int r = lin / nx;
      lj = r % ny;
      lk = r / ny;
   }
}

__device__ __forceinline__ int coarsen_index(int i, int r)
{
   return i < 0 ? (i + 1) / r - 1 : i / r;
}

// settype1cells{2,3}d (robinbchelper2d.f:10-72): ghost value from the
// interior value next to the boundary.
template <class T>
__device__ __forceinline__ T robin_abg(T uin, T a, T b, T g, T h, int hom)
{
   const T half = (T)0.5;
   if (hom) return (uin * (b - half * h * a)) / (b + half * h * a);
   return (h * g + uin * (b - half * h * a)) / (b + half * h * a);
}

template <class T>
__device__ __forceinline__ T robin(T uin, int loc, T h, int hom, const BcCoefs &bc)
{
   return robin_abg<T>(uin, (T)bc.a[loc], (T)bc.b[loc], (T)bc.g[loc], h, hom);
}

// The Robin ghost value across location loc of a boundary item of level
// lvl and problem prob, inward cell ci: the coefficients of that face when
// the level has per-face coefficients on that side (RobinBcCoefStrategy::
// setBcCoefs arrays), else the side's constants.
template <class T>
__device__ __forceinline__ T robin_at(T uin, int loc, T h, int hom, const BcCoefs &bc, int lvl,
                                      int prob, const int *ci)
{
   if (bc.face_base) {
      const long long off = bc.face_off[((long long)lvl * 6 + loc) * bc.face_nprob + prob];
      if (off >= 0) {
         const int *dm = bc.face_dom + ((long long)lvl * bc.face_nprob + prob) * 6;
         const int a = loc >> 1;
         long long idx = 0, stride = 1;
         for (int t = 0; t < 3; ++t) {
            if (t == a) continue;
            idx += stride * (ci[t] - dm[t]);
            stride *= dm[3 + t];
         }
         const double *f = bc.face_base + off + 3 * idx;
         return robin_abg<T>(uin, (T)f[0], (T)f[1], (T)f[2], h, hom);
      }
   }
   return robin<T>(uin, loc, h, hom, bc);
}

// One red-black point update from the six face fluxes (low/high per axis),
// the six face coefficients, C and f (rbgswithfluxmax*, 2d.f:136-160,
// 3d.f:196-226): returns the new value and the residual.  FP64 keeps the
// Fortran's evaluation order with every product and sum rounded separately
// (the build has no contraction).  FP32, used only for the error equation
// inside the mixed cycle whose FP64 outer loop restores the accuracy, fuses
// the sums of products into FMAs; the reciprocal is the correctly rounded
// one in both.
template <int DIM, class T>
__device__ __forceinline__ T rb_point(T fv, T uc, T scv, T dxi, T dyi, T dzi, T fxl, T fxh,
                                      T fyl, T fyh, T fzl, T fzh, T dx0, T dx1, T dy0, T dy1,
                                      T dz0, T dz1, T &residual)
{
   const T one = (T)1;
   if constexpr (sizeof(T) == 8) {
      T dudr;
      if (DIM == 2) {
         residual = fv - (dxi * (fxh - fxl) + dyi * (fyh - fyl)) - scv * uc;
         dudr = one / ((dxi * dxi * (dx1 + dx0) + dyi * dyi * (dy1 + dy0)) - scv);
      } else {
         const T dxi2 = dxi * dxi, dyi2 = dyi * dyi, dzi2 = dzi * dzi;
         residual = fv - (dxi * (fxh - fxl) + dyi * (fyh - fyl) + dzi * (fzh - fzl)) - scv * uc;
         dudr = one / ((dxi2 * (dx1 + dx0) + dyi2 * (dy1 + dy0) + dzi2 * (dz1 + dz0)) - scv);
      }
      const T du = -residual * dudr;
      const T rcoef = one;
      return uc + du * rcoef;
   } else {
      T div = dxi * (fxh - fxl);
      div = __fmaf_rn(dyi, fyh - fyl, div);
      T diag = dxi * dxi * (dx1 + dx0);
      diag = __fmaf_rn(dyi * dyi, dy1 + dy0, diag);
      if (DIM == 3) {
         div = __fmaf_rn(dzi, fzh - fzl, div);
         diag = __fmaf_rn(dzi * dzi, dz1 + dz0, diag);
      }
      residual = __fmaf_rn(-scv, uc, fv - div);
      const T dudr = __frcp_rn(diag - scv);
      return __fmaf_rn(-residual, dudr, uc);
   }
}

}  // namespace dev
}  // namespace samrai_b200

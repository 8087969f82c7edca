// FP64 kernels of the FAC Poisson hot path (sm_100a).
//
// Built with --fmad=false: every multiply and add is rounded separately, in
// the order of the reference's Fortran expressions, so results are
// bit-identical to the reference arithmetic (solv_cellpoissonfacops{2,3}d.f,
// geom_m4cart{refine,coarsen}ops{2,3}d.i, solv_cartesianrobinbchelper{2,3}d.f).
//
// All kernels are table driven: a level of every problem in the context is
// processed by one launch whose blocks each take one Chunk (a run of cells of
// one patch or one transaction), so patches of uneven size share the grid.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <mutex>
#include <stdexcept>
#include <unordered_map>

#include "fac_device.h"
#include "fac_internal.h"
#include "fac_kernels.h"

namespace samrai_b200 {

namespace {

using namespace dev;

__device__ __forceinline__ void atomic_max_nonneg(unsigned long long *addr, double v)
{
   atomicMax(addr, (unsigned long long)__double_as_longlong(v));
}

// ---------------------------------------------------------------------------
// ghost fill
// ---------------------------------------------------------------------------

// Cell lin of fill item it (x fastest, then y, then z).
template <class T>
__device__ __forceinline__ void fill_element(const FillItem &it, int lin, T *__restrict__ dst,
                                             const T *__restrict__ src_same,
                                             const T *__restrict__ src_coarse, int homogeneous,
                                             const BcCoefs &bc)
{
   const T *src = it.src_is_coarse ? src_coarse : src_same;
   const int nx = it.hi[0] - it.lo[0] + 1;
   const int ny = it.hi[1] - it.lo[1] + 1;
   const int i = it.lo[0] + lin % nx;
   const int r = lin / nx;
   const int j = it.lo[1] + r % ny;
   const int k = it.lo[2] + r / ny;
   T v;
   if (it.kind == kFillCopy) {
      v = src[aidx(it.src, i, j, k)];
   } else if (it.kind == kFillCoarse) {
      v = src[aidx(it.src, coarsen_index(i, it.ratio[0]), coarsen_index(j, it.ratio[1]),
                   coarsen_index(k, it.ratio[2]))];
   } else {
      // Every ghost value of codimension m depends only on the interior
      // cell reached by moving inward along all m outside axes
      // (settype1/2/3cells{2,3}d applied in codimension order).
      const int ci[3] = {i - it.side[0], j - it.side[1], k - it.side[2]};
      const T uin = src[aidx(it.src, ci[0], ci[1], ci[2])];
      T f[3];
      int m = 0;
      for (int a = 0; a < 3; ++a) {
         if (it.side[a]) {
            f[a] = robin_at<T>(uin, 2 * a + (it.side[a] > 0), (T)it.h[a], homogeneous, bc,
                               it.bc_level, it.prob, ci);
            ++m;
         } else {
            f[a] = (T)0;
         }
      }
      if (m == 1) {
         v = it.side[0] ? f[0] : (it.side[1] ? f[1] : f[2]);
      } else if (m == 2) {
         T s0 = (T)0, s1 = (T)0;
         int n = 0;
         for (int a = 0; a < 3; ++a)
            if (it.side[a]) {
               if (n == 0) s0 = f[a];
               else s1 = f[a];
               ++n;
            }
         v = -uin + (s1 + s0);
      } else {
         const T two3 = (T)(2.0f / 3.0f);
         v = -uin + two3 * ((f[0] + f[1]) + f[2]);
      }
   }
   dst[aidx(it.dst, i, j, k)] = v;
}

template <class T>
__global__ void __launch_bounds__(kThreads)
k_fill(const FillItem *__restrict__ items, const Chunk *__restrict__ chunks, int nwork,
       const int *__restrict__ prefix, T *__restrict__ dst, const T *__restrict__ src_same,
       const T *__restrict__ src_coarse, int homogeneous, BcCoefs bc,
       const int *__restrict__ active)
{
   WORK_LOOP(ch) {
      for (int t = threadIdx.x; t < ch.count; t += blockDim.x) {
         int lin;
         const FillItem &it = items[chunk_item(ch, prefix, t, lin)];
         if (active && !active[it.prob]) continue;
         fill_element<T>(it, lin, dst, src_same, src_coarse, homogeneous, bc);
      }
   }
}

// Ghost fill from a gather list: element e sets dst[to[e]] from the same
// level (from[e] >= 0) or from the coarser level's element -from[e] - 1
// (constant refine), when its problem prob[e] is active.  A flat launch:
// each thread of the first nblk blocks has kFillPer elements in flight (its
// index loads, then its value loads).  The blocks after them walk the
// physical-boundary items of the same fill.
constexpr int kFillPer = 4;

template <class T>
__global__ void __launch_bounds__(kThreads)
k_fill_gather(long long n, int nblk, const unsigned *__restrict__ to,
              const int *__restrict__ from, const unsigned short *__restrict__ prob,
              const FillItem *__restrict__ bc_items, const Chunk *__restrict__ bc_chunks, int nbc,
              const int *__restrict__ bc_prefix, T *__restrict__ dst,
              const T *__restrict__ src_same, const T *__restrict__ src_coarse, int homogeneous,
              BcCoefs bc, const int *__restrict__ active)
{
   if ((int)blockIdx.x < nblk) {
      const long long e0 = (long long)blockIdx.x * (kThreads * kFillPer) + threadIdx.x;
      unsigned d[kFillPer];
      int sx[kFillPer];
      bool on[kFillPer];
#pragma unroll
      for (int q = 0; q < kFillPer; ++q) {
         const long long e = e0 + q * kThreads;
         on[q] = e < n;
         d[q] = 0u;
         sx[q] = 0;
         if (on[q]) {
            d[q] = to[e];
            sx[q] = from[e];
            if (active) on[q] = active[prob[e]] != 0;
         }
      }
      T v[kFillPer];
#pragma unroll
      for (int q = 0; q < kFillPer; ++q)
         if (on[q]) v[q] = sx[q] >= 0 ? src_same[sx[q]] : src_coarse[-(sx[q] + 1)];
#pragma unroll
      for (int q = 0; q < kFillPer; ++q)
         if (on[q]) dst[d[q]] = v[q];
      return;
   }
   for (int w = (int)blockIdx.x - nblk; w < nbc; w += (int)gridDim.x - nblk) {
      const Chunk ch = bc_chunks[w];
      if (ch.patch < 0) break;
      for (int t = threadIdx.x; t < ch.count; t += blockDim.x) {
         int lin;
         const FillItem &it = bc_items[chunk_item(ch, bc_prefix, t, lin)];
         if (active && !active[it.prob]) continue;
         fill_element<T>(it, lin, dst, src_same, src_coarse, homogeneous, bc);
      }
   }
}

// ---------------------------------------------------------------------------
// Ewing coarse-fine flux (ewingfixflux{vardc,condc}{2,3}d, 2d.f:460-686,
// 3d.f:604-1012), evaluated from the current u.
// ---------------------------------------------------------------------------

template <class T>
__device__ __forceinline__ T ewing_flux(const T *__restrict__ u, const T *__restrict__ dside,
                                        const CfFace &cf, const PatchDesc &p, int dvar,
                                        T dconst, const double *tranwt, const double *longwt)
{
   const int a = cf.axis;
   const T d = dvar ? dside[cf.sidx] : dconst;
   const T h = (T)p.dx[a];
   const T dxi = (T)1 / h;
   const T uc = u[cf.cell], ug = u[cf.ghost], um = u[cf.mirror];
   const T tw = (T)tranwt[a], lw = (T)longwt[a];
   T flux;
   if (cf.side == 0) {
      flux = dxi * d * (uc - ug);
      return lw * flux + tw * d * (um - uc) / h;
   }
   flux = dxi * d * (ug - uc);
   return lw * flux - tw * d * (um - uc) / h;
}

struct EwingWeights {
   double tranwt[3];
   double longwt[3];
};

template <class T>
__global__ void __launch_bounds__(kThreads)
k_cf_flux(const CfFace *__restrict__ faces, int nfaces,
          const PatchDesc *__restrict__ patches, const T *__restrict__ u,
          const T *__restrict__ dside, int dvar, T dconst,
          EwingWeights w, T *__restrict__ cfflux,
          const int *__restrict__ run)
{
   const int t = blockIdx.x * blockDim.x + threadIdx.x;
   if (t >= nfaces) return;
   const CfFace cf = faces[t];
   const PatchDesc &p = patches[cf.patch];
   if (run && !run[p.prob]) return;
   cfflux[cf.oidx] = ewing_flux<T>(u, dside, cf, p, dvar, dconst, w.tranwt, w.longwt);
}

// ---------------------------------------------------------------------------
// red-black Gauss-Seidel colour pass with on-the-fly fluxes
// (compflux* + rbgswithfluxmax*, 2d.f:10-364, 3d.f:10-484)
// ---------------------------------------------------------------------------

// FUSED: values across patch faces are read where they live instead of from
// the patch's ghost cells -- the neighbour patch's interior cell (which has
// the other colour, so it does not change during the pass), the Robin value
// of the cell itself at a physical boundary (homogeneous, as the
// smoother's fills are), or the precomputed Ewing flux at a coarse-fine
// face -- so the three ghost fills around each colour pass are not needed.
// One slot s of a colour pass over patch p (the cell of the active colour
// in row s / hx): the update of compflux + rbgswithfluxmax and the running
// maximum of |residual|.
template <int DIM, bool DVAR, int CKIND, class T, bool FUSED>
__device__ __forceinline__ void rb_slot(const PatchDesc &p, int s, int nx, int ny, int hx, T dxi,
                                        T dyi, T dzi, bool has_cf, T *__restrict__ u,
                                        const T *__restrict__ f, const T *__restrict__ dside,
                                        const T *__restrict__ cfield,
                                        const T *__restrict__ cfflux,
                                        const unsigned char *__restrict__ cfmask, int offset,
                                        T dconst, T cconst, const long long *__restrict__ facemap,
                                        const BcCoefs &bc, double &maxres)
{
      const int row = s / hx;
      const int mm = s - row * hx;
      const int j = p.lo[1] + row % ny;
      const int k = DIM == 3 ? p.lo[2] + row / ny : 0;
      int ioffset;
      if (DIM == 2) {
         const int q = p.lo[1] + j;
         ioffset = (q - (q / 2) * 2) != offset ? 1 : 0;
      } else {
         const int q = p.lo[0] + j + k;
         ioffset = (q - (q / 2) * 2) != offset ? 1 : 0;
      }
      const int i = p.lo[0] + ioffset + 2 * mm;
      if (i > p.hi[0]) return;
      const long long c = cidx<DIM>(p, p.off1, 1, i, j, k);
      const long long sx = 1;
      const long long sy = nx + 2;
      const long long sz = (long long)(nx + 2) * (ny + 2);
      const T uc = u[c];
      T dx0, dx1, dy0, dy1, dz0 = (T)0, dz1 = (T)0;
      if (DVAR) {
         dx0 = dside[sidx(p, 0, i, j, k)];
         dx1 = dside[sidx(p, 0, i + 1, j, k)];
         dy0 = dside[sidx(p, 1, i, j, k)];
         dy1 = dside[sidx(p, 1, i, j + 1, k)];
         if (DIM == 3) {
            dz0 = dside[sidx(p, 2, i, j, k)];
            dz1 = dside[sidx(p, 2, i, j, k + 1)];
         }
      } else {
         dx0 = dx1 = dy0 = dy1 = dz0 = dz1 = dconst;
      }
      T nxl, nxh, nyl, nyh, nzl = (T)0, nzh = (T)0;
      if (FUSED) {
         auto across = [&](int a, int sd, long long own) -> T {
            const long long m = facemap[oidx(p, a, sd, i, j, k)];
            if (m >= 0) return u[m];
            if (m == -1) return robin<T>(uc, 2 * a + sd, (T)p.dx[a], 1, bc);
            return u[own];
         };
         nxl = i == p.lo[0] ? across(0, 0, c - sx) : u[c - sx];
         nxh = i == p.hi[0] ? across(0, 1, c + sx) : u[c + sx];
         nyl = j == p.lo[1] ? across(1, 0, c - sy) : u[c - sy];
         nyh = j == p.hi[1] ? across(1, 1, c + sy) : u[c + sy];
         if (DIM == 3) {
            nzl = k == p.lo[2] ? across(2, 0, c - sz) : u[c - sz];
            nzh = k == p.hi[2] ? across(2, 1, c + sz) : u[c + sz];
         }
      } else {
         nxl = u[c - sx];
         nxh = u[c + sx];
         nyl = u[c - sy];
         nyh = u[c + sy];
         if (DIM == 3) {
            nzl = u[c - sz];
            nzh = u[c + sz];
         }
      }
      T fxl = dxi * dx0 * (uc - nxl);
      T fxh = dxi * dx1 * (nxh - uc);
      T fyl = dyi * dy0 * (uc - nyl);
      T fyh = dyi * dy1 * (nyh - uc);
      T fzl = (T)0, fzh = (T)0;
      if (DIM == 3) {
         fzl = dzi * dz0 * (uc - nzl);
         fzh = dzi * dz1 * (nzh - uc);
      }
      if (has_cf) {
         if (i == p.lo[0]) {
            const long long o = oidx(p, 0, 0, i, j, k);
            if (cfmask[o]) fxl = cfflux[o];
         }
         if (i == p.hi[0]) {
            const long long o = oidx(p, 0, 1, i, j, k);
            if (cfmask[o]) fxh = cfflux[o];
         }
         if (j == p.lo[1]) {
            const long long o = oidx(p, 1, 0, i, j, k);
            if (cfmask[o]) fyl = cfflux[o];
         }
         if (j == p.hi[1]) {
            const long long o = oidx(p, 1, 1, i, j, k);
            if (cfmask[o]) fyh = cfflux[o];
         }
         if (DIM == 3) {
            if (k == p.lo[2]) {
               const long long o = oidx(p, 2, 0, i, j, k);
               if (cfmask[o]) fzl = cfflux[o];
            }
            if (k == p.hi[2]) {
               const long long o = oidx(p, 2, 1, i, j, k);
               if (cfmask[o]) fzh = cfflux[o];
            }
         }
      }
      const T sf = CKIND == 2 ? cfield[cidx<DIM>(p, p.off0, 0, i, j, k)]
                              : (CKIND == 1 ? cconst : (T)0);
      const T fv = f[cidx<DIM>(p, p.off0, 0, i, j, k)];
      T residual;
      u[c] = rb_point<DIM, T>(fv, uc, sf, dxi, dyi, dzi, fxl, fxh, fyl, fyh, fzl, fzh, dx0, dx1,
                              dy0, dy1, dz0, dz1, residual);
      const double ar = fabs((double)residual);
      if (maxres < ar) maxres = ar;
}

template <int DIM, bool DVAR, int CKIND, class T, bool FUSED>
__global__ void __launch_bounds__(kThreads, 3)
k_rbgs(const PatchDesc *__restrict__ patches, const Chunk *__restrict__ chunks, int nwork,
       T *__restrict__ u, const T *__restrict__ f,
       const T *__restrict__ dside, const T *__restrict__ cfield,
       const T *__restrict__ cfflux, const unsigned char *__restrict__ cfmask,
       int offset, T dconst, T cconst,
       unsigned long long *__restrict__ maxres_patch, const int *__restrict__ run,
       const long long *__restrict__ facemap, BcCoefs bc)
{
   WORK_LOOP(ch) {
      const PatchDesc p = patches[ch.patch];
      if (run && !run[p.prob]) continue;
      const int nx = p.hi[0] - p.lo[0] + 1;
      const int ny = p.hi[1] - p.lo[1] + 1;
      const int hx = (nx + 1) >> 1;
      const T one = (T)1;
      const T dxi = one / (T)p.dx[0], dyi = one / (T)p.dx[1];
      const T dzi = DIM == 3 ? one / (T)p.dx[2] : (T)0;
      const bool has_cf = (p.flags & 1) != 0;
      double maxres = 0.0;
      for (int t = threadIdx.x; t < ch.count; t += blockDim.x)
         rb_slot<DIM, DVAR, CKIND, T, FUSED>(p, ch.begin + t, nx, ny, hx, dxi, dyi, dzi, has_cf, u,
                                             f, dside, cfield, cfflux, cfmask, offset, dconst,
                                             cconst, facemap, bc, maxres);
      // block max, then one atomic per block
      __shared__ double red[kThreads / 32];
      for (int o = 16; o > 0; o >>= 1) {
         const double other = __shfl_down_sync(0xffffffffu, maxres, o);
         maxres = other > maxres ? other : maxres;
      }
      if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = maxres;
      __syncthreads();
      if (threadIdx.x == 0) {
         double m = red[0];
         for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = red[w] > m ? red[w] : m;
         if (maxres_patch) atomic_max_nonneg(&maxres_patch[ch.patch], m);
      }
      __syncthreads();  // shared memory is reused by the next chunk
   }
}

// Red-black smoothing to a tolerance of a level with one patch per problem
// and no coarser level, all sweeps in one launch: block b owns patch b
// (problem patches[b].prob) and runs up to nsweeps sweeps of a red and a
// black pass, __syncthreads between passes, with the fused neighbour reads
// (physical boundaries through the facemap).  After each sweep the block
// applies the sweep check of smoothErrorByRedBlack: the sweep counts, and
// with tol >= 0 the problem stops once max(red, black) max |residual| <=
// tol.  Same cells, order and arithmetic as k_rbgs + k_sweep_check, so the
// same bits.
template <int DIM, bool DVAR, int CKIND, class T>
__global__ void __launch_bounds__(kThreads)
k_rbgs_solve(const PatchDesc *__restrict__ patches, T *__restrict__ u, const T *__restrict__ f,
             const T *__restrict__ dside, const T *__restrict__ cfield, T dconst, T cconst,
             const long long *__restrict__ facemap, BcCoefs bc, int nsweeps, double tol,
             int *__restrict__ run, long long *__restrict__ sweeps,
             unsigned long long *__restrict__ maxres_red,
             unsigned long long *__restrict__ maxres_blk)
{
   const int ip = blockIdx.x;
   const PatchDesc p = patches[ip];
   const int pr = p.prob;
   if (!run[pr]) return;
   const int nx = p.hi[0] - p.lo[0] + 1;
   const int ny = p.hi[1] - p.lo[1] + 1;
   const int nz = DIM == 3 ? p.hi[2] - p.lo[2] + 1 : 1;
   const int hx = (nx + 1) >> 1;
   const int nslots = hx * ny * nz;
   const T one = (T)1;
   const T dxi = one / (T)p.dx[0], dyi = one / (T)p.dx[1];
   const T dzi = DIM == 3 ? one / (T)p.dx[2] : (T)0;
   __shared__ double red[kThreads / 32];
   bool going = true;
   double mcol[2] = {0.0, 0.0};
   for (int sw = 0; sw < nsweeps && going; ++sw) {
      for (int color = 0; color < 2; ++color) {
         double maxres = 0.0;
         for (int t = threadIdx.x; t < nslots; t += blockDim.x)
            rb_slot<DIM, DVAR, CKIND, T, true>(p, t, nx, ny, hx, dxi, dyi, dzi, false, u, f,
                                               dside, cfield, nullptr, nullptr, color, dconst,
                                               cconst, facemap, bc, maxres);
         for (int o = 16; o > 0; o >>= 1) {
            const double other = __shfl_down_sync(0xffffffffu, maxres, o);
            maxres = other > maxres ? other : maxres;
         }
         if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = maxres;
         // the pass's writes and maxima are visible to the whole block
         __syncthreads();
         double m = red[0];
         for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = red[w] > m ? red[w] : m;
         mcol[color] = m;
         __syncthreads();  // red is reused
      }
      if (threadIdx.x == 0) sweeps[pr] += 1;
      if (tol >= 0.0) going = (mcol[0] > mcol[1] ? mcol[0] : mcol[1]) > tol;
   }
   if (threadIdx.x == 0) {
      run[pr] = going ? 1 : 0;
      maxres_red[ip] = (unsigned long long)__double_as_longlong(mcol[0]);
      maxres_blk[ip] = (unsigned long long)__double_as_longlong(mcol[1]);
   }
}

// k_rbgs_solve with the patch held in shared memory: u (ghosted), f, the
// side arrays of D and the C field are copied in once, every sweep runs on
// the copies, and u is copied back.  rb_slot sees a patch descriptor whose
// offsets point into the shared copies, so the arithmetic and the order of
// the updates are those of k_rbgs_solve (the same bits).  For levels whose
// face table has no same-level neighbour (one patch covering the domain),
// patch by patch within the shared-memory limit.
constexpr int kSolveSmemThreads = 512;

template <int DIM, bool DVAR, int CKIND, class T>
__global__ void __launch_bounds__(kSolveSmemThreads)
k_rbgs_solve_smem(const PatchDesc *__restrict__ patches, T *__restrict__ u,
                  const T *__restrict__ f, const T *__restrict__ dside,
                  const T *__restrict__ cfield, T dconst, T cconst,
                  const long long *__restrict__ facemap, BcCoefs bc, int nsweeps, double tol,
                  int *__restrict__ run, long long *__restrict__ sweeps,
                  unsigned long long *__restrict__ maxres_red,
                  unsigned long long *__restrict__ maxres_blk)
{
   extern __shared__ __align__(16) unsigned char psm[];
   const int ip = blockIdx.x;
   const PatchDesc p = patches[ip];
   const int pr = p.prob;
   if (!run[pr]) return;
   const int nx = p.hi[0] - p.lo[0] + 1;
   const int ny = p.hi[1] - p.lo[1] + 1;
   const int nz = DIM == 3 ? p.hi[2] - p.lo[2] + 1 : 1;
   const long long n1 = (long long)(nx + 2) * (ny + 2) * (DIM == 3 ? nz + 2 : 1);
   const long long n0 = (long long)nx * ny * nz;
   long long ns[3] = {0, 0, 0};
   for (int a = 0; a < DIM; ++a)
      ns[a] = (long long)(nx + (a == 0)) * (ny + (a == 1)) * (DIM == 3 ? nz + (a == 2) : 1);
   T *su = reinterpret_cast<T *>(psm);
   T *sf = su + n1;
   T *sd = sf + n0;
   T *sc = sd + (DVAR ? ns[0] + ns[1] + ns[2] : 0);
   for (long long q = threadIdx.x; q < n1; q += blockDim.x) su[q] = u[p.off1 + q];
   for (long long q = threadIdx.x; q < n0; q += blockDim.x) sf[q] = f[p.off0 + q];
   if (DVAR) {
      long long o = 0;
      for (int a = 0; a < DIM; ++a) {
         for (long long q = threadIdx.x; q < ns[a]; q += blockDim.x) sd[o + q] = dside[p.offs[a] + q];
         o += ns[a];
      }
   }
   if (CKIND == 2)
      for (long long q = threadIdx.x; q < n0; q += blockDim.x) sc[q] = cfield[p.off0 + q];
   PatchDesc pl = p;
   pl.off1 = 0;
   pl.off0 = 0;
   pl.offs[0] = 0;
   pl.offs[1] = ns[0];
   pl.offs[2] = ns[0] + ns[1];
   __syncthreads();
   const int hx = (nx + 1) >> 1;
   const int nslots = hx * ny * nz;
   const T one = (T)1;
   const T dxi = one / (T)p.dx[0], dyi = one / (T)p.dx[1];
   const T dzi = DIM == 3 ? one / (T)p.dx[2] : (T)0;
   __shared__ double red[kSolveSmemThreads / 32];
   bool going = true;
   double mcol[2] = {0.0, 0.0};
   for (int sw = 0; sw < nsweeps && going; ++sw) {
      for (int color = 0; color < 2; ++color) {
         double maxres = 0.0;
         for (int t = threadIdx.x; t < nslots; t += blockDim.x)
            rb_slot<DIM, DVAR, CKIND, T, true>(pl, t, nx, ny, hx, dxi, dyi, dzi, false, su, sf,
                                               sd, sc, nullptr, nullptr, color, dconst, cconst,
                                               facemap, bc, maxres);
         for (int o = 16; o > 0; o >>= 1) {
            const double other = __shfl_down_sync(0xffffffffu, maxres, o);
            maxres = other > maxres ? other : maxres;
         }
         if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = maxres;
         __syncthreads();
         double m = red[0];
         for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = red[w] > m ? red[w] : m;
         mcol[color] = m;
         __syncthreads();
      }
      if (threadIdx.x == 0) sweeps[pr] += 1;
      if (tol >= 0.0) going = (mcol[0] > mcol[1] ? mcol[0] : mcol[1]) > tol;
   }
   for (long long q = threadIdx.x; q < n1; q += blockDim.x) u[p.off1 + q] = su[q];
   if (threadIdx.x == 0) {
      run[pr] = going ? 1 : 0;
      maxres_red[ip] = (unsigned long long)__double_as_longlong(mcol[0]);
      maxres_blk[ip] = (unsigned long long)__double_as_longlong(mcol[1]);
   }
}

// ---------------------------------------------------------------------------
// fluxes into side arrays, with the Ewing fix on coarse-fine faces
// (computeFluxOnPatch, CellPoissonFACOps.C:2157-2267)
// ---------------------------------------------------------------------------

template <int DIM, bool DVAR, class TU>
__global__ void __launch_bounds__(kThreads)
k_flux(const PatchDesc *__restrict__ patches, const Chunk *__restrict__ chunks, int nwork,
       const TU *__restrict__ u, const double *__restrict__ dside,
       double dconst, const unsigned char *__restrict__ cfmask, EwingWeights w,
       const int *ratio_to_coarser, double *__restrict__ flux,
       const int *__restrict__ run)
{
   WORK_LOOP(ch) {
      const PatchDesc p = patches[ch.patch];
      if (run && !run[p.prob]) continue;
      const int a = ch.aux;
      const int nx = p.hi[0] - p.lo[0] + 1 + (a == 0);
      const int ny = p.hi[1] - p.lo[1] + 1 + (a == 1);
      const double dai = 1. / p.dx[a];
      const bool has_cf = (p.flags & 1) != 0;
      for (int t = threadIdx.x; t < ch.count; t += blockDim.x) {
         const int lin = ch.begin + t;
         const int i = p.lo[0] + lin % nx;
         const int r = lin / nx;
         const int j = p.lo[1] + r % ny;
         const int k = DIM == 3 ? p.lo[2] + r / ny : 0;
         int cm[3] = {i, j, k};
         cm[a] -= 1;
         const long long cp = cidx<DIM>(p, p.off1, 1, i, j, k);
         const long long cq = cidx<DIM>(p, p.off1, 1, cm[0], cm[1], cm[2]);
         const long long si = sidx(p, a, i, j, k);
         const double d = DVAR ? dside[si] : dconst;
         double fl = dai * d * ((double)u[cp] - (double)u[cq]);
         if (has_cf) {
            const int fc[3] = {i, j, k};
            int s = -1;
            if (fc[a] == p.lo[a]) s = 0;
            else if (fc[a] == p.hi[a] + 1) s = 1;
            if (s >= 0) {
               int cc[3] = {i, j, k};
               if (s == 1) cc[a] -= 1;
               const long long o = oidx(p, a, s, cc[0], cc[1], cc[2]);
               if (cfmask[o]) {
                  int mq[3] = {cc[0], cc[1], cc[2]};
                  for (int tt = 0; tt < DIM; ++tt) {
                     if (tt == a) continue;
                     const int rr = ratio_to_coarser[tt];
                     const int base = coarsen_index(cc[tt], rr) * rr;
                     mq[tt] = base + (rr - (cc[tt] - base) - 1);
                  }
                  const double uc = (double)u[cidx<DIM>(p, p.off1, 1, cc[0], cc[1], cc[2])];
                  const double um = (double)u[cidx<DIM>(p, p.off1, 1, mq[0], mq[1], mq[2])];
                  if (s == 0) fl = w.longwt[a] * fl + w.tranwt[a] * d * (um - uc) / p.dx[a];
                  else fl = w.longwt[a] * fl - w.tranwt[a] * d * (um - uc) / p.dx[a];
               }
            }
         }
         flux[si] = fl;
      }
   }
}

// Ewing fix of the flux on face (a, s) of cell (i, j, k) of patch p
// (ewingfixflux*, 2d.f:460-686, 3d.f:604-1012); out of line: only
// coarse-fine faces take it.
template <int DIM, class TU>
__device__ __noinline__ double ewing_face(const PatchDesc &p, const TU *__restrict__ u, int a,
                                          int s, int i, int j, int k, double fl, double d,
                                          const EwingWeights &w, const int *ratio_to_coarser)
{
   const int cc[3] = {i, j, k};
   int mq[3] = {i, j, k};
   for (int tt = 0; tt < DIM; ++tt) {
      if (tt == a) continue;
      const int rr = ratio_to_coarser[tt];
      const int base = coarsen_index(cc[tt], rr) * rr;
      mq[tt] = base + (rr - (cc[tt] - base) - 1);
   }
   const double uc = (double)u[cidx<DIM>(p, p.off1, 1, i, j, k)];
   const double um = (double)u[cidx<DIM>(p, p.off1, 1, mq[0], mq[1], mq[2])];
   if (s == 0) return w.longwt[a] * fl + w.tranwt[a] * d * (um - uc) / p.dx[a];
   return w.longwt[a] * fl - w.tranwt[a] * d * (um - uc) / p.dx[a];
}

// Fluxes of every face of the level, one thread per cell: the lower face of
// each axis, and the upper one as well for the last cell of a row -- the
// arithmetic of computeFluxOnPatch with one cell decode for all axes.  The
// Ewing fix of the coarse-fine faces follows in k_ewing_fix.
template <int DIM, bool DVAR, class TU>
__global__ void __launch_bounds__(kThreads, 4)
k_flux_cells(const PatchDesc *__restrict__ patches, const Chunk *__restrict__ chunks, int nwork,
             const TU *__restrict__ u, const double *__restrict__ dside, double dconst,
             const unsigned char *__restrict__ cfmask, EwingWeights w,
             const int *ratio_to_coarser, double *__restrict__ flux,
             const int *__restrict__ run)
{
   WORK_LOOP(ch) {
      const PatchDesc &p = patches[ch.patch];
      if (run && !run[p.prob]) continue;
      const int nx = p.hi[0] - p.lo[0] + 1;
      const int ny = p.hi[1] - p.lo[1] + 1;
      const int nz = DIM == 3 ? p.hi[2] - p.lo[2] + 1 : 1;
      const int gx = nx + 2, gxy = (nx + 2) * (ny + 2);
      const TU *up = u + p.off1;
      const double dai[3] = {1. / p.dx[0], 1. / p.dx[1], DIM == 3 ? 1. / p.dx[2] : 0.0};
      for (int t = threadIdx.x; t < ch.count; t += blockDim.x) {
         const int lin = ch.begin + t;
         int li, lj, lk;
         patch_cell(p, lin, nx, ny, li, lj, lk);
         const int c = (li + 1) + gx * (lj + 1) + (DIM == 3 ? gxy * (lk + 1) : 0);
         const double uc = (double)up[c];
         // side-array positions of the cell's lower faces
         const int sx = li + (nx + 1) * (lj + ny * lk);
         const int sy = li + nx * (lj + (ny + 1) * lk);
         const int sz = li + nx * (lj + ny * lk);
#pragma unroll
         for (int a = 0; a < DIM; ++a) {
            const int la = a == 0 ? li : (a == 1 ? lj : lk);
            const int na = a == 0 ? nx : (a == 1 ? ny : nz);
            const int st = a == 0 ? 1 : (a == 1 ? gx : gxy);
            const long long sbase = p.offs[a] + (a == 0 ? sx : (a == 1 ? sy : sz));
            const int sup = a == 0 ? 1 : (a == 1 ? nx : nx * ny);
#pragma unroll
            for (int s = 0; s < 2; ++s) {
               if (s == 1 && la != na - 1) break;
               const long long si = sbase + (s ? sup : 0);
               const double d = DVAR ? dside[si] : dconst;
               const double ulo = s ? uc : (double)up[c - st];
               const double uhi = s ? (double)up[c + st] : uc;
               flux[si] = dai[a] * d * (uhi - ulo);
            }
         }
      }
   }
}

// Ewing fix of the stored flux on every coarse-fine face of the level
// (ewingfixflux*, 2d.f:460-686, 3d.f:604-1012): flux = longwt*flux
// +/- tranwt*D*(u(mirror) - u(cell))/h, after k_flux_cells.
template <class TU>
__global__ void __launch_bounds__(kThreads)
k_ewing_fix(const CfFace *__restrict__ faces, int nfaces, const PatchDesc *__restrict__ patches,
            const TU *__restrict__ u, const double *__restrict__ dside, int dvar,
            double dconst, EwingWeights w, double *__restrict__ flux,
            const int *__restrict__ run)
{
   const int t = blockIdx.x * blockDim.x + threadIdx.x;
   if (t >= nfaces) return;
   const CfFace cf = faces[t];
   const PatchDesc &p = patches[cf.patch];
   if (run && !run[p.prob]) return;
   const int a = cf.axis;
   const double d = dvar ? dside[cf.sidx] : dconst;
   const double fl = flux[cf.sidx];
   const double uc = (double)u[cf.cell], um = (double)u[cf.mirror];
   if (cf.side == 0) flux[cf.sidx] = w.longwt[a] * fl + w.tranwt[a] * d * (um - uc) / p.dx[a];
   else flux[cf.sidx] = w.longwt[a] * fl - w.tranwt[a] * d * (um - uc) / p.dx[a];
}

// ---------------------------------------------------------------------------
// residual from side fluxes (compres{var,con}sca{2,3}d) and outer-side save
// ---------------------------------------------------------------------------

template <int DIM, int CKIND, class TU>
__global__ void __launch_bounds__(kThreads, 4)
k_residual(const PatchDesc *__restrict__ patches, const Chunk *__restrict__ chunks, int nwork,
           const TU *__restrict__ u, const double *__restrict__ f,
           const double *__restrict__ flux, const double *__restrict__ cfield,
           double cconst, double *__restrict__ res, double *__restrict__ oflux,
           const int *__restrict__ run)
{
   WORK_LOOP(ch) {
      const PatchDesc &p = patches[ch.patch];
      if (run && !run[p.prob]) continue;
      const int nx = p.hi[0] - p.lo[0] + 1;
      const int ny = p.hi[1] - p.lo[1] + 1;
      const int nz = DIM == 3 ? p.hi[2] - p.lo[2] + 1 : 1;
      const int gx = nx + 2, gxy = (nx + 2) * (ny + 2);
      const double dxi = 1. / p.dx[0], dyi = 1. / p.dx[1];
      const double dzi = DIM == 3 ? 1. / p.dx[2] : 0.0;
      const double *fx = flux + p.offs[0], *fy = flux + p.offs[1];
      const double *fz = DIM == 3 ? flux + p.offs[2] : nullptr;
      for (int t = threadIdx.x; t < ch.count; t += blockDim.x) {
         const int lin = ch.begin + t;
         int li, lj, lk;
         patch_cell(p, lin, nx, ny, li, lj, lk);
         const int sx = li + (nx + 1) * (lj + ny * lk);
         const int sy = li + nx * (lj + (ny + 1) * lk);
         const double fxl = fx[sx], fxh = fx[sx + 1];
         const double fyl = fy[sy], fyh = fy[sy + nx];
         const long long c0 = p.off0 + lin;
         const double uc =
            (double)u[p.off1 + (li + 1) + gx * (lj + 1) + (DIM == 3 ? gxy * (lk + 1) : 0)];
         const double sf = CKIND == 2 ? cfield[c0] : (CKIND == 1 ? cconst : 0.0);
         double rv, fzl = 0.0, fzh = 0.0;
         if (DIM == 2) {
            rv = f[c0] - (dxi * (fxh - fxl) + dyi * (fyh - fyl)) - sf * uc;
         } else {
            const int sz = li + nx * (lj + ny * lk);
            fzl = fz[sz];
            fzh = fz[sz + nx * ny];
            rv = f[c0] - (dxi * (fxh - fxl) + dyi * (fyh - fyl) + dzi * (fzh - fzl)) - sf * uc;
         }
         res[c0] = rv;
         if (oflux) {
            const int i = p.lo[0] + li, j = p.lo[1] + lj, k = DIM == 3 ? p.lo[2] + lk : 0;
            if (li == 0) oflux[oidx(p, 0, 0, i, j, k)] = fxl;
            if (li == nx - 1) oflux[oidx(p, 0, 1, i, j, k)] = fxh;
            if (lj == 0) oflux[oidx(p, 1, 0, i, j, k)] = fyl;
            if (lj == ny - 1) oflux[oidx(p, 1, 1, i, j, k)] = fyh;
            if (DIM == 3) {
               if (lk == 0) oflux[oidx(p, 2, 0, i, j, k)] = fzl;
               if (lk == nz - 1) oflux[oidx(p, 2, 1, i, j, k)] = fzh;
            }
         }
      }
   }
}

// ---------------------------------------------------------------------------
// composite residual with the fluxes formed on the fly: the arithmetic of
// k_flux (Ewing fix on coarse-fine faces) and k_residual in one pass, so the
// side-array fluxes are neither written nor read back.  Faces that carry a
// coarsened finer-level flux (fcmask) take it from fcflux, where
// k_flux_coarsen put it, as the two-kernel sequence does.
// ---------------------------------------------------------------------------

// The residual of cell (li, lj, lk) of patch p (linear index lin) with its
// fluxes formed on the spot; writes res and, where oflux is given, the
// cell's patch-face fluxes.
template <int DIM, bool DVAR, int CKIND, class TU>
__device__ __forceinline__ void residual_cell(
   const PatchDesc &p, int lin, int li, int lj, int lk, const double dai[3],
   const TU *__restrict__ u, const double *__restrict__ dside, double dconst,
   const unsigned char *__restrict__ cfmask, const EwingWeights &w, const int *ratio_to_coarser,
   const unsigned char *__restrict__ fcmask, const double *__restrict__ fcflux,
   const double *__restrict__ f, const double *__restrict__ cfield, double cconst,
   double *__restrict__ res, double *__restrict__ oflux)
{
   const int nx = p.hi[0] - p.lo[0] + 1;
   const int ny = p.hi[1] - p.lo[1] + 1;
   const int nz = DIM == 3 ? p.hi[2] - p.lo[2] + 1 : 1;
   const bool has_cf = (p.flags & 1) != 0;
   // faces taking a coarsened finer-level flux exist on this patch
   const bool has_fc = fcmask && (p.flags & 2) != 0;
   const int gx = nx + 2, gxy = (nx + 2) * (ny + 2);
   const TU *up = u + p.off1;
   const int c = (li + 1) + gx * (lj + 1) + (DIM == 3 ? gxy * (lk + 1) : 0);
   const double uc = (double)up[c];
   const int sx = li + (nx + 1) * (lj + ny * lk);
   const int sy = li + nx * (lj + (ny + 1) * lk);
   const int sz = li + nx * (lj + ny * lk);
   // every face's loads are issued before any test of a mask: the plain
   // fluxes first, then the Ewing fix on coarse-fine faces, then the
   // coarsened finer-level fluxes over the faces that take them
   double fl[3][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
   double dd[3][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
   for (int a = 0; a < DIM; ++a) {
      const int st = a == 0 ? 1 : (a == 1 ? gx : gxy);
      const long long sbase = p.offs[a] + (a == 0 ? sx : (a == 1 ? sy : sz));
      const int sup = a == 0 ? 1 : (a == 1 ? nx : nx * ny);
#pragma unroll
      for (int s = 0; s < 2; ++s) {
         const long long si = sbase + (s ? sup : 0);
         const double d = DVAR ? dside[si] : dconst;
         const double ulo = s ? uc : (double)up[c - st];
         const double uhi = s ? (double)up[c + st] : uc;
         dd[a][s] = d;
         fl[a][s] = dai[a] * d * (uhi - ulo);
      }
   }
   if (has_cf) {
#pragma unroll
      for (int a = 0; a < DIM; ++a) {
         const int la = a == 0 ? li : (a == 1 ? lj : lk);
         const int na = a == 0 ? nx : (a == 1 ? ny : nz);
#pragma unroll
         for (int s = 0; s < 2; ++s) {
            if (!(s ? la == na - 1 : la == 0)) continue;
            const int i = p.lo[0] + li, j = p.lo[1] + lj;
            const int k = DIM == 3 ? p.lo[2] + lk : 0;
            if (cfmask[oidx(p, a, s, i, j, k)])
               fl[a][s] = ewing_face<DIM, TU>(p, u, a, s, i, j, k, fl[a][s], dd[a][s], w,
                                              ratio_to_coarser);
         }
      }
   }
   if (has_fc) {
#pragma unroll
      for (int a = 0; a < DIM; ++a) {
         const long long sbase = p.offs[a] + (a == 0 ? sx : (a == 1 ? sy : sz));
         const int sup = a == 0 ? 1 : (a == 1 ? nx : nx * ny);
#pragma unroll
         for (int s = 0; s < 2; ++s) {
            const long long si = sbase + (s ? sup : 0);
            if (fcmask[si]) fl[a][s] = fcflux[si];
         }
      }
   }
   const long long c0 = p.off0 + lin;
   const double sf = CKIND == 2 ? cfield[c0] : (CKIND == 1 ? cconst : 0.0);
   double rv;
   if (DIM == 2)
      rv = f[c0] - (dai[0] * (fl[0][1] - fl[0][0]) + dai[1] * (fl[1][1] - fl[1][0])) - sf * uc;
   else
      rv = f[c0] - (dai[0] * (fl[0][1] - fl[0][0]) + dai[1] * (fl[1][1] - fl[1][0]) +
                    dai[2] * (fl[2][1] - fl[2][0])) -
           sf * uc;
   res[c0] = rv;
   if (oflux) {
      const int i = p.lo[0] + li, j = p.lo[1] + lj, k = DIM == 3 ? p.lo[2] + lk : 0;
      if (li == 0) oflux[oidx(p, 0, 0, i, j, k)] = fl[0][0];
      if (li == nx - 1) oflux[oidx(p, 0, 1, i, j, k)] = fl[0][1];
      if (lj == 0) oflux[oidx(p, 1, 0, i, j, k)] = fl[1][0];
      if (lj == ny - 1) oflux[oidx(p, 1, 1, i, j, k)] = fl[1][1];
      if (DIM == 3) {
         if (lk == 0) oflux[oidx(p, 2, 0, i, j, k)] = fl[2][0];
         if (lk == nz - 1) oflux[oidx(p, 2, 1, i, j, k)] = fl[2][1];
      }
   }
}

template <int DIM, bool DVAR, int CKIND, class TU>
__global__ void __launch_bounds__(kThreads, 4)
k_residual_fused(const PatchDesc *__restrict__ patches, const Chunk *__restrict__ chunks,
                 int nwork, const TU *__restrict__ u, const double *__restrict__ dside,
                 double dconst, const unsigned char *__restrict__ cfmask, EwingWeights w,
                 const int *ratio_to_coarser, const unsigned char *__restrict__ fcmask,
                 const double *__restrict__ fcflux, const double *__restrict__ f,
                 const double *__restrict__ cfield, double cconst, double *__restrict__ res,
                 double *__restrict__ oflux, const int *__restrict__ run)
{
   WORK_LOOP(ch) {
      const PatchDesc &p = patches[ch.patch];
      if (run && !run[p.prob]) continue;
      const int nx = p.hi[0] - p.lo[0] + 1;
      const int ny = p.hi[1] - p.lo[1] + 1;
      const double dai[3] = {1. / p.dx[0], 1. / p.dx[1], DIM == 3 ? 1. / p.dx[2] : 0.0};
      for (int t = threadIdx.x; t < ch.count; t += blockDim.x) {
         const int lin = ch.begin + t;
         int li, lj, lk;
         patch_cell(p, lin, nx, ny, li, lj, lk);
         residual_cell<DIM, DVAR, CKIND, TU>(p, lin, li, lj, lk, dai, u, dside, dconst, cfmask, w,
                                             ratio_to_coarser, fcmask, fcflux, f, cfield, cconst,
                                             res, oflux);
      }
   }
}

// The fix-up after the staged residual: the listed cells (those with a
// coarse-fine face or a face under a finer patch) as k_residual_fused
// forms them, over the values the staged pass wrote.
template <int DIM, bool DVAR, int CKIND, class TU>
__global__ void __launch_bounds__(kThreads)
k_residual_cells(const CellRef *__restrict__ cells, int ncells,
                 const PatchDesc *__restrict__ patches, const TU *__restrict__ u,
                 const double *__restrict__ dside, double dconst,
                 const unsigned char *__restrict__ cfmask, EwingWeights w,
                 const int *ratio_to_coarser, const unsigned char *__restrict__ fcmask,
                 const double *__restrict__ fcflux, const double *__restrict__ f,
                 const double *__restrict__ cfield, double cconst, double *__restrict__ res,
                 double *__restrict__ oflux, const int *__restrict__ run)
{
   const int e = blockIdx.x * blockDim.x + threadIdx.x;
   if (e >= ncells) return;
   const CellRef cr = cells[e];
   const PatchDesc &p = patches[cr.patch];
   if (run && !run[p.prob]) return;
   const int nx = p.hi[0] - p.lo[0] + 1;
   const int ny = p.hi[1] - p.lo[1] + 1;
   int li, lj, lk;
   patch_cell(p, cr.lin, nx, ny, li, lj, lk);
   const double dai[3] = {1. / p.dx[0], 1. / p.dx[1], DIM == 3 ? 1. / p.dx[2] : 0.0};
   residual_cell<DIM, DVAR, CKIND, TU>(p, cr.lin, li, lj, lk, dai, u, dside, dconst, cfmask, w,
                                       ratio_to_coarser, fcmask, fcflux, f, cfield, cconst, res,
                                       oflux);
}

// ---------------------------------------------------------------------------
// flux coarsening (cartwgtavgoutsidedoub*, OutersideData::copy2)
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(kThreads)
k_flux_coarsen(const FluxCoarsenItem *__restrict__ items, const Chunk *__restrict__ chunks, int nwork,
               const int *__restrict__ prefix, const PatchDesc *__restrict__ fine,
               const PatchDesc *__restrict__ coarse, const double *__restrict__ oflux_fine,
               double *__restrict__ flux_coarse, const int *__restrict__ run)
{
   WORK_LOOP(ch) {
      for (int t = threadIdx.x; t < ch.count; t += blockDim.x) {
         int lin;
         const FluxCoarsenItem &it = items[chunk_item(ch, prefix, t, lin)];
         if (run && !run[it.prob]) continue;
         const PatchDesc &fp = fine[it.fine_patch];
         const PatchDesc &cp = coarse[it.coarse_patch];
         const int a = it.axis;
         const int nx = it.hi[0] - it.lo[0] + 1;
         const int ny = it.hi[1] - it.lo[1] + 1;
         double wf, wc;
         if (it.t1 < 0) {
            wf = fp.dx[it.t0];
            wc = cp.dx[it.t0];
         } else {
            wf = fp.dx[it.t0] * fp.dx[it.t1];
            wc = cp.dx[it.t0] * cp.dx[it.t1];
         }
         // refinement ratios along the tangential axes
         const int r0 = it.ratio & 0xff;
         const int r1 = (it.ratio >> 8) & 0xff;
         int c[3];
         c[0] = it.lo[0] + lin % nx;
         const int rr = lin / nx;
         c[1] = it.lo[1] + rr % ny;
         c[2] = it.lo[2] + rr / ny;
         double acc = 0.0;
         if (it.t1 < 0) {
            for (int ir = 0; ir < r0; ++ir) {
               int fc[3] = {0, 0, 0};
               fc[a] = it.fface;
               fc[it.t0] = c[it.t0] * r0 + ir;
               int cc[3] = {fc[0], fc[1], fc[2]};
               if (it.side == 1) cc[a] -= 1;
               acc = acc + oflux_fine[oidx(fp, a, it.side, cc[0], cc[1], cc[2])] * wf;
            }
         } else {
            for (int ro = 0; ro < r1; ++ro)
               for (int ri = 0; ri < r0; ++ri) {
                  int fc[3];
                  fc[a] = it.fface;
                  fc[it.t0] = c[it.t0] * r0 + ri;
                  fc[it.t1] = c[it.t1] * r1 + ro;
                  int cc[3] = {fc[0], fc[1], fc[2]};
                  if (it.side == 1) cc[a] -= 1;
                  acc = acc + oflux_fine[oidx(fp, a, it.side, cc[0], cc[1], cc[2])] * wf;
               }
         }
         acc = acc / wc;
         flux_coarse[sidx(cp, a, c[0], c[1], c[2])] = acc;
      }
   }
}

// ---------------------------------------------------------------------------
// restriction (cartwgtavgcelldoub{2,3}d)
// ---------------------------------------------------------------------------

template <int DIM>
__global__ void __launch_bounds__(kThreads)
k_restrict(const RestrictItem *__restrict__ items, const Chunk *__restrict__ chunks, int nwork,
           const int *__restrict__ prefix, const PatchDesc *__restrict__ fine,
           const PatchDesc *__restrict__ coarse, const double *__restrict__ src, int src_g,
           double *__restrict__ dst, int dst_g, const int *__restrict__ run)
{
   WORK_LOOP(ch) {
      for (int t = threadIdx.x; t < ch.count; t += blockDim.x) {
         int lin;
         const RestrictItem &it = items[chunk_item(ch, prefix, t, lin)];
         if (run && !run[it.prob]) continue;
         const PatchDesc &fp = fine[it.fine_patch];
         const PatchDesc &cp = coarse[it.coarse_patch];
         const int nx = it.hi[0] - it.lo[0] + 1;
         const int ny = it.hi[1] - it.lo[1] + 1;
         const int r0 = it.ratio & 0xff, r1 = (it.ratio >> 8) & 0xff,
                   r2 = (it.ratio >> 16) & 0xff;
         double dVf, dVc;
         if (DIM == 2) {
            dVf = fp.dx[0] * fp.dx[1];
            dVc = cp.dx[0] * cp.dx[1];
         } else {
            dVf = fp.dx[0] * fp.dx[1] * fp.dx[2];
            dVc = cp.dx[0] * cp.dx[1] * cp.dx[2];
         }
         const long long soff = src_g ? fp.off1 : fp.off0;
         const long long doff = dst_g ? cp.off1 : cp.off0;
         const int i = it.lo[0] + lin % nx;
         const int rr = lin / nx;
         const int j = it.lo[1] + rr % ny;
         const int k = it.lo[2] + rr / ny;
         double acc = 0.0;
         if (r0 == 2 && r1 == 2 && (DIM == 2 || r2 == 2)) {
            // ratio 2: all fine values loaded first, summed in the loop order
            // below (i2 outer, i1, i0 inner)
            constexpr int NF = DIM == 3 ? 8 : 4;
            const long long b = cidx<DIM>(fp, soff, src_g, 2 * i, 2 * j, DIM == 3 ? 2 * k : 0);
            const long long sy = fp.hi[0] - fp.lo[0] + 1 + 2 * src_g;
            const long long sz = sy * (fp.hi[1] - fp.lo[1] + 1 + 2 * src_g);
            double v[NF];
#pragma unroll
            for (int q = 0; q < NF; ++q)
               v[q] = src[b + (q & 1) + ((q >> 1) & 1) * sy + (q >> 2) * sz];
#pragma unroll
            for (int q = 0; q < NF; ++q) acc = acc + v[q] * dVf;
         } else {
            const int nr2 = DIM == 3 ? r2 : 1;
            for (int i2 = 0; i2 < nr2; ++i2)
               for (int i1 = 0; i1 < r1; ++i1)
                  for (int i0 = 0; i0 < r0; ++i0) {
                     const int fk = DIM == 3 ? k * r2 + i2 : 0;
                     acc = acc +
                           src[cidx<DIM>(fp, soff, src_g, i * r0 + i0, j * r1 + i1, fk)] * dVf;
                  }
         }
         acc = acc / dVc;
         dst[cidx<DIM>(cp, doff, dst_g, i, j, k)] = acc;
      }
   }
}

// ---------------------------------------------------------------------------
// linear refine of the coarse interpolation array + correction
// (cartlinrefcelldoub{2,3}d, HierarchyCellDataOpsReal::add)
// ---------------------------------------------------------------------------

template <int DIM, class T>
__global__ void __launch_bounds__(kThreads)
k_prolong_add(const ProlongItem *__restrict__ items, const Chunk *__restrict__ chunks, int nwork,
              const int *__restrict__ prefix, const PatchDesc *__restrict__ fine,
              const T *__restrict__ tmp, const double *__restrict__ dxc_prob, int ratio0,
              int ratio1, int ratio2, T *__restrict__ e, const int *__restrict__ run)
{
   const T half = (T)0.5, one = (T)1;
   const int r[3] = {ratio0, ratio1, ratio2};
   // per axis and fine offset ir within the coarse cell: the interpolation
   // weight x and the shift of the lower coarse cell (0 or -1).  They
   // depend on the problem only (all patches of a problem on a level share
   // dx), and a chunk holds one problem's cells.
   __shared__ T s_x[3][kProlongRatioMax];
   __shared__ int s_sh[3][kProlongRatioMax];
   WORK_LOOP(ch) {
      const int prob = items[ch.patch].prob;
      if (run && !run[prob]) continue;
      __syncthreads();  // the previous chunk's table is no longer read
      if ((int)threadIdx.x < DIM * kProlongRatioMax) {
         const int a = threadIdx.x / kProlongRatioMax, ir = threadIdx.x % kProlongRatioMax;
         if (ir < r[a]) {
            const double *dxc = dxc_prob + 3 * prob;
            const PatchDesc &p0 = fine[items[ch.patch].fine_patch];
            const T deltax = ((T)ir + half) * (T)p0.dx[a] - (T)dxc[a] * half;
            T x = deltax / (T)dxc[a];
            int sh = 0;
            if (x < 0.0) {
               sh = -1;
               x = x + one;
            }
            s_x[a][ir] = x;
            s_sh[a][ir] = sh;
         }
      }
      __syncthreads();
      for (int t = threadIdx.x; t < ch.count; t += blockDim.x) {
         int lin;
         const ProlongItem &it = items[chunk_item(ch, prefix, t, lin)];
         const PatchDesc &p = fine[it.fine_patch];
         const int nx = p.hi[0] - p.lo[0] + 1;
         const int ny = p.hi[1] - p.lo[1] + 1;
         int ci, cj, ck;
         patch_cell(p, lin, nx, ny, ci, cj, ck);
         const int fi[3] = {p.lo[0] + ci, p.lo[1] + cj, DIM == 3 ? p.lo[2] + ck : 0};
         int ic[3] = {0, 0, 0};
         T x[3];
#pragma unroll
         for (int a = 0; a < DIM; ++a) {
            const int c0 = coarsen_index(fi[a], r[a]);
            const int ir = fi[a] - c0 * r[a];
            x[a] = s_x[a][ir];
            ic[a] = c0 + s_sh[a][ir];
         }
         const ArrDesc &A = it.tmp;
         const long long b = aidx(A, ic[0], ic[1], ic[2]);
         const int sy = A.n[0];
         T v;
         if (DIM == 2) {
            const T c00 = tmp[b];
            const T c10 = tmp[b + 1];
            const T c01 = tmp[b + sy];
            const T c11 = tmp[b + sy + 1];
            v = (c00 + (c10 - c00) * x[0]) * (one - x[1]) + (c01 + (c11 - c01) * x[0]) * x[1];
         } else {
            const int sz = A.n[0] * A.n[1];
            const T c000 = tmp[b];
            const T c100 = tmp[b + 1];
            const T c010 = tmp[b + sy];
            const T c110 = tmp[b + sy + 1];
            const T c001 = tmp[b + sz];
            const T c101 = tmp[b + sz + 1];
            const T c011 = tmp[b + sz + sy];
            const T c111 = tmp[b + sz + sy + 1];
            const T y = x[1], z = x[2], xx = x[0];
            v = ((c000 + (c100 - c000) * xx) * (one - y) + (c010 + (c110 - c010) * xx) * y) *
                   (one - z) +
                ((c001 + (c101 - c001) * xx) * (one - y) + (c011 + (c111 - c011) * xx) * y) * z;
         }
         const long long c = cidx<DIM>(p, p.off1, 1, fi[0], fi[1], fi[2]);
         e[c] = e[c] + v;
      }
   }
}

// k_prolong_add for ratio 2 on every axis: one thread per coarse cell of a
// fine patch (fine patches are whole coarse cells), which loads the 3^DIM
// values of the interpolation array around it once and updates its 2^DIM
// fine cells.  Each fine cell takes the same corner values and weights as
// in k_prolong_add (lower corner at the coarse cell plus the tabulated
// shift, -1 for the lower fine cell and 0 for the upper one), so the same
// bits; the loads are the union of those the fine cells read.
template <int DIM, class T>
__global__ void __launch_bounds__(kThreads)
k_prolong_add_r2(const ProlongItem *__restrict__ items, const Chunk *__restrict__ chunks,
                 int nwork, const int *__restrict__ prefix, const PatchDesc *__restrict__ fine,
                 const T *__restrict__ tmp, const double *__restrict__ dxc_prob,
                 T *__restrict__ e, const int *__restrict__ run)
{
   const T half = (T)0.5, one = (T)1;
   __shared__ T s_x[3][2];
   __shared__ int s_sh[3][2];
   WORK_LOOP(ch) {
      const int prob = items[ch.patch].prob;
      if (run && !run[prob]) continue;
      __syncthreads();  // the previous chunk's table is no longer read
      if ((int)threadIdx.x < DIM * 2) {
         const int a = threadIdx.x / 2, ir = threadIdx.x % 2;
         const double *dxc = dxc_prob + 3 * prob;
         const PatchDesc &p0 = fine[items[ch.patch].fine_patch];
         const T deltax = ((T)ir + half) * (T)p0.dx[a] - (T)dxc[a] * half;
         T x = deltax / (T)dxc[a];
         int sh = 0;
         if (x < 0.0) {
            sh = -1;
            x = x + one;
         }
         s_x[a][ir] = x;
         s_sh[a][ir] = sh;
      }
      __syncthreads();
      for (int t = threadIdx.x; t < ch.count; t += blockDim.x) {
         int lin;
         const ProlongItem &it = items[chunk_item(ch, prefix, t, lin)];
         const PatchDesc &p = fine[it.fine_patch];
         const int nxc = (p.hi[0] - p.lo[0] + 1) >> 1;
         const int nyc = (p.hi[1] - p.lo[1] + 1) >> 1;
         const int q = lin / nxc;
         int c0[3];
         c0[0] = coarsen_index(p.lo[0], 2) + (lin - q * nxc);
         c0[1] = coarsen_index(p.lo[1], 2) + (DIM == 3 ? q % nyc : q);
         c0[2] = DIM == 3 ? coarsen_index(p.lo[2], 2) + q / nyc : 0;
         const ArrDesc &A = it.tmp;
         const int sy = A.n[0];
         const long long sz = (long long)A.n[0] * A.n[1];
         const long long b = aidx(A, c0[0] - 1, c0[1] - 1, DIM == 3 ? c0[2] - 1 : 0);
         constexpr int NZ = DIM == 3 ? 3 : 1;
         T nb[NZ][3][3];
#pragma unroll
         for (int dz = 0; dz < NZ; ++dz)
#pragma unroll
            for (int dy = 0; dy < 3; ++dy)
#pragma unroll
               for (int dx = 0; dx < 3; ++dx) nb[dz][dy][dx] = tmp[b + dx + sy * dy + sz * dz];
#pragma unroll
         for (int iz = 0; iz < (DIM == 3 ? 2 : 1); ++iz)
#pragma unroll
            for (int iy = 0; iy < 2; ++iy)
#pragma unroll
               for (int ix = 0; ix < 2; ++ix) {
                  const int ox = 1 + s_sh[0][ix], oy = 1 + s_sh[1][iy];
                  const T xx = s_x[0][ix], y = s_x[1][iy];
                  T v;
                  if (DIM == 2) {
                     const T c00 = nb[0][oy][ox], c10 = nb[0][oy][ox + 1];
                     const T c01 = nb[0][oy + 1][ox], c11 = nb[0][oy + 1][ox + 1];
                     v = (c00 + (c10 - c00) * xx) * (one - y) + (c01 + (c11 - c01) * xx) * y;
                  } else {
                     const int oz = 1 + s_sh[2][iz];
                     const T z = s_x[2][iz];
                     const T c000 = nb[oz][oy][ox], c100 = nb[oz][oy][ox + 1];
                     const T c010 = nb[oz][oy + 1][ox], c110 = nb[oz][oy + 1][ox + 1];
                     const T c001 = nb[oz + 1][oy][ox], c101 = nb[oz + 1][oy][ox + 1];
                     const T c011 = nb[oz + 1][oy + 1][ox], c111 = nb[oz + 1][oy + 1][ox + 1];
                     v = ((c000 + (c100 - c000) * xx) * (one - y) +
                          (c010 + (c110 - c010) * xx) * y) *
                            (one - z) +
                         ((c001 + (c101 - c001) * xx) * (one - y) +
                          (c011 + (c111 - c011) * xx) * y) *
                            z;
                  }
                  const long long c = cidx<DIM>(p, p.off1, 1, 2 * c0[0] + ix, 2 * c0[1] + iy,
                                                DIM == 3 ? 2 * c0[2] + iz : 0);
                  e[c] = e[c] + v;
               }
      }
   }
}

// ---------------------------------------------------------------------------
// interior cell helpers
// ---------------------------------------------------------------------------

template <int DIM, class T>
__global__ void __launch_bounds__(kThreads)
k_add_interior(const PatchDesc *__restrict__ patches, const Chunk *__restrict__ chunks, int nwork,
               double *__restrict__ u, const T *__restrict__ e,
               const int *__restrict__ run)
{
   WORK_LOOP(ch) {
      const PatchDesc p = patches[ch.patch];
      if (run && !run[p.prob]) continue;
      const int nx = p.hi[0] - p.lo[0] + 1;
      const int ny = p.hi[1] - p.lo[1] + 1;
      for (int t = threadIdx.x; t < ch.count; t += blockDim.x) {
         const int lin = ch.begin + t;
         int ci, cj, ck;
         patch_cell(p, lin, nx, ny, ci, cj, ck);
         const int i = p.lo[0] + ci;
         const int j = p.lo[1] + cj;
         const int k = DIM == 3 ? p.lo[2] + ck : 0;
         const long long c = cidx<DIM>(p, p.off1, 1, i, j, k);
         u[c] = u[c] + (double)e[c];
      }
   }
}

// Weighted sums sum(w x^2), sum(w) per chunk.
template <int DIM>
__global__ void __launch_bounds__(kThreads)
k_norm_partial(const PatchDesc *__restrict__ patches, const Chunk *__restrict__ chunks, int nwork,
               const double *__restrict__ x, int xg, const double *__restrict__ w,
               double2 *__restrict__ partial)
{
   WORK_LOOP(ch) {
      const PatchDesc p = patches[ch.patch];
      const int nx = p.hi[0] - p.lo[0] + 1;
      const int ny = p.hi[1] - p.lo[1] + 1;
      const long long xoff = xg ? p.off1 : p.off0;
      double sd = 0.0, sv = 0.0;
      if (!xg) {
         // ghost-0 field: the same linear index as the weights
         for (int t = threadIdx.x; t < ch.count; t += blockDim.x) {
            const long long c = p.off0 + ch.begin + t;
            const double xv = x[c];
            const double wv = w[c];
            sd += xv * xv * wv;
            sv += wv;
         }
      } else {
         for (int t = threadIdx.x; t < ch.count; t += blockDim.x) {
            const int lin = ch.begin + t;
            int ci, cj, ck;
            patch_cell(p, lin, nx, ny, ci, cj, ck);
            const int i = p.lo[0] + ci;
            const int j = p.lo[1] + cj;
            const int k = DIM == 3 ? p.lo[2] + ck : 0;
            const double xv = x[cidx<DIM>(p, xoff, xg, i, j, k)];
            const double wv = w[p.off0 + lin];
            sd += xv * xv * wv;
            sv += wv;
         }
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
      if (threadIdx.x == 0) partial[ch.aux] = make_double2(rs[0], rv[0]);
      __syncthreads();  // shared memory is reused by the next chunk
   }
}

// Composite-vector reductions (SAMRAIVectorReal::dot and maxNorm with
// control volumes, SAMRAIVectorReal.C:821-960 over HierarchyCellDataOpsReal
// dot/maxNorm, HierarchyCellDataOpsReal.C:877-1036): MODE 0, per chunk the
// sum of w x y (and of w); MODE 1, the largest |x| over cells with w > 0.
// Interior cells of fields of any ghost width.
template <int DIM, int MODE>
__global__ void __launch_bounds__(kThreads)
k_vec_partial(const PatchDesc *__restrict__ patches, const Chunk *__restrict__ chunks, int nwork,
              const double *__restrict__ x, int xg, const double *__restrict__ y, int yg,
              const double *__restrict__ w, double2 *__restrict__ partial)
{
   WORK_LOOP(ch) {
      const PatchDesc p = patches[ch.patch];
      const int nx = p.hi[0] - p.lo[0] + 1;
      const int ny = p.hi[1] - p.lo[1] + 1;
      const long long xoff = xg ? p.off1 : p.off0, yoff = yg ? p.off1 : p.off0;
      double sd = 0.0, sv = 0.0;
      for (int t = threadIdx.x; t < ch.count; t += blockDim.x) {
         const int lin = ch.begin + t;
         int ci, cj, ck;
         patch_cell(p, lin, nx, ny, ci, cj, ck);
         const int i = p.lo[0] + ci;
         const int j = p.lo[1] + cj;
         const int k = DIM == 3 ? p.lo[2] + ck : 0;
         const double xv = x[cidx<DIM>(p, xoff, xg, i, j, k)];
         const double wv = w[p.off0 + lin];
         if (MODE == 0) {
            const double yv = y[cidx<DIM>(p, yoff, yg, i, j, k)];
            sd += xv * yv * wv;
            sv += wv;
         } else if (wv > 0.0) {
            sd = fmax(sd, fabs(xv));
         }
      }
      __shared__ double rs[kThreads], rv[kThreads];
      rs[threadIdx.x] = sd;
      rv[threadIdx.x] = sv;
      __syncthreads();
      for (int o = kThreads / 2; o > 0; o >>= 1) {
         if ((int)threadIdx.x < o) {
            rs[threadIdx.x] = MODE == 0 ? rs[threadIdx.x] + rs[threadIdx.x + o]
                                        : fmax(rs[threadIdx.x], rs[threadIdx.x + o]);
            rv[threadIdx.x] += rv[threadIdx.x + o];
         }
         __syncthreads();
      }
      if (threadIdx.x == 0) partial[ch.aux] = make_double2(rs[0], rv[0]);
      __syncthreads();
   }
}

// Per problem: the partials of its chunks in chunk order, added to (MODE 0)
// or maxed into (MODE 1) acc[prob]; levels in level order by the caller.
template <int MODE>
__global__ void k_vec_reduce(const double2 *__restrict__ partial,
                             const int *__restrict__ prob_chunk_begin, int nprob,
                             double2 *__restrict__ acc)
{
   const int pr = blockIdx.x;
   if (pr >= nprob) return;
   const int b = prob_chunk_begin[pr], e = prob_chunk_begin[pr + 1];
   __shared__ double rs[kThreads], rv[kThreads];
   double sd = 0.0, sv = 0.0;
   for (int c = b + threadIdx.x; c < e; c += blockDim.x) {
      sd = MODE == 0 ? sd + partial[c].x : fmax(sd, partial[c].x);
      sv += partial[c].y;
   }
   rs[threadIdx.x] = sd;
   rv[threadIdx.x] = sv;
   __syncthreads();
   for (int o = kThreads / 2; o > 0; o >>= 1) {
      if ((int)threadIdx.x < o) {
         rs[threadIdx.x] = MODE == 0 ? rs[threadIdx.x] + rs[threadIdx.x + o]
                                     : fmax(rs[threadIdx.x], rs[threadIdx.x + o]);
         rv[threadIdx.x] += rv[threadIdx.x + o];
      }
      __syncthreads();
   }
   if (threadIdx.x == 0) {
      double2 a = acc[pr];
      a.x = MODE == 0 ? a.x + rs[0] : fmax(a.x, rs[0]);
      a.y += rv[0];
      acc[pr] = a;
   }
}

// z = a[prob] x + b[prob] y on interior cells (SAMRAIVectorReal::linearSum,
// ArrayDataBasicOps: dst = alpha src1 + beta src2)
template <int DIM>
__global__ void __launch_bounds__(kThreads)
k_vec_lincomb(const PatchDesc *__restrict__ patches, const Chunk *__restrict__ chunks, int nwork,
              double *z, int zg, const double *x, int xg, const double *y, int yg,
              const double *__restrict__ a, const double *__restrict__ b)
{
   WORK_LOOP(ch) {
      const PatchDesc p = patches[ch.patch];
      const int nx = p.hi[0] - p.lo[0] + 1;
      const int ny = p.hi[1] - p.lo[1] + 1;
      const double ap = a[p.prob], bp = b[p.prob];
      for (int t = threadIdx.x; t < ch.count; t += blockDim.x) {
         const int lin = ch.begin + t;
         int ci, cj, ck;
         patch_cell(p, lin, nx, ny, ci, cj, ck);
         const int i = p.lo[0] + ci;
         const int j = p.lo[1] + cj;
         const int k = DIM == 3 ? p.lo[2] + ck : 0;
         const double xv = x[cidx<DIM>(p, xg ? p.off1 : p.off0, xg, i, j, k)];
         const double yv = y[cidx<DIM>(p, yg ? p.off1 : p.off0, yg, i, j, k)];
         z[cidx<DIM>(p, zg ? p.off1 : p.off0, zg, i, j, k)] = ap * xv + bp * yv;
      }
   }
}

// Per problem: sum the partials of its chunks (in chunk order) and add them
// to acc[prob] (levels are summed in level order by the caller).
__global__ void k_norm_reduce(const double2 *__restrict__ partial,
                              const int *__restrict__ prob_chunk_begin, int nprob,
                              double2 *__restrict__ acc)
{
   const int pr = blockIdx.x;
   if (pr >= nprob) return;
   const int b = prob_chunk_begin[pr], e = prob_chunk_begin[pr + 1];
   __shared__ double rs[kThreads], rv[kThreads];
   double sd = 0.0, sv = 0.0;
   for (int c = b + threadIdx.x; c < e; c += blockDim.x) {
      sd += partial[c].x;
      sv += partial[c].y;
   }
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
   if (threadIdx.x == 0) {
      acc[pr].x += rs[0];
      acc[pr].y += rv[0];
   }
}

// Convergence test of one red-black sweep per problem
// (CellPoissonFACOps.C:1496-1508 with the last patch's max residuals).
__global__ void k_sweep_check(const unsigned long long *__restrict__ red,
                              const unsigned long long *__restrict__ blk,
                              const int *__restrict__ last_patch, int nprob,
                              double tol, int *__restrict__ run,
                              long long *__restrict__ sweeps)
{
   const int pr = blockIdx.x * blockDim.x + threadIdx.x;
   if (pr >= nprob) return;
   if (!run[pr]) return;
   sweeps[pr] += 1;
   if (tol >= 0.0) {
      const int lp = last_patch[pr];
      const double r = __longlong_as_double((long long)red[lp]);
      const double b = __longlong_as_double((long long)blk[lp]);
      const double m = r > b ? r : b;
      run[pr] = m > tol ? 1 : 0;
   }
}

template <class S, class D>
__global__ void k_convert(const S *__restrict__ src, D *__restrict__ dst, long long n)
{
   const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (t < n) dst[t] = (D)src[t];
}

__global__ void k_accumulate(const long long *__restrict__ src, long long *__restrict__ dst,
                             int n)
{
   const int t = blockIdx.x * blockDim.x + threadIdx.x;
   if (t < n) dst[t] += src[t];
}

__global__ void k_gather(const long long *__restrict__ idx, long long n,
                         const double *__restrict__ src, double *__restrict__ dst)
{
   const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (t < n) dst[t] = src[idx[t]];
}

__global__ void k_scatter(const long long *__restrict__ idx, long long n,
                          const double *__restrict__ src, double *__restrict__ dst)
{
   const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (t < n) dst[idx[t]] = src[t];
}

// ---------------------------------------------------------------------------
// learned correction: per-patch samples in and out of the CNN's S^3 boxes
// ---------------------------------------------------------------------------

// interior of a ghost-0 field copied into the interior of a ghost-1 field
template <int DIM>
__global__ void __launch_bounds__(kThreads)
k_g0_to_g1(const PatchDesc *__restrict__ patches, const Chunk *__restrict__ chunks, int nwork,
           const double *__restrict__ src, double *__restrict__ dst)
{
   WORK_LOOP(ch) {
      const PatchDesc p = patches[ch.patch];
      const int nx = p.hi[0] - p.lo[0] + 1;
      const int ny = p.hi[1] - p.lo[1] + 1;
      for (int t = threadIdx.x; t < ch.count; t += blockDim.x) {
         const int lin = ch.begin + t;
         int ci, cj, ck;
         patch_cell(p, lin, nx, ny, ci, cj, ck);
         const int i = p.lo[0] + ci;
         const int j = p.lo[1] + cj;
         const int k = DIM == 3 ? p.lo[2] + ck : 0;
         dst[cidx<DIM>(p, p.off1, 1, i, j, k)] = src[cidx<DIM>(p, p.off0, 0, i, j, k)];
      }
   }
}

// RMS of a ghost-0 field over each patch's interior (one block per patch)
template <int DIM>
__global__ void k_patch_rms(const PatchDesc *__restrict__ patches, const double *__restrict__ x,
                            double *__restrict__ rms)
{
   const PatchDesc p = patches[blockIdx.x];
   const long long n = (long long)(p.hi[0] - p.lo[0] + 1) * (p.hi[1] - p.lo[1] + 1) *
                       (p.hi[2] - p.lo[2] + 1);
   double sum = 0.0;
   for (long long t = threadIdx.x; t < n; t += blockDim.x) {
      const double v = x[p.off0 + t];
      sum += v * v;
   }
   __shared__ double red[kThreads];
   red[threadIdx.x] = sum;
   __syncthreads();
   for (int o = kThreads / 2; o > 0; o >>= 1) {
      if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
      __syncthreads();
   }
   if (threadIdx.x == 0) rms[blockIdx.x] = n > 0 ? sqrt(red[0] / (double)n) : 0.0;
}

// sample p = ghosted box of patch p of a ghost-1 field, divided by scale[p],
// at offset (0,0,0) of an S^3 box (the patch interior starts at 1), zeros
// elsewhere; 2-D patches fill the middle z-plane
template <int DIM>
__global__ void k_gather_samples(const PatchDesc *__restrict__ patches,
                                 const double *__restrict__ x, const double *__restrict__ scale,
                                 float *__restrict__ out, int S)
{
   const int ip = blockIdx.y;
   const PatchDesc p = patches[ip];
   const long long S3 = (long long)S * S * S;
   const double sc = scale[ip];
   const double inv = sc > 0.0 ? 1.0 / sc : 0.0;
   const int gx = p.hi[0] - p.lo[0] + 3, gy = p.hi[1] - p.lo[1] + 3;
   const int gz = DIM == 3 ? p.hi[2] - p.lo[2] + 3 : 1;
   for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < S3;
        c += (long long)gridDim.x * blockDim.x) {
      const int sx = (int)(c % S), sy = (int)((c / S) % S), sz = (int)(c / ((long long)S * S));
      const int zz = DIM == 3 ? sz : sz - S / 2;
      float v = 0.f;
      if (sx < gx && sy < gy && zz >= 0 && zz < gz) {
         const long long idx = p.off1 + sx + (long long)gx * (sy + (long long)gy * zz);
         v = (float)(x[idx] * inv);
      }
      out[(long long)ip * S3 + c] = v;
   }
}

// interior cells of patch p of a ghost-1 field = y[p] * scale[p] * dx^2
template <int DIM>
__global__ void __launch_bounds__(kThreads)
k_scatter_samples(const PatchDesc *__restrict__ patches, const Chunk *__restrict__ chunks, int nwork,
                  const float *__restrict__ y, const double *__restrict__ scale, int S,
                  double *__restrict__ dst)
{
   WORK_LOOP(ch) {
      const PatchDesc p = patches[ch.patch];
      const int nx = p.hi[0] - p.lo[0] + 1;
      const int ny = p.hi[1] - p.lo[1] + 1;
      const long long S3 = (long long)S * S * S;
      const double f = scale[ch.patch] * p.dx[0] * p.dx[0];
      for (int t = threadIdx.x; t < ch.count; t += blockDim.x) {
         const int lin = ch.begin + t;
         const int a = lin % nx;
         const int r = lin / nx;
         const int b = r % ny;
         const int cz = DIM == 3 ? r / ny : 0;
         const int sz = DIM == 3 ? cz + 1 : S / 2;
         const long long sidx = (long long)ch.patch * S3 + (a + 1) + (long long)S * ((b + 1) + (long long)S * sz);
         dst[cidx<DIM>(p, p.off1, 1, p.lo[0] + a, p.lo[1] + b, DIM == 3 ? p.lo[2] + cz : 0)] =
            (double)y[sidx] * f;
      }
   }
}

// per chunk: sum w r d and sum w d d with d = r - r2 (ghost-0 fields)
template <int DIM>
__global__ void __launch_bounds__(kThreads)
k_dot_pair(const PatchDesc *__restrict__ patches, const Chunk *__restrict__ chunks, int nwork,
           const double *__restrict__ r, const double *__restrict__ r2,
           const double *__restrict__ w, double2 *__restrict__ partial)
{
   WORK_LOOP(ch) {
      const PatchDesc p = patches[ch.patch];
      double a = 0.0, b = 0.0;
      for (int t = threadIdx.x; t < ch.count; t += blockDim.x) {
         const long long c = p.off0 + ch.begin + t;
         const double d = r[c] - r2[c];
         a += w[c] * r[c] * d;
         b += w[c] * d * d;
      }
      __shared__ double ra[kThreads], rb[kThreads];
      ra[threadIdx.x] = a;
      rb[threadIdx.x] = b;
      __syncthreads();
      for (int o = kThreads / 2; o > 0; o >>= 1) {
         if ((int)threadIdx.x < o) {
            ra[threadIdx.x] += ra[threadIdx.x + o];
            rb[threadIdx.x] += rb[threadIdx.x + o];
         }
         __syncthreads();
      }
      if (threadIdx.x == 0) partial[ch.aux] = make_double2(ra[0], rb[0]);
      __syncthreads();  // shared memory is reused by the next chunk
   }
}

// minimal-residual step length per problem: alpha = <r, d> / <d, d>, kept
// at 0 when it would not lower the residual
__global__ void k_alpha(const double2 *__restrict__ acc, const int *__restrict__ active,
                        int nprob, double *__restrict__ alpha)
{
   const int pr = blockIdx.x * blockDim.x + threadIdx.x;
   if (pr >= nprob) return;
   const double a = acc[pr].x, b = acc[pr].y;
   alpha[pr] = (active[pr] && b > 0.0 && a > 0.0) ? a / b : 0.0;
}

// u += alpha e (interior) and r = r - alpha (r - r2)
template <int DIM>
__global__ void __launch_bounds__(kThreads)
k_apply_alpha(const PatchDesc *__restrict__ patches, const Chunk *__restrict__ chunks, int nwork,
              const double *__restrict__ alpha, double *__restrict__ u,
              const double *__restrict__ e, double *__restrict__ r,
              const double *__restrict__ r2)
{
   WORK_LOOP(ch) {
      const PatchDesc p = patches[ch.patch];
      const double al = alpha[p.prob];
      if (al == 0.0) continue;
      const int nx = p.hi[0] - p.lo[0] + 1;
      const int ny = p.hi[1] - p.lo[1] + 1;
      for (int t = threadIdx.x; t < ch.count; t += blockDim.x) {
         const int lin = ch.begin + t;
         int ci, cj, ck;
         patch_cell(p, lin, nx, ny, ci, cj, ck);
         const int i = p.lo[0] + ci;
         const int j = p.lo[1] + cj;
         const int k = DIM == 3 ? p.lo[2] + ck : 0;
         const long long c1 = cidx<DIM>(p, p.off1, 1, i, j, k);
         const long long c0 = p.off0 + lin;
         u[c1] = u[c1] + al * e[c1];
         r[c0] = r[c0] - al * (r[c0] - r2[c0]);
      }
   }
}

// Block (list, problem): copy the problem's chunks of one work list to their
// place in the compacted list when the problem is active; the block of the
// last problem also writes the end markers.
__global__ void __launch_bounds__(kThreads)
k_compact(const WorkReg *__restrict__ regs, const int *__restrict__ active, int nprob)
{
   const WorkReg r = regs[blockIdx.x];
   const int p = blockIdx.y;
   int before = 0;
   for (int q = threadIdx.x; q < p; q += blockDim.x)
      if (active[q]) before += r.pcb[q + 1] - r.pcb[q];
   __shared__ int part[kThreads / 32];
   for (int o = 16; o > 0; o >>= 1) before += __shfl_down_sync(0xffffffffu, before, o);
   if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = before;
   __syncthreads();
   int pos = 0;
   for (int w = 0; w < kThreads / 32; ++w) pos += part[w];
   const int b = r.pcb[p], n = r.pcb[p + 1] - b;
   const bool on = active[p] != 0;
   if (on)
      for (int t = threadIdx.x; t < n; t += blockDim.x) r.list[pos + t] = r.all[b + t];
   if (p == nprob - 1) {
      const int total = pos + (on ? n : 0);
      for (int t = total + threadIdx.x; t < r.n; t += blockDim.x) r.list[t] = Chunk{-1, 0, 0, 0};
   }
}

// ---------------------------------------------------------------------------
// Krylov vector operations on composite vectors (ghost-0 cell arrays of a
// level, one vector every vstride elements), per problem, deterministic
// ---------------------------------------------------------------------------

// Vectors a multi-dot or combination takes per pass over the cells: their
// loads are independent, so a thread keeps that many in flight.
constexpr int kVecBlock = 8;

// partial[chunk * K + i] = sum over the chunk of w x V_i, chunks being runs
// of one problem's cells {problem, first cell, cells, chunk index}: one pass
// over the cells reads w and x once per kVecBlock vectors; each sum
// accumulates thread-strided cells, then a warp tree, then warps in order.
// With SELF, entry K is <x, x>: x taken as one more vector after the K.
template <bool SELF>
__global__ void __launch_bounds__(kThreads)
k_multidot(const Chunk *__restrict__ chunks, int nwork, const double *__restrict__ w,
           const double *__restrict__ x, const double *__restrict__ V, long long vstride, int K,
           double *__restrict__ partial)
{
   __shared__ double red[kVecBlock][kThreads / 32];
   const int KT = K + (SELF ? 1 : 0);
   WORK_LOOP(ch) {
      const long long c0 = ch.begin;
      for (int i0 = 0; i0 < KT; i0 += kVecBlock) {
         const int nb = KT - i0 < kVecBlock ? KT - i0 : kVecBlock;
         const double *vb = V + (long long)i0 * vstride;
         double sum[kVecBlock];
#pragma unroll
         for (int q = 0; q < kVecBlock; ++q) sum[q] = 0.0;
         for (int t = threadIdx.x; t < ch.count; t += blockDim.x) {
            const long long c = c0 + t;
            const double xc = x[c];
            const double wx = w[c] * xc;
            double v[kVecBlock];
#pragma unroll
            for (int q = 0; q < kVecBlock; ++q)
               v[q] = i0 + q < K ? vb[(long long)q * vstride + c]
                                 : (SELF && i0 + q == K ? xc : 0.0);
#pragma unroll
            for (int q = 0; q < kVecBlock; ++q) sum[q] += wx * v[q];
         }
#pragma unroll
         for (int q = 0; q < kVecBlock; ++q) {
            double b = sum[q];
            for (int o = 16; o > 0; o >>= 1) b += __shfl_down_sync(0xffffffffu, b, o);
            if ((threadIdx.x & 31) == 0) red[q][threadIdx.x >> 5] = b;
         }
         __syncthreads();
         if ((int)threadIdx.x < nb) {
            double b = 0.0;
            for (int r = 0; r < (int)(blockDim.x >> 5); ++r) b += red[threadIdx.x][r];
            partial[(long long)ch.aux * KT + i0 + threadIdx.x] = b;
         }
         __syncthreads();
      }
   }
}

// out[p * K + i] += sum of the problem's chunk partials, in chunk order
__global__ void k_multidot_reduce(const double *__restrict__ partial,
                                  const int *__restrict__ prob_chunk_begin, int K,
                                  const int *__restrict__ active, double *__restrict__ out)
{
   const int p = blockIdx.x, i = blockIdx.y;
   if (active && !active[p]) return;
   const int b = prob_chunk_begin[p], e = prob_chunk_begin[p + 1];
   __shared__ double red[kThreads];
   double sum = 0.0;
   for (int c = b + threadIdx.x; c < e; c += blockDim.x) sum += partial[(long long)c * K + i];
   red[threadIdx.x] = sum;
   __syncthreads();
   for (int o = kThreads / 2; o > 0; o >>= 1) {
      if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
      __syncthreads();
   }
   if (threadIdx.x == 0) out[(long long)p * K + i] += red[0];
}

// x = a[p] x + sum_i coef[p * K + i] V_i over the chunks of problem runs,
// summed in the order of i; the loads of kVecBlock vectors are issued ahead
// of their terms.  NORM: also partial[chunk] = sum over the chunk of w x x
// of the new x, accumulated exactly as k_multidot accumulates <x, x> (the
// same cells per thread in the same order, the same warp tree, warps in
// order), so the pass that would reread x for its norm is saved.
// The old x is read from xin (x itself when xin is null) and the new one
// is also written to x2 when that is not null, so a copy before or after
// the combination needs no pass of its own; xin and x2 may be the same
// array (each element is read before it is written, by the same thread).
template <bool NORM>
__global__ void __launch_bounds__(kThreads)
k_combine(const Chunk *__restrict__ chunks, int nwork, double *x, const double *xin,
          double *x2, const double *__restrict__ a, const double *__restrict__ V,
          long long vstride, int K, const double *__restrict__ coef,
          const double *__restrict__ w, double *__restrict__ partial)
{
   if (!xin) xin = x;
   __shared__ double red[NORM ? kThreads / 32 : 1];
   WORK_LOOP(ch) {
      const double ap = a[ch.patch];
      const double *cp = coef + (long long)ch.patch * K;
      // a problem's trailing zero coefficients add nothing: their vectors
      // are not read (a problem that needs no second Gram-Schmidt pass
      // reads only x)
      int Kp = K;
      while (Kp > 0 && cp[Kp - 1] == 0.0) --Kp;
      double sum = 0.0;
      // four cells of a thread at a time keep (K + 1) x 4 loads in flight
#pragma unroll 4
      for (int t = threadIdx.x; t < ch.count; t += blockDim.x) {
         const long long c = (long long)ch.begin + t;
         double v = ap * xin[c];
         for (int i0 = 0; i0 < Kp; i0 += kVecBlock) {
            const double *vb = V + (long long)i0 * vstride + c;
            double vv[kVecBlock];
#pragma unroll
            for (int q = 0; q < kVecBlock; ++q) vv[q] = i0 + q < Kp ? vb[(long long)q * vstride] : 0.0;
#pragma unroll
            for (int q = 0; q < kVecBlock; ++q)
               if (i0 + q < Kp) v = v + cp[i0 + q] * vv[q];
         }
         x[c] = v;
         if (x2) x2[c] = v;
         if (NORM) {
            const double wx = w[c] * v;
            sum += wx * v;
         }
      }
      if (NORM) {
         for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
         if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sum;
         __syncthreads();
         if (threadIdx.x == 0) {
            double b = 0.0;
            for (int r = 0; r < (int)(blockDim.x >> 5); ++r) b += red[r];
            partial[ch.aux] = b;
         }
         __syncthreads();
      }
   }
}

// x = a[p] xin + sum_i coef[p * K + i] V_i as k_combine (the same terms in
// the same order), and in the same pass partial[chunk * (K + 1) + i] = sum
// over the chunk of w x V_i of the new x, entry K being <x, x>: the
// multi-dot of the new vector against the vectors it was formed from,
// accumulated exactly as k_multidot<true> accumulates it (the same cells per
// thread in the same order, the same warp tree, warps in order), so the
// second Gram-Schmidt pass needs no multi-dot pass of its own.  The K vector
// values of a cell stay in registers between the combination and the
// products (K <= KB); the coefficients sit in shared memory.
template <int KB>
__global__ void __launch_bounds__(kThreads)
k_combine_dots(const Chunk *__restrict__ chunks, int nwork, double *x, const double *xin,
               const double *__restrict__ a, const double *__restrict__ V, long long vstride,
               int K, const double *__restrict__ coef, const double *__restrict__ w,
               double *__restrict__ partial)
{
   if (!xin) xin = x;
   __shared__ double red[KB + 1][kThreads / 32];
   __shared__ double scoef[KB];
   const int KT = K + 1;
   WORK_LOOP(ch) {
      if ((int)threadIdx.x < K) scoef[threadIdx.x] = coef[(long long)ch.patch * K + threadIdx.x];
      __syncthreads();
      const double ap = a[ch.patch];
      double sum[KB + 1];
#pragma unroll
      for (int q = 0; q <= KB; ++q) sum[q] = 0.0;
      // UNR cells of a thread per round, all their loads issued before the
      // first store (x may be xin, so a store would otherwise hold back the
      // next cell's loads); the sums still take the cells in the order t,
      // t + blockDim.x, ... of the one-cell loop
      constexpr int UNR = KB <= 8 ? 2 : 1;
      for (int t0 = threadIdx.x; t0 < ch.count; t0 += UNR * blockDim.x) {
         double vv[UNR][KB], xi[UNR], wv[UNR];
#pragma unroll
         for (int u = 0; u < UNR; ++u) {
            const int t = t0 + u * (int)blockDim.x;
            const long long c = (long long)ch.begin + t;
            const bool in = t < ch.count;
#pragma unroll
            for (int q = 0; q < KB; ++q)
               vv[u][q] = in && q < K ? V[(long long)q * vstride + c] : 0.0;
            xi[u] = in ? xin[c] : 0.0;
            wv[u] = in ? w[c] : 0.0;
         }
#pragma unroll
         for (int u = 0; u < UNR; ++u) {
            const int t = t0 + u * (int)blockDim.x;
            if (t >= ch.count) break;
            const long long c = (long long)ch.begin + t;
            double v = ap * xi[u];
#pragma unroll
            for (int q = 0; q < KB; ++q)
               if (q < K) v = v + scoef[q] * vv[u][q];
            x[c] = v;
            const double wx = wv[u] * v;
#pragma unroll
            for (int q = 0; q < KB; ++q)
               if (q < K) sum[q] += wx * vv[u][q];
            sum[KB] += wx * v;
         }
      }
#pragma unroll
      for (int q = 0; q <= KB; ++q) {
         if (q < K || q == KB) {
            double b = sum[q];
            for (int o = 16; o > 0; o >>= 1) b += __shfl_down_sync(0xffffffffu, b, o);
            if ((threadIdx.x & 31) == 0) red[q][threadIdx.x >> 5] = b;
         }
      }
      __syncthreads();
      if ((int)threadIdx.x < KT) {
         const int q = (int)threadIdx.x < K ? (int)threadIdx.x : KB;
         double b = 0.0;
         for (int r = 0; r < (int)(blockDim.x >> 5); ++r) b += red[q][r];
         partial[(long long)ch.aux * KT + threadIdx.x] = b;
      }
      __syncthreads();
   }
}

// dst (ghost-0, FP64) = src interior (ghost-1)
template <int DIM, class TS>
__global__ void __launch_bounds__(kThreads)
k_g1_to_g0(const PatchDesc *__restrict__ patches, const Chunk *__restrict__ chunks, int nwork,
           const TS *__restrict__ src, double *__restrict__ dst, int add,
           const double *__restrict__ scale, double *__restrict__ dst1)
{
   WORK_LOOP(ch) {
      const PatchDesc &p = patches[ch.patch];
      const int nx = p.hi[0] - p.lo[0] + 1;
      const int ny = p.hi[1] - p.lo[1] + 1;
      for (int t = threadIdx.x; t < ch.count; t += blockDim.x) {
         const int lin = ch.begin + t;
         int ci, cj, ck;
         patch_cell(p, lin, nx, ny, ci, cj, ck);
         const int i = p.lo[0] + ci;
         const int j = p.lo[1] + cj;
         const int k = DIM == 3 ? p.lo[2] + ck : 0;
         const long long c1 = cidx<DIM>(p, p.off1, 1, i, j, k);
         double v = (double)src[c1];
         if (scale) v = scale[p.prob] * v;
         dst[p.off0 + lin] = add ? dst[p.off0 + lin] + v : v;
         if (dst1) dst1[c1] = v;
      }
   }
}

// u interior (ghost-1) += sum_i y[p * K + i] Z_i (ghost-0)
template <int DIM>
__global__ void __launch_bounds__(kThreads)
k_add_combination(const PatchDesc *__restrict__ patches, const Chunk *__restrict__ chunks,
                  int nwork, double *__restrict__ u, const double *__restrict__ Z,
                  long long zstride, int K, const double *__restrict__ y)
{
   WORK_LOOP(ch) {
      const PatchDesc &p = patches[ch.patch];
      const int nx = p.hi[0] - p.lo[0] + 1;
      const int ny = p.hi[1] - p.lo[1] + 1;
      const double *yp = y + (long long)p.prob * K;
      for (int t = threadIdx.x; t < ch.count; t += blockDim.x) {
         const int lin = ch.begin + t;
         int ci, cj, ck;
         patch_cell(p, lin, nx, ny, ci, cj, ck);
         const int i = p.lo[0] + ci;
         const int j = p.lo[1] + cj;
         const int k = DIM == 3 ? p.lo[2] + ck : 0;
         const long long c0 = p.off0 + lin;
         double s = 0.0;
         for (int q0 = 0; q0 < K; q0 += kVecBlock) {
            const double *zb = Z + (long long)q0 * zstride + c0;
            double zz[kVecBlock];
#pragma unroll
            for (int q = 0; q < kVecBlock; ++q) zz[q] = q0 + q < K ? zb[(long long)q * zstride] : 0.0;
#pragma unroll
            for (int q = 0; q < kVecBlock; ++q)
               if (q0 + q < K) s = s + yp[q0 + q] * zz[q];
         }
         const long long c1 = cidx<DIM>(p, p.off1, 1, i, j, k);
         u[c1] = u[c1] + s;
      }
   }
}

std::atomic<long long> g_launches{0};

std::mutex g_occ_mutex;
std::unordered_map<const void *, int> g_occ;

}  // namespace

namespace dev {

int resident_blocks(const void *fn)
{
   std::lock_guard<std::mutex> lock(g_occ_mutex);
   const auto it = g_occ.find(fn);
   if (it != g_occ.end()) return it->second;
   int device = 0, nsm = 0, per_sm = 0;
   int cap = kGridCap;
   if (cudaGetDevice(&device) == cudaSuccess &&
       cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device) == cudaSuccess &&
       cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kThreads, 0) == cudaSuccess &&
       nsm > 0 && per_sm > 0)
      cap = nsm * per_sm;
   else
      (void)cudaGetLastError();  // the launch reports real faults
   g_occ[fn] = cap;
   return cap;
}

}  // namespace dev

long long kernel_launch_count() { return g_launches.load(); }

void add_kernel_launches(long long n) { g_launches += n; }

void launch_multidot(cudaStream_t s, int nchunks, const Chunk *chunks, const double *w,
                     const double *x, const double *V, long long vstride, int K,
                     double *partial, const int *prob_chunk_begin, int nprob, const int *active,
                     double *out, bool self_dot)
{
   const int KT = K + (self_dot ? 1 : 0);
   if (KT <= 0) return;
   if (nchunks > 0) {
      g_launches.fetch_add(1, std::memory_order_relaxed);
      if (self_dot)
         k_multidot<true><<<work_grid(k_multidot<true>, nchunks), kThreads, 0, s>>>(
            chunks, nchunks, w, x, V, vstride, K, partial);
      else
         k_multidot<false><<<work_grid(k_multidot<false>, nchunks), kThreads, 0, s>>>(
            chunks, nchunks, w, x, V, vstride, K, partial);
   }
   g_launches.fetch_add(1, std::memory_order_relaxed);
   k_multidot_reduce<<<dim3(nprob, KT), kThreads, 0, s>>>(partial, prob_chunk_begin, KT, active,
                                                          out);
}

void launch_combine(cudaStream_t s, int nchunks, const Chunk *chunks, double *x, const double *a,
                    const double *V, long long vstride, int K, const double *coef,
                    const double *xin, double *x2)
{
   if (nchunks <= 0) return;
   g_launches.fetch_add(1, std::memory_order_relaxed);
   k_combine<false><<<work_grid(k_combine<false>, nchunks), kThreads, 0, s>>>(
      chunks, nchunks, x, xin, x2, a, V, vstride, K, coef, nullptr, nullptr);
}

void launch_combine_norm(cudaStream_t s, int nchunks, const Chunk *chunks, double *x,
                         const double *a, const double *V, long long vstride, int K,
                         const double *coef, const double *w, double *partial,
                         const int *prob_chunk_begin, int nprob, const int *active, double *out,
                         const double *xin)
{
   if (nchunks > 0) {
      g_launches.fetch_add(1, std::memory_order_relaxed);
      k_combine<true><<<work_grid(k_combine<true>, nchunks), kThreads, 0, s>>>(
         chunks, nchunks, x, xin, nullptr, a, V, vstride, K, coef, w, partial);
   }
   g_launches.fetch_add(1, std::memory_order_relaxed);
   k_multidot_reduce<<<dim3(nprob, 1), kThreads, 0, s>>>(partial, prob_chunk_begin, 1, active,
                                                         out);
}

bool launch_combine_dots(cudaStream_t s, int nchunks, const Chunk *chunks, double *x,
                         const double *a, const double *V, long long vstride, int K,
                         const double *coef, const double *w, double *partial,
                         const int *prob_chunk_begin, int nprob, const int *active, double *out,
                         const double *xin)
{
   if (K < 1 || K > kCombineDotsMax) return false;
   if (nchunks > 0) {
      g_launches.fetch_add(1, std::memory_order_relaxed);
      if (K <= 8)
         k_combine_dots<8><<<work_grid(k_combine_dots<8>, nchunks), kThreads, 0, s>>>(
            chunks, nchunks, x, xin, a, V, vstride, K, coef, w, partial);
      else if (K <= 16)
         k_combine_dots<16><<<work_grid(k_combine_dots<16>, nchunks), kThreads, 0, s>>>(
            chunks, nchunks, x, xin, a, V, vstride, K, coef, w, partial);
      else
         k_combine_dots<kCombineDotsMax>
            <<<work_grid(k_combine_dots<kCombineDotsMax>, nchunks), kThreads, 0, s>>>(
               chunks, nchunks, x, xin, a, V, vstride, K, coef, w, partial);
   }
   g_launches.fetch_add(1, std::memory_order_relaxed);
   k_multidot_reduce<<<dim3(nprob, K + 1), kThreads, 0, s>>>(partial, prob_chunk_begin, K + 1,
                                                             active, out);
   return true;
}

template <class TS>
void launch_g1_to_g0(cudaStream_t s, int dim, int nchunks, const PatchDesc *patches,
                     const Chunk *chunks, const TS *src, double *dst, bool add,
                     const double *scale, double *dst1)
{
   if (nchunks <= 0) return;
   g_launches.fetch_add(1, std::memory_order_relaxed);
   if (dim == 2)
      k_g1_to_g0<2, TS><<<work_grid(k_g1_to_g0<2, TS>, nchunks), kThreads, 0, s>>>(
         patches, chunks, nchunks, src, dst, add ? 1 : 0, scale, dst1);
   else
      k_g1_to_g0<3, TS><<<work_grid(k_g1_to_g0<3, TS>, nchunks), kThreads, 0, s>>>(
         patches, chunks, nchunks, src, dst, add ? 1 : 0, scale, dst1);
}
template void launch_g1_to_g0<double>(cudaStream_t, int, int, const PatchDesc *, const Chunk *,
                                      const double *, double *, bool, const double *, double *);
template void launch_g1_to_g0<float>(cudaStream_t, int, int, const PatchDesc *, const Chunk *,
                                     const float *, double *, bool, const double *, double *);

void launch_add_combination(cudaStream_t s, int dim, int nchunks, const PatchDesc *patches,
                            const Chunk *chunks, double *u, const double *Z, long long zstride,
                            int K, const double *y)
{
   if (nchunks <= 0 || K <= 0) return;
   g_launches.fetch_add(1, std::memory_order_relaxed);
   if (dim == 2)
      k_add_combination<2><<<work_grid(k_add_combination<2>, nchunks), kThreads, 0, s>>>(patches, chunks, nchunks, u, Z,
                                                                    zstride, K, y);
   else
      k_add_combination<3><<<work_grid(k_add_combination<3>, nchunks), kThreads, 0, s>>>(patches, chunks, nchunks, u, Z,
                                                                    zstride, K, y);
}

void launch_compact(cudaStream_t s, const WorkReg *regs, int nregs, const int *active, int nprob)
{
   if (nregs <= 0 || nprob <= 0) return;
   g_launches.fetch_add(1, std::memory_order_relaxed);
   k_compact<<<dim3(nregs, nprob), kThreads, 0, s>>>(regs, active, nprob);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------

template <class T>
void launch_fill(cudaStream_t s, const FillItem *items, const Chunk *chunks, int nchunks,
                 const int *prefix, T *dst, const T *src_same, const T *src_coarse,
                 int homogeneous, const BcCoefs &bc, const int *active)
{
   if (nchunks <= 0) return;
   g_launches.fetch_add(1, std::memory_order_relaxed);
   k_fill<T><<<work_grid(k_fill<T>, nchunks), kThreads, 0, s>>>(items, chunks, nchunks, prefix, dst, src_same, src_coarse,
                                          homogeneous, bc, active);
}

bool allow_solve_smem(int bytes)
{
   bool ok = true;
   auto set = [&](auto kern) {
      ok = ok && cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      bytes) == cudaSuccess;
   };
   set(k_rbgs_solve_smem<2, false, 0, double>);
   set(k_rbgs_solve_smem<2, false, 1, double>);
   set(k_rbgs_solve_smem<2, false, 2, double>);
   set(k_rbgs_solve_smem<2, true, 0, double>);
   set(k_rbgs_solve_smem<2, true, 1, double>);
   set(k_rbgs_solve_smem<2, true, 2, double>);
   set(k_rbgs_solve_smem<3, false, 0, double>);
   set(k_rbgs_solve_smem<3, false, 1, double>);
   set(k_rbgs_solve_smem<3, false, 2, double>);
   set(k_rbgs_solve_smem<3, true, 0, double>);
   set(k_rbgs_solve_smem<3, true, 1, double>);
   set(k_rbgs_solve_smem<3, true, 2, double>);
   return ok;
}

template <class T>
void launch_rbgs_solve(cudaStream_t s, int dim, const PoissonSpec &spec, int npatch,
                       const PatchDesc *patches, T *u, const T *f, const T *dside,
                       const T *cfield, const long long *facemap, const BcCoefs &bc,
                       int nsweeps, double tol, int *run, long long *sweeps,
                       unsigned long long *maxres_red, unsigned long long *maxres_blk,
                       int smem)
{
   if (npatch <= 0 || nsweeps <= 0) return;
   g_launches.fetch_add(1, std::memory_order_relaxed);
   const T dc = (T)spec.d_const, cc = (T)spec.c_const;
#define RS(D, V, C)                                                                           \
   do {                                                                                       \
      if (smem > 0) {                                                                         \
         k_rbgs_solve_smem<D, V, C, T><<<npatch, kSolveSmemThreads, smem, s>>>(               \
            patches, u, f, dside, cfield, dc, cc, facemap, bc, nsweeps, tol, run, sweeps,     \
            maxres_red, maxres_blk);                                                          \
      } else {                                                                                \
         k_rbgs_solve<D, V, C, T><<<npatch, kThreads, 0, s>>>(patches, u, f, dside, cfield,   \
                                                              dc, cc, facemap, bc, nsweeps,   \
                                                              tol, run, sweeps, maxres_red,   \
                                                              maxres_blk);                    \
      }                                                                                       \
   } while (0)
   if (dim == 2) {
      if (spec.d_variable) {
         if (spec.c_kind == 2) RS(2, true, 2);
         else if (spec.c_kind == 1) RS(2, true, 1);
         else RS(2, true, 0);
      } else {
         if (spec.c_kind == 2) RS(2, false, 2);
         else if (spec.c_kind == 1) RS(2, false, 1);
         else RS(2, false, 0);
      }
   } else {
      if (spec.d_variable) {
         if (spec.c_kind == 2) RS(3, true, 2);
         else if (spec.c_kind == 1) RS(3, true, 1);
         else RS(3, true, 0);
      } else {
         if (spec.c_kind == 2) RS(3, false, 2);
         else if (spec.c_kind == 1) RS(3, false, 1);
         else RS(3, false, 0);
      }
   }
#undef RS
}

template <class T>
void launch_fill_gather(cudaStream_t s, long long n, const unsigned *to, const int *from,
                        const unsigned short *prob, const FillItem *bc_items,
                        const Chunk *bc_chunks, int nbc, const int *bc_prefix, T *dst,
                        const T *src_same, const T *src_coarse, int homogeneous,
                        const BcCoefs &bc, const int *active)
{
   const long long nblk = (n + kThreads * kFillPer - 1) / (kThreads * kFillPer);
   const int gbc = nbc > 0 ? work_grid(k_fill_gather<T>, nbc) : 0;
   if (nblk + gbc <= 0) return;
   if (nblk + gbc > (1ll << 31) - 1) throw std::runtime_error("fill gather list too long");
   g_launches.fetch_add(1, std::memory_order_relaxed);
   k_fill_gather<T><<<(unsigned)(nblk + gbc), kThreads, 0, s>>>(
      n, (int)nblk, to, from, prob, bc_items, bc_chunks, nbc, bc_prefix, dst, src_same,
      src_coarse, homogeneous, bc, active);
}

template <class T>
void launch_cf_flux(cudaStream_t s, const CfFace *faces, int nfaces, const PatchDesc *patches,
                    const T *u, const T *dside, int dvar, double dconst, const double *tranwt,
                    const double *longwt, T *cfflux, const int *run)
{
   if (nfaces <= 0) return;
   g_launches.fetch_add(1, std::memory_order_relaxed);
   EwingWeights w;
   for (int a = 0; a < 3; ++a) {
      w.tranwt[a] = tranwt[a];
      w.longwt[a] = longwt[a];
   }
   const int nb = (nfaces + kThreads - 1) / kThreads;
   k_cf_flux<T><<<nb, kThreads, 0, s>>>(faces, nfaces, patches, u, dside, dvar, (T)dconst, w,
                                        cfflux, run);
}

template <int DIM, bool DVAR, int CK, class T>
static void rbgs_inst(cudaStream_t s, int nchunks, const PatchDesc *patches,
                      const Chunk *chunks, T *u, const T *f, const T *dside, const T *cfield,
                      const T *cfflux, const unsigned char *cfmask, int offset, double dconst,
                      double cconst, unsigned long long *maxres, const int *run,
                      const long long *facemap, const BcCoefs &bc)
{
   if (facemap)
      k_rbgs<DIM, DVAR, CK, T, true><<<work_grid(k_rbgs<DIM, DVAR, CK, T, true>, nchunks), kThreads, 0, s>>>(
         patches, chunks, nchunks, u, f, dside, cfield, cfflux, cfmask, offset, (T)dconst, (T)cconst,
         maxres, run, facemap, bc);
   else
      k_rbgs<DIM, DVAR, CK, T, false><<<work_grid(k_rbgs<DIM, DVAR, CK, T, false>, nchunks), kThreads, 0, s>>>(
         patches, chunks, nchunks, u, f, dside, cfield, cfflux, cfmask, offset, (T)dconst, (T)cconst,
         maxres, run, facemap, bc);
}

template <class T>
void launch_rbgs(cudaStream_t s, int dim, const PoissonSpec &spec, int nchunks,
                 const PatchDesc *patches, const Chunk *chunks, T *u, const T *f,
                 const T *dside, const T *cfield, const T *cfflux,
                 const unsigned char *cfmask, int offset, unsigned long long *maxres,
                 const int *run, const long long *facemap, const BcCoefs &bc)
{
   if (nchunks <= 0) return;
   g_launches.fetch_add(1, std::memory_order_relaxed);
#define RB(D, V, C)                                                                        \
   rbgs_inst<D, V, C, T>(s, nchunks, patches, chunks, u, f, dside, cfield, cfflux, cfmask, \
                         offset, spec.d_const, spec.c_const, maxres, run, facemap, bc)
   if (dim == 2) {
      if (spec.d_variable) {
         if (spec.c_kind == 2) RB(2, true, 2);
         else if (spec.c_kind == 1) RB(2, true, 1);
         else RB(2, true, 0);
      } else {
         if (spec.c_kind == 2) RB(2, false, 2);
         else if (spec.c_kind == 1) RB(2, false, 1);
         else RB(2, false, 0);
      }
   } else {
      if (spec.d_variable) {
         if (spec.c_kind == 2) RB(3, true, 2);
         else if (spec.c_kind == 1) RB(3, true, 1);
         else RB(3, true, 0);
      } else {
         if (spec.c_kind == 2) RB(3, false, 2);
         else if (spec.c_kind == 1) RB(3, false, 1);
         else RB(3, false, 0);
      }
   }
#undef RB
}

template <class TU>
void launch_flux(cudaStream_t s, int dim, const PoissonSpec &spec, int nchunks,
                 const PatchDesc *patches, const Chunk *chunks, const TU *u,
                 const double *dside, const unsigned char *cfmask, const double *tranwt,
                 const double *longwt, const int *ratio_dev, double *flux, const int *run)
{
   if (nchunks <= 0) return;
   g_launches.fetch_add(1, std::memory_order_relaxed);
   EwingWeights w;
   for (int a = 0; a < 3; ++a) {
      w.tranwt[a] = tranwt[a];
      w.longwt[a] = longwt[a];
   }
   if (dim == 2) {
      if (spec.d_variable)
         k_flux<2, true, TU><<<work_grid(k_flux<2, true, TU>, nchunks), kThreads, 0, s>>>(patches, chunks, nchunks, u, dside,
                                                          spec.d_const, cfmask, w, ratio_dev,
                                                          flux, run);
      else
         k_flux<2, false, TU><<<work_grid(k_flux<2, false, TU>, nchunks), kThreads, 0, s>>>(patches, chunks, nchunks, u, dside,
                                                           spec.d_const, cfmask, w,
                                                           ratio_dev, flux, run);
   } else {
      if (spec.d_variable)
         k_flux<3, true, TU><<<work_grid(k_flux<3, true, TU>, nchunks), kThreads, 0, s>>>(patches, chunks, nchunks, u, dside,
                                                          spec.d_const, cfmask, w, ratio_dev,
                                                          flux, run);
      else
         k_flux<3, false, TU><<<work_grid(k_flux<3, false, TU>, nchunks), kThreads, 0, s>>>(patches, chunks, nchunks, u, dside,
                                                           spec.d_const, cfmask, w,
                                                           ratio_dev, flux, run);
   }
}

template <class TU>
void launch_flux_cells(cudaStream_t s, int dim, const PoissonSpec &spec, int nchunks,
                       const PatchDesc *patches, const Chunk *cell_chunks, const TU *u,
                       const double *dside, const unsigned char *cfmask, const double *tranwt,
                       const double *longwt, const int *ratio_dev, double *flux, const int *run)
{
   if (nchunks <= 0) return;
   g_launches.fetch_add(1, std::memory_order_relaxed);
   EwingWeights w;
   for (int a = 0; a < 3; ++a) {
      w.tranwt[a] = tranwt[a];
      w.longwt[a] = longwt[a];
   }
#define FC(D, V)                                                                            \
   k_flux_cells<D, V, TU><<<work_grid(k_flux_cells<D, V, TU>, nchunks), kThreads, 0, s>>>(                          \
      patches, cell_chunks, nchunks, u, dside, spec.d_const, cfmask, w, ratio_dev, flux, run)
   if (dim == 2) {
      if (spec.d_variable) FC(2, true);
      else FC(2, false);
   } else {
      if (spec.d_variable) FC(3, true);
      else FC(3, false);
   }
#undef FC
}

template <class TU>
void launch_ewing_fix(cudaStream_t s, const CfFace *faces, int nfaces, const PatchDesc *patches,
                      const TU *u, const double *dside, int dvar, double dconst,
                      const double *tranwt, const double *longwt, double *flux, const int *run)
{
   if (nfaces <= 0) return;
   g_launches.fetch_add(1, std::memory_order_relaxed);
   EwingWeights w;
   for (int a = 0; a < 3; ++a) {
      w.tranwt[a] = tranwt[a];
      w.longwt[a] = longwt[a];
   }
   k_ewing_fix<TU><<<(nfaces + kThreads - 1) / kThreads, kThreads, 0, s>>>(
      faces, nfaces, patches, u, dside, dvar, dconst, w, flux, run);
}

template <class TU>
void launch_residual_fused(cudaStream_t s, int dim, const PoissonSpec &spec, int nchunks,
                           const PatchDesc *patches, const Chunk *chunks, const TU *u,
                           const double *dside, const unsigned char *cfmask,
                           const double *tranwt, const double *longwt, const int *ratio_dev,
                           const unsigned char *fcmask, const double *fcflux, const double *f,
                           const double *cfield, double *res, double *oflux, const int *run)
{
   if (nchunks <= 0) return;
   g_launches.fetch_add(1, std::memory_order_relaxed);
   EwingWeights w;
   for (int a = 0; a < 3; ++a) {
      w.tranwt[a] = tranwt[a];
      w.longwt[a] = longwt[a];
   }
#define RF(D, V, C)                                                                         \
   k_residual_fused<D, V, C, TU><<<work_grid(k_residual_fused<D, V, C, TU>, nchunks), kThreads, 0, s>>>(                   \
      patches, chunks, nchunks, u, dside, spec.d_const, cfmask, w, ratio_dev, fcmask, fcflux, \
      f, cfield, spec.c_const, res, oflux, run)
   if (dim == 2) {
      if (spec.d_variable) {
         if (spec.c_kind == 2) RF(2, true, 2);
         else if (spec.c_kind == 1) RF(2, true, 1);
         else RF(2, true, 0);
      } else {
         if (spec.c_kind == 2) RF(2, false, 2);
         else if (spec.c_kind == 1) RF(2, false, 1);
         else RF(2, false, 0);
      }
   } else {
      if (spec.d_variable) {
         if (spec.c_kind == 2) RF(3, true, 2);
         else if (spec.c_kind == 1) RF(3, true, 1);
         else RF(3, true, 0);
      } else {
         if (spec.c_kind == 2) RF(3, false, 2);
         else if (spec.c_kind == 1) RF(3, false, 1);
         else RF(3, false, 0);
      }
   }
#undef RF
}

template <class TU>
void launch_residual_cells(cudaStream_t s, int dim, const PoissonSpec &spec, int ncells,
                           const CellRef *cells, const PatchDesc *patches, const TU *u,
                           const double *dside, const unsigned char *cfmask,
                           const double *tranwt, const double *longwt,
                           const int *ratio_to_coarser, const unsigned char *fcmask,
                           const double *fcflux, const double *f, const double *cfield,
                           double *res, double *oflux, const int *run)
{
   if (ncells <= 0) return;
   g_launches.fetch_add(1, std::memory_order_relaxed);
   EwingWeights w;
   for (int a = 0; a < 3; ++a) {
      w.tranwt[a] = tranwt[a];
      w.longwt[a] = longwt[a];
   }
   const int grid = (ncells + kThreads - 1) / kThreads;
#define RC(D, V, C)                                                                          \
   k_residual_cells<D, V, C, TU><<<grid, kThreads, 0, s>>>(                                   \
      cells, ncells, patches, u, dside, spec.d_const, cfmask, w, ratio_to_coarser, fcmask,    \
      fcflux, f, cfield, spec.c_const, res, oflux, run)
   if (dim == 2) {
      if (spec.d_variable) {
         if (spec.c_kind == 2) RC(2, true, 2);
         else if (spec.c_kind == 1) RC(2, true, 1);
         else RC(2, true, 0);
      } else {
         if (spec.c_kind == 2) RC(2, false, 2);
         else if (spec.c_kind == 1) RC(2, false, 1);
         else RC(2, false, 0);
      }
   } else {
      if (spec.d_variable) {
         if (spec.c_kind == 2) RC(3, true, 2);
         else if (spec.c_kind == 1) RC(3, true, 1);
         else RC(3, true, 0);
      } else {
         if (spec.c_kind == 2) RC(3, false, 2);
         else if (spec.c_kind == 1) RC(3, false, 1);
         else RC(3, false, 0);
      }
   }
#undef RC
}

template <class TU>
void launch_residual(cudaStream_t s, int dim, const PoissonSpec &spec, int nchunks,
                     const PatchDesc *patches, const Chunk *chunks, const TU *u,
                     const double *f, const double *flux, const double *cfield,
                     double *res, double *oflux, const int *run)
{
   if (nchunks <= 0) return;
   g_launches.fetch_add(1, std::memory_order_relaxed);
#define RS(D, C)                                                                         \
   k_residual<D, C, TU><<<work_grid(k_residual<D, C, TU>, nchunks), kThreads, 0, s>>>(patches, chunks, nchunks, u, f, flux, cfield, \
                                                     spec.c_const, res, oflux, run)
   if (dim == 2) {
      if (spec.c_kind == 2) RS(2, 2);
      else if (spec.c_kind == 1) RS(2, 1);
      else RS(2, 0);
   } else {
      if (spec.c_kind == 2) RS(3, 2);
      else if (spec.c_kind == 1) RS(3, 1);
      else RS(3, 0);
   }
#undef RS
}

void launch_flux_coarsen(cudaStream_t s, const FluxCoarsenItem *items, const Chunk *chunks,
                         int nchunks, const int *prefix, const PatchDesc *fine,
                         const PatchDesc *coarse, const double *oflux_fine, double *flux_coarse,
                         const int *run)
{
   if (nchunks <= 0) return;
   g_launches.fetch_add(1, std::memory_order_relaxed);
   k_flux_coarsen<<<work_grid(k_flux_coarsen, nchunks), kThreads, 0, s>>>(items, chunks, nchunks, prefix, fine,
                                                          coarse, oflux_fine, flux_coarse, run);
}

void launch_restrict(cudaStream_t s, int dim, const RestrictItem *items, const Chunk *chunks,
                     int nchunks, const int *prefix, const PatchDesc *fine,
                     const PatchDesc *coarse, const double *src, int src_g, double *dst,
                     int dst_g, const int *run)
{
   if (nchunks <= 0) return;
   g_launches.fetch_add(1, std::memory_order_relaxed);
   if (dim == 2)
      k_restrict<2><<<work_grid(k_restrict<2>, nchunks), kThreads, 0, s>>>(items, chunks, nchunks, prefix, fine,
                                                            coarse, src, src_g, dst, dst_g, run);
   else
      k_restrict<3><<<work_grid(k_restrict<3>, nchunks), kThreads, 0, s>>>(items, chunks, nchunks, prefix, fine,
                                                            coarse, src, src_g, dst, dst_g, run);
}

template <class T>
void launch_prolong_add(cudaStream_t s, int dim, const ProlongItem *items, const Chunk *chunks,
                        int nchunks, const int *prefix, const PatchDesc *fine, const T *tmp,
                        const double *dxc_prob, const int *ratio, T *e, const int *run)
{
   if (nchunks <= 0) return;
   g_launches.fetch_add(1, std::memory_order_relaxed);
   if (dim == 2)
      k_prolong_add<2, T><<<work_grid(k_prolong_add<2, T>, nchunks), kThreads, 0, s>>>(
         items, chunks, nchunks, prefix, fine, tmp, dxc_prob, ratio[0], ratio[1], ratio[2], e, run);
   else
      k_prolong_add<3, T><<<work_grid(k_prolong_add<3, T>, nchunks), kThreads, 0, s>>>(
         items, chunks, nchunks, prefix, fine, tmp, dxc_prob, ratio[0], ratio[1], ratio[2], e, run);
}

template <class T>
void launch_prolong_add_r2(cudaStream_t s, int dim, const ProlongItem *items,
                           const Chunk *chunks, int nchunks, const int *prefix,
                           const PatchDesc *fine, const T *tmp, const double *dxc_prob, T *e,
                           const int *run)
{
   if (nchunks <= 0) return;
   g_launches.fetch_add(1, std::memory_order_relaxed);
   if (dim == 2)
      k_prolong_add_r2<2, T><<<work_grid(k_prolong_add_r2<2, T>, nchunks), kThreads, 0, s>>>(
         items, chunks, nchunks, prefix, fine, tmp, dxc_prob, e, run);
   else
      k_prolong_add_r2<3, T><<<work_grid(k_prolong_add_r2<3, T>, nchunks), kThreads, 0, s>>>(
         items, chunks, nchunks, prefix, fine, tmp, dxc_prob, e, run);
}

template <class T>
void launch_add_interior(cudaStream_t s, int dim, int nchunks, const PatchDesc *patches,
                         const Chunk *chunks, double *u, const T *e, const int *run)
{
   if (nchunks <= 0) return;
   g_launches.fetch_add(1, std::memory_order_relaxed);
   if (dim == 2)
      k_add_interior<2, T><<<work_grid(k_add_interior<2, T>, nchunks), kThreads, 0, s>>>(patches, chunks, nchunks, u, e, run);
   else
      k_add_interior<3, T><<<work_grid(k_add_interior<3, T>, nchunks), kThreads, 0, s>>>(patches, chunks, nchunks, u, e, run);
}

template <class S, class D>
void launch_convert(cudaStream_t s, const S *src, D *dst, long long n)
{
   if (n <= 0) return;
   g_launches.fetch_add(1, std::memory_order_relaxed);
   k_convert<S, D><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(src, dst, n);
}

void launch_norm(cudaStream_t s, int dim, int nchunks, const PatchDesc *patches,
                 const Chunk *chunks, const double *x, int xg, const double *w,
                 double2 *partial, const int *prob_chunk_begin, int nprob, double2 *acc)
{
   if (nchunks <= 0) return;
   g_launches.fetch_add(2, std::memory_order_relaxed);
   if (dim == 2)
      k_norm_partial<2><<<work_grid(k_norm_partial<2>, nchunks), kThreads, 0, s>>>(patches, chunks, nchunks, x, xg, w, partial);
   else
      k_norm_partial<3><<<work_grid(k_norm_partial<3>, nchunks), kThreads, 0, s>>>(patches, chunks, nchunks, x, xg, w, partial);
   k_norm_reduce<<<nprob, kThreads, 0, s>>>(partial, prob_chunk_begin, nprob, acc);
}

void launch_vec_reduce(cudaStream_t s, int dim, int mode, int nchunks, const PatchDesc *patches,
                       const Chunk *chunks, const double *x, int xg, const double *y, int yg,
                       const double *w, double2 *partial, const int *prob_chunk_begin,
                       int nprob, double2 *acc)
{
   if (nchunks <= 0) return;
   g_launches.fetch_add(2, std::memory_order_relaxed);
#define VP(D, M)                                                                          \
   k_vec_partial<D, M><<<work_grid(k_vec_partial<D, M>, nchunks), kThreads, 0, s>>>(       \
      patches, chunks, nchunks, x, xg, y, yg, w, partial)
   if (dim == 2) {
      if (mode == 0) VP(2, 0);
      else VP(2, 1);
   } else {
      if (mode == 0) VP(3, 0);
      else VP(3, 1);
   }
#undef VP
   if (mode == 0) k_vec_reduce<0><<<nprob, kThreads, 0, s>>>(partial, prob_chunk_begin, nprob, acc);
   else k_vec_reduce<1><<<nprob, kThreads, 0, s>>>(partial, prob_chunk_begin, nprob, acc);
}

void launch_vec_lincomb(cudaStream_t s, int dim, int nchunks, const PatchDesc *patches,
                        const Chunk *chunks, double *z, int zg, const double *x, int xg,
                        const double *y, int yg, const double *a, const double *b)
{
   if (nchunks <= 0) return;
   g_launches.fetch_add(1, std::memory_order_relaxed);
   if (dim == 2)
      k_vec_lincomb<2><<<work_grid(k_vec_lincomb<2>, nchunks), kThreads, 0, s>>>(
         patches, chunks, nchunks, z, zg, x, xg, y, yg, a, b);
   else
      k_vec_lincomb<3><<<work_grid(k_vec_lincomb<3>, nchunks), kThreads, 0, s>>>(
         patches, chunks, nchunks, z, zg, x, xg, y, yg, a, b);
}

void launch_sweep_check(cudaStream_t s, const unsigned long long *red,
                        const unsigned long long *blk, const int *last_patch, int nprob,
                        double tol, int *run, long long *sweeps)
{
   g_launches.fetch_add(1, std::memory_order_relaxed);
   const int nb = (nprob + 127) / 128;
   k_sweep_check<<<nb, 128, 0, s>>>(red, blk, last_patch, nprob, tol, run, sweeps);
}

void launch_accumulate(cudaStream_t s, const long long *src, long long *dst, int n)
{
   if (n <= 0) return;
   g_launches.fetch_add(1, std::memory_order_relaxed);
   k_accumulate<<<(n + 127) / 128, 128, 0, s>>>(src, dst, n);
}

void launch_g0_to_g1(cudaStream_t s, int dim, int nchunks, const PatchDesc *patches,
                     const Chunk *chunks, const double *src, double *dst)
{
   if (nchunks <= 0) return;
   g_launches.fetch_add(1, std::memory_order_relaxed);
   if (dim == 2) k_g0_to_g1<2><<<work_grid(k_g0_to_g1<2>, nchunks), kThreads, 0, s>>>(patches, chunks, nchunks, src, dst);
   else k_g0_to_g1<3><<<work_grid(k_g0_to_g1<3>, nchunks), kThreads, 0, s>>>(patches, chunks, nchunks, src, dst);
}

void launch_patch_rms(cudaStream_t s, int dim, int npatch, const PatchDesc *patches,
                      const double *x, double *rms)
{
   if (npatch <= 0) return;
   g_launches.fetch_add(1, std::memory_order_relaxed);
   if (dim == 2) k_patch_rms<2><<<npatch, kThreads, 0, s>>>(patches, x, rms);
   else k_patch_rms<3><<<npatch, kThreads, 0, s>>>(patches, x, rms);
}

void launch_gather_samples(cudaStream_t s, int dim, int npatch, const PatchDesc *patches,
                           const double *x, const double *scale, float *out, int S)
{
   if (npatch <= 0) return;
   g_launches.fetch_add(1, std::memory_order_relaxed);
   const long long S3 = (long long)S * S * S;
   dim3 grid((unsigned)((S3 + kThreads - 1) / kThreads), (unsigned)npatch);
   if (dim == 2) k_gather_samples<2><<<grid, kThreads, 0, s>>>(patches, x, scale, out, S);
   else k_gather_samples<3><<<grid, kThreads, 0, s>>>(patches, x, scale, out, S);
}

void launch_scatter_samples(cudaStream_t s, int dim, int nchunks, const PatchDesc *patches,
                            const Chunk *chunks, const float *y, const double *scale, int S,
                            double *dst)
{
   if (nchunks <= 0) return;
   g_launches.fetch_add(1, std::memory_order_relaxed);
   if (dim == 2)
      k_scatter_samples<2><<<work_grid(k_scatter_samples<2>, nchunks), kThreads, 0, s>>>(patches, chunks, nchunks, y, scale, S, dst);
   else
      k_scatter_samples<3><<<work_grid(k_scatter_samples<3>, nchunks), kThreads, 0, s>>>(patches, chunks, nchunks, y, scale, S, dst);
}

void launch_dot_pair(cudaStream_t s, int dim, int nchunks, const PatchDesc *patches,
                     const Chunk *chunks, const double *r, const double *r2, const double *w,
                     double2 *partial, const int *prob_chunk_begin, int nprob, double2 *acc)
{
   if (nchunks <= 0) return;
   g_launches.fetch_add(2, std::memory_order_relaxed);
   if (dim == 2)
      k_dot_pair<2><<<work_grid(k_dot_pair<2>, nchunks), kThreads, 0, s>>>(patches, chunks, nchunks, r, r2, w, partial);
   else
      k_dot_pair<3><<<work_grid(k_dot_pair<3>, nchunks), kThreads, 0, s>>>(patches, chunks, nchunks, r, r2, w, partial);
   k_norm_reduce<<<nprob, kThreads, 0, s>>>(partial, prob_chunk_begin, nprob, acc);
}

void launch_alpha(cudaStream_t s, const double2 *acc, const int *active, int nprob,
                  double *alpha)
{
   g_launches.fetch_add(1, std::memory_order_relaxed);
   k_alpha<<<(nprob + 127) / 128, 128, 0, s>>>(acc, active, nprob, alpha);
}

void launch_apply_alpha(cudaStream_t s, int dim, int nchunks, const PatchDesc *patches,
                        const Chunk *chunks, const double *alpha, double *u, const double *e,
                        double *r, const double *r2)
{
   if (nchunks <= 0) return;
   g_launches.fetch_add(1, std::memory_order_relaxed);
   if (dim == 2)
      k_apply_alpha<2><<<work_grid(k_apply_alpha<2>, nchunks), kThreads, 0, s>>>(patches, chunks, nchunks, alpha, u, e, r, r2);
   else
      k_apply_alpha<3><<<work_grid(k_apply_alpha<3>, nchunks), kThreads, 0, s>>>(patches, chunks, nchunks, alpha, u, e, r, r2);
}

void launch_gather(cudaStream_t s, const long long *idx, long long n, const double *src,
                   double *dst)
{
   if (n <= 0) return;
   g_launches.fetch_add(1, std::memory_order_relaxed);
   k_gather<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(idx, n, src, dst);
}

void launch_scatter(cudaStream_t s, const long long *idx, long long n, const double *src,
                    double *dst)
{
   if (n <= 0) return;
   g_launches.fetch_add(1, std::memory_order_relaxed);
   k_scatter<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(idx, n, src, dst);
}

// explicit instantiations: FP64 (reference arithmetic) and FP32 (mixed
// precision smoothing and transfer of the error)
#define INST_T(T)                                                                          \
   template void launch_fill<T>(cudaStream_t, const FillItem *, const Chunk *, int, const int *, T *,    \
                                const T *, const T *, int, const BcCoefs &, const int *);   \
   template void launch_rbgs_solve<T>(cudaStream_t, int, const PoissonSpec &, int,          \
                                      const PatchDesc *, T *, const T *, const T *,         \
                                      const T *, const long long *, const BcCoefs &, int,   \
                                      double, int *, long long *, unsigned long long *,     \
                                      unsigned long long *, int);                           \
   template void launch_fill_gather<T>(cudaStream_t, long long, const unsigned *,           \
                                       const int *, const unsigned short *,                 \
                                       const FillItem *, const Chunk *, int, const int *,   \
                                       T *, const T *, const T *, int, const BcCoefs &,     \
                                       const int *);                                        \
   template void launch_cf_flux<T>(cudaStream_t, const CfFace *, int, const PatchDesc *,    \
                                   const T *, const T *, int, double, const double *,       \
                                   const double *, T *, const int *);                       \
   template void launch_rbgs<T>(cudaStream_t, int, const PoissonSpec &, int,                \
                                const PatchDesc *, const Chunk *, T *, const T *, const T *, \
                                const T *, const T *, const unsigned char *, int,           \
                                unsigned long long *, const int *, const long long *,       \
                                const BcCoefs &);                                           \
   template void launch_flux<T>(cudaStream_t, int, const PoissonSpec &, int,                \
                                const PatchDesc *, const Chunk *, const T *, const double *, \
                                const unsigned char *, const double *, const double *,      \
                                const int *, double *, const int *);                        \
   template void launch_residual<T>(cudaStream_t, int, const PoissonSpec &, int,            \
                                    const PatchDesc *, const Chunk *, const T *,            \
                                    const double *, const double *, const double *,         \
                                    double *, double *, const int *);                       \
   template void launch_ewing_fix<T>(cudaStream_t, const CfFace *, int, const PatchDesc *,   \
                                     const T *, const double *, int, double, const double *, \
                                     const double *, double *, const int *);                \
   template void launch_flux_cells<T>(cudaStream_t, int, const PoissonSpec &, int,          \
                                      const PatchDesc *, const Chunk *, const T *,          \
                                      const double *, const unsigned char *,                \
                                      const double *, const double *, const int *, double *, \
                                      const int *);                                          \
   template void launch_residual_fused<T>(                                                  \
      cudaStream_t, int, const PoissonSpec &, int, const PatchDesc *, const Chunk *, const T *, \
      const double *, const unsigned char *, const double *, const double *, const int *,   \
      const unsigned char *, const double *, const double *, const double *, double *,      \
      double *, const int *);                                                               \
   template void launch_residual_cells<T>(                                                  \
      cudaStream_t, int, const PoissonSpec &, int, const CellRef *, const PatchDesc *,        \
      const T *, const double *, const unsigned char *, const double *, const double *,     \
      const int *, const unsigned char *, const double *, const double *, const double *,   \
      double *, double *, const int *);                                                     \
   template void launch_prolong_add<T>(cudaStream_t, int, const ProlongItem *,              \
                                       const Chunk *, int, const int *, const PatchDesc *, const T *, \
                                       const double *, const int *, T *, const int *);      \
   template void launch_prolong_add_r2<T>(cudaStream_t, int, const ProlongItem *,           \
                                          const Chunk *, int, const int *, const PatchDesc *, \
                                          const T *, const double *, T *, const int *);     \
   template void launch_add_interior<T>(cudaStream_t, int, int, const PatchDesc *,          \
                                        const Chunk *, double *, const T *, const int *);
INST_T(double)
INST_T(float)
#undef INST_T
template void launch_convert<double, float>(cudaStream_t, const double *, float *, long long);
template void launch_convert<float, double>(cudaStream_t, const float *, double *, long long);

}  // namespace samrai_b200

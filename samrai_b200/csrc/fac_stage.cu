// Staged red-black colour pass (sm_100a), warp specialised.
//
// A CTA walks its share of the level's work units -- runs of slices of one
// patch along the patch's slowest axis -- through a ring of shared-memory
// stages (2 to 4, a launch parameter).  One producer warp copies each unit's
// data from HBM into a stage with TMA bulk copies (cp.async.bulk, completion
// counted on the stage's "full" mbarrier): u over the unit's slices and one
// slice either side, ghost cells included, f, the side arrays of D, C, and
// for the unit's patch faces the push targets and Ewing fluxes.  Eight
// consumer warps then treat the unit in two phases.  Update: the cells of
// the active colour get their new values from the staged values with the
// arithmetic of compflux + rbgswithfluxmax (2d.f:10-364, 3d.f:10-484;
// --fmad=false), stored to HBM and over the staged old value.  Push: after
// a named barrier of the consumers, the new values of the active face cells
// go where the ghost fill would have put them -- into the neighbour patch's
// ghost cell, or the homogeneous Robin value into the patch's own ghost
// cell at a physical boundary.  Each consumer warp then releases the stage
// on its "empty" mbarrier.
//
// Race freedom within a pass: a unit reads cells of the other colour only
// (its own slices, the neighbouring slices and the ghost cells that hold the
// other colour's pushed values) besides each active cell's own old value,
// and writes cells of the active colour and ghost cells next to cells of
// the other colour, which no unit reads in this pass.  The ghost cells must
// be filled before the first pass of a smoothing call; they are then kept
// current by the pushes except the edge and corner ghost cells, which the
// 7-point stencil never reads.
#include <cuda_runtime.h>

#include "fac_device.h"
#include "fac_internal.h"
#include "fac_kernels.h"

namespace samrai_b200 {

namespace {

using namespace dev;

// A wait gives up after this many SM clock cycles (about 2 s), far beyond
// any real copy; the thread sleeps in try_wait up to the hint per test.
constexpr long long kWaitCycles = 4000000000ll;
constexpr unsigned kSuspendHintNs = 20000;

__device__ __forceinline__ unsigned smem_addr(const void *p)
{
   return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes)
{
   asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                "r"(bytes)
                : "memory");
}

// Test the phase; a thread whose phase is not complete may be suspended up
// to the hint (ns) before the test returns false.
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity)
{
   unsigned ok;
   asm volatile(
      "{\n"
      " .reg .pred p;\n"
      " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n"
      " selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity), "r"(kSuspendHintNs)
      : "memory");
   return ok != 0;
}

__device__ __forceinline__ void bulk_load(void *sdst, const void *gsrc, unsigned bytes,
                                          unsigned long long *bar)
{
   asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
         "r"(smem_addr(sdst)),
      "l"(gsrc), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

constexpr int kConsumerWarps = 8;
constexpr int kConsumers = kConsumerWarps * 32;
constexpr int kStageBlock = kConsumers + 32;  // + one producer warp
// full[depth], empty[depth] mbarriers and the copy sources (StageBases)
constexpr int kBarrierBytes = kStageBarrierBytes;

// q / d with m = ceil(2^32 / d) = (2^32 + r) / d, 0 <= r < d: q m / 2^32 =
// q / d + q r / (d 2^32), and the excess stays below 1 / d (so the high word
// of the product is the quotient) whenever q d < 2^32.  The host checks
// that bound for every decode of a unit (integer pipe, no conversions).
__device__ __forceinline__ int udiv(int q, unsigned m)
{
   return (int)__umulhi((unsigned)q, m);
}

__device__ __forceinline__ void mbar_init_count(unsigned long long *bar, unsigned count)
{
   asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
                : "memory");
}

__device__ __forceinline__ void mbar_arrive(unsigned long long *bar)
{
   asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// bounded wait of one thread; false on timeout
__device__ __forceinline__ bool wait_phase(unsigned long long *bar, unsigned parity,
                                           long long limit = kWaitCycles)
{
   const long long t0 = clock64();
   while (!mbar_try_wait(bar, parity))
      if (clock64() - t0 > limit) return false;
   return true;
}

// OR of a predicate over the consumer warps: named barrier 1, which the
// producer warp never takes.  Orders the consumers' shared-memory accesses
// before it against those after it.
__device__ __forceinline__ bool consumers_any(bool p)
{
   unsigned r;
   asm volatile(
      "{\n"
      " .reg .pred pi, po;\n"
      " setp.ne.u32 pi, %1, 0;\n"
      " bar.red.or.pred po, 1, %2, pi;\n"
      " selp.u32 %0, 1, 0, po;\n"
      "}\n"
      : "=r"(r)
      : "r"((unsigned)p), "n"(kConsumers)
      : "memory");
   return r != 0;
}

// Source arrays of the bulk copies, indexed by StageSrc.
struct StageBases {
   const char *p[kSrcCount];
};

// full[depth], empty[depth], the copy sources, and one mbarrier nothing
// arrives on (the test of the bounded wait waits on it)
static_assert(2 * kStageDepthMax * 8 + sizeof(StageBases) + 8 <= kBarrierBytes, "barrier area");
static_assert((2 * kStageDepthMax * 8 + sizeof(StageBases)) % 8 == 0, "mbarrier alignment");

// Red-black parity of a row of a unit: the first active cell of the row is
// at li = ioffset (2d.f:141-147, 3d.f:201-207 with their integer modulo).
__device__ __forceinline__ int row_ioffset(int q, int offset)
{
   return (q - (q / 2) * 2) != offset ? 1 : 0;
}

// Phase 1 of a unit: the new values of the active colour, stored to HBM and
// over the staged old values (which no other cell of this pass reads).
template <int DIM, bool DVAR, int CKIND, class T>
__device__ __forceinline__ void stage_update(unsigned char *stage, int tid, T *__restrict__ u,
                                             int offset, T dconst, T cconst)
{
   const UnitHdr *h = reinterpret_cast<const UnitHdr *>(stage);
   const int s0 = h->s0;
   const int lo0 = h->lo[0], lo1 = h->lo[1], lo2 = DIM == 3 ? h->lo[2] : 0;
   const int nx = h->hi[0] - lo0 + 1;
   const int ny = h->hi[1] - lo1 + 1;
   const int gx = nx + 2, gy = ny + 2;
   const int sy = gx, sz = gx * gy;
   T *su = reinterpret_cast<T *>(stage + h->off_u);
   const T *sf = reinterpret_cast<const T *>(stage + h->off_f);
   const T *sdx = reinterpret_cast<const T *>(stage + h->off_d[0]);
   const T *sdy = reinterpret_cast<const T *>(stage + h->off_d[1]);
   const T *sdz = reinterpret_cast<const T *>(stage + h->off_d[2]);
   const T *sc = reinterpret_cast<const T *>(stage + h->off_c);
   // faces of the unit with coarse-fine entries, whose fluxes are the
   // staged Ewing fluxes
   const int cfm = h->cfmask;
   const int ns = h->ns;
   // global element of staged u element 0 (the slice before the unit)
   T *gu = u + h->off1 + (long long)s0 * (DIM == 3 ? (long long)sz : (long long)gx);
   const int hx = h->hx;
   const int nslots = h->nslots;
   const unsigned mhx = h->mhx, mny = h->mny;
   const bool f64 = sizeof(T) == 8;
   const T dxi = f64 ? (T)h->dxi_d[0] : (T)h->dxi_f[0];
   const T dyi = f64 ? (T)h->dxi_d[1] : (T)h->dxi_f[1];
   const T dzi = DIM == 3 ? (f64 ? (T)h->dxi_d[2] : (T)h->dxi_f[2]) : (T)0;
   // parity of the first cell of each row: lo1 + j (2-D), lo0 + j + k (3-D)
   const int qbase = DIM == 3 ? lo0 + lo1 + lo2 + s0 : 2 * lo1 + s0;
   // two slots per thread in flight: their shared-memory loads overlap
#pragma unroll 2
   for (int t = tid; t < nslots; t += kConsumers) {
      const int row = udiv(t, mhx);
      const int mm = t - row * hx;
      int lj, ls;
      if (DIM == 3) {
         ls = udiv(row, mny);
         lj = row - ls * ny;
      } else {
         lj = s0 + row;
         ls = row;
      }
      const int li = row_ioffset(DIM == 3 ? qbase + lj + ls : qbase + row, offset) + 2 * mm;
      if (li >= nx) continue;
      const int c = DIM == 3 ? (li + 1) + gx * ((lj + 1) + gy * (ls + 1))
                             : (li + 1) + gx * (ls + 1);
      const T uc = su[c];
      T dx0, dx1, dy0, dy1, dz0 = (T)0, dz1 = (T)0;
      if (DVAR) {
         if (DIM == 3) {
            const int bx = li + (nx + 1) * (lj + ny * ls);
            dx0 = sdx[bx];
            dx1 = sdx[bx + 1];
            const int by = li + nx * (lj + (ny + 1) * ls);
            dy0 = sdy[by];
            dy1 = sdy[by + nx];
            const int bz = li + nx * (lj + ny * ls);
            dz0 = sdz[bz];
            dz1 = sdz[bz + nx * ny];
         } else {
            const int bx = li + (nx + 1) * ls;
            dx0 = sdx[bx];
            dx1 = sdx[bx + 1];
            const int by = li + nx * ls;
            dy0 = sdy[by];
            dy1 = sdy[by + nx];
         }
      } else {
         dx0 = dx1 = dy0 = dy1 = dz0 = dz1 = dconst;
      }
      const T nxl = su[c - 1], nxh = su[c + 1];
      const T nyl = su[c - sy], nyh = su[c + sy];
      T nzl = (T)0, nzh = (T)0;
      if (DIM == 3) {
         nzl = su[c - sz];
         nzh = su[c + sz];
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
      if (cfm) {
         // coarse-fine faces this cell lies on (bit 2*axis+side)
         int on = 0;
         on |= li == 0 ? 1 : 0;
         on |= li == nx - 1 ? 2 : 0;
         on |= lj == 0 ? 4 : 0;
         on |= lj == ny - 1 ? 8 : 0;
         if (DIM == 3) {
            on |= ls == 0 ? 16 : 0;
            on |= ls == ns - 1 ? 32 : 0;
         }
         on &= cfm;
         if (on) {
#pragma unroll
            for (int fid = 0; fid < 2 * DIM; ++fid) {
               if (!(on & (1 << fid))) continue;
               const int a = fid >> 1;
               // index of the cell in the face region of axis a
               const int e = a == 0 ? (DIM == 3 ? lj + ny * ls : ls)
                                    : (a == DIM - 1 ? (DIM == 3 ? li + nx * lj : li)
                                                    : li + nx * ls);
               if (reinterpret_cast<const int *>(stage + h->off_push[fid])[e] != -2) continue;
               const T fl = reinterpret_cast<const T *>(stage + h->off_cff[fid])[e];
               switch (fid) {
                  case 0: fxl = fl; break;
                  case 1: fxh = fl; break;
                  case 2: fyl = fl; break;
                  case 3: fyh = fl; break;
                  case 4: fzl = fl; break;
                  default: fzh = fl; break;
               }
            }
         }
      }
      const int l0 = DIM == 3 ? li + nx * (lj + ny * ls) : li + nx * ls;
      const T scv = CKIND == 2 ? sc[l0] : (CKIND == 1 ? cconst : (T)0);
      const T fv = sf[l0];
      T residual;
      const T v = rb_point<DIM, T>(fv, uc, scv, dxi, dyi, dzi, fxl, fxh, fyl, fyh, fzl, fzh, dx0,
                                   dx1, dy0, dy1, dz0, dz1, residual);
      gu[c] = v;
      su[c] = v;
   }
}

// Phase 2 of a unit: the new values of the active cells on the unit's patch
// faces go where the ghost fill would put them -- the neighbour patch's
// ghost cell, or the homogeneous Robin value into the patch's own ghost cell
// at a physical boundary.  One flat loop over the entries of the faces
// with push targets (pmask), so that no thread walks six face tests.
template <int DIM, class T>
__device__ __forceinline__ void stage_push(const unsigned char *stage, int tid,
                                           T *__restrict__ u, int offset, const BcCoefs &bc)
{
   const UnitHdr *h = reinterpret_cast<const UnitHdr *>(stage);
   const int pm = h->pmask;
   if (!pm) return;
   const int s0 = h->s0, ns = h->ns;
   const int lo0 = h->lo[0], lo1 = h->lo[1], lo2 = DIM == 3 ? h->lo[2] : 0;
   const int nx = h->hi[0] - lo0 + 1;
   const int ny = h->hi[1] - lo1 + 1;
   const int gx = nx + 2, gy = ny + 2;
   const int sz = gx * gy;
   const T *su = reinterpret_cast<const T *>(stage + h->off_u);
   T *gu = u + h->off1 + (long long)s0 * (DIM == 3 ? (long long)sz : (long long)gx);
   const unsigned mnx = h->mnx, mny = h->mny;
   const int qbase = DIM == 3 ? lo0 + lo1 + lo2 + s0 : 2 * lo1 + s0;
   // entries of each face region (0 for faces without push targets)
   int cnt[2 * DIM];
   int total = 0;
#pragma unroll
   for (int f = 0; f < 2 * DIM; ++f) {
      const int a = f >> 1;
      const int n = a == 0 ? (DIM == 3 ? ny * ns : ns) : (a == DIM - 1 ? (DIM == 3 ? nx * ny : nx)
                                                                       : nx * ns);
      cnt[f] = (pm >> f) & 1 ? n : 0;
      total += cnt[f];
   }
   for (int t = tid; t < total; t += kConsumers) {
      int f = 0, e = t;
#pragma unroll
      for (int q = 0; q < 2 * DIM - 1; ++q)
         if (f == q && e >= cnt[q]) {
            e -= cnt[q];
            f = q + 1;
         }
      const int a = f >> 1, side = f & 1;
      int li, lj, ls;
      if (DIM == 3) {
         if (a == 0) {
            ls = udiv(e, mny);
            lj = e - ls * ny;
            li = side ? nx - 1 : 0;
         } else if (a == 1) {
            ls = udiv(e, mnx);
            li = e - ls * nx;
            lj = side ? ny - 1 : 0;
         } else {
            lj = udiv(e, mnx);
            li = e - lj * nx;
            ls = side ? ns - 1 : 0;
         }
      } else {
         if (a == 0) {
            ls = e;
            li = side ? nx - 1 : 0;
         } else {
            li = e;
            ls = side ? ns - 1 : 0;
         }
         lj = s0 + ls;
      }
      const int q = DIM == 3 ? qbase + lj + ls : qbase + ls;
      if ((li & 1) != row_ioffset(q, offset)) continue;  // not of the active colour
      const int tgt = reinterpret_cast<const int *>(stage + h->off_push[f])[e];
      if (tgt < -1) continue;  // coarse-fine face: no push
      const int c = DIM == 3 ? (li + 1) + gx * ((lj + 1) + gy * (ls + 1))
                             : (li + 1) + gx * (ls + 1);
      const T v = su[c];
      if (tgt >= 0) {
         u[tgt] = v;
      } else {
         const int step = a == 0 ? 1 : (a == 1 ? gx : sz);
         gu[side ? c + step : c - step] = robin<T>(v, f, (T)h->dx[a], 1, bc);
      }
   }
}

// The walk of a block over its units, shared by the staged passes: the
// producer warp streams the units' copies into the ring, the consumer warps
// run the pass's first phase on each unit, meet at a named barrier (where a
// wait that ran out ends the walk for all of them), run its second phase
// and free the stage.
template <class Pass>
__device__ __forceinline__ void staged_walk(const Chunk *__restrict__ chunks, int nwork,
                                            const UnitCopy *__restrict__ copies,
                                            const StageBases &bases, int stage_bytes, int depth,
                                            int *__restrict__ err, const WaitTest &wt,
                                            const Pass &pass)
{
   extern __shared__ __align__(128) unsigned char smem[];
   unsigned long long *full = reinterpret_cast<unsigned long long *>(smem);
   unsigned long long *empty = full + kStageDepthMax;
   StageBases *sbases = reinterpret_cast<StageBases *>(smem + 2 * kStageDepthMax * 8);
   unsigned long long *never_bar = reinterpret_cast<unsigned long long *>(
      smem + 2 * kStageDepthMax * 8 + sizeof(StageBases));
   unsigned char *stages = smem + kBarrierBytes;
   // the list holds active problems only (compacted), so unit k of this
   // block is entry k G + b (G blocks, b this block) up to the end marker
   auto unit_at = [&](int k) { return k * (int)gridDim.x + (int)blockIdx.x; };
   auto valid = [&](int w) { return w < nwork && chunks[w].patch >= 0; };
   if (threadIdx.x == 0) {
      for (int k = 0; k < depth; ++k) {
         mbar_init_count(&full[k], 1);
         mbar_init_count(&empty[k], kConsumerWarps);
      }
      mbar_init_count(never_bar, 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      *sbases = bases;
   }
   __syncthreads();
   const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
   if (warp == kConsumerWarps) {
      // producer warp: lane i issues copy i of a unit (the host-built copy
      // list, header first; its first entry carries the byte total)
      // two units ahead of the copies it issues: the chunk of the unit after
      // next and the copy entry of the next unit are loaded while this
      // unit's stage comes free, so no dependent load waits per unit
      const Chunk end = {-1, 0, 0, 0};
      const UnitCopy none = {0, 0, 0, 0, 0};
      int w = unit_at(0);
      Chunk ch = w < nwork ? chunks[w] : end;
      UnitCopy cp = ch.patch >= 0 && lane < ch.count ? copies[ch.begin + lane] : none;
      w = unit_at(1);
      Chunk chn = ch.patch >= 0 && w < nwork ? chunks[w] : end;
      int k = 0;  // units issued
      for (; ch.patch >= 0; ++k) {
         const UnitCopy cpn = chn.patch >= 0 && lane < chn.count ? copies[chn.begin + lane] : none;
         const int w2 = unit_at(k + 2);
         const Chunk chnn = chn.patch >= 0 && w2 < nwork ? chunks[w2] : end;
         const int st = k % depth;
         bool ok = true;
         if (k >= depth && lane == 0) ok = wait_phase(&empty[st], ((k / depth) & 1) ^ 1u);
         if (!__shfl_sync(0xffffffffu, ok ? 1 : 0, 0)) {
            if (lane == 0) atomicExch(err, 1);
            break;
         }
         unsigned char *stage = stages + st * stage_bytes;
         if (lane == 0) mbar_expect_tx(&full[st], (unsigned)cp.total);
         __syncwarp();
         if (lane < ch.count)
            bulk_load(stage + cp.dst_off, sbases->p[cp.src] + cp.src_off, (unsigned)cp.nbytes,
                      &full[st]);
         ch = chn;
         cp = cpn;
         chn = chnn;
      }
      // the block's shared memory must outlive every copy issued into it:
      // the last `depth` units (one per stage; no later unit was issued
      // into those stages) have landed before this warp leaves, whether
      // or not the consumers took them
      if (lane == 0)
         for (int q = k - 1; q >= 0 && q >= k - depth; --q)
            if (!wait_phase(&full[q % depth], (q / depth) & 1)) atomicExch(err, 1);
      __syncwarp();
      return;
   }
   const int tid = threadIdx.x;  // 0 .. kConsumers-1
   int k = 0;
   bool cur = valid(unit_at(0));
   for (; cur; ++k) {
      const bool nxt = valid(unit_at(k + 1));  // prefetched, used at the loop end
      const int st = k % depth;
      const unsigned par = (k / depth) & 1;
      unsigned char *stage = stages + st * stage_bytes;
      // (the test of the bounded wait waits on a barrier nothing arrives on)
      const bool ok = wt.never ? wait_phase(never_bar, 0u, wt.limit)
                               : wait_phase(&full[st], par, wt.limit);
      if (ok) pass.first(stage, tid);
      // every consumer passes here once per unit: all leave together when
      // any wait ran out, and the pushes read the updated stage
      if (consumers_any(!ok)) {
         if (tid == 0) atomicExch(err, 1);
         wait_phase(&full[st], par);  // copies still in flight land before the exit
         return;
      }
      pass.second(stage, tid);
      // the next copies into this stage (async proxy) follow the stores above
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[st]);
      cur = nxt;
   }
}

// Red-black colour pass: update of the active colour, then the pushes.
template <int DIM, bool DVAR, int CKIND, class T>
struct ColourPass {
   T *u;
   int offset;
   T dconst, cconst;
   BcCoefs bc;
   __device__ __forceinline__ void first(unsigned char *stage, int tid) const
   {
      stage_update<DIM, DVAR, CKIND, T>(stage, tid, u, offset, dconst, cconst);
   }
   __device__ __forceinline__ void second(unsigned char *stage, int tid) const
   {
      stage_push<DIM, T>(stage, tid, u, offset, bc);
   }
};

template <int DIM, bool DVAR, int CKIND, class T>
__global__ void __launch_bounds__(kStageBlock)
k_rb_staged(const Chunk *__restrict__ chunks, int nwork, const UnitCopy *__restrict__ copies,
            StageBases bases, int stage_bytes, int depth, ColourPass<DIM, DVAR, CKIND, T> pass,
            int *__restrict__ err, WaitTest wt)
{
   staged_walk(chunks, nwork, copies, bases, stage_bytes, depth, err, wt, pass);
}

// One unit of the staged composite residual: for every cell of the unit,
// the face fluxes from the staged u and D (computeFluxOnPatch, the
// compflux* arithmetic: flux = (1/dx) D (u_hi - u_lo)) and the residual
// r = f - div flux - C u (compres{var,con}sca{2,3}d), the operation order
// of k_flux_cells + k_residual, FP64 throughout (--fmad=false); the fluxes
// on the patch's faces go to the outer-side arrays.  Cells with a
// coarse-fine face or a face under a finer patch are redone by the fix-up
// pass afterwards.
template <int DIM, bool DVAR, int CKIND, class TU>
__device__ __forceinline__ void stage_residual(const unsigned char *stage, int tid, double dconst,
                                               double cconst, double *__restrict__ res,
                                               double *__restrict__ oflux)
{
   const ResHdr *h = reinterpret_cast<const ResHdr *>(stage);
   const int s0 = h->s0;
   const int lo0 = h->lo[0], lo1 = h->lo[1], lo2 = DIM == 3 ? h->lo[2] : 0;
   const int nx = h->hi[0] - lo0 + 1;
   const int ny = h->hi[1] - lo1 + 1;
   const int nslow = DIM == 3 ? h->hi[2] - lo2 + 1 : ny;
   const int gx = nx + 2, gy = ny + 2, sz = gx * gy;
   const TU *su = reinterpret_cast<const TU *>(stage + h->off_u);
   const bool hasf = h->off_f >= 0;
   const double *sf = reinterpret_cast<const double *>(stage + (hasf ? h->off_f : 0));
   const double *sdx = reinterpret_cast<const double *>(stage + h->off_d[0]);
   const double *sdy = reinterpret_cast<const double *>(stage + h->off_d[1]);
   const double *sdz = reinterpret_cast<const double *>(stage + h->off_d[2]);
   const double *sc = reinterpret_cast<const double *>(stage + h->off_c);
   const double dxi = h->dxi[0], dyi = h->dxi[1], dzi = DIM == 3 ? h->dxi[2] : 0.0;
   double *gr = res + h->off0s;
   const bool wo = oflux != nullptr && h->has_oflux;
   const int n = h->ncells;
   const unsigned mnx = h->mnx, mny = h->mny;
   for (int t = tid; t < n; t += kConsumers) {
      int li, lj, ls;
      if (DIM == 3) {
         const int row = udiv(t, mnx);
         li = t - row * nx;
         ls = udiv(row, mny);
         lj = row - ls * ny;
      } else {
         ls = udiv(t, mnx);
         li = t - ls * nx;
         lj = s0 + ls;
      }
      const int c = DIM == 3 ? (li + 1) + gx * ((lj + 1) + gy * (ls + 1))
                             : (li + 1) + gx * (ls + 1);
      const double uc = (double)su[c];
      double dx0, dx1, dy0, dy1, dz0 = 0.0, dz1 = 0.0;
      if (DVAR) {
         if (DIM == 3) {
            const int bx = li + (nx + 1) * (lj + ny * ls);
            dx0 = sdx[bx];
            dx1 = sdx[bx + 1];
            const int by = li + nx * (lj + (ny + 1) * ls);
            dy0 = sdy[by];
            dy1 = sdy[by + nx];
            const int bz = li + nx * (lj + ny * ls);
            dz0 = sdz[bz];
            dz1 = sdz[bz + nx * ny];
         } else {
            const int bx = li + (nx + 1) * ls;
            dx0 = sdx[bx];
            dx1 = sdx[bx + 1];
            const int by = li + nx * ls;
            dy0 = sdy[by];
            dy1 = sdy[by + nx];
         }
      } else {
         dx0 = dx1 = dy0 = dy1 = dz0 = dz1 = dconst;
      }
      const double fxl = dxi * dx0 * (uc - (double)su[c - 1]);
      const double fxh = dxi * dx1 * ((double)su[c + 1] - uc);
      const double fyl = dyi * dy0 * (uc - (double)su[c - gx]);
      const double fyh = dyi * dy1 * ((double)su[c + gx] - uc);
      double fzl = 0.0, fzh = 0.0;
      if (DIM == 3) {
         fzl = dzi * dz0 * (uc - (double)su[c - sz]);
         fzh = dzi * dz1 * ((double)su[c + sz] - uc);
      }
      const double scv = CKIND == 2 ? sc[t] : (CKIND == 1 ? cconst : 0.0);
      const double fv = hasf ? sf[t] : 0.0;
      double rv;
      if (DIM == 2)
         rv = fv - (dxi * (fxh - fxl) + dyi * (fyh - fyl)) - scv * uc;
      else
         rv = fv - (dxi * (fxh - fxl) + dyi * (fyh - fyl) + dzi * (fzh - fzl)) - scv * uc;
      gr[t] = rv;
      if (wo) {
         const int kk = DIM == 3 ? s0 + ls : 0;  // slow-axis index in the patch (3-D)
         if (li == 0) oflux[h->offo[0][0] + (DIM == 3 ? lj + ny * kk : lj)] = fxl;
         if (li == nx - 1) oflux[h->offo[0][1] + (DIM == 3 ? lj + ny * kk : lj)] = fxh;
         if (lj == 0) oflux[h->offo[1][0] + (DIM == 3 ? li + nx * kk : li)] = fyl;
         if (lj == ny - 1) oflux[h->offo[1][1] + (DIM == 3 ? li + nx * kk : li)] = fyh;
         if (DIM == 3) {
            if (kk == 0) oflux[h->offo[2][0] + li + nx * lj] = fzl;
            if (kk == nslow - 1) oflux[h->offo[2][1] + li + nx * lj] = fzh;
         }
      }
   }
}

template <int DIM, bool DVAR, int CKIND, class TU>
struct ResidualPass {
   double dconst, cconst;
   double *res, *oflux;
   __device__ __forceinline__ void first(unsigned char *stage, int tid) const
   {
      stage_residual<DIM, DVAR, CKIND, TU>(stage, tid, dconst, cconst, res, oflux);
   }
   __device__ __forceinline__ void second(unsigned char *, int) const {}
};

template <int DIM, bool DVAR, int CKIND, class TU>
__global__ void __launch_bounds__(kStageBlock)
k_res_staged(const Chunk *__restrict__ chunks, int nwork, const UnitCopy *__restrict__ copies,
             StageBases bases, int stage_bytes, int depth, ResidualPass<DIM, DVAR, CKIND, TU> pass,
             int *__restrict__ err, WaitTest wt)
{
   staged_walk(chunks, nwork, copies, bases, stage_bytes, depth, err, wt, pass);
}

// Grid of a staged kernel: one wave of resident blocks, each walking its
// share of the units.
template <class K>
int staged_grid(K *kernel, int nunits, int smem)
{
   static int nsm = 0;
   if (nsm == 0) {
      int dev = 0;
      if (cudaGetDevice(&dev) != cudaSuccess ||
          cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
         nsm = 148;
   }
   int per_sm = 1;
   cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kStageBlock, smem);
   per_sm = per_sm < 1 ? 1 : per_sm;
   return nunits < nsm * per_sm ? nunits : nsm * per_sm;
}

template <int DIM, bool DVAR, int CK, class TU>
void res_staged_inst(cudaStream_t s, int nunits, int stage_bytes, int depth, const Chunk *units,
                     const UnitCopy *copies, const StageBases &bases, double dconst,
                     double cconst, double *res, double *oflux, int *err, const WaitTest &wt)
{
   static bool attr = false;
   if (!attr) {
      cudaFuncSetAttribute(k_res_staged<DIM, DVAR, CK, TU>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, kStageSmemMax);
      attr = true;
   }
   const int smem = kBarrierBytes + depth * stage_bytes;
   const int grid = staged_grid(k_res_staged<DIM, DVAR, CK, TU>, nunits, smem);
   const ResidualPass<DIM, DVAR, CK, TU> pass{dconst, cconst, res, oflux};
   k_res_staged<DIM, DVAR, CK, TU><<<grid, kStageBlock, smem, s>>>(
      units, nunits, copies, bases, stage_bytes, depth, pass, err, wt);
}

template <int DIM, bool DVAR, int CK, class T>
void staged_inst(cudaStream_t s, int nunits, int stage_bytes, int depth, const Chunk *units,
                 const UnitCopy *copies, const StageBases &bases, T *u, int offset,
                 double dconst, double cconst, const BcCoefs &bc, int *err, const WaitTest &wt)
{
   static bool attr = false;
   static int nsm = 148;
   if (!attr) {
      cudaFuncSetAttribute(k_rb_staged<DIM, DVAR, CK, T>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, kStageSmemMax);
      int dev = 0;
      if (cudaGetDevice(&dev) == cudaSuccess)
         cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
      attr = true;
   }
   const int smem = kBarrierBytes + depth * stage_bytes;
   // one wave of resident blocks: each walks its share of the units
   int per_sm = 1;
   cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_rb_staged<DIM, DVAR, CK, T>,
                                                 kStageBlock, smem);
   per_sm = per_sm < 1 ? 1 : per_sm;
   const int grid = nunits < nsm * per_sm ? nunits : nsm * per_sm;
   const ColourPass<DIM, DVAR, CK, T> pass{u, offset, (T)dconst, (T)cconst, bc};
   k_rb_staged<DIM, DVAR, CK, T><<<grid, kStageBlock, smem, s>>>(
      units, nunits, copies, bases, stage_bytes, depth, pass, err, wt);
}

}  // namespace

template <class T>
void launch_rb_staged(cudaStream_t s, int dim, const PoissonSpec &spec, int nunits,
                      int stage_bytes, int depth, const Chunk *units, const UnitCopy *copies,
                      const unsigned char *headers, T *u, const T *f, const T *dside,
                      const T *cfield, const T *cfflux, int offset, const int *pushmap,
                      const BcCoefs &bc, int *err, const WaitTest &wt)
{
   if (nunits <= 0) return;
   add_kernel_launches(1);
   StageBases bases;
   bases.p[kSrcU] = reinterpret_cast<const char *>(u);
   bases.p[kSrcF] = reinterpret_cast<const char *>(f);
   bases.p[kSrcD] = reinterpret_cast<const char *>(dside);
   bases.p[kSrcC] = reinterpret_cast<const char *>(cfield);
   bases.p[kSrcPush] = reinterpret_cast<const char *>(pushmap);
   bases.p[kSrcFlux] = reinterpret_cast<const char *>(cfflux);
   bases.p[kSrcHdr] = reinterpret_cast<const char *>(headers);
#define SG(D, V, C)                                                                       \
   staged_inst<D, V, C, T>(s, nunits, stage_bytes, depth, units, copies, bases, u, offset, \
                           spec.d_const, spec.c_const, bc, err, wt)
   if (dim == 2) {
      if (spec.d_variable) {
         if (spec.c_kind == 2) SG(2, true, 2);
         else if (spec.c_kind == 1) SG(2, true, 1);
         else SG(2, true, 0);
      } else {
         if (spec.c_kind == 2) SG(2, false, 2);
         else if (spec.c_kind == 1) SG(2, false, 1);
         else SG(2, false, 0);
      }
   } else {
      if (spec.d_variable) {
         if (spec.c_kind == 2) SG(3, true, 2);
         else if (spec.c_kind == 1) SG(3, true, 1);
         else SG(3, true, 0);
      } else {
         if (spec.c_kind == 2) SG(3, false, 2);
         else if (spec.c_kind == 1) SG(3, false, 1);
         else SG(3, false, 0);
      }
   }
#undef SG
}

#define INST_STAGED(T)                                                                       \
   template void launch_rb_staged<T>(cudaStream_t, int, const PoissonSpec &, int, int, int,    \
                                     const Chunk *, const UnitCopy *, const unsigned char *,   \
                                     T *, const T *, const T *, const T *, const T *, int,     \
                                     const int *, const BcCoefs &, int *, const WaitTest &);
INST_STAGED(double)
INST_STAGED(float)
#undef INST_STAGED

template <class TU>
void launch_res_staged(cudaStream_t s, int dim, const PoissonSpec &spec, int nunits,
                       int stage_bytes, int depth, const Chunk *units, const UnitCopy *copies,
                       const unsigned char *headers, const TU *u, const double *f,
                       const double *dside, const double *cfield, double *res, double *oflux,
                       int *err, const WaitTest &wt)
{
   if (nunits <= 0) return;
   add_kernel_launches(1);
   StageBases bases;
   for (int k = 0; k < kSrcCount; ++k) bases.p[k] = nullptr;
   bases.p[kSrcU] = reinterpret_cast<const char *>(u);
   bases.p[kSrcF] = reinterpret_cast<const char *>(f);
   bases.p[kSrcD] = reinterpret_cast<const char *>(dside);
   bases.p[kSrcC] = reinterpret_cast<const char *>(cfield);
   bases.p[kSrcHdr] = reinterpret_cast<const char *>(headers);
#define RG(D, V, C)                                                                        \
   res_staged_inst<D, V, C, TU>(s, nunits, stage_bytes, depth, units, copies, bases,        \
                                spec.d_const, spec.c_const, res, oflux, err, wt)
   if (dim == 2) {
      if (spec.d_variable) {
         if (spec.c_kind == 2) RG(2, true, 2);
         else if (spec.c_kind == 1) RG(2, true, 1);
         else RG(2, true, 0);
      } else {
         if (spec.c_kind == 2) RG(2, false, 2);
         else if (spec.c_kind == 1) RG(2, false, 1);
         else RG(2, false, 0);
      }
   } else {
      if (spec.d_variable) {
         if (spec.c_kind == 2) RG(3, true, 2);
         else if (spec.c_kind == 1) RG(3, true, 1);
         else RG(3, true, 0);
      } else {
         if (spec.c_kind == 2) RG(3, false, 2);
         else if (spec.c_kind == 1) RG(3, false, 1);
         else RG(3, false, 0);
      }
   }
#undef RG
}

#define INST_RES_STAGED(TU)                                                                    \
   template void launch_res_staged<TU>(cudaStream_t, int, const PoissonSpec &, int, int, int,  \
                                       const Chunk *, const UnitCopy *, const unsigned char *, \
                                       const TU *, const double *, const double *,             \
                                       const double *, double *, double *, int *,              \
                                       const WaitTest &);
INST_RES_STAGED(double)
INST_RES_STAGED(float)
#undef INST_RES_STAGED

}  // namespace samrai_b200

// Learned coarse-correction network: forward, backward and Adam kernels.
//
// Four 3x3x3 convolutions 1 -> 16 -> 16 -> 16 -> 1 channels, ReLU after
// the first three, no biases (so the network is positively homogeneous and
// the residual's scale passes straight through), zero padding at the edge
// of each sample.  Weights and stored activations are BF16; accumulation is
// FP32.  One sample is a patch plus a one-cell halo padded to an S^3 box
// (S = 18: patches of up to 16^3 cells).
//
// The 16 -> 16 layers run as implicit GEMMs on the 5th-generation tensor
// cores (k_conv_mid_tc: tcgen05.mma, BF16 operands in shared memory, FP32
// accumulators in tensor memory): a CTA stages a slab of z-planes of one
// sample with a zero halo in shared memory, and for each 128-row tile of
// the slab's cells one thread issues 27 MMAs (one per tap, M = 128 cells,
// N = 16 output channels, K = 16 input channels), the tap being a shift of
// the A operand's start address.  The same kernel computes the backward
// pass with respect to the data (taps reversed, weights transposed, gated by
// the forward ReLU mask).  Weight gradients of the 16 -> 16 layers are 27
// 16 x 16 GEMMs reducing over all cells, from the same staged slabs
// (ldmatrix + mma.sync, three taps per warp).  Layer 4 (16 -> 1) runs on
// the same tensor-core kernel with its weights padded to 16 output
// channels; layer 1 (1 -> 16), its weight gradient and the other small
// gradients run on the FP32 cores.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/samrai_fac_b200.h"
#include "fac_kernels.h"

namespace {

constexpr int S = FAC_CNN_BOX;       // sample box side (patch + halo)
constexpr int S3 = S * S * S;
constexpr int C = 16;                // hidden channels
constexpr int T = 27;                // taps

__device__ __forceinline__ void cell_coords(long long cell, int &x, int &y, int &z)
{
   const int rem = (int)(cell % S3);
   x = rem % S;
   y = (rem / S) % S;
   z = rem / (S * S);
}

__device__ __forceinline__ int tap_dx(int t) { return t % 3 - 1; }
__device__ __forceinline__ int tap_dy(int t) { return (t / 3) % 3 - 1; }
__device__ __forceinline__ int tap_dz(int t) { return t / 9 - 1; }

// Flat index of the neighbour of `cell` at tap t, or -1 outside the sample.
__device__ __forceinline__ long long neighbour(long long cell, int x, int y, int z, int t)
{
   const int dx = tap_dx(t), dy = tap_dy(t), dz = tap_dz(t);
   if (x + dx < 0 || x + dx >= S || y + dy < 0 || y + dy >= S || z + dz < 0 || z + dz >= S)
      return -1;
   return cell + dz * S * S + dy * S + dx;
}

__device__ __forceinline__ void mma_bf16(float *d, const uint32_t *a, uint32_t b0, uint32_t b1)
{
   asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// ---------------------------------------------------------------------------
// layer 1: 1 -> 16, ReLU
// ---------------------------------------------------------------------------
__global__ void k_conv_in(const __nv_bfloat16 *__restrict__ x, const float *__restrict__ w1,
                          __nv_bfloat16 *__restrict__ y, long long ncells)
{
   __shared__ float w[T * C];
   for (int i = threadIdx.x; i < T * C; i += blockDim.x) w[i] = w1[i];
   __syncthreads();
   const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (cell >= ncells) return;
   int cx, cy, cz;
   cell_coords(cell, cx, cy, cz);
   float acc[C];
#pragma unroll
   for (int c = 0; c < C; ++c) acc[c] = 0.f;
   for (int t = 0; t < T; ++t) {
      const long long nb = neighbour(cell, cx, cy, cz, t);
      if (nb < 0) continue;
      const float v = __bfloat162float(x[nb]);
#pragma unroll
      for (int c = 0; c < C; ++c) acc[c] = __fmaf_rn(w[t * C + c], v, acc[c]);
   }
#pragma unroll
   for (int c = 0; c < C; c += 2) {
      __nv_bfloat162 o = __floats2bfloat162_rn(fmaxf(acc[c], 0.f), fmaxf(acc[c + 1], 0.f));
      *reinterpret_cast<__nv_bfloat162 *>(y + cell * C + c) = o;
   }
}

// ---------------------------------------------------------------------------
// layers 2, 3 (and their data gradients) on tcgen05.
//
// A CTA takes slabs of kTcNz output z-planes of one sample in turn.  It
// stages the slab's input planes z0-1 .. z0+kTcNz with a one-cell zero halo
// in x and y (kTcPx x kTcPx cells per plane) in shared memory, channels
// split in two planes of 8 (16 bytes per cell each): with cells as rows and
// channels as K, that is the K-major canonical layout without swizzle (8
// consecutive cells form a core matrix of 8 rows x 16 bytes; SBO = 128 bytes
// between groups of 8 cells, LBO = the distance of the two channel planes).
// Output row r (a padded cell index) needs input row r + off(tap), so tap t
// is the same descriptor with its start moved by off(t) cells.  The padded
// rows of halo positions are computed and dropped.  Weights: per tap the
// 16 x 16 block as B (N = output channels, K = input channels, K-major).
// Accumulators: tile i of 128 rows in tensor-memory columns 16 i .. 16 i +
// 15, lane = row; warp w reads lanes 32 (w % 4) .. + 31.
// ---------------------------------------------------------------------------
constexpr int kTcPx = S + 2;                         // padded row length
constexpr int kTcPlane = kTcPx * kTcPx;              // padded plane
constexpr int kTcNz = 3;                             // output planes per slab
constexpr int kTcSlabs = S / kTcNz;                  // slabs per sample
constexpr int kTcBox = (kTcNz + 2) * kTcPlane;       // staged cells
constexpr int kTcTiles = (kTcNz * kTcPlane + 127) / 128;
constexpr int kTcReach = 1 + kTcPx + kTcPlane;       // largest |tap offset|
constexpr int kTcFront = 32;                         // cells before the box
constexpr int kTcSpan = kTcFront + kTcBox + 128;     // cells per channel plane
constexpr int kTcCols = 256;                         // tensor-memory columns
constexpr int kTcPlaneBytes = kTcSpan * 16;
constexpr int kTcWBytes = T * 512;
constexpr int kTcSmem = 2 * kTcPlaneBytes + kTcWBytes + 16;
constexpr int kTcThreads = 256;
static_assert(S % kTcNz == 0, "whole slabs");
static_assert(kTcFront + kTcPlane - kTcReach >= 0, "front guard");
static_assert(kTcFront + kTcPlane + 128 * kTcTiles + kTcReach <= kTcSpan, "back guard");
static_assert(16 * kTcTiles <= kTcCols, "accumulator columns");
static_assert(kTcPlaneBytes % 16 == 0 && (kTcPlaneBytes >> 4) < (1 << 14), "LBO field");
static_assert(3 * kTcSmem > 228 * 1024, "at most two CTAs per SM share the tensor memory");
// instruction descriptor, kind::f16: FP32 accumulator (bits 4-5 = 1), BF16
// A and B (bits 7-9, 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at
// bit 24
constexpr unsigned kTcIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((16u >> 3) << 17) |
                              ((128u >> 4) << 24);
// a wait gives up after this many SM cycles (about 2 s)
constexpr long long kTcWaitCycles = 4000000000ll;

__device__ __forceinline__ unsigned tc_smem(const void *p)
{
   return (unsigned)__cvta_generic_to_shared(p);
}

// shared-memory matrix descriptor: start, leading and stride byte offsets
// (16-byte units), descriptor version 1, no swizzle
__device__ __forceinline__ unsigned long long tc_desc(unsigned addr, unsigned lbo, unsigned sbo)
{
   return (unsigned long long)((addr >> 4) & 0x3FFFu) |
          ((unsigned long long)((lbo >> 4) & 0x3FFFu) << 16) |
          ((unsigned long long)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void tc_mma(unsigned d, unsigned long long a, unsigned long long b,
                                       unsigned idesc, unsigned accumulate)
{
   asm volatile(
      "{\n"
      " .reg .pred p;\n"
      " setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n"
      "}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ bool tc_try_wait(unsigned bar, unsigned parity)
{
   unsigned ok;
   asm volatile(
      "{\n"
      " .reg .pred p;\n"
      " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
   return ok != 0;
}

__device__ __forceinline__ void tc_ld16(unsigned taddr, unsigned *v)
{
   asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15}, [%16];\n"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
        "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
   asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// wt: [27][16 out][16 in] BF16.  mode 0: y = relu(acc); mode 1: y = acc *
// (gate > 0); mode 2 (layer 4, its weights padded to 16 output channels):
// yf = output channel 0 in FP32.  A wait that runs out sets *err and ends
// the CTA's work.
__global__ void __launch_bounds__(kTcThreads)
k_conv_mid_tc(const __nv_bfloat16 *__restrict__ x, const __nv_bfloat16 *__restrict__ wt,
              __nv_bfloat16 *__restrict__ y, const __nv_bfloat16 *__restrict__ gate,
              float *__restrict__ yf, long long nsamp, int mode, int *__restrict__ err)
{
   extern __shared__ __align__(128) unsigned char tsm[];
   uint4 *p0 = reinterpret_cast<uint4 *>(tsm);                   // channels 0..7
   uint4 *p1 = reinterpret_cast<uint4 *>(tsm + kTcPlaneBytes);   // channels 8..15
   unsigned char *ws = tsm + 2 * kTcPlaneBytes;
   unsigned long long *bar = reinterpret_cast<unsigned long long *>(ws + kTcWBytes);
   unsigned *tslot = reinterpret_cast<unsigned *>(bar + 1);
   const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

   // weights per tap as [in-channel half][out channel][8 in-channels]
   for (int i = tid; i < T * C * 2; i += kTcThreads) {
      const int half = i & 1, tco = i >> 1, t = tco / C, co = tco - t * C;
      *reinterpret_cast<uint4 *>(ws + t * 512 + half * 256 + co * 16) =
         *reinterpret_cast<const uint4 *>(wt + (size_t)tco * C + half * 8);
   }
   for (int i = tid; i < kTcSpan; i += kTcThreads) {
      p0[i] = make_uint4(0u, 0u, 0u, 0u);
      p1[i] = make_uint4(0u, 0u, 0u, 0u);
   }
   if (tid == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem(bar)) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
   }
   if (warp == 0) {
      asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                      tc_smem(tslot)),
                   "r"(kTcCols)
                   : "memory");
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
   }
   asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
   __syncthreads();
   asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
   const unsigned tmem = *tslot;
   const unsigned s0 = tc_smem(p0), s1 = tc_smem(p1), sw = tc_smem(ws), sb = tc_smem(bar);
   unsigned phase = 0;
   const long long nslab = nsamp * kTcSlabs;
   for (long long slab = blockIdx.x; slab < nslab; slab += gridDim.x) {
      const long long smp = slab / kTcSlabs;
      const int z0 = (int)(slab - smp * kTcSlabs) * kTcNz;
      const __nv_bfloat16 *xs = x + smp * (long long)S3 * C;
      for (int i = tid; i < kTcBox; i += kTcThreads) {
         const int zz = i / kTcPlane, r = i - zz * kTcPlane;
         const int py = r / kTcPx, px = r - py * kTcPx;
         const int cx = px - 1, cy = py - 1, cz = z0 - 1 + zz;
         uint4 lo = make_uint4(0u, 0u, 0u, 0u), hi = lo;
         if (cx >= 0 && cx < S && cy >= 0 && cy < S && cz >= 0 && cz < S) {
            const uint4 *src =
               reinterpret_cast<const uint4 *>(xs + ((long long)cx + S * (cy + S * cz)) * C);
            lo = src[0];
            hi = src[1];
         }
         p0[kTcFront + i] = lo;
         p1[kTcFront + i] = hi;
      }
      // the tensor cores read shared memory through the async proxy; the
      // previous slab's accumulator reads come before these MMAs
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
      if (tid == 0) {
         asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
         for (int i = 0; i < kTcTiles; ++i)
            for (int t = 0; t < T; ++t) {
               const int off = tap_dx(t) + kTcPx * tap_dy(t) + kTcPlane * tap_dz(t);
               const unsigned row = (unsigned)(kTcFront + kTcPlane + 128 * i + off);
               tc_mma(tmem + 16u * i, tc_desc(s0 + 16u * row, s1 - s0, 128u),
                      tc_desc(sw + 512u * t, 256u, 128u), kTcIdesc, t > 0 ? 1u : 0u);
            }
         asm volatile(
            "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(sb)
            : "memory");
      }
      bool ok = true;
      {
         const long long t0 = clock64();
         while (!tc_try_wait(sb, phase))
            if (clock64() - t0 > kTcWaitCycles) {
               ok = false;
               break;
            }
      }
      phase ^= 1u;
      if (!__syncthreads_and(ok)) {
         if (tid == 0) atomicExch(err, 1);
         break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int q = warp & 3;
      for (int i = warp >> 2; i < kTcTiles; i += kTcThreads / 128) {
         unsigned v[16];
         tc_ld16(tmem + ((unsigned)(32 * q) << 16) + 16u * i, v);
         const int r = kTcPlane + 128 * i + 32 * q + lane;  // padded box row
         const int zz = r / kTcPlane, rr = r - zz * kTcPlane;
         const int py = rr / kTcPx, px = rr - py * kTcPx;
         if (zz > kTcNz || px < 1 || px > S || py < 1 || py > S) continue;
         const long long cell =
            smp * S3 + (px - 1) + S * ((py - 1) + (long long)S * (z0 - 1 + zz));
         if (mode == 2) {
            yf[cell] = __uint_as_float(v[0]);
            continue;
         }
         float o[16];
#pragma unroll
         for (int c = 0; c < 16; ++c) o[c] = __uint_as_float(v[c]);
         if (mode == 0) {
#pragma unroll
            for (int c = 0; c < 16; ++c) o[c] = fmaxf(o[c], 0.f);
         } else {
            const uint4 *gp = reinterpret_cast<const uint4 *>(gate + cell * C);
            uint4 gg[2] = {gp[0], gp[1]};
            const __nv_bfloat16 *g = reinterpret_cast<const __nv_bfloat16 *>(gg);
#pragma unroll
            for (int c = 0; c < 16; ++c)
               if (!(__bfloat162float(g[c]) > 0.f)) o[c] = 0.f;
         }
         uint4 out[2];
         __nv_bfloat162 *ob = reinterpret_cast<__nv_bfloat162 *>(out);
#pragma unroll
         for (int c = 0; c < 8; ++c) ob[c] = __floats2bfloat162_rn(o[2 * c], o[2 * c + 1]);
         uint4 *dst = reinterpret_cast<uint4 *>(y + cell * C);
         dst[0] = out[0];
         dst[1] = out[1];
      }
   }
   // every accumulator read is done before the tensor memory is released
   asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
   __syncthreads();
   if (warp == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                   "r"(kTcCols)
                   : "memory");
   }
}

// masked MSE: dy = 2/m * mask * (y - target); loss += sum(mask*(y-target)^2)
__global__ void k_loss_grad(const float *__restrict__ y, const float *__restrict__ target,
                            const float *__restrict__ mask, float inv_m, float *__restrict__ dy,
                            double *__restrict__ loss, long long ncells)
{
   const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   double l = 0.0;
   if (cell < ncells) {
      const float d = (y[cell] - target[cell]) * mask[cell];
      dy[cell] = 2.f * inv_m * d;
      l = (double)d * (double)d;
   }
   for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
   if ((threadIdx.x & 31) == 0 && l != 0.0) atomicAdd(loss, l);
}

// data gradient through layer 4, gated by layer 3's ReLU
__global__ void k_bwd_out_data(const float *__restrict__ dy, const float *__restrict__ w4,
                               const __nv_bfloat16 *__restrict__ a3,
                               __nv_bfloat16 *__restrict__ d3, long long ncells)
{
   __shared__ float w[T * C];
   for (int i = threadIdx.x; i < T * C; i += blockDim.x)
      w[i] = __bfloat162float(__float2bfloat16_rn(w4[i]));
   __syncthreads();
   const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (cell >= ncells) return;
   int cx, cy, cz;
   cell_coords(cell, cx, cy, cz);
   float acc[C];
#pragma unroll
   for (int c = 0; c < C; ++c) acc[c] = 0.f;
   for (int t = 0; t < T; ++t) {
      // dx[cell] += w[t] * dy[cell - off_t]: the neighbour at the reversed tap
      const long long nb = neighbour(cell, cx, cy, cz, T - 1 - t);
      if (nb < 0) continue;
      const float g = dy[nb];
#pragma unroll
      for (int c = 0; c < C; ++c) acc[c] = __fmaf_rn(w[t * C + c], g, acc[c]);
   }
#pragma unroll
   for (int c = 0; c < C; c += 2) {
      const __nv_bfloat162 gg = *reinterpret_cast<const __nv_bfloat162 *>(a3 + cell * C + c);
      const float o0 = __bfloat162float(gg.x) > 0.f ? acc[c] : 0.f;
      const float o1 = __bfloat162float(gg.y) > 0.f ? acc[c + 1] : 0.f;
      *reinterpret_cast<__nv_bfloat162 *>(d3 + cell * C + c) = __floats2bfloat162_rn(o0, o1);
   }
}

// weight gradient of a 16 -> 16 layer: dw[t][ci][co] += sum over cells of
// x[cell + off_t][ci] * dy[cell][co].  Slabs as in k_conv_mid_tc: the
// slab's input box (zero halo) and the gradient at its output rows (zero at
// the halo rows) are staged in shared memory in channel planes of 16 bytes
// per cell; warp w owns taps 3w .. 3w + 2 (one x-row of taps) and multiplies
// A = x^T (16 in-channels x 16 cells, ldmatrix.trans at the tap's shifted
// rows) by B = dy (16 cells x 8 out-channels, ldmatrix.trans) with
// mma.sync m16n8k16 over every 16 rows of the slab.  The tensor cores'
// tcgen05 form needs M >= 64 output rows, and with 16 x 16 outputs per tap
// and the tap as a row shift no operand layout gives that.  Each CTA sums
// its slabs in registers and adds them once.
constexpr int kWgWarps = T / 3;                      // 9 warps, 3 taps each
constexpr int kWgThreads = 32 * kWgWarps;
constexpr int kWgRows = 128 * kTcTiles;              // output rows per slab
constexpr int kWgSmem = 2 * kTcPlaneBytes + 2 * kWgRows * 16;
static_assert(T % 3 == 0, "three taps per warp");
static_assert(kWgRows % 16 == 0, "whole k-steps");
static_assert(kTcFront + kTcPlane + kWgRows + kTcReach <= kTcSpan, "x rows in the box");

__device__ __forceinline__ void ldm_x4_trans(unsigned addr, uint32_t *r)
{
   asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0, %1, %2, %3}, [%4];\n"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                : "r"(addr));
}

__global__ void __launch_bounds__(kWgThreads)
k_bwd_weight_mid(const __nv_bfloat16 *__restrict__ x, const __nv_bfloat16 *__restrict__ dy,
                 float *__restrict__ dw, long long nsamp)
{
   extern __shared__ __align__(128) unsigned char wsm[];
   uint4 *x0 = reinterpret_cast<uint4 *>(wsm);
   uint4 *x1 = reinterpret_cast<uint4 *>(wsm + kTcPlaneBytes);
   uint4 *g0 = reinterpret_cast<uint4 *>(wsm + 2 * kTcPlaneBytes);
   uint4 *g1 = g0 + kWgRows;
   const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
   for (int i = tid; i < kTcSpan; i += kWgThreads) {
      x0[i] = make_uint4(0u, 0u, 0u, 0u);
      x1[i] = make_uint4(0u, 0u, 0u, 0u);
   }
   const unsigned sx0 = tc_smem(x0), sx1 = tc_smem(x1), sg0 = tc_smem(g0), sg1 = tc_smem(g1);
   // ldmatrix.x4: lanes 8j .. 8j + 7 give the rows of matrix j
   const int mrow = lane & 7, mj = lane >> 3;
   float acc[3][2][4];
#pragma unroll
   for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b)
#pragma unroll
         for (int c = 0; c < 4; ++c) acc[a][b][c] = 0.f;
   int off[3];
#pragma unroll
   for (int a = 0; a < 3; ++a) {
      const int t = 3 * warp + a;
      off[a] = tap_dx(t) + kTcPx * tap_dy(t) + kTcPlane * tap_dz(t);
   }
   const long long nslab = nsamp * kTcSlabs;
   for (long long slab = blockIdx.x; slab < nslab; slab += gridDim.x) {
      const long long smp = slab / kTcSlabs;
      const int z0 = (int)(slab - smp * kTcSlabs) * kTcNz;
      const __nv_bfloat16 *xs = x + smp * (long long)S3 * C;
      const __nv_bfloat16 *gs = dy + smp * (long long)S3 * C;
      __syncthreads();  // the previous slab's reads are done
      for (int i = tid; i < kTcBox; i += kWgThreads) {
         const int zz = i / kTcPlane, r = i - zz * kTcPlane;
         const int py = r / kTcPx, px = r - py * kTcPx;
         const int cx = px - 1, cy = py - 1, cz = z0 - 1 + zz;
         uint4 lo = make_uint4(0u, 0u, 0u, 0u), hi = lo;
         if (cx >= 0 && cx < S && cy >= 0 && cy < S && cz >= 0 && cz < S) {
            const uint4 *src =
               reinterpret_cast<const uint4 *>(xs + ((long long)cx + S * (cy + S * cz)) * C);
            lo = src[0];
            hi = src[1];
         }
         x0[kTcFront + i] = lo;
         x1[kTcFront + i] = hi;
      }
      for (int i = tid; i < kWgRows; i += kWgThreads) {
         const int rr = kTcPlane + i;  // padded box row of output row i
         const int zz = rr / kTcPlane, r = rr - zz * kTcPlane;
         const int py = r / kTcPx, px = r - py * kTcPx;
         uint4 lo = make_uint4(0u, 0u, 0u, 0u), hi = lo;
         if (zz <= kTcNz && px >= 1 && px <= S && py >= 1 && py <= S) {
            const uint4 *src = reinterpret_cast<const uint4 *>(
               gs + ((long long)(px - 1) + S * ((py - 1) + (long long)S * (z0 - 1 + zz))) * C);
            lo = src[0];
            hi = src[1];
         }
         g0[i] = lo;
         g1[i] = hi;
      }
      __syncthreads();
      for (int k0 = 0; k0 < kWgRows; k0 += 16) {
         // B: dy rows k0 .. k0 + 15; matrices (co 0-7, rows +0), (co 0-7,
         // rows +8), (co 8-15, rows +0), (co 8-15, rows +8)
         uint32_t b[4];
         {
            const unsigned base = (mj >> 1) ? sg1 : sg0;
            ldm_x4_trans(base + 16u * (unsigned)(k0 + 8 * (mj & 1) + mrow), b);
         }
#pragma unroll
         for (int a = 0; a < 3; ++a) {
            // A = x^T at the tap's rows: matrices (ci 0-7, rows +0),
            // (ci 8-15, rows +0), (ci 0-7, rows +8), (ci 8-15, rows +8)
            uint32_t av[4];
            const unsigned base = (mj & 1) ? sx1 : sx0;
            const int row = kTcFront + kTcPlane + k0 + off[a] + 8 * (mj >> 1) + mrow;
            ldm_x4_trans(base + 16u * (unsigned)row, av);
            mma_bf16(acc[a][0], av, b[0], b[1]);
            mma_bf16(acc[a][1], av, b[2], b[3]);
         }
      }
   }
   const int g = lane >> 2, q = lane & 3;
#pragma unroll
   for (int a = 0; a < 3; ++a) {
      const int t = 3 * warp + a;
#pragma unroll
      for (int j = 0; j < 2; ++j) {
         const int co = 8 * j + 2 * q;
         atomicAdd(&dw[(t * C + g) * C + co], acc[a][j][0]);
         atomicAdd(&dw[(t * C + g) * C + co + 1], acc[a][j][1]);
         atomicAdd(&dw[(t * C + g + 8) * C + co], acc[a][j][2]);
         atomicAdd(&dw[(t * C + g + 8) * C + co + 1], acc[a][j][3]);
      }
   }
}

// Weight gradients of layers 1 and 4 from staged slabs (the slabs of
// k_conv_mid_tc), on the FP32 cores with fused multiply-adds (the network's
// arithmetic needs no particular rounding): thread (tap t, row group g)
// sums rows g, g + kSgGroups, ... of the slab's output rows into 16
// accumulators, and each CTA adds its sums once after all its slabs.
//   layer 1: dw1[t][co] += sum_cells x0[cell + off_t] * d1[cell][co]
//   layer 4: dw4[t][ci] += sum_cells a3[cell + off_t][ci] * dy[cell]
constexpr int kSgGroups = 8;
constexpr int kSgThreads = T * kSgGroups;            // 216
constexpr int kSgInSmem = kTcSpan * 4 + kWgRows * 32;
constexpr int kSgOutSmem = kTcSpan * 32 + kWgRows * 4;

// padded box row i of the slab (z0, sample base) -> cell index in the
// sample, or -1 outside it
__device__ __forceinline__ int slab_box_cell(int i, int z0)
{
   const int zz = i / kTcPlane, r = i - zz * kTcPlane;
   const int py = r / kTcPx, px = r - py * kTcPx;
   const int cx = px - 1, cy = py - 1, cz = z0 - 1 + zz;
   if (cx < 0 || cx >= S || cy < 0 || cy >= S || cz < 0 || cz >= S) return -1;
   return cx + S * (cy + S * cz);
}

// output row i of the slab -> cell index in the sample, or -1 (halo row)
__device__ __forceinline__ int slab_out_cell(int i, int z0)
{
   const int rr = kTcPlane + i;
   const int zz = rr / kTcPlane, r = rr - zz * kTcPlane;
   const int py = r / kTcPx, px = r - py * kTcPx;
   if (zz > kTcNz || px < 1 || px > S || py < 1 || py > S) return -1;
   return (px - 1) + S * ((py - 1) + S * (z0 - 1 + zz));
}

__global__ void __launch_bounds__(kSgThreads)
k_bwd_weight_in(const __nv_bfloat16 *__restrict__ x0, const __nv_bfloat16 *__restrict__ d1,
                float *__restrict__ dw1, long long nsamp)
{
   extern __shared__ __align__(128) unsigned char ssm[];
   float *xs = reinterpret_cast<float *>(ssm);                       // kTcSpan
   uint4 *ds = reinterpret_cast<uint4 *>(ssm + kTcSpan * 4);         // 2 per row
   const int tid = threadIdx.x, t = tid / kSgGroups, g = tid - t * kSgGroups;
   const int off = tap_dx(t) + kTcPx * tap_dy(t) + kTcPlane * tap_dz(t);
   for (int i = tid; i < kTcSpan; i += kSgThreads) xs[i] = 0.f;
   float acc[C];
#pragma unroll
   for (int c = 0; c < C; ++c) acc[c] = 0.f;
   const long long nslab = nsamp * kTcSlabs;
   for (long long slab = blockIdx.x; slab < nslab; slab += gridDim.x) {
      const long long smp = slab / kTcSlabs;
      const int z0 = (int)(slab - smp * kTcSlabs) * kTcNz;
      __syncthreads();
      for (int i = tid; i < kTcBox; i += kSgThreads) {
         const int cell = slab_box_cell(i, z0);
         xs[kTcFront + i] = cell >= 0 ? __bfloat162float(x0[smp * S3 + cell]) : 0.f;
      }
      for (int i = tid; i < kWgRows; i += kSgThreads) {
         const int cell = slab_out_cell(i, z0);
         uint4 lo = make_uint4(0u, 0u, 0u, 0u), hi = lo;
         if (cell >= 0) {
            const uint4 *src = reinterpret_cast<const uint4 *>(d1 + (smp * S3 + cell) * C);
            lo = src[0];
            hi = src[1];
         }
         ds[2 * i] = lo;
         ds[2 * i + 1] = hi;
      }
      __syncthreads();
      for (int k = g; k < kWgRows; k += kSgGroups) {
         const float xv = xs[kTcFront + kTcPlane + k + off];
         uint4 dd[2] = {ds[2 * k], ds[2 * k + 1]};
         const __nv_bfloat16 *dv = reinterpret_cast<const __nv_bfloat16 *>(dd);
#pragma unroll
         for (int c = 0; c < C; ++c) acc[c] = __fmaf_rn(xv, __bfloat162float(dv[c]), acc[c]);
      }
   }
#pragma unroll
   for (int c = 0; c < C; ++c) atomicAdd(&dw1[t * C + c], acc[c]);
}

__global__ void __launch_bounds__(kSgThreads)
k_bwd_weight_out(const __nv_bfloat16 *__restrict__ a3, const float *__restrict__ dy,
                 float *__restrict__ dw4, long long nsamp)
{
   extern __shared__ __align__(128) unsigned char ssm[];
   uint4 *as = reinterpret_cast<uint4 *>(ssm);                       // 2 per cell
   float *ys = reinterpret_cast<float *>(ssm + kTcSpan * 32);        // kWgRows
   const int tid = threadIdx.x, t = tid / kSgGroups, g = tid - t * kSgGroups;
   const int off = tap_dx(t) + kTcPx * tap_dy(t) + kTcPlane * tap_dz(t);
   for (int i = tid; i < 2 * kTcSpan; i += kSgThreads) as[i] = make_uint4(0u, 0u, 0u, 0u);
   float acc[C];
#pragma unroll
   for (int c = 0; c < C; ++c) acc[c] = 0.f;
   const long long nslab = nsamp * kTcSlabs;
   for (long long slab = blockIdx.x; slab < nslab; slab += gridDim.x) {
      const long long smp = slab / kTcSlabs;
      const int z0 = (int)(slab - smp * kTcSlabs) * kTcNz;
      __syncthreads();
      for (int i = tid; i < kTcBox; i += kSgThreads) {
         const int cell = slab_box_cell(i, z0);
         uint4 lo = make_uint4(0u, 0u, 0u, 0u), hi = lo;
         if (cell >= 0) {
            const uint4 *src = reinterpret_cast<const uint4 *>(a3 + (smp * S3 + cell) * C);
            lo = src[0];
            hi = src[1];
         }
         as[2 * (kTcFront + i)] = lo;
         as[2 * (kTcFront + i) + 1] = hi;
      }
      for (int i = tid; i < kWgRows; i += kSgThreads) {
         const int cell = slab_out_cell(i, z0);
         ys[i] = cell >= 0 ? dy[smp * S3 + cell] : 0.f;
      }
      __syncthreads();
      for (int k = g; k < kWgRows; k += kSgGroups) {
         const float yv = ys[k];
         const int row = kTcFront + kTcPlane + k + off;
         uint4 aa[2] = {as[2 * row], as[2 * row + 1]};
         const __nv_bfloat16 *av = reinterpret_cast<const __nv_bfloat16 *>(aa);
#pragma unroll
         for (int c = 0; c < C; ++c) acc[c] = __fmaf_rn(__bfloat162float(av[c]), yv, acc[c]);
      }
   }
#pragma unroll
   for (int c = 0; c < C; ++c) atomicAdd(&dw4[t * C + c], acc[c]);
}

// BF16 copies of the 16 -> 16 weights: forward [t][co][ci] and data-gradient
// [t'][ci][co] with t' = 26 - t.
__global__ void k_pack_mid(const float *__restrict__ w, __nv_bfloat16 *__restrict__ wf,
                           __nv_bfloat16 *__restrict__ wd)
{
   const int i = blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= T * C * C) return;
   const int t = i / (C * C), ci = (i / C) % C, co = i % C;
   const __nv_bfloat16 v = __float2bfloat16_rn(w[i]);
   wf[(t * C + co) * C + ci] = v;
   wd[((T - 1 - t) * C + ci) * C + co] = v;
}

// BF16 copy of the 16 -> 1 weights as a 16 -> 16 block [t][co][ci] whose
// output channels 1..15 are zero (layer 4 on the tensor-core kernel)
__global__ void k_pack_out(const float *__restrict__ w4, __nv_bfloat16 *__restrict__ wo)
{
   const int i = blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= T * C * C) return;
   const int t = i / (C * C), co = (i / C) % C, ci = i % C;
   wo[i] = __float2bfloat16_rn(co == 0 ? w4[t * C + ci] : 0.f);
}

__global__ void k_round_bf16(const float *__restrict__ w, float *__restrict__ wr, int n)
{
   const int i = blockIdx.x * blockDim.x + threadIdx.x;
   if (i < n) wr[i] = __bfloat162float(__float2bfloat16_rn(w[i]));
}

__global__ void k_adam(float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2)
{
   const int i = blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= n) return;
   const float gi = g[i];
   const float mi = b1 * m[i] + (1.f - b1) * gi;
   const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
   m[i] = mi;
   v[i] = vi;
   w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

__global__ void k_to_bf16(const float *__restrict__ x, __nv_bfloat16 *__restrict__ y, long long n)
{
   const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (i < n) y[i] = __float2bfloat16_rn(x[i]);
}

thread_local std::string t_cnn_error;

}  // namespace

// ---------------------------------------------------------------------------
// network object
// ---------------------------------------------------------------------------

struct fac_cnn {
   int device = 0;
   int max_batch = 0;
   cudaStream_t stream = nullptr;
   // FP32 masters, Adam moments and gradients: w1 [27*16], w2, w3 [27*16*16], w4 [27*16]
   float *w[4] = {nullptr}, *gw[4] = {nullptr}, *m[4] = {nullptr}, *v[4] = {nullptr};
   float *w1r = nullptr;                 // BF16-rounded w1 for the first layer
   __nv_bfloat16 *wf[2] = {nullptr}, *wd[2] = {nullptr};  // layers 2, 3
   __nv_bfloat16 *wo = nullptr;          // layer 4 padded to 16 x 16 per tap
   __nv_bfloat16 *x0 = nullptr, *a[3] = {nullptr}, *d[3] = {nullptr};
   float *y = nullptr, *dy = nullptr;
   double *loss = nullptr;
   int *kerr = nullptr;                  // set by a tensor-core wait that ran out
   int tc_grid = 0;                      // CTAs of k_conv_mid_tc (two per SM)
   int steps = 0;
   std::vector<void *> allocs;
};

namespace {

const int kSizes[4] = {T * C, T * C * C, T * C * C, T * C};

#define CNN_CHECK(x)                                                                \
   do {                                                                             \
      cudaError_t _e = (x);                                                         \
      if (_e != cudaSuccess) {                                                      \
         t_cnn_error = std::string(#x) + ": " + cudaGetErrorString(_e);             \
         return FAC_ERR_CUDA;                                                       \
      }                                                                             \
   } while (0)

template <class P>
int dalloc(fac_cnn *n, P **p, size_t bytes)
{
   cudaError_t e = cudaMalloc((void **)p, bytes);
   if (e != cudaSuccess) {
      t_cnn_error = std::string("cudaMalloc: ") + cudaGetErrorString(e);
      return FAC_ERR_NOMEM;
   }
   n->allocs.push_back((void *)*p);
   return FAC_OK;
}

int pack(fac_cnn *n)
{
   for (int l = 0; l < 2; ++l) {
      k_pack_mid<<<(T * C * C + 255) / 256, 256, 0, n->stream>>>(n->w[l + 1], n->wf[l], n->wd[l]);
   }
   k_round_bf16<<<(T * C + 127) / 128, 128, 0, n->stream>>>(n->w[0], n->w1r, T * C);
   k_pack_out<<<(T * C * C + 255) / 256, 256, 0, n->stream>>>(n->w[3], n->wo);
   samrai_b200::add_kernel_launches(4);
   CNN_CHECK(cudaGetLastError());
   return FAC_OK;
}

void conv_mid(fac_cnn *n, const __nv_bfloat16 *x, const __nv_bfloat16 *wt, __nv_bfloat16 *y,
              const __nv_bfloat16 *gate, long long nsamp, int mode, cudaStream_t st,
              float *yf = nullptr)
{
   const long long slabs = nsamp * kTcSlabs;
   const unsigned grid = (unsigned)std::min<long long>(slabs, n->tc_grid);
   k_conv_mid_tc<<<grid, kTcThreads, kTcSmem, st>>>(x, wt, y, gate, yf, nsamp, mode, n->kerr);
}

void weight_mid(fac_cnn *n, const __nv_bfloat16 *x, const __nv_bfloat16 *dy, float *dw,
                long long nsamp)
{
   const long long slabs = nsamp * kTcSlabs;
   const unsigned grid = (unsigned)std::min<long long>(slabs, n->tc_grid);
   k_bwd_weight_mid<<<grid, kWgThreads, kWgSmem, n->stream>>>(x, dy, dw, nsamp);
}

// the device error flag, after the stream has drained
int device_status(fac_cnn *n)
{
   int e = 0;
   CNN_CHECK(cudaMemcpyAsync(&e, n->kerr, sizeof(int), cudaMemcpyDeviceToHost, n->stream));
   CNN_CHECK(cudaStreamSynchronize(n->stream));
   if (e) {
      t_cnn_error = "a tensor-core wait ran out (k_conv_mid_tc)";
      return FAC_ERR_DEVICE;
   }
   return FAC_OK;
}

int forward_on(fac_cnn *n, const float *x, long long nsamp, cudaStream_t st)
{
   const long long cells = nsamp * S3;
   const int tb = 256;
   const unsigned gb = (unsigned)((cells + tb - 1) / tb);
   k_to_bf16<<<gb, tb, 0, st>>>(x, n->x0, cells);
   k_conv_in<<<gb, tb, 0, st>>>(n->x0, n->w1r, n->a[0], cells);
   conv_mid(n, n->a[0], n->wf[0], n->a[1], nullptr, nsamp, 0, st);
   conv_mid(n, n->a[1], n->wf[1], n->a[2], nullptr, nsamp, 0, st);
   conv_mid(n, n->a[2], n->wo, nullptr, nullptr, nsamp, 2, st, n->y);
   samrai_b200::add_kernel_launches(5);
   CNN_CHECK(cudaGetLastError());
   return FAC_OK;
}

int forward(fac_cnn *n, const float *x, long long nsamp)
{
   return forward_on(n, x, nsamp, n->stream);
}

int backward(fac_cnn *n, const float *target, const float *mask, long long nsamp, float inv_m)
{
   const long long cells = nsamp * S3;
   const int tb = 256;
   const unsigned gb = (unsigned)((cells + tb - 1) / tb);
   for (int l = 0; l < 4; ++l)
      CNN_CHECK(cudaMemsetAsync(n->gw[l], 0, kSizes[l] * sizeof(float), n->stream));
   CNN_CHECK(cudaMemsetAsync(n->loss, 0, sizeof(double), n->stream));
   k_loss_grad<<<gb, tb, 0, n->stream>>>(n->y, target, mask, inv_m, n->dy, n->loss, cells);
   const unsigned sg = (unsigned)std::min<long long>(nsamp * kTcSlabs, n->tc_grid);
   k_bwd_weight_out<<<sg, kSgThreads, kSgOutSmem, n->stream>>>(n->a[2], n->dy, n->gw[3], nsamp);
   k_bwd_out_data<<<gb, tb, 0, n->stream>>>(n->dy, n->w[3], n->a[2], n->d[2], cells);
   weight_mid(n, n->a[1], n->d[2], n->gw[2], nsamp);
   conv_mid(n, n->d[2], n->wd[1], n->d[1], n->a[1], nsamp, 1, n->stream);
   weight_mid(n, n->a[0], n->d[1], n->gw[1], nsamp);
   conv_mid(n, n->d[1], n->wd[0], n->d[0], n->a[0], nsamp, 1, n->stream);
   k_bwd_weight_in<<<sg, kSgThreads, kSgInSmem, n->stream>>>(n->x0, n->d[0], n->gw[0], nsamp);
   samrai_b200::add_kernel_launches(8);
   CNN_CHECK(cudaGetLastError());
   return FAC_OK;
}

int check_batch(fac_cnn *n, long long nsamp)
{
   if (!n) {
      t_cnn_error = "null network";
      return FAC_ERR_ARG;
   }
   if (nsamp < 1 || nsamp > n->max_batch) {
      t_cnn_error = "batch size out of range";
      return FAC_ERR_ARG;
   }
   return FAC_OK;
}

}  // namespace

namespace samrai_b200 {
// Forward pass on the caller's stream (used inside the FAC cycle); *y points
// at the network's output buffer (nsamp * S^3 floats).
int cnn_forward_on_stream(fac_cnn *n, const float *x, long long nsamp, cudaStream_t st,
                          const float **y)
{
   int rc = check_batch(n, nsamp);
   if (rc) return rc;
   rc = forward_on(n, x, nsamp, st);
   if (y) *y = n->y;
   return rc;
}
int cnn_max_batch(const fac_cnn *n) { return n ? n->max_batch : 0; }
int cnn_device(const fac_cnn *n) { return n ? n->device : -1; }
}  // namespace samrai_b200

extern "C" {

const char *fac_cnn_last_error(void) { return t_cnn_error.c_str(); }

int fac_cnn_create(fac_cnn **out, int device, int max_batch, unsigned long long seed)
{
   if (!out || max_batch < 1) {
      t_cnn_error = "bad arguments";
      return FAC_ERR_ARG;
   }
   CNN_CHECK(cudaSetDevice(device));
   fac_cnn *n = new fac_cnn();
   n->device = device;
   n->max_batch = max_batch;
   int rc = FAC_OK;
   auto fail = [&](int r) {
      for (void *p : n->allocs) cudaFree(p);
      delete n;
      return r;
   };
   if (cudaStreamCreateWithFlags(&n->stream, cudaStreamNonBlocking) != cudaSuccess)
      return fail(FAC_ERR_CUDA);
   const long long cells = (long long)max_batch * S3;
   for (int l = 0; l < 4; ++l) {
      if ((rc = dalloc(n, &n->w[l], kSizes[l] * sizeof(float))) ||
          (rc = dalloc(n, &n->gw[l], kSizes[l] * sizeof(float))) ||
          (rc = dalloc(n, &n->m[l], kSizes[l] * sizeof(float))) ||
          (rc = dalloc(n, &n->v[l], kSizes[l] * sizeof(float))))
         return fail(rc);
   }
   if ((rc = dalloc(n, &n->w1r, T * C * sizeof(float))) ||
       (rc = dalloc(n, &n->wo, T * C * C * 2)))
      return fail(rc);
   for (int l = 0; l < 2; ++l)
      if ((rc = dalloc(n, &n->wf[l], T * C * C * 2)) || (rc = dalloc(n, &n->wd[l], T * C * C * 2)))
         return fail(rc);
   if ((rc = dalloc(n, &n->x0, cells * 2))) return fail(rc);
   for (int l = 0; l < 3; ++l)
      if ((rc = dalloc(n, &n->a[l], cells * C * 2)) || (rc = dalloc(n, &n->d[l], cells * C * 2)))
         return fail(rc);
   if ((rc = dalloc(n, &n->y, cells * 4)) || (rc = dalloc(n, &n->dy, cells * 4)) ||
       (rc = dalloc(n, &n->loss, sizeof(double))) || (rc = dalloc(n, &n->kerr, sizeof(int))))
      return fail(rc);
   int sms = 0;
   if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
       cudaFuncSetAttribute(k_conv_mid_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            kTcSmem) != cudaSuccess ||
       cudaFuncSetAttribute(k_bwd_weight_mid, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            kWgSmem) != cudaSuccess ||
       cudaFuncSetAttribute(k_bwd_weight_out, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            kSgOutSmem) != cudaSuccess ||
       cudaFuncSetAttribute(k_bwd_weight_in, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            kSgInSmem) != cudaSuccess)
      return fail(FAC_ERR_CUDA);
   n->tc_grid = 2 * sms;
   if (cudaMemsetAsync(n->kerr, 0, sizeof(int), n->stream) != cudaSuccess)
      return fail(FAC_ERR_CUDA);
   // He initialisation from a seeded host generator (splitmix64 + Box-Muller)
   unsigned long long st = seed * 0x9E3779B97F4A7C15ull + 1;
   auto next = [&]() {
      st += 0x9E3779B97F4A7C15ull;
      unsigned long long z = st;
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
      return ((z ^ (z >> 31)) >> 11) * (1.0 / 9007199254740992.0);
   };
   const int fan_in[4] = {T, T * C, T * C, T * C};
   for (int l = 0; l < 4; ++l) {
      std::vector<float> h(kSizes[l]);
      const double sd = std::sqrt(2.0 / fan_in[l]);
      for (auto &x : h) {
         const double u1 = next() + 1e-300, u2 = next();
         x = (float)(sd * std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2));
      }
      if (l == 3)
         for (auto &x : h) x *= 0.1f;  // start close to a zero correction
      CNN_CHECK(cudaMemcpyAsync(n->w[l], h.data(), kSizes[l] * 4, cudaMemcpyHostToDevice,
                                n->stream));
      CNN_CHECK(cudaMemsetAsync(n->m[l], 0, kSizes[l] * 4, n->stream));
      CNN_CHECK(cudaMemsetAsync(n->v[l], 0, kSizes[l] * 4, n->stream));
   }
   if ((rc = pack(n))) return fail(rc);
   CNN_CHECK(cudaStreamSynchronize(n->stream));
   *out = n;
   return FAC_OK;
}

int fac_cnn_destroy(fac_cnn *n)
{
   if (!n) return FAC_OK;
   cudaSetDevice(n->device);
   cudaStreamSynchronize(n->stream);
   for (void *p : n->allocs) cudaFree(p);
   cudaStreamDestroy(n->stream);
   delete n;
   return FAC_OK;
}

int fac_cnn_set_weights(fac_cnn *n, const float *w1, const float *w2, const float *w3,
                        const float *w4)
{
   if (!n || !w1 || !w2 || !w3 || !w4) {
      t_cnn_error = "null argument";
      return FAC_ERR_ARG;
   }
   const float *src[4] = {w1, w2, w3, w4};
   for (int l = 0; l < 4; ++l)
      CNN_CHECK(cudaMemcpyAsync(n->w[l], src[l], kSizes[l] * 4, cudaMemcpyHostToDevice,
                                n->stream));
   int rc = pack(n);
   if (rc) return rc;
   CNN_CHECK(cudaStreamSynchronize(n->stream));
   return FAC_OK;
}

int fac_cnn_get_weights(fac_cnn *n, float *w1, float *w2, float *w3, float *w4)
{
   if (!n || !w1 || !w2 || !w3 || !w4) {
      t_cnn_error = "null argument";
      return FAC_ERR_ARG;
   }
   float *dst[4] = {w1, w2, w3, w4};
   for (int l = 0; l < 4; ++l)
      CNN_CHECK(cudaMemcpyAsync(dst[l], n->w[l], kSizes[l] * 4, cudaMemcpyDeviceToHost,
                                n->stream));
   CNN_CHECK(cudaStreamSynchronize(n->stream));
   return FAC_OK;
}

int fac_cnn_forward(fac_cnn *n, const float *x, long long nsamp, float *y)
{
   int rc = check_batch(n, nsamp);
   if (rc) return rc;
   if (!x || !y) {
      t_cnn_error = "null argument";
      return FAC_ERR_ARG;
   }
   if ((rc = forward(n, x, nsamp))) return rc;
   CNN_CHECK(cudaMemcpyAsync(y, n->y, nsamp * S3 * sizeof(float), cudaMemcpyDeviceToDevice,
                             n->stream));
   return device_status(n);
}

int fac_cnn_gradients(fac_cnn *n, const float *x, const float *target, const float *mask,
                      long long nsamp, double *loss, float *g1, float *g2, float *g3, float *g4)
{
   int rc = check_batch(n, nsamp);
   if (rc) return rc;
   if (!x || !target || !mask) {
      t_cnn_error = "null argument";
      return FAC_ERR_ARG;
   }
   std::vector<float> hm(nsamp * S3);
   CNN_CHECK(cudaMemcpyAsync(hm.data(), mask, hm.size() * 4, cudaMemcpyDeviceToHost, n->stream));
   CNN_CHECK(cudaStreamSynchronize(n->stream));
   double msum = 0;
   for (float v : hm) msum += v;
   if (msum <= 0) {
      t_cnn_error = "empty mask";
      return FAC_ERR_ARG;
   }
   if ((rc = forward(n, x, nsamp))) return rc;
   if ((rc = backward(n, target, mask, nsamp, (float)(1.0 / msum)))) return rc;
   double l = 0;
   CNN_CHECK(cudaMemcpyAsync(&l, n->loss, sizeof(double), cudaMemcpyDeviceToHost, n->stream));
   float *dst[4] = {g1, g2, g3, g4};
   for (int k = 0; k < 4; ++k)
      if (dst[k])
         CNN_CHECK(cudaMemcpyAsync(dst[k], n->gw[k], kSizes[k] * 4, cudaMemcpyDeviceToHost,
                                   n->stream));
   if ((rc = device_status(n))) return rc;
   if (loss) *loss = l / msum;
   return FAC_OK;
}

int fac_cnn_train_step(fac_cnn *n, const float *x, const float *target, const float *mask,
                       long long nsamp, double mask_sum, float lr, double *loss)
{
   int rc = check_batch(n, nsamp);
   if (rc) return rc;
   if (!x || !target || !mask || !(mask_sum > 0)) {
      t_cnn_error = "bad arguments";
      return FAC_ERR_ARG;
   }
   if ((rc = forward(n, x, nsamp))) return rc;
   if ((rc = backward(n, target, mask, nsamp, (float)(1.0 / mask_sum)))) return rc;
   n->steps += 1;
   const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
   const float c1 = 1.f - std::pow(b1, (float)n->steps), c2 = 1.f - std::pow(b2, (float)n->steps);
   for (int l = 0; l < 4; ++l)
      k_adam<<<(kSizes[l] + 255) / 256, 256, 0, n->stream>>>(n->w[l], n->gw[l], n->m[l], n->v[l],
                                                              kSizes[l], lr, b1, b2, eps, c1, c2);
   samrai_b200::add_kernel_launches(4);
   if ((rc = pack(n))) return rc;
   if (loss) {
      double l = 0;
      CNN_CHECK(cudaMemcpyAsync(&l, n->loss, sizeof(double), cudaMemcpyDeviceToHost, n->stream));
      if ((rc = device_status(n))) return rc;
      *loss = l / mask_sum;
   }
   return FAC_OK;
}

}  // extern "C"

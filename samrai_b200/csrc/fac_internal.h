// Internal types shared by the host-side table builder and the CUDA kernels.
//
// Device layout of one level (all problems of a context concatenated, then
// patches in order): every cell field of ghost width g is one buffer holding
// each patch's array over its ghosted box (pdat::ArrayData layout, i
// fastest); side fields hold per patch the side arrays of axes 0..dim-1;
// outer-side fields hold per patch, axis and side (lower, upper) the face
// arrays.  The per-problem slice of a level buffer is contiguous and equals
// the host layout of fac_upload_field / fac_download_field.
#pragma once

#include <cstdint>

namespace samrai_b200 {

constexpr int kMaxLevels = 8;
constexpr int kChunk = 1024;  // cells per work chunk of the cell kernels
constexpr int kSpanChunk = 2048;  // cells per chunk of the Krylov vector kernels
// Largest refinement ratio per axis: the prolongation tabulates its
// interpolation offsets per chunk in shared memory.
constexpr int kProlongRatioMax = 16;

// One patch of a (batched) level.
struct PatchDesc {
   int lo[3], hi[3];
   int prob;           // problem index within the context
   int flags;          // bit0: has coarse-fine boundary faces; bit1: has faces
                       // that take a coarsened finer-level flux
   // ceil(2^32 / nx), ceil(2^32 / ny) for the cell decode of a linear
   // index (exact while cells * max(nx, ny) < 2^32); 0: divide instead
   unsigned mx, my;
   long long off1;     // start of this patch in ghost-1 cell buffers
   long long off0;     // start in ghost-0 cell buffers
   long long offs[3];  // start of the side array of each axis
   long long offo[3][2];  // start of the outer-side array of axis a, side s
   double dx[3];
};

// Chunk of work over one patch: cells [begin, begin+count) of a
// linearisation chosen by the kernel that consumes it.  Transaction lists
// (fills, restriction, flux coarsening, prolongation) pack small items of
// one problem into one chunk: then patch is the first item, aux > 1 the
// number of items and the chunk covers their cells back to back (a list's
// item prefix sums give each item's first cell).
struct Chunk {
   int patch;
   int begin;
   int count;
   int aux;
};

// A work list that is compacted on the device: `all` holds the full list
// (chunks in problem order, problem p owning [pcb[p], pcb[p+1])), `list` the
// chunks of the active problems followed by end markers (patch = -1).
struct WorkReg {
   const Chunk *all;
   Chunk *list;
   const int *pcb;
   int n;
   int pad;
};

// Array descriptor: element (i,j,k) of the box lo..lo+n-1 lives at
// base + (i-lo0) + n0*((j-lo1) + n1*(k-lo2)).
struct ArrDesc {
   long long base;
   int lo[3];
   int n[3];
};

enum FillKind : int {
   kFillCopy = 0,     // dst(c) = src(c)
   kFillCoarse = 1,   // dst(c) = src(coarsen(c))   (constant refine)
   kFillBc = 2        // physical boundary value from src(c moved inward)
};

// One ghost-fill transaction over a box of destination cells.
struct FillItem {
   int kind;
   int prob;
   int lo[3], hi[3];    // destination cells
   int side[3];         // kFillBc: -1/0/+1 outside direction per axis
   int ratio[3];        // kFillCoarse
   ArrDesc dst;
   ArrDesc src;
   double h[3];         // kFillBc: grid spacing of the destination
   int src_is_coarse;   // read from the coarser level's buffer
   int bc_level;        // kFillBc: level whose boundary coefficients apply
};

// A coarse-fine boundary face of a patch (Ewing fix-up).
struct CfFace {
   long long cell;     // interior cell next to the face (ghost-1 buffer)
   long long mirror;   // the other fine cell of the same coarse cell
   long long ghost;    // ghost cell across the face
   long long oidx;     // index in the outer-side buffers
   long long sidx;     // index in the side buffers
   int patch;
   int axis;
   int side;           // 0 lower, 1 upper
   int pad;
};

// Flux coarsening: coarse faces of one coarse patch fed by one fine patch's
// outer-side flux (CartesianOutersideDoubleWeightedAverage + copy2).
struct FluxCoarsenItem {
   int prob;
   int axis;
   int side;
   int fine_patch;
   int coarse_patch;
   int lo[3], hi[3];   // coarse face cells (index space of the side box)
   int fface;          // fine face index along the axis
   int t0, t1;         // tangential axes (t1 = -1 in 2-D); t1 is outer
   int ratio;          // refinement ratios along t0 (bits 0-7) and t1 (bits 8-15)
};

// Restriction: coarse cells of one destination patch covered by one fine
// patch (CartesianCellDoubleWeightedAverage + CoarsenSchedule copy).
struct RestrictItem {
   int prob;
   int fine_patch;
   int coarse_patch;
   int lo[3], hi[3];   // coarse cells
   int ratio;          // refinement ratios, 8 bits per axis
};

// Prolongation: one fine patch with its coarse interpolation array.
struct ProlongItem {
   int prob;
   int fine_patch;
   ArrDesc tmp;        // coarse interpolation array (in the tmp buffer)
};

struct BcCoefs {
   double a[6], b[6], g[6];
   // Robin coefficients varying along the boundary (fac_set_bc_faces):
   // (a, b, g) triples; face_off[(level * 6 + location) * face_nprob +
   // problem] is a problem's offset for one side of one level's domain
   // face (-1: the constants above), face_dom[(level * face_nprob +
   // problem) * 6] that level's domain box (lower corner, extents).  Null
   // base: constants everywhere.
   const double *face_base = nullptr;
   const long long *face_off = nullptr;
   const int *face_dom = nullptr;
   int face_nprob = 0;
};

// The staged colour pass's wait for a unit's copies: it gives up after
// `limit` SM clock cycles (about 2 s by default).  never = 1 is the test of
// that bound: the wait is on an mbarrier nothing arrives on, so it runs
// out (the stage's copies still land before the block exits).
struct WaitTest {
   long long limit = 4000000000ll;
   int never = 0;
};

#ifdef __CUDACC__
#define FAC_HD __host__ __device__
#else
#define FAC_HD
#endif

// Largest dynamic shared memory of one CTA of the staged colour pass.
constexpr int kStageSmemMax = 227 * 1024;
// dynamic shared memory of the one-launch coarsest solve on shared copies
// (its static reduction array takes part of the per-block limit)
constexpr int kSolveSmemMax = kStageSmemMax - 1024;
// staged pass: mbarriers and copy sources ahead of the stages, and the
// largest ring of stages a CTA holds
constexpr int kStageBarrierBytes = 128;
constexpr int kStageDepthMax = 4;

// Shared-memory plan of one unit of the staged colour pass: a run of ns
// slices (planes in 3-D, rows in 2-D) along the slowest axis of an nx x ny
// (x nz) patch.  A stage holds a 256-byte unit header and the regions
//   0 u over the slices and one slice either side (ghosted rows), 1 f,
//   2..1+dim the side arrays of D, then C when variable,
//   then per patch face of the unit (x lo/hi, y lo/hi (3-D), slow-axis
//   lo/hi where the unit reaches the patch's end) the push targets (int32),
//   then, for a patch with coarse-fine faces, the Ewing fluxes of the same
//   faces.
// Each region is sized for its elements plus a 16-byte alignment shift;
// off[r] is its start from the stage start (16-byte multiples).
constexpr int kStageHeader = 256;
constexpr int kStageMaxRegions = 18;

struct StagePlan {
   int nreg;
   int nbase;        // u, f, D, C regions
   int face0;        // first push-target region
   int cff0;         // first Ewing-flux region (== nreg when none)
   int off[kStageMaxRegions];
   long long count[kStageMaxRegions];  // elements
   int esize[kStageMaxRegions];        // element bytes
   int face[6];      // face id (2*axis + side) of the k-th face region
   int nface;
   int bytes;
};

FAC_HD inline StagePlan stage_plan(int dim, int nx, int ny, int ns, int tsize, bool dvar,
                                   bool cvar, bool slo, bool shi, bool cf)
{
   StagePlan sp;
   const long long g1 = dim == 3 ? (long long)(nx + 2) * (ny + 2) : nx + 2;
   const long long g0 = dim == 3 ? (long long)nx * ny : nx;
   int r = 0;
   sp.count[r] = (ns + 2) * g1;
   sp.esize[r++] = tsize;
   sp.count[r] = ns * g0;
   sp.esize[r++] = tsize;
   if (dvar) {
      for (int a = 0; a < dim; ++a) {
         long long n;
         if (dim == 3) {
            n = a == 0 ? (long long)ns * (nx + 1) * ny
                       : (a == 1 ? (long long)ns * nx * (ny + 1) : (long long)(ns + 1) * nx * ny);
         } else {
            n = a == 0 ? (long long)ns * (nx + 1) : (long long)(ns + 1) * nx;
         }
         sp.count[r] = n;
         sp.esize[r++] = tsize;
      }
   }
   if (cvar) {
      sp.count[r] = ns * g0;
      sp.esize[r++] = tsize;
   }
   sp.nbase = r;
   // faces of the unit
   sp.nface = 0;
   const long long lat0 = dim == 3 ? (long long)ny * ns : ns;  // x faces
   const long long lat1 = (long long)nx * ns;                   // y faces (3-D)
   const long long slow = dim == 3 ? (long long)nx * ny : nx;   // slow-axis faces
   long long fcount[6];
   for (int s = 0; s < 2; ++s) {
      sp.face[sp.nface] = s;
      fcount[sp.nface++] = lat0;
   }
   if (dim == 3)
      for (int s = 0; s < 2; ++s) {
         sp.face[sp.nface] = 2 + s;
         fcount[sp.nface++] = lat1;
      }
   if (slo) {
      sp.face[sp.nface] = 2 * (dim - 1);
      fcount[sp.nface++] = slow;
   }
   if (shi) {
      sp.face[sp.nface] = 2 * (dim - 1) + 1;
      fcount[sp.nface++] = slow;
   }
   sp.face0 = r;
   for (int k = 0; k < sp.nface; ++k) {
      sp.count[r] = fcount[k];
      sp.esize[r++] = 4;
   }
   sp.cff0 = r;
   if (cf)
      for (int k = 0; k < sp.nface; ++k) {
         sp.count[r] = fcount[k];
         sp.esize[r++] = tsize;
      }
   sp.nreg = r;
   long long o = kStageHeader;
   for (int k = 0; k < r; ++k) {
      sp.off[k] = (int)o;
      o += ((sp.count[k] * sp.esize[k] + 15) / 16) * 16 + 16;
   }
   for (int k = r; k < kStageMaxRegions; ++k) {
      sp.off[k] = (int)o;
      sp.count[k] = 0;
      sp.esize[k] = 0;
   }
   sp.bytes = o > 0x3fffffff ? 0x3fffffff : (int)o;
   return sp;
}

// Header of one staged unit (built on the host, copied into the stage
// ahead of the unit's data): the patch geometry the consumers need, values
// computed once per unit (reciprocals in both precisions, slot counts) and
// the stage offsets (bytes from the stage start to element 0) of the regions.
struct UnitHdr {
   int lo[3], hi[3];
   int flags, s0, ns, hx;  // hx: active cells per row, (nx + 1) / 2
   long long off1;         // patch start in ghost-1 cell buffers
   double dx[3];
   double dxi_d[3];        // 1 / dx in FP64
   float dxi_f[3];         // 1 / dx rounded from FP32 dx, in FP32
   unsigned mhx, mny, mnx; // ceil(2^32 / d) for d = hx, ny, nx: q / d = umulhi(q, m)
                           // for the slot and face decodes (exact for q d < 2^32)
   int nslots;             // hx * rows
   int fmask;              // bit 2*axis+side: the unit has that patch face
   int cfmask;             // faces of fmask with coarse-fine entries (-2)
   int pmask;              // faces of fmask with push targets (>= -1)
   int off_u, off_f, off_d[3], off_c;
   int off_push[6];        // per face id 2*axis+side: push targets, -1 if none
   int off_cff[6];         // Ewing fluxes of the same faces, -1 if none
};

// Shared-memory plan of one unit of the staged composite residual: the
// 256-byte header, then u over the unit's slices and one slice either side
// (ghosted rows, element size tu: FP64, or FP32 for the error of the mixed
// cycle), f when the right-hand side is not zero, the side arrays of D and
// C when variable (all FP64).
FAC_HD inline StagePlan res_plan(int dim, int nx, int ny, int ns, int tu, bool hasf, bool dvar,
                                 bool cvar)
{
   StagePlan sp;
   const long long g1 = dim == 3 ? (long long)(nx + 2) * (ny + 2) : nx + 2;
   const long long g0 = dim == 3 ? (long long)nx * ny : nx;
   int r = 0;
   sp.count[r] = (ns + 2) * g1;
   sp.esize[r++] = tu;
   if (hasf) {
      sp.count[r] = ns * g0;
      sp.esize[r++] = 8;
   }
   if (dvar) {
      for (int a = 0; a < dim; ++a) {
         long long n;
         if (dim == 3) {
            n = a == 0 ? (long long)ns * (nx + 1) * ny
                       : (a == 1 ? (long long)ns * nx * (ny + 1) : (long long)(ns + 1) * nx * ny);
         } else {
            n = a == 0 ? (long long)ns * (nx + 1) : (long long)(ns + 1) * nx;
         }
         sp.count[r] = n;
         sp.esize[r++] = 8;
      }
   }
   if (cvar) {
      sp.count[r] = ns * g0;
      sp.esize[r++] = 8;
   }
   sp.nbase = sp.face0 = sp.cff0 = sp.nreg = r;
   sp.nface = 0;
   long long o = kStageHeader;
   for (int k = 0; k < r; ++k) {
      sp.off[k] = (int)o;
      o += ((sp.count[k] * sp.esize[k] + 15) / 16) * 16 + 16;
   }
   for (int k = r; k < kStageMaxRegions; ++k) {
      sp.off[k] = (int)o;
      sp.count[k] = 0;
      sp.esize[k] = 0;
   }
   sp.bytes = o > 0x3fffffff ? 0x3fffffff : (int)o;
   return sp;
}

// Header of one unit of the staged residual.
struct ResHdr {
   int lo[3], hi[3];
   int s0, ns;             // first slice (patch-relative) and slices of the unit
   int ncells;             // cells of the unit, x fastest
   int has_oflux;          // the level stores its patches' outer-side fluxes
   unsigned mnx, mny;      // ceil(2^32 / d) for d = nx, ny (exact for q d < 2^32)
   long long off0s;        // ghost-0 element of the unit's first cell
   long long offo[3][2];   // outer-side flux arrays of the patch (axis, side)
   double dxi[3];          // 1 / dx, FP64
   int off_u, off_f, off_d[3], off_c;  // stage offsets of the regions (-1 none)
};
static_assert(sizeof(ResHdr) <= kStageHeader, "residual unit header");

// Kinds of residual unit lists: the error or solution in FP64 with a
// right-hand side, the same with a zero right-hand side (operator
// application), the FP32 error of the mixed cycle with a right-hand side.
enum ResKind : int { kResF64 = 0, kResF64Zero = 1, kResF32 = 2, kResKinds = 3 };

// A cell of a patch (linear index x fastest) whose residual the staged pass
// leaves to the fix-up pass: it has a coarse-fine face (Ewing) or a face
// that takes a coarsened finer-level flux.
struct CellRef {
   int patch;
   int lin;
};

// Berger-Rigoutsos node box on the device (3-D extents, 1 for unused axes),
// its problem's dense tag array and where its histograms start: x counts,
// then y, then z.
struct BrNode {
   int lo[3], hi[3];
   int dlo[3], dn[3];   // the problem's dense tag array: lower corner, extents
   long long hoff;
   long long doff;      // where that array starts
};
// A run of rows (along x) of one node box for one block of the histogram
// kernel; rows are numbered y fastest, then z.
struct BrItem {
   int node;
   int row0;
   int nrows;
   int pad;
};
// Block of the histogram kernel and x positions per thread: node boxes up
// to kBrThreads * kBrMaxXPerThread cells along x.
constexpr int kBrThreads = 256;
constexpr int kBrMaxXPerThread = 4;

// One bulk copy of a staged unit: nbytes (a multiple of 16) from byte
// src_off (16-byte aligned) of source array src into the stage at dst_off.
// The first copy of a unit carries the unit's total in total.
enum StageSrc : int {
   kSrcU = 0, kSrcF, kSrcD, kSrcC, kSrcPush, kSrcFlux, kSrcHdr, kSrcCount
};
struct UnitCopy {
   long long src_off;
   int src;
   int nbytes;
   int dst_off;
   int total;
};

struct PoissonSpec {
   int d_variable;
   int c_kind;        // 0 zero, 1 constant, 2 variable
   double d_const;
   double c_const;
};

}  // namespace samrai_b200

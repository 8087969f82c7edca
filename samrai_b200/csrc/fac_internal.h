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

// One patch of a (batched) level.
struct PatchDesc {
   int lo[3], hi[3];
   int prob;           // problem index within the context
   int flags;          // bit0: has coarse-fine boundary faces
   long long off1;     // start of this patch in ghost-1 cell buffers
   long long off0;     // start in ghost-0 cell buffers
   long long offs[3];  // start of the side array of each axis
   long long offo[3][2];  // start of the outer-side array of axis a, side s
   double dx[3];
};

// Chunk of work over one patch: cells [begin, begin+count) of a
// linearisation chosen by the kernel that consumes it.
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
   int pad;
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
};

// Restriction: coarse cells of one destination patch covered by one fine
// patch (CartesianCellDoubleWeightedAverage + CoarsenSchedule copy).
struct RestrictItem {
   int prob;
   int fine_patch;
   int coarse_patch;
   int lo[3], hi[3];   // coarse cells
};

// Prolongation: one fine patch with its coarse interpolation array.
struct ProlongItem {
   int prob;
   int fine_patch;
   ArrDesc tmp;        // coarse interpolation array (in the tmp buffer)
};

struct BcCoefs {
   double a[6], b[6], g[6];
};

struct PoissonSpec {
   int d_variable;
   int c_kind;        // 0 zero, 1 constant, 2 variable
   double d_const;
   double c_const;
};

}  // namespace samrai_b200

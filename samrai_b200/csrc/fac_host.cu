// Host side of the FAC hot path: hierarchy tables (the device form of
// SAMRAI's refine/coarsen schedules), the FAC algorithm
// (FACPreconditioner + CellPoissonFACOps) and the C ABI.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <climits>
#include <limits>
#include <map>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/samrai_fac_b200.h"
#include "fac_internal.h"
#include "fac_kernels.h"

namespace samrai_b200 {

int cnn_forward_on_stream(fac_cnn *n, const float *x, long long nsamp, cudaStream_t st,
                          const float **y);
int cnn_max_batch(const fac_cnn *n);
int cnn_device(const fac_cnn *n);

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------

static thread_local std::string g_last_error;
// Host-only mode (device index -1): tables are built and validated but no
// device memory is allocated and no kernel can run.
static thread_local bool g_dry = false;

struct FacError : std::runtime_error {
   int code;
   FacError(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

#define CUDA_CHECK(x)                                                             \
   do {                                                                           \
      cudaError_t _e = (x);                                                       \
      if (_e != cudaSuccess)                                                      \
         throw FacError(FAC_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(_e)); \
   } while (0)

// ---------------------------------------------------------------------------
// box algebra (hier::Box semantics: inclusive lower/upper corners)
// ---------------------------------------------------------------------------

struct Box {
   int lo[3] = {0, 0, 0}, hi[3] = {-1, -1, -1};
   bool empty() const { return lo[0] > hi[0] || lo[1] > hi[1] || lo[2] > hi[2]; }
   long long size() const
   {
      if (empty()) return 0;
      return (long long)(hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1);
   }
   bool contains(int i, int j, int k) const
   {
      return i >= lo[0] && i <= hi[0] && j >= lo[1] && j <= hi[1] && k >= lo[2] && k <= hi[2];
   }
};

static Box isect(const Box &a, const Box &b)
{
   Box r;
   for (int d = 0; d < 3; ++d) {
      r.lo[d] = std::max(a.lo[d], b.lo[d]);
      r.hi[d] = std::min(a.hi[d], b.hi[d]);
   }
   return r;
}

static Box grow(Box b, int dim, int g)
{
   for (int a = 0; a < dim; ++a) {
      b.lo[a] -= g;
      b.hi[a] += g;
   }
   return b;
}

static int coarsen_index(int i, int r) { return i < 0 ? (i + 1) / r - 1 : i / r; }

static Box coarsen(Box b, int dim, const int *r)
{
   for (int a = 0; a < dim; ++a) {
      b.lo[a] = coarsen_index(b.lo[a], r[a]);
      b.hi[a] = coarsen_index(b.hi[a], r[a]);
   }
   return b;
}

static Box refine(Box b, int dim, const int *r)
{
   for (int a = 0; a < dim; ++a) {
      b.lo[a] = b.lo[a] * r[a];
      b.hi[a] = (b.hi[a] + 1) * r[a] - 1;
   }
   return b;
}

// a minus b as a list of disjoint boxes
static void subtract(const Box &a, const Box &b, std::vector<Box> &out)
{
   Box I = isect(a, b);
   if (I.empty()) {
      out.push_back(a);
      return;
   }
   Box rem = a;
   for (int d = 0; d < 3; ++d) {
      if (rem.lo[d] < I.lo[d]) {
         Box piece = rem;
         piece.hi[d] = I.lo[d] - 1;
         out.push_back(piece);
         rem.lo[d] = I.lo[d];
      }
      if (rem.hi[d] > I.hi[d]) {
         Box piece = rem;
         piece.lo[d] = I.hi[d] + 1;
         out.push_back(piece);
         rem.hi[d] = I.hi[d];
      }
   }
}

static void subtract_all(std::vector<Box> &region, const Box &b)
{
   std::vector<Box> out;
   for (const Box &r : region) subtract(r, b, out);
   region.swap(out);
}

static ArrDesc make_desc(long long base, const Box &gb)
{
   ArrDesc d;
   d.base = base;
   for (int a = 0; a < 3; ++a) {
      d.lo[a] = gb.lo[a];
      d.n[a] = gb.hi[a] - gb.lo[a] + 1;
   }
   return d;
}

// ---------------------------------------------------------------------------
// device buffers
// ---------------------------------------------------------------------------

template <class T>
struct DevArray {
   T *p = nullptr;
   size_t n = 0;
   void alloc(size_t count)
   {
      free();
      n = count;
      if (g_dry) return;
      if (count) {
         // 64 spare bytes: bulk copies round their ends out to 16 bytes
         cudaError_t e = cudaMalloc((void **)&p, count * sizeof(T) + 64);
         if (e != cudaSuccess) {
            p = nullptr;
            throw FacError(FAC_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
         }
      }
   }
   void upload(const std::vector<T> &v, cudaStream_t s)
   {
      alloc(v.size());
      if (!v.empty() && !g_dry)
         CUDA_CHECK(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
   }
   void free()
   {
      if (p) cudaFree(p);
      p = nullptr;
      n = 0;
   }
   ~DevArray() { free(); }
   DevArray() = default;
   DevArray(const DevArray &) = delete;
   DevArray &operator=(const DevArray &) = delete;
};

// The full chunk list and per-problem chunk ranges behind a work list that
// the device compacts to the active problems (k_compact).
struct WorkSrc {
   DevArray<Chunk> all;
   DevArray<int> pcb;
};

template <class I>
struct ItemList {
   std::vector<I> items;
   std::vector<long long> cells;  // per item
   std::vector<Chunk> chunks;
   std::vector<int> prefix;       // first cell of each item (list order)
   DevArray<I> d_items;
   DevArray<Chunk> d_chunks;
   DevArray<int> d_prefix;
   WorkSrc ws;
   void add(const I &it, long long ncells)
   {
      items.push_back(it);
      cells.push_back(ncells);
   }
   // Chunks: an item larger than kChunk cells gets chunks of its own; runs
   // of smaller items of one problem share a chunk of up to kChunk cells.
   void pack()
   {
      chunks.clear();
      prefix.assign(items.size() + 1, 0);
      long long run = 0;
      for (size_t i = 0; i < items.size(); ++i) {
         if (run + cells[i] >= (1ll << 31)) throw FacError(FAC_ERR_ARG, "transaction list too long");
         prefix[i] = (int)run;
         run += cells[i];
      }
      prefix[items.size()] = (int)run;
      size_t i = 0;
      while (i < items.size()) {
         if (cells[i] > kChunk) {
            for (long long b = 0; b < cells[i]; b += kChunk)
               chunks.push_back({(int)i, (int)b, (int)std::min<long long>(kChunk, cells[i] - b), 1});
            ++i;
            continue;
         }
         size_t j = i;
         long long n = 0;
         while (j < items.size() && cells[j] <= kChunk && n + cells[j] <= kChunk &&
                items[j].prob == items[i].prob) {
            n += cells[j];
            ++j;
         }
         if (n > 0) chunks.push_back({(int)i, 0, (int)n, (int)(j - i)});
         i = j;
      }
   }
   void upload(cudaStream_t s)
   {
      pack();
      d_items.upload(items, s);
      d_chunks.upload(chunks, s);
      d_prefix.upload(prefix, s);
   }
   int nchunks() const { return (int)chunks.size(); }
   void clear()
   {
      items.clear();
      cells.clear();
      chunks.clear();
      prefix.clear();
      d_items.free();
      d_chunks.free();
      d_prefix.free();
      ws.all.free();
      ws.pcb.free();
   }
};

// A ghost fill as a gather list: per element of the copy and constant-refine
// items its destination, source element (coarser level: -source - 1) and
// problem; the physical-boundary items stay items (bc).
struct FillGather {
   std::vector<unsigned> to;
   std::vector<int> from;
   std::vector<unsigned short> prob;
   DevArray<unsigned> d_to;
   DevArray<int> d_from;
   DevArray<unsigned short> d_prob;
   ItemList<FillItem> bc;
   bool ok = false;  // element indices and problems fit their fields
};

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------

struct HostProblem {
   int n0[3];
   double xlo[3], xup[3];
   int nlev;
   int ratio[kMaxLevels][3];
   std::vector<Box> boxes[kMaxLevels];
};

// internal field id: the all-zero ghost-0 field
constexpr int kFieldZero = 100;

struct LevelState {
   int npatch = 0;
   std::vector<PatchDesc> hp;
   std::vector<Box> box;               // patch boxes
   std::vector<int> prob_patch_begin;  // size nprob+1
   long long n1 = 0, n0 = 0, ns = 0, no = 0;
   std::vector<long long> prob_off1, prob_off0, prob_offs, prob_offo;  // size nprob+1
   int ratio[3] = {1, 1, 1};
   double tranwt[3] = {0, 0, 0}, longwt[3] = {0, 0, 0};
   double rb_bytes = 0, fill_bytes = 0;  // algorithmic bytes per launch (all problems)
   std::vector<double> rb_bytes_prob, fill_bytes_prob;  // per problem
   std::vector<Box> domain;            // per problem
   std::vector<double> dx;             // per problem x3

   DevArray<PatchDesc> d_patches;
   DevArray<double> u, e, f, r, tr, w, c, d, flux, oflux, cfflux;
   DevArray<double> zero;  // all-zero ghost-0 field (right-hand side of A x)
   // Krylov workspace (fac_solve_fgmres): V_0..V_m then Z_0..Z_{m-1}, n0
   // apart, and per-chunk partial sums of the multi-dot products
   DevArray<double> kry, kry_partial;
   // FP32 copies for the mixed-precision cycle (error, smoother rhs, D, C,
   // Ewing fluxes, coarse interpolation arrays)
   DevArray<float> e32, r32, d32, c32, cfflux32, tmp32;
   DevArray<unsigned char> cfmask;
   // per face cell: index (ghost-1 buffer) of the same-level cell across the
   // face, -1 physical boundary, -2 coarse-fine face (fused colour pass)
   DevArray<long long> facemap;
   DevArray<int> pushmap;
   std::vector<int> pushmap_h;  // host copy (face masks of the staged units)
   // side-array faces that carry a coarsened finer-level flux
   DevArray<unsigned char> fcmask;
   bool fused_ok = false;
   // staged colour pass: units (runs of slices of one patch) for FP64 [0]
   // and FP32 [1] data, and the largest shared memory of a unit
   std::vector<Chunk> units[2];  // {patch, first copy, copies, header}
   DevArray<Chunk> d_units[2];
   DevArray<UnitCopy> d_copies[2];
   DevArray<unsigned char> d_hdrs[2];
   WorkSrc ws_units[2];
   int unit_smem[2] = {0, 0};
   // staged composite residual: units per ResKind (largest first) and
   // their largest shared memory (0: the level runs the unstaged kernels)
   std::vector<Chunk> runits[kResKinds];
   DevArray<Chunk> d_runits[kResKinds];
   DevArray<UnitCopy> d_rcopies[kResKinds];
   DevArray<unsigned char> d_rhdrs[kResKinds];
   WorkSrc ws_runits[kResKinds];
   int runit_smem[kResKinds] = {0, 0, 0};
   // cells the staged residual leaves to the fix-up pass
   std::vector<CellRef> rfix;
   DevArray<CellRef> d_rfix;
   // host copies of cfmask and fcmask
   std::vector<unsigned char> cfmask_h, fcmask_h;
   // regrid step: tags of the level's cells (ghost-0 layout), allocated on first use
   DevArray<unsigned char> tag;
   DevArray<int> d_ratio;

   // work chunks
   std::vector<Chunk> cell_chunks, slot_chunks, flux_chunks;
   DevArray<Chunk> d_cell_chunks, d_slot_chunks, d_flux_chunks;
   WorkSrc ws_cell, ws_slot, ws_flux;
   std::vector<int> prob_cell_chunk_begin;
   DevArray<int> d_prob_cell_chunk_begin;
   // Krylov vector chunks: runs of up to kSpanChunk ghost-0 cells of one
   // problem, {problem, first cell, cells, chunk index}; a problem's patches
   // are contiguous in the ghost-0 buffers
   std::vector<Chunk> span_chunks;
   DevArray<Chunk> d_span_chunks;
   WorkSrc ws_span;
   std::vector<int> prob_span_begin;
   DevArray<int> d_prob_span_begin;
   std::vector<double> cells_prob;  // ghost-0 cells per problem
   DevArray<double2> norm_partial;

   ItemList<FillItem> fill_nc, fill_wc;   // ghost fill without / with coarser level
   FillGather gather_nc, gather_wc;       // the same fills as gather lists
   FillGather gather_tmp;                 // tmp_fill as a gather list
   std::vector<CfFace> cf;
   DevArray<CfFace> d_cf;
   ItemList<RestrictItem> restrict_g1, restrict_g0;  // from level ln+1 into this
   ItemList<FluxCoarsenItem> fcoarsen;               // from level ln+1 into this
   ItemList<FillItem> tmp_fill;                      // coarse interpolation arrays
   ItemList<ProlongItem> prolong;                    // from level ln-1 into this
   ItemList<ProlongItem> prolong2;                   // the same, counted in coarse cells
   bool prolong_r2 = false;                          // ratio 2 on every axis
   DevArray<double> tmp;
   DevArray<double> dxc_prob;                        // per problem dx of level ln-1
   DevArray<unsigned long long> maxres_red, maxres_blk;
   bool one_patch_per_prob = false;  // patch p is problem p's only patch, <= 16384 cells
   bool facemap_local = false;       // no face of the level has a same-level neighbour
   int solve_smem = 0;               // shared bytes of the one-launch solve on shared
                                     // copies (0: that form does not fit)
   DevArray<int> last_patch;
   std::vector<long long> dir_idx;
   DevArray<long long> d_dir_idx;
   DevArray<double> dir_cache;
};

}  // namespace samrai_b200

using namespace samrai_b200;

struct fac_ctx {
   int dim = 2;
   int device = 0;
   cudaStream_t stream = nullptr;
   bool initialized = false;
   std::vector<HostProblem> probs;
   int nlev = 0;
   PoissonSpec spec{0, 0, 1.0, 0.0};
   BcCoefs bc;
   // FACPreconditioner / CellPoissonFACOps parameters (reference defaults,
   // FACPreconditioner.C:37-48 and CellPoissonFACOps.C:588-600)
   int max_cycles = 10;
   double residual_tol = 1e-6;
   double rel_residual_tol = -1.0;
   int pre_sweeps = 1, post_sweeps = 1;
   double coarse_tol = 1e-8;
   int coarse_max_it = 500;
   int ewing = 1;
   int mixed = 0;            // 1: FP32 smoothing and error transfer
   int use_graph = 1;        // capture one FAC cycle into a CUDA graph and replay it
   int fused = 1;            // colour passes read across patch faces directly
   int staged = 1;           // fused passes on shared-memory staged units
   // coefficients came from fac_set_bc / fac_set_bc_faces (a caller's
   // RobinBcCoefStrategy): the solves leave the boundary ghost values of u
   // as their last fill leaves them instead of restoring them
   bool bc_object = false;
   // residual kernels form the fluxes on the fly: 1 on every level, 0 on
   // none, -1 on the levels of large patches (fused_residual_on)
   int fused_residual = -1;
   int stage_budget = 32 * 1024;  // shared memory of one stage (unit) of the staged pass
   int stage_depth = 2;           // stages per CTA of the staged pass
   DevArray<int> kerr;       // set by kernels whose bounded waits ran out
   WaitTest wait_test;       // bound of the staged pass's waits (fac_set_wait_test)
   // Robin coefficients varying along the boundary (fac_set_bc_faces);
   // while any are set the colour passes take the fill-based path, whose
   // boundary fills read them
   bool bc_faces = false;
   std::vector<double> face_host;
   std::vector<long long> face_off_host;
   std::vector<int> face_dom_host;
   DevArray<double> face_dev;
   DevArray<long long> face_off_dev;
   DevArray<int> face_dom_dev;
   bool capturing = false;   // inside stream capture: no host synchronisation
   cudaGraphExec_t cycle_exec = nullptr;
   // captured FGMRES pieces: FAC cycle on R into E (the preconditioner) and
   // the composite operator on E into TR; our kernels in each graph
   cudaGraphExec_t prec_exec = nullptr, apply_exec = nullptr;
   long long prec_launches = 0, apply_launches = 0;
   int kry_m = 0;
   DevArray<double> kry_dots, kry_coef, kry_a;
   DevArray<double> vec_coef;  // per-problem scalars of fac_vec_linear_sum
   DevArray<unsigned long long> tag_counts;  // per-problem tag counts
   // clustering scratch, grown as needed and kept between calls
   DevArray<unsigned char> br_dense;
   DevArray<BrNode> br_nodes;
   DevArray<BrItem> br_items;
   DevArray<int> br_hist;
   int krylov = 0;  // > 0: fac_solve runs FGMRES(krylov) around the FAC cycle
   // fac_set_coarse_extension: domain-covering coarser levels added below
   // every problem's level 0, and whether their coefficients need to be
   // derived again from the caller's level 0 before the next solve
   int ext_levels = 0;
   bool ext_dirty = false;
   // learned correction after every cycle (fac_set_learned)
   fac_cnn *cnn = nullptr;
   int learned_level = -1;
   DevArray<float> cnn_in;
   DevArray<double> cnn_scale, alpha;
   DevArray<double2> dot_acc;
   long long learned_applied = 0;
   std::vector<int> host_active;  // host copy of the active flags (instrumentation)
   int check_interval = 8;   // sweeps between host checks of convergence flags

   // optional per-kernel timing with CUDA events on the context stream
   struct ProfRec {
      int kind;
      cudaEvent_t a, b;
      double bytes;
      // records inside the captured cycle: bytes of the problems active in
      // each replay = scale x sum of per_prob over the active problems
      const std::vector<double> *per_prob;
      double scale;
   };
   bool profiling = false;
   // the captured cycle: its event records, how many of our kernels it
   // launches, and whether it was captured with profiling on
   std::vector<ProfRec> graph_prof;
   long long graph_launches = 0;
   bool graph_profiled = false;
   struct KindAcc {
      long long n = 0;
      double ms = 0, bytes = 0;
   };
   KindAcc graph_acc[6];
   // per-operation wall time with a stream synchronisation on both sides
   // (tbox::Timer::barrierAndStart semantics, tbox/Timer.C:174)
   bool tracing = false;
   std::map<std::string, std::pair<long long, double>> trace;
   std::vector<ProfRec> prof;
   std::vector<cudaEvent_t> ev_pool;
   size_t ev_next = 0;
   cudaEvent_t t0 = nullptr, t1 = nullptr;

   LevelState L[kMaxLevels];
   DevArray<int> active, run;
   // every work list of the context, compacted after each change of active
   std::vector<WorkReg> work_regs;
   DevArray<WorkReg> d_work_regs;
   DevArray<long long> sweeps_call, sweeps_coarse;
   DevArray<double2> norm_acc;
   std::vector<std::vector<double>> hist;  // per problem residual history

   void drop_graph()
   {
      if (cycle_exec) cudaGraphExecDestroy(cycle_exec);
      cycle_exec = nullptr;
      if (prec_exec) cudaGraphExecDestroy(prec_exec);
      if (apply_exec) cudaGraphExecDestroy(apply_exec);
      prec_exec = apply_exec = nullptr;
      prec_launches = apply_launches = 0;
      for (const ProfRec &r : graph_prof) {
         cudaEventDestroy(r.a);
         cudaEventDestroy(r.b);
      }
      graph_prof.clear();
      graph_launches = 0;
   }

   ~fac_ctx()
   {
      drop_graph();
      for (cudaEvent_t e : ev_pool) cudaEventDestroy(e);
      if (t0) cudaEventDestroy(t0);
      if (t1) cudaEventDestroy(t1);
   }
};

namespace {

int nprob(const fac_ctx *c) { return (int)c->probs.size(); }

struct OpTimer {
   fac_ctx *c;
   std::string name;
   std::chrono::steady_clock::time_point t0;
   OpTimer(fac_ctx *ctx, const char *n, int ln) : c(ctx)
   {
      if (!c->tracing) return;
      name = std::string(n) + "@L" + std::to_string(ln);
      cudaStreamSynchronize(c->stream);
      t0 = std::chrono::steady_clock::now();
   }
   ~OpTimer()
   {
      if (!c->tracing) return;
      cudaStreamSynchronize(c->stream);
      const double ms =
         std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
      auto &e = c->trace[name];
      e.first += 1;
      e.second += ms;
   }
};

cudaEvent_t next_event(fac_ctx *c)
{
   if (c->ev_next == c->ev_pool.size()) {
      cudaEvent_t e;
      CUDA_CHECK(cudaEventCreate(&e));
      c->ev_pool.push_back(e);
   }
   return c->ev_pool[c->ev_next++];
}

double active_bytes(const fac_ctx *c, const std::vector<double> &per_prob)
{
   double b = 0;
   for (size_t p = 0; p < per_prob.size(); ++p)
      if (p >= c->host_active.size() || c->host_active[p]) b += per_prob[p];
   return b;
}

// Record the start of a profiled launch; returns its index or -1.  During
// stream capture the two events become event-record nodes of the cycle graph
// (external records), read back after every replay (harvest_graph_profile).
int prof_begin(fac_ctx *c, int kind, const std::vector<double> &per_prob, double scale)
{
   if (!c->profiling) return -1;
   fac_ctx::ProfRec r;
   r.kind = kind;
   r.per_prob = &per_prob;
   r.scale = scale;
   if (c->capturing) {
      r.bytes = 0;
      CUDA_CHECK(cudaEventCreate(&r.a));
      CUDA_CHECK(cudaEventCreate(&r.b));
      CUDA_CHECK(cudaEventRecordWithFlags(r.a, c->stream, cudaEventRecordExternal));
      c->graph_prof.push_back(r);
      return (int)c->graph_prof.size() - 1;
   }
   r.bytes = scale * active_bytes(c, per_prob);
   r.a = next_event(c);
   r.b = next_event(c);
   CUDA_CHECK(cudaEventRecord(r.a, c->stream));
   c->prof.push_back(r);
   return (int)c->prof.size() - 1;
}

void prof_end(fac_ctx *c, int idx)
{
   if (idx < 0) return;
   if (c->capturing)
      CUDA_CHECK(cudaEventRecordWithFlags(c->graph_prof[idx].b, c->stream,
                                          cudaEventRecordExternal));
   else
      CUDA_CHECK(cudaEventRecord(c->prof[idx].b, c->stream));
}

// After a replay of the cycle graph has completed: add its launch times and
// the bytes of the problems that were active in it.
void harvest_graph_profile(fac_ctx *c)
{
   for (const fac_ctx::ProfRec &r : c->graph_prof) {
      float e = 0.f;
      CUDA_CHECK(cudaEventElapsedTime(&e, r.a, r.b));
      fac_ctx::KindAcc &acc = c->graph_acc[r.kind];
      acc.n += 1;
      acc.ms += e;
      acc.bytes += r.scale * active_bytes(c, *r.per_prob);
   }
}

double *field_ptr(LevelState &L, int fid)
{
   switch (fid) {
      case kFieldZero: return L.zero.p;
      case FAC_U: return L.u.p;
      case FAC_F: return L.f.p;
      case FAC_E: return L.e.p;
      case FAC_R: return L.r.p;
      case FAC_TR: return L.tr.p;
      case FAC_W: return L.w.p;
      case FAC_C: return L.c.p;
   }
   throw FacError(FAC_ERR_ARG, "bad field id");
}

int field_ghost(int fid)
{
   if (fid == kFieldZero) return 0;
   if (fid < 0 || fid > FAC_C) throw FacError(FAC_ERR_ARG, "bad field id");
   return (fid == FAC_U || fid == FAC_E) ? 1 : 0;
}

Box ghost_box(int dim, const Box &b, int g) { return grow(b, dim, g); }

long long cell_count(int dim, const Box &b, int g) { return ghost_box(dim, b, g).size(); }

Box side_box(const Box &b, int a)
{
   Box s = b;
   s.hi[a] += 1;
   return s;
}

Box face_box(const Box &b, int a, int s)
{
   Box f = side_box(b, a);
   if (s == 0) f.hi[a] = f.lo[a];
   else f.lo[a] = f.hi[a];
   return f;
}

void check_state(fac_ctx *c, bool need_init)
{
   if (!c) throw FacError(FAC_ERR_ARG, "null context");
   if (need_init && !c->initialized) throw FacError(FAC_ERR_STATE, "fac_initialize not called");
   if (!need_init && c->initialized) throw FacError(FAC_ERR_STATE, "context already initialized");
}

void check_ops(fac_ctx *c)
{
   check_state(c, true);
   if (c->device < 0)
      throw FacError(FAC_ERR_STATE, "host-only context (device -1) cannot run operations");
}

// ---------------------------------------------------------------------------
// table construction (CellPoissonFACOps::initializeOperatorState)
// ---------------------------------------------------------------------------

void build_level_layout(fac_ctx *c, int ln)
{
   LevelState &L = c->L[ln];
   const int dim = c->dim;
   const int np = nprob(c);
   L.hp.clear();
   L.box.clear();
   L.prob_patch_begin.assign(np + 1, 0);
   L.prob_off1.assign(np + 1, 0);
   L.prob_off0.assign(np + 1, 0);
   L.prob_offs.assign(np + 1, 0);
   L.prob_offo.assign(np + 1, 0);
   L.domain.resize(np);
   L.dx.assign(3 * np, 1.0);
   for (int a = 0; a < 3; ++a) L.ratio[a] = c->probs[0].ratio[ln][a];
   long long o1 = 0, o0 = 0, os = 0, oo = 0;
   for (int p = 0; p < np; ++p) {
      const HostProblem &P = c->probs[p];
      L.prob_patch_begin[p] = (int)L.hp.size();
      L.prob_off1[p] = o1;
      L.prob_off0[p] = o0;
      L.prob_offs[p] = os;
      L.prob_offo[p] = oo;
      int rz[3] = {1, 1, 1};
      for (int l = 1; l <= ln; ++l)
         for (int a = 0; a < 3; ++a) rz[a] *= P.ratio[l][a];
      Box dom;
      for (int a = 0; a < 3; ++a) {
         dom.lo[a] = 0;
         dom.hi[a] = a < dim ? P.n0[a] * rz[a] - 1 : 0;
         // CartesianGridGeometry.C:308-312, 373-379
         const double dx0 = a < dim ? (P.xup[a] - P.xlo[a]) / ((double)P.n0[a]) : 1.0;
         L.dx[3 * p + a] = a < dim ? dx0 / ((double)rz[a]) : 1.0;
      }
      L.domain[p] = dom;
      for (const Box &b : P.boxes[ln]) {
         PatchDesc d;
         std::memset(&d, 0, sizeof(d));
         for (int a = 0; a < 3; ++a) {
            d.lo[a] = b.lo[a];
            d.hi[a] = b.hi[a];
            d.dx[a] = L.dx[3 * p + a];
         }
         d.prob = p;
         d.flags = 0;
         {
            const long long nx = b.hi[0] - b.lo[0] + 1, ny = dim > 1 ? b.hi[1] - b.lo[1] + 1 : 1;
            const long long cells = b.size();
            if (nx > 0 && ny > 0 && cells * std::max(nx, ny) < (1ll << 32)) {
               d.mx = (unsigned)(((1ull << 32) + nx - 1) / nx);
               d.my = (unsigned)(((1ull << 32) + ny - 1) / ny);
            }
         }
         d.off1 = o1;
         d.off0 = o0;
         o1 += cell_count(dim, b, 1);
         o0 += cell_count(dim, b, 0);
         for (int a = 0; a < 3; ++a) {
            d.offs[a] = os;
            if (a < dim) os += side_box(b, a).size();
         }
         for (int a = 0; a < 3; ++a)
            for (int s = 0; s < 2; ++s) {
               d.offo[a][s] = oo;
               if (a < dim) oo += face_box(b, a, s).size();
            }
         L.hp.push_back(d);
         L.box.push_back(b);
      }
   }
   L.prob_patch_begin[np] = (int)L.hp.size();
   L.prob_off1[np] = o1;
   L.prob_off0[np] = o0;
   L.prob_offs[np] = os;
   L.prob_offo[np] = oo;
   L.npatch = (int)L.hp.size();
   L.n1 = o1;
   L.n0 = o0;
   L.ns = os;
   L.no = oo;
   for (int a = 0; a < 3; ++a) {
      // ewingfixflux*: tranwt = 1.0/(1+r) in REAL*4 (2d.f:502), longwt = 2*tranwt
      L.tranwt[a] = (double)(1.0f / (float)(1 + L.ratio[a]));
      L.longwt[a] = 2 * L.tranwt[a];
   }
}

ArrDesc patch_desc(const fac_ctx *c, const LevelState &L, int ip, int g)
{
   const Box gb = ghost_box(c->dim, L.box[ip], g);
   return make_desc(g ? L.hp[ip].off1 : L.hp[ip].off0, gb);
}

// Boxes of ghost cells of box b whose outside pattern is `side`
// (physical boundary, trimmed to b's extent on the other axes).
bool bc_box(int dim, const Box &b, const Box &dom, const int *side, Box &out)
{
   out = b;
   for (int a = 0; a < 3; ++a) {
      if (a >= dim) {
         if (side[a]) return false;
         continue;
      }
      if (side[a] < 0) {
         if (b.lo[a] != dom.lo[a]) return false;
         out.lo[a] = out.hi[a] = b.lo[a] - 1;
      } else if (side[a] > 0) {
         if (b.hi[a] != dom.hi[a]) return false;
         out.lo[a] = out.hi[a] = b.hi[a] + 1;
      }
   }
   return true;
}

std::vector<std::array<int, 3>> all_sides(int dim)
{
   std::vector<std::array<int, 3>> v;
   for (int z = (dim == 3 ? -1 : 0); z <= (dim == 3 ? 1 : 0); ++z)
      for (int y = -1; y <= 1; ++y)
         for (int x = -1; x <= 1; ++x) {
            if (!x && !y && !z) continue;
            v.push_back({x, y, z});
         }
   return v;
}

void build_fill_tables(fac_ctx *c, int ln)
{
   LevelState &L = c->L[ln];
   const int dim = c->dim;
   const int np = nprob(c);
   L.fill_nc.clear();
   L.fill_wc.clear();
   auto sides = all_sides(dim);
   for (int p = 0; p < np; ++p) {
      const int pb = L.prob_patch_begin[p], pe = L.prob_patch_begin[p + 1];
      for (int ip = pb; ip < pe; ++ip) {
         const Box gb = ghost_box(dim, L.box[ip], 1);
         const ArrDesc dst = patch_desc(c, L, ip, 1);
         // same-level copies (CellGeometry overlap: dst ghost box x src box)
         for (int iq = pb; iq < pe; ++iq) {
            if (iq == ip) continue;
            Box ov = isect(gb, L.box[iq]);
            if (ov.empty()) continue;
            FillItem it;
            std::memset(&it, 0, sizeof(it));
            it.kind = kFillCopy;
            it.prob = p;
            for (int a = 0; a < 3; ++a) {
               it.lo[a] = ov.lo[a];
               it.hi[a] = ov.hi[a];
            }
            it.dst = dst;
            it.src = patch_desc(c, L, iq, 1);
            L.fill_nc.add(it, ov.size());
            L.fill_wc.add(it, ov.size());
         }
         // physical boundary
         for (auto &s : sides) {
            Box bb;
            if (!bc_box(dim, L.box[ip], L.domain[p], s.data(), bb)) continue;
            FillItem it;
            std::memset(&it, 0, sizeof(it));
            it.kind = kFillBc;
            it.prob = p;
            for (int a = 0; a < 3; ++a) {
               it.lo[a] = bb.lo[a];
               it.hi[a] = bb.hi[a];
               it.side[a] = s[a];
               it.h[a] = L.dx[3 * p + a];
            }
            it.bc_level = ln;
            it.dst = dst;
            it.src = dst;
            L.fill_nc.add(it, bb.size());
            L.fill_wc.add(it, bb.size());
         }
         // coarse-level fill of ghost cells not covered by the level
         if (ln > 0) {
            const LevelState &C = c->L[ln - 1];
            std::vector<Box> region{isect(gb, L.domain[p])};
            for (int iq = pb; iq < pe; ++iq) subtract_all(region, L.box[iq]);
            const int cb = C.prob_patch_begin[p], ce = C.prob_patch_begin[p + 1];
            for (const Box &rg : region) {
               if (rg.empty()) continue;
               std::vector<Box> left{rg};
               for (int iq = cb; iq < ce; ++iq) {
                  Box fr = refine(C.box[iq], dim, L.ratio);
                  Box sub = isect(rg, fr);
                  if (sub.empty()) continue;
                  subtract_all(left, fr);
                  FillItem it;
                  std::memset(&it, 0, sizeof(it));
                  it.kind = kFillCoarse;
                  it.prob = p;
                  for (int a = 0; a < 3; ++a) {
                     it.lo[a] = sub.lo[a];
                     it.hi[a] = sub.hi[a];
                     it.ratio[a] = L.ratio[a];
                  }
                  it.dst = dst;
                  it.src = patch_desc(c, C, iq, 1);
                  it.src_is_coarse = 1;
                  L.fill_wc.add(it, sub.size());
               }
               for (const Box &lb : left)
                  if (!lb.empty())
                     throw FacError(FAC_ERR_NESTING, "level " + std::to_string(ln) +
                                                          " is not properly nested");
            }
         }
      }
   }
}

void build_cf_faces(fac_ctx *c, int ln)
{
   LevelState &L = c->L[ln];
   const int dim = c->dim;
   std::vector<unsigned char> mask(L.no, 0);
   L.cf.clear();
   if (ln == 0) {
      L.cfmask.upload(mask, c->stream);
      L.cfmask_h = mask;
      return;
   }
   for (int ip = 0; ip < L.npatch; ++ip) {
      PatchDesc &d = L.hp[ip];
      const int p = d.prob;
      const int pb = L.prob_patch_begin[p], pe = L.prob_patch_begin[p + 1];
      const Box &b = L.box[ip];
      const Box gb1 = ghost_box(dim, b, 1);
      auto c1 = [&](int i, int j, int k) {
         const long long nx = gb1.hi[0] - gb1.lo[0] + 1, ny = gb1.hi[1] - gb1.lo[1] + 1;
         return d.off1 + (i - gb1.lo[0]) + nx * ((j - gb1.lo[1]) + ny * (k - gb1.lo[2]));
      };
      for (int a = 0; a < dim; ++a)
         for (int s = 0; s < 2; ++s) {
            Box layer = b;
            const int g = s == 0 ? b.lo[a] - 1 : b.hi[a] + 1;
            layer.lo[a] = layer.hi[a] = g;
            std::vector<Box> region{isect(layer, L.domain[p])};
            for (int iq = pb; iq < pe; ++iq) subtract_all(region, L.box[iq]);
            const Box fb = face_box(b, a, s);
            const Box sb = side_box(b, a);
            for (const Box &rg : region)
               for (int k = rg.lo[2]; k <= rg.hi[2]; ++k)
                  for (int j = rg.lo[1]; j <= rg.hi[1]; ++j)
                     for (int i = rg.lo[0]; i <= rg.hi[0]; ++i) {
                        int cc[3] = {i, j, k};
                        cc[a] = s == 0 ? b.lo[a] : b.hi[a];
                        int fc[3] = {cc[0], cc[1], cc[2]};
                        if (s == 1) fc[a] += 1;
                        int mq[3] = {cc[0], cc[1], cc[2]};
                        for (int t = 0; t < dim; ++t) {
                           if (t == a) continue;
                           const int rr = L.ratio[t];
                           const int base = coarsen_index(cc[t], rr) * rr;
                           mq[t] = base + (rr - (cc[t] - base) - 1);
                           if (mq[t] < b.lo[t] || mq[t] > b.hi[t])
                              throw FacError(FAC_ERR_NESTING,
                                             "patch box not aligned to the refinement ratio");
                        }
                        CfFace f;
                        std::memset(&f, 0, sizeof(f));
                        f.cell = c1(cc[0], cc[1], cc[2]);
                        f.mirror = c1(mq[0], mq[1], mq[2]);
                        f.ghost = c1(i, j, k);
                        const long long fnx = fb.hi[0] - fb.lo[0] + 1, fny = fb.hi[1] - fb.lo[1] + 1;
                        const int ti = cc[0] - fb.lo[0], tj = cc[1] - fb.lo[1], tk = cc[2] - fb.lo[2];
                        long long tlin;
                        if (a == 0) tlin = tj + (long long)(b.hi[1] - b.lo[1] + 1) * tk;
                        else if (a == 1) tlin = ti + (long long)(b.hi[0] - b.lo[0] + 1) * tk;
                        else tlin = ti + (long long)(b.hi[0] - b.lo[0] + 1) * tj;
                        (void)fnx;
                        (void)fny;
                        f.oidx = d.offo[a][s] + tlin;
                        const long long snx = sb.hi[0] - sb.lo[0] + 1, sny = sb.hi[1] - sb.lo[1] + 1;
                        f.sidx = d.offs[a] + (fc[0] - sb.lo[0]) +
                                 snx * ((fc[1] - sb.lo[1]) + sny * (fc[2] - sb.lo[2]));
                        f.patch = ip;
                        f.axis = a;
                        f.side = s;
                        L.cf.push_back(f);
                        mask[f.oidx] = 1;
                        d.flags |= 1;
                     }
         }
   }
   L.cfmask.upload(mask, c->stream);
   L.cfmask_h = mask;
   L.d_cf.upload(L.cf, c->stream);
}

// Units of the staged colour pass: each patch is cut along its slowest axis
// into runs of slices whose shared-memory plan fits the budget (one slice at
// least; a level whose single slice does not fit is not staged).  For every
// unit the host writes its header and its list of bulk copies (byte ranges
// of the level arrays, rounded out to 16 bytes, and where they land in the
// stage), so the producer warp only streams them.
void build_stage_units(fac_ctx *c, int ln)
{
   LevelState &L = c->L[ln];
   const int dim = c->dim;
   const bool dvar = c->spec.d_variable != 0, cvar = c->spec.c_kind == 2;
   struct HdrRec {
      UnitHdr h;
      char pad[kStageHeader - sizeof(UnitHdr)];
   };
   static_assert(sizeof(HdrRec) == kStageHeader, "header record size");
   for (int t = 0; t < 2; ++t) {
      const int ts = t == 0 ? 8 : 4;
      std::vector<Chunk> &U = L.units[t];
      std::vector<UnitCopy> copies;
      std::vector<HdrRec> hdrs;
      U.clear();
      int maxb = 0;
      bool decode_ok = true;
      for (int ip = 0; ip < L.npatch; ++ip) {
         const Box &b = L.box[ip];
         const int nx = b.hi[0] - b.lo[0] + 1, ny = b.hi[1] - b.lo[1] + 1;
         const int nslow = dim == 3 ? b.hi[2] - b.lo[2] + 1 : ny;
         const PatchDesc &d = L.hp[ip];
         const bool cf = (d.flags & 1) != 0;
         // plan of a unit of ns slices; sizing takes both slow-axis faces
         auto bytes = [&](int ns) {
            return stage_plan(dim, nx, ny, ns, ts, dvar, cvar, true, true, cf).bytes;
         };
         // the slot decode wants fewer than 2^14 active cells per unit
         const long long row_slots = (long long)((nx + 1) / 2) * (dim == 3 ? ny : 1);
         int nsmax = 1;
         while (nsmax < nslow && bytes(nsmax + 1) <= c->stage_budget &&
                row_slots * (nsmax + 1) < (1 << 14))
            ++nsmax;
         const int nunit = (nslow + nsmax - 1) / nsmax;
         const int base = nslow / nunit, rem = nslow % nunit;
         int s0 = 0;
         const long long g1 = dim == 3 ? (long long)(nx + 2) * (ny + 2) : nx + 2;
         const long long g0 = dim == 3 ? (long long)nx * ny : nx;
         for (int u = 0; u < nunit; ++u) {
            const int ns = base + (u < rem ? 1 : 0);
            const bool slo = s0 == 0, shi = s0 + ns == nslow;
            const StagePlan sp = stage_plan(dim, nx, ny, ns, ts, dvar, cvar, slo, shi, cf);
            maxb = std::max(maxb, sp.bytes);
            HdrRec rec;
            std::memset(&rec, 0, sizeof(rec));
            UnitHdr &h = rec.h;
            for (int a = 0; a < 3; ++a) {
               h.lo[a] = d.lo[a];
               h.hi[a] = d.hi[a];
               h.dx[a] = d.dx[a];
               // the reciprocals the kernels would form: IEEE divisions in
               // the working precision
               h.dxi_d[a] = 1.0 / d.dx[a];
               h.dxi_f[a] = 1.0f / (float)d.dx[a];
            }
            h.flags = d.flags;
            h.off1 = d.off1;
            h.s0 = s0;
            h.ns = ns;
            h.hx = (nx + 1) / 2;
            h.mhx = (unsigned)(((1ull << 32) + h.hx - 1) / h.hx);
            h.mny = (unsigned)(((1ull << 32) + ny - 1) / ny);
            h.mnx = (unsigned)(((1ull << 32) + nx - 1) / nx);
            h.nslots = h.hx * (dim == 3 ? ny * ns : ns);
            // exact magic divisions: quotient q by divisor d with q d < 2^32
            // (slots by hx, rows by ny, face entries by ny or nx)
            const long long lim = 1ll << 32;
            if ((long long)h.nslots * h.hx >= lim || (long long)ny * ns * ny >= lim ||
                (long long)nx * ns * nx >= lim || (long long)nx * ny * nx >= lim)
               decode_ok = false;
            h.fmask = h.cfmask = h.pmask = 0;
            for (int k = 0; k < 6; ++k) h.off_push[k] = h.off_cff[k] = -1;
            const int first = (int)copies.size();
            copies.push_back({(long long)hdrs.size() * kStageHeader, kSrcHdr, kStageHeader, 0, 0});
            long long total = kStageHeader;
            for (int r = 0; r < sp.nreg; ++r) {
               int src;
               long long e0;  // first element
               long long limit;  // end of the source array (elements)
               if (r == 0) {
                  src = kSrcU;
                  e0 = d.off1 + (long long)s0 * g1;
                  limit = std::min<long long>(L.n1, d.off1 + cell_count(dim, b, 1));
               } else if (r == 1) {
                  src = kSrcF;
                  e0 = d.off0 + (long long)s0 * g0;
                  limit = std::min<long long>(L.n0, d.off0 + b.size());
               } else if (r < sp.nbase) {
                  const int a = r - 2;
                  if (dvar && a < dim) {
                     const long long per =
                        dim == 3 ? (a == 0 ? (long long)(nx + 1) * ny
                                           : (a == 1 ? (long long)nx * (ny + 1) : g0))
                                 : (a == 0 ? nx + 1 : nx);
                     src = kSrcD;
                     e0 = d.offs[a] + (long long)s0 * per;
                     limit = std::min<long long>(L.ns, d.offs[a] + side_box(b, a).size());
                  } else {
                     src = kSrcC;
                     e0 = d.off0 + (long long)s0 * g0;
                     limit = std::min<long long>(L.n0, d.off0 + b.size());
                  }
               } else {
                  const bool flux = r >= sp.cff0;
                  const int fid = sp.face[flux ? r - sp.cff0 : r - sp.face0];
                  const int a = fid >> 1, sd = fid & 1;
                  long long st;
                  if (a == dim - 1) st = 0;  // slow-axis face: the whole face
                  else if (dim == 3) st = (long long)s0 * (a == 0 ? ny : nx);
                  else st = s0;
                  src = flux ? kSrcFlux : kSrcPush;
                  e0 = d.offo[a][sd] + st;
                  const long long fsize = dim == 3 ? (a == 0 ? (long long)ny * (b.hi[2] - b.lo[2] + 1)
                                                   : (a == 1 ? (long long)nx * (b.hi[2] - b.lo[2] + 1)
                                                             : (long long)nx * ny))
                                             : (a == 0 ? ny : nx);
                  limit = std::min<long long>(L.no, d.offo[a][sd] + fsize);
               }
               if (e0 < 0 || e0 + sp.count[r] > limit)
                  throw FacError(FAC_ERR_ARG, "staged unit outside its patch arrays");
               const long long b0 = e0 * sp.esize[r], b1 = b0 + sp.count[r] * sp.esize[r];
               const long long a0 = b0 & ~15ll, a1 = (b1 + 15) & ~15ll;
               const int off = sp.off[r] + (int)(b0 - a0);
               if (r == 0) h.off_u = off;
               else if (r == 1) h.off_f = off;
               else if (r < sp.nbase) {
                  if (dvar && r - 2 < dim) h.off_d[r - 2] = off;
                  else h.off_c = off;
               } else if (r >= sp.cff0) {
                  h.off_cff[sp.face[r - sp.cff0]] = off;
               } else {
                  const int fid = sp.face[r - sp.face0];
                  h.off_push[fid] = off;
                  h.fmask |= 1 << fid;
                  for (long long q = e0; q < e0 + sp.count[r]; ++q) {
                     if (L.pushmap_h[q] == -2) h.cfmask |= 1 << fid;
                     else h.pmask |= 1 << fid;
                  }
               }
               copies.push_back({a0, src, (int)(a1 - a0), sp.off[r], 0});
               total += a1 - a0;
            }
            copies[first].total = (int)total;
            U.push_back({ip, first, (int)copies.size() - first, (int)hdrs.size()});
            hdrs.push_back(rec);
            s0 += ns;
         }
         if (s0 != nslow) throw FacError(FAC_ERR_ARG, "staged units do not tile the patch");
      }
      // stage_depth stages per CTA after the barriers and copy sources; a
      // level whose units do not fit runs the unstaged pass
      L.unit_smem[t] =
         decode_ok && kStageBarrierBytes + (long long)c->stage_depth * maxb <= kStageSmemMax
            ? maxb
            : 0;
      L.d_units[t].upload(U, c->stream);
      L.d_copies[t].upload(copies, c->stream);
      std::vector<unsigned char> raw(hdrs.size() * kStageHeader);
      if (!hdrs.empty()) std::memcpy(raw.data(), hdrs.data(), raw.size());
      L.d_hdrs[t].upload(raw, c->stream);
   }
}

// Units of the staged composite residual, one list per ResKind: every
// patch cut along its slowest axis into runs of slices whose plan fits the
// stage budget (one slice at least), header and bulk-copy list per unit as
// for the colour pass.
void build_res_units(fac_ctx *c, int ln)
{
   LevelState &L = c->L[ln];
   const int dim = c->dim;
   const bool dvar = c->spec.d_variable != 0, cvar = c->spec.c_kind == 2;
   struct HdrRec {
      ResHdr h;
      char pad[kStageHeader - sizeof(ResHdr)];
   };
   static_assert(sizeof(HdrRec) == kStageHeader, "header record size");
   for (int kind = 0; kind < kResKinds; ++kind) {
      const int tu = kind == kResF32 ? 4 : 8;
      const bool hasf = kind != kResF64Zero;
      std::vector<Chunk> &U = L.runits[kind];
      std::vector<UnitCopy> copies;
      std::vector<HdrRec> hdrs;
      U.clear();
      int maxb = 0;
      bool decode_ok = true;
      for (int ip = 0; ip < L.npatch; ++ip) {
         const Box &b = L.box[ip];
         const PatchDesc &d = L.hp[ip];
         const int nx = b.hi[0] - b.lo[0] + 1, ny = b.hi[1] - b.lo[1] + 1;
         const int nslow = dim == 3 ? b.hi[2] - b.lo[2] + 1 : ny;
         const long long g1 = dim == 3 ? (long long)(nx + 2) * (ny + 2) : nx + 2;
         const long long g0 = dim == 3 ? (long long)nx * ny : nx;
         auto bytes = [&](int ns) { return res_plan(dim, nx, ny, ns, tu, hasf, dvar, cvar).bytes; };
         int nsmax = 1;
         while (nsmax < nslow && bytes(nsmax + 1) <= c->stage_budget) ++nsmax;
         const int nunit = (nslow + nsmax - 1) / nsmax;
         const int base = nslow / nunit, rem = nslow % nunit;
         int s0 = 0;
         for (int u = 0; u < nunit; ++u) {
            const int ns = base + (u < rem ? 1 : 0);
            const StagePlan sp = res_plan(dim, nx, ny, ns, tu, hasf, dvar, cvar);
            maxb = std::max(maxb, sp.bytes);
            HdrRec rec;
            std::memset(&rec, 0, sizeof(rec));
            ResHdr &h = rec.h;
            for (int a = 0; a < 3; ++a) {
               h.lo[a] = d.lo[a];
               h.hi[a] = d.hi[a];
               // the reciprocal the kernels would form: an IEEE division
               h.dxi[a] = 1.0 / d.dx[a];
               for (int sd = 0; sd < 2; ++sd) h.offo[a][sd] = a < dim ? d.offo[a][sd] : 0;
            }
            h.s0 = s0;
            h.ns = ns;
            h.ncells = (int)(g0 * ns);
            h.has_oflux = ln > 0 ? 1 : 0;
            h.mnx = (unsigned)(((1ull << 32) + nx - 1) / nx);
            h.mny = (unsigned)(((1ull << 32) + ny - 1) / ny);
            // exact magic divisions: cells by nx, rows by ny (3-D)
            const long long lim = 1ll << 32;
            if ((long long)h.ncells * nx >= lim || (long long)ny * ns * ny >= lim)
               decode_ok = false;
            h.off0s = d.off0 + (long long)s0 * g0;
            h.off_u = h.off_f = h.off_c = -1;
            for (int a = 0; a < 3; ++a) h.off_d[a] = -1;
            const int first = (int)copies.size();
            copies.push_back({(long long)hdrs.size() * kStageHeader, kSrcHdr, kStageHeader, 0, 0});
            long long total = kStageHeader;
            for (int r = 0; r < sp.nreg; ++r) {
               // region r: u, then f (hasf), then D per axis (dvar), then C (cvar)
               int q = r;
               int what;  // 0 u, 1 f, 2.. D axis, 5 C
               if (q == 0) what = 0;
               else if (hasf && q == 1) what = 1;
               else {
                  q -= hasf ? 2 : 1;
                  what = dvar && q < dim ? 2 + q : 5;
               }
               int src;
               long long e0, limit;
               if (what == 0) {
                  src = kSrcU;
                  e0 = d.off1 + (long long)s0 * g1;
                  limit = std::min<long long>(L.n1, d.off1 + cell_count(dim, b, 1));
               } else if (what == 1 || what == 5) {
                  src = what == 1 ? kSrcF : kSrcC;
                  e0 = d.off0 + (long long)s0 * g0;
                  limit = std::min<long long>(L.n0, d.off0 + b.size());
               } else {
                  const int a = what - 2;
                  const long long per =
                     dim == 3 ? (a == 0 ? (long long)(nx + 1) * ny
                                        : (a == 1 ? (long long)nx * (ny + 1) : g0))
                              : (a == 0 ? nx + 1 : nx);
                  src = kSrcD;
                  e0 = d.offs[a] + (long long)s0 * per;
                  limit = std::min<long long>(L.ns, d.offs[a] + side_box(b, a).size());
               }
               if (e0 < 0 || e0 + sp.count[r] > limit)
                  throw FacError(FAC_ERR_ARG, "residual unit outside its patch arrays");
               const long long b0 = e0 * sp.esize[r], b1 = b0 + sp.count[r] * sp.esize[r];
               const long long a0 = b0 & ~15ll, a1 = (b1 + 15) & ~15ll;
               const int off = sp.off[r] + (int)(b0 - a0);
               if (what == 0) h.off_u = off;
               else if (what == 1) h.off_f = off;
               else if (what == 5) h.off_c = off;
               else h.off_d[what - 2] = off;
               copies.push_back({a0, src, (int)(a1 - a0), sp.off[r], 0});
               total += a1 - a0;
            }
            copies[first].total = (int)total;
            U.push_back({ip, first, (int)copies.size() - first, (int)hdrs.size()});
            hdrs.push_back(rec);
            s0 += ns;
         }
         if (s0 != nslow) throw FacError(FAC_ERR_ARG, "residual units do not tile the patch");
      }
      L.runit_smem[kind] =
         decode_ok && kStageBarrierBytes + (long long)c->stage_depth * maxb <= kStageSmemMax
            ? maxb
            : 0;
      L.d_runits[kind].upload(U, c->stream);
      L.d_rcopies[kind].upload(copies, c->stream);
      std::vector<unsigned char> raw(hdrs.size() * kStageHeader);
      if (!hdrs.empty()) std::memcpy(raw.data(), hdrs.data(), raw.size());
      L.d_rhdrs[kind].upload(raw, c->stream);
   }
}

// Cells whose residual the staged pass leaves to the fix-up pass, each once
// in patch order: a cell on a coarse-fine face of the level (the Ewing fix
// changes that face's flux) and a cell next to a face that takes a
// coarsened finer-level flux -- exactly the faces k_residual_fused treats
// apart (patch flags bit 0 with cfmask, bit 1 with fcmask).  Cells under
// the finer level count too: the V-cycle restricts their residual to the
// coarser level (facCycle_Recursive's restrictResidual of the level's
// whole residual).
void build_residual_fixups(fac_ctx *c, int ln)
{
   LevelState &L = c->L[ln];
   const int dim = c->dim;
   L.rfix.clear();
   std::vector<unsigned char> mark;
   for (int ip = 0; ip < L.npatch; ++ip) {
      const PatchDesc &d = L.hp[ip];
      if (!(d.flags & 3)) continue;
      const int n[3] = {d.hi[0] - d.lo[0] + 1, d.hi[1] - d.lo[1] + 1,
                        dim == 3 ? d.hi[2] - d.lo[2] + 1 : 1};
      mark.assign((size_t)n[0] * n[1] * n[2], 0);
      auto cell = [&](const int *x) { return x[0] + (long long)n[0] * (x[1] + (long long)n[1] * x[2]); };
      if ((d.flags & 1) && !L.cfmask_h.empty()) {
         for (int a = 0; a < dim; ++a) {
            // outer-side layout: tangential axes t0 (fastest) and t1
            const int t0 = a == 0 ? 1 : 0, t1 = a == 2 ? 1 : 2;
            const int m0 = n[t0], m1 = dim == 3 ? n[t1] : 1;
            for (int sd = 0; sd < 2; ++sd)
               for (int q1 = 0; q1 < m1; ++q1)
                  for (int q0 = 0; q0 < m0; ++q0) {
                     const long long o = d.offo[a][sd] + q0 + (long long)m0 * q1;
                     if (o < 0 || o >= (long long)L.cfmask_h.size())
                        throw FacError(FAC_ERR_ARG, "coarse-fine mask index");
                     if (!L.cfmask_h[o]) continue;
                     int x[3] = {0, 0, 0};
                     x[a] = sd ? n[a] - 1 : 0;
                     x[t0] = q0;
                     if (dim == 3) x[t1] = q1;
                     mark[cell(x)] = 1;
                  }
         }
      }
      if ((d.flags & 2) && !L.fcmask_h.empty()) {
         for (int a = 0; a < dim; ++a) {
            const int e0 = n[0] + (a == 0), e1 = n[1] + (a == 1), e2 = n[2] + (dim == 3 && a == 2);
            for (int k = 0; k < e2; ++k)
               for (int j = 0; j < e1; ++j)
                  for (int i = 0; i < e0; ++i) {
                     const long long si = d.offs[a] + i + (long long)e0 * (j + (long long)e1 * k);
                     if (si < 0 || si >= (long long)L.fcmask_h.size())
                        throw FacError(FAC_ERR_ARG, "finer-flux mask index");
                     if (!L.fcmask_h[si]) continue;
                     int x[3] = {i, j, k};
                     if (x[a] < n[a]) mark[cell(x)] = 1;  // the cell above the face
                     if (x[a] > 0) {                      // and the one below
                        --x[a];
                        mark[cell(x)] = 1;
                     }
                  }
         }
      }
      for (size_t q = 0; q < mark.size(); ++q)
         if (mark[q]) L.rfix.push_back({ip, (int)q});
   }
   L.d_rfix.upload(L.rfix, c->stream);
}

// Same-level neighbour of every face cell of every patch (fused colour
// pass).  The fused pass reads a neighbour patch's cell during a colour
// pass; that is exact only when the neighbour has the other colour, which
// holds for the global 3-D colouring and, in 2-D, when every patch of the
// level starts on the same parity of ifirst+jfirst (2d.f:140-147).
void build_facemap(fac_ctx *c, int ln)
{
   LevelState &L = c->L[ln];
   const int dim = c->dim;
   std::vector<long long> fmap(std::max<long long>(1, L.no), -3);
   // push targets: where a face cell's value goes in the neighbour's ghost
   // cells (staged pass), same -1 / -2 codes
   std::vector<int> pmap(std::max<long long>(1, L.no), -3);
   bool ok = L.n1 < (1ll << 31);
   int parity = -1;
   for (int ip = 0; ip < L.npatch && dim == 2; ++ip) {
      const int q = ((L.box[ip].lo[0] + L.box[ip].lo[1]) % 2 + 2) % 2;
      if (parity < 0) parity = q;
      else if (q != parity) ok = false;
   }
   for (int ip = 0; ip < L.npatch; ++ip) {
      const PatchDesc &d = L.hp[ip];
      const int p = d.prob;
      const Box &b = L.box[ip];
      const int pb = L.prob_patch_begin[p], pe = L.prob_patch_begin[p + 1];
      for (int a = 0; a < dim; ++a)
         for (int s = 0; s < 2; ++s) {
            Box layer = b;
            const int g = s == 0 ? b.lo[a] - 1 : b.hi[a] + 1;
            layer.lo[a] = layer.hi[a] = g;
            auto tlin = [&](int i, int j, int k) -> long long {
               if (a == 0) return (j - b.lo[1]) + (long long)(b.hi[1] - b.lo[1] + 1) * (k - b.lo[2]);
               if (a == 1) return (i - b.lo[0]) + (long long)(b.hi[0] - b.lo[0] + 1) * (k - b.lo[2]);
               return (i - b.lo[0]) + (long long)(b.hi[0] - b.lo[0] + 1) * (j - b.lo[1]);
            };
            const bool outside = g < L.domain[p].lo[a] || g > L.domain[p].hi[a];
            for (int k = layer.lo[2]; k <= layer.hi[2]; ++k)
               for (int j = layer.lo[1]; j <= layer.hi[1]; ++j)
                  for (int i = layer.lo[0]; i <= layer.hi[0]; ++i)
                     fmap[d.offo[a][s] + tlin(i, j, k)] = pmap[d.offo[a][s] + tlin(i, j, k)] =
                        outside ? -1 : -2;
            if (outside) continue;
            for (int iq = pb; iq < pe; ++iq) {
               if (iq == ip) continue;
               const Box ov = isect(layer, L.box[iq]);
               if (ov.empty()) continue;
               const Box qg = ghost_box(dim, L.box[iq], 1);
               const long long qnx = qg.hi[0] - qg.lo[0] + 1, qny = qg.hi[1] - qg.lo[1] + 1;
               for (int k = ov.lo[2]; k <= ov.hi[2]; ++k)
                  for (int j = ov.lo[1]; j <= ov.hi[1]; ++j)
                     for (int i = ov.lo[0]; i <= ov.hi[0]; ++i) {
                        fmap[d.offo[a][s] + tlin(i, j, k)] =
                           L.hp[iq].off1 + (i - qg.lo[0]) + qnx * ((j - qg.lo[1]) + qny * (k - qg.lo[2]));
                        // the face cell itself, one step back into patch ip
                        int x[3] = {i, j, k};
                        x[a] += s == 0 ? 1 : -1;
                        pmap[d.offo[a][s] + tlin(i, j, k)] = (int)(
                           L.hp[iq].off1 + (x[0] - qg.lo[0]) +
                           qnx * ((x[1] - qg.lo[1]) + qny * (x[2] - qg.lo[2])));
                     }
            }
         }
   }
   // -2 (not covered) must be exactly the coarse-fine faces
   std::vector<unsigned char> mask(std::max<long long>(1, L.no), 0);
   for (const CfFace &f : L.cf) mask[f.oidx] = 1;
   for (long long t = 0; t < L.no; ++t) {
      if (fmap[t] == -3) ok = false;
      if (fmap[t] >= L.n1 || pmap[t] >= L.n1 || (pmap[t] < 0) != (fmap[t] < 0) ||
          (fmap[t] < 0 && pmap[t] != fmap[t]))
         throw FacError(FAC_ERR_ARG, "face table index out of range");
      if ((fmap[t] == -2) != (mask[t] != 0))
         throw FacError(FAC_ERR_NESTING, "face table disagrees with the coarse-fine boundary");
   }
   L.fused_ok = ok;
   L.facemap_local = true;
   for (long long t = 0; t < L.no; ++t)
      if (fmap[t] >= 0) L.facemap_local = false;
   L.facemap.upload(fmap, c->stream);
   L.pushmap.upload(pmap, c->stream);
   L.pushmap_h = std::move(pmap);
   build_stage_units(c, ln);
}

void build_chunks(fac_ctx *c, int ln)
{
   LevelState &L = c->L[ln];
   const int dim = c->dim;
   const int np = nprob(c);
   L.cell_chunks.clear();
   L.slot_chunks.clear();
   L.flux_chunks.clear();
   L.prob_cell_chunk_begin.assign(np + 1, 0);
   int cur_prob = -1;
   for (int ip = 0; ip < L.npatch; ++ip) {
      const Box &b = L.box[ip];
      while (cur_prob < L.hp[ip].prob) {
         ++cur_prob;
         L.prob_cell_chunk_begin[cur_prob] = (int)L.cell_chunks.size();
      }
      const long long n = b.size();
      // aux: the chunk's own index (slot of its partial sums)
      for (long long s = 0; s < n; s += kChunk)
         L.cell_chunks.push_back({ip, (int)s, (int)std::min<long long>(kChunk, n - s),
                                  (int)L.cell_chunks.size()});
      const long long nx = b.hi[0] - b.lo[0] + 1;
      const long long slots = ((nx + 1) / 2) * (n / nx);
      for (long long s = 0; s < slots; s += kChunk)
         L.slot_chunks.push_back({ip, (int)s, (int)std::min<long long>(kChunk, slots - s), 0});
      for (int a = 0; a < dim; ++a) {
         const long long ns = side_box(b, a).size();
         for (long long s = 0; s < ns; s += kChunk)
            L.flux_chunks.push_back({ip, (int)s, (int)std::min<long long>(kChunk, ns - s), a});
      }
   }
   while (cur_prob < np) {
      ++cur_prob;
      L.prob_cell_chunk_begin[cur_prob] = (int)L.cell_chunks.size();
   }
   L.d_cell_chunks.upload(L.cell_chunks, c->stream);
   L.d_slot_chunks.upload(L.slot_chunks, c->stream);
   L.d_flux_chunks.upload(L.flux_chunks, c->stream);
   L.d_prob_cell_chunk_begin.upload(L.prob_cell_chunk_begin, c->stream);
   L.span_chunks.clear();
   L.prob_span_begin.assign(np + 1, 0);
   for (int p = 0; p < np; ++p) {
      L.prob_span_begin[p] = (int)L.span_chunks.size();
      const int pb = L.prob_patch_begin[p], pe = L.prob_patch_begin[p + 1];
      if (pb == pe) continue;
      const long long b0 = L.hp[pb].off0;
      long long e0 = b0;
      for (int ip = pb; ip < pe; ++ip) {
         if (L.hp[ip].off0 != e0) throw FacError(FAC_ERR_ARG, "problem cells not contiguous");
         e0 += L.box[ip].size();
      }
      if (e0 >= (1ll << 31)) throw FacError(FAC_ERR_ARG, "level too large for 32-bit chunks");
      for (long long q = b0; q < e0; q += kSpanChunk)
         L.span_chunks.push_back({p, (int)q, (int)std::min<long long>(kSpanChunk, e0 - q),
                                  (int)L.span_chunks.size()});
   }
   L.prob_span_begin[np] = (int)L.span_chunks.size();
   L.cells_prob.assign(np, 0.0);
   for (int ip = 0; ip < L.npatch; ++ip) L.cells_prob[L.hp[ip].prob] += (double)L.box[ip].size();
   L.d_span_chunks.upload(L.span_chunks, c->stream);
   L.d_prob_span_begin.upload(L.prob_span_begin, c->stream);
   L.norm_partial.alloc(std::max<size_t>(1, L.cell_chunks.size()));
   std::vector<int> last(np, 0);
   for (int p = 0; p < np; ++p) last[p] = L.prob_patch_begin[p + 1] - 1;
   L.last_patch.upload(last, c->stream);
   L.maxres_red.alloc(std::max(1, L.npatch));
   L.maxres_blk.alloc(std::max(1, L.npatch));
   // one block per problem pays off for small patches only
   L.one_patch_per_prob = L.npatch == np;
   for (int ip = 0; ip < L.npatch; ++ip)
      if (L.hp[ip].prob != ip || L.box[ip].size() > 16384) L.one_patch_per_prob = false;
   // the one-launch solve on shared copies of u, f, D and C (FP64)
   L.solve_smem = 0;
   if (L.one_patch_per_prob && L.facemap_local) {
      long long most = 0;
      for (int ip = 0; ip < L.npatch; ++ip) {
         const Box &b = L.box[ip];
         long long n = cell_count(c->dim, b, 1) + b.size();
         if (c->spec.d_variable)
            for (int a = 0; a < c->dim; ++a) n += side_box(b, a).size();
         if (c->spec.c_kind == 2) n += b.size();
         most = std::max(most, 8 * n);
      }
      if (most <= kSolveSmemMax) L.solve_smem = (int)most;
   }
   // one colour pass reads u over the ghosted boxes, f at the active half,
   // writes u at the active half, and reads D on all faces when variable
   double n = 0, ng = 0;
   for (int ip = 0; ip < L.npatch; ++ip) {
      n += (double)L.box[ip].size();
      ng += (double)cell_count(dim, L.box[ip], 1);
   }
   L.rb_bytes = 8.0 * (ng + n) + (c->spec.d_variable ? 8.0 * dim * n : 0.0) +
                (c->spec.c_kind == 2 ? 4.0 * n : 0.0);
   L.rb_bytes_prob.assign(np, 0.0);
   for (int ip = 0; ip < L.npatch; ++ip) {
      const double pn = (double)L.box[ip].size(), pg = (double)cell_count(dim, L.box[ip], 1);
      L.rb_bytes_prob[L.hp[ip].prob] += 8.0 * (pg + pn) +
                                         (c->spec.d_variable ? 8.0 * dim * pn : 0.0) +
                                         (c->spec.c_kind == 2 ? 4.0 * pn : 0.0);
   }
   double gcells = 0;
   L.fill_bytes_prob.assign(np, 0.0);
   for (const FillItem &it : L.fill_nc.items) {
      Box b;
      for (int a = 0; a < 3; ++a) {
         b.lo[a] = it.lo[a];
         b.hi[a] = it.hi[a];
      }
      gcells += (double)b.size();
      L.fill_bytes_prob[it.prob] += 16.0 * (double)b.size();
   }
   L.fill_bytes = 16.0 * gcells;
}

// Inter-level tables with the next finer level (restriction, flux coarsening).
void build_coarsen_tables(fac_ctx *c, int ln)
{
   LevelState &C = c->L[ln];
   LevelState &Fl = c->L[ln + 1];
   const int dim = c->dim;
   const int np = nprob(c);
   C.restrict_g1.clear();
   C.restrict_g0.clear();
   C.fcoarsen.clear();
   const int *r = Fl.ratio;
   const int raux = r[0] | (r[1] << 8) | ((dim == 3 ? r[2] : 1) << 16);
   for (int p = 0; p < np; ++p) {
      const int fb = Fl.prob_patch_begin[p], fe = Fl.prob_patch_begin[p + 1];
      const int cb = C.prob_patch_begin[p], ce = C.prob_patch_begin[p + 1];
      std::vector<FluxCoarsenItem> fcs;  // this problem's, in the reference's order
      for (int ip = fb; ip < fe; ++ip) {
         const Box cbox = coarsen(Fl.box[ip], dim, r);
         for (int iq = cb; iq < ce; ++iq) {
            for (int g = 0; g < 2; ++g) {
               Box ov = isect(cbox, ghost_box(dim, C.box[iq], g));
               if (ov.empty()) continue;
               RestrictItem it;
               it.prob = p;
               it.fine_patch = ip;
               it.coarse_patch = iq;
               for (int a = 0; a < 3; ++a) {
                  it.lo[a] = ov.lo[a];
                  it.hi[a] = ov.hi[a];
               }
               it.ratio = raux;
               (g ? C.restrict_g1 : C.restrict_g0).add(it, ov.size());
            }
         }
         for (int a = 0; a < dim; ++a) {
            int t0 = -1, t1 = -1;
            for (int t = 0; t < dim; ++t)
               if (t != a) {
                  if (t0 < 0) t0 = t;
                  else t1 = t;
               }
            for (int s = 0; s < 2; ++s) {
               Box T = cbox;
               const int cf = s == 0 ? cbox.lo[a] : cbox.hi[a] + 1;
               T.lo[a] = T.hi[a] = cf;
               for (int iq = cb; iq < ce; ++iq) {
                  Box ov = isect(T, side_box(C.box[iq], a));
                  if (ov.empty()) continue;
                  FluxCoarsenItem it;
                  it.prob = p;
                  it.axis = a;
                  it.side = s;
                  it.fine_patch = ip;
                  it.coarse_patch = iq;
                  for (int d = 0; d < 3; ++d) {
                     it.lo[d] = ov.lo[d];
                     it.hi[d] = ov.hi[d];
                  }
                  it.fface = s == 0 ? Fl.box[ip].lo[a] : Fl.box[ip].hi[a] + 1;
                  it.t0 = t0;
                  it.t1 = t1;
                  const int aux = r[t0] | ((t1 >= 0 ? r[t1] : 1) << 8);
                  it.ratio = aux;
                  fcs.push_back(it);
               }
            }
         }
      }
      // Two fine patches that share a face both coarsen it onto the same
      // coarse faces.  Their values agree only as far as the two patches'
      // copies of D on the shared face do; the reference's schedule writes
      // the items in order and the last one stays (xfer/CoarsenSchedule.C:
      // 275-330 over the fine patches in order, lower side before upper).
      // Each item keeps only the faces no later item writes, so every
      // coarse face has one writer and the result is the reference's.
      for (size_t i = 0; i < fcs.size(); ++i) {
         const FluxCoarsenItem &it = fcs[i];
         Box bi;
         for (int d = 0; d < 3; ++d) {
            bi.lo[d] = it.lo[d];
            bi.hi[d] = it.hi[d];
         }
         std::vector<Box> keep{bi};
         for (size_t j = i + 1; j < fcs.size() && !keep.empty(); ++j) {
            const FluxCoarsenItem &jt = fcs[j];
            if (jt.coarse_patch != it.coarse_patch || jt.axis != it.axis ||
                jt.lo[it.axis] != it.lo[it.axis])
               continue;
            Box bj;
            for (int d = 0; d < 3; ++d) {
               bj.lo[d] = jt.lo[d];
               bj.hi[d] = jt.hi[d];
            }
            subtract_all(keep, bj);
         }
         for (const Box &k : keep) {
            if (k.empty()) continue;
            FluxCoarsenItem piece = it;
            for (int d = 0; d < 3; ++d) {
               piece.lo[d] = k.lo[d];
               piece.hi[d] = k.hi[d];
            }
            C.fcoarsen.add(piece, k.size());
         }
      }
   }
   C.restrict_g1.upload(c->stream);
   C.restrict_g0.upload(c->stream);
   C.fcoarsen.upload(c->stream);
   // faces of level ln written by the flux coarsening
   std::vector<unsigned char> fm(std::max<long long>(1, C.ns), 0);
   for (const FluxCoarsenItem &it : C.fcoarsen.items) {
      const PatchDesc &cp = C.hp[it.coarse_patch];
      const int a = it.axis;
      const long long nxa = cp.hi[0] - cp.lo[0] + 1 + (a == 0);
      const long long nya = cp.hi[1] - cp.lo[1] + 1 + (a == 1);
      for (int k = it.lo[2]; k <= it.hi[2]; ++k)
         for (int j = it.lo[1]; j <= it.hi[1]; ++j)
            for (int i = it.lo[0]; i <= it.hi[0]; ++i) {
               const long long si = cp.offs[a] + (i - cp.lo[0]) +
                                    nxa * ((j - cp.lo[1]) + nya * (k - cp.lo[2]));
               if (si < 0 || si >= C.ns) throw FacError(FAC_ERR_ARG, "flux coarsening face");
               fm[si] = 1;
            }
      C.hp[it.coarse_patch].flags |= 2;
   }
   C.fcmask.upload(fm, c->stream);
   C.fcmask_h = std::move(fm);
}

// Coarse interpolation arrays for prolongation into level ln
// (RefineSchedule coarse interpolation level, RefineSchedule.C:1353-1560).
void build_fill_gather(fac_ctx *c, ItemList<FillItem> &F, FillGather &G, long long dstlen,
                       long long samelen, long long coarselen);

void build_prolong_tables(fac_ctx *c, int ln)
{
   LevelState &Fl = c->L[ln];
   LevelState &C = c->L[ln - 1];
   const int dim = c->dim;
   Fl.tmp_fill.clear();
   Fl.prolong.clear();
   Fl.prolong2.clear();
   Fl.prolong_r2 = Fl.ratio[0] == 2 && Fl.ratio[1] == 2 && (dim == 2 || Fl.ratio[2] == 2);
   auto sides = all_sides(dim);
   long long toff = 0;
   for (int ip = 0; ip < Fl.npatch; ++ip) {
      const int p = Fl.hp[ip].prob;
      const Box fill = ghost_box(dim, Fl.box[ip], 1);
      const Box B = isect(coarsen(fill, dim, Fl.ratio), C.domain[p]);
      const Box Bg = ghost_box(dim, B, 1);
      const ArrDesc T = make_desc(toff, Bg);
      toff += Bg.size();
      const int cb = C.prob_patch_begin[p], ce = C.prob_patch_begin[p + 1];
      for (int iq = cb; iq < ce; ++iq) {
         Box ov = isect(Bg, C.box[iq]);
         if (ov.empty()) continue;
         FillItem it;
         std::memset(&it, 0, sizeof(it));
         it.kind = kFillCopy;
         it.prob = p;
         for (int a = 0; a < 3; ++a) {
            it.lo[a] = ov.lo[a];
            it.hi[a] = ov.hi[a];
         }
         it.dst = T;
         it.src = patch_desc(c, C, iq, 1);
         it.src_is_coarse = 1;
         Fl.tmp_fill.add(it, ov.size());
      }
      for (auto &s : sides) {
         Box bb;
         if (!bc_box(dim, B, C.domain[p], s.data(), bb)) continue;
         Box inward = bb;
         for (int a = 0; a < 3; ++a) {
            inward.lo[a] -= s[a];
            inward.hi[a] -= s[a];
         }
         for (int iq = cb; iq < ce; ++iq) {
            Box sub = isect(inward, C.box[iq]);
            if (sub.empty()) continue;
            FillItem it;
            std::memset(&it, 0, sizeof(it));
            it.kind = kFillBc;
            it.prob = p;
            for (int a = 0; a < 3; ++a) {
               it.lo[a] = sub.lo[a] + s[a];
               it.hi[a] = sub.hi[a] + s[a];
               it.side[a] = s[a];
               it.h[a] = C.dx[3 * p + a];
            }
            it.bc_level = ln - 1;  // the coarse level's boundary coefficients
            it.dst = T;
            it.src = patch_desc(c, C, iq, 1);
            it.src_is_coarse = 1;
            Fl.tmp_fill.add(it, sub.size());
         }
      }
      ProlongItem pi;
      pi.prob = p;
      pi.fine_patch = ip;
      pi.tmp = T;
      Fl.prolong.add(pi, Fl.box[ip].size());
      if (Fl.prolong_r2) Fl.prolong2.add(pi, Fl.box[ip].size() / (dim == 3 ? 8 : 4));
   }
   Fl.tmp.alloc(std::max<long long>(1, toff));
   if (c->mixed) {
      Fl.tmp32.alloc(std::max<long long>(1, toff));
      if (!g_dry)
         CUDA_CHECK(cudaMemsetAsync(Fl.tmp32.p, 0xff, Fl.tmp32.n * sizeof(float), c->stream));
   }
   // cells of the interpolation array that nothing fills stay NaN
   if (!g_dry)
      CUDA_CHECK(cudaMemsetAsync(Fl.tmp.p, 0xff, Fl.tmp.n * sizeof(double), c->stream));
   Fl.tmp_fill.upload(c->stream);
   // every source of the interpolation array is on the coarser level
   build_fill_gather(c, Fl.tmp_fill, Fl.gather_tmp, toff, 0, C.n1);
   Fl.prolong.upload(c->stream);
   Fl.prolong2.upload(c->stream);
   std::vector<double> dxc(3 * nprob(c));
   for (int p = 0; p < nprob(c); ++p)
      for (int a = 0; a < 3; ++a) dxc[3 * p + a] = C.dx[3 * p + a];
   Fl.dxc_prob.upload(dxc, c->stream);
}

// Cells of the codimension-1 physical boundary boxes of u (untrimmed:
// BaseGridGeometry::getBoundaryBoxes grows them one cell tangentially),
// saved and restored by SimpleCellRobinBcCoefs::cacheDirichletData /
// restoreDirichletData.
void build_dirichlet_index(fac_ctx *c, int ln)
{
   LevelState &L = c->L[ln];
   const int dim = c->dim;
   L.dir_idx.clear();
   for (int ip = 0; ip < L.npatch; ++ip) {
      const int p = L.hp[ip].prob;
      const Box &b = L.box[ip];
      const Box &dom = L.domain[p];
      const Box gb = ghost_box(dim, b, 1);
      const long long nx = gb.hi[0] - gb.lo[0] + 1, ny = gb.hi[1] - gb.lo[1] + 1;
      for (int k = gb.lo[2]; k <= gb.hi[2]; ++k)
         for (int j = gb.lo[1]; j <= gb.hi[1]; ++j)
            for (int i = gb.lo[0]; i <= gb.hi[0]; ++i) {
               const int cc[3] = {i, j, k};
               int out = 0;
               bool ok = true;
               for (int a = 0; a < dim; ++a)
                  if (cc[a] < dom.lo[a] || cc[a] > dom.hi[a]) {
                     ++out;
                     if (!((cc[a] == b.lo[a] - 1 && b.lo[a] == dom.lo[a]) ||
                           (cc[a] == b.hi[a] + 1 && b.hi[a] == dom.hi[a])))
                        ok = false;
                  }
               if (!ok || out != 1) continue;
               L.dir_idx.push_back(L.hp[ip].off1 + (i - gb.lo[0]) +
                                   nx * ((j - gb.lo[1]) + ny * (k - gb.lo[2])));
            }
   }
   L.d_dir_idx.upload(L.dir_idx, c->stream);
   L.dir_cache.alloc(std::max<size_t>(1, L.dir_idx.size()));
}

// CellPoissonFACOps::computeVectorWeights (CellPoissonFACOps.C:2005-2102).
void compute_weights_host(fac_ctx *c)
{
   if (g_dry) return;
   const int dim = c->dim;
   for (int ln = c->nlev - 1; ln >= 0; --ln) {
      LevelState &L = c->L[ln];
      std::vector<double> w(std::max<long long>(1, L.n0), 0.0);
      for (int ip = 0; ip < L.npatch; ++ip) {
         const int p = L.hp[ip].prob;
         double vol = L.dx[3 * p + 0];
         vol *= L.dx[3 * p + 1];
         if (dim > 2) vol *= L.dx[3 * p + 2];
         const Box &b = L.box[ip];
         const long long n = b.size();
         for (long long t = 0; t < n; ++t) w[L.hp[ip].off0 + t] = vol;
         if (ln < c->nlev - 1) {
            LevelState &Fl = c->L[ln + 1];
            const long long nx = b.hi[0] - b.lo[0] + 1, ny = b.hi[1] - b.lo[1] + 1;
            for (int iq = Fl.prob_patch_begin[p]; iq < Fl.prob_patch_begin[p + 1]; ++iq) {
               Box ov = isect(coarsen(Fl.box[iq], dim, Fl.ratio), b);
               if (ov.empty()) continue;
               for (int k = ov.lo[2]; k <= ov.hi[2]; ++k)
                  for (int j = ov.lo[1]; j <= ov.hi[1]; ++j)
                     for (int i = ov.lo[0]; i <= ov.hi[0]; ++i)
                        w[L.hp[ip].off0 + (i - b.lo[0]) + nx * ((j - b.lo[1]) + ny * (k - b.lo[2]))] =
                           0.0;
            }
         }
      }
      CUDA_CHECK(cudaMemcpyAsync(L.w.p, w.data(), L.n0 * sizeof(double), cudaMemcpyHostToDevice,
                                 c->stream));
   }
}

// Host-side bounds check of every device table before any kernel runs:
// each transaction's destination and source cells must lie inside the
// arrays they address, and every array inside its buffer.
void vcheck(bool ok, const char *what)
{
   if (!ok) throw FacError(FAC_ERR_ARG, std::string("table validation failed: ") + what);
}

bool desc_contains(const ArrDesc &d, const Box &b, long long buflen)
{
   if (b.empty()) return true;
   for (int a = 0; a < 3; ++a)
      if (b.lo[a] < d.lo[a] || b.hi[a] > d.lo[a] + d.n[a] - 1) return false;
   const long long n = (long long)d.n[0] * d.n[1] * d.n[2];
   return d.base >= 0 && d.base + n <= buflen;
}

Box item_box(const int *lo, const int *hi)
{
   Box b;
   for (int a = 0; a < 3; ++a) {
      b.lo[a] = lo[a];
      b.hi[a] = hi[a];
   }
   return b;
}

// Packed chunk ranges of a transaction list (see ItemList::pack).
template <class I>
void validate_chunks(ItemList<I> &L, const char *what)
{
   L.pack();
   for (const Chunk &ch : L.chunks) {
      vcheck(ch.patch >= 0 && ch.aux >= 1 && ch.patch + ch.aux <= (int)L.items.size(), what);
      if (ch.aux == 1)
         vcheck(ch.begin >= 0 && ch.count > 0 && ch.begin + ch.count <= L.cells[ch.patch], what);
      else
         vcheck(ch.begin == 0 && ch.count == L.prefix[ch.patch + ch.aux] - L.prefix[ch.patch] &&
                   ch.count <= kChunk,
                what);
      for (int j = ch.patch; j < ch.patch + ch.aux; ++j)
         vcheck(L.items[j].prob == L.items[ch.patch].prob, what);
   }
}

void validate_fill(ItemList<FillItem> &L, long long dstlen, long long samelen,
                   long long coarselen)
{
   for (const FillItem &it : L.items) {
      const Box b = item_box(it.lo, it.hi);
      vcheck(!b.empty(), "empty fill item");
      vcheck(desc_contains(it.dst, b, dstlen), "fill destination");
      Box sb = b;
      if (it.kind == kFillCoarse) {
         for (int a = 0; a < 3; ++a) {
            vcheck(it.ratio[a] >= 1, "fill ratio");
            sb.lo[a] = coarsen_index(b.lo[a], it.ratio[a]);
            sb.hi[a] = coarsen_index(b.hi[a], it.ratio[a]);
         }
      } else if (it.kind == kFillBc) {
         for (int a = 0; a < 3; ++a) {
            sb.lo[a] -= it.side[a];
            sb.hi[a] -= it.side[a];
         }
      }
      vcheck(desc_contains(it.src, sb, it.src_is_coarse ? coarselen : samelen), "fill source");
   }
   for (size_t i = 0; i < L.items.size(); ++i)
      vcheck(L.cells[i] == item_box(L.items[i].lo, L.items[i].hi).size(), "fill item cells");
   validate_chunks(L, "fill chunk range");
}

// Gather list of a validated fill.  Falls back to the item kernel (ok =
// false) when an element index does not fit its 32-bit field or two items
// share a destination element.
void build_fill_gather(fac_ctx *c, ItemList<FillItem> &F, FillGather &G, long long dstlen,
                       long long samelen, long long coarselen)
{
   G.to.clear();
   G.from.clear();
   G.prob.clear();
   G.bc.clear();
   G.ok = dstlen <= 0xffffffffll && samelen < (1ll << 31) && coarselen < (1ll << 31) &&
          nprob(c) <= 0xffff;
   auto idx = [](const ArrDesc &A, int i, int j, int k) {
      return A.base + (long long)(i - A.lo[0]) +
             (long long)A.n[0] * ((long long)(j - A.lo[1]) + (long long)A.n[1] * (k - A.lo[2]));
   };
   auto crs = [](int i, int r) { return i < 0 ? (i + 1) / r - 1 : i / r; };
   std::vector<unsigned char> seen(G.ok ? std::max<long long>(1, dstlen) : 1, 0);
   for (const FillItem &it : F.items) {
      if (!G.ok) break;
      const Box b = item_box(it.lo, it.hi);
      if (it.kind == kFillBc) {
         for (int k = b.lo[2]; k <= b.hi[2]; ++k)
            for (int j = b.lo[1]; j <= b.hi[1]; ++j)
               for (int i = b.lo[0]; i <= b.hi[0]; ++i) {
                  const long long d = idx(it.dst, i, j, k);
                  if (seen[d]) G.ok = false;
                  seen[d] = 1;
               }
         G.bc.add(it, b.size());
         continue;
      }
      const bool coarse = it.src_is_coarse != 0;
      const long long slen = coarse ? coarselen : samelen;
      for (int k = b.lo[2]; k <= b.hi[2] && G.ok; ++k)
         for (int j = b.lo[1]; j <= b.hi[1]; ++j)
            for (int i = b.lo[0]; i <= b.hi[0]; ++i) {
               const long long d = idx(it.dst, i, j, k);
               const long long sidx =
                  it.kind == kFillCopy
                     ? idx(it.src, i, j, k)
                     : idx(it.src, crs(i, it.ratio[0]), crs(j, it.ratio[1]), crs(k, it.ratio[2]));
               vcheck(d >= 0 && d < dstlen && sidx >= 0 && sidx < slen, "fill gather element");
               if (seen[d]) G.ok = false;
               seen[d] = 1;
               G.to.push_back((unsigned)d);
               G.from.push_back(coarse ? -(int)sidx - 1 : (int)sidx);
               G.prob.push_back((unsigned short)it.prob);
            }
      if (G.to.size() >= (size_t)1 << 31) G.ok = false;
   }
   if (!G.ok) {
      G.to.clear();
      G.from.clear();
      G.prob.clear();
      G.bc.clear();
      return;
   }
   G.d_to.upload(G.to, c->stream);
   G.d_from.upload(G.from, c->stream);
   G.d_prob.upload(G.prob, c->stream);
   G.bc.upload(c->stream);
}

void validate_tables(fac_ctx *c)
{
   const int dim = c->dim;
   for (int ln = 0; ln < c->nlev; ++ln) {
      LevelState &L = c->L[ln];
      const long long clen = ln > 0 ? c->L[ln - 1].n1 : 0;
      validate_fill(L.fill_nc, L.n1, L.n1, clen);
      validate_fill(L.fill_wc, L.n1, L.n1, clen);
      for (int ip = 0; ip < L.npatch; ++ip) {
         const PatchDesc &d = L.hp[ip];
         vcheck(d.off1 + cell_count(dim, L.box[ip], 1) <= L.n1, "patch ghost-1 extent");
         vcheck(d.off0 + cell_count(dim, L.box[ip], 0) <= L.n0, "patch ghost-0 extent");
         for (int a = 0; a < dim; ++a) {
            vcheck(d.offs[a] + side_box(L.box[ip], a).size() <= L.ns, "patch side extent");
            for (int s = 0; s < 2; ++s)
               vcheck(d.offo[a][s] + face_box(L.box[ip], a, s).size() <= L.no,
                      "patch outer-side extent");
         }
      }
      for (const CfFace &f : L.cf) {
         vcheck(f.cell >= 0 && f.cell < L.n1 && f.mirror >= 0 && f.mirror < L.n1 &&
                   f.ghost >= 0 && f.ghost < L.n1,
                "cf cell index");
         vcheck(f.oidx >= 0 && f.oidx < L.no && f.sidx >= 0 && f.sidx < L.ns, "cf face index");
      }
      for (const Chunk &ch : L.cell_chunks)
         vcheck(ch.patch >= 0 && ch.patch < L.npatch &&
                   ch.begin + ch.count <= L.box[ch.patch].size(),
                "cell chunk");
      for (const Chunk &ch : L.slot_chunks) {
         const Box &b = L.box[ch.patch];
         const long long nx = b.hi[0] - b.lo[0] + 1;
         vcheck(ch.begin + ch.count <= ((nx + 1) / 2) * (b.size() / nx), "slot chunk");
      }
      for (const Chunk &ch : L.flux_chunks)
         vcheck(ch.aux >= 0 && ch.aux < dim &&
                   ch.begin + ch.count <= side_box(L.box[ch.patch], ch.aux).size(),
                "flux chunk");
      if (ln > 0) {
         LevelState &C = c->L[ln - 1];
         validate_fill(L.tmp_fill, (long long)L.tmp.n, 0, C.n1);
         for (const ProlongItem &pi : L.prolong.items) {
            // linear refine reads coarse cells coarsen(box) -1 .. +1
            Box need = grow(coarsen(L.box[pi.fine_patch], dim, L.ratio), dim, 1);
            vcheck(desc_contains(pi.tmp, need, (long long)L.tmp.n), "prolong stencil");
         }
      }
      if (ln + 1 < c->nlev) {
         LevelState &Fl = c->L[ln + 1];
         for (int g = 0; g < 2; ++g) {
            const ItemList<RestrictItem> &R = g ? L.restrict_g1 : L.restrict_g0;
            for (const RestrictItem &it : R.items) {
               const Box b = item_box(it.lo, it.hi);
               vcheck(isect(b, ghost_box(dim, L.box[it.coarse_patch], g)).size() == b.size(),
                      "restrict destination");
               vcheck(isect(refine(b, dim, Fl.ratio), Fl.box[it.fine_patch]).size() ==
                         refine(b, dim, Fl.ratio).size(),
                      "restrict source");
            }
         }
         for (const FluxCoarsenItem &it : L.fcoarsen.items) {
            const Box b = item_box(it.lo, it.hi);
            vcheck(isect(b, side_box(L.box[it.coarse_patch], it.axis)).size() == b.size(),
                   "flux coarsen destination");
            Box fb = refine(b, dim, Fl.ratio);
            fb.lo[it.axis] = fb.hi[it.axis] = it.fface;
            vcheck(isect(fb, face_box(Fl.box[it.fine_patch], it.axis, it.side)).size() ==
                      fb.size(),
                   "flux coarsen source");
         }
      }
   }
   for (int ln = 0; ln < c->nlev; ++ln) {
      LevelState &L = c->L[ln];
      validate_chunks(L.restrict_g1, "restrict chunk range");
      validate_chunks(L.restrict_g0, "restrict chunk range");
      validate_chunks(L.fcoarsen, "flux coarsening chunk range");
      validate_chunks(L.tmp_fill, "coarse interpolation chunk range");
      validate_chunks(L.prolong, "prolongation chunk range");
   }
}

// Record one work list for device-side compaction; its chunks must be in
// problem order.
template <class ProbOf>
void register_work(fac_ctx *c, WorkSrc &ws, const std::vector<Chunk> &chunks, Chunk *list,
                   ProbOf prob_of)
{
   const int np = nprob(c);
   std::vector<int> pcb(np + 1, 0);
   int prev = 0;
   for (const Chunk &ch : chunks) {
      const int p = prob_of(ch);
      if (p < prev || p >= np) throw FacError(FAC_ERR_ARG, "work list not in problem order");
      prev = p;
      pcb[p + 1] += 1;
   }
   for (int p = 0; p < np; ++p) pcb[p + 1] += pcb[p];
   if (!chunks.empty() && !list && !g_dry)
      throw FacError(FAC_ERR_STATE, "work list registered before its upload");
   ws.all.upload(chunks, c->stream);
   ws.pcb.upload(pcb, c->stream);
   if (!chunks.empty()) c->work_regs.push_back({ws.all.p, list, ws.pcb.p, (int)chunks.size(), 0});
}

template <class I>
void register_items(fac_ctx *c, ItemList<I> &it)
{
   register_work(c, it.ws, it.chunks, it.d_chunks.p,
                 [&](const Chunk &ch) { return it.items[ch.patch].prob; });
}

void register_work_lists(fac_ctx *c)
{
   c->work_regs.clear();
   for (int ln = 0; ln < c->nlev; ++ln) {
      LevelState &L = c->L[ln];
      auto pp = [&](const Chunk &ch) { return L.hp[ch.patch].prob; };
      register_work(c, L.ws_cell, L.cell_chunks, L.d_cell_chunks.p, pp);
      register_work(c, L.ws_slot, L.slot_chunks, L.d_slot_chunks.p, pp);
      register_work(c, L.ws_flux, L.flux_chunks, L.d_flux_chunks.p, pp);
      register_work(c, L.ws_span, L.span_chunks, L.d_span_chunks.p,
                    [](const Chunk &ch) { return ch.patch; });
      register_items(c, L.fill_nc);
      register_items(c, L.fill_wc);
      for (FillGather *G : {&L.gather_nc, &L.gather_wc})
         if (G->ok) register_items(c, G->bc);
      register_items(c, L.restrict_g1);
      register_items(c, L.restrict_g0);
      register_items(c, L.fcoarsen);
      register_items(c, L.tmp_fill);
      if (L.gather_tmp.ok) register_items(c, L.gather_tmp.bc);
      register_items(c, L.prolong);
      register_items(c, L.prolong2);
      for (int t = 0; t < 2; ++t)
         register_work(c, L.ws_units[t], L.units[t], L.d_units[t].p, pp);
      for (int k = 0; k < kResKinds; ++k)
         register_work(c, L.ws_runits[k], L.runits[k], L.d_runits[k].p, pp);
   }
   c->d_work_regs.upload(c->work_regs, c->stream);
}

// New active flags: upload them and compact every work list to the chunks of
// the active problems (stream ordered, so graph replays see the new lists).
void set_active(fac_ctx *c, const std::vector<int> &act)
{
   const int np = nprob(c);
   CUDA_CHECK(cudaMemcpyAsync(c->active.p, act.data(), np * sizeof(int), cudaMemcpyHostToDevice,
                              c->stream));
   launch_compact(c->stream, c->d_work_regs.p, (int)c->work_regs.size(), c->active.p, np);
   CUDA_CHECK(cudaGetLastError());
}

void initialize(fac_ctx *c)
{
   if (c->probs.empty()) throw FacError(FAC_ERR_STATE, "no problems added");
   if (!c->ewing) throw FacError(FAC_ERR_ARG, "only cf_discretization Ewing is implemented");
   c->nlev = c->probs[0].nlev;
   for (auto &P : c->probs) {
      if (P.nlev != c->nlev) throw FacError(FAC_ERR_ARG, "problems must share the level count");
      for (int ln = 0; ln < c->nlev; ++ln)
         for (int a = 0; a < 3; ++a)
            if (P.ratio[ln][a] != c->probs[0].ratio[ln][a])
               throw FacError(FAC_ERR_ARG, "problems must share refinement ratios");
   }
   g_dry = c->device < 0;
   struct DryReset {
      ~DryReset() { g_dry = false; }
   } dry_reset;
   if (!g_dry) CUDA_CHECK(cudaSetDevice(c->device));
   const int np = nprob(c);
   for (int ln = 0; ln < c->nlev; ++ln) {
      LevelState &L = c->L[ln];
      build_level_layout(c, ln);
      const size_t n1 = std::max<long long>(1, L.n1), n0 = std::max<long long>(1, L.n0);
      L.u.alloc(n1);
      L.e.alloc(n1);
      L.f.alloc(n0);
      L.r.alloc(n0);
      L.tr.alloc(n0);
      L.w.alloc(n0);
      L.c.alloc(c->spec.c_kind == 2 ? n0 : 1);
      L.d.alloc(c->spec.d_variable ? std::max<long long>(1, L.ns) : 1);
      L.flux.alloc(std::max<long long>(1, L.ns));
      L.oflux.alloc(std::max<long long>(1, L.no));
      L.cfflux.alloc(std::max<long long>(1, L.no));
      L.zero.alloc(n0);
      if (!g_dry) CUDA_CHECK(cudaMemsetAsync(L.zero.p, 0, n0 * sizeof(double), c->stream));
      if (!g_dry)
         for (auto *b : {&L.u, &L.e, &L.f, &L.r, &L.tr, &L.w, &L.c, &L.d, &L.flux, &L.oflux,
                         &L.cfflux})
            CUDA_CHECK(cudaMemsetAsync(b->p, 0, b->n * sizeof(double), c->stream));
      std::vector<int> rr(L.ratio, L.ratio + 3);
      L.d_ratio.upload(rr, c->stream);
      if (c->mixed) {
         L.e32.alloc(n1);
         L.r32.alloc(n0);
         L.d32.alloc(c->spec.d_variable ? std::max<long long>(1, L.ns) : 1);
         L.c32.alloc(c->spec.c_kind == 2 ? n0 : 1);
         L.cfflux32.alloc(std::max<long long>(1, L.no));
         if (!g_dry)
            for (auto *b : {&L.e32, &L.r32, &L.d32, &L.c32, &L.cfflux32})
               CUDA_CHECK(cudaMemsetAsync(b->p, 0, b->n * sizeof(float), c->stream));
      }
   }
   for (int ln = 0; ln < c->nlev; ++ln) {
      build_fill_tables(c, ln);
      build_cf_faces(c, ln);
      build_facemap(c, ln);
      build_chunks(c, ln);
      build_dirichlet_index(c, ln);
      if (ln > 0) build_prolong_tables(c, ln);
   }
   for (int ln = 0; ln + 1 < c->nlev; ++ln) build_coarsen_tables(c, ln);
   for (int ln = 0; ln < c->nlev; ++ln) {
      build_res_units(c, ln);
      build_residual_fixups(c, ln);
   }
   validate_tables(c);
   for (int ln = 0; ln < c->nlev; ++ln) {
      LevelState &L = c->L[ln];
      L.d_patches.upload(L.hp, c->stream);  // after cf flags are set
      L.fill_nc.upload(c->stream);
      L.fill_wc.upload(c->stream);
      const long long clen = ln > 0 ? c->L[ln - 1].n1 : 0;
      build_fill_gather(c, L.fill_nc, L.gather_nc, L.n1, L.n1, clen);
      build_fill_gather(c, L.fill_wc, L.gather_wc, L.n1, L.n1, clen);
   }
   register_work_lists(c);
   c->kerr.alloc(1);
   if (!g_dry) CUDA_CHECK(cudaMemsetAsync(c->kerr.p, 0, sizeof(int), c->stream));
   std::vector<int> ones(np, 1);
   c->active.upload(ones, c->stream);
   c->run.upload(ones, c->stream);
   c->sweeps_call.alloc(np);
   c->sweeps_coarse.alloc(np);
   c->norm_acc.alloc(np);
   c->hist.assign(np, {});
   if (!g_dry) {
      CUDA_CHECK(cudaMemsetAsync(c->sweeps_coarse.p, 0, np * sizeof(long long), c->stream));
      compute_weights_host(c);
      CUDA_CHECK(cudaStreamSynchronize(c->stream));
   }
   c->initialized = true;
}

// ---------------------------------------------------------------------------
// level operators
// ---------------------------------------------------------------------------

void ghost_fill(fac_ctx *c, int fid, int ln, bool with_coarse, int homogeneous, const int *mask)
{
   LevelState &L = c->L[ln];
   if (field_ghost(fid) != 1) return;  // ghost-0 fields have no ghosts to fill
   double *dst = field_ptr(L, fid);
   const double *coarse = ln > 0 ? field_ptr(c->L[ln - 1], fid) : nullptr;
   ItemList<FillItem> &it = (with_coarse && ln > 0) ? L.fill_wc : L.fill_nc;
   FillGather &G = (with_coarse && ln > 0) ? L.gather_wc : L.gather_nc;
   const int pi = prof_begin(c, 1, L.fill_bytes_prob, 1.0);
   if (G.ok)
      launch_fill_gather(c->stream, (long long)G.to.size(), G.d_to.p, G.d_from.p, G.d_prob.p,
                         G.bc.d_items.p, G.bc.d_chunks.p, G.bc.nchunks(), G.bc.d_prefix.p, dst,
                         dst, coarse, homogeneous, c->bc, mask);
   else
      launch_fill(c->stream, it.d_items.p, it.d_chunks.p, it.nchunks(), it.d_prefix.p, dst, dst,
                  coarse, homogeneous, c->bc, mask);
   prof_end(c, pi);
}

// CellPoissonFACOps::smoothErrorByRedBlack (CellPoissonFACOps.C:1339-1514).
void smooth(fac_ctx *c, int fid_e, int fid_r, int ln, int nsweeps, double tol)
{
   OpTimer ot(c, tol >= 0 ? "smooth_to_tol" : "smooth", ln);
   LevelState &L = c->L[ln];
   const int np = nprob(c);
   double *e = field_ptr(L, fid_e);
   const double *r = field_ptr(L, fid_r);
   CUDA_CHECK(cudaMemcpyAsync(c->run.p, c->active.p, np * sizeof(int), cudaMemcpyDeviceToDevice,
                              c->stream));
   CUDA_CHECK(cudaMemsetAsync(c->sweeps_call.p, 0, np * sizeof(long long), c->stream));
   const long long *fmap = (c->fused && L.fused_ok && !c->bc_faces) ? L.facemap.p : nullptr;
   // the staged pass computes no residual maxima: fixed sweep counts only
   const bool staged = fmap && c->staged && tol < 0.0 && L.unit_smem[0] > 0;
   // The fill with the coarser level is a full fill.  Pulling fused passes
   // read only its coarse-fine ghosts; staged passes read face ghost cells,
   // which their pushes keep current after this fill.
   if (ln > 0) ghost_fill(c, fid_e, ln, true, 1, c->run.p);
   else if (!fmap || staged) ghost_fill(c, fid_e, ln, false, 1, c->run.p);
   std::vector<int> hrun(np);
   // smoothing to a tolerance on a level without a coarser one and with one
   // patch per problem (the coarsest level): every sweep in one launch
   const bool one_launch = tol >= 0.0 && ln == 0 && fmap && L.one_patch_per_prob;
   if (one_launch) {
      const int pi = prof_begin(c, 0, L.rb_bytes_prob, 2.0 * nsweeps);
      launch_rbgs_solve<double>(c->stream, c->dim, c->spec, L.npatch, L.d_patches.p, e, r,
                                L.d.p, L.c.p, fmap, c->bc, nsweeps, tol, c->run.p,
                                c->sweeps_call.p, L.maxres_red.p, L.maxres_blk.p,
                                L.solve_smem);
      prof_end(c, pi);
   }
   for (int isweep = 0; isweep < (one_launch ? 0 : nsweeps); ++isweep) {
      if (tol >= 0.0 && isweep > 0 && isweep % c->check_interval == 0 && !c->capturing) {
         CUDA_CHECK(cudaMemcpyAsync(hrun.data(), c->run.p, np * sizeof(int),
                                    cudaMemcpyDeviceToHost, c->stream));
         CUDA_CHECK(cudaStreamSynchronize(c->stream));
         bool any = false;
         for (int v : hrun) any = any || v;
         if (!any) break;
      }
      CUDA_CHECK(cudaMemsetAsync(L.maxres_red.p, 0, L.maxres_red.n * sizeof(unsigned long long),
                                 c->stream));
      CUDA_CHECK(cudaMemsetAsync(L.maxres_blk.p, 0, L.maxres_blk.n * sizeof(unsigned long long),
                                 c->stream));
      for (int color = 0; color < 2; ++color) {
         if (!fmap) ghost_fill(c, fid_e, ln, false, 1, c->run.p);
         if (ln > 0)
            launch_cf_flux(c->stream, L.d_cf.p, (int)L.cf.size(), L.d_patches.p, e, L.d.p,
                           c->spec.d_variable, c->spec.d_const, L.tranwt, L.longwt, L.cfflux.p,
                           c->run.p);
         const int pi = prof_begin(c, 0, L.rb_bytes_prob, 1.0);
         if (staged)
            launch_rb_staged<double>(c->stream, c->dim, c->spec, (int)L.units[0].size(),
                                     L.unit_smem[0], c->stage_depth, L.d_units[0].p,
                                     L.d_copies[0].p, L.d_hdrs[0].p, e, r, L.d.p, L.c.p,
                                     L.cfflux.p, color, L.pushmap.p, c->bc, c->kerr.p,
                                     c->wait_test);
         else
            launch_rbgs(c->stream, c->dim, c->spec, (int)L.slot_chunks.size(), L.d_patches.p,
                        L.d_slot_chunks.p, e, r, L.d.p, L.c.p, L.cfflux.p, L.cfmask.p, color,
                        color == 0 ? L.maxres_red.p : L.maxres_blk.p, c->run.p, fmap, c->bc);
         prof_end(c, pi);
      }
      if (!fmap) ghost_fill(c, fid_e, ln, false, 1, c->run.p);
      launch_sweep_check(c->stream, L.maxres_red.p, L.maxres_blk.p, L.last_patch.p, np, tol,
                         c->run.p, c->sweeps_call.p);
   }
   // Fused passes leave the same-level ghosts stale; one fill of every active
   // problem gives the ghost values the per-sweep fills would have left (a
   // fill depends only on the interior, which a stopped problem no longer
   // changes).
   if (fmap && nsweeps > 0) ghost_fill(c, fid_e, ln, false, 1, c->active.p);
   CUDA_CHECK(cudaGetLastError());
}

// CellPoissonFACOps::computeCompositeResidualOnLevel (CellPoissonFACOps.C:1792-1956).
// Mean patch size (cells) from which the automatic setting fuses the
// residual: on levels of 32^3 patches the one-pass kernel measured faster
// than the flux-array pair, on levels of 8^3..16^3 patches slower.
constexpr long long kFusedResidualCells = 8192;

bool fused_residual_on(const fac_ctx *c, int ln)
{
   if (c->fused_residual >= 0) return c->fused_residual != 0;
   const LevelState &L = c->L[ln];
   return L.npatch > 0 && L.n0 >= kFusedResidualCells * (long long)L.npatch;
}

// The staged residual (TMA-staged units, then the fix-up of the special
// cells) runs wherever the staged passes are on and two CTAs of the level's
// largest unit fit an SM's shared memory; with one CTA per SM (FP64 slices
// of 32 x 32 patches) it measured slower than the one-pass kernel.  It
// gives the same bits as the other two forms.
bool staged_residual_on(const fac_ctx *c, int ln, int kind)
{
   const LevelState &L = c->L[ln];
   if (!c->staged || L.runit_smem[kind] <= 0 || L.runits[kind].empty()) return false;
   return 2LL * (kStageBarrierBytes + (long long)c->stage_depth * L.runit_smem[kind]) <=
          kStageSmemMax;
}

void comp_residual(fac_ctx *c, int fid_r, int fid_u, int fid_f, int ln, int error_eq)
{
   OpTimer ot(c, "comp_residual", ln);
   LevelState &L = c->L[ln];
   const int *run = c->active.p;
   ghost_fill(c, fid_u, ln, ln > 0, error_eq, run);
   const double *u = field_ptr(L, fid_u);
   const bool finer = ln < c->nlev - 1;
   const int kind = fid_f == kFieldZero ? kResF64Zero : kResF64;
   const bool staged = staged_residual_on(c, ln, kind);
   const bool fused = !staged && fused_residual_on(c, ln);
   if (!staged && !fused) {
      launch_flux_cells(c->stream, c->dim, c->spec, (int)L.cell_chunks.size(), L.d_patches.p,
                        L.d_cell_chunks.p, u, L.d.p, L.cfmask.p, L.tranwt, L.longwt,
                        L.d_ratio.p, L.flux.p, run);
      if (ln > 0)
         launch_ewing_fix(c->stream, L.d_cf.p, (int)L.cf.size(), L.d_patches.p, u, L.d.p,
                          c->spec.d_variable, c->spec.d_const, L.tranwt, L.longwt, L.flux.p,
                          run);
   }
   if (finer) {
      LevelState &Fl = c->L[ln + 1];
      launch_flux_coarsen(c->stream, L.fcoarsen.d_items.p, L.fcoarsen.d_chunks.p,
                          L.fcoarsen.nchunks(), L.fcoarsen.d_prefix.p, Fl.d_patches.p, L.d_patches.p, Fl.oflux.p,
                          L.flux.p, run);
   }
   if (staged) {
      launch_res_staged<double>(c->stream, c->dim, c->spec, (int)L.runits[kind].size(),
                                L.runit_smem[kind], c->stage_depth, L.d_runits[kind].p,
                                L.d_rcopies[kind].p, L.d_rhdrs[kind].p, u,
                                field_ptr(L, fid_f), L.d.p, L.c.p, field_ptr(L, fid_r),
                                ln > 0 ? L.oflux.p : nullptr, c->kerr.p, c->wait_test);
      launch_residual_cells<double>(c->stream, c->dim, c->spec, (int)L.rfix.size(), L.d_rfix.p,
                                    L.d_patches.p, u, L.d.p, L.cfmask.p, L.tranwt, L.longwt,
                                    L.d_ratio.p, finer ? L.fcmask.p : nullptr, L.flux.p,
                                    field_ptr(L, fid_f), L.c.p, field_ptr(L, fid_r),
                                    ln > 0 ? L.oflux.p : nullptr, run);
   } else if (fused) {
      launch_residual_fused(c->stream, c->dim, c->spec, (int)L.cell_chunks.size(),
                            L.d_patches.p, L.d_cell_chunks.p, u, L.d.p, L.cfmask.p, L.tranwt,
                            L.longwt, L.d_ratio.p, finer ? L.fcmask.p : nullptr, L.flux.p,
                            field_ptr(L, fid_f), L.c.p, field_ptr(L, fid_r),
                            ln > 0 ? L.oflux.p : nullptr, run);
   } else {
      launch_residual(c->stream, c->dim, c->spec, (int)L.cell_chunks.size(), L.d_patches.p,
                      L.d_cell_chunks.p, u, field_ptr(L, fid_f), L.flux.p, L.c.p,
                      field_ptr(L, fid_r), ln > 0 ? L.oflux.p : nullptr, run);
   }
   CUDA_CHECK(cudaGetLastError());
}

void restrict_op(fac_ctx *c, int fid_src, int fid_dst, int dest_ln)
{
   OpTimer ot(c, "restrict", dest_ln);
   LevelState &C = c->L[dest_ln];
   LevelState &Fl = c->L[dest_ln + 1];
   const int sg = field_ghost(fid_src), dg = field_ghost(fid_dst);
   ItemList<RestrictItem> &it = dg ? C.restrict_g1 : C.restrict_g0;
   launch_restrict(c->stream, c->dim, it.d_items.p, it.d_chunks.p, it.nchunks(), it.d_prefix.p,
                   Fl.d_patches.p, C.d_patches.p, field_ptr(Fl, fid_src), sg,
                   field_ptr(C, fid_dst), dg, c->active.p);
   CUDA_CHECK(cudaGetLastError());
}

void restrict_solution(fac_ctx *c, int fid, int dest_ln)
{
   OpTimer ot(c, "restrict_solution", dest_ln);
   restrict_op(c, fid, fid, dest_ln);
   ghost_fill(c, fid, dest_ln, dest_ln > 0, 0, c->active.p);
}

// CellPoissonFACOps::prolongErrorAndCorrect (CellPoissonFACOps.C:1254-1304).
void prolong_correct(fac_ctx *c, int fid_src, int fid_dst, int dest_ln)
{
   OpTimer ot(c, "prolong", dest_ln);
   LevelState &Fl = c->L[dest_ln];
   LevelState &C = c->L[dest_ln - 1];
   if (field_ghost(fid_src) != 1 || field_ghost(fid_dst) != 1)
      throw FacError(FAC_ERR_ARG, "prolongation needs ghosted cell fields");
   const FillGather &G = Fl.gather_tmp;
   if (G.ok)
      launch_fill_gather<double>(c->stream, (long long)G.to.size(), G.d_to.p, G.d_from.p,
                                 G.d_prob.p, G.bc.d_items.p, G.bc.d_chunks.p, G.bc.nchunks(),
                                 G.bc.d_prefix.p, Fl.tmp.p, nullptr, field_ptr(C, fid_src), 1,
                                 c->bc, c->active.p);
   else
      launch_fill<double>(c->stream, Fl.tmp_fill.d_items.p, Fl.tmp_fill.d_chunks.p,
                          Fl.tmp_fill.nchunks(), Fl.tmp_fill.d_prefix.p, Fl.tmp.p, nullptr,
                          field_ptr(C, fid_src), 1, c->bc, c->active.p);
   if (Fl.prolong_r2)
      launch_prolong_add_r2<double>(c->stream, c->dim, Fl.prolong2.d_items.p,
                                    Fl.prolong2.d_chunks.p, Fl.prolong2.nchunks(),
                                    Fl.prolong2.d_prefix.p, Fl.d_patches.p, Fl.tmp.p,
                                    Fl.dxc_prob.p, field_ptr(Fl, fid_dst), c->active.p);
   else
      launch_prolong_add(c->stream, c->dim, Fl.prolong.d_items.p, Fl.prolong.d_chunks.p,
                         Fl.prolong.nchunks(), Fl.prolong.d_prefix.p, Fl.d_patches.p, Fl.tmp.p,
                         Fl.dxc_prob.p, Fl.ratio, field_ptr(Fl, fid_dst), c->active.p);
   CUDA_CHECK(cudaGetLastError());
}

void rms_norm_launch(fac_ctx *c, int fid)
{
   const int np = nprob(c);
   CUDA_CHECK(cudaMemsetAsync(c->norm_acc.p, 0, np * sizeof(double2), c->stream));
   const int g = field_ghost(fid);
   for (int ln = 0; ln < c->nlev; ++ln) {
      LevelState &L = c->L[ln];
      launch_norm(c->stream, c->dim, (int)L.cell_chunks.size(), L.d_patches.p, L.d_cell_chunks.p,
                  field_ptr(L, fid), g, L.w.p, L.norm_partial.p, L.d_prob_cell_chunk_begin.p, np,
                  c->norm_acc.p);
   }
}

void rms_norm_read(fac_ctx *c, std::vector<double> &out)
{
   const int np = nprob(c);
   std::vector<double2> acc(np);
   CUDA_CHECK(cudaMemcpyAsync(acc.data(), c->norm_acc.p, np * sizeof(double2),
                              cudaMemcpyDeviceToHost, c->stream));
   int kerr = 0;
   CUDA_CHECK(cudaMemcpyAsync(&kerr, c->kerr.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
   CUDA_CHECK(cudaStreamSynchronize(c->stream));
   if (kerr)
      throw FacError(FAC_ERR_CUDA, "a bounded wait of a staged colour pass ran out (device error "
                                   "flag; fac_clear_device_error resets it)");
   out.resize(np);
   for (int p = 0; p < np; ++p) {
      const double num = std::sqrt(acc[p].x);
      out[p] = acc[p].y > 0.0 ? num / std::sqrt(acc[p].y) : 0.0;
   }
}

void rms_norm(fac_ctx *c, int fid, std::vector<double> &out)
{
   OpTimer ot(c, "rms_norm", 0);
   rms_norm_launch(c, fid);
   rms_norm_read(c, out);
}

void solve_coarsest(fac_ctx *c)
{
   OpTimer ot(c, "solve_coarsest", 0);
   smooth(c, FAC_E, FAC_R, 0, c->coarse_max_it, c->coarse_tol);
   // accumulate the per-call sweep counts on the device
   launch_accumulate(c->stream, c->sweeps_call.p, c->sweeps_coarse.p, nprob(c));
   ghost_fill(c, FAC_E, 0, false, 1, c->active.p);
}

// FACPreconditioner::facCycle_Recursive (FACPreconditioner.C:462-518).
void fac_cycle_recursive(fac_ctx *c, int ln)
{
   if (ln == 0) {
      solve_coarsest(c);
   } else {
      if (c->pre_sweeps > 0) {
         smooth(c, FAC_E, FAC_R, ln, c->pre_sweeps, -1.0);
         comp_residual(c, FAC_TR, FAC_E, FAC_R, ln, 1);
         restrict_op(c, FAC_TR, FAC_R, ln - 1);
      } else {
         // Without pre-smoothing the error is still zero on this level and
         // on the coarser ones (zeroed before the cycle, visited later), so
         // the composite residual f - A 0 is f itself, bit for bit (every
         // flux is D (0 - 0) = +0, and the finer level's saved fluxes, which
         // nothing in this cycle reads, would be +0 too): f is restricted as
         // it is.
         restrict_op(c, FAC_R, FAC_R, ln - 1);
      }
      fac_cycle_recursive(c, ln - 1);
      prolong_correct(c, FAC_E, FAC_E, ln);
      smooth(c, FAC_E, FAC_R, ln, c->post_sweeps, -1.0);
   }
}

// FACPreconditioner::computeFullCompositeResidual (FACPreconditioner.C:775-814).
void full_composite_residual_launch(fac_ctx *c)
{
   const int lmax = c->nlev - 1;
   comp_residual(c, FAC_R, FAC_U, FAC_F, lmax, 0);
   for (int ln = lmax - 1; ln >= 0; --ln) {
      restrict_solution(c, FAC_U, ln);
      comp_residual(c, FAC_R, FAC_U, FAC_F, ln, 0);
      restrict_op(c, FAC_R, FAC_R, ln);
   }
   rms_norm_launch(c, FAC_R);
}

void full_composite_residual(fac_ctx *c, std::vector<double> &norms)
{
   full_composite_residual_launch(c);
   rms_norm_read(c, norms);
}

void zero_field(fac_ctx *c, int fid)
{
   OpTimer ot(c, "zero_field", fid);
   for (int ln = 0; ln < c->nlev; ++ln) {
      LevelState &L = c->L[ln];
      const size_t n = field_ghost(fid) ? L.u.n : L.f.n;
      CUDA_CHECK(cudaMemsetAsync(field_ptr(L, fid), 0, n * sizeof(double), c->stream));
   }
}

// CellPoissonFACSolver::solveSystem with the solver's own boundary object
// (CellPoissonFACSolver.C:327-349): the physical-boundary ghost values of u
// are cached before the solve and put back after it.  With a caller's
// coefficient object the reference does neither.
void dirichlet(fac_ctx *c, bool restore)
{
   if (c->bc_object) return;
   for (int ln = 0; ln < c->nlev; ++ln) {
      LevelState &L = c->L[ln];
      const long long n = (long long)L.dir_idx.size();
      if (restore) launch_scatter(c->stream, L.d_dir_idx.p, n, L.dir_cache.p, L.u.p);
      else launch_gather(c->stream, L.d_dir_idx.p, n, L.u.p, L.dir_cache.p);
   }
}

// ---------------------------------------------------------------------------
// mixed precision cycle: FP32 smoothing, prolongation and error storage;
// FP64 composite residual (fluxes, Ewing fix, flux sums), residual
// restriction and coarsest-level solve.  The outer FACPreconditioner loop
// (u, f, full composite residual, norms) stays FP64, so each cycle is a
// defect correction that recovers FP64 accuracy.
// ---------------------------------------------------------------------------

void ghost_fill32(fac_ctx *c, int ln, bool with_coarse, int homogeneous, const int *mask)
{
   LevelState &L = c->L[ln];
   const float *coarse = ln > 0 ? c->L[ln - 1].e32.p : nullptr;
   ItemList<FillItem> &it = (with_coarse && ln > 0) ? L.fill_wc : L.fill_nc;
   FillGather &G = (with_coarse && ln > 0) ? L.gather_wc : L.gather_nc;
   const int pi = prof_begin(c, 3, L.fill_bytes_prob, 0.5);
   if (G.ok)
      launch_fill_gather<float>(c->stream, (long long)G.to.size(), G.d_to.p, G.d_from.p,
                                G.d_prob.p, G.bc.d_items.p, G.bc.d_chunks.p, G.bc.nchunks(),
                                G.bc.d_prefix.p, L.e32.p, L.e32.p, coarse, homogeneous, c->bc,
                                mask);
   else
      launch_fill<float>(c->stream, it.d_items.p, it.d_chunks.p, it.nchunks(), it.d_prefix.p,
                         L.e32.p, L.e32.p, coarse, homogeneous, c->bc, mask);
   prof_end(c, pi);
}

// zero_start: e32 of this level and of the coarser level are zero (interior
// and ghosts), so the entry fill, which would write the zeros the ghost
// cells already hold, is skipped.
void smooth32(fac_ctx *c, int ln, int nsweeps, bool zero_start = false)
{
   OpTimer ot(c, "smooth32", ln);
   LevelState &L = c->L[ln];
   const int np = nprob(c);
   const int *run = c->active.p;
   const long long *fmap = (c->fused && L.fused_ok && !c->bc_faces) ? L.facemap.p : nullptr;
   const bool staged = fmap && c->staged && L.unit_smem[1] > 0;
   if (zero_start && fmap) {
      // entry fill skipped (see above); passes that fill around themselves
      // (!fmap) fill as usual
   } else if (ln > 0) {
      ghost_fill32(c, ln, true, 1, run);
   } else if (!fmap || staged) {
      ghost_fill32(c, ln, false, 1, run);
   }
   for (int isweep = 0; isweep < nsweeps; ++isweep) {
      for (int color = 0; color < 2; ++color) {
         if (!fmap) ghost_fill32(c, ln, false, 1, run);
         if (ln > 0)
            launch_cf_flux<float>(c->stream, L.d_cf.p, (int)L.cf.size(), L.d_patches.p, L.e32.p,
                                  L.d32.p, c->spec.d_variable, c->spec.d_const, L.tranwt,
                                  L.longwt, L.cfflux32.p, run);
         const int pi =
            prof_begin(c, 2, L.rb_bytes_prob, 0.5);
         if (staged)
            launch_rb_staged<float>(c->stream, c->dim, c->spec, (int)L.units[1].size(),
                                    L.unit_smem[1], c->stage_depth, L.d_units[1].p,
                                    L.d_copies[1].p, L.d_hdrs[1].p, L.e32.p, L.r32.p,
                                    L.d32.p, L.c32.p, L.cfflux32.p, color, L.pushmap.p,
                                    c->bc, c->kerr.p, c->wait_test);
         else
            launch_rbgs<float>(c->stream, c->dim, c->spec, (int)L.slot_chunks.size(),
                               L.d_patches.p, L.d_slot_chunks.p, L.e32.p, L.r32.p, L.d32.p,
                               L.c32.p, L.cfflux32.p, L.cfmask.p, color, nullptr, run, fmap,
                               c->bc);
         prof_end(c, pi);
      }
      if (!fmap) ghost_fill32(c, ln, false, 1, run);
   }
   // after fused passes the same-level ghosts of e32 are left stale: every
   // reader in the mixed cycle fills them first (comp_residual_mixed) or
   // reads interiors only (prolongation sources, u += e)
   (void)np;
   CUDA_CHECK(cudaGetLastError());
}

void comp_residual_mixed(fac_ctx *c, int ln)
{
   OpTimer ot(c, "comp_residual_mixed", ln);
   LevelState &L = c->L[ln];
   const int *run = c->active.p;
   ghost_fill32(c, ln, ln > 0, 1, run);
   const bool finer = ln < c->nlev - 1;
   const bool staged = staged_residual_on(c, ln, kResF32);
   const bool fused = !staged && fused_residual_on(c, ln);
   if (!staged && !fused) {
      launch_flux_cells<float>(c->stream, c->dim, c->spec, (int)L.cell_chunks.size(),
                               L.d_patches.p, L.d_cell_chunks.p, L.e32.p, L.d.p, L.cfmask.p,
                               L.tranwt, L.longwt, L.d_ratio.p, L.flux.p, run);
      if (ln > 0)
         launch_ewing_fix<float>(c->stream, L.d_cf.p, (int)L.cf.size(), L.d_patches.p, L.e32.p,
                                 L.d.p, c->spec.d_variable, c->spec.d_const, L.tranwt,
                                 L.longwt, L.flux.p, run);
   }
   if (finer) {
      LevelState &Fl = c->L[ln + 1];
      launch_flux_coarsen(c->stream, L.fcoarsen.d_items.p, L.fcoarsen.d_chunks.p,
                          L.fcoarsen.nchunks(), L.fcoarsen.d_prefix.p, Fl.d_patches.p, L.d_patches.p, Fl.oflux.p,
                          L.flux.p, run);
   }
   if (staged) {
      launch_res_staged<float>(c->stream, c->dim, c->spec, (int)L.runits[kResF32].size(),
                               L.runit_smem[kResF32], c->stage_depth, L.d_runits[kResF32].p,
                               L.d_rcopies[kResF32].p, L.d_rhdrs[kResF32].p, L.e32.p, L.r.p,
                               L.d.p, L.c.p, L.tr.p, ln > 0 ? L.oflux.p : nullptr, c->kerr.p,
                               c->wait_test);
      launch_residual_cells<float>(c->stream, c->dim, c->spec, (int)L.rfix.size(), L.d_rfix.p,
                                   L.d_patches.p, L.e32.p, L.d.p, L.cfmask.p, L.tranwt,
                                   L.longwt, L.d_ratio.p, finer ? L.fcmask.p : nullptr,
                                   L.flux.p, L.r.p, L.c.p, L.tr.p,
                                   ln > 0 ? L.oflux.p : nullptr, run);
   } else if (fused) {
      launch_residual_fused<float>(c->stream, c->dim, c->spec, (int)L.cell_chunks.size(),
                                   L.d_patches.p, L.d_cell_chunks.p, L.e32.p, L.d.p, L.cfmask.p,
                                   L.tranwt, L.longwt, L.d_ratio.p,
                                   finer ? L.fcmask.p : nullptr, L.flux.p, L.r.p, L.c.p, L.tr.p,
                                   ln > 0 ? L.oflux.p : nullptr, run);
   } else {
      launch_residual<float>(c->stream, c->dim, c->spec, (int)L.cell_chunks.size(),
                             L.d_patches.p, L.d_cell_chunks.p, L.e32.p, L.r.p, L.flux.p, L.c.p,
                             L.tr.p, ln > 0 ? L.oflux.p : nullptr, run);
   }
   CUDA_CHECK(cudaGetLastError());
}

void prolong32(fac_ctx *c, int dest_ln)
{
   OpTimer ot(c, "prolong32", dest_ln);
   LevelState &Fl = c->L[dest_ln];
   LevelState &C = c->L[dest_ln - 1];
   const FillGather &G = Fl.gather_tmp;
   if (G.ok)
      launch_fill_gather<float>(c->stream, (long long)G.to.size(), G.d_to.p, G.d_from.p,
                                G.d_prob.p, G.bc.d_items.p, G.bc.d_chunks.p, G.bc.nchunks(),
                                G.bc.d_prefix.p, Fl.tmp32.p, nullptr, C.e32.p, 1, c->bc,
                                c->active.p);
   else
      launch_fill<float>(c->stream, Fl.tmp_fill.d_items.p, Fl.tmp_fill.d_chunks.p,
                         Fl.tmp_fill.nchunks(), Fl.tmp_fill.d_prefix.p, Fl.tmp32.p, nullptr,
                         C.e32.p, 1, c->bc, c->active.p);
   if (Fl.prolong_r2)
      launch_prolong_add_r2<float>(c->stream, c->dim, Fl.prolong2.d_items.p,
                                   Fl.prolong2.d_chunks.p, Fl.prolong2.nchunks(),
                                   Fl.prolong2.d_prefix.p, Fl.d_patches.p, Fl.tmp32.p,
                                   Fl.dxc_prob.p, Fl.e32.p, c->active.p);
   else
      launch_prolong_add<float>(c->stream, c->dim, Fl.prolong.d_items.p, Fl.prolong.d_chunks.p,
                                Fl.prolong.nchunks(), Fl.prolong.d_prefix.p, Fl.d_patches.p,
                                Fl.tmp32.p, Fl.dxc_prob.p, Fl.ratio, Fl.e32.p, c->active.p);
   CUDA_CHECK(cudaGetLastError());
}

void fac_cycle_mixed(fac_ctx *c, int ln)
{
   LevelState &L = c->L[ln];
   if (ln == 0) {
      solve_coarsest(c);
      launch_convert<double, float>(c->stream, L.e.p, L.e32.p, (long long)L.e.n);
      return;
   }
   launch_convert<double, float>(c->stream, L.r.p, L.r32.p, (long long)L.r.n);
   if (c->pre_sweeps > 0) {
      // every e32 is zeroed before the cycle, and coarser levels are reached
      // only after this pre-smoothing
      smooth32(c, ln, c->pre_sweeps, true);
      comp_residual_mixed(c, ln);
      restrict_op(c, FAC_TR, FAC_R, ln - 1);
   } else {
      // no pre-smoothing: the residual of the still zero error is f, bit
      // for bit (fac_cycle_recursive)
      restrict_op(c, FAC_R, FAC_R, ln - 1);
   }
   fac_cycle_mixed(c, ln - 1);
   prolong32(c, ln);
   smooth32(c, ln, c->post_sweeps);
}

void mixed_prepare(fac_ctx *c)
{
   for (int ln = 0; ln < c->nlev; ++ln) {
      LevelState &L = c->L[ln];
      if (c->spec.d_variable)
         launch_convert<double, float>(c->stream, L.d.p, L.d32.p, (long long)L.d.n);
      if (c->spec.c_kind == 2)
         launch_convert<double, float>(c->stream, L.c.p, L.c32.p, (long long)L.c.n);
   }
}

// ---------------------------------------------------------------------------
// learned correction (no reference counterpart).  After a cycle's composite
// residual r: the network predicts the error on every patch of one level
// from r on the patch and a one-cell halo; the prediction e is carried to
// the coarser levels by restriction, d = A e is formed as r minus the
// composite residual of the error equation, and u += alpha e, r -= alpha d
// with alpha = <r,d>/<d,d> per problem (weighted inner products; alpha = 0
// when it would not lower the residual).  The FAC residual therefore never
// grows: plain FAC is the fallback and the judge.
// ---------------------------------------------------------------------------

void learned_gather(fac_ctx *c, int ln)
{
   LevelState &L = c->L[ln];
   const int S = FAC_CNN_BOX;
   CUDA_CHECK(cudaMemsetAsync(L.e.p, 0, L.e.n * sizeof(double), c->stream));
   launch_g0_to_g1(c->stream, c->dim, (int)L.cell_chunks.size(), L.d_patches.p,
                   L.d_cell_chunks.p, L.r.p, L.e.p);
   ghost_fill(c, FAC_E, ln, false, 1, nullptr);
   launch_patch_rms(c->stream, c->dim, L.npatch, L.d_patches.p, L.r.p, c->cnn_scale.p);
   launch_gather_samples(c->stream, c->dim, L.npatch, L.d_patches.p, L.e.p, c->cnn_scale.p,
                         c->cnn_in.p, S);
}

void learned_step(fac_ctx *c)
{
   const int ln = c->learned_level;
   LevelState &L = c->L[ln];
   const int np = nprob(c);
   learned_gather(c, ln);
   const float *y = nullptr;
   if (cnn_forward_on_stream(c->cnn, c->cnn_in.p, L.npatch, c->stream, &y) != FAC_OK)
      throw FacError(FAC_ERR_CUDA, "learned correction: network forward failed");
   zero_field(c, FAC_E);
   launch_scatter_samples(c->stream, c->dim, (int)L.cell_chunks.size(), L.d_patches.p,
                          L.d_cell_chunks.p, y, c->cnn_scale.p, FAC_CNN_BOX, L.e.p);
   // composite residual of the error equation with rhs r: TR = r - A e
   const int lmax = c->nlev - 1;
   for (int l = ln - 1; l >= 0; --l) {
      restrict_op(c, FAC_E, FAC_E, l);
   }
   comp_residual(c, FAC_TR, FAC_E, FAC_R, lmax, 1);
   for (int l = lmax - 1; l >= 0; --l) {
      comp_residual(c, FAC_TR, FAC_E, FAC_R, l, 1);
      restrict_op(c, FAC_TR, FAC_TR, l);
   }
   CUDA_CHECK(cudaMemsetAsync(c->dot_acc.p, 0, np * sizeof(double2), c->stream));
   for (int l = 0; l < c->nlev; ++l) {
      LevelState &Ll = c->L[l];
      launch_dot_pair(c->stream, c->dim, (int)Ll.cell_chunks.size(), Ll.d_patches.p,
                      Ll.d_cell_chunks.p, Ll.r.p, Ll.tr.p, Ll.w.p, Ll.norm_partial.p,
                      Ll.d_prob_cell_chunk_begin.p, np, c->dot_acc.p);
   }
   launch_alpha(c->stream, c->dot_acc.p, c->active.p, np, c->alpha.p);
   for (int l = 0; l < c->nlev; ++l) {
      LevelState &Ll = c->L[l];
      launch_apply_alpha(c->stream, c->dim, (int)Ll.cell_chunks.size(), Ll.d_patches.p,
                         Ll.d_cell_chunks.p, c->alpha.p, Ll.u.p, Ll.e.p, Ll.r.p, Ll.tr.p);
   }
   CUDA_CHECK(cudaGetLastError());
}

// FACPreconditioner::solveSystem (FACPreconditioner.C:277-452) inside
// CellPoissonFACSolver::solveSystem (CellPoissonFACSolver.C:310-352).
void fgmres_solve(fac_ctx *c, int m, int *converged, int *iterations, double *residual);

void solve(fac_ctx *c, int *converged, int *iterations, double *residual)
{
   if (c->krylov > 0) {
      fgmres_solve(c, c->krylov, converged, iterations, residual);
      return;
   }
   const int np = nprob(c);
   std::vector<int> act(np, 1);
   c->host_active = act;
   set_active(c, act);
   dirichlet(c, false);
   zero_field(c, FAC_E);
   zero_field(c, FAC_R);
   std::vector<double> res, fnorm;
   full_composite_residual(c, res);
   rms_norm(c, FAC_F, fnorm);
   std::vector<double> eff(np);
   for (int p = 0; p < np; ++p) {
      eff[p] = c->residual_tol;
      if (c->rel_residual_tol >= 0) {
         const double t = fnorm[p] * c->rel_residual_tol;
         if (eff[p] < t) eff[p] = t;
      }
      c->hist[p].assign(1, res[p]);
   }
   std::vector<int> its(np, 0);
   int it = 0;
   bool any = true;
   if (c->mixed) mixed_prepare(c);
   // one FACPreconditioner cycle up to the norm kernels (no host sync)
   auto cycle_body = [&]() {
      if (c->mixed) {
         // the error lives in e32; E is the FP64 coarsest-level solve's
         CUDA_CHECK(cudaMemsetAsync(c->L[0].e.p, 0, c->L[0].e.n * sizeof(double), c->stream));
         for (int ln = 0; ln < c->nlev; ++ln)
            CUDA_CHECK(cudaMemsetAsync(c->L[ln].e32.p, 0, c->L[ln].e32.n * sizeof(float),
                                       c->stream));
         fac_cycle_mixed(c, c->nlev - 1);
      } else {
         zero_field(c, FAC_E);
         fac_cycle_recursive(c, c->nlev - 1);
      }
      for (int ln = 0; ln < c->nlev; ++ln) {
         LevelState &L = c->L[ln];
         if (c->mixed)
            launch_add_interior<float>(c->stream, c->dim, (int)L.cell_chunks.size(),
                                       L.d_patches.p, L.d_cell_chunks.p, L.u.p, L.e32.p,
                                       c->active.p);
         else
            launch_add_interior<double>(c->stream, c->dim, (int)L.cell_chunks.size(),
                                        L.d_patches.p, L.d_cell_chunks.p, L.u.p, L.e.p,
                                        c->active.p);
      }
      for (int ln = c->nlev - 2; ln >= 0; --ln) restrict_solution(c, FAC_U, ln);
      full_composite_residual_launch(c);
      if (c->cnn) {
         learned_step(c);
         rms_norm_launch(c, FAC_R);
      }
   };
   // The whole cycle is one CUDA graph, captured on first use and replayed:
   // the launch sequence is fixed (converged problems are skipped on the
   // device through the active flags), so only the norms come back per cycle.
   // With profiling on, the cycle is captured with event-record nodes around
   // the profiled launches, so their times carry no host launch gaps.
   const bool graph = c->use_graph && !c->tracing;
   if (graph && c->cycle_exec && c->graph_profiled != c->profiling) c->drop_graph();
   if (graph && !c->cycle_exec) {
      cudaGraph_t g = nullptr;
      const long long n0 = kernel_launch_count();
      CUDA_CHECK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
      c->capturing = true;
      try {
         cycle_body();
      } catch (...) {
         c->capturing = false;
         cudaStreamEndCapture(c->stream, &g);
         if (g) cudaGraphDestroy(g);
         c->drop_graph();
         throw;
      }
      c->capturing = false;
      CUDA_CHECK(cudaStreamEndCapture(c->stream, &g));
      c->graph_launches = kernel_launch_count() - n0;
      add_kernel_launches(-c->graph_launches);  // captured, not launched
      c->graph_profiled = c->profiling;
      cudaError_t e = cudaGraphInstantiate(&c->cycle_exec, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) {
         c->cycle_exec = nullptr;
         c->drop_graph();
         throw FacError(FAC_ERR_CUDA, std::string("cudaGraphInstantiate: ") +
                                          cudaGetErrorString(e));
      }
   }
   while (any) {
      if (graph) {
         CUDA_CHECK(cudaGraphLaunch(c->cycle_exec, c->stream));
         add_kernel_launches(c->graph_launches);
      } else {
         cycle_body();
      }
      std::vector<double> nr;
      rms_norm_read(c, nr);
      if (graph && c->profiling) harvest_graph_profile(c);
      ++it;
      any = false;
      for (int p = 0; p < np; ++p) {
         if (!act[p]) continue;
         res[p] = nr[p];
         its[p] = it;
         c->hist[p].push_back(nr[p]);
         if (!(nr[p] > eff[p] && it < c->max_cycles)) act[p] = 0;
         any = any || act[p];
      }
      if (act != c->host_active) set_active(c, act);
      c->host_active = act;
   }
   c->host_active.assign(np, 1);
   set_active(c, c->host_active);
   dirichlet(c, true);
   CUDA_CHECK(cudaStreamSynchronize(c->stream));
   for (int p = 0; p < np; ++p) {
      if (converged) converged[p] = res[p] < eff[p];
      if (iterations) iterations[p] = its[p];
      if (residual) residual[p] = res[p];
   }
}

// ---------------------------------------------------------------------------
// FGMRES(m) with one FAC cycle as the (flexible) right preconditioner, for
// every problem of the context at once: each problem has its own Krylov
// basis, Hessenberg matrix and Givens rotations; the level operations run
// on all problems that are still iterating.  Inner products are the
// control-volume-weighted sums of the RMS norm (weights 0 under finer
// levels), so the stopping test is FACPreconditioner's: weighted RMS
// residual <= max(residual_tol, relative_residual_tol * ||f||).  The
// preconditioner (a FAC cycle, FP32 in the mixed precision) changes from
// one application to the next only through its arithmetic, which the
// flexible variant allows for.  The composite operator is the residual of
// the error equation with a zero right-hand side (fills with the coarser
// level, Ewing fluxes, flux coarsening, restriction of finer values).
// ---------------------------------------------------------------------------

namespace {

double *kry_vec(fac_ctx *c, int ln, int slot)
{
   return c->L[ln].kry.p + (size_t)slot * (size_t)std::max<long long>(1, c->L[ln].n0);
}

void kry_alloc(fac_ctx *c, int m)
{
   if (c->kry_m == m) return;
   const int np = nprob(c);
   for (int ln = 0; ln < c->nlev; ++ln) {
      LevelState &L = c->L[ln];
      L.kry.alloc((size_t)(2 * m + 1) * (size_t)std::max<long long>(1, L.n0));
      L.kry_partial.alloc((size_t)std::max<size_t>(1, L.span_chunks.size()) * (m + 1));
      // finite contents: slots a problem did not reach enter x += Z y with y = 0
      CUDA_CHECK(cudaMemsetAsync(L.kry.p, 0, L.kry.n * sizeof(double), c->stream));
   }
   c->kry_dots.alloc((size_t)np * (m + 1));
   c->kry_coef.alloc((size_t)np * (m + 1));
   c->kry_a.alloc(np);
   c->kry_m = m;
}

// Krylov operands that are not slots: the residual field TR (the operator's
// output) and R (the preconditioner's input), ghost-0 level arrays of the
// same layout as the slots
constexpr int kNoField = -1;

double *kry_field(fac_ctx *c, int ln, int field)
{
   if (field == FAC_TR) return c->L[ln].tr.p;
   if (field == FAC_R) return c->L[ln].r.p;
   return nullptr;
}

// out[p*KT + i] = <x, V_i> (weighted) over all levels, for i < K, x slot
// xslot or the field xfield; with self_dot KT = K + 1 and entry K is <x, x>
void kry_dots(fac_ctx *c, int xslot, int vslot, int K, std::vector<double> &out,
              int xfield = kNoField, bool self_dot = false)
{
   OpTimer ot(c, "kry_dots", -1);
   const int np = nprob(c);
   const int KT = K + (self_dot ? 1 : 0);
   CUDA_CHECK(cudaMemsetAsync(c->kry_dots.p, 0, (size_t)np * KT * sizeof(double), c->stream));
   for (int ln = 0; ln < c->nlev; ++ln) {
      LevelState &L = c->L[ln];
      const int pi = prof_begin(c, 4, L.cells_prob, 8.0 * (K + 2));
      const double *x = xfield != kNoField ? kry_field(c, ln, xfield) : kry_vec(c, ln, xslot);
      launch_multidot(c->stream, (int)L.span_chunks.size(), L.d_span_chunks.p, L.w.p, x,
                      kry_vec(c, ln, vslot), std::max<long long>(1, L.n0), K, L.kry_partial.p,
                      L.d_prob_span_begin.p, np, c->active.p, c->kry_dots.p, self_dot);
      prof_end(c, pi);
   }
   out.resize((size_t)np * KT);
   CUDA_CHECK(cudaMemcpyAsync(out.data(), c->kry_dots.p, (size_t)np * KT * sizeof(double),
                              cudaMemcpyDeviceToHost, c->stream));
   CUDA_CHECK(cudaStreamSynchronize(c->stream));
}

// V_x = a[p] X + sum_i coef[p*K+i] V_{vslot+i}, X = V_x or the field
// xin_field; the result also goes to the field x2_field when one is given
// (not with norm).  With norm: also norm[p] = <V_x, V_x> (weighted) of the
// result, the same numbers as kry_dots(c, xslot, xslot, 1, norm) without
// rereading V_x.
void kry_combine(fac_ctx *c, int xslot, const std::vector<double> &a, int vslot, int K,
                 const std::vector<double> &coef, std::vector<double> *norm = nullptr,
                 int xin_field = kNoField, int x2_field = kNoField)
{
   OpTimer ot(c, "kry_combine", -1);
   const int np = nprob(c);
   CUDA_CHECK(cudaMemcpyAsync(c->kry_a.p, a.data(), np * sizeof(double), cudaMemcpyHostToDevice,
                              c->stream));
   if (K > 0)
      CUDA_CHECK(cudaMemcpyAsync(c->kry_coef.p, coef.data(), (size_t)np * K * sizeof(double),
                                 cudaMemcpyHostToDevice, c->stream));
   if (norm) CUDA_CHECK(cudaMemsetAsync(c->kry_dots.p, 0, (size_t)np * sizeof(double), c->stream));
   for (int ln = 0; ln < c->nlev; ++ln) {
      LevelState &L = c->L[ln];
      const int pi = prof_begin(c, 5, L.cells_prob, 8.0 * (K + (norm ? 3 : 2)));
      const double *xin = xin_field != kNoField ? kry_field(c, ln, xin_field) : nullptr;
      if (norm)
         launch_combine_norm(c->stream, (int)L.span_chunks.size(), L.d_span_chunks.p,
                             kry_vec(c, ln, xslot), c->kry_a.p,
                             K > 0 ? kry_vec(c, ln, vslot) : nullptr,
                             std::max<long long>(1, L.n0), K, c->kry_coef.p, L.w.p,
                             L.kry_partial.p, L.d_prob_span_begin.p, np, c->active.p,
                             c->kry_dots.p, xin);
      else
         launch_combine(c->stream, (int)L.span_chunks.size(), L.d_span_chunks.p,
                        kry_vec(c, ln, xslot), c->kry_a.p,
                        K > 0 ? kry_vec(c, ln, vslot) : nullptr, std::max<long long>(1, L.n0),
                        K, c->kry_coef.p, xin,
                        x2_field != kNoField ? kry_field(c, ln, x2_field) : nullptr);
      prof_end(c, pi);
   }
   if (norm) {
      norm->resize(np);
      CUDA_CHECK(cudaMemcpyAsync(norm->data(), c->kry_dots.p, (size_t)np * sizeof(double),
                                 cudaMemcpyDeviceToHost, c->stream));
      CUDA_CHECK(cudaStreamSynchronize(c->stream));
   }
}

// V_x = a[p] X + sum_i coef[p*K+i] V_{vslot+i} as kry_combine, and
// dots[p*(K+1)+i] = <V_x, V_{vslot+i}>, dots[p*(K+1)+K] = <V_x, V_x> of the
// result: the numbers kry_dots(c, xslot, vslot, K, dots, kNoField, true)
// would give, from the combination's own pass.  False (nothing done) when K
// is outside the fused kernel's range.
bool kry_combine_dots(fac_ctx *c, int xslot, const std::vector<double> &a, int vslot, int K,
                      const std::vector<double> &coef, std::vector<double> &dots,
                      int xin_field = kNoField)
{
   if (K < 1 || K > kCombineDotsMax) return false;
   OpTimer ot(c, "kry_combine_dots", -1);
   const int np = nprob(c);
   const int KT = K + 1;
   CUDA_CHECK(cudaMemcpyAsync(c->kry_a.p, a.data(), np * sizeof(double), cudaMemcpyHostToDevice,
                              c->stream));
   CUDA_CHECK(cudaMemcpyAsync(c->kry_coef.p, coef.data(), (size_t)np * K * sizeof(double),
                              cudaMemcpyHostToDevice, c->stream));
   CUDA_CHECK(cudaMemsetAsync(c->kry_dots.p, 0, (size_t)np * KT * sizeof(double), c->stream));
   for (int ln = 0; ln < c->nlev; ++ln) {
      LevelState &L = c->L[ln];
      const int pi = prof_begin(c, 5, L.cells_prob, 8.0 * (K + 3));
      const double *xin = xin_field != kNoField ? kry_field(c, ln, xin_field) : nullptr;
      launch_combine_dots(c->stream, (int)L.span_chunks.size(), L.d_span_chunks.p,
                          kry_vec(c, ln, xslot), c->kry_a.p, kry_vec(c, ln, vslot),
                          std::max<long long>(1, L.n0), K, c->kry_coef.p, L.w.p,
                          L.kry_partial.p, L.d_prob_span_begin.p, np, c->active.p,
                          c->kry_dots.p, xin);
      prof_end(c, pi);
   }
   dots.resize((size_t)np * KT);
   CUDA_CHECK(cudaMemcpyAsync(dots.data(), c->kry_dots.p, (size_t)np * KT * sizeof(double),
                              cudaMemcpyDeviceToHost, c->stream));
   CUDA_CHECK(cudaStreamSynchronize(c->stream));
   return true;
}

// Run body() through a CUDA graph captured on first use (eager when graphs
// are off or the context traces / profiles).
template <class Body>
void run_graph(fac_ctx *c, cudaGraphExec_t &exec, long long &launches, Body body)
{
   if (!c->use_graph || c->tracing || c->profiling) {
      body();
      return;
   }
   if (!exec) {
      cudaGraph_t g = nullptr;
      const long long n0 = kernel_launch_count();
      CUDA_CHECK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
      c->capturing = true;
      try {
         body();
      } catch (...) {
         c->capturing = false;
         cudaStreamEndCapture(c->stream, &g);
         if (g) cudaGraphDestroy(g);
         throw;
      }
      c->capturing = false;
      CUDA_CHECK(cudaStreamEndCapture(c->stream, &g));
      launches = kernel_launch_count() - n0;
      add_kernel_launches(-launches);
      cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) {
         exec = nullptr;
         throw FacError(FAC_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
      }
   }
   CUDA_CHECK(cudaGraphLaunch(exec, c->stream));
   add_kernel_launches(launches);
}

}  // namespace

// The learned correction as the second stage of FGMRES's preconditioner:
// the cycle's correction z (Krylov slot zslot) for v (slot vslot) leaves
// the residual s = v - A z of the error equation; the network predicts the
// error e for s on the learned level (carried to the coarser levels by
// restriction), and z += alpha e with the per-problem minimal-residual
// alpha = <s, A e> / <A e, A e> (weighted; 0 when it would not lower the
// residual), so the stage never makes the preconditioner's residual worse.
void learned_precondition(fac_ctx *c, int vslot, int zslot)
{
   OpTimer ot(c, "kry_learned", -1);
   const int ln = c->learned_level;
   const int lmax = c->nlev - 1;
   const int np = nprob(c);
   LevelState &Lc = c->L[ln];
   // the cycle left restricted residuals in R on the coarser levels: R = v
   for (int l = 0; l < c->nlev; ++l) {
      LevelState &L = c->L[l];
      if (L.n0 > 0)
         CUDA_CHECK(cudaMemcpyAsync(L.r.p, kry_vec(c, l, vslot), (size_t)L.n0 * sizeof(double),
                                    cudaMemcpyDeviceToDevice, c->stream));
   }
   // composite residual of the error equation with rhs R into TR for the
   // correction in E (finer values restricted onto covered cells first)
   auto residual_of_e = [&]() {
      for (int l = lmax - 1; l >= 0; --l) restrict_op(c, FAC_E, FAC_E, l);
      comp_residual(c, FAC_TR, FAC_E, FAC_R, lmax, 1);
      for (int l = lmax - 1; l >= 0; --l) {
         comp_residual(c, FAC_TR, FAC_E, FAC_R, l, 1);
         restrict_op(c, FAC_TR, FAC_TR, l);
      }
   };
   zero_field(c, FAC_E);
   for (int l = 0; l < c->nlev; ++l) {
      LevelState &L = c->L[l];
      launch_g0_to_g1(c->stream, c->dim, (int)L.cell_chunks.size(), L.d_patches.p,
                      L.d_cell_chunks.p, kry_vec(c, l, zslot), L.e.p);
   }
   residual_of_e();
   // R = s
   for (int l = 0; l < c->nlev; ++l) {
      LevelState &L = c->L[l];
      if (L.n0 > 0)
         CUDA_CHECK(cudaMemcpyAsync(L.r.p, L.tr.p, (size_t)L.n0 * sizeof(double),
                                    cudaMemcpyDeviceToDevice, c->stream));
   }
   learned_gather(c, ln);
   const float *y = nullptr;
   if (cnn_forward_on_stream(c->cnn, c->cnn_in.p, Lc.npatch, c->stream, &y) != FAC_OK)
      throw FacError(FAC_ERR_CUDA, "learned correction: network forward failed");
   zero_field(c, FAC_E);
   launch_scatter_samples(c->stream, c->dim, (int)Lc.cell_chunks.size(), Lc.d_patches.p,
                          Lc.d_cell_chunks.p, y, c->cnn_scale.p, FAC_CNN_BOX, Lc.e.p);
   // TR = s - A e, then alpha from <s, s - TR> and <s - TR, s - TR>
   residual_of_e();
   CUDA_CHECK(cudaMemsetAsync(c->dot_acc.p, 0, np * sizeof(double2), c->stream));
   for (int l = 0; l < c->nlev; ++l) {
      LevelState &L = c->L[l];
      launch_dot_pair(c->stream, c->dim, (int)L.cell_chunks.size(), L.d_patches.p,
                      L.d_cell_chunks.p, L.r.p, L.tr.p, L.w.p, L.norm_partial.p,
                      L.d_prob_cell_chunk_begin.p, np, c->dot_acc.p);
   }
   launch_alpha(c->stream, c->dot_acc.p, c->active.p, np, c->alpha.p);
   for (int l = 0; l < c->nlev; ++l) {
      LevelState &L = c->L[l];
      launch_g1_to_g0<double>(c->stream, c->dim, (int)L.cell_chunks.size(), L.d_patches.p,
                              L.d_cell_chunks.p, L.e.p, kry_vec(c, l, zslot), true,
                              c->alpha.p);
   }
   CUDA_CHECK(cudaGetLastError());
}

// Relative size of the second Gram-Schmidt correction below which FGMRES
// skips it (see the Gram-Schmidt step).
constexpr double kReorthTol = 1e-10;

void fgmres_solve(fac_ctx *c, int m, int *converged, int *iterations, double *residual)
{
   const int np = nprob(c);
   if (m < 1 || m > 64) throw FacError(FAC_ERR_ARG, "restart length must be 1..64");
   kry_alloc(c, m);
   const int zslot0 = m + 1;
   std::vector<int> act(np, 1);
   c->host_active = act;
   set_active(c, act);
   dirichlet(c, false);
   zero_field(c, FAC_E);
   zero_field(c, FAC_R);
   std::vector<double> res, fnorm, wsum(np, 0.0);
   full_composite_residual(c, res);
   rms_norm(c, FAC_F, fnorm);
   {
      // sum of the weights per problem (the RMS norm's denominator)
      std::vector<double2> acc(np);
      CUDA_CHECK(cudaMemcpyAsync(acc.data(), c->norm_acc.p, np * sizeof(double2),
                                 cudaMemcpyDeviceToHost, c->stream));
      CUDA_CHECK(cudaStreamSynchronize(c->stream));
      for (int p = 0; p < np; ++p) wsum[p] = acc[p].y;
   }
   std::vector<double> eff(np);
   for (int p = 0; p < np; ++p) {
      eff[p] = c->residual_tol;
      if (c->rel_residual_tol >= 0) eff[p] = std::max(eff[p], fnorm[p] * c->rel_residual_tol);
      c->hist[p].assign(1, res[p]);
   }
   if (c->mixed) mixed_prepare(c);
   std::vector<int> its(np, 0), done(np, 0);
   for (int p = 0; p < np; ++p)
      if (!(res[p] > eff[p])) done[p] = 1;
   auto prec_body = [&]() {
      if (c->mixed) {
         // the mixed cycle keeps the error in e32 and solves the coarsest
         // level in FP64 on E: only level 0 of E needs its zero start
         CUDA_CHECK(cudaMemsetAsync(c->L[0].e.p, 0, c->L[0].e.n * sizeof(double), c->stream));
         for (int ln = 0; ln < c->nlev; ++ln)
            CUDA_CHECK(cudaMemsetAsync(c->L[ln].e32.p, 0, c->L[ln].e32.n * sizeof(float),
                                       c->stream));
         fac_cycle_mixed(c, c->nlev - 1);
      } else {
         zero_field(c, FAC_E);
         fac_cycle_recursive(c, c->nlev - 1);
      }
   };
   auto apply_body = [&]() {
      // as for u in the solve: finer values restricted onto covered cells
      // first (finest first, so each level passes on what it received),
      // then the composite residual level by level.  Each residual fills
      // its level's ghost cells itself (homogeneous boundary values of the
      // error equation), so the restrictions need no fills of their own.
      const int lmax = c->nlev - 1;
      for (int ln = lmax - 1; ln >= 0; --ln) restrict_op(c, FAC_E, FAC_E, ln);
      comp_residual(c, FAC_TR, FAC_E, kFieldZero, lmax, 1);
      for (int ln = lmax - 1; ln >= 0; --ln) {
         comp_residual(c, FAC_TR, FAC_E, kFieldZero, ln, 1);
         restrict_op(c, FAC_TR, FAC_TR, ln);
      }
   };
   const int H = m + 1;  // Hessenberg rows
   std::vector<double> h((size_t)np * H * m), cs((size_t)np * m), sn((size_t)np * m),
      g((size_t)np * H);
   std::vector<int> kp(np);
   std::vector<double> dots, coef, a(np);
   while (true) {
      for (int p = 0; p < np; ++p) act[p] = !done[p] && its[p] < c->max_cycles;
      bool any = false;
      for (int v : act) any = any || v;
      if (!any) break;
      set_active(c, act);
      c->host_active = act;
      // V_0 = r / beta
      std::vector<int> cyc = act;
      std::fill(g.begin(), g.end(), 0.0);
      std::fill(h.begin(), h.end(), 0.0);
      for (int p = 0; p < np; ++p) {
         const double beta = res[p] * std::sqrt(wsum[p]);
         g[(size_t)p * H] = beta;
         a[p] = cyc[p] && beta > 0 ? 1.0 / beta : 0.0;
         kp[p] = 0;
      }
      // V_0 = R / beta, also back into R, the preconditioner's input
      kry_combine(c, 0, a, 0, 0, coef, nullptr, FAC_R, FAC_R);
      for (int j = 0; j < m; ++j) {
         bool live = false;
         for (int v : act) live = live || v;
         if (!live) break;
         // Z_j = M^-1 V_j: one FAC cycle on the residual V_j (R holds V_j)
         {
            OpTimer ot(c, "kry_precondition", -1);
            run_graph(c, c->prec_exec, c->prec_launches, prec_body);
         }
         // Z_j into its slot and into E for W = A Z_j; the mixed cycle's
         // correction is in e32, so one pass writes both.  E's interior is
         // then Z_j on every level, and its ghost cells need no zeroing: the
         // operator fills every face ghost of a level before its residual
         // reads it, and edge and corner ghosts are not read
         const bool both = c->mixed && !c->cnn;
         for (int ln = 0; ln < c->nlev; ++ln) {
            LevelState &L = c->L[ln];
            if (c->mixed)
               launch_g1_to_g0<float>(c->stream, c->dim, (int)L.cell_chunks.size(),
                                      L.d_patches.p, L.d_cell_chunks.p, L.e32.p,
                                      kry_vec(c, ln, zslot0 + j), false, nullptr,
                                      both ? L.e.p : nullptr);
            else
               launch_g1_to_g0<double>(c->stream, c->dim, (int)L.cell_chunks.size(),
                                       L.d_patches.p, L.d_cell_chunks.p, L.e.p,
                                       kry_vec(c, ln, zslot0 + j));
         }
         if (c->cnn) learned_precondition(c, j, zslot0 + j);
         if (!both) {
            zero_field(c, FAC_E);
            for (int ln = 0; ln < c->nlev; ++ln) {
               LevelState &L = c->L[ln];
               launch_g0_to_g1(c->stream, c->dim, (int)L.cell_chunks.size(), L.d_patches.p,
                               L.d_cell_chunks.p, kry_vec(c, ln, zslot0 + j), L.e.p);
            }
         }
         // W = A Z_j = -(0 - A Z_j)
         {
            OpTimer ot(c, "kry_apply", -1);
            run_graph(c, c->apply_exec, c->apply_launches, apply_body);
         }
         // classical Gram-Schmidt, W = -TR - sum h_i V_i into slot j + 1,
         // repeated once for the problems that need it (below)
         const int K = j + 1;
         kry_dots(c, 0, 0, K, dots, FAC_TR, true);  // <TR, V_i>, i <= j, and <TR, TR>
         std::vector<double> before(np, 0.0);
         coef.assign((size_t)np * K, 0.0);
         for (int p = 0; p < np; ++p) {
            a[p] = -1.0;
            before[p] = dots[(size_t)p * (K + 1) + K];
            for (int i = 0; i < K; ++i) {
               const double hi = act[p] ? -dots[(size_t)p * (K + 1) + i] : 0.0;
               h[((size_t)p * H + i) * m + j] = hi;
               coef[(size_t)p * K + i] = -hi;
            }
         }
         // W' = -TR - sum h_i V_i into slot j + 1 with <W', W'>; with the
         // fused pass also the second-pass coefficients d_i = <W', V_i>
         std::vector<double> nw(np, 0.0), d2;
         const bool fused = kry_combine_dots(c, j + 1, a, 0, K, coef, d2, FAC_TR);
         if (fused) {
            for (int p = 0; p < np; ++p) nw[p] = d2[(size_t)p * (K + 1) + K];
         } else {
            kry_combine(c, j + 1, a, 0, K, coef, &dots, FAC_TR);
            for (int p = 0; p < np; ++p) nw[p] = dots[p];
         }
         // Second pass where it is needed.  With the fused pass the d_i are
         // measured: the pass would move W' by ||d||, so it runs where
         // ||d|| > kReorthTol ||W'||.  Skipping it leaves V_{j+1} that far from
         // orthogonal to the V_i; the Arnoldi relation A Z = V H holds either
         // way, and a basis that far from orthonormal changes the residual
         // estimate only by a factor 1 + O(j kReorthTol).  Without the d_i:
         // where W' lost more than half its norm (cancellation).
         bool again = false;
         std::vector<int> reo(np, 0);
         // squared norm of V_{j+1} before its normalisation, and -d_i of the
         // second pass (0 for the problems that need none)
         std::vector<double> hn2(nw), dcoef((size_t)np * K, 0.0);
         bool exact = false;
         if (fused) {
            for (int p = 0; p < np; ++p) {
               if (!act[p]) continue;
               double s2 = 0.0;
               for (int i = 0; i < K; ++i) {
                  const double d = d2[(size_t)p * (K + 1) + i];
                  s2 += d * d;
               }
               if (!(s2 > kReorthTol * kReorthTol * nw[p])) continue;
               reo[p] = again = true;
               for (int i = 0; i < K; ++i) {
                  const double d = d2[(size_t)p * (K + 1) + i];
                  h[((size_t)p * H + i) * m + j] += d;
                  dcoef[(size_t)p * K + i] = -d;
               }
               // W' - sum d_i V_i is orthogonal to the V_i: its norm follows
               // from ||W'|| and the d_i while these are small against W'
               hn2[p] = nw[p] - s2;
               if (!(hn2[p] > 0.5 * nw[p])) exact = true;
            }
         } else {
            for (int p = 0; p < np; ++p)
               if (act[p] && nw[p] < 0.25 * before[p]) reo[p] = again = true;
            exact = again;
         }
         if (exact) {
            // second pass as its own combination, with the norm of the result
            if (!fused) {
               kry_dots(c, j + 1, 0, K, dots);
               for (int p = 0; p < np; ++p)
                  for (int i = 0; i < K; ++i) {
                     const double d = reo[p] ? dots[(size_t)p * K + i] : 0.0;
                     h[((size_t)p * H + i) * m + j] += d;
                     dcoef[(size_t)p * K + i] = -d;
                  }
            }
            std::fill(a.begin(), a.end(), 1.0);
            kry_combine(c, j + 1, a, 0, K, dcoef, &dots);
            for (int p = 0; p < np; ++p) hn2[p] = dots[p];
            std::fill(dcoef.begin(), dcoef.end(), 0.0);
            again = false;
         }
         for (int p = 0; p < np; ++p) {
            if (!act[p]) {
               a[p] = 0.0;
               continue;
            }
            double *hp = &h[(size_t)p * H * m];
            const double hn = std::sqrt(std::max(0.0, hn2[p]));
            hp[(size_t)(j + 1) * m + j] = hn;
            a[p] = hn > 0 ? 1.0 / hn : 0.0;
            // Givens rotations on column j
            for (int i = 0; i < j; ++i) {
               const double x = hp[(size_t)i * m + j], y = hp[(size_t)(i + 1) * m + j];
               hp[(size_t)i * m + j] = cs[(size_t)p * m + i] * x + sn[(size_t)p * m + i] * y;
               hp[(size_t)(i + 1) * m + j] = -sn[(size_t)p * m + i] * x + cs[(size_t)p * m + i] * y;
            }
            const double x = hp[(size_t)j * m + j], y = hp[(size_t)(j + 1) * m + j];
            const double r = std::hypot(x, y);
            const double cj = r > 0 ? x / r : 1.0, sj = r > 0 ? y / r : 0.0;
            cs[(size_t)p * m + j] = cj;
            sn[(size_t)p * m + j] = sj;
            hp[(size_t)j * m + j] = r;
            hp[(size_t)(j + 1) * m + j] = 0.0;
            double *gp = &g[(size_t)p * H];
            gp[j + 1] = -sj * gp[j];
            gp[j] = cj * gp[j];
            its[p] += 1;
            kp[p] = j + 1;
            const double est = std::fabs(gp[j + 1]) / std::sqrt(std::max(wsum[p], 1e-300));
            c->hist[p].push_back(est);
            if (!(est > eff[p]) || its[p] >= c->max_cycles || !(hn > 0)) act[p] = 0;
         }
         // V_{j+1} = (W' - sum d_i V_i) / ||.||, the second Gram-Schmidt pass
         // and the normalisation in one combination, also into R for the
         // next preconditioning
         if (again) {
            for (int p = 0; p < np; ++p)
               for (int i = 0; i < K; ++i) dcoef[(size_t)p * K + i] *= a[p];
            kry_combine(c, j + 1, a, 0, K, dcoef, nullptr, kNoField, FAC_R);
         } else {
            kry_combine(c, j + 1, a, 0, 0, coef, nullptr, kNoField, FAC_R);
         }
         set_active(c, act);
         c->host_active = act;
      }
      // x += Z y for every problem of this restart cycle
      std::vector<double> y((size_t)np * m, 0.0);
      for (int p = 0; p < np; ++p) {
         if (!cyc[p]) continue;
         const double *hp = &h[(size_t)p * H * m];
         const double *gp = &g[(size_t)p * H];
         for (int i = kp[p] - 1; i >= 0; --i) {
            double sum = gp[i];
            for (int q = i + 1; q < kp[p]; ++q) sum -= hp[(size_t)i * m + q] * y[(size_t)p * m + q];
            y[(size_t)p * m + i] = hp[(size_t)i * m + i] != 0 ? sum / hp[(size_t)i * m + i] : 0.0;
         }
      }
      set_active(c, cyc);
      c->host_active = cyc;
      int kmax = 0;
      for (int p = 0; p < np; ++p)
         if (cyc[p]) kmax = std::max(kmax, kp[p]);
      std::vector<double> yk((size_t)np * std::max(1, kmax), 0.0);
      for (int p = 0; p < np; ++p)
         for (int i = 0; i < kmax; ++i) yk[(size_t)p * kmax + i] = y[(size_t)p * m + i];
      if (kmax > 0)
         CUDA_CHECK(cudaMemcpyAsync(c->kry_coef.p, yk.data(), (size_t)np * kmax * sizeof(double),
                                    cudaMemcpyHostToDevice, c->stream));
      for (int ln = 0; ln < c->nlev; ++ln) {
         LevelState &L = c->L[ln];
         launch_add_combination(c->stream, c->dim, (int)L.cell_chunks.size(), L.d_patches.p,
                                L.d_cell_chunks.p, L.u.p, kry_vec(c, ln, zslot0),
                                std::max<long long>(1, L.n0), kmax, c->kry_coef.p);
      }
      for (int ln = c->nlev - 2; ln >= 0; --ln) restrict_solution(c, FAC_U, ln);
      std::vector<double> nr;
      full_composite_residual(c, nr);
      for (int p = 0; p < np; ++p) {
         if (!cyc[p]) continue;
         res[p] = nr[p];
         if (!c->hist[p].empty()) c->hist[p].back() = nr[p];
         if (!(nr[p] > eff[p])) done[p] = 1;
      }
   }
   c->host_active.assign(np, 1);
   set_active(c, c->host_active);
   dirichlet(c, true);
   CUDA_CHECK(cudaStreamSynchronize(c->stream));
   for (int p = 0; p < np; ++p) {
      if (converged) converged[p] = res[p] < eff[p];
      if (iterations) iterations[p] = its[p];
      if (residual) residual[p] = res[p];
   }
}

size_t field_slice(const fac_ctx *c, int fid, int p, int ln, long long &off)
{
   const LevelState &L = c->L[ln];
   if (fid == FAC_U || fid == FAC_E) {
      off = L.prob_off1[p];
      return (size_t)(L.prob_off1[p + 1] - L.prob_off1[p]);
   }
   off = L.prob_off0[p];
   return (size_t)(L.prob_off0[p + 1] - L.prob_off0[p]);
}

void check_pl(fac_ctx *c, int p, int ln)
{
   if (p < 0 || p >= nprob(c)) throw FacError(FAC_ERR_ARG, "bad problem index");
   if (ln < 0 || ln >= c->nlev) throw FacError(FAC_ERR_ARG, "bad level number");
}

template <class F>
int guarded(F &&f)
{
   try {
      f();
      return FAC_OK;
   } catch (const FacError &e) {
      g_last_error = e.what();
      return e.code;
   } catch (const std::exception &e) {
      g_last_error = e.what();
      return FAC_ERR_ARG;
   }
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

extern "C" {

const char *fac_last_error(void) { return g_last_error.c_str(); }

namespace {

// The problem with k domain-covering levels below its level 0, each
// coarsening the domain by 2 (one patch each): every cell of an added level
// is covered by the next finer level, so the composite problem, its weights
// and its residual norm are unchanged and the FAC cycle becomes a full
// multigrid V-cycle whose coarsest solve is cheap (the reference reaches the
// same end with its hypre coarse solver, CellPoissonFACOps.C:1741-1781).
HostProblem extend_problem(const HostProblem &P, int k, int dim)
{
   if (P.nlev + k > kMaxLevels) throw FacError(FAC_ERR_ARG, "too many levels with the extension");
   long long domain = 1, covered = 0;
   for (int a = 0; a < dim; ++a) {
      if (P.n0[a] % (1 << k) != 0)
         throw FacError(FAC_ERR_ARG, "level 0 not divisible by 2^levels for the extension");
      domain *= P.n0[a];
   }
   for (const Box &b : P.boxes[0]) covered += b.size();
   if (covered != domain)
      throw FacError(FAC_ERR_ARG, "the extension needs a level 0 that covers the domain");
   HostProblem E;
   for (int a = 0; a < 3; ++a) {
      E.n0[a] = a < dim ? P.n0[a] >> k : 1;
      E.xlo[a] = P.xlo[a];
      E.xup[a] = P.xup[a];
   }
   E.nlev = P.nlev + k;
   for (int j = k; j >= 1; --j) {
      const int ln = k - j;
      Box b;
      for (int a = 0; a < 3; ++a) {
         b.lo[a] = 0;
         b.hi[a] = a < dim ? (P.n0[a] >> j) - 1 : 0;
         E.ratio[ln][a] = (ln == 0 || a >= dim) ? 1 : 2;
      }
      E.boxes[ln].push_back(b);
   }
   for (int ln = 0; ln < P.nlev; ++ln) {
      for (int a = 0; a < 3; ++a)
         E.ratio[ln + k][a] = ln == 0 ? (a < dim ? 2 : 1) : P.ratio[ln][a];
      E.boxes[ln + k] = P.boxes[ln];
   }
   return E;
}

// D on the added levels from D of the caller's level 0 (level k): on each
// coarse face the mean of the 2^(dim-1) fine faces it covers, averaged in
// pairs along the tangential axes in increasing order; f, u and C there
// are zero (covered cells).  Host side, once per change of D.
void extend_coefficients(fac_ctx *c)
{
   const int k = c->ext_levels, dim = c->dim;
   for (int ln = 0; ln < k; ++ln) {
      LevelState &L = c->L[ln];
      CUDA_CHECK(cudaMemsetAsync(L.f.p, 0, L.f.n * sizeof(double), c->stream));
      CUDA_CHECK(cudaMemsetAsync(L.u.p, 0, L.u.n * sizeof(double), c->stream));
      if (c->spec.c_kind == 2)
         CUDA_CHECK(cudaMemsetAsync(L.c.p, 0, L.c.n * sizeof(double), c->stream));
   }
   if (c->spec.d_variable) {
      const LevelState &L0 = c->L[k];
      for (int p = 0; p < nprob(c); ++p) {
         const HostProblem &P = c->probs[p];
         // dense per-axis face arrays of the caller's level 0 (patches in
         // order; a face two patches share takes the later patch's value)
         int n[3];
         for (int a = 0; a < 3; ++a) n[a] = a < dim ? P.n0[a] << k : 1;
         std::vector<double> fine(L0.prob_offs[p + 1] - L0.prob_offs[p]);
         CUDA_CHECK(cudaMemcpyAsync(fine.data(), L0.d.p + L0.prob_offs[p],
                                    fine.size() * sizeof(double), cudaMemcpyDeviceToHost,
                                    c->stream));
         CUDA_CHECK(cudaStreamSynchronize(c->stream));
         std::vector<std::vector<double> > dense(dim);
         int ext[3][3];
         for (int a = 0; a < dim; ++a) {
            for (int q = 0; q < 3; ++q) ext[a][q] = n[q] + (q == a ? 1 : 0);
            dense[a].assign((size_t)ext[a][0] * ext[a][1] * ext[a][2], 0.0);
         }
         size_t off = 0;
         for (const Box &b : P.boxes[k]) {
            for (int a = 0; a < dim; ++a) {
               const Box sb = side_box(b, a);
               for (int z = sb.lo[2]; z <= sb.hi[2]; ++z)
                  for (int y = sb.lo[1]; y <= sb.hi[1]; ++y)
                     for (int x = sb.lo[0]; x <= sb.hi[0]; ++x)
                        dense[a][((size_t)z * ext[a][1] + y) * ext[a][0] + x] = fine[off++];
            }
         }
         for (int ln = k - 1; ln >= 0; --ln) {
            for (int q = 0; q < 3; ++q) n[q] = q < dim ? n[q] / 2 : 1;
            std::vector<std::vector<double> > coarse(dim);
            for (int a = 0; a < dim; ++a) {
               int ce[3];
               for (int q = 0; q < 3; ++q) ce[q] = n[q] + (q == a ? 1 : 0);
               // every other face along the normal, then pair means along
               // each tangential axis in turn
               std::vector<double> t = dense[a];
               int te[3] = {ext[a][0], ext[a][1], ext[a][2]};
               auto take = [&](int ax) {
                  int ne[3] = {te[0], te[1], te[2]};
                  const bool normal = ax == a;
                  ne[ax] = normal ? (te[ax] + 1) / 2 : te[ax] / 2;
                  std::vector<double> o((size_t)ne[0] * ne[1] * ne[2]);
                  for (int z = 0; z < ne[2]; ++z)
                     for (int y = 0; y < ne[1]; ++y)
                        for (int x = 0; x < ne[0]; ++x) {
                           int i0[3] = {x, y, z};
                           int i1[3] = {x, y, z};
                           i0[ax] *= 2;
                           i1[ax] = i0[ax] + 1;
                           const double v0 =
                              t[((size_t)i0[2] * te[1] + i0[1]) * te[0] + i0[0]];
                           o[((size_t)z * ne[1] + y) * ne[0] + x] =
                              normal ? v0
                                     : 0.5 * (v0 + t[((size_t)i1[2] * te[1] + i1[1]) * te[0] +
                                                     i1[0]]);
                        }
                  t.swap(o);
                  for (int q = 0; q < 3; ++q) te[q] = ne[q];
               };
               take(a);
               for (int tt = 0; tt < dim; ++tt)
                  if (tt != a) take(tt);
               for (int q = 0; q < 3; ++q)
                  if (te[q] != ce[q]) throw FacError(FAC_ERR_STATE, "extension face count");
               coarse[a].swap(t);
               for (int q = 0; q < 3; ++q) ext[a][q] = ce[q];
            }
            dense.swap(coarse);
            // the added level is one patch over the domain: its side arrays
            // per axis are the dense arrays
            const LevelState &L = c->L[ln];
            long long o = L.prob_offs[p];
            for (int a = 0; a < dim; ++a) {
               if (o + (long long)dense[a].size() > L.prob_offs[p + 1])
                  throw FacError(FAC_ERR_STATE, "extension side layout");
               CUDA_CHECK(cudaMemcpyAsync(L.d.p + o, dense[a].data(),
                                          dense[a].size() * sizeof(double),
                                          cudaMemcpyHostToDevice, c->stream));
               o += (long long)dense[a].size();
            }
            CUDA_CHECK(cudaStreamSynchronize(c->stream));
         }
      }
   }
   c->ext_dirty = false;
}

void ensure_extension(fac_ctx *c)
{
   if (c->ext_levels > 0 && c->ext_dirty) extend_coefficients(c);
}

}  // namespace

int fac_set_coarse_extension(fac_ctx *ctx, int levels)
{
   return guarded([&] {
      check_state(ctx, false);
      if (!ctx->probs.empty())
         throw FacError(FAC_ERR_STATE, "set the extension before adding problems");
      if (levels < 0 || levels > kMaxLevels - 1) throw FacError(FAC_ERR_ARG, "bad level count");
      ctx->ext_levels = levels;
   });
}

int fac_extend_coefficients(fac_ctx *ctx)
{
   return guarded([&] {
      check_ops(ctx);
      ctx->ext_dirty = true;
      ensure_extension(ctx);
   });
}

namespace {

// Composite-vector operations act on every problem: lists compacted to
// converged problems are restored first.
void vec_all_active(fac_ctx *c)
{
   const int np = nprob(c);
   bool all = (int)c->host_active.size() == np;
   for (int v : c->host_active) all = all && v;
   if (!all) {
      c->host_active.assign(np, 1);
      set_active(c, c->host_active);
   }
}

std::vector<double2> vec_reduce(fac_ctx *c, int mode, int fid_x, int fid_y)
{
   vec_all_active(c);
   const int np = nprob(c);
   const int gx = field_ghost(fid_x), gy = field_ghost(fid_y);
   CUDA_CHECK(cudaMemsetAsync(c->norm_acc.p, 0, np * sizeof(double2), c->stream));
   for (int ln = 0; ln < c->nlev; ++ln) {
      LevelState &L = c->L[ln];
      launch_vec_reduce(c->stream, c->dim, mode, (int)L.cell_chunks.size(), L.d_patches.p,
                        L.d_cell_chunks.p, field_ptr(L, fid_x), gx, field_ptr(L, fid_y), gy,
                        L.w.p, L.norm_partial.p, L.d_prob_cell_chunk_begin.p, np,
                        c->norm_acc.p);
   }
   CUDA_CHECK(cudaGetLastError());
   std::vector<double2> acc(np);
   CUDA_CHECK(cudaMemcpyAsync(acc.data(), c->norm_acc.p, np * sizeof(double2),
                              cudaMemcpyDeviceToHost, c->stream));
   CUDA_CHECK(cudaStreamSynchronize(c->stream));
   return acc;
}

}  // namespace

int fac_vec_dot(fac_ctx *ctx, int fid_x, int fid_y, double *dots)
{
   return guarded([&] {
      check_ops(ctx);
      if (!dots) throw FacError(FAC_ERR_ARG, "null output");
      const std::vector<double2> acc = vec_reduce(ctx, 0, fid_x, fid_y);
      for (int p = 0; p < nprob(ctx); ++p) dots[p] = acc[p].x;
   });
}

int fac_vec_l2_norm(fac_ctx *ctx, int fid, double *norms)
{
   return guarded([&] {
      check_ops(ctx);
      if (!norms) throw FacError(FAC_ERR_ARG, "null output");
      const std::vector<double2> acc = vec_reduce(ctx, 0, fid, fid);
      for (int p = 0; p < nprob(ctx); ++p) norms[p] = std::sqrt(acc[p].x);
   });
}

int fac_vec_max_norm(fac_ctx *ctx, int fid, double *norms)
{
   return guarded([&] {
      check_ops(ctx);
      if (!norms) throw FacError(FAC_ERR_ARG, "null output");
      const std::vector<double2> acc = vec_reduce(ctx, 1, fid, fid);
      for (int p = 0; p < nprob(ctx); ++p) norms[p] = acc[p].x;
   });
}

int fac_vec_linear_sum(fac_ctx *ctx, int fid_z, const double *a, int fid_x, const double *b,
                       int fid_y)
{
   return guarded([&] {
      check_ops(ctx);
      if (!a || !b) throw FacError(FAC_ERR_ARG, "null coefficients");
      if (fid_z == FAC_W) throw FacError(FAC_ERR_ARG, "the weights are not a vector");
      vec_all_active(ctx);
      const int np = nprob(ctx);
      ctx->vec_coef.alloc(2 * (size_t)np);
      CUDA_CHECK(cudaMemcpyAsync(ctx->vec_coef.p, a, np * sizeof(double),
                                 cudaMemcpyHostToDevice, ctx->stream));
      CUDA_CHECK(cudaMemcpyAsync(ctx->vec_coef.p + np, b, np * sizeof(double),
                                 cudaMemcpyHostToDevice, ctx->stream));
      const int gz = field_ghost(fid_z), gx = field_ghost(fid_x), gy = field_ghost(fid_y);
      for (int ln = 0; ln < ctx->nlev; ++ln) {
         LevelState &L = ctx->L[ln];
         launch_vec_lincomb(ctx->stream, ctx->dim, (int)L.cell_chunks.size(), L.d_patches.p,
                            L.d_cell_chunks.p, field_ptr(L, fid_z), gz, field_ptr(L, fid_x), gx,
                            field_ptr(L, fid_y), gy, ctx->vec_coef.p, ctx->vec_coef.p + np);
      }
      CUDA_CHECK(cudaGetLastError());
      CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
   });
}

// ---------------------------------------------------------------------------
// regrid step: tagging and Berger-Rigoutsos clustering
// ---------------------------------------------------------------------------

int fac_tag_gradient(fac_ctx *ctx, int fid, int ln, double threshold, long long *ntagged)
{
   return guarded([&] {
      check_ops(ctx);
      check_pl(ctx, 0, ln);
      if (field_ghost(fid) != 1 || fid == FAC_W)
         throw FacError(FAC_ERR_ARG, "tagging reads a ghosted FP64 cell field (U or E)");
      vec_all_active(ctx);
      LevelState &L = ctx->L[ln];
      const int np = nprob(ctx);
      if (L.tag.n != (size_t)std::max<long long>(1, L.n0))
         L.tag.alloc(std::max<long long>(1, L.n0));
      ctx->tag_counts.alloc(np);
      CUDA_CHECK(cudaMemsetAsync(ctx->tag_counts.p, 0, np * sizeof(unsigned long long),
                                 ctx->stream));
      launch_adaption_tags(ctx->stream, ctx->dim, (int)L.cell_chunks.size(), L.d_patches.p,
                           L.d_cell_chunks.p, field_ptr(L, fid), threshold, L.tag.p,
                           ctx->tag_counts.p, nullptr);
      CUDA_CHECK(cudaGetLastError());
      std::vector<unsigned long long> cnt(np);
      CUDA_CHECK(cudaMemcpyAsync(cnt.data(), ctx->tag_counts.p, np * sizeof(unsigned long long),
                                 cudaMemcpyDeviceToHost, ctx->stream));
      CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
      if (ntagged)
         for (int p = 0; p < np; ++p) ntagged[p] = (long long)cnt[p];
   });
}

int fac_download_tags(fac_ctx *ctx, int problem, int ln, unsigned char *host)
{
   return guarded([&] {
      check_ops(ctx);
      check_pl(ctx, problem, ln);
      if (!host) throw FacError(FAC_ERR_ARG, "null output");
      LevelState &L = ctx->L[ln];
      if (!L.tag.p) throw FacError(FAC_ERR_STATE, "no tags on this level (fac_tag_gradient)");
      const long long off = L.prob_off0[problem], n = L.prob_off0[problem + 1] - off;
      CUDA_CHECK(cudaMemcpyAsync(host, L.tag.p + off, (size_t)n, cudaMemcpyDeviceToHost,
                                 ctx->stream));
      CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
   });
}

namespace {

// One node of the clustering tree (BergerRigoutsosNode on one process).
struct BrTree {
   int lo[3], hi[3];          // box (after the shrink to the tags' bounding box)
   int left = -1, right = -1;
   int state = 0;             // 1 accepted, 2 split, 3 no tag
   std::vector<int> h[3];     // histograms of the (shrunken) box
};

// C integer division (toward zero), as the reference's int arithmetic
inline int cdiv(int a, int b) { return a / b; }

struct BrParams {
   int dim;
   int min_box[3], max_box[3];
   double efficiency, combine;
};

// findZeroCutSwath (mesh/BergerRigoutsosNode.C:1636-1700)
bool zero_cut(const BrParams &P, const BrTree &n, int a, int &cut_lo, int &cut_hi)
{
   const int lo = n.lo[a], hi = n.hi[a];
   const int lim_lo = lo + P.min_box[a], lim_hi = hi - P.min_box[a];
   const std::vector<int> &h = n.h[a];
   cut_lo = cut_hi = cdiv(lo + hi, 2);
   while (cut_lo >= lim_lo && cut_hi <= lim_hi) {
      if (h[cut_lo - lo] == 0) {
         cut_hi = cut_lo;
         while (cut_lo > lim_lo && h[cut_lo - lo - 1] == 0) --cut_lo;
         return true;
      }
      if (h[cut_hi - lo] == 0) {
         cut_lo = cut_hi;
         while (cut_hi < lim_hi && h[cut_hi - lo + 1] == 0) ++cut_hi;
         return true;
      }
      --cut_lo;
      ++cut_hi;
   }
   return false;
}

// cutAtInflection (mesh/BergerRigoutsosNode.C:1718-1812), with the
// reference's defaults DEV_max_inflection_cut_from_center = 1 and
// DEV_min_box_size_from_cutting = 0; the product of the two Laplacians is
// formed in 64 bits (its sign is what the reference tests)
void inflection_cut(const BrParams &P, const BrTree &n, int a, int &cut_pt, int &inflection)
{
   const std::vector<int> &h = n.h[a];
   const int size = (int)h.size();
   if (size < 4) {
      cut_pt = 1;
      for (int i = 2; i < size; ++i)
         if (std::abs(h[cut_pt] - h[cut_pt - 1]) < std::abs(h[i] - h[i - 1])) cut_pt = i;
      cut_pt += n.lo[a];
      inflection = 0;
      return;
   }
   const int min_size = std::max(P.min_box[a], 0);
   const int box_lo = 0, box_hi = size - 1;
   const int max_dist = (int)(1.0 * size / 2);
   const int mid = cdiv(box_lo + box_hi + 1, 2);
   const int lim_lo = std::max(box_lo + min_size, mid - max_dist);
   const int lim_hi = std::min(box_hi - min_size + 1, mid + max_dist);
   cut_pt = mid;
   inflection = std::abs((h[cut_pt - 1] - 2 * h[cut_pt] + h[cut_pt + 1]) -
                         (h[cut_pt - 2] - 2 * h[cut_pt - 1] + h[cut_pt]));
   int cl = mid - 1, ch = mid + 1;
   auto test = [&](int c) {
      const int la = h[c - 1] - 2 * h[c] + h[c + 1];
      const int lb = h[c - 2] - 2 * h[c - 1] + h[c];
      if ((long long)la * (long long)lb <= 0) {
         const int t = std::abs(la - lb);
         if (t > inflection) {
            cut_pt = c;
            inflection = t;
         }
      }
   };
   while (cl > lim_lo || ch < lim_hi) {
      if (cl > lim_lo) test(cl);
      if (ch < lim_hi) test(ch);
      --cl;
      ++ch;
   }
   cut_pt += n.lo[a];
}

// computeMinimalBoundingBoxForTags + acceptOrSplitBox
// (mesh/BergerRigoutsosNode.C:1251-1590) for a node whose histograms are
// known: shrink, then accept (state 1), find no tags (3), or cut into the
// children's boxes (state 2, boxes in lchild/rchild).
void decide(const BrParams &P, BrTree &n, int lchild[6], int rchild[6])
{
   const int d = P.dim;
   for (int a = 0; a < d; ++a) {
      std::vector<int> &h = n.h[a];
      int size = n.hi[a] - n.lo[a] + 1, b = 0, e = (int)h.size() - 1;
      while (h[b] == 0 && size > P.min_box[a]) {
         ++n.lo[a];
         ++b;
         --size;
      }
      while (h[e] == 0 && size > P.min_box[a]) {
         --n.hi[a];
         --e;
         --size;
      }
      h = std::vector<int>(h.begin() + b, h.begin() + e + 1);
   }
   int dims[3] = {1, 1, 1};
   long long size = 1;
   for (int a = 0; a < d; ++a) {
      dims[a] = n.hi[a] - n.lo[a] + 1;
      size *= dims[a];
   }
   bool over = false;
   for (int a = 0; a < d; ++a) over = over || dims[a] > P.max_box[a];
   if (!over) {
      long long tagged = 0;
      for (int v : n.h[0]) tagged += v;
      const double eff = size == 0 ? 1.0 : (double)tagged / (double)size;
      if (eff >= P.efficiency) {
         n.state = 1;
         return;
      }
      if (tagged == 0) {
         n.state = 3;
         return;
      }
   }
   int margin[3];
   bool none = true;  // IntVector's < : no direction can be cut
   for (int a = 0; a < d; ++a) {
      margin[a] = dims[a] - 2 * P.min_box[a];
      none = none && margin[a] < 0;
   }
   if (none) {
      n.state = 1;
      return;
   }
   int order[3] = {0, 1, 2};
   for (int d0 = 0; d0 < d - 1; ++d0)
      for (int d1 = d0 + 1; d1 < d; ++d1)
         if (margin[order[d0]] < margin[order[d1]]) std::swap(order[d0], order[d1]);
   int lft_hi[3] = {n.hi[0], n.hi[1], n.hi[2]}, rht_lo[3] = {n.lo[0], n.lo[1], n.lo[2]};
   int cut_dir = 0, k = 0;
   for (; k < d; ++k) {
      cut_dir = order[k];
      if (margin[cut_dir] < 0) continue;
      int cl, ch;
      if (zero_cut(P, n, cut_dir, cl, ch)) {
         lft_hi[cut_dir] = cl - 1;
         rht_lo[cut_dir] = ch + 1;
         break;
      }
   }
   if (k == d) {
      // DEV_inflection_cut_threshold_ar = 0: only the direction(s) of the
      // largest margin are cut
      const int leave = dims[order[0]] - 1;
      int inflection = -1, cut_pt = 0;
      for (int a = 0; a < d; ++a) {
         if (margin[a] < 0 || dims[a] <= leave) continue;
         int cp, ti;
         inflection_cut(P, n, a, cp, ti);
         if (inflection < ti || (inflection == ti && margin[a] > margin[cut_dir])) {
            cut_dir = a;
            cut_pt = cp;
            inflection = ti;
         }
      }
      lft_hi[cut_dir] = cut_pt - 1;
      rht_lo[cut_dir] = cut_pt;
   }
   for (int a = 0; a < 3; ++a) {
      lchild[a] = n.lo[a];
      lchild[3 + a] = lft_hi[a];
      rchild[a] = rht_lo[a];
      rchild[3 + a] = n.hi[a];
   }
   n.state = 2;
}

}  // namespace

namespace {

// Berger-Rigoutsos over the tags of level ln of the listed problems at once:
// problem probs[q] clusters inside its nbound[q] bound boxes (back to back
// in bound).  One dense tag array per problem; the trees are walked breadth
// first together, one histogram launch per depth for all open nodes.
// Boxes go out problem by problem (depth first, left before right);
// counts[q] gets problem probs[q]'s number of boxes, the return value their
// total (boxes beyond cap are counted, not written).
long long cluster_levels(fac_ctx *ctx, int ln, const std::vector<int> &probs,
                         const int *nbound, const int *bound, const BrParams &P, int cap,
                         int *boxes, int *counts)
{
   LevelState &L = ctx->L[ln];
   if (!L.tag.p) throw FacError(FAC_ERR_STATE, "no tags on this level (fac_tag_gradient)");
   const int d = ctx->dim;
   const int nq = (int)probs.size();
   // dense tag arrays over the bounding box of each problem's patches and
   // bound boxes (cells outside the patches hold no tags)
   std::vector<std::array<int, 3> > dlo(nq), dn(nq);
   std::vector<long long> doff(nq + 1, 0);
   std::vector<int> boff(nq + 1, 0);
   for (int q = 0; q < nq; ++q) boff[q + 1] = boff[q] + nbound[q];
   for (int q = 0; q < nq; ++q) {
      int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
      auto grow = [&](const int *blo, const int *bhi) {
         for (int a = 0; a < 3; ++a) {
            const int l = a < d ? blo[a] : 0, h = a < d ? bhi[a] : 0;
            lo[a] = std::min(lo[a], l);
            hi[a] = std::max(hi[a], h);
         }
      };
      for (int ip = L.prob_patch_begin[probs[q]]; ip < L.prob_patch_begin[probs[q] + 1]; ++ip)
         grow(L.hp[ip].lo, L.hp[ip].hi);
      for (int b = boff[q]; b < boff[q + 1]; ++b) {
         const int *bb = bound + 6 * b;
         for (int a = 0; a < d; ++a)
            if (bb[3 + a] < bb[a]) throw FacError(FAC_ERR_ARG, "empty bound box");
         grow(bb, bb + 3);
      }
      long long cells = 1;
      for (int a = 0; a < 3; ++a) {
         dlo[q][a] = lo[a];
         dn[q][a] = hi[a] - lo[a] + 1;
         cells *= dn[q][a];
      }
      doff[q + 1] = doff[q] + ((cells + 255) / 256) * 256;
   }
   DevArray<unsigned char> &dense = ctx->br_dense;
   if (dense.n < (size_t)std::max<long long>(1, doff[nq])) dense.alloc((size_t)std::max<long long>(1, doff[nq]));
   CUDA_CHECK(cudaMemsetAsync(dense.p, 0, (size_t)std::max<long long>(1, doff[nq]), ctx->stream));
   for (int q = 0; q < nq; ++q) {
      // the problem's own chunks of the full (uncompacted) cell list
      const int ch0 = L.prob_cell_chunk_begin[probs[q]];
      const int ch1 = L.prob_cell_chunk_begin[probs[q] + 1];
      launch_tags_dense(ctx->stream, d, ch1 - ch0, L.d_patches.p, L.ws_cell.all.p + ch0, L.tag.p,
                        probs[q], dlo[q].data(), dn[q].data(), dense.p + doff[q]);
   }
   CUDA_CHECK(cudaGetLastError());
   std::vector<BrTree> tree;
   std::vector<int> owner;  // problem slot q of each tree node
   std::vector<int> frontier;
   std::vector<std::vector<int> > roots(nq);
   for (int q = 0; q < nq; ++q)
      for (int b = boff[q]; b < boff[q + 1]; ++b) {
         BrTree t;
         for (int a = 0; a < 3; ++a) {
            t.lo[a] = a < d ? bound[6 * b + a] : 0;
            t.hi[a] = a < d ? bound[6 * b + 3 + a] : 0;
         }
         roots[q].push_back((int)tree.size());
         frontier.push_back((int)tree.size());
         tree.push_back(t);
         owner.push_back(q);
      }
   DevArray<BrNode> &d_nodes = ctx->br_nodes;
   DevArray<BrItem> &d_items = ctx->br_items;
   DevArray<int> &d_hist = ctx->br_hist;
   auto put = [&](auto &dev, const auto &host) {
      if (dev.n < host.size()) dev.alloc(host.size() * 2);
      if (!host.empty())
         CUDA_CHECK(cudaMemcpyAsync(dev.p, host.data(), host.size() * sizeof(host[0]),
                                    cudaMemcpyHostToDevice, ctx->stream));
   };
   while (!frontier.empty()) {
      std::vector<BrNode> nodes;
      std::vector<BrItem> items;
      long long hsize = 0;
      for (int f = 0; f < (int)frontier.size(); ++f) {
         const BrTree &t = tree[frontier[f]];
         const int q = owner[frontier[f]];
         BrNode nd;
         int e[3];
         for (int a = 0; a < 3; ++a) {
            nd.lo[a] = t.lo[a];
            nd.hi[a] = t.hi[a];
            nd.dlo[a] = dlo[q][a];
            nd.dn[a] = dn[q][a];
            e[a] = t.hi[a] - t.lo[a] + 1;
         }
         if (e[0] > kBrThreads * kBrMaxXPerThread)
            throw FacError(FAC_ERR_ARG, "clustering box too long along x");
         nd.hoff = hsize;
         nd.doff = doff[q];
         hsize += e[0] + e[1] + e[2];
         nodes.push_back(nd);
         // runs of rows of at most ~64k cells per block
         const int rows = e[1] * e[2];
         const int per = std::max(1, 65536 / e[0]);
         for (int r0 = 0; r0 < rows; r0 += per) items.push_back({f, r0, std::min(per, rows - r0), 0});
      }
      put(d_nodes, nodes);
      put(d_items, items);
      const size_t hn = (size_t)std::max<long long>(1, hsize);
      if (d_hist.n < hn) d_hist.alloc(hn * 2);
      CUDA_CHECK(cudaMemsetAsync(d_hist.p, 0, hn * sizeof(int), ctx->stream));
      launch_br_histogram(ctx->stream, (int)items.size(), d_items.p, d_nodes.p, dense.p, d_hist.p);
      CUDA_CHECK(cudaGetLastError());
      std::vector<int> hist(hn);
      CUDA_CHECK(cudaMemcpyAsync(hist.data(), d_hist.p, hn * sizeof(int), cudaMemcpyDeviceToHost,
                                 ctx->stream));
      CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
      std::vector<int> next;
      for (int f = 0; f < (int)frontier.size(); ++f) {
         const int id = frontier[f];
         const BrNode &nd = nodes[f];
         long long o = nd.hoff;
         for (int a = 0; a < 3; ++a) {
            const int e = nd.hi[a] - nd.lo[a] + 1;
            if (a < d) tree[id].h[a].assign(hist.begin() + o, hist.begin() + o + e);
            o += e;
         }
         int lc[6], rc[6];
         decide(P, tree[id], lc, rc);
         if (tree[id].state == 2) {
            for (int side = 0; side < 2; ++side) {
               const int *cb = side ? rc : lc;
               BrTree t;
               for (int a = 0; a < 3; ++a) {
                  t.lo[a] = cb[a];
                  t.hi[a] = cb[3 + a];
               }
               (side ? tree[id].right : tree[id].left) = (int)tree.size();
               next.push_back((int)tree.size());
               tree.push_back(t);
               owner.push_back(owner[id]);
            }
         }
      }
      frontier.swap(next);
   }
   // recombination, children before parents (runChildren_check,
   // mesh/BergerRigoutsosNode.C:719-790)
   auto box_size = [&](const BrTree &t) {
      long long sz = 1;
      for (int a = 0; a < d; ++a) sz *= t.hi[a] - t.lo[a] + 1;
      return sz;
   };
   for (int id = (int)tree.size() - 1; id >= 0; --id) {
      BrTree &t = tree[id];
      if (t.state != 2) continue;
      const BrTree &l = tree[t.left], &r = tree[t.right];
      bool fits = true;
      for (int a = 0; a < d; ++a) fits = fits && t.hi[a] - t.lo[a] + 1 <= P.max_box[a];
      const double reduction = (double)(box_size(l) + box_size(r)) / (double)box_size(t);
      if (l.state == 1 && r.state == 1 && fits && reduction >= P.combine) t.state = 1;
   }
   // the accepted boxes, problem by problem, depth first, left before right
   long long total = 0;
   for (int q = 0; q < nq; ++q) {
      int count = 0;
      std::vector<int> stack(roots[q].rbegin(), roots[q].rend());
      while (!stack.empty()) {
         const int id = stack.back();
         stack.pop_back();
         const BrTree &t = tree[id];
         if (t.state == 1) {
            if (total < cap)
               for (int a = 0; a < 3; ++a) {
                  boxes[6 * total + a] = t.lo[a];
                  boxes[6 * total + 3 + a] = t.hi[a];
               }
            ++count;
            ++total;
         } else if (t.state == 2) {
            stack.push_back(t.right);
            stack.push_back(t.left);
         }
      }
      counts[q] = count;
   }
   return total;
}

BrParams br_params(int d, const int *min_box, const int *max_box, double efficiency,
                   double combine)
{
   if (!min_box || !max_box) throw FacError(FAC_ERR_ARG, "bad clustering arguments");
   if (!(efficiency >= 0.0 && efficiency <= 1.0) || !(combine >= 0.0 && combine <= 1.0))
      throw FacError(FAC_ERR_ARG, "efficiency and combine efficiency must lie in [0, 1]");
   BrParams P;
   P.dim = d;
   P.efficiency = efficiency;
   P.combine = combine;
   for (int a = 0; a < 3; ++a) {
      P.min_box[a] = a < d ? min_box[a] : 1;
      P.max_box[a] = a < d && max_box[a] > 0 ? max_box[a] : std::numeric_limits<int>::max();
      if (a < d && P.min_box[a] < 1) throw FacError(FAC_ERR_ARG, "min_box must be >= 1");
   }
   return P;
}

}  // namespace

int fac_cluster_tags(fac_ctx *ctx, int problem, int ln, int nbound, const int *bound,
                     const int *min_box, const int *max_box, double efficiency, double combine,
                     int cap, int *boxes, int *nboxes)
{
   return guarded([&] {
      check_ops(ctx);
      check_pl(ctx, problem, ln);
      if (nbound < 1 || !bound || !nboxes || (cap > 0 && !boxes))
         throw FacError(FAC_ERR_ARG, "bad clustering arguments");
      const BrParams P = br_params(ctx->dim, min_box, max_box, efficiency, combine);
      int count = 0;
      cluster_levels(ctx, ln, std::vector<int>{problem}, &nbound, bound, P, cap, boxes, &count);
      *nboxes = count;
   });
}

int fac_cluster_tags_all(fac_ctx *ctx, int ln, const int *nbound, const int *bound,
                         const int *min_box, const int *max_box, double efficiency,
                         double combine, int cap, int *boxes, int *counts)
{
   return guarded([&] {
      check_ops(ctx);
      check_pl(ctx, 0, ln);
      const int np = nprob(ctx);
      if (!nbound || !bound || !counts || (cap > 0 && !boxes))
         throw FacError(FAC_ERR_ARG, "bad clustering arguments");
      for (int p = 0; p < np; ++p)
         if (nbound[p] < 1) throw FacError(FAC_ERR_ARG, "every problem needs a bound box");
      const BrParams P = br_params(ctx->dim, min_box, max_box, efficiency, combine);
      std::vector<int> probs(np);
      for (int p = 0; p < np; ++p) probs[p] = p;
      cluster_levels(ctx, ln, probs, nbound, bound, P, cap, boxes, counts);
   });
}

int fac_ctx_create(fac_ctx **ctx, int dim, int device)
{
   return guarded([&] {
      if (!ctx) throw FacError(FAC_ERR_ARG, "null output pointer");
      if (dim != 2 && dim != 3) throw FacError(FAC_ERR_ARG, "dim must be 2 or 3");
      if (device >= 0) {
         int ndev = 0;
         CUDA_CHECK(cudaGetDeviceCount(&ndev));
         if (device >= ndev) throw FacError(FAC_ERR_ARG, "bad device index");
         CUDA_CHECK(cudaSetDevice(device));
         // outside any stream capture: the shared-memory limit of the
         // one-launch coarsest solve (stays set for the process)
         if (!allow_solve_smem(kSolveSmemMax))
            throw FacError(FAC_ERR_CUDA, "shared-memory limit of the coarsest solve refused");
      }
      fac_ctx *c = new fac_ctx();
      c->dim = dim;
      c->device = device;
      for (int l = 0; l < 6; ++l) {
         c->bc.a[l] = 1.0;
         c->bc.b[l] = 0.0;
         c->bc.g[l] = 0.0;
      }
      if (device >= 0) {
         cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
         if (e != cudaSuccess) {
            delete c;
            throw FacError(FAC_ERR_CUDA, cudaGetErrorString(e));
         }
      }
      *ctx = c;
   });
}

int fac_ctx_destroy(fac_ctx *ctx)
{
   return guarded([&] {
      if (!ctx) return;
      if (ctx->device < 0) {
         g_dry = true;
         delete ctx;
         g_dry = false;
         return;
      }
      cudaSetDevice(ctx->device);
      cudaStreamSynchronize(ctx->stream);
      cudaStream_t s = ctx->stream;
      delete ctx;
      cudaStreamDestroy(s);
   });
}

int fac_add_problem(fac_ctx *ctx, const int *n0, const double *xlo, const double *xup, int nlev,
                    const int *ratio, const int *npatch, const int *boxes, int *problem)
{
   return guarded([&] {
      check_state(ctx, false);
      if (!n0 || !xlo || !xup || !ratio || !npatch || !boxes)
         throw FacError(FAC_ERR_ARG, "null argument");
      if (nlev < 1 || nlev > kMaxLevels) throw FacError(FAC_ERR_ARG, "bad level count");
      HostProblem P;
      const int dim = ctx->dim;
      for (int a = 0; a < 3; ++a) {
         P.n0[a] = a < dim ? n0[a] : 1;
         P.xlo[a] = a < dim ? xlo[a] : 0.0;
         P.xup[a] = a < dim ? xup[a] : 1.0;
         if (P.n0[a] < 1) throw FacError(FAC_ERR_ARG, "bad n0");
      }
      P.nlev = nlev;
      int off = 0;
      for (int ln = 0; ln < nlev; ++ln) {
         for (int a = 0; a < 3; ++a) {
            P.ratio[ln][a] = a < dim ? ratio[3 * ln + a] : 1;
            if (P.ratio[ln][a] < 1 || P.ratio[ln][a] > kProlongRatioMax)
               throw FacError(FAC_ERR_ARG, "bad ratio (1 .. 16 per axis)");
         }
         if (npatch[ln] < 1) throw FacError(FAC_ERR_ARG, "empty level");
         for (int ip = 0; ip < npatch[ln]; ++ip, ++off) {
            Box b;
            for (int a = 0; a < 3; ++a) {
               b.lo[a] = boxes[6 * off + a];
               b.hi[a] = boxes[6 * off + 3 + a];
            }
            if (dim == 2) b.lo[2] = b.hi[2] = 0;
            if (b.empty()) throw FacError(FAC_ERR_ARG, "empty patch box");
            P.boxes[ln].push_back(b);
         }
      }
      if (ctx->ext_levels > 0) P = extend_problem(P, ctx->ext_levels, dim);
      ctx->probs.push_back(P);
      if (problem) *problem = (int)ctx->probs.size() - 1;
   });
}

int fac_set_poisson(fac_ctx *ctx, int d_variable, double d_const, int c_kind, double c_const)
{
   return guarded([&] {
      check_state(ctx, false);
      if (c_kind < 0 || c_kind > 2) throw FacError(FAC_ERR_ARG, "bad c_kind");
      ctx->spec.d_variable = d_variable ? 1 : 0;
      ctx->spec.d_const = d_const;
      ctx->spec.c_kind = c_kind;
      ctx->spec.c_const = c_const;
   });
}

int fac_set_bc(fac_ctx *ctx, const double *a, const double *b, const double *g)
{
   return guarded([&] {
      if (!ctx || !a || !b || !g) throw FacError(FAC_ERR_ARG, "null argument");
      for (int l = 0; l < 2 * ctx->dim; ++l) {
         ctx->bc.a[l] = a[l];
         ctx->bc.b[l] = b[l];
         ctx->bc.g[l] = g[l];
      }
      ctx->bc_object = true;
      // kernels take the coefficients by value: graphs captured with the
      // old ones are captured again
      ctx->drop_graph();
   });
}

int fac_set_params(fac_ctx *ctx, int max_cycles, double residual_tol, double relative_residual_tol,
                   int pre_sweeps, int post_sweeps, double coarse_tol, int coarse_max_it, int ewing)
{
   return guarded([&] {
      if (!ctx) throw FacError(FAC_ERR_ARG, "null context");
      // FACPreconditioner::getFromInput range checks (FACPreconditioner.C:80-114)
      if (max_cycles < 1) throw FacError(FAC_ERR_ARG, "max_cycles");
      if (!(residual_tol > 0)) throw FacError(FAC_ERR_ARG, "residual_tol");
      if (pre_sweeps < 0 || post_sweeps < 0) throw FacError(FAC_ERR_ARG, "sweeps");
      if (!(coarse_tol > 0)) throw FacError(FAC_ERR_ARG, "coarse_solver_tolerance");
      if (coarse_max_it < 1) throw FacError(FAC_ERR_ARG, "coarse_solver_max_iterations");
      ctx->max_cycles = max_cycles;
      ctx->residual_tol = residual_tol;
      ctx->rel_residual_tol = relative_residual_tol;
      ctx->pre_sweeps = pre_sweeps;
      ctx->post_sweeps = post_sweeps;
      ctx->coarse_tol = coarse_tol;
      ctx->coarse_max_it = coarse_max_it;
      ctx->ewing = ewing;
      ctx->drop_graph();  // sweep counts are part of the captured cycle
   });
}

// Stage size and depth of the staged pass; rebuilds the unit tables of an
// initialised context.
void set_stage_shape(fac_ctx *ctx, int bytes, int depth)
{
   if (bytes < 4096 || bytes > (kStageSmemMax - kStageBarrierBytes) / 2)
      throw FacError(FAC_ERR_ARG, "stage budget out of range");
   if (depth < 2 || depth > kStageDepthMax) throw FacError(FAC_ERR_ARG, "stage depth out of range");
   ctx->stage_budget = bytes;
   ctx->stage_depth = depth;
   if (ctx->initialized && ctx->device >= 0) {
      CUDA_CHECK(cudaSetDevice(ctx->device));
      CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
      ctx->drop_graph();
      for (int ln = 0; ln < ctx->nlev; ++ln) {
         build_stage_units(ctx, ln);
         build_res_units(ctx, ln);
      }
      register_work_lists(ctx);
      launch_compact(ctx->stream, ctx->d_work_regs.p, (int)ctx->work_regs.size(),
                     ctx->active.p, nprob(ctx));
      CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
   }
}

int fac_set_stage_budget(fac_ctx *ctx, int bytes)
{
   return guarded([&] {
      if (!ctx) throw FacError(FAC_ERR_ARG, "null context");
      set_stage_shape(ctx, bytes, ctx->stage_depth);
   });
}

int fac_set_stage_depth(fac_ctx *ctx, int depth)
{
   return guarded([&] {
      if (!ctx) throw FacError(FAC_ERR_ARG, "null context");
      set_stage_shape(ctx, ctx->stage_budget, depth);
   });
}

int fac_set_fused_residual(fac_ctx *ctx, int on)
{
   return guarded([&] {
      if (!ctx) throw FacError(FAC_ERR_ARG, "null context");
      if (on < -1 || on > 1) throw FacError(FAC_ERR_ARG, "fused residual setting must be -1, 0 or 1");
      ctx->fused_residual = on;
      ctx->drop_graph();
   });
}

// Autotuner of the staged pass: rebuild the units for each candidate stage
// size and depth, time a red-black sweep of every staged level (CUDA
// events, best of three), keep the fastest.  Uses the smoothing fields (E,
// R or their FP32 copies) as scratch, so it belongs before a solve.
int fac_autotune(fac_ctx *ctx, int *chosen_bytes, int *chosen_depth, double *ms_per_candidate)
{
   return guarded([&] {
      check_ops(ctx);
      if (ctx->device < 0) throw FacError(FAC_ERR_STATE, "host-only context");
      static const int cand[] = {12 * 1024, 16 * 1024, 24 * 1024, 32 * 1024, 48 * 1024};
      const int nc = (int)(sizeof(cand) / sizeof(cand[0]));
      static const int depths[] = {2, 3};
      cudaEvent_t e0, e1;
      CUDA_CHECK(cudaEventCreate(&e0));
      CUDA_CHECK(cudaEventCreate(&e1));
      struct Ev {
         cudaEvent_t a, b;
         ~Ev()
         {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
         }
      } ev{e0, e1};
      const bool was_tracing = ctx->tracing, was_prof = ctx->profiling;
      ctx->tracing = ctx->profiling = false;
      int best = ctx->stage_budget, best_depth = ctx->stage_depth;
      float best_ms = 1e30f;
      for (int kd = 0; kd < 2; ++kd)
         for (int k = 0; k < nc; ++k) {
            set_stage_shape(ctx, cand[k], depths[kd]);
            float t = 1e30f;
            for (int rep = 0; rep < 3; ++rep) {
               CUDA_CHECK(cudaEventRecord(e0, ctx->stream));
               for (int ln = 1; ln < ctx->nlev; ++ln) {
                  if (ctx->mixed) smooth32(ctx, ln, 1);
                  else smooth(ctx, FAC_E, FAC_R, ln, 1, -1.0);
               }
               CUDA_CHECK(cudaEventRecord(e1, ctx->stream));
               CUDA_CHECK(cudaEventSynchronize(e1));
               float ms = 0.f;
               CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
               t = std::min(t, ms);
            }
            if (ms_per_candidate) ms_per_candidate[kd * nc + k] = t;
            if (t < best_ms) {
               best_ms = t;
               best = cand[k];
               best_depth = depths[kd];
            }
         }
      ctx->tracing = was_tracing;
      ctx->profiling = was_prof;
      set_stage_shape(ctx, best, best_depth);
      if (chosen_bytes) *chosen_bytes = best;
      if (chosen_depth) *chosen_depth = best_depth;
   });
}

int fac_set_bc_faces(fac_ctx *ctx, int problem, int ln, int location, const double *abg)
{
   return guarded([&] {
      check_ops(ctx);
      check_pl(ctx, problem, ln);
      const int dim = ctx->dim, np = nprob(ctx);
      if (location < 0 || location >= 2 * dim) throw FacError(FAC_ERR_ARG, "bad location index");
      if (!abg) throw FacError(FAC_ERR_ARG, "null coefficients");
      if (ctx->face_off_host.empty()) {
         ctx->face_off_host.assign((size_t)kMaxLevels * 6 * np, -1);
         ctx->face_dom_host.assign((size_t)kMaxLevels * np * 6, 0);
         for (int l = 0; l < ctx->nlev; ++l)
            for (int p = 0; p < np; ++p) {
               const Box &d = ctx->L[l].domain[p];
               int *dm = &ctx->face_dom_host[((size_t)l * np + p) * 6];
               for (int a = 0; a < 3; ++a) {
                  dm[a] = d.lo[a];
                  dm[3 + a] = d.hi[a] - d.lo[a] + 1;
               }
            }
      }
      const Box &d = ctx->L[ln].domain[problem];
      long long n = 1;
      for (int t = 0; t < 3; ++t)
         if (t != location / 2) n *= d.hi[t] - d.lo[t] + 1;
      long long &off = ctx->face_off_host[((size_t)ln * 6 + location) * np + problem];
      if (off < 0) {
         off = (long long)ctx->face_host.size();
         ctx->face_host.resize(ctx->face_host.size() + 3 * (size_t)n);
      }
      std::copy(abg, abg + 3 * n, ctx->face_host.begin() + off);
      ctx->face_dev.upload(ctx->face_host, ctx->stream);
      ctx->face_off_dev.upload(ctx->face_off_host, ctx->stream);
      ctx->face_dom_dev.upload(ctx->face_dom_host, ctx->stream);
      CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
      ctx->bc.face_base = ctx->face_dev.p;
      ctx->bc.face_off = ctx->face_off_dev.p;
      ctx->bc.face_dom = ctx->face_dom_dev.p;
      ctx->bc.face_nprob = np;
      ctx->bc_faces = true;
      ctx->bc_object = true;
      ctx->drop_graph();  // kernels take the coefficients by value
   });
}

int fac_set_wait_test(fac_ctx *ctx, long long limit_cycles, int never)
{
   return guarded([&] {
      if (!ctx) throw FacError(FAC_ERR_ARG, "null context");
      if (limit_cycles < 1 || never < 0 || never > 1) throw FacError(FAC_ERR_ARG, "bad wait test");
      ctx->wait_test.limit = limit_cycles;
      ctx->wait_test.never = never;
      ctx->drop_graph();  // launches take the bound by value
   });
}

int fac_clear_device_error(fac_ctx *ctx)
{
   return guarded([&] {
      check_ops(ctx);
      CUDA_CHECK(cudaMemsetAsync(ctx->kerr.p, 0, sizeof(int), ctx->stream));
      CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
   });
}

int fac_set_staged(fac_ctx *ctx, int on)
{
   return guarded([&] {
      if (!ctx) throw FacError(FAC_ERR_ARG, "null context");
      ctx->staged = on != 0;
      ctx->drop_graph();
   });
}

int fac_set_fused(fac_ctx *ctx, int on)
{
   return guarded([&] {
      if (!ctx) throw FacError(FAC_ERR_ARG, "null context");
      ctx->fused = on != 0;
      ctx->drop_graph();
   });
}

int fac_set_graph(fac_ctx *ctx, int on)
{
   return guarded([&] {
      if (!ctx) throw FacError(FAC_ERR_ARG, "null context");
      ctx->use_graph = on != 0;
      ctx->drop_graph();
   });
}

int fac_set_learned(fac_ctx *ctx, fac_cnn *net, int level)
{
   return guarded([&] {
      check_ops(ctx);
      ctx->drop_graph();
      if (!net) {
         ctx->cnn = nullptr;
         ctx->learned_level = -1;
         return;
      }
      if (level < 1 || level >= ctx->nlev) throw FacError(FAC_ERR_ARG, "bad learned level");
      if (cnn_device(net) != ctx->device) throw FacError(FAC_ERR_ARG, "network on another device");
      LevelState &L = ctx->L[level];
      for (const Box &b : L.box)
         for (int a = 0; a < ctx->dim; ++a)
            if (b.hi[a] - b.lo[a] + 3 > FAC_CNN_BOX)
               throw FacError(FAC_ERR_ARG, "patch too large for the network's sample box");
      if (L.npatch > cnn_max_batch(net))
         throw FacError(FAC_ERR_ARG, "network batch smaller than the level's patch count");
      ctx->cnn = net;
      ctx->learned_level = level;
      ctx->cnn_in.alloc((size_t)L.npatch * FAC_CNN_BOX * FAC_CNN_BOX * FAC_CNN_BOX);
      ctx->cnn_scale.alloc(std::max(1, L.npatch));
      ctx->alpha.alloc(nprob(ctx));
      ctx->dot_acc.alloc(nprob(ctx));
   });
}

int fac_learned_samples(fac_ctx *ctx, int level, float *x, double *scale)
{
   return guarded([&] {
      check_ops(ctx);
      if (level < 0 || level >= ctx->nlev) throw FacError(FAC_ERR_ARG, "bad level");
      LevelState &L = ctx->L[level];
      for (const Box &b : L.box)
         for (int a = 0; a < ctx->dim; ++a)
            if (b.hi[a] - b.lo[a] + 3 > FAC_CNN_BOX)
               throw FacError(FAC_ERR_ARG, "patch too large for the network's sample box");
      DevArray<double> sc;
      sc.alloc(std::max(1, L.npatch));
      CUDA_CHECK(cudaMemsetAsync(L.e.p, 0, L.e.n * sizeof(double), ctx->stream));
      launch_g0_to_g1(ctx->stream, ctx->dim, (int)L.cell_chunks.size(), L.d_patches.p,
                      L.d_cell_chunks.p, L.r.p, L.e.p);
      ghost_fill(ctx, FAC_E, level, false, 1, nullptr);
      launch_patch_rms(ctx->stream, ctx->dim, L.npatch, L.d_patches.p, L.r.p, sc.p);
      launch_gather_samples(ctx->stream, ctx->dim, L.npatch, L.d_patches.p, L.e.p, sc.p, x,
                            FAC_CNN_BOX);
      if (scale)
         CUDA_CHECK(cudaMemcpyAsync(scale, sc.p, L.npatch * sizeof(double),
                                    cudaMemcpyDeviceToHost, ctx->stream));
      CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
   });
}

int fac_set_precision(fac_ctx *ctx, int mixed)
{
   return guarded([&] {
      check_state(ctx, false);
      if (mixed != 0 && mixed != 1) throw FacError(FAC_ERR_ARG, "precision must be 0 or 1");
      ctx->mixed = mixed;
   });
}

int fac_initialize(fac_ctx *ctx)
{
   return guarded([&] {
      check_state(ctx, false);
      initialize(ctx);
      ctx->ext_dirty = ctx->ext_levels > 0;
   });
}

int fac_field_size(fac_ctx *ctx, int fid, int problem, int ln, size_t *n)
{
   return guarded([&] {
      check_state(ctx, true);
      check_pl(ctx, problem, ln);
      field_ghost(fid);
      long long off;
      *n = field_slice(ctx, fid, problem, ln, off);
   });
}

int fac_side_size(fac_ctx *ctx, int problem, int ln, size_t *n)
{
   return guarded([&] {
      check_state(ctx, true);
      check_pl(ctx, problem, ln);
      const LevelState &L = ctx->L[ln];
      *n = (size_t)(L.prob_offs[problem + 1] - L.prob_offs[problem]);
   });
}

int fac_oside_size(fac_ctx *ctx, int problem, int ln, size_t *n)
{
   return guarded([&] {
      check_state(ctx, true);
      check_pl(ctx, problem, ln);
      const LevelState &L = ctx->L[ln];
      *n = (size_t)(L.prob_offo[problem + 1] - L.prob_offo[problem]);
   });
}

int fac_upload_field(fac_ctx *ctx, int fid, int problem, int ln, const double *host)
{
   return guarded([&] {
      check_ops(ctx);
      check_pl(ctx, problem, ln);
      if (!host) throw FacError(FAC_ERR_ARG, "null host pointer");
      if (fid == FAC_C && ctx->spec.c_kind != 2) throw FacError(FAC_ERR_ARG, "C is not variable");
      if (fid == FAC_C && ln == ctx->ext_levels) ctx->ext_dirty = true;
      long long off;
      const size_t n = field_slice(ctx, fid, problem, ln, off);
      CUDA_CHECK(cudaMemcpyAsync(field_ptr(ctx->L[ln], fid) + off, host, n * sizeof(double),
                                 cudaMemcpyHostToDevice, ctx->stream));
      CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
   });
}

int fac_download_field(fac_ctx *ctx, int fid, int problem, int ln, double *host)
{
   return guarded([&] {
      check_ops(ctx);
      check_pl(ctx, problem, ln);
      if (!host) throw FacError(FAC_ERR_ARG, "null host pointer");
      long long off;
      const size_t n = field_slice(ctx, fid, problem, ln, off);
      CUDA_CHECK(cudaMemcpyAsync(host, field_ptr(ctx->L[ln], fid) + off, n * sizeof(double),
                                 cudaMemcpyDeviceToHost, ctx->stream));
      CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
   });
}

int fac_upload_side(fac_ctx *ctx, int problem, int ln, const double *host)
{
   return guarded([&] {
      check_ops(ctx);
      check_pl(ctx, problem, ln);
      if (!ctx->spec.d_variable) throw FacError(FAC_ERR_ARG, "D is not variable");
      if (ln == ctx->ext_levels) ctx->ext_dirty = true;
      if (!host) throw FacError(FAC_ERR_ARG, "null host pointer");
      const LevelState &L = ctx->L[ln];
      const long long off = L.prob_offs[problem], n = L.prob_offs[problem + 1] - off;
      CUDA_CHECK(cudaMemcpyAsync(ctx->L[ln].d.p + off, host, n * sizeof(double),
                                 cudaMemcpyHostToDevice, ctx->stream));
      CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
   });
}

int fac_download_side(fac_ctx *ctx, int problem, int ln, double *host)
{
   return guarded([&] {
      check_ops(ctx);
      check_pl(ctx, problem, ln);
      if (!host) throw FacError(FAC_ERR_ARG, "null host pointer");
      const LevelState &L = ctx->L[ln];
      const long long off = L.prob_offs[problem], n = L.prob_offs[problem + 1] - off;
      CUDA_CHECK(cudaMemcpyAsync(host, ctx->L[ln].d.p + off, n * sizeof(double),
                                 cudaMemcpyDeviceToHost, ctx->stream));
      CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
   });
}

int fac_download_flux(fac_ctx *ctx, int problem, int ln, double *host)
{
   return guarded([&] {
      check_ops(ctx);
      check_pl(ctx, problem, ln);
      if (!host) throw FacError(FAC_ERR_ARG, "null host pointer");
      const LevelState &L = ctx->L[ln];
      const long long off = L.prob_offs[problem], n = L.prob_offs[problem + 1] - off;
      CUDA_CHECK(cudaMemcpyAsync(host, ctx->L[ln].flux.p + off, n * sizeof(double),
                                 cudaMemcpyDeviceToHost, ctx->stream));
      CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
   });
}

int fac_download_oside(fac_ctx *ctx, int problem, int ln, double *host)
{
   return guarded([&] {
      check_ops(ctx);
      check_pl(ctx, problem, ln);
      if (!host) throw FacError(FAC_ERR_ARG, "null host pointer");
      const LevelState &L = ctx->L[ln];
      const long long off = L.prob_offo[problem], n = L.prob_offo[problem + 1] - off;
      CUDA_CHECK(cudaMemcpyAsync(host, ctx->L[ln].oflux.p + off, n * sizeof(double),
                                 cudaMemcpyDeviceToHost, ctx->stream));
      CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
   });
}

int fac_fill_table(fac_ctx *ctx, int ln, int with_coarse, long long *dst, long long *src,
                   size_t cap, size_t *n)
{
   return guarded([&] {
      check_state(ctx, true);
      check_pl(ctx, 0, ln);
      if (!n) throw FacError(FAC_ERR_ARG, "null count");
      if (with_coarse && ln == 0) throw FacError(FAC_ERR_ARG, "level 0 has no coarser level");
      const FillGather &G = with_coarse ? ctx->L[ln].gather_wc : ctx->L[ln].gather_nc;
      if (!G.ok)
         throw FacError(FAC_ERR_STATE, "this level's fill has no element table (item fill)");
      *n = G.to.size();
      if (cap == 0) return;
      if (cap < G.to.size() || !dst || !src) throw FacError(FAC_ERR_ARG, "table too small");
      for (size_t q = 0; q < G.to.size(); ++q) {
         dst[q] = (long long)G.to[q];
         src[q] = (long long)G.from[q];
      }
   });
}

int fac_ghost_fill(fac_ctx *ctx, int fid, int ln, int with_coarse, int homogeneous)
{
   return guarded([&] {
      check_ops(ctx);
      check_pl(ctx, 0, ln);
      ghost_fill(ctx, fid, ln, with_coarse != 0, homogeneous ? 1 : 0, ctx->active.p);
      CUDA_CHECK(cudaGetLastError());
      CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
   });
}

int fac_smooth(fac_ctx *ctx, int fid_e, int fid_r, int ln, int nsweeps, double tol, int *sweeps)
{
   return guarded([&] {
      check_ops(ctx);
      check_pl(ctx, 0, ln);
      if (field_ghost(fid_e) != 1 || field_ghost(fid_r) != 0)
         throw FacError(FAC_ERR_ARG, "smooth needs a ghosted unknown and a ghost-0 rhs");
      smooth(ctx, fid_e, fid_r, ln, nsweeps, tol);
      if (sweeps) {
         std::vector<long long> s(nprob(ctx));
         CUDA_CHECK(cudaMemcpyAsync(s.data(), ctx->sweeps_call.p, s.size() * sizeof(long long),
                                    cudaMemcpyDeviceToHost, ctx->stream));
         CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
         for (size_t p = 0; p < s.size(); ++p) sweeps[p] = (int)s[p];
      }
      CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
   });
}

int fac_comp_residual(fac_ctx *ctx, int fid_r, int fid_u, int fid_f, int ln, int error_equation)
{
   return guarded([&] {
      check_ops(ctx);
      check_pl(ctx, 0, ln);
      if (field_ghost(fid_u) != 1 || field_ghost(fid_r) != 0 || field_ghost(fid_f) != 0)
         throw FacError(FAC_ERR_ARG, "bad field kinds for the residual");
      // this entry point leaves the face fluxes in the flux side data, as
      // the reference operator does; solves use the staged or fused kernels
      struct Restore {
         fac_ctx *c;
         int v, st;
         ~Restore()
         {
            c->fused_residual = v;
            c->staged = st;
         }
      } restore{ctx, ctx->fused_residual, ctx->staged};
      ctx->fused_residual = 0;
      ctx->staged = 0;
      comp_residual(ctx, fid_r, fid_u, fid_f, ln, error_equation ? 1 : 0);
      CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
   });
}

int fac_restrict(fac_ctx *ctx, int fid_src, int fid_dst, int dest_ln)
{
   return guarded([&] {
      check_ops(ctx);
      check_pl(ctx, 0, dest_ln);
      if (dest_ln + 1 >= ctx->nlev) throw FacError(FAC_ERR_ARG, "no finer level");
      restrict_op(ctx, fid_src, fid_dst, dest_ln);
      CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
   });
}

int fac_restrict_solution(fac_ctx *ctx, int fid, int dest_ln)
{
   return guarded([&] {
      check_ops(ctx);
      check_pl(ctx, 0, dest_ln);
      if (dest_ln + 1 >= ctx->nlev) throw FacError(FAC_ERR_ARG, "no finer level");
      restrict_solution(ctx, fid, dest_ln);
      CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
   });
}

int fac_prolong_correct(fac_ctx *ctx, int fid_src, int fid_dst, int dest_ln)
{
   return guarded([&] {
      check_ops(ctx);
      check_pl(ctx, 0, dest_ln);
      if (dest_ln < 1) throw FacError(FAC_ERR_ARG, "no coarser level");
      prolong_correct(ctx, fid_src, fid_dst, dest_ln);
      CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
   });
}

int fac_compute_weights(fac_ctx *ctx)
{
   return guarded([&] {
      check_ops(ctx);
      compute_weights_host(ctx);
      CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
   });
}

int fac_rms_norm(fac_ctx *ctx, int fid, double *norms)
{
   return guarded([&] {
      check_ops(ctx);
      if (!norms) throw FacError(FAC_ERR_ARG, "null output");
      std::vector<double> v;
      rms_norm(ctx, fid, v);
      for (size_t p = 0; p < v.size(); ++p) norms[p] = v[p];
   });
}

int fac_solve_coarsest(fac_ctx *ctx, int *sweeps)
{
   return guarded([&] {
      check_ops(ctx);
      solve_coarsest(ctx);
      if (sweeps) {
         std::vector<long long> s(nprob(ctx));
         CUDA_CHECK(cudaMemcpyAsync(s.data(), ctx->sweeps_call.p, s.size() * sizeof(long long),
                                    cudaMemcpyDeviceToHost, ctx->stream));
         CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
         for (size_t p = 0; p < s.size(); ++p) sweeps[p] = (int)s[p];
      }
      CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
   });
}

int fac_fac_cycle(fac_ctx *ctx)
{
   return guarded([&] {
      check_ops(ctx);
      fac_cycle_recursive(ctx, ctx->nlev - 1);
      CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
   });
}

int fac_solve(fac_ctx *ctx, int *converged, int *iterations, double *residual)
{
   return guarded([&] {
      check_ops(ctx);
      ensure_extension(ctx);
      solve(ctx, converged, iterations, residual);
   });
}

int fac_set_krylov(fac_ctx *ctx, int restart)
{
   return guarded([&] {
      if (!ctx) throw FacError(FAC_ERR_ARG, "null context");
      if (restart < 0 || restart > 64) throw FacError(FAC_ERR_ARG, "restart length must be 0..64");
      ctx->krylov = restart;
   });
}

int fac_solve_fgmres(fac_ctx *ctx, int restart, int *converged, int *iterations, double *residual)
{
   return guarded([&] {
      check_ops(ctx);
      ensure_extension(ctx);
      fgmres_solve(ctx, restart, converged, iterations, residual);
   });
}

int fac_solve_host(fac_ctx *ctx, const double *const *f_host, const double *const *u0_host,
                   double *const *u_host, int *converged, int *iterations, double *residual)
{
   return guarded([&] {
      check_ops(ctx);
      if (!f_host || !u_host) throw FacError(FAC_ERR_ARG, "null host array table");
      ensure_extension(ctx);
      const int np = nprob(ctx);
      // the tables hold the caller's levels; the added coarser ones keep
      // their zero f and start from a zero u
      const int lx = ctx->ext_levels, nl = ctx->nlev - lx;
      for (int ln = 0; ln < lx; ++ln)
         CUDA_CHECK(cudaMemsetAsync(ctx->L[ln].u.p, 0, ctx->L[ln].u.n * sizeof(double),
                                    ctx->stream));
      for (int p = 0; p < np; ++p)
         for (int ln = lx; ln < ctx->nlev; ++ln) {
            const int k = p * nl + ln - lx;
            long long off;
            size_t n = field_slice(ctx, FAC_F, p, ln, off);
            CUDA_CHECK(cudaMemcpyAsync(ctx->L[ln].f.p + off, f_host[k], n * sizeof(double),
                                       cudaMemcpyHostToDevice, ctx->stream));
            n = field_slice(ctx, FAC_U, p, ln, off);
            if (u0_host && u0_host[k])
               CUDA_CHECK(cudaMemcpyAsync(ctx->L[ln].u.p + off, u0_host[k], n * sizeof(double),
                                          cudaMemcpyHostToDevice, ctx->stream));
            else
               CUDA_CHECK(cudaMemsetAsync(ctx->L[ln].u.p + off, 0, n * sizeof(double),
                                          ctx->stream));
         }
      solve(ctx, converged, iterations, residual);
      for (int p = 0; p < np; ++p)
         for (int ln = lx; ln < ctx->nlev; ++ln) {
            const int k = p * nl + ln - lx;
            long long off;
            const size_t n = field_slice(ctx, FAC_U, p, ln, off);
            CUDA_CHECK(cudaMemcpyAsync(u_host[k], ctx->L[ln].u.p + off, n * sizeof(double),
                                       cudaMemcpyDeviceToHost, ctx->stream));
         }
      CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
   });
}

int fac_residual_history(fac_ctx *ctx, int problem, double *hist, int cap, int *n)
{
   return guarded([&] {
      check_state(ctx, true);
      check_pl(ctx, problem, 0);
      const auto &h = ctx->hist[problem];
      const int m = (int)std::min<size_t>(h.size(), (size_t)std::max(cap, 0));
      for (int t = 0; t < m; ++t) hist[t] = h[t];
      if (n) *n = (int)h.size();
   });
}

int fac_coarse_sweeps(fac_ctx *ctx, long long *sweeps)
{
   return guarded([&] {
      check_ops(ctx);
      CUDA_CHECK(cudaMemcpyAsync(sweeps, ctx->sweeps_coarse.p, nprob(ctx) * sizeof(long long),
                                 cudaMemcpyDeviceToHost, ctx->stream));
      CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
   });
}

int fac_reset_stats(fac_ctx *ctx)
{
   return guarded([&] {
      check_ops(ctx);
      CUDA_CHECK(cudaMemsetAsync(ctx->sweeps_coarse.p, 0, nprob(ctx) * sizeof(long long),
                                 ctx->stream));
      CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
   });
}

int fac_zero_field(fac_ctx *ctx, int fid)
{
   return guarded([&] {
      check_ops(ctx);
      zero_field(ctx, fid);
   });
}

int fac_trace_enable(fac_ctx *ctx, int on)
{
   return guarded([&] {
      check_ops(ctx);
      ctx->tracing = on != 0;
      ctx->trace.clear();
   });
}

int fac_trace_read(fac_ctx *ctx, char *buf, int cap, int *len)
{
   return guarded([&] {
      check_ops(ctx);
      std::string j = "{";
      bool first = true;
      for (const auto &kv : ctx->trace) {
         char tmp[256];
         std::snprintf(tmp, sizeof(tmp), "%s\"%s\": [%lld, %.6f]", first ? "" : ", ",
                       kv.first.c_str(), kv.second.first, kv.second.second);
         j += tmp;
         first = false;
      }
      j += "}";
      if (len) *len = (int)j.size();
      if (buf && cap > 0) {
         const int n = std::min<int>(cap - 1, (int)j.size());
         std::memcpy(buf, j.data(), n);
         buf[n] = 0;
      }
   });
}

int fac_kernel_launches(long long *n)
{
   return guarded([&] {
      if (!n) throw FacError(FAC_ERR_ARG, "null output");
      *n = kernel_launch_count();
   });
}

int fac_profile_enable(fac_ctx *ctx, int on)
{
   return guarded([&] {
      check_ops(ctx);
      CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
      ctx->profiling = on != 0;
      ctx->prof.clear();
      ctx->ev_next = 0;
      for (auto &a : ctx->graph_acc) a = fac_ctx::KindAcc();
   });
}

int fac_profile_read(fac_ctx *ctx, int kind, long long *launches, double *ms, double *bytes)
{
   return guarded([&] {
      check_ops(ctx);
      CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
      if (kind < 0 || kind > 5) throw FacError(FAC_ERR_ARG, "profile kind out of range");
      long long n = ctx->graph_acc[kind].n;
      double t = ctx->graph_acc[kind].ms, b = ctx->graph_acc[kind].bytes;
      for (const auto &r : ctx->prof) {
         if (r.kind != kind) continue;
         float e = 0.f;
         CUDA_CHECK(cudaEventElapsedTime(&e, r.a, r.b));
         ++n;
         t += e;
         b += r.bytes;
      }
      if (launches) *launches = n;
      if (ms) *ms = t;
      if (bytes) *bytes = b;
   });
}

int fac_profile_reset(fac_ctx *ctx)
{
   return guarded([&] {
      check_ops(ctx);
      CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
      ctx->prof.clear();
      ctx->ev_next = 0;
      for (auto &a : ctx->graph_acc) a = fac_ctx::KindAcc();
   });
}

int fac_timer(fac_ctx *ctx, int stop, double *ms)
{
   return guarded([&] {
      check_ops(ctx);
      if (!ctx->t0) {
         CUDA_CHECK(cudaEventCreate(&ctx->t0));
         CUDA_CHECK(cudaEventCreate(&ctx->t1));
      }
      if (!stop) {
         CUDA_CHECK(cudaEventRecord(ctx->t0, ctx->stream));
         return;
      }
      CUDA_CHECK(cudaEventRecord(ctx->t1, ctx->stream));
      CUDA_CHECK(cudaEventSynchronize(ctx->t1));
      float e = 0.f;
      CUDA_CHECK(cudaEventElapsedTime(&e, ctx->t0, ctx->t1));
      if (ms) *ms = e;
   });
}

int fac_synchronize(fac_ctx *ctx)
{
   return guarded([&] {
      if (!ctx) throw FacError(FAC_ERR_ARG, "null context");
      CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
   });
}

}  // extern "C"

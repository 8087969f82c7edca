/*
 * fac_ref_driver.C -- runs the reference's own FAC Poisson solver on one
 * problem read from a file and writes what it computed.
 *
 * TEST INFRASTRUCTURE ONLY: built by oracle/ref/build_ref.py against the
 * reference's headers and objects into oracle/_ref/, it produces the golden
 * fixtures that pin the oracle and the CUDA path.  It is modelled on the
 * reference's static-refinement test (source/test/FAC_staticrefinement/
 * FACPoisson.C:244-300): hierarchy -> variables -> CellPoissonFACSolver ->
 * initializeSolverState -> solveSystem.  The hierarchy is made from boxes
 * the way source/test/dataops/cell_hiertest.C:131-189 makes its one.
 *
 *    fac_ref_driver <in.bin> <out.bin>
 *
 * Built with WITH_B200_OPS (fac_dropin_driver), the same solver runs the
 * B200 library's operators through samrai_b200::B200CellPoissonFACOps in
 * place of CellPoissonFACOps: the drop-in, checked against the reference's
 * own results.
 *
 * File format (both directions): records of
 *    int32 name length, name bytes, int32 type (0 = f64, 1 = i32),
 *    int64 count, count values.
 * Input records: dim, nlev, n0[3], ratio[nlev*3], npatch[nlev],
 * boxes[npatch_total*6] (lo0 lo1 lo2 hi0 hi1 hi2 in the level's index space),
 * xlo[3], xup[3], poisson[4] (D variable, D constant, C kind, C constant),
 * bc[18] (a, b, g per location index 0..5; absent: Dirichlet through the
 * solver's setBoundaries, values from u0's ghost cells), bc_faces (present:
 * Robin coefficients varying along the boundary, FaceRobin), params[7] (max_cycles,
 * residual_tol, relative_residual_tol, pre sweeps, post sweeps, coarse
 * tolerance, coarse max iterations), and per level f<ln> (cells, ghost 0),
 * u0<ln> (ghost 1), d<ln> (side data, when D is variable), c<ln> (when C is
 * a field).  Arrays of a level are its patches' ghosted arrays in patch
 * order, each column-major (pdat::ArrayData layout); side data per patch,
 * axis 0..dim-1.
 * With a "skip_u" record the solution is not written back.
 * Output records: converged, iterations, residual, hist (composite residual
 * norm after each cycle), factors (average, final), seconds (wall time of
 * initializeSolverState and of solveSystem), u<ln> (ghost 1).
 */
#include "SAMRAI/SAMRAI_config.h"

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "SAMRAI/geom/CartesianGridGeometry.h"
#include "SAMRAI/hier/BoundaryBox.h"
#include "SAMRAI/hier/BoxLevel.h"
#include "SAMRAI/hier/PatchHierarchy.h"
#include "SAMRAI/hier/VariableDatabase.h"
#include "SAMRAI/pdat/ArrayData.h"
#include "SAMRAI/pdat/CellData.h"
#include "SAMRAI/pdat/CellVariable.h"
#include "SAMRAI/pdat/SideData.h"
#include "SAMRAI/pdat/SideVariable.h"
#include "SAMRAI/solv/CellPoissonFACOps.h"
#include "SAMRAI/solv/CellPoissonFACSolver.h"
#include "SAMRAI/solv/FACPreconditioner.h"
#include "SAMRAI/solv/RobinBcCoefStrategy.h"
#include "SAMRAI/tbox/InputManager.h"
#include "SAMRAI/tbox/MemoryDatabase.h"
#include "SAMRAI/tbox/SAMRAIManager.h"
#include "SAMRAI/tbox/SAMRAI_MPI.h"

#ifdef WITH_B200_OPS
// the drop-in: SAMRAI's solver running the B200 library's operators
#include "B200CellPoissonFACOps.h"
typedef samrai_b200::B200CellPoissonFACOps BaseOps;
#else
typedef SAMRAI::solv::CellPoissonFACOps BaseOps;
#endif

using namespace SAMRAI;

namespace {

struct Records {
   std::map<std::string, std::vector<double> > f64;
   std::map<std::string, std::vector<int> > i32;
};

Records read_records(const char *path)
{
   Records r;
   std::ifstream in(path, std::ios::binary);
   if (!in) throw std::runtime_error("cannot open input");
   while (true) {
      int32_t len;
      if (!in.read(reinterpret_cast<char *>(&len), 4)) break;
      std::string name(len, '\0');
      in.read(&name[0], len);
      int32_t type;
      int64_t n;
      in.read(reinterpret_cast<char *>(&type), 4);
      in.read(reinterpret_cast<char *>(&n), 8);
      if (type == 0) {
         std::vector<double> v(n);
         in.read(reinterpret_cast<char *>(v.data()), n * 8);
         r.f64[name] = v;
      } else {
         std::vector<int> v(n);
         in.read(reinterpret_cast<char *>(v.data()), n * 4);
         r.i32[name] = v;
      }
   }
   return r;
}

void write_record(std::ofstream &out, const std::string &name, const std::vector<double> &v)
{
   int32_t len = (int32_t)name.size(), type = 0;
   int64_t n = (int64_t)v.size();
   out.write(reinterpret_cast<const char *>(&len), 4);
   out.write(name.data(), len);
   out.write(reinterpret_cast<const char *>(&type), 4);
   out.write(reinterpret_cast<const char *>(&n), 8);
   out.write(reinterpret_cast<const char *>(v.data()), n * 8);
}

/*
 * Constant Robin coefficients a u + b du/dn = g per location index, filling
 * no tangential extensions, as the solver's default SimpleCellRobinBcCoefs
 * (SimpleCellRobinBcCoefs.C:483-486) does.
 */
class ConstantRobin : public solv::RobinBcCoefStrategy {
public:
   ConstantRobin(const tbox::Dimension &dim, const std::vector<double> &abg)
      : d_dim(dim), d_abg(abg) {}

   void setBcCoefs(const std::shared_ptr<pdat::ArrayData<double> > &acoef_data,
                   const std::shared_ptr<pdat::ArrayData<double> > &bcoef_data,
                   const std::shared_ptr<pdat::ArrayData<double> > &gcoef_data,
                   const std::shared_ptr<hier::Variable> &,
                   const hier::Patch &, const hier::BoundaryBox &bdry_box,
                   const double) const override
   {
      const int loc = bdry_box.getLocationIndex();
      if (acoef_data) acoef_data->fill(d_abg[loc]);
      if (bcoef_data) bcoef_data->fill(d_abg[6 + loc]);
      if (gcoef_data) gcoef_data->fill(d_abg[12 + loc]);
   }

   hier::IntVector numberOfExtensionsFillable() const override
   {
      return hier::IntVector::getZero(d_dim);
   }

private:
   const tbox::Dimension d_dim;
   std::vector<double> d_abg;
};

/*
 * Robin coefficients varying along the boundary: a polynomial of the face
 * centre's tangential coordinates (t = sum of x = xlo + (i + 1/2) dx over
 * the tangential axes, dx of the patch's level), a = 1 + t/4, b = 1/2 + t/8,
 * g = t/10 - 1/20 + location/100, written per face into the arrays the
 * helper asks for, without tangential extensions.
 */
class FaceRobin : public solv::RobinBcCoefStrategy {
public:
   FaceRobin(const tbox::Dimension &dim, const std::vector<double> &xlo,
             const std::vector<double> &xup, const std::vector<int> &n0)
      : d_dim(dim), d_xlo(xlo), d_xup(xup), d_n0(n0) {}

   void setBcCoefs(const std::shared_ptr<pdat::ArrayData<double> > &acoef_data,
                   const std::shared_ptr<pdat::ArrayData<double> > &bcoef_data,
                   const std::shared_ptr<pdat::ArrayData<double> > &gcoef_data,
                   const std::shared_ptr<hier::Variable> &, const hier::Patch &patch,
                   const hier::BoundaryBox &bdry_box, const double) const override
   {
      const int dim = d_dim.getValue();
      const int loc = bdry_box.getLocationIndex();
      const int normal = loc / 2;
      const hier::IntVector &ratio = patch.getPatchGeometry()->getRatio();
      double dx[3] = {1, 1, 1};
      for (int a = 0; a < dim; ++a)
         dx[a] = ((d_xup[a] - d_xlo[a]) / (double)d_n0[a]) / (double)ratio(a);
      const std::shared_ptr<pdat::ArrayData<double> > arrs[3] = {acoef_data, bcoef_data,
                                                                  gcoef_data};
      for (int q = 0; q < 3; ++q) {
         if (!arrs[q]) continue;
         const hier::Box &box = arrs[q]->getBox();
         for (hier::Box::iterator bi(box.begin()); bi != box.end(); ++bi) {
            const hier::Index &idx = *bi;
            double t = 0.0;
            for (int a = 0; a < dim; ++a)
               if (a != normal) t = t + (d_xlo[a] + ((double)idx(a) + 0.5) * dx[a]);
            const double v = q == 0 ? 1.0 + 0.25 * t
                                    : (q == 1 ? 0.5 + 0.125 * t : 0.1 * t - 0.05 + 0.01 * loc);
            (*arrs[q])(idx, 0) = v;
         }
      }
   }

   hier::IntVector numberOfExtensionsFillable() const override
   {
      return hier::IntVector::getZero(d_dim);
   }

private:
   const tbox::Dimension d_dim;
   std::vector<double> d_xlo, d_xup;
   std::vector<int> d_n0;
};

/*
 * CellPoissonFACOps that records the composite residual norm after every
 * cycle: FACPreconditioner::solveSystem calls postprocessOneCycle after it
 * has stored the new norm (FACPreconditioner.C:425-436).
 */
class RecordingOps : public BaseOps {
public:
   RecordingOps(const tbox::Dimension &dim, const std::string &name,
                const std::shared_ptr<tbox::Database> &db)
      : BaseOps(dim, name, db) {}

   void setRecordingPreconditioner(const solv::FACPreconditioner *p) { d_pre = p; }

   void postprocessOneCycle(int it, const solv::SAMRAIVectorReal<double> &u,
                            const solv::SAMRAIVectorReal<double> &r) override
   {
      BaseOps::postprocessOneCycle(it, u, r);
      hist.push_back(d_pre->getResidualNorm());
   }

   std::vector<double> hist;

private:
   const solv::FACPreconditioner *d_pre = nullptr;
};

/* Copy between a level's canonical array and its patches' data. */
template <class F>
void for_patches(const std::shared_ptr<hier::PatchLevel> &level, F f)
{
   // patches in LocalId order, as the boxes were given
   std::vector<std::shared_ptr<hier::Patch> > patches(level->getLocalNumberOfPatches());
   for (hier::PatchLevel::iterator ip(level->begin()); ip != level->end(); ++ip) {
      const int id = (*ip)->getBox().getLocalId().getValue();
      patches.at(id) = *ip;
   }
   for (auto &p : patches) f(*p);
}

std::vector<double> &need(Records &r, const std::string &n)
{
   auto it = r.f64.find(n);
   if (it == r.f64.end()) throw std::runtime_error("missing record " + n);
   return it->second;
}

std::vector<int> &needi(Records &r, const std::string &n)
{
   auto it = r.i32.find(n);
   if (it == r.i32.end()) throw std::runtime_error("missing record " + n);
   return it->second;
}

void load_cell(const std::shared_ptr<hier::PatchLevel> &level, int id, const std::vector<double> &v)
{
   size_t off = 0;
   for_patches(level, [&](hier::Patch &p) {
      auto d = SAMRAI_SHARED_PTR_CAST<pdat::CellData<double>, hier::PatchData>(p.getPatchData(id));
      const size_t n = d->getGhostBox().size();
      if (off + n > v.size()) throw std::runtime_error("cell array too short");
      std::memcpy(d->getPointer(), v.data() + off, n * 8);
      off += n;
   });
   if (off != v.size()) throw std::runtime_error("cell array size mismatch");
}

std::vector<double> save_cell(const std::shared_ptr<hier::PatchLevel> &level, int id)
{
   std::vector<double> v;
   for_patches(level, [&](hier::Patch &p) {
      auto d = SAMRAI_SHARED_PTR_CAST<pdat::CellData<double>, hier::PatchData>(p.getPatchData(id));
      const size_t n = d->getGhostBox().size();
      v.insert(v.end(), d->getPointer(), d->getPointer() + n);
   });
   return v;
}

void load_side(const std::shared_ptr<hier::PatchLevel> &level, int id, int dim,
               const std::vector<double> &v)
{
   size_t off = 0;
   for_patches(level, [&](hier::Patch &p) {
      auto d = SAMRAI_SHARED_PTR_CAST<pdat::SideData<double>, hier::PatchData>(p.getPatchData(id));
      for (int a = 0; a < dim; ++a) {
         const size_t n = d->getArrayData(a).getBox().size();
         if (off + n > v.size()) throw std::runtime_error("side array too short");
         std::memcpy(d->getPointer(a), v.data() + off, n * 8);
         off += n;
      }
   });
   if (off != v.size()) throw std::runtime_error("side array size mismatch");
}

#ifdef DRIVER_TRACE
#define TRACE(x) std::fprintf(stderr, "trace: %s\n", x)
#else
#define TRACE(x)
#endif

/*
 * Cache the overlap Connectors between each level and itself and between
 * each level and the next coarser one, with the widths the hierarchy
 * requires, as the reference's gridding does when it makes a level
 * (mesh/GriddingAlgorithm.C:1719-1731) and its communication tester does
 * (source/test/communication/CommTester.C:270-282): refine schedules with a
 * coarser level and no source level rely on them.
 */
void cache_connectors(const std::shared_ptr<hier::PatchHierarchy> &h)
{
   for (int ln = 0; ln < h->getNumberOfLevels(); ++ln) {
      h->getPatchLevel(ln)->findConnector(*h->getPatchLevel(ln),
                                          h->getRequiredConnectorWidth(ln, ln, true),
                                          hier::CONNECTOR_CREATE, false);
      if (ln > 0)
         h->getPatchLevel(ln)->findConnectorWithTranspose(
            *h->getPatchLevel(ln - 1), h->getRequiredConnectorWidth(ln, ln - 1, true),
            h->getRequiredConnectorWidth(ln - 1, ln), hier::CONNECTOR_CREATE, false);
   }
}

int run(Records &in, const char *out_path)
{
   const int d = needi(in, "dim")[0];
   const int nlev = needi(in, "nlev")[0];
   const tbox::Dimension dim(static_cast<unsigned short>(d));
   const std::vector<int> &n0 = needi(in, "n0");
   const std::vector<int> &ratio = needi(in, "ratio");
   const std::vector<int> &npatch = needi(in, "npatch");
   const std::vector<int> &boxes = needi(in, "boxes");
   const std::vector<double> &xlo = need(in, "xlo"), &xup = need(in, "xup");
   const std::vector<double> &poisson = need(in, "poisson");
   // no "bc" record: the solver's own Dirichlet path (setBoundaries
   // "Dirichlet", boundary values taken from u's ghost cells and restored
   // after the solve, CellPoissonFACSolver.C:342-349)
   const bool robin_bc = in.f64.count("bc") != 0;
   const std::vector<double> bc = robin_bc ? need(in, "bc") : std::vector<double>(18, 0.0);
   const std::vector<double> &prm = need(in, "params");
   const bool dvar = poisson[0] != 0.0;
   const int ckind = (int)poisson[2];

   // Every variable first -- the driver's, then the solver's and the FAC
   // operators' internal ones, which their constructors register -- since
   // the grid geometry fixes the largest ghost width when the first level
   // is made (hier/BaseGridGeometry.C:520-530).  The reference's drivers
   // construct their solver before gridding for the same reason.
   hier::VariableDatabase *vdb = hier::VariableDatabase::getDatabase();
   std::shared_ptr<hier::VariableContext> ctx(vdb->getContext("driver"));
   std::shared_ptr<pdat::CellVariable<double> > u_var(new pdat::CellVariable<double>(dim, "u"));
   std::shared_ptr<pdat::CellVariable<double> > f_var(new pdat::CellVariable<double>(dim, "f"));
   std::shared_ptr<pdat::CellVariable<double> > c_var(new pdat::CellVariable<double>(dim, "c"));
   std::shared_ptr<pdat::SideVariable<double> > d_var(
      new pdat::SideVariable<double>(dim, "D", hier::IntVector::getOne(dim)));
   const int u_id = vdb->registerVariableAndContext(u_var, ctx, hier::IntVector(dim, 1));
   const int f_id = vdb->registerVariableAndContext(f_var, ctx, hier::IntVector(dim, 0));
   const int c_id = vdb->registerVariableAndContext(c_var, ctx, hier::IntVector(dim, 0));
   const int d_id = vdb->registerVariableAndContext(d_var, ctx, hier::IntVector(dim, 0));

   std::shared_ptr<tbox::MemoryDatabase> ops_db(new tbox::MemoryDatabase("fac_ops"));
   ops_db->putString("prolongation_method", "LINEAR_REFINE");
   ops_db->putString("cf_discretization", "Ewing");
   ops_db->putString("coarse_solver_choice", "redblack");
   ops_db->putDouble("coarse_solver_tolerance", prm[5]);
   ops_db->putInteger("coarse_solver_max_iterations", (int)prm[6]);
   std::shared_ptr<tbox::MemoryDatabase> pre_db(new tbox::MemoryDatabase("fac_precond"));
   pre_db->putInteger("max_cycles", (int)prm[0]);
   pre_db->putDouble("residual_tol", prm[1]);
   pre_db->putDouble("relative_residual_tol", prm[2]);
   pre_db->putInteger("num_pre_sweeps", (int)prm[3]);
   pre_db->putInteger("num_post_sweeps", (int)prm[4]);
   std::shared_ptr<RecordingOps> ops(new RecordingOps(dim, "fac_ops", ops_db));
   std::shared_ptr<solv::FACPreconditioner> pre(
      new solv::FACPreconditioner("fac_precond", ops, pre_db));
   ops->setRecordingPreconditioner(pre.get());
   ConstantRobin robin(dim, bc);
   FaceRobin face_robin(dim, xlo, xup, n0);
   const bool face_bc = in.i32.count("bc_faces") != 0;
   solv::CellPoissonFACSolver solver(dim, "solver", pre, ops);
   TRACE("solver made");

   hier::Index lo(dim, 0), hi(dim, 0);
   for (int a = 0; a < d; ++a) hi(a) = n0[a] - 1;
   hier::BoxContainer domain;
   domain.pushBack(hier::Box(lo, hi, hier::BlockId(0)));
   std::shared_ptr<geom::CartesianGridGeometry> geometry(
      new geom::CartesianGridGeometry("CartesianGeometry", xlo.data(), xup.data(), domain));
   std::shared_ptr<hier::PatchHierarchy> hierarchy(
      new hier::PatchHierarchy("PatchHierarchy", geometry));
   hierarchy->setMaxNumberOfLevels(nlev);
   hier::IntVector to_zero(dim, 1);
   int b0 = 0;
   for (int ln = 0; ln < nlev; ++ln) {
      hier::IntVector r(dim, 1);
      for (int a = 0; a < d; ++a) r(a) = ratio[3 * ln + a];
      if (ln > 0) {
         hierarchy->setRatioToCoarserLevel(r, ln);
         to_zero *= r;
      }
      std::shared_ptr<hier::BoxLevel> layer(std::make_shared<hier::BoxLevel>(to_zero, geometry));
      for (int ib = 0; ib < npatch[ln]; ++ib, ++b0) {
         hier::Index blo(dim, 0), bhi(dim, 0);
         for (int a = 0; a < d; ++a) {
            blo(a) = boxes[6 * b0 + a];
            bhi(a) = boxes[6 * b0 + 3 + a];
         }
         layer->addBox(hier::Box(hier::Box(blo, bhi, hier::BlockId(0)), hier::LocalId(ib), 0));
      }
      hierarchy->makeNewPatchLevel(ln, layer);
   }
   cache_connectors(hierarchy);
   TRACE("hierarchy built");

   for (int ln = 0; ln < nlev; ++ln) {
      std::shared_ptr<hier::PatchLevel> level(hierarchy->getPatchLevel(ln));
      level->allocatePatchData(u_id);
      level->allocatePatchData(f_id);
      load_cell(level, u_id, need(in, "u0" + std::to_string(ln)));
      load_cell(level, f_id, need(in, "f" + std::to_string(ln)));
      if (dvar) {
         level->allocatePatchData(d_id);
         load_side(level, d_id, d, need(in, "d" + std::to_string(ln)));
      }
      if (ckind == 2) {
         level->allocatePatchData(c_id);
         load_cell(level, c_id, need(in, "c" + std::to_string(ln)));
      }
   }
   TRACE("data loaded");

   if (dvar) solver.setDPatchDataId(d_id);
   else solver.setDConstant(poisson[1]);
   if (ckind == 2) solver.setCPatchDataId(c_id);
   else solver.setCConstant(ckind == 1 ? poisson[3] : 0.0);
   if (face_bc) solver.setBcObject(&face_robin);
   else if (robin_bc) solver.setBcObject(&robin);
   else solver.setBoundaries("Dirichlet");
   using clock = std::chrono::steady_clock;
   const clock::time_point t0 = clock::now();
   solver.initializeSolverState(u_id, f_id, hierarchy, 0, nlev - 1);
   TRACE("state initialized");
   const clock::time_point t1 = clock::now();
   const int converged = solver.solveSystem(u_id, f_id) ? 1 : 0;
   const clock::time_point t2 = clock::now();
   TRACE("solved");
   double avg = 0.0, fin = 0.0;
   solver.getConvergenceFactors(avg, fin);
   std::ofstream out(out_path, std::ios::binary);
   write_record(out, "converged", {(double)converged});
   write_record(out, "iterations", {(double)solver.getNumberOfIterations()});
   write_record(out, "residual", {solver.getResidualNorm()});
   write_record(out, "factors", {avg, fin});
   write_record(out, "hist", ops->hist);
   write_record(out, "seconds", {std::chrono::duration<double>(t1 - t0).count(),
                                 std::chrono::duration<double>(t2 - t1).count()});
   if (!in.i32.count("skip_u"))
      for (int ln = 0; ln < nlev; ++ln)
         write_record(out, "u" + std::to_string(ln),
                      save_cell(hierarchy->getPatchLevel(ln), u_id));
   solver.deallocateSolverState();
   return 0;
}

}  // namespace

#ifdef DRIVER_TRACE
#include <csignal>
#include <execinfo.h>
#include <unistd.h>
static void on_segv(int)
{
   void *frames[64];
   const int n = backtrace(frames, 64);
   backtrace_symbols_fd(frames, n, 2);
   _exit(3);
}
#endif

int main(int argc, char **argv)
{
#ifdef DRIVER_TRACE
   std::signal(SIGSEGV, on_segv);
#endif
   if (argc != 3) {
      std::fprintf(stderr, "usage: %s in.bin out.bin\n", argv[0]);
      return 2;
   }
   tbox::SAMRAI_MPI::init(&argc, &argv);
   tbox::SAMRAIManager::initialize();
   tbox::SAMRAIManager::startup();
   int rc = 0;
   try {
      Records in = read_records(argv[1]);
      rc = run(in, argv[2]);
   } catch (const std::exception &e) {
      std::fprintf(stderr, "fac_ref_driver: %s\n", e.what());
      rc = 1;
   }
   tbox::SAMRAIManager::shutdown();
   tbox::SAMRAIManager::finalize();
   tbox::SAMRAI_MPI::finalize();
   return rc;
}

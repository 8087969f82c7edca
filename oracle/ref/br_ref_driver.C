/*
 * br_ref_driver.C -- the reference's own tagging and Berger-Rigoutsos
 * clustering on one level read from a file, with what they computed written
 * back.
 *
 * TEST INFRASTRUCTURE ONLY: built by oracle/ref/build_ref.py against the
 * reference's headers and objects (mesh package and the FAC_adaptive test's
 * AdaptivePoisson) into oracle/_ref/; it produces the golden fixtures of the
 * regrid step.  The steps are those of an adaptive FAC run before gridding
 * (source/test/FAC_adaptive/AdaptivePoisson.C:464-533, applyGradientDetector:
 * tag = computeAdaptionEstimate(u) > adaption_threshold) and of the
 * GriddingAlgorithm's box generator (mesh/BergerRigoutsos.C:251-420,
 * findBoxesContainingTags on the tag level within bound boxes).
 *
 *    br_ref_driver <in.bin> <out.bin>
 *
 * Records as in fac_ref_driver.C.  Input: dim, n0[3] (the tag level is
 * level 0 of a hierarchy over the box [0, n0)), boxes[npatch*6] (lo, hi),
 * xlo[3], xup[3], u (ghost-1 arrays of the patches in order, column-major),
 * threshold, bound[nbound*6], min_box[3], max_box[3] (0: unlimited),
 * efficiency, combine.  Output: tags (ghost-0 arrays of the patches, 0/1),
 * boxes[nbox*6] (the new BoxLevel's boxes in its order), seconds (wall time
 * of the tagging and of the clustering).
 */
#include "SAMRAI/SAMRAI_config.h"

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "AdaptivePoisson.h"
#include "SAMRAI/geom/CartesianGridGeometry.h"
#include "SAMRAI/hier/BoxLevel.h"
#include "SAMRAI/hier/Connector.h"
#include "SAMRAI/hier/PatchHierarchy.h"
#include "SAMRAI/hier/VariableDatabase.h"
#include "SAMRAI/mesh/BergerRigoutsos.h"
#include "SAMRAI/pdat/CellData.h"
#include "SAMRAI/pdat/CellVariable.h"
#include "SAMRAI/solv/CellPoissonFACOps.h"
#include "SAMRAI/solv/FACPreconditioner.h"
#include "SAMRAI/tbox/MemoryDatabase.h"
#include "SAMRAI/tbox/SAMRAIManager.h"
#include "SAMRAI/tbox/SAMRAI_MPI.h"

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

template <class T>
void write_record(std::ofstream &out, const std::string &name, const std::vector<T> &v)
{
   int32_t len = (int32_t)name.size(), type = sizeof(T) == 8 ? 0 : 1;
   int64_t n = (int64_t)v.size();
   out.write(reinterpret_cast<const char *>(&len), 4);
   out.write(name.data(), len);
   out.write(reinterpret_cast<const char *>(&type), 4);
   out.write(reinterpret_cast<const char *>(&n), 8);
   out.write(reinterpret_cast<const char *>(v.data()), n * sizeof(T));
}

const std::vector<double> &need(const Records &r, const std::string &k)
{
   auto it = r.f64.find(k);
   if (it == r.f64.end()) throw std::runtime_error("missing record " + k);
   return it->second;
}

const std::vector<int> &needi(const Records &r, const std::string &k)
{
   auto it = r.i32.find(k);
   if (it == r.i32.end()) throw std::runtime_error("missing record " + k);
   return it->second;
}

int run(const Records &in, const char *out_path)
{
   const int d = needi(in, "dim")[0];
   const tbox::Dimension dim(static_cast<unsigned short>(d));
   const std::vector<int> &n0 = needi(in, "n0");
   const std::vector<int> &boxes = needi(in, "boxes");
   const std::vector<double> &xlo = need(in, "xlo"), &xup = need(in, "xup");
   const std::vector<double> &u = need(in, "u");
   const double threshold = need(in, "threshold")[0];
   const std::vector<int> &bound = needi(in, "bound");
   const std::vector<int> &min_box = needi(in, "min_box");
   const std::vector<int> &max_box = needi(in, "max_box");
   const double efficiency = need(in, "efficiency")[0];
   const double combine = need(in, "combine")[0];

   hier::VariableDatabase *vdb = hier::VariableDatabase::getDatabase();
   std::shared_ptr<hier::VariableContext> ctx = vdb->getContext("br_driver");
   std::shared_ptr<pdat::CellVariable<double> > u_var(
      new pdat::CellVariable<double>(dim, "br_driver:u"));
   std::shared_ptr<pdat::CellVariable<int> > tag_var(
      new pdat::CellVariable<int>(dim, "br_driver:tag"));
   const int u_id = vdb->registerVariableAndContext(u_var, ctx, hier::IntVector(dim, 1));
   const int tag_id = vdb->registerVariableAndContext(tag_var, ctx, hier::IntVector(dim, 0));

   // the test problem's own object, for its adaption estimate
   std::shared_ptr<tbox::MemoryDatabase> ops_db(new tbox::MemoryDatabase("ops"));
   std::shared_ptr<solv::CellPoissonFACOps> ops(new solv::CellPoissonFACOps(dim, "ops", ops_db));
   std::shared_ptr<tbox::MemoryDatabase> pre_db(new tbox::MemoryDatabase("pre"));
   std::shared_ptr<solv::FACPreconditioner> pre(new solv::FACPreconditioner("pre", ops, pre_db));
   tbox::MemoryDatabase ap_db("ap");
   AdaptivePoisson ap("ap", dim, ops, pre, ap_db);

   hier::Index lo(dim, 0), hi(dim, 0);
   for (int a = 0; a < d; ++a) hi(a) = n0[a] - 1;
   hier::BoxContainer domain;
   domain.pushBack(hier::Box(lo, hi, hier::BlockId(0)));
   std::shared_ptr<geom::CartesianGridGeometry> geometry(
      new geom::CartesianGridGeometry("CartesianGeometry", xlo.data(), xup.data(), domain));
   std::shared_ptr<hier::PatchHierarchy> hierarchy(
      new hier::PatchHierarchy("PatchHierarchy", geometry));
   hierarchy->setMaxNumberOfLevels(1);
   std::shared_ptr<hier::BoxLevel> layer(
      std::make_shared<hier::BoxLevel>(hier::IntVector(dim, 1), geometry));
   const int npatch = (int)boxes.size() / 6;
   for (int ib = 0; ib < npatch; ++ib) {
      hier::Index blo(dim, 0), bhi(dim, 0);
      for (int a = 0; a < d; ++a) {
         blo(a) = boxes[6 * ib + a];
         bhi(a) = boxes[6 * ib + 3 + a];
      }
      layer->addBox(hier::Box(hier::Box(blo, bhi, hier::BlockId(0)), hier::LocalId(ib), 0));
   }
   hierarchy->makeNewPatchLevel(0, layer);
   std::shared_ptr<hier::PatchLevel> level(hierarchy->getPatchLevel(0));
   level->findConnector(*level, hierarchy->getRequiredConnectorWidth(0, 0, true),
                        hier::CONNECTOR_CREATE, false);
   level->allocatePatchData(u_id);
   level->allocatePatchData(tag_id);

   // u from the file, patch by patch in LocalId order
   size_t off = 0;
   for (int ib = 0; ib < npatch; ++ib) {
      std::shared_ptr<hier::Patch> patch(level->getPatch(hier::GlobalId(hier::LocalId(ib), 0)));
      std::shared_ptr<pdat::CellData<double> > ud(
         SAMRAI_SHARED_PTR_CAST<pdat::CellData<double>, hier::PatchData>(
            patch->getPatchData(u_id)));
      pdat::ArrayData<double> &arr = ud->getArrayData();
      const size_t n = arr.getBox().size();
      if (off + n > u.size()) throw std::runtime_error("u record too short");
      std::copy(u.begin() + off, u.begin() + off + n, arr.getPointer());
      off += n;
   }

   using clock = std::chrono::steady_clock;
   const clock::time_point t0 = clock::now();
   // AdaptivePoisson::applyGradientDetector: tags where the estimate
   // exceeds the threshold
   std::vector<int> tags_out;
   for (int ib = 0; ib < npatch; ++ib) {
      std::shared_ptr<hier::Patch> patch(level->getPatch(hier::GlobalId(hier::LocalId(ib), 0)));
      std::shared_ptr<pdat::CellData<double> > ud(
         SAMRAI_SHARED_PTR_CAST<pdat::CellData<double>, hier::PatchData>(
            patch->getPatchData(u_id)));
      std::shared_ptr<pdat::CellData<int> > td(
         SAMRAI_SHARED_PTR_CAST<pdat::CellData<int>, hier::PatchData>(
            patch->getPatchData(tag_id)));
      pdat::CellData<double> estimate(patch->getBox(), 1, hier::IntVector(dim, 0));
      ap.computeAdaptionEstimate(estimate, *ud);
      td->fill(0);
      hier::Box::iterator iend(patch->getBox().end());
      for (hier::Box::iterator i(patch->getBox().begin()); i != iend; ++i) {
         const pdat::CellIndex ci(*i);
         if (estimate(ci) > threshold) (*td)(ci) = 1;
      }
      const int *tp = td->getArrayData().getPointer();
      tags_out.insert(tags_out.end(), tp, tp + td->getArrayData().getBox().size());
   }
   const clock::time_point t1 = clock::now();

   std::shared_ptr<tbox::MemoryDatabase> br_db(new tbox::MemoryDatabase("br"));
   br_db->putDoubleVector("efficiency_tolerance", std::vector<double>(1, efficiency));
   br_db->putDoubleVector("combine_efficiency", std::vector<double>(1, combine));
   bool limited = false;
   for (int a = 0; a < d; ++a) limited = limited || max_box[a] > 0;
   if (limited) {
      std::vector<int> mb(d);
      for (int a = 0; a < d; ++a) mb[a] = max_box[a] > 0 ? max_box[a] : tbox::MathUtilities<int>::getMax();
      br_db->putIntegerVector("max_box_size", mb);
   }
   mesh::BergerRigoutsos br(dim, br_db);
   hier::BoxContainer bound_boxes;
   for (size_t ib = 0; ib < bound.size() / 6; ++ib) {
      hier::Index blo(dim, 0), bhi(dim, 0);
      for (int a = 0; a < d; ++a) {
         blo(a) = bound[6 * ib + a];
         bhi(a) = bound[6 * ib + 3 + a];
      }
      bound_boxes.pushBack(hier::Box(blo, bhi, hier::BlockId(0)));
   }
   hier::IntVector minb(dim, 1);
   for (int a = 0; a < d; ++a) minb(a) = min_box[a];
   std::shared_ptr<hier::BoxLevel> new_level;
   std::shared_ptr<hier::Connector> tag_to_new;
   br.findBoxesContainingTags(new_level, tag_to_new, level, tag_id, 1, bound_boxes, minb,
                              hier::IntVector(dim, 0));
   const clock::time_point t2 = clock::now();

   std::vector<int> out_boxes;
   const hier::BoxContainer &nb = new_level->getBoxes();
   for (hier::BoxContainer::const_iterator bi = nb.begin(); bi != nb.end(); ++bi) {
      for (int a = 0; a < 3; ++a) out_boxes.push_back(a < d ? bi->lower(a) : 0);
      for (int a = 0; a < 3; ++a) out_boxes.push_back(a < d ? bi->upper(a) : 0);
   }
   std::ofstream out(out_path, std::ios::binary);
   write_record(out, "tags", tags_out);
   write_record(out, "boxes", out_boxes);
   write_record(out, "seconds", std::vector<double>{std::chrono::duration<double>(t1 - t0).count(),
                                                    std::chrono::duration<double>(t2 - t1).count()});
   return 0;
}

}  // namespace

int main(int argc, char **argv)
{
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
      std::fprintf(stderr, "br_ref_driver: %s\n", e.what());
      rc = 1;
   }
   tbox::SAMRAIManager::shutdown();
   tbox::SAMRAIManager::finalize();
   tbox::SAMRAI_MPI::finalize();
   return rc;
}

/*
 * B200CellPoissonFACOps: see B200CellPoissonFACOps.h.
 *
 * Each FACOperatorStrategy operation maps onto one C-ABI operation of the
 * library, on the device fields of its context (U and E with one ghost
 * cell, F, R and TR without): the vectors the operation reads are copied
 * level by level from their patch data into the field chosen for them, the
 * operation runs, and the vector it writes is copied back, ghost cells
 * included.  State the reference keeps inside its operators between calls
 * (the fine fluxes saved for the coarser level's composite residual, the
 * control-volume weights) stays in the device context the same way.
 */
#include "B200CellPoissonFACOps.h"

#include <array>
#include <cmath>
#include <cstring>
#include <map>

#include "SAMRAI/geom/CartesianGridGeometry.h"
#include "SAMRAI/geom/CartesianPatchGeometry.h"
#include "SAMRAI/hier/BoundaryBox.h"
#include "SAMRAI/hier/PatchLevel.h"
#include "SAMRAI/pdat/ArrayData.h"
#include "SAMRAI/pdat/CellData.h"
#include "SAMRAI/pdat/SideData.h"
#include "SAMRAI/solv/PoissonSpecifications.h"
#include "SAMRAI/solv/RobinBcCoefStrategy.h"
#include "SAMRAI/tbox/Utilities.h"

#include "samrai_fac_b200.h"

using namespace SAMRAI;

namespace {

// CellPoissonFACOps keeps what its public setters receive (the Poisson
// specification, the boundary object, the coarse-solver settings and the
// input keys) in private members without getters.  The derived operators
// read them there through explicit template instantiation, which the
// language exempts from access checking, so the caller's calls on the base
// class reach the GPU operators unchanged.
template <class Tag, typename Tag::type M>
struct Grant {
   friend typename Tag::type member(Tag) { return M; }
};

#define B200_BASE_MEMBER(TAG, TYPE, NAME)                                    \
   struct TAG {                                                              \
      typedef TYPE solv::CellPoissonFACOps::*type;                          \
      friend type member(TAG);                                               \
   };                                                                        \
   template struct Grant<TAG, &solv::CellPoissonFACOps::NAME>;

B200_BASE_MEMBER(SpecTag, solv::PoissonSpecifications, d_poisson_spec)
B200_BASE_MEMBER(BcTag, const solv::RobinBcCoefStrategy *, d_physical_bc_coef)
B200_BASE_MEMBER(CoarseChoiceTag, std::string, d_coarse_solver_choice)
B200_BASE_MEMBER(CfTag, std::string, d_cf_discretization)
B200_BASE_MEMBER(ProlongTag, std::string, d_prolongation_method)
B200_BASE_MEMBER(CoarseTolTag, double, d_coarse_solver_tolerance)
B200_BASE_MEMBER(CoarseMaxTag, int, d_coarse_solver_max_iterations)
#undef B200_BASE_MEMBER

// Ghost width of each device field (include/samrai_fac_b200.h).
int field_ghost(int fid) { return (fid == FAC_U || fid == FAC_E) ? 1 : 0; }

}  // namespace

namespace samrai_b200 {

B200CellPoissonFACOps::B200CellPoissonFACOps(const tbox::Dimension &dim,
                                             const std::string &object_name,
                                             const std::shared_ptr<tbox::Database> &input_db,
                                             int device)
   : solv::CellPoissonFACOps(dim, object_name, input_db), d_b200_dim(dim), d_device(device)
{
}

B200CellPoissonFACOps::~B200CellPoissonFACOps() { deallocateOperatorState(); }

void B200CellPoissonFACOps::check(int rc, const char *what) const
{
   if (rc != FAC_OK) TBOX_ERROR("B200CellPoissonFACOps: " << what << ": " << fac_last_error());
}

void B200CellPoissonFACOps::initializeOperatorState(
   const solv::SAMRAIVectorReal<double> &solution, const solv::SAMRAIVectorReal<double> &rhs)
{
   NULL_USE(rhs);
   deallocateOperatorState();
   const int dim = d_b200_dim.getValue();
   const std::string &choice = this->*member(CoarseChoiceTag());
   const std::string &cf = this->*member(CfTag());
   const std::string &prolong = this->*member(ProlongTag());
   if (choice != "redblack")
      TBOX_ERROR("B200CellPoissonFACOps: coarse_solver_choice must be redblack");
   if (cf != "Ewing") TBOX_ERROR("B200CellPoissonFACOps: cf_discretization must be Ewing");
   if (prolong != "LINEAR_REFINE")
      TBOX_ERROR("B200CellPoissonFACOps: prolongation_method must be LINEAR_REFINE");
   if (solution.getCoarsestLevelNumber() != 0)
      TBOX_ERROR("B200CellPoissonFACOps: the levels must start at level 0");

   d_hier = solution.getPatchHierarchy();
   const int nlev = solution.getFinestLevelNumber() + 1;
   std::shared_ptr<geom::CartesianGridGeometry> geom(
      SAMRAI_SHARED_PTR_CAST<geom::CartesianGridGeometry, hier::BaseGridGeometry>(
         d_hier->getGridGeometry()));
   if (!geom) TBOX_ERROR("B200CellPoissonFACOps: needs a CartesianGridGeometry");
   const hier::BoxContainer &domain = geom->getPhysicalDomain();
   if (domain.size() != 1)
      TBOX_ERROR("B200CellPoissonFACOps: the physical domain must be one box");
   const hier::Box &dbox = domain.front();
   int n0[3] = {1, 1, 1};
   double xlo[3] = {0, 0, 0}, xup[3] = {1, 1, 1};
   for (int a = 0; a < dim; ++a) {
      if (dbox.lower()(a) != 0)
         TBOX_ERROR("B200CellPoissonFACOps: the domain box must start at the origin");
      n0[a] = dbox.upper()(a) + 1;
      xlo[a] = geom->getXLower()[a];
      xup[a] = geom->getXUpper()[a];
   }
   std::vector<int> ratio(3 * nlev, 1), npatch(nlev), boxes;
   d_patches.assign(nlev, {});
   for (int ln = 0; ln < nlev; ++ln) {
      std::shared_ptr<hier::PatchLevel> level(d_hier->getPatchLevel(ln));
      std::map<int, std::shared_ptr<hier::Patch> > by_id;
      for (hier::PatchLevel::iterator ip(level->begin()); ip != level->end(); ++ip)
         by_id[(*ip)->getBox().getLocalId().getValue()] = *ip;
      for (auto &kv : by_id) {
         d_patches[ln].push_back(kv.second);
         const hier::Box &b = kv.second->getBox();
         for (int a = 0; a < 3; ++a) boxes.push_back(a < dim ? b.lower()(a) : 0);
         for (int a = 0; a < 3; ++a) boxes.push_back(a < dim ? b.upper()(a) : 0);
      }
      npatch[ln] = (int)by_id.size();
      if (ln > 0)
         for (int a = 0; a < dim; ++a) ratio[3 * ln + a] = level->getRatioToCoarserLevel()(a);
   }

   const solv::PoissonSpecifications &spec = this->*member(SpecTag());
   const int ckind = spec.cIsZero() ? 0 : (spec.cIsConstant() ? 1 : 2);
   check(fac_ctx_create(&d_ctx, dim, d_device), "fac_ctx_create");
   check(fac_set_poisson(d_ctx, spec.dIsConstant() ? 0 : 1,
                         spec.dIsConstant() ? spec.getDConstant() : 1.0, ckind,
                         ckind == 1 ? spec.getCConstant() : 0.0),
         "fac_set_poisson");
   check(fac_set_params(d_ctx, 1, 1e-300, -1.0, 1, 1, this->*member(CoarseTolTag()),
                        this->*member(CoarseMaxTag()), 1),
         "fac_set_params");
   int problem = 0;
   check(fac_add_problem(d_ctx, n0, xlo, xup, nlev, ratio.data(), npatch.data(),
                         boxes.data(), &problem),
         "fac_add_problem");
   check(fac_initialize(d_ctx), "fac_initialize");
   upload_coefficients();
   d_bc_known = false;
}

void B200CellPoissonFACOps::deallocateOperatorState()
{
   if (d_ctx) fac_ctx_destroy(d_ctx);
   d_ctx = nullptr;
   d_patches.clear();
   d_hier.reset();
}

// D (side data) and C (cell data) of the Poisson specification
void B200CellPoissonFACOps::upload_coefficients()
{
   const int dim = d_b200_dim.getValue();
   const solv::PoissonSpecifications &spec = this->*member(SpecTag());
   for (int ln = 0; ln < (int)d_patches.size(); ++ln) {
      if (!spec.dIsConstant()) {
         size_t n = 0;
         check(fac_side_size(d_ctx, 0, ln, &n), "fac_side_size");
         d_buf.assign(n, 0.0);
         size_t off = 0;
         for (auto &patch : d_patches[ln]) {
            std::shared_ptr<pdat::SideData<double> > d(
               SAMRAI_SHARED_PTR_CAST<pdat::SideData<double>, hier::PatchData>(
                  patch->getPatchData(spec.getDPatchDataId())));
            const hier::Box &b = patch->getBox();
            for (int a = 0; a < dim; ++a) {
               const pdat::ArrayData<double> &ad = d->getArrayData(a);
               const hier::Box &gb = ad.getBox();
               hier::Box sb(b);
               sb.growUpper(static_cast<tbox::Dimension::dir_t>(a), 1);
               const int lo2 = dim == 3 ? sb.lower()(2) : 0, hi2 = dim == 3 ? sb.upper()(2) : 0;
               for (int k = lo2; k <= hi2; ++k)
                  for (int j = sb.lower()(1); j <= sb.upper()(1); ++j)
                     for (int i = sb.lower()(0); i <= sb.upper()(0); ++i) {
                        const long long gi = (i - gb.lower()(0)) +
                           (long long)gb.numberCells(0) *
                              ((j - gb.lower()(1)) +
                               (dim == 3 ? (long long)gb.numberCells(1) * (k - gb.lower()(2))
                                         : 0));
                        if (off >= n) TBOX_ERROR("B200CellPoissonFACOps: side layout");
                        d_buf[off++] = ad.getPointer()[gi];
                     }
            }
         }
         check(fac_upload_side(d_ctx, 0, ln, d_buf.data()), "fac_upload_side");
      }
      if (!spec.cIsZero() && !spec.cIsConstant()) {
         solv::SAMRAIVectorReal<double> *none = nullptr;
         NULL_USE(none);
         size_t n = 0;
         check(fac_field_size(d_ctx, FAC_C, 0, ln, &n), "fac_field_size");
         d_buf.assign(n, 0.0);
         size_t off = 0;
         for (auto &patch : d_patches[ln]) {
            std::shared_ptr<pdat::CellData<double> > c(
               SAMRAI_SHARED_PTR_CAST<pdat::CellData<double>, hier::PatchData>(
                  patch->getPatchData(spec.getCPatchDataId())));
            const hier::Box &b = patch->getBox();
            const hier::Box &gb = c->getGhostBox();
            const int lo2 = dim == 3 ? b.lower()(2) : 0, hi2 = dim == 3 ? b.upper()(2) : 0;
            for (int k = lo2; k <= hi2; ++k)
               for (int j = b.lower()(1); j <= b.upper()(1); ++j)
                  for (int i = b.lower()(0); i <= b.upper()(0); ++i) {
                     const long long gi = (i - gb.lower()(0)) +
                        (long long)gb.numberCells(0) *
                           ((j - gb.lower()(1)) +
                            (dim == 3 ? (long long)gb.numberCells(1) * (k - gb.lower()(2)) : 0));
                     d_buf[off++] = c->getPointer()[gi];
                  }
         }
         check(fac_upload_field(d_ctx, FAC_C, 0, ln, d_buf.data()), "fac_upload_field C");
      }
   }
}

// Robin coefficients a, b, g from the boundary object, asked over every
// physical boundary box of every patch (the faces next to the patch,
// without tangential extensions, as CartesianRobinBcHelper asks
// SimpleCellRobinBcCoefs for them, CartesianRobinBcHelper.C:215-241), at
// the first operation of a solve, when the solver has cached its Dirichlet
// values.  Constant sides go to fac_set_bc (the fused and staged colour
// passes stay on); otherwise every level's side arrays go to
// fac_set_bc_faces.
void B200CellPoissonFACOps::sync_bc()
{
   if (d_bc_known) return;
   const solv::RobinBcCoefStrategy *bc = this->*member(BcTag());
   if (!bc) TBOX_ERROR("B200CellPoissonFACOps: no boundary condition object");
   const int dim = d_b200_dim.getValue();
   const int nlev = (int)d_patches.size();
   double a[6] = {1, 1, 1, 1, 1, 1}, b[6] = {0, 0, 0, 0, 0, 0}, g[6] = {0, 0, 0, 0, 0, 0};
   bool seen[6] = {false, false, false, false, false, false};
   bool varies = false;
   // per level and side, the faces of the level's domain face: (a, b, g)
   std::vector<std::vector<double> > faces((size_t)nlev * 6);
   std::vector<std::array<int, 6> > dom(nlev);
   std::shared_ptr<hier::Variable> var;
   for (int ln = 0; ln < nlev; ++ln) {
      const hier::BoxContainer &pd =
         d_hier->getPatchLevel(ln)->getPhysicalDomain(hier::BlockId::zero());
      const hier::Box &dbox = pd.front();
      for (int t = 0; t < 3; ++t) {
         dom[ln][t] = t < dim ? dbox.lower()(t) : 0;
         dom[ln][3 + t] = t < dim ? dbox.upper()(t) - dbox.lower()(t) + 1 : 1;
      }
      for (auto &patch : d_patches[ln]) {
         std::shared_ptr<geom::CartesianPatchGeometry> pg(
            SAMRAI_SHARED_PTR_CAST<geom::CartesianPatchGeometry, hier::PatchGeometry>(
               patch->getPatchGeometry()));
         const std::vector<hier::BoundaryBox> &bb = pg->getCodimensionBoundaries(1);
         for (const hier::BoundaryBox &bx : bb) {
            const int loc = bx.getLocationIndex();
            const int nd = loc / 2;
            // trimmed to the patch in the tangential directions
            hier::Box cells(bx.getBox());
            for (int t = 0; t < dim; ++t) {
               if (t == nd) continue;
               cells.setLower(static_cast<tbox::Dimension::dir_t>(t),
                              std::max(cells.lower()(t), patch->getBox().lower()(t)));
               cells.setUpper(static_cast<tbox::Dimension::dir_t>(t),
                              std::min(cells.upper()(t), patch->getBox().upper()(t)));
            }
            const hier::BoundaryBox trimmed(cells, 1, loc);
            hier::Box fbox(cells);
            if (loc % 2 == 0) fbox.shift(static_cast<tbox::Dimension::dir_t>(nd), 1);
            std::shared_ptr<pdat::ArrayData<double> > ad(
               std::make_shared<pdat::ArrayData<double> >(fbox, 1));
            std::shared_ptr<pdat::ArrayData<double> > bd(
               std::make_shared<pdat::ArrayData<double> >(fbox, 1));
            std::shared_ptr<pdat::ArrayData<double> > gd(
               std::make_shared<pdat::ArrayData<double> >(fbox, 1));
            bc->setBcCoefs(ad, bd, gd, var, *patch, trimmed, 0.0);
            std::vector<double> &f = faces[(size_t)ln * 6 + loc];
            if (f.empty()) {
               size_t n = 1;
               for (int t = 0; t < 3; ++t)
                  if (t != nd) n *= (size_t)dom[ln][3 + t];
               f.assign(3 * n, 0.0);
            }
            size_t q = 0;
            for (hier::Box::iterator bi(fbox.begin()); bi != fbox.end(); ++bi, ++q) {
               const hier::Index &idx = *bi;
               const double av = ad->getPointer()[q], bv = bd->getPointer()[q],
                            gv = gd->getPointer()[q];
               long long fi = 0, stride = 1;
               for (int t = 0; t < dim; ++t) {
                  if (t == nd) continue;
                  fi += stride * (idx(t) - dom[ln][t]);
                  stride *= dom[ln][3 + t];
               }
               f[3 * fi] = av;
               f[3 * fi + 1] = bv;
               f[3 * fi + 2] = gv;
               if (!seen[loc]) {
                  a[loc] = av;
                  b[loc] = bv;
                  g[loc] = gv;
                  seen[loc] = true;
               } else if (av != a[loc] || bv != b[loc] || gv != g[loc]) {
                  varies = true;
               }
            }
         }
      }
   }
   check(fac_set_bc(d_ctx, a, b, g), "fac_set_bc");
   if (varies)
      for (int ln = 0; ln < nlev; ++ln)
         for (int loc = 0; loc < 2 * dim; ++loc)
            if (!faces[(size_t)ln * 6 + loc].empty())
               check(fac_set_bc_faces(d_ctx, 0, ln, loc, faces[(size_t)ln * 6 + loc].data()),
                     "fac_set_bc_faces");
   d_bc_known = true;
}

// vector component 0 of level ln -> device field fid (the field's ghost
// width; cells outside the patch data's ghost box stay 0)
void B200CellPoissonFACOps::upload(const solv::SAMRAIVectorReal<double> &v, int ln, int fid)
{
   const int dim = d_b200_dim.getValue();
   const int g = field_ghost(fid);
   size_t n = 0;
   check(fac_field_size(d_ctx, fid, 0, ln, &n), "fac_field_size");
   d_buf.assign(n, 0.0);
   size_t off = 0;
   const int id = v.getComponentDescriptorIndex(0);
   for (auto &patch : d_patches[ln]) {
      std::shared_ptr<pdat::CellData<double> > c(
         SAMRAI_SHARED_PTR_CAST<pdat::CellData<double>, hier::PatchData>(
            patch->getPatchData(id)));
      hier::Box b(patch->getBox());
      b.grow(hier::IntVector(d_b200_dim, g));
      const hier::Box &gb = c->getGhostBox();
      const int lo2 = dim == 3 ? b.lower()(2) : 0, hi2 = dim == 3 ? b.upper()(2) : 0;
      for (int k = lo2; k <= hi2; ++k)
         for (int j = b.lower()(1); j <= b.upper()(1); ++j)
            for (int i = b.lower()(0); i <= b.upper()(0); ++i, ++off) {
               hier::Index idx(d_b200_dim);
               idx(0) = i;
               idx(1) = j;
               if (dim == 3) idx(2) = k;
               if (!gb.contains(idx)) continue;
               const long long gi = (i - gb.lower()(0)) +
                  (long long)gb.numberCells(0) *
                     ((j - gb.lower()(1)) +
                      (dim == 3 ? (long long)gb.numberCells(1) * (k - gb.lower()(2)) : 0));
               d_buf[off] = c->getPointer()[gi];
            }
   }
   if (off != n) TBOX_ERROR("B200CellPoissonFACOps: cell layout");
   check(fac_upload_field(d_ctx, fid, 0, ln, d_buf.data()), "fac_upload_field");
}

// device field fid of level ln -> vector component 0 (cells of the patch
// data's ghost box that the field has)
void B200CellPoissonFACOps::download(solv::SAMRAIVectorReal<double> &v, int ln, int fid)
{
   const int dim = d_b200_dim.getValue();
   const int g = field_ghost(fid);
   size_t n = 0;
   check(fac_field_size(d_ctx, fid, 0, ln, &n), "fac_field_size");
   d_buf.assign(n, 0.0);
   check(fac_download_field(d_ctx, fid, 0, ln, d_buf.data()), "fac_download_field");
   size_t off = 0;
   const int id = v.getComponentDescriptorIndex(0);
   for (auto &patch : d_patches[ln]) {
      std::shared_ptr<pdat::CellData<double> > c(
         SAMRAI_SHARED_PTR_CAST<pdat::CellData<double>, hier::PatchData>(
            patch->getPatchData(id)));
      hier::Box b(patch->getBox());
      b.grow(hier::IntVector(d_b200_dim, g));
      const hier::Box &gb = c->getGhostBox();
      const int lo2 = dim == 3 ? b.lower()(2) : 0, hi2 = dim == 3 ? b.upper()(2) : 0;
      for (int k = lo2; k <= hi2; ++k)
         for (int j = b.lower()(1); j <= b.upper()(1); ++j)
            for (int i = b.lower()(0); i <= b.upper()(0); ++i, ++off) {
               hier::Index idx(d_b200_dim);
               idx(0) = i;
               idx(1) = j;
               if (dim == 3) idx(2) = k;
               if (!gb.contains(idx)) continue;
               const long long gi = (i - gb.lower()(0)) +
                  (long long)gb.numberCells(0) *
                     ((j - gb.lower()(1)) +
                      (dim == 3 ? (long long)gb.numberCells(1) * (k - gb.lower()(2)) : 0));
               c->getPointer()[gi] = d_buf[off];
            }
   }
}

void B200CellPoissonFACOps::restrictSolution(const solv::SAMRAIVectorReal<double> &source,
                                             solv::SAMRAIVectorReal<double> &dest, int dest_ln)
{
   sync_bc();
   upload(source, dest_ln + 1, FAC_U);
   upload(dest, dest_ln, FAC_U);
   check(fac_restrict_solution(d_ctx, FAC_U, dest_ln), "fac_restrict_solution");
   download(dest, dest_ln, FAC_U);
}

void B200CellPoissonFACOps::restrictResidual(const solv::SAMRAIVectorReal<double> &source,
                                             solv::SAMRAIVectorReal<double> &dest, int dest_ln)
{
   upload(source, dest_ln + 1, FAC_TR);
   upload(dest, dest_ln, FAC_R);
   check(fac_restrict(d_ctx, FAC_TR, FAC_R, dest_ln), "fac_restrict");
   download(dest, dest_ln, FAC_R);
}

void B200CellPoissonFACOps::prolongErrorAndCorrect(const solv::SAMRAIVectorReal<double> &source,
                                                   solv::SAMRAIVectorReal<double> &dest,
                                                   int dest_ln)
{
   sync_bc();
   upload(source, dest_ln - 1, FAC_E);
   upload(dest, dest_ln, FAC_E);
   check(fac_prolong_correct(d_ctx, FAC_E, FAC_E, dest_ln), "fac_prolong_correct");
   download(dest, dest_ln, FAC_E);
}

void B200CellPoissonFACOps::smoothError(solv::SAMRAIVectorReal<double> &error,
                                        const solv::SAMRAIVectorReal<double> &residual, int ln,
                                        int num_sweeps)
{
   sync_bc();
   if (ln > 0) upload(error, ln - 1, FAC_E);
   upload(error, ln, FAC_E);
   upload(residual, ln, FAC_R);
   int sweeps = 0;
   check(fac_smooth(d_ctx, FAC_E, FAC_R, ln, num_sweeps, -1.0, &sweeps), "fac_smooth");
   download(error, ln, FAC_E);
}

int B200CellPoissonFACOps::solveCoarsestLevel(solv::SAMRAIVectorReal<double> &error,
                                              const solv::SAMRAIVectorReal<double> &residual,
                                              int coarsest_ln)
{
   if (coarsest_ln != 0) TBOX_ERROR("B200CellPoissonFACOps: the coarsest level must be 0");
   sync_bc();
   // the coarse-solver setters may have changed the settings since the
   // operator state was made
   check(fac_set_params(d_ctx, 1, 1e-300, -1.0, 1, 1, this->*member(CoarseTolTag()),
                        this->*member(CoarseMaxTag()), 1),
         "fac_set_params");
   upload(error, 0, FAC_E);
   upload(residual, 0, FAC_R);
   int sweeps = 0;
   check(fac_solve_coarsest(d_ctx, &sweeps), "fac_solve_coarsest");
   download(error, 0, FAC_E);
   return 0;
}

void B200CellPoissonFACOps::computeCompositeResidualOnLevel(
   solv::SAMRAIVectorReal<double> &residual, const solv::SAMRAIVectorReal<double> &solution,
   const solv::SAMRAIVectorReal<double> &rhs, int ln, bool error_equation_indicator)
{
   sync_bc();
   if (ln > 0) upload(solution, ln - 1, FAC_E);
   upload(solution, ln, FAC_E);
   upload(rhs, ln, FAC_R);
   check(fac_comp_residual(d_ctx, FAC_TR, FAC_E, FAC_R, ln, error_equation_indicator ? 1 : 0),
         "fac_comp_residual");
   download(residual, ln, FAC_TR);
   // the solution's ghost cells as the residual computation filled them
   download(const_cast<solv::SAMRAIVectorReal<double> &>(solution), ln, FAC_E);
}

double B200CellPoissonFACOps::computeResidualNorm(const solv::SAMRAIVectorReal<double> &residual,
                                                  int fine_ln, int coarse_ln)
{
   if (coarse_ln != 0 || fine_ln != (int)d_patches.size() - 1)
      TBOX_ERROR("B200CellPoissonFACOps: the norm is taken over all levels");
   for (int ln = coarse_ln; ln <= fine_ln; ++ln) upload(residual, ln, FAC_R);
   double norm = 0.0;
   check(fac_rms_norm(d_ctx, FAC_R, &norm), "fac_rms_norm");
   return norm;
}

}  // namespace samrai_b200

/*
 * B200CellPoissonFACOps -- SAMRAI's cell-centred Poisson FAC operators
 * (solv::CellPoissonFACOps) with every FACOperatorStrategy operation run by
 * the B200 library through its C ABI (include/samrai_fac_b200.h).
 *
 * A drop-in for code that builds its solver from SAMRAI's classes: pass a
 * B200CellPoissonFACOps where a CellPoissonFACOps goes (the class derives
 * from it), e.g. to CellPoissonFACSolver's constructor
 * (solv/CellPoissonFACSolver.h:134-140) or to a FACPreconditioner
 * (solv/FACPreconditioner.h:137-141).  The caller keeps using the
 * reference's public API unchanged: setPoissonSpecifications,
 * setPhysicalBcCoefObject, the coarse-solver setters and the input keys are
 * read from the base object.  The FACOperatorStrategy virtuals
 * (solv/FACOperatorStrategy.h:83-364, CellPoissonFACOps.h:408-466) copy the
 * patch data they read from the hierarchy to the device, run the operation
 * on the GPU and copy what it writes back, so FACPreconditioner's own vector
 * arithmetic on the host sees the same data as with the CPU operators.
 *
 * Supported as the GPU path implements them: prolongation_method
 * LINEAR_REFINE, cf_discretization Ewing, coarse_solver_choice redblack, a
 * level-0 domain of one box at the origin, levels from 0 up.  Robin
 * coefficients may vary along the boundary (then the library's
 * fill-based colour passes run).  Other settings stop with TBOX_ERROR in
 * initializeOperatorState.
 */
#ifndef SAMRAI_B200_CELL_POISSON_FAC_OPS_H
#define SAMRAI_B200_CELL_POISSON_FAC_OPS_H

#include "SAMRAI/SAMRAI_config.h"

#include <memory>
#include <string>
#include <vector>

#include "SAMRAI/hier/Patch.h"
#include "SAMRAI/hier/PatchHierarchy.h"
#include "SAMRAI/solv/CellPoissonFACOps.h"
#include "SAMRAI/solv/SAMRAIVectorReal.h"

struct fac_ctx;

namespace samrai_b200 {

class B200CellPoissonFACOps : public SAMRAI::solv::CellPoissonFACOps {
public:
   B200CellPoissonFACOps(const SAMRAI::tbox::Dimension &dim,
                         const std::string &object_name = std::string(),
                         const std::shared_ptr<SAMRAI::tbox::Database> &input_db =
                            std::shared_ptr<SAMRAI::tbox::Database>(),
                         int device = 0);
   ~B200CellPoissonFACOps() override;

   void restrictSolution(const SAMRAI::solv::SAMRAIVectorReal<double> &source,
                         SAMRAI::solv::SAMRAIVectorReal<double> &dest, int dest_ln) override;
   void restrictResidual(const SAMRAI::solv::SAMRAIVectorReal<double> &source,
                         SAMRAI::solv::SAMRAIVectorReal<double> &dest, int dest_ln) override;
   void prolongErrorAndCorrect(const SAMRAI::solv::SAMRAIVectorReal<double> &source,
                               SAMRAI::solv::SAMRAIVectorReal<double> &dest,
                               int dest_ln) override;
   void smoothError(SAMRAI::solv::SAMRAIVectorReal<double> &error,
                    const SAMRAI::solv::SAMRAIVectorReal<double> &residual, int ln,
                    int num_sweeps) override;
   int solveCoarsestLevel(SAMRAI::solv::SAMRAIVectorReal<double> &error,
                          const SAMRAI::solv::SAMRAIVectorReal<double> &residual,
                          int coarsest_ln) override;
   void computeCompositeResidualOnLevel(SAMRAI::solv::SAMRAIVectorReal<double> &residual,
                                        const SAMRAI::solv::SAMRAIVectorReal<double> &solution,
                                        const SAMRAI::solv::SAMRAIVectorReal<double> &rhs,
                                        int ln, bool error_equation_indicator) override;
   double computeResidualNorm(const SAMRAI::solv::SAMRAIVectorReal<double> &residual,
                              int fine_ln, int coarse_ln) override;
   void initializeOperatorState(const SAMRAI::solv::SAMRAIVectorReal<double> &solution,
                                const SAMRAI::solv::SAMRAIVectorReal<double> &rhs) override;
   void deallocateOperatorState() override;

private:
   // device field of the library a vector component is copied into
   void upload(const SAMRAI::solv::SAMRAIVectorReal<double> &v, int ln, int fid);
   void download(SAMRAI::solv::SAMRAIVectorReal<double> &v, int ln, int fid);
   void upload_coefficients();
   void sync_bc();
   void check(int rc, const char *what) const;

   const SAMRAI::tbox::Dimension d_b200_dim;
   int d_device;
   fac_ctx *d_ctx = nullptr;
   std::shared_ptr<SAMRAI::hier::PatchHierarchy> d_hier;
   // patches of each level in LocalId order, the order of the device layout
   std::vector<std::vector<std::shared_ptr<SAMRAI::hier::Patch> > > d_patches;
   std::vector<double> d_buf;
   bool d_bc_known = false;
};

}  // namespace samrai_b200

#endif

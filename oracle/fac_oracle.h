/*
 * fac_oracle.h -- CPU restatement of SAMRAI's cell-centred FAC Poisson path.
 *
 * TEST INFRASTRUCTURE ONLY.  This oracle is the checker for the CUDA path in
 * samrai_b200: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it.  The product path never calls it.
 *
 * Parity status: pinned against the reference's own known-answer tests for
 * this path (linear refine of linear data is exact, conservative coarsening
 * of linear data is exact: source/test/communication/CellDataTest.C:554-643;
 * FAC discretisation error of the sine problem:
 * source/test/FAC_adaptive/main.C:282-392).  The reference's Fortran kernels
 * cannot be compiled in this image (no gfortran, no m4) and its C++ needs a
 * CMake-generated configuration header, so no binary of the reference itself
 * runs here; every routine below restates the reference routine it cites.
 *
 * Data layout follows pdat::ArrayData (source/SAMRAI/pdat/ArrayData.C:79-127):
 * one column-major array per patch over the ghosted box, i fastest.  The
 * "canonical" export layout of a level is the concatenation of its patches'
 * ghosted arrays in patch order (side data: per patch, axis 0..dim-1; outer-
 * side data: per patch, axis, lower/upper side).
 */
#ifndef FAC_ORACLE_H
#define FAC_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Cell fields (ghost width in brackets). */
enum {
   ORC_U = 0,   /* solution u            [1] */
   ORC_F,       /* right-hand side f     [0] */
   ORC_E,       /* error e               [1] */
   ORC_R,       /* residual r            [0] */
   ORC_TR,      /* coarser residual      [0] */
   ORC_W,       /* control volume weight [0] */
   ORC_C,       /* Poisson C field       [0] */
   ORC_NCELL
};
/* Side fields (ghost 0). */
enum { ORC_SD = 0, ORC_SFLUX, ORC_NSIDE };

typedef struct orc_hier orc_hier;

/*
 * Create a hierarchy.  boxes holds, for every patch of every level in level
 * order, lo0 lo1 lo2 hi0 hi1 hi2 (2-D: lo2 = hi2 = 0).  ratio holds, per
 * level, the refinement ratio to the next coarser level (level 0: 1 1 1).
 * The physical domain is level 0's box [0, n0-1] x ... with physical extent
 * [xlo, xup].
 */
orc_hier *orc_create(int dim, const int *n0, const double *xlo,
                     const double *xup, int nlev, const int *ratio,
                     const int *npatch, const int *boxes);
void orc_destroy(orc_hier *h);

/* Poisson specification (PoissonSpecifications.h): D constant or side
 * field; C kind 0 = zero, 1 = constant, 2 = cell field. */
void orc_set_poisson(orc_hier *h, int d_variable, double d_const,
                     int c_kind, double c_const);
/* Robin coefficients per location index 0..2*dim-1 (a u + b un = g). */
void orc_set_bc(orc_hier *h, const double *a, const double *b,
                const double *g);
/* Robin coefficients per face of location index loc of level ln: abg holds
 * (a, b, g) triples over the level's whole domain face, the lowest
 * tangential axis fastest (NULL: back to the constants of orc_set_bc). */
void orc_set_bc_faces(orc_hier *h, int ln, int loc, const double *abg);
/* Solver parameters (FACPreconditioner / CellPoissonFACOps input keys). */
void orc_set_params(orc_hier *h, int max_cycles, double residual_tol,
                    double relative_residual_tol, int pre_sweeps,
                    int post_sweeps, double coarse_tol, int coarse_max_it,
                    int ewing);

long orc_field_size(const orc_hier *h, int fid, int ln);
void orc_get_field(const orc_hier *h, int fid, int ln, double *out);
void orc_set_field(orc_hier *h, int fid, int ln, const double *in);
long orc_side_size(const orc_hier *h, int sid, int ln);
void orc_get_side(const orc_hier *h, int sid, int ln, double *out);
void orc_set_side(orc_hier *h, int sid, int ln, const double *in);
long orc_oside_size(const orc_hier *h, int ln);
void orc_get_oside(const orc_hier *h, int ln, double *out);

/* Operations (each mirrors one CellPoissonFACOps / FACPreconditioner step). */
void orc_ghost_fill(orc_hier *h, int fid, int ln, int with_coarse,
                    int homogeneous);
int orc_smooth(orc_hier *h, int fid_e, int fid_r, int ln, int nsweeps,
               double tol, double *maxres_out);
void orc_comp_residual(orc_hier *h, int fid_r, int fid_u, int fid_f, int ln,
                       int error_equation);
void orc_restrict(orc_hier *h, int fid_src, int fid_dst, int dest_ln);
void orc_restrict_solution(orc_hier *h, int fid, int dest_ln);
void orc_prolong_correct(orc_hier *h, int fid_src, int fid_dst, int dest_ln);
void orc_compute_weights(orc_hier *h);
double orc_rms_norm(const orc_hier *h, int fid);
int orc_solve_coarsest(orc_hier *h, int fid_e, int fid_r, int ln);
void orc_fac_cycle(orc_hier *h);
/* Full CellPoissonFACSolver::solveSystem.  Returns 1 if converged.
 * hist (length >= max_cycles+1, may be NULL) receives the residual norm
 * before the first cycle and after each cycle. */
int orc_solve(orc_hier *h, int *iterations, double *residual_norm,
              double *hist);
/* Number of red-black sweeps taken by the last coarsest-level solves,
 * summed since the last reset. */
long orc_coarse_sweeps(const orc_hier *h);
void orc_reset_stats(orc_hier *h);

#ifdef __cplusplus
}
#endif
#endif

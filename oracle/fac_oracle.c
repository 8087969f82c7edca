/*
 * fac_oracle.c -- CPU restatement of SAMRAI's cell-centred FAC Poisson path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker for the CUDA path; never part of the
 * product).  Compile with -ffp-contract=off so every floating-point operation
 * is rounded exactly where the reference's Fortran rounds it.
 *
 * Each routine cites the reference routine it restates (paths relative to the
 * SAMRAI source tree; "2d.f"/"3d.f" = solv/fortran/solv_cellpoissonfacops{2,3}d.f).
 */
#include "fac_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define OMAXL 8

static const int k_cell_ghost[ORC_NCELL] = {1, 0, 1, 0, 0, 0, 0};

typedef struct {
   int lo[3], hi[3];
} obox;

typedef struct {
   double *p;
   int lo[3];   /* lower corner of the array's box */
   int n[3];    /* extents of the array's box */
} oarr;

#define AT(A, i, j, k)                                                   \
   ((A).p[((long)(i) - (A).lo[0]) +                                      \
          (long)(A).n[0] * (((long)(j) - (A).lo[1]) +                    \
                            (long)(A).n[1] * ((long)(k) - (A).lo[2]))])

typedef struct {
   obox box;
   double *cell[ORC_NCELL];
   double *side[ORC_NSIDE][3];
   double *oside[3][2];
   unsigned char *cfmask[3][2];  /* coarse-fine boundary mask per face */
} opatch;

typedef struct {
   int np;
   opatch *p;
   int ratio[3];   /* ratio to next coarser level */
   int rzero[3];   /* ratio to level 0 */
   double dx[3];
   obox domain;
} olevel;

struct orc_hier {
   int dim;
   double xlo[3], xup[3];
   int nlev;
   olevel L[OMAXL];
   int d_variable;
   double d_const;
   int c_kind;
   double c_const;
   double bc_a[6], bc_b[6], bc_g[6];
   /* per-face Robin coefficients (a, b, g triples) over each level's domain
    * face of each location index, or NULL for the constants above */
   double *bcf[OMAXL][6];
   /* FACPreconditioner / CellPoissonFACOps parameters */
   int max_cycles;
   double residual_tol, rel_residual_tol;
   int pre_sweeps, post_sweeps;
   double coarse_tol;
   int coarse_max_it;
   int ewing;
   long coarse_sweeps;
   /* Dirichlet data cached from u's ghost cells (SimpleCellRobinBcCoefs) */
   double *cached[OMAXL];
};

/* ------------------------------------------------------------------ */
/* box helpers                                                          */
/* ------------------------------------------------------------------ */

static obox box_grow(obox b, int dim, int g)
{
   for (int a = 0; a < dim; ++a) {
      b.lo[a] -= g;
      b.hi[a] += g;
   }
   return b;
}

static int box_empty(const obox *b)
{
   return b->lo[0] > b->hi[0] || b->lo[1] > b->hi[1] || b->lo[2] > b->hi[2];
}

static obox box_isect(obox a, obox b)
{
   obox r;
   for (int d = 0; d < 3; ++d) {
      r.lo[d] = a.lo[d] > b.lo[d] ? a.lo[d] : b.lo[d];
      r.hi[d] = a.hi[d] < b.hi[d] ? a.hi[d] : b.hi[d];
   }
   return r;
}

static int box_contains(const obox *b, int i, int j, int k)
{
   return i >= b->lo[0] && i <= b->hi[0] && j >= b->lo[1] &&
          j <= b->hi[1] && k >= b->lo[2] && k <= b->hi[2];
}

/* hier::Index coarsen: floor division (geom_m4cartopstuff.i:8-14). */
static int coarsen_index(int i, int r)
{
   return i < 0 ? (i + 1) / r - 1 : i / r;
}

static obox box_coarsen(obox b, int dim, const int *r)
{
   for (int a = 0; a < dim; ++a) {
      b.lo[a] = coarsen_index(b.lo[a], r[a]);
      b.hi[a] = coarsen_index(b.hi[a], r[a]);
   }
   return b;
}

static long box_size(const obox *b)
{
   if (box_empty(b)) return 0;
   return (long)(b->hi[0] - b->lo[0] + 1) * (b->hi[1] - b->lo[1] + 1) *
          (b->hi[2] - b->lo[2] + 1);
}

/* ------------------------------------------------------------------ */
/* array accessors                                                      */
/* ------------------------------------------------------------------ */

static obox cell_gbox(const orc_hier *h, const opatch *p, int fid)
{
   return box_grow(p->box, h->dim, k_cell_ghost[fid]);
}

static oarr arr_from_box(double *ptr, obox b)
{
   oarr A;
   A.p = ptr;
   for (int d = 0; d < 3; ++d) {
      A.lo[d] = b.lo[d];
      A.n[d] = b.hi[d] - b.lo[d] + 1;
   }
   return A;
}

static oarr cell_arr(const orc_hier *h, const opatch *p, int fid)
{
   return arr_from_box(p->cell[fid], cell_gbox(h, p, fid));
}

/* Side data box for axis a: upper(a)+1 (pdat/SideGeometry.C:194). */
static obox side_box(const opatch *p, int a)
{
   obox b = p->box;
   b.hi[a] += 1;
   return b;
}

static oarr side_arr(const opatch *p, int sid, int a)
{
   return arr_from_box(p->side[sid][a], side_box(p, a));
}

/* Outerside data for axis a, side s: the side box restricted to the face. */
static obox oside_box(const opatch *p, int a, int s)
{
   obox b = side_box(p, a);
   if (s == 0) b.hi[a] = b.lo[a];
   else b.lo[a] = b.hi[a];
   return b;
}

static oarr oside_arr(const opatch *p, int a, int s)
{
   return arr_from_box(p->oside[a][s], oside_box(p, a, s));
}

/* ------------------------------------------------------------------ */
/* creation                                                             */
/* ------------------------------------------------------------------ */

static void compute_cf_masks(orc_hier *h, int ln);

orc_hier *orc_create(int dim, const int *n0, const double *xlo,
                     const double *xup, int nlev, const int *ratio,
                     const int *npatch, const int *boxes)
{
   if (dim < 2 || dim > 3 || nlev < 1 || nlev > OMAXL) return NULL;
   orc_hier *h = (orc_hier *)calloc(1, sizeof(orc_hier));
   h->dim = dim;
   h->nlev = nlev;
   for (int d = 0; d < 3; ++d) {
      h->xlo[d] = d < dim ? xlo[d] : 0.0;
      h->xup[d] = d < dim ? xup[d] : 1.0;
   }
   /* CartesianGridGeometry.C:308-312 and :373-379: dx0 = length/ncells,
    * dx on a refined level = dx0 / ratio_to_level_zero. */
   double dx0[3];
   for (int d = 0; d < 3; ++d)
      dx0[d] = d < dim ? (h->xup[d] - h->xlo[d]) / ((double)n0[d]) : 1.0;
   int off = 0;
   for (int ln = 0; ln < nlev; ++ln) {
      olevel *L = &h->L[ln];
      for (int d = 0; d < 3; ++d) {
         L->ratio[d] = d < dim ? ratio[3 * ln + d] : 1;
         L->rzero[d] = (ln == 0 ? 1 : h->L[ln - 1].rzero[d]) * L->ratio[d];
         L->dx[d] = d < dim ? dx0[d] / ((double)L->rzero[d]) : 1.0;
         L->domain.lo[d] = 0;
         L->domain.hi[d] = d < dim ? n0[d] * L->rzero[d] - 1 : 0;
      }
      L->np = npatch[ln];
      L->p = (opatch *)calloc((size_t)L->np, sizeof(opatch));
      for (int ip = 0; ip < L->np; ++ip) {
         opatch *p = &L->p[ip];
         for (int d = 0; d < 3; ++d) {
            p->box.lo[d] = boxes[6 * off + d];
            p->box.hi[d] = boxes[6 * off + 3 + d];
         }
         if (dim == 2) p->box.lo[2] = p->box.hi[2] = 0;
         ++off;
         for (int f = 0; f < ORC_NCELL; ++f) {
            obox gb = cell_gbox(h, p, f);
            p->cell[f] = (double *)calloc((size_t)box_size(&gb), sizeof(double));
         }
         for (int s = 0; s < ORC_NSIDE; ++s)
            for (int a = 0; a < dim; ++a) {
               obox sb = side_box(p, a);
               p->side[s][a] =
                  (double *)calloc((size_t)box_size(&sb), sizeof(double));
            }
         for (int a = 0; a < dim; ++a)
            for (int s = 0; s < 2; ++s) {
               obox ob = oside_box(p, a, s);
               p->oside[a][s] =
                  (double *)calloc((size_t)box_size(&ob), sizeof(double));
               p->cfmask[a][s] = (unsigned char *)calloc((size_t)box_size(&ob), 1);
            }
      }
   }
   h->d_variable = 0;
   h->d_const = 1.0;
   h->c_kind = 0;
   h->c_const = 0.0;
   for (int l = 0; l < 6; ++l) {
      h->bc_a[l] = 1.0;  /* Dirichlet: SimpleCellRobinBcCoefs.C:283-290 */
      h->bc_b[l] = 0.0;
      h->bc_g[l] = 0.0;
   }
   h->max_cycles = 10;
   h->residual_tol = 1e-6;
   h->rel_residual_tol = -1.0;
   h->pre_sweeps = 1;
   h->post_sweeps = 1;
   h->coarse_tol = 1e-8;
   h->coarse_max_it = 500;
   h->ewing = 1;
   for (int ln = 1; ln < nlev; ++ln) compute_cf_masks(h, ln);
   return h;
}

void orc_destroy(orc_hier *h)
{
   if (!h) return;
   for (int ln = 0; ln < h->nlev; ++ln) {
      olevel *L = &h->L[ln];
      for (int loc = 0; loc < 6; ++loc) free(h->bcf[ln][loc]);
      for (int ip = 0; ip < L->np; ++ip) {
         opatch *p = &L->p[ip];
         for (int f = 0; f < ORC_NCELL; ++f) free(p->cell[f]);
         for (int s = 0; s < ORC_NSIDE; ++s)
            for (int a = 0; a < 3; ++a) free(p->side[s][a]);
         for (int a = 0; a < 3; ++a)
            for (int s = 0; s < 2; ++s) {
               free(p->oside[a][s]);
               free(p->cfmask[a][s]);
            }
      }
      free(L->p);
      free(h->cached[ln]);
   }
   free(h);
}

void orc_set_poisson(orc_hier *h, int d_variable, double d_const,
                     int c_kind, double c_const)
{
   h->d_variable = d_variable;
   h->d_const = d_const;
   h->c_kind = c_kind;
   h->c_const = c_const;
}

void orc_set_bc(orc_hier *h, const double *a, const double *b,
                const double *g)
{
   for (int l = 0; l < 2 * h->dim; ++l) {
      h->bc_a[l] = a[l];
      h->bc_b[l] = b[l];
      h->bc_g[l] = g[l];
   }
}

void orc_set_bc_faces(orc_hier *h, int ln, int loc, const double *abg)
{
   if (ln < 0 || ln >= h->nlev || loc < 0 || loc >= 2 * h->dim) return;
   const obox *d = &h->L[ln].domain;
   long n = 1;
   for (int t = 0; t < h->dim; ++t)
      if (t != loc / 2) n *= d->hi[t] - d->lo[t] + 1;
   free(h->bcf[ln][loc]);
   h->bcf[ln][loc] = NULL;
   if (!abg) return;
   h->bcf[ln][loc] = malloc(3 * n * sizeof(double));
   memcpy(h->bcf[ln][loc], abg, 3 * n * sizeof(double));
}

void orc_set_params(orc_hier *h, int max_cycles, double residual_tol,
                    double relative_residual_tol, int pre_sweeps,
                    int post_sweeps, double coarse_tol, int coarse_max_it,
                    int ewing)
{
   h->max_cycles = max_cycles;
   h->residual_tol = residual_tol;
   h->rel_residual_tol = relative_residual_tol;
   h->pre_sweeps = pre_sweeps;
   h->post_sweeps = post_sweeps;
   h->coarse_tol = coarse_tol;
   h->coarse_max_it = coarse_max_it;
   h->ewing = ewing;
}

/* ------------------------------------------------------------------ */
/* canonical field I/O                                                  */
/* ------------------------------------------------------------------ */

long orc_field_size(const orc_hier *h, int fid, int ln)
{
   long n = 0;
   for (int ip = 0; ip < h->L[ln].np; ++ip) {
      obox gb = cell_gbox(h, &h->L[ln].p[ip], fid);
      n += box_size(&gb);
   }
   return n;
}

void orc_get_field(const orc_hier *h, int fid, int ln, double *out)
{
   for (int ip = 0; ip < h->L[ln].np; ++ip) {
      const opatch *p = &h->L[ln].p[ip];
      obox gb = cell_gbox(h, p, fid);
      long n = box_size(&gb);
      memcpy(out, p->cell[fid], (size_t)n * sizeof(double));
      out += n;
   }
}

void orc_set_field(orc_hier *h, int fid, int ln, const double *in)
{
   for (int ip = 0; ip < h->L[ln].np; ++ip) {
      opatch *p = &h->L[ln].p[ip];
      obox gb = cell_gbox(h, p, fid);
      long n = box_size(&gb);
      memcpy(p->cell[fid], in, (size_t)n * sizeof(double));
      in += n;
   }
}

long orc_side_size(const orc_hier *h, int sid, int ln)
{
   (void)sid;
   long n = 0;
   for (int ip = 0; ip < h->L[ln].np; ++ip)
      for (int a = 0; a < h->dim; ++a) {
         obox sb = side_box(&h->L[ln].p[ip], a);
         n += box_size(&sb);
      }
   return n;
}

void orc_get_side(const orc_hier *h, int sid, int ln, double *out)
{
   for (int ip = 0; ip < h->L[ln].np; ++ip)
      for (int a = 0; a < h->dim; ++a) {
         const opatch *p = &h->L[ln].p[ip];
         obox sb = side_box(p, a);
         long n = box_size(&sb);
         memcpy(out, p->side[sid][a], (size_t)n * sizeof(double));
         out += n;
      }
}

void orc_set_side(orc_hier *h, int sid, int ln, const double *in)
{
   for (int ip = 0; ip < h->L[ln].np; ++ip)
      for (int a = 0; a < h->dim; ++a) {
         opatch *p = &h->L[ln].p[ip];
         obox sb = side_box(p, a);
         long n = box_size(&sb);
         memcpy(p->side[sid][a], in, (size_t)n * sizeof(double));
         in += n;
      }
}

long orc_oside_size(const orc_hier *h, int ln)
{
   long n = 0;
   for (int ip = 0; ip < h->L[ln].np; ++ip)
      for (int a = 0; a < h->dim; ++a)
         for (int s = 0; s < 2; ++s) {
            obox ob = oside_box(&h->L[ln].p[ip], a, s);
            n += box_size(&ob);
         }
   return n;
}

void orc_get_oside(const orc_hier *h, int ln, double *out)
{
   for (int ip = 0; ip < h->L[ln].np; ++ip)
      for (int a = 0; a < h->dim; ++a)
         for (int s = 0; s < 2; ++s) {
            const opatch *p = &h->L[ln].p[ip];
            obox ob = oside_box(p, a, s);
            long n = box_size(&ob);
            memcpy(out, p->oside[a][s], (size_t)n * sizeof(double));
            out += n;
         }
}

/* ------------------------------------------------------------------ */
/* level coverage queries                                               */
/* ------------------------------------------------------------------ */

static int level_find_patch(const orc_hier *h, int ln, int i, int j, int k)
{
   const olevel *L = &h->L[ln];
   for (int ip = 0; ip < L->np; ++ip)
      if (box_contains(&L->p[ip].box, i, j, k)) return ip;
   return -1;
}

/*
 * Coarse-fine boundary faces of every patch of level ln
 * (hier/CoarseFineBoundary.C:130-260 with BaseGridGeometry::getBoundaryBoxes,
 * hier/BaseGridGeometry.C:1077-1222): a face cell of the patch is on the
 * coarse-fine boundary when the ghost cell across it lies inside the
 * physical domain and is not covered by any patch of the level.  The Ewing
 * fix-up clips the boundary boxes to the patch's own tangential extent
 * (2d.f:495-499), so the mask is over the patch face only.
 */
static void compute_cf_masks(orc_hier *h, int ln)
{
   olevel *L = &h->L[ln];
   for (int ip = 0; ip < L->np; ++ip) {
      opatch *p = &L->p[ip];
      for (int a = 0; a < h->dim; ++a)
         for (int s = 0; s < 2; ++s) {
            int g = s == 0 ? p->box.lo[a] - 1 : p->box.hi[a] + 1;
            obox ob = oside_box(p, a, s);
            unsigned char *m = p->cfmask[a][s];
            long idx = 0;
            for (int k = ob.lo[2]; k <= ob.hi[2]; ++k)
               for (int j = ob.lo[1]; j <= ob.hi[1]; ++j)
                  for (int i = ob.lo[0]; i <= ob.hi[0]; ++i, ++idx) {
                     int c[3] = {i, j, k};
                     c[a] = g;
                     int inside = box_contains(&L->domain, c[0], c[1], c[2]);
                     int covered = level_find_patch(h, ln, c[0], c[1], c[2]) >= 0;
                     m[idx] = (unsigned char)(inside && !covered);
                  }
         }
   }
}

/* ------------------------------------------------------------------ */
/* physical boundary conditions                                         */
/* ------------------------------------------------------------------ */

/*
 * Robin ghost values on the ghost layer (width 1) of an array over box b:
 * solv/CartesianRobinBcHelper.C:125-593 with SimpleCellRobinBcCoefs
 * (numberOfExtensionsFillable() == 0, SimpleCellRobinBcCoefs.C:483-486, so
 * every boundary box is trimmed to the patch box along its tangential
 * directions, CartesianRobinBcHelper.C:215-218).
 *   codimension 1: settype1cells{2,3}d (robinbchelper2d.f:10-72)
 *   codimension 2: settype2cells2d (robinbchelper2d.f:74-108),
 *                  settype2cells3d (robinbchelper3d.f:110-246)
 *   codimension 3: settype3cells3d (robinbchelper3d.f:247-333)
 * Codimension 1 is done for all faces first, then 2, then 3, as in the
 * reference.
 */
/* Index of the face at the tangential coordinates of cell c on location
 * loc of a level's domain face: lowest tangential axis fastest. */
static long face_index(int dim, const obox *domain, int loc, const int *c)
{
   const int a = loc / 2;
   long idx = 0, stride = 1;
   for (int t = 0; t < dim; ++t) {
      if (t == a) continue;
      idx += stride * (c[t] - domain->lo[t]);
      stride *= domain->hi[t] - domain->lo[t] + 1;
   }
   return idx;
}

static void bc_fill_box(const orc_hier *h, oarr A, obox b, const obox *domain,
                        const double *dx, int homogeneous, double *const *faces)
{
   const int dim = h->dim;
   obox gb = box_grow(b, dim, 1);
   for (int codim = 1; codim <= dim; ++codim) {
      for (int k = gb.lo[2]; k <= gb.hi[2]; ++k)
         for (int j = gb.lo[1]; j <= gb.hi[1]; ++j)
            for (int i = gb.lo[0]; i <= gb.hi[0]; ++i) {
               int c[3] = {i, j, k};
               int out = 0, ok = 1;
               int side[3] = {0, 0, 0}; /* -1 below domain, +1 above */
               for (int a = 0; a < dim; ++a) {
                  if (c[a] < domain->lo[a] || c[a] > domain->hi[a]) {
                     /* outside the domain: must be the ghost layer next to
                      * the box face lying on the domain boundary */
                     if (c[a] == b.lo[a] - 1 && b.lo[a] == domain->lo[a])
                        side[a] = -1;
                     else if (c[a] == b.hi[a] + 1 && b.hi[a] == domain->hi[a])
                        side[a] = 1;
                     else
                        ok = 0;
                     ++out;
                  } else if (c[a] < b.lo[a] || c[a] > b.hi[a]) {
                     ok = 0; /* tangential extension trimmed away */
                  }
               }
               if (!ok || out != codim) continue;
               if (codim == 1) {
                  int a = side[0] ? 0 : (side[1] ? 1 : 2);
                  int loc = 2 * a + (side[a] > 0 ? 1 : 0);
                  int ci[3] = {i, j, k};
                  ci[a] -= side[a];
                  double av = h->bc_a[loc], bv = h->bc_b[loc], gv = h->bc_g[loc];
                  if (faces && faces[loc]) {
                     /* the coefficients of the face between ghost and
                      * interior cell (RobinBcCoefStrategy::setBcCoefs
                      * arrays, RobinBcCoefStrategy.h:138-145) */
                     const double *f = faces[loc] + 3 * face_index(dim, domain, loc, c);
                     av = f[0];
                     bv = f[1];
                     gv = f[2];
                  }
                  double hh = dx[a];
                  double uin = AT(A, ci[0], ci[1], ci[2]);
                  double v;
                  if (homogeneous)
                     v = (uin * (bv - 0.5 * hh * av)) / (bv + 0.5 * hh * av);
                  else
                     v = (hh * gv + uin * (bv - 0.5 * hh * av)) /
                         (bv + 0.5 * hh * av);
                  AT(A, i, j, k) = v;
               } else if (codim == 2) {
                  int ax[2], n = 0;
                  for (int a = 0; a < dim; ++a)
                     if (side[a]) ax[n++] = a;
                  int s0 = -side[ax[0]], s1 = -side[ax[1]];
                  int d0[3] = {0, 0, 0}, d1[3] = {0, 0, 0};
                  d0[ax[0]] = s0;
                  d1[ax[1]] = s1;
                  double vboth = AT(A, i + d0[0] + d1[0], j + d0[1] + d1[1],
                                    k + d0[2] + d1[2]);
                  double v0 = AT(A, i + d0[0], j + d0[1], k + d0[2]);
                  double v1 = AT(A, i + d1[0], j + d1[1], k + d1[2]);
                  AT(A, i, j, k) = -vboth + (v0 + v1);
               } else {
                  /* settype3cells3d: -d(all inward) + 2./3.*(d(i fixed) +
                   * d(j fixed) + d(k fixed)); 2./3. is a REAL*4 constant. */
                  int si = -side[0], sj = -side[1], sk = -side[2];
                  double vall = AT(A, i + si, j + sj, k + sk);
                  double vi = AT(A, i, j + sj, k + sk);
                  double vj = AT(A, i + si, j, k + sk);
                  double vk = AT(A, i + si, j + sj, k);
                  const double two3 = (double)(2.0f / 3.0f);
                  AT(A, i, j, k) = -vall + two3 * ((vi + vj) + vk);
               }
            }
   }
}

/* ------------------------------------------------------------------ */
/* ghost fill (RefineSchedule::fillData)                                */
/* ------------------------------------------------------------------ */

/*
 * Same-level copies: dst ghost box intersect src interior
 * (pdat/CellGeometry.C:96-124 with src_mask = src box,
 * xfer/RefineSchedule.C:4670-4683); transactions whose src and dst are the
 * same patch are skipped (RefineSchedule.C:4793-4797).
 */
static void fill_same_level(orc_hier *h, int fid, int ln)
{
   olevel *L = &h->L[ln];
   for (int ip = 0; ip < L->np; ++ip) {
      opatch *p = &L->p[ip];
      oarr D = cell_arr(h, p, fid);
      obox gb = cell_gbox(h, p, fid);
      for (int iq = 0; iq < L->np; ++iq) {
         if (iq == ip) continue;
         opatch *q = &L->p[iq];
         obox ov = box_isect(gb, q->box);
         if (box_empty(&ov)) continue;
         oarr S = cell_arr(h, q, fid);
         for (int k = ov.lo[2]; k <= ov.hi[2]; ++k)
            for (int j = ov.lo[1]; j <= ov.hi[1]; ++j)
               for (int i = ov.lo[0]; i <= ov.hi[0]; ++i)
                  AT(D, i, j, k) = AT(S, i, j, k);
      }
   }
}

/*
 * Ghost cells not covered by the level and inside the domain are filled by
 * CONSTANT_REFINE from the next coarser level (the Ewing choice,
 * CellPoissonFACOps.C:940-943; pdat/CellConstantRefine.C:32-130 and
 * pdat_m4conrefineops2d.i:33: fine = coarse(coarsen(i))).  The coarse
 * interpolation level is filled from the coarser level's interiors only.
 */
static void fill_from_coarse(orc_hier *h, int fid, int ln)
{
   olevel *L = &h->L[ln];
   olevel *C = &h->L[ln - 1];
   for (int ip = 0; ip < L->np; ++ip) {
      opatch *p = &L->p[ip];
      oarr D = cell_arr(h, p, fid);
      obox gb = cell_gbox(h, p, fid);
      for (int k = gb.lo[2]; k <= gb.hi[2]; ++k)
         for (int j = gb.lo[1]; j <= gb.hi[1]; ++j)
            for (int i = gb.lo[0]; i <= gb.hi[0]; ++i) {
               if (box_contains(&p->box, i, j, k)) continue;
               if (!box_contains(&L->domain, i, j, k)) continue;
               if (level_find_patch(h, ln, i, j, k) >= 0) continue;
               int ci = coarsen_index(i, L->ratio[0]);
               int cj = coarsen_index(j, L->ratio[1]);
               int ck = coarsen_index(k, L->ratio[2]);
               int q = level_find_patch(h, ln - 1, ci, cj, ck);
               if (q < 0) {
                  fprintf(stderr, "oracle: level %d not properly nested\n", ln);
                  abort();
               }
               oarr S = cell_arr(h, &C->p[q], fid);
               AT(D, i, j, k) = AT(S, ci, cj, ck);
            }
   }
}

static void fill_physical(orc_hier *h, int fid, int ln, int homogeneous)
{
   olevel *L = &h->L[ln];
   if (k_cell_ghost[fid] < 1) return;
   for (int ip = 0; ip < L->np; ++ip) {
      opatch *p = &L->p[ip];
      bc_fill_box(h, cell_arr(h, p, fid), p->box, &L->domain, L->dx, homogeneous,
                  h->bcf[ln]);
   }
}

/* xeqScheduleGhostFillNoCoarse / xeqScheduleGhostFill
 * (CellPoissonFACOps.C:2861-2900; RefineSchedule::recursiveFill,
 * RefineSchedule.C:2148-2397: coarse interpolation, then same-level copies,
 * then physical boundary conditions). */
void orc_ghost_fill(orc_hier *h, int fid, int ln, int with_coarse,
                    int homogeneous)
{
   if (with_coarse && ln > 0) fill_from_coarse(h, fid, ln);
   fill_same_level(h, fid, ln);
   fill_physical(h, fid, ln, homogeneous);
}

/* ------------------------------------------------------------------ */
/* flux, Ewing fix, smoother, residual (solv_cellpoissonfacops{2,3}d.f) */
/* ------------------------------------------------------------------ */

/* compfluxvardc2d / compfluxcondc2d (2d.f:10-92);
 * compfluxvardc3d / compfluxcondc3d (3d.f:10-135). */
static void compute_flux_on_patch(orc_hier *h, opatch *p, double *dx,
                                  oarr U)
{
   const obox b = p->box;
   const int dim = h->dim;
   double dxi = 1. / dx[0], dyi = 1. / dx[1];
   double dzi = dim == 3 ? 1. / dx[2] : 0.0;
   oarr FX = side_arr(p, ORC_SFLUX, 0), FY = side_arr(p, ORC_SFLUX, 1), FZ = {0};
   oarr DX = {0}, DY = {0}, DZ = {0};
   if (h->d_variable) {
      DX = side_arr(p, ORC_SD, 0);
      DY = side_arr(p, ORC_SD, 1);
   }
   if (dim == 3) {
      FZ = side_arr(p, ORC_SFLUX, 2);
      if (h->d_variable) DZ = side_arr(p, ORC_SD, 2);
   }
   const double dc = h->d_const;
   for (int k = b.lo[2]; k <= b.hi[2]; ++k)
      for (int j = b.lo[1]; j <= b.hi[1]; ++j)
         for (int i = b.lo[0]; i <= b.hi[0] + 1; ++i) {
            double d = h->d_variable ? AT(DX, i, j, k) : dc;
            AT(FX, i, j, k) = dxi * d * (AT(U, i, j, k) - AT(U, i - 1, j, k));
         }
   for (int k = b.lo[2]; k <= b.hi[2]; ++k)
      for (int j = b.lo[1]; j <= b.hi[1] + 1; ++j)
         for (int i = b.lo[0]; i <= b.hi[0]; ++i) {
            double d = h->d_variable ? AT(DY, i, j, k) : dc;
            AT(FY, i, j, k) = dyi * d * (AT(U, i, j, k) - AT(U, i, j - 1, k));
         }
   if (dim == 3)
      for (int k = b.lo[2]; k <= b.hi[2] + 1; ++k)
         for (int j = b.lo[1]; j <= b.hi[1]; ++j)
            for (int i = b.lo[0]; i <= b.hi[0]; ++i) {
               double d = h->d_variable ? AT(DZ, i, j, k) : dc;
               AT(FZ, i, j, k) = dzi * d * (AT(U, i, j, k) - AT(U, i, j, k - 1));
            }
}

/*
 * ewingfixflux{vardc,condc}{2,3}d (2d.f:460-686, 3d.f:604-1012):
 *   flux = longwt*flux +/- tranwt*D*(u(mirror) - u(cell))/h
 * with tranwt = 1.0/(1+r) evaluated in REAL*4 and longwt = 2*tranwt.
 * Mirror = the other fine cell of the same coarse cell, along every
 * tangential direction.  Applied to every coarse-fine boundary face
 * (CellPoissonFACOps::ewingFixFlux, CellPoissonFACOps.C:1524-1671).
 */
static void ewing_fix_flux(orc_hier *h, int ln, opatch *p, oarr U)
{
   olevel *L = &h->L[ln];
   const int dim = h->dim;
   for (int a = 0; a < dim; ++a) {
      const double tranwt = (double)(1.0f / (float)(1 + L->ratio[a]));
      const double longwt = 2 * tranwt;
      const double hh = L->dx[a];
      oarr FA = side_arr(p, ORC_SFLUX, a);
      oarr DA = {0};
      if (h->d_variable) DA = side_arr(p, ORC_SD, a);
      for (int s = 0; s < 2; ++s) {
         obox ob = oside_box(p, a, s);
         const unsigned char *m = p->cfmask[a][s];
         int ifc = s == 0 ? p->box.lo[a] : p->box.hi[a] + 1; /* face */
         int icl = s == 0 ? p->box.lo[a] : p->box.hi[a];     /* cell */
         long idx = 0;
         for (int k = ob.lo[2]; k <= ob.hi[2]; ++k)
            for (int j = ob.lo[1]; j <= ob.hi[1]; ++j)
               for (int i = ob.lo[0]; i <= ob.hi[0]; ++i, ++idx) {
                  if (!m[idx]) continue;
                  int f[3] = {i, j, k};
                  f[a] = ifc;
                  int c[3] = {i, j, k};
                  c[a] = icl;
                  int q[3] = {c[0], c[1], c[2]};
                  for (int t = 0; t < dim; ++t) {
                     if (t == a) continue;
                     int r = L->ratio[t];
                     int base = coarsen_index(c[t], r) * r;
                     int pp = c[t] - base;
                     q[t] = base + (r - pp - 1);
                  }
                  double d = h->d_variable ? AT(DA, f[0], f[1], f[2]) : h->d_const;
                  double du = AT(U, q[0], q[1], q[2]) - AT(U, c[0], c[1], c[2]);
                  double old = AT(FA, f[0], f[1], f[2]);
                  if (s == 0)
                     AT(FA, f[0], f[1], f[2]) = longwt * old + tranwt * d * du / hh;
                  else
                     AT(FA, f[0], f[1], f[2]) = longwt * old - tranwt * d * du / hh;
               }
      }
   }
}

/* CellPoissonFACOps::computeFluxOnPatch (CellPoissonFACOps.C:2157-2267). */
static void flux_on_patch(orc_hier *h, int ln, opatch *p, int fid_u)
{
   oarr U = cell_arr(h, p, fid_u);
   compute_flux_on_patch(h, p, h->L[ln].dx, U);
   if (h->ewing && ln > 0) ewing_fix_flux(h, ln, p, U);
}

/* rbgswithfluxmax*2d (2d.f:95-364) and *3d (3d.f:136-484). */
static double rbgs_on_patch(orc_hier *h, int ln, opatch *p, int fid_e,
                            int fid_r, int offset)
{
   const int dim = h->dim;
   const obox b = p->box;
   double *dx = h->L[ln].dx;
   double dxi = 1. / dx[0], dyi = 1. / dx[1];
   double dzi = dim == 3 ? 1. / dx[2] : 0.0;
   oarr U = cell_arr(h, p, fid_e), F = cell_arr(h, p, fid_r);
   oarr FX = side_arr(p, ORC_SFLUX, 0), FY = side_arr(p, ORC_SFLUX, 1), FZ = {0};
   oarr DX = {0}, DY = {0}, DZ = {0}, CF = {0};
   if (dim == 3) FZ = side_arr(p, ORC_SFLUX, 2);
   if (h->d_variable) {
      DX = side_arr(p, ORC_SD, 0);
      DY = side_arr(p, ORC_SD, 1);
      if (dim == 3) DZ = side_arr(p, ORC_SD, 2);
   }
   if (h->c_kind == 2) CF = cell_arr(h, p, ORC_C);
   const double sfc = h->c_kind == 1 ? h->c_const : 0.0;
   const double dc = h->d_const;
   const double rcoef = 1.0;
   double maxres = 0.0;
   if (dim == 2) {
      const int ifirst = b.lo[0], ilast = b.hi[0];
      const int jfirst = b.lo[1], jlast = b.hi[1];
      for (int j = jfirst; j <= jlast; ++j) {
         int ioffset = ((jfirst + j) - ((jfirst + j) / 2 * 2)) != offset ? 1 : 0;
         for (int i = ifirst + ioffset; i <= ilast; i += 2) {
            double sf = h->c_kind == 2 ? AT(CF, i, j, 0) : sfc;
            double residual =
               AT(F, i, j, 0) -
               (dxi * (AT(FX, i + 1, j, 0) - AT(FX, i, j, 0)) +
                dyi * (AT(FY, i, j + 1, 0) - AT(FY, i, j, 0))) -
               sf * AT(U, i, j, 0);
            double dudr;
            if (h->d_variable)
               dudr = 1. / ((dxi * dxi * (AT(DX, i + 1, j, 0) + AT(DX, i, j, 0)) +
                             dyi * dyi * (AT(DY, i, j + 1, 0) + AT(DY, i, j, 0))) -
                            sf);
            else
               dudr = 1. / ((dxi * dxi * (dc + dc) + dyi * dyi * (dc + dc)) - sf);
            double du = -residual * dudr;
            AT(U, i, j, 0) = AT(U, i, j, 0) + du * rcoef;
            if (maxres < fabs(residual)) maxres = fabs(residual);
         }
      }
   } else {
      const int ifirst = b.lo[0], ilast = b.hi[0];
      const double dxi2 = dxi * dxi, dyi2 = dyi * dyi, dzi2 = dzi * dzi;
      for (int k = b.lo[2]; k <= b.hi[2]; ++k)
         for (int j = b.lo[1]; j <= b.hi[1]; ++j) {
            int ioffset =
               ((ifirst + j + k) - ((ifirst + j + k) / 2 * 2)) != offset ? 1 : 0;
            for (int i = ifirst + ioffset; i <= ilast; i += 2) {
               double sf = h->c_kind == 2 ? AT(CF, i, j, k) : sfc;
               double residual =
                  AT(F, i, j, k) -
                  (dxi * (AT(FX, i + 1, j, k) - AT(FX, i, j, k)) +
                   dyi * (AT(FY, i, j + 1, k) - AT(FY, i, j, k)) +
                   dzi * (AT(FZ, i, j, k + 1) - AT(FZ, i, j, k))) -
                  sf * AT(U, i, j, k);
               double dudr;
               if (h->d_variable)
                  dudr = 1. / ((dxi2 * (AT(DX, i + 1, j, k) + AT(DX, i, j, k)) +
                                dyi2 * (AT(DY, i, j + 1, k) + AT(DY, i, j, k)) +
                                dzi2 * (AT(DZ, i, j, k + 1) + AT(DZ, i, j, k))) -
                               sf);
               else
                  dudr = 1. / ((dxi2 * (dc + dc) + dyi2 * (dc + dc) +
                                dzi2 * (dc + dc)) -
                               sf);
               double du = -residual * dudr;
               AT(U, i, j, k) = AT(U, i, j, k) + du * rcoef;
               if (maxres < fabs(residual)) maxres = fabs(residual);
            }
         }
   }
   return maxres;
}

/*
 * CellPoissonFACOps::smoothErrorByRedBlack (CellPoissonFACOps.C:1339-1514).
 * Note the reference's convergence test: redOrBlackSmoothingOnPatch assigns
 * (does not accumulate) *p_maxres (CellPoissonFACOps.C:2776), so the value
 * tested is the last patch's max residual of each colour.
 */
int orc_smooth(orc_hier *h, int fid_e, int fid_r, int ln, int nsweeps,
               double tol, double *maxres_out)
{
   olevel *L = &h->L[ln];
   orc_ghost_fill(h, fid_e, ln, 0, 1);
   if (ln > 0) orc_ghost_fill(h, fid_e, ln, 1, 1);
   double red_maxres, blk_maxres, maxres = 0;
   red_maxres = blk_maxres = tol + 1;
   int not_converged = 1;
   int isweep;
   for (isweep = 0; isweep < nsweeps && not_converged; ++isweep) {
      red_maxres = blk_maxres = 0;
      orc_ghost_fill(h, fid_e, ln, 0, 1);
      for (int ip = 0; ip < L->np; ++ip) {
         flux_on_patch(h, ln, &L->p[ip], fid_e);
         red_maxres = rbgs_on_patch(h, ln, &L->p[ip], fid_e, fid_r, 0);
      }
      orc_ghost_fill(h, fid_e, ln, 0, 1);
      for (int ip = 0; ip < L->np; ++ip) {
         flux_on_patch(h, ln, &L->p[ip], fid_e);
         blk_maxres = rbgs_on_patch(h, ln, &L->p[ip], fid_e, fid_r, 1);
      }
      orc_ghost_fill(h, fid_e, ln, 0, 1);
      if (tol >= 0.0) {
         maxres = red_maxres > blk_maxres ? red_maxres : blk_maxres;
         not_converged = maxres > tol;
      }
   }
   if (maxres_out) *maxres_out = maxres;
   return isweep;
}

/* compres{var,con}sca{2,3}d (2d.f:368-456, 3d.f:485-603). */
static void residual_on_patch(orc_hier *h, int ln, opatch *p, int fid_r,
                              int fid_u, int fid_f)
{
   const int dim = h->dim;
   const obox b = p->box;
   double *dx = h->L[ln].dx;
   double dxi = 1. / dx[0], dyi = 1. / dx[1];
   double dzi = dim == 3 ? 1. / dx[2] : 0.0;
   oarr U = cell_arr(h, p, fid_u), F = cell_arr(h, p, fid_f),
        R = cell_arr(h, p, fid_r);
   oarr FX = side_arr(p, ORC_SFLUX, 0), FY = side_arr(p, ORC_SFLUX, 1), FZ = {0}, CF = {0};
   if (dim == 3) FZ = side_arr(p, ORC_SFLUX, 2);
   if (h->c_kind == 2) CF = cell_arr(h, p, ORC_C);
   const double sfc = h->c_kind == 1 ? h->c_const : 0.0;
   for (int k = b.lo[2]; k <= b.hi[2]; ++k)
      for (int j = b.lo[1]; j <= b.hi[1]; ++j)
         for (int i = b.lo[0]; i <= b.hi[0]; ++i) {
            double sf = h->c_kind == 2 ? AT(CF, i, j, k) : sfc;
            if (dim == 2)
               AT(R, i, j, k) =
                  AT(F, i, j, k) -
                  (dxi * (AT(FX, i + 1, j, k) - AT(FX, i, j, k)) +
                   dyi * (AT(FY, i, j + 1, k) - AT(FY, i, j, k))) -
                  sf * AT(U, i, j, k);
            else
               AT(R, i, j, k) =
                  AT(F, i, j, k) -
                  (dxi * (AT(FX, i + 1, j, k) - AT(FX, i, j, k)) +
                   dyi * (AT(FY, i, j + 1, k) - AT(FY, i, j, k)) +
                   dzi * (AT(FZ, i, j, k + 1) - AT(FZ, i, j, k))) -
                  sf * AT(U, i, j, k);
         }
}

/*
 * Flux coarsening of the finer level's saved outerside flux into this
 * level's flux (xeqScheduleFluxCoarsen, CellPoissonFACOps.C:2841-2858;
 * CoarsenSchedule::coarsenData, xfer/CoarsenSchedule.C:275-330;
 * cartwgtavgoutsidedoub{2,3}d* bodies, geom_m4cartcoarsenops2d.i:233-261
 * and geom_m4cartcoarsenops3d.i:343-410; OutersideData::copy2 into
 * SideData, pdat/OutersideData.C:326-340, lower side then upper side).
 */
static void flux_coarsen(orc_hier *h, int ln)
{
   olevel *L = &h->L[ln];
   olevel *Fl = &h->L[ln + 1];
   const int dim = h->dim;
   const int *r = Fl->ratio;
   const double *dxf = Fl->dx, *dxc = L->dx;
   for (int ip = 0; ip < Fl->np; ++ip) {
      opatch *fp = &Fl->p[ip];
      obox cb = box_coarsen(fp->box, dim, r);
      for (int a = 0; a < dim; ++a) {
         int t0 = -1, t1 = -1; /* tangential axes, outer = t1 */
         for (int t = 0; t < dim; ++t)
            if (t != a) {
               if (t0 < 0) t0 = t;
               else t1 = t;
            }
         double wf, wc;
         if (dim == 2) {
            wf = dxf[t0];
            wc = dxc[t0];
         } else {
            wf = dxf[t0] * dxf[t1];
            wc = dxc[t0] * dxc[t1];
         }
         for (int s = 0; s < 2; ++s) {
            oarr FO = oside_arr(fp, a, s);
            int cface = s == 0 ? cb.lo[a] : cb.hi[a] + 1;
            int fface = s == 0 ? fp->box.lo[a] : fp->box.hi[a] + 1;
            /* coarse outerside values over cb's face */
            obox tb = cb;
            tb.lo[a] = tb.hi[a] = cface;
            for (int k = tb.lo[2]; k <= tb.hi[2]; ++k)
               for (int j = tb.lo[1]; j <= tb.hi[1]; ++j)
                  for (int i = tb.lo[0]; i <= tb.hi[0]; ++i) {
                     int c[3] = {i, j, k};
                     double acc = 0.0;
                     if (dim == 2) {
                        for (int ir = 0; ir < r[t0]; ++ir) {
                           int f[3] = {0, 0, 0};
                           f[a] = fface;
                           f[t0] = c[t0] * r[t0] + ir;
                           acc = acc + AT(FO, f[0], f[1], f[2]) * wf;
                        }
                     } else {
                        for (int ro = 0; ro < r[t1]; ++ro)
                           for (int ri = 0; ri < r[t0]; ++ri) {
                              int f[3];
                              f[a] = fface;
                              f[t0] = c[t0] * r[t0] + ri;
                              f[t1] = c[t1] * r[t1] + ro;
                              acc = acc + AT(FO, f[0], f[1], f[2]) * wf;
                           }
                     }
                     acc = acc / wc;
                     /* copy into every coarse patch side box holding it */
                     for (int iq = 0; iq < L->np; ++iq) {
                        opatch *cp = &L->p[iq];
                        obox sb = side_box(cp, a);
                        if (!box_contains(&sb, i, j, k)) continue;
                        oarr FS = side_arr(cp, ORC_SFLUX, a);
                        AT(FS, i, j, k) = acc;
                     }
                  }
         }
      }
   }
}

/* CellPoissonFACOps::computeCompositeResidualOnLevel
 * (CellPoissonFACOps.C:1792-1956). */
void orc_comp_residual(orc_hier *h, int fid_r, int fid_u, int fid_f, int ln,
                       int error_equation)
{
   olevel *L = &h->L[ln];
   /* S1 */
   orc_ghost_fill(h, fid_u, ln, ln > 0, error_equation);
   /* S2 */
   for (int ip = 0; ip < L->np; ++ip) flux_on_patch(h, ln, &L->p[ip], fid_u);
   /* S3 */
   if (ln < h->nlev - 1) flux_coarsen(h, ln);
   /* S4 */
   for (int ip = 0; ip < L->np; ++ip) {
      opatch *p = &L->p[ip];
      residual_on_patch(h, ln, p, fid_r, fid_u, fid_f);
      if (ln > 0) {
         /* OutersideData::copy(SideData) (pdat/OutersideData.C:306-322) */
         for (int a = 0; a < h->dim; ++a)
            for (int s = 0; s < 2; ++s) {
               oarr O = oside_arr(p, a, s), S = side_arr(p, ORC_SFLUX, a);
               obox ob = oside_box(p, a, s);
               for (int k = ob.lo[2]; k <= ob.hi[2]; ++k)
                  for (int j = ob.lo[1]; j <= ob.hi[1]; ++j)
                     for (int i = ob.lo[0]; i <= ob.hi[0]; ++i)
                        AT(O, i, j, k) = AT(S, i, j, k);
            }
      }
   }
}

/* ------------------------------------------------------------------ */
/* inter-level transfer                                                 */
/* ------------------------------------------------------------------ */

/*
 * Volume-weighted restriction cartwgtavgcelldoub{2,3}d
 * (geom_m4cartcoarsenops2d.i:31-69, geom_m4cartcoarsenops3d.i:31-76):
 * accumulate arrayf*dVf in loop order (ir2,) ir1, ir0, then divide by dVc.
 * The coarsened values are copied into every coarse patch over the
 * destination's ghost box (CoarsenSchedule overlap with dst_fill_box = dst
 * ghost box, xfer/CoarsenSchedule.C:886-940).
 */
void orc_restrict(orc_hier *h, int fid_src, int fid_dst, int dest_ln)
{
   olevel *C = &h->L[dest_ln];
   olevel *Fl = &h->L[dest_ln + 1];
   const int dim = h->dim;
   const int *r = Fl->ratio;
   double dVf = Fl->dx[0] * Fl->dx[1];
   double dVc = C->dx[0] * C->dx[1];
   if (dim == 3) {
      dVf = Fl->dx[0] * Fl->dx[1] * Fl->dx[2];
      dVc = C->dx[0] * C->dx[1] * C->dx[2];
   }
   for (int ip = 0; ip < Fl->np; ++ip) {
      opatch *fp = &Fl->p[ip];
      oarr S = cell_arr(h, fp, fid_src);
      obox cb = box_coarsen(fp->box, dim, r);
      for (int k = cb.lo[2]; k <= cb.hi[2]; ++k)
         for (int j = cb.lo[1]; j <= cb.hi[1]; ++j)
            for (int i = cb.lo[0]; i <= cb.hi[0]; ++i) {
               double acc = 0.0;
               int r2 = dim == 3 ? r[2] : 1;
               for (int i2 = 0; i2 < r2; ++i2)
                  for (int i1 = 0; i1 < r[1]; ++i1)
                     for (int i0 = 0; i0 < r[0]; ++i0) {
                        int f2 = dim == 3 ? k * r[2] + i2 : 0;
                        acc = acc + AT(S, i * r[0] + i0, j * r[1] + i1, f2) * dVf;
                     }
               acc = acc / dVc;
               for (int iq = 0; iq < C->np; ++iq) {
                  opatch *cp = &C->p[iq];
                  obox gb = cell_gbox(h, cp, fid_dst);
                  if (!box_contains(&gb, i, j, k)) continue;
                  oarr D = cell_arr(h, cp, fid_dst);
                  AT(D, i, j, k) = acc;
               }
            }
   }
}

/* CellPoissonFACOps::restrictSolution (CellPoissonFACOps.C:1197-1220). */
void orc_restrict_solution(orc_hier *h, int fid, int dest_ln)
{
   orc_restrict(h, fid, fid, dest_ln);
   orc_ghost_fill(h, fid, dest_ln, dest_ln > 0, 0);
}

/*
 * CellPoissonFACOps::prolongErrorAndCorrect (CellPoissonFACOps.C:1254-1304):
 * linear refine (cartlinrefcelldoub{2,3}d, geom_m4cartrefineops2d.i:64-98,
 * geom_m4cartrefineops3d.i:64-116; deltax from geom_m4cartopstuff.i:39-43)
 * of a coarse interpolation patch, then e_fine += scratch over the patch
 * interior (HierarchyCellDataOpsReal::add).  The coarse interpolation patch
 * (RefineSchedule::setupCoarseInterpBoxLevel, xfer/RefineSchedule.C:
 * 1353-1560) covers coarsen(fine box grown by the scratch ghost width),
 * sheared to the domain; it is filled from the coarser level's interiors
 * and then gets homogeneous physical boundary values on its ghost layer.
 */
void orc_prolong_correct(orc_hier *h, int fid_src, int fid_dst, int dest_ln)
{
   olevel *Fl = &h->L[dest_ln];
   olevel *C = &h->L[dest_ln - 1];
   const int dim = h->dim;
   const int *r = Fl->ratio;
   const double *dxf = Fl->dx, *dxc = C->dx;
   const double half = 0.5, one = 1.0;
   double deltax[3][16];
   for (int a = 0; a < dim; ++a)
      for (int ir = 0; ir < r[a]; ++ir)
         deltax[a][ir] = ((double)ir + half) * dxf[a] - dxc[a] * half;
   for (int ip = 0; ip < Fl->np; ++ip) {
      opatch *fp = &Fl->p[ip];
      /* coarse interpolation patch */
      obox fill = box_grow(fp->box, dim, 1);
      obox B = box_isect(box_coarsen(fill, dim, r), C->domain);
      obox Bg = box_grow(B, dim, 1);
      long n = box_size(&Bg);
      double *tmp = (double *)malloc((size_t)n * sizeof(double));
      for (long t = 0; t < n; ++t) tmp[t] = NAN;
      oarr T = arr_from_box(tmp, Bg);
      for (int iq = 0; iq < C->np; ++iq) {
         opatch *cp = &C->p[iq];
         obox ov = box_isect(Bg, cp->box);
         if (box_empty(&ov)) continue;
         oarr S = cell_arr(h, cp, fid_src);
         for (int k = ov.lo[2]; k <= ov.hi[2]; ++k)
            for (int j = ov.lo[1]; j <= ov.hi[1]; ++j)
               for (int i = ov.lo[0]; i <= ov.hi[0]; ++i)
                  AT(T, i, j, k) = AT(S, i, j, k);
      }
      bc_fill_box(h, T, B, &C->domain, C->dx, 1, h->bcf[dest_ln - 1]);
      oarr D = cell_arr(h, fp, fid_dst);
      const obox b = fp->box;
      for (int k = b.lo[2]; k <= b.hi[2]; ++k) {
         int ic2 = 0;
         double z = 0.0;
         if (dim == 3) {
            ic2 = coarsen_index(k, r[2]);
            int ir2 = k - ic2 * r[2];
            z = deltax[2][ir2] / dxc[2];
            if (z < 0.0) {
               ic2 = ic2 - 1;
               z = z + one;
            }
         }
         for (int j = b.lo[1]; j <= b.hi[1]; ++j) {
            int ic1 = coarsen_index(j, r[1]);
            int ir1 = j - ic1 * r[1];
            double y = deltax[1][ir1] / dxc[1];
            if (y < 0.0) {
               ic1 = ic1 - 1;
               y = y + one;
            }
            for (int i = b.lo[0]; i <= b.hi[0]; ++i) {
               int ic0 = coarsen_index(i, r[0]);
               int ir0 = i - ic0 * r[0];
               double x = deltax[0][ir0] / dxc[0];
               if (x < 0.0) {
                  ic0 = ic0 - 1;
                  x = x + one;
               }
               double v;
               if (dim == 2) {
                  v = (AT(T, ic0, ic1, 0) +
                       (AT(T, ic0 + 1, ic1, 0) - AT(T, ic0, ic1, 0)) * x) *
                         (one - y) +
                      (AT(T, ic0, ic1 + 1, 0) +
                       (AT(T, ic0 + 1, ic1 + 1, 0) - AT(T, ic0, ic1 + 1, 0)) * x) *
                         y;
               } else {
                  v = ((AT(T, ic0, ic1, ic2) +
                        (AT(T, ic0 + 1, ic1, ic2) - AT(T, ic0, ic1, ic2)) * x) *
                          (one - y) +
                       (AT(T, ic0, ic1 + 1, ic2) +
                        (AT(T, ic0 + 1, ic1 + 1, ic2) - AT(T, ic0, ic1 + 1, ic2)) * x) *
                          y) *
                         (one - z) +
                      ((AT(T, ic0, ic1, ic2 + 1) +
                        (AT(T, ic0 + 1, ic1, ic2 + 1) - AT(T, ic0, ic1, ic2 + 1)) * x) *
                          (one - y) +
                       (AT(T, ic0, ic1 + 1, ic2 + 1) +
                        (AT(T, ic0 + 1, ic1 + 1, ic2 + 1) - AT(T, ic0, ic1 + 1, ic2 + 1)) *
                           x) *
                          y) *
                         z;
               }
               AT(D, i, j, k) = AT(D, i, j, k) + v;
            }
         }
      }
      free(tmp);
   }
}

/* ------------------------------------------------------------------ */
/* norms and weights                                                    */
/* ------------------------------------------------------------------ */

/* CellPoissonFACOps::computeVectorWeights (CellPoissonFACOps.C:2005-2102). */
void orc_compute_weights(orc_hier *h)
{
   const int dim = h->dim;
   for (int ln = h->nlev - 1; ln >= 0; --ln) {
      olevel *L = &h->L[ln];
      double vol = L->dx[0];
      vol *= L->dx[1];
      if (dim > 2) vol *= L->dx[2];
      for (int ip = 0; ip < L->np; ++ip) {
         opatch *p = &L->p[ip];
         long n = box_size(&p->box);
         for (long t = 0; t < n; ++t) p->cell[ORC_W][t] = vol;
      }
      if (ln < h->nlev - 1) {
         olevel *Fl = &h->L[ln + 1];
         for (int ip = 0; ip < L->np; ++ip) {
            opatch *p = &L->p[ip];
            oarr W = cell_arr(h, p, ORC_W);
            for (int iq = 0; iq < Fl->np; ++iq) {
               obox cb = box_coarsen(Fl->p[iq].box, dim, Fl->ratio);
               obox ov = box_isect(cb, p->box);
               if (box_empty(&ov)) continue;
               for (int k = ov.lo[2]; k <= ov.hi[2]; ++k)
                  for (int j = ov.lo[1]; j <= ov.hi[1]; ++j)
                     for (int i = ov.lo[0]; i <= ov.hi[0]; ++i)
                        AT(W, i, j, k) = 0.0;
            }
         }
      }
   }
}

/* SAMRAIVectorReal::RMSNorm (solv/SAMRAIVectorReal.C:821-840) with
 * HierarchyCellDataOpsReal::dot and sumControlVolumes
 * (math/HierarchyCellDataOpsReal.C:777-890, 1036-1090). */
double orc_rms_norm(const orc_hier *h, int fid)
{
   double dot = 0.0, vol = 0.0;
   for (int ln = 0; ln < h->nlev; ++ln) {
      const olevel *L = &h->L[ln];
      for (int ip = 0; ip < L->np; ++ip) {
         const opatch *p = &L->p[ip];
         oarr X = cell_arr(h, p, fid);
         oarr W = cell_arr(h, p, ORC_W);
         const obox b = p->box;
         double pd = 0.0, pv = 0.0;
         for (int k = b.lo[2]; k <= b.hi[2]; ++k)
            for (int j = b.lo[1]; j <= b.hi[1]; ++j)
               for (int i = b.lo[0]; i <= b.hi[0]; ++i) {
                  double x = AT(X, i, j, k), w = AT(W, i, j, k);
                  pd += x * x * w;
                  pv += w;
               }
         dot += pd;
         vol += pv;
      }
   }
   double num = sqrt(dot);
   return vol > 0.0 ? num / sqrt(vol) : 0.0;
}

/* ------------------------------------------------------------------ */
/* FAC algorithm (FACPreconditioner.C)                                  */
/* ------------------------------------------------------------------ */

/* CellPoissonFACOps::solveCoarsestLevel, redblack choice
 * (CellPoissonFACOps.C:1681-1730). */
int orc_solve_coarsest(orc_hier *h, int fid_e, int fid_r, int ln)
{
   int n = orc_smooth(h, fid_e, fid_r, ln, h->coarse_max_it, h->coarse_tol,
                      NULL);
   h->coarse_sweeps += n;
   orc_ghost_fill(h, fid_e, ln, 0, 1);
   return 0;
}

/* FACPreconditioner::facCycle_Recursive (FACPreconditioner.C:462-518). */
static void fac_cycle_recursive(orc_hier *h, int ln)
{
   if (ln == 0) {
      orc_solve_coarsest(h, ORC_E, ORC_R, ln);
   } else {
      orc_smooth(h, ORC_E, ORC_R, ln, h->pre_sweeps, -1.0, NULL);
      orc_comp_residual(h, ORC_TR, ORC_E, ORC_R, ln, 1);
      orc_restrict(h, ORC_TR, ORC_R, ln - 1);
      fac_cycle_recursive(h, ln - 1);
      orc_prolong_correct(h, ORC_E, ORC_E, ln);
      orc_smooth(h, ORC_E, ORC_R, ln, h->post_sweeps, -1.0, NULL);
   }
}

void orc_fac_cycle(orc_hier *h) { fac_cycle_recursive(h, h->nlev - 1); }

/* FACPreconditioner::computeFullCompositeResidual (FACPreconditioner.C:775-814). */
static double full_composite_residual(orc_hier *h)
{
   int lmax = h->nlev - 1;
   orc_comp_residual(h, ORC_R, ORC_U, ORC_F, lmax, 0);
   for (int ln = lmax - 1; ln >= 0; --ln) {
      orc_restrict_solution(h, ORC_U, ln);
      orc_comp_residual(h, ORC_R, ORC_U, ORC_F, ln, 0);
      orc_restrict(h, ORC_R, ORC_R, ln);
   }
   return orc_rms_norm(h, ORC_R);
}

static void set_zero(orc_hier *h, int fid, int with_ghosts)
{
   for (int ln = 0; ln < h->nlev; ++ln) {
      olevel *L = &h->L[ln];
      for (int ip = 0; ip < L->np; ++ip) {
         opatch *p = &L->p[ip];
         if (with_ghosts) {
            obox gb = cell_gbox(h, p, fid);
            memset(p->cell[fid], 0, (size_t)box_size(&gb) * sizeof(double));
         } else {
            oarr A = cell_arr(h, p, fid);
            const obox b = p->box;
            for (int k = b.lo[2]; k <= b.hi[2]; ++k)
               for (int j = b.lo[1]; j <= b.hi[1]; ++j)
                  for (int i = b.lo[0]; i <= b.hi[0]; ++i) AT(A, i, j, k) = 0.0;
         }
      }
   }
}

/*
 * SimpleCellRobinBcCoefs::cacheDirichletData / restoreDirichletData
 * (solv/SimpleCellRobinBcCoefs.C:488-560): the ghost values of u on the
 * codimension-1 physical boundary boxes are saved before the solve and
 * written back afterwards.  Boundary boxes extend one cell tangentially
 * inside the domain (BaseGridGeometry::getBoundaryBoxes).
 */
static void dirichlet_cache(orc_hier *h, int restore)
{
   const int dim = h->dim;
   for (int ln = 0; ln < h->nlev; ++ln) {
      olevel *L = &h->L[ln];
      long count = 0;
      for (int pass = 0; pass < 2; ++pass) {
         long t = 0;
         for (int ip = 0; ip < L->np; ++ip) {
            opatch *p = &L->p[ip];
            oarr U = cell_arr(h, p, ORC_U);
            obox gb = box_grow(p->box, dim, 1);
            for (int k = gb.lo[2]; k <= gb.hi[2]; ++k)
               for (int j = gb.lo[1]; j <= gb.hi[1]; ++j)
                  for (int i = gb.lo[0]; i <= gb.hi[0]; ++i) {
                     int c[3] = {i, j, k}, out = 0, ok = 1;
                     for (int a = 0; a < dim; ++a) {
                        if (c[a] < L->domain.lo[a] || c[a] > L->domain.hi[a]) {
                           if (!((c[a] == p->box.lo[a] - 1 &&
                                  p->box.lo[a] == L->domain.lo[a]) ||
                                 (c[a] == p->box.hi[a] + 1 &&
                                  p->box.hi[a] == L->domain.hi[a])))
                              ok = 0;
                           ++out;
                        }
                     }
                     if (!ok || out != 1) continue;
                     if (pass == 0) {
                        ++count;
                     } else if (restore) {
                        AT(U, i, j, k) = h->cached[ln][t++];
                     } else {
                        h->cached[ln][t++] = AT(U, i, j, k);
                     }
                  }
         }
         if (pass == 0) {
            if (!restore) {
               free(h->cached[ln]);
               h->cached[ln] = (double *)malloc((size_t)(count + 1) * sizeof(double));
            }
         }
      }
   }
}

/* FACPreconditioner::solveSystem (FACPreconditioner.C:277-452) wrapped by
 * CellPoissonFACSolver::solveSystem (CellPoissonFACSolver.C:310-352). */
int orc_solve(orc_hier *h, int *iterations, double *residual_norm,
              double *hist)
{
   dirichlet_cache(h, 0);
   orc_compute_weights(h);
   set_zero(h, ORC_E, 1);
   set_zero(h, ORC_R, 0);
   double initial = full_composite_residual(h);
   double res = initial;
   if (hist) hist[0] = res;
   double eff_tol = h->residual_tol;
   if (h->rel_residual_tol >= 0) {
      double tmp = orc_rms_norm(h, ORC_F) * h->rel_residual_tol;
      if (eff_tol < tmp) eff_tol = tmp;
   }
   int it = 0;
   do {
      set_zero(h, ORC_E, 1);
      fac_cycle_recursive(h, h->nlev - 1);
      for (int ln = 0; ln < h->nlev; ++ln) {
         olevel *L = &h->L[ln];
         for (int ip = 0; ip < L->np; ++ip) {
            opatch *p = &L->p[ip];
            oarr U = cell_arr(h, p, ORC_U), E = cell_arr(h, p, ORC_E);
            const obox b = p->box;
            for (int k = b.lo[2]; k <= b.hi[2]; ++k)
               for (int j = b.lo[1]; j <= b.hi[1]; ++j)
                  for (int i = b.lo[0]; i <= b.hi[0]; ++i)
                     AT(U, i, j, k) = AT(U, i, j, k) + AT(E, i, j, k);
         }
      }
      for (int ln = h->nlev - 2; ln >= 0; --ln) orc_restrict_solution(h, ORC_U, ln);
      res = full_composite_residual(h);
      ++it;
      if (hist) hist[it] = res;
   } while (res > eff_tol && it < h->max_cycles);
   dirichlet_cache(h, 1);
   if (iterations) *iterations = it;
   if (residual_norm) *residual_norm = res;
   return res < eff_tol;
}

long orc_coarse_sweeps(const orc_hier *h) { return h->coarse_sweeps; }
void orc_reset_stats(orc_hier *h) { h->coarse_sweeps = 0; }

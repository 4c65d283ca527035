/*
 * mg_oracle.c -- CPU oracle: a plain-C restatement of the reference's
 * multigrid Poisson--Helmholtz solver.
 *
 * TEST INFRASTRUCTURE ONLY (see mg_oracle.h).  The checker and the CPU
 * baseline; never part of the product path.
 *
 * What it restates, by reference file:line (paths inside the Basilisk tree):
 *   level layout, GHOSTS = 2, C-order index   grid/multigrid.h:2,49-73
 *   parent/child index arithmetic             grid/multigrid.h:136-157
 *   loop order of foreach_level / foreach     grid/multigrid.h:191-241
 *   box boundary conditions, BGHOSTS = 1,     grid/multigrid.h:543-594,
 *     sides right,left,top,bottom,front,back    common.h:949-960
 *   periodic ghost copies (2 layers, level 0) grid/multigrid.h:638-695
 *   boundary list order: box, then periodic   grid/multigrid.h:733-745
 *   cell/face restriction, bilinear           grid/multigrid-common.h:26-63,
 *                                               124-140, 368-404
 *   coordinates and Delta                      grid/cartesian-common.h:10-34
 *   mg_cycle                                  poisson.h:32-90
 *   mg_solve (nrelax adaptation, warning)     poisson.h:139-235
 *   relax (GS / JACOBI)                       poisson.h:271-338
 *   residual (uniform-grid branch)            poisson.h:373-389
 *   poisson()                                 poisson.h:402-441
 *
 * Arithmetic is written in the reference's evaluation order so that the
 * results are reproducible bit for bit by any implementation that keeps the
 * same order (build with -ffp-contract=off).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "mg_oracle.h"

#ifndef DIM
#define DIM 2
#endif

#define GH 2          /* grid/multigrid.h:2 */
#define sq_(x) ((x)*(x))   /* common.h:58 */
#define MAXLEVEL 16

int og_NITERMAX = 100, og_NITERMIN = 1;   /* poisson.h:102 */
double og_TOLERANCE = 1e-3;               /* poisson.h:103 */

typedef struct {
  double * lv[MAXLEVEL + 1];
} field;

struct og_grid {
  int depth;
  double L0, X0, Y0, Z0;
  int periodic[3];
  int bctype[6];
  double bcconst[6];
  double * bcval[6];          /* finest-level values, NULL = bcconst */
  int relax_mode;
  field a, b, res, da, c, lambda, alpha[DIM], uf[DIM];
  /* viscosity: u, its r.h.s., correction, residual, work; mu, rho */
  field vu[DIM], vr[DIM], vda[DIM], vres[DIM], vw[DIM], mu[DIM], rho;
  int vbctype[DIM][6];
  double vbcval[DIM][6];
  int mu_const, rho_const;
  double mu_c, rho_c;
  int alpha_const, lambda_const;
  double alpha_c, lambda_c;
};

int og_dimension (void) { return DIM; }

static inline int P_of (int l) { return (1 << l) + 2*GH; }

static size_t level_size (int l)
{
  size_t P = P_of (l), s = 1;
  for (int d = 0; d < DIM; d++) s *= P;
  return s;
}

static inline size_t IX (int P, int i, int j, int k)
{
#if DIM == 1
  (void) P; (void) j; (void) k;
  return i;
#elif DIM == 2
  (void) k;
  return (size_t) i*P + j;
#else
  return ((size_t) i*P + j)*P + k;
#endif
}

/* strides of dimension d at a level with padded extent P */
static inline size_t stride (int P, int d)
{
  size_t s = 1;
  for (int e = DIM - 1; e > d; e--) s *= P;
  return s;
}

static void field_alloc (og_grid * g, field * f)
{
  for (int l = 0; l <= g->depth; l++) {
    size_t n = level_size (l);
    f->lv[l] = malloc (n*sizeof (double));
    for (size_t i = 0; i < n; i++) f->lv[l][i] = 0.;
  }
}

static void field_free (og_grid * g, field * f)
{
  for (int l = 0; l <= g->depth; l++)
    free (f->lv[l]);
}

static field * field_of (og_grid * g, int which)
{
  switch (which) {
  case OG_A: return &g->a;
  case OG_B: return &g->b;
  case OG_RES: return &g->res;
  case OG_LAMBDA: return &g->lambda;
  case OG_DA: return &g->da;
  case OG_ALPHA_X: return &g->alpha[0];
  case OG_UF_X: return &g->uf[0];
  case OG_U_X: return &g->vu[0];
  case OG_MU_X: return &g->mu[0];
  case OG_RHO: return &g->rho;
#if DIM > 1
  case OG_ALPHA_Y: return &g->alpha[1];
  case OG_UF_Y: return &g->uf[1];
  case OG_U_Y: return &g->vu[1];
  case OG_MU_Y: return &g->mu[1];
#endif
#if DIM > 2
  case OG_ALPHA_Z: return &g->alpha[2];
  case OG_UF_Z: return &g->uf[2];
  case OG_U_Z: return &g->vu[2];
  case OG_MU_Z: return &g->mu[2];
#endif
  }
  return NULL;
}

og_grid * og_new (int depth, double L0, double X0, double Y0, double Z0)
{
  if (depth < 0 || depth > MAXLEVEL) return NULL;
  og_grid * g = calloc (1, sizeof (og_grid));
  g->depth = depth;
  g->L0 = L0; g->X0 = X0; g->Y0 = Y0; g->Z0 = Z0;
  for (int d = 0; d < 6; d++) g->bctype[d] = OG_NEUMANN; /* symmetry */
  field_alloc (g, &g->a); field_alloc (g, &g->b); field_alloc (g, &g->res);
  field_alloc (g, &g->da); field_alloc (g, &g->c); field_alloc (g, &g->lambda);
  for (int d = 0; d < DIM; d++) {
    field_alloc (g, &g->alpha[d]); field_alloc (g, &g->uf[d]);
    field_alloc (g, &g->vu[d]); field_alloc (g, &g->vr[d]); field_alloc (g, &g->vda[d]);
    field_alloc (g, &g->vres[d]); field_alloc (g, &g->vw[d]); field_alloc (g, &g->mu[d]);
    for (int s = 0; s < 6; s++) g->vbctype[d][s] = OG_NEUMANN;
  }
  field_alloc (g, &g->rho);
  g->mu_const = 1; g->mu_c = 1.; g->rho_const = 1; g->rho_c = 1.;
  g->alpha_const = 1; g->alpha_c = 1.;   /* unityf, common.h:1276 */
  g->lambda_const = 1; g->lambda_c = 0.; /* zeroc, common.h:1277 */
  return g;
}

void og_free (og_grid * g)
{
  if (!g) return;
  field_free (g, &g->a); field_free (g, &g->b); field_free (g, &g->res);
  field_free (g, &g->da); field_free (g, &g->c); field_free (g, &g->lambda);
  for (int d = 0; d < DIM; d++) {
    field_free (g, &g->alpha[d]); field_free (g, &g->uf[d]);
    field_free (g, &g->vu[d]); field_free (g, &g->vr[d]); field_free (g, &g->vda[d]);
    field_free (g, &g->vres[d]); field_free (g, &g->vw[d]); field_free (g, &g->mu[d]);
  }
  field_free (g, &g->rho);
  for (int d = 0; d < 6; d++) free (g->bcval[d]);
  free (g);
}

void og_set_periodic (og_grid * g, int dim)
{
  if (dim >= 0 && dim < DIM) {
    g->periodic[dim] = 1;
    g->bctype[2*dim] = g->bctype[2*dim + 1] = OG_PERIODIC;
  }
}

void og_set_bc (og_grid * g, int side, int type, double value, const double * values)
{
  if (side < 0 || side >= 2*DIM) return;
  g->bctype[side] = type;
  g->bcconst[side] = value;
  free (g->bcval[side]);
  g->bcval[side] = NULL;
  if (values) {
    size_t n = 1;
    for (int d = 1; d < DIM; d++) n *= (1 << g->depth);
    g->bcval[side] = malloc (n*sizeof (double));
    memcpy (g->bcval[side], values, n*sizeof (double));
  }
  if (type == OG_PERIODIC) g->periodic[side/2] = 1;
}

void og_set_relax (og_grid * g, int mode) { g->relax_mode = mode; }

void og_set_threads (int n)
{
#ifdef _OPENMP
  omp_set_num_threads (n > 0 ? n : 1);
#else
  (void) n;
#endif
}

int og_get_threads (void)
{
#ifdef _OPENMP
  return omp_get_max_threads ();
#else
  return 1;
#endif
}

void og_set_alpha_const (og_grid * g, double v) { g->alpha_const = 1; g->alpha_c = v; }
void og_set_lambda_const (og_grid * g, double v) { g->lambda_const = 1; g->lambda_c = v; }

/* ------------------------------------------------------------------ */
/* Boundary conditions                                                 */
/* ------------------------------------------------------------------ */

/* value of the boundary data of side d at tangential padded coordinates
   (t1, t2), clamped to the interior (ghost tangential positions only occur
   in corners, which the solver never reads for inhomogeneous fields). */
static double bc_value (og_grid * g, int side, int n, int t1, int t2)
{
  if (!g->bcval[side]) return g->bcconst[side];
  int u = t1 - GH, v = t2 - GH;
  if (u < 0) u = 0; if (u > n - 1) u = n - 1;
  if (v < 0) v = 0; if (v > n - 1) v = n - 1;
#if DIM == 1
  (void) u; (void) v;
  return g->bcval[side][0];
#elif DIM == 2
  (void) v;
  return g->bcval[side][u];
#else
  return g->bcval[side][(size_t) u*n + v];
#endif
}

/* box_boundary_level (grid/multigrid.h:543-594) for one cell-centred field:
   sides in enum order, one ghost layer, full tangential range. */
static void box_boundary (og_grid * g, double * s, int l, int homogeneous)
{
  int n = 1 << l, P = P_of (l);
  double Delta = g->L0*(1./(1 << l));
  for (int side = 0; side < 2*DIM; side++) {
    int dim = side/2;
    if (g->periodic[dim]) continue;
    int type = g->bctype[side];
    int c = (side % 2 == 0) ? n + GH - 1 : GH;   /* boundary cell */
    int gi = (side % 2 == 0) ? c + 1 : c - 1;    /* its ghost */
    int T1 = DIM > 1 ? P : 1, T2 = DIM > 2 ? P : 1;
#pragma omp parallel for schedule(static)
    for (int t1 = 0; t1 < T1; t1++)
      for (int t2 = 0; t2 < T2; t2++) {
        int p[3], q[3];
        /* tangential coordinates in increasing dimension order */
        int tt[2] = {t1, t2}, m = 0;
        for (int e = 0; e < DIM; e++)
          if (e == dim) { p[e] = c; q[e] = gi; }
          else { p[e] = q[e] = tt[m++]; }
        for (int e = DIM; e < 3; e++) p[e] = q[e] = 0;
        double v = s[IX (P, p[0], p[1], p[2])], r;
        if (homogeneous)
          r = type == OG_DIRICHLET ? - v : v;   /* common.h:958,960 */
        else {
          double val = bc_value (g, side, n, tt[0], tt[1]);
          if (type == OG_DIRICHLET)
            r = 2.*(val) - v;                  /* common.h:957 */
          else
            r = Delta*(val) + v;               /* common.h:959 */
        }
        s[IX (P, q[0], q[1], q[2])] = r;
      }
  }
}

/* periodic_boundary_level_x (grid/multigrid.h:638-695), applied for x, y, z
   in that order; at level 0 every neighbour takes the cell value. */
static void periodic_boundary (og_grid * g, double * s, int l)
{
  int n = 1 << l, P = P_of (l);
  for (int dim = 0; dim < DIM; dim++) {
    if (!g->periodic[dim]) continue;
    if (l == 0) {
      double v = s[IX (P, GH, GH, GH)];
      for (int i = 0; i < P; i++)
        for (int j = 0; j < (DIM > 1 ? P : 1); j++)
          for (int k = 0; k < (DIM > 2 ? P : 1); k++)
            s[IX (P, i, j, k)] = v;
      continue;
    }
    size_t sd = stride (P, dim);
    int T1 = DIM > 1 ? P : 1, T2 = DIM > 2 ? P : 1;
#pragma omp parallel for schedule(static)
    for (int t1 = 0; t1 < T1; t1++)
      for (int t2 = 0; t2 < T2; t2++) {
        int tt[2] = {t1, t2}, m = 0, p[3] = {0, 0, 0};
        for (int e = 0; e < DIM; e++)
          p[e] = (e == dim) ? 0 : tt[m++];
        size_t base = IX (P, p[0], p[1], p[2]);
        for (int i = 0; i < GH; i++)
          s[base + i*sd] = s[base + (i + n)*sd];
        for (int i = n + GH; i < n + 2*GH; i++)
          s[base + i*sd] = s[base + (i - n)*sd];
      }
  }
}

static void boundary_level (og_grid * g, double * s, int l, int homogeneous)
{
  box_boundary (g, s, l, homogeneous);
  periodic_boundary (g, s, l);
}

void og_boundary_level (og_grid * g, int which, int level, int homogeneous)
{
  field * f = field_of (g, which);
  if (f && level >= 0 && level <= g->depth)
    boundary_level (g, f->lv[level], level, homogeneous);
}

/* face vectors: only periodic copies apply (box BCs of face vectors are
   NULL, cartesian-common.h:566-576; periodic_boundary copies them). */
static void face_boundary (og_grid * g, int l)
{
  for (int d = 0; d < DIM; d++)
    periodic_boundary (g, g->alpha[d].lv[l], l);
}

/* ------------------------------------------------------------------ */
/* Field I/O                                                           */
/* ------------------------------------------------------------------ */

static void copy_in (og_grid * g, double * s, int l, const double * v, int face_dim)
{
  int n = 1 << l, P = P_of (l);
  int ni = n + (face_dim == 0), nj = DIM > 1 ? n + (face_dim == 1) : 1,
    nk = DIM > 2 ? n + (face_dim == 2) : 1;
  size_t m = 0;
  for (int i = 0; i < ni; i++)
    for (int j = 0; j < nj; j++)
      for (int k = 0; k < nk; k++)
        s[IX (P, i + GH, j + GH, k + GH)] = v[m++];
}

static void copy_out (og_grid * g, const double * s, int l, double * v, int face_dim)
{
  int n = 1 << l, P = P_of (l);
  int ni = n + (face_dim == 0), nj = DIM > 1 ? n + (face_dim == 1) : 1,
    nk = DIM > 2 ? n + (face_dim == 2) : 1;
  size_t m = 0;
  for (int i = 0; i < ni; i++)
    for (int j = 0; j < nj; j++)
      for (int k = 0; k < nk; k++)
        v[m++] = s[IX (P, i + GH, j + GH, k + GH)];
}

static int face_dim_of (int which)
{
  return which == OG_ALPHA_X || which == OG_UF_X || which == OG_MU_X ? 0 :
    which == OG_ALPHA_Y || which == OG_UF_Y || which == OG_MU_Y ? 1 :
    which == OG_ALPHA_Z || which == OG_UF_Z || which == OG_MU_Z ? 2 : -1;
}

void og_set_field (og_grid * g, int which, const double * values)
{
  field * f = field_of (g, which);
  if (!f) return;
  int fd = face_dim_of (which);
  copy_in (g, f->lv[g->depth], g->depth, values, fd);
  if (fd >= 0) {
    if (which >= OG_ALPHA_X && which <= OG_ALPHA_Z) g->alpha_const = 0;
    if (which >= OG_MU_X && which <= OG_MU_Z) g->mu_const = 0;
    /* the automatic boundary of a dirty face vector copies periodic
       ghosts before the first stencil read (stencils.h:228+). */
    periodic_boundary (g, f->lv[g->depth], g->depth);
  }
  if (which == OG_LAMBDA) g->lambda_const = 0;
  if (which == OG_RHO) g->rho_const = 0;
}

void og_get_field (og_grid * g, int which, double * out)
{
  field * f = field_of (g, which);
  if (f) copy_out (g, f->lv[g->depth], g->depth, out, face_dim_of (which));
}

void og_get_level (og_grid * g, int which, int level, double * out)
{
  field * f = field_of (g, which);
  if (f && level >= 0 && level <= g->depth)
    copy_out (g, f->lv[level], level, out, face_dim_of (which));
}

void og_set_level (og_grid * g, int which, int level, const double * values)
{
  field * f = field_of (g, which);
  if (f && level >= 0 && level <= g->depth)
    copy_in (g, f->lv[level], level, values, face_dim_of (which));
}

/* ------------------------------------------------------------------ */
/* Inter-level operators                                               */
/* ------------------------------------------------------------------ */

/* restriction_average (grid/multigrid-common.h:26-32), children in
   foreach_child order (grid/multigrid.h:323-338). */
static void restrict_average (og_grid * g, double * coarse, const double * fine, int l)
{
  int n = 1 << l, P = P_of (l), Pf = P_of (l + 1);
#pragma omp parallel for schedule(static)
  for (int i = GH; i < n + GH; i++)
    for (int j = (DIM > 1 ? GH : 0); j < (DIM > 1 ? n + GH : 1); j++)
      for (int k = (DIM > 2 ? GH : 0); k < (DIM > 2 ? n + GH : 1); k++) {
        double sum = 0.;
        int fi = 2*i - GH, fj = 2*j - GH, fk = 2*k - GH;
#if DIM == 1
        for (int a = 0; a < 2; a++) sum += fine[IX (Pf, fi + a, 0, 0)];
#elif DIM == 2
        for (int a = 0; a < 2; a++)
          for (int b = 0; b < 2; b++)
            sum += fine[IX (Pf, fi + a, fj + b, 0)];
#else
        for (int a = 0; a < 2; a++)
          for (int b = 0; b < 2; b++)
            for (int c = 0; c < 2; c++)
              sum += fine[IX (Pf, fi + a, fj + b, fk + c)];
#endif
        (void) fj; (void) fk;
        coarse[IX (P, i, j, k)] = sum/(1 << DIM);
      }
}

/* fine(v, o0, o1, o2) of the coarse cell (i, j, k) */
static inline double finev (const double * f, int Pf, int i, int j, int k,
                            int o0, int o1, int o2)
{
  return f[IX (Pf, 2*i - GH + o0, DIM > 1 ? 2*j - GH + o1 : 0,
               DIM > 2 ? 2*k - GH + o2 : 0)];
}

/* face_average (grid/multigrid-common.h:42-58), with the index rotation
   that foreach_dimension applies to the fine() offsets (rotate.lex). */
static void restrict_faces_of (og_grid * g, field * comps, int l)
{
  int n = 1 << l, P = P_of (l), Pf = P_of (l + 1);
#pragma omp parallel for schedule(static)
  for (int i = GH; i < n + GH; i++)
    for (int j = (DIM > 1 ? GH : 0); j < (DIM > 1 ? n + GH : 1); j++)
      for (int k = (DIM > 2 ? GH : 0); k < (DIM > 2 ? n + GH : 1); k++) {
        for (int d = 0; d < DIM; d++) {
          const double * f = comps[d].lv[l + 1];
          double * c = comps[d].lv[l];
          size_t sd = stride (P, d), id = IX (P, i, j, k);
          for (int side = 0; side < 2; side++) {
            int o = 2*side;
            double v;
#if DIM == 1
            v = finev (f, Pf, i, j, k, o, 0, 0);
#elif DIM == 2
            if (d == 0)
              v = (finev (f, Pf, i, j, k, o, 0, 0) + finev (f, Pf, i, j, k, o, 1, 0))/2.;
            else
              v = (finev (f, Pf, i, j, k, 0, o, 0) + finev (f, Pf, i, j, k, 1, o, 0))/2.;
#else
            if (d == 0)
              v = (finev (f, Pf, i, j, k, o, 0, 0) + finev (f, Pf, i, j, k, o, 1, 0) +
                   finev (f, Pf, i, j, k, o, 0, 1) + finev (f, Pf, i, j, k, o, 1, 1))/4.;
            else if (d == 1)
              v = (finev (f, Pf, i, j, k, 0, o, 0) + finev (f, Pf, i, j, k, 0, o, 1) +
                   finev (f, Pf, i, j, k, 1, o, 0) + finev (f, Pf, i, j, k, 1, o, 1))/4.;
            else
              v = (finev (f, Pf, i, j, k, 0, 0, o) + finev (f, Pf, i, j, k, 1, 0, o) +
                   finev (f, Pf, i, j, k, 0, 1, o) + finev (f, Pf, i, j, k, 1, 1, o))/4.;
#endif
            c[id + side*sd] = v;
          }
        }
      }
}

static void restrict_faces (og_grid * g, int l) { restrict_faces_of (g, g->alpha, l); }

/* poisson.h:418-420: restriction ({alpha, lambda}) through all levels,
   each level followed by its boundary (multigrid-common.h:398). */
void og_restrict_coefficients (og_grid * g)
{
  for (int l = g->depth - 1; l >= 0; l--) {
    if (!g->alpha_const) {
      restrict_faces (g, l);
      face_boundary (g, l);
    }
    if (!g->lambda_const)
      restrict_average (g, g->lambda.lv[l], g->lambda.lv[l + 1], l);
  }
}

/* restriction (res): multigrid_restriction (multigrid-common.h:368-404).
   The boundary applied after each level touches ghosts of res only, which
   no operator reads. */
void og_restrict_res (og_grid * g)
{
  for (int l = g->depth - 1; l >= 0; l--)
    restrict_average (g, g->res.lv[l], g->res.lv[l + 1], l);
}

/* bilinear (grid/multigrid-common.h:124-140) of da from level l-1 */
static void prolong_field (og_grid * g, field * fd, int l)
{
  int n = 1 << l, P = P_of (l), Pc = P_of (l - 1);
  (void) Pc;
  const double * s = fd->lv[l - 1];
  double * f = fd->lv[l];
#pragma omp parallel for schedule(static)
  for (int i = GH; i < n + GH; i++)
    for (int j = (DIM > 1 ? GH : 0); j < (DIM > 1 ? n + GH : 1); j++)
      for (int k = (DIM > 2 ? GH : 0); k < (DIM > 2 ? n + GH : 1); k++) {
        int pi = (i + GH)/2, cx = 2*((i + GH) % 2) - 1;
#if DIM == 1
        f[IX (P, i, j, k)] = (3.*s[pi] + s[pi + cx])/4.;
#elif DIM == 2
        int pj = (j + GH)/2, cy = 2*((j + GH) % 2) - 1;
        f[IX (P, i, j, k)] =
          (9.*s[IX (Pc, pi, pj, 0)] +
           3.*(s[IX (Pc, pi + cx, pj, 0)] + s[IX (Pc, pi, pj + cy, 0)]) +
           s[IX (Pc, pi + cx, pj + cy, 0)])/16.;
#else
        int pj = (j + GH)/2, cy = 2*((j + GH) % 2) - 1;
        int pk = (k + GH)/2, cz = 2*((k + GH) % 2) - 1;
        f[IX (P, i, j, k)] =
          (27.*s[IX (Pc, pi, pj, pk)] +
           9.*(s[IX (Pc, pi + cx, pj, pk)] + s[IX (Pc, pi, pj + cy, pk)] +
               s[IX (Pc, pi, pj, pk + cz)]) +
           3.*(s[IX (Pc, pi + cx, pj + cy, pk)] + s[IX (Pc, pi + cx, pj, pk + cz)] +
               s[IX (Pc, pi, pj + cy, pk + cz)]) +
           s[IX (Pc, pi + cx, pj + cy, pk + cz)])/64.;
#endif
      }
}

static void prolong_bilinear (og_grid * g, int l) { prolong_field (g, &g->da, l); }

/* ------------------------------------------------------------------ */
/* relax and residual                                                  */
/* ------------------------------------------------------------------ */

#define ALPHA(d, l, id) (g->alpha_const ? g->alpha_c : g->alpha[d].lv[l][id])
#define LAMBDA(l, id) (g->lambda_const ? g->lambda_c : g->lambda.lv[l][id])

/* one relaxation cell update (poisson.h:303-319); returns n/d */
static inline double relax_cell (og_grid * g, const double * a, const double * b,
                                 int l, size_t id, const size_t * st, double Delta)
{
  double n = - sq_(Delta)*b[id], d = - LAMBDA (l, id)*sq_(Delta);
  for (int e = 0; e < DIM; e++) {
    double a1 = ALPHA (e, l, id + st[e]), a0 = ALPHA (e, l, id);
    n += a1*a[id + st[e]] + a0*a[id - st[e]];
    d += a1 + a0;
  }
  return n/d;
}

/* relax (poisson.h:271-338) on level l, in the variant selected */
void og_relax_level (og_grid * g, int l)
{
  int n = 1 << l, P = P_of (l);
  double Delta = g->L0*(1./(1 << l));
  size_t st[3];
  for (int e = 0; e < DIM; e++) st[e] = stride (P, e);
  double * a = g->da.lv[l];
  const double * b = g->res.lv[l];
  int J0 = DIM > 1 ? GH : 0, J1 = DIM > 1 ? n + GH : 1;
  int K0 = DIM > 2 ? GH : 0, K1 = DIM > 2 ? n + GH : 1;
  if (g->relax_mode == OG_RELAX_JACOBI) {
    double * c = g->c.lv[l];
#pragma omp parallel for schedule(static)
    for (int i = GH; i < n + GH; i++)
      for (int j = J0; j < J1; j++)
        for (int k = K0; k < K1; k++) {
          size_t id = IX (P, i, j, k);
          c[id] = relax_cell (g, a, b, l, id, st, Delta);
        }
#pragma omp parallel for schedule(static)
    for (int i = GH; i < n + GH; i++)
      for (int j = J0; j < J1; j++)
        for (int k = K0; k < K1; k++) {
          size_t id = IX (P, i, j, k);
          a[id] = (a[id] + 2.*c[id])/3.;          /* poisson.h:326-327 */
        }
  }
  else if (g->relax_mode == OG_RELAX_RBGS) {
    /* red cells, boundary, black cells: the black pass sees the updated
       red values everywhere, periodic images included */
    for (int color = 0; color < 2; color++) {
      if (color == 1)
        boundary_level (g, a, l, 1);
#pragma omp parallel for schedule(static)
      for (int i = GH; i < n + GH; i++)
        for (int j = J0; j < J1; j++)
          for (int k = K0; k < K1; k++) {
            if (((i + j + k) & 1) != color) continue;   /* GH even: parity of interior index */
            size_t id = IX (P, i, j, k);
            a[id] = relax_cell (g, a, b, l, id, st, Delta);
          }
    }
  }
  else {
    /* in-place sweep, c aliased to a (poisson.h:296).  Under OpenMP the
       threads race at chunk borders, as in the reference (poisson.h:284). */
#pragma omp parallel for schedule(static)
    for (int i = GH; i < n + GH; i++)
      for (int j = J0; j < J1; j++)
        for (int k = K0; k < K1; k++) {
          size_t id = IX (P, i, j, k);
          a[id] = relax_cell (g, a, b, l, id, st, Delta);
        }
  }
}

/* residual (poisson.h:345-391, the uniform-grid branch 373-389), after the
   automatic boundary of a (stencils.h:228+).  Returns max |res|. */
double og_residual (og_grid * g)
{
  int l = g->depth, n = 1 << l, P = P_of (l);
  double Delta = g->L0*(1./(1 << l));
  boundary_level (g, g->a.lv[l], l, 0);
  size_t st[3];
  for (int e = 0; e < DIM; e++) st[e] = stride (P, e);
  const double * a = g->a.lv[l], * b = g->b.lv[l];
  double * res = g->res.lv[l];
  double maxres = 0.;
  int J0 = DIM > 1 ? GH : 0, J1 = DIM > 1 ? n + GH : 1;
  int K0 = DIM > 2 ? GH : 0, K1 = DIM > 2 ? n + GH : 1;
#pragma omp parallel for schedule(static) reduction(max:maxres)
  for (int i = GH; i < n + GH; i++)
    for (int j = J0; j < J1; j++)
      for (int k = K0; k < K1; k++) {
        size_t id = IX (P, i, j, k);
        double r = b[id] - LAMBDA (l, id)*a[id];
        for (int e = 0; e < DIM; e++)
          r += (ALPHA (e, l, id)*((a[id] - a[id - st[e]])/Delta) -
                ALPHA (e, l, id + st[e])*((a[id + st[e]] - a[id])/Delta))/Delta;
        res[id] = r;
        if (fabs (r) > maxres)
          maxres = fabs (r);
      }
  return maxres;
}

/* ------------------------------------------------------------------ */
/* mg_cycle, mg_solve, poisson                                         */
/* ------------------------------------------------------------------ */

/* mg_cycle (poisson.h:32-90) */
void og_mg_cycle (og_grid * g, int nrelax, int minlevel, int maxlevel)
{
  og_restrict_res (g);
  minlevel = minlevel < maxlevel ? minlevel : maxlevel;
  for (int l = minlevel; l <= maxlevel; l++) {
    if (l == minlevel) {
      size_t m = level_size (l);
      double * s = g->da.lv[l];
      int n = 1 << l, P = P_of (l);
      (void) m;
      for (int i = GH; i < n + GH; i++)
        for (int j = (DIM > 1 ? GH : 0); j < (DIM > 1 ? n + GH : 1); j++)
          for (int k = (DIM > 2 ? GH : 0); k < (DIM > 2 ? n + GH : 1); k++)
            s[IX (P, i, j, k)] = 0.;
    }
    else
      prolong_bilinear (g, l);
    boundary_level (g, g->da.lv[l], l, 1);
    for (int i = 0; i < nrelax; i++) {
      og_relax_level (g, l);
      boundary_level (g, g->da.lv[l], l, 1);
    }
  }
  /* a += da on the leaves (the finest level) */
  int l = g->depth, n = 1 << l, P = P_of (l);
  double * a = g->a.lv[l];
  const double * da = g->da.lv[l];
#pragma omp parallel for schedule(static)
  for (int i = GH; i < n + GH; i++)
    for (int j = (DIM > 1 ? GH : 0); j < (DIM > 1 ? n + GH : 1); j++)
      for (int k = (DIM > 2 ? GH : 0); k < (DIM > 2 ? n + GH : 1); k++) {
        size_t id = IX (P, i, j, k);
        a[id] += da[id];
      }
}

double og_sum_b (og_grid * g)
{
  int l = g->depth, n = 1 << l, P = P_of (l);
  const double * b = g->b.lv[l];
  double sum = 0.;
#pragma omp parallel for schedule(static) reduction(+:sum)
  for (int i = GH; i < n + GH; i++)
    for (int j = (DIM > 1 ? GH : 0); j < (DIM > 1 ? n + GH : 1); j++)
      for (int k = (DIM > 2 ? GH : 0); k < (DIM > 2 ? n + GH : 1); k++)
        sum += b[IX (P, i, j, k)];
  return sum;
}

/* mg_solve (poisson.h:139-235) with the Poisson residual and relax */
og_mgstats og_mg_solve (og_grid * g, double tolerance, int nrelax, int minlevel)
{
  og_mgstats s = {0};
  s.sum = og_sum_b (g);
  s.nrelax = nrelax > 0 ? nrelax : 4;
  double resb;
  resb = s.resb = s.resa = og_residual (g);
  if (tolerance == 0.)
    tolerance = og_TOLERANCE;
  for (s.i = 0;
       s.i < og_NITERMAX && (s.i < og_NITERMIN || s.resa > tolerance);
       s.i++) {
    og_mg_cycle (g, s.nrelax, minlevel, g->depth);
    s.resa = og_residual (g);
    if (s.resa > tolerance) {
      if (resb/s.resa < 1.2 && s.nrelax < 100)
        s.nrelax++;
      else if (resb/s.resa > 10 && s.nrelax > 2)
        s.nrelax--;
    }
    resb = s.resa;
  }
  s.minlevel = minlevel;
  if (s.resa > tolerance) {
    fprintf (stderr,
             "WARNING: convergence for %s not reached after %d iterations\n"
             "  res: %g sum: %g nrelax: %d\n", "a",
             s.i, s.resa, s.sum, s.nrelax), fflush (stderr);
  }
  return s;
}

/* poisson (poisson.h:402-441) */
og_mgstats og_poisson (og_grid * g, double tolerance, int nrelax, int minlevel)
{
  og_restrict_coefficients (g);
  double defaultol = og_TOLERANCE;
  if (tolerance)
    og_TOLERANCE = tolerance;
  og_mgstats s = og_mg_solve (g, 0., nrelax, minlevel > 1 ? minlevel : 1);
  if (tolerance)
    og_TOLERANCE = defaultol;
  return s;
}

/* project (poisson.h:468-509) on the finest level: div = sum of the face
   differences of uf over dt Delta, poisson (p, div, alpha, TOLERANCE/dt^2,
   nrelax), then uf -= dt alpha grad p on every face (foreach_face visits
   faces 0..n along their direction, multigrid.h:255-320) */
og_mgstats og_project (og_grid * g, double dt, int nrelax)
{
  dt = dt ? dt : 1.;
  nrelax = nrelax ? nrelax : 4;
  const int l = g->depth, n = 1 << l, P = P_of (l);
  const double Delta = g->L0*(1./(1 << l));
  size_t st[3];
  for (int e = 0; e < DIM; e++) st[e] = stride (P, e);
  double * div = g->b.lv[l];
  int J0 = DIM > 1 ? GH : 0, J1 = DIM > 1 ? n + GH : 1;
  int K0 = DIM > 2 ? GH : 0, K1 = DIM > 2 ? n + GH : 1;
  for (int i = GH; i < n + GH; i++)
    for (int j = J0; j < J1; j++)
      for (int k = K0; k < K1; k++) {
        size_t id = IX (P, i, j, k);
        double d = 0.;
        for (int e = 0; e < DIM; e++)
          d += g->uf[e].lv[l][id + st[e]] - g->uf[e].lv[l][id];
        d /= dt*Delta;
        div[id] = d;
      }
  og_mgstats s = og_poisson (g, og_TOLERANCE/sq_(dt), nrelax, 0);
  const double * p = g->a.lv[l];
  for (int e = 0; e < DIM; e++) {
    double * u = g->uf[e].lv[l];
    int I1 = n + GH + (e == 0), Jx = J1 + (e == 1 && DIM > 1), Kx = K1 + (e == 2 && DIM > 2);
    for (int i = GH; i < I1; i++)
      for (int j = J0; j < Jx; j++)
        for (int k = K0; k < Kx; k++) {
          size_t id = IX (P, i, j, k);
          u[id] -= dt*ALPHA (e, l, id)*((p[id] - p[id - st[e]])/Delta);
        }
  }
  return s;
}

/* ------------------------------------------------------------------ */
/* implicit viscosity (viscosity.h)                                    */
/* ------------------------------------------------------------------ */

void og_set_visc_bc (og_grid * g, int comp, int side, int type, double value)
{
  if (comp >= 0 && comp < DIM && side >= 0 && side < 2*DIM) {
    g->vbctype[comp][side] = type;
    g->vbcval[comp][side] = value;
  }
}

void og_set_mu_const (og_grid * g, double v) { g->mu_const = 1; g->mu_c = v; }
void og_set_rho_const (og_grid * g, double v) { g->rho_const = 1; g->rho_c = v; }

#define MU(d, l, id) (g->mu_const ? g->mu_c : g->mu[d].lv[l][id])
#define RHO(l, id) (g->rho_const ? g->rho_c : g->rho.lv[l][id])

/* boundary_level of component c of the vector (its own box conditions,
   constant data), as the list boundaries of mg_cycle apply them */
static void comp_boundary (og_grid * g, int c, double * s, int l, int homogeneous)
{
  int t[6], save_t[6];
  double v[6], save_v[6];
  double * save_p[6];
  for (int k = 0; k < 6; k++) {
    t[k] = k < 2*DIM ? g->vbctype[c][k] : OG_NEUMANN; v[k] = k < 2*DIM ? g->vbcval[c][k] : 0.;
    save_t[k] = g->bctype[k]; save_v[k] = g->bcconst[k]; save_p[k] = g->bcval[k];
    g->bctype[k] = t[k]; g->bcconst[k] = v[k]; g->bcval[k] = NULL;
  }
  boundary_level (g, s, l, homogeneous);
  for (int k = 0; k < 6; k++) {
    g->bctype[k] = save_t[k]; g->bcconst[k] = save_v[k]; g->bcval[k] = save_p[k];
  }
}

/* the tangential directions of component c in foreach_dimension order
   (rotate.lex: x -> y -> z -> x) */
static inline int tang (int c, int m) { return DIM == 2 ? 1 - c : (c + 1 + m) % 3; }

/* w.c of relax_viscosity (viscosity.h:36-67) at cell id of level l, from
   the components U and the r.h.s. R of component c */
static double visc_w (og_grid * g, int c, int l, size_t id, double * const * U,
                      const double * R, double dt)
{
  const int P = P_of (l);
  const double Delta = g->L0*(1./(1 << l));
  size_t st[3];
  for (int e = 0; e < DIM; e++) st[e] = stride (P, e);
  const size_t sn = st[c];
  const double * un = U[c];
  const double mn1 = MU (c, l, id + sn), mn0 = MU (c, l, id);
  double A = 2.*mn1*un[id + sn] + 2.*mn0*un[id - sn];
  double den = 2.*mn1 + 2.*mn0;
  for (int m = 0; m < DIM - 1; m++) {
    const int t = tang (c, m);
    const size_t s = st[t];
    const double * ut = U[t];
    const double mt1 = MU (t, l, id + s), mt0 = MU (t, l, id);
    A = A + mt1*(un[id + s] + (ut[id + sn] + ut[id + sn + s])/4. -
                 (ut[id - sn] + ut[id - sn + s])/4.);
    A = A - mt0*(- un[id - s] + (ut[id + sn - s] + ut[id + sn])/4. -
                 (ut[id - sn - s] + ut[id - sn])/4.);
    den = den + mt1;
    den = den + mt0;
  }
  const double rho = RHO (l, id);
  return (dt/rho*A + R[id]*sq_(Delta))/(sq_(Delta)*1. + dt/rho*den);
}

/* relax_viscosity over level l, in the variant selected: the reference's
   in-place sweep (w = u, components in turn per cell), its JACOBI branch,
   or red-black with every colour computed from the values before it
   (the same-colour diagonal neighbours it reads keep their old values) */
static void visc_relax (og_grid * g, int l, double dt)
{
  const int n = 1 << l, P = P_of (l);
  double * U[3] = {NULL, NULL, NULL}, * W[3] = {NULL, NULL, NULL};
  for (int c = 0; c < DIM; c++) { U[c] = g->vda[c].lv[l]; W[c] = g->vw[c].lv[l]; }
  int J0 = DIM > 1 ? GH : 0, J1 = DIM > 1 ? n + GH : 1;
  int K0 = DIM > 2 ? GH : 0, K1 = DIM > 2 ? n + GH : 1;
  if (g->relax_mode == OG_RELAX_GS) {
    for (int i = GH; i < n + GH; i++)
      for (int j = J0; j < J1; j++)
        for (int k = K0; k < K1; k++) {
          size_t id = IX (P, i, j, k);
          for (int c = 0; c < DIM; c++)
            U[c][id] = visc_w (g, c, l, id, U, g->vres[c].lv[l], dt);
        }
    return;
  }
  for (int color = 0; color < 2; color++) {
    const int jac = g->relax_mode == OG_RELAX_JACOBI;
    if (jac && color == 1) break;
    if (!jac && color == 1)
      for (int c = 0; c < DIM; c++) comp_boundary (g, c, U[c], l, 1);
    for (int i = GH; i < n + GH; i++)
      for (int j = J0; j < J1; j++)
        for (int k = K0; k < K1; k++) {
          if (!jac && ((i + j + k) & 1) != color) continue;
          size_t id = IX (P, i, j, k);
          for (int c = 0; c < DIM; c++)
            W[c][id] = visc_w (g, c, l, id, U, g->vres[c].lv[l], dt);
        }
    for (int i = GH; i < n + GH; i++)
      for (int j = J0; j < J1; j++)
        for (int k = K0; k < K1; k++) {
          if (!jac && ((i + j + k) & 1) != color) continue;
          size_t id = IX (P, i, j, k);
          for (int c = 0; c < DIM; c++)
            U[c][id] = jac ? (U[c][id] + 2.*W[c][id])/3. : W[c][id];
        }
  }
}

/* residual_viscosity, uniform-grid branch (viscosity.h:121-147), after
   the boundary of u; res of every component, returns the maximum */
double og_residual_viscosity (og_grid * g, double dt)
{
  const int l = g->depth, n = 1 << l, P = P_of (l);
  const double Delta = g->L0*(1./(1 << l));
  double * U[3] = {NULL, NULL, NULL};
  for (int c = 0; c < DIM; c++) {
    U[c] = g->vu[c].lv[l];
    comp_boundary (g, c, U[c], l, 0);
  }
  size_t st[3];
  for (int e = 0; e < DIM; e++) st[e] = stride (P, e);
  double maxres = 0.;
  int J0 = DIM > 1 ? GH : 0, J1 = DIM > 1 ? n + GH : 1;
  int K0 = DIM > 2 ? GH : 0, K1 = DIM > 2 ? n + GH : 1;
  for (int i = GH; i < n + GH; i++)
    for (int j = J0; j < J1; j++)
      for (int k = K0; k < K1; k++) {
        size_t id = IX (P, i, j, k);
        for (int c = 0; c < DIM; c++) {
          const size_t sn = st[c];
          const double * un = U[c];
          double B = 2.*MU (c, l, id + sn)*(un[id + sn] - un[id]) -
            2.*MU (c, l, id)*(un[id] - un[id - sn]);
          for (int m = 0; m < DIM - 1; m++) {
            const int t = tang (c, m);
            const size_t s = st[t];
            const double * ut = U[t];
            B = B + MU (t, l, id + s)*(un[id + s] - un[id] +
                                      (ut[id + sn] + ut[id + sn + s])/4. -
                                      (ut[id - sn] + ut[id - sn + s])/4.);
            B = B - MU (t, l, id)*(un[id] - un[id - s] +
                                  (ut[id + sn - s] + ut[id + sn])/4. -
                                  (ut[id - sn - s] + ut[id - sn])/4.);
          }
          const double r = g->vr[c].lv[l][id] - 1.*un[id] + dt/RHO (l, id)*B/sq_(Delta);
          g->vres[c].lv[l][id] = r;
          if (fabs (r) > maxres)
            maxres = fabs (r);
        }
      }
  return maxres;
}

/* mg_cycle (poisson.h:32-90) on the vector list {da.x, da.y, (da.z)} */
static void visc_cycle (og_grid * g, int nrelax, int minlevel, int maxlevel, double dt)
{
  for (int c = 0; c < DIM; c++)
    for (int l = g->depth - 1; l >= 0; l--)
      restrict_average (g, g->vres[c].lv[l], g->vres[c].lv[l + 1], l);
  minlevel = minlevel < maxlevel ? minlevel : maxlevel;
  for (int l = minlevel; l <= maxlevel; l++) {
    for (int c = 0; c < DIM; c++) {
      if (l == minlevel) {
        double * s = g->vda[c].lv[l];
        for (size_t q = 0; q < level_size (l); q++) s[q] = 0.;
      }
      else
        prolong_field (g, &g->vda[c], l);
      comp_boundary (g, c, g->vda[c].lv[l], l, 1);
    }
    for (int i = 0; i < nrelax; i++) {
      visc_relax (g, l, dt);
      for (int c = 0; c < DIM; c++)
        comp_boundary (g, c, g->vda[c].lv[l], l, 1);
    }
  }
  const int l = g->depth, n = 1 << l, P = P_of (l);
  for (int c = 0; c < DIM; c++)
    for (int i = GH; i < n + GH; i++)
      for (int j = (DIM > 1 ? GH : 0); j < (DIM > 1 ? n + GH : 1); j++)
        for (int k = (DIM > 2 ? GH : 0); k < (DIM > 2 ? n + GH : 1); k++) {
          size_t id = IX (P, i, j, k);
          g->vu[c].lv[l][id] += g->vda[c].lv[l][id];
        }
}

/* viscosity (viscosity.h:169-183): r = u, restriction ({mu, rho}), then
   mg_solve with residual_viscosity / relax_viscosity (minlevel 0) */
og_mgstats og_viscosity (og_grid * g, double dt, int nrelax)
{
  const int l = g->depth, n = 1 << l, P = P_of (l);
  for (int c = 0; c < DIM; c++)
    memcpy (g->vr[c].lv[l], g->vu[c].lv[l], level_size (l)*sizeof (double));
  for (int m = g->depth - 1; m >= 0; m--) {
    if (!g->mu_const) {
      restrict_faces_of (g, g->mu, m);
      for (int d = 0; d < DIM; d++) periodic_boundary (g, g->mu[d].lv[m], m);
    }
    if (!g->rho_const)
      restrict_average (g, g->rho.lv[m], g->rho.lv[m + 1], m);
  }
  og_mgstats s = {0};
  /* sum of the r.h.s. components (poisson.h:162-167) */
  for (int i = GH; i < n + GH; i++)
    for (int j = (DIM > 1 ? GH : 0); j < (DIM > 1 ? n + GH : 1); j++)
      for (int k = (DIM > 2 ? GH : 0); k < (DIM > 2 ? n + GH : 1); k++)
        for (int c = 0; c < DIM; c++)
          s.sum += g->vr[c].lv[l][IX (P, i, j, k)];
  s.nrelax = nrelax > 0 ? nrelax : 4;
  double resb;
  resb = s.resb = s.resa = og_residual_viscosity (g, dt);
  const double tolerance = og_TOLERANCE;
  for (s.i = 0; s.i < og_NITERMAX && (s.i < og_NITERMIN || s.resa > tolerance); s.i++) {
    visc_cycle (g, s.nrelax, 0, g->depth, dt);
    s.resa = og_residual_viscosity (g, dt);
    if (s.resa > tolerance) {
      if (resb/s.resa < 1.2 && s.nrelax < 100)
        s.nrelax++;
      else if (resb/s.resa > 10 && s.nrelax > 2)
        s.nrelax--;
    }
    resb = s.resa;
  }
  s.minlevel = 0;
  if (s.resa > tolerance)
    fprintf (stderr,
             "WARNING: convergence for %s not reached after %d iterations\n"
             "  res: %g sum: %g nrelax: %d\n", "u.x",
             s.i, s.resa, s.sum, s.nrelax), fflush (stderr);
  return s;
}

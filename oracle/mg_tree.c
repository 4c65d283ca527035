/*
 * mg_tree.c -- CPU oracle: a plain-C restatement of the reference's quadtree
 * multigrid Poisson--Helmholtz solver (two dimensions).
 *
 * TEST INFRASTRUCTURE ONLY (see mg_tree.h).  The checker for the CUDA tree
 * path and its CPU baseline; never part of the product path.
 *
 * What it restates, by reference file:line (paths inside the Basilisk tree):
 *   refine_cell with the 2:1 rule (TWO_ONE)     grid/tree-common.h:22-55
 *   refine (cond) fixed-point loop              grid/tree-common.h:308-326
 *   neighbour counts, halo children             grid/tree.h:1032-1041, 929-970
 *   caches: active, leaves, prolongation        grid/tree.h:556-684
 *   traversal order of foreach_cell             grid/foreach_cell.h:80-120
 *   foreach_level_or_leaf                       grid/tree.h:735-740
 *   tree_boundary_level (restriction from l     grid/tree-common.h:588-716
 *     down, then bilinear halo prolongation)
 *   box boundary on trees (normal neighbour,    grid/tree.h:1139-1209,
 *     then diagonal)                              1286-1367
 *   halo_face (conservative coarse faces)       grid/tree-common.h:374-411
 *   restriction_average, face_average, bilinear grid/multigrid-common.h:26-55,
 *                                                 124-146
 *   BC formulas                                 common.h:957-960
 *   mg_cycle, mg_solve, relax, poisson          poisson.h:32-90, 139-235,
 *                                                 271-338, 402-441
 *   residual, tree branch                       poisson.h:355-372
 *
 * The relaxation variants are the reference's in-place sweep in its
 * traversal order (level l in foreach_cell order, then the leaves of the
 * coarser levels, finest first), its JACOBI branch, and red-black
 * Gauss-Seidel (red cells of every level of the set, tree boundary, black
 * cells), which pins the GPU smoother of that name.
 *
 * Arithmetic is written in the reference's evaluation order (build with
 * -ffp-contract=off).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include "mg_tree.h"

#define TL 14
#define sq_(x) ((x)*(x))
#define NF 8                 /* A, B, RES, LAMBDA, ALPHA_X, ALPHA_Y, DA, C */
#define OT_C 7

int ot_NITERMAX = 100, ot_NITERMIN = 1;
double ot_TOLERANCE = 1e-3;

struct ot_tree {
  int maxdepth, depth;
  double L0, X0, Y0;
  unsigned char * fl[TL + 1];
  unsigned short * nb[TL + 1];      /* refined cells in the 3x3 neighbourhood */
  double * f[NF][TL + 1];
  int bctype[4];
  double bcconst[4];
  double * bcv[4][TL + 1];
  int relax_mode;
  int alpha_const, lambda_const;
  double alpha_c, lambda_c;
  int * order[TL + 1];              /* active cells of a level, foreach_cell order */
  int norder[TL + 1];
  int * leafs;                      /* all leaves, foreach_cell order (level, index) */
  long nleaves;
};

static inline int NN (int l) { return 1 << l; }
static inline int PP (int l) { return (1 << l) + 2; }
static inline size_t IX (int l, int i, int j) { return (size_t) (i + 1)*PP (l) + (j + 1); }
static inline double DELTA (const ot_tree * t, int l) { return t->L0*(1./(1 << l)); }

ot_tree * ot_new (int maxdepth, double L0, double X0, double Y0)
{
  if (maxdepth < 0 || maxdepth >= TL) return NULL;
  ot_tree * t = calloc (1, sizeof (ot_tree));
  t->maxdepth = maxdepth;
  t->L0 = L0; t->X0 = X0; t->Y0 = Y0;
  for (int l = 0; l <= maxdepth; l++) {
    size_t m = (size_t) PP (l)*PP (l);
    t->fl[l] = calloc (m, 1);
    t->nb[l] = calloc (m, sizeof (unsigned short));
    for (int k = 0; k < NF; k++)
      if (k != OT_LAMBDA)
        t->f[k][l] = calloc (m, sizeof (double));
  }
  for (int s = 0; s < 4; s++) t->bctype[s] = OT_NEUMANN;   /* symmetry */
  t->fl[0][IX (0, 0, 0)] = OT_ACTIVE | OT_LEAF;           /* init_grid (1) */
  t->alpha_const = 1; t->alpha_c = 1.;                     /* unityf */
  t->lambda_const = 1; t->lambda_c = 0.;                   /* zeroc */
  t->relax_mode = OT_RELAX_GS;
  t->nleaves = 1;
  t->leafs = NULL;
  return t;
}

void ot_free (ot_tree * t)
{
  if (!t) return;
  for (int l = 0; l <= t->maxdepth; l++) {
    free (t->fl[l]); free (t->nb[l]); free (t->order[l]);
    for (int k = 0; k < NF; k++) free (t->f[k][l]);
    for (int s = 0; s < 4; s++) free (t->bcv[s][l]);
  }
  free (t->leafs);
  free (t);
}

int ot_depth (const ot_tree * t) { return t->depth; }
long ot_leaves (const ot_tree * t) { return t->nleaves; }
void ot_set_relax (ot_tree * t, int mode) { t->relax_mode = mode; }
void ot_set_alpha_const (ot_tree * t, double v) { t->alpha_const = 1; t->alpha_c = v; }

void ot_set_lambda_const (ot_tree * t, double v) { t->lambda_const = 1; t->lambda_c = v; }

/* ------------------------------------------------------------------ */
/* the tree                                                            */
/* ------------------------------------------------------------------ */

/* refine_cell (tree-common.h:22-55): first the coarse neighbours of the
   parent in the direction of this child, if they are leaves, then this
   cell; increment_neighbors (tree.h:1032-1041) counts it in the 3x3
   neighbourhood (itself included) */
static void refine_cell (ot_tree * t, int l, int i, int j, int * err)
{
  if (l + 1 > t->maxdepth) { *err = 1; return; }
  if (l > 0) {
    int pi = i >> 1, pj = j >> 1, cx = (i & 1) ? 1 : -1, cy = (j & 1) ? 1 : -1;
    int np = NN (l - 1);
    for (int k = 0; k != 2*cx; k += cx)
      for (int m = 0; m != 2*cy; m += cy) {
        int ni = pi + k, nj = pj + m;
        if (ni < 0 || nj < 0 || ni >= np || nj >= np) continue;    /* box boundary */
        if (t->fl[l - 1][IX (l - 1, ni, nj)] & OT_LEAF)
          refine_cell (t, l - 1, ni, nj, err);
      }
  }
  int n = NN (l);
  for (int di = -1; di <= 1; di++)
    for (int dj = -1; dj <= 1; dj++) {
      int a = i + di, b = j + dj;
      if (a >= 0 && b >= 0 && a < n && b < n)
        t->nb[l][IX (l, a, b)]++;
    }
  unsigned char cf = (t->fl[l][IX (l, i, j)] & OT_ACTIVE) ? (OT_ACTIVE | OT_LEAF) : OT_LEAF;
  for (int ci = 0; ci < 2; ci++)
    for (int cj = 0; cj < 2; cj++)
      t->fl[l + 1][IX (l + 1, 2*i + ci, 2*j + cj)] |= cf;
  t->fl[l][IX (l, i, j)] &= ~OT_LEAF;
  if (l + 1 > t->depth) t->depth = l + 1;
}

/* one foreach_leaf() pass of refine (): pre-order, children in the order
   (left,bottom), (left,top), (right,bottom), (right,top) */
static int refine_pass (ot_tree * t, int l, int i, int j, ot_cond cond, void * data, int * err)
{
  unsigned char f = t->fl[l][IX (l, i, j)];
  if (!(f & OT_ACTIVE) || *err) return 0;
  if (f & OT_LEAF) {
    double D = DELTA (t, l);
    double x = (i + 0.5)*D + t->X0, y = (j + 0.5)*D + t->Y0;
    if (cond (l, x, y, data)) {
      refine_cell (t, l, i, j, err);
      return 1;
    }
    return 0;
  }
  int r = 0;
  for (int ci = 0; ci < 2; ci++)
    for (int cj = 0; cj < 2; cj++)
      r += refine_pass (t, l + 1, 2*i + ci, 2*j + cj, cond, data, err);
  return r;
}

static void collect (ot_tree * t, int l, int i, int j, long * nl)
{
  size_t id = IX (l, i, j);
  unsigned char f = t->fl[l][id];
  if (!(f & OT_ACTIVE)) return;
  t->order[l][t->norder[l]++] = (int) id;
  if (f & OT_LEAF) {
    t->leafs[2*(*nl)] = l;
    t->leafs[2*(*nl) + 1] = (int) id;
    (*nl)++;
    return;
  }
  for (int ci = 0; ci < 2; ci++)
    for (int cj = 0; cj < 2; cj++)
      collect (t, l + 1, 2*i + ci, 2*j + cj, nl);
}

/* flags of halo cells and prolongation leaves (update_cache_f), and the
   traversal orders */
static void finalize (ot_tree * t)
{
  long leaves = 0;
  for (int l = 0; l <= t->maxdepth; l++) {
    size_t m = (size_t) PP (l)*PP (l);
    for (size_t id = 0; id < m; id++)
      t->fl[l][id] &= ~(OT_HALO | OT_PROL);
  }
  for (int l = 0; l <= t->depth; l++) {
    int n = NN (l);
    long cnt = 0;
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) {
        size_t id = IX (l, i, j);
        if (t->fl[l][id] & OT_ACTIVE) cnt++;
        if ((t->fl[l][id] & OT_LEAF) && t->nb[l][id] > 0) {
          t->fl[l][id] |= OT_PROL;
          for (int ci = 0; ci < 2; ci++)
            for (int cj = 0; cj < 2; cj++)
              t->fl[l + 1][IX (l + 1, 2*i + ci, 2*j + cj)] |= OT_HALO;
        }
        if (t->fl[l][id] & OT_LEAF) leaves++;
      }
    free (t->order[l]);
    t->order[l] = malloc ((cnt + 1)*sizeof (int));
    t->norder[l] = 0;
  }
  free (t->leafs);
  t->leafs = malloc ((2*leaves + 2)*sizeof (int));
  long nl = 0;
  collect (t, 0, 0, 0, &nl);
  t->nleaves = nl;
}

int ot_refine (ot_tree * t, ot_cond cond, void * data)
{
  int err = 0, total = 0, r;
  do {
    r = refine_pass (t, 0, 0, 0, cond, data, &err);
    total += r;
  } while (r && !err);
  finalize (t);
  return err ? -1 : total;
}

void ot_get_flags (const ot_tree * t, int level, unsigned char * out)
{
  int n = NN (level);
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++)
      out[(size_t) i*n + j] = level <= t->maxdepth ? t->fl[level][IX (level, i, j)] : 0;
}

/* ------------------------------------------------------------------ */
/* fields                                                              */
/* ------------------------------------------------------------------ */

void ot_set_level (ot_tree * t, int which, int level, const double * v)
{
  int n = NN (level);
  if (which == OT_LAMBDA && !t->f[OT_LAMBDA][0])
    for (int l = 0; l <= t->maxdepth; l++)
      t->f[OT_LAMBDA][l] = calloc ((size_t) PP (l)*PP (l), sizeof (double));
  if (which == OT_LAMBDA) t->lambda_const = 0;
  if (which == OT_ALPHA_X || which == OT_ALPHA_Y) t->alpha_const = 0;
  double * s = t->f[which][level];
  int ni = which == OT_ALPHA_X ? n + 1 : n, nj = which == OT_ALPHA_Y ? n + 1 : n;
  for (int i = 0; i < ni; i++)
    for (int j = 0; j < nj; j++)
      s[IX (level, i, j)] = v[(size_t) i*nj + j];
}

void ot_get_level (const ot_tree * t, int which, int level, double * v)
{
  int n = NN (level);
  const double * s = t->f[which][level];
  int ni = which == OT_ALPHA_X ? n + 1 : n, nj = which == OT_ALPHA_Y ? n + 1 : n;
  for (int i = 0; i < ni; i++)
    for (int j = 0; j < nj; j++)
      v[(size_t) i*nj + j] = s ? s[IX (level, i, j)] : 0.;
}

void ot_set_bc (ot_tree * t, int side, int type, double value, int level,
                const double * values)
{
  t->bctype[side] = type;
  if (!values) {
    t->bcconst[side] = value;
    for (int l = 0; l <= t->maxdepth; l++) { free (t->bcv[side][l]); t->bcv[side][l] = NULL; }
    return;
  }
  int n = NN (level);
  if (!t->bcv[side][level]) t->bcv[side][level] = malloc (n*sizeof (double));
  memcpy (t->bcv[side][level], values, n*sizeof (double));
}

#define AX(l, id) (t->alpha_const ? t->alpha_c : t->f[OT_ALPHA_X][l][id])
#define AY(l, id) (t->alpha_const ? t->alpha_c : t->f[OT_ALPHA_Y][l][id])
#define LAM(l, id) (t->lambda_const ? t->lambda_c : t->f[OT_LAMBDA][l][id])

/* ------------------------------------------------------------------ */
/* boundaries                                                          */
/* ------------------------------------------------------------------ */

static inline int allocated_interior (const ot_tree * t, int l, int i, int j)
{
  int n = NN (l);
  if (i < 0 || j < 0 || i >= n || j >= n) return 0;
  return (t->fl[l][IX (l, i, j)] & (OT_ACTIVE | OT_HALO)) != 0;
}

static inline int is_ghost (int l, int i, int j)
{
  int n = NN (l);
  if (i < -1 || j < -1 || i > n || j > n) return 0;
  return i == -1 || j == -1 || i == n || j == n;
}

/* the boundary id of a ghost cell: the pids of init_grid (tree.h:1530-1542)
   give corners their x side, children inherit them */
static inline int side_of (int l, int i, int j)
{
  int n = NN (l);
  if (i < 0) return OT_LEFT;
  if (i >= n) return OT_RIGHT;
  if (j >= n) return OT_TOP;
  return OT_BOTTOM;
}

/* s.boundary[side](n, ghost) of common.h:957-960; tidx is the tangential
   index of the boundary face of the interior cell n */
static inline double bc_apply (const ot_tree * t, const double * s, int side, int l,
                               int tidx, size_t n, int homog)
{
  double v = t->bcv[side][l] ? t->bcv[side][l][tidx] : t->bcconst[side];
  if (t->bctype[side] == OT_DIRICHLET)
    return homog ? - s[n] : 2.*v - s[n];
  return homog ? s[n] : DELTA (t, l)*v + s[n];
}

/* box_boundary_level on trees (tree.h:1286-1367): a ghost takes the value
   given by its first normal interior neighbour (x then y, -1 then +1), else
   by a diagonal interior neighbour whose two normal cells are ghosts */
static void box_bc (ot_tree * t, double * s, int l, int homog)
{
  int n = NN (l);
  for (int gi = -1; gi <= n; gi++)
    for (int gj = -1; gj <= n; gj++) {
      if (!is_ghost (l, gi, gj)) continue;
      static const int dirs[4][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}};
      int done = 0;
      for (int q = 0; q < 4 && !done; q++) {
        int a = gi + dirs[q][0], b = gj + dirs[q][1];
        if (allocated_interior (t, l, a, b)) {
          int side = side_of (l, gi, gj);
          int tidx = (side == OT_LEFT || side == OT_RIGHT) ? b : a;
          s[IX (l, gi, gj)] = bc_apply (t, s, side, l, tidx, IX (l, a, b), homog);
          done = 1;
        }
      }
      for (int di = -1; di <= 1 && !done; di += 2)
        for (int dj = -1; dj <= 1 && !done; dj += 2) {
          int a = gi + di, b = gj + dj;
          if (allocated_interior (t, l, a, b) && is_ghost (l, a, gj) && is_ghost (l, gi, b)) {
            int s1 = side_of (l, a, gj), s2 = side_of (l, gi, b);
            size_t nid = IX (l, a, b);
            int t1 = (s1 == OT_LEFT || s1 == OT_RIGHT) ? b : a;
            int t2 = (s2 == OT_LEFT || s2 == OT_RIGHT) ? b : a;
            s[IX (l, gi, gj)] = (bc_apply (t, s, s1, l, t1, nid, homog) +
                                 bc_apply (t, s, s2, l, t2, nid, homog) -
                                 s[nid]);
            done = 1;
          }
        }
    }
}

/* restriction_average (multigrid-common.h:26-32) on the refined cells of
   level l */
static void restrict_cells (ot_tree * t, double ** s, int l)
{
  int n = NN (l);
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) {
      unsigned char f = t->fl[l][IX (l, i, j)];
      if (!(f & OT_ACTIVE) || (f & OT_LEAF)) continue;
      double sum = 0.;
      for (int ci = 0; ci < 2; ci++)
        for (int cj = 0; cj < 2; cj++)
          sum += s[l + 1][IX (l + 1, 2*i + ci, 2*j + cj)];
      s[l][IX (l, i, j)] = sum/(1 << 2);
    }
}

/* bilinear (multigrid-common.h:124-140) of child (i, j) of level l */
static inline double bilinear (const ot_tree * t, double ** s, int l, int i, int j)
{
  int pi = i >> 1, pj = j >> 1, cx = (i & 1) ? 1 : -1, cy = (j & 1) ? 1 : -1;
  const double * c = s[l - 1];
  (void) t;
  return (9.*c[IX (l - 1, pi, pj)] +
          3.*(c[IX (l - 1, pi + cx, pj)] + c[IX (l - 1, pi, pj + cy)]) +
          c[IX (l - 1, pi + cx, pj + cy)])/16.;
}

/* refine_bilinear of the halo children of the prolongation leaves of level l */
static void prolong_halo (ot_tree * t, double ** s, int l)
{
  int n = NN (l);
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++)
      if (t->fl[l][IX (l, i, j)] & OT_PROL)
        for (int ci = 0; ci < 2; ci++)
          for (int cj = 0; cj < 2; cj++)
            s[l + 1][IX (l + 1, 2*i + ci, 2*j + cj)] = bilinear (t, s, l + 1, 2*i + ci, 2*j + cj);
}

static int tree_full (const ot_tree * t)
{
  return t->nleaves == (1L << (2*t->depth));
}

/* tree_boundary_level (tree-common.h:588-716) of a cell scalar with the
   default restriction/prolongation, up to level l */
static void tree_boundary (ot_tree * t, double ** s, int l, int homog)
{
  if (tree_full (t)) {
    box_bc (t, s[l], l, homog);
    return;
  }
  for (int m = l - 1; m >= 0; m--)
    restrict_cells (t, s, m);
  box_bc (t, s[0], 0, homog);
  for (int i = 0; i < l; i++) {
    prolong_halo (t, s, i);
    box_bc (t, s[i + 1], i + 1, homog);
  }
}

void ot_boundary (ot_tree * t, int which, int level, int homogeneous)
{
  tree_boundary (t, t->f[which], level < 0 ? t->depth : level, homogeneous);
}

/* restriction ({alpha, lambda}): face_average / restriction_average on the
   refined cells, finest first (the halo faces of halo_face get the same
   averages from the refined neighbour) */
void ot_restrict_coefficients (ot_tree * t)
{
  for (int l = t->depth - 1; l >= 0; l--) {
    int n = NN (l);
    if (!t->alpha_const) {
      double * ax = t->f[OT_ALPHA_X][l], * ay = t->f[OT_ALPHA_Y][l];
      const double * fx = t->f[OT_ALPHA_X][l + 1], * fy = t->f[OT_ALPHA_Y][l + 1];
      for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) {
          unsigned char f = t->fl[l][IX (l, i, j)];
          if (!(f & OT_ACTIVE) || (f & OT_LEAF)) continue;
          ax[IX (l, i, j)] = (fx[IX (l + 1, 2*i, 2*j)] + fx[IX (l + 1, 2*i, 2*j + 1)])/2.;
          ax[IX (l, i + 1, j)] = (fx[IX (l + 1, 2*i + 2, 2*j)] + fx[IX (l + 1, 2*i + 2, 2*j + 1)])/2.;
          ay[IX (l, i, j)] = (fy[IX (l + 1, 2*i, 2*j)] + fy[IX (l + 1, 2*i + 1, 2*j)])/2.;
          ay[IX (l, i, j + 1)] = (fy[IX (l + 1, 2*i, 2*j + 2)] + fy[IX (l + 1, 2*i + 1, 2*j + 2)])/2.;
        }
    }
    if (!t->lambda_const)
      restrict_cells (t, t->f[OT_LAMBDA], l);
  }
}

/* ------------------------------------------------------------------ */
/* relax, residual                                                     */
/* ------------------------------------------------------------------ */

static inline double relax_cell (const ot_tree * t, const double * a, const double * b,
                                 int l, size_t id)
{
  int P = PP (l);
  double Delta = DELTA (t, l);
  double n = - sq_(Delta)*b[id], d = - LAM (l, id)*sq_(Delta);
  n += AX (l, id + P)*a[id + P] + AX (l, id)*a[id - P];
  d += AX (l, id + P) + AX (l, id);
  n += AY (l, id + 1)*a[id + 1] + AY (l, id)*a[id - 1];
  d += AY (l, id + 1) + AY (l, id);
  return n/d;
}

static inline int parity (int l, size_t id)
{
  int P = PP (l), i = (int) (id/P) - 1, j = (int) (id % P) - 1;
  return (i + j) & 1;
}

/* relax (poisson.h:271-338) over foreach_level_or_leaf (l) */
void ot_relax_level (ot_tree * t, int l)
{
  double ** a = t->f[OT_DA], ** b = t->f[OT_RES];
  if (t->relax_mode == OT_RELAX_JACOBI) {
    double ** c = t->f[OT_C];
    for (int m = l; m >= 0; m--)
      for (int k = 0; k < t->norder[m]; k++) {
        size_t id = t->order[m][k];
        if (m == l || (t->fl[m][id] & OT_LEAF))
          c[m][id] = relax_cell (t, a[m], b[m], m, id);
      }
    for (int m = l; m >= 0; m--)
      for (int k = 0; k < t->norder[m]; k++) {
        size_t id = t->order[m][k];
        if (m == l || (t->fl[m][id] & OT_LEAF))
          a[m][id] = (a[m][id] + 2.*c[m][id])/3.;
      }
  }
  else if (t->relax_mode == OT_RELAX_RBGS) {
    for (int color = 0; color < 2; color++) {
      if (color == 1)
        tree_boundary (t, a, l, 1);
      for (int m = l; m >= 0; m--)
        for (int k = 0; k < t->norder[m]; k++) {
          size_t id = t->order[m][k];
          if ((m == l || (t->fl[m][id] & OT_LEAF)) && parity (m, id) == color)
            a[m][id] = relax_cell (t, a[m], b[m], m, id);
        }
    }
  }
  else {
    for (int m = l; m >= 0; m--)
      for (int k = 0; k < t->norder[m]; k++) {
        size_t id = t->order[m][k];
        if (m == l || (t->fl[m][id] & OT_LEAF))
          a[m][id] = relax_cell (t, a[m], b[m], m, id);
      }
  }
}

/* g.x = alpha.x face_gradient_x (a, 0) on the face to the left of cell
   (i, j) of level l (stored at that cell) */
static inline double gx (const ot_tree * t, double ** a, int l, int i, int j)
{
  size_t id = IX (l, i, j);
  return AX (l, id)*((a[l][id] - a[l][id - PP (l)])/DELTA (t, l));
}

static inline double gy (const ot_tree * t, double ** a, int l, int i, int j)
{
  size_t id = IX (l, i, j);
  return AY (l, id)*((a[l][id] - a[l][id - 1])/DELTA (t, l));
}

static inline int refined (const ot_tree * t, int l, int i, int j)
{
  int n = NN (l);
  if (i < 0 || j < 0 || i >= n || j >= n) return 0;
  unsigned char f = t->fl[l][IX (l, i, j)];
  return (f & OT_ACTIVE) && !(f & OT_LEAF);
}

/* residual (poisson.h:355-372): fluxes on the faces of each leaf, a face
   shared with a refined neighbour being the mean of the two fine faces
   (halo_face, tree-common.h:374-411), after boundary (a) */
double ot_residual (ot_tree * t)
{
  double ** a = t->f[OT_A];
  tree_boundary (t, a, t->depth, 0);
  double maxres = 0.;
  for (long k = 0; k < t->nleaves; k++) {
    int l = t->leafs[2*k];
    size_t id = t->leafs[2*k + 1];
    int P = PP (l), i = (int) (id/P) - 1, j = (int) (id % P) - 1;
    double Delta = DELTA (t, l);
    double gl, gr, gb, gt;
    gl = refined (t, l, i - 1, j) ?
      (gx (t, a, l + 1, 2*i, 2*j) + gx (t, a, l + 1, 2*i, 2*j + 1))/2. : gx (t, a, l, i, j);
    gr = refined (t, l, i + 1, j) ?
      (gx (t, a, l + 1, 2*i + 2, 2*j) + gx (t, a, l + 1, 2*i + 2, 2*j + 1))/2. : gx (t, a, l, i + 1, j);
    gb = refined (t, l, i, j - 1) ?
      (gy (t, a, l + 1, 2*i, 2*j) + gy (t, a, l + 1, 2*i + 1, 2*j))/2. : gy (t, a, l, i, j);
    gt = refined (t, l, i, j + 1) ?
      (gy (t, a, l + 1, 2*i, 2*j + 2) + gy (t, a, l + 1, 2*i + 1, 2*j + 2))/2. : gy (t, a, l, i, j + 1);
    double r = t->f[OT_B][l][id] - LAM (l, id)*a[l][id];
    r -= (gr - gl)/Delta;
    r -= (gt - gb)/Delta;
    t->f[OT_RES][l][id] = r;
    if (fabs (r) > maxres)
      maxres = fabs (r);
  }
  return maxres;
}

double ot_sum_b (const ot_tree * t)
{
  double sum = 0.;
  for (long k = 0; k < t->nleaves; k++)
    sum += t->f[OT_B][t->leafs[2*k]][t->leafs[2*k + 1]];
  return sum;
}

/* ------------------------------------------------------------------ */
/* mg_cycle, mg_solve, poisson                                         */
/* ------------------------------------------------------------------ */

/* mg_cycle (poisson.h:32-90) on the tree */
void ot_mg_cycle (ot_tree * t, int nrelax, int minlevel, int maxlevel)
{
  double ** da = t->f[OT_DA];
  /* restriction (res): tree_restriction = boundary (res), whose restriction
     part is all the relaxation reads */
  for (int m = t->depth - 1; m >= 0; m--)
    restrict_cells (t, t->f[OT_RES], m);
  minlevel = minlevel < maxlevel ? minlevel : maxlevel;
  for (int l = minlevel; l <= maxlevel; l++) {
    if (l == minlevel) {
      for (int m = l; m >= 0; m--)
        for (int k = 0; k < t->norder[m]; k++) {
          size_t id = t->order[m][k];
          if (m == l || (t->fl[m][id] & OT_LEAF))
            da[m][id] = 0.;
        }
    }
    else
      for (int k = 0; k < t->norder[l]; k++) {
        size_t id = t->order[l][k];
        int P = PP (l), i = (int) (id/P) - 1, j = (int) (id % P) - 1;
        da[l][id] = bilinear (t, da, l, i, j);
      }
    tree_boundary (t, da, l, 1);
    for (int i = 0; i < nrelax; i++) {
      ot_relax_level (t, l);
      tree_boundary (t, da, l, 1);
    }
  }
  for (long k = 0; k < t->nleaves; k++) {
    int l = t->leafs[2*k];
    size_t id = t->leafs[2*k + 1];
    t->f[OT_A][l][id] += da[l][id];
  }
}

ot_mgstats ot_mg_solve (ot_tree * t, double tolerance, int nrelax, int minlevel)
{
  ot_mgstats s = {0};
  s.sum = ot_sum_b (t);
  s.nrelax = nrelax > 0 ? nrelax : 4;
  double resb;
  resb = s.resb = s.resa = ot_residual (t);
  if (tolerance == 0.)
    tolerance = ot_TOLERANCE;
  for (s.i = 0;
       s.i < ot_NITERMAX && (s.i < ot_NITERMIN || s.resa > tolerance);
       s.i++) {
    ot_mg_cycle (t, s.nrelax, minlevel, t->depth);
    s.resa = ot_residual (t);
    if (s.resa > tolerance) {
      if (resb/s.resa < 1.2 && s.nrelax < 100)
        s.nrelax++;
      else if (resb/s.resa > 10 && s.nrelax > 2)
        s.nrelax--;
    }
    resb = s.resa;
  }
  s.minlevel = minlevel;
  if (s.resa > tolerance)
    fprintf (stderr,
             "WARNING: convergence for %s not reached after %d iterations\n"
             "  res: %g sum: %g nrelax: %d\n", "a",
             s.i, s.resa, s.sum, s.nrelax), fflush (stderr);
  return s;
}

ot_mgstats ot_poisson (ot_tree * t, double tolerance, int nrelax, int minlevel)
{
  ot_restrict_coefficients (t);
  double defaultol = ot_TOLERANCE;
  if (tolerance)
    ot_TOLERANCE = tolerance;
  ot_mgstats s = ot_mg_solve (t, 0., nrelax, minlevel > 1 ? minlevel : 1);
  if (tolerance)
    ot_TOLERANCE = defaultol;
  return s;
}

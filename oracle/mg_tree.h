/*
 * mg_tree.h -- CPU oracle for the quadtree variant of the multigrid
 * Poisson--Helmholtz solver.
 *
 * TEST INFRASTRUCTURE ONLY.  A plain-C99 restatement of the reference's tree
 * multigrid (Basilisk poisson.h mg_cycle / relax / residual, tree branch,
 * on grid/quadtree.h = grid/tree.h + grid/tree-common.h, two dimensions).
 * It is the checker for the CUDA tree path; the product never links it.
 *
 * Storage: every level l = 0..maxdepth is a dense (2^l + 2)^2 array with one
 * ghost layer; the tree is a set of flags per cell.  Arrays at this
 * interface are the interior n x n values of one level (C order, j, the y
 * index, contiguous); x faces are (n+1) x n, y faces n x (n+1), face f the
 * left/bottom face of cell f.
 */
#ifndef MG_TREE_H
#define MG_TREE_H
#ifdef __cplusplus
extern "C" {
#endif

/* cell flags (grid/tree.h:27-47): active and leaf as in the reference;
   HALO marks an allocated cell that is not active (a "prolongation" cell,
   tree.h:399), PROL a leaf whose children are such halo cells (the
   prolongation cache of update_cache_f, tree.h:646-648) */
enum { OT_ACTIVE = 1, OT_LEAF = 2, OT_HALO = 4, OT_PROL = 8 };

/* sides (common.h:949) and BC kinds, as in mg_oracle.h */
enum { OT_RIGHT = 0, OT_LEFT, OT_TOP, OT_BOTTOM };
enum { OT_NEUMANN = 0, OT_DIRICHLET = 1 };
enum { OT_RELAX_GS = 0, OT_RELAX_JACOBI = 1, OT_RELAX_RBGS = 2 };
enum { OT_A = 0, OT_B, OT_RES, OT_LAMBDA, OT_ALPHA_X, OT_ALPHA_Y, OT_DA };

typedef struct {
  int i;
  double resb, resa;
  double sum;
  int nrelax;
  int minlevel;
} ot_mgstats;

typedef struct ot_tree ot_tree;
typedef int (* ot_cond) (int level, double x, double y, void * data);

extern int ot_NITERMAX, ot_NITERMIN;
extern double ot_TOLERANCE;

ot_tree * ot_new (int maxdepth, double L0, double X0, double Y0);
void ot_free (ot_tree * t);
/* refine (cond) (tree-common.h:308-326) with the 2:1 rule of refine_cell
   (tree-common.h:22-55); returns the number of refinements, -1 when a
   refinement would go past maxdepth */
int ot_refine (ot_tree * t, ot_cond cond, void * data);
int ot_depth (const ot_tree * t);
long ot_leaves (const ot_tree * t);
void ot_get_flags (const ot_tree * t, int level, unsigned char * out);
void ot_set_relax (ot_tree * t, int mode);
/* s[side] = dirichlet / neumann: a constant (values == NULL) or the n
   values of one level's boundary faces, over the tangential index */
void ot_set_bc (ot_tree * t, int side, int type, double value, int level,
                const double * values);
void ot_set_level (ot_tree * t, int which, int level, const double * values);
void ot_get_level (const ot_tree * t, int which, int level, double * out);
void ot_set_alpha_const (ot_tree * t, double v);
void ot_set_lambda_const (ot_tree * t, double v);
/* restriction ({alpha, lambda}) on the tree (tree-common.h:588-716 with
   face_average / restriction_average, multigrid-common.h:26-55) */
void ot_restrict_coefficients (ot_tree * t);
/* boundary (a) or boundary_level (da, l) (tree_boundary_level) */
void ot_boundary (ot_tree * t, int which, int level, int homogeneous);
void ot_relax_level (ot_tree * t, int level);
double ot_residual (ot_tree * t);
double ot_sum_b (const ot_tree * t);
void ot_mg_cycle (ot_tree * t, int nrelax, int minlevel, int maxlevel);
ot_mgstats ot_mg_solve (ot_tree * t, double tolerance, int nrelax, int minlevel);
ot_mgstats ot_poisson (ot_tree * t, double tolerance, int nrelax, int minlevel);

#ifdef __cplusplus
}
#endif
#endif

/*
 * mg_tree.h -- internal interface of the quadtree path: the host layer
 * (mg_tree_host.c) and its CUDA kernels (mg_tree.cu).  Plain C types only.
 *
 * A tree lives on the dense levels of a grid (the level layout of
 * mg_launch.h): every level l keeps its (2^l + 2)^2 padded array, and the
 * tree is a set of per-cell flags plus cell lists.  A list entry packs one
 * cell as level << 28 | (i + 1) << 14 | (j + 1), interior indices i (x) and
 * j (y) from -1 (the ghost layer) to n.
 */
#ifndef MG_TREE_H
#define MG_TREE_H

#include <stdint.h>
#include <cuda_runtime_api.h>
#include "mg_launch.h"

#ifdef __cplusplus
extern "C" {
#endif

#define BMG_TREE_MAXLEVEL 13

/* cell flags (grid/tree.h:27-47, 398-399): ACTIVE and LEAF as in the
   reference, HALO an allocated cell that is not active (a prolongation
   cell), PROL a leaf whose children are halo cells (the prolongation cache,
   grid/tree.h:646-648) */
enum { BMG_T_ACTIVE = 1, BMG_T_LEAF = 2, BMG_T_HALO = 4, BMG_T_PROL = 8 };

/* rule of one ghost cell of the box boundary (grid/tree.h:1139-1209):
   NORMAL takes bc(side1) of the interior cell, DIAGONAL
   bc(side1) + bc(side2) - s[interior] */
enum { BMG_T_NORMAL = 1, BMG_T_DIAGONAL = 2 };
typedef struct {
  uint32_t ghost, inner;   /* packed cells, same level */
  uint32_t kind_sides;     /* kind << 8 | side2 << 4 | side1 */
  uint32_t tidx;           /* tidx2 << 16 | tidx1: tangential face index */
} bmg_tree_rule;

/* the levels of the grid as the tree kernels see them: an all-level field
   buffer holds level l at element offset off[l] with geometry g[l] */
typedef struct {
  bmg_geom g[BMG_TREE_MAXLEVEL + 1];
  long long off[BMG_TREE_MAXLEVEL + 1];
  double Delta[BMG_TREE_MAXLEVEL + 1];
} bmg_tree_levels;

/* a coefficient over all levels: an all-level array, or a constant */
typedef struct {
  const double * p;
  double c;
} bmg_tree_coef;

/* a coefficient of the mixed form's FP32 cycle: an all-level FP32 array
   (the same element layout as the FP64 one), or a constant */
typedef struct {
  const float * p;
  double c;
} bmg_tree_coef32;

/* box conditions of one cell field, per level (NULL values: the constant) */
typedef struct {
  int type[4];
  double cval[4];
  const double * val[4][BMG_TREE_MAXLEVEL + 1];
} bmg_tree_bc;

int bmg_tree_launch_set (const uint32_t * list, long n, const bmg_tree_levels * T,
                         double * s, double v, cudaStream_t st);
int bmg_tree_launch_prolong (const uint32_t * list, long n, const bmg_tree_levels * T,
                             double * s, cudaStream_t st);
int bmg_tree_launch_halo (const uint32_t * list, long n, const bmg_tree_levels * T,
                          double * s, cudaStream_t st);
int bmg_tree_launch_restrict (const uint32_t * list, long n, const bmg_tree_levels * T,
                              double * s, cudaStream_t st);
int bmg_tree_launch_restrict_faces (const uint32_t * list, long n, const bmg_tree_levels * T,
                                    const unsigned char * flags, double * ax, double * ay,
                                    cudaStream_t st);
int bmg_tree_launch_bc (const bmg_tree_rule * rules, long n, const bmg_tree_levels * T,
                        double * s, const bmg_tree_bc * bc, int homogeneous, cudaStream_t st);
/* one stage of a scheduled tree boundary: op (restriction of the listed
   refined cells, or bilinear prolongation into the halo children of the
   listed prolongation leaves, or nothing) together with a span of ghost
   rules, in one launch */
enum { BMG_T_OP_NONE = 0, BMG_T_OP_RESTRICT = 1, BMG_T_OP_HALO = 2 };
int bmg_tree_launch_stage (const uint32_t * list, long n, int op, const bmg_tree_rule * rules,
                           long nrules, const bmg_tree_levels * T, double * s,
                           const bmg_tree_bc * bc, int homogeneous, cudaStream_t st);
/* out = n/d of relax (poisson.h:303-320) for the listed cells: out = a for
   an in-place colour pass, the Jacobi temporary otherwise */
int bmg_tree_launch_relax (const uint32_t * list, long n, const bmg_tree_levels * T,
                           const double * a, const double * b, bmg_tree_coef ax,
                           bmg_tree_coef ay, bmg_tree_coef lambda, double * out,
                           cudaStream_t st);
int bmg_tree_launch_jacobi (const uint32_t * list, long n, const bmg_tree_levels * T,
                            double * a, const double * c, cudaStream_t st);
int bmg_tree_launch_residual (const uint32_t * leaves, long n, const bmg_tree_levels * T,
                              const unsigned char * flags, const double * a, const double * b,
                              bmg_tree_coef ax, bmg_tree_coef ay, bmg_tree_coef lambda,
                              double * res, unsigned long long * maxres, cudaStream_t st);
int bmg_tree_launch_add (const uint32_t * leaves, long n, const bmg_tree_levels * T,
                         double * a, const double * da, cudaStream_t st);
/* one operation of the schedule interpreter: the one-operation launch it
   stands for (type), its cell list and ghost rules, the field it works on
   (0 a, 1 da, 2 res, 3 the Jacobi temporary), the boundary conditions of a
   ghost rule (bcsel: 0 those of a, 1 those of da) and whether they are
   homogeneous; sub is a stage's operation, or for a relaxation 1 when it
   writes the Jacobi temporary; v is the value of a set; local marks an
   operation small enough for one CTA (the interpreter runs it on the
   cluster's first CTA alone and separates two consecutive local
   operations by a CTA barrier instead of a cluster barrier) */
enum { BMG_TI_SET = 0, BMG_TI_PROLONG, BMG_TI_RESTRICT, BMG_TI_STAGE, BMG_TI_RELAX,
       BMG_TI_JACOBI, BMG_TI_ADD, BMG_TI_RESIDUAL };
typedef struct {
  const uint32_t * list;
  long long n;
  const bmg_tree_rule * rules;
  long long nr;
  int type, sub, field, bcsel, homog, local;
  double v;
} bmg_tree_op;
/* the operations ops[0..nops) in order, in one launch of one thread-block
   cluster (16 CTAs, or 8 where 16 cannot be scheduled): fields = {a, da,
   res, tmp}, b the right-hand side, coefs = {alpha_x, alpha_y, lambda},
   bcs = {those of a, those of da}; the residual operations' maximum goes
   to maxres */
int bmg_tree_interp_available (void);
int bmg_tree_launch_interp (const bmg_tree_op * ops, int nops, const bmg_tree_levels * T,
                            double * const * fields, const double * b, const unsigned char * flags,
                            const bmg_tree_coef * coefs, const bmg_tree_bc * bcs,
                            unsigned long long * maxres, cudaStream_t st);

/* the same operations in the mixed form: the cycle's fields
   fields32 = {da, res, tmp} and its coefficients coefs32 are FP32 (same
   element layout as the FP64 arrays), a, b and the residual (coefs) FP64;
   the residual operation stores the FP64 residual rounded to FP32 into
   res, and the correction adds the FP32 da to the FP64 a */
int bmg_tree_launch_interp_mixed (const bmg_tree_op * ops, int nops, const bmg_tree_levels * T,
                                  double * a, float * const * fields32, const double * b,
                                  const unsigned char * flags, const bmg_tree_coef * coefs,
                                  const bmg_tree_coef32 * coefs32, const bmg_tree_bc * bcs,
                                  unsigned long long * maxres, cudaStream_t st);
/* dst[k] = (float) src[k], 0 <= k < n */
int bmg_tree_launch_to_f32 (const double * src, float * dst, long long n, cudaStream_t st);

/* deterministic sum over the listed cells: per-block partials, then one
   block; npartials at most 1024 */
int bmg_tree_launch_sum (const uint32_t * list, long n, const bmg_tree_levels * T,
                         const double * s, double * partials, int npartials, double * out,
                         cudaStream_t st);

#ifdef __cplusplus
}
#endif
#endif

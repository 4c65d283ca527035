/*
 * mg_tree.cu -- CUDA kernels of the quadtree path (two dimensions, FP64).
 *
 * Every kernel walks a cell list (mg_tree.h) with a grid-stride loop: the
 * tree's cells of one kind on one or several levels, whose data sit in the
 * dense level arrays of the grid.  The arithmetic follows the reference's
 * evaluation order, so that FP64 results are bit-identical to the oracle
 * (built with --fmad=false like the rest of the library):
 *   restriction_average, face_average   grid/multigrid-common.h:26-55
 *   bilinear, refine_bilinear           grid/multigrid-common.h:124-146
 *   box boundary on trees               grid/tree.h:1139-1209, 1286-1367
 *   relax                               poisson.h:303-320
 *   residual, tree branch + halo_face   poisson.h:355-372,
 *                                       grid/tree-common.h:374-411
 */
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>
#include "basilisk_mg.h"
#include "mg_device.cuh"
#include "mg_tree.h"

using namespace bmgd;

namespace {

typedef bmg_tree_levels TL;

__device__ __forceinline__ void unpack (uint32_t e, int & l, int & i, int & j)
{
  l = (int) (e >> 28);
  i = (int) ((e >> 14) & 0x3FFFu) - 1;
  j = (int) (e & 0x3FFFu) - 1;
}

/* element index of cell (i, j) of level l in an all-level buffer */
__device__ __forceinline__ long long gidx (const TL & T, int l, int i, int j)
{
  return T.off[l] + cidx<2> (T.g[l], i, j, 0);
}

__device__ __forceinline__ double coef (const bmg_tree_coef & c, long long id)
{
  return c.p ? c.p[id] : c.c;
}

/* a field value: a plain load in the one-operation kernels, an L2 load
   (ld.global.cg) in the interpreter, whose fields other CTAs write during
   the launch (L1 is not coherent across SMs) */
template <bool CG, typename R>
__device__ __forceinline__ R ldf (const R * p)
{
  return CG ? __ldcg (p) : *p;
}

/* a coefficient of the mixed form's FP32 cycle */
__device__ __forceinline__ float coef (const bmg_tree_coef32 & c, long long id)
{
  return c.p ? c.p[id] : (float) c.c;
}

#define GRID_STRIDE(k, n) \
  for (long k = (long) blockIdx.x*blockDim.x + threadIdx.x; k < (n); k += (long) gridDim.x*blockDim.x)

__global__ void k_set (const uint32_t * __restrict__ list, long n, TL T, double * s, double v)
{
  pdl_wait ();
  pdl_trigger ();
  GRID_STRIDE (k, n) {
    int l, i, j;
    unpack (list[k], l, i, j);
    s[gidx (T, l, i, j)] = v;
  }
}

/* bilinear (multigrid-common.h:124-140) of child (i, j) of level l from
   level l - 1 */
template <bool CG = false, typename R = double>
__device__ __forceinline__ R bilinear (const TL & T, const R * s, int l, int i, int j)
{
  const int pi = i >> 1, pj = j >> 1, cx = (i & 1) ? 1 : -1, cy = (j & 1) ? 1 : -1;
  const R * c = s + T.off[l - 1];
  const bmg_geom & gc = T.g[l - 1];
  return ((R) 9*ldf<CG> (c + cidx<2> (gc, pi, pj, 0)) +
          (R) 3*(ldf<CG> (c + cidx<2> (gc, pi + cx, pj, 0)) + ldf<CG> (c + cidx<2> (gc, pi, pj + cy, 0))) +
          ldf<CG> (c + cidx<2> (gc, pi + cx, pj + cy, 0)))/(R) 16;
}

/* foreach_level (l) s[] = bilinear (point, s) (poisson.h:64-68) */
__global__ void k_prolong (const uint32_t * __restrict__ list, long n, TL T, double * s)
{
  pdl_wait ();
  pdl_trigger ();
  GRID_STRIDE (k, n) {
    int l, i, j;
    unpack (list[k], l, i, j);
    s[gidx (T, l, i, j)] = bilinear (T, s, l, i, j);
  }
}

/* refine_bilinear of the halo children of prolongation leaves: one thread
   per child */
template <bool CG = false, typename R = double>
__device__ __forceinline__ void halo_child (const uint32_t * list, long k, const TL & T, R * s)
{
  int l, i, j;
  unpack (list[k >> 2], l, i, j);
  const int ci = 2*i + (int) ((k >> 1) & 1), cj = 2*j + (int) (k & 1);
  s[gidx (T, l + 1, ci, cj)] = bilinear<CG> (T, s, l + 1, ci, cj);
}

__global__ void k_halo (const uint32_t * __restrict__ list, long n, TL T, double * s)
{
  pdl_wait ();
  pdl_trigger ();
  GRID_STRIDE (k, 4*n)
    halo_child (list, k, T, s);
}

/* restriction_average (multigrid-common.h:26-32), children in foreach_child
   order */
template <bool CG = false, typename R = double>
__device__ __forceinline__ void restrict_cell (const uint32_t * list, long k, const TL & T, R * s)
{
  int l, i, j;
  unpack (list[k], l, i, j);
  const R * f = s + T.off[l + 1];
  const bmg_geom & gf = T.g[l + 1];
  R sum = 0.;
  sum += ldf<CG> (f + cidx<2> (gf, 2*i, 2*j, 0));
  sum += ldf<CG> (f + cidx<2> (gf, 2*i, 2*j + 1, 0));
  sum += ldf<CG> (f + cidx<2> (gf, 2*i + 1, 2*j, 0));
  sum += ldf<CG> (f + cidx<2> (gf, 2*i + 1, 2*j + 1, 0));
  s[gidx (T, l, i, j)] = sum/(R) (1 << 2);
}

__global__ void k_restrict (const uint32_t * __restrict__ list, long n, TL T, double * s)
{
  pdl_wait ();
  pdl_trigger ();
  GRID_STRIDE (k, n)
    restrict_cell (list, k, T, s);
}

__device__ __forceinline__ bool refined_at (const TL & T, const unsigned char * fl, int l, int i, int j)
{
  const int n = T.g[l].n;
  if (i < 0 || j < 0 || i >= n || j >= n) return false;
  const unsigned char f = fl[gidx (T, l, i, j)];
  return (f & BMG_T_ACTIVE) && !(f & BMG_T_LEAF);
}

/* face_average (multigrid-common.h:42-55) of the refined cells of one
   level: each cell writes its left and bottom faces, and its right and top
   faces unless the neighbour there is refined too (which writes the same
   value as its own left/bottom face) */
__global__ void k_restrict_faces (const uint32_t * __restrict__ list, long n, TL T,
                                  const unsigned char * __restrict__ fl, double * ax, double * ay)
{
  pdl_wait ();
  pdl_trigger ();
  GRID_STRIDE (k, n) {
    int l, i, j;
    unpack (list[k], l, i, j);
    const bmg_geom & gf = T.g[l + 1];
    const double * fx = ax + T.off[l + 1], * fy = ay + T.off[l + 1];
    ax[gidx (T, l, i, j)] = (fx[cidx<2> (gf, 2*i, 2*j, 0)] + fx[cidx<2> (gf, 2*i, 2*j + 1, 0)])/2.;
    if (!refined_at (T, fl, l, i + 1, j))
      ax[gidx (T, l, i + 1, j)] = (fx[cidx<2> (gf, 2*i + 2, 2*j, 0)] +
                                   fx[cidx<2> (gf, 2*i + 2, 2*j + 1, 0)])/2.;
    ay[gidx (T, l, i, j)] = (fy[cidx<2> (gf, 2*i, 2*j, 0)] + fy[cidx<2> (gf, 2*i + 1, 2*j, 0)])/2.;
    if (!refined_at (T, fl, l, i, j + 1))
      ay[gidx (T, l, i, j + 1)] = (fy[cidx<2> (gf, 2*i, 2*j + 2, 0)] +
                                   fy[cidx<2> (gf, 2*i + 1, 2*j + 2, 0)])/2.;
  }
}

/* s.boundary[side](interior, ghost) of common.h:957-960 */
__device__ __forceinline__ double bc_of (const bmg_tree_bc & bc, int side, int l, int tidx,
                                         double sn, double Delta, int homog)
{
  const double * v = bc.val[side][l];
  const double val = v ? v[tidx] : bc.cval[side];
  if (bc.type[side] == BMG_DIRICHLET)
    return homog ? - sn : 2.*val - sn;
  return homog ? sn : Delta*val + sn;
}

template <bool CG = false, typename R = double>
__device__ __forceinline__ void ghost_value (const bmg_tree_rule & r, const TL & T, R * s,
                                             const bmg_tree_bc & bc, int homog)
{
  int l, gi, gj, l2, a, b;
  unpack (r.ghost, l, gi, gj);
  unpack (r.inner, l2, a, b);
  const long long nid = gidx (T, l, a, b);
  const double sn = ldf<CG> (s + nid), D = T.Delta[l];
  const int s1 = r.kind_sides & 15, s2 = (r.kind_sides >> 4) & 15, kind = r.kind_sides >> 8;
  const int t1 = r.tidx & 0xFFFF, t2 = r.tidx >> 16;
  double v = bc_of (bc, s1, l, t1, sn, D, homog);
  if (kind == BMG_T_DIAGONAL)
    v = (v + bc_of (bc, s2, l, t2, sn, D, homog) - sn);
  s[gidx (T, l, gi, gj)] = (R) v;
}

__global__ void k_bc (const bmg_tree_rule * __restrict__ rules, long n, TL T, double * s,
                      bmg_tree_bc bc, int homog)
{
  pdl_wait ();
  pdl_trigger ();
  GRID_STRIDE (k, n)
    ghost_value (rules[k], T, s, bc, homog);
}

/* one stage of a scheduled tree boundary: a restriction or halo
   prolongation level (op) and, in the same launch, ghost cells whose
   interior values were final before it and which it does not read */
__global__ void k_stage (const uint32_t * __restrict__ list, long n, int op,
                         const bmg_tree_rule * __restrict__ rules, long nr, TL T, double * s,
                         bmg_tree_bc bc, int homog)
{
  pdl_wait ();
  pdl_trigger ();
  const long w = op == BMG_T_OP_HALO ? 4*n : op == BMG_T_OP_RESTRICT ? n : 0;
  GRID_STRIDE (k, w + nr) {
    if (k >= w) ghost_value (rules[k - w], T, s, bc, homog);
    else if (op == BMG_T_OP_HALO) halo_child (list, k, T, s);
    else restrict_cell (list, k, T, s);
  }
}

/* relax (poisson.h:303-320) of one listed cell; x is the first index
   (stride P), y the second */
template <bool CG = false, typename R = double, typename CO = bmg_tree_coef>
__device__ __forceinline__ void relax_item (uint32_t e, const TL & T, const R * a,
                                            const R * b, const CO & ax, const CO & ay,
                                            const CO & lam, R * out)
{
  int l, i, j;
  unpack (e, l, i, j);
  const long long id = gidx (T, l, i, j), P = T.g[l].P;
  const R Delta = (R) T.Delta[l];
  R nn = - (Delta*Delta)*ldf<CG> (b + id), d = - coef (lam, id)*(Delta*Delta);
  const R x1 = coef (ax, id + P), x0 = coef (ax, id);
  nn += x1*ldf<CG> (a + id + P) + x0*ldf<CG> (a + id - P);
  d += x1 + x0;
  const R y1 = coef (ay, id + 1), y0 = coef (ay, id);
  nn += y1*ldf<CG> (a + id + 1) + y0*ldf<CG> (a + id - 1);
  d += y1 + y0;
  out[id] = nn/d;
}

__global__ void k_relax (const uint32_t * __restrict__ list, long n, TL T,
                         const double * a, const double * __restrict__ b,
                         bmg_tree_coef ax, bmg_tree_coef ay, bmg_tree_coef lam, double * out)
{
  pdl_wait ();
  pdl_trigger ();
  GRID_STRIDE (k, n)
    relax_item (list[k], T, a, b, ax, ay, lam, out);
}

/* weighted Jacobi (poisson.h:325-328) */
__global__ void k_jacobi (const uint32_t * __restrict__ list, long n, TL T, double * a,
                          const double * __restrict__ c)
{
  pdl_wait ();
  pdl_trigger ();
  GRID_STRIDE (k, n) {
    int l, i, j;
    unpack (list[k], l, i, j);
    const long long id = gidx (T, l, i, j);
    a[id] = (a[id] + 2.*c[id])/3.;
  }
}

/* g.x = alpha.x face_gradient_x (a, 0) on the left face of (i, j) */
template <bool CG = false>
__device__ __forceinline__ double gx (const TL & T, const double * a, const bmg_tree_coef & ax,
                                      int l, int i, int j)
{
  const long long id = gidx (T, l, i, j);
  return coef (ax, id)*((ldf<CG> (a + id) - ldf<CG> (a + id - T.g[l].P))/T.Delta[l]);
}

template <bool CG = false>
__device__ __forceinline__ double gy (const TL & T, const double * a, const bmg_tree_coef & ay,
                                      int l, int i, int j)
{
  const long long id = gidx (T, l, i, j);
  return coef (ay, id)*((ldf<CG> (a + id) - ldf<CG> (a + id - 1))/T.Delta[l]);
}

/* atomicMax on the bits of a non-negative double (NaN sorts above inf) */
__device__ __forceinline__ void max_bits (unsigned long long * m, double v)
{
  atomicMax (m, (unsigned long long) __double_as_longlong (v));
}

/* residual, tree branch (poisson.h:355-372): a leaf face shared with a
   refined neighbour carries the mean of the two fine fluxes (halo_face) */
template <bool CG = false, typename R = double>
__device__ __forceinline__ double residual_item (uint32_t e, const TL & T, const unsigned char * fl,
                                                 const double * a, const double * b,
                                                 const bmg_tree_coef & ax, const bmg_tree_coef & ay,
                                                 const bmg_tree_coef & lam, R * res)
{
  int l, i, j;
  unpack (e, l, i, j);
  const long long id = gidx (T, l, i, j);
  const double Delta = T.Delta[l];
  const double gl = refined_at (T, fl, l, i - 1, j) ?
    (gx<CG> (T, a, ax, l + 1, 2*i, 2*j) + gx<CG> (T, a, ax, l + 1, 2*i, 2*j + 1))/2. :
    gx<CG> (T, a, ax, l, i, j);
  const double gr = refined_at (T, fl, l, i + 1, j) ?
    (gx<CG> (T, a, ax, l + 1, 2*i + 2, 2*j) + gx<CG> (T, a, ax, l + 1, 2*i + 2, 2*j + 1))/2. :
    gx<CG> (T, a, ax, l, i + 1, j);
  const double gb = refined_at (T, fl, l, i, j - 1) ?
    (gy<CG> (T, a, ay, l + 1, 2*i, 2*j) + gy<CG> (T, a, ay, l + 1, 2*i + 1, 2*j))/2. :
    gy<CG> (T, a, ay, l, i, j);
  const double gt = refined_at (T, fl, l, i, j + 1) ?
    (gy<CG> (T, a, ay, l + 1, 2*i, 2*j + 2) + gy<CG> (T, a, ay, l + 1, 2*i + 1, 2*j + 2))/2. :
    gy<CG> (T, a, ay, l, i, j + 1);
  double r = b[id] - coef (lam, id)*ldf<CG> (a + id);
  r -= (gr - gl)/Delta;
  r -= (gt - gb)/Delta;
  res[id] = (R) r;
  return r;
}

__global__ void k_residual (const uint32_t * __restrict__ list, long n, TL T,
                            const unsigned char * __restrict__ fl, const double * __restrict__ a,
                            const double * __restrict__ b, bmg_tree_coef ax, bmg_tree_coef ay,
                            bmg_tree_coef lam, double * res, unsigned long long * maxres)
{
  pdl_wait ();
  pdl_trigger ();
  double m = 0.;
  GRID_STRIDE (k, n) {
    const double ar = fabs (residual_item (list[k], T, fl, a, b, ax, ay, lam, res));
    if (m == m && !(ar <= m)) m = ar;       /* a NaN sticks */
  }
  /* warp maximum, then one atomic per warp */
  for (int o = 16; o > 0; o >>= 1) {
    const double v = __shfl_down_sync (0xffffffffu, m, o);
    if (m == m && !(v <= m)) m = v;
  }
  if ((threadIdx.x & 31) == 0 && m != 0.)
    max_bits (maxres, m);
}

__global__ void k_add (const uint32_t * __restrict__ list, long n, TL T, double * a,
                       const double * __restrict__ da)
{
  pdl_wait ();
  pdl_trigger ();
  GRID_STRIDE (k, n) {
    int l, i, j;
    unpack (list[k], l, i, j);
    const long long id = gidx (T, l, i, j);
    a[id] += da[id];
  }
}

/* two-stage deterministic sum: fixed grid, fixed reduction tree */
__global__ void k_sum_partial (const uint32_t * __restrict__ list, long n, TL T,
                               const double * __restrict__ s, double * partials)
{
  pdl_wait ();
  pdl_trigger ();
  __shared__ double sh[256];
  double v = 0.;
  GRID_STRIDE (k, n) {
    int l, i, j;
    unpack (list[k], l, i, j);
    v += s[gidx (T, l, i, j)];
  }
  sh[threadIdx.x] = v;
  __syncthreads ();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int) threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads ();
  }
  if (threadIdx.x == 0) partials[blockIdx.x] = sh[0];
}

__global__ void k_sum_final (const double * __restrict__ partials, int np, double * out)
{
  pdl_wait ();
  pdl_trigger ();
  __shared__ double sh[1024];
  sh[threadIdx.x] = (int) threadIdx.x < np ? partials[threadIdx.x] : 0.;
  __syncthreads ();
  for (int w = 512; w > 0; w >>= 1) {
    if ((int) threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads ();
  }
  if (threadIdx.x == 0) *out = sh[0];
}

/* ---------------------------------------------------------------- */
/* the schedule interpreter                                          */
/* ---------------------------------------------------------------- */

/* One mg_solve iteration on a tree (the cycle and the residual) is a fixed
   sequence of a few thousand small list operations, each of which depends
   on the one before.  k_tree_interp runs such a sequence (bmg_tree_op
   records, built on the host in the order of the launches they replace)
   in one launch of one thread-block cluster: every operation's items are
   spread over the cluster's threads, and the cluster barrier
   (release/acquire at cluster scope) separates an operation from the next;
   field values are loaded from L2, since other CTAs of the cluster wrote
   them.  Every item is computed by the function the one-operation kernel
   uses, so the results are bit-identical.  The residual's maximum is
   reduced per warp into maxres (zeroed before the launch). */
/* How the interpreter loads field values that earlier operations of the
   launch wrote: plain (L1-cached) loads.  Every operation is separated
   from the next by a cluster barrier with release/acquire semantics at
   cluster scope, or, between two operations the first CTA runs alone, by
   that CTA's barrier; under the PTX memory model these order every write
   of one operation before every read of the next (the program has no data
   race), so weak loads observe them -- the L1 of an SM cannot serve a
   value older than the acquire. */
constexpr bool ICG = false;

/* The list operations that work on one field s of the scalar type S: a
   set, prolongation, restriction or boundary stage (the interpreter's
   field 0, a, is FP64; the cycle's fields have the cycle's type) */
template <typename S>
__device__ __forceinline__ void field_op (const bmg_tree_op & op, long gt, long gs, uint32_t first,
                                          const TL & T, S * s, const bmg_tree_bc & bc)
{
  const uint32_t * list = op.list;
#define ENTRY(k) ((k) == gt ? first : list[k])
  switch (op.type) {
  case BMG_TI_SET:
    for (long k = gt; k < op.n; k += gs) {
      int l, i, j;
      unpack (ENTRY (k), l, i, j);
      s[gidx (T, l, i, j)] = (S) op.v;
    }
    break;
  case BMG_TI_PROLONG:
    for (long k = gt; k < op.n; k += gs) {
      int l, i, j;
      unpack (ENTRY (k), l, i, j);
      s[gidx (T, l, i, j)] = bilinear<ICG> (T, s, l, i, j);
    }
    break;
  case BMG_TI_RESTRICT:
    for (long k = gt; k < op.n; k += gs)
      restrict_cell<ICG> (list, k, T, s);
    break;
  case BMG_TI_STAGE: {
    const long w = op.sub == BMG_T_OP_HALO ? 4*op.n : op.sub == BMG_T_OP_RESTRICT ? op.n : 0;
    for (long k = gt; k < w + op.nr; k += gs) {
      if (k >= w) ghost_value<ICG> (op.rules[k - w], T, s, bc, op.homog);
      else if (op.sub == BMG_T_OP_HALO) halo_child<ICG> (list, k, T, s);
      else restrict_cell<ICG> (list, k, T, s);
    }
    break;
  }
  }
#undef ENTRY
}

/* One mg_solve iteration on a tree (the cycle and the residual) is a fixed
   sequence of a few thousand small list operations, each of which depends
   on the one before.  k_tree_interp runs such a sequence (bmg_tree_op
   records, built on the host in the order of the launches they replace)
   in one launch of one thread-block cluster: every operation's items are
   spread over the cluster's threads, and the cluster barrier
   (release/acquire at cluster scope) separates an operation from the next;
   field values are loaded from L2, since other CTAs of the cluster wrote
   them.  Every item is computed by the function the one-operation kernel
   uses, so the results are bit-identical.  The residual's maximum is
   reduced per warp into maxres (zeroed before the launch).
   R is the cycle's type: double for the plain form; float for the mixed
   form, whose correction da, restricted residual res and Jacobi temporary
   are FP32 with FP32 coefficients (rax, ray, rlam), while a, b and the
   residual itself (ax, ay, lam) stay FP64 and res receives the FP64
   residual rounded to FP32.
   A local operation (few items, most of a tree boundary's stages) runs on
   the first CTA alone; two consecutive local operations are separated by
   that CTA's barrier (its own global writes are visible to it after
   bar.sync), and a cluster barrier separates every other pair, so the
   other CTAs wait at the cluster barrier that ends a run of local
   operations. */
template <int C, typename R, typename CO>
__global__ void __launch_bounds__ (1024, 1)
k_tree_interp (const bmg_tree_op * __restrict__ ops, int nops, TL Tp, double * fa, R * fda,
               R * fres, R * ftmp, const double * __restrict__ b,
               const unsigned char * __restrict__ fl, bmg_tree_coef ax, bmg_tree_coef ay,
               bmg_tree_coef lam, CO rax, CO ray, CO rlam, bmg_tree_bc bc0, bmg_tree_bc bc1,
               unsigned long long * maxres)
{
  constexpr int CH = 256;                       /* operations staged per chunk */
  __shared__ TL T;
  __shared__ bmg_tree_bc B[2];
  __shared__ bmg_tree_op sops[CH];
  if (threadIdx.x == 0) { T = Tp; B[0] = bc0; B[1] = bc1; }
  unsigned rank;
  asm volatile ("mov.u32 %0, %%cluster_ctarank;" : "=r"(rank));
  const long gt = (long) rank*blockDim.x + threadIdx.x, gs = (long) C*blockDim.x;
  R * const F[4] = {NULL, fda, fres, ftmp};
  double m = 0.;
  /* the list entry of the thread's first item of the current operation,
     loaded while the previous one waited at the barrier */
  uint32_t first = 0;
  for (int o = 0; o < nops; o++) {
    if (o % CH == 0) {
      /* the next chunk of operations into shared memory (after the
         barrier that ended the last chunk's operation) */
      __syncthreads ();
      const int nc = nops - o < CH ? nops - o : CH;
      const int words = nc*(int) (sizeof (bmg_tree_op)/8);
      const unsigned long long * src = (const unsigned long long *) (ops + o);
      unsigned long long * dst = (unsigned long long *) sops;
      for (int w = threadIdx.x; w < words; w += blockDim.x) dst[w] = src[w];
      __syncthreads ();
      const long n0 = sops[0].local ? (rank == 0 ? (long) threadIdx.x : 1L << 62) : gt;
      if (n0 < sops[0].n && sops[0].list) first = sops[0].list[n0];
    }
    const bmg_tree_op & op = sops[o % CH];
    const uint32_t * list = op.list;
    /* the items of this CTA: the whole cluster's share, or all of a local
       operation on the first CTA (none on the others) */
    const long g0 = op.local ? (rank == 0 ? (long) threadIdx.x : 1L << 62) : gt;
    const long gsx = op.local ? (long) blockDim.x : gs;
#define ENTRY(k) ((k) == g0 ? first : list[k])
    switch (op.type) {
    case BMG_TI_SET:
    case BMG_TI_PROLONG:
    case BMG_TI_RESTRICT:
    case BMG_TI_STAGE:
      if (op.field == 0) field_op (op, g0, gsx, first, T, fa, B[op.bcsel]);
      else field_op (op, g0, gsx, first, T, F[op.field], B[op.bcsel]);
      break;
    case BMG_TI_RELAX:
      for (long k = g0; k < op.n; k += gsx)
        relax_item<ICG> (ENTRY (k), T, (const R *) fda, (const R *) fres, rax, ray, rlam,
                          op.sub ? ftmp : fda);
      break;
    case BMG_TI_JACOBI:
      for (long k = g0; k < op.n; k += gsx) {
        int l, i, j;
        unpack (ENTRY (k), l, i, j);
        const long long id = gidx (T, l, i, j);
        fda[id] = (ldf<ICG> (fda + id) + (R) 2*ldf<ICG> (ftmp + id))/(R) 3;
      }
      break;
    case BMG_TI_ADD:
      for (long k = g0; k < op.n; k += gsx) {
        int l, i, j;
        unpack (ENTRY (k), l, i, j);
        const long long id = gidx (T, l, i, j);
        fa[id] = ldf<ICG> (fa + id) + (double) ldf<ICG> (fda + id);
      }
      break;
    case BMG_TI_RESIDUAL:
      for (long k = g0; k < op.n; k += gsx) {
        const double ar = fabs (residual_item<ICG> (ENTRY (k), T, fl, fa, b, ax, ay, lam, fres));
        if (m == m && !(ar <= m)) m = ar;   /* a NaN sticks */
      }
      break;
    }
#undef ENTRY
    /* the next operation's first list entry of this thread (the lists are
       constant during the launch), then the barrier: a CTA barrier of the
       first CTA between two local operations, else a cluster barrier */
    const int nlocal = o + 1 < nops ? ((o + 1) % CH ? sops[(o + 1) % CH].local
                                                    : __ldg (&ops[o + 1].local)) : 0;
    if (o + 1 < nops && (o + 1) % CH != 0) {
      const bmg_tree_op & nx = sops[(o + 1) % CH];
      const long n0 = nx.local ? (rank == 0 ? (long) threadIdx.x : 1L << 62) : gt;
      if (n0 < nx.n && nx.list) first = nx.list[n0];
    }
    if (op.local && nlocal) {
      if (rank == 0) __syncthreads ();
    }
    else
      asm volatile ("barrier.cluster.arrive.release.aligned;\n"
                    "barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double v = __shfl_down_sync (0xffffffffu, m, o);
    if (m == m && !(v <= m)) m = v;
  }
  if ((threadIdx.x & 31) == 0 && m != 0.)
    max_bits (maxres, m);
}

template <int C, typename R, typename CO>
int launch_interp (const bmg_tree_op * ops, int nops, const TL & T, double * fa, R * const * f,
                   const double * b, const unsigned char * fl, const bmg_tree_coef * co,
                   const CO * rco, const bmg_tree_bc * bc, unsigned long long * maxres,
                   cudaStream_t st)
{
  auto kern = k_tree_interp<C, R, CO>;
  static int ok[64];
  int dev = 0;
  cudaGetDevice (&dev);
  if (dev < 0 || dev >= 64) return (int) cudaErrorInvalidDevice;
  cudaLaunchConfig_t cfg;
  memset (&cfg, 0, sizeof cfg);
  cfg.gridDim = dim3 (C, 1, 1);
  cfg.blockDim = dim3 (1024, 1, 1);
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = C; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  if (!ok[dev]) {
    cudaError_t e = cudaSuccess;
    if (C > 8) e = cudaFuncSetAttribute (kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    int nc = 0;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveClusters (&nc, kern, &cfg);
    cudaGetLastError ();
    ok[dev] = e == cudaSuccess && nc >= 1 ? 1 : -1;
  }
  if (ok[dev] < 0) return -1;
  return (int) cudaLaunchKernelEx (&cfg, kern, ops, nops, T, fa, f[0], f[1], f[2], b, fl,
                                   co[0], co[1], co[2], rco[0], rco[1], rco[2], bc[0], bc[1],
                                   maxres);
}

/* double -> float of n consecutive values (the mixed form's FP32 copies
   of the coefficients and of the initial residual, all levels at once) */
__global__ void k_to_f32 (const double * __restrict__ src, float * __restrict__ dst, long long n)
{
  for (long long k = (long long) blockIdx.x*blockDim.x + threadIdx.x; k < n;
       k += (long long) gridDim.x*blockDim.x)
    dst[k] = (float) src[k];
}

const int NT = 256;

int blocks_for (long work)
{
  long b = (work + NT - 1)/NT;
  if (b > 148*16) b = 148*16;
  return b < 1 ? 1 : (int) b;
}

int status ()
{
  cudaError_t e = cudaGetLastError ();
  return e == cudaSuccess ? 0 : (int) e;
}

} // namespace

extern "C" {

int bmg_tree_launch_set (const uint32_t * list, long n, const bmg_tree_levels * T,
                         double * s, double v, cudaStream_t st)
{
  if (n <= 0) return 0;
  pdl_launch (k_set, dim3 (blocks_for (n)), dim3 (NT), 0, st, list, n, *T, s, v);
  return status ();
}

int bmg_tree_launch_prolong (const uint32_t * list, long n, const bmg_tree_levels * T,
                             double * s, cudaStream_t st)
{
  if (n <= 0) return 0;
  pdl_launch (k_prolong, dim3 (blocks_for (n)), dim3 (NT), 0, st, list, n, *T, s);
  return status ();
}

int bmg_tree_launch_halo (const uint32_t * list, long n, const bmg_tree_levels * T,
                          double * s, cudaStream_t st)
{
  if (n <= 0) return 0;
  pdl_launch (k_halo, dim3 (blocks_for (4*n)), dim3 (NT), 0, st, list, n, *T, s);
  return status ();
}

int bmg_tree_launch_restrict (const uint32_t * list, long n, const bmg_tree_levels * T,
                              double * s, cudaStream_t st)
{
  if (n <= 0) return 0;
  pdl_launch (k_restrict, dim3 (blocks_for (n)), dim3 (NT), 0, st, list, n, *T, s);
  return status ();
}

int bmg_tree_launch_restrict_faces (const uint32_t * list, long n, const bmg_tree_levels * T,
                                    const unsigned char * flags, double * ax, double * ay,
                                    cudaStream_t st)
{
  if (n <= 0) return 0;
  pdl_launch (k_restrict_faces, dim3 (blocks_for (n)), dim3 (NT), 0, st, list, n, *T, flags, ax, ay);
  return status ();
}

int bmg_tree_launch_bc (const bmg_tree_rule * rules, long n, const bmg_tree_levels * T,
                        double * s, const bmg_tree_bc * bc, int homogeneous, cudaStream_t st)
{
  if (n <= 0) return 0;
  pdl_launch (k_bc, dim3 (blocks_for (n)), dim3 (NT), 0, st, rules, n, *T, s, *bc, homogeneous);
  return status ();
}

int bmg_tree_launch_stage (const uint32_t * list, long n, int op, const bmg_tree_rule * rules,
                           long nrules, const bmg_tree_levels * T, double * s,
                           const bmg_tree_bc * bc, int homogeneous, cudaStream_t st)
{
  const long w = (op == BMG_T_OP_HALO ? 4*n : op == BMG_T_OP_RESTRICT ? n : 0) + nrules;
  if (w <= 0) return 0;
  pdl_launch (k_stage, dim3 (blocks_for (w)), dim3 (NT), 0, st, list, n, op, rules, nrules, *T, s, *bc, homogeneous);
  return status ();
}

int bmg_tree_launch_relax (const uint32_t * list, long n, const bmg_tree_levels * T,
                           const double * a, const double * b, bmg_tree_coef ax,
                           bmg_tree_coef ay, bmg_tree_coef lambda, double * out,
                           cudaStream_t st)
{
  if (n <= 0) return 0;
  pdl_launch (k_relax, dim3 (blocks_for (n)), dim3 (NT), 0, st, list, n, *T, a, b, ax, ay, lambda, out);
  return status ();
}

int bmg_tree_launch_jacobi (const uint32_t * list, long n, const bmg_tree_levels * T,
                            double * a, const double * c, cudaStream_t st)
{
  if (n <= 0) return 0;
  pdl_launch (k_jacobi, dim3 (blocks_for (n)), dim3 (NT), 0, st, list, n, *T, a, c);
  return status ();
}

int bmg_tree_launch_residual (const uint32_t * leaves, long n, const bmg_tree_levels * T,
                              const unsigned char * flags, const double * a, const double * b,
                              bmg_tree_coef ax, bmg_tree_coef ay, bmg_tree_coef lambda,
                              double * res, unsigned long long * maxres, cudaStream_t st)
{
  if (n <= 0) return 0;
  pdl_launch (k_residual, dim3 (blocks_for (n)), dim3 (NT), 0, st, leaves, n, *T, flags, a, b, ax, ay, lambda, res, maxres);
  return status ();
}

int bmg_tree_launch_add (const uint32_t * leaves, long n, const bmg_tree_levels * T,
                         double * a, const double * da, cudaStream_t st)
{
  if (n <= 0) return 0;
  pdl_launch (k_add, dim3 (blocks_for (n)), dim3 (NT), 0, st, leaves, n, *T, a, da);
  return status ();
}

int bmg_tree_interp_available (void)
{
  /* a cluster of 16 or 8 CTAs of 1024 threads can be scheduled */
  int dev = 0;
  if (cudaGetDevice (&dev) != cudaSuccess) { cudaGetLastError (); return 0; }
  for (int C = 16; C >= 8; C /= 2) {
    cudaLaunchConfig_t cfg;
    memset (&cfg, 0, sizeof cfg);
    cfg.gridDim = dim3 (C, 1, 1);
    cfg.blockDim = dim3 (1024, 1, 1);
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = C; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int nc = 0;
    cudaError_t e = C > 8 ?
      cudaFuncSetAttribute (k_tree_interp<16, double, bmg_tree_coef>,
                            cudaFuncAttributeNonPortableClusterSizeAllowed, 1) :
      cudaSuccess;
    if (e == cudaSuccess)
      e = C > 8 ? cudaOccupancyMaxActiveClusters (&nc, k_tree_interp<16, double, bmg_tree_coef>, &cfg)
                : cudaOccupancyMaxActiveClusters (&nc, k_tree_interp<8, double, bmg_tree_coef>, &cfg);
    cudaGetLastError ();
    if (e == cudaSuccess && nc >= 1) return 1;
  }
  return 0;
}

int bmg_tree_launch_interp (const bmg_tree_op * ops, int nops, const bmg_tree_levels * T,
                            double * const * fields, const double * b, const unsigned char * flags,
                            const bmg_tree_coef * coefs, const bmg_tree_bc * bcs,
                            unsigned long long * maxres, cudaStream_t st)
{
  if (nops < 1) return 0;
  double * const f[3] = {fields[1], fields[2], fields[3]};
  int e = launch_interp<16> (ops, nops, *T, fields[0], f, b, flags, coefs, coefs, bcs, maxres, st);
  if (e == -1)
    e = launch_interp<8> (ops, nops, *T, fields[0], f, b, flags, coefs, coefs, bcs, maxres, st);
  if (e) return e;
  return status ();
}

int bmg_tree_launch_interp_mixed (const bmg_tree_op * ops, int nops, const bmg_tree_levels * T,
                                  double * a, float * const * fields32, const double * b,
                                  const unsigned char * flags, const bmg_tree_coef * coefs,
                                  const bmg_tree_coef32 * coefs32, const bmg_tree_bc * bcs,
                                  unsigned long long * maxres, cudaStream_t st)
{
  if (nops < 1) return 0;
  int e = launch_interp<16> (ops, nops, *T, a, fields32, b, flags, coefs, coefs32, bcs, maxres, st);
  if (e == -1)
    e = launch_interp<8> (ops, nops, *T, a, fields32, b, flags, coefs, coefs32, bcs, maxres, st);
  if (e) return e;
  return status ();
}

int bmg_tree_launch_to_f32 (const double * src, float * dst, long long n, cudaStream_t st)
{
  if (n <= 0) return 0;
  long long nb = (n + NT - 1)/NT;
  if (nb > 148*8) nb = 148*8;
  k_to_f32<<<(int) nb, NT, 0, st>>> (src, dst, n);
  return status ();
}

int bmg_tree_launch_sum (const uint32_t * list, long n, const bmg_tree_levels * T,
                         const double * s, double * partials, int npartials, double * out,
                         cudaStream_t st)
{
  if (npartials < 1 || npartials > 1024) return (int) cudaErrorInvalidValue;
  pdl_launch (k_sum_partial, dim3 (npartials), dim3 (256), 0, st, list, n, *T, s, partials);
  pdl_launch (k_sum_final, dim3 (1), dim3 (1024), 0, st, partials, npartials, out);
  return status ();
}

} // extern "C"

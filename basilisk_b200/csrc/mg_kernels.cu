/*
 * mg_kernels.cu -- sm_100a stencil kernels of the multigrid
 * Poisson--Helmholtz solver, and their C launchers.
 *
 * One kernel per operation of the reference's V-cycle (Basilisk poisson.h,
 * grid/multigrid.h, grid/multigrid-common.h), each templated on the
 * dimension and on the storage type (double for the plain form, float for
 * the inner cycles of the mixed form):
 *
 *   k_relax        relax (poisson.h:271-338): red/black Gauss-Seidel sweep
 *                  in place, or the -DJACOBI weighted-Jacobi update
 *                  (poisson.h:325-328) from one buffer into another
 *   k_prolong      bilinear prolongation (multigrid-common.h:124-140) or the
 *                  coarsest-level zero (poisson.h:54-58)
 *   k_restrict     restriction_average (multigrid-common.h:26-32)
 *   k_restrict_face face_average (multigrid-common.h:42-58)
 *   k_residual     residual (poisson.h:373-389) fused with the max|res|
 *                  reduction (warp shuffles, one atomic per block)
 *   k_correct      a += da (poisson.h:84-89) fused with the boundary
 *                  conditions of a (the automatic BC of stencils.h:228+)
 *
 * Ghost cells are written by the thread that writes the interior cell they
 * mirror, in the same kernel: box conditions one layer deep in the
 * reference's side order with corners composed dimension by dimension
 * (grid/multigrid.h:543-594), periodic images (grid/multigrid.h:638-695),
 * and the level-0 rule that a periodic level-0 cell is its own neighbour in
 * every direction (grid/multigrid.h:655-664).  No kernel needs a separate
 * boundary pass.
 *
 * Arithmetic follows the reference's evaluation order; the library is
 * compiled with --fmad=false so that the FP64 results are bit-identical to
 * a C build of the same expressions.
 */
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include "mg_launch.h"

#include <string.h>
#include <type_traits>
#include "mg_device.cuh"

using namespace bmgd;

namespace {

template <int DIM, typename T, int MODE>
__global__ void k_relax (bmg_geom g, T * out, const T * in, const T * __restrict__ rhs,
                         Coef<T> ax, Coef<T> ay, Coef<T> az, Coef<T> lam, T Delta, BCH bc)
{
  int i, j, k;
  if (!cell_of_thread<DIM> (g.n, i, j, k)) return;
  if (MODE != BMG_SWEEP_JACOBI && ((i + j + k) & 1) != MODE) return;
  const long long id = cidx<DIM> (g, i, j, k);
  const T D2 = Delta*Delta;
  T c = relax_value<DIM, T> (g, id, in, rhs, ax, ay, az, lam, D2);
  T v;
  if (MODE == BMG_SWEEP_JACOBI)
    v = (in[id] + T(2)*c)/T(3);
  else
    v = c;
  out[id] = v;
  ghosts_homog<DIM, T> (out, g, i, j, k, v, bc);
}

/* one colour pass of a 3D level by cell pairs: thread (q, j, i) owns the
   cells 2q and 2q + 1 of a row, one of each colour, and relaxes the one of
   colour MODE with relax_value's expression and order (bit-identical to
   k_relax); every array is read as aligned pairs, which halves the load
   instructions per byte moved */
template <typename T, int MODE, bool COR>
__global__ void k_relax3_pair (bmg_geom g, T * out, const T * in, const T * __restrict__ rhs,
                               Coef<T> ax, Coef<T> ay, Coef<T> az, Coef<T> lam, T Delta, BCH bc,
                               double * acor, bmg_geom ga, bmg_bcdesc abc)
{
  typedef typename std::conditional<sizeof (T) == 8, double2, float2>::type T2;
  const int q = blockIdx.x*blockDim.x + threadIdx.x;
  const int j = blockIdx.y*blockDim.y + threadIdx.y;
  const int i = blockIdx.z*blockDim.z + threadIdx.z;
  const int n = g.n;
  if (2*q >= n || j >= n || i >= n) return;
  const int o = (MODE + i + j) & 1;              /* the cell of colour MODE */
  const long long p0 = cidx<3> (g, i, j, 2*q), id = p0 + o;
  auto pick = [o] (T2 v) { return o ? v.y : v.x; };
  auto pair = [] (const T * a, long long at) { return *(const T2 *) (a + at); };
  const T D2 = Delta*Delta;
  const T2 c0 = pair (in, p0);
  T nn = (-D2)*pick (pair (rhs, p0));
  T d = (-(lam.p ? pick (pair (lam.p, p0)) : lam.c))*D2;
  {
    const long long s = g.plane;
    const T a1 = ax.p ? pick (pair (ax.p, p0 + s)) : ax.c, a0 = ax.p ? pick (pair (ax.p, p0)) : ax.c;
    nn += a1*pick (pair (in, p0 + s)) + a0*pick (pair (in, p0 - s));
    d += a1 + a0;
  }
  {
    const long long s = g.P;
    const T a1 = ay.p ? pick (pair (ay.p, p0 + s)) : ay.c, a0 = ay.p ? pick (pair (ay.p, p0)) : ay.c;
    nn += a1*pick (pair (in, p0 + s)) + a0*pick (pair (in, p0 - s));
    d += a1 + a0;
  }
  {
    T a1, a0, v1, v0;
    if (o == 0) {
      if (az.p) { const T2 z = pair (az.p, p0); a0 = z.x; a1 = z.y; }
      else a0 = a1 = az.c;
      v1 = c0.y; v0 = in[p0 - 1];
    }
    else {
      if (az.p) { a0 = az.p[p0 + 1]; a1 = az.p[p0 + 2]; }
      else a0 = a1 = az.c;
      v1 = in[p0 + 2]; v0 = c0.x;
    }
    nn += a1*v1 + a0*v0;
    d += a1 + a0;
  }
  const T v = nn/d;
  out[id] = v;
  ghosts_homog<3, T> (out, g, i, j, 2*q + o, v, bc);
  if (COR) {
    /* the last pass of the finest level: both cells of the pair are final
       (the other one since the previous pass), so a += da for the pair,
       with k_correct's expression and the ghost images of a */
    const T d0 = o ? c0.x : v, d1 = o ? v : c0.y;
    const long long ia = cidx<3> (ga, i, j, 2*q);
    const double2 av = *(const double2 *) (acor + ia);
    const double a0 = av.x + (double) d0, a1 = av.y + (double) d1;
    *(double2 *) (acor + ia) = make_double2 (a0, a1);
    ghosts_inhomog<3> (acor, ga, i, j, 2*q, a0, abc);
    ghosts_inhomog<3> (acor, ga, i, j, 2*q + 1, a1, abc);
  }
}

/* ---------------------------------------------------------------- */
/* prolongation / restriction                                        */
/* ---------------------------------------------------------------- */

template <int DIM, typename TC, typename TF>
__global__ void k_prolong (bmg_geom gc, bmg_geom gf, const TC * __restrict__ s,
                           TF * __restrict__ f, BCH bc, int zero)
{
  pdl_wait ();
  pdl_trigger ();
  int i, j, k;
  if (!cell_of_thread<DIM> (gf.n, i, j, k)) return;
  TC v = TC(0);
  if (!zero) {
    const int pi = i >> 1, cx = (i & 1) ? 1 : -1;
    if (DIM == 1)
      v = (TC(3)*s[cidx<1> (gc, pi, 0, 0)] + s[cidx<1> (gc, pi + cx, 0, 0)])/TC(4);
    else if (DIM == 2) {
      const int pj = j >> 1, cy = (j & 1) ? 1 : -1;
      v = (TC(9)*s[cidx<2> (gc, pi, pj, 0)] +
           TC(3)*(s[cidx<2> (gc, pi + cx, pj, 0)] + s[cidx<2> (gc, pi, pj + cy, 0)]) +
           s[cidx<2> (gc, pi + cx, pj + cy, 0)])/TC(16);
    }
    else {
      const int pj = j >> 1, cy = (j & 1) ? 1 : -1;
      const int pk = k >> 1, cz = (k & 1) ? 1 : -1;
      v = (TC(27)*s[cidx<3> (gc, pi, pj, pk)] +
           TC(9)*(s[cidx<3> (gc, pi + cx, pj, pk)] + s[cidx<3> (gc, pi, pj + cy, pk)] +
                  s[cidx<3> (gc, pi, pj, pk + cz)]) +
           TC(3)*(s[cidx<3> (gc, pi + cx, pj + cy, pk)] + s[cidx<3> (gc, pi + cx, pj, pk + cz)] +
                  s[cidx<3> (gc, pi, pj + cy, pk + cz)]) +
           s[cidx<3> (gc, pi + cx, pj + cy, pk + cz)])/TC(64);
    }
  }
  const TF w = (TF) v;
  f[cidx<DIM> (gf, i, j, k)] = w;
  ghosts_homog<DIM, TF> (f, gf, i, j, k, w, bc);
}

/* the 2D bilinear prolongation by coarse cell: one thread reads the 3 x 3
   coarse neighbourhood (ghosts included) once and writes the four children,
   each with k_prolong's expression and order (bit-identical) */
template <typename TC, typename TF>
__global__ void k_prolong2d_blk (bmg_geom gc, bmg_geom gf, const TC * __restrict__ s,
                                 TF * __restrict__ f, BCH bc)
{
  pdl_wait ();
  pdl_trigger ();
  const int cj = blockIdx.x*blockDim.x + threadIdx.x, ci = blockIdx.y*blockDim.y + threadIdx.y;
  if (ci >= gc.n || cj >= gc.n) return;
  TC m[3][3];
#pragma unroll
  for (int di = 0; di < 3; di++)
#pragma unroll
    for (int dj = 0; dj < 3; dj++)
      m[di][dj] = s[cidx<2> (gc, ci + di - 1, cj + dj - 1, 0)];
#pragma unroll
  for (int a = 0; a < 2; a++) {
    TF w[2];
#pragma unroll
    for (int b = 0; b < 2; b++) {
      const int cx = a ? 1 : -1, cy = b ? 1 : -1;
      const TC v = (TC(9)*m[1][1] + TC(3)*(m[1 + cx][1] + m[1][1 + cy]) + m[1 + cx][1 + cy])/TC(16);
      w[b] = (TF) v;
    }
    const int i = 2*ci + a, j = 2*cj;
    TF * q = f + cidx<2> (gf, i, j, 0);
    q[0] = w[0];
    q[1] = w[1];
    ghosts_homog<2, TF> (f, gf, i, j, 0, w[0], bc);
    ghosts_homog<2, TF> (f, gf, i, j + 1, 0, w[1], bc);
  }
}

/* the 3D trilinear prolongation by coarse cell: one thread reads the
   3 x 3 x 3 coarse neighbourhood (ghosts included) once and writes the
   eight children, each with k_prolong's expression and order
   (bit-identical); children along the contiguous axis are written in
   pairs */
template <typename TC, typename TF>
__global__ void k_prolong3d_blk (bmg_geom gc, bmg_geom gf, const TC * __restrict__ s,
                                 TF * __restrict__ f, BCH bc)
{
  pdl_wait ();
  pdl_trigger ();
  const int ck = blockIdx.x*blockDim.x + threadIdx.x;
  const int cj = blockIdx.y*blockDim.y + threadIdx.y;
  const int ci = blockIdx.z*blockDim.z + threadIdx.z;
  if (ci >= gc.n || cj >= gc.n || ck >= gc.n) return;
  TC m[3][3][3];
#pragma unroll
  for (int di = 0; di < 3; di++)
#pragma unroll
    for (int dj = 0; dj < 3; dj++)
#pragma unroll
      for (int dk = 0; dk < 3; dk++)
        m[di][dj][dk] = s[cidx<3> (gc, ci + di - 1, cj + dj - 1, ck + dk - 1)];
#pragma unroll
  for (int a = 0; a < 2; a++)
#pragma unroll
    for (int b = 0; b < 2; b++) {
      TF w[2];
#pragma unroll
      for (int c = 0; c < 2; c++) {
        const int cx = a ? 2 : 0, cy = b ? 2 : 0, cz = c ? 2 : 0;
        const TC v = (TC(27)*m[1][1][1] +
                      TC(9)*(m[cx][1][1] + m[1][cy][1] + m[1][1][cz]) +
                      TC(3)*(m[cx][cy][1] + m[cx][1][cz] + m[1][cy][cz]) +
                      m[cx][cy][cz])/TC(64);
        w[c] = (TF) v;
      }
      const int i = 2*ci + a, j = 2*cj + b, k = 2*ck;
      TF * q = f + cidx<3> (gf, i, j, k);
      q[0] = w[0];
      q[1] = w[1];
      ghosts_homog<3, TF> (f, gf, i, j, k, w[0], bc);
      ghosts_homog<3, TF> (f, gf, i, j, k + 1, w[1], bc);
    }
}

/* coarse = mean of the children, summed in foreach_child order */
template <int DIM, typename TF, typename TC>
__global__ void k_restrict (bmg_geom gf, bmg_geom gc, const TF * __restrict__ f,
                            TC * __restrict__ c)
{
  pdl_wait ();
  pdl_trigger ();
  int i, j, k;
  if (!cell_of_thread<DIM> (gc.n, i, j, k)) return;
  TC sum = TC(0);
  const int fi = 2*i, fj = 2*j, fk = 2*k;
  if (DIM == 1) {
    for (int a = 0; a < 2; a++) sum += (TC) f[cidx<1> (gf, fi + a, 0, 0)];
  }
  else if (DIM == 2) {
    for (int a = 0; a < 2; a++)
      for (int b = 0; b < 2; b++)
        sum += (TC) f[cidx<2> (gf, fi + a, fj + b, 0)];
  }
  else {
    for (int a = 0; a < 2; a++)
      for (int b = 0; b < 2; b++)
        for (int d = 0; d < 2; d++)
          sum += (TC) f[cidx<3> (gf, fi + a, fj + b, fk + d)];
  }
  c[cidx<DIM> (gc, i, j, k)] = sum/TC(1 << DIM);
}

struct FacePtrs {
  const double * f[3];
  double * c[3];
};

/* face_average (multigrid-common.h:42-58) with the foreach_dimension
   rotation of the fine() offsets; every coarse cell writes its lower face,
   the last cell along each axis also its upper face. */
template <int DIM>
__global__ void k_restrict_face (bmg_geom gf, bmg_geom gc, FacePtrs p, int level0p)
{
  int i, j, k;
  if (!cell_of_thread<DIM> (gc.n, i, j, k)) return;
  const int n = gc.n;
#define FV(o0, o1, o2) f[cidx<DIM> (gf, 2*i + (o0), DIM > 1 ? 2*j + (o1) : 0, DIM > 2 ? 2*k + (o2) : 0)]
  for (int e = 0; e < DIM; e++) {
    const double * f = p.f[e];
    double * c = p.c[e];
    const int ce = e == 0 ? i : e == 1 ? j : k;
    for (int side = 0; side < 2; side++) {
      if (side == 1 && ce != n - 1) break;
      const int o = 2*side;
      double v;
      if (DIM == 1)
        v = FV (o, 0, 0);
      else if (DIM == 2)
        v = e == 0 ? (FV (o, 0, 0) + FV (o, 1, 0))/2. : (FV (0, o, 0) + FV (1, o, 0))/2.;
      else {
        if (e == 0)
          v = (FV (o, 0, 0) + FV (o, 1, 0) + FV (o, 0, 1) + FV (o, 1, 1))/4.;
        else if (e == 1)
          v = (FV (0, o, 0) + FV (0, o, 1) + FV (1, o, 0) + FV (1, o, 1))/4.;
        else
          v = (FV (0, 0, o) + FV (1, 0, o) + FV (0, 1, o) + FV (1, 1, o))/4.;
      }
      const int ii = e == 0 ? i + side : i, jj = e == 1 ? j + side : j, kk = e == 2 ? k + side : k;
      c[cidx<DIM> (gc, ii, jj, kk)] = v;
      if (level0p) {
        /* periodic level 0: the upper face is a copy of the lower one */
        c[cidx<DIM> (gc, e == 0 ? 1 : 0, e == 1 ? 1 : 0, e == 2 ? 1 : 0)] = v;
        break;
      }
    }
  }
#undef FV
}

/* ---------------------------------------------------------------- */
/* residual + max reduction                                          */
/* ---------------------------------------------------------------- */

/* max that keeps NaN */
__device__ __forceinline__ double nanmax (double a, double b)
{
  return (a > b || a != a) ? a : b;
}

__device__ __forceinline__ void block_max_atomic (double m, unsigned long long * out)
{
  __shared__ double sm[32];
  const int tid = threadIdx.x + blockDim.x*(threadIdx.y + blockDim.y*threadIdx.z);
  const int lane = tid & 31;
  const int nth = blockDim.x*blockDim.y*blockDim.z;
  for (int o = 16; o > 0; o >>= 1)
    m = nanmax (m, __shfl_xor_sync (0xffffffffu, m, o));
  const int warp = tid >> 5;
  if ((tid & 31) == 0) sm[warp] = m;
  __syncthreads ();
  if (warp == 0) {
    const int nw = (nth + 31) >> 5;
    double v = lane < nw ? sm[lane] : 0.;
    for (int o = 16; o > 0; o >>= 1)
      v = nanmax (v, __shfl_xor_sync (0xffffffffu, v, o));
    if (lane == 0)
      atomicMax (out, (unsigned long long) __double_as_longlong (v));
  }
}

/* x/Delta; when Delta is a power of two (L0 = 1, Delta = 2^-l) the
   division is an exact scaling and x*(1/Delta) is the same double, at a
   fraction of the cost of the IEEE division */
template <bool POW2>
__device__ __forceinline__ double over_delta (double x, double Delta, double rDelta)
{
  return POW2 ? x*rDelta : x/Delta;
}

template <int DIM, typename TR, bool POW2>
__global__ void k_residual (bmg_geom g, bmg_geom gr, const double * __restrict__ a,
                            const double * __restrict__ b, Coef<double> ax,
                            Coef<double> ay, Coef<double> az, Coef<double> lam,
                            double Delta, TR * __restrict__ res,
                            unsigned long long * maxres)
{
  pdl_wait ();
  pdl_trigger ();
  int i, j, k;
  double m = 0.;
  const double rD = 1./Delta;
  if (cell_of_thread<DIM> (g.n, i, j, k)) {
    const long long id = cidx<DIM> (g, i, j, k);
    const double ac = a[id];
    double r = b[id] - lam.at (id)*ac;
    {
      long long s = cstride<DIM> (g, 0);
      r += over_delta<POW2> (ax.at (id)*over_delta<POW2> (ac - a[id - s], Delta, rD) -
                             ax.at (id + s)*over_delta<POW2> (a[id + s] - ac, Delta, rD), Delta, rD);
    }
    if (DIM > 1) {
      long long s = cstride<DIM> (g, 1);
      r += over_delta<POW2> (ay.at (id)*over_delta<POW2> (ac - a[id - s], Delta, rD) -
                             ay.at (id + s)*over_delta<POW2> (a[id + s] - ac, Delta, rD), Delta, rD);
    }
    if (DIM > 2) {
      long long s = cstride<DIM> (g, 2);
      r += over_delta<POW2> (az.at (id)*over_delta<POW2> (ac - a[id - s], Delta, rD) -
                             az.at (id + s)*over_delta<POW2> (a[id + s] - ac, Delta, rD), Delta, rD);
    }
    res[cidx<DIM> (gr, i, j, k)] = (TR) r;
    m = fabs (r);
  }
  block_max_atomic (m, maxres);
}

/* the residual of the finest 2D level fused with its restriction into the
   level below (multigrid-common.h:368-404): each thread computes the four
   residuals of one coarse cell's children with k_residual's expression and
   order, stores them, and stores their mean in k_restrict's order (children
   in foreach_child order, from the stored values), so the results are
   bit-identical to k_residual followed by k_restrict */
template <typename TR, typename TC, bool POW2>
__global__ void k_residual_restrict2d (bmg_geom g, bmg_geom gr, bmg_geom gc,
                                       const double * __restrict__ a,
                                       const double * __restrict__ b, Coef<double> ax,
                                       Coef<double> ay, Coef<double> lam, double Delta,
                                       TR * __restrict__ res, TC * __restrict__ resc,
                                       unsigned long long * maxres)
{
  pdl_wait ();
  pdl_trigger ();
  const int cj = blockIdx.x*blockDim.x + threadIdx.x, ci = blockIdx.y*blockDim.y + threadIdx.y;
  double m = 0.;
  const double rD = 1./Delta;
  if (ci < gc.n && cj < gc.n) {
    TC sum = TC(0);
#pragma unroll
    for (int u = 0; u < 2; u++)
#pragma unroll
      for (int v = 0; v < 2; v++) {
        const int i = 2*ci + u, j = 2*cj + v;
        const long long id = cidx<2> (g, i, j, 0);
        const double ac = a[id];
        double r = b[id] - lam.at (id)*ac;
        {
          const long long s = g.P;
          r += over_delta<POW2> (ax.at (id)*over_delta<POW2> (ac - a[id - s], Delta, rD) -
                                 ax.at (id + s)*over_delta<POW2> (a[id + s] - ac, Delta, rD), Delta, rD);
        }
        r += over_delta<POW2> (ay.at (id)*over_delta<POW2> (ac - a[id - 1], Delta, rD) -
                               ay.at (id + 1)*over_delta<POW2> (a[id + 1] - ac, Delta, rD), Delta, rD);
        const TR rs = (TR) r;
        res[cidx<2> (gr, i, j, 0)] = rs;
        sum += (TC) rs;
        m = nanmax (m, fabs (r));
      }
    resc[cidx<2> (gc, ci, cj, 0)] = sum/TC(4);
  }
  block_max_atomic (m, maxres);
}

/* the same in 3D: each thread computes the eight residuals of one coarse
   cell's children (k_residual's expression and order), stores them, and
   stores their mean in k_restrict's order (children a, b, d nested as in
   foreach_child, from the stored values): bit-identical to k_residual
   followed by k_restrict */
template <typename TR, typename TC, bool POW2>
__global__ void k_residual_restrict3d (bmg_geom g, bmg_geom gr, bmg_geom gc,
                                       const double * __restrict__ a,
                                       const double * __restrict__ b, Coef<double> ax,
                                       Coef<double> ay, Coef<double> az, Coef<double> lam,
                                       double Delta, TR * __restrict__ res, TC * __restrict__ resc,
                                       unsigned long long * maxres)
{
  pdl_wait ();
  pdl_trigger ();
  const int ck = blockIdx.x*blockDim.x + threadIdx.x;
  const int cj = blockIdx.y*blockDim.y + threadIdx.y;
  const int ci = blockIdx.z*blockDim.z + threadIdx.z;
  double m = 0.;
  const double rD = 1./Delta;
  if (ci < gc.n && cj < gc.n && ck < gc.n) {
    TC sum = TC(0);
#pragma unroll
    for (int u = 0; u < 2; u++)
#pragma unroll
      for (int v = 0; v < 2; v++)
#pragma unroll
        for (int w = 0; w < 2; w++) {
          const int i = 2*ci + u, j = 2*cj + v, k = 2*ck + w;
          const long long id = cidx<3> (g, i, j, k);
          const double ac = a[id];
          double r = b[id] - lam.at (id)*ac;
          {
            const long long s = g.plane;
            r += over_delta<POW2> (ax.at (id)*over_delta<POW2> (ac - a[id - s], Delta, rD) -
                                   ax.at (id + s)*over_delta<POW2> (a[id + s] - ac, Delta, rD), Delta, rD);
          }
          {
            const long long s = g.P;
            r += over_delta<POW2> (ay.at (id)*over_delta<POW2> (ac - a[id - s], Delta, rD) -
                                   ay.at (id + s)*over_delta<POW2> (a[id + s] - ac, Delta, rD), Delta, rD);
          }
          r += over_delta<POW2> (az.at (id)*over_delta<POW2> (ac - a[id - 1], Delta, rD) -
                                 az.at (id + 1)*over_delta<POW2> (a[id + 1] - ac, Delta, rD), Delta, rD);
          const TR rs = (TR) r;
          res[cidx<3> (gr, i, j, k)] = rs;
          sum += (TC) rs;
          m = nanmax (m, fabs (r));
        }
    resc[cidx<3> (gc, ci, cj, ck)] = sum/TC(8);
  }
  block_max_atomic (m, maxres);
}

/* ---------------------------------------------------------------- */
/* correction a += da, boundary conditions                           */
/* ---------------------------------------------------------------- */

template <int DIM, typename TD>
__global__ void k_correct (bmg_geom g, bmg_geom gd, double * a, const TD * __restrict__ da,
                           bmg_bcdesc bc)
{
  pdl_wait ();
  pdl_trigger ();
  int i, j, k;
  if (!cell_of_thread<DIM> (g.n, i, j, k)) return;
  const long long id = cidx<DIM> (g, i, j, k);
  const double v = a[id] + (double) da[cidx<DIM> (gd, i, j, k)];
  a[id] = v;
  ghosts_inhomog<DIM> (a, g, i, j, k, v, bc);
}

template <int DIM, typename T>
__global__ void k_apply_bc (bmg_geom g, T * f, bmg_bcdesc bc, BCH h, int homogeneous)
{
  int i, j, k;
  if (!cell_of_thread<DIM> (g.n, i, j, k)) return;
  if (!on_boundary<DIM> (g.n, i, j, k)) return;
  const long long id = cidx<DIM> (g, i, j, k);
  if (homogeneous)
    ghosts_homog<DIM, T> (f, g, i, j, k, f[id], h);
  else
    ghosts_inhomog<DIM> ((double *) f, g, i, j, k, (double) f[id], bc);
}

/* ---------------------------------------------------------------- */
/* sums, packing, conversion                                         */
/* ---------------------------------------------------------------- */

template <int DIM>
__device__ __forceinline__ void decode (long long q, int ni, int nj, int nk, int & i, int & j, int & k)
{
  if (DIM == 1) { i = (int) q; j = k = 0; return; }
  if (DIM == 2) { i = (int) (q/nj); j = (int) (q - (long long) i*nj); k = 0; return; }
  long long ij = q/nk;
  k = (int) (q - ij*nk);
  i = (int) (ij/nj);
  j = (int) (ij - (long long) i*nj);
}

__device__ __forceinline__ double block_sum (double v, double * sm)
{
  const int tid = threadIdx.x;
  for (int o = 16; o > 0; o >>= 1)
    v += __shfl_down_sync (0xffffffffu, v, o);
  if ((tid & 31) == 0) sm[tid >> 5] = v;
  __syncthreads ();
  double r = 0.;
  if (tid < 32) {
    const int nw = blockDim.x >> 5;
    r = tid < nw ? sm[tid] : 0.;
    for (int o = 16; o > 0; o >>= 1)
      r += __shfl_down_sync (0xffffffffu, r, o);
  }
  return r;
}

/* deterministic two-stage sum of the interior (fixed partition, fixed order) */
template <int DIM>
__global__ void k_sum_partial (bmg_geom g, const double * __restrict__ b, double * partials)
{
  __shared__ double sm[32];
  const int n = g.n;
  const long long total = DIM == 1 ? n : DIM == 2 ? (long long) n*n : (long long) n*n*n;
  double s = 0.;
  for (long long q = (long long) blockIdx.x*blockDim.x + threadIdx.x; q < total;
       q += (long long) gridDim.x*blockDim.x) {
    int i, j, k;
    decode<DIM> (q, n, n, n, i, j, k);
    s += b[cidx<DIM> (g, i, j, k)];
  }
  s = block_sum (s, sm);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

__global__ void k_sum_final (const double * partials, int np, double * out)
{
  __shared__ double sm[32];
  double s = 0.;
  for (int q = threadIdx.x; q < np; q += blockDim.x) s += partials[q];
  s = block_sum (s, sm);
  if (threadIdx.x == 0) *out = s;
}

template <int DIM, typename T>
__global__ void k_pack (bmg_geom g, int ni, int nj, int nk, const double * __restrict__ src,
                        T * __restrict__ dst)
{
  const long long total = (long long) ni*nj*nk;
  for (long long q = (long long) blockIdx.x*blockDim.x + threadIdx.x; q < total;
       q += (long long) gridDim.x*blockDim.x) {
    int i, j, k;
    decode<DIM> (q, ni, nj, nk, i, j, k);
    dst[cidx<DIM> (g, i, j, k)] = (T) src[q];
  }
}

template <int DIM>
__global__ void k_unpack (bmg_geom g, int ni, int nj, int nk, const double * __restrict__ src,
                          double * __restrict__ dst)
{
  const long long total = (long long) ni*nj*nk;
  for (long long q = (long long) blockIdx.x*blockDim.x + threadIdx.x; q < total;
       q += (long long) gridDim.x*blockDim.x) {
    int i, j, k;
    decode<DIM> (q, ni, nj, nk, i, j, k);
    dst[q] = src[cidx<DIM> (g, i, j, k)];
  }
}

template <int DIM>
__global__ void k_convert (bmg_geom g64, bmg_geom g32, int ni, int nj, int nk,
                           const double * __restrict__ src, float * __restrict__ dst)
{
  const long long total = (long long) ni*nj*nk;
  for (long long q = (long long) blockIdx.x*blockDim.x + threadIdx.x; q < total;
       q += (long long) gridDim.x*blockDim.x) {
    int i, j, k;
    decode<DIM> (q, ni, nj, nk, i, j, k);
    dst[cidx<DIM> (g32, i, j, k)] = (float) src[cidx<DIM> (g64, i, j, k)];
  }
}

template <typename T>
__global__ void k_fill (T * f, long long n, T v)
{
  for (long long q = (long long) blockIdx.x*blockDim.x + threadIdx.x; q < n;
       q += (long long) gridDim.x*blockDim.x)
    f[q] = v;
}

template <int DIM>
__global__ void k_shift (bmg_geom g, double * f, const double * sum, double scale)
{
  int i, j, k;
  if (!cell_of_thread<DIM> (g.n, i, j, k)) return;
  f[cidx<DIM> (g, i, j, k)] -= (*sum)*scale;
}

/* face n along a periodic direction = face 0 */
template <int DIM>
__global__ void k_face_wrap (bmg_geom g, int e, double * f)
{
  const int n = g.n;
  const long long total = DIM == 1 ? 1 : DIM == 2 ? n : (long long) n*n;
  const long long q = (long long) blockIdx.x*blockDim.x + threadIdx.x;
  if (q >= total) return;
  int t1 = DIM > 1 ? (int) (DIM == 2 ? q : q/n) : 0, t2 = DIM > 2 ? (int) (q % n) : 0;
  int c0[3], c1[3], m = 0;
  const int tt[2] = {t1, t2};
  for (int d = 0; d < 3; d++) {
    if (d == e) { c0[d] = 0; c1[d] = n; }
    else if (d < DIM) { c0[d] = c1[d] = tt[m++]; }
    else c0[d] = c1[d] = 0;
  }
  f[cidx<DIM> (g, c1[0], c1[1], c1[2])] = f[cidx<DIM> (g, c0[0], c0[1], c0[2])];
}

int lin_blocks (long long total)
{
  long long b = (total + 255)/256;
  if (b > 148*16) b = 148*16;
  if (b < 1) b = 1;
  return (int) b;
}

int status_of_launch ()
{
  cudaError_t e = cudaGetLastError ();
  return e == cudaSuccess ? 0 : (int) e;
}

/* ---------------------------------------------------------------- */
/* dimension dispatch                                                */
/* ---------------------------------------------------------------- */

template <int DIM, typename T>
void relax_dim (int mode, bmg_geom g, void * out, const void * in, const void * rhs,
                const bmg_coef * alpha, bmg_coef lambda, double Delta, BCH h,
                cudaStream_t s)
{
  Coef<T> ax = coef_of<T> (alpha[0]), ay = coef_of<T> (alpha[1]),
    az = coef_of<T> (alpha[2]), lam = coef_of<T> (lambda);
  if (DIM == 3 && mode != BMG_SWEEP_JACOBI && g.n >= 2) {
    const dim3 bb (32, 4, 2), gb ((g.n/2 + 31)/32, (g.n + 3)/4, (g.n + 1)/2);
    bmg_bcdesc none;
    memset (&none, 0, sizeof none);
    if (mode == BMG_SWEEP_RED)
      k_relax3_pair<T, BMG_SWEEP_RED, false><<<gb, bb, 0, s>>> (
        g, (T *) out, (const T *) in, (const T *) rhs, ax, ay, az, lam, (T) Delta, h, NULL, g, none);
    else
      k_relax3_pair<T, BMG_SWEEP_BLACK, false><<<gb, bb, 0, s>>> (
        g, (T *) out, (const T *) in, (const T *) rhs, ax, ay, az, lam, (T) Delta, h, NULL, g, none);
    return;
  }
  dim3 gb = grid_shape<DIM> (g.n), bb = block_shape<DIM> ();
  if (mode == BMG_SWEEP_JACOBI)
    k_relax<DIM, T, BMG_SWEEP_JACOBI><<<gb, bb, 0, s>>> (g, (T *) out, (const T *) in,
                                                          (const T *) rhs, ax, ay, az, lam, (T) Delta, h);
  else if (mode == BMG_SWEEP_RED)
    k_relax<DIM, T, BMG_SWEEP_RED><<<gb, bb, 0, s>>> (g, (T *) out, (const T *) in,
                                                       (const T *) rhs, ax, ay, az, lam, (T) Delta, h);
  else
    k_relax<DIM, T, BMG_SWEEP_BLACK><<<gb, bb, 0, s>>> (g, (T *) out, (const T *) in,
                                                         (const T *) rhs, ax, ay, az, lam, (T) Delta, h);
}

#define DISPATCH_DIM(dim, F, ...)                         \
  do {                                                    \
    if ((dim) == 1) F<1> (__VA_ARGS__);                   \
    else if ((dim) == 2) F<2> (__VA_ARGS__);              \
    else F<3> (__VA_ARGS__);                              \
  } while (0)

template <int DIM>
void relax_st (int st, int mode, bmg_geom g, void * out, const void * in, const void * rhs,
               const bmg_coef * alpha, bmg_coef lambda, double Delta, BCH h, cudaStream_t s)
{
  if (st == BMG_ST_F64) relax_dim<DIM, double> (mode, g, out, in, rhs, alpha, lambda, Delta, h, s);
  else relax_dim<DIM, float> (mode, g, out, in, rhs, alpha, lambda, Delta, h, s);
}

template <int DIM>
void prolong_dim (int stc, int stf, bmg_geom gc, bmg_geom gf, const void * c, void * f,
                  BCH h, int zero, cudaStream_t s)
{
  if (DIM == 2 && !zero && gf.n == 2*gc.n) {
    dim3 gb = grid_shape<2> (gc.n), bb = block_shape<2> ();
    if (stc == BMG_ST_F64 && stf == BMG_ST_F64)
      pdl_launch (k_prolong2d_blk<double, double>, gb, bb, 0, s, gc, gf, (const double *) c, (double *) f, h);
    else if (stc == BMG_ST_F32 && stf == BMG_ST_F32)
      pdl_launch (k_prolong2d_blk<float, float>, gb, bb, 0, s, gc, gf, (const float *) c, (float *) f, h);
    else if (stc == BMG_ST_F64 && stf == BMG_ST_F32)
      pdl_launch (k_prolong2d_blk<double, float>, gb, bb, 0, s, gc, gf, (const double *) c, (float *) f, h);
    else
      pdl_launch (k_prolong2d_blk<float, double>, gb, bb, 0, s, gc, gf, (const float *) c, (double *) f, h);
    return;
  }
  if (DIM == 3 && !zero && gf.n == 2*gc.n) {
    dim3 gb = grid_shape<3> (gc.n), bb = block_shape<3> ();
    if (stc == BMG_ST_F64 && stf == BMG_ST_F64)
      pdl_launch (k_prolong3d_blk<double, double>, gb, bb, 0, s, gc, gf, (const double *) c, (double *) f, h);
    else if (stc == BMG_ST_F32 && stf == BMG_ST_F32)
      pdl_launch (k_prolong3d_blk<float, float>, gb, bb, 0, s, gc, gf, (const float *) c, (float *) f, h);
    else if (stc == BMG_ST_F64 && stf == BMG_ST_F32)
      pdl_launch (k_prolong3d_blk<double, float>, gb, bb, 0, s, gc, gf, (const double *) c, (float *) f, h);
    else
      pdl_launch (k_prolong3d_blk<float, double>, gb, bb, 0, s, gc, gf, (const float *) c, (double *) f, h);
    return;
  }
  dim3 gb = grid_shape<DIM> (gf.n), bb = block_shape<DIM> ();
  if (stc == BMG_ST_F64 && stf == BMG_ST_F64)
    pdl_launch (k_prolong<DIM, double, double>, gb, bb, 0, s, gc, gf, (const double *) c, (double *) f, h, zero);
  else if (stc == BMG_ST_F32 && stf == BMG_ST_F32)
    pdl_launch (k_prolong<DIM, float, float>, gb, bb, 0, s, gc, gf, (const float *) c, (float *) f, h, zero);
  else if (stc == BMG_ST_F64 && stf == BMG_ST_F32)
    pdl_launch (k_prolong<DIM, double, float>, gb, bb, 0, s, gc, gf, (const double *) c, (float *) f, h, zero);
  else
    pdl_launch (k_prolong<DIM, float, double>, gb, bb, 0, s, gc, gf, (const float *) c, (double *) f, h, zero);
}

template <int DIM>
void restrict_dim (int stf, int stc, bmg_geom gf, bmg_geom gc, const void * f, void * c,
                   cudaStream_t s)
{
  dim3 gb = grid_shape<DIM> (gc.n), bb = block_shape<DIM> ();
  if (stf == BMG_ST_F64 && stc == BMG_ST_F64)
    pdl_launch (k_restrict<DIM, double, double>, gb, bb, 0, s, gf, gc, (const double *) f, (double *) c);
  else if (stf == BMG_ST_F32 && stc == BMG_ST_F32)
    pdl_launch (k_restrict<DIM, float, float>, gb, bb, 0, s, gf, gc, (const float *) f, (float *) c);
  else if (stf == BMG_ST_F32 && stc == BMG_ST_F64)
    pdl_launch (k_restrict<DIM, float, double>, gb, bb, 0, s, gf, gc, (const float *) f, (double *) c);
  else
    pdl_launch (k_restrict<DIM, double, float>, gb, bb, 0, s, gf, gc, (const double *) f, (float *) c);
}

template <int DIM>
void restrict_face_dim (bmg_geom gf, bmg_geom gc, FacePtrs p, int level0p, cudaStream_t s)
{
  k_restrict_face<DIM><<<grid_shape<DIM> (gc.n), block_shape<DIM> (), 0, s>>> (gf, gc, p, level0p);
}

template <int DIM>
void residual_dim (int st, bmg_geom g, bmg_geom gr, const double * a, const double * b,
                   const bmg_coef * alpha, bmg_coef lambda, double Delta, void * res,
                   unsigned long long * maxres, cudaStream_t s)
{
  Coef<double> ax = coef_of<double> (alpha[0]), ay = coef_of<double> (alpha[1]),
    az = coef_of<double> (alpha[2]), lam = coef_of<double> (lambda);
  dim3 gb = grid_shape<DIM> (g.n), bb = block_shape<DIM> ();
  int ex;
  const bool pow2 = Delta > 0. && frexp (Delta, &ex) == 0.5 && ex > -1000 && ex < 1000;
  if (st == BMG_ST_F64) {
    if (pow2) pdl_launch (k_residual<DIM, double, true>, gb, bb, 0, s, g, gr, a, b, ax, ay, az, lam, Delta, (double *) res, maxres);
    else pdl_launch (k_residual<DIM, double, false>, gb, bb, 0, s, g, gr, a, b, ax, ay, az, lam, Delta, (double *) res, maxres);
  }
  else {
    if (pow2) pdl_launch (k_residual<DIM, float, true>, gb, bb, 0, s, g, gr, a, b, ax, ay, az, lam, Delta, (float *) res, maxres);
    else pdl_launch (k_residual<DIM, float, false>, gb, bb, 0, s, g, gr, a, b, ax, ay, az, lam, Delta, (float *) res, maxres);
  }
}

template <typename TR, typename TC>
void residual_restrict_2d (bmg_geom g, bmg_geom gr, bmg_geom gc, const double * a,
                           const double * b, const bmg_coef * alpha, bmg_coef lambda,
                           double Delta, void * res, void * resc, unsigned long long * maxres,
                           cudaStream_t s)
{
  Coef<double> ax = coef_of<double> (alpha[0]), ay = coef_of<double> (alpha[1]),
    lam = coef_of<double> (lambda);
  const dim3 bb (32, 8, 1), gb ((gc.n + 31)/32, (gc.n + 7)/8, 1);
  int ex;
  const bool pow2 = Delta > 0. && frexp (Delta, &ex) == 0.5 && ex > -1000 && ex < 1000;
  if (pow2)
    pdl_launch (k_residual_restrict2d<TR, TC, true>, gb, bb, 0, s, g, gr, gc, a, b, ax, ay, lam,
                Delta, (TR *) res, (TC *) resc, maxres);
  else
    pdl_launch (k_residual_restrict2d<TR, TC, false>, gb, bb, 0, s, g, gr, gc, a, b, ax, ay, lam,
                Delta, (TR *) res, (TC *) resc, maxres);
}

template <typename TR, typename TC>
void residual_restrict_3d (bmg_geom g, bmg_geom gr, bmg_geom gc, const double * a,
                           const double * b, const bmg_coef * alpha, bmg_coef lambda,
                           double Delta, void * res, void * resc, unsigned long long * maxres,
                           cudaStream_t s)
{
  Coef<double> ax = coef_of<double> (alpha[0]), ay = coef_of<double> (alpha[1]),
    az = coef_of<double> (alpha[2]), lam = coef_of<double> (lambda);
  const dim3 bb = block_shape<3> (), gb = grid_shape<3> (gc.n);
  int ex;
  const bool pow2 = Delta > 0. && frexp (Delta, &ex) == 0.5 && ex > -1000 && ex < 1000;
  if (pow2)
    pdl_launch (k_residual_restrict3d<TR, TC, true>, gb, bb, 0, s, g, gr, gc, a, b, ax, ay, az,
                lam, Delta, (TR *) res, (TC *) resc, maxres);
  else
    pdl_launch (k_residual_restrict3d<TR, TC, false>, gb, bb, 0, s, g, gr, gc, a, b, ax, ay, az,
                lam, Delta, (TR *) res, (TC *) resc, maxres);
}

template <int DIM>
void correct_dim (int st, bmg_geom g, bmg_geom gd, double * a, const void * da,
                  bmg_bcdesc bc, cudaStream_t s)
{
  dim3 gb = grid_shape<DIM> (g.n), bb = block_shape<DIM> ();
  if (st == BMG_ST_F64)
    pdl_launch (k_correct<DIM, double>, gb, bb, 0, s, g, gd, a, (const double *) da, bc);
  else
    pdl_launch (k_correct<DIM, float>, gb, bb, 0, s, g, gd, a, (const float *) da, bc);
}

template <int DIM>
void apply_bc_dim (int st, bmg_geom g, void * f, bmg_bcdesc bc, BCH h, int homogeneous,
                   cudaStream_t s)
{
  dim3 gb = grid_shape<DIM> (g.n), bb = block_shape<DIM> ();
  if (st == BMG_ST_F64)
    k_apply_bc<DIM, double><<<gb, bb, 0, s>>> (g, (double *) f, bc, h, homogeneous);
  else
    k_apply_bc<DIM, float><<<gb, bb, 0, s>>> (g, (float *) f, bc, h, homogeneous);
}

template <int DIM>
void extents (int n, int face_dim, int & ni, int & nj, int & nk)
{
  ni = n + (face_dim == 0);
  nj = DIM > 1 ? n + (face_dim == 1) : 1;
  nk = DIM > 2 ? n + (face_dim == 2) : 1;
}

template <int DIM>
void pack_dim (int st, bmg_geom g, int face_dim, const double * c, void * p, cudaStream_t s)
{
  int ni, nj, nk;
  extents<DIM> (g.n, face_dim, ni, nj, nk);
  int nb = lin_blocks ((long long) ni*nj*nk);
  if (st == BMG_ST_F64)
    k_pack<DIM, double><<<nb, 256, 0, s>>> (g, ni, nj, nk, c, (double *) p);
  else
    k_pack<DIM, float><<<nb, 256, 0, s>>> (g, ni, nj, nk, c, (float *) p);
}

template <int DIM>
void unpack_dim (bmg_geom g, int face_dim, const double * p, double * c, cudaStream_t s)
{
  int ni, nj, nk;
  extents<DIM> (g.n, face_dim, ni, nj, nk);
  k_unpack<DIM><<<lin_blocks ((long long) ni*nj*nk), 256, 0, s>>> (g, ni, nj, nk, p, c);
}

template <int DIM>
void convert_dim (bmg_geom g64, bmg_geom g32, int face_dim, const double * src, float * dst,
                  cudaStream_t s)
{
  int ni, nj, nk;
  extents<DIM> (g64.n, face_dim, ni, nj, nk);
  k_convert<DIM><<<lin_blocks ((long long) ni*nj*nk), 256, 0, s>>> (g64, g32, ni, nj, nk, src, dst);
}

template <int DIM>
void sum_dim (bmg_geom g, const double * b, double * partials, int np, double * out,
              cudaStream_t s)
{
  k_sum_partial<DIM><<<np, 256, 0, s>>> (g, b, partials);
  k_sum_final<<<1, 1024, 0, s>>> (partials, np, out);
}

template <int DIM>
void shift_dim (bmg_geom g, double * f, const double * sum, double scale, cudaStream_t s)
{
  k_shift<DIM><<<grid_shape<DIM> (g.n), block_shape<DIM> (), 0, s>>> (g, f, sum, scale);
}


/* ---------------------------------------------------------------- */
/* adjoint coefficient gradients (differentiable solve)              */
/* ---------------------------------------------------------------- */

/* For a = L^{-1} b with (L a)_p = lambda_p a_p + sum over faces f of p of
   alpha_f (a_neighbour - a_p)/Delta^2 (the operator whose residual
   poisson.h:373-389 computes), and mu the adjoint (L mu = dl/da, homogeneous
   conditions; L is symmetric):
     dl/dalpha_f = -[mu_p (a_q - a_p) + mu_q (a_p - a_q)]/Delta^2
   over the cells p (lower) and q (upper) of face f that are interior (a
   boundary face has one; ghosts hold the boundary images of a and mu), and
     dl/dlambda_c = -mu_c a_c.
   Face n of a periodic direction is the image of face 0: its gradient is
   carried by face 0 and its own entry is 0. */
template <int DIM>
__global__ void k_adjoint_faces (bmg_geom g, int e, int periodic, const double * __restrict__ mu,
                                 const double * __restrict__ a, double Delta, double * __restrict__ out)
{
  const int n = g.n;
  const int ne = n + 1;
  const long long total = DIM == 1 ? ne : DIM == 2 ? (long long) ne*n : (long long) ne*n*n;
  for (long long q = (long long) blockIdx.x*blockDim.x + threadIdx.x; q < total;
       q += (long long) gridDim.x*blockDim.x) {
    /* compact face index, C order with n+1 entries along e */
    int c[3] = {0, 0, 0};
    {
      long long r = q;
      for (int d = DIM - 1; d >= 0; d--) {
        const int ext = d == e ? ne : n;
        c[d] = (int) (r % ext);
        r /= ext;
      }
    }
    const int f = c[e];
    double v = 0.;
    if (!(periodic && f == n)) {
      int lo[3] = {c[0], c[1], c[2]}, hi[3] = {c[0], c[1], c[2]};
      lo[e] = f - 1; hi[e] = f;
      if (periodic && f == 0) lo[e] = n - 1;
      const bool lin = periodic || f >= 1, hin = periodic || f <= n - 1;
      const long long il = cidx<DIM> (g, lo[0], lo[1], lo[2]), ih = cidx<DIM> (g, hi[0], hi[1], hi[2]);
      const double al = a[il], ah = a[ih];
      if (lin) v -= mu[il]*(ah - al);
      if (hin) v -= mu[ih]*(al - ah);
      v /= Delta*Delta;
    }
    out[q] = v;
  }
}

template <int DIM>
__global__ void k_adjoint_cells (bmg_geom g, const double * __restrict__ mu,
                                 const double * __restrict__ a, double * __restrict__ out)
{
  int i, j, k;
  if (!cell_of_thread<DIM> (g.n, i, j, k)) return;
  const long long id = cidx<DIM> (g, i, j, k);
  long long q = DIM == 1 ? i : DIM == 2 ? (long long) i*g.n + j : ((long long) i*g.n + j)*g.n + k;
  out[q] = -mu[id]*a[id];
}

/* ---------------------------------------------------------------- */
/* implicit viscosity (viscosity.h)                                  */
/* ---------------------------------------------------------------- */

/* components of a cell vector, and of a face coefficient */
struct VecP { double * p[3]; };
struct VecC { Coef<double> c[3]; };

/* the tangential directions of component c in foreach_dimension order
   (x -> y -> z -> x) */
template <int DIM>
__device__ __forceinline__ int vtang (int c, int m) { return DIM == 2 ? 1 - c : (c + 1 + m) % 3; }

/* w.c of relax_viscosity (viscosity.h:36-67), lambda = 1, in the
   reference's evaluation order */
template <int DIM>
__device__ double visc_w (const bmg_geom & g, int c, long long id, const VecP & U, const double * R,
                          const VecC & mu, const Coef<double> & rho, double dt, double Delta)
{
  const long long sn = cstride<DIM> (g, c);
  const double * un = U.p[c];
  const double mn1 = mu.c[c].p ? mu.c[c].p[id + sn] : mu.c[c].c;
  const double mn0 = mu.c[c].p ? mu.c[c].p[id] : mu.c[c].c;
  double A = 2.*mn1*un[id + sn] + 2.*mn0*un[id - sn];
  double den = 2.*mn1 + 2.*mn0;
#pragma unroll
  for (int m = 0; m < DIM - 1; m++) {
    const int t = vtang<DIM> (c, m);
    const long long s = cstride<DIM> (g, t);
    const double * ut = U.p[t];
    const double mt1 = mu.c[t].p ? mu.c[t].p[id + s] : mu.c[t].c;
    const double mt0 = mu.c[t].p ? mu.c[t].p[id] : mu.c[t].c;
    A = A + mt1*(un[id + s] + (ut[id + sn] + ut[id + sn + s])/4. -
                 (ut[id - sn] + ut[id - sn + s])/4.);
    A = A - mt0*(- un[id - s] + (ut[id + sn - s] + ut[id + sn])/4. -
                 (ut[id - sn - s] + ut[id - sn])/4.);
    den = den + mt1;
    den = den + mt0;
  }
  const double r = rho.p ? rho.p[id] : rho.c;
  return (dt/r*A + R[id]*(Delta*Delta))/((Delta*Delta)*1. + dt/r*den);
}

/* mode 0: every cell (Jacobi); 1 / 2: the red / black cells, all
   computed from the values before the pass into W */
template <int DIM>
__global__ void k_visc_relax (bmg_geom g, int mode, VecP U, VecP R, VecP W, VecC mu,
                              Coef<double> rho, double dt, double Delta)
{
  int i, j, k;
  if (!cell_of_thread<DIM> (g.n, i, j, k)) return;
  if (mode && ((i + j + k) & 1) != mode - 1) return;
  const long long id = cidx<DIM> (g, i, j, k);
#pragma unroll
  for (int c = 0; c < DIM; c++)
    W.p[c][id] = visc_w<DIM> (g, c, id, U, R.p[c], mu, rho, dt, Delta);
}

/* u = (u + 2 w)/3 (JACOBI, viscosity.h:71-74), or u = w on one colour */
template <int DIM>
__global__ void k_visc_commit (bmg_geom g, int mode, VecP U, VecP W)
{
  int i, j, k;
  if (!cell_of_thread<DIM> (g.n, i, j, k)) return;
  if (mode && ((i + j + k) & 1) != mode - 1) return;
  const long long id = cidx<DIM> (g, i, j, k);
#pragma unroll
  for (int c = 0; c < DIM; c++)
    U.p[c][id] = mode ? W.p[c][id] : (U.p[c][id] + 2.*W.p[c][id])/3.;
}

/* residual_viscosity, uniform-grid branch (viscosity.h:121-147), lambda =
   1; max |res| over the components into maxres */
template <int DIM>
__global__ void k_visc_residual (bmg_geom g, VecP U, VecP R, VecP RES, VecC mu,
                                 Coef<double> rho, double dt, double Delta,
                                 unsigned long long * maxres)
{
  int i, j, k;
  double m = 0.;
  if (cell_of_thread<DIM> (g.n, i, j, k)) {
    const long long id = cidx<DIM> (g, i, j, k);
    const double rh = rho.p ? rho.p[id] : rho.c;
#pragma unroll
    for (int c = 0; c < DIM; c++) {
      const long long sn = cstride<DIM> (g, c);
      const double * un = U.p[c];
      const double mn1 = mu.c[c].p ? mu.c[c].p[id + sn] : mu.c[c].c;
      const double mn0 = mu.c[c].p ? mu.c[c].p[id] : mu.c[c].c;
      double B = 2.*mn1*(un[id + sn] - un[id]) - 2.*mn0*(un[id] - un[id - sn]);
#pragma unroll
      for (int q = 0; q < DIM - 1; q++) {
        const int t = vtang<DIM> (c, q);
        const long long s = cstride<DIM> (g, t);
        const double * ut = U.p[t];
        const double mt1 = mu.c[t].p ? mu.c[t].p[id + s] : mu.c[t].c;
        const double mt0 = mu.c[t].p ? mu.c[t].p[id] : mu.c[t].c;
        B = B + mt1*(un[id + s] - un[id] + (ut[id + sn] + ut[id + sn + s])/4. -
                     (ut[id - sn] + ut[id - sn + s])/4.);
        B = B - mt0*(un[id] - un[id - s] + (ut[id + sn - s] + ut[id + sn])/4. -
                     (ut[id - sn - s] + ut[id - sn])/4.);
      }
      const double r = R.p[c][id] - 1.*un[id] + dt/rh*B/(Delta*Delta);
      RES.p[c][id] = r;
      const double ar = fabs (r);
      if (m == m && !(ar <= m)) m = ar;       /* a NaN sticks */
    }
  }
  block_max_atomic (m, maxres);
}

/* project (poisson.h:468-509), first step: div = sum over dimensions of
   uf.x[1] - uf.x[], over dt Delta (poisson.h:482-487) */
template <int DIM>
__global__ void k_divergence (bmg_geom g, const double * __restrict__ ux,
                              const double * __restrict__ uy, const double * __restrict__ uz,
                              double dt, double Delta, double * __restrict__ div)
{
  int i, j, k;
  if (!cell_of_thread<DIM> (g.n, i, j, k)) return;
  const long long id = cidx<DIM> (g, i, j, k);
  double d = 0.;
  d += ux[id + cstride<DIM> (g, 0)] - ux[id];
  if (DIM > 1) d += uy[id + cstride<DIM> (g, 1)] - uy[id];
  if (DIM > 2) d += uz[id + cstride<DIM> (g, 2)] - uz[id];
  d /= dt*Delta;
  div[id] = d;
}

/* project, last step: uf.x[] -= dt alpha.x[] face_gradient_x (p, 0) on
   every face of direction e, faces 0..n along e (foreach_face,
   multigrid.h:255-320) */
template <int DIM>
__global__ void k_project_faces (bmg_geom g, int e, double * __restrict__ u, Coef<double> al,
                                 const double * __restrict__ p, double dt, double Delta)
{
  const int n = g.n, ne = n + 1;
  const long long total = DIM == 1 ? ne : DIM == 2 ? (long long) ne*n : (long long) ne*n*n;
  for (long long q = (long long) blockIdx.x*blockDim.x + threadIdx.x; q < total;
       q += (long long) gridDim.x*blockDim.x) {
    int c[3] = {0, 0, 0};
    long long r = q;
    for (int d = DIM - 1; d >= 0; d--) {
      const int ext = d == e ? ne : n;
      c[d] = (int) (r % ext);
      r /= ext;
    }
    const long long id = cidx<DIM> (g, c[0], c[1], c[2]);
    const long long st = cstride<DIM> (g, e);
    const double a = al.p ? al.p[id] : al.c;
    u[id] -= dt*a*((p[id] - p[id - st])/Delta);
  }
}

/* ---------------------------------------------------------------- */
/* ghost slabs of a decomposed domain                                */
/* ---------------------------------------------------------------- */

/* at most this many blocks per launch (the descriptors go by value) */
#define HALO_BATCH 128
struct HaloBatch { bmg_halo h[HALO_BATCH]; };

/* element offset of position t of the slab at index i of direction e: the
   slab spans -1..n of each other direction (ghosts included) */
template <int DIM>
__device__ __forceinline__ long long slab_elem (const bmg_geom & g, int e, int i, int t)
{
  if (DIM == 1) return (long long) g.xo + i;
  const int w = g.n + 2;
  if (DIM == 2)
    return e == 0 ? (long long) (i + 1)*g.P + g.xo + (t - 1) : (long long) t*g.P + g.xo + i;
  const int u = t/w, v = t - u*w;      /* the two other directions, in order */
  if (e == 0) return (long long) (i + 1)*g.plane + (long long) u*g.P + g.xo + (v - 1);
  if (e == 1) return (long long) u*g.plane + (long long) (i + 1)*g.P + g.xo + (v - 1);
  return (long long) u*g.plane + (long long) v*g.P + g.xo + i;
}

/* blockIdx.y: the block; blockIdx.z: the side (0: ghost slab -1 from the
   low neighbour's slab n - 1, 1: ghost slab n from the high neighbour's
   slab 0) */
template <int DIM>
__global__ void k_halo (bmg_geom g, int e, HaloBatch hb)
{
  const bmg_halo & h = hb.h[blockIdx.y];
  const double * src = blockIdx.z ? h.hi : h.lo;
  if (!src) return;
  const long long S = DIM == 1 ? 1 : DIM == 2 ? g.n + 2 : (long long) (g.n + 2)*(g.n + 2);
  const long long t = (long long) blockIdx.x*blockDim.x + threadIdx.x;
  if (t >= S) return;
  const int gi = blockIdx.z ? g.n : -1, si = blockIdx.z ? 0 : g.n - 1;
  h.dst[slab_elem<DIM> (g, e, gi, (int) t)] = src[slab_elem<DIM> (g, e, si, (int) t)];
}

} // namespace


/* ---------------------------------------------------------------- */
/* allocation-free sum                                               */
/* ---------------------------------------------------------------- */

/* Scratch of bmg_sum_noalloc: one partial sum per tile of BMG_NOALLOC_TILE
   values.  A file-scope device array, so every GPU that loads the library
   holds these 32 KB until the process exits, and every call shares them. */
#define BMG_NOALLOC_THREADS 256
#define BMG_NOALLOC_TILE (BMG_NOALLOC_THREADS*16)
#define BMG_NOALLOC_PARTIALS 4096
static __device__ __align__(256) double bmg_noalloc_scratch[BMG_NOALLOC_PARTIALS];

namespace {

/* stage 1: block b sums values [b*TILE, (b+1)*TILE) in a fixed order */
__global__ void k_sum_noalloc_partial (const double * __restrict__ v, long long count,
                                       double * partials)
{
  __shared__ double sm[32];
  const long long base = (long long) blockIdx.x*BMG_NOALLOC_TILE;
  double s = 0.;
  for (int r = 0; r < BMG_NOALLOC_TILE/BMG_NOALLOC_THREADS; r++) {
    const long long q = base + (long long) r*BMG_NOALLOC_THREADS + threadIdx.x;
    if (q < count) s += v[q];
  }
  s = block_sum (s, sm);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

/* stage 2: one block sums the partials written by this call's stage 1 */
__global__ void k_sum_noalloc_final (const double * partials, int np, double * out)
{
  __shared__ double sm[32];
  double s = 0.;
  for (int q = threadIdx.x; q < np; q += blockDim.x) s += partials[q];
  s = block_sum (s, sm);
  if (threadIdx.x == 0) *out = s;
}

} // namespace

#define BMG_NOALLOC_MAXDEV 64
static double * noalloc_scratch_ptr[BMG_NOALLOC_MAXDEV];

extern "C" int bmg_sum_noalloc (const double * values, size_t count, double * result,
                                void * stream)
{
  const size_t maxcount = (size_t) BMG_NOALLOC_PARTIALS*BMG_NOALLOC_TILE;
  if (!result || (count > 0 && !values))
    return 1; /* BMG_EINVAL */
  if (count > maxcount) {
    fprintf (stderr, "bmg_sum_noalloc: %zu values exceed the maximum of %zu "
             "(%d partial sums of %d values in the static scratch)\n",
             count, maxcount, BMG_NOALLOC_PARTIALS, BMG_NOALLOC_TILE);
    return 1; /* BMG_EINVAL */
  }
  int dev = 0;
  if (cudaGetDevice (&dev) != cudaSuccess || dev < 0 || dev >= BMG_NOALLOC_MAXDEV) {
    cudaGetLastError ();
    return 7; /* BMG_ENODEV */
  }
  cudaStream_t s = (cudaStream_t) stream;
  /* the device address of the scratch array (its name in host code is only
     a stand-in), looked up with the device current.  Outside a stream
     capture it is looked up on every call, so that a context that was torn
     down and created again (cudaDeviceReset) gets the module's new address;
     inside a capture the address cached by the last call outside one is
     used (the first call on a device must come before any capture). */
  enum cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing (s, &cs) != cudaSuccess) {
    cudaGetLastError ();
    return 2; /* BMG_ECUDA */
  }
  if (cs == cudaStreamCaptureStatusNone || !noalloc_scratch_ptr[dev]) {
    if (cs != cudaStreamCaptureStatusNone) {
      fprintf (stderr, "bmg_sum_noalloc: the first call on device %d is inside a stream "
               "capture; call it once before capturing\n", dev);
      return 1; /* BMG_EINVAL */
    }
    void * p = NULL;
    cudaError_t e = cudaGetSymbolAddress (&p, bmg_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      fprintf (stderr, "bmg_sum_noalloc: cudaGetSymbolAddress failed: %s\n",
               cudaGetErrorString (e));
      return 2; /* BMG_ECUDA */
    }
    noalloc_scratch_ptr[dev] = (double *) p;
  }
  const int np = (int) ((count + BMG_NOALLOC_TILE - 1)/BMG_NOALLOC_TILE);
  /* nothing accumulates across calls: stage 1 overwrites the np partials
     that stage 2 reads, and stage 2 overwrites *result (count 0: one empty
     partial, a sum of 0) */
  const int nb = np > 0 ? np : 1;
  k_sum_noalloc_partial<<<nb, BMG_NOALLOC_THREADS, 0, s>>> (values, (long long) count,
                                                             noalloc_scratch_ptr[dev]);
  k_sum_noalloc_final<<<1, 1024, 0, s>>> (noalloc_scratch_ptr[dev], nb, result);
  return cudaGetLastError () == cudaSuccess ? 0 : 2;
}

/* ---------------------------------------------------------------- */
/* C launchers                                                       */
/* ---------------------------------------------------------------- */

extern "C" {

int bmg_launch_relax (int dim, int st, int mode, bmg_geom g, void * out, const void * in,
                      const void * rhs, const bmg_coef * alpha, bmg_coef lambda,
                      double Delta, const bmg_bcdesc * bc, cudaStream_t s)
{
  BCH h = bch_of (bc);
  DISPATCH_DIM (dim, relax_st, st, mode, g, out, in, rhs, alpha, lambda, Delta, h, s);
  return status_of_launch ();
}

int bmg_launch_prolong (int dim, int st_coarse, int st_fine, bmg_geom gc, bmg_geom gf,
                        const void * coarse, void * fine, const bmg_bcdesc * bc, int zero,
                        cudaStream_t s)
{
  BCH h = bch_of (bc);
  DISPATCH_DIM (dim, prolong_dim, st_coarse, st_fine, gc, gf, coarse, fine, h, zero, s);
  return status_of_launch ();
}

int bmg_launch_restrict (int dim, int st_fine, int st_coarse, bmg_geom gf, bmg_geom gc,
                         const void * fine, void * coarse, cudaStream_t s)
{
  DISPATCH_DIM (dim, restrict_dim, st_fine, st_coarse, gf, gc, fine, coarse, s);
  return status_of_launch ();
}

int bmg_launch_restrict_face (int dim, bmg_geom gf, bmg_geom gc, const double * const * fine,
                              double * const * coarse, int level0p, cudaStream_t s)
{
  FacePtrs p;
  for (int e = 0; e < 3; e++) {
    p.f[e] = e < dim ? fine[e] : 0;
    p.c[e] = e < dim ? coarse[e] : 0;
  }
  DISPATCH_DIM (dim, restrict_face_dim, gf, gc, p, level0p, s);
  return status_of_launch ();
}

int bmg_launch_residual (int dim, int st_res, bmg_geom g, bmg_geom gres, const double * a,
                         const double * b, const bmg_coef * alpha, bmg_coef lambda,
                         double Delta, void * res, unsigned long long * maxres,
                         cudaStream_t s)
{
  DISPATCH_DIM (dim, residual_dim, st_res, g, gres, a, b, alpha, lambda, Delta, res, maxres, s);
  return status_of_launch ();
}

int bmg_launch_residual_restrict (int st_res, int st_coarse, bmg_geom g, bmg_geom gres,
                                  bmg_geom gcoarse, const double * a, const double * b,
                                  const bmg_coef * alpha, bmg_coef lambda, double Delta,
                                  void * res, void * coarse, unsigned long long * maxres,
                                  cudaStream_t s)
{
  if (g.n < 2 || gcoarse.n*2 != g.n) return (int) cudaErrorInvalidValue;
  if (st_res == BMG_ST_F64 && st_coarse == BMG_ST_F64)
    residual_restrict_2d<double, double> (g, gres, gcoarse, a, b, alpha, lambda, Delta, res, coarse, maxres, s);
  else if (st_res == BMG_ST_F32 && st_coarse == BMG_ST_F32)
    residual_restrict_2d<float, float> (g, gres, gcoarse, a, b, alpha, lambda, Delta, res, coarse, maxres, s);
  else if (st_res == BMG_ST_F32 && st_coarse == BMG_ST_F64)
    residual_restrict_2d<float, double> (g, gres, gcoarse, a, b, alpha, lambda, Delta, res, coarse, maxres, s);
  else
    residual_restrict_2d<double, float> (g, gres, gcoarse, a, b, alpha, lambda, Delta, res, coarse, maxres, s);
  cudaError_t r = cudaGetLastError ();
  return r == cudaSuccess ? 0 : (int) r;
}

int bmg_launch_residual_restrict3d (int st_res, int st_coarse, bmg_geom g, bmg_geom gres,
                                    bmg_geom gcoarse, const double * a, const double * b,
                                    const bmg_coef * alpha, bmg_coef lambda, double Delta,
                                    void * res, void * coarse, unsigned long long * maxres,
                                    cudaStream_t s)
{
  if (g.n < 2 || gcoarse.n*2 != g.n) return (int) cudaErrorInvalidValue;
  if (st_res == BMG_ST_F64 && st_coarse == BMG_ST_F64)
    residual_restrict_3d<double, double> (g, gres, gcoarse, a, b, alpha, lambda, Delta, res, coarse, maxres, s);
  else if (st_res == BMG_ST_F32 && st_coarse == BMG_ST_F32)
    residual_restrict_3d<float, float> (g, gres, gcoarse, a, b, alpha, lambda, Delta, res, coarse, maxres, s);
  else if (st_res == BMG_ST_F32 && st_coarse == BMG_ST_F64)
    residual_restrict_3d<float, double> (g, gres, gcoarse, a, b, alpha, lambda, Delta, res, coarse, maxres, s);
  else
    residual_restrict_3d<double, float> (g, gres, gcoarse, a, b, alpha, lambda, Delta, res, coarse, maxres, s);
  cudaError_t r = cudaGetLastError ();
  return r == cudaSuccess ? 0 : (int) r;
}

int bmg_launch_relax_correct3d (int st, bmg_geom g, void * out, const void * in, const void * rhs,
                                const bmg_coef * alpha, bmg_coef lambda, double Delta,
                                const bmg_bcdesc * bc, double * acor, bmg_geom ga,
                                const bmg_bcdesc * abc, cudaStream_t s)
{
  if (g.n < 2 || g.n != ga.n || !acor || !abc) return (int) cudaErrorInvalidValue;
  BCH h = bch_of (bc);
  const dim3 bb (32, 4, 2), gb ((g.n/2 + 31)/32, (g.n + 3)/4, (g.n + 1)/2);
  if (st == BMG_ST_F64)
    k_relax3_pair<double, BMG_SWEEP_BLACK, true><<<gb, bb, 0, s>>> (
      g, (double *) out, (const double *) in, (const double *) rhs, coef_of<double> (alpha[0]),
      coef_of<double> (alpha[1]), coef_of<double> (alpha[2]), coef_of<double> (lambda),
      Delta, h, acor, ga, *abc);
  else
    k_relax3_pair<float, BMG_SWEEP_BLACK, true><<<gb, bb, 0, s>>> (
      g, (float *) out, (const float *) in, (const float *) rhs, coef_of<float> (alpha[0]),
      coef_of<float> (alpha[1]), coef_of<float> (alpha[2]), coef_of<float> (lambda),
      (float) Delta, h, acor, ga, *abc);
  return status_of_launch ();
}

int bmg_launch_correct (int dim, int st_da, bmg_geom g, bmg_geom gda, double * a,
                        const void * da, const bmg_bcdesc * bc, cudaStream_t s)
{
  DISPATCH_DIM (dim, correct_dim, st_da, g, gda, a, da, *bc, s);
  return status_of_launch ();
}

int bmg_launch_apply_bc (int dim, int st, bmg_geom g, void * f, const bmg_bcdesc * bc,
                         int homogeneous, cudaStream_t s)
{
  BCH h = bch_of (bc);
  DISPATCH_DIM (dim, apply_bc_dim, st, g, f, *bc, h, homogeneous, s);
  return status_of_launch ();
}

int bmg_sum_partials (int dim, bmg_geom g)
{
  long long total = dim == 1 ? g.n : dim == 2 ? (long long) g.n*g.n : (long long) g.n*g.n*g.n;
  long long nb = (total + 255)/256;
  if (nb > 1024) nb = 1024;
  if (nb < 1) nb = 1;
  return (int) nb;
}

int bmg_launch_sum (int dim, bmg_geom g, const double * b, double * partials, int npartials,
                    double * out, cudaStream_t s)
{
  DISPATCH_DIM (dim, sum_dim, g, b, partials, npartials, out, s);
  return status_of_launch ();
}

int bmg_launch_pack (int dim, int st, bmg_geom g, int face_dim, const double * compact,
                     void * padded, cudaStream_t s)
{
  DISPATCH_DIM (dim, pack_dim, st, g, face_dim, compact, padded, s);
  return status_of_launch ();
}

int bmg_launch_unpack (int dim, bmg_geom g, int face_dim, const double * padded,
                       double * compact, cudaStream_t s)
{
  DISPATCH_DIM (dim, unpack_dim, g, face_dim, padded, compact, s);
  return status_of_launch ();
}

int bmg_launch_convert (int dim, bmg_geom g64, bmg_geom g32, int face_dim, const double * src,
                        float * dst, cudaStream_t s)
{
  DISPATCH_DIM (dim, convert_dim, g64, g32, face_dim, src, dst, s);
  return status_of_launch ();
}

int bmg_launch_fill (int dim, int st, bmg_geom g, void * f, double v, cudaStream_t s)
{
  (void) dim;
  int nb = lin_blocks (g.size);
  if (st == BMG_ST_F64) k_fill<double><<<nb, 256, 0, s>>> ((double *) f, g.size, v);
  else k_fill<float><<<nb, 256, 0, s>>> ((float *) f, g.size, (float) v);
  return status_of_launch ();
}

int bmg_launch_halo (int dim, bmg_geom g, int e, const bmg_halo * blocks, int nb, cudaStream_t s)
{
  const long long S = dim == 1 ? 1 : dim == 2 ? g.n + 2 : (long long) (g.n + 2)*(g.n + 2);
  const int gx = (int) ((S + 255)/256);
  for (int b0 = 0; b0 < nb; b0 += HALO_BATCH) {
    HaloBatch hb;
    const int m = nb - b0 < HALO_BATCH ? nb - b0 : HALO_BATCH;
    for (int k = 0; k < m; k++) hb.h[k] = blocks[b0 + k];
    dim3 grid (gx, m, 2);
    if (dim == 1) k_halo<1><<<grid, 256, 0, s>>> (g, e, hb);
    else if (dim == 2) k_halo<2><<<grid, 256, 0, s>>> (g, e, hb);
    else k_halo<3><<<grid, 256, 0, s>>> (g, e, hb);
    const int st = status_of_launch ();
    if (st) return st;
  }
  return 0;
}

int bmg_launch_face_wrap (int dim, bmg_geom g, int face_dim, double * f, cudaStream_t s)
{
  long long total = dim == 1 ? 1 : dim == 2 ? g.n : (long long) g.n*g.n;
  int nb = (int) ((total + 255)/256);
  if (dim == 1) k_face_wrap<1><<<nb, 256, 0, s>>> (g, face_dim, f);
  else if (dim == 2) k_face_wrap<2><<<nb, 256, 0, s>>> (g, face_dim, f);
  else k_face_wrap<3><<<nb, 256, 0, s>>> (g, face_dim, f);
  return status_of_launch ();
}

int bmg_launch_adjoint_faces (int dim, bmg_geom g, int e, int periodic, const double * mu,
                              const double * a, double Delta, double * out, cudaStream_t s)
{
  long long total = (long long) (g.n + 1);
  for (int d = 1; d < dim; d++) total *= g.n;
  const int nb = lin_blocks (total);
  if (dim == 1) k_adjoint_faces<1><<<nb, 256, 0, s>>> (g, e, periodic, mu, a, Delta, out);
  else if (dim == 2) k_adjoint_faces<2><<<nb, 256, 0, s>>> (g, e, periodic, mu, a, Delta, out);
  else k_adjoint_faces<3><<<nb, 256, 0, s>>> (g, e, periodic, mu, a, Delta, out);
  return status_of_launch ();
}

int bmg_launch_adjoint_cells (int dim, bmg_geom g, const double * mu, const double * a,
                              double * out, cudaStream_t s)
{
  if (dim == 1) k_adjoint_cells<1><<<grid_shape<1> (g.n), block_shape<1> (), 0, s>>> (g, mu, a, out);
  else if (dim == 2) k_adjoint_cells<2><<<grid_shape<2> (g.n), block_shape<2> (), 0, s>>> (g, mu, a, out);
  else k_adjoint_cells<3><<<grid_shape<3> (g.n), block_shape<3> (), 0, s>>> (g, mu, a, out);
  return status_of_launch ();
}

int bmg_launch_visc_relax (int dim, bmg_geom g, int mode, double * const * u,
                           double * const * r, double * const * w, const bmg_coef * mu,
                           bmg_coef rho, double dt, double Delta, cudaStream_t s)
{
  VecP U, R, W;
  VecC M;
  for (int c = 0; c < 3; c++) {
    U.p[c] = c < dim ? u[c] : NULL; R.p[c] = c < dim ? r[c] : NULL;
    W.p[c] = c < dim ? w[c] : NULL;
    M.c[c] = coef_of<double> (mu[c]);
  }
  const Coef<double> rh = coef_of<double> (rho);
  if (dim == 2) k_visc_relax<2><<<grid_shape<2> (g.n), block_shape<2> (), 0, s>>> (g, mode, U, R, W, M, rh, dt, Delta);
  else if (dim == 3) k_visc_relax<3><<<grid_shape<3> (g.n), block_shape<3> (), 0, s>>> (g, mode, U, R, W, M, rh, dt, Delta);
  else return (int) cudaErrorInvalidValue;
  return status_of_launch ();
}

int bmg_launch_visc_commit (int dim, bmg_geom g, int mode, double * const * u,
                            double * const * w, cudaStream_t s)
{
  VecP U, W;
  for (int c = 0; c < 3; c++) { U.p[c] = c < dim ? u[c] : NULL; W.p[c] = c < dim ? w[c] : NULL; }
  if (dim == 2) k_visc_commit<2><<<grid_shape<2> (g.n), block_shape<2> (), 0, s>>> (g, mode, U, W);
  else if (dim == 3) k_visc_commit<3><<<grid_shape<3> (g.n), block_shape<3> (), 0, s>>> (g, mode, U, W);
  else return (int) cudaErrorInvalidValue;
  return status_of_launch ();
}

int bmg_launch_visc_residual (int dim, bmg_geom g, double * const * u, double * const * r,
                              double * const * res, const bmg_coef * mu, bmg_coef rho,
                              double dt, double Delta, unsigned long long * maxres,
                              cudaStream_t s)
{
  VecP U, R, RES;
  VecC M;
  for (int c = 0; c < 3; c++) {
    U.p[c] = c < dim ? u[c] : NULL; R.p[c] = c < dim ? r[c] : NULL;
    RES.p[c] = c < dim ? res[c] : NULL;
    M.c[c] = coef_of<double> (mu[c]);
  }
  const Coef<double> rh = coef_of<double> (rho);
  if (dim == 2) k_visc_residual<2><<<grid_shape<2> (g.n), block_shape<2> (), 0, s>>> (g, U, R, RES, M, rh, dt, Delta, maxres);
  else if (dim == 3) k_visc_residual<3><<<grid_shape<3> (g.n), block_shape<3> (), 0, s>>> (g, U, R, RES, M, rh, dt, Delta, maxres);
  else return (int) cudaErrorInvalidValue;
  return status_of_launch ();
}

int bmg_launch_divergence (int dim, bmg_geom g, const double * const * uf, double dt,
                           double Delta, double * div, cudaStream_t s)
{
  const double * ux = uf[0], * uy = dim > 1 ? uf[1] : NULL, * uz = dim > 2 ? uf[2] : NULL;
  if (dim == 1) k_divergence<1><<<grid_shape<1> (g.n), block_shape<1> (), 0, s>>> (g, ux, uy, uz, dt, Delta, div);
  else if (dim == 2) k_divergence<2><<<grid_shape<2> (g.n), block_shape<2> (), 0, s>>> (g, ux, uy, uz, dt, Delta, div);
  else k_divergence<3><<<grid_shape<3> (g.n), block_shape<3> (), 0, s>>> (g, ux, uy, uz, dt, Delta, div);
  return status_of_launch ();
}

int bmg_launch_project_faces (int dim, bmg_geom g, int e, double * u, bmg_coef alpha,
                              const double * p, double dt, double Delta, cudaStream_t s)
{
  long long total = (long long) (g.n + 1);
  for (int d = 1; d < dim; d++) total *= g.n;
  const int nb = lin_blocks (total);
  const Coef<double> al = coef_of<double> (alpha);
  if (dim == 1) k_project_faces<1><<<nb, 256, 0, s>>> (g, e, u, al, p, dt, Delta);
  else if (dim == 2) k_project_faces<2><<<nb, 256, 0, s>>> (g, e, u, al, p, dt, Delta);
  else k_project_faces<3><<<nb, 256, 0, s>>> (g, e, u, al, p, dt, Delta);
  return status_of_launch ();
}

int bmg_launch_shift (int dim, bmg_geom g, double * f, const double * sum, double scale,
                      cudaStream_t s)
{
  DISPATCH_DIM (dim, shift_dim, g, f, sum, scale, s);
  return status_of_launch ();
}

} // extern "C"

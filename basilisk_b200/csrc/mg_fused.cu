/*
 * mg_fused.cu -- fused relaxation kernels of the multigrid solver.
 *
 * The reference's V-cycle (poisson.h:32-90) relaxes every level nrelax times,
 * and mg_solve raises nrelax while a cycle reduces the residual by less than
 * 1.2 (poisson.h:198-204): on stiff problems nrelax reaches 30-50, so the
 * solve is a long chain of small relaxation sweeps.  These kernels replace
 * the one-launch-per-colour sweeps of mg_kernels.cu on the red-black path:
 *
 *   k_relax_tile2d    S complete red-black sweeps of a 2D level in one
 *                     launch.  Each CTA stages a TS x TS tile plus a
 *                     2S-cell halo of da, res, alpha_x, alpha_y (and lambda)
 *                     in shared memory, updates red then black cells on a
 *                     region that shrinks by one cell per colour pass, and
 *                     writes the TS x TS interior back to the partner buffer
 *                     (CTAs read halos that other CTAs own, so a launch never
 *                     writes what it reads).  The halo is recomputed
 *                     redundantly, so each array is read about once per S
 *                     sweeps instead of twice per sweep.  FP64 levels (in the
 *                     reference's evaluation order) and the small FP32
 *                     levels.
 *   k_relax_tile2d_w  the same temporal blocking for the large FP32 levels of
 *                     the mixed form, with each thread's cells' coefficients
 *                     divided by the diagonal once per launch and kept in
 *                     registers: only the iterate is staged.
 *   k_bottom          the coarse end of the cycle in one single-CTA launch:
 *                     restriction of res down to minlevel, the coarsest zero,
 *                     then for each level up to a small one the bilinear
 *                     prolongation and all nrelax sweeps, with barriers
 *                     between colour passes.  Those levels are pure latency
 *                     when each pass is a launch.
 *
 * The FP64 paths compute every cell update with relax_value's expression and
 * order and write the same ghost images as the unfused kernels, so their
 * results are bit-identical to the red / boundary / black sequence of the
 * oracle; the FP32 paths of the mixed form relax the same operator up to
 * FP32 rounding.
 */
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "mg_device.cuh"

using namespace bmgd;

namespace {

/* ---------------------------------------------------------------- */
/* tile-fused red-black sweeps, 2D                                    */
/* ---------------------------------------------------------------- */

/* a global index along one axis: its periodic image, or -1 when it is a
   box ghost or outside the domain (never updated) */
__device__ __forceinline__ int real_index (int gi, int n, int periodic)
{
  if (gi >= 0 && gi < n) return gi;
  if (!periodic) return -1;
  int r = gi % n;
  return r < 0 ? r + n : r;
}

/* a face index along its own axis (faces 0..n; face n of a periodic
   direction is face 0) */
__device__ __forceinline__ int real_face (int f, int n, int periodic)
{
  if (f >= 0 && f <= n) return (periodic && f == n) ? 0 : f;
  if (!periodic) return -1;
  int r = f % n;
  return r < 0 ? r + n : r;
}

/* Shared-memory tile of TS x TS cells plus a 2S halo, stored split by
   colour: colour c = (i + j) & 1 of cell (i, j) (global indices); cell
   (p, q) of the staged region lives in the colour-c arrays at [p][q >> 1].
   A colour pass then reads its neighbours (all of the other colour) with
   unit stride: up/down at [p -+ 1][m], left/right at [p][m - 1 + o] and
   [p][m + o], o the column offset of colour c in row p. */
/* asynchronous global -> shared copy of one element (cp.async, sm_80+), with
   zero fill when the source is not a real cell: all staging loads of a
   thread are in flight at once instead of one dependent load per step */
template <typename T>
__device__ __forceinline__ void cp_async_elem (T * smem, const T * gmem, bool valid)
{
  const unsigned s = (unsigned) __cvta_generic_to_shared (smem);
  const int sz = valid ? (int) sizeof (T) : 0;
  if (sizeof (T) == 8)
    asm volatile ("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" :: "r"(s), "l"(gmem), "r"(sz) : "memory");
  else
    asm volatile ("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" :: "r"(s), "l"(gmem), "r"(sz) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all ()
{
  asm volatile ("cp.async.commit_group;\n" ::: "memory");
  asm volatile ("cp.async.wait_group 0;\n" ::: "memory");
}

/* programmatic dependent launch (sm_90+): with the launch attribute set,
   a dependent grid may start before this one ends; wait () blocks until
   the preceding grid has completed and its writes are visible, and is a
   no-op in a grid launched without the attribute */
__device__ __forceinline__ void grid_dependency_wait ()
{
  asm volatile ("griddepcontrol.wait;" ::: "memory");
}

__device__ __forceinline__ void grid_dependents_launch ()
{
  asm volatile ("griddepcontrol.launch_dependents;" ::: "memory");
}

template <typename T, int TS, int S>
struct TileShape {
  static constexpr int H = 2*S;        /* halo: one cell per colour pass */
  static constexpr int W = TS + 2*H;   /* staged cells per side (even) */
  static constexpr int M = W/2;        /* cells of one colour per row */
  static_assert (W % 2 == 0, "staged width must be even");
  static constexpr int MY = M + 4;     /* y-face row pitch (16-byte aligned rows) */
  /* da, res, (lambda): 2 colours x W x M; alpha_x faces: 2 x (W+1) x M;
     alpha_y faces: 2 x W x MY */
  static constexpr size_t elems (bool lam)
  {
    return (size_t) 2*W*M*(lam ? 3 : 2) + (size_t) 2*(W + 1)*M + (size_t) 2*W*MY;
  }
  static constexpr size_t bytes (bool lam) { return sizeof (T)*elems (lam); }
};

/* the cell update's division: IEEE for FP64 (the plain form is
   bit-compared with the oracle), the fast reciprocal-multiply for the FP32
   smoothing of the mixed form, whose rounding the FP64 outer residual
   corrects anyway */
__device__ __forceinline__ double relax_div (double n, double d) { return n/d; }
__device__ __forceinline__ float relax_div (float n, float d) { return __fdividef (n, d); }

/* n += x1 v1 + x0 v0: the reference's order in FP64, fused multiply-adds
   in FP32 */
__device__ __forceinline__ double tile_acc (double n, double x1, double v1, double x0, double v0)
{
  return n + (x1*v1 + x0*v0);
}
__device__ __forceinline__ float tile_acc (float n, float x1, float v1, float x0, float v0)
{
  return fmaf (x0, v0, fmaf (x1, v1, n));
}

template <typename T> struct Pair;
template <> struct Pair<float> { typedef float2 type; };
template <> struct Pair<double> { typedef double2 type; };

/* four consecutive elements of a row (16-byte aligned in global memory) */
template <typename T> struct Quad { T x, y, z, w; };

__device__ __forceinline__ Quad<float> load_quad (const float * p)
{
  const float4 v = *(const float4 *) p;
  Quad<float> q = {v.x, v.y, v.z, v.w};
  return q;
}

__device__ __forceinline__ Quad<double> load_quad (const double * p)
{
  const double2 a = *(const double2 *) p, b = *(const double2 *) (p + 2);
  Quad<double> q = {a.x, a.y, b.x, b.y};
  return q;
}

__device__ __forceinline__ void store_quad (float * p, const Quad<float> & q)
{
  *(float4 *) p = make_float4 (q.x, q.y, q.z, q.w);
}

__device__ __forceinline__ void store_quad (double * p, const Quad<double> & q)
{
  *(double2 *) p = make_double2 (q.x, q.y);
  *(double2 *) (p + 2) = make_double2 (q.z, q.w);
}

/* a quad starting at an even column q (m = q/2, even): elements q and q + 2
   belong to colour c0, q + 1 and q + 3 to the other colour, each pair at
   [m, m + 1] of its colour array */
template <typename T>
__device__ __forceinline__ void put_quad (T * a0, T * a1, int off, const Quad<T> & v)
{
  typedef typename Pair<T>::type T2;
  T2 e, o;
  e.x = v.x; e.y = v.z; o.x = v.y; o.y = v.w;
  *(T2 *) (a0 + off) = e;
  *(T2 *) (a1 + off) = o;
}

/* The bilinear prolongation (multigrid-common.h:124-140) of fine cell
   (i, j) from the coarse level c (geometry gc, ghosts filled), with
   k_prolong2d_blk's expression and order, so that a tile launch that
   stages it instead of the iterate gives the values the prolongation
   launch would have written (bit-identical in FP64). */
template <typename T>
__device__ __forceinline__ T prolong_cell (const T * __restrict__ c, const bmg_geom & gc, int i, int j)
{
  const int ci = i >> 1, cj = j >> 1, cx = (i & 1) ? 1 : -1, cy = (j & 1) ? 1 : -1;
  const T m = c[cidx<2> (gc, ci, cj, 0)], mx = c[cidx<2> (gc, ci + cx, cj, 0)];
  const T my = c[cidx<2> (gc, ci, cj + cy, 0)], mxy = c[cidx<2> (gc, ci + cx, cj + cy, 0)];
  return (T(9)*m + T(3)*(mx + my) + mxy)/T(16);
}

/* the same for the K fine cells (i, j0) .. (i, j0 + K - 1) of one row, j0
   even: the K/2 + 2 coarse values of the two coarse rows involved read
   once */
template <typename T, int K>
__device__ __forceinline__ void prolong_row (const T * __restrict__ c, const bmg_geom & gc, int i, int j0,
                                             T * v)
{
  const int ci = i >> 1, cx = (i & 1) ? 1 : -1, cb = (j0 >> 1) - 1;
  const T * c0 = c + cidx<2> (gc, ci, cb, 0), * c1 = c + cidx<2> (gc, ci + cx, cb, 0);
  T r0[K/2 + 2], r1[K/2 + 2];
#pragma unroll
  for (int u = 0; u < K/2 + 2; u++) { r0[u] = c0[u]; r1[u] = c1[u]; }
#pragma unroll
  for (int q = 0; q < K; q++) {
    const int u = 1 + (q >> 1), cy = (q & 1) ? 1 : -1;
    v[q] = (T(9)*r0[u] + T(3)*(r1[u] + r0[u + cy]) + r1[u + cy])/T(16);
  }
}

/* BX x BY threads: thread (tx, ty) updates the CPT = 2 cells 2 tx, 2 tx + 1
   of each colour of row ty + lo in every colour pass; MINB CTAs per SM bound
   the registers */
template <typename T, int TS, int S, bool LAM, int BX, int BY, int CPT, int MINB>
__global__ void __launch_bounds__ (BX*BY, MINB)
k_relax_tile2d (bmg_geom g, T * __restrict__ out, const T * __restrict__ in,
                const T * __restrict__ res, Coef<T> ax, Coef<T> ay, Coef<T> lam, T Delta, BCH bc,
                int nsweeps)
{
  typedef TileShape<T, TS, S> Sh;
  constexpr int H = Sh::H, W = Sh::W, M = Sh::M, MY = Sh::MY;
  static_assert (M % CPT == 0 && M <= CPT*BX && W - 2 <= BY, "CPT cells per thread per row");
  static_assert (CPT == 2, "pairs of cells per thread and colour");
  typedef typename Pair<T>::type T2;
  extern __shared__ __align__ (16) unsigned char smem_raw[];
  /* the colour-c arrays, as offsets from one shared base (no pointer
     tables: those would live in local memory) */
  T * const smb = (T *) smem_raw;
  constexpr int WM = W*M, WX = (W + 1)*M, WY = W*MY;
  constexpr int OR = 2*WM, OX = 4*WM, OY = OX + 2*WX, OL = OY + 2*WY;
  auto sa = [smb] (int c) { return smb + c*WM; };
  auto sr = [smb] (int c) { return smb + OR + c*WM; };
  auto sx = [smb] (int c) { return smb + OX + c*WX; };
  auto sy = [smb] (int c) { return smb + OY + c*WY; };
  auto sl = [smb] (int c) { return smb + OL + c*WM; };
  const int n = g.n, tx = threadIdx.x, ty = threadIdx.y;
  const int tid = ty*BX + tx, nth = BX*BY;
  constexpr int RW = 32/BX;     /* rows per warp */
  static_assert (32 % BX == 0 && BY % (2*RW) == 0, "warps cover whole row pairs");
  const int pr = 2*RW*(ty/(2*RW)) + 2*(ty % RW) + ((ty/RW) & 1);
  const int i0 = blockIdx.y*TS - H, j0 = blockIdx.x*TS - H;   /* global index of (0,0) */
  const int px = bc.periodic[0], py = bc.periodic[1];
  const int base = (i0 + j0) & 1;                             /* colour of (0,0) */
  /* the whole staged region inside the domain: no cell checks needed */
  const bool inner = i0 >= 0 && i0 + W <= n && j0 >= 0 && j0 + W <= n;
  /* the next launch may start staging its coefficients now: it waits for
     this grid before it reads the iterate this grid writes */
  grid_dependents_launch ();

  if (inner) {
    /* the staged region lies inside the domain: 16-byte loads of four
       cells, split into the colour arrays with pair stores (all loads of
       one thread are issued before its stores) */
    constexpr int QW = W/4;
    static_assert (W % 4 == 0 && TS % 4 == 0 && H % 4 == 0, "quads of cells");
    for (int idx = tid; idx < W*QW; idx += nth) {
      const int p = idx/QW, k = idx - p*QW, q = 4*k;
      const int c0 = (base + p + q) & 1;
      const long long id = cidx<2> (g, i0 + p, j0 + q, 0);
      const Quad<T> vr = load_quad (res + id);
      Quad<T> vl, vx, vy;
      if (LAM) vl = load_quad (lam.p + id);
      if (ax.p) vx = load_quad (ax.p + id);
      else vx.x = vx.y = vx.z = vx.w = ax.c;
      if (ay.p) vy = load_quad (ay.p + id);
      else vy.x = vy.y = vy.z = vy.w = ay.c;
      put_quad (sr(c0), sr(c0 ^ 1), p*M + 2*k, vr);
      if (LAM) put_quad (sl(c0), sl(c0 ^ 1), p*M + 2*k, vl);
      put_quad (sx(c0), sx(c0 ^ 1), p*M + 2*k, vx);
      put_quad (sy(c0), sy(c0 ^ 1), p*MY + 2*k, vy);
    }
    /* the last x-face row (face i0 + W <= n) and y-face column (j0 + W <= n;
       face n of a periodic direction is face 0) */
    const int fi = real_face (i0 + W, n, px), fj = real_face (j0 + W, n, py);
    for (int idx = tid; idx < QW + W; idx += nth) {
      if (idx < QW) {
        const int q = 4*idx, c0 = (base + W + q) & 1;
        Quad<T> vx;
        if (ax.p) vx = load_quad (ax.p + cidx<2> (g, fi, j0 + q, 0));
        else vx.x = vx.y = vx.z = vx.w = ax.c;
        put_quad (sx(c0), sx(c0 ^ 1), W*M + 2*idx, vx);
      }
      else {
        const int p = idx - QW, c = (base + p + W) & 1;
        sy(c)[p*MY + W/2] = ay.p ? ay.p[cidx<2> (g, i0 + p, fj, 0)] : ay.c;
      }
    }
    /* the iterate is the previous launch's output */
    grid_dependency_wait ();
    for (int idx = tid; idx < W*QW; idx += nth) {
      const int p = idx/QW, k = idx - p*QW, q = 4*k;
      const int c0 = (base + p + q) & 1;
      const Quad<T> va = load_quad (in + cidx<2> (g, i0 + p, j0 + q, 0));
      put_quad (sa(c0), sa(c0 ^ 1), p*M + 2*k, va);
    }
  }
  else {
  /* stage cells and faces with asynchronous copies (zero fill outside) */
  for (int idx = tid; idx < W*W; idx += nth) {
    const int p = idx/W, q = idx - p*W;
    const int c = (base + p + q) & 1, m = q >> 1;
    const int ri = real_index (i0 + p, n, px), rj = real_index (j0 + q, n, py);
    const bool ok = ri >= 0 && rj >= 0;
    const long long id = ok ? cidx<2> (g, ri, rj, 0) : 0;
    cp_async_elem (&sr(c)[p*M + m], res + id, ok);
    if (LAM) cp_async_elem (&sl(c)[p*M + m], lam.p + id, ok);
  }
  /* x faces: W+1 rows of W (face (p, q): lower face of cell (p, q)) */
  for (int idx = tid; idx < (W + 1)*W; idx += nth) {
    const int p = idx/W, q = idx - p*W;
    const int c = (base + p + q) & 1;
    const int fi = real_face (i0 + p, n, px), rj = real_index (j0 + q, n, py);
    const bool ok = fi >= 0 && rj >= 0;
    if (ax.p) cp_async_elem (&sx(c)[p*M + (q >> 1)], ax.p + (ok ? cidx<2> (g, fi, rj, 0) : 0), ok);
    else sx(c)[p*M + (q >> 1)] = ok ? ax.c : T(0);
  }
  /* y faces: W rows of W+1 (face (p, q): left face of cell (p, q)) */
  for (int idx = tid; idx < W*(W + 1); idx += nth) {
    const int p = idx/(W + 1), q = idx - p*(W + 1);
    const int c = (base + p + q) & 1;
    const int ri = real_index (i0 + p, n, px), fj = real_face (j0 + q, n, py);
    const bool ok = ri >= 0 && fj >= 0;
    if (ay.p) cp_async_elem (&sy(c)[p*MY + (q >> 1)], ay.p + (ok ? cidx<2> (g, ri, fj, 0) : 0), ok);
    else sy(c)[p*MY + (q >> 1)] = ok ? ay.c : T(0);
  }
  grid_dependency_wait ();
  for (int idx = tid; idx < W*W; idx += nth) {
    const int p = idx/W, q = idx - p*W;
    const int c = (base + p + q) & 1, m = q >> 1;
    const int ri = real_index (i0 + p, n, px), rj = real_index (j0 + q, n, py);
    const bool ok = ri >= 0 && rj >= 0;
    cp_async_elem (&sa(c)[p*M + m], in + (ok ? cidx<2> (g, ri, rj, 0) : 0), ok);
  }
  }
  cp_async_wait_all ();
  __syncthreads ();

  /* box ghosts (global -1 and n) of the staged region: ghost = factor x
     mirror, both of opposite colours at the same or adjacent column index */
  const int glo_i = px ? -1 : -1 - i0, ghi_i = px ? -1 : n - i0;
  const int glo_j = py ? -1 : -1 - j0, ghi_j = py ? -1 : n - j0;
  const bool has_ghosts = !inner &&
    ((glo_i >= 0 && glo_i < W) || (ghi_i >= 0 && ghi_i < W) ||
     (glo_j >= 0 && glo_j < W) || (ghi_j >= 0 && ghi_j < W));
  auto refresh = [&] () {
    for (int t = tid; t < 4*W; t += nth) {
      const int line = t/W, u = t - line*W;
      int p, q, pm, qm, f;
      if (line == 0) { p = glo_i; q = u; pm = p + 1; qm = q; f = bc.fac[1]; }
      else if (line == 1) { p = ghi_i; q = u; pm = p - 1; qm = q; f = bc.fac[0]; }
      else if (line == 2) { p = u; q = glo_j; pm = p; qm = q + 1; f = bc.fac[3]; }
      else { p = u; q = ghi_j; pm = p; qm = q - 1; f = bc.fac[2]; }
      if (p < 0 || p >= W || q < 0 || q >= W || pm < 0 || pm >= W || qm < 0 || qm >= W)
        continue;
      if (line < 2 ? real_index (j0 + q, n, py) < 0 : real_index (i0 + p, n, px) < 0)
        continue;
      const int c = (base + p + q) & 1;
      sa(c)[p*M + (q >> 1)] = sa(c ^ 1)[pm*M + (qm >> 1)]*T(f);
    }
  };
  if (has_ghosts) refresh ();
  __syncthreads ();

  const T D2 = Delta*Delta;
  for (int sw = 0; sw < nsweeps; sw++)
#pragma unroll
    for (int c = 0; c < 2; c++) {
      const int k = 2*sw + c;
      const int lo = k + 1, hi = W - k - 1;      /* valid update region [lo, hi)^2 */
      const T * __restrict__ o_a = sa(c ^ 1);
      const T * __restrict__ xr = sx(c), * __restrict__ xo = sx(c ^ 1);
      const T * __restrict__ yr = sy(c), * __restrict__ yo = sy(c ^ 1);
      T * __restrict__ a = sa(c);
      const T * __restrict__ r = sr(c);
      const T * __restrict__ l = sl(c);
      /* thread (tx, ty): cells m0 = CPT tx .. m0 + CPT - 1 of colour c in row
         lo + pr; a warp covers RW rows of one parity (pr interleaves them),
         so the colour offset o, and every branch on it, is uniform per warp */
      const int p = lo + pr;
      if (p < hi) {
        const int o = (c - base - p) & 1;        /* column offset of colour c */
        const int mlo = (lo - o + 1) >> 1, mhi = (hi - o + 1) >> 1;
        const int m0 = 2*tx;
        bool ok0 = m0 >= mlo && m0 < mhi, ok1 = m0 + 1 >= mlo && m0 + 1 < mhi;
        if (!inner) {
          const int gi = i0 + p, gj = j0 + 2*m0 + o;
          const bool rowok = px || (unsigned) gi < (unsigned) n;
          ok0 = ok0 && rowok && (py || (unsigned) gj < (unsigned) n);
          ok1 = ok1 && rowok && (py || (unsigned) (gj + 2) < (unsigned) n);
        }
        if (ok0 || ok1) {
          const int ci = p*M + m0;
          const T2 up = *(const T2 *) &o_a[ci - M], dn = *(const T2 *) &o_a[ci + M];
          /* the other colour's cells left and right: [m0-1+o], [m0+o], [m0+1+o] */
          T vl, vm, vr;
          if (o == 0) {
            const T2 v = *(const T2 *) &o_a[ci];
            vl = o_a[ci - 1]; vm = v.x; vr = v.y;
          }
          else {
            const T2 v = *(const T2 *) &o_a[ci];
            vl = v.x; vm = v.y; vr = o_a[ci + 2];
          }
          const T2 rr = *(const T2 *) &r[ci];
          const T2 xl = *(const T2 *) &xr[ci], xu = *(const T2 *) &xo[ci + M];
          const T2 yl = *(const T2 *) &yr[p*MY + m0];
          T yr0, yr1;
          if (o == 0) { const T2 v = *(const T2 *) &yo[p*MY + m0]; yr0 = v.x; yr1 = v.y; }
          else { yr0 = yo[p*MY + m0 + 1]; yr1 = yo[p*MY + m0 + 2]; }
          T2 lv;
          if (LAM) lv = *(const T2 *) &l[ci];
          else { lv.x = lam.c; lv.y = lam.c; }
          /* relax_value's expression and order (poisson.h:303-319), two cells */
          T n0 = (-D2)*rr.x, d0 = (-lv.x)*D2;
          T n1 = (-D2)*rr.y, d1 = (-lv.y)*D2;
          n0 = tile_acc (n0, xu.x, dn.x, xl.x, up.x); d0 += xu.x + xl.x;
          n1 = tile_acc (n1, xu.y, dn.y, xl.y, up.y); d1 += xu.y + xl.y;
          n0 = tile_acc (n0, yr0, vm, yl.x, vl);      d0 += yr0 + yl.x;
          n1 = tile_acc (n1, yr1, vr, yl.y, vm);      d1 += yr1 + yl.y;
          const T a0 = relax_div (n0, d0), a1 = relax_div (n1, d1);
          if (ok0 && ok1) { T2 w; w.x = a0; w.y = a1; *(T2 *) &a[ci] = w; }
          else if (ok0) a[ci] = a0;
          else a[ci + 1] = a1;
        }
      }
      __syncthreads ();
      if (has_ghosts) {
        refresh ();
        __syncthreads ();
      }
    }

  /* write the tile interior back, with its ghost images */
  if (inner) {
    /* no domain-boundary cell in the interior: 16-byte stores, no ghosts */
    constexpr int QT = TS/4;
    for (int idx = tid; idx < TS*QT; idx += nth) {
      const int rr = idx/QT, k = idx - rr*QT;
      const int p = rr + H, q = H + 4*k, c0 = (base + p + q) & 1, m = q >> 1;
      Quad<T> v;
      v.x = sa(c0)[p*M + m]; v.z = sa(c0)[p*M + m + 1];
      v.y = sa(c0 ^ 1)[p*M + m]; v.w = sa(c0 ^ 1)[p*M + m + 1];
      store_quad (out + cidx<2> (g, blockIdx.y*TS + rr, blockIdx.x*TS + 4*k, 0), v);
    }
    return;
  }
  for (int idx = tid; idx < TS*TS; idx += nth) {
    const int rr = idx/TS, s = idx - rr*TS;
    const int gi = blockIdx.y*TS + rr, gj = blockIdx.x*TS + s;
    if (gi >= n || gj >= n) continue;
    const int p = rr + H, q = s + H;
    const T v = sa((base + p + q) & 1)[p*M + (q >> 1)];
    out[cidx<2> (g, gi, gj, 0)] = v;
    ghosts_homog<2, T> (out, g, gi, gj, 0, v, bc);
  }
}

/* ---------------------------------------------------------------- */
/* FP32 tiles with register-resident weights                         */
/* ---------------------------------------------------------------- */

/* The FP32 red-black sweeps of the mixed form on large 2D levels, S per
   launch on TS x TS tiles staged with a 2S halo, as k_relax_tile2d, but
   with the roles of registers and shared memory swapped: each of the 512
   threads owns eight cells of the staged W x W region for the whole launch
   (one row, four cells of each colour), reads their coefficients from
   global memory once and divides them by the diagonal,

     a = beta + w_xl a[-1,0] + w_xu a[1,0] + w_yl a[0,-1] + w_yr a[0,1],
     w = alpha/d,  beta = -Delta^2 res/d,  d = sum of the four alpha - lambda Delta^2,

   the relaxation of relax_value (poisson.h:303-319) up to FP32 rounding.
   Only the iterate lives in shared memory (16 KB, split by colour), so a
   colour pass reads four operands per cell instead of nine and issues four
   fused multiply-adds per cell instead of a division and eleven
   operations: the shared-memory pipe, which bounds k_relax_tile2d, carries
   less than half the traffic. */
namespace tw {
constexpr int W = 64, M = W/2, WM = W*M, BX = 8, BY = 64;
static_assert (W == 8*BX && W - 2 <= BY && BY % 8 == 0, "one row of eight cells per thread");
/* a tile of TS x TS cells in the W x W staged region: a halo of
   H = (W - TS)/2 cells, S = H/2 sweeps per launch (48: 4 sweeps, 32: 8) */
template <int TS> struct Tile {
  static constexpr int H = (W - TS)/2, S = H/2;
  static_assert (TS % 4 == 0 && H % 2 == 0 && H > 0, "tile of quads, even halo");
};
}

/* shared-memory accesses by 32-bit byte address plus a constant offset
   (volatile: kept in program order with the barriers) */
template <int OFF>
__device__ __forceinline__ float4 lds_f4 (unsigned a)
{
  float4 v;
  asm volatile ("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4+%5];"
                : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(a), "n"(OFF));
  return v;
}

template <int OFF>
__device__ __forceinline__ float lds_f1 (unsigned a)
{
  float v;
  asm volatile ("ld.shared.f32 %0, [%1+%2];" : "=f"(v) : "r"(a), "n"(OFF));
  return v;
}

__device__ __forceinline__ void sts_f4 (unsigned a, float4 v)
{
  asm volatile ("st.shared.v4.f32 [%0], {%1, %2, %3, %4};"
                :: "r"(a), "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w) : "memory");
}

__device__ __forceinline__ void sts_f1 (unsigned a, float v)
{
  asm volatile ("st.shared.f32 [%0], %1;" :: "r"(a), "f"(v) : "memory");
}

template <int TS, bool LAM>
__global__ void __launch_bounds__ (tw::BX*tw::BY, 2)
k_relax_tile2d_w (bmg_geom g, float * __restrict__ out, const float * __restrict__ in,
                  const float * __restrict__ res, Coef<float> ax, Coef<float> ay, Coef<float> lam,
                  float Delta, BCH bc, int nsweeps, double * __restrict__ acor, bmg_geom ga,
                  bmg_bcdesc abc, const float * __restrict__ coarse, bmg_geom gc)
{
  using namespace tw;
  constexpr int H = Tile<TS>::H;
  __shared__ __align__ (16) float sa[2*WM];     /* colour c of staged cell (p, q) at c*WM + p*M + q/2 */
  const int n = g.n, tx = threadIdx.x, ty = threadIdx.y, tid = ty*BX + tx, nth = BX*BY;
  constexpr int RW = 32/BX;                     /* rows per warp, all of one parity */
  const int p = 2*RW*(ty/(2*RW)) + 2*(ty % RW) + ((ty/RW) & 1);
  const int i0 = blockIdx.y*TS - H, j0 = blockIdx.x*TS - H;
  const int px = bc.periodic[0], py = bc.periodic[1];
  const int base = (i0 + j0) & 1;
  const bool inner = i0 >= 0 && i0 + W <= n && j0 >= 0 && j0 + W <= n;
  const int q0 = 8*tx, m0 = 4*tx, gi = i0 + p;
  const float D2 = Delta*Delta;
  grid_dependents_launch ();

  /* the coefficients of the thread's eight columns q0 .. q0 + 7 of row p
     (x faces below and above, y faces left of each column and right of the
     last), res and lambda */
  float r8[8], xl8[8], xu8[8], yl8[9], l8[8];
  if (inner) {
    const long long id = cidx<2> (g, gi, j0 + q0, 0);
    const Quad<float> r0 = load_quad (res + id), r1 = load_quad (res + id + 4);
    r8[0] = r0.x; r8[1] = r0.y; r8[2] = r0.z; r8[3] = r0.w;
    r8[4] = r1.x; r8[5] = r1.y; r8[6] = r1.z; r8[7] = r1.w;
    if (ax.p) {
      const Quad<float> a0 = load_quad (ax.p + id), a1 = load_quad (ax.p + id + 4);
      const Quad<float> b0 = load_quad (ax.p + id + g.P), b1 = load_quad (ax.p + id + g.P + 4);
      xl8[0] = a0.x; xl8[1] = a0.y; xl8[2] = a0.z; xl8[3] = a0.w;
      xl8[4] = a1.x; xl8[5] = a1.y; xl8[6] = a1.z; xl8[7] = a1.w;
      xu8[0] = b0.x; xu8[1] = b0.y; xu8[2] = b0.z; xu8[3] = b0.w;
      xu8[4] = b1.x; xu8[5] = b1.y; xu8[6] = b1.z; xu8[7] = b1.w;
    }
    else
#pragma unroll
      for (int q = 0; q < 8; q++) xl8[q] = xu8[q] = ax.c;
    if (ay.p) {
      const Quad<float> a0 = load_quad (ay.p + id), a1 = load_quad (ay.p + id + 4);
      yl8[0] = a0.x; yl8[1] = a0.y; yl8[2] = a0.z; yl8[3] = a0.w;
      yl8[4] = a1.x; yl8[5] = a1.y; yl8[6] = a1.z; yl8[7] = a1.w;
      yl8[8] = ay.p[id + 8];
    }
    else
#pragma unroll
      for (int q = 0; q < 9; q++) yl8[q] = ay.c;
    if (LAM) {
      const Quad<float> a0 = load_quad (lam.p + id), a1 = load_quad (lam.p + id + 4);
      l8[0] = a0.x; l8[1] = a0.y; l8[2] = a0.z; l8[3] = a0.w;
      l8[4] = a1.x; l8[5] = a1.y; l8[6] = a1.z; l8[7] = a1.w;
    }
  }
  else {
    /* outside the domain: zero, or the periodic image */
    const int ri = real_index (gi, n, px);
    const int flo = real_face (gi, n, px), fhi = real_face (gi + 1, n, px);
#pragma unroll
    for (int q = 0; q < 9; q++) {
      const int rj = real_index (j0 + q0 + q, n, py), fj = real_face (j0 + q0 + q, n, py);
      yl8[q] = ri >= 0 && fj >= 0 ? ay.at (cidx<2> (g, ri, fj, 0)) : 0.f;
      if (q == 8) break;
      const bool ok = ri >= 0 && rj >= 0;
      r8[q] = ok ? res[cidx<2> (g, ri, rj, 0)] : 0.f;
      xl8[q] = flo >= 0 && rj >= 0 ? ax.at (cidx<2> (g, flo, rj, 0)) : 0.f;
      xu8[q] = fhi >= 0 && rj >= 0 ? ax.at (cidx<2> (g, fhi, rj, 0)) : 0.f;
      if (LAM) l8[q] = ok ? lam.p[cidx<2> (g, ri, rj, 0)] : 0.f;
    }
  }
  /* the iterate is the previous launch's output: its loads are issued
     before the weights are computed, so that both round trips overlap */
  grid_dependency_wait ();
  const int cq = (base + p) & 1;                /* colour of the even columns */
  if (coarse) {
    /* the level's first launch: the iterate is the prolongation of the
       coarse level, computed here instead of by its own launch */
    if (inner) {
      float v8[8];
      prolong_row<float, 8> (coarse, gc, gi, j0 + q0, v8);
      const Quad<float> va = {v8[0], v8[1], v8[2], v8[3]}, vb = {v8[4], v8[5], v8[6], v8[7]};
      put_quad (sa + cq*WM, sa + (cq ^ 1)*WM, p*M + m0, va);
      put_quad (sa + cq*WM, sa + (cq ^ 1)*WM, p*M + m0 + 2, vb);
    }
    else {
      const int ri = real_index (gi, n, px);
#pragma unroll
      for (int q = 0; q < 8; q++) {
        const int rj = real_index (j0 + q0 + q, n, py);
        sa[((cq + q) & 1)*WM + p*M + ((q0 + q) >> 1)] =
          ri >= 0 && rj >= 0 ? prolong_cell<float> (coarse, gc, ri, rj) : 0.f;
      }
    }
  }
  else if (inner) {
    const long long id = cidx<2> (g, gi, j0 + q0, 0);
    const Quad<float> va = load_quad (in + id), vb = load_quad (in + id + 4);
    put_quad (sa + cq*WM, sa + (cq ^ 1)*WM, p*M + m0, va);
    put_quad (sa + cq*WM, sa + (cq ^ 1)*WM, p*M + m0 + 2, vb);
  }
  else {
    const int ri = real_index (gi, n, px);
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const int rj = real_index (j0 + q0 + q, n, py);
      sa[((cq + q) & 1)*WM + p*M + ((q0 + q) >> 1)] =
        ri >= 0 && rj >= 0 ? in[cidx<2> (g, ri, rj, 0)] : 0.f;
    }
  }
  /* weights of cell e of colour c: column 2e + o_c of the eight */
  float wxl[2][4], wxu[2][4], wyl[2][4], wyr[2][4], be[2][4];
  unsigned valid = 0;                           /* bit 4c + e: a cell that is updated */
  const bool rowok = px || (unsigned) gi < (unsigned) n;
#pragma unroll
  for (int c = 0; c < 2; c++)
#pragma unroll
    for (int e = 0; e < 4; e++) {
      /* column 2e or 2e + 1 (selects with constant indices: a runtime
         index would put the arrays in local memory) */
      const bool odd = (c ^ base ^ p) & 1;
      const int q = 2*e + (odd ? 1 : 0);
      const float xl = odd ? xl8[2*e + 1] : xl8[2*e], xu = odd ? xu8[2*e + 1] : xu8[2*e];
      const float yl = odd ? yl8[2*e + 1] : yl8[2*e], yr = odd ? yl8[2*e + 2] : yl8[2*e + 1];
      const float rv = odd ? r8[2*e + 1] : r8[2*e];
      const float lv = LAM ? (odd ? l8[2*e + 1] : l8[2*e]) : lam.c;
      const bool ok = rowok && (py || (unsigned) (j0 + q0 + q) < (unsigned) n);
      float d = (-lv)*D2;
      d += xu + xl;
      d += yr + yl;
      const float inv = ok ? __fdividef (1.f, d) : 0.f;
      wxl[c][e] = xl*inv; wxu[c][e] = xu*inv;
      wyl[c][e] = yl*inv; wyr[c][e] = yr*inv;
      be[c][e] = ((-D2)*rv)*inv;
      valid |= (ok ? 1u : 0u) << (4*c + e);
    }

  __syncthreads ();

  /* box ghosts (global -1 and n) of the staged region: ghost = factor x
     mirror */
  const int glo_i = px ? -1 : -1 - i0, ghi_i = px ? -1 : n - i0;
  const int glo_j = py ? -1 : -1 - j0, ghi_j = py ? -1 : n - j0;
  const bool has_ghosts = !inner &&
    ((glo_i >= 0 && glo_i < W) || (ghi_i >= 0 && ghi_i < W) ||
     (glo_j >= 0 && glo_j < W) || (ghi_j >= 0 && ghi_j < W));
  auto refresh = [&] () {
    for (int t = tid; t < 4*W; t += nth) {
      const int line = t/W, u = t - line*W;
      int pp, q, pm, qm, f;
      if (line == 0) { pp = glo_i; q = u; pm = pp + 1; qm = q; f = bc.fac[1]; }
      else if (line == 1) { pp = ghi_i; q = u; pm = pp - 1; qm = q; f = bc.fac[0]; }
      else if (line == 2) { pp = u; q = glo_j; pm = pp; qm = q + 1; f = bc.fac[3]; }
      else { pp = u; q = ghi_j; pm = pp; qm = q - 1; f = bc.fac[2]; }
      if (pp < 0 || pp >= W || q < 0 || q >= W || pm < 0 || pm >= W || qm < 0 || qm >= W)
        continue;
      if (line < 2 ? real_index (j0 + q, n, py) < 0 : real_index (i0 + pp, n, px) < 0)
        continue;
      const int c = (base + pp + q) & 1;
      sa[c*WM + pp*M + (q >> 1)] = sa[(c ^ 1)*WM + pm*M + (qm >> 1)]*float(f);
    }
  };
  if (has_ghosts) {
    refresh ();
    __syncthreads ();
  }

  /* the colour passes.  Rows shrink by one per pass (whole warps drop out);
     columns do not: a cell next to the staged region's edge may be updated
     from stale neighbours, but staleness moves inward by one cell per pass
     and never reaches the TS x TS interior after 2S passes, so only cells
     outside the domain (box ghosts, refreshed from their mirrors) are
     masked.  Shared memory is addressed by 32-bit byte offsets with the
     row offsets as immediates. */
  const unsigned sbase = (unsigned) __cvta_generic_to_shared (sa);
  const int o0 = (base ^ p) & 1;               /* column offset of colour 0 in row p */
  for (int sw = 0; sw < nsweeps; sw++)
#pragma unroll
    for (int c = 0; c < 2; c++) {
      const int k = 2*sw + c;
      if (p >= k + 1 && p < W - k - 1) {
        const int o = o0 ^ c;
        /* the other colour's quad at rows p - 1, p, p + 1 and its left or
           right neighbour in row p */
        const unsigned aup = sbase + 4u*((c ^ 1)*WM + (p - 1)*M + m0);
        const float4 up = lds_f4<0> (aup), mid = lds_f4<4*M> (aup), dn = lds_f4<8*M> (aup);
        float v[5];
        if (o == 0) { v[0] = lds_f1<4*M - 4> (aup); v[1] = mid.x; v[2] = mid.y; v[3] = mid.z; v[4] = mid.w; }
        else { v[0] = mid.x; v[1] = mid.y; v[2] = mid.z; v[3] = mid.w; v[4] = lds_f1<4*M + 16> (aup); }
        const float upv[4] = {up.x, up.y, up.z, up.w}, dnv[4] = {dn.x, dn.y, dn.z, dn.w};
        float nv[4];
#pragma unroll
        for (int e = 0; e < 4; e++)
          nv[e] = fmaf (wyr[c][e], v[e + 1], fmaf (wyl[c][e], v[e],
                  fmaf (wxu[c][e], dnv[e], fmaf (wxl[c][e], upv[e], be[c][e]))));
        const unsigned aw = sbase + 4u*(c*WM + p*M + m0);
        const unsigned vc = (valid >> (4*c)) & 15u;
        if (vc == 15u)
          sts_f4 (aw, make_float4 (nv[0], nv[1], nv[2], nv[3]));
        else {
          if (vc & 1u) sts_f1 (aw, nv[0]);
          if (vc & 2u) sts_f1 (aw + 4, nv[1]);
          if (vc & 4u) sts_f1 (aw + 8, nv[2]);
          if (vc & 8u) sts_f1 (aw + 12, nv[3]);
        }
      }
      __syncthreads ();
      if (has_ghosts) {
        refresh ();
        __syncthreads ();
      }
    }

  /* the tile interior back, with its ghost images; the last launch of a
     cycle's finest level also applies the correction a += da
     (poisson.h:84-89, k_correct's expression) to its tile, with the
     boundary conditions of a */
  if (inner) {
    constexpr int QT = TS/4;
    for (int idx = tid; idx < TS*QT; idx += nth) {
      const int rr = idx/QT, k = idx - rr*QT;
      const int pp = rr + H, q = H + 4*k, c0 = (base + pp + q) & 1, m = q >> 1;
      Quad<float> v;
      v.x = sa[c0*WM + pp*M + m]; v.z = sa[c0*WM + pp*M + m + 1];
      v.y = sa[(c0 ^ 1)*WM + pp*M + m]; v.w = sa[(c0 ^ 1)*WM + pp*M + m + 1];
      const int oi = blockIdx.y*TS + rr, oj = blockIdx.x*TS + 4*k;
      store_quad (out + cidx<2> (g, oi, oj, 0), v);
      if (acor) {
        double * ap = acor + cidx<2> (ga, oi, oj, 0);
        Quad<double> av = load_quad (ap);
        av.x = av.x + (double) v.x; av.y = av.y + (double) v.y;
        av.z = av.z + (double) v.z; av.w = av.w + (double) v.w;
        store_quad (ap, av);
      }
    }
    return;
  }
  for (int idx = tid; idx < TS*TS; idx += nth) {
    const int rr = idx/TS, s = idx - rr*TS;
    const int oi = blockIdx.y*TS + rr, oj = blockIdx.x*TS + s;
    if (oi >= n || oj >= n) continue;
    const int pp = rr + H, q = s + H;
    const float v = sa[((base + pp + q) & 1)*WM + pp*M + (q >> 1)];
    out[cidx<2> (g, oi, oj, 0)] = v;
    ghosts_homog<2, float> (out, g, oi, oj, 0, v, bc);
    if (acor) {
      const long long ia = cidx<2> (ga, oi, oj, 0);
      const double an = acor[ia] + (double) v;
      acor[ia] = an;
      ghosts_inhomog<2> (acor, ga, oi, oj, 0, an, abc);
    }
  }
}

/* ---------------------------------------------------------------- */
/* cluster level kernel: all nrelax sweeps of a middle FP32 level     */
/* ---------------------------------------------------------------- */

/* The 128^2 and 256^2 levels of the mixed form's cycle are pure latency as
   launches of four sweeps (about 7 us per launch for a few microseconds of
   arithmetic).  This kernel relaxes such a level nrelax times in one launch
   of one thread-block cluster of C CTAs, with the level held on chip for
   the whole launch:

     - CTA r owns R = N/C full rows [rR, rR + R) and stages them with H = 8
       rows of halo on either side (R + 2H rows x N columns, colour-split
       in shared memory as in k_relax_tile2d_w, with a ghost column on each
       side);
     - every thread owns eight consecutive cells of one staged row per
       segment (SEG segments) and keeps their weights -- the coefficients
       divided by the diagonal, computed once per launch -- in registers;
     - a block of S = 4 sweeps stages the owned rows from the CTA's own
       exchange buffer and the halo rows from its neighbours' exchange
       buffers (distributed shared memory), runs 2S colour passes on the
       staged rows (staleness moves in one row per pass and never reaches
       the owned rows), writes the owned rows to its exchange buffer and
       meets the cluster at one barrier.  Exchange buffers alternate, so a
       block never overwrites what a neighbour may still be reading;
     - the first block stages the bilinear prolongation of the coarse level
       (multigrid-common.h:124-140, the expression of k_prolong2d_blk)
       instead, which fuses the level's prolongation in;
     - box ghost cells (rows -1 and N on the first and last CTA, columns -1
       and N everywhere) and periodic ghost columns are written by the
       thread that updates their mirror cell, right after the update: only
       that cell reads them in a colour pass.  Periodic rows come from the
       neighbour across the wrap.
   The level's final iterate, with every ghost image, goes to out.  The
   weights and the arithmetic of a cell update are those of
   k_relax_tile2d_w (the relaxation of relax_value, poisson.h:303-319, up
   to FP32 rounding).  Row and column indices: i along x (rows, sides
   left/right), j along y (the contiguous axis, sides bottom/top). */
namespace cl {
template <int N, int C, int SEG> struct Shape {
  static constexpr int R = N/C, H = 8, S = 4;
  static constexpr int BYR = R + 2*H;             /* staged rows */
  static constexpr int BX = N/(8*SEG);            /* threads per row */
  static constexpr int NT = BX*BYR;
  static constexpr int RW = 32/BX;                /* rows per warp */
  static constexpr int OFS = 4;                   /* interior m = 0; ghost m = -1 at OFS - 1 */
  static constexpr int MP = N/2 + 8;              /* colour row pitch (16-byte rows) */
  static constexpr int SAW = BYR*MP, OWW = R*MP;  /* one colour of the staged / owned rows */
  static constexpr size_t bytes = sizeof (float)*(2*SAW + 4*OWW);
  static_assert (R >= H && 32 % BX == 0 && BYR % (2*RW) == 0 && NT <= 1024, "cluster level shape");
};
}

__device__ __forceinline__ void cluster_barrier ()
{
  asm volatile ("barrier.cluster.arrive.release.aligned;\n"
                "barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

__device__ __forceinline__ unsigned cluster_rank ()
{
  unsigned r;
  asm volatile ("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}

/* the generic address of the same shared-memory location in CTA rank */
template <typename T>
__device__ __forceinline__ T * cluster_map (T * p, unsigned rank)
{
  unsigned long long r;
  asm volatile ("mapa.u64 %0, %1, %2;" : "=l"(r) : "l"(p), "r"(rank));
  return (T *) r;
}

template <int N, int C, int SEG, bool LAM>
__global__ void __launch_bounds__ (cl::Shape<N, C, SEG>::NT, 1)
k_level_cluster (bmg_geom g, float * __restrict__ out, const float * __restrict__ res,
                 Coef<float> ax, Coef<float> ay, Coef<float> lam, float Delta, BCH bc, int nrelax,
                 bmg_geom gc, const float * __restrict__ coarse)
{
  typedef cl::Shape<N, C, SEG> Sh;
  constexpr int R = Sh::R, H = Sh::H, S = Sh::S, BYR = Sh::BYR, BX = Sh::BX, RW = Sh::RW;
  constexpr int OFS = Sh::OFS, MP = Sh::MP, SAW = Sh::SAW, OWW = Sh::OWW;
  extern __shared__ __align__ (16) float csm[];
  float * sa = csm;                       /* [2][BYR][MP] staged rows */
  float * own = csm + 2*SAW;              /* [2 buffers][2][R][MP] owned rows */
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int p = 2*RW*(ty/(2*RW)) + 2*(ty % RW) + ((ty/RW) & 1);
  const int rank = (int) cluster_rank ();
  const int px = bc.periodic[0], py = bc.periodic[1];
  const int gi = rank*R - H + p;          /* global row of staged row p */
  const int ri = real_index (gi, N, px);  /* its real row, -1: none */
  const bool rowok = ri >= 0;
  const int ce = gi & 1;                  /* colour of the even columns */
  const float D2 = Delta*Delta;
  pdl_trigger ();

  /* weights of the thread's cells: segment sg covers columns q0 .. q0 + 7,
     q0 = 8 (tx + sg BX); colour c's cells are e = 0..3 at column
     q0 + 2e + (c ^ ce) */
  float wxl[SEG][2][4], wxu[SEG][2][4], wyl[SEG][2][4], wyr[SEG][2][4], be[SEG][2][4];
#pragma unroll
  for (int sg = 0; sg < SEG; sg++) {
    const int q0 = 8*(tx + sg*BX);
    float r8[8], xl8[8], xu8[8], yl8[9], l8[8];
#pragma unroll
    for (int q = 0; q < 8; q++) { r8[q] = xl8[q] = xu8[q] = yl8[q] = l8[q] = 0.f; }
    yl8[8] = 0.f;
    if (rowok) {
      const int flo = real_face (gi, N, px), fhi = real_face (gi + 1, N, px);
      const long long id = cidx<2> (g, ri, q0, 0);
      const Quad<float> r0 = load_quad (res + id), r1 = load_quad (res + id + 4);
      r8[0] = r0.x; r8[1] = r0.y; r8[2] = r0.z; r8[3] = r0.w;
      r8[4] = r1.x; r8[5] = r1.y; r8[6] = r1.z; r8[7] = r1.w;
      if (ax.p) {
        const long long il = cidx<2> (g, flo, q0, 0), iu = cidx<2> (g, fhi, q0, 0);
        const Quad<float> a0 = load_quad (ax.p + il), a1 = load_quad (ax.p + il + 4);
        const Quad<float> b0 = load_quad (ax.p + iu), b1 = load_quad (ax.p + iu + 4);
        xl8[0] = a0.x; xl8[1] = a0.y; xl8[2] = a0.z; xl8[3] = a0.w;
        xl8[4] = a1.x; xl8[5] = a1.y; xl8[6] = a1.z; xl8[7] = a1.w;
        xu8[0] = b0.x; xu8[1] = b0.y; xu8[2] = b0.z; xu8[3] = b0.w;
        xu8[4] = b1.x; xu8[5] = b1.y; xu8[6] = b1.z; xu8[7] = b1.w;
      }
      else
#pragma unroll
        for (int q = 0; q < 8; q++) xl8[q] = xu8[q] = ax.c;
      if (ay.p) {
        const Quad<float> a0 = load_quad (ay.p + id), a1 = load_quad (ay.p + id + 4);
        yl8[0] = a0.x; yl8[1] = a0.y; yl8[2] = a0.z; yl8[3] = a0.w;
        yl8[4] = a1.x; yl8[5] = a1.y; yl8[6] = a1.z; yl8[7] = a1.w;
        /* face q0 + 8: face N of a periodic direction is face 0 */
        yl8[8] = ay.p[cidx<2> (g, ri, real_face (q0 + 8, N, py), 0)];
      }
      else
#pragma unroll
        for (int q = 0; q < 9; q++) yl8[q] = ay.c;
      if (LAM) {
        const Quad<float> a0 = load_quad (lam.p + id), a1 = load_quad (lam.p + id + 4);
        l8[0] = a0.x; l8[1] = a0.y; l8[2] = a0.z; l8[3] = a0.w;
        l8[4] = a1.x; l8[5] = a1.y; l8[6] = a1.z; l8[7] = a1.w;
      }
    }
#pragma unroll
    for (int c = 0; c < 2; c++)
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const bool odd = (c ^ ce) & 1;
        const float xl = odd ? xl8[2*e + 1] : xl8[2*e], xu = odd ? xu8[2*e + 1] : xu8[2*e];
        const float yl = odd ? yl8[2*e + 1] : yl8[2*e], yr = odd ? yl8[2*e + 2] : yl8[2*e + 1];
        const float rv = odd ? r8[2*e + 1] : r8[2*e];
        const float lv = LAM ? (odd ? l8[2*e + 1] : l8[2*e]) : lam.c;
        float d = (-lv)*D2;
        d += xu + xl;
        d += yr + yl;
        const float inv = rowok ? __fdividef (1.f, d) : 0.f;
        wxl[sg][c][e] = xl*inv; wxu[sg][c][e] = xu*inv;
        wyl[sg][c][e] = yl*inv; wyr[sg][c][e] = yr*inv;
        be[sg][c][e] = ((-D2)*rv)*inv;
      }
  }

  /* ghost cells this thread writes after updating a cell: the box row
     ghost of rows 0 and N - 1, the column ghost of columns 0 and N - 1
     (box: the factor times the cell; periodic: the image across the wrap) */
  /* (a staged row 0 or BYR - 1 is never updated and has no ghost row
     inside the staged region: when R == H a neighbour's halo reaches the
     domain's first or last row there) */
  const bool rowghost_lo = !px && gi == 0 && p >= 1, rowghost_hi = !px && gi == N - 1 && p <= BYR - 2;
  const float frow = rowghost_lo ? (float) bc.fac[1] : (float) bc.fac[0];
  const float fbot = (float) bc.fac[3], ftop = (float) bc.fac[2];
  const bool first_col = tx == 0, last_col = tx == BX - 1;
  auto put_ghosts = [&] (int sg, int c, const float * nv) {
    /* colour-c cells of segment sg in row p were just written (values nv) */
    const int m0 = 4*(tx + sg*BX);
    if (rowghost_lo || rowghost_hi) {
      float * gr = sa + (c ^ 1)*SAW + (rowghost_lo ? p - 1 : p + 1)*MP + OFS + m0;
#pragma unroll
      for (int e = 0; e < 4; e++) gr[e] = nv[e]*frow;
    }
    const int o = c ^ ce;
    if (sg == 0 && first_col && o == 0) {          /* cell j = 0 */
      if (py) sa[c*SAW + p*MP + OFS + N/2] = nv[0];
      else sa[(c ^ 1)*SAW + p*MP + OFS - 1] = nv[0]*fbot;
    }
    if (sg == SEG - 1 && last_col && o == 1) {     /* cell j = N - 1 */
      if (py) sa[c*SAW + p*MP + OFS - 1] = nv[3];
      else sa[(c ^ 1)*SAW + p*MP + OFS + N/2] = nv[3]*ftop;
    }
  };
  /* the ghosts of a freshly staged row (both colours), from its cells */
  auto stage_ghosts = [&] () {
    if (!rowok) return;
    const int c0 = ce;               /* colour of column 0 */
    const int cl = ce ^ 1;           /* colour of column N - 1 */
    if (first_col) {
      const float v = sa[c0*SAW + p*MP + OFS];
      if (py) sa[c0*SAW + p*MP + OFS + N/2] = v;
      else sa[(c0 ^ 1)*SAW + p*MP + OFS - 1] = v*fbot;
    }
    if (last_col) {
      const float v = sa[cl*SAW + p*MP + OFS + N/2 - 1];
      if (py) sa[cl*SAW + p*MP + OFS - 1] = v;
      else sa[(cl ^ 1)*SAW + p*MP + OFS + N/2] = v*ftop;
    }
    if (rowghost_lo || rowghost_hi) {
      const int pg = rowghost_lo ? p - 1 : p + 1;
#pragma unroll
      for (int sg = 0; sg < SEG; sg++) {
        const int m0 = 4*(tx + sg*BX);
#pragma unroll
        for (int c = 0; c < 2; c++)
#pragma unroll
          for (int e = 0; e < 4; e++)
            sa[(c ^ 1)*SAW + pg*MP + OFS + m0 + e] = sa[c*SAW + p*MP + OFS + m0 + e]*frow;
      }
    }
  };

  const unsigned sbase = (unsigned) __cvta_generic_to_shared (sa);
  const int nblk = (nrelax + S - 1)/S;
  /* neighbours across the rows, -1: none (a box side) */
  const int up = rank > 0 ? rank - 1 : (px ? C - 1 : -1);
  const int dn = rank < C - 1 ? rank + 1 : (px ? 0 : -1);
  grid_dependency_wait ();

  for (int blk = 0; blk < nblk; blk++) {
    const int ks = nrelax - blk*S < S ? nrelax - blk*S : S;
    if (blk == 0) {
      /* the bilinear prolongation of the coarse level: the thread's eight
         cells of a segment have six consecutive coarse parents (with
         their neighbours) in each of two coarse rows */
#pragma unroll
      for (int sg = 0; sg < SEG; sg++) {
        const int q0 = 8*(tx + sg*BX), m0 = 4*(tx + sg*BX);
        float v8[8];
        if (rowok) {
          const int ci = ri >> 1, cx = (ri & 1) ? 1 : -1, cj0 = (q0 >> 1) - 1;
          const long long b0 = cidx<2> (gc, ci, cj0, 0), b1 = cidx<2> (gc, ci + cx, cj0, 0);
          float r0[6], r1[6];
#pragma unroll
          for (int u = 0; u < 6; u++) { r0[u] = coarse[b0 + u]; r1[u] = coarse[b1 + u]; }
#pragma unroll
          for (int q = 0; q < 8; q++) {
            const int u = 1 + (q >> 1), cy = (q & 1) ? 1 : -1;
            v8[q] = (9.f*r0[u] + 3.f*(r1[u] + r0[u + cy]) + r1[u + cy])/16.f;
          }
        }
        else
#pragma unroll
          for (int q = 0; q < 8; q++) v8[q] = 0.f;
        /* even columns have colour ce */
        *(float4 *) (sa + ce*SAW + p*MP + OFS + m0) = make_float4 (v8[0], v8[2], v8[4], v8[6]);
        *(float4 *) (sa + (ce ^ 1)*SAW + p*MP + OFS + m0) = make_float4 (v8[1], v8[3], v8[5], v8[7]);
      }
    }
    else {
      /* owned rows from this CTA's exchange buffer, halo rows from the
         neighbours' (written in the previous block) */
      const int src = (blk - 1) & 1;
      int u = rank, r = p - H;
      if (p < H) { u = up; r = R - H + p; }
      else if (p >= H + R) { u = dn; r = p - H - R; }
      const float * ob = own + src*2*OWW;
      const float * q = u < 0 ? NULL : (u == rank ? ob : cluster_map (ob, (unsigned) u));
#pragma unroll
      for (int sg = 0; sg < SEG; sg++) {
        const int m0 = 4*(tx + sg*BX);
#pragma unroll
        for (int c = 0; c < 2; c++) {
          float4 v = make_float4 (0.f, 0.f, 0.f, 0.f);
          if (q) v = *(const float4 *) (q + c*OWW + r*MP + OFS + m0);
          *(float4 *) (sa + c*SAW + p*MP + OFS + m0) = v;
        }
      }
    }
    __syncthreads ();
    stage_ghosts ();
    __syncthreads ();

    for (int sw = 0; sw < ks; sw++)
#pragma unroll
      for (int c = 0; c < 2; c++) {
        const int k = 2*sw + c;
        if (rowok && p >= k + 1 && p < BYR - k - 1) {
          const int o = c ^ ce;
#pragma unroll
          for (int sg = 0; sg < SEG; sg++) {
            const int m0 = 4*(tx + sg*BX);
            const unsigned aup = sbase + 4u*((c ^ 1)*SAW + (p - 1)*MP + OFS + m0);
            const float4 upq = lds_f4<0> (aup), mid = lds_f4<4*MP> (aup), dnq = lds_f4<8*MP> (aup);
            float v[5];
            if (o == 0) { v[0] = lds_f1<4*MP - 4> (aup); v[1] = mid.x; v[2] = mid.y; v[3] = mid.z; v[4] = mid.w; }
            else { v[0] = mid.x; v[1] = mid.y; v[2] = mid.z; v[3] = mid.w; v[4] = lds_f1<4*MP + 16> (aup); }
            const float upv[4] = {upq.x, upq.y, upq.z, upq.w}, dnv[4] = {dnq.x, dnq.y, dnq.z, dnq.w};
            float nv[4];
#pragma unroll
            for (int e = 0; e < 4; e++)
              nv[e] = fmaf (wyr[sg][c][e], v[e + 1], fmaf (wyl[sg][c][e], v[e],
                      fmaf (wxu[sg][c][e], dnv[e], fmaf (wxl[sg][c][e], upv[e], be[sg][c][e]))));
            sts_f4 (sbase + 4u*(c*SAW + p*MP + OFS + m0), make_float4 (nv[0], nv[1], nv[2], nv[3]));
            put_ghosts (sg, c, nv);
          }
        }
        __syncthreads ();
      }
    /* the owned rows into this block's exchange buffer, then the cluster
       barrier: the buffer is complete before any neighbour stages from it,
       and every CTA has staged from the other buffer before it is reused */
    if (p >= H && p < H + R) {
      float * ob = own + (blk & 1)*2*OWW;
#pragma unroll
      for (int sg = 0; sg < SEG; sg++) {
        const int m0 = 4*(tx + sg*BX);
#pragma unroll
        for (int c = 0; c < 2; c++)
          *(float4 *) (ob + c*OWW + (p - H)*MP + OFS + m0) =
            *(const float4 *) (sa + c*SAW + p*MP + OFS + m0);
      }
    }
    cluster_barrier ();
  }

  /* the owned rows, with every ghost image, to global memory */
  if (p >= H && p < H + R) {
#pragma unroll
    for (int sg = 0; sg < SEG; sg++) {
      const int q0 = 8*(tx + sg*BX), m0 = 4*(tx + sg*BX);
      const float4 a = *(const float4 *) (sa + ce*SAW + p*MP + OFS + m0);
      const float4 b = *(const float4 *) (sa + (ce ^ 1)*SAW + p*MP + OFS + m0);
      const float v8[8] = {a.x, b.x, a.y, b.y, a.z, b.z, a.w, b.w};
      float * o8 = out + cidx<2> (g, gi, q0, 0);
      *(float4 *) o8 = make_float4 (v8[0], v8[1], v8[2], v8[3]);
      *(float4 *) (o8 + 4) = make_float4 (v8[4], v8[5], v8[6], v8[7]);
      if (gi == 0 || gi == N - 1 || q0 == 0 || q0 + 8 == N)
#pragma unroll
        for (int q = 0; q < 8; q++)
          ghosts_homog<2, float> (out, g, gi, q0 + q, 0, v8[q], bc);
    }
  }
}

/* FP64 shared-memory accesses by 32-bit byte address plus a constant
   offset */
template <int OFF>
__device__ __forceinline__ double2 lds_d2 (unsigned a)
{
  double2 v;
  asm volatile ("ld.shared.v2.f64 {%0, %1}, [%2+%3];" : "=d"(v.x), "=d"(v.y) : "r"(a), "n"(OFF));
  return v;
}

template <int OFF>
__device__ __forceinline__ double lds_d1 (unsigned a)
{
  double v;
  asm volatile ("ld.shared.f64 %0, [%1+%2];" : "=d"(v) : "r"(a), "n"(OFF));
  return v;
}

__device__ __forceinline__ void sts_d2 (unsigned a, double2 v)
{
  asm volatile ("st.shared.v2.f64 [%0], {%1, %2};" :: "r"(a), "d"(v.x), "d"(v.y) : "memory");
}

__device__ __forceinline__ void sts_d1 (unsigned a, double v)
{
  asm volatile ("st.shared.f64 [%0], %1;" :: "r"(a), "d"(v) : "memory");
}

/* The plain FP64 form of k_relax_tile2d_w on large levels: the same
   temporal blocking (48^2 tiles staged with an 8-cell halo, only the
   iterate in shared memory, 32 KB), with four cells per thread (two of
   each colour, 16 x 64 threads) whose exact coefficients and -Delta^2 b
   stay in registers for the launch, and every update in relax_value's
   expression and order with the IEEE division, so that the result is
   bit-identical to the reference's red-black sequence (and to
   k_relax_tile2d).  Four cells per thread keep the coefficients within 64
   registers, so an SM holds 32 warps to cover the latency of the dependent
   FP64 chains (eight cells per thread at 128 registers held 16 and were
   14 % slower per launch). */
namespace tx4 {
constexpr int W = 64, M = W/2, WM = W*M, BX = 16, BY = 64;
static_assert (W == 4*BX && BY == W, "one row of four cells per thread");
}

template <int TS, bool LAM>
__global__ void __launch_bounds__ (tx4::BX*tx4::BY, 1)
k_relax_tile2d_x4 (bmg_geom g, double * __restrict__ out, const double * __restrict__ in,
                   const double * __restrict__ res, Coef<double> ax, Coef<double> ay, Coef<double> lam,
                   double Delta, BCH bc, int nsweeps, double * __restrict__ acor, bmg_bcdesc abc,
                   const double * __restrict__ coarse, bmg_geom gc)
{
  using namespace tx4;
  constexpr int H = (W - TS)/2;
  __shared__ __align__ (16) double sa[2*WM];
  const int n = g.n, tx = threadIdx.x, ty = threadIdx.y, tid = ty*BX + tx, nth = BX*BY;
  constexpr int RW = 32/BX;
  const int p = 2*RW*(ty/(2*RW)) + 2*(ty % RW) + ((ty/RW) & 1);
  const int i0 = blockIdx.y*TS - H, j0 = blockIdx.x*TS - H;
  const int px = bc.periodic[0], py = bc.periodic[1];
  const int base = (i0 + j0) & 1;
  const bool inner = i0 >= 0 && i0 + W <= n && j0 >= 0 && j0 + W <= n;
  const int q0 = 4*tx, m0 = 2*tx, gi = i0 + p;
  const double D2 = Delta*Delta;
  grid_dependents_launch ();

  double r4[4], xl4[4], xu4[4], yl4[5], l4[4];
  if (inner) {
    const long long id = cidx<2> (g, gi, j0 + q0, 0);
    const Quad<double> r0 = load_quad (res + id);
    r4[0] = r0.x; r4[1] = r0.y; r4[2] = r0.z; r4[3] = r0.w;
    if (ax.p) {
      const Quad<double> a0 = load_quad (ax.p + id), b0 = load_quad (ax.p + id + g.P);
      xl4[0] = a0.x; xl4[1] = a0.y; xl4[2] = a0.z; xl4[3] = a0.w;
      xu4[0] = b0.x; xu4[1] = b0.y; xu4[2] = b0.z; xu4[3] = b0.w;
    }
    else
#pragma unroll
      for (int q = 0; q < 4; q++) xl4[q] = xu4[q] = ax.c;
    if (ay.p) {
      const Quad<double> a0 = load_quad (ay.p + id);
      yl4[0] = a0.x; yl4[1] = a0.y; yl4[2] = a0.z; yl4[3] = a0.w;
      yl4[4] = ay.p[id + 4];
    }
    else
#pragma unroll
      for (int q = 0; q < 5; q++) yl4[q] = ay.c;
    if (LAM) {
      const Quad<double> a0 = load_quad (lam.p + id);
      l4[0] = a0.x; l4[1] = a0.y; l4[2] = a0.z; l4[3] = a0.w;
    }
  }
  else {
    const int ri = real_index (gi, n, px);
    const int flo = real_face (gi, n, px), fhi = real_face (gi + 1, n, px);
#pragma unroll
    for (int q = 0; q < 5; q++) {
      const int rj = real_index (j0 + q0 + q, n, py), fj = real_face (j0 + q0 + q, n, py);
      yl4[q] = ri >= 0 && fj >= 0 ? ay.at (cidx<2> (g, ri, fj, 0)) : 0.;
      if (q == 4) break;
      const bool ok = ri >= 0 && rj >= 0;
      r4[q] = ok ? res[cidx<2> (g, ri, rj, 0)] : 0.;
      xl4[q] = flo >= 0 && rj >= 0 ? ax.at (cidx<2> (g, flo, rj, 0)) : 0.;
      xu4[q] = fhi >= 0 && rj >= 0 ? ax.at (cidx<2> (g, fhi, rj, 0)) : 0.;
      if (LAM) l4[q] = ok ? lam.p[cidx<2> (g, ri, rj, 0)] : 0.;
    }
  }
  grid_dependency_wait ();
  const int cq = (base + p) & 1;
  if (coarse) {
    /* the level's first launch: the iterate is the prolongation of the
       coarse level (bit-identical to the prolongation launch) */
    if (inner) {
      double v4[4];
      prolong_row<double, 4> (coarse, gc, gi, j0 + q0, v4);
      const Quad<double> va = {v4[0], v4[1], v4[2], v4[3]};
      put_quad (sa + cq*WM, sa + (cq ^ 1)*WM, p*M + m0, va);
    }
    else {
      const int ri = real_index (gi, n, px);
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int rj = real_index (j0 + q0 + q, n, py);
        sa[((cq + q) & 1)*WM + p*M + ((q0 + q) >> 1)] =
          ri >= 0 && rj >= 0 ? prolong_cell<double> (coarse, gc, ri, rj) : 0.;
      }
    }
  }
  else if (inner) {
    const long long id = cidx<2> (g, gi, j0 + q0, 0);
    const Quad<double> va = load_quad (in + id);
    put_quad (sa + cq*WM, sa + (cq ^ 1)*WM, p*M + m0, va);
  }
  else {
    const int ri = real_index (gi, n, px);
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int rj = real_index (j0 + q0 + q, n, py);
      sa[((cq + q) & 1)*WM + p*M + ((q0 + q) >> 1)] =
        ri >= 0 && rj >= 0 ? in[cidx<2> (g, ri, rj, 0)] : 0.;
    }
  }
  double cxl[2][2], cxu[2][2], cyl[2][2], cyr[2][2], cnb[2][2], cdl[2][LAM ? 2 : 1];
  const double dlc = (-lam.c)*D2;
  unsigned valid = 0;
  const bool rowok = px || (unsigned) gi < (unsigned) n;
#pragma unroll
  for (int c = 0; c < 2; c++)
#pragma unroll
    for (int e = 0; e < 2; e++) {
      const bool odd = (c ^ base ^ p) & 1;
      const int q = 2*e + (odd ? 1 : 0);
      const double xl = odd ? xl4[2*e + 1] : xl4[2*e], xu = odd ? xu4[2*e + 1] : xu4[2*e];
      const double yl = odd ? yl4[2*e + 1] : yl4[2*e], yr = odd ? yl4[2*e + 2] : yl4[2*e + 1];
      const double rv = odd ? r4[2*e + 1] : r4[2*e];
      const double lv = LAM ? (odd ? l4[2*e + 1] : l4[2*e]) : lam.c;
      const bool ok = rowok && (py || (unsigned) (j0 + q0 + q) < (unsigned) n);
      cxl[c][e] = xl; cxu[c][e] = xu; cyl[c][e] = yl; cyr[c][e] = yr;
      cnb[c][e] = (-D2)*rv;
      if (LAM) cdl[c][LAM ? e : 0] = (-lv)*D2;
      valid |= (ok ? 1u : 0u) << (2*c + e);
    }

  __syncthreads ();

  const int glo_i = px ? -1 : -1 - i0, ghi_i = px ? -1 : n - i0;
  const int glo_j = py ? -1 : -1 - j0, ghi_j = py ? -1 : n - j0;
  const bool has_ghosts = !inner &&
    ((glo_i >= 0 && glo_i < W) || (ghi_i >= 0 && ghi_i < W) ||
     (glo_j >= 0 && glo_j < W) || (ghi_j >= 0 && ghi_j < W));
  auto refresh = [&] () {
    for (int t = tid; t < 4*W; t += nth) {
      const int line = t/W, u = t - line*W;
      int pp, q, pm, qm, f;
      if (line == 0) { pp = glo_i; q = u; pm = pp + 1; qm = q; f = bc.fac[1]; }
      else if (line == 1) { pp = ghi_i; q = u; pm = pp - 1; qm = q; f = bc.fac[0]; }
      else if (line == 2) { pp = u; q = glo_j; pm = pp; qm = q + 1; f = bc.fac[3]; }
      else { pp = u; q = ghi_j; pm = pp; qm = q - 1; f = bc.fac[2]; }
      if (pp < 0 || pp >= W || q < 0 || q >= W || pm < 0 || pm >= W || qm < 0 || qm >= W)
        continue;
      if (line < 2 ? real_index (j0 + q, n, py) < 0 : real_index (i0 + pp, n, px) < 0)
        continue;
      const int c = (base + pp + q) & 1;
      sa[c*WM + pp*M + (q >> 1)] = sa[(c ^ 1)*WM + pm*M + (qm >> 1)]*double(f);
    }
  };
  if (has_ghosts) {
    refresh ();
    __syncthreads ();
  }

  const unsigned sbase = (unsigned) __cvta_generic_to_shared (sa);
  const int o0 = (base ^ p) & 1;
  for (int sw = 0; sw < nsweeps; sw++)
#pragma unroll
    for (int c = 0; c < 2; c++) {
      const int k = 2*sw + c;
      if (p >= k + 1 && p < W - k - 1) {
        const int o = o0 ^ c;
        /* the other colour's pair at rows p - 1, p, p + 1 and its left or
           right neighbour in row p */
        const unsigned aup = sbase + 8u*((c ^ 1)*WM + (p - 1)*M + m0);
        const double2 u0 = lds_d2<0> (aup), m0v = lds_d2<8*M> (aup), d0 = lds_d2<16*M> (aup);
        double v[3];
        if (o == 0) { v[0] = lds_d1<8*M - 8> (aup); v[1] = m0v.x; v[2] = m0v.y; }
        else { v[0] = m0v.x; v[1] = m0v.y; v[2] = lds_d1<8*M + 16> (aup); }
        const double upv[2] = {u0.x, u0.y}, dnv[2] = {d0.x, d0.y};
        double nv[2];
#pragma unroll
        for (int e = 0; e < 2; e++) {
          /* relax_value's expression and order (poisson.h:303-319) */
          double d = LAM ? cdl[c][LAM ? e : 0] : dlc;
          d += cxu[c][e] + cxl[c][e];
          d += cyr[c][e] + cyl[c][e];
          double nn = cnb[c][e] + (cxu[c][e]*dnv[e] + cxl[c][e]*upv[e]);
          nn = nn + (cyr[c][e]*v[e + 1] + cyl[c][e]*v[e]);
          nv[e] = nn/d;
        }
        const unsigned aw = sbase + 8u*(c*WM + p*M + m0);
        const unsigned vc = (valid >> (2*c)) & 3u;
        if (vc == 3u)
          sts_d2 (aw, make_double2 (nv[0], nv[1]));
        else {
          if (vc & 1u) sts_d1 (aw, nv[0]);
          if (vc & 2u) sts_d1 (aw + 8, nv[1]);
        }
      }
      __syncthreads ();
      if (has_ghosts) {
        refresh ();
        __syncthreads ();
      }
    }

  /* (and a += da on the cycle's last launch of the finest level, as in
     k_relax_tile2d_w) */
  if (inner) {
    constexpr int QT = TS/4;
    for (int idx = tid; idx < TS*QT; idx += nth) {
      const int rr = idx/QT, k = idx - rr*QT;
      const int pp = rr + H, q = H + 4*k, c0 = (base + pp + q) & 1, m = q >> 1;
      Quad<double> v;
      v.x = sa[c0*WM + pp*M + m]; v.z = sa[c0*WM + pp*M + m + 1];
      v.y = sa[(c0 ^ 1)*WM + pp*M + m]; v.w = sa[(c0 ^ 1)*WM + pp*M + m + 1];
      const long long id = cidx<2> (g, blockIdx.y*TS + rr, blockIdx.x*TS + 4*k, 0);
      store_quad (out + id, v);
      if (acor) {
        Quad<double> av = load_quad (acor + id);
        av.x = av.x + v.x; av.y = av.y + v.y; av.z = av.z + v.z; av.w = av.w + v.w;
        store_quad (acor + id, av);
      }
    }
    return;
  }
  for (int idx = tid; idx < TS*TS; idx += nth) {
    const int rr = idx/TS, s = idx - rr*TS;
    const int oi = blockIdx.y*TS + rr, oj = blockIdx.x*TS + s;
    if (oi >= n || oj >= n) continue;
    const int pp = rr + H, q = s + H;
    const double v = sa[((base + pp + q) & 1)*WM + pp*M + (q >> 1)];
    const long long id = cidx<2> (g, oi, oj, 0);
    out[id] = v;
    ghosts_homog<2, double> (out, g, oi, oj, 0, v, bc);
    if (acor) {
      const double an = acor[id] + v;
      acor[id] = an;
      ghosts_inhomog<2> (acor, g, oi, oj, 0, an, abc);
    }
  }
}

/* The plain FP64 form of k_level_cluster, for the 64^2 and 128^2 levels:
   the same strips, exchanges and barriers, eight cells per thread (four
   of each colour) whose exact coefficients and -Delta^2 b stay in
   registers, and every update in relax_value's expression and order with
   the IEEE division (as k_relax_tile2d_x4), so that the result is
   bit-identical to the single-CTA bottom and the tile launches it
   replaces; the fused prolongation is bilinear's expression in FP64. */
namespace clx {
template <int N, int C> struct Shape {
  static constexpr int R = N/C, H = 8, S = 4;
  static constexpr int BYR = R + 2*H, BX = N/8, NT = BX*BYR, RW = 32/BX;
  static constexpr int OFS = 4, MP = N/2 + 8;
  static constexpr int SAW = BYR*MP, OWW = R*MP;
  static constexpr size_t bytes = sizeof (double)*(2*SAW + 4*OWW);
  static_assert (R >= H && 32 % BX == 0 && BYR % (2*RW) == 0 && NT <= 1024, "cluster level shape");
};
}

template <int N, int C, bool LAM>
__global__ void __launch_bounds__ (clx::Shape<N, C>::NT, 1)
k_level_cluster_x (bmg_geom g, double * __restrict__ out, const double * __restrict__ res,
                   Coef<double> ax, Coef<double> ay, Coef<double> lam, double Delta, BCH bc,
                   int nrelax, bmg_geom gc, const double * __restrict__ coarse)
{
  typedef clx::Shape<N, C> Sh;
  constexpr int R = Sh::R, H = Sh::H, S = Sh::S, BYR = Sh::BYR, BX = Sh::BX, RW = Sh::RW;
  constexpr int OFS = Sh::OFS, MP = Sh::MP, SAW = Sh::SAW, OWW = Sh::OWW;
  extern __shared__ __align__ (16) double xsm[];
  double * sa = xsm, * own = xsm + 2*SAW;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int p = 2*RW*(ty/(2*RW)) + 2*(ty % RW) + ((ty/RW) & 1);
  const int rank = (int) cluster_rank ();
  const int px = bc.periodic[0], py = bc.periodic[1];
  const int gi = rank*R - H + p, ri = real_index (gi, N, px);
  const bool rowok = ri >= 0;
  const int ce = gi & 1, q0 = 8*tx, m0 = 4*tx;
  const double D2 = Delta*Delta;
  pdl_trigger ();

  /* the exact coefficients of the thread's eight cells */
  double cxl[2][4], cxu[2][4], cyl[2][4], cyr[2][4], cnb[2][4], cdl[2][LAM ? 4 : 1];
  {
    double r8[8], xl8[8], xu8[8], yl8[9], l8[8];
#pragma unroll
    for (int q = 0; q < 8; q++) { r8[q] = xl8[q] = xu8[q] = yl8[q] = l8[q] = 0.; }
    yl8[8] = 0.;
    if (rowok) {
      const int flo = real_face (gi, N, px), fhi = real_face (gi + 1, N, px);
      const long long id = cidx<2> (g, ri, q0, 0);
      const Quad<double> r0 = load_quad (res + id), r1 = load_quad (res + id + 4);
      r8[0] = r0.x; r8[1] = r0.y; r8[2] = r0.z; r8[3] = r0.w;
      r8[4] = r1.x; r8[5] = r1.y; r8[6] = r1.z; r8[7] = r1.w;
      if (ax.p) {
        const long long il = cidx<2> (g, flo, q0, 0), iu = cidx<2> (g, fhi, q0, 0);
        const Quad<double> a0 = load_quad (ax.p + il), a1 = load_quad (ax.p + il + 4);
        const Quad<double> b0 = load_quad (ax.p + iu), b1 = load_quad (ax.p + iu + 4);
        xl8[0] = a0.x; xl8[1] = a0.y; xl8[2] = a0.z; xl8[3] = a0.w;
        xl8[4] = a1.x; xl8[5] = a1.y; xl8[6] = a1.z; xl8[7] = a1.w;
        xu8[0] = b0.x; xu8[1] = b0.y; xu8[2] = b0.z; xu8[3] = b0.w;
        xu8[4] = b1.x; xu8[5] = b1.y; xu8[6] = b1.z; xu8[7] = b1.w;
      }
      else
#pragma unroll
        for (int q = 0; q < 8; q++) xl8[q] = xu8[q] = ax.c;
      if (ay.p) {
        const Quad<double> a0 = load_quad (ay.p + id), a1 = load_quad (ay.p + id + 4);
        yl8[0] = a0.x; yl8[1] = a0.y; yl8[2] = a0.z; yl8[3] = a0.w;
        yl8[4] = a1.x; yl8[5] = a1.y; yl8[6] = a1.z; yl8[7] = a1.w;
        yl8[8] = ay.p[cidx<2> (g, ri, real_face (q0 + 8, N, py), 0)];
      }
      else
#pragma unroll
        for (int q = 0; q < 9; q++) yl8[q] = ay.c;
      if (LAM) {
        const Quad<double> a0 = load_quad (lam.p + id), a1 = load_quad (lam.p + id + 4);
        l8[0] = a0.x; l8[1] = a0.y; l8[2] = a0.z; l8[3] = a0.w;
        l8[4] = a1.x; l8[5] = a1.y; l8[6] = a1.z; l8[7] = a1.w;
      }
    }
#pragma unroll
    for (int c = 0; c < 2; c++)
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const bool odd = (c ^ ce) & 1;
        cxl[c][e] = odd ? xl8[2*e + 1] : xl8[2*e]; cxu[c][e] = odd ? xu8[2*e + 1] : xu8[2*e];
        cyl[c][e] = odd ? yl8[2*e + 1] : yl8[2*e]; cyr[c][e] = odd ? yl8[2*e + 2] : yl8[2*e + 1];
        cnb[c][e] = (-D2)*(odd ? r8[2*e + 1] : r8[2*e]);
        if (LAM) cdl[c][LAM ? e : 0] = (-(odd ? l8[2*e + 1] : l8[2*e]))*D2;
      }
  }
  const double dlc = (-lam.c)*D2;

  const bool rowghost_lo = !px && gi == 0 && p >= 1, rowghost_hi = !px && gi == N - 1 && p <= BYR - 2;
  const double frow = rowghost_lo ? (double) bc.fac[1] : (double) bc.fac[0];
  const double fbot = (double) bc.fac[3], ftop = (double) bc.fac[2];
  const bool first_col = tx == 0, last_col = tx == BX - 1;
  auto put_ghosts = [&] (int c, const double * nv) {
    if (rowghost_lo || rowghost_hi) {
      double * gr = sa + (c ^ 1)*SAW + (rowghost_lo ? p - 1 : p + 1)*MP + OFS + m0;
#pragma unroll
      for (int e = 0; e < 4; e++) gr[e] = nv[e]*frow;
    }
    const int o = c ^ ce;
    if (first_col && o == 0) {
      if (py) sa[c*SAW + p*MP + OFS + N/2] = nv[0];
      else sa[(c ^ 1)*SAW + p*MP + OFS - 1] = nv[0]*fbot;
    }
    if (last_col && o == 1) {
      if (py) sa[c*SAW + p*MP + OFS - 1] = nv[3];
      else sa[(c ^ 1)*SAW + p*MP + OFS + N/2] = nv[3]*ftop;
    }
  };
  auto stage_ghosts = [&] () {
    if (!rowok) return;
    const int c0 = ce, cl = ce ^ 1;
    if (first_col) {
      const double v = sa[c0*SAW + p*MP + OFS];
      if (py) sa[c0*SAW + p*MP + OFS + N/2] = v;
      else sa[(c0 ^ 1)*SAW + p*MP + OFS - 1] = v*fbot;
    }
    if (last_col) {
      const double v = sa[cl*SAW + p*MP + OFS + N/2 - 1];
      if (py) sa[cl*SAW + p*MP + OFS - 1] = v;
      else sa[(cl ^ 1)*SAW + p*MP + OFS + N/2] = v*ftop;
    }
    if (rowghost_lo || rowghost_hi) {
      const int pg = rowghost_lo ? p - 1 : p + 1;
#pragma unroll
      for (int c = 0; c < 2; c++)
#pragma unroll
        for (int e = 0; e < 4; e++)
          sa[(c ^ 1)*SAW + pg*MP + OFS + m0 + e] = sa[c*SAW + p*MP + OFS + m0 + e]*frow;
    }
  };

  const unsigned sbase = (unsigned) __cvta_generic_to_shared (sa);
  const int nblk = (nrelax + S - 1)/S;
  const int up = rank > 0 ? rank - 1 : (px ? C - 1 : -1);
  const int dn = rank < C - 1 ? rank + 1 : (px ? 0 : -1);
  grid_dependency_wait ();

  for (int blk = 0; blk < nblk; blk++) {
    const int ks = nrelax - blk*S < S ? nrelax - blk*S : S;
    if (blk == 0) {
      double v8[8];
      if (rowok) {
        const int ci = ri >> 1, cx = (ri & 1) ? 1 : -1, cj0 = (q0 >> 1) - 1;
        const long long b0 = cidx<2> (gc, ci, cj0, 0), b1 = cidx<2> (gc, ci + cx, cj0, 0);
        double r0[6], r1[6];
#pragma unroll
        for (int u = 0; u < 6; u++) { r0[u] = coarse[b0 + u]; r1[u] = coarse[b1 + u]; }
#pragma unroll
        for (int q = 0; q < 8; q++) {
          const int u = 1 + (q >> 1), cy = (q & 1) ? 1 : -1;
          v8[q] = (9.*r0[u] + 3.*(r1[u] + r0[u + cy]) + r1[u + cy])/16.;
        }
      }
      else
#pragma unroll
        for (int q = 0; q < 8; q++) v8[q] = 0.;
      double * se = sa + ce*SAW + p*MP + OFS + m0, * so = sa + (ce ^ 1)*SAW + p*MP + OFS + m0;
      *(double2 *) se = make_double2 (v8[0], v8[2]); *(double2 *) (se + 2) = make_double2 (v8[4], v8[6]);
      *(double2 *) so = make_double2 (v8[1], v8[3]); *(double2 *) (so + 2) = make_double2 (v8[5], v8[7]);
    }
    else {
      const int src = (blk - 1) & 1;
      int u = rank, r = p - H;
      if (p < H) { u = up; r = R - H + p; }
      else if (p >= H + R) { u = dn; r = p - H - R; }
      const double * ob = own + src*2*OWW;
      const double * q = u < 0 ? NULL : (u == rank ? ob : cluster_map (ob, (unsigned) u));
#pragma unroll
      for (int c = 0; c < 2; c++) {
        double2 v0 = make_double2 (0., 0.), v1 = v0;
        if (q) {
          v0 = *(const double2 *) (q + c*OWW + r*MP + OFS + m0);
          v1 = *(const double2 *) (q + c*OWW + r*MP + OFS + m0 + 2);
        }
        *(double2 *) (sa + c*SAW + p*MP + OFS + m0) = v0;
        *(double2 *) (sa + c*SAW + p*MP + OFS + m0 + 2) = v1;
      }
    }
    __syncthreads ();
    stage_ghosts ();
    __syncthreads ();

    for (int sw = 0; sw < ks; sw++)
#pragma unroll
      for (int c = 0; c < 2; c++) {
        const int k = 2*sw + c;
        if (rowok && p >= k + 1 && p < BYR - k - 1) {
          const int o = c ^ ce;
          const unsigned aup = sbase + 8u*((c ^ 1)*SAW + (p - 1)*MP + OFS + m0);
          const double2 u0 = lds_d2<0> (aup), u1 = lds_d2<16> (aup);
          const double2 mA = lds_d2<8*MP> (aup), mB = lds_d2<8*MP + 16> (aup);
          const double2 d0 = lds_d2<16*MP> (aup), d1 = lds_d2<16*MP + 16> (aup);
          double v[5];
          if (o == 0) { v[0] = lds_d1<8*MP - 8> (aup); v[1] = mA.x; v[2] = mA.y; v[3] = mB.x; v[4] = mB.y; }
          else { v[0] = mA.x; v[1] = mA.y; v[2] = mB.x; v[3] = mB.y; v[4] = lds_d1<8*MP + 32> (aup); }
          const double upv[4] = {u0.x, u0.y, u1.x, u1.y}, dnv[4] = {d0.x, d0.y, d1.x, d1.y};
          double nv[4];
#pragma unroll
          for (int e = 0; e < 4; e++) {
            /* relax_value's expression and order (poisson.h:303-319) */
            double d = LAM ? cdl[c][LAM ? e : 0] : dlc;
            d += cxu[c][e] + cxl[c][e];
            d += cyr[c][e] + cyl[c][e];
            double nn = cnb[c][e] + (cxu[c][e]*dnv[e] + cxl[c][e]*upv[e]);
            nn = nn + (cyr[c][e]*v[e + 1] + cyl[c][e]*v[e]);
            nv[e] = nn/d;
          }
          const unsigned aw = sbase + 8u*(c*SAW + p*MP + OFS + m0);
          sts_d2 (aw, make_double2 (nv[0], nv[1]));
          sts_d2 (aw + 16, make_double2 (nv[2], nv[3]));
          put_ghosts (c, nv);
        }
        __syncthreads ();
      }
    if (p >= H && p < H + R) {
      double * ob = own + (blk & 1)*2*OWW;
#pragma unroll
      for (int c = 0; c < 2; c++) {
        *(double2 *) (ob + c*OWW + (p - H)*MP + OFS + m0) =
          *(const double2 *) (sa + c*SAW + p*MP + OFS + m0);
        *(double2 *) (ob + c*OWW + (p - H)*MP + OFS + m0 + 2) =
          *(const double2 *) (sa + c*SAW + p*MP + OFS + m0 + 2);
      }
    }
    cluster_barrier ();
  }

  if (p >= H && p < H + R) {
    const double * se = sa + ce*SAW + p*MP + OFS + m0, * so = sa + (ce ^ 1)*SAW + p*MP + OFS + m0;
    const double v8[8] = {se[0], so[0], se[1], so[1], se[2], so[2], se[3], so[3]};
    double * o8 = out + cidx<2> (g, gi, q0, 0);
    *(double2 *) o8 = make_double2 (v8[0], v8[1]); *(double2 *) (o8 + 2) = make_double2 (v8[2], v8[3]);
    *(double2 *) (o8 + 4) = make_double2 (v8[4], v8[5]); *(double2 *) (o8 + 6) = make_double2 (v8[6], v8[7]);
    if (gi == 0 || gi == N - 1 || q0 == 0 || q0 + 8 == N)
#pragma unroll
      for (int q = 0; q < 8; q++)
        ghosts_homog<2, double> (out, g, gi, q0 + q, 0, v8[q], bc);
  }
}

template <int N, int C, bool LAM>
int launch_level_cluster_x (bmg_geom g, double * out, const double * res, const bmg_coef * alpha,
                            bmg_coef lambda, double Delta, BCH h, int nrelax, bmg_geom gc,
                            const double * coarse, cudaStream_t s)
{
  typedef clx::Shape<N, C> Sh;
  auto kern = k_level_cluster_x<N, C, LAM>;
  static int ok[64];
  int dev = 0;
  cudaGetDevice (&dev);
  if (dev < 0 || dev >= 64) return (int) cudaErrorInvalidDevice;
  cudaLaunchConfig_t cfg;
  memset (&cfg, 0, sizeof cfg);
  cfg.gridDim = dim3 (C, 1, 1);
  cfg.blockDim = dim3 (Sh::BX, Sh::BYR, 1);
  cfg.dynamicSmemBytes = Sh::bytes;
  cfg.stream = s;
  cudaLaunchAttribute at[2];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = C; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
  at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 2;
  if (!ok[dev]) {
    cudaError_t e = cudaFuncSetAttribute (kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) Sh::bytes);
    if (e == cudaSuccess && C > 8)
      e = cudaFuncSetAttribute (kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    int nc = 0;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveClusters (&nc, kern, &cfg);
    cudaGetLastError ();
    ok[dev] = e == cudaSuccess && nc >= 1 ? 1 : -1;
  }
  if (ok[dev] < 0) return -1;
  return (int) cudaLaunchKernelEx (&cfg, kern, g, out, res, coef_of<double> (alpha[0]),
                                   coef_of<double> (alpha[1]), coef_of<double> (lambda),
                                   Delta, h, nrelax, gc, coarse);
}

template <bool LAM>
int launch_tile_x4 (bmg_geom g, void * out, const void * in, const void * res,
                    const bmg_coef * alpha, bmg_coef lambda, double Delta, BCH h, int nsweeps,
                    double * acor, const bmg_bcdesc & abc, const void * coarse, bmg_geom gc,
                    cudaStream_t s)
{
  using namespace tx4;
  constexpr int TS = 48;
  cudaLaunchConfig_t cfg;
  memset (&cfg, 0, sizeof cfg);
  cfg.gridDim = dim3 ((g.n + TS - 1)/TS, (g.n + TS - 1)/TS, 1);
  cfg.blockDim = dim3 (BX, BY, 1);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return (int) cudaLaunchKernelEx (&cfg, k_relax_tile2d_x4<TS, LAM>, g, (double *) out,
                                   (const double *) in, (const double *) res,
                                   coef_of<double> (alpha[0]), coef_of<double> (alpha[1]),
                                   coef_of<double> (lambda), Delta, h, nsweeps, acor, abc,
                                   (const double *) coarse, gc);
}


template <int TS, bool LAM>
int launch_tile_w (bmg_geom g, void * out, const void * in, const void * res,
                   const bmg_coef * alpha, bmg_coef lambda, double Delta, BCH h, int nsweeps,
                   double * acor, bmg_geom ga, const bmg_bcdesc & abc, const void * coarse,
                   bmg_geom gc, cudaStream_t s)
{
  using namespace tw;
  cudaLaunchConfig_t cfg;
  memset (&cfg, 0, sizeof cfg);
  cfg.gridDim = dim3 ((g.n + TS - 1)/TS, (g.n + TS - 1)/TS, 1);
  cfg.blockDim = dim3 (BX, BY, 1);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return (int) cudaLaunchKernelEx (&cfg, k_relax_tile2d_w<TS, LAM>, g, (float *) out, (const float *) in,
                                   (const float *) res, coef_of<float> (alpha[0]),
                                   coef_of<float> (alpha[1]), coef_of<float> (lambda),
                                   (float) Delta, h, nsweeps, acor, ga, abc,
                                   (const float *) coarse, gc);
}

/* ---------------------------------------------------------------- */
/* single-CTA bottom of the cycle                                    */
/* ---------------------------------------------------------------- */

typedef bmg_bottom_level BotLevel;

#define BOT_MAXLEVELS 14
/* threads of the bottom CTA: 512 leaves each up to 128 registers, enough
   for the register-resident weights of four cells per colour without
   spilling */
#define BOT_THREADS 512
/* levels up to this size use the small relaxation tiles */
#define BMG_SMALL_TILE_N 256
/* staged levels up to this many padded cells are relaxed by one warp */
#define BOT_WARP_CELLS 100

/* a staged level: its global arrays and their shared-memory copies, which
   use a compact padded layout described by a bmg_geom of its own (pitch
   n+2, offset 1), so relax_value and ghosts_homog apply unchanged */
struct BotStage {
  bmg_geom gs;                  /* shared-memory geometry */
  unsigned off_da, off_res, off_alpha[3], off_lambda;   /* byte offsets, ~0u = absent */
};

struct BotParams {
  BotLevel lv[BOT_MAXLEVELS];   /* levels lo..hi at indices 0..hi-lo */
  BotStage sm[BOT_MAXLEVELS];
  bmg_geom g_src;               /* level hi+1: the restricted res comes from it */
  const void * res_src;
  int st_src;
  int nlev, nrelax, restrict_src;
  BCH bc;
};

__device__ __forceinline__ void * sm_at (unsigned char * base, unsigned off)
{
  return off == ~0u ? NULL : (void *) (base + off);
}

template <int DIM>
__device__ __forceinline__ void decode_padded (long long q, int e, int & i, int & j, int & k)
{
  /* q over (n+2)^DIM positions -> (i, j, k) in [-1, n]^DIM, e = n + 2 */
  if (DIM == 1) { i = (int) q - 1; j = k = 0; }
  else if (DIM == 2) { i = (int) (q/e) - 1; j = (int) (q % e) - 1; k = 0; }
  else { i = (int) (q/((long long) e*e)) - 1; long long r = q % ((long long) e*e); j = (int) (r/e) - 1; k = (int) (r % e) - 1; }
}

/* copy every position [-1, n]^DIM of a level array between global and shared
   memory: one warp per row of the contiguous axis, no index divisions */
template <int DIM, typename T>
__device__ __forceinline__ void bot_copy (const bmg_geom & gg, T * gp, const bmg_geom & gs, T * sp,
                                          int to_shared)
{
  const int e = gs.n + 2;
  const int rows = DIM == 1 ? 1 : DIM == 2 ? e : e*e;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int r = warp; r < rows; r += nw) {
    int i, j;
    if (DIM == 1) { i = 0; j = 0; }
    else if (DIM == 2) { i = r - 1; j = 0; }
    else { i = r/e - 1; j = r - (i + 1)*e - 1; }
    for (int k = lane - 1; k < e - 1; k += 32) {
      long long gi, si;
      if (DIM == 1) { gi = cidx<1> (gg, k, 0, 0); si = cidx<1> (gs, k, 0, 0); }
      else if (DIM == 2) { gi = cidx<2> (gg, i, k, 0); si = cidx<2> (gs, i, k, 0); }
      else { gi = cidx<3> (gg, i, j, k); si = cidx<3> (gs, i, j, k); }
      if (to_shared) cp_async_elem (&sp[si], &gp[gi], true);   /* waited for by the caller */
      else gp[gi] = sp[si];
    }
  }
}

template <int DIM>
__device__ __forceinline__ void bot_copy_st (int st, const bmg_geom & gg, const void * gp, const bmg_geom & gs,
                             void * sp, int to_shared)
{
  if (st == BMG_ST_F64) bot_copy<DIM, double> (gg, (double *) gp, gs, (double *) sp, to_shared);
  else bot_copy<DIM, float> (gg, (float *) gp, gs, (float *) sp, to_shared);
}

template <typename T>
__device__ __forceinline__ T ld (const void * p, long long i) { return ((const T *) p)[i]; }

template <int DIM, typename TF, typename TC>
__device__ __forceinline__ void bot_restrict (const bmg_geom & gf, const void * f, const bmg_geom & gc, void * c)
{
  const int n = gc.n;
  const long long total = DIM == 1 ? n : DIM == 2 ? (long long) n*n : (long long) n*n*n;
  for (long long q = threadIdx.x; q < total; q += blockDim.x) {
    int i, j = 0, k = 0;
    const int ln = 31 - __clz (n), qq = (int) q;
    if (DIM == 1) i = qq;
    else if (DIM == 2) { i = qq >> ln; j = qq & (n - 1); }
    else { i = qq >> (2*ln); j = (qq >> ln) & (n - 1); k = qq & (n - 1); }
    TC sum = TC(0);
    if (DIM == 1) {
      for (int a = 0; a < 2; a++) sum += (TC) ld<TF> (f, cidx<1> (gf, 2*i + a, 0, 0));
    }
    else if (DIM == 2) {
      for (int a = 0; a < 2; a++)
        for (int b = 0; b < 2; b++)
          sum += (TC) ld<TF> (f, cidx<2> (gf, 2*i + a, 2*j + b, 0));
    }
    else {
      for (int a = 0; a < 2; a++)
        for (int b = 0; b < 2; b++)
          for (int d = 0; d < 2; d++)
            sum += (TC) ld<TF> (f, cidx<3> (gf, 2*i + a, 2*j + b, 2*k + d));
    }
    ((TC *) c)[cidx<DIM> (gc, i, j, k)] = sum/TC(1 << DIM);
  }
}

template <int DIM, typename TC, typename TF>
__device__ __forceinline__ void bot_prolong (const bmg_geom & gc, const void * cv, const bmg_geom & gf, void * fv,
                             const BCH & bc, int zero)
{
  const TC * s = (const TC *) cv;
  TF * f = (TF *) fv;
  const int n = gf.n;
  const long long total = DIM == 1 ? n : DIM == 2 ? (long long) n*n : (long long) n*n*n;
  for (long long q = threadIdx.x; q < total; q += blockDim.x) {
    int i, j = 0, k = 0;
    const int ln = 31 - __clz (n), qq = (int) q;
    if (DIM == 1) i = qq;
    else if (DIM == 2) { i = qq >> ln; j = qq & (n - 1); }
    else { i = qq >> (2*ln); j = (qq >> ln) & (n - 1); k = qq & (n - 1); }
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
}

/* ghost images of a 2D cell (homogeneous BCs) without local arrays: the
   edge images and the corner image, composed as in ghosts_homog */
template <typename T>
__device__ __forceinline__ void ghosts_homog_2d (T * f, const bmg_geom & g, int i, int j, T v,
                                                 const BCH & bc)
{
  const int n = g.n;
  if (i != 0 && i != n - 1 && j != 0 && j != n - 1) return;
  if (n == 1) { ghosts_homog<2, T> (f, g, i, j, 0, v, bc); return; }
  int gi = i, gj = j;
  T fi = T(1), fj = T(1);
  if (i == 0) { gi = bc.periodic[0] ? n : -1; fi = bc.periodic[0] ? T(1) : T(bc.fac[1]); }
  else if (i == n - 1) { gi = bc.periodic[0] ? -1 : n; fi = bc.periodic[0] ? T(1) : T(bc.fac[0]); }
  if (j == 0) { gj = bc.periodic[1] ? n : -1; fj = bc.periodic[1] ? T(1) : T(bc.fac[3]); }
  else if (j == n - 1) { gj = bc.periodic[1] ? -1 : n; fj = bc.periodic[1] ? T(1) : T(bc.fac[2]); }
  if (gi != i) f[cidx<2> (g, gi, j, 0)] = v*fi;
  if (gj != j) f[cidx<2> (g, i, gj, 0)] = v*fj;
  if (gi != i && gj != j) f[cidx<2> (g, gi, gj, 0)] = v*fi*fj;
}

/* one colour pass of red-black relaxation over a whole staged level, by
   threads [t0, t0 + nt) of the block */
template <int DIM, typename T>
__device__ __forceinline__ void bot_pass (const bmg_geom & g, void * dav, const void * resv, const void * const * al,
                          const BotLevel & L, const void * lamp, const BCH & bc, int color,
                          int t0, int nt)
{
  T * a = (T *) dav;
  const T * b = (const T *) resv;
  Coef<T> ax, ay, az, lam;
  ax.p = (const T *) al[0]; ax.c = (T) L.alpha[0].c;
  ay.p = (const T *) al[1]; ay.c = (T) L.alpha[1].c;
  az.p = (const T *) al[2]; az.c = (T) L.alpha[2].c;
  lam.p = (const T *) lamp; lam.c = (T) L.lambda.c;
  const T D2 = (T) L.Delta*(T) L.Delta;
  const int n = g.n;
  /* cells of one colour: the contiguous index runs over half the row
     (n is a power of two: shifts, no divisions) */
  const int ln = 31 - __clz (n), nh = n > 1 ? n >> 1 : 1, lh = n > 1 ? ln - 1 : 0;
  const int rows = DIM == 1 ? 1 : DIM == 2 ? n : n*n;
  const int total = rows*nh;
  for (int q = threadIdx.x - t0; q < total; q += nt) {
    const int row = q >> lh, h = q & (nh - 1);
    int i, j, k;
    if (DIM == 1) { i = 2*h + color; j = k = 0; if (i >= n) continue; }
    else if (DIM == 2) { i = row; j = 2*h + ((color + i) & 1); k = 0; if (j >= n) continue; }
    else { i = row >> ln; j = row & (n - 1); k = 2*h + ((color + i + j) & 1); if (k >= n) continue; }
    const long long id = cidx<DIM> (g, i, j, k);
    const T v = relax_value<DIM, T> (g, id, a, b, ax, ay, az, lam, D2);
    a[id] = v;
    if (DIM == 2) ghosts_homog_2d<T> (a, g, i, j, v, bc);
    else ghosts_homog<DIM, T> (a, g, i, j, k, v, bc);
  }
}

/* the 2D pass of the bottom solve with instruction-level parallelism: each
   thread first gathers the operands of up to K cells (independent loads,
   no stores in between), then divides and stores */
template <typename T, bool AST, bool LST, int K>
__device__ __forceinline__ void bot_pass2d (const bmg_geom & g, T * a, const T * b, const T * ax, const T * ay,
                            T axc, T ayc, const T * lam, T lamc, T D2, const BCH & bc,
                            int color, int nt)
{
  const int n = g.n, P = g.P;
  if (n == 1) {   /* level 0: the generic path handles its single cell */
    if (threadIdx.x == 0 && color == 0) {
      Coef<T> cx, cy, cz, cl;
      cx.p = AST ? ax : NULL; cx.c = axc; cy.p = AST ? ay : NULL; cy.c = ayc;
      cz.p = NULL; cz.c = T(0); cl.p = LST ? lam : NULL; cl.c = lamc;
      const long long id = cidx<2> (g, 0, 0, 0);
      const T v = relax_value<2, T> (g, id, a, b, cx, cy, cz, cl, D2);
      a[id] = v;
      ghosts_homog<2, T> (a, g, 0, 0, 0, v, bc);
    }
    return;
  }
  const int ln = 31 - __clz (n), lh = ln - 1, nh = n >> 1;
  const int total = n*nh;
  for (int q0 = threadIdx.x; q0 < total; q0 += nt*K) {
    T nn[K], dd[K];
    int ids[K], is[K], js[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
      const int q = q0 + k*nt;
      const int i = q >> lh, j = 2*(q & (nh - 1)) + ((color + i) & 1);
      is[k] = i; js[k] = j;
      const int id = (i + 1)*P + 1 + j;
      ids[k] = q < total ? id : -1;
      if (q < total) {
        const T ax0 = AST ? ax[id] : axc, ax1 = AST ? ax[id + P] : axc;
        const T ay0 = AST ? ay[id] : ayc, ay1 = AST ? ay[id + 1] : ayc;
        T m = (-D2)*b[id], d = (-(LST ? lam[id] : lamc))*D2;
        m += ax1*a[id + P] + ax0*a[id - P];
        d += ax1 + ax0;
        m += ay1*a[id + 1] + ay0*a[id - 1];
        d += ay1 + ay0;
        nn[k] = m; dd[k] = d;
      }
    }
#pragma unroll
    for (int k = 0; k < K; k++)
      if (ids[k] >= 0) {
        const T v = relax_div (nn[k], dd[k]);
        a[ids[k]] = v;
        ghosts_homog_2d<T> (a, g, is[k], js[k], v, bc);
      }
  }
}

template <typename T>
__device__ __forceinline__ void bot_pass2d_any (const bmg_geom & g, void * dav, const void * resv,
                                const void * const * al, const BotLevel & L, const void * lamp,
                                const BCH & bc, int color, int nt)
{
  T * a = (T *) dav;
  const T * b = (const T *) resv;
  const T * ax = (const T *) al[0], * ay = (const T *) al[1], * lam = (const T *) lamp;
  const T axc = (T) L.alpha[0].c, ayc = (T) L.alpha[1].c, lamc = (T) L.lambda.c;
  const T D2 = (T) L.Delta*(T) L.Delta;
  if ((ax == NULL) != (ay == NULL))   /* one component stored, one constant */
    bot_pass<2, T> (g, dav, resv, al, L, lamp, bc, color, 0, nt);
  else if (ax && lam) bot_pass2d<T, true, true, 1> (g, a, b, ax, ay, axc, ayc, lam, lamc, D2, bc, color, nt);
  else if (ax) bot_pass2d<T, true, false, 1> (g, a, b, ax, ay, axc, ayc, lam, lamc, D2, bc, color, nt);
  else if (lam) bot_pass2d<T, false, true, 1> (g, a, b, ax, ay, axc, ayc, lam, lamc, D2, bc, color, nt);
  else bot_pass2d<T, false, false, 1> (g, a, b, ax, ay, axc, ayc, lam, lamc, D2, bc, color, nt);
}

/* all nrelax sweeps of one 2D level, every parameter in registers (the
   per-level parameters live in the kernel's parameter space, and reading
   them inside the sweep loop costs a constant-cache miss per pass) */
template <typename T, bool AST, bool LST>
__device__ __forceinline__ void bot_sweeps2d (const bmg_geom g, T * a, const T * b, const T * ax,
                                              const T * ay, T axc, T ayc, const T * lam, T lamc,
                                              T D2, const BCH bc, int nrelax, int nt, bool small)
{
  for (int sw = 0; sw < nrelax; sw++)
    for (int color = 0; color < 2; color++) {
      bot_pass2d<T, AST, LST, 1> (g, a, b, ax, ay, axc, ayc, lam, lamc, D2, bc, color, nt);
      if (small) __syncwarp ();
      else __syncthreads ();
    }
}

/* all nrelax sweeps of one 2D level of the mixed form whose cells of one
   colour number at most K nt: each thread keeps its (up to K per colour)
   cells' coefficients in registers, divided by the diagonal once per
   level, so a pass reads only the four neighbours of each cell from shared
   memory and needs no division: a = beta + sum of w a_neighbour with
   w = alpha/d and beta = -Delta^2 b/d, the relaxation of relax_value
   (poisson.h:303-319) up to rounding.  The pass is bound by the
   shared-memory bandwidth of the one SM, which this cuts from nine operands
   per cell to four. */
__device__ __forceinline__ float fma_t (float a, float b, float c) { return fmaf (a, b, c); }
__device__ __forceinline__ double fma_t (double a, double b, double c) { return fma (a, b, c); }

template <typename T, int K, bool EXACT>
__device__ __forceinline__ void bot_sweeps2d_reg (const bmg_geom g, T * a, const T * b,
                                                  const T * ax, const T * ay, T axc,
                                                  T ayc, const T * lam, T lamc,
                                                  T D2, const BCH bc, int nrelax, int nt,
                                                  bool small)
{
  const int n = g.n, P = g.P, nh = n >> 1, total = n*nh;
  const int lh = 30 - __clz (n);              /* log2 (n) - 1 */
  int ij[2][K];                               /* i << 16 | j, or -1: no cell */
  /* the ghost images of a boundary cell (ghosts_homog_2d, with the box
     factors +-1 as signs): bits 0/1 a column / row ghost, bits 2/3 their
     signs, bits 8-15 the column offset, bits 16-31 the row offset in
     elements; 0 for an interior cell */
  int gw[2][K];
  T wx0[2][K], wx1[2][K], wy0[2][K], wy1[2][K], beta[2][K];
#pragma unroll
  for (int c = 0; c < 2; c++)
#pragma unroll
    for (int k = 0; k < K; k++) {
      const int q = threadIdx.x + k*nt;
      const int i = q >> lh, j = 2*(q & (nh - 1)) + ((c + i) & 1);
      ij[c][k] = q < total ? (i << 16) | j : -1;
      {
        int w = 0;
        if (q < total && (i == 0 || i == n - 1 || j == 0 || j == n - 1)) {
          int ro = 0, co = 0, si = 0, sj = 0;
          if (i == 0) { ro = (bc.periodic[0] ? n : -1)*P; si = bc.periodic[0] ? 0 : bc.fac[1] < 0; }
          else if (i == n - 1) { ro = (bc.periodic[0] ? -n : 1)*P; si = bc.periodic[0] ? 0 : bc.fac[0] < 0; }
          if (j == 0) { co = bc.periodic[1] ? n : -1; sj = bc.periodic[1] ? 0 : bc.fac[3] < 0; }
          else if (j == n - 1) { co = bc.periodic[1] ? -n : 1; sj = bc.periodic[1] ? 0 : bc.fac[2] < 0; }
          w = (ro << 16) | ((co & 0xff) << 8) | (si << 3) | (sj << 2) | (ro ? 2 : 0) | (co ? 1 : 0);
        }
        gw[c][k] = w;
      }
      wx0[c][k] = wx1[c][k] = wy0[c][k] = wy1[c][k] = beta[c][k] = T(0);
      if (q < total) {
        const int e = (i + 1)*P + 1 + j;
        const T x0 = ax ? ax[e] : axc, x1 = ax ? ax[e + P] : axc;
        const T y0 = ay ? ay[e] : ayc, y1 = ay ? ay[e + 1] : ayc;
        if (EXACT) {
          /* the plain form: the coefficients as they are, and -Delta^2 b */
          wx0[c][k] = x0; wx1[c][k] = x1; wy0[c][k] = y0; wy1[c][k] = y1;
          beta[c][k] = (-D2)*b[e];
        }
        else {
          T d = (-(lam ? lam[e] : lamc))*D2;
          d += x1 + x0;
          d += y1 + y0;
          const T inv = T(1)/d;
          wx0[c][k] = x0*inv; wx1[c][k] = x1*inv; wy0[c][k] = y0*inv; wy1[c][k] = y1*inv;
          beta[c][k] = ((-D2)*b[e])*inv;
        }
      }
    }
  const T dl = (-lamc)*D2;                    /* lambda constant in the exact form */
  for (int sw = 0; sw < nrelax; sw++)
#pragma unroll
    for (int c = 0; c < 2; c++) {
      T v[K];
      int e[K];
#pragma unroll
      for (int k = 0; k < K; k++) {
        const int t = ij[c][k] < 0 ? 0 : ij[c][k];
        e[k] = ((t >> 16) + 1)*P + 1 + (t & 0xffff);
        if (EXACT) {
          /* relax_value's expression and order (poisson.h:303-319) */
          T d = dl;
          d += wx1[c][k] + wx0[c][k];
          d += wy1[c][k] + wy0[c][k];
          T m = beta[c][k] + (wx1[c][k]*a[e[k] + P] + wx0[c][k]*a[e[k] - P]);
          m = m + (wy1[c][k]*a[e[k] + 1] + wy0[c][k]*a[e[k] - 1]);
          v[k] = m/d;
        }
        else
          v[k] = fma_t (wy0[c][k], a[e[k] - 1], fma_t (wy1[c][k], a[e[k] + 1],
                 fma_t (wx0[c][k], a[e[k] - P], fma_t (wx1[c][k], a[e[k] + P], beta[c][k]))));
      }
#pragma unroll
      for (int k = 0; k < K; k++)
        if (ij[c][k] >= 0) {
          a[e[k]] = v[k];
          const int w = gw[c][k];
          if (w) {
            const int ro = w >> 16, co = (signed char) ((w >> 8) & 0xff);
            const T vi = (w & 8) ? -v[k] : v[k], vj = (w & 4) ? -v[k] : v[k];
            if (w & 2) a[e[k] + ro] = vi;
            if (w & 1) a[e[k] + co] = vj;
            if ((w & 3) == 3) a[e[k] + ro + co] = (w & 4) ? -vi : vi;
          }
        }
      if (small) __syncwarp ();
      else __syncthreads ();
    }
}

template <typename T>
__device__ __forceinline__ void bot_level2d (const bmg_geom g, void * dav, const void * resv,
                                             const void * axv, const void * ayv, double axc,
                                             double ayc, const void * lamv, double lamc,
                                             double Delta, const BCH bc, int nrelax, int nt,
                                             bool small, int fast)
{
  T * a = (T *) dav;
  const T * b = (const T *) resv, * ax = (const T *) axv, * ay = (const T *) ayv,
    * lam = (const T *) lamv;
  const T D2 = (T) Delta*(T) Delta;
  /* up to four cells per colour per thread in FP32, two in FP64
     (registers); one where the level's cells of a colour fit the threads,
     so that the small levels' passes carry no empty slots */
  constexpr int K = sizeof (T) == 4 ? 4 : 2;
  if (fast && g.n >= 2 && g.n*(g.n >> 1) <= nt) {
    bot_sweeps2d_reg<T, 1, false> (g, a, b, ax, ay, (T) axc, (T) ayc, lam, (T) lamc, D2, bc, nrelax, nt, small);
    return;
  }
  if (fast && g.n >= 2 && g.n*(g.n >> 1) <= K*nt) {
    bot_sweeps2d_reg<T, K, false> (g, a, b, ax, ay, (T) axc, (T) ayc, lam, (T) lamc, D2, bc, nrelax, nt, small);
    return;
  }
  /* the plain FP64 form with lambda constant, on the levels whose cells of
     a colour fit the threads: the same register ownership with the exact
     coefficients, in the reference's evaluation order */
  if (!fast && sizeof (T) == 8 && !lam && g.n >= 2 && g.n*(g.n >> 1) <= nt) {
    bot_sweeps2d_reg<T, 1, true> (g, a, b, ax, ay, (T) axc, (T) ayc, lam, (T) lamc, D2, bc, nrelax, nt, small);
    return;
  }
  if (ax && lam)
    bot_sweeps2d<T, true, true> (g, a, b, ax, ay, (T) axc, (T) ayc, lam, (T) lamc, D2, bc, nrelax, nt, small);
  else if (ax)
    bot_sweeps2d<T, true, false> (g, a, b, ax, ay, (T) axc, (T) ayc, lam, (T) lamc, D2, bc, nrelax, nt, small);
  else if (lam)
    bot_sweeps2d<T, false, true> (g, a, b, ax, ay, (T) axc, (T) ayc, lam, (T) lamc, D2, bc, nrelax, nt, small);
  else
    bot_sweeps2d<T, false, false> (g, a, b, ax, ay, (T) axc, (T) ayc, lam, (T) lamc, D2, bc, nrelax, nt, small);
}

template <int DIM>
__device__ __forceinline__ void bot_restrict_st (int stf, const bmg_geom & gf, const void * f, int stc,
                                 const bmg_geom & gc, void * c)
{
  if (stf == BMG_ST_F64 && stc == BMG_ST_F64) bot_restrict<DIM, double, double> (gf, f, gc, c);
  else if (stf == BMG_ST_F32 && stc == BMG_ST_F32) bot_restrict<DIM, float, float> (gf, f, gc, c);
  else if (stf == BMG_ST_F32 && stc == BMG_ST_F64) bot_restrict<DIM, float, double> (gf, f, gc, c);
  else bot_restrict<DIM, double, float> (gf, f, gc, c);
}

template <int DIM>
__device__ __forceinline__ void bot_prolong_st (int stc, const bmg_geom & gc, const void * c, int stf,
                                const bmg_geom & gf, void * f, const BCH & bc, int zero)
{
  if (stc == BMG_ST_F64 && stf == BMG_ST_F64) bot_prolong<DIM, double, double> (gc, c, gf, f, bc, zero);
  else if (stc == BMG_ST_F32 && stf == BMG_ST_F32) bot_prolong<DIM, float, float> (gc, c, gf, f, bc, zero);
  else if (stc == BMG_ST_F64 && stf == BMG_ST_F32) bot_prolong<DIM, double, float> (gc, c, gf, f, bc, zero);
  else bot_prolong<DIM, float, double> (gc, c, gf, f, bc, zero);
}

template <int DIM>
__global__ void __launch_bounds__ (BOT_THREADS, 1) k_bottom (const __grid_constant__ BotParams P)
{
  extern __shared__ __align__ (16) unsigned char bsm[];
  const BCH bc = P.bc;
  pdl_wait ();
  pdl_trigger ();
  /* stage the coefficients of every level (asynchronous copies) */
  for (int m = 0; m < P.nlev; m++) {
    const BotLevel & L = P.lv[m];
    const BotStage & S = P.sm[m];
    for (int d = 0; d < DIM; d++)
      if (S.off_alpha[d] != ~0u)
        bot_copy_st<DIM> (L.st, L.g, L.alpha[d].p, S.gs, sm_at (bsm, S.off_alpha[d]), 1);
    if (S.off_lambda != ~0u)
      bot_copy_st<DIM> (L.st, L.g, L.lambda.p, S.gs, sm_at (bsm, S.off_lambda), 1);
  }
  /* res of the top staged level: restricted from level hi+1, or as given */
  const int top = P.nlev - 1;
  if (P.restrict_src)
    bot_restrict_st<DIM> (P.st_src, P.g_src, P.res_src, P.lv[top].st, P.sm[top].gs,
                          sm_at (bsm, P.sm[top].off_res));
  else
    bot_copy_st<DIM> (P.lv[top].st, P.lv[top].g, P.lv[top].res, P.sm[top].gs,
                      sm_at (bsm, P.sm[top].off_res), 1);
  cp_async_wait_all ();
  __syncthreads ();
  /* restriction down to the coarsest level (multigrid-common.h:368-404) */
  for (int m = top - 1; m >= 0; m--) {
    bot_restrict_st<DIM> (P.lv[m + 1].st, P.sm[m + 1].gs, sm_at (bsm, P.sm[m + 1].off_res),
                          P.lv[m].st, P.sm[m].gs, sm_at (bsm, P.sm[m].off_res));
    __syncthreads ();
  }
  /* coarse to fine: zero / bilinear, then nrelax red-black sweeps */
  for (int m = 0; m < P.nlev; m++) {
    const BotLevel & L = P.lv[m];
    const BotStage & S = P.sm[m];
    void * da = sm_at (bsm, S.off_da);
    if (m == 0)
      bot_prolong_st<DIM> (L.st, S.gs, NULL, L.st, S.gs, da, P.bc, 1);
    else
      bot_prolong_st<DIM> (P.lv[m - 1].st, P.sm[m - 1].gs, sm_at (bsm, P.sm[m - 1].off_da),
                           L.st, S.gs, da, P.bc, 0);
    __syncthreads ();
    const void * al[3];
    for (int d = 0; d < 3; d++) al[d] = d < DIM ? sm_at (bsm, S.off_alpha[d]) : NULL;
    const void * res = sm_at (bsm, S.off_res);
    const void * lam = sm_at (bsm, S.off_lambda);
    /* levels of at most BOT_WARP_CELLS cells are relaxed by warp 0 alone,
       with warp barriers; the other warps wait at the level's end */
    const bmg_geom gs = S.gs;
    const bool small = gs.size <= BOT_WARP_CELLS;
    const int nt = small ? 32 : blockDim.x, nrelax = P.nrelax, st = L.st;
    if (DIM == 2 && (al[0] == NULL) == (al[1] == NULL)) {
      /* x and y coefficients both stored or both constant */
      const double axc = L.alpha[0].c, ayc = L.alpha[1].c, lamc = L.lambda.c, Delta = L.Delta;
      if (!small || threadIdx.x < 32) {
        if (st == BMG_ST_F64)
          bot_level2d<double> (gs, da, res, al[0], al[1], axc, ayc, lam, lamc, Delta, bc, nrelax, nt, small, L.fast);
        else
          bot_level2d<float> (gs, da, res, al[0], al[1], axc, ayc, lam, lamc, Delta, bc, nrelax, nt, small, L.fast);
      }
    }
    else if (!small || threadIdx.x < 32)
      for (int sw = 0; sw < nrelax; sw++)
        for (int color = 0; color < 2; color++) {
          if (st == BMG_ST_F64)
            bot_pass<DIM, double> (gs, da, res, al, L, lam, bc, color, 0, nt);
          else
            bot_pass<DIM, float> (gs, da, res, al, L, lam, bc, color, 0, nt);
          if (small) __syncwarp ();
          else __syncthreads ();
        }
    if (small) __syncthreads ();
  }
  /* da of every staged level, ghosts included, back to global memory (the
     next level's prolongation reads it) */
  for (int m = 0; m < P.nlev; m++)
    bot_copy_st<DIM> (P.lv[m].st, P.lv[m].g, P.lv[m].da, P.sm[m].gs, sm_at (bsm, P.sm[m].off_da), 0);
}

/* one launch of k_level_cluster (one cluster of C CTAs); -1 when this
   device cannot schedule such a cluster (the caller then uses tile
   launches) */
template <int N, int C, int SEG, bool LAM>
int launch_level_cluster (bmg_geom g, float * out, const float * res, const bmg_coef * alpha,
                          bmg_coef lambda, double Delta, BCH h, int nrelax, bmg_geom gc,
                          const float * coarse, cudaStream_t s)
{
  typedef cl::Shape<N, C, SEG> Sh;
  auto kern = k_level_cluster<N, C, SEG, LAM>;
  static int ok[64];
  int dev = 0;
  cudaGetDevice (&dev);
  if (dev < 0 || dev >= 64) return (int) cudaErrorInvalidDevice;
  cudaLaunchConfig_t cfg;
  memset (&cfg, 0, sizeof cfg);
  cfg.gridDim = dim3 (C, 1, 1);
  cfg.blockDim = dim3 (Sh::BX, Sh::BYR, 1);
  cfg.dynamicSmemBytes = Sh::bytes;
  cfg.stream = s;
  cudaLaunchAttribute at[2];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = C; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
  at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 2;
  if (!ok[dev]) {
    cudaError_t e = cudaFuncSetAttribute (kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) Sh::bytes);
    if (e == cudaSuccess && C > 8)
      e = cudaFuncSetAttribute (kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    int nc = 0;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveClusters (&nc, kern, &cfg);
    cudaGetLastError ();
    ok[dev] = e == cudaSuccess && nc >= 1 ? 1 : -1;
  }
  if (ok[dev] < 0) return -1;
  return (int) cudaLaunchKernelEx (&cfg, kern, g, out, res, coef_of<float> (alpha[0]),
                                   coef_of<float> (alpha[1]), coef_of<float> (lambda),
                                   (float) Delta, h, nrelax, gc, coarse);
}

template <typename T, int TS, int S, bool LAM, int BX, int BY, int CPT, int MINB>
int launch_tile_v (bmg_geom g, void * out, const void * in, const void * res,
                   const bmg_coef * alpha, bmg_coef lambda, double Delta, BCH h, int nsweeps,
                   cudaStream_t s)
{
  typedef TileShape<T, TS, S> Sh;
  const size_t bytes = Sh::bytes (LAM);
  /* the shared-memory opt-in, once per device */
  static unsigned char configured[64];
  int dev = 0;
  cudaGetDevice (&dev);
  if (dev < 0 || dev >= 64) return (int) cudaErrorInvalidDevice;
  if (!configured[dev]) {
    cudaError_t e = cudaFuncSetAttribute (k_relax_tile2d<T, TS, S, LAM, BX, BY, CPT, MINB>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int) bytes);
    if (e != cudaSuccess) return (int) e;
    configured[dev] = 1;
  }
  cudaLaunchConfig_t cfg;
  memset (&cfg, 0, sizeof cfg);
  cfg.gridDim = dim3 ((g.n + TS - 1)/TS, (g.n + TS - 1)/TS, 1);
  cfg.blockDim = dim3 (BX, BY, 1);
  cfg.dynamicSmemBytes = bytes;
  cfg.stream = s;
  /* programmatic dependent launch: the kernel stages res and alpha before
     it waits for the preceding grid, which wrote the iterate it reads */
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return (int) cudaLaunchKernelEx (&cfg, k_relax_tile2d<T, TS, S, LAM, BX, BY, CPT, MINB>, g, (T *) out,
                                   (const T *) in, (const T *) res, coef_of<T> (alpha[0]),
                                   coef_of<T> (alpha[1]), coef_of<T> (lambda), (T) Delta, h,
                                   nsweeps);
}

template <typename T, int TS, int S, int BX, int BY, int CPT = 2, int MINB = 1>
int launch_tile (bmg_geom g, void * out, const void * in, const void * res,
                 const bmg_coef * alpha, bmg_coef lambda, double Delta, BCH h, int nsweeps,
                 cudaStream_t s)
{
  if (lambda.p)
    return launch_tile_v<T, TS, S, true, BX, BY, CPT, MINB> (g, out, in, res, alpha, lambda, Delta, h, nsweeps, s);
  return launch_tile_v<T, TS, S, false, BX, BY, CPT, MINB> (g, out, in, res, alpha, lambda, Delta, h, nsweeps, s);
}

} // namespace

extern "C" {

/* the FP32 level whose register-weight tiles are 32 x 32 (eight sweeps per
   launch): a latency-bound level, where halving the launches and doubling
   the CTAs outweighs the deeper halo */
#define BMG_DEEP_TILE_N 512

int bmg_tile_sweeps (int st, int n)
{
  return st == BMG_ST_F32 && n == BMG_DEEP_TILE_N ? 8 : 4;
}

int bmg_tile_corrects (int st, int n)
{
  return n > BMG_SMALL_TILE_N;
}

int bmg_tile_prolongs (int st, int n)
{
  (void) st;
  return n > BMG_SMALL_TILE_N;
}

int bmg_launch_relax_tile (int dim, int st, bmg_geom g, void * out, const void * in,
                           const void * res, const bmg_coef * alpha, bmg_coef lambda,
                           double Delta, const bmg_bcdesc * bc, int nsweeps, double * acor,
                           bmg_geom ga, const bmg_bcdesc * abc, const void * coarse, bmg_geom gc,
                           cudaStream_t s)
{
  if (dim != 2 || nsweeps < 1 || nsweeps > bmg_tile_sweeps (st, g.n)) return (int) cudaErrorInvalidValue;
  if (acor && (!abc || !bmg_tile_corrects (st, g.n))) return (int) cudaErrorInvalidValue;
  if (coarse && (!bmg_tile_prolongs (st, g.n) || 2*gc.n != g.n)) return (int) cudaErrorInvalidValue;
  BCH h = bch_of (bc);
  bmg_bcdesc abc0;
  memset (&abc0, 0, sizeof abc0);
  const bmg_bcdesc & ab = abc ? *abc : abc0;
  int e;
  /* small levels: 16 x 16 tiles (more CTAs, a shorter critical path per
     CTA); large levels: big tiles (less halo recomputation).  A deeper halo
     on the small levels (twelve sweeps per launch) measured slower: the
     redundant halo work outweighs the saved launches. */
  const bool small = g.n <= BMG_SMALL_TILE_N;
  if (st == BMG_ST_F64)
    e = small ? launch_tile<double, 16, 4, 8, 32> (g, out, in, res, alpha, lambda, Delta, h, nsweeps, s)
      : lambda.p ? launch_tile_x4<true> (g, out, in, res, alpha, lambda, Delta, h, nsweeps, acor, ab, coarse, gc, s)
      : launch_tile_x4<false> (g, out, in, res, alpha, lambda, Delta, h, nsweeps, acor, ab, coarse, gc, s);
  else
    e = small ? launch_tile<float, 16, 4, 8, 32> (g, out, in, res, alpha, lambda, Delta, h, nsweeps, s)
      : g.n == BMG_DEEP_TILE_N ?
        (lambda.p ? launch_tile_w<32, true> (g, out, in, res, alpha, lambda, Delta, h, nsweeps, acor, ga, ab, coarse, gc, s)
                  : launch_tile_w<32, false> (g, out, in, res, alpha, lambda, Delta, h, nsweeps, acor, ga, ab, coarse, gc, s))
      : lambda.p ? launch_tile_w<48, true> (g, out, in, res, alpha, lambda, Delta, h, nsweeps, acor, ga, ab, coarse, gc, s)
      : launch_tile_w<48, false> (g, out, in, res, alpha, lambda, Delta, h, nsweeps, acor, ga, ab, coarse, gc, s);
  if (e) return e;
  cudaError_t r = cudaGetLastError ();
  return r == cudaSuccess ? 0 : (int) r;
}

int bmg_level_cluster_ok (int st, int n)
{
  if (st == BMG_ST_F64) return n == 64 || n == 128;
  return n == 64 || n == 128 || n == 256;
}

int bmg_launch_level_cluster (int st, bmg_geom g, void * out, const void * res,
                              const bmg_coef * alpha, bmg_coef lambda, double Delta,
                              const bmg_bcdesc * bc, int nrelax, bmg_geom gc, const void * coarse,
                              cudaStream_t s)
{
  if (nrelax < 1 || !bmg_level_cluster_ok (st, g.n)) return -1;
  BCH h = bch_of (bc);
  if (st == BMG_ST_F64) {
    double * o = (double *) out;
    const double * r = (const double *) res, * c = (const double *) coarse;
    int e = g.n == 128 ?
      (lambda.p ? launch_level_cluster_x<128, 16, true> (g, o, r, alpha, lambda, Delta, h, nrelax, gc, c, s)
                : launch_level_cluster_x<128, 16, false> (g, o, r, alpha, lambda, Delta, h, nrelax, gc, c, s))
      : lambda.p ? launch_level_cluster_x<64, 8, true> (g, o, r, alpha, lambda, Delta, h, nrelax, gc, c, s)
      : launch_level_cluster_x<64, 8, false> (g, o, r, alpha, lambda, Delta, h, nrelax, gc, c, s);
    if (e) return e;
    cudaError_t q = cudaGetLastError ();
    return q == cudaSuccess ? 0 : (int) q;
  }
  float * o = (float *) out;
  const float * r = (const float *) res, * c = (const float *) coarse;
  int e;
  if (g.n == 256)
    e = lambda.p ? launch_level_cluster<256, 16, 2, true> (g, o, r, alpha, lambda, Delta, h, nrelax, gc, c, s)
      : launch_level_cluster<256, 16, 2, false> (g, o, r, alpha, lambda, Delta, h, nrelax, gc, c, s);
  else if (g.n == 128)
    e = lambda.p ? launch_level_cluster<128, 16, 1, true> (g, o, r, alpha, lambda, Delta, h, nrelax, gc, c, s)
      : launch_level_cluster<128, 16, 1, false> (g, o, r, alpha, lambda, Delta, h, nrelax, gc, c, s);
  else
    e = lambda.p ? launch_level_cluster<64, 8, 1, true> (g, o, r, alpha, lambda, Delta, h, nrelax, gc, c, s)
      : launch_level_cluster<64, 8, 1, false> (g, o, r, alpha, lambda, Delta, h, nrelax, gc, c, s);
  if (e) return e;
  cudaError_t q = cudaGetLastError ();
  return q == cudaSuccess ? 0 : (int) q;
}

size_t bmg_bottom_smem (int dim, const bmg_bottom_level * lv, int nlev)
{
  size_t off = 0;
  for (int m = 0; m < nlev; m++) {
    size_t cells = 1;
    for (int d = 0; d < dim; d++) cells *= (size_t) lv[m].g.n + 2;
    const size_t arr = (cells*(lv[m].st == BMG_ST_F64 ? 8 : 4) + 15)/16*16;
    int narr = 2 + (lv[m].lambda.p ? 1 : 0);
    for (int d = 0; d < dim; d++) narr += lv[m].alpha[d].p ? 1 : 0;
    off += narr*arr;
  }
  return off;
}

int bmg_launch_bottom (int dim, const bmg_bottom_level * lv, int nlev, bmg_geom g_src,
                       const void * res_src, int st_src, int restrict_src, int nrelax,
                       const bmg_bcdesc * bc, cudaStream_t s)
{
  if (nlev < 1 || nlev > BOT_MAXLEVELS) return (int) cudaErrorInvalidValue;
  const size_t bytes = bmg_bottom_smem (dim, lv, nlev);
  if (bytes > BMG_BOTTOM_SMEM) return (int) cudaErrorInvalidValue;
  BotParams P;
  memset (&P, 0, sizeof P);
  size_t off = 0;
  for (int m = 0; m < nlev; m++) {
    P.lv[m] = lv[m];
    BotStage & S = P.sm[m];
    const int n = lv[m].g.n;
    S.gs.n = n; S.gs.P = n + 2; S.gs.xo = 1;
    S.gs.plane = dim == 3 ? (long long) (n + 2)*(n + 2) : dim == 2 ? n + 2 : 1;
    size_t cells = 1;
    for (int d = 0; d < dim; d++) cells *= (size_t) n + 2;
    S.gs.size = (long long) cells;
    const size_t arr = (cells*(lv[m].st == BMG_ST_F64 ? 8 : 4) + 15)/16*16;
    S.off_da = (unsigned) off; off += arr;
    S.off_res = (unsigned) off; off += arr;
    for (int d = 0; d < 3; d++)
      if (d < dim && lv[m].alpha[d].p) { S.off_alpha[d] = (unsigned) off; off += arr; }
      else S.off_alpha[d] = ~0u;
    if (lv[m].lambda.p) { S.off_lambda = (unsigned) off; off += arr; }
    else S.off_lambda = ~0u;
  }
  P.g_src = g_src; P.res_src = res_src; P.st_src = st_src;
  P.nlev = nlev; P.nrelax = nrelax; P.restrict_src = restrict_src;
  P.bc = bch_of (bc);
  static unsigned char configured[64][3];
  int dev = 0;
  cudaGetDevice (&dev);
  if (dev < 0 || dev >= 64) return (int) cudaErrorInvalidDevice;
  if (!configured[dev][dim - 1]) {
    cudaError_t e = dim == 1 ? cudaFuncSetAttribute (k_bottom<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, BMG_BOTTOM_SMEM)
      : dim == 2 ? cudaFuncSetAttribute (k_bottom<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, BMG_BOTTOM_SMEM)
      : cudaFuncSetAttribute (k_bottom<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, BMG_BOTTOM_SMEM);
    if (e != cudaSuccess) return (int) e;
    configured[dev][dim - 1] = 1;
  }
  if (dim == 1) pdl_launch (k_bottom<1>, dim3 (1), dim3 (BOT_THREADS), bytes, s, P);
  else if (dim == 2) pdl_launch (k_bottom<2>, dim3 (1), dim3 (BOT_THREADS), bytes, s, P);
  else pdl_launch (k_bottom<3>, dim3 (1), dim3 (BOT_THREADS), bytes, s, P);
  cudaError_t r = cudaGetLastError ();
  return r == cudaSuccess ? 0 : (int) r;
}

} // extern "C"

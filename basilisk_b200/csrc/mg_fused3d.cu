/*
 * mg_fused3d.cu -- one complete red-black sweep of a 3D level in one launch.
 *
 * The one-pass kernels (k_relax in mg_kernels.cu) relax the red cells, then
 * the black cells, in two launches that each read the iterate, the
 * right-hand side and every coefficient array of the whole level: with
 * 8-byte cells in 32-byte sectors a colour pass moves the arrays of both
 * colours.  k_relax3d_rb does the sweep in one pass over the level: each
 * CTA owns a TJ x TK column of cells (the second and third indices) and
 * marches along the first index through a chunk of ZB planes, keeping a
 * ring of planes of the iterate in shared memory (the tile plus two halo
 * rings, staged from global memory one plane ahead with cp.async):
 *
 *   step x: stage plane x; relax the red cells of plane x - 1 (the tile and
 *   its first halo ring); relax the black cells of plane x - 2 (the tile)
 *   and store plane x - 2.
 *
 * Red at x - 1 reads the black cells of planes x - 2 .. x, none of which
 * the launch has updated yet; black at x - 2 reads red cells of planes
 * x - 3 .. x - 1, all updated, the first halo ring included -- the order
 * of a red pass over the whole level followed by a black pass.  Each cell
 * is updated by the expression of relax_value (poisson.h:303-319, same
 * order, same division), so the result equals the two one-pass launches
 * bit for bit, in FP64 and in FP32.  Every array is read once per sweep
 * (the halo rings from L2), the iterate written once.
 *
 * Boundaries: a box ghost of a cell is the image of that cell alone
 * (dirichlet -s[], neumann s[]), read only by that cell's own update, and
 * no cell is updated twice in a sweep, so the ghosts of the input are the
 * values both passes need; along a periodic direction the halo is staged
 * from the wrapped cells and its red cells are relaxed like the others.
 * The output gets the ghost images of its boundary cells (as k_relax
 * writes them).
 */
#include <cuda_runtime.h>
#include <stdlib.h>
#include "mg_device.cuh"

using namespace bmgd;

namespace {

/* index of a staged position along one axis: the real cell, the box ghost
   slot (-1 or n, whose input value is valid), or -2 when nothing is there
   (beyond a box ghost) */
__device__ __forceinline__ int stage_index (int gi, int n, int periodic)
{
  if (gi >= 0 && gi < n) return gi;
  if (periodic) { int r = gi % n; return r < 0 ? r + n : r; }
  return (gi == -1 || gi == n) ? gi : -2;
}

/* a position whose cell is relaxed: inside the level or wrapped */
__device__ __forceinline__ bool real_cell (int gi, int n, int periodic)
{
  return periodic || (gi >= 0 && gi < n);
}

template <typename T>
__device__ __forceinline__ void cp_async_el (T * smem, const T * gmem, bool valid)
{
  const unsigned s = (unsigned) __cvta_generic_to_shared (smem);
  const int sz = valid ? (int) sizeof (T) : 0;
  if (sizeof (T) == 8)
    asm volatile ("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" :: "r"(s), "l"(gmem), "r"(sz) : "memory");
  else
    asm volatile ("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" :: "r"(s), "l"(gmem), "r"(sz) : "memory");
}

__device__ __forceinline__ void cp_async_commit () { asm volatile ("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0 () { asm volatile ("cp.async.wait_group 0;\n" ::: "memory"); }

/* the tile: TJ x TK cells; threads own pairs (k, k + 1) of one row */
template <int TJ, int TK>
struct Sh3 {
  static constexpr int WJ = TJ + 4, WK = TK + 4;     /* staged plane: two halo rings */
  static constexpr int PL = WJ*WK;                    /* elements per staged plane */
  static constexpr int NT = TJ*TK/2;                  /* threads */
  static constexpr int RING = 5;                      /* planes x - 3 .. x + 1 */
  static constexpr int NRING = 2*(TK + 2) + 2*TJ;     /* first-ring positions */
};

/* relax_value (poisson.h:303-319) of the cell at staged position (pj, pk)
   of ring plane c (neighbour planes m below, p above), global index id */
template <typename T, int WK>
__device__ __forceinline__ T relax_cell (const T * sm, int m, int c, int p, int pj, int pk,
                                         long long id, const bmg_geom & g, const T * rhs,
                                         const Coef<T> & ax, const Coef<T> & ay,
                                         const Coef<T> & az, const Coef<T> & lam, T D2)
{
  const int o = pj*WK + pk;
  T nn = (-D2)*rhs[id], d = (-lam.at (id))*D2;
  {
    const T a1 = ax.at (id + g.plane), a0 = ax.at (id);
    nn += a1*sm[p + o] + a0*sm[m + o];
    d += a1 + a0;
  }
  {
    const T a1 = ay.at (id + g.P), a0 = ay.at (id);
    nn += a1*sm[c + o + WK] + a0*sm[c + o - WK];
    d += a1 + a0;
  }
  {
    const T a1 = az.at (id + 1), a0 = az.at (id);
    nn += a1*sm[c + o + 1] + a0*sm[c + o - 1];
    d += a1 + a0;
  }
  return nn/d;
}

template <typename T, int TJ, int TK>
__global__ void __launch_bounds__ (Sh3<TJ, TK>::NT)
k_relax3d_rb (bmg_geom g, T * __restrict__ out, const T * __restrict__ in,
              const T * __restrict__ rhs, Coef<T> ax, Coef<T> ay, Coef<T> az, Coef<T> lam,
              T Delta, BCH bc, int ZB)
{
  typedef Sh3<TJ, TK> S;
  constexpr int WJ = S::WJ, WK = S::WK, PL = S::PL, NT = S::NT, R = S::RING;
  extern __shared__ __align__ (16) unsigned char smem_raw[];
  T * const sm = (T *) smem_raw;                   /* R planes of PL */
  const int n = g.n, t = threadIdx.x;
  const int j0 = blockIdx.y*TJ, k0 = blockIdx.x*TK;
  const int i0 = blockIdx.z*ZB, i1 = min (n, i0 + ZB);
  const int px = bc.periodic[0], py = bc.periodic[1], pz = bc.periodic[2];
  const T D2 = Delta*Delta;
  /* the thread's pair: row u, cells 2q, 2q + 1 of the tile */
  const int u = t/(TK/2), q = t - u*(TK/2);
  const int pj = u + 2, pk0 = 2*q + 2;
  const int gj = j0 + u, gk = k0 + 2*q;
  /* its extra first-ring position (t < NRING): (rj, rk) staged */
  int rj = -1, rk = -1;
  if (t < S::NRING) {
    if (t < TK + 2) { rj = 1; rk = 1 + t; }
    else if (t < 2*(TK + 2)) { rj = TJ + 2; rk = 1 + t - (TK + 2); }
    else if (t < 2*(TK + 2) + TJ) { rj = 2 + t - 2*(TK + 2); rk = 1; }
    else { rj = 2 + t - 2*(TK + 2) - TJ; rk = TK + 2; }
  }
  const int rgj = j0 - 2 + rj, rgk = k0 - 2 + rk;
  const bool ring_real = t < S::NRING && real_cell (rgj, n, py) && real_cell (rgk, n, pz);
  const int rrj = stage_index (rgj, n, py), rrk = stage_index (rgk, n, pz);

  /* stage plane x of the iterate into ring slot x mod R */
  auto stage = [&] (int x) {
    const int xi = stage_index (x, n, px);
    T * dst = sm + ((x + 3*R) % R)*PL;
    for (int e = t; e < PL; e += NT) {
      const int a = e/WK, b = e - a*WK;
      const int sj = stage_index (j0 - 2 + a, n, py), sk = stage_index (k0 - 2 + b, n, pz);
      const bool ok = xi != -2 && sj != -2 && sk != -2;
      cp_async_el (dst + e, in + (ok ? cidx<3> (g, xi, sj, sk) : 0), ok);
    }
  };

  /* the window: planes i0 - 2 .. i1 + 1 */
  stage (i0 - 2);
  cp_async_commit ();
  for (int x = i0 - 2; x <= i1 + 1; x++) {
    /* plane x is in, and every thread is done with step x - 1: the slot of
       plane x - 4 (= x + 1 mod R), last read by the black pass of step
       x - 1, can take plane x + 1 */
    cp_async_wait0 ();
    __syncthreads ();
    if (x + 1 <= i1 + 1) {
      stage (x + 1);
      cp_async_commit ();
    }
    /* red cells of plane x - 1: the tile and its first ring */
    const int xr = x - 1;
    if (xr >= i0 - 1 && xr <= i1 && real_cell (xr, n, px)) {
      const int xi = stage_index (xr, n, px);
      const int c = ((xr + 3*R) % R)*PL, m = ((xr - 1 + 3*R) % R)*PL, p = ((xr + 1 + 3*R) % R)*PL;
      /* the tile cell of the pair that is red */
      const int odd = (xr + gj + gk) & 1;            /* cell 2q is black */
      const int kk = gk + odd, pk = pk0 + odd;
      if (gj < n && kk < n) {
        const long long id = cidx<3> (g, xi, gj, kk);
        sm[c + pj*WK + pk] = relax_cell<T, WK> (sm, m, c, p, pj, pk, id, g, rhs, ax, ay, az, lam, D2);
      }
      if (ring_real && ((xr + rgj + rgk) & 1) == 0) {
        const long long id = cidx<3> (g, xi, rrj, rrk);
        sm[c + rj*WK + rk] = relax_cell<T, WK> (sm, m, c, p, rj, rk, id, g, rhs, ax, ay, az, lam, D2);
      }
    }
    __syncthreads ();
    /* black cells of plane x - 2 (the tile), then the pair to the output */
    const int xb = x - 2;
    if (xb >= i0 && xb < i1) {
      const int c = ((xb + 3*R) % R)*PL, m = ((xb - 1 + 3*R) % R)*PL, p = ((xb + 1 + 3*R) % R)*PL;
      const int odd = (xb + gj + gk + 1) & 1;        /* 1: cell 2q + 1 is black */
      const int kk = gk + odd, pk = pk0 + odd;
      if (gj < n && kk < n) {
        const long long id = cidx<3> (g, xb, gj, kk);
        sm[c + pj*WK + pk] = relax_cell<T, WK> (sm, m, c, p, pj, pk, id, g, rhs, ax, ay, az, lam, D2);
      }
      if (gj < n && gk < n) {
        const T v0 = sm[c + pj*WK + pk0], v1 = sm[c + pj*WK + pk0 + 1];
        const long long id = cidx<3> (g, xb, gj, gk);
        out[id] = v0;
        out[id + 1] = v1;
        ghosts_homog<3, T> (out, g, xb, gj, gk, v0, bc);
        ghosts_homog<3, T> (out, g, xb, gj, gk + 1, v1, bc);
      }
    }
  }
}

/* ---------------------------------------------------------------- */
/* the same sweep with the coefficients staged too                   */
/* ---------------------------------------------------------------- */

/* k_relax3d_rb reads each cell's coefficients from global memory at the
   moment it relaxes the cell, so every step waits for two round trips to
   memory (one per colour pass).  k_relax3d_rbs stages them like the
   iterate, one plane ahead, with cp.async: the right-hand side, lambda and
   the y and z faces of a plane over the tile and its first halo ring (the
   cells a pass relaxes), the x faces of a plane likewise; the passes then
   read shared memory only.  Rings: the iterate of planes x - 3 .. x + 1,
   the cell coefficients of planes x - 2 .. x, the x faces of planes
   x - 2 .. x + 1.  Same arithmetic, same order: bit-identical again. */

/* a real face along an axis of n cells (faces 0..n; face n of a periodic
   direction is face 0, as the library stores it), or -1 */
__device__ __forceinline__ int face_index (int f, int n, int periodic)
{
  if (f >= 0 && f <= n) return (periodic && f == n) ? 0 : f;
  if (!periodic) return -1;
  int r = f % n;
  return r < 0 ? r + n : r;
}

/* a real cell along an axis (wrapped when periodic), or -1 */
__device__ __forceinline__ int cell_index (int gi, int n, int periodic)
{
  if (gi >= 0 && gi < n) return gi;
  if (!periodic) return -1;
  int r = gi % n;
  return r < 0 ? r + n : r;
}

template <int TJ, int TK>
struct Sh3s {
  static constexpr int WJ = TJ + 4, WK = TK + 4, PL = WJ*WK;   /* iterate plane */
  static constexpr int CJ = TJ + 2, CK = TK + 2, CP = CJ*CK;   /* cell coefficients */
  static constexpr int YP = (CJ + 1)*CK;                       /* y faces of a plane */
  static constexpr int ZK = CK + 1, ZP = CJ*ZK;                /* z faces of a plane */
  static constexpr int NT = TJ*TK/2;
  static constexpr int R = 5, RC = 3, RX = 4;
  static constexpr int NRING = 2*(TK + 2) + 2*TJ;
};

/* element offsets of the staged arrays in shared memory (0: not staged) */
struct Off3 { int b, l, x, y, z, total; };

template <typename T, int TJ, int TK>
__global__ void __launch_bounds__ (Sh3s<TJ, TK>::NT)
k_relax3d_rbs (bmg_geom g, T * __restrict__ out, const T * __restrict__ in,
               const T * __restrict__ rhs, Coef<T> ax, Coef<T> ay, Coef<T> az, Coef<T> lam,
               T Delta, BCH bc, int ZB, Off3 so)
{
  typedef Sh3s<TJ, TK> S;
  constexpr int WK = S::WK, PL = S::PL, CK = S::CK, CP = S::CP, YP = S::YP, ZK = S::ZK,
    ZP = S::ZP, NT = S::NT, R = S::R, RC = S::RC, RX = S::RX;
  extern __shared__ __align__ (16) unsigned char smem_raw[];
  T * const sm = (T *) smem_raw;
  const int n = g.n, t = threadIdx.x;
  const int j0 = blockIdx.y*TJ, k0 = blockIdx.x*TK;
  const int i0 = blockIdx.z*ZB, i1 = min (n, i0 + ZB);
  const int px = bc.periodic[0], py = bc.periodic[1], pz = bc.periodic[2];
  const T D2 = Delta*Delta;
  const bool sx = ax.p, sy = ay.p, sz = az.p, sl = lam.p;
  const int u = t/(TK/2), q = t - u*(TK/2);
  const int pj = u + 2, pk0 = 2*q + 2;
  const int gj = j0 + u, gk = k0 + 2*q;
  int rj = -1, rk = -1;
  if (t < S::NRING) {
    if (t < TK + 2) { rj = 1; rk = 1 + t; }
    else if (t < 2*(TK + 2)) { rj = TJ + 2; rk = 1 + t - (TK + 2); }
    else if (t < 2*(TK + 2) + TJ) { rj = 2 + t - 2*(TK + 2); rk = 1; }
    else { rj = 2 + t - 2*(TK + 2) - TJ; rk = TK + 2; }
  }
  const int rgj = j0 - 2 + rj, rgk = k0 - 2 + rk;
  const bool ring_real = t < S::NRING && real_cell (rgj, n, py) && real_cell (rgk, n, pz);

  /* ring slots (x >= -2) */
  auto slot = [] (int x, int r) { return (x + 4*r) % r; };

  /* stage the iterate of plane x */
  auto stage_a = [&] (int x) {
    const int xi = stage_index (x, n, px);
    T * dst = sm + slot (x, R)*PL;
    for (int e = t; e < PL; e += NT) {
      const int a = e/WK, b = e - a*WK;
      const int sj = stage_index (j0 - 2 + a, n, py), sk = stage_index (k0 - 2 + b, n, pz);
      const bool ok = xi != -2 && sj != -2 && sk != -2;
      cp_async_el (dst + e, in + (ok ? cidx<3> (g, xi, sj, sk) : 0), ok);
    }
  };
  /* stage the cell coefficients (rhs, lambda, y and z faces) of plane x:
     region rows j0 - 1 .. j0 + TJ, columns k0 - 1 .. k0 + TK */
  auto stage_c = [&] (int x) {
    const int xi = cell_index (x, n, px);
    const int sc = slot (x, RC);
    for (int e = t; e < CP; e += NT) {
      const int a = e/CK, b = e - a*CK;
      const int cj = cell_index (j0 - 1 + a, n, py), ck = cell_index (k0 - 1 + b, n, pz);
      const bool ok = xi >= 0 && cj >= 0 && ck >= 0;
      const long long id = ok ? cidx<3> (g, xi, cj, ck) : 0;
      cp_async_el (sm + so.b + sc*CP + e, rhs + id, ok);
      if (sl) cp_async_el (sm + so.l + sc*CP + e, lam.p + id, ok);
    }
    if (sy)
      for (int e = t; e < YP; e += NT) {
        const int a = e/CK, b = e - a*CK;
        const int fj = face_index (j0 - 1 + a, n, py), ck = cell_index (k0 - 1 + b, n, pz);
        const bool ok = xi >= 0 && fj >= 0 && ck >= 0;
        cp_async_el (sm + so.y + sc*YP + e, ay.p + (ok ? cidx<3> (g, xi, fj, ck) : 0), ok);
      }
    if (sz)
      for (int e = t; e < ZP; e += NT) {
        const int a = e/ZK, b = e - a*ZK;
        const int cj = cell_index (j0 - 1 + a, n, py), fk = face_index (k0 - 1 + b, n, pz);
        const bool ok = xi >= 0 && cj >= 0 && fk >= 0;
        cp_async_el (sm + so.z + sc*ZP + e, az.p + (ok ? cidx<3> (g, xi, cj, fk) : 0), ok);
      }
  };
  /* stage the x faces of plane x (the lower faces of its cells) */
  auto stage_x = [&] (int x) {
    if (!sx) return;
    const int fx = face_index (x, n, px);
    const int sc = slot (x, RX);
    for (int e = t; e < CP; e += NT) {
      const int a = e/CK, b = e - a*CK;
      const int cj = cell_index (j0 - 1 + a, n, py), ck = cell_index (k0 - 1 + b, n, pz);
      const bool ok = fx >= 0 && cj >= 0 && ck >= 0;
      cp_async_el (sm + so.x + sc*CP + e, ax.p + (ok ? cidx<3> (g, fx, cj, ck) : 0), ok);
    }
  };
  /* relax_value (poisson.h:303-319) of the cell at staged position (pj, pk)
     of plane x, everything from shared memory */
  auto relax = [&] (int x, int pj_, int pk_) -> T {
    const int c = slot (x, R)*PL, m = slot (x - 1, R)*PL, p = slot (x + 1, R)*PL;
    const int o = pj_*WK + pk_;
    const int ci = (pj_ - 1)*CK + (pk_ - 1);
    const int cs = slot (x, RC);
    T nn = (-D2)*sm[so.b + cs*CP + ci];
    T d = (-(sl ? sm[so.l + cs*CP + ci] : lam.c))*D2;
    {
      const T a1 = sx ? sm[so.x + slot (x + 1, RX)*CP + ci] : ax.c;
      const T a0 = sx ? sm[so.x + slot (x, RX)*CP + ci] : ax.c;
      nn += a1*sm[p + o] + a0*sm[m + o];
      d += a1 + a0;
    }
    {
      const T a1 = sy ? sm[so.y + cs*YP + ci + CK] : ay.c;
      const T a0 = sy ? sm[so.y + cs*YP + ci] : ay.c;
      nn += a1*sm[c + o + WK] + a0*sm[c + o - WK];
      d += a1 + a0;
    }
    {
      const int zi = so.z + cs*ZP + (pj_ - 1)*ZK + (pk_ - 1);
      const T a1 = sz ? sm[zi + 1] : az.c;
      const T a0 = sz ? sm[zi] : az.c;
      nn += a1*sm[c + o + 1] + a0*sm[c + o - 1];
      d += a1 + a0;
    }
    return nn/d;
  };

  /* prologue: the iterate of plane i0 - 2; then at step x the iterate of
     plane x + 1, the cell coefficients of plane x and the x faces of
     plane x + 1 */
  stage_a (i0 - 2);
  stage_x (i0 - 2);
  cp_async_commit ();
  for (int x = i0 - 2; x <= i1 + 1; x++) {
    /* everything staged at step x - 1 is in, and every thread is done with
       step x - 1 (whose passes read the slots restaged below last) */
    cp_async_wait0 ();
    __syncthreads ();
    if (x + 1 <= i1 + 1) stage_a (x + 1);
    if (x >= i0 - 1 && x <= i1) stage_c (x);
    if (x + 1 <= i1 + 1) stage_x (x + 1);
    cp_async_commit ();
    /* red cells of plane x - 1: the tile and its first ring */
    const int xr = x - 1;
    if (xr >= i0 - 1 && xr <= i1 && real_cell (xr, n, px)) {
      const int c = slot (xr, R)*PL;
      const int odd = (xr + gj + gk) & 1;
      const int pk = pk0 + odd;
      if (gj < n && gk + odd < n) sm[c + pj*WK + pk] = relax (xr, pj, pk);
      if (ring_real && ((xr + rgj + rgk) & 1) == 0) sm[c + rj*WK + rk] = relax (xr, rj, rk);
    }
    __syncthreads ();
    /* black cells of plane x - 2, then the pair to the output */
    const int xb = x - 2;
    if (xb >= i0 && xb < i1) {
      const int c = slot (xb, R)*PL;
      const int odd = (xb + gj + gk + 1) & 1;
      const int pk = pk0 + odd;
      if (gj < n && gk + odd < n) sm[c + pj*WK + pk] = relax (xb, pj, pk);
      if (gj < n && gk < n) {
        const T v0 = sm[c + pj*WK + pk0], v1 = sm[c + pj*WK + pk0 + 1];
        const long long id = cidx<3> (g, xb, gj, gk);
        out[id] = v0;
        out[id + 1] = v1;
        ghosts_homog<3, T> (out, g, xb, gj, gk, v0, bc);
        ghosts_homog<3, T> (out, g, xb, gj, gk + 1, v1, bc);
      }
    }
  }
  cp_async_wait0 ();
}

template <typename T, int TJ, int TK>
int launch_rbs (bmg_geom g, void * out, const void * in, const void * rhs, const bmg_coef * alpha,
                bmg_coef lambda, double Delta, const bmg_bcdesc * bc, cudaStream_t s)
{
  typedef Sh3s<TJ, TK> S;
  const int n = g.n;
  Off3 so;
  int o = S::R*S::PL;
  so.b = o; o += S::RC*S::CP;
  so.l = o; if (lambda.p) o += S::RC*S::CP;
  so.y = o; if (alpha[1].p) o += S::RC*S::YP;
  so.z = o; if (alpha[2].p) o += S::RC*S::ZP;
  so.x = o; if (alpha[0].p) o += S::RX*S::CP;
  so.total = o;
  const size_t smem = (size_t) o*sizeof (T);
  const size_t smax = (size_t) (S::R*S::PL + S::RC*(2*S::CP + S::YP + S::ZP) + S::RX*S::CP)*sizeof (T);
  static int slots[64][16];
  int dev = 0;
  cudaGetDevice (&dev);
  if (dev < 0 || dev >= 64) return (int) cudaErrorInvalidDevice;
  const int key = (lambda.p ? 1 : 0) | (alpha[0].p ? 2 : 0) | (alpha[1].p ? 4 : 0) | (alpha[2].p ? 8 : 0);
  if (!slots[dev][key]) {
    cudaError_t e = cudaFuncSetAttribute (k_relax3d_rbs<T, TJ, TK>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smax);
    int per = 0, sms = 0;
    if (e == cudaSuccess)
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor (&per, k_relax3d_rbs<T, TJ, TK>, S::NT, smem);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute (&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return (int) e;
    slots[dev][key] = per*sms > 0 ? per*sms : 1;
  }
  const int tiles = ((n + TK - 1)/TK)*((n + TJ - 1)/TJ);
  int chunks = slots[dev][key]/tiles;
  if (chunks > n/8) chunks = n/8;
  if (chunks < 1) chunks = 1;
  const int ZB = (n + chunks - 1)/chunks;
  chunks = (n + ZB - 1)/ZB;
  dim3 grid ((n + TK - 1)/TK, (n + TJ - 1)/TJ, chunks);
  k_relax3d_rbs<T, TJ, TK><<<grid, S::NT, smem, s>>> (
    g, (T *) out, (const T *) in, (const T *) rhs, coef_of<T> (alpha[0]), coef_of<T> (alpha[1]),
    coef_of<T> (alpha[2]), coef_of<T> (lambda), (T) Delta, bch_of (bc), ZB, so);
  return (int) cudaGetLastError ();
}

template <typename T, int TJ, int TK>
int launch_rb3 (bmg_geom g, void * out, const void * in, const void * rhs, const bmg_coef * alpha,
                bmg_coef lambda, double Delta, const bmg_bcdesc * bc, cudaStream_t s)
{
  typedef Sh3<TJ, TK> S;
  const int n = g.n;
  const size_t smem = (size_t) S::RING*S::PL*sizeof (T);
  /* resident CTAs of the device (once per device) */
  static int slots[64];
  int dev = 0;
  cudaGetDevice (&dev);
  if (dev < 0 || dev >= 64) return (int) cudaErrorInvalidDevice;
  if (!slots[dev]) {
    cudaError_t e = cudaFuncSetAttribute (k_relax3d_rb<T, TJ, TK>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
    int per = 0, sms = 0;
    if (e == cudaSuccess)
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor (&per, k_relax3d_rb<T, TJ, TK>, S::NT, smem);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute (&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return (int) e;
    slots[dev] = per*sms > 0 ? per*sms : 1;
  }
  /* chunks along the first index: as many CTAs as fit on the device at
     once, in one wave (a partial second wave would double the time) */
  const int tiles = ((n + TK - 1)/TK)*((n + TJ - 1)/TJ);
  int chunks = slots[dev]/tiles;
  if (chunks > n/8) chunks = n/8;
  if (chunks < 1) chunks = 1;
  const int ZB = (n + chunks - 1)/chunks;
  chunks = (n + ZB - 1)/ZB;
  dim3 grid ((n + TK - 1)/TK, (n + TJ - 1)/TJ, chunks);
  k_relax3d_rb<T, TJ, TK><<<grid, S::NT, smem, s>>> (
    g, (T *) out, (const T *) in, (const T *) rhs, coef_of<T> (alpha[0]), coef_of<T> (alpha[1]),
    coef_of<T> (alpha[2]), coef_of<T> (lambda), (T) Delta, bch_of (bc), ZB);
  return (int) cudaGetLastError ();
}

} // namespace

extern "C" {

int bmg_relax3d_rb_ok (int n)
{
  return n >= 16 && n % 16 == 0;
}

int bmg_launch_relax3d_rb (int st, bmg_geom g, void * out, const void * in, const void * rhs,
                           const bmg_coef * alpha, bmg_coef lambda, double Delta,
                           const bmg_bcdesc * bc, cudaStream_t s)
{
  if (!bmg_relax3d_rb_ok (g.n) || out == in) return (int) cudaErrorInvalidValue;
  static int staged = -1;
  if (staged < 0) staged = getenv ("BMG_FUSED3D_GLOBAL") == NULL;
  if (staged) {
    if (g.n >= 32)
      return st == BMG_ST_F64 ? launch_rbs<double, 16, 32> (g, out, in, rhs, alpha, lambda, Delta, bc, s)
                              : launch_rbs<float, 16, 32> (g, out, in, rhs, alpha, lambda, Delta, bc, s);
    return st == BMG_ST_F64 ? launch_rbs<double, 16, 16> (g, out, in, rhs, alpha, lambda, Delta, bc, s)
                            : launch_rbs<float, 16, 16> (g, out, in, rhs, alpha, lambda, Delta, bc, s);
  }
  if (g.n >= 32)
    return st == BMG_ST_F64 ? launch_rb3<double, 16, 32> (g, out, in, rhs, alpha, lambda, Delta, bc, s)
                            : launch_rb3<float, 16, 32> (g, out, in, rhs, alpha, lambda, Delta, bc, s);
  return st == BMG_ST_F64 ? launch_rb3<double, 16, 16> (g, out, in, rhs, alpha, lambda, Delta, bc, s)
                          : launch_rb3<float, 16, 16> (g, out, in, rhs, alpha, lambda, Delta, bc, s);
}

} // extern "C"

/*
 * mg_device.cuh -- device helpers shared by the kernels of the multigrid
 * solver: level layout, coefficients, ghost-image writers (the boundary
 * conditions of grid/multigrid.h:543-695 and common.h:957-960) and the
 * relax update of poisson.h:303-319.
 */
#ifndef MG_DEVICE_CUH
#define MG_DEVICE_CUH

#include <cuda_runtime.h>
#include "mg_launch.h"

namespace bmgd {

/* programmatic dependent launch (sm_90+).  A kernel launched with
   pdl_launch starts while its predecessor in the stream drains; it calls
   pdl_wait () before touching global memory (the predecessor has then
   completed and its writes are visible) and pdl_trigger () to let its own
   successor be scheduled.  Only the launch latency overlaps: the order of
   every memory access is that of plain stream order. */
__device__ __forceinline__ void pdl_wait ()
{
  asm volatile ("griddepcontrol.wait;" ::: "memory");
}

__device__ __forceinline__ void pdl_trigger ()
{
  asm volatile ("griddepcontrol.launch_dependents;" ::: "memory");
}

template <typename... KArgs, typename... Args>
inline cudaError_t pdl_launch (void (*k) (KArgs...), dim3 grid, dim3 block, size_t smem,
                               cudaStream_t s, Args... args)
{
  cudaLaunchConfig_t cfg;
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx (&cfg, k, ((KArgs) args)...);
}

/* ---------------------------------------------------------------- */
/* layout                                                            */
/* ---------------------------------------------------------------- */

template <int DIM>
__device__ __forceinline__ long long cidx (const bmg_geom & g, int i, int j, int k)
{
  if (DIM == 1) return (long long) g.xo + i;
  if (DIM == 2) return (long long) (i + 1)*g.P + g.xo + j;
  return (long long) (i + 1)*g.plane + (long long) (j + 1)*g.P + g.xo + k;
}

template <int DIM>
__device__ __forceinline__ long long cstride (const bmg_geom & g, int e)
{
  if (DIM == 1) return 1;
  if (DIM == 2) return e == 0 ? (long long) g.P : 1;
  return e == 0 ? g.plane : e == 1 ? (long long) g.P : 1;
}

/* thread -> interior cell; the contiguous axis maps to threadIdx.x */
template <int DIM>
__device__ __forceinline__ bool cell_of_thread (int n, int & i, int & j, int & k)
{
  if (DIM == 1) {
    i = blockIdx.x*blockDim.x + threadIdx.x; j = k = 0;
    return i < n;
  }
  if (DIM == 2) {
    j = blockIdx.x*blockDim.x + threadIdx.x;
    i = blockIdx.y*blockDim.y + threadIdx.y; k = 0;
    return i < n && j < n;
  }
  k = blockIdx.x*blockDim.x + threadIdx.x;
  j = blockIdx.y*blockDim.y + threadIdx.y;
  i = blockIdx.z*blockDim.z + threadIdx.z;
  return i < n && j < n && k < n;
}

template <int DIM> dim3 block_shape ()
{
  if (DIM == 1) return dim3 (256, 1, 1);
  if (DIM == 2) return dim3 (32, 8, 1);
  return dim3 (32, 4, 2);
}

template <int DIM> dim3 grid_shape (int n)
{
  dim3 b = block_shape<DIM> ();
  dim3 g ((n + b.x - 1)/b.x, 1, 1);
  if (DIM >= 2) g.y = (n + b.y - 1)/b.y;
  if (DIM >= 3) g.z = (n + b.z - 1)/b.z;
  return g;
}

template <typename T>
struct Coef {
  const T * p;
  T c;
  __device__ __forceinline__ T at (long long id) const { return p ? p[id] : c; }
};

template <typename T>
__host__ __device__ inline Coef<T> coef_of (const bmg_coef & c)
{
  Coef<T> r;
  r.p = (const T *) c.p;
  r.c = (T) c.c;
  return r;
}

/* homogeneous boundary factors of a field: ghost = fac*cell for box sides
   (dirichlet_homogeneous -s[], neumann_homogeneous s[], common.h:958,960) */
struct BCH {
  int periodic[3];
  int fac[6];
};

inline BCH bch_of (const bmg_bcdesc * bc)
{
  BCH h;
  for (int e = 0; e < 3; e++) h.periodic[e] = bc ? bc->periodic[e] : 0;
  for (int s = 0; s < 6; s++)
    h.fac[s] = (bc && bc->type[s] == 1 /* BMG_DIRICHLET */) ? -1 : 1;
  return h;
}

template <int DIM>
__device__ __forceinline__ bool on_boundary (int n, int i, int j, int k)
{
  bool b = (i == 0 || i == n - 1);
  if (DIM > 1) b = b || j == 0 || j == n - 1;
  if (DIM > 2) b = b || k == 0 || k == n - 1;
  return b;
}

/* write the ghost images of cell (i, j, k) of value v, homogeneous BCs */
template <int DIM, typename T>
__device__ void ghosts_homog (T * f, const bmg_geom & g, int i, int j, int k,
                              T v, const BCH & bc)
{
  const int n = g.n;
  if (!on_boundary<DIM> (n, i, j, k)) return;
  const int c[3] = {i, j, k};
  int pos[3][3];
  T fac[3][3];
  int cnt[3];
  const bool l0p = (n == 1) && (bc.periodic[0] || bc.periodic[1] || bc.periodic[2]);
#pragma unroll
  for (int e = 0; e < 3; e++) {
    pos[e][0] = c[e]; fac[e][0] = T(1); cnt[e] = 1;
    if (e < DIM) {
      if (c[e] == 0) {
        if (bc.periodic[e]) { pos[e][cnt[e]] = n; fac[e][cnt[e]] = T(1); }
        else { pos[e][cnt[e]] = -1; fac[e][cnt[e]] = l0p ? T(1) : T(bc.fac[2*e + 1]); }
        cnt[e]++;
      }
      if (c[e] == n - 1) {
        if (bc.periodic[e]) { pos[e][cnt[e]] = -1; fac[e][cnt[e]] = T(1); }
        else { pos[e][cnt[e]] = n; fac[e][cnt[e]] = l0p ? T(1) : T(bc.fac[2*e]); }
        cnt[e]++;
      }
    }
  }
  for (int a = 0; a < cnt[0]; a++)
    for (int b = 0; b < cnt[1]; b++)
      for (int d = 0; d < cnt[2]; d++) {
        if (a == 0 && b == 0 && d == 0) continue;
        f[cidx<DIM> (g, pos[0][a], pos[1][b], pos[2][d])] = v*fac[0][a]*fac[1][b]*fac[2][d];
      }
}

/* boundary value of side s at the tangential indices of cell (i, j, k) */
template <int DIM>
__device__ __forceinline__ double bc_data (const bmg_bcdesc & bc, int s, int n,
                                           int i, int j, int k)
{
  const double * v = bc.val[s];
  if (!v) return bc.cval[s];
  int e = s/2;
  long long t = 0;
  if (DIM == 2) t = e == 0 ? j : i;
  if (DIM == 3) t = e == 0 ? (long long) j*n + k : e == 1 ? (long long) i*n + k : (long long) i*n + j;
  return v[t];
}

/* ghost images with the inhomogeneous BCs of a field on the finest level:
   dirichlet 2v - s[], neumann Delta*v + s[] (common.h:957,959), composed
   dimension by dimension for edges and corners */
template <int DIM>
__device__ void ghosts_inhomog (double * f, const bmg_geom & g, int i, int j, int k,
                                double v, const bmg_bcdesc & bc)
{
  const int n = g.n;
  if (!on_boundary<DIM> (n, i, j, k)) return;
  const int c[3] = {i, j, k};
  int pos[3][3], side[3][3], cnt[3];
  const bool l0p = (n == 1) && (bc.periodic[0] || bc.periodic[1] || bc.periodic[2]);
#pragma unroll
  for (int e = 0; e < 3; e++) {
    pos[e][0] = c[e]; side[e][0] = -1; cnt[e] = 1;
    if (e < DIM) {
      if (c[e] == 0) {
        pos[e][cnt[e]] = bc.periodic[e] ? n : -1;
        side[e][cnt[e]] = bc.periodic[e] ? -1 : 2*e + 1;
        cnt[e]++;
      }
      if (c[e] == n - 1) {
        pos[e][cnt[e]] = bc.periodic[e] ? -1 : n;
        side[e][cnt[e]] = bc.periodic[e] ? -1 : 2*e;
        cnt[e]++;
      }
    }
  }
  for (int a = 0; a < cnt[0]; a++)
    for (int b = 0; b < cnt[1]; b++)
      for (int d = 0; d < cnt[2]; d++) {
        if (a == 0 && b == 0 && d == 0) continue;
        double r = v;
        if (!l0p) {
          const int sd[3] = {side[0][a], side[1][b], side[2][d]};
          for (int e = 0; e < DIM; e++)
            if (sd[e] >= 0) {
              double w = bc_data<DIM> (bc, sd[e], n, i, j, k);
              if (bc.type[sd[e]] == 1 /* BMG_DIRICHLET */)
                r = 2.*(w) - r;
              else
                r = bc.Delta*(w) + r;
            }
        }
        f[cidx<DIM> (g, pos[0][a], pos[1][b], pos[2][d])] = r;
      }
}

/* ---------------------------------------------------------------- */
/* relax                                                             */
/* ---------------------------------------------------------------- */

/* one cell of relax (poisson.h:303-319) */
template <int DIM, typename T>
__device__ __forceinline__ T relax_value (const bmg_geom & g, long long id, const T * in,
                                          const T * rhs, const Coef<T> & ax,
                                          const Coef<T> & ay, const Coef<T> & az,
                                          const Coef<T> & lam, T D2)
{
  T nn = (-D2)*rhs[id], d = (-lam.at (id))*D2;
  {
    long long s = cstride<DIM> (g, 0);
    T a1 = ax.at (id + s), a0 = ax.at (id);
    nn += a1*in[id + s] + a0*in[id - s];
    d += a1 + a0;
  }
  if (DIM > 1) {
    long long s = cstride<DIM> (g, 1);
    T a1 = ay.at (id + s), a0 = ay.at (id);
    nn += a1*in[id + s] + a0*in[id - s];
    d += a1 + a0;
  }
  if (DIM > 2) {
    long long s = cstride<DIM> (g, 2);
    T a1 = az.at (id + s), a0 = az.at (id);
    nn += a1*in[id + s] + a0*in[id - s];
    d += a1 + a0;
  }
  return nn/d;
}

} // namespace bmgd

#endif

/*
 * mg_launch.h -- internal interface between the C host layer (mg_host.c)
 * and the CUDA kernels (mg_kernels.cu).  Plain C types only.
 *
 * Device level layout (one array per field per level, structure of arrays):
 *   interior cell (i, j, k), 0 <= i, j, k < n, of a level lives at
 *     1D:  xo + i
 *     2D:  (i + 1)*P + xo + j
 *     3D:  (i + 1)*plane + (j + 1)*P + xo + k
 *   with one ghost layer on every side (the reference keeps GHOSTS = 2 but
 *   its box conditions fill only BGHOSTS = 1, grid/multigrid.h:2-9, and no
 *   operator of this path reads the second layer).  xo puts interior index 0
 *   of the contiguous axis on a 32-byte boundary; P is padded to 128 bytes.
 *   Face component d uses the same array shape: face f along d sits at the
 *   slot of cell f, so face n is the ghost slot (as alpha.x[1] of the last
 *   cell in the reference).
 */
#ifndef MG_LAUNCH_H
#define MG_LAUNCH_H

#include <cuda_runtime_api.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BMG_MAXLEVEL 15

typedef struct {
  int n;             /* interior cells per side */
  int P;             /* elements per row of the contiguous axis */
  int xo;            /* element offset of interior index 0 on that axis */
  int pad_;
  long long plane;   /* elements per slab of the first axis (3D) */
  long long size;    /* elements of the level array */
} bmg_geom;

/* boundary conditions of one field (finest level for inhomogeneous data) */
typedef struct {
  int periodic[3];
  int type[6];             /* BMG_NEUMANN / BMG_DIRICHLET / BMG_PERIODIC */
  const double * val[6];   /* device boundary values, NULL = cval */
  double cval[6];
  double Delta;            /* finest-level cell size, for Neumann data */
} bmg_bcdesc;

/* a coefficient on one level: array of the storage type, or a constant */
typedef struct {
  const void * p;
  double c;
} bmg_coef;

/* storage types */
enum { BMG_ST_F64 = 0, BMG_ST_F32 = 1 };
/* relax modes */
enum { BMG_SWEEP_RED = 0, BMG_SWEEP_BLACK = 1, BMG_SWEEP_JACOBI = 2 };

int bmg_launch_relax (int dim, int st, int mode, bmg_geom g, void * out,
                      const void * in, const void * rhs, const bmg_coef * alpha,
                      bmg_coef lambda, double Delta, const bmg_bcdesc * bc,
                      cudaStream_t s);

int bmg_launch_prolong (int dim, int st_coarse, int st_fine, bmg_geom gc,
                        bmg_geom gf, const void * coarse, void * fine,
                        const bmg_bcdesc * bc, int zero, cudaStream_t s);

int bmg_launch_restrict (int dim, int st_fine, int st_coarse, bmg_geom gf,
                         bmg_geom gc, const void * fine, void * coarse,
                         cudaStream_t s);

/* level0p: the coarse level is a periodic level 0, whose upper faces are
   copies of the lower ones */
int bmg_launch_restrict_face (int dim, bmg_geom gf, bmg_geom gc,
                              const double * const * fine, double * const * coarse,
                              int level0p, cudaStream_t s);

int bmg_launch_residual (int dim, int st_res, bmg_geom g, bmg_geom gres,
                         const double * a, const double * b,
                         const bmg_coef * alpha, bmg_coef lambda, double Delta,
                         void * res, unsigned long long * maxres,
                         cudaStream_t s);

/* the 2D residual of the finest level (as bmg_launch_residual, max into
   maxres) fused with its restriction into the level below (coarse, storage
   st_coarse, geometry gcoarse): bit-identical to bmg_launch_residual then
   bmg_launch_restrict */
int bmg_launch_residual_restrict (int st_res, int st_coarse, bmg_geom g, bmg_geom gres,
                                  bmg_geom gcoarse, const double * a, const double * b,
                                  const bmg_coef * alpha, bmg_coef lambda, double Delta,
                                  void * res, void * coarse, unsigned long long * maxres,
                                  cudaStream_t s);

/* the same for the finest 3D level (eight children per coarse cell) */
int bmg_launch_residual_restrict3d (int st_res, int st_coarse, bmg_geom g, bmg_geom gres,
                                    bmg_geom gcoarse, const double * a, const double * b,
                                    const bmg_coef * alpha, bmg_coef lambda, double Delta,
                                    void * res, void * coarse, unsigned long long * maxres,
                                    cudaStream_t s);

/* the black pass of a 3D red-black sweep (in place, out == in) that also
   applies a += out to the FP64 finest level acor (geometry ga) with the
   ghost images of its boundary conditions abc: the last pass of a cycle's
   finest level, bit-identical to the pass followed by bmg_launch_correct */
int bmg_launch_relax_correct3d (int st, bmg_geom g, void * out, const void * in, const void * rhs,
                                const bmg_coef * alpha, bmg_coef lambda, double Delta,
                                const bmg_bcdesc * bc, double * acor, bmg_geom ga,
                                const bmg_bcdesc * abc, cudaStream_t s);

int bmg_launch_correct (int dim, int st_da, bmg_geom g, bmg_geom gda, double * a,
                        const void * da, const bmg_bcdesc * bc, cudaStream_t s);

int bmg_launch_apply_bc (int dim, int st, bmg_geom g, void * f,
                         const bmg_bcdesc * bc, int homogeneous, cudaStream_t s);

int bmg_launch_sum (int dim, bmg_geom g, const double * b, double * partials,
                    int npartials, double * out, cudaStream_t s);

int bmg_launch_pack (int dim, int st, bmg_geom g, int face_dim,
                     const double * compact, void * padded, cudaStream_t s);

int bmg_launch_unpack (int dim, bmg_geom g, int face_dim, const double * padded,
                       double * compact, cudaStream_t s);

int bmg_launch_convert (int dim, bmg_geom g64, bmg_geom g32, int face_dim,
                        const double * src, float * dst, cudaStream_t s);

int bmg_launch_fill (int dim, int st, bmg_geom g, void * f, double v, cudaStream_t s);

int bmg_launch_shift (int dim, bmg_geom g, double * f, const double * sum,
                      double scale, cudaStream_t s);

/* adjoint coefficient gradients: face component e into a compact face
   array, and -mu*a into a compact cell array */
int bmg_launch_adjoint_faces (int dim, bmg_geom g, int e, int periodic, const double * mu,
                              const double * a, double Delta, double * out, cudaStream_t s);
int bmg_launch_adjoint_cells (int dim, bmg_geom g, const double * mu, const double * a,
                              double * out, cudaStream_t s);

int bmg_launch_face_wrap (int dim, bmg_geom g, int face_dim, double * f, cudaStream_t s);

/* ghost slabs of direction e of nb blocks' level arrays (geometry g), for
   the decomposed solve: the ghost slab -1 of dst takes slab n - 1 of lo,
   the ghost slab n takes slab 0 of hi (NULL: that side is not
   exchanged); a slab spans -1..n of the other directions, ghosts included,
   so that exchanging the directions in order fills edges and corners from
   the diagonal blocks.  lo and hi may be another device's memory (peer
   access enabled). */
typedef struct { double * dst; const double * lo, * hi; } bmg_halo;
int bmg_launch_halo (int dim, bmg_geom g, int e, const bmg_halo * blocks, int nb, cudaStream_t s);

/* fused red-black relaxation (mg_fused.cu) */
int bmg_tile_sweeps (int st, int n);   /* sweeps one tile launch can do on an n x n level */
/* whether the tile launch of an n x n level can apply the correction: with
   acor != NULL (the FP64 finest level of a, geometry ga, boundary conditions
   abc) the launch also does a += out on every cell it writes, with the
   ghost images of a (poisson.h:84-89) */
int bmg_tile_corrects (int st, int n);
/* whether the tile launch of an n x n level can stage the level's
   prolongation itself: with coarse != NULL (the level below, of the same
   storage type, geometry gc, ghosts filled) the launch relaxes the bilinear
   prolongation of coarse (multigrid-common.h:124-140, the values
   bmg_launch_prolong would write) instead of in, so that the level's first
   launch replaces its prolongation launch */
int bmg_tile_prolongs (int st, int n);
int bmg_launch_relax_tile (int dim, int st, bmg_geom g, void * out, const void * in,
                           const void * res, const bmg_coef * alpha, bmg_coef lambda,
                           double Delta, const bmg_bcdesc * bc, int nsweeps, double * acor,
                           bmg_geom ga, const bmg_bcdesc * abc, const void * coarse, bmg_geom gc,
                           cudaStream_t s);

/* all nrelax red-black sweeps of a 2D level (FP32: 64^2 to 256^2; FP64,
   bit-identical: 64^2 and 128^2) in one launch of one thread-block
   cluster, the bilinear prolongation of coarse (the level below, same
   storage type, ghosts included) fused in; the final iterate, with its
   ghost images, goes to out.  bmg_level_cluster_ok () tells whether a
   level has such a kernel.  Returns 0, -1 when the device cannot schedule
   the cluster (use tile launches), or a CUDA error. */
int bmg_level_cluster_ok (int st, int n);
int bmg_launch_level_cluster (int st, bmg_geom g, void * out, const void * res,
                              const bmg_coef * alpha, bmg_coef lambda, double Delta,
                              const bmg_bcdesc * bc, int nrelax, bmg_geom gc, const void * coarse,
                              cudaStream_t s);

/* one level of the single-CTA bottom solve */
typedef struct {
  bmg_geom g;
  void * da;
  void * res;
  bmg_coef alpha[3];
  bmg_coef lambda;
  double Delta;
  int st;
  int fast;     /* relax from weights divided by the diagonal once per level
                   (not in the reference's evaluation order: mixed form only) */
} bmg_bottom_level;

/* levels lv[0..nlev-1] (coarse to fine): restriction of res (from the level
   above, g_src/res_src, when restrict_src), zero, prolongations and nrelax
   red-black sweeps per level, in one launch of one CTA, with every level
   staged in shared memory (at most BMG_BOTTOM_SMEM bytes, see
   bmg_bottom_smem) */
#define BMG_BOTTOM_SMEM (200*1024)
size_t bmg_bottom_smem (int dim, const bmg_bottom_level * lv, int nlev);
int bmg_launch_bottom (int dim, const bmg_bottom_level * lv, int nlev, bmg_geom g_src,
                       const void * res_src, int st_src, int restrict_src, int nrelax,
                       const bmg_bcdesc * bc, cudaStream_t s);

/* number of partial sums bmg_launch_sum needs for a level */
int bmg_sum_partials (int dim, bmg_geom g);

/* implicit viscosity (viscosity.h), 2D and 3D, FP64: one pass of
   relax_viscosity into w (mode 0: every cell, 1/2: red/black cells), its
   commit into u (Jacobi average, or the colour's cells), and
   residual_viscosity with max |res| */
int bmg_launch_visc_relax (int dim, bmg_geom g, int mode, double * const * u,
                           double * const * r, double * const * w, const bmg_coef * mu,
                           bmg_coef rho, double dt, double Delta, cudaStream_t s);
int bmg_launch_visc_commit (int dim, bmg_geom g, int mode, double * const * u,
                            double * const * w, cudaStream_t s);
int bmg_launch_visc_residual (int dim, bmg_geom g, double * const * u, double * const * r,
                              double * const * res, const bmg_coef * mu, bmg_coef rho,
                              double dt, double Delta, unsigned long long * maxres,
                              cudaStream_t s);

/* project (poisson.h:468-509): the divergence of a face vector over
   dt Delta, and the face correction uf -= dt alpha grad p of direction e */
int bmg_launch_divergence (int dim, bmg_geom g, const double * const * uf, double dt,
                           double Delta, double * div, cudaStream_t s);
int bmg_launch_project_faces (int dim, bmg_geom g, int e, double * u, bmg_coef alpha,
                              const double * p, double dt, double Delta, cudaStream_t s);

#ifdef __cplusplus
}
#endif
#endif

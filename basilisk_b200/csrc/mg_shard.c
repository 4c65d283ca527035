/*
 * mg_shard.c -- mg_solve over a Cartesian decomposition of the domain into
 * blocks, the device counterpart of grid/multigrid-mpi.h.
 *
 * The reference splits a multigrid domain into dims[0] x dims[1] (x dims[2])
 * blocks (MPI_Dims_create, MPI_Cart_create: multigrid-mpi.h:94-130), each a
 * complete multigrid hierarchy of the same depth on its own rank.  A side
 * that faces another block is marked periodic so that no box condition is
 * applied there, and mpi_boundary_level (multigrid-mpi.h:52-85) fills the
 * ghost layer of that side from the neighbour after every operation that
 * ends with a boundary: direction by direction (x, then y, then z), each
 * message a slab of the padded level including the ghosts of the directions
 * already exchanged, so that edge and corner ghosts come from the diagonal
 * neighbours.  The reductions of mg_solve (the sum of b, the maximum
 * residual) become MPI_Allreduce (common.h:681-718).
 *
 * Here every block is a bmg_grid on a CUDA device, and one host thread
 * drives all the blocks of the decomposition: the blocks of one device
 * share one stream, the exchange of a direction is one kernel per device
 * (bmg_launch_halo) that copies every neighbour's edge slab straight into
 * its blocks' ghost slabs -- reading the neighbour by peer access over
 * NVLink when it lives on another device -- ordered across devices by
 * events, and the reductions are the maximum / sum of the blocks' values
 * on the host, which reads them back every cycle as the single-grid solve
 * does.
 *
 * Boundary conditions: a side of a block that faces another block keeps
 * the field's box condition type (its kernels write box images there,
 * which the exchange then overwrites); a direction is periodic on a block
 * only when the domain is periodic in it and it holds a single block.
 *
 * The solve is the reference's mg_solve / mg_cycle (poisson.h:32-90,
 * 139-235) with one relaxation pass per launch and a boundary exchange
 * after each pass, exactly where the single-grid solve has a boundary: the
 * zero or prolonged correction of a level, each colour pass of a red-black
 * sweep (red, boundary, black, boundary) or each Jacobi sweep, and a after
 * the correction a += da.  Every value is computed by the kernels the
 * single-grid solve uses, in the same order, so a decomposed solve gives
 * the single grid's solution bit for bit (FP64) when the single grid's
 * minlevel is the blocks' minlevel plus log2 (dims[0]); mgstats.sum is the
 * sum of the blocks' sums, a reduction in another order.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <cuda_runtime_api.h>

#include "mg_grid.h"

#define MAXB 4096

struct bmg_shard {
  int dim, nb, dims[3], periodic[3];
  bmg_grid ** blk;
  int (*nbr)[6];              /* neighbour block of each side, -1: box side */
  int ndev;
  int dev[16];                /* the devices holding blocks */
  cudaStream_t stream[16];    /* one stream per device */
  cudaEvent_t ev[16];
  int * bdev;                 /* device slot of each block */
  bmg_halo * halo;            /* exchange descriptors, one per block */
  long long nhalo;            /* exchange launches */
};

#define FAIL(s) bmg_i_fail (s)
#define CKS(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) { \
      fprintf (stderr, "bmg shard: %s failed: %s (%s:%d)\n", #call,      \
               cudaGetErrorString (e_), __FILE__, __LINE__);              \
      return FAIL (e_ == cudaErrorMemoryAllocation ? BMG_ENOMEM : BMG_ECUDA); } } while (0)
#define CLS(call) do { int e_ = (call); if (e_) {                         \
      fprintf (stderr, "bmg shard: launch %s failed: %s (%s:%d)\n", #call, \
               cudaGetErrorString ((cudaError_t) e_), __FILE__, __LINE__); \
      return FAIL (BMG_ECUDA); } } while (0)

/* ------------------------------------------------------------------ */
/* the decomposition                                                   */
/* ------------------------------------------------------------------ */

/* MPI_Dims_create (n, dimension, dims) with all dims free: the factors of
   n spread as evenly as possible over the dimensions, in non-increasing
   order (the largest prime factors first, each onto the currently
   smallest dimension) */
int bmg_shard_dims (int n, int dimension, int * dims)
{
  if (n < 1 || dimension < 1 || dimension > 3 || !dims) return FAIL (BMG_EINVAL);
  int f[64], nf = 0, m = n;
  for (int p = 2; p*p <= m; p++)
    while (m % p == 0) { f[nf++] = p; m /= p; }
  if (m > 1) f[nf++] = m;
  int d[3] = {1, 1, 1};
  for (int k = nf - 1; k >= 0; k--) {
    int s = 0;
    for (int e = 1; e < dimension; e++) if (d[e] < d[s]) s = e;
    d[s] *= f[k];
  }
  /* non-increasing */
  for (int a = 0; a < dimension; a++)
    for (int b = a + 1; b < dimension; b++)
      if (d[b] > d[a]) { int t = d[a]; d[a] = d[b]; d[b] = t; }
  for (int e = 0; e < 3; e++) dims[e] = e < dimension ? d[e] : 1;
  return BMG_OK;
}

/* the neighbours of block b (MPI_Cart_shift over a row-major Cartesian
   order: b = (c0 dims[1] + c1) dims[2] + c2), sides in the reference's
   order right, left, top, bottom, front, back: -1 where the side is a box
   side */
int bmg_shard_neighbours (int dimension, const int * dims, const int * periodic, int b,
                          int * out)
{
  if (dimension < 1 || dimension > 3 || !dims || !out) return FAIL (BMG_EINVAL);
  int nd[3] = {1, 1, 1}, total = 1;
  for (int e = 0; e < dimension; e++) {
    if (dims[e] < 1) return FAIL (BMG_EINVAL);
    nd[e] = dims[e];
    total *= dims[e];
  }
  if (b < 0 || b >= total) return FAIL (BMG_EINVAL);
  int c[3] = {b/(nd[1]*nd[2]), (b/nd[2]) % nd[1], b % nd[2]};
  for (int s = 0; s < 6; s++) out[s] = -1;
  for (int e = 0; e < dimension; e++)
    for (int hi = 1; hi >= 0; hi--) {
      int cc[3] = {c[0], c[1], c[2]};
      cc[e] += hi ? 1 : -1;
      if (cc[e] < 0 || cc[e] >= nd[e]) {
        if (!(periodic && periodic[e]) || nd[e] == 1) continue;
        cc[e] = (cc[e] + nd[e]) % nd[e];
      }
      out[2*e + (hi ? 0 : 1)] = (cc[0]*nd[1] + cc[1])*nd[2] + cc[2];
    }
  return BMG_OK;
}

static int devslot (bmg_shard * s, int dev)
{
  for (int k = 0; k < s->ndev; k++) if (s->dev[k] == dev) return k;
  return -1;
}

void bmg_shard_free (bmg_shard * s)
{
  if (!s) return;
  /* give the blocks streams of their own again */
  for (int b = 0; b < s->nb; b++)
    if (s->blk[b]) {
      cudaSetDevice (s->blk[b]->device);
      cudaStreamSynchronize (s->blk[b]->stream);
      bmg_set_stream (s->blk[b], NULL);
    }
  for (int k = 0; k < s->ndev; k++) {
    cudaSetDevice (s->dev[k]);
    if (s->stream[k]) cudaStreamDestroy (s->stream[k]);
    if (s->ev[k]) cudaEventDestroy (s->ev[k]);
  }
  free (s->blk); free (s->nbr); free (s->bdev); free (s->halo);
  free (s);
}

int bmg_shard_new (bmg_shard ** out, bmg_grid * const * blocks, const int * dims,
                   const int * periodic)
{
  if (!out || !blocks || !dims) return FAIL (BMG_EINVAL);
  *out = NULL;
  const int dim = blocks[0] ? blocks[0]->dim : 0;
  if (dim < 1) return FAIL (BMG_EINVAL);
  int nb = 1;
  for (int e = 0; e < dim; e++) {
    if (dims[e] < 1) return FAIL (BMG_EINVAL);
    nb *= dims[e];
  }
  if (nb > MAXB) return FAIL (BMG_EINVAL);
  for (int b = 0; b < nb; b++) {
    const bmg_grid * g = blocks[b];
    if (!g || g->dim != dim || g->depth != blocks[0]->depth || g->tree ||
        g->precision != BMG_FP64 || g->relax != blocks[0]->relax)
      return FAIL (BMG_EINVAL);
    for (int e = 0; e < dim; e++) {
      const int want = periodic && periodic[e] && dims[e] == 1;
      if (g->periodic[e] != want) return FAIL (BMG_EINVAL);
    }
  }
  bmg_shard * s = calloc (1, sizeof *s);
  if (!s) return FAIL (BMG_ENOMEM);
  s->dim = dim; s->nb = nb;
  for (int e = 0; e < 3; e++) {
    s->dims[e] = e < dim ? dims[e] : 1;
    s->periodic[e] = e < dim && periodic ? periodic[e] != 0 : 0;
  }
  s->blk = calloc (nb, sizeof (bmg_grid *));
  s->nbr = calloc (nb, sizeof *s->nbr);
  s->bdev = calloc (nb, sizeof (int));
  s->halo = calloc (nb, sizeof (bmg_halo));
  if (!s->blk || !s->nbr || !s->bdev || !s->halo) { bmg_shard_free (s); return FAIL (BMG_ENOMEM); }
  for (int b = 0; b < nb; b++) {
    int k = devslot (s, blocks[b]->device);
    if (k < 0) {
      if (s->ndev == 16) { bmg_shard_free (s); return FAIL (BMG_EINVAL); }
      k = s->ndev++;
      s->dev[k] = blocks[b]->device;
    }
    s->bdev[b] = k;
    bmg_shard_neighbours (dim, s->dims, s->periodic, b, s->nbr[b]);
  }
  int cur = 0;
  cudaGetDevice (&cur);
  for (int k = 0; k < s->ndev; k++) {
    cudaError_t e = cudaSetDevice (s->dev[k]);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags (&s->stream[k], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags (&s->ev[k], cudaEventDisableTiming);
    /* peer access to the devices of the neighbours (NVLink copies) */
    for (int j = 0; j < s->ndev && e == cudaSuccess; j++)
      if (j != k) {
        int ok = 0;
        cudaDeviceCanAccessPeer (&ok, s->dev[k], s->dev[j]);
        if (ok) {
          cudaError_t pe = cudaDeviceEnablePeerAccess (s->dev[j], 0);
          if (pe != cudaSuccess && pe != cudaErrorPeerAccessAlreadyEnabled) e = pe;
          else cudaGetLastError ();
        }
      }
    if (e != cudaSuccess) {
      fprintf (stderr, "bmg shard: device %d: %s\n", s->dev[k], cudaGetErrorString (e));
      cudaSetDevice (cur);
      bmg_shard_free (s);
      return FAIL (BMG_ECUDA);
    }
  }
  cudaSetDevice (cur);
  /* the blocks of a device share its stream */
  for (int b = 0; b < nb; b++) {
    s->blk[b] = blocks[b];
    int r = bmg_set_stream (blocks[b], s->stream[s->bdev[b]]);
    if (r) { bmg_shard_free (s); return FAIL (r); }
  }
  *out = s;
  return BMG_OK;
}

/* every stream waits for the work issued so far on every other stream */
static int sync_devices (bmg_shard * s)
{
  if (s->ndev < 2) return BMG_OK;
  for (int k = 0; k < s->ndev; k++) {
    CKS (cudaSetDevice (s->dev[k]));
    CKS (cudaEventRecord (s->ev[k], s->stream[k]));
  }
  for (int k = 0; k < s->ndev; k++) {
    CKS (cudaSetDevice (s->dev[k]));
    for (int j = 0; j < s->ndev; j++)
      if (j != k) CKS (cudaStreamWaitEvent (s->stream[k], s->ev[j], 0));
  }
  return BMG_OK;
}

/* mpi_boundary_level (multigrid-mpi.h:52-85) of a level array of every
   block: ptr (b) is the level-l array of block b.  Direction by direction,
   one bmg_launch_halo per device copies the neighbours' edge slabs into
   the ghost slabs of its blocks (reading a neighbour on another device by
   peer access); every device has finished a direction before any starts
   the next, so that the slabs of the later directions carry the ghosts of
   the earlier ones (edges and corners). */
typedef double * (*lvptr_t) (bmg_shard * s, int b, int l, void * data);

static int exchange (bmg_shard * s, int l, lvptr_t ptr, void * data)
{
  const bmg_geom g = s->blk[0]->g64[l];
  for (int e = 0; e < s->dim; e++) {
    if (s->dims[e] == 1) continue;     /* nothing to exchange: box or own periodic images */
    int r = sync_devices (s);
    if (r) return r;
    for (int k = 0; k < s->ndev; k++) {
      int m = 0;
      for (int b = 0; b < s->nb; b++) {
        if (s->bdev[b] != k) continue;
        const int lo = s->nbr[b][2*e + 1], hi = s->nbr[b][2*e];
        if (lo < 0 && hi < 0) continue;
        s->halo[m].dst = ptr (s, b, l, data);
        s->halo[m].lo = lo >= 0 ? ptr (s, lo, l, data) : NULL;
        s->halo[m].hi = hi >= 0 ? ptr (s, hi, l, data) : NULL;
        m++;
      }
      if (!m) continue;
      CKS (cudaSetDevice (s->dev[k]));
      CLS (bmg_launch_halo (s->dim, g, e, s->halo, m, s->stream[k]));
      s->nhalo++;
    }
    r = sync_devices (s);
    if (r) return r;
  }
  return BMG_OK;
}

/* ------------------------------------------------------------------ */
/* the solve                                                           */
/* ------------------------------------------------------------------ */

typedef struct {
  field_t * a, * b, * res;
  bmg_coef alpha[BMG_MAXLEVEL + 1][3], lambda[BMG_MAXLEVEL + 1];
  int alpha_stored, lambda_stored;
  bmg_bcdesc abc, dabc;
} blk_t;

static double * ptr_a (bmg_shard * s, int b, int l, void * data)
{
  (void) s;
  return ((blk_t *) data)[b].a->lv[l];
}

static double * ptr_da (bmg_shard * s, int b, int l, void * data)
{
  (void) data;
  return bmg_i_ws64 (s->blk[b], BMG_WS_DA, l);
}

static double delta_of (const bmg_grid * g, int l) { return g->L0*(1./(1 << l)); }

static int level0_periodic (const bmg_grid * g, int l)
{
  return l == 0 && (g->periodic[0] || g->periodic[1] || g->periodic[2]);
}

/* the Poisson coefficients of block g: unityf / zeroc defaults
   (poisson.h:410-413), per level, and restriction ({alpha, lambda})
   (poisson.h:418-420) */
static int block_coefs (bmg_grid * g, const struct Poisson * p, blk_t * k)
{
  const int ah[3] = {p->alpha.x.i, p->alpha.y.i, p->alpha.z.i};
  for (int l = 0; l <= g->depth; l++) {
    for (int d = 0; d < 3; d++) { k->alpha[l][d].p = NULL; k->alpha[l][d].c = 1.; }
    k->lambda[l].p = NULL; k->lambda[l].c = 0.;
  }
  k->alpha_stored = k->lambda_stored = 0;
  if (ah[0])
    for (int d = 0; d < g->dim; d++) {
      field_t * f = bmg_i_field (g, ah[d]);
      if (!f || f->face_dim != d) return FAIL (BMG_EINVAL);
      for (int l = 0; l <= g->depth; l++) {
        if (f->is_const) k->alpha[l][d].c = f->cval;
        else k->alpha[l][d].p = f->lv[l];
      }
      if (!f->is_const) k->alpha_stored = 1;
    }
  if (p->lambda.i) {
    field_t * f = bmg_i_field (g, p->lambda.i);
    if (!f || f->face_dim >= 0) return FAIL (BMG_EINVAL);
    for (int l = 0; l <= g->depth; l++) {
      if (f->is_const) k->lambda[l].c = f->cval;
      else k->lambda[l].p = f->lv[l];
    }
    if (!f->is_const) k->lambda_stored = 1;
  }
  for (int l = g->depth - 1; l >= 0; l--) {
    if (k->alpha_stored) {
      const double * fine[3] = {0, 0, 0};
      double * coarse[3] = {0, 0, 0};
      for (int d = 0; d < g->dim; d++) {
        fine[d] = (const double *) k->alpha[l + 1][d].p;
        coarse[d] = (double *) k->alpha[l][d].p;
      }
      CLS (bmg_launch_restrict_face (g->dim, g->g64[l + 1], g->g64[l], fine, coarse,
                                     level0_periodic (g, l), g->stream));
    }
    if (k->lambda_stored)
      CLS (bmg_launch_restrict (g->dim, BMG_ST_F64, BMG_ST_F64, g->g64[l + 1], g->g64[l],
                                k->lambda[l + 1].p, (void *) k->lambda[l].p, g->stream));
  }
  return BMG_OK;
}

/* the residual of every block (after the exchange of a), each block's
   maximum into its pinned host word; with done, an event on block 0's
   stream after every device's residual */
static int residual_issue (bmg_shard * s, blk_t * k, cudaEvent_t done)
{
  const int L = s->blk[0]->depth;
  int r = exchange (s, L, ptr_a, k);
  if (r) return r;
  for (int b = 0; b < s->nb; b++) {
    bmg_grid * g = s->blk[b];
    CKS (cudaSetDevice (g->device));
    CKS (cudaMemsetAsync (g->d_maxres, 0, sizeof (unsigned long long), g->stream));
    CLS (bmg_launch_residual (g->dim, BMG_ST_F64, g->g64[L], g->g64[L], k[b].a->lv[L],
                              k[b].b->lv[L], k[b].alpha[L], k[b].lambda[L], delta_of (g, L),
                              bmg_i_ws64 (g, BMG_WS_RES, L), g->d_maxres, g->stream));
  }
  if (done) {
    int r2 = sync_devices (s);
    if (r2) return r2;
    CKS (cudaSetDevice (s->blk[0]->device));
    CKS (cudaEventRecord (done, s->blk[0]->stream));
  }
  for (int b = 0; b < s->nb; b++) {
    bmg_grid * g = s->blk[b];
    CKS (cudaSetDevice (g->device));
    CKS (cudaMemcpyAsync (g->h_pinned, g->d_maxres, sizeof (double),
                          cudaMemcpyDeviceToHost, g->stream));
  }
  return BMG_OK;
}

/* max over the blocks of their residual maxima (non-negative doubles, or
   NaN, compared by their bits as the kernels' atomicMax does) */
static int residual_collect (bmg_shard * s, double * maxres)
{
  unsigned long long m = 0;
  for (int b = 0; b < s->nb; b++) {
    bmg_grid * g = s->blk[b];
    CKS (cudaSetDevice (g->device));
    CKS (cudaStreamSynchronize (g->stream));
    unsigned long long v;
    memcpy (&v, &g->h_pinned[0], sizeof v);
    if (v > m) m = v;
  }
  memcpy (maxres, &m, sizeof m);
  return BMG_OK;
}

static int residual_all (bmg_shard * s, blk_t * k, double * maxres, cudaEvent_t done)
{
  int r = residual_issue (s, k, done);
  return r ? r : residual_collect (s, maxres);
}

/* mg_cycle (poisson.h:32-90) over the blocks, one pass per launch, with
   the boundary exchanges of the single-grid cycle */
static long long cells_of (int dim, int l)
{
  long long c = 1;
  for (int d = 0; d < dim; d++) c *= 1LL << l;
  return c;
}

/* the algorithmic bytes of one cycle over all blocks (each array pass once,
   8 bytes a value, ghosts excluded), as the single-grid solve counts them */
static double cycle_bytes (const bmg_shard * s, const blk_t * k, int nrelax, int minlevel,
                           int maxlevel)
{
  const int dim = s->dim, L = s->blk[0]->depth;
  const double narr = 3. + (k->alpha_stored ? dim : 0) + (k->lambda_stored ? 1 : 0);
  double b = 0.;
  for (int l = L - 1; l >= minlevel; l--) b += 8.*(cells_of (dim, l + 1) + cells_of (dim, l));
  for (int l = minlevel; l <= maxlevel; l++) {
    b += 8.*cells_of (dim, l) + (l > minlevel ? 8.*cells_of (dim, l - 1) : 0.);
    b += nrelax*narr*8.*cells_of (dim, l);
  }
  b += 24.*cells_of (dim, L);                                        /* a += da */
  b += 8.*cells_of (dim, L)*(3. + (k->alpha_stored ? dim : 0) + (k->lambda_stored ? 1 : 0));
  return b*s->nb;
}

static int shard_cycle (bmg_shard * s, blk_t * k, int nrelax, int minlevel, int maxlevel,
                        long long * launches)
{
  const int dim = s->dim, L = s->blk[0]->depth;
  const int jacobi = s->blk[0]->relax == BMG_RELAX_JACOBI;
  /* restriction (res) (multigrid-common.h:368-404): interior cells only */
  for (int b = 0; b < s->nb; b++) {
    bmg_grid * g = s->blk[b];
    CKS (cudaSetDevice (g->device));
    for (int l = L - 1; l >= minlevel; l--) {
      CLS (bmg_launch_restrict (dim, BMG_ST_F64, BMG_ST_F64, g->g64[l + 1], g->g64[l],
                                bmg_i_ws64 (g, BMG_WS_RES, l + 1), bmg_i_ws64 (g, BMG_WS_RES, l),
                                g->stream));
      (*launches)++;
    }
  }
  for (int l = minlevel; l <= maxlevel; l++) {
    for (int b = 0; b < s->nb; b++) {
      bmg_grid * g = s->blk[b];
      CKS (cudaSetDevice (g->device));
      double * da = bmg_i_ws64 (g, BMG_WS_DA, l);
      if (l == minlevel)
        CLS (bmg_launch_prolong (dim, BMG_ST_F64, BMG_ST_F64, g->g64[l], g->g64[l], NULL, da,
                                 &k[b].dabc, 1, g->stream));
      else
        CLS (bmg_launch_prolong (dim, BMG_ST_F64, BMG_ST_F64, g->g64[l - 1], g->g64[l],
                                 bmg_i_ws64 (g, BMG_WS_DA, l - 1), da, &k[b].dabc, 0, g->stream));
      (*launches)++;
    }
    int r = exchange (s, l, ptr_da, k);
    if (r) return r;
    for (int i = 0; i < nrelax; i++) {
      const int passes = jacobi ? 1 : 2;
      for (int c = 0; c < passes; c++) {
        for (int b = 0; b < s->nb; b++) {
          bmg_grid * g = s->blk[b];
          CKS (cudaSetDevice (g->device));
          double * da = bmg_i_ws64 (g, BMG_WS_DA, l);
          double * res = bmg_i_ws64 (g, BMG_WS_RES, l);
          if (jacobi) {
            /* out = (da + 2 n/d)/3 into the partner, then copied back so
               that da stays the current iterate */
            double * da2 = bmg_i_ws64 (g, BMG_WS_DA2, l);
            CLS (bmg_launch_relax (dim, BMG_ST_F64, BMG_SWEEP_JACOBI, g->g64[l], da2, da, res,
                                   k[b].alpha[l], k[b].lambda[l], delta_of (g, l), &k[b].dabc,
                                   g->stream));
            CKS (cudaMemcpyAsync (da, da2, g->g64[l].size*sizeof (double),
                                  cudaMemcpyDeviceToDevice, g->stream));
          }
          else
            CLS (bmg_launch_relax (dim, BMG_ST_F64, c ? BMG_SWEEP_BLACK : BMG_SWEEP_RED,
                                   g->g64[l], da, da, res, k[b].alpha[l], k[b].lambda[l],
                                   delta_of (g, l), &k[b].dabc, g->stream));
          (*launches)++;
        }
        r = exchange (s, l, ptr_da, k);
        if (r) return r;
      }
    }
  }
  /* a += da with the boundary conditions of a (poisson.h:84-89) */
  for (int b = 0; b < s->nb; b++) {
    bmg_grid * g = s->blk[b];
    CKS (cudaSetDevice (g->device));
    CLS (bmg_launch_correct (dim, BMG_ST_F64, g->g64[L], g->g64[L], k[b].a->lv[L],
                             bmg_i_ws64 (g, BMG_WS_DA, L), &k[b].abc, g->stream));
    (*launches)++;
  }
  return BMG_OK;
}

int bmg_shard_poisson (bmg_shard * s, struct Poisson p, mgstats * out)
{
  if (!s || !out) return FAIL (BMG_EINVAL);
  const int L = s->blk[0]->depth;
  int cur = 0;
  cudaGetDevice (&cur);
  blk_t * k = calloc (s->nb, sizeof (blk_t));
  if (!k) return FAIL (BMG_ENOMEM);
  int r = BMG_OK;
  for (int b = 0; b < s->nb && !r; b++) {
    bmg_grid * g = s->blk[b];
    cudaSetDevice (g->device);
    k[b].a = bmg_i_field (g, p.a.i);
    k[b].b = bmg_i_field (g, p.b.i);
    if (!k[b].a || !k[b].b || k[b].a->face_dim >= 0 || k[b].b->face_dim >= 0 ||
        k[b].a->is_const || k[b].b->is_const) { r = FAIL (BMG_EINVAL); break; }
    if (p.res && p.res[0].i) {
      k[b].res = bmg_i_field (g, p.res[0].i);
      if (!k[b].res || k[b].res->face_dim >= 0 || k[b].res->is_const) { r = FAIL (BMG_EINVAL); break; }
    }
    r = bmg_i_workspace (g);
    if (!r) r = block_coefs (g, &p, &k[b]);
    if (!r) {
      bmg_i_bcdesc (g, k[b].a, &k[b].abc);
      k[b].dabc = k[b].abc;
    }
  }
  if (r) { free (k); cudaSetDevice (cur); return r; }
  const int minlevel = p.minlevel > 1 ? (p.minlevel < L ? p.minlevel : L) : (L < 1 ? L : 1);
  const double tolerance = p.tolerance ? p.tolerance : TOLERANCE;
  mgstats st;
  memset (&st, 0, sizeof st);
  long long launches = 0;
  s->nhalo = 0;
  /* the sum of b over every block (an MPI_Allreduce in the reference) */
  for (int b = 0; b < s->nb && !r; b++) {
    bmg_grid * g = s->blk[b];
    cudaSetDevice (g->device);
    r = bmg_launch_sum (s->dim, g->g64[L], k[b].b->lv[L], g->d_partials, g->npartials,
                        g->d_sum, g->stream);
    if (!r && cudaMemcpyAsync (g->h_pinned + 1, g->d_sum, sizeof (double),
                               cudaMemcpyDeviceToHost, g->stream) != cudaSuccess)
      r = BMG_ECUDA;
    if (!r && cudaStreamSynchronize (g->stream) != cudaSuccess) r = BMG_ECUDA;
    if (!r) st.sum += g->h_pinned[1];
  }
  if (r) { free (k); cudaSetDevice (cur); return FAIL (BMG_ECUDA); }
  st.nrelax = p.nrelax > 0 ? p.nrelax : 4;
  r = residual_all (s, k, &st.resb, NULL);
  double resb = st.resa = st.resb;
  int status = BMG_OK;
  bmg_grid * g0 = s->blk[0];
  for (st.i = 0; !r && st.i < NITERMAX && (st.i < NITERMIN || st.resa > tolerance); st.i++) {
    /* with timing on, the cycle and its residual between two events on
       block 0's stream, which waits for every device at both ends */
    if (g0->timing) {
      r = sync_devices (s);
      if (!r && (cudaSetDevice (g0->device) != cudaSuccess ||
                 cudaEventRecord (g0->ev0, g0->stream) != cudaSuccess)) r = FAIL (BMG_ECUDA);
    }
    const double bytes = cycle_bytes (s, k, st.nrelax, minlevel, L);
    if (!r) r = shard_cycle (s, k, st.nrelax, minlevel, L, &launches);
    if (!r) r = residual_all (s, k, &st.resa, g0->timing ? g0->ev1 : NULL);
    if (r) break;
    g0->counters.cycles++;
    g0->counters.bytes += bytes;
    if (g0->timing) {
      float ms = 0.f;
      cudaSetDevice (g0->device);
      if (cudaEventElapsedTime (&ms, g0->ev0, g0->ev1) != cudaSuccess) { r = FAIL (BMG_ECUDA); break; }
      g0->counters.cycle_ms += ms;
    }
    if (!isfinite (st.resa)) { status = BMG_ENAN; st.i++; break; }
    /* nrelax adaptation (poisson.h:198-204) */
    if (st.resa > tolerance) {
      if (resb/st.resa < 1.2 && st.nrelax < 100)
        st.nrelax++;
      else if (resb/st.resa > 10 && st.nrelax > 2)
        st.nrelax--;
    }
    resb = st.resa;
  }
  s->blk[0]->counters.launches += launches + s->nhalo;
  s->nhalo = 0;
  if (!r) {
    st.minlevel = minlevel;
    if (st.resa > tolerance) {
      fprintf (stderr,
               "WARNING: convergence for %s not reached after %d iterations\n"
               "  res: %g sum: %g nrelax: %d\n", "a",
               st.i, st.resa, st.sum, st.nrelax), fflush (stderr);
      if (status == BMG_OK) status = BMG_ENOTCONV;
    }
    for (int b = 0; b < s->nb && !r; b++)
      if (k[b].res) {
        bmg_grid * g = s->blk[b];
        cudaSetDevice (g->device);
        if (cudaMemcpyAsync (k[b].res->lv[L], bmg_i_ws64 (g, BMG_WS_RES, L),
                             g->g64[L].size*sizeof (double), cudaMemcpyDeviceToDevice,
                             g->stream) != cudaSuccess ||
            cudaStreamSynchronize (g->stream) != cudaSuccess)
          r = FAIL (BMG_ECUDA);
      }
    *out = st;
  }
  free (k);
  cudaSetDevice (cur);
  return r ? r : FAIL (status);
}

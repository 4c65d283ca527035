/*
 * mg_host.c -- C host layer of the B200 multigrid Poisson--Helmholtz solver.
 *
 * Grid and field management (the device counterpart of grid/multigrid.h and
 * grid/cartesian-common.h), and the control flow of Basilisk's poisson.h:
 * poisson() (poisson.h:402-441), mg_solve() (poisson.h:139-235) and
 * mg_cycle() (poisson.h:32-90).  Every arithmetic operation on field data
 * runs on the device through the launchers of mg_kernels.cu; this file only
 * sequences them, adapts nrelax and reads one 8-byte residual maximum back
 * per cycle.  There is no CPU fallback: without a CUDA device every entry
 * point fails with BMG_ENODEV.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <cuda_runtime_api.h>

#include "basilisk_mg.h"
#include "mg_launch.h"
#include "mg_grid.h"

int NITERMAX = 100, NITERMIN = 1;   /* poisson.h:102 */
double TOLERANCE = 1e-3;            /* poisson.h:103 */

static __thread int last_error = BMG_OK;
static bmg_grid * current_grid = NULL;

#define XO64 4
#define XO32 8
/* levels with at most this many cells are solved by the single-CTA bottom
   kernel on the red-black path */
#define BMG_BOTTOM_CELLS 4096



const char * bmg_error_string (int s)
{
  switch (s) {
  case BMG_OK: return "ok";
  case BMG_EINVAL: return "invalid argument";
  case BMG_ECUDA: return "CUDA runtime error";
  case BMG_ENOMEM: return "device allocation failed";
  case BMG_ENAN: return "residual is not finite";
  case BMG_ENOTCONV: return "tolerance not reached";
  case BMG_EUNSUPPORTED: return "unsupported callbacks (only bmg_relax/bmg_residual run on the device)";
  case BMG_ENODEV: return "no CUDA device";
  }
  return "unknown status";
}

int bmg_last_error (void) { return last_error; }

static int fail (int s) { last_error = s; return s; }

#define CK(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) { \
      fprintf (stderr, "bmg: %s failed: %s (%s:%d)\n", #call,           \
               cudaGetErrorString (e_), __FILE__, __LINE__);             \
      return fail (e_ == cudaErrorMemoryAllocation ? BMG_ENOMEM : BMG_ECUDA); } } while (0)
#define CL(call) do { int e_ = (call); if (e_) { \
      fprintf (stderr, "bmg: launch %s failed: %s (%s:%d)\n", #call,     \
               cudaGetErrorString ((cudaError_t) e_), __FILE__, __LINE__); \
      return fail (BMG_ECUDA); } } while (0)

/* captured V-cycles: the launch sequence of one mg_solve iteration is a
   pure function of its parameters (cycle_key), so each distinct key is
   captured once into a CUDA graph and replayed afterwards */
#define NGRAPH_MAX 256
#define NGRAPH_DEFAULT 64
struct graph_entry {
  int valid;
  unsigned long long stamp;
  void * key;            /* malloc'd copy of the cycle_key */
  size_t keylen;
  cudaGraphExec_t exec;
  work_t w;
};

static void graphs_clear (struct bmg_grid * g)
{
  bmg_tree_graphs_clear (g);
  if (!g->graphs) return;
  for (int i = 0; i < NGRAPH_MAX; i++)
    if (g->graphs[i].valid) {
      cudaGraphExecDestroy (g->graphs[i].exec);
      free (g->graphs[i].key);
      g->graphs[i].valid = 0;
    }
}

/* ------------------------------------------------------------------ */
/* geometry                                                            */
/* ------------------------------------------------------------------ */

static int roundup (int v, int m) { return (v + m - 1)/m*m; }

static bmg_geom make_geom (int dim, int l, int xo, int align)
{
  bmg_geom g;
  memset (&g, 0, sizeof g);
  g.n = 1 << l;
  g.xo = xo;
  g.P = roundup (xo + g.n + 1, align);
  if (dim == 1) { g.plane = 1; g.size = g.P; }
  else if (dim == 2) { g.plane = g.P; g.size = (long long) (g.n + 2)*g.P; }
  else { g.plane = (long long) (g.n + 2)*g.P; g.size = (long long) (g.n + 2)*g.plane; }
  return g;
}

static void init_geometry (bmg_grid * g)
{
  size_t o64 = 0, o32 = 0;
  for (int l = 0; l <= g->depth; l++) {
    g->g64[l] = make_geom (g->dim, l, XO64, 16);
    g->g32[l] = make_geom (g->dim, l, XO32, 32);
    g->off64[l] = o64; g->off32[l] = o32;
    o64 += roundup ((int) 0, 1) + (size_t) ((g->g64[l].size + 63)/64*64);
    o32 += (size_t) ((g->g32[l].size + 63)/64*64);
  }
  g->off64[g->depth + 1] = o64;
  g->off32[g->depth + 1] = o32;
}

static size_t total64 (const bmg_grid * g) { return g->off64[g->depth + 1]; }
static size_t total32 (const bmg_grid * g) { return g->off32[g->depth + 1]; }

static long long ncells (const bmg_grid * g, int l)
{
  long long n = 1;
  for (int d = 0; d < g->dim; d++) n *= (1 << l);
  return n;
}

/* level 0 of a grid with a periodic direction: the reference's periodic
   boundary makes every neighbour of the single cell a copy of it */
static int level0_periodic (const bmg_grid * g, int l)
{
  return l == 0 && (g->periodic[0] || g->periodic[1] || g->periodic[2]);
}

static double delta_of (const bmg_grid * g, int l)
{
  return g->L0*(1./(1 << l));    /* cartesian-common.h:11, multigrid.h:14 */
}

/* ------------------------------------------------------------------ */
/* grid                                                                */
/* ------------------------------------------------------------------ */

int bmg_grid_new (bmg_grid ** out, int dim, int depth)
{
  if (!out || dim < 1 || dim > 3 || depth < 0 || depth > BMG_MAXLEVEL)
    return fail (BMG_EINVAL);
  if (dim == 3 && depth > 10) return fail (BMG_EINVAL);
  int ndev = 0;
  if (cudaGetDeviceCount (&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError ();
    return fail (BMG_ENODEV);
  }
  bmg_grid * g = calloc (1, sizeof (bmg_grid));
  if (!g) return fail (BMG_ENOMEM);
  g->dim = dim; g->depth = depth; g->L0 = 1.;
  g->relax = BMG_RELAX_RBGS; g->precision = BMG_FP64; g->use_graphs = NGRAPH_DEFAULT;
  CK (cudaGetDevice (&g->device));
  CK (cudaStreamCreateWithFlags (&g->stream, cudaStreamNonBlocking));
  g->own_stream = 1;
  init_geometry (g);
  g->cap = 16;
  g->fields = calloc (g->cap, sizeof (field_t));
  g->nfields = 1;   /* handle 0 means "unset" */
  CK (cudaMalloc ((void **) &g->d_maxres, 2*sizeof (unsigned long long)));
  g->cluster_levels = getenv ("BMG_NO_CLUSTER") == NULL;
  g->npartials = bmg_sum_partials (dim, g->g64[depth]);
  CK (cudaMalloc ((void **) &g->d_partials, (g->npartials + 1)*sizeof (double)));
  CK (cudaMalloc ((void **) &g->d_sum, 2*sizeof (double)));
  CK (cudaMallocHost ((void **) &g->h_pinned, 4*sizeof (double)));
  CK (cudaEventCreate (&g->ev0));
  CK (cudaEventCreate (&g->ev1));
  CK (cudaEventCreate (&g->evr0));
  CK (cudaEventCreate (&g->evr1));
  g->graphs = calloc (NGRAPH_MAX, sizeof (struct graph_entry));
  *out = g;
  current_grid = g;
  return fail (BMG_OK);
}

void bmg_grid_free (bmg_grid * g)
{
  if (!g) return;
  cudaSetDevice (g->device);
  cudaStreamSynchronize (g->stream);
  graphs_clear (g);
  bmg_tree_free (g);
  free (g->graphs);
  for (int i = 1; i < g->nfields; i++)
    if (g->fields[i].used) {
      cudaFree (g->fields[i].buf);
      for (int s = 0; s < 6; s++) {
        cudaFree (g->fields[i].bcval[s]);
        for (int l = 0; l <= BMG_MAXLEVEL; l++) cudaFree (g->fields[i].bclv[s][l]);
      }
    }
  free (g->fields);
  cudaFree (g->ws64); cudaFree (g->ws32); cudaFree (g->bproj); cudaFree (g->visc_ws);
  cudaFree (g->stage);
  cudaFree (g->d_maxres); cudaFree (g->d_partials); cudaFree (g->d_sum);
  cudaFreeHost (g->h_pinned);
  cudaEventDestroy (g->ev0); cudaEventDestroy (g->ev1);
  cudaEventDestroy (g->evr0); cudaEventDestroy (g->evr1);
  if (g->own_stream) cudaStreamDestroy (g->stream);
  if (current_grid == g) current_grid = NULL;
  free (g);
}

int bmg_grid_select (bmg_grid * g) { if (!g) return fail (BMG_EINVAL); current_grid = g; return BMG_OK; }
bmg_grid * bmg_grid_current (void) { return current_grid; }

int bmg_grid_info (const bmg_grid * g, int * dim, int * depth)
{
  if (!g) return fail (BMG_EINVAL);
  if (dim) *dim = g->dim;
  if (depth) *depth = g->depth;
  return BMG_OK;
}

int bmg_origin (bmg_grid * g, double x, double y, double z)
{
  if (!g) return fail (BMG_EINVAL);
  if (g->X0 != x || g->Y0 != y || g->Z0 != z) graphs_clear (g);   /* boundary data */
  g->X0 = x; g->Y0 = y; g->Z0 = z;
  return BMG_OK;
}

int bmg_size (bmg_grid * g, double L0)
{
  if (!g || !(L0 > 0.)) return fail (BMG_EINVAL);
  if (g->L0 != L0) graphs_clear (g);     /* Delta is a launch argument */
  g->L0 = L0;
  return BMG_OK;
}

static int refresh_bc_ghosts (bmg_grid * g, int h);

/* periodic (cartesian-common.h:920-933): both sides of the direction, for
   every field of the grid */
int bmg_periodic (bmg_grid * g, int dir)
{
  if (!g || dir < 0 || dir >= 2*g->dim) return fail (BMG_EINVAL);
  int d = dir/2;
  g->periodic[d] = 1;
  for (int i = 1; i < g->nfields; i++)
    if (g->fields[i].used) {
      g->fields[i].bctype[2*d] = g->fields[i].bctype[2*d + 1] = BMG_PERIODIC;
      if (g->fields[i].face_dim < 0 && !g->fields[i].is_const) {
        int s = refresh_bc_ghosts (g, i);
        if (s) return s;
      }
    }
  graphs_clear (g);
  return BMG_OK;
}

int bmg_set_relax (bmg_grid * g, int relax)
{
  if (!g || (relax != BMG_RELAX_RBGS && relax != BMG_RELAX_JACOBI)) return fail (BMG_EINVAL);
  g->relax = relax;
  return BMG_OK;
}

int bmg_set_precision (bmg_grid * g, int p)
{
  if (!g || (p != BMG_FP64 && p != BMG_MIXED)) return fail (BMG_EINVAL);
  g->precision = p;
  return BMG_OK;
}

int bmg_set_stream (bmg_grid * g, void * stream)
{
  if (!g) return fail (BMG_EINVAL);
  cudaSetDevice (g->device);
  cudaStreamSynchronize (g->stream);
  if (g->own_stream && stream) { cudaStreamDestroy (g->stream); g->own_stream = 0; }
  if (stream) g->stream = (cudaStream_t) stream;
  else if (!g->own_stream) {
    CK (cudaStreamCreateWithFlags (&g->stream, cudaStreamNonBlocking));
    g->own_stream = 1;
  }
  graphs_clear (g);
  return BMG_OK;
}

int bmg_synchronize (bmg_grid * g)
{
  if (!g) return fail (BMG_EINVAL);
  CK (cudaStreamSynchronize (g->stream));
  return BMG_OK;
}

int bmg_set_graphs (bmg_grid * g, int n)
{
  if (!g || n < 0) return fail (BMG_EINVAL);
  graphs_clear (g);
  g->use_graphs = n == 1 ? NGRAPH_DEFAULT : n > NGRAPH_MAX ? NGRAPH_MAX : n;
  return BMG_OK;
}
int bmg_set_timing (bmg_grid * g, int on) { if (!g) return fail (BMG_EINVAL); g->timing = on; return BMG_OK; }

int bmg_get_counters (bmg_grid * g, bmg_counters * c)
{
  if (!g || !c) return fail (BMG_EINVAL);
  *c = g->counters;
  return BMG_OK;
}

int bmg_reset_counters (bmg_grid * g)
{
  if (!g) return fail (BMG_EINVAL);
  memset (&g->counters, 0, sizeof g->counters);
  return BMG_OK;
}

/* ------------------------------------------------------------------ */
/* fields                                                              */
/* ------------------------------------------------------------------ */

static int new_field (bmg_grid * g, int face_dim, int is_const, double v, int * handle)
{
  if (g->nfields == g->cap) {
    int cap = 2*g->cap;
    field_t * f = realloc (g->fields, cap*sizeof (field_t));
    if (!f) return fail (BMG_ENOMEM);
    memset (f + g->cap, 0, (cap - g->cap)*sizeof (field_t));
    g->fields = f; g->cap = cap;
  }
  int h = g->nfields++;
  field_t * f = &g->fields[h];
  memset (f, 0, sizeof *f);
  f->used = 1; f->face_dim = face_dim; f->is_const = is_const; f->cval = v;
  for (int s = 0; s < 6; s++)
    f->bctype[s] = g->periodic[s/2] ? BMG_PERIODIC : BMG_NEUMANN; /* symmetry */
  if (!is_const) {
    CK (cudaSetDevice (g->device));
    CK (cudaMalloc ((void **) &f->buf, total64 (g)*sizeof (double)));
    CK (cudaMemsetAsync (f->buf, 0, total64 (g)*sizeof (double), g->stream));
    for (int l = 0; l <= g->depth; l++) f->lv[l] = f->buf + g->off64[l];
  }
  *handle = h;
  return BMG_OK;
}

static field_t * field_get (bmg_grid * g, int h)
{
  if (!g || h <= 0 || h >= g->nfields || !g->fields[h].used) return NULL;
  return &g->fields[h];
}

int bmg_scalar_new (bmg_grid * g, bmg_scalar * s)
{
  if (!g || !s) return fail (BMG_EINVAL);
  return new_field (g, -1, 0, 0., &s->i);
}

int bmg_face_vector_new (bmg_grid * g, bmg_vector * v)
{
  if (!g || !v) return fail (BMG_EINVAL);
  int h[3] = {0, 0, 0};
  for (int d = 0; d < g->dim; d++) {
    int s = new_field (g, d, 0, 0., &h[d]);
    if (s) return s;
  }
  v->x.i = h[0]; v->y.i = h[1]; v->z.i = h[2];
  return BMG_OK;
}

int bmg_const_scalar (bmg_grid * g, double value, bmg_scalar * s)
{
  if (!g || !s) return fail (BMG_EINVAL);
  return new_field (g, -1, 1, value, &s->i);
}

int bmg_const_face_vector (bmg_grid * g, double value, bmg_vector * v)
{
  if (!g || !v) return fail (BMG_EINVAL);
  int h[3] = {0, 0, 0};
  for (int d = 0; d < g->dim; d++) {
    int s = new_field (g, d, 1, value, &h[d]);
    if (s) return s;
  }
  v->x.i = h[0]; v->y.i = h[1]; v->z.i = h[2];
  return BMG_OK;
}

int bmg_field_delete (bmg_grid * g, bmg_scalar s)
{
  field_t * f = field_get (g, s.i);
  if (!f) return fail (BMG_EINVAL);
  cudaSetDevice (g->device);
  cudaStreamSynchronize (g->stream);
  cudaFree (f->buf);
  for (int k = 0; k < 6; k++) {
    cudaFree (f->bcval[k]);
    for (int l = 0; l <= BMG_MAXLEVEL; l++) cudaFree (f->bclv[k][l]);
  }
  memset (f, 0, sizeof *f);
  graphs_clear (g);
  return BMG_OK;
}

static size_t field_count (const bmg_grid * g, int l, int face_dim)
{
  size_t c = 1;
  for (int d = 0; d < g->dim; d++) c *= (size_t) (1 << l) + (d == face_dim);
  return c;
}

/* the grid's staging buffer for host values, grown on demand and kept
   (set and get are synchronous, so one buffer serves every call) */
static double * stage_buf (bmg_grid * g, size_t count)
{
  if (g->stage_n < count) {
    cudaStreamSynchronize (g->stream);
    cudaFree (g->stage);
    g->stage = NULL;
    g->stage_n = 0;
    if (cudaMalloc ((void **) &g->stage, count*sizeof (double)) != cudaSuccess) {
      g->stage = NULL;
      return NULL;
    }
    g->stage_n = count;
  }
  return g->stage;
}

/* staging: compact values on the device (copied from the host if needed) */
static int stage_in (bmg_grid * g, const double * values, size_t count, int memory,
                     const double ** dptr)
{
  if (memory == BMG_DEVICE) { *dptr = values; return BMG_OK; }
  double * tmp = stage_buf (g, count);
  if (!tmp) return fail (BMG_ENOMEM);
  CK (cudaMemcpyAsync (tmp, values, count*sizeof (double), cudaMemcpyHostToDevice, g->stream));
  *dptr = tmp;
  return BMG_OK;
}

static int refresh_bc_ghosts (bmg_grid * g, int h);

int bmg_field_set_level (bmg_grid * g, bmg_scalar s, int level, const double * values,
                         size_t count, int memory)
{
  field_t * f = field_get (g, s.i);
  if (!f || f->is_const || !values || level < 0 || level > g->depth ||
      count != field_count (g, level, f->face_dim))
    return fail (BMG_EINVAL);
  CK (cudaSetDevice (g->device));
  const double * d;
  int st = stage_in (g, values, count, memory, &d);
  if (st) return st;
  CL (bmg_launch_pack (g->dim, BMG_ST_F64, g->g64[level], f->face_dim, d, f->lv[level], g->stream));
  if (f->face_dim >= 0 && (g->periodic[f->face_dim] || level0_periodic (g, level)))
    /* periodic face vectors: the last face is the image of the first
       (periodic_boundary_level_x copies face vectors, multigrid.h:644-647);
       on a periodic level 0 every neighbour slot takes the cell's value,
       the upper face of every component included (multigrid.h:655-664) */
    CL (bmg_launch_face_wrap (g->dim, g->g64[level], f->face_dim, f->lv[level], g->stream));
  if (f->face_dim < 0 && level == g->depth) {
    int r = refresh_bc_ghosts (g, s.i);
    if (r) return r;
  }
  CK (cudaStreamSynchronize (g->stream));
  return BMG_OK;
}

int bmg_field_set (bmg_grid * g, bmg_scalar s, const double * values, size_t count, int memory)
{
  if (!g) return fail (BMG_EINVAL);
  return bmg_field_set_level (g, s, g->depth, values, count, memory);
}

int bmg_field_get_level (bmg_grid * g, bmg_scalar s, int level, double * values,
                         size_t count, int memory)
{
  field_t * f = field_get (g, s.i);
  if (!f || f->is_const || !values || level < 0 || level > g->depth ||
      count != field_count (g, level, f->face_dim))
    return fail (BMG_EINVAL);
  CK (cudaSetDevice (g->device));
  double * d = values, * tmp = NULL;
  if (memory != BMG_DEVICE) {
    if (!(tmp = stage_buf (g, count))) return fail (BMG_ENOMEM);
    d = tmp;
  }
  CL (bmg_launch_unpack (g->dim, g->g64[level], f->face_dim, f->lv[level], d, g->stream));
  if (tmp)
    CK (cudaMemcpyAsync (values, tmp, count*sizeof (double), cudaMemcpyDeviceToHost, g->stream));
  CK (cudaStreamSynchronize (g->stream));
  return BMG_OK;
}

int bmg_field_get (bmg_grid * g, bmg_scalar s, double * values, size_t count, int memory)
{
  if (!g) return fail (BMG_EINVAL);
  return bmg_field_get_level (g, s, g->depth, values, count, memory);
}

static void bcdesc_of (const bmg_grid * g, const field_t * f, bmg_bcdesc * bc)
{
  memset (bc, 0, sizeof *bc);
  for (int d = 0; d < 3; d++) bc->periodic[d] = d < g->dim ? g->periodic[d] : 0;
  for (int s = 0; s < 6; s++) {
    bc->type[s] = f ? f->bctype[s] : BMG_NEUMANN;
    bc->val[s] = f ? f->bcval[s] : NULL;
    bc->cval[s] = f ? f->bccval[s] : 0.;
  }
  bc->Delta = delta_of (g, g->depth);
}

/* ghosts of a cell field's finest level from its (inhomogeneous) BCs */
static int refresh_bc_ghosts (bmg_grid * g, int h)
{
  field_t * f = &g->fields[h];
  bmg_bcdesc bc;
  bcdesc_of (g, f, &bc);
  CL (bmg_launch_apply_bc (g->dim, BMG_ST_F64, g->g64[g->depth], f->lv[g->depth], &bc, 0, g->stream));
  return BMG_OK;
}

int bmg_bc (bmg_grid * g, bmg_scalar s, int side, int type, double value,
            const double * values, int memory)
{
  field_t * f = field_get (g, s.i);
  if (!f || side < 0 || side >= 2*g->dim ||
      (type != BMG_NEUMANN && type != BMG_DIRICHLET) || f->face_dim >= 0)
    return fail (BMG_EINVAL);
  if (g->periodic[side/2]) return fail (BMG_EINVAL);
  CK (cudaSetDevice (g->device));
  f->bctype[side] = type;
  f->bccval[side] = value;
  if (f->bcval[side]) { CK (cudaFree (f->bcval[side])); f->bcval[side] = NULL; }
  if (values) {
    size_t n = 1;
    for (int d = 1; d < g->dim; d++) n *= (size_t) 1 << g->depth;
    CK (cudaMalloc ((void **) &f->bcval[side], n*sizeof (double)));
    CK (cudaMemcpyAsync (f->bcval[side], values, n*sizeof (double),
                         memory == BMG_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                         g->stream));
  }
  if (!f->is_const) {
    int r = refresh_bc_ghosts (g, s.i);
    if (r) return r;
  }
  CK (cudaStreamSynchronize (g->stream));
  graphs_clear (g);
  return BMG_OK;
}

int bmg_bc_level (bmg_grid * g, bmg_scalar s, int side, int type, int level,
                  const double * values, int memory)
{
  field_t * f = field_get (g, s.i);
  if (!f || side < 0 || side >= 2*g->dim || level < 0 || level > g->depth || !values ||
      (type != BMG_NEUMANN && type != BMG_DIRICHLET) || f->face_dim >= 0 ||
      (memory != BMG_HOST && memory != BMG_DEVICE))
    return fail (BMG_EINVAL);
  if (g->periodic[side/2]) return fail (BMG_EINVAL);
  CK (cudaSetDevice (g->device));
  f->bctype[side] = type;
  size_t n = 1;
  for (int d = 1; d < g->dim; d++) n *= (size_t) 1 << level;
  if (!f->bclv[side][level])
    CK (cudaMalloc ((void **) &f->bclv[side][level], n*sizeof (double)));
  CK (cudaMemcpyAsync (f->bclv[side][level], values, n*sizeof (double),
                       memory == BMG_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                       g->stream));
  CK (cudaStreamSynchronize (g->stream));
  graphs_clear (g);
  return BMG_OK;
}

/* ------------------------------------------------------------------ */
/* workspace                                                           */
/* ------------------------------------------------------------------ */

enum { WS_DA = 0, WS_DA2 = 1, WS_RES = 2 };
enum { W32_DA = 0, W32_DA2, W32_RES, W32_AX, W32_AY, W32_AZ, W32_LAMBDA, W32_N };

static double * ws64 (bmg_grid * g, int which, int l)
{
  return g->ws64 + which*total64 (g) + g->off64[l];
}

static float * ws32 (bmg_grid * g, int which, int l)
{
  return g->ws32 + which*total32 (g) + g->off32[l];
}

static int ensure_workspace (bmg_grid * g, int mixed)
{
  if (!g->ws64) {
    CK (cudaMalloc ((void **) &g->ws64, 3*total64 (g)*sizeof (double)));
    CK (cudaMemsetAsync (g->ws64, 0, 3*total64 (g)*sizeof (double), g->stream));
  }
  if (mixed && !g->ws32) {
    CK (cudaMalloc ((void **) &g->ws32, W32_N*total32 (g)*sizeof (float)));
    CK (cudaMemsetAsync (g->ws32, 0, W32_N*total32 (g)*sizeof (float), g->stream));
  }
  /* the zero-mean copy of b of the mixed form's singular problems: part of
     the workspace, so that a solve itself allocates nothing */
  if (mixed && !g->bproj)
    CK (cudaMalloc ((void **) &g->bproj, g->g64[g->depth].size*sizeof (double)));
  return BMG_OK;
}

int bmg_i_fail (int status) { return fail (status); }
void bmg_i_bcdesc (const bmg_grid * g, const field_t * f, bmg_bcdesc * bc) { bcdesc_of (g, f, bc); }
field_t * bmg_i_field (bmg_grid * g, int handle) { return field_get (g, handle); }
int bmg_i_workspace (bmg_grid * g) { return ensure_workspace (g, 0); }
double * bmg_i_ws64 (bmg_grid * g, int which, int level) { return ws64 (g, which, level); }

/* ------------------------------------------------------------------ */
/* the solver proper                                                   */
/* ------------------------------------------------------------------ */

/* coefficients of one solve, per level and storage type */
typedef struct {
  bmg_coef alpha64[BMG_MAXLEVEL + 1][3], lambda64[BMG_MAXLEVEL + 1];
  bmg_coef alpha32[BMG_MAXLEVEL + 1][3], lambda32[BMG_MAXLEVEL + 1];
  int alpha_stored, lambda_stored;
} coefs_t;

/* the level arrays a cycle works on */
typedef struct {
  void * da[BMG_MAXLEVEL + 1];
  void * da2[BMG_MAXLEVEL + 1];    /* Jacobi ping-pong partner */
  void * res[BMG_MAXLEVEL + 1];
  int st[BMG_MAXLEVEL + 1];        /* storage type of each level */
} levels_t;

static bmg_geom geom_st (const bmg_grid * g, int l, int st)
{
  return st == BMG_ST_F64 ? g->g64[l] : g->g32[l];
}

static double es_of (int st) { return st == BMG_ST_F64 ? 8. : 4.; }

static int resolve_coefs (bmg_grid * g, bmg_vector alpha, bmg_scalar lambda, coefs_t * c)
{
  memset (c, 0, sizeof *c);
  int ah[3] = {alpha.x.i, alpha.y.i, alpha.z.i};
  if (!ah[0]) {
    /* unityf (poisson.h:410-411) */
    for (int l = 0; l <= g->depth; l++)
      for (int d = 0; d < 3; d++) { c->alpha64[l][d].c = 1.; c->alpha32[l][d].c = 1.; }
  }
  else {
    for (int d = 0; d < g->dim; d++) {
      field_t * f = field_get (g, ah[d]);
      if (!f || f->face_dim != d) return fail (BMG_EINVAL);
      for (int l = 0; l <= g->depth; l++) {
        if (f->is_const) { c->alpha64[l][d].c = f->cval; c->alpha32[l][d].c = f->cval; }
        else c->alpha64[l][d].p = f->lv[l];
      }
      if (!f->is_const) c->alpha_stored = 1;
    }
  }
  if (!lambda.i) {
    for (int l = 0; l <= g->depth; l++) { c->lambda64[l].c = 0.; c->lambda32[l].c = 0.; }
  }
  else {
    field_t * f = field_get (g, lambda.i);
    if (!f || f->face_dim >= 0) return fail (BMG_EINVAL);
    for (int l = 0; l <= g->depth; l++) {
      if (f->is_const) { c->lambda64[l].c = f->cval; c->lambda32[l].c = f->cval; }
      else c->lambda64[l].p = f->lv[l];
    }
    if (!f->is_const) c->lambda_stored = 1;
  }
  return BMG_OK;
}

/* restriction ({alpha, lambda}) (poisson.h:418-420) */
static int restrict_coefs (bmg_grid * g, const coefs_t * c)
{
  for (int l = g->depth - 1; l >= 0; l--) {
    if (c->alpha_stored) {
      const double * fine[3] = {0, 0, 0};
      double * coarse[3] = {0, 0, 0};
      for (int d = 0; d < g->dim; d++) {
        fine[d] = (const double *) c->alpha64[l + 1][d].p;
        coarse[d] = (double *) c->alpha64[l][d].p;
      }
      CL (bmg_launch_restrict_face (g->dim, g->g64[l + 1], g->g64[l], fine, coarse,
                                    level0_periodic (g, l), g->stream));
    }
    if (c->lambda_stored)
      CL (bmg_launch_restrict (g->dim, BMG_ST_F64, BMG_ST_F64, g->g64[l + 1], g->g64[l],
                               c->lambda64[l + 1].p, (void *) c->lambda64[l].p, g->stream));
  }
  return BMG_OK;
}

/* FP32 copies of the coefficients for the inner cycles of the mixed form */
static int convert_coefs (bmg_grid * g, coefs_t * c)
{
  for (int l = 0; l <= g->depth; l++) {
    for (int d = 0; d < g->dim; d++)
      if (c->alpha64[l][d].p) {
        float * dst = ws32 (g, W32_AX + d, l);
        CL (bmg_launch_convert (g->dim, g->g64[l], g->g32[l], d, c->alpha64[l][d].p, dst, g->stream));
        c->alpha32[l][d].p = dst;
      }
    if (c->lambda64[l].p) {
      float * dst = ws32 (g, W32_LAMBDA, l);
      CL (bmg_launch_convert (g->dim, g->g64[l], g->g32[l], -1, c->lambda64[l].p, dst, g->stream));
      c->lambda32[l].p = dst;
    }
  }
  return BMG_OK;
}

static double relax_arrays (const bmg_grid * g, const coefs_t * c)
{
  return 3. + (c->alpha_stored ? g->dim : 0) + (c->lambda_stored ? 1 : 0);
}

/* one residual of the finest level into res (storage st); with sync, the
   maximum is read back into *maxres */
static int residual_max (bmg_grid * g, field_t * a, const double * b, const coefs_t * c,
                         void * res, int st, double * maxres, int sync, work_t * w)
{
  int L = g->depth;
  CK (cudaMemsetAsync (g->d_maxres, 0, sizeof (unsigned long long), g->stream));
  CL (bmg_launch_residual (g->dim, st, g->g64[L], geom_st (g, L, st), a->lv[L], b,
                           c->alpha64[L], c->lambda64[L], delta_of (g, L), res,
                           g->d_maxres, g->stream));
  w->launches += 1;
  w->bytes += ncells (g, L)*(8.*(2. + (c->alpha_stored ? g->dim : 0) +
                                 (c->lambda_stored ? 1 : 0)) + es_of (st));
  if (sync) {
    CK (cudaMemcpyAsync (g->h_pinned, g->d_maxres, sizeof (double), cudaMemcpyDeviceToHost, g->stream));
    CK (cudaStreamSynchronize (g->stream));
    *maxres = g->h_pinned[0];
  }
  return BMG_OK;
}

/* the residual of an mg_solve iteration: on 2D grids fused with the
   restriction of res into the level below, which the next cycle then
   skips (returns 1 when it restricted) */
static int fused_tail (const bmg_grid * g) { return g->dim >= 2 && g->depth >= 1; }

static int residual_tail (bmg_grid * g, field_t * a, const double * b, const coefs_t * c,
                          const levels_t * lv, double * maxres, int sync, work_t * w)
{
  const int L = g->depth;
  if (!fused_tail (g))
    return residual_max (g, a, b, c, lv->res[L], lv->st[L], maxres, sync, w);
  CK (cudaMemsetAsync (g->d_maxres, 0, sizeof (unsigned long long), g->stream));
  if (g->dim == 2)
    CL (bmg_launch_residual_restrict (lv->st[L], lv->st[L - 1], g->g64[L], geom_st (g, L, lv->st[L]),
                                      geom_st (g, L - 1, lv->st[L - 1]), a->lv[L], b,
                                      c->alpha64[L], c->lambda64[L], delta_of (g, L),
                                      lv->res[L], lv->res[L - 1], g->d_maxres, g->stream));
  else
    CL (bmg_launch_residual_restrict3d (lv->st[L], lv->st[L - 1], g->g64[L], geom_st (g, L, lv->st[L]),
                                        geom_st (g, L - 1, lv->st[L - 1]), a->lv[L], b,
                                        c->alpha64[L], c->lambda64[L], delta_of (g, L),
                                        lv->res[L], lv->res[L - 1], g->d_maxres, g->stream));
  w->launches += 1;
  w->bytes += ncells (g, L)*(8.*(2. + (c->alpha_stored ? g->dim : 0) +
                                 (c->lambda_stored ? 1 : 0)) + es_of (lv->st[L])) +
    ncells (g, L - 1)*es_of (lv->st[L - 1]);
  if (sync) {
    CK (cudaMemcpyAsync (g->h_pinned, g->d_maxres, sizeof (double), cudaMemcpyDeviceToHost, g->stream));
    CK (cudaStreamSynchronize (g->stream));
    *maxres = g->h_pinned[0];
  }
  return BMG_OK;
}

/* an event on stream s: a graph node of its own while s is being captured
   (the external flag), a plain record otherwise (the flag is refused
   outside a capture) */
static cudaError_t record_event (cudaEvent_t e, cudaStream_t s)
{
  enum cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaError_t r = cudaStreamIsCapturing (s, &cs);
  if (r != cudaSuccess) return r;
  return cs == cudaStreamCaptureStatusActive ?
    cudaEventRecordWithFlags (e, s, cudaEventRecordExternal) : cudaEventRecord (e, s);
}

/* the levels of the single-CTA bottom solve: minlevel up to the largest
   level with at most BMG_BOTTOM_CELLS cells whose staged arrays fit the
   bottom kernel's shared memory; fills bl[0..top-minlevel] */
static int use_cluster (const bmg_grid * g, const levels_t * lv, int l, int minlevel, int maxlevel);

static int bottom_top (const bmg_grid * g, const levels_t * lv, const coefs_t * c,
                       int minlevel, int maxlevel, bmg_bottom_level * bl)
{
  int top = minlevel - 1;
  for (int l = minlevel; l <= maxlevel; l++) {
    /* in 3D a 16^3 level is 4096 cells of one CTA's generic passes: the
       one-pass launches over the whole device are faster from 16^3 up */
    if (l > minlevel && ncells (g, l) > (g->dim == 3 ? 512 : BMG_BOTTOM_CELLS)) break;
    /* a level that has a cluster kernel is relaxed by it, not by the
       single CTA */
    if (use_cluster (g, lv, l, minlevel, maxlevel)) break;
    bmg_bottom_level * b = &bl[l - minlevel];
    memset (b, 0, sizeof *b);
    b->st = lv->st[l];
    b->g = geom_st (g, l, b->st);
    b->da = lv->da[l];
    b->res = lv->res[l];
    for (int d = 0; d < 3; d++)
      b->alpha[d] = b->st == BMG_ST_F64 ? c->alpha64[l][d] : c->alpha32[l][d];
    b->lambda = b->st == BMG_ST_F64 ? c->lambda64[l] : c->lambda32[l];
    b->Delta = delta_of (g, l);
    b->fast = g->precision == BMG_MIXED;
    if (l > minlevel && bmg_bottom_smem (g->dim, bl, l - minlevel + 1) > BMG_BOTTOM_SMEM) break;
    top = l;
  }
  return top < minlevel ? minlevel : top;
}

/* whether level l of a cycle is relaxed by the cluster level kernel: a
   level of a red-black 2D cycle above minlevel that has such a kernel in
   its storage type (FP32: 64^2 to 256^2; FP64: 64^2 and 128^2), whose
   coarse level has the same storage type; not the finest level while its
   sweeps are being timed */
static int use_cluster (const bmg_grid * g, const levels_t * lv, int l, int minlevel, int maxlevel)
{
  return g->cluster_levels && g->relax == BMG_RELAX_RBGS && g->dim == 2 && l > minlevel &&
    lv->st[l] == lv->st[l - 1] && bmg_level_cluster_ok (lv->st[l], 1 << l) &&
    !(g->timing && l == g->depth && maxlevel == g->depth);
}

/* the launches of one mg_cycle (poisson.h:32-90).  Each level's final
   iterate of da is returned in fin[] (the Jacobi sweeps alternate between
   the da and da2 buffers). */
static int cycle_launches (bmg_grid * g, field_t * a, const levels_t * lv, const coefs_t * c,
                           const bmg_bcdesc * dabc, int nrelax, int minlevel, int maxlevel,
                           int top_restricted, void ** fin, work_t * w)
{
  const int dim = g->dim, L = g->depth;
  cudaStream_t s = g->stream;
  double bytes = 0.;
  long long launches = 0, sweeps = 0;
  bmg_bcdesc abc;                   /* the boundary conditions of a */
  bcdesc_of (g, a, &abc);
  int corrected = 0;
  /* restriction (res) down to minlevel (multigrid-common.h:368-404); on the
     red-black path the levels of the bottom solve are restricted inside it */
  int rlow = minlevel;
  if (g->relax == BMG_RELAX_RBGS) {
    bmg_bottom_level bl[BMG_MAXLEVEL + 1];
    rlow = bottom_top (g, lv, c, minlevel, maxlevel, bl) + 1;
  }
  /* (res of level L - 1 may already be the restriction of the finest
     residual, made by the residual that ended the previous iteration) */
  for (int l = top_restricted ? L - 2 : L - 1; l >= rlow; l--) {
    CL (bmg_launch_restrict (dim, lv->st[l + 1], lv->st[l], geom_st (g, l + 1, lv->st[l + 1]),
                             geom_st (g, l, lv->st[l]), lv->res[l + 1], lv->res[l], s));
    bytes += ncells (g, l + 1)*es_of (lv->st[l + 1]) + ncells (g, l)*es_of (lv->st[l]);
    launches++;
  }
  void * cur[BMG_MAXLEVEL + 1], * oth[BMG_MAXLEVEL + 1];
  const double narr = relax_arrays (g, c);
  int first = minlevel;
  if (g->relax == BMG_RELAX_RBGS) {
    /* the coarse end in one single-CTA launch: levels minlevel..top */
    bmg_bottom_level bl[BMG_MAXLEVEL + 1];
    const int top = bottom_top (g, lv, c, minlevel, maxlevel, bl);
    for (int l = minlevel; l <= top; l++) {
      const int st = lv->st[l];
      cur[l] = lv->da[l]; oth[l] = lv->da2[l];
      if (l < L)   /* restriction of res into this level */
        bytes += ncells (g, l + 1)*es_of (lv->st[l + 1]) + ncells (g, l)*es_of (st);
      bytes += ncells (g, l)*es_of (st);            /* zero or prolongation */
      if (l > minlevel)
        bytes += ncells (g, l - 1)*es_of (lv->st[l - 1]);
      bytes += nrelax*narr*ncells (g, l)*es_of (st);
      sweeps += nrelax;
    }
    const int src = top < L;
    CL (bmg_launch_bottom (dim, bl, top - minlevel + 1,
                           src ? geom_st (g, top + 1, lv->st[top + 1]) : g->g64[L],
                           src ? lv->res[top + 1] : NULL, src ? lv->st[top + 1] : 0, src,
                           nrelax, dabc, s));
    launches++;
    first = top + 1;
  }
  for (int l = first; l <= maxlevel; l++) {
    const int st = lv->st[l];
    const bmg_geom gl = geom_st (g, l, st);
    cur[l] = lv->da[l]; oth[l] = lv->da2[l];
    /* a middle level of the mixed form: prolongation and all nrelax sweeps
       in one thread-block cluster (falls through when it does not apply) */
    if (use_cluster (g, lv, l, minlevel, maxlevel)) {
      const int e = bmg_launch_level_cluster (st, gl, lv->da[l], lv->res[l],
                                              st == BMG_ST_F64 ? c->alpha64[l] : c->alpha32[l],
                                              st == BMG_ST_F64 ? c->lambda64[l] : c->lambda32[l],
                                              delta_of (g, l), dabc, nrelax,
                                              geom_st (g, l - 1, st), cur[l - 1], s);
      if (e > 0) CL (e);
      if (e == 0) {
        bytes += ncells (g, l - 1)*es_of (BMG_ST_F32) + ncells (g, l)*es_of (st);
        bytes += nrelax*narr*ncells (g, l)*es_of (st);
        sweeps += nrelax;
        launches++;
        continue;
      }
    }
    /* the prolongation goes into the level's first tile launch where that
       launch can stage it (red-black tiles, same storage type) */
    const int tiled = g->relax == BMG_RELAX_RBGS && dim == 2;
    const int pfused = tiled && l > minlevel && lv->st[l - 1] == st && bmg_tile_prolongs (st, gl.n);
    if (l == minlevel) {
      /* zero on the coarsest level (poisson.h:54-58) */
      CL (bmg_launch_prolong (dim, st, st, gl, gl, NULL, cur[l], dabc, 1, s));
      bytes += ncells (g, l)*es_of (st);
      launches++;
    }
    else if (pfused)
      bytes += ncells (g, l - 1)*es_of (st);
    else {
      /* bilinear from the coarser level (poisson.h:64-68) */
      const int stc = lv->st[l - 1];
      CL (bmg_launch_prolong (dim, stc, st, geom_st (g, l - 1, stc), gl, cur[l - 1], cur[l], dabc, 0, s));
      bytes += ncells (g, l - 1)*es_of (stc) + ncells (g, l)*es_of (st);
      launches++;
    }
    const bmg_coef * al = st == BMG_ST_F64 ? c->alpha64[l] : c->alpha32[l];
    const bmg_coef la = st == BMG_ST_F64 ? c->lambda64[l] : c->lambda32[l];
    const int timed = g->timing && l == L && maxlevel == L;
    if (timed) CK (record_event (g->evr0, s));
    if (tiled) {
      /* several complete red-black sweeps per launch, ping-pong buffers;
         the first launch of a level stages its prolongation (pfused), the
         last launch of the finest level also applies a += da */
      const int S = bmg_tile_sweeps (st, gl.n);
      const int fuse = l == L && maxlevel == L && bmg_tile_corrects (st, gl.n);
      for (int done = 0; done < nrelax; ) {
        const int k = nrelax - done < S ? nrelax - done : S;
        const int last = fuse && done + k >= nrelax;
        const int pro = pfused && done == 0;
        CL (bmg_launch_relax_tile (dim, st, gl, oth[l], cur[l], lv->res[l], al, la,
                                   delta_of (g, l), dabc, k, last ? a->lv[L] : NULL,
                                   g->g64[L], last ? &abc : NULL, pro ? cur[l - 1] : NULL,
                                   geom_st (g, l - 1, st), s));
        void * t = cur[l]; cur[l] = oth[l]; oth[l] = t;
        launches++;
        done += k;
      }
      if (fuse) {
        corrected = 1;
        bytes += ncells (g, L)*16.;
        if (timed) w->relax_bytes += ncells (g, L)*16.;
      }
    }
    else
      for (int i = 0; i < nrelax; i++) {
        if (g->relax == BMG_RELAX_JACOBI) {
          CL (bmg_launch_relax (dim, st, BMG_SWEEP_JACOBI, gl, oth[l], cur[l], lv->res[l], al, la,
                                delta_of (g, l), dabc, s));
          void * t = cur[l]; cur[l] = oth[l]; oth[l] = t;
          launches++;
        }
        else {
          CL (bmg_launch_relax (dim, st, BMG_SWEEP_RED, gl, cur[l], cur[l], lv->res[l], al, la,
                                delta_of (g, l), dabc, s));
          if (dim == 3 && l == L && maxlevel == L && i == nrelax - 1) {
            /* the finest level's last pass also applies a += da */
            CL (bmg_launch_relax_correct3d (st, gl, cur[l], cur[l], lv->res[l], al, la,
                                            delta_of (g, l), dabc, a->lv[L], g->g64[L], &abc, s));
            corrected = 1;
            bytes += ncells (g, L)*16.;
            if (timed) w->relax_bytes += ncells (g, L)*16.;
          }
          else
            CL (bmg_launch_relax (dim, st, BMG_SWEEP_BLACK, gl, cur[l], cur[l], lv->res[l], al, la,
                                  delta_of (g, l), dabc, s));
          launches += 2;
        }
      }
    bytes += nrelax*narr*ncells (g, l)*es_of (st);
    sweeps += nrelax;
    if (timed) {
      CK (record_event (g->evr1, s));
      w->relax_bytes += nrelax*narr*ncells (g, l)*es_of (st);
      w->relax_sweeps += nrelax;
    }
  }
  /* a += da on the finest level, with the BCs of a (poisson.h:84-89),
     unless the finest level's last tile launch applied it */
  if (!corrected) {
    const int st = lv->st[L];
    CL (bmg_launch_correct (dim, st, g->g64[L], geom_st (g, L, st), a->lv[L], cur[L], &abc, s));
    bytes += ncells (g, L)*(16. + es_of (st));
    launches++;
  }
  for (int l = 0; l <= L; l++)
    fin[l] = (l >= minlevel && l <= maxlevel) ? cur[l] : lv->da[l];
  w->bytes += bytes;
  w->launches += launches;
  w->sweeps += sweeps;
  return BMG_OK;
}

/* everything that determines the launches of one solver iteration */
typedef struct {
  int nrelax, minlevel, relax, precision, dim, depth, timing;
  cudaStream_t stream;
  const void * a, * b;
  levels_t lv;
  coefs_t c;
  bmg_bcdesc dabc, abc;
  const void * maxres, * pinned;
} cycle_key;

/* one mg_solve iteration: mg_cycle, the residual with its maximum, and the
   read-back of that maximum into pinned memory; replayed from a CUDA graph
   when one was captured for the same key. */
static int run_cycle (bmg_grid * g, field_t * a, const double * bdata, const levels_t * lv,
                      const coefs_t * c, const bmg_bcdesc * dabc, int nrelax, int minlevel)
{
  const int L = g->depth;
  cycle_key key;
  memset (&key, 0, sizeof key);
  key.nrelax = nrelax; key.minlevel = minlevel; key.relax = g->relax;
  key.precision = g->precision; key.dim = g->dim; key.depth = L; key.timing = g->timing;
  key.stream = g->stream; key.a = a->lv[L]; key.b = bdata;
  key.lv = *lv; key.c = *c; key.dabc = *dabc;
  bcdesc_of (g, a, &key.abc);
  key.maxres = g->d_maxres; key.pinned = g->h_pinned;

  work_t w = {0., 0, 0, 0., 0};
  void * fin[BMG_MAXLEVEL + 1];
  if (g->use_graphs) {
    struct graph_entry * e = NULL, * victim = &g->graphs[0];
    for (int i = 0; i < g->use_graphs; i++) {
      struct graph_entry * q = &g->graphs[i];
      if (q->valid && q->keylen == sizeof key && !memcmp (q->key, &key, sizeof key)) { e = q; break; }
      if (!q->valid || q->stamp < victim->stamp) victim = q;
    }
    if (!e) {
      if (victim->valid) {
        cudaGraphExecDestroy (victim->exec);
        free (victim->key);
        victim->valid = 0;
      }
      cudaGraph_t graph;
      memset (&victim->w, 0, sizeof victim->w);
      CK (cudaStreamBeginCapture (g->stream, cudaStreamCaptureModeThreadLocal));
      int r = cycle_launches (g, a, lv, c, dabc, nrelax, minlevel, L, fused_tail (g), fin,
                              &victim->w);
      double dummy;
      if (!r) r = residual_tail (g, a, bdata, c, lv, &dummy, 0, &victim->w);
      cudaError_t me = cudaMemcpyAsync (g->h_pinned, g->d_maxres, sizeof (double),
                                        cudaMemcpyDeviceToHost, g->stream);

      cudaError_t ee = cudaStreamEndCapture (g->stream, &graph);
      if (r) return r;
      CK (me);
      CK (ee);
      cudaError_t ie = cudaGraphInstantiate (&victim->exec, graph, 0);
      cudaGraphDestroy (graph);
      CK (ie);
      victim->key = malloc (sizeof key);
      memcpy (victim->key, &key, sizeof key);
      victim->keylen = sizeof key;
      victim->valid = 1;
      e = victim;
    }
    e->stamp = ++g->clock;
    CK (cudaGraphLaunch (e->exec, g->stream));
    w = e->w;
  }
  else {
    int r = cycle_launches (g, a, lv, c, dabc, nrelax, minlevel, L, fused_tail (g), fin, &w);
    if (r) return r;
    double dummy;
    r = residual_tail (g, a, bdata, c, lv, &dummy, 0, &w);
    if (r) return r;
    CK (cudaMemcpyAsync (g->h_pinned, g->d_maxres, sizeof (double), cudaMemcpyDeviceToHost,
                         g->stream));
  }
  g->counters.bytes += w.bytes;
  g->counters.launches += w.launches;
  g->counters.sweeps += w.sweeps;
  if (g->timing) {
    g->counters.relax_bytes += w.relax_bytes;
    g->counters.relax_sweeps += w.relax_sweeps;
  }
  return BMG_OK;
}

static int is_singular (const bmg_grid * g, const field_t * a, const coefs_t * c)
{
  if (c->lambda_stored || c->lambda64[g->depth].c != 0.) return 0;
  for (int s = 0; s < 2*g->dim; s++)
    if (a->bctype[s] == BMG_DIRICHLET) return 0;
  return 1;
}

/* mg_solve (poisson.h:139-235) with the Poisson callbacks */
static int solve (bmg_grid * g, field_t * a, field_t * b, coefs_t * c, int nrelax,
                  field_t * resout, int minlevel, double tolerance, mgstats * out)
{
  const int L = g->depth;
  const int mixed = g->precision == BMG_MIXED;
  int r = ensure_workspace (g, mixed);
  if (r) return r;
  if (minlevel > L) minlevel = L;
  if (minlevel < 0) minlevel = 0;
  if (mixed) { r = convert_coefs (g, c); if (r) return r; }

  /* zeroed: the struct is part of the graph cache key (memcmp), so the
     entries of levels above the depth must not be stack garbage */
  levels_t lv;
  memset (&lv, 0, sizeof lv);
  for (int l = 0; l <= L; l++) {
    int st = (mixed && l != minlevel) ? BMG_ST_F32 : BMG_ST_F64;
    lv.st[l] = st;
    if (st == BMG_ST_F64) {
      lv.da[l] = ws64 (g, WS_DA, l); lv.da2[l] = ws64 (g, WS_DA2, l); lv.res[l] = ws64 (g, WS_RES, l);
    }
    else {
      lv.da[l] = ws32 (g, W32_DA, l); lv.da2[l] = ws32 (g, W32_DA2, l); lv.res[l] = ws32 (g, W32_RES, l);
    }
  }
  bmg_bcdesc dabc;
  bcdesc_of (g, a, &dabc);

  mgstats s;
  memset (&s, 0, sizeof s);
  /* sum of the r.h.s. (poisson.h:162-167) */
  CL (bmg_launch_sum (g->dim, g->g64[L], b->lv[L], g->d_partials, g->npartials, g->d_sum, g->stream));
  CK (cudaMemcpyAsync (g->h_pinned + 1, g->d_sum, sizeof (double), cudaMemcpyDeviceToHost, g->stream));
  CK (cudaStreamSynchronize (g->stream));
  s.sum = g->h_pinned[1];
  s.nrelax = nrelax > 0 ? nrelax : 4;

  /* mixed form, singular problem: FP64 zero-mean projection of b */
  const double * bdata = b->lv[L];
  if (mixed && is_singular (g, a, c)) {
    CK (cudaMemcpyAsync (g->bproj, b->lv[L], g->g64[L].size*sizeof (double),
                         cudaMemcpyDeviceToDevice, g->stream));
    CL (bmg_launch_shift (g->dim, g->g64[L], g->bproj, g->d_sum, 1./(double) ncells (g, L), g->stream));
    bdata = g->bproj;
  }

  double resb;
  work_t w0 = {0., 0, 0, 0., 0};
  r = residual_tail (g, a, bdata, c, &lv, &s.resb, 1, &w0);
  if (r) return r;
  resb = s.resa = s.resb;
  if (tolerance == 0.)
    tolerance = TOLERANCE;
  int status = BMG_OK;
  for (s.i = 0; s.i < NITERMAX && (s.i < NITERMIN || s.resa > tolerance); s.i++) {
    if (g->timing) CK (cudaEventRecord (g->ev0, g->stream));
    r = run_cycle (g, a, bdata, &lv, c, &dabc, s.nrelax, minlevel);
    if (r) return r;
    if (g->timing) CK (cudaEventRecord (g->ev1, g->stream));
    CK (cudaStreamSynchronize (g->stream));
    s.resa = g->h_pinned[0];
    g->counters.cycles++;
    if (g->timing) {
      float ms = 0.f, rms = 0.f;
      CK (cudaEventElapsedTime (&ms, g->ev0, g->ev1));
      CK (cudaEventElapsedTime (&rms, g->evr0, g->evr1));
      g->counters.cycle_ms += ms;
      g->counters.relax_ms += rms;
    }
    if (!isfinite (s.resa)) { status = BMG_ENAN; s.i++; break; }
    /* nrelax adaptation (poisson.h:198-204) */
    if (s.resa > tolerance) {
      if (resb/s.resa < 1.2 && s.nrelax < 100)
        s.nrelax++;
      else if (resb/s.resa > 10 && s.nrelax > 2)
        s.nrelax--;
    }
    resb = s.resa;
  }
  s.minlevel = minlevel;
  if (s.resa > tolerance) {
    fprintf (stderr,
             "WARNING: convergence for %s not reached after %d iterations\n"
             "  res: %g sum: %g nrelax: %d\n", "a",
             s.i, s.resa, s.sum, s.nrelax), fflush (stderr);
    if (status == BMG_OK) status = BMG_ENOTCONV;
  }
  if (resout && !resout->is_const && resout->face_dim < 0) {
    if (lv.st[L] == BMG_ST_F64)
      CK (cudaMemcpyAsync (resout->lv[L], lv.res[L], g->g64[L].size*sizeof (double),
                           cudaMemcpyDeviceToDevice, g->stream));
    else {
      /* widen the FP32 residual: recompute it in FP64 into the caller's field */
      double dummy;
      work_t wr = {0., 0, 0, 0., 0};
      r = residual_max (g, a, bdata, c, resout->lv[L], BMG_ST_F64, &dummy, 0, &wr);
      if (r) return r;
    }
    CK (cudaStreamSynchronize (g->stream));
  }
  *out = s;
  return fail (status);
}

/* ------------------------------------------------------------------ */
/* reference-facing entry points                                       */
/* ------------------------------------------------------------------ */

static int check_cell (bmg_grid * g, int h, field_t ** f)
{
  *f = field_get (g, h);
  if (!*f || (*f)->is_const || (*f)->face_dim >= 0) return fail (BMG_EINVAL);
  return BMG_OK;
}

int bmg_poisson (bmg_grid * g, struct Poisson p, mgstats * out)
{
  mgstats zero;
  memset (&zero, 0, sizeof zero);
  if (out) *out = zero;
  if (!g || !out) return fail (BMG_EINVAL);
  CK (cudaSetDevice (g->device));
  if (g->tree) return bmg_tree_poisson (g, p, out);
  field_t * a, * b, * res = NULL;
  if (check_cell (g, p.a.i, &a) || check_cell (g, p.b.i, &b)) return fail (BMG_EINVAL);
  if (p.res && p.res[0].i && check_cell (g, p.res[0].i, &res)) return fail (BMG_EINVAL);
  coefs_t c;
  int r = resolve_coefs (g, p.alpha, p.lambda, &c);
  if (r) return r;
  r = restrict_coefs (g, &c);
  if (r) return r;
  /* the reference sets TOLERANCE to p.tolerance for the duration of the
     solve and restores it (poisson.h:426-438); mg_solve then reads it.
     Here the solve is given that tolerance directly, which is the same
     solve and leaves the global untouched, so that solves on different
     grids can run from different host threads at once. */
  r = solve (g, a, b, &c, p.nrelax, res, p.minlevel > 1 ? p.minlevel : 1,
             p.tolerance ? p.tolerance : TOLERANCE, out);
  return fail (r);
}

mgstats poisson (struct Poisson p)
{
  mgstats s;
  bmg_poisson (current_grid, p, &s);
  return s;
}

/* project (poisson.h:468-509): div = (sum of uf.x[1] - uf.x[])/(dt Delta),
   poisson (p, div, alpha, tolerance = TOLERANCE/sq(dt), nrelax), then
   uf.x[] -= dt alpha.x[] face_gradient_x (p, 0) on every face */
int bmg_project (bmg_grid * g, struct Project q, mgstats * out)
{
  mgstats zero;
  memset (&zero, 0, sizeof zero);
  if (out) *out = zero;
  if (!g || !out) return fail (BMG_EINVAL);
  if (g->tree) return fail (BMG_EUNSUPPORTED);
  CK (cudaSetDevice (g->device));
  const int L = g->depth;
  /* scalar div[] (poisson.h:482): one field of the grid, created on first
     use (before any field pointer is taken: creation may move the table) */
  if (!g->div_h) {
    int r = new_field (g, -1, 0, 0., &g->div_h);
    if (r) return fail (r);
  }
  field_t * p, * div = field_get (g, g->div_h);
  if (!div || check_cell (g, q.p.i, &p)) return fail (BMG_EINVAL);
  const int uh[3] = {q.uf.x.i, q.uf.y.i, q.uf.z.i};
  double * u[3] = {NULL, NULL, NULL};
  for (int d = 0; d < g->dim; d++) {
    field_t * f = field_get (g, uh[d]);
    if (!f || f->face_dim != d || f->is_const) return fail (BMG_EINVAL);
    u[d] = f->lv[L];
  }
  const double dt = q.dt ? q.dt : 1.;
  const int nrelax = q.nrelax ? q.nrelax : 4;
  CL (bmg_launch_divergence (g->dim, g->g64[L], (const double * const *) u, dt, delta_of (g, L),
                             div->lv[L], g->stream));
  struct Poisson pp;
  memset (&pp, 0, sizeof pp);
  pp.a = q.p;
  pp.b.i = g->div_h;
  pp.alpha = q.alpha;
  pp.tolerance = TOLERANCE/(dt*dt);
  pp.nrelax = nrelax;
  int r = bmg_poisson (g, pp, out);
  if (r != BMG_OK && r != BMG_ENOTCONV) return fail (r);
  coefs_t c;
  bmg_scalar nolambda = {0};
  if (resolve_coefs (g, q.alpha, nolambda, &c)) return fail (BMG_EINVAL);
  for (int d = 0; d < g->dim; d++)
    CL (bmg_launch_project_faces (g->dim, g->g64[L], d, u[d], c.alpha64[L][d], p->lv[L], dt,
                                  delta_of (g, L), g->stream));
  CK (cudaStreamSynchronize (g->stream));
  return fail (r);
}

mgstats project (struct Project q)
{
  mgstats s;
  bmg_project (current_grid, q, &s);
  return s;
}

/* bmg_relax / bmg_residual: the Poisson callbacks (poisson.h:271-391) */
void bmg_relax (bmg_scalar * da, bmg_scalar * res, int l, void * data)
{
  bmg_grid * g = current_grid;
  struct Poisson * p = (struct Poisson *) data;
  field_t * fa, * fr;
  if (!g || !p || !da || !res || check_cell (g, da[0].i, &fa) || check_cell (g, res[0].i, &fr) ||
      l < 0 || l > g->depth) { fail (BMG_EINVAL); return; }
  if (g->tree) { bmg_tree_relax (g, fa, fr, l, p); return; }
  coefs_t c;
  if (resolve_coefs (g, p->alpha, p->lambda, &c)) return;
  bmg_bcdesc bc;
  bcdesc_of (g, fa, &bc);
  if (g->relax == BMG_RELAX_JACOBI) {
    if (ensure_workspace (g, 0)) return;
    double * tmp = ws64 (g, WS_DA2, l);
    if (bmg_launch_relax (g->dim, BMG_ST_F64, BMG_SWEEP_JACOBI, g->g64[l], tmp, fa->lv[l],
                          fr->lv[l], c.alpha64[l], c.lambda64[l], delta_of (g, l), &bc, g->stream) ||
        cudaMemcpyAsync (fa->lv[l], tmp, g->g64[l].size*sizeof (double), cudaMemcpyDeviceToDevice,
                         g->stream) != cudaSuccess) { fail (BMG_ECUDA); return; }
  }
  else if (bmg_launch_relax (g->dim, BMG_ST_F64, BMG_SWEEP_RED, g->g64[l], fa->lv[l], fa->lv[l],
                             fr->lv[l], c.alpha64[l], c.lambda64[l], delta_of (g, l), &bc, g->stream) ||
           bmg_launch_relax (g->dim, BMG_ST_F64, BMG_SWEEP_BLACK, g->g64[l], fa->lv[l], fa->lv[l],
                             fr->lv[l], c.alpha64[l], c.lambda64[l], delta_of (g, l), &bc, g->stream)) {
    fail (BMG_ECUDA); return;
  }
  if (cudaStreamSynchronize (g->stream) != cudaSuccess) { fail (BMG_ECUDA); return; }
  fail (BMG_OK);
}

double bmg_residual (bmg_scalar * al, bmg_scalar * bl, bmg_scalar * resl, void * data)
{
  bmg_grid * g = current_grid;
  struct Poisson * p = (struct Poisson *) data;
  field_t * a, * b, * res;
  if (!g || !p || !al || !bl || !resl || check_cell (g, al[0].i, &a) ||
      check_cell (g, bl[0].i, &b) || check_cell (g, resl[0].i, &res)) {
    fail (BMG_EINVAL);
    return NAN;
  }
  if (g->tree) {
    double m = NAN;
    if (bmg_tree_residual (g, a, b, res, p, &m)) return NAN;
    return m;
  }
  coefs_t c;
  if (resolve_coefs (g, p->alpha, p->lambda, &c)) return NAN;
  double m = NAN;
  work_t w = {0., 0, 0, 0., 0};
  if (residual_max (g, a, b->lv[g->depth], &c, res->lv[g->depth], BMG_ST_F64, &m, 1, &w)) return NAN;
  fail (BMG_OK);
  return m;
}

mgstats mg_solve (struct MGSolve p)
{
  mgstats s;
  memset (&s, 0, sizeof s);
  bmg_grid * g = current_grid;
  if (!g || !p.a || !p.b) { fail (BMG_EINVAL); return s; }
  if (p.residual != bmg_residual || p.relax != bmg_relax || !p.data) {
    fail (BMG_EUNSUPPORTED);
    return s;
  }
  if (cudaSetDevice (g->device) != cudaSuccess) { fail (BMG_ECUDA); return s; }
  if (g->tree) { bmg_tree_mg_solve (g, p, &s); return s; }
  struct Poisson * pp = (struct Poisson *) p.data;
  field_t * a, * b, * res = NULL;
  if (check_cell (g, p.a[0].i, &a) || check_cell (g, p.b[0].i, &b)) return s;
  if (p.res && p.res[0].i && check_cell (g, p.res[0].i, &res)) return s;
  coefs_t c;
  if (resolve_coefs (g, pp->alpha, pp->lambda, &c)) return s;
  /* mg_solve uses the coefficients as they are on each level; poisson()
     restricts them beforehand (poisson.h:420) */
  solve (g, a, b, &c, p.nrelax, res, p.minlevel, p.tolerance, &s);
  return s;
}

void mg_cycle (bmg_scalar * al, bmg_scalar * resl, bmg_scalar * dal,
               void (* relax) (bmg_scalar *, bmg_scalar *, int, void *),
               void * data, int nrelax, int minlevel, int maxlevel)
{
  bmg_grid * g = current_grid;
  if (!g || !al || !resl || !dal || !data) { fail (BMG_EINVAL); return; }
  if (relax != bmg_relax) { fail (BMG_EUNSUPPORTED); return; }
  if (cudaSetDevice (g->device) != cudaSuccess) { fail (BMG_ECUDA); return; }
  struct Poisson * p = (struct Poisson *) data;
  field_t * a, * res, * da;
  if (check_cell (g, al[0].i, &a) || check_cell (g, resl[0].i, &res) ||
      check_cell (g, dal[0].i, &da)) return;
  if (g->tree) { bmg_tree_mg_cycle (g, a, res, da, p, nrelax, minlevel, maxlevel); return; }
  coefs_t c;
  if (resolve_coefs (g, p->alpha, p->lambda, &c)) return;
  if (ensure_workspace (g, 0)) return;
  if (maxlevel > g->depth) maxlevel = g->depth;
  minlevel = minlevel < maxlevel ? minlevel : maxlevel;   /* poisson.h:48 */
  if (minlevel < 0) minlevel = 0;
  levels_t lv;
  memset (&lv, 0, sizeof lv);
  for (int l = 0; l <= g->depth; l++) {
    lv.st[l] = BMG_ST_F64;
    lv.da[l] = da->lv[l];
    lv.da2[l] = ws64 (g, WS_DA2, l);
    lv.res[l] = res->lv[l];
  }
  bmg_bcdesc dabc;
  bcdesc_of (g, da, &dabc);
  void * fin[BMG_MAXLEVEL + 1];
  work_t w = {0., 0, 0, 0., 0};
  if (cycle_launches (g, a, &lv, &c, &dabc, nrelax, minlevel, maxlevel, 0, fin, &w)) return;
  /* Jacobi may leave a level's final iterate in the workspace partner */
  for (int l = minlevel; l <= maxlevel; l++)
    if (fin[l] != da->lv[l])
      if (cudaMemcpyAsync (da->lv[l], fin[l], g->g64[l].size*sizeof (double),
                           cudaMemcpyDeviceToDevice, g->stream) != cudaSuccess) { fail (BMG_ECUDA); return; }
  if (cudaStreamSynchronize (g->stream) != cudaSuccess) { fail (BMG_ECUDA); return; }
  g->counters.bytes += w.bytes;
  g->counters.launches += w.launches;
  g->counters.sweeps += w.sweeps;
  g->counters.cycles++;
  fail (BMG_OK);
}

int bmg_adjoint_gradients (bmg_grid * g, bmg_scalar mu, bmg_scalar a, double * const * grad_alpha,
                           double * grad_lambda, int memory)
{
  field_t * fm, * fa;
  if (!g || check_cell (g, mu.i, &fm) || check_cell (g, a.i, &fa)) return fail (BMG_EINVAL);
  if (g->tree) return fail (BMG_EUNSUPPORTED);
  if (memory != BMG_DEVICE && memory != BMG_HOST) return fail (BMG_EINVAL);
  CK (cudaSetDevice (g->device));
  const int L = g->depth;
  for (int d = 0; d < g->dim; d++) {
    if (!grad_alpha || !grad_alpha[d]) continue;
    const size_t count = field_count (g, L, d);
    double * dst = grad_alpha[d], * tmp = NULL;
    if (memory == BMG_HOST) {
      /* the staging buffer: reused in stream order by the next copy */
      if (!(tmp = stage_buf (g, count))) return fail (BMG_ENOMEM);
      dst = tmp;
    }
    CL (bmg_launch_adjoint_faces (g->dim, g->g64[L], d, g->periodic[d], fm->lv[L], fa->lv[L],
                                  delta_of (g, L), dst, g->stream));
    if (tmp) {
      CK (cudaMemcpyAsync (grad_alpha[d], tmp, count*sizeof (double), cudaMemcpyDeviceToHost, g->stream));
    }
  }
  if (grad_lambda) {
    const size_t count = field_count (g, L, -1);
    double * dst = grad_lambda, * tmp = NULL;
    if (memory == BMG_HOST) {
      /* the staging buffer: reused in stream order by the next copy */
      if (!(tmp = stage_buf (g, count))) return fail (BMG_ENOMEM);
      dst = tmp;
    }
    CL (bmg_launch_adjoint_cells (g->dim, g->g64[L], fm->lv[L], fa->lv[L], dst, g->stream));
    if (tmp) {
      CK (cudaMemcpyAsync (grad_lambda, tmp, count*sizeof (double), cudaMemcpyDeviceToHost, g->stream));
    }
  }
  CK (cudaStreamSynchronize (g->stream));
  return fail (BMG_OK);
}

int bmg_restriction (bmg_grid * g, const bmg_scalar * list)
{
  if (!g || !list) return fail (BMG_EINVAL);
  CK (cudaSetDevice (g->device));
  if (g->tree) return bmg_tree_restriction (g, list);
  for (const bmg_scalar * s = list; s->i; s++) {
    field_t * f = field_get (g, s->i);
    if (!f) return fail (BMG_EINVAL);
    if (f->is_const) continue;
    if (f->face_dim >= 0) {
      /* a face component: restrict the whole vector it belongs to; the
         components of one vector are consecutive handles */
      if (f->face_dim != 0) continue;
      const double * fine[3] = {0, 0, 0};
      double * coarse[3] = {0, 0, 0};
      for (int l = g->depth - 1; l >= 0; l--) {
        for (int d = 0; d < g->dim; d++) {
          field_t * fd = field_get (g, s->i + d);
          if (!fd || fd->face_dim != d) return fail (BMG_EINVAL);
          fine[d] = fd->lv[l + 1]; coarse[d] = fd->lv[l];
        }
        CL (bmg_launch_restrict_face (g->dim, g->g64[l + 1], g->g64[l], fine, coarse,
                                      level0_periodic (g, l), g->stream));
      }
    }
    else
      for (int l = g->depth - 1; l >= 0; l--)
        CL (bmg_launch_restrict (g->dim, BMG_ST_F64, BMG_ST_F64, g->g64[l + 1], g->g64[l],
                                 f->lv[l + 1], f->lv[l], g->stream));
  }
  CK (cudaStreamSynchronize (g->stream));
  return fail (BMG_OK);
}

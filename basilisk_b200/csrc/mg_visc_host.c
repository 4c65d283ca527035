/*
 * mg_visc_host.c -- viscosity () of viscosity.h (implicit viscous step)
 * on the device, uniform grids, two and three dimensions, FP64.
 *
 * viscosity (viscosity.h:169-183) copies u into the r.h.s. r, restricts mu
 * and rho, and calls mg_solve (poisson.h:139-235) on the vector list
 * {u.x, u.y, (u.z)} with residual_viscosity / relax_viscosity
 * (viscosity.h:25-160).  Here the same control flow drives the kernels of
 * mg_kernels.cu: the multigrid transfer operators of the Poisson path on
 * every component, and the coupled relaxation and residual of the
 * viscous operator.  The smoothers are the reference's JACOBI branch, and
 * red-black: each colour computed from the values before it (the
 * same-colour diagonal neighbours the stencil reads keep their old
 * values), then the boundary, then the other colour.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <cuda_runtime_api.h>

#include "mg_grid.h"

#define FAIL(s) bmg_i_fail (s)
#define CKV(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) { \
      fprintf (stderr, "bmg: %s failed: %s (%s:%d)\n", #call,            \
               cudaGetErrorString (e_), __FILE__, __LINE__);              \
      return FAIL (e_ == cudaErrorMemoryAllocation ? BMG_ENOMEM : BMG_ECUDA); } } while (0)
#define LV(call) do { int e_ = (call); if (e_) {                          \
      fprintf (stderr, "bmg: launch %s failed: %s (%s:%d)\n", #call,      \
               cudaGetErrorString ((cudaError_t) e_), __FILE__, __LINE__); \
      return FAIL (BMG_ECUDA); } (*nl)++; } while (0)

typedef struct {
  bmg_grid * g;
  int dim, L;
  double dt;
  double * u[3];                  /* all-level buffers of the fields */
  double * da[3], * res[3], * w[3], * r[3];   /* workspace, all levels */
  bmg_coef mu[BMG_MAXLEVEL + 1][3], rho[BMG_MAXLEVEL + 1];
  bmg_bcdesc bc[3];               /* box conditions of each component of u */
  long long launches;
} visc_t;

static double * at (const visc_t * v, double * base, int l) { return base + v->g->off64[l]; }

static double delta (const bmg_grid * g, int l) { return g->L0*(1./(1 << l)); }

/* residual_viscosity (viscosity.h:91-160) after the boundary of u; the
   maximum goes to g->d_maxres */
static int v_residual (visc_t * v)
{
  bmg_grid * g = v->g;
  const int L = v->L;
  long long * nl = &v->launches;
  double * u[3], * r[3], * res[3];
  for (int c = 0; c < v->dim; c++) {
    LV (bmg_launch_apply_bc (v->dim, BMG_ST_F64, g->g64[L], at (v, v->u[c], L), &v->bc[c], 0, g->stream));
    u[c] = at (v, v->u[c], L); r[c] = at (v, v->r[c], L); res[c] = at (v, v->res[c], L);
  }
  CKV (cudaMemsetAsync (g->d_maxres, 0, sizeof (unsigned long long), g->stream));
  LV (bmg_launch_visc_residual (v->dim, g->g64[L], u, r, res, v->mu[L], v->rho[L], v->dt,
                                delta (g, L), g->d_maxres, g->stream));
  return BMG_OK;
}

static int v_boundary (visc_t * v, int l)
{
  long long * nl = &v->launches;
  for (int c = 0; c < v->dim; c++)
    LV (bmg_launch_apply_bc (v->dim, BMG_ST_F64, v->g->g64[l], at (v, v->da[c], l), &v->bc[c], 1,
                             v->g->stream));
  return BMG_OK;
}

/* relax_viscosity (viscosity.h:25-84) on level l */
static int v_relax (visc_t * v, int l)
{
  bmg_grid * g = v->g;
  long long * nl = &v->launches;
  double * u[3], * res[3], * w[3];
  for (int c = 0; c < v->dim; c++) {
    u[c] = at (v, v->da[c], l); res[c] = at (v, v->res[c], l); w[c] = at (v, v->w[c], l);
  }
  if (g->relax == BMG_RELAX_JACOBI) {
    LV (bmg_launch_visc_relax (v->dim, g->g64[l], 0, u, res, w, v->mu[l], v->rho[l], v->dt,
                               delta (g, l), g->stream));
    LV (bmg_launch_visc_commit (v->dim, g->g64[l], 0, u, w, g->stream));
    return BMG_OK;
  }
  for (int colour = 1; colour <= 2; colour++) {
    if (colour == 2) {
      int r = v_boundary (v, l);
      if (r) return r;
    }
    LV (bmg_launch_visc_relax (v->dim, g->g64[l], colour, u, res, w, v->mu[l], v->rho[l], v->dt,
                               delta (g, l), g->stream));
    LV (bmg_launch_visc_commit (v->dim, g->g64[l], colour, u, w, g->stream));
  }
  return BMG_OK;
}

/* mg_cycle (poisson.h:32-90) on the vector list, minlevel 0 */
static int v_cycle (visc_t * v, int nrelax)
{
  bmg_grid * g = v->g;
  const int L = v->L, dim = v->dim;
  long long * nl = &v->launches;
  for (int c = 0; c < dim; c++)
    for (int l = L - 1; l >= 0; l--)
      LV (bmg_launch_restrict (dim, BMG_ST_F64, BMG_ST_F64, g->g64[l + 1], g->g64[l],
                               at (v, v->res[c], l + 1), at (v, v->res[c], l), g->stream));
  for (int l = 0; l <= L; l++) {
    for (int c = 0; c < dim; c++) {
      if (l == 0)
        LV (bmg_launch_prolong (dim, BMG_ST_F64, BMG_ST_F64, g->g64[l], g->g64[l], NULL,
                                at (v, v->da[c], l), &v->bc[c], 1, g->stream));
      else
        LV (bmg_launch_prolong (dim, BMG_ST_F64, BMG_ST_F64, g->g64[l - 1], g->g64[l],
                                at (v, v->da[c], l - 1), at (v, v->da[c], l), &v->bc[c], 0,
                                g->stream));
    }
    int r = v_boundary (v, l);
    if (r) return r;
    for (int i = 0; i < nrelax; i++) {
      r = v_relax (v, l);
      if (!r) r = v_boundary (v, l);
      if (r) return r;
    }
  }
  for (int c = 0; c < dim; c++)
    LV (bmg_launch_correct (dim, BMG_ST_F64, g->g64[L], g->g64[L], at (v, v->u[c], L),
                            at (v, v->da[c], L), &v->bc[c], g->stream));
  return BMG_OK;
}

static int read_max (bmg_grid * g, double * m)
{
  CKV (cudaMemcpyAsync (g->h_pinned, g->d_maxres, sizeof (double), cudaMemcpyDeviceToHost, g->stream));
  CKV (cudaStreamSynchronize (g->stream));
  *m = g->h_pinned[0];
  return BMG_OK;
}

int bmg_viscosity (bmg_grid * g, struct Viscosity p, mgstats * out)
{
  mgstats s;
  memset (&s, 0, sizeof s);
  if (out) *out = s;
  if (!g || !out) return FAIL (BMG_EINVAL);
  if (g->tree || g->dim < 2) return FAIL (BMG_EUNSUPPORTED);
  CKV (cudaSetDevice (g->device));
  visc_t v;
  memset (&v, 0, sizeof v);
  v.g = g; v.dim = g->dim; v.L = g->depth; v.dt = p.dt;
  const size_t T = g->off64[g->depth + 1];
  if (!g->visc_ws) {
    CKV (cudaMalloc ((void **) &g->visc_ws, 12*T*sizeof (double)));
    CKV (cudaMemsetAsync (g->visc_ws, 0, 12*T*sizeof (double), g->stream));
  }
  const int uh[3] = {p.u.x.i, p.u.y.i, p.u.z.i}, mh[3] = {p.mu.x.i, p.mu.y.i, p.mu.z.i};
  field_t * uf[3] = {NULL, NULL, NULL};
  for (int c = 0; c < v.dim; c++) {
    uf[c] = bmg_i_field (g, uh[c]);
    if (!uf[c] || uf[c]->is_const || uf[c]->face_dim >= 0) return FAIL (BMG_EINVAL);
    v.u[c] = uf[c]->buf;
    v.da[c] = g->visc_ws + (0*3 + c)*T; v.res[c] = g->visc_ws + (1*3 + c)*T;
    v.w[c] = g->visc_ws + (2*3 + c)*T; v.r[c] = g->visc_ws + (3*3 + c)*T;
    bmg_i_bcdesc (g, uf[c], &v.bc[c]);
  }
  /* mu, rho: (const) fields (viscosity.h:29-30); restriction ({mu, rho})
     (viscosity.h:178) */
  field_t * mf[3] = {NULL, NULL, NULL}, * rf = bmg_i_field (g, p.rho.i);
  for (int d = 0; d < v.dim; d++) {
    mf[d] = bmg_i_field (g, mh[d]);
    if (!mf[d] || mf[d]->face_dim != d) return FAIL (BMG_EINVAL);
  }
  if (!rf || rf->face_dim >= 0) return FAIL (BMG_EINVAL);
  long long * nl = &v.launches;
  for (int l = v.L - 1; l >= 0; l--) {
    if (!mf[0]->is_const) {
      const double * fine[3] = {0, 0, 0};
      double * coarse[3] = {0, 0, 0};
      for (int d = 0; d < v.dim; d++) { fine[d] = mf[d]->lv[l + 1]; coarse[d] = mf[d]->lv[l]; }
      const int l0p = l == 0 && (g->periodic[0] || g->periodic[1] || g->periodic[2]);
      LV (bmg_launch_restrict_face (v.dim, g->g64[l + 1], g->g64[l], fine, coarse, l0p, g->stream));
    }
    if (!rf->is_const)
      LV (bmg_launch_restrict (v.dim, BMG_ST_F64, BMG_ST_F64, g->g64[l + 1], g->g64[l],
                               rf->lv[l + 1], rf->lv[l], g->stream));
  }
  for (int l = 0; l <= v.L; l++) {
    for (int d = 0; d < 3; d++) {
      v.mu[l][d].p = d < v.dim && !mf[d]->is_const ? mf[d]->lv[l] : NULL;
      v.mu[l][d].c = d < v.dim && mf[d]->is_const ? mf[d]->cval : 0.;
    }
    v.rho[l].p = rf->is_const ? NULL : rf->lv[l];
    v.rho[l].c = rf->is_const ? rf->cval : 0.;
  }
  /* r = u (viscosity.h:173-175) */
  for (int c = 0; c < v.dim; c++)
    CKV (cudaMemcpyAsync (at (&v, v.r[c], v.L), at (&v, v.u[c], v.L),
                          g->g64[v.L].size*sizeof (double), cudaMemcpyDeviceToDevice, g->stream));
  /* sum of the r.h.s. (poisson.h:162-167), component by component */
  for (int c = 0; c < v.dim; c++) {
    LV (bmg_launch_sum (v.dim, g->g64[v.L], at (&v, v.r[c], v.L), g->d_partials, g->npartials,
                        g->d_sum, g->stream));
    CKV (cudaMemcpyAsync (g->h_pinned + 1, g->d_sum, sizeof (double), cudaMemcpyDeviceToHost,
                          g->stream));
    CKV (cudaStreamSynchronize (g->stream));
    s.sum += g->h_pinned[1];
  }
  s.nrelax = p.nrelax > 0 ? p.nrelax : 4;
  int r = v_residual (&v);
  if (!r) r = read_max (g, &s.resb);
  if (r) return r;
  double resb = s.resa = s.resb;
  const double tolerance = TOLERANCE;
  int status = BMG_OK;
  for (s.i = 0; s.i < NITERMAX && (s.i < NITERMIN || s.resa > tolerance); s.i++) {
    r = v_cycle (&v, s.nrelax);
    if (!r) r = v_residual (&v);
    if (!r) r = read_max (g, &s.resa);
    if (r) return r;
    g->counters.cycles++;
    if (!isfinite (s.resa)) { status = BMG_ENAN; s.i++; break; }
    if (s.resa > tolerance) {
      if (resb/s.resa < 1.2 && s.nrelax < 100)
        s.nrelax++;
      else if (resb/s.resa > 10 && s.nrelax > 2)
        s.nrelax--;
    }
    resb = s.resa;
  }
  s.minlevel = 0;
  if (s.resa > tolerance) {
    fprintf (stderr,
             "WARNING: convergence for %s not reached after %d iterations\n"
             "  res: %g sum: %g nrelax: %d\n", "u.x",
             s.i, s.resa, s.sum, s.nrelax), fflush (stderr);
    if (status == BMG_OK) status = BMG_ENOTCONV;
  }
  /* p.res: the caller's residual fields, one per component */
  if (p.res)
    for (int c = 0; c < v.dim && p.res[c].i; c++) {
      field_t * f = bmg_i_field (g, p.res[c].i);
      if (!f || f->is_const || f->face_dim >= 0) return FAIL (BMG_EINVAL);
      CKV (cudaMemcpyAsync (f->lv[v.L], at (&v, v.res[c], v.L), g->g64[v.L].size*sizeof (double),
                            cudaMemcpyDeviceToDevice, g->stream));
    }
  CKV (cudaStreamSynchronize (g->stream));
  g->counters.launches += v.launches;
  *out = s;
  return FAIL (status);
}

mgstats viscosity (struct Viscosity p)
{
  mgstats s;
  bmg_viscosity (bmg_grid_current (), p, &s);
  return s;
}

/*
 * mg_grid.h -- internal: the grid and field records shared by the host
 * layers of the uniform multigrid (mg_host.c) and of the quadtree
 * (mg_tree_host.c).  Not part of the public C-ABI.
 */
#ifndef MG_GRID_H
#define MG_GRID_H

#include <cuda_runtime_api.h>
#include "basilisk_mg.h"
#include "mg_launch.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int used;
  int face_dim;         /* -1: cell field; d: component d of a face vector */
  int is_const;
  double cval;
  double * buf;         /* all levels */
  double * lv[BMG_MAXLEVEL + 1];
  int bctype[6];
  double bccval[6];
  double * bcval[6];    /* device, n^(dim-1) values of the finest level */
  double * bclv[6][BMG_MAXLEVEL + 1];   /* device, per-level values (trees) */
} field_t;

typedef struct { double bytes; long long launches, sweeps; double relax_bytes; long long relax_sweeps; } work_t;

struct graph_entry;
struct bmg_tree;

struct bmg_grid {
  int dim, depth, device;
  double L0, X0, Y0, Z0;
  int periodic[3];
  int relax, precision, use_graphs, timing;
  cudaStream_t stream;
  int own_stream;
  bmg_geom g64[BMG_MAXLEVEL + 1], g32[BMG_MAXLEVEL + 1];
  size_t off64[BMG_MAXLEVEL + 2], off32[BMG_MAXLEVEL + 2];
  field_t * fields;
  int nfields, cap;
  /* workspace (allocated on first solve) */
  double * ws64;        /* da, da2, res: 3 all-level FP64 arrays */
  float * ws32;         /* da, da2, res, alpha x/y/z, lambda: FP32 levels */
  double * bproj;       /* zero-mean copy of b (mixed form, singular problems) */
  unsigned long long * d_maxres;
  int cluster_levels;   /* cluster kernels for the middle levels of the mixed form
                           (on unless BMG_NO_CLUSTER is set in the environment) */
  double * d_sum, * d_partials;
  int npartials;
  double * h_pinned;
  bmg_counters counters;
  cudaEvent_t ev0, ev1, evr0, evr1;
  struct graph_entry * graphs;     /* captured V-cycles, see run_cycle() */
  struct bmg_tree * tree;          /* quadtree over the levels, or NULL */
  int div_h;                       /* handle of project ()'s div field, 0 = none yet */
  double * visc_ws;                /* viscosity (): da, res, w, r of each component */
  double * stage;                  /* host <-> device staging of field values */
  size_t stage_n;                  /* its size in doubles */
  unsigned long long clock;
};

/* helpers of mg_host.c used by the tree layer */
int bmg_i_fail (int status);                 /* sets bmg_last_error () */
void bmg_i_bcdesc (const bmg_grid * g, const field_t * f, bmg_bcdesc * bc);
field_t * bmg_i_field (bmg_grid * g, int handle);
int bmg_i_workspace (bmg_grid * g);          /* FP64 da, da2, res on all levels */
double * bmg_i_ws64 (bmg_grid * g, int which, int level);
enum { BMG_WS_DA = 0, BMG_WS_DA2 = 1, BMG_WS_RES = 2 };

/* the tree layer (mg_tree_host.c) */
void bmg_tree_free (bmg_grid * g);
void bmg_tree_graphs_clear (bmg_grid * g);
int bmg_tree_poisson (bmg_grid * g, struct Poisson p, mgstats * out);
int bmg_tree_mg_solve (bmg_grid * g, struct MGSolve p, mgstats * out);
int bmg_tree_mg_cycle (bmg_grid * g, field_t * a, field_t * res, field_t * da,
                       struct Poisson * p, int nrelax, int minlevel, int maxlevel);
int bmg_tree_relax (bmg_grid * g, field_t * da, field_t * res, int level, struct Poisson * p);
int bmg_tree_residual (bmg_grid * g, field_t * a, field_t * b, field_t * res,
                       struct Poisson * p, double * maxres);
int bmg_tree_restriction (bmg_grid * g, const bmg_scalar * list);

#ifdef __cplusplus
}
#endif
#endif

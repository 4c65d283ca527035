/*
 * basilisk_mg.h -- C-ABI of the B200 multigrid Poisson--Helmholtz solver.
 *
 * A device-resident replacement for Basilisk's multigrid Poisson solver
 * (poisson.h: mg_cycle, mg_solve, poisson; grid/multigrid.h levels).  The
 * reference-facing entry points keep the reference's names, argument
 * meaning and result struct; the grid/field functions are the device
 * counterpart of what grid/multigrid.h and grid/cartesian-common.h give a
 * Basilisk program (init_grid, new scalar fields, boundary conditions,
 * origin/size/periodic).
 *
 * Conventions
 *   - Fields live on the device, on every level 0..depth of one grid, as
 *     padded, level-contiguous structure-of-arrays buffers.  Host code moves
 *     finest-level values in and out with bmg_field_set / bmg_field_get, from
 *     host or device memory, in the compact layout: n^dimension values in C
 *     order with the last index contiguous (the reference's index order,
 *     grid/multigrid.h:59-73).  Face component d has n+1 values along d; face
 *     f is the left/bottom/back face of cell f (alpha.x[] / alpha.x[1],
 *     poisson.h:306).
 *   - Handles are small integers, 0 meaning "unset" (poisson.h:410-413 tests
 *     alpha.x.i and lambda.i against 0).
 *   - Every call is on one host thread per grid; the grid owns one CUDA
 *     stream; calls are not re-entrant on one grid.
 *   - The library never aborts the process and never traps on the device:
 *     failures are status codes (bmg_* functions) or bmg_last_error() (the
 *     reference-named functions, which return mgstats by value).
 */
#ifndef BASILISK_MG_H
#define BASILISK_MG_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- result and globals: poisson.h:102-114 ---------------------------- */

/* byte-identical to the reference's mgstats (poisson.h:108-114) */
typedef struct {
  int i;              /* number of iterations */
  double resb, resa;  /* maximum residual before and after the iterations */
  double sum;         /* sum of r.h.s. */
  int nrelax;         /* number of relaxations */
  int minlevel;       /* minimum level of the multigrid hierarchy */
} mgstats;

/* poisson.h:102-103: same names, same defaults (100, 1, 1e-3) */
extern int NITERMAX, NITERMIN;
extern double TOLERANCE;

/* ---- status codes --------------------------------------------------- */
enum {
  BMG_OK = 0,
  BMG_EINVAL = 1,        /* invalid argument or handle */
  BMG_ECUDA = 2,         /* a CUDA runtime call failed */
  BMG_ENOMEM = 3,        /* device allocation failed */
  BMG_ENAN = 4,          /* the residual became NaN or Inf */
  BMG_ENOTCONV = 5,      /* tolerance not reached after NITERMAX cycles */
  BMG_EUNSUPPORTED = 6,  /* callbacks other than the Poisson ones */
  BMG_ENODEV = 7         /* no CUDA device */
};
const char * bmg_error_string (int status);
int bmg_last_error (void);           /* status of the last call on this thread */

/* ---- grid: grid/multigrid.h init_grid, common.h origin/size/periodic -- */

/* sides in the reference's order (common.h:949) */
enum { BMG_RIGHT = 0, BMG_LEFT, BMG_TOP, BMG_BOTTOM, BMG_FRONT, BMG_BACK };

/* boundary-condition kinds (common.h:957-960; periodic: cartesian-common.h:898) */
enum { BMG_NEUMANN = 0, BMG_DIRICHLET = 1, BMG_PERIODIC = 2 };

/* smoother: red-black Gauss-Seidel, or the reference's -DJACOBI weighted
   Jacobi (poisson.h:293-328), which gives results independent of the
   traversal order and therefore bit-comparable with the reference. */
enum { BMG_RELAX_RBGS = 0, BMG_RELAX_JACOBI = 1 };

/* arithmetic of the solve: FP64 throughout, or FP32 cycles inside an FP64
   iterative-refinement loop (outer residual, accumulation, compatibility
   projection and coarsest level in FP64).  On a quadtree the mixed form
   runs its cycle in FP32 on every level, keeps the residual and a += da
   in FP64, does not project b, and needs the schedule interpreter's
   thread-block cluster (16 or 8 CTAs of 1024 threads): without it the
   solve returns BMG_EUNSUPPORTED. */
enum { BMG_FP64 = 0, BMG_MIXED = 1 };

/* where the pointers given to bmg_field_set / get / bmg_bc point */
enum { BMG_HOST = 0, BMG_DEVICE = 1 };

typedef struct bmg_grid bmg_grid;

/* init_grid (grid/multigrid.h:723-759): levels 0..depth of a 2^depth per
   side box, dimension 1, 2 or 3, on the current CUDA device.  The new grid
   becomes the current grid used by poisson(), mg_solve() and mg_cycle(). */
int bmg_grid_new (bmg_grid ** grid, int dimension, int depth);
void bmg_grid_free (bmg_grid * grid);
int bmg_grid_select (bmg_grid * grid);      /* make it the current grid */
bmg_grid * bmg_grid_current (void);
int bmg_grid_info (const bmg_grid * grid, int * dimension, int * depth);
/* origin (common.h:935) and size (common.h:939) */
int bmg_origin (bmg_grid * grid, double x, double y, double z);
int bmg_size (bmg_grid * grid, double L0);
/* periodic (cartesian-common.h:920-933): dir is a side (BMG_RIGHT, BMG_TOP,
   BMG_FRONT or their opposite); applies to every field of the grid */
int bmg_periodic (bmg_grid * grid, int dir);
int bmg_set_relax (bmg_grid * grid, int relax);
int bmg_set_precision (bmg_grid * grid, int precision);
/* optional: run on a caller's stream (cudaStream_t); NULL = the grid's own */
int bmg_set_stream (bmg_grid * grid, void * stream);
int bmg_synchronize (bmg_grid * grid);

/* ---- fields: scalar / face vector handles ---------------------------- */

/* layout-compatible with Basilisk's scalar {int i;} and vector {scalar x, y, z;} */
typedef struct { int i; } bmg_scalar;
typedef struct { bmg_scalar x, y, z; } bmg_vector;

/* a new cell-centred field, zero on every level (cartesian-common.h:62-106) */
int bmg_scalar_new (bmg_grid * grid, bmg_scalar * s);
/* a new face vector; its components have no box BCs (cartesian-common.h:566) */
int bmg_face_vector_new (bmg_grid * grid, bmg_vector * v);
/* constant fields (common.h:1275-1277): stored as one value, never as arrays */
int bmg_const_scalar (bmg_grid * grid, double value, bmg_scalar * s);
int bmg_const_face_vector (bmg_grid * grid, double value, bmg_vector * v);
int bmg_field_delete (bmg_grid * grid, bmg_scalar s);
/* finest-level values in the compact layout; count = number of doubles */
int bmg_field_set (bmg_grid * grid, bmg_scalar s, const double * values, size_t count, int memory);
int bmg_field_get (bmg_grid * grid, bmg_scalar s, double * values, size_t count, int memory);
/* values of any level (tests, diagnostics) */
int bmg_field_get_level (bmg_grid * grid, bmg_scalar s, int level, double * values, size_t count, int memory);
int bmg_field_set_level (bmg_grid * grid, bmg_scalar s, int level, const double * values, size_t count, int memory);

/* s[side] = dirichlet(v) / neumann(v) (common.h:957-960): a constant v, or,
   when values != NULL, one value per boundary face of the finest level
   (n^(dimension-1) values over the tangential indices in increasing
   dimension order).  The homogeneous twin (-s[] / s[]) is used for the
   correction field of mg_solve (poisson.h:155-157). */
int bmg_bc (bmg_grid * grid, bmg_scalar s, int side, int type, double value,
            const double * values, int memory);

/* ---- the solver: poisson.h ----------------------------------------- */

/* struct Poisson (poisson.h:258-265), same members and order */
struct Poisson {
  bmg_scalar a, b;
  bmg_vector alpha;      /* 0 = unityf */
  bmg_scalar lambda;     /* 0 = zeroc */
  double tolerance;      /* 0 = TOLERANCE */
  int nrelax, minlevel;
  bmg_scalar * res;      /* optional: receives the final residual */
};

/* poisson (poisson.h:402-441) on the current grid.  Status: bmg_last_error(). */
mgstats poisson (struct Poisson p);
/* the same on a given grid, returning a status */
int bmg_poisson (bmg_grid * grid, struct Poisson p, mgstats * stats);
/* struct Project (poisson.h:461-467), same members and order */
struct Project {
  bmg_vector uf;         /* face velocity, corrected in place */
  bmg_scalar p;          /* pressure, solved in place */
  bmg_vector alpha;      /* 0 = unityf */
  double dt;             /* 0 = 1 */
  int nrelax;            /* 0 = 4 */
};
/* project (poisson.h:468-509) on the current grid: div of uf over dt Delta,
   poisson (p, div, alpha, tolerance = TOLERANCE/dt^2, nrelax), then
   uf -= dt alpha grad p on every face.  Status: bmg_last_error ().
   Uniform grids only (BMG_EUNSUPPORTED on a tree). */
mgstats project (struct Project q);
int bmg_project (bmg_grid * grid, struct Project q, mgstats * stats);


/* struct Viscosity (viscosity.h:3-10), same members and order */
struct Viscosity {
  bmg_vector u;          /* cell velocity components, solved in place */
  bmg_vector mu;         /* face viscosity (a constant face vector allowed) */
  bmg_scalar rho;        /* density (a constant scalar allowed) */
  double dt;
  int nrelax;            /* 0 = 4 */
  bmg_scalar * res;      /* optional: receives the residual of each component */
};
/* viscosity (viscosity.h:169-183) on the current grid: the implicit
   viscous step rho (u - u*)/dt = div (2 mu D) as mg_solve with the
   coupled relax_viscosity / residual_viscosity (viscosity.h:25-160),
   lambda = 1 (no AXI), two or three dimensions, uniform grids, FP64.
   Status: bmg_last_error (). */
mgstats viscosity (struct Viscosity p);
int bmg_viscosity (bmg_grid * grid, struct Viscosity p, mgstats * stats);

/* the Poisson--Helmholtz callbacks (poisson.h:271-391); data is a
   struct Poisson *.  These are the only callbacks mg_solve/mg_cycle accept:
   they run on the device, host callbacks cannot. */
void bmg_relax (bmg_scalar * da, bmg_scalar * res, int level, void * data);
double bmg_residual (bmg_scalar * a, bmg_scalar * b, bmg_scalar * res, void * data);

/* struct MGSolve (poisson.h:125-137), same members and order */
struct MGSolve {
  bmg_scalar * a, * b;
  double (* residual) (bmg_scalar * a, bmg_scalar * b, bmg_scalar * res, void * data);
  void (* relax) (bmg_scalar * da, bmg_scalar * res, int depth, void * data);
  void * data;
  int nrelax;
  bmg_scalar * res;
  int minlevel;
  double tolerance;
};

/* mg_solve (poisson.h:139-235).  Status: bmg_last_error(). */
mgstats mg_solve (struct MGSolve p);

/* mg_cycle (poisson.h:32-90): restriction of res, coarse-to-fine
   correction of da with nrelax relaxations per level, then a += da.  da
   takes the homogeneous BCs of a. */
void mg_cycle (bmg_scalar * a, bmg_scalar * res, bmg_scalar * da,
               void (* relax) (bmg_scalar * da, bmg_scalar * res, int depth, void * data),
               void * data, int nrelax, int minlevel, int maxlevel);

/* restriction of a list of fields to all levels (multigrid-common.h:368-404),
   as test/variable.c calls it for its face coefficients; list ends with .i=0 */
int bmg_restriction (bmg_grid * grid, const bmg_scalar * list);

/* ---- quadtree grids: grid/quadtree.h (grid/tree.h, tree-common.h) --- */

/* refine (cond) (tree-common.h:308-326) on a two-dimensional, non-periodic
   grid: the grid's levels become a quadtree whose root is init_grid (1);
   every leaf for which cond (level, x, y, z, data) is non-zero is refined,
   with the 2:1 balance of refine_cell (tree-common.h:22-55), until no leaf
   asks for refinement.  The tree's depth is at most the grid's depth
   (deeper refinement fails with BMG_EINVAL).  Returns the number of
   refined cells (>= 0) or a negative status.  Once a grid is a tree,
   poisson, mg_solve, mg_cycle, bmg_relax, bmg_residual and bmg_restriction
   follow the reference's tree branch: relaxation over
   foreach_level_or_leaf, the tree boundary (restriction then bilinear halo
   prolongation, tree-common.h:588-716), the conservative residual
   (poisson.h:355-372).  Cell values live in the grid's level arrays
   (bmg_field_set_level / get_level); a field's leaves are the cells whose
   flags have BMG_TREE_LEAF.  The tree path computes in FP64. */
typedef int (* bmg_refine_cond) (int level, double x, double y, double z, void * data);
int bmg_tree_refine (bmg_grid * grid, bmg_refine_cond cond, void * data);
/* depth () and the number of leaves of a tree grid */
int bmg_tree_info (const bmg_grid * grid, int * depth, long long * leaves);
/* cell flags of one level, n x n bytes in the compact layout
   (grid/tree.h:27-47, 398-399): */
enum { BMG_TREE_ACTIVE = 1, BMG_TREE_LEAF = 2, BMG_TREE_HALO = 4, BMG_TREE_PROLONGATION = 8 };
int bmg_tree_flags (const bmg_grid * grid, int level, unsigned char * flags);
/* s[side] = dirichlet / neumann with one value per boundary face of one
   level (n values over the tangential index): a tree applies the condition
   of a field on every level (tree_boundary_level), with the expression
   evaluated at that level's face centres */
int bmg_bc_level (bmg_grid * grid, bmg_scalar s, int side, int type, int level,
                  const double * values, int memory);

/* ---- snapshots: dump () and restore () (output.h:1043-1400) ---------- */

/* dump (file, list) (output.h:1138-1171): writes the fields of list (ends
   with .i = 0), named by names[], in the reference's binary format
   (dump_version 170901): header {t, len, i, depth, npe = 1, version, n},
   the names with "size" first, {X0, Y0, Z0, L0}, then every cell of
   foreach_cell () with its flags (leaf = 2), its subtree's cell count and
   the values.  A uniform grid writes all its levels (its leaves are the
   finest level); a tree grid its active cells.  t and iter go into the
   header. */
int bmg_dump (bmg_grid * grid, const char * file, const bmg_scalar * list,
              const char * const * names, double t, int iter);
/* restore (file, list) (output.h:1220-1400): reads a file of the format
   above (or the older, unnamed 161020 one, whose columns must be list's
   fields in order).  Columns whose name matches names[k] go to list[k];
   the others are skipped.  The origin and size of the file are applied.
   A tree grid, or any grid given a file that holds a tree, is rebuilt
   from init_grid (1) by refining the cells the file holds refined (as
   refine_cell does in restore); a uniform grid takes a uniform file of
   its own depth.  Fields that are not listed keep their values (the
   reference resets them to 0; here the caller owns them).  *t and *iter
   (when not NULL) receive the header's time and iteration. */
int bmg_restore (bmg_grid * grid, const char * file, const bmg_scalar * list,
                 const char * const * names, double * t, int * iter);

/* ---- decomposition into blocks: grid/multigrid-mpi.h ----------------- */

/* A domain of dims[0] x dims[1] (x dims[2]) blocks, each a grid of the same
   dimension and depth (the reference's per-rank multigrid, multigrid-mpi.h:
   94-130): block b sits at Cartesian coordinates c with
   b = (c0 dims[1] + c1) dims[2] + c2 (MPI_Cart_create's row-major order),
   and covers cells c_e 2^depth .. (c_e + 1) 2^depth - 1 along direction e;
   set each block's origin and size accordingly (bmg_origin, bmg_size).
   periodic[e] makes the domain periodic along e: a direction of a single
   block is then periodic on that block (bmg_periodic), a direction of
   several blocks wraps its neighbours and must not be periodic on the
   blocks.  Blocks may live on different CUDA devices (each created with its
   device current); the decomposition puts the blocks of a device on one
   stream of its own, and gives them their own streams back when it is
   freed, so free the decomposition before its blocks.  Every block must
   create its fields in the same order, so that a field has the same handle
   in every block.  The solve is FP64. */
typedef struct bmg_shard bmg_shard;
int bmg_shard_new (bmg_shard ** shard, bmg_grid * const * blocks, const int * dims,
                   const int * periodic);
void bmg_shard_free (bmg_shard * shard);
/* poisson () (poisson.h:402-441) over the blocks: mg_solve with the
   boundary exchange of mpi_boundary_level (multigrid-mpi.h:52-85) after
   every pass, the sum of b and the residual maximum reduced over the
   blocks (the MPI_Allreduce of common.h:681-718).  Field handles of p are
   those of every block; minlevel counts a block's levels (at least 1). */
int bmg_shard_poisson (bmg_shard * shard, struct Poisson p, mgstats * out);
/* MPI_Dims_create (n, dimension, dims) with all dims free */
int bmg_shard_dims (int n, int dimension, int * dims);
/* MPI_Cart_shift of block b: out[side] is the neighbouring block on each
   side (BMG_RIGHT .. BMG_BACK), -1 on a box side */
int bmg_shard_neighbours (int dimension, const int * dims, const int * periodic, int b,
                          int * out);

/* ---- differentiation ----------------------------------------------- */

/* Gradients of a loss l(a) with respect to the coefficients of the solve
   a = L^{-1} b, given the adjoint mu (solved with poisson() from the
   right-hand side dl/da on a field with the homogeneous conditions of a;
   L is symmetric): grad_alpha[d] receives dl/dalpha for face component d
   (compact face arrays, n+1 along d; NULL skips), grad_lambda receives
   dl/dlambda = -mu a (compact cell array; NULL skips).  dl/db is mu
   itself.  No counterpart in the reference (whose solver has no
   derivatives); it differentiates the discrete operator of poisson.h:373-389. */
int bmg_adjoint_gradients (bmg_grid * grid, bmg_scalar mu, bmg_scalar a,
                           double * const * grad_alpha, double * grad_lambda, int memory);

/* ---- allocation-free sum ------------------------------------------- */

/* The sum of count doubles at values (device memory), written to *result
   (device memory) on stream (a cudaStream_t, NULL = the default stream):
   the Sigma b that mg_solve reports in mgstats.sum, for callers that cannot
   allocate device memory -- code running while a stream is captured into a
   CUDA graph in global capture mode, where cudaMalloc is refused, or
   programs that hand all device memory to their own pool at start-up and
   let nothing else allocate.  It allocates nothing: its scratch is a static
   32 KB device array inside the library (4096 partial sums), so count is at
   most 16,777,216 (4096^2 in 2D, 256^3 in 3D); larger counts are rejected
   with BMG_EINVAL and a message on stderr.  Every call outside a stream
   capture looks up the scratch's device address with the current device
   (so a context created again after cudaDeviceReset is followed); a call
   inside a capture uses the address found by the last call outside one, so
   make one call on each device before any stream capture (a first call
   inside a capture fails with BMG_EINVAL).  All calls share the scratch: calls
   that overlap on the GPU (different streams, no ordering) race.  The
   result is asynchronous on stream.  No counterpart in the reference. */
int bmg_sum_noalloc (const double * values, size_t count, double * result, void * stream);

/* ---- measurement ---------------------------------------------------- */

/* totals since the grid was created: V-cycles, relaxation sweeps per level
   (summed), algorithmic bytes moved by the cycle kernels (each array pass
   counted once at its storage precision, ghosts excluded) and the device
   time of the cycles in milliseconds (CUDA events), when timing is on. */
typedef struct {
  long long cycles;
  long long sweeps;
  double bytes;
  double cycle_ms;
  long long launches;
  /* the finest level's relaxation sweeps of each timed cycle, bracketed by
     CUDA events: their device time and algorithmic bytes */
  double relax_ms;
  double relax_bytes;
  long long relax_sweeps;
} bmg_counters;
int bmg_get_counters (bmg_grid * grid, bmg_counters * c);
int bmg_reset_counters (bmg_grid * grid);
int bmg_set_timing (bmg_grid * grid, int on);
/* CUDA graphs for the V-cycles: 0 = off, 1 = on with the default cache
   (64 captured cycles, one per distinct nrelax), n > 1 = a cache of n (<= 256) */
int bmg_set_graphs (bmg_grid * grid, int n);

#ifdef __cplusplus
}
#endif
#endif

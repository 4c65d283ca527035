/*
 * mg_tree_host.c -- host layer of the quadtree path (two dimensions).
 *
 * A grid becomes a quadtree with bmg_tree_refine (): the device counterpart
 * of Basilisk's init_grid (1) + refine (cond) on grid/quadtree.h.  The tree
 * keeps the grid's dense level arrays; it adds per-cell flags and the cell
 * lists the tree kernels walk (mg_tree.h).  The control flow follows the
 * reference's tree branch:
 *   refine_cell with TWO_ONE, refine ()     grid/tree-common.h:22-55, 308-326
 *   halo cells, caches                      grid/tree.h:556-684, 929-1041
 *   tree_boundary_level                     grid/tree-common.h:588-716
 *   box boundary on trees                   grid/tree.h:1139-1209, 1286-1367
 *   mg_cycle / mg_solve / poisson           poisson.h:32-90, 139-235, 402-441
 *   relax over foreach_level_or_leaf        poisson.h:271-338, grid/tree.h:735-740
 *   residual, tree branch                   poisson.h:355-372
 * Every operation on field data runs in mg_tree.cu; this file builds the
 * tree, sequences launches (captured into CUDA graphs per solve key) and
 * reads one residual maximum back per cycle.
 *
 * The red-black smoother relaxes the red cells of every level of the set,
 * refreshes the tree boundary, then the black cells; the Jacobi smoother is
 * the reference's JACOBI branch.
 *
 * Two forms, as on uniform grids: the plain form computes in FP64; the
 * mixed form (grid precision BMG_MIXED) runs the cycle -- restriction of
 * the residual, prolongation, relaxation and the tree boundaries of the
 * correction -- in FP32, and keeps FP64 for a, b, the residual r = b - L a
 * (its boundary of a included) and the accumulation a += da, so that every
 * iteration is an FP64 iterative-refinement step.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <stdint.h>
#include <cuda_runtime_api.h>

#include "mg_grid.h"
#include "mg_tree.h"

#define TMAX BMG_TREE_MAXLEVEL
#define NTGRAPH 16

typedef struct { long off, n; } span_t;

/* one launch of a scheduled tree boundary (bmg_tree_launch_stage) */
typedef struct { int op; span_t list; span_t rules; } tstage;
enum { SCHED_FULL = 0, SCHED_PRUNED = 1 };

/* everything a captured solve iteration depends on */
typedef struct {
  int nrelax, minlevel, maxlevel, relax, mixed;
  const void * a, * b, * da, * res, * tmp;
  bmg_tree_coef ax, ay, lam;
  bmg_tree_bc abc;
  cudaStream_t stream;
  const void * maxres, * pinned;
} tkey;

struct tgraph {
  int valid;
  unsigned long long stamp;
  tkey key;
  cudaGraphExec_t exec;
  long long launches;
  bmg_tree_op * dops;     /* the interpreter's operations of the iteration */
  long nops;
  double bytes;           /* algorithmic bytes of the iteration */
};

struct bmg_tree {
  int depth, hmax;
  long long nleaves;
  int full;
  unsigned char * fl[TMAX + 1];       /* host flags, (n + 2)^2 with the ghost ring */
  unsigned short * nb[TMAX + 1];      /* refined cells in the 3x3 neighbourhood */
  unsigned char * dflags;             /* device flags, FP64 level layout */
  uint32_t * dlist;
  bmg_tree_rule * drules;
  span_t act[TMAX + 1], ref[TMAX + 1], prol[TMAX + 1], rl[TMAX + 1], ghost[TMAX + 1], leaves;
  long rl1[TMAX + 1];                 /* colour-1 part of rl[l] starts here */
  /* tree boundary schedules: [SCHED_FULL / SCHED_PRUNED][level] spans of
     stages, whose rules live in dsrules */
  tstage * stages;
  long nstages;
  span_t sched[2][TMAX + 1];
  bmg_tree_rule * dsrules;
  bmg_tree_levels T;
  double * dpart;
  int npart;
  struct tgraph graphs[NTGRAPH];
  unsigned long long clock;
  int interp;                         /* run solve iterations through the interpreter */
  float * ws32;                       /* mixed form: da, res, tmp, alpha x, alpha y, lambda in
                                         FP32, each an all-level array in the FP64 element layout */
};
enum { W32_DA = 0, W32_RES, W32_TMP, W32_AX, W32_AY, W32_LAM, W32_N };

#define FAIL(s) bmg_i_fail (s)
#define CKT(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) { \
      fprintf (stderr, "bmg: %s failed: %s (%s:%d)\n", #call,            \
               cudaGetErrorString (e_), __FILE__, __LINE__);              \
      return FAIL (e_ == cudaErrorMemoryAllocation ? BMG_ENOMEM : BMG_ECUDA); } } while (0)
#define LT(call) do { int e_ = (call); if (e_) {                          \
      fprintf (stderr, "bmg: launch %s failed: %s (%s:%d)\n", #call,      \
               cudaGetErrorString ((cudaError_t) e_), __FILE__, __LINE__); \
      return FAIL (BMG_ECUDA); } (*nl)++; } while (0)

static inline size_t HX (int l, int i, int j) { return (size_t) (i + 1)*((1 << l) + 2) + (j + 1); }

static inline uint32_t pack (int l, int i, int j)
{
  return ((uint32_t) l << 28) | ((uint32_t) (i + 1) << 14) | (uint32_t) (j + 1);
}

/* ------------------------------------------------------------------ */
/* building the tree                                                   */
/* ------------------------------------------------------------------ */

static void graph_drop (struct tgraph * q)
{
  if (q->valid) cudaGraphExecDestroy (q->exec);
  cudaFree (q->dops);
  q->dops = NULL; q->nops = 0;
  q->valid = 0;
}

static void tree_release (struct bmg_tree * t)
{
  if (!t) return;
  for (int i = 0; i < NTGRAPH; i++) graph_drop (&t->graphs[i]);
  for (int l = 0; l <= TMAX; l++) { free (t->fl[l]); free (t->nb[l]); }
  cudaFree (t->dflags); cudaFree (t->dlist); cudaFree (t->drules); cudaFree (t->dpart);
  cudaFree (t->dsrules); cudaFree (t->ws32);
  free (t->stages);
  free (t);
}

void bmg_tree_free (bmg_grid * g)
{
  if (!g || !g->tree) return;
  tree_release (g->tree);
  g->tree = NULL;
}

void bmg_tree_graphs_clear (bmg_grid * g)
{
  if (!g || !g->tree) return;
  for (int i = 0; i < NTGRAPH; i++) graph_drop (&g->tree->graphs[i]);
}

/* refine_cell (tree-common.h:22-55): the leaves among the parent's
   neighbours on this child's side are refined first (TWO_ONE), then the
   cell; its 3x3 neighbourhood counts it (increment_neighbors) */
static int split (struct bmg_tree * t, int l, int i, int j)
{
  if (l + 1 > t->hmax) return BMG_EINVAL;
  if (l > 0) {
    const int pi = i >> 1, pj = j >> 1, np = 1 << (l - 1);
    const int sx = (i & 1) ? 1 : -1, sy = (j & 1) ? 1 : -1;
    const int side[3][2] = {{0, sy}, {sx, 0}, {sx, sy}};
    for (int q = 0; q < 3; q++) {
      const int ni = pi + side[q][0], nj = pj + side[q][1];
      if (ni < 0 || nj < 0 || ni >= np || nj >= np) continue;
      if (t->fl[l - 1][HX (l - 1, ni, nj)] & BMG_T_LEAF) {
        int r = split (t, l - 1, ni, nj);
        if (r) return r;
      }
    }
  }
  const int n = 1 << l;
  for (int a = i - 1; a <= i + 1; a++)
    for (int b = j - 1; b <= j + 1; b++)
      if (a >= 0 && b >= 0 && a < n && b < n)
        t->nb[l][HX (l, a, b)]++;
  for (int c = 0; c < 4; c++)
    t->fl[l + 1][HX (l + 1, 2*i + (c >> 1), 2*j + (c & 1))] |= BMG_T_ACTIVE | BMG_T_LEAF;
  t->fl[l][HX (l, i, j)] &= ~BMG_T_LEAF;
  if (l + 1 > t->depth) t->depth = l + 1;
  return BMG_OK;
}

/* one foreach_leaf () pass of refine (): depth first, children in the
   order (left,bottom), (left,top), (right,bottom), (right,top) */
static int refine_pass (bmg_grid * g, struct bmg_tree * t, bmg_refine_cond cond, void * data,
                        long * count)
{
  struct { int l, i, j; } stack[4*(TMAX + 2)];
  int top = 0;
  stack[top].l = 0; stack[top].i = 0; stack[top].j = 0; top++;
  while (top > 0) {
    top--;
    const int l = stack[top].l, i = stack[top].i, j = stack[top].j;
    const unsigned char f = t->fl[l][HX (l, i, j)];
    if (!(f & BMG_T_ACTIVE)) continue;
    if (f & BMG_T_LEAF) {
      const double Delta = g->L0*(1./(1 << l));
      const double x = (i + 0.5)*Delta + g->X0, y = (j + 0.5)*Delta + g->Y0;
      if (cond (l, x, y, 0., data)) {
        int r = split (t, l, i, j);
        if (r) return r;
        (*count)++;
      }
      continue;
    }
    for (int c = 3; c >= 0; c--) {          /* pushed in reverse: popped in order */
      stack[top].l = l + 1; stack[top].i = 2*i + (c >> 1); stack[top].j = 2*j + (c & 1);
      top++;
    }
  }
  return BMG_OK;
}

static inline int interior_allocated (const struct bmg_tree * t, int l, int i, int j)
{
  const int n = 1 << l;
  if (i < 0 || j < 0 || i >= n || j >= n) return 0;
  return (t->fl[l][HX (l, i, j)] & (BMG_T_ACTIVE | BMG_T_HALO)) != 0;
}

static inline int ghost_at (int l, int i, int j)
{
  const int n = 1 << l;
  if (i < -1 || j < -1 || i > n || j > n) return 0;
  return i == -1 || j == -1 || i == n || j == n;
}

/* boundary id of a ghost: init_grid's pids give corners their x side
   (tree.h:1530-1542) */
static inline int ghost_side (int l, int i, int j)
{
  const int n = 1 << l;
  if (i < 0) return BMG_LEFT;
  if (i >= n) return BMG_RIGHT;
  if (j >= n) return BMG_TOP;
  return BMG_BOTTOM;
}

static inline int tangential (int side, int i, int j)
{
  return (side == BMG_LEFT || side == BMG_RIGHT) ? j : i;
}

/* the rule of ghost (gi, gj): normal_neighbor, else diagonal_neighbor_2D
   (tree.h:1139-1209); 0 when the ghost touches no allocated cell */
static int ghost_rule (const struct bmg_tree * t, int l, int gi, int gj, bmg_tree_rule * r)
{
  static const int nrm[4][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}};
  for (int q = 0; q < 4; q++) {
    const int a = gi + nrm[q][0], b = gj + nrm[q][1];
    if (interior_allocated (t, l, a, b)) {
      const int s = ghost_side (l, gi, gj);
      r->ghost = pack (l, gi, gj); r->inner = pack (l, a, b);
      r->kind_sides = (BMG_T_NORMAL << 8) | s;
      r->tidx = (uint32_t) tangential (s, a, b);
      return 1;
    }
  }
  for (int di = -1; di <= 1; di += 2)
    for (int dj = -1; dj <= 1; dj += 2) {
      const int a = gi + di, b = gj + dj;
      if (interior_allocated (t, l, a, b) && ghost_at (l, a, gj) && ghost_at (l, gi, b)) {
        const int s1 = ghost_side (l, a, gj), s2 = ghost_side (l, gi, b);
        r->ghost = pack (l, gi, gj); r->inner = pack (l, a, b);
        r->kind_sides = (BMG_T_DIAGONAL << 8) | (s2 << 4) | s1;
        r->tidx = ((uint32_t) tangential (s2, a, b) << 16) | (uint32_t) tangential (s1, a, b);
        return 1;
      }
    }
  return 0;
}

/* The launches of tree_boundary_level (s, l), as stages.  The events are
   the restriction of levels l-1 down to mlo, then the halo prolongation of
   levels mlo up to l-1 (tree-common.h:672-712); the ghost cells of levels
   mlo..l ride along: a ghost can run in the first event after the one that
   produces its interior value (restriction of its level for a refined
   cell, halo prolongation of the level below for a halo cell, none for a
   leaf or a cell of level l), provided that event does not read it (the
   halo prolongation of its own level does); otherwise it gets a launch of
   its own at that point.  With mlo = 0 every value of the reference's
   sequence is computed; SCHED_PRUNED starts at the coarsest level holding a
   leaf, below which no value computed here is ever read (no leaf relaxes
   there, no halo is prolonged from there). */
static int schedule (struct bmg_tree * t, int l, int mlo, const bmg_tree_rule * hr,
                     tstage ** st, long * nst, long * cap, bmg_tree_rule ** rs, long * nrs,
                     long * rcap)
{
  typedef struct { int op, level; } event_t;
  event_t ev[2*(TMAX + 1)];
  int E = 0, Ridx[TMAX + 1], Hidx[TMAX + 1];
  for (int m = 0; m <= TMAX; m++) Ridx[m] = Hidx[m] = -1;
  if (mlo > l) mlo = l;
  for (int m = l - 1; m >= mlo; m--)
    if (t->ref[m].n) { Ridx[m] = E; ev[E].op = BMG_T_OP_RESTRICT; ev[E++].level = m; }
  for (int i = mlo; i < l; i++)
    if (t->prol[i].n) { Hidx[i] = E; ev[E].op = BMG_T_OP_HALO; ev[E++].level = i; }
  /* slot of every rule: 2*k = a launch of its own before event k,
     2*k + 1 = fused into event k */
  long nr = 0;
  for (int m = mlo; m <= l; m++) nr += t->ghost[m].n;
  int * slot = malloc ((nr + 1)*sizeof (int));
  const bmg_tree_rule ** rp = malloc ((nr + 1)*sizeof (*rp));
  if (!slot || !rp) { free (slot); free (rp); return BMG_ENOMEM; }
  long q = 0;
  for (int m = mlo; m <= l; m++)
    for (long k = 0; k < t->ghost[m].n; k++, q++) {
      const bmg_tree_rule * r = &hr[t->ghost[m].off + k];
      const int ii = (int) ((r->inner >> 14) & 0x3FFF) - 1, jj = (int) (r->inner & 0x3FFF) - 1;
      const unsigned char f = t->fl[m][HX (m, ii, jj)];
      int p = -1;
      if (m < l && (f & BMG_T_ACTIVE) && !(f & BMG_T_LEAF)) p = Ridx[m];
      else if (f & BMG_T_HALO) p = m >= 1 ? Hidx[m - 1] : -1;
      const int c = (m < l && Hidx[m] >= 0) ? Hidx[m] : E;
      const int e = p + 1;
      slot[q] = (e < c && e < E) ? 2*e + 1 : 2*e;
      rp[q] = r;
    }
  for (int sl = 0; sl <= 2*E; sl++) {
    const int k = sl/2, fused = sl & 1;
    if (fused && k >= E) break;
    long first = *nrs;
    for (long u = 0; u < nr; u++)
      if (slot[u] == sl) {
        if (*nrs == *rcap) {
          *rcap = 2*(*rcap) + 1024;
          bmg_tree_rule * nrp = realloc (*rs, *rcap*sizeof (bmg_tree_rule));
          if (!nrp) { free (slot); free (rp); return BMG_ENOMEM; }
          *rs = nrp;
        }
        (*rs)[(*nrs)++] = *rp[u];
      }
    if (!fused && *nrs == first) continue;          /* no launch of its own needed */
    if (*nst == *cap) {
      *cap = 2*(*cap) + 64;
      tstage * ns = realloc (*st, *cap*sizeof (tstage));
      if (!ns) { free (slot); free (rp); return BMG_ENOMEM; }
      *st = ns;
    }
    tstage * sg = &(*st)[(*nst)++];
    memset (sg, 0, sizeof *sg);
    sg->rules.off = first; sg->rules.n = *nrs - first;
    if (fused) {
      sg->op = ev[k].op;
      sg->list = ev[k].op == BMG_T_OP_RESTRICT ? t->ref[ev[k].level] : t->prol[ev[k].level];
    }
    else
      sg->op = BMG_T_OP_NONE;
  }
  free (slot); free (rp);
  return BMG_OK;
}

/* flags of halo cells and prolongation leaves, cell lists, ghost rules:
   the caches of update_cache_f (tree.h:556-684), uploaded */
static int derive (bmg_grid * g, struct bmg_tree * t)
{
  const int D = t->depth;
  long nact[TMAX + 1] = {0}, nref[TMAX + 1] = {0}, nprol[TMAX + 1] = {0}, nleaf[TMAX + 1] = {0};
  long long leaves = 0;
  for (int l = 0; l <= t->hmax; l++) {
    const size_t m = (size_t) ((1 << l) + 2)*((1 << l) + 2);
    for (size_t k = 0; k < m; k++) t->fl[l][k] &= ~(BMG_T_HALO | BMG_T_PROL);
  }
  for (int l = 0; l <= D; l++) {
    const int n = 1 << l;
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) {
        unsigned char * f = &t->fl[l][HX (l, i, j)];
        if (!(*f & BMG_T_ACTIVE)) continue;
        nact[l]++;
        if (!(*f & BMG_T_LEAF)) { nref[l]++; continue; }
        nleaf[l]++; leaves++;
        if (t->nb[l][HX (l, i, j)] > 0) {
          *f |= BMG_T_PROL;
          nprol[l]++;
          for (int c = 0; c < 4; c++)
            t->fl[l + 1][HX (l + 1, 2*i + (c >> 1), 2*j + (c & 1))] |= BMG_T_HALO;
        }
      }
  }
  t->nleaves = leaves;
  t->full = leaves == (1LL << (2*D));

  /* list layout: act, ref, prol per level, leaves, relax sets per level */
  long total = 0;
  for (int l = 0; l <= D; l++) {
    t->act[l].off = total; t->act[l].n = nact[l]; total += nact[l];
    t->ref[l].off = total; t->ref[l].n = nref[l]; total += nref[l];
    t->prol[l].off = total; t->prol[l].n = nprol[l]; total += nprol[l];
  }
  t->leaves.off = total; t->leaves.n = leaves; total += leaves;
  long below = 0;                      /* leaves of the levels under l */
  for (int l = 0; l <= D; l++) {
    t->rl[l].off = total; t->rl[l].n = nact[l] + below; total += t->rl[l].n;
    below += nleaf[l];
  }
  uint32_t * h = malloc ((total + 1)*sizeof (uint32_t));
  if (!h) return FAIL (BMG_ENOMEM);
  long pa[TMAX + 1], pr[TMAX + 1], pp[TMAX + 1], pl = t->leaves.off;
  for (int l = 0; l <= D; l++) { pa[l] = t->act[l].off; pr[l] = t->ref[l].off; pp[l] = t->prol[l].off; }
  for (int l = 0; l <= D; l++) {
    const int n = 1 << l;
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) {
        const unsigned char f = t->fl[l][HX (l, i, j)];
        if (!(f & BMG_T_ACTIVE)) continue;
        const uint32_t e = pack (l, i, j);
        h[pa[l]++] = e;
        if (!(f & BMG_T_LEAF)) h[pr[l]++] = e;
        else {
          h[pl++] = e;
          if (f & BMG_T_PROL) h[pp[l]++] = e;
        }
      }
  }
  /* relax set of level l (foreach_level_or_leaf): its active cells and the
     leaves below, red first */
  for (int l = 0; l <= D; l++) {
    long w = t->rl[l].off;
    for (int c = 0; c < 2; c++) {
      if (c == 1) t->rl1[l] = w - t->rl[l].off;
      for (int m = l; m >= 0; m--) {
        const int n = 1 << m;
        for (int i = 0; i < n; i++)
          for (int j = 0; j < n; j++) {
            const unsigned char f = t->fl[m][HX (m, i, j)];
            if (!(f & BMG_T_ACTIVE) || (m < l && !(f & BMG_T_LEAF)) || ((i + j) & 1) != c) continue;
            h[w++] = pack (m, i, j);
          }
      }
    }
  }
  /* ghost rules */
  long nrules = 0;
  for (int l = 0; l <= D; l++) nrules += 4L*(1 << l) + 4;
  bmg_tree_rule * hr = malloc ((nrules + 1)*sizeof (bmg_tree_rule));
  if (!hr) { free (h); return FAIL (BMG_ENOMEM); }
  long k = 0;
  for (int l = 0; l <= D; l++) {
    const int n = 1 << l;
    t->ghost[l].off = k;
    for (int gi = -1; gi <= n; gi++)
      for (int gj = -1; gj <= n; gj++) {
        if (!ghost_at (l, gi, gj)) continue;
        if (ghost_rule (t, l, gi, gj, &hr[k])) k++;
      }
    t->ghost[l].n = k - t->ghost[l].off;
  }
  /* device flags in the FP64 level layout */
  const size_t nfl = g->off64[g->depth + 1];
  unsigned char * hf = calloc (nfl, 1);
  if (!hf) { free (h); free (hr); return FAIL (BMG_ENOMEM); }
  for (int l = 0; l <= D; l++) {
    const int n = 1 << l;
    const bmg_geom * gg = &g->g64[l];
    for (int i = -1; i <= n; i++)
      for (int j = -1; j <= n; j++)
        hf[g->off64[l] + (size_t) (i + 1)*gg->P + gg->xo + j] = t->fl[l][HX (l, i, j)];
  }
  cudaFree (t->dflags); cudaFree (t->dlist); cudaFree (t->drules);
  t->dflags = NULL; t->dlist = NULL; t->drules = NULL;
  int st = BMG_OK;
  if (cudaMalloc ((void **) &t->dflags, nfl) != cudaSuccess ||
      cudaMalloc ((void **) &t->dlist, (total + 1)*sizeof (uint32_t)) != cudaSuccess ||
      cudaMalloc ((void **) &t->drules, (k + 1)*sizeof (bmg_tree_rule)) != cudaSuccess ||
      cudaMemcpy (t->dflags, hf, nfl, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy (t->dlist, h, total*sizeof (uint32_t), cudaMemcpyHostToDevice) != cudaSuccess ||
      (k && cudaMemcpy (t->drules, hr, k*sizeof (bmg_tree_rule), cudaMemcpyHostToDevice) != cudaSuccess))
    st = BMG_ENOMEM;
  free (h); free (hf);
  if (st) { free (hr); return FAIL (st); }
  /* boundary schedules */
  int mleaf = D;
  for (int l = D; l >= 0; l--) if (nleaf[l]) mleaf = l;
  free (t->stages); t->stages = NULL; t->nstages = 0;
  long cap = 0, nrs = 0, rcap = 0;
  bmg_tree_rule * rs = NULL;
  for (int kind = 0; kind < 2 && !st; kind++)
    for (int l = 0; l <= D && !st; l++) {
      const long first = t->nstages;
      st = schedule (t, l, kind == SCHED_FULL ? 0 : mleaf, hr, &t->stages, &t->nstages, &cap,
                     &rs, &nrs, &rcap);
      t->sched[kind][l].off = first;
      t->sched[kind][l].n = t->nstages - first;
    }
  free (hr);
  cudaFree (t->dsrules); t->dsrules = NULL;
  if (!st && (cudaMalloc ((void **) &t->dsrules, (nrs + 1)*sizeof (bmg_tree_rule)) != cudaSuccess ||
              (nrs && cudaMemcpy (t->dsrules, rs, nrs*sizeof (bmg_tree_rule),
                                  cudaMemcpyHostToDevice) != cudaSuccess)))
    st = BMG_ENOMEM;
  free (rs);
  if (st) return FAIL (st);
  memset (&t->T, 0, sizeof t->T);
  for (int l = 0; l <= g->depth && l <= TMAX; l++) {
    t->T.g[l] = g->g64[l];
    t->T.off[l] = (long long) g->off64[l];
    t->T.Delta[l] = g->L0*(1./(1 << l));
  }
  if (!t->dpart) {
    t->npart = 256;
    CKT (cudaMalloc ((void **) &t->dpart, (t->npart + 1)*sizeof (double)));
  }
  return BMG_OK;
}

int bmg_tree_refine (bmg_grid * g, bmg_refine_cond cond, void * data)
{
  if (!g || !cond || g->dim != 2 || g->depth > TMAX || g->periodic[0] || g->periodic[1])
    return FAIL (BMG_EINVAL);
  CKT (cudaSetDevice (g->device));
  struct bmg_tree * t = g->tree;
  if (!t) {
    t = calloc (1, sizeof (struct bmg_tree));
    if (!t) return FAIL (BMG_ENOMEM);
    t->hmax = g->depth;
    for (int l = 0; l <= t->hmax; l++) {
      const size_t m = (size_t) ((1 << l) + 2)*((1 << l) + 2);
      t->fl[l] = calloc (m, 1);
      t->nb[l] = calloc (m, sizeof (unsigned short));
      if (!t->fl[l] || !t->nb[l]) { tree_release (t); return FAIL (BMG_ENOMEM); }
    }
    t->fl[0][HX (0, 0, 0)] = BMG_T_ACTIVE | BMG_T_LEAF;     /* init_grid (1) */
    t->interp = getenv ("BMG_NO_TREE_INTERP") == NULL && bmg_tree_interp_available ();
    g->tree = t;
  }
  long count = 0, pass;
  int r;
  do {
    pass = 0;
    r = refine_pass (g, t, cond, data, &pass);
    count += pass;
  } while (!r && pass);
  if (r) { bmg_tree_free (g); return FAIL (r); }
  bmg_tree_graphs_clear (g);
  r = derive (g, t);
  if (r) { bmg_tree_free (g); return r; }
  FAIL (BMG_OK);
  return (int) (count > 0x7fffffff ? 0x7fffffff : count);
}

int bmg_tree_info (const bmg_grid * g, int * depth, long long * leaves)
{
  if (!g || !g->tree) return FAIL (BMG_EINVAL);
  if (depth) *depth = g->tree->depth;
  if (leaves) *leaves = g->tree->nleaves;
  return FAIL (BMG_OK);
}

int bmg_tree_flags (const bmg_grid * g, int level, unsigned char * out)
{
  if (!g || !g->tree || !out || level < 0 || level > g->tree->hmax) return FAIL (BMG_EINVAL);
  const int n = 1 << level;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++)
      out[(size_t) i*n + j] = g->tree->fl[level][HX (level, i, j)];
  return FAIL (BMG_OK);
}

/* ------------------------------------------------------------------ */
/* launch sequences                                                    */
/* ------------------------------------------------------------------ */

static bmg_tree_coef coef_of_field (bmg_grid * g, int handle, int want_face, double dflt, int * ok)
{
  bmg_tree_coef c = {NULL, dflt};
  if (!handle) return c;
  field_t * f = bmg_i_field (g, handle);
  if (!f || f->face_dim != want_face) { *ok = 0; return c; }
  if (f->is_const) c.c = f->cval;
  else c.p = f->buf;
  return c;
}

typedef struct { bmg_tree_coef ax, ay, lam; int ax_h, lam_h; } tcoefs;

static int resolve (bmg_grid * g, const struct Poisson * p, tcoefs * c)
{
  int ok = 1;
  memset (c, 0, sizeof *c);
  c->ax_h = p->alpha.x.i;
  c->lam_h = p->lambda.i;
  c->ax = coef_of_field (g, p->alpha.x.i, 0, 1., &ok);      /* unityf */
  c->ay = coef_of_field (g, p->alpha.x.i ? p->alpha.y.i : 0, 1, 1., &ok);
  c->lam = coef_of_field (g, p->lambda.i, -1, 0., &ok);     /* zeroc */
  return ok ? BMG_OK : FAIL (BMG_EINVAL);
}

/* the box conditions of field f on every level of the tree */
static void bc_of_field (const bmg_grid * g, const field_t * f, bmg_tree_bc * bc)
{
  memset (bc, 0, sizeof *bc);
  for (int s = 0; s < 4; s++) {
    bc->type[s] = f->bctype[s];
    bc->cval[s] = f->bccval[s];
    for (int l = 0; l <= g->depth && l <= TMAX; l++)
      bc->val[s][l] = f->bclv[s][l] ? f->bclv[s][l] : (l == g->depth ? f->bcval[s] : NULL);
  }
}

#define LIST(sp) (t->dlist + (sp).off), (sp).n

static int t_bc (bmg_grid * g, struct bmg_tree * t, double * s, int l, const bmg_tree_bc * bc,
                 int homog, long long * nl)
{
  if (t->ghost[l].n)
    LT (bmg_tree_launch_bc (t->drules + t->ghost[l].off, t->ghost[l].n, &t->T, s, bc, homog, g->stream));
  return BMG_OK;
}

/* tree_boundary_level (tree-common.h:588-716) of a cell field up to level
   l, by the stages of schedule () */
static int t_boundary (bmg_grid * g, struct bmg_tree * t, double * s, int l, const bmg_tree_bc * bc,
                       int homog, int kind, long long * nl)
{
  if (t->full) return t_bc (g, t, s, l, bc, homog, nl);
  const span_t sp = t->sched[kind][l];
  for (long k = 0; k < sp.n; k++) {
    const tstage * sg = &t->stages[sp.off + k];
    LT (bmg_tree_launch_stage (t->dlist + sg->list.off, sg->list.n, sg->op,
                               t->dsrules + sg->rules.off, sg->rules.n, &t->T, s, bc, homog,
                               g->stream));
  }
  return BMG_OK;
}

/* relax (poisson.h:271-338) of foreach_level_or_leaf (l) */
static int t_relax (bmg_grid * g, struct bmg_tree * t, double * da, const double * res, double * tmp,
                    const tcoefs * c, int l, const bmg_tree_bc * dabc, long long * nl)
{
  const span_t all = t->rl[l];
  if (g->relax == BMG_RELAX_JACOBI) {
    LT (bmg_tree_launch_relax (LIST (all), &t->T, da, res, c->ax, c->ay, c->lam, tmp, g->stream));
    LT (bmg_tree_launch_jacobi (LIST (all), &t->T, da, tmp, g->stream));
    return BMG_OK;
  }
  const span_t red = {all.off, t->rl1[l]}, black = {all.off + t->rl1[l], all.n - t->rl1[l]};
  if (red.n) LT (bmg_tree_launch_relax (LIST (red), &t->T, da, res, c->ax, c->ay, c->lam, da, g->stream));
  int r = t_boundary (g, t, da, l, dabc, 1, SCHED_PRUNED, nl);
  if (r) return r;
  if (black.n) LT (bmg_tree_launch_relax (LIST (black), &t->T, da, res, c->ax, c->ay, c->lam, da, g->stream));
  return BMG_OK;
}

/* mg_cycle (poisson.h:32-90) on the tree */
static int t_cycle (bmg_grid * g, struct bmg_tree * t, double * a, double * da, double * res,
                    double * tmp, const tcoefs * c, const bmg_tree_bc * dabc, int nrelax,
                    int minlevel, int maxlevel, long long * nl)
{
  /* restriction (res): the restriction part of tree_restriction */
  for (int m = t->depth - 1; m >= 0; m--)
    if (t->ref[m].n) LT (bmg_tree_launch_restrict (LIST (t->ref[m]), &t->T, res, g->stream));
  for (int l = minlevel; l <= maxlevel; l++) {
    if (l == minlevel)
      LT (bmg_tree_launch_set (LIST (t->rl[l]), &t->T, da, 0., g->stream));
    else
      LT (bmg_tree_launch_prolong (LIST (t->act[l]), &t->T, da, g->stream));
    int r = t_boundary (g, t, da, l, dabc, 1, SCHED_PRUNED, nl);
    if (r) return r;
    for (int i = 0; i < nrelax; i++) {
      r = t_relax (g, t, da, res, tmp, c, l, dabc, nl);
      if (r) return r;
      r = t_boundary (g, t, da, l, dabc, 1, SCHED_PRUNED, nl);
      if (r) return r;
    }
  }
  LT (bmg_tree_launch_add (LIST (t->leaves), &t->T, a, da, g->stream));
  return BMG_OK;
}

/* residual (poisson.h:355-372) into res, maximum into g->d_maxres */
static int t_residual (bmg_grid * g, struct bmg_tree * t, double * a, const double * b, double * res,
                       const tcoefs * c, const bmg_tree_bc * abc, long long * nl)
{
  int r = t_boundary (g, t, a, t->depth, abc, 0, SCHED_FULL, nl);
  if (r) return r;
  CKT (cudaMemsetAsync (g->d_maxres, 0, sizeof (unsigned long long), g->stream));
  LT (bmg_tree_launch_residual (LIST (t->leaves), &t->T, t->dflags, a, b, c->ax, c->ay, c->lam,
                                res, g->d_maxres, g->stream));
  return BMG_OK;
}

/* ------------------------------------------------------------------ */
/* the iteration as interpreter operations                             */
/* ------------------------------------------------------------------ */

/* the same operations, in the same order, as the launches of t_cycle and
   t_residual (an empty operation, which those skip, is left out) */
typedef struct {
  bmg_tree_op * v; long n, cap; int err; double bytes; int astored, lstored;
  double vb;            /* bytes of a value of the cycle's fields: 8, or 4 (mixed form) */
} opvec;
enum { F_A = 0, F_DA = 1, F_RES = 2, F_TMP = 3 };

/* algorithmic bytes of one item of an operation: each array value it
   reads or writes once at its storage precision (a, b and the residual's
   coefficients 8 B, the cycle's fields and coefficients o->vb), its list
   index (4 B) or ghost rule (16 B); alpha and lambda only when they are
   stored */
static double item_bytes (const opvec * o, int type, int sub, int rule, int field)
{
  const double w = field == F_A ? 8. : o->vb;
  const double ax = o->astored ? o->vb : 0., lam = o->lstored ? o->vb : 0.;
  const double ax8 = o->astored ? 8. : 0., lam8 = o->lstored ? 8. : 0.;
  if (rule) return 16. + w + w;                       /* rule, interior value, ghost */
  switch (type) {
  case BMG_TI_SET: return 4. + w;
  case BMG_TI_PROLONG: return 4. + 4*w + w;
  case BMG_TI_RESTRICT: return 4. + 4*w + w;
  case BMG_TI_STAGE: return sub == BMG_T_OP_HALO ? 1. + 4*w + w : 4. + 4*w + w;
  case BMG_TI_RELAX: return 4. + w + 4*w + 4*ax + lam + w;
  case BMG_TI_JACOBI: return 4. + 2*w + w;
  case BMG_TI_ADD: return 4. + 2*8. + o->vb;
  case BMG_TI_RESIDUAL: return 4. + 8. + 5*8. + 4*ax8 + lam8 + o->vb + 4.;
  }
  return 0.;
}

static void r_push (opvec * o, int type, int field, int sub, int homog, const uint32_t * list,
                    long n, const bmg_tree_rule * rules, long nr, double v)
{
  if (o->err) return;
  if (o->n == o->cap) {
    long cap = 2*o->cap + 256;
    bmg_tree_op * nv = realloc (o->v, cap*sizeof (bmg_tree_op));
    if (!nv) { o->err = 1; return; }
    o->v = nv; o->cap = cap;
  }
  const long items = type == BMG_TI_STAGE ? (sub == BMG_T_OP_HALO ? 4*n : sub == BMG_T_OP_RESTRICT ? n : 0) : n;
  o->bytes += items*item_bytes (o, type, sub, 0, field) + nr*item_bytes (o, type, sub, 1, field);
  bmg_tree_op * q = &o->v[o->n++];
  memset (q, 0, sizeof *q);
  q->type = type; q->field = field; q->sub = sub; q->homog = homog; q->bcsel = 0;
  q->list = list; q->n = n; q->rules = rules; q->nr = nr; q->v = v;
  /* at most two items a thread of one 1024-thread CTA: run on one CTA
     (measured on the depth-11 band tree: 772 ms per solve with no local
     operations, 645-684 with at most 1024-2048 items, 690-1034 above) */
  q->local = items + nr <= 2048;
}

static void r_boundary (struct bmg_tree * t, opvec * o, int field, int l, int homog, int kind)
{
  if (t->full) {
    if (t->ghost[l].n)
      r_push (o, BMG_TI_STAGE, field, BMG_T_OP_NONE, homog, NULL, 0,
              t->drules + t->ghost[l].off, t->ghost[l].n, 0.);
    return;
  }
  const span_t sp = t->sched[kind][l];
  for (long k = 0; k < sp.n; k++) {
    const tstage * sg = &t->stages[sp.off + k];
    const long w = (sg->op == BMG_T_OP_HALO ? 4*sg->list.n : sg->op == BMG_T_OP_RESTRICT ?
                    sg->list.n : 0) + sg->rules.n;
    if (w <= 0) continue;
    r_push (o, BMG_TI_STAGE, field, sg->op, homog, t->dlist + sg->list.off, sg->list.n,
            t->dsrules + sg->rules.off, sg->rules.n, 0.);
  }
}

static void r_relax (bmg_grid * g, struct bmg_tree * t, opvec * o, int l)
{
  const span_t all = t->rl[l];
  if (g->relax == BMG_RELAX_JACOBI) {
    if (all.n) {
      r_push (o, BMG_TI_RELAX, F_DA, 1, 0, t->dlist + all.off, all.n, NULL, 0, 0.);
      r_push (o, BMG_TI_JACOBI, F_DA, 0, 0, t->dlist + all.off, all.n, NULL, 0, 0.);
    }
    return;
  }
  const span_t red = {all.off, t->rl1[l]}, black = {all.off + t->rl1[l], all.n - t->rl1[l]};
  if (red.n) r_push (o, BMG_TI_RELAX, F_DA, 0, 0, t->dlist + red.off, red.n, NULL, 0, 0.);
  r_boundary (t, o, F_DA, l, 1, SCHED_PRUNED);
  if (black.n) r_push (o, BMG_TI_RELAX, F_DA, 0, 0, t->dlist + black.off, black.n, NULL, 0, 0.);
}

static void r_iteration (bmg_grid * g, struct bmg_tree * t, opvec * o, int nrelax, int minlevel,
                         int maxlevel)
{
  for (int m = t->depth - 1; m >= 0; m--)
    if (t->ref[m].n)
      r_push (o, BMG_TI_RESTRICT, F_RES, 0, 0, t->dlist + t->ref[m].off, t->ref[m].n, NULL, 0, 0.);
  for (int l = minlevel; l <= maxlevel; l++) {
    if (l == minlevel) {
      if (t->rl[l].n)
        r_push (o, BMG_TI_SET, F_DA, 0, 0, t->dlist + t->rl[l].off, t->rl[l].n, NULL, 0, 0.);
    }
    else if (t->act[l].n)
      r_push (o, BMG_TI_PROLONG, F_DA, 0, 0, t->dlist + t->act[l].off, t->act[l].n, NULL, 0, 0.);
    r_boundary (t, o, F_DA, l, 1, SCHED_PRUNED);
    for (int i = 0; i < nrelax; i++) {
      r_relax (g, t, o, l);
      r_boundary (t, o, F_DA, l, 1, SCHED_PRUNED);
    }
  }
  if (t->leaves.n)
    r_push (o, BMG_TI_ADD, F_A, 0, 0, t->dlist + t->leaves.off, t->leaves.n, NULL, 0, 0.);
  r_boundary (t, o, F_A, t->depth, 0, SCHED_FULL);
  if (t->leaves.n)
    r_push (o, BMG_TI_RESIDUAL, F_RES, 0, 0, t->dlist + t->leaves.off, t->leaves.n, NULL, 0, 0.);
}

static int read_max (bmg_grid * g, double * m)
{
  CKT (cudaMemcpyAsync (g->h_pinned, g->d_maxres, sizeof (double), cudaMemcpyDeviceToHost, g->stream));
  CKT (cudaStreamSynchronize (g->stream));
  *m = g->h_pinned[0];
  return BMG_OK;
}

/* one mg_solve iteration (cycle, residual, maximum to pinned memory),
   captured once per key and replayed */
static int t_iteration (bmg_grid * g, struct bmg_tree * t, const tkey * key, double * a,
                        const double * b, double * da, double * res, double * tmp, const tcoefs * c,
                        const bmg_tree_bc * abc)
{
  long long launches = 0, * nl = &launches;
  if (!g->use_graphs) {
    int r = t_cycle (g, t, a, da, res, tmp, c, abc, key->nrelax, key->minlevel, key->maxlevel, nl);
    if (!r) r = t_residual (g, t, a, b, res, c, abc, nl);
    if (r) return r;
    CKT (cudaMemcpyAsync (g->h_pinned, g->d_maxres, sizeof (double), cudaMemcpyDeviceToHost, g->stream));
    g->counters.launches += launches;
    return BMG_OK;
  }
  struct tgraph * e = NULL, * victim = &t->graphs[0];
  for (int i = 0; i < NTGRAPH; i++) {
    struct tgraph * q = &t->graphs[i];
    if (q->valid && !memcmp (&q->key, key, sizeof *key)) { e = q; break; }
    if (!q->valid || q->stamp < victim->stamp) victim = q;
  }
  if (!e && t->interp) {
    /* the iteration as one interpreter launch, its operations uploaded once */
    graph_drop (victim);
    opvec o = {NULL, 0, 0, 0, 0., c->ax.p != NULL, c->lam.p != NULL, 8.};
    r_iteration (g, t, &o, key->nrelax, key->minlevel, key->maxlevel);
    victim->bytes = o.bytes;
    if (o.err) { free (o.v); return FAIL (BMG_ENOMEM); }
    if (cudaMalloc ((void **) &victim->dops, (o.n + 1)*sizeof (bmg_tree_op)) != cudaSuccess ||
        (o.n && cudaMemcpy (victim->dops, o.v, o.n*sizeof (bmg_tree_op), cudaMemcpyHostToDevice)
         != cudaSuccess)) {
      free (o.v);
      cudaGetLastError ();
      graph_drop (victim);
      return FAIL (BMG_ENOMEM);
    }
    victim->nops = o.n;
    free (o.v);
    double * fields[4] = {a, da, res, tmp};
    const bmg_tree_coef co[3] = {c->ax, c->ay, c->lam};
    const bmg_tree_bc bcs[2] = {*abc, *abc};
    cudaGraph_t graph;
    CKT (cudaStreamBeginCapture (g->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t me = cudaMemsetAsync (g->d_maxres, 0, sizeof (unsigned long long), g->stream);
    int r = me == cudaSuccess ?
      bmg_tree_launch_interp (victim->dops, (int) victim->nops, &t->T, fields, b, t->dflags, co,
                              bcs, g->d_maxres, g->stream) : (int) me;
    me = cudaMemcpyAsync (g->h_pinned, g->d_maxres, sizeof (double), cudaMemcpyDeviceToHost,
                          g->stream);
    cudaError_t ee = cudaStreamEndCapture (g->stream, &graph);
    if (r) {
      if (ee == cudaSuccess) cudaGraphDestroy (graph);
      fprintf (stderr, "bmg: tree interpreter launch failed (%d)\n", r);
      graph_drop (victim);
      return FAIL (BMG_ECUDA);
    }
    CKT (me);
    CKT (ee);
    cudaError_t ie = cudaGraphInstantiate (&victim->exec, graph, 0);
    cudaGraphDestroy (graph);
    CKT (ie);
    victim->key = *key;
    victim->launches = 1;
    victim->valid = 1;
    e = victim;
  }
  if (!e) {
    graph_drop (victim);
    {
      /* the same iteration's algorithmic bytes, from its operation list */
      opvec o = {NULL, 0, 0, 0, 0., c->ax.p != NULL, c->lam.p != NULL, 8.};
      r_iteration (g, t, &o, key->nrelax, key->minlevel, key->maxlevel);
      victim->bytes = o.bytes;
      free (o.v);
    }
    cudaGraph_t graph;
    CKT (cudaStreamBeginCapture (g->stream, cudaStreamCaptureModeThreadLocal));
    int r = t_cycle (g, t, a, da, res, tmp, c, abc, key->nrelax, key->minlevel, key->maxlevel, nl);
    if (!r) r = t_residual (g, t, a, b, res, c, abc, nl);
    cudaError_t me = cudaMemcpyAsync (g->h_pinned, g->d_maxres, sizeof (double),
                                      cudaMemcpyDeviceToHost, g->stream);
    cudaError_t ee = cudaStreamEndCapture (g->stream, &graph);
    if (r) { if (ee == cudaSuccess) cudaGraphDestroy (graph); return r; }
    CKT (me);
    CKT (ee);
    cudaError_t ie = cudaGraphInstantiate (&victim->exec, graph, 0);
    cudaGraphDestroy (graph);
    CKT (ie);
    victim->key = *key;
    victim->launches = launches;
    victim->valid = 1;
    e = victim;
  }
  e->stamp = ++t->clock;
  CKT (cudaGraphLaunch (e->exec, g->stream));
  g->counters.launches += e->launches;
  g->counters.bytes += e->bytes;
  return BMG_OK;
}

/* one iteration of the mixed form: the operations of r_iteration run by
   the FP32 interpreter (bmg_tree_launch_interp_mixed), captured once per
   key with the upload of its operations, and replayed */
static int t_iteration_mixed (bmg_grid * g, struct bmg_tree * t, const tkey * key, double * a,
                              const double * b, float * const * f32, const tcoefs * c,
                              const bmg_tree_coef32 * c32, const bmg_tree_bc * abc)
{
  struct tgraph * e = NULL, * victim = &t->graphs[0];
  for (int i = 0; i < NTGRAPH; i++) {
    struct tgraph * q = &t->graphs[i];
    if (q->valid && !memcmp (&q->key, key, sizeof *key)) { e = q; break; }
    if (!q->valid || q->stamp < victim->stamp) victim = q;
  }
  if (!e) {
    graph_drop (victim);
    opvec o = {NULL, 0, 0, 0, 0., c->ax.p != NULL, c->lam.p != NULL, 4.};
    r_iteration (g, t, &o, key->nrelax, key->minlevel, key->maxlevel);
    victim->bytes = o.bytes;
    if (o.err) { free (o.v); return FAIL (BMG_ENOMEM); }
    if (cudaMalloc ((void **) &victim->dops, (o.n + 1)*sizeof (bmg_tree_op)) != cudaSuccess ||
        (o.n && cudaMemcpy (victim->dops, o.v, o.n*sizeof (bmg_tree_op), cudaMemcpyHostToDevice)
         != cudaSuccess)) {
      free (o.v);
      cudaGetLastError ();
      graph_drop (victim);
      return FAIL (BMG_ENOMEM);
    }
    victim->nops = o.n;
    free (o.v);
    const bmg_tree_coef co[3] = {c->ax, c->ay, c->lam};
    const bmg_tree_bc bcs[2] = {*abc, *abc};
    cudaGraph_t graph;
    CKT (cudaStreamBeginCapture (g->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t me = cudaMemsetAsync (g->d_maxres, 0, sizeof (unsigned long long), g->stream);
    int r = me == cudaSuccess ?
      bmg_tree_launch_interp_mixed (victim->dops, (int) victim->nops, &t->T, a, f32, b,
                                    t->dflags, co, c32, bcs, g->d_maxres, g->stream) : (int) me;
    me = cudaMemcpyAsync (g->h_pinned, g->d_maxres, sizeof (double), cudaMemcpyDeviceToHost,
                          g->stream);
    cudaError_t ee = cudaStreamEndCapture (g->stream, &graph);
    if (r) {
      if (ee == cudaSuccess) cudaGraphDestroy (graph);
      fprintf (stderr, "bmg: tree interpreter launch (mixed) failed (%d)\n", r);
      graph_drop (victim);
      return FAIL (BMG_ECUDA);
    }
    CKT (me);
    CKT (ee);
    cudaError_t ie = cudaGraphInstantiate (&victim->exec, graph, 0);
    cudaGraphDestroy (graph);
    CKT (ie);
    victim->key = *key;
    victim->launches = 1;
    victim->valid = 1;
    e = victim;
  }
  e->stamp = ++t->clock;
  CKT (cudaGraphLaunch (e->exec, g->stream));
  g->counters.launches += e->launches;
  g->counters.bytes += e->bytes;
  return BMG_OK;
}

/* the mixed form's FP32 workspace, allocated on its first solve */
static int t_workspace32 (bmg_grid * g, struct bmg_tree * t)
{
  if (t->ws32) return BMG_OK;
  const size_t n = g->off64[g->depth + 1];
  CKT (cudaMalloc ((void **) &t->ws32, (size_t) W32_N*n*sizeof (float)));
  CKT (cudaMemsetAsync (t->ws32, 0, (size_t) W32_N*n*sizeof (float), g->stream));
  return BMG_OK;
}

/* mg_solve (poisson.h:139-235) on the tree, Poisson callbacks */
static int t_solve (bmg_grid * g, field_t * a, field_t * b, const tcoefs * c, int nrelax,
                    field_t * resout, int minlevel, double tolerance, mgstats * out)
{
  struct bmg_tree * t = g->tree;
  const int mixed = g->precision == BMG_MIXED;
  /* the mixed form runs its iterations through the interpreter only */
  if (mixed && !t->interp) return FAIL (BMG_EUNSUPPORTED);
  int r = bmg_i_workspace (g);
  if (r) return r;
  if (mixed && (r = t_workspace32 (g, t))) return r;
  if (minlevel > t->depth) minlevel = t->depth;
  if (minlevel < 0) minlevel = 0;
  double * da = bmg_i_ws64 (g, BMG_WS_DA, 0), * tmp = bmg_i_ws64 (g, BMG_WS_DA2, 0);
  double * res = bmg_i_ws64 (g, BMG_WS_RES, 0);
  bmg_tree_bc abc;
  bc_of_field (g, a, &abc);
  mgstats s;
  memset (&s, 0, sizeof s);
  long long launches = 0, * nl = &launches;
  /* sum of the r.h.s. over the leaves (poisson.h:162-167) */
  LT (bmg_tree_launch_sum (LIST (t->leaves), &t->T, b->buf, t->dpart, t->npart, g->d_sum, g->stream));
  CKT (cudaMemcpyAsync (g->h_pinned + 1, g->d_sum, sizeof (double), cudaMemcpyDeviceToHost, g->stream));
  CKT (cudaStreamSynchronize (g->stream));
  s.sum = g->h_pinned[1];
  s.nrelax = nrelax > 0 ? nrelax : 4;
  r = t_residual (g, t, a->buf, b->buf, res, c, &abc, nl);
  if (r) return r;
  /* mixed form: FP32 copies of the initial residual and of the
     coefficients the cycle reads (all levels) */
  const long long n32 = (long long) g->off64[g->depth + 1];
  float * const f32[3] = {t->ws32 ? t->ws32 + (size_t) W32_DA*n32 : NULL,
                          t->ws32 ? t->ws32 + (size_t) W32_RES*n32 : NULL,
                          t->ws32 ? t->ws32 + (size_t) W32_TMP*n32 : NULL};
  bmg_tree_coef32 c32[3] = {{NULL, c->ax.c}, {NULL, c->ay.c}, {NULL, c->lam.c}};
  if (mixed) {
    LT (bmg_tree_launch_to_f32 (res, f32[1], n32, g->stream));
    const bmg_tree_coef * c64[3] = {&c->ax, &c->ay, &c->lam};
    for (int k = 0; k < 3; k++)
      if (c64[k]->p) {
        float * dst = t->ws32 + (size_t) (W32_AX + k)*n32;
        LT (bmg_tree_launch_to_f32 (c64[k]->p, dst, n32, g->stream));
        c32[k].p = dst;
      }
  }
  r = read_max (g, &s.resb);
  if (r) return r;
  g->counters.launches += launches;
  double resb = s.resa = s.resb;
  if (tolerance == 0.)
    tolerance = TOLERANCE;
  tkey key;
  memset (&key, 0, sizeof key);
  key.minlevel = minlevel; key.maxlevel = t->depth; key.relax = g->relax; key.mixed = mixed;
  key.a = a->buf; key.b = b->buf;
  key.da = mixed ? (const void *) f32[0] : da;
  key.res = mixed ? (const void *) f32[1] : res;
  key.tmp = mixed ? (const void *) f32[2] : tmp;
  key.ax = c->ax; key.ay = c->ay; key.lam = c->lam; key.abc = abc;
  key.stream = g->stream; key.maxres = g->d_maxres; key.pinned = g->h_pinned;
  int status = BMG_OK;
  for (s.i = 0; s.i < NITERMAX && (s.i < NITERMIN || s.resa > tolerance); s.i++) {
    key.nrelax = s.nrelax;
    if (g->timing) CKT (cudaEventRecord (g->ev0, g->stream));
    r = mixed ? t_iteration_mixed (g, t, &key, a->buf, b->buf, f32, c, c32, &abc)
              : t_iteration (g, t, &key, a->buf, b->buf, da, res, tmp, c, &abc);
    if (r) return r;
    if (g->timing) CKT (cudaEventRecord (g->ev1, g->stream));
    CKT (cudaStreamSynchronize (g->stream));
    s.resa = g->h_pinned[0];
    g->counters.cycles++;
    if (g->timing) {
      float ms = 0.f;
      CKT (cudaEventElapsedTime (&ms, g->ev0, g->ev1));
      g->counters.cycle_ms += ms;
    }
    if (!isfinite (s.resa)) { status = BMG_ENAN; s.i++; break; }
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
    if (mixed) {
      /* the FP64 residual of the final a (the iterations kept it in FP32) */
      launches = 0;
      r = t_residual (g, t, a->buf, b->buf, res, c, &abc, nl);
      if (r) return r;
      g->counters.launches += launches;
    }
    CKT (cudaMemcpyAsync (resout->buf, res, g->off64[g->depth + 1]*sizeof (double),
                          cudaMemcpyDeviceToDevice, g->stream));
  }
  CKT (cudaStreamSynchronize (g->stream));
  *out = s;
  return FAIL (status);
}

/* restriction ({alpha, lambda}) on the tree (poisson.h:418-420) */
static int t_restrict_coefs (bmg_grid * g, struct bmg_tree * t, const tcoefs * c)
{
  long long n0 = 0, * nl = &n0;
  for (int m = t->depth - 1; m >= 0; m--) {
    if (c->ax.p && c->ay.p && t->ref[m].n)
      LT (bmg_tree_launch_restrict_faces (LIST (t->ref[m]), &t->T, t->dflags,
                                          (double *) c->ax.p, (double *) c->ay.p, g->stream));
    if (c->lam.p && t->ref[m].n)
      LT (bmg_tree_launch_restrict (LIST (t->ref[m]), &t->T, (double *) c->lam.p, g->stream));
  }
  return BMG_OK;
}

static int cell_field (bmg_grid * g, int h, field_t ** f)
{
  *f = bmg_i_field (g, h);
  if (!*f || (*f)->is_const || (*f)->face_dim >= 0) return FAIL (BMG_EINVAL);
  return BMG_OK;
}

int bmg_tree_poisson (bmg_grid * g, struct Poisson p, mgstats * out)
{
  field_t * a, * b, * res = NULL;
  if (cell_field (g, p.a.i, &a) || cell_field (g, p.b.i, &b)) return FAIL (BMG_EINVAL);
  if (p.res && p.res[0].i && cell_field (g, p.res[0].i, &res)) return FAIL (BMG_EINVAL);
  tcoefs c;
  int r = resolve (g, &p, &c);
  if (r) return r;
  r = t_restrict_coefs (g, g->tree, &c);
  if (r) return r;
  /* p.tolerance for this solve, without touching the global TOLERANCE
     (see bmg_poisson) */
  r = t_solve (g, a, b, &c, p.nrelax, res, p.minlevel > 1 ? p.minlevel : 1,
               p.tolerance ? p.tolerance : TOLERANCE, out);
  return FAIL (r);
}

int bmg_tree_mg_solve (bmg_grid * g, struct MGSolve p, mgstats * out)
{
  field_t * a, * b, * res = NULL;
  if (cell_field (g, p.a[0].i, &a) || cell_field (g, p.b[0].i, &b)) return FAIL (BMG_EINVAL);
  if (p.res && p.res[0].i && cell_field (g, p.res[0].i, &res)) return FAIL (BMG_EINVAL);
  tcoefs c;
  int r = resolve (g, (struct Poisson *) p.data, &c);
  if (r) return r;
  return t_solve (g, a, b, &c, p.nrelax, res, p.minlevel, p.tolerance, out);
}

int bmg_tree_mg_cycle (bmg_grid * g, field_t * a, field_t * res, field_t * da,
                       struct Poisson * p, int nrelax, int minlevel, int maxlevel)
{
  struct bmg_tree * t = g->tree;
  tcoefs c;
  int r = resolve (g, p, &c);
  if (r) return r;
  r = bmg_i_workspace (g);
  if (r) return r;
  if (maxlevel > t->depth) maxlevel = t->depth;
  minlevel = minlevel < maxlevel ? minlevel : maxlevel;      /* poisson.h:48 */
  if (minlevel < 0) minlevel = 0;
  bmg_tree_bc dabc;
  bc_of_field (g, da, &dabc);
  long long launches = 0;
  r = t_cycle (g, t, a->buf, da->buf, res->buf, bmg_i_ws64 (g, BMG_WS_DA2, 0), &c, &dabc,
               nrelax, minlevel, maxlevel, &launches);
  if (r) return r;
  CKT (cudaStreamSynchronize (g->stream));
  g->counters.launches += launches;
  g->counters.cycles++;
  return FAIL (BMG_OK);
}

int bmg_tree_relax (bmg_grid * g, field_t * da, field_t * res, int level, struct Poisson * p)
{
  struct bmg_tree * t = g->tree;
  if (level > t->depth) return FAIL (BMG_EINVAL);
  tcoefs c;
  int r = resolve (g, p, &c);
  if (r) return r;
  r = bmg_i_workspace (g);
  if (r) return r;
  bmg_tree_bc dabc;
  bc_of_field (g, da, &dabc);
  long long launches = 0;
  r = t_relax (g, t, da->buf, res->buf, bmg_i_ws64 (g, BMG_WS_DA2, 0), &c, level, &dabc, &launches);
  if (r) return r;
  CKT (cudaStreamSynchronize (g->stream));
  return FAIL (BMG_OK);
}

int bmg_tree_residual (bmg_grid * g, field_t * a, field_t * b, field_t * res,
                       struct Poisson * p, double * maxres)
{
  tcoefs c;
  int r = resolve (g, p, &c);
  if (r) return r;
  bmg_tree_bc abc;
  bc_of_field (g, a, &abc);
  long long launches = 0;
  r = t_residual (g, g->tree, a->buf, b->buf, res->buf, &c, &abc, &launches);
  if (r) return r;
  r = read_max (g, maxres);
  if (r) return r;
  return FAIL (BMG_OK);
}

/* restriction (list) on a tree (tree_restriction = boundary (list),
   tree-common.h:795-799): face vectors by face_average, cell fields by the
   whole tree boundary with their own conditions */
int bmg_tree_restriction (bmg_grid * g, const bmg_scalar * list)
{
  struct bmg_tree * t = g->tree;
  long long launches = 0, * nl = &launches;
  for (const bmg_scalar * s = list; s->i; s++) {
    field_t * f = bmg_i_field (g, s->i);
    if (!f) return FAIL (BMG_EINVAL);
    if (f->is_const) continue;
    if (f->face_dim >= 0) {
      if (f->face_dim != 0) continue;
      field_t * fy = bmg_i_field (g, s->i + 1);
      if (!fy || fy->face_dim != 1) return FAIL (BMG_EINVAL);
      for (int m = t->depth - 1; m >= 0; m--)
        if (t->ref[m].n)
          LT (bmg_tree_launch_restrict_faces (LIST (t->ref[m]), &t->T, t->dflags, f->buf, fy->buf,
                                              g->stream));
    }
    else {
      bmg_tree_bc bc;
      bc_of_field (g, f, &bc);
      int r = t_boundary (g, t, f->buf, t->depth, &bc, 0, SCHED_FULL, nl);
      if (r) return r;
    }
  }
  CKT (cudaStreamSynchronize (g->stream));
  return FAIL (BMG_OK);
}

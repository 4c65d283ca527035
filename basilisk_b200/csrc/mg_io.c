/*
 * mg_io.c -- Basilisk snapshots: dump () and restore () (output.h:1043-1300)
 * for the grids of this library, so that fields of a reference simulation
 * can be solved for here and results read back by the reference's tools.
 *
 * The file is the reference's (dump_version 170901, single process):
 *   struct DumpHeader {double t; long len; int i, depth, npe, version;
 *                      coord n;}                         (output.h:1049-1053)
 *   len names: unsigned length, then the characters (no terminator); the
 *     first is "size", the number of cells of each subtree (subtree_size,
 *     multigrid-common.h:422-440)                          (output.h:1070-1086)
 *   double o[4] = {X0, Y0, Z0, L0}                         (output.h:1087-1091)
 *   every cell of foreach_cell () (depth first, children in index order,
 *   not below leaves): unsigned flags (leaf = 2), then one double per name
 *                                                          (output.h:1122-1135)
 * A uniform grid dumps every cell of every level (its leaves are the
 * finest level, grid/multigrid.h:244); a tree its active cells.  restore ()
 * matches the names of the file with the caller's fields, skips the
 * others, and turns the grid into a quadtree when the file holds one
 * (refine_cell where a dumped cell is not a leaf, output.h:1357-1360).
 * This is host I/O around the device fields; no solver arithmetic.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <cuda_runtime_api.h>

#include "mg_grid.h"

#define FAIL(s) bmg_i_fail (s)
#define DUMP_VERSION 170901
#define LEAF 2

typedef struct {
  double t;
  long len;
  int i, depth, npe, version;
  double n[3];
} dump_header;

/* the level arrays of the listed fields, in host memory (compact layout) */
typedef struct {
  int nf, depth, dim;
  double * v[64][BMG_MAXLEVEL + 1];
} host_fields;

static void free_fields (host_fields * h)
{
  for (int f = 0; f < h->nf; f++)
    for (int l = 0; l <= h->depth; l++) free (h->v[f][l]);
}

static size_t ncells (int dim, int l)
{
  size_t n = 1;
  for (int d = 0; d < dim; d++) n *= (size_t) 1 << l;
  return n;
}

static size_t cell_index (int dim, int l, int i, int j, int k)
{
  const size_t n = (size_t) 1 << l;
  return dim == 1 ? (size_t) i : dim == 2 ? (size_t) i*n + j : ((size_t) i*n + j)*n + k;
}

static int is_leaf_cell (bmg_grid * g, const unsigned char * const * fl, int l, int i, int j, int k)
{
  if (!g->tree) return l == g->depth;
  (void) k;
  return (fl[l][cell_index (2, l, i, j, 0)] & BMG_TREE_LEAF) != 0;
}

/* the number of cells of every cell's subtree, level by level from the
   deepest: 1 for a leaf, 1 + the children's sums otherwise
   (subtree_size (size, false), multigrid-common.h:422-440) */
static int subtree_sizes (bmg_grid * g, const unsigned char * const * fl, int depth, double ** sz)
{
  for (int l = depth; l >= 0; l--) {
    const int n = 1 << l;
    const size_t nc = ncells (g->dim, l);
    if (!(sz[l] = malloc (nc*sizeof (double)))) return BMG_ENOMEM;
    for (size_t q = 0; q < nc; q++) {
      const int i = g->dim == 1 ? (int) q : g->dim == 2 ? (int) (q/n) : (int) (q/((size_t) n*n));
      const int j = g->dim == 1 ? 0 : g->dim == 2 ? (int) (q % n) : (int) ((q/n) % n);
      const int k = g->dim == 3 ? (int) (q % n) : 0;
      double s = 1.;
      if (l < depth && !is_leaf_cell (g, fl, l, i, j, k))
        for (int c = 0; c < (1 << g->dim); c++) {
          const int ci = 2*i + ((c >> (g->dim - 1)) & 1);
          const int cj = g->dim > 1 ? 2*j + ((c >> (g->dim - 2)) & 1) : 0;
          const int ck = g->dim > 2 ? 2*k + (c & 1) : 0;
          s += sz[l + 1][cell_index (g->dim, l + 1, ci, cj, ck)];
        }
      sz[l][q] = s;
    }
  }
  return BMG_OK;
}

typedef struct {
  FILE * fp;
  bmg_grid * g;
  const unsigned char * const * fl;
  host_fields * h;
  double ** sz;
  int depth, err;
} dump_ctx;

static void dump_cell (dump_ctx * c, int l, int i, int j, int k)
{
  if (c->err) return;
  const int leaf = is_leaf_cell (c->g, c->fl, l, i, j, k);
  const unsigned flags = leaf ? LEAF : 0;
  const size_t id = cell_index (c->g->dim, l, i, j, k);
  const double size = c->sz[l][id];
  if (fwrite (&flags, sizeof flags, 1, c->fp) != 1 || fwrite (&size, sizeof size, 1, c->fp) != 1) {
    c->err = 1;
    return;
  }
  for (int f = 0; f < c->h->nf; f++)
    if (fwrite (&c->h->v[f][l][id], sizeof (double), 1, c->fp) != 1) { c->err = 1; return; }
  if (leaf) return;
  const int nc = 1 << c->g->dim;
  for (int q = 0; q < nc; q++) {
    const int ci = 2*i + ((q >> (c->g->dim - 1)) & 1);
    const int cj = c->g->dim > 1 ? 2*j + ((q >> (c->g->dim - 2)) & 1) : 0;
    const int ck = c->g->dim > 2 ? 2*k + (q & 1) : 0;
    dump_cell (c, l + 1, ci, cj, ck);
  }
}

static int load_fields (bmg_grid * g, const bmg_scalar * list, int depth, host_fields * h)
{
  memset (h, 0, sizeof *h);
  h->depth = depth; h->dim = g->dim;
  for (const bmg_scalar * s = list; s && s->i; s++) {
    if (h->nf == 64) return BMG_EINVAL;
    for (int l = 0; l <= depth; l++) {
      const size_t n = ncells (g->dim, l);
      h->v[h->nf][l] = malloc (n*sizeof (double));
      if (!h->v[h->nf][l]) { h->nf++; return BMG_ENOMEM; }
      int r = bmg_field_get_level (g, *s, l, h->v[h->nf][l], n, BMG_HOST);
      if (r) { h->nf++; return r; }
    }
    h->nf++;
  }
  return BMG_OK;
}

int bmg_dump (bmg_grid * g, const char * file, const bmg_scalar * list,
              const char * const * names, double t, int iter)
{
  if (!g || !file || !list || !names) return FAIL (BMG_EINVAL);
  if (g->tree && g->dim != 2) return FAIL (BMG_EINVAL);
  int depth = g->depth;
  long long leaves = 0;
  unsigned char * fl[BMG_MAXLEVEL + 1] = {NULL};
  if (g->tree) {
    int d;
    if (bmg_tree_info (g, &d, &leaves)) return FAIL (BMG_EINVAL);
    depth = d;
    for (int l = 0; l <= depth; l++) {
      fl[l] = malloc (ncells (2, l));
      if (!fl[l] || bmg_tree_flags (g, l, fl[l])) {
        for (int m = 0; m <= l; m++) free (fl[m]);
        return FAIL (BMG_ENOMEM);
      }
    }
  }
  host_fields h;
  double * sz[BMG_MAXLEVEL + 1] = {NULL};
  int r = load_fields (g, list, depth, &h);
  if (!r) r = subtree_sizes (g, (const unsigned char * const *) fl, depth, sz);
  /* written to file~ then renamed (output.h:1101-1108, 1138-1143) */
  char * tmp = malloc (strlen (file) + 2);
  if (!tmp) r = BMG_ENOMEM;
  else { strcpy (tmp, file); strcat (tmp, "~"); }
  FILE * fp = r ? NULL : fopen (tmp, "wb");
  if (!r && !fp) r = BMG_EINVAL;
  if (!r) {
    dump_header hd;
    memset (&hd, 0, sizeof hd);
    hd.t = t; hd.len = h.nf + 1; hd.i = iter; hd.depth = depth; hd.npe = 1;
    hd.version = DUMP_VERSION;
    int ok = fwrite (&hd, sizeof hd, 1, fp) == 1;
    const char * size = "size";
    for (int f = -1; ok && f < h.nf; f++) {
      const char * nm = f < 0 ? size : names[f];
      const unsigned len = (unsigned) strlen (nm);
      ok = fwrite (&len, sizeof len, 1, fp) == 1 && fwrite (nm, 1, len, fp) == len;
    }
    const double o[4] = {g->X0, g->Y0, g->Z0, g->L0};
    ok = ok && fwrite (o, sizeof (double), 4, fp) == 4;
    dump_ctx c = {fp, g, (const unsigned char * const *) fl, &h, sz, depth, !ok};
    dump_cell (&c, 0, 0, 0, 0);
    if (fclose (fp) || c.err || rename (tmp, file)) r = BMG_EINVAL;
  }
  free (tmp);
  free_fields (&h);
  for (int l = 0; l <= depth; l++) { free (fl[l]); free (sz[l]); }
  return FAIL (r);
}

/* ------------------------------------------------------------------ */
/* restore                                                             */
/* ------------------------------------------------------------------ */

/* the cells of a dump, as read: (level, index, leaf) and the values of the
   matched fields */
typedef struct {
  int dim;
  long ncell, cap;
  unsigned char * level, * leaf;
  int * ii, * jj, * kk;
} cells_t;

/* grows *p to n elements of size sz; on failure *p is left as it was (and
   freed by the caller) */
static int grow (void ** p, size_t n, size_t sz)
{
  void * q = realloc (*p, n*sz);
  if (!q) return BMG_ENOMEM;
  *p = q;
  return BMG_OK;
}

static int push_cell (cells_t * c, int l, int i, int j, int k, int leaf)
{
  if (c->ncell == c->cap) {
    const long cap = 2*c->cap + 1024;
    if (grow ((void **) &c->level, cap, 1) || grow ((void **) &c->leaf, cap, 1) ||
        grow ((void **) &c->ii, cap, sizeof (int)) || grow ((void **) &c->jj, cap, sizeof (int)) ||
        grow ((void **) &c->kk, cap, sizeof (int)))
      return BMG_ENOMEM;
    c->cap = cap;
  }
  c->level[c->ncell] = (unsigned char) l; c->leaf[c->ncell] = (unsigned char) leaf;
  c->ii[c->ncell] = i; c->jj[c->ncell] = j; c->kk[c->ncell] = k;
  c->ncell++;
  return BMG_OK;
}

typedef struct {
  FILE * fp;
  int dim, maxdepth, nvals, err;
  cells_t * cells;
  double * vals;            /* nvals per cell, appended */
  long vcap;
} read_ctx;

static void read_cell (read_ctx * c, int l, int i, int j, int k)
{
  if (c->err) return;
  if (l > c->maxdepth) { c->err = BMG_EINVAL; return; }
  unsigned flags;
  if (fread (&flags, sizeof flags, 1, c->fp) != 1) { c->err = BMG_EINVAL; return; }
  const long at = c->cells->ncell;
  if (push_cell (c->cells, l, i, j, k, (flags & LEAF) != 0)) { c->err = BMG_ENOMEM; return; }
  if ((at + 1)*c->nvals > c->vcap) {
    const long vcap = 2*c->vcap + 1024*c->nvals;
    if (grow ((void **) &c->vals, vcap, sizeof (double))) { c->err = BMG_ENOMEM; return; }
    c->vcap = vcap;
  }
  if (fread (c->vals + at*c->nvals, sizeof (double), c->nvals, c->fp) != (size_t) c->nvals) {
    c->err = BMG_EINVAL;
    return;
  }
  if (flags & LEAF) return;
  const int nc = 1 << c->dim;
  for (int q = 0; q < nc; q++) {
    const int ci = 2*i + ((q >> (c->dim - 1)) & 1);
    const int cj = c->dim > 1 ? 2*j + ((q >> (c->dim - 2)) & 1) : 0;
    const int ck = c->dim > 2 ? 2*k + (q & 1) : 0;
    read_cell (c, l + 1, ci, cj, ck);
  }
}

/* refine () predicate: the cells the dump holds refined, by level and
   index (a sorted key list per level) */
typedef struct {
  bmg_grid * g;
  long * keys[BMG_MAXLEVEL + 1];
  long nkeys[BMG_MAXLEVEL + 1];
} refined_set;

static int cmp_long (const void * a, const void * b)
{
  const long x = *(const long *) a, y = *(const long *) b;
  return x < y ? -1 : x > y;
}

static int refined_cond (int level, double x, double y, double z, void * data)
{
  (void) z;
  refined_set * r = (refined_set *) data;
  if (level > BMG_MAXLEVEL || !r->nkeys[level]) return 0;
  const double Delta = r->g->L0*(1./(1 << level));
  const long i = lround ((x - r->g->X0)/Delta - 0.5), j = lround ((y - r->g->Y0)/Delta - 0.5);
  const long key = (i << 20) | j;
  return bsearch (&key, r->keys[level], r->nkeys[level], sizeof (long), cmp_long) != NULL;
}

int bmg_restore (bmg_grid * g, const char * file, const bmg_scalar * list,
                 const char * const * names, double * t, int * iter)
{
  if (!g || !file || !list || !names) return FAIL (BMG_EINVAL);
  FILE * fp = fopen (file, "rb");
  if (!fp) return FAIL (BMG_EINVAL);
  dump_header hd;
  int r = BMG_OK;
  if (fread (&hd, sizeof hd, 1, fp) != 1 || (hd.version != DUMP_VERSION && hd.version != 161020) ||
      hd.len < 1 || hd.len > 1024 || hd.depth < 0 || hd.depth > g->depth || hd.npe != 1)
    r = BMG_EINVAL;
  /* names of the file -> the caller's fields (-1: skipped); the older
     format 161020 has no names: its columns are the list's fields in order
     (output.h:1265-1273) */
  int match[1024];
  int nlist = 0;
  while (list[nlist].i) nlist++;
  if (!r && hd.version == 161020) {
    if (hd.len - 1 != nlist) r = BMG_EINVAL;
    for (long f = 0; !r && f < hd.len; f++) match[f] = (int) f - 1;
  }
  for (long f = 0; !r && hd.version == DUMP_VERSION && f < hd.len; f++) {
    unsigned len;
    char name[1024];
    if (fread (&len, sizeof len, 1, fp) != 1 || len >= sizeof name ||
        fread (name, 1, len, fp) != len) { r = BMG_EINVAL; break; }
    name[len] = '\0';
    match[f] = -1;
    for (int q = 0; f > 0 && q < nlist; q++)
      if (!strcmp (names[q], name)) match[f] = q;
  }
  double o[4];
  if (!r && fread (o, sizeof (double), 4, fp) != 4) r = BMG_EINVAL;
  cells_t cells;
  memset (&cells, 0, sizeof cells);
  read_ctx c = {fp, g->dim, hd.depth, (int) hd.len, 0, &cells, NULL, 0};
  if (!r) {
    read_cell (&c, 0, 0, 0, 0);
    r = c.err;
  }
  fclose (fp);
  /* geometry (output.h:1325-1326) */
  if (!r) {
    r = bmg_origin (g, o[0], o[1], o[2]);
    if (!r) r = bmg_size (g, o[3]);
  }
  /* a tree grid, or a file holding a tree (a leaf above the deepest level),
     is rebuilt from init_grid (1) by refining the cells the file holds
     refined (output.h:1237-1242, 1357-1358); a uniform grid takes a
     uniform file of its own depth (init_grid (1 << header.depth),
     output.h:1256) */
  int tree = g->tree != NULL;
  for (long q = 0; !r && q < cells.ncell; q++)
    if (cells.leaf[q] && cells.level[q] < hd.depth) tree = 1;
  if (!r && !tree && hd.depth != g->depth) r = BMG_EINVAL;
  if (!r && tree) {
    if (g->dim != 2) r = BMG_EINVAL;
    if (!r) bmg_tree_free (g);
    refined_set rs;
    memset (&rs, 0, sizeof rs);
    rs.g = g;
    for (long q = 0; !r && q < cells.ncell; q++)
      if (!cells.leaf[q]) rs.nkeys[cells.level[q]]++;
    for (int l = 0; !r && l <= hd.depth; l++)
      if (rs.nkeys[l] && !(rs.keys[l] = malloc (rs.nkeys[l]*sizeof (long)))) r = BMG_ENOMEM;
    long at[BMG_MAXLEVEL + 1] = {0};
    for (long q = 0; !r && q < cells.ncell; q++)
      if (!cells.leaf[q]) {
        const int l = cells.level[q];
        rs.keys[l][at[l]++] = ((long) cells.ii[q] << 20) | cells.jj[q];
      }
    for (int l = 0; !r && l <= hd.depth; l++)
      if (rs.nkeys[l]) qsort (rs.keys[l], rs.nkeys[l], sizeof (long), cmp_long);
    if (!r && bmg_tree_refine (g, refined_cond, &rs) < 0) r = BMG_EINVAL;
    for (int l = 0; l <= hd.depth; l++) free (rs.keys[l]);
  }
  /* the values of the matched fields, level by level */
  for (int q = 0; !r && q < nlist; q++) {
    int col = -1;
    for (long f = 1; f < hd.len; f++) if (match[f] == q) col = (int) f;
    if (col < 0) continue;
    for (int l = 0; !r && l <= hd.depth; l++) {
      const size_t n = ncells (g->dim, l);
      double * v = calloc (n, sizeof (double));
      if (!v) { r = BMG_ENOMEM; break; }
      r = bmg_field_get_level (g, list[q], l, v, n, BMG_HOST);
      for (long k = 0; !r && k < cells.ncell; k++)
        if (cells.level[k] == l)
          v[cell_index (g->dim, l, cells.ii[k], cells.jj[k], cells.kk[k])] = c.vals[k*hd.len + col];
      if (!r) r = bmg_field_set_level (g, list[q], l, v, n, BMG_HOST);
      free (v);
    }
  }
  free (cells.level); free (cells.leaf); free (cells.ii); free (cells.jj); free (cells.kk);
  free (c.vals);
  if (!r) {
    if (t) *t = hd.t;
    if (iter) *iter = hd.i;
  }
  return FAIL (r);
}

/*
 * mg_oracle.h -- CPU oracle for the multigrid Poisson--Helmholtz solver.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C99 restatement of the
 * reference's CPU algorithm (Basilisk poisson.h mg_cycle / mg_solve / relax /
 * residual / poisson on grid/multigrid.h levels).  It is the checker for the
 * CUDA path and the timed CPU baseline.  Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg may load it; the product library never
 * links or calls it.
 *
 * The oracle is compiled once per dimension (-DDIM=1, 2 or 3), like the
 * reference, whose dimension is a compile-time constant (grid/multigrid.h,
 * grid/multigrid1D.h, grid/multigrid3D.h).
 *
 * Array conventions at this interface (all finest-level, no ghosts, C order,
 * last index contiguous as in grid/multigrid.h:59-73):
 *   cell field          n^DIM values, index (i, j, k)
 *   face component d    extents n in every dimension but d, which has n+1
 *                       faces; face index f along d is the left/bottom/back
 *                       face of cell f (the reference stores alpha.x[] of
 *                       cell i at its left face, poisson.h:306).
 *   boundary values     per side, n^(DIM-1) values over the tangential
 *                       indices in increasing dimension order.
 */
#ifndef MG_ORACLE_H
#define MG_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* side order of common.h:949 (right, left, top, bottom, front, back) */
enum { OG_RIGHT = 0, OG_LEFT, OG_TOP, OG_BOTTOM, OG_FRONT, OG_BACK };

/* boundary-condition kinds (common.h:957-960, cartesian-common.h:464) */
enum { OG_NEUMANN = 0, OG_DIRICHLET = 1, OG_PERIODIC = 2 };

/* relaxation variants: poisson.h:293-328 (GS = default in-place sweep,
   JACOBI = the -DJACOBI branch) and red-black Gauss-Seidel, an oracle
   extension that pins the GPU smoother of the same name. */
enum { OG_RELAX_GS = 0, OG_RELAX_JACOBI = 1, OG_RELAX_RBGS = 2 };

/* same field order as poisson.h:108-114 */
typedef struct {
  int i;
  double resb, resa;
  double sum;
  int nrelax;
  int minlevel;
} og_mgstats;

enum { OG_A = 0, OG_B, OG_RES, OG_LAMBDA, OG_ALPHA_X, OG_ALPHA_Y, OG_ALPHA_Z, OG_DA,
       OG_UF_X, OG_UF_Y, OG_UF_Z,
       OG_U_X, OG_U_Y, OG_U_Z, OG_MU_X, OG_MU_Y, OG_MU_Z, OG_RHO };

typedef struct og_grid og_grid;

/* poisson.h:102-103 */
extern int og_NITERMAX, og_NITERMIN;
extern double og_TOLERANCE;

int og_dimension (void);
og_grid * og_new (int depth, double L0, double X0, double Y0, double Z0);
void og_free (og_grid * g);
void og_set_periodic (og_grid * g, int dim);
void og_set_bc (og_grid * g, int side, int type, double value, const double * values);
void og_set_relax (og_grid * g, int mode);
void og_set_threads (int n);
int og_get_threads (void);
void og_set_field (og_grid * g, int which, const double * values);
void og_get_field (og_grid * g, int which, double * out);
void og_set_alpha_const (og_grid * g, double v);
void og_set_lambda_const (og_grid * g, double v);
void og_restrict_coefficients (og_grid * g);
double og_residual (og_grid * g);
void og_mg_cycle (og_grid * g, int nrelax, int minlevel, int maxlevel);
og_mgstats og_mg_solve (og_grid * g, double tolerance, int nrelax, int minlevel);
og_mgstats og_poisson (og_grid * g, double tolerance, int nrelax, int minlevel);
/* project (poisson.h:468-509): uf = the OG_UF_* face vector, p = OG_A, alpha
   as set (unityf by default), div in OG_B; dt = 0 / nrelax = 0: defaults */
og_mgstats og_project (og_grid * g, double dt, int nrelax);
/* viscosity (viscosity.h:169-183): implicit viscous step of the cell
   vector OG_U_* with face viscosity OG_MU_* (or a constant) and density
   OG_RHO (or a constant); component c of u has its own box conditions */
void og_set_visc_bc (og_grid * g, int comp, int side, int type, double value);
void og_set_mu_const (og_grid * g, double v);
void og_set_rho_const (og_grid * g, double v);
og_mgstats og_viscosity (og_grid * g, double dt, int nrelax);
double og_residual_viscosity (og_grid * g, double dt);
double og_sum_b (og_grid * g);
/* level access for fine-grained tests: interior values of a level */
void og_get_level (og_grid * g, int which, int level, double * out);
void og_set_level (og_grid * g, int which, int level, const double * values);
void og_relax_level (og_grid * g, int level);
void og_boundary_level (og_grid * g, int which, int level, int homogeneous);
void og_restrict_res (og_grid * g);

#ifdef __cplusplus
}
#endif
#endif

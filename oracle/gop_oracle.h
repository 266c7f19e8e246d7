/*
 * gop_oracle -- CPU restatement of GAMERA-OP's single-domain MHD time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the CUDA path is compared
 * against; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg may load it.  The product library never links it.
 *
 * It restates, in plain C and in the reference's own operation order, the
 * step driver src/solver_solve.c:23-536 and the numerics it calls in
 * src/solver_func.c (PDMU7 215-253, get_dt_normal 255-298,
 * get_derived_variables 308-383, get_AB2_variables 385-492,
 * reconstruct_3dv_* 503-685, center2corner_* 686-778, get_e_fields_*
 * 779-932, get_fluid_flux_rusanov_* 934-1266, get_magnetic_stress_rusanov_*
 * 1268-1529, check_positivity 2117-2135), the geometry and reconstruction
 * weights of src/cartesian/cartesian_general.c:42-367 and
 * src/spherical/spherical_general.c:42-603 (spherical source terms 605-698),
 * the single-domain halo exchange of src/boundary_exchange.c:7-201 with the
 * index sets of src/setup_mpi.c:62-253, and the ghost-fill library of
 * src/boundary_conditions.c.  Background field B0 and gravity are zero in
 * every supported problem and are omitted (adding +0.0 is exact).
 *
 * All arrays use the reference layout: field-major, then i, j, k with k
 * fastest, each axis ghost-extended to n + 2*4 + 1 points.
 */
#ifndef GOP_ORACLE_H
#define GOP_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int ni, nj, nk;        /* active cells per axis (each >= 4) */
  int coord;             /* 0 Cartesian, 2 spherical (COORD_TYPE) */
  const double *x1;      /* face coordinates, ni+9 values (x1[i][0][0]) */
  const double *x2;      /* nj+9 values */
  const double *x3;      /* nk+9 values */
  double gamma, cfl, ca, pdmb, rho_floor, p_floor;
  char bc[6];            /* i-lo,i-hi,j-lo,j-hi,k-lo,k-hi: p s r f e n */
} og_desc;

typedef struct og og_t;

og_t *og_create(const og_desc *d);
void og_destroy(og_t *g);

/* W: 6 primitives (rho v1 v2 v3 p pS), B: 3 face fields (bi bj bk), each
 * NI*NJ*NK doubles.  Wp/Bp may be NULL (fresh start). */
int og_set_state(og_t *g, const double *W, const double *B, const double *Wp,
                 const double *Bp, double time, double dt0);
/* The part of solve() before the time loop (src/solver_solve.c:25-99). */
int og_prepare(og_t *g, int restart);
/* nsteps passes of the time loop (src/solver_solve.c:102-529). */
int og_run(og_t *g, int nsteps);
/* scal[0..4] = time, dt, dt0, divB_max, steps done */
int og_get_state(og_t *g, double *W, double *B, double *Wp, double *Bp,
                 double *scal);
/* Half-step fields of the last step (W_h 6 fields, B_h 3 fields) and the
 * edge electric fields (3 fields), for stage-level checks. */
int og_get_stage(og_t *g, double *Wh, double *Bh, double *E);

#ifdef __cplusplus
}
#endif
#endif

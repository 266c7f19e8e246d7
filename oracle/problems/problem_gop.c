/*
 * Problem hooks for running GAMERA-OP's own solver as the CPU oracle on the
 * workloads this project measures.  Test infrastructure only: compiled
 * together with the reference sources (which are left untouched) behind
 * -DPROBLEM_GOP, in place of the reference's problem_*.c files.
 *
 * It implements the three hooks of src/problem.h:5-12
 * (set_problem_config / problem_init / boundary_conditions) and is driven by
 * environment variables so one binary per coordinate system covers every
 * parity case:
 *
 *   GOP_PROBLEM  ot | blast | loop_cart | loop_sph        (default blast)
 *   GOP_DOMAIN   "x1min,x1max,x2min,x2max,x3min,x3max"
 *   GOP_BC       6 letters for faces i-lo,i-hi,j-lo,j-hi,k-lo,k-hi:
 *                p periodic, s symmetric, r reflective, f fixed,
 *                e extrapolated, n none, o pole (j faces of spherical
 *                grids, src/spherical/spherical_boundary.c)
 *                                                       (default pppppp)
 *   GOP_RING     1: doRingAverage = 1 (the pole ring average)
 *   GOP_CA       Boris "speed of light" CA               (default 10)
 *   blast:  GOP_RHO, GOP_P_IN, GOP_P_OUT, GOP_RADIUS, GOP_CENTER "x,y,z",
 *           GOP_B "b1,b2,b3" (uniform face field), GOP_RHO_IN (density
 *           inside the radius, default GOP_RHO: below the density floor
 *           it drives the positivity floors of check_positivity)
 *   loop_sph: GOP_V "vx,vy,vz" (Cartesian), GOP_RHO, GOP_P, GOP_LOOP
 *           "xc,yc,R,A0"
 *   GOP_PS   f: the entropy channel p_S = f * p in every initialised cell
 *            (default 0: p_S stays 0, as in the reference's own problems)
 *   GOP_B0   uniform | dipole: the background field hooks B10/B20/B30 of
 *            src/common.c (B10_uniform..., B10_dipole...), integrated by the
 *            reference's set_background_field after problem_init (default:
 *            none)
 *
 * The Orszag-Tang and Cartesian field-loop initial states follow the
 * reference problems (src/problem_test_OT_cartesion.c:50-130,
 * src/problem_FieldLoop_cartesian.c:51-84); the blast generalises
 * src/problem_test_Blast_cartesion.c:179-234 to a configurable centre and
 * field; loop_sph is the pole-free spherical-shell field loop.
 */
#ifdef PROBLEM_GOP
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "common.h"
#include "config.h"
#include "curvilinear.h"
#include "log.h"
#include "problem.h"
#include "solver.h"

static double env_d(const char *name, double def) {
  const char *s = getenv(name);
  return s ? atof(s) : def;
}

static int env_vec(const char *name, double *v, int n) {
  const char *s = getenv(name);
  if (!s) return 0;
  char buf[256];
  snprintf(buf, sizeof(buf), "%s", s);
  int k = 0;
  for (char *tok = strtok(buf, ","); tok && k < n; tok = strtok(NULL, ","))
    v[k++] = atof(tok);
  return k == n;
}

static const char *problem_kind(void) {
  const char *s = getenv("GOP_PROBLEM");
  return s ? s : "blast";
}

static char bc_letter(int face) {
  const char *s = getenv("GOP_BC");
  if (!s || (int)strlen(s) < 6) return 'p';
  return s[face];
}

void set_problem_config() {
  double dom[6] = {-0.5, 0.5, -0.5, 0.5, -0.5, 0.5};
  const char *kind = problem_kind();
  if (strcmp(kind, "ot") == 0) {
    double d[6] = {0.0, 1.0, 0.0, 1.0, 0.0, 1.0};
    memcpy(dom, d, sizeof(d));
  } else if (strcmp(kind, "loop_cart") == 0) {
    double d[6] = {-2.0, 2.0, -2.0, 2.0, -2.0, 2.0};
    memcpy(dom, d, sizeof(d));
  } else if (strcmp(kind, "loop_sph") == 0) {
    double d[6] = {1.0, 2.0, 0.25 * PI, 0.75 * PI, -0.25 * PI, 0.25 * PI};
    memcpy(dom, d, sizeof(d));
  }
  env_vec("GOP_DOMAIN", dom, 6);
  x1min_global = dom[0];
  x1max_global = dom[1];
  x2min_global = dom[2];
  x2max_global = dom[3];
  x3min_global = dom[4];
  x3max_global = dom[5];
  CA = env_d("GOP_CA", 10.0);
  doRingAverage = env_d("GOP_RING", 0.0) != 0.0 ? 1 : 0;
  problem_config.Boundary_i =
      (bc_letter(0) == 'p' && bc_letter(1) == 'p') ? BC_PERIODIC
                                                   : BC_NON_PERIODIC;
  problem_config.Boundary_j =
      (bc_letter(2) == 'p' && bc_letter(3) == 'p') ? BC_PERIODIC
                                                   : BC_NON_PERIODIC;
  problem_config.Boundary_k =
      (bc_letter(4) == 'p' && bc_letter(5) == 'p') ? BC_PERIODIC
                                                   : BC_NON_PERIODIC;
}

typedef void (*bc_fn)(void);

/* [face][kind] tables of the reference's BC library (src/common.h:18-87) */
static void apply_face_bc(int face) {
  static bc_fn gas_tab[6][5] = {
      {gas_bc_symmetric_i_low, gas_bc_reflective_i_low, gas_bc_fixed_i_low,
       gas_bc_extrapolated_i_low, gas_bc_none_i_low},
      {gas_bc_symmetric_i_high, gas_bc_reflective_i_high, gas_bc_fixed_i_high,
       gas_bc_extrapolated_i_high, gas_bc_none_i_high},
      {gas_bc_symmetric_j_low, gas_bc_reflective_j_low, gas_bc_fixed_j_low,
       gas_bc_extrapolated_j_low, gas_bc_none_j_low},
      {gas_bc_symmetric_j_high, gas_bc_reflective_j_high, gas_bc_fixed_j_high,
       gas_bc_extrapolated_j_high, gas_bc_none_j_high},
      {gas_bc_symmetric_k_low, gas_bc_reflective_k_low, gas_bc_fixed_k_low,
       gas_bc_extrapolated_k_low, gas_bc_none_k_low},
      {gas_bc_symmetric_k_high, gas_bc_reflective_k_high, gas_bc_fixed_k_high,
       gas_bc_extrapolated_k_high, gas_bc_none_k_high}};
  static bc_fn gem_tab[6][5] = {
      {gem_bc_symmetric_i_low, gem_bc_reflective_i_low, gem_bc_fixed_i_low,
       gem_bc_extrapolated_i_low, gem_bc_none_i_low},
      {gem_bc_symmetric_i_high, gem_bc_reflective_i_high, gem_bc_fixed_i_high,
       gem_bc_extrapolated_i_high, gem_bc_none_i_high},
      {gem_bc_symmetric_j_low, gem_bc_reflective_j_low, gem_bc_fixed_j_low,
       gem_bc_extrapolated_j_low, gem_bc_none_j_low},
      {gem_bc_symmetric_j_high, gem_bc_reflective_j_high, gem_bc_fixed_j_high,
       gem_bc_extrapolated_j_high, gem_bc_none_j_high},
      {gem_bc_symmetric_k_low, gem_bc_reflective_k_low, gem_bc_fixed_k_low,
       gem_bc_extrapolated_k_low, gem_bc_none_k_low},
      {gem_bc_symmetric_k_high, gem_bc_reflective_k_high, gem_bc_fixed_k_high,
       gem_bc_extrapolated_k_high, gem_bc_none_k_high}};
#ifdef GOP_HAVE_POLE_BC
  if (bc_letter(face) == 'o' && (face == 2 || face == 3)) {
    if (face == 2) {
      gas_bc_pole_j_low();
      gem_bc_pole_j_low();
    } else {
      gas_bc_pole_j_high();
      gem_bc_pole_j_high();
    }
    return;
  }
#endif
  int kind;
  switch (bc_letter(face)) {
    case 's': kind = 0; break;
    case 'r': kind = 1; break;
    case 'f': kind = 2; break;
    case 'e': kind = 3; break;
    case 'n': kind = 4; break;
    default: return; /* periodic: handled by the halo exchange */
  }
  gas_tab[face][kind]();
  gem_tab[face][kind]();
}

void boundary_conditions() {
  for (int face = 0; face < 6; face++) apply_face_bc(face);
}

static double ot_az(double x, double y, double z) {
  (void)z;
  return (cos(4.0 * PI * x) / PI / 4.0 + cos(2.0 * PI * y) / PI / 2.0) /
         sqrt(PI * 4.0);
}

static double loopc_az(double x, double y, double z) {
  const double b0 = 1e-3, sigma = 0.2, rad = 0.5;
  const double x0 = -sqrt(2.0) / 2.0, y0 = 0.0, z0 = sqrt(2.0) / 2.0;
  double d = sqrt((x - x0) * (x - x0) + (y - y0) * (y - y0));
  return b0 * exp(-(z - z0) * (z - z0) / sigma / sigma) * fmax(0.0, rad - d);
}

static double g_loop[4] = {1.5, 0.0, 0.15, 1e-3};

static double loops_az_cart(double x, double y) {
  double d = sqrt((x - g_loop[0]) * (x - g_loop[0]) +
                  (y - g_loop[1]) * (y - g_loop[1]));
  return d < g_loop[2] ? g_loop[3] * (g_loop[2] - d) : 0.0;
}

/* spherical components of A = (0, 0, A_z(x, y)) at curvilinear (r,th,ph) */
static void loops_a(double x1, double x2, double x3, double *a) {
  double x, y, z;
  curvilinear_to_cartesian_coord(x1, x2, x3, &x, &y, &z);
  cartesian_to_curvilinear_vector(x, y, z, 0.0, 0.0, loops_az_cart(x, y),
                                  &a[0], &a[1], &a[2]);
}
static double loops_a1(double x1, double x2, double x3) {
  double a[3];
  loops_a(x1, x2, x3, a);
  return a[0];
}
static double loops_a2(double x1, double x2, double x3) {
  double a[3];
  loops_a(x1, x2, x3, a);
  return a[1];
}
static double loops_a3(double x1, double x2, double x3) {
  double a[3];
  loops_a(x1, x2, x3, a);
  return a[2];
}

/* the reference's dipole hooks (src/common.c:30-41; not declared in its
 * headers) */
double B10_dipole(double x, double y, double z);
double B20_dipole(double x, double y, double z);
double B30_dipole(double x, double y, double z);

static void select_background(void) {
  const char *s = getenv("GOP_B0");
  if (!s) return;
  if (strcmp(s, "uniform") == 0) {
    B10 = B10_uniform;
    B20 = B20_uniform;
    B30 = B30_uniform;
  } else if (strcmp(s, "dipole") == 0) {
    B10 = B10_dipole;
    B20 = B20_dipole;
    B30 = B30_dipole;
  }
}

void problem_init() {
  const char *kind = problem_kind();
  log_info("Initializing GOP problem %s", kind);
  select_background();
  Field b_none = Field_Default;
  if (strcmp(kind, "ot") == 0) {
    A3 = ot_az;
    for (int s = 0; s < NS1; s++)
      for (int i = is; i <= ie; i++)
        for (int j = js; j <= je; j++)
          for (int k = ks; k <= ke; k++) {
            gas[s][gas_rho][i][j][k] = 25.0 / (PI * 36.0);
            gas[s][gas_p][i][j][k] = 5.0 / (PI * 12.0);
            gas[s][gas_v1][i][j][k] = -sin(2 * PI * x2c[i][j][k]);
            gas[s][gas_v2][i][j][k] = sin(2 * PI * x1c[i][j][k]);
            gas[s][gas_v3][i][j][k] = 0.0;
          }
    AinitB(gem[mag_bi], gem[mag_bj], gem[mag_bk], A1, A2, A3, b_none, b_none,
           b_none);
  } else if (strcmp(kind, "loop_cart") == 0) {
    A3 = loopc_az;
    for (int s = 0; s < NS1; s++)
      for (int i = is; i <= ie; i++)
        for (int j = js; j <= je; j++)
          for (int k = ks; k <= ke; k++) {
            gas[s][gas_rho][i][j][k] = 1.0;
            gas[s][gas_v1][i][j][k] = 1.0;
            gas[s][gas_v2][i][j][k] = 0.0;
            gas[s][gas_v3][i][j][k] = 0.0;
            gas[s][gas_p][i][j][k] = 0.5;
          }
    AinitB(gem[mag_bi], gem[mag_bj], gem[mag_bk], A1, A2, A3, b_none, b_none,
           b_none);
  } else if (strcmp(kind, "loop_sph") == 0) {
    double vc[3] = {0.0, 1.0, 0.5};
    env_vec("GOP_V", vc, 3);
    env_vec("GOP_LOOP", g_loop, 4);
    double rho = env_d("GOP_RHO", 1.0), p = env_d("GOP_P", 1.0);
    A1 = loops_a1;
    A2 = loops_a2;
    A3 = loops_a3;
    for (int s = 0; s < NS1; s++)
      for (int i = isg; i <= ieg; i++)
        for (int j = jsg; j <= jeg; j++)
          for (int k = ksg; k <= keg; k++) {
            double x, y, z;
            gas[s][gas_rho][i][j][k] = rho;
            curvilinear_to_cartesian_coord(x1ctr[i][j][k], x2ctr[i][j][k],
                                           x3ctr[i][j][k], &x, &y, &z);
            cartesian_to_curvilinear_vector(
                x, y, z, vc[0], vc[1], vc[2], &gas[s][gas_v1][i][j][k],
                &gas[s][gas_v2][i][j][k], &gas[s][gas_v3][i][j][k]);
            gas[s][gas_p][i][j][k] = p;
          }
    AinitB(gem[mag_bi], gem[mag_bj], gem[mag_bk], A1, A2, A3, b_none, b_none,
           b_none);
  } else { /* blast */
    double c[3] = {0.0, 0.0, 0.0};
    double b[3] = {1.0 / sqrt(2), 1.0 / sqrt(2), 0.0};
    env_vec("GOP_CENTER", c, 3);
    env_vec("GOP_B", b, 3);
    double rho = env_d("GOP_RHO", 1.0);
    double p_in = env_d("GOP_P_IN", 10.0), p_out = env_d("GOP_P_OUT", 0.1);
    double rad = env_d("GOP_RADIUS", 0.1);
    double rho_in = env_d("GOP_RHO_IN", rho);
    for (int s = 0; s < NS1; s++)
      for (int i = is; i <= ie; i++)
        for (int j = js; j <= je; j++)
          for (int k = ks; k <= ke; k++) {
            double dx = x1c[i][j][k] - c[0], dy = x2c[i][j][k] - c[1],
                   dz = x3c[i][j][k] - c[2];
            double r = sqrt(dx * dx + dy * dy + dz * dz);
            gas[s][gas_rho][i][j][k] = r < rad ? rho_in : rho;
            gas[s][gas_v1][i][j][k] = 0.0;
            gas[s][gas_v2][i][j][k] = 0.0;
            gas[s][gas_v3][i][j][k] = 0.0;
            gas[s][gas_p][i][j][k] = r < rad ? p_in : p_out;
          }
    for (int i = is; i <= ie + 1; i++)
      for (int j = js; j <= je; j++)
        for (int k = ks; k <= ke; k++) gem[mag_bi][i][j][k] = b[0];
    for (int i = is; i <= ie; i++)
      for (int j = js; j <= je + 1; j++)
        for (int k = ks; k <= ke; k++) gem[mag_bj][i][j][k] = b[1];
    for (int i = is; i <= ie; i++)
      for (int j = js; j <= je; j++)
        for (int k = ks; k <= ke + 1; k++) gem[mag_bk][i][j][k] = b[2];
  }
  double fps = env_d("GOP_PS", 0.0);
  if (fps != 0.0)
    for (int s = 0; s < NS1; s++)
      for (int i = isg; i <= ieg; i++)
        for (int j = jsg; j <= jeg; j++)
          for (int k = ksg; k <= keg; k++)
            gas[s][gas_p_S][i][j][k] = fps * gas[s][gas_p][i][j][k];
}
#endif

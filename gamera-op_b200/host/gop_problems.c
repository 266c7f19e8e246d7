/*
 * Host-side initial conditions for the measured workloads, written against
 * the C ABI's array layout (reference layout: [f][i][j][k], k fastest,
 * ghost-extended by 4 + 1 points per axis).
 *
 * In a drop-in deployment the reference's own problem_*.c hooks build the
 * initial state; these helpers exist so this library can build the same
 * states standalone (bench, tests, serving).  They follow:
 *   - the default uniform grid, src/solver_init.c:297-321;
 *   - face B from a vector potential by 12-point Gauss line integrals and
 *     Stokes' theorem, AinitB / GaussianLineIntegral in
 *     src/solver_func.c:15-125;
 *   - Orszag-Tang, src/problem_test_OT_cartesion.c:50-130;
 *   - blast wave, src/problem_test_Blast_cartesion.c:179-234 (generalised to
 *     any centre and uniform field);
 *   - field loops, src/problem_FieldLoop_cartesian.c:51-84 and a pole-free
 *     spherical-shell loop with the velocity projection of
 *     src/problem_FieldLoop_spherical.c:185-203.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "gamera_op.h"

#define NG 4
#define GOP_PI 3.14159265358979323846

int gop_grid_uniform(int n, double xmin, double xmax, double *x) {
  if (n < NG || !x || !(xmax > xmin)) return GOP_EINVAL;
  for (int i = 0; i <= n + 2 * NG; i++)
    x[i] = xmin - (xmax - xmin) * NG / n + i * (xmax - xmin) / n;
  return GOP_OK;
}

void gop_problem_defaults(int kind, gop_problem *p) {
  memset(p, 0, sizeof(*p));
  p->kind = kind;
  switch (kind) {
    case GOP_PROBLEM_OT:
      break;
    case GOP_PROBLEM_BLAST:
      p->rho = 1.0;
      p->p_in = 10.0;
      p->p_out = 0.1;
      p->radius = 0.1;
      p->b[0] = 1.0 / sqrt(2);
      p->b[1] = 1.0 / sqrt(2);
      break;
    case GOP_PROBLEM_LOOP_CART:
      p->rho = 1.0;
      p->p_out = 0.5;
      p->v[0] = 1.0;
      break;
    case GOP_PROBLEM_LOOP_SPH:
      p->rho = 1.0;
      p->p_out = 1.0;
      p->v[1] = 1.0;
      p->v[2] = 0.5;
      p->loop[0] = 1.5;
      p->loop[1] = 0.0;
      p->loop[2] = 0.15;
      p->loop[3] = 1e-3;
      break;
  }
}

typedef double (*field_fn)(const gop_problem *p, double x1, double x2, double x3);

static double zero_fn(const gop_problem *p, double a, double b, double c) {
  (void)p; (void)a; (void)b; (void)c;
  return 0.0;
}

static double ot_az(const gop_problem *p, double x, double y, double z) {
  (void)p; (void)z;
  return (cos(4 * GOP_PI * x) / GOP_PI / 4 + cos(2 * GOP_PI * y) / GOP_PI / 2) / sqrt(GOP_PI * 4);
}

static double loopc_az(const gop_problem *p, double x, double y, double z) {
  (void)p;
  double b0 = 1e-3, sigma = 0.2, r = 0.5;
  double x0 = -sqrt(2) / 2.0, y0 = 0, z0 = sqrt(2.0) / 2.0;
  return b0 * exp(-(z - z0) * (z - z0) / sigma / sigma) *
         fmax(0, r - sqrt((x - x0) * (x - x0) + (y - y0) * (y - y0)));
}

/* spherical <-> Cartesian (src/spherical/spherical_general.c:745-796) */
static void sph_to_cart(double r, double t, double f, double *x, double *y, double *z) {
  *x = r * sin(t) * cos(f);
  *y = r * sin(t) * sin(f);
  *z = r * cos(t);
}

static void cart_vec_to_sph(double x, double y, double z, double vx, double vy, double vz,
                            double *v1, double *v2, double *v3) {
  double r = sqrt(x * x + y * y + z * z), t = 0.0, f = 0.0;
  if (r != 0.0) {
    t = acos(z / r);
    f = atan2(y, x);
    if (f < 0.0) f += 2.0 * GOP_PI;
  }
  double st = sin(t), ct = cos(t), sf = sin(f), cf = cos(f);
  *v1 = vx * st * cf + vy * st * sf + vz * ct;
  *v2 = vx * ct * cf + vy * ct * sf - vz * st;
  *v3 = -vx * sf + vy * cf;
}

static void loops_a(const gop_problem *p, double x1, double x2, double x3, double a[3]) {
  double x, y, z;
  sph_to_cart(x1, x2, x3, &x, &y, &z);
  double d = sqrt((x - p->loop[0]) * (x - p->loop[0]) + (y - p->loop[1]) * (y - p->loop[1]));
  double az = d < p->loop[2] ? p->loop[3] * (p->loop[2] - d) : 0.0;
  cart_vec_to_sph(x, y, z, 0.0, 0.0, az, &a[0], &a[1], &a[2]);
}
static double loops_a1(const gop_problem *p, double a, double b, double c) {
  double v[3];
  loops_a(p, a, b, c, v);
  return v[0];
}
static double loops_a2(const gop_problem *p, double a, double b, double c) {
  double v[3];
  loops_a(p, a, b, c, v);
  return v[1];
}
static double loops_a3(const gop_problem *p, double a, double b, double c) {
  double v[3];
  loops_a(p, a, b, c, v);
  return v[2];
}

/* mean of f on the segment a -> b by 12-point Gauss-Legendre quadrature
 * (GaussianLineIntegral, src/solver_func.c:97-125: the 10-digit abscissas
 * and weights of the reference) */
static double line_mean(field_fn f, const gop_problem *p, double xa, double ya, double za,
                        double xb, double yb, double zb) {
  static const double node[6] = {0.1252334085, 0.3678314989, 0.5873179542,
                                 0.7699026741, 0.9041172563, 0.9815606342};
  static const double wt[6] = {0.2491470458, 0.2334925365, 0.2031674267,
                               0.1600783285, 0.1069393259, 0.0471753363};
  double hx = (xb - xa) / 2.0, hy = (yb - ya) / 2.0, hz = (zb - za) / 2.0;
  double mx = (xa + xb) / 2.0, my = (ya + yb) / 2.0, mz = (za + zb) / 2.0;
  double s = 0;
  for (int k = 0; k < 6; k++)
    s += wt[k] * (f(p, mx + node[k] * hx, my + node[k] * hy, mz + node[k] * hz) +
                  f(p, mx - node[k] * hx, my - node[k] * hy, mz - node[k] * hz));
  s /= 2.0;
  return s;
}

typedef struct {
  int N[3];
  const double *x[3];
  int sph;
} grid_t;

static size_t at(const grid_t *g, int i, int j, int k) {
  return ((size_t)i * g->N[1] + j) * g->N[2] + k;
}

/* edge lengths and face areas of the reference geometry (cartesian_general.c
 * and spherical_general.c set_geometry_arrays) at one point */
static double edge_len(const grid_t *g, int a, int i, int j, int k) {
  const double *x1 = g->x[0], *x2 = g->x[1], *x3 = g->x[2];
  if (a == 0) return x1[i + 1] - x1[i];
  if (a == 1) return g->sph ? x1[i] * (x2[j + 1] - x2[j]) : x2[j + 1] - x2[j];
  return g->sph ? x1[i] * sin(x2[j]) * (x3[k + 1] - x3[k]) : x3[k + 1] - x3[k];
}

static double face_area(const grid_t *g, int a, int i, int j, int k) {
  const double *x1 = g->x[0], *x2 = g->x[1], *x3 = g->x[2];
  if (!g->sph) {
    double d1 = x1[i + 1] - x1[i], d2 = x2[j + 1] - x2[j], d3 = x3[k + 1] - x3[k];
    return a == 0 ? d2 * d3 : (a == 1 ? d1 * d3 : d1 * d2);
  }
  if (a == 0) return -x1[i] * x1[i] * (cos(x2[j + 1]) - cos(x2[j])) * (x3[k + 1] - x3[k]);
  if (a == 1)
    return 0.5 * (x1[i + 1] * x1[i + 1] - x1[i] * x1[i]) * sin(x2[j]) * (x3[k + 1] - x3[k]);
  return 0.5 * (x1[i + 1] * x1[i + 1] - x1[i] * x1[i]) * (x2[j + 1] - x2[j]);
}

/* AinitB (src/solver_func.c:15-95): line integrals of A along every edge,
 * then the circulation around every face divided by its area */
static int face_b_from_potential(const grid_t *g, const gop_problem *p, field_fn A[3], double *B) {
  size_t n3 = (size_t)g->N[0] * g->N[1] * g->N[2];
  double *LA = (double *)calloc(3 * n3, sizeof(double));
  if (!LA) return GOP_ENOMEM;
  const double *x1 = g->x[0], *x2 = g->x[1], *x3 = g->x[2];
  int gi = g->N[0] - 2, gj = g->N[1] - 2, gk = g->N[2] - 2; /* ieg, jeg, keg */
  for (int i = 0; i <= gi; i++)
    for (int j = 0; j <= gj + 1; j++)
      for (int k = 0; k <= gk + 1; k++)
        LA[at(g, i, j, k)] = edge_len(g, 0, i, j, k) *
                             line_mean(A[0], p, x1[i + 1], x2[j], x3[k], x1[i], x2[j], x3[k]);
  for (int i = 0; i <= gi + 1; i++)
    for (int j = 0; j <= gj; j++)
      for (int k = 0; k <= gk + 1; k++)
        LA[n3 + at(g, i, j, k)] = edge_len(g, 1, i, j, k) *
                                  line_mean(A[1], p, x1[i], x2[j + 1], x3[k], x1[i], x2[j], x3[k]);
  for (int i = 0; i <= gi + 1; i++)
    for (int j = 0; j <= gj + 1; j++)
      for (int k = 0; k <= gk; k++)
        LA[2 * n3 + at(g, i, j, k)] =
            edge_len(g, 2, i, j, k) * line_mean(A[2], p, x1[i], x2[j], x3[k + 1], x1[i], x2[j], x3[k]);
  const double *Li = LA, *Lj = LA + n3, *Lk = LA + 2 * n3;
  size_t si = (size_t)g->N[1] * g->N[2], sj = g->N[2];
  for (int i = 0; i <= gi + 1; i++)
    for (int j = 0; j <= gj; j++)
      for (int k = 0; k <= gk; k++) {
        size_t c = at(g, i, j, k);
        double f = face_area(g, 0, i, j, k);
        B[c] = f < 1e-10 ? 0.0 : (Lj[c] - Lj[c + 1] + Lk[c + sj] - Lk[c]) / f;
      }
  for (int i = 0; i <= gi; i++)
    for (int j = 0; j <= gj + 1; j++)
      for (int k = 0; k <= gk; k++) {
        size_t c = at(g, i, j, k);
        double f = face_area(g, 1, i, j, k);
        B[n3 + c] = f < 1e-10 ? 0.0 : -(Li[c] - Li[c + 1] + Lk[c + si] - Lk[c]) / f;
      }
  for (int i = 0; i <= gi; i++)
    for (int j = 0; j <= gj; j++)
      for (int k = 0; k <= gk + 1; k++) {
        size_t c = at(g, i, j, k);
        double f = face_area(g, 2, i, j, k);
        B[2 * n3 + c] = f < 1e-10 ? 0.0 : (Li[c] - Li[c + sj] + Lj[c + si] - Lj[c]) / f;
      }
  free(LA);
  return GOP_OK;
}

int gop_problem_init(const gop_desc *d, const gop_problem *p, double *gas, double *face_b) {
  if (!d || !p || !gas || !face_b) return GOP_EINVAL;
  grid_t g;
  g.N[0] = d->ni + 2 * NG + 1;
  g.N[1] = d->nj + 2 * NG + 1;
  g.N[2] = d->nk + 2 * NG + 1;
  g.x[0] = d->x1;
  g.x[1] = d->x2;
  g.x[2] = d->x3;
  g.sph = d->coord == GOP_COORD_SPHERICAL;
  size_t n3 = (size_t)g.N[0] * g.N[1] * g.N[2];
  memset(gas, 0, 6 * n3 * sizeof(double));
  memset(face_b, 0, 3 * n3 * sizeof(double));
  double *rho = gas, *v1 = gas + n3, *v2 = gas + 2 * n3, *v3 = gas + 3 * n3, *pr = gas + 4 * n3;
  const double *x1 = d->x1, *x2 = d->x2, *x3 = d->x3;
  int lo = NG, hi[3] = {NG + d->ni - 1, NG + d->nj - 1, NG + d->nk - 1};
  if (p->kind == GOP_PROBLEM_OT) {
    if (g.sph) return GOP_EINVAL;
    for (int i = lo; i <= hi[0]; i++)
      for (int j = lo; j <= hi[1]; j++)
        for (int k = lo; k <= hi[2]; k++) {
          size_t c = at(&g, i, j, k);
          double xc = 0.5 * (x1[i] + x1[i + 1]), yc = 0.5 * (x2[j] + x2[j + 1]);
          rho[c] = 25.0 / (GOP_PI * 36.0);
          pr[c] = 5.0 / (GOP_PI * 12.0);
          v1[c] = -sin(2 * GOP_PI * yc);
          v2[c] = sin(2 * GOP_PI * xc);
          v3[c] = 0.0;
        }
    field_fn A[3] = {zero_fn, zero_fn, ot_az};
    return face_b_from_potential(&g, p, A, face_b);
  }
  if (p->kind == GOP_PROBLEM_LOOP_CART) {
    if (g.sph) return GOP_EINVAL;
    for (int i = lo; i <= hi[0]; i++)
      for (int j = lo; j <= hi[1]; j++)
        for (int k = lo; k <= hi[2]; k++) {
          size_t c = at(&g, i, j, k);
          rho[c] = p->rho;
          v1[c] = p->v[0];
          v2[c] = p->v[1];
          v3[c] = p->v[2];
          pr[c] = p->p_out;
        }
    field_fn A[3] = {zero_fn, zero_fn, loopc_az};
    return face_b_from_potential(&g, p, A, face_b);
  }
  if (p->kind == GOP_PROBLEM_LOOP_SPH) {
    if (!g.sph) return GOP_EINVAL;
    for (int i = 0; i <= g.N[0] - 2; i++)
      for (int j = 0; j <= g.N[1] - 2; j++)
        for (int k = 0; k <= g.N[2] - 2; k++) {
          size_t c = at(&g, i, j, k);
          /* volume centroids x1ctr / x2ctr (spherical_general.c:205-234) */
          double rc = 0.5 * (x1[i] + x1[i + 1]), dr = x1[i + 1] - x1[i];
          double r = rc + 2.0 * rc * dr * dr / (12.0 * rc * rc + dr * dr);
          double t = (sin(x2[j + 1]) - sin(x2[j]) - (x2[j + 1] * cos(x2[j + 1]) - x2[j] * cos(x2[j]))) /
                     (-cos(x2[j + 1]) + cos(x2[j]));
          double f = 0.5 * (x3[k] + x3[k + 1]);
          double x, y, z;
          sph_to_cart(r, t, f, &x, &y, &z);
          rho[c] = p->rho;
          cart_vec_to_sph(x, y, z, p->v[0], p->v[1], p->v[2], &v1[c], &v2[c], &v3[c]);
          pr[c] = p->p_out;
        }
    field_fn A[3] = {loops_a1, loops_a2, loops_a3};
    return face_b_from_potential(&g, p, A, face_b);
  }
  if (p->kind == GOP_PROBLEM_BLAST) {
    if (g.sph) return GOP_EINVAL;
    for (int i = lo; i <= hi[0]; i++)
      for (int j = lo; j <= hi[1]; j++)
        for (int k = lo; k <= hi[2]; k++) {
          size_t c = at(&g, i, j, k);
          double dx = 0.5 * (x1[i] + x1[i + 1]) - p->center[0];
          double dy = 0.5 * (x2[j] + x2[j + 1]) - p->center[1];
          double dz = 0.5 * (x3[k] + x3[k + 1]) - p->center[2];
          double r = sqrt(dx * dx + dy * dy + dz * dz);
          rho[c] = p->rho;
          pr[c] = r < p->radius ? p->p_in : p->p_out;
        }
    double *bi = face_b, *bj = face_b + n3, *bk = face_b + 2 * n3;
    for (int i = lo; i <= hi[0] + 1; i++)
      for (int j = lo; j <= hi[1]; j++)
        for (int k = lo; k <= hi[2]; k++) bi[at(&g, i, j, k)] = p->b[0];
    for (int i = lo; i <= hi[0]; i++)
      for (int j = lo; j <= hi[1] + 1; j++)
        for (int k = lo; k <= hi[2]; k++) bj[at(&g, i, j, k)] = p->b[1];
    for (int i = lo; i <= hi[0]; i++)
      for (int j = lo; j <= hi[1]; j++)
        for (int k = lo; k <= hi[2] + 1; k++) bk[at(&g, i, j, k)] = p->b[2];
    return GOP_OK;
  }
  return GOP_EINVAL;
}

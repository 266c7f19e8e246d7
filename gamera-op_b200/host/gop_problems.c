/*
 * Host-side initial conditions for the measured workloads, written against
 * the C ABI's array layout (reference layout: [f][i][j][k], k fastest,
 * ghost-extended by 4 + 1 points per axis).
 *
 * In a drop-in deployment the reference's own problem_*.c hooks build the
 * initial state; these helpers exist so this library can build the same
 * states standalone (bench, tests, serving).  They follow:
 *   - the default uniform grid, src/solver_init.c:297-321;
 *   - face B from a vector potential (AinitB, src/solver_func.c:15-95), with
 *     the potentials, line integrals and geometry of csrc/gop_fields.h
 *     (shared with the device set-up, csrc/gop_init.cu);
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
#include "../csrc/gop_fields.h"

#define NG 4

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

typedef struct {
  int N[3];
  const double *x[3];
  int sph;
} grid_t;

static size_t at(const grid_t *g, int i, int j, int k) {
  return ((size_t)i * g->N[1] + j) * g->N[2] + k;
}

/* AinitB (src/solver_func.c:15-95): line integrals of A along every edge,
 * then the circulation around every face divided by its area */
static int face_b_from_potential(const grid_t *g, const gop_problem *p, double *B) {
  size_t n3 = (size_t)g->N[0] * g->N[1] * g->N[2];
  double *LA = (double *)calloc(3 * n3, sizeof(double));
  if (!LA) return GOP_ENOMEM;
  const double *x1 = g->x[0], *x2 = g->x[1], *x3 = g->x[2];
  int gi = g->N[0] - 2, gj = g->N[1] - 2, gk = g->N[2] - 2; /* ieg, jeg, keg */
  for (int i = 0; i <= gi; i++)
    for (int j = 0; j <= gj + 1; j++)
      for (int k = 0; k <= gk + 1; k++)
        LA[at(g, i, j, k)] = gop_edge_integral(p, x1, x2, x3, g->sph, 0, i, j, k);
  for (int i = 0; i <= gi + 1; i++)
    for (int j = 0; j <= gj; j++)
      for (int k = 0; k <= gk + 1; k++)
        LA[n3 + at(g, i, j, k)] = gop_edge_integral(p, x1, x2, x3, g->sph, 1, i, j, k);
  for (int i = 0; i <= gi + 1; i++)
    for (int j = 0; j <= gj + 1; j++)
      for (int k = 0; k <= gk; k++)
        LA[2 * n3 + at(g, i, j, k)] = gop_edge_integral(p, x1, x2, x3, g->sph, 2, i, j, k);
  const double *Li = LA, *Lj = LA + n3, *Lk = LA + 2 * n3;
  size_t si = (size_t)g->N[1] * g->N[2], sj = g->N[2];
  for (int i = 0; i <= gi + 1; i++)
    for (int j = 0; j <= gj; j++)
      for (int k = 0; k <= gk; k++) {
        size_t c = at(g, i, j, k);
        double f = gop_face_area(x1, x2, x3, g->sph, 0, i, j, k);
        B[c] = f < 1e-10 ? 0.0 : (Lj[c] - Lj[c + 1] + Lk[c + sj] - Lk[c]) / f;
      }
  for (int i = 0; i <= gi; i++)
    for (int j = 0; j <= gj + 1; j++)
      for (int k = 0; k <= gk; k++) {
        size_t c = at(g, i, j, k);
        double f = gop_face_area(x1, x2, x3, g->sph, 1, i, j, k);
        B[n3 + c] = f < 1e-10 ? 0.0 : -(Li[c] - Li[c + 1] + Lk[c + si] - Lk[c]) / f;
      }
  for (int i = 0; i <= gi; i++)
    for (int j = 0; j <= gj; j++)
      for (int k = 0; k <= gk + 1; k++) {
        size_t c = at(g, i, j, k);
        double f = gop_face_area(x1, x2, x3, g->sph, 2, i, j, k);
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
    return face_b_from_potential(&g, p, face_b);
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
    return face_b_from_potential(&g, p, face_b);
  }
  if (p->kind == GOP_PROBLEM_LOOP_SPH) {
    if (!g.sph) return GOP_EINVAL;
    for (int i = 0; i <= g.N[0] - 2; i++)
      for (int j = 0; j <= g.N[1] - 2; j++)
        for (int k = 0; k <= g.N[2] - 2; k++) {
          size_t c = at(&g, i, j, k);
          double r, t, f, x, y, z;
          gop_sph_centroid(x1, x2, x3, i, j, k, &r, &t, &f);
          gop_sph_to_cart(r, t, f, &x, &y, &z);
          rho[c] = p->rho;
          gop_cart_vec_to_sph(x, y, z, p->v[0], p->v[1], p->v[2], &v1[c], &v2[c], &v3[c]);
          pr[c] = p->p_out;
        }
    return face_b_from_potential(&g, p, face_b);
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

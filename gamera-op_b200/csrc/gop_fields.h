/*
 * Initial-condition fields shared by the host set-up (host/gop_problems.c,
 * compiled as C by gcc) and the device set-up (csrc/gop_init.cu, compiled by
 * nvcc): the same source evaluates the problems' vector potentials, the
 * reference's 12-point Gauss line mean and the edge lengths and face areas
 * of the reference geometry on either side.
 *
 * They follow:
 *   - face B from a vector potential by 12-point Gauss line integrals and
 *     Stokes' theorem, AinitB / GaussianLineIntegral in
 *     src/solver_func.c:15-125;
 *   - Orszag-Tang A_z, src/problem_test_OT_cartesion.c:50-130;
 *   - the Cartesian field loop, src/problem_FieldLoop_cartesian.c:51-84, and a
 *     pole-free spherical-shell loop with the vector projection of
 *     src/spherical/spherical_general.c:745-796.
 */
#ifndef GOP_FIELDS_H
#define GOP_FIELDS_H

#include <math.h>

#include "gamera_op.h"

#ifdef __CUDACC__
#define GOP_HD __host__ __device__ static inline
#else
#define GOP_HD static inline
#endif

#define GOP_PI 3.14159265358979323846

/* A_z of the Orszag-Tang vortex */
GOP_HD double gop_ot_az(double x, double y) {
  return (cos(4 * GOP_PI * x) / GOP_PI / 4 + cos(2 * GOP_PI * y) / GOP_PI / 2) / sqrt(GOP_PI * 4);
}

/* A_z of the Cartesian field loop (a Gaussian-weighted cone) */
GOP_HD double gop_loopc_az(double x, double y, double z) {
  double b0 = 1e-3, sigma = 0.2, r = 0.5;
  double x0 = -sqrt(2.0) / 2.0, y0 = 0, z0 = sqrt(2.0) / 2.0;
  return b0 * exp(-(z - z0) * (z - z0) / sigma / sigma) *
         fmax(0.0, r - sqrt((x - x0) * (x - x0) + (y - y0) * (y - y0)));
}

/* spherical <-> Cartesian (src/spherical/spherical_general.c:745-796) */
GOP_HD void gop_sph_to_cart(double r, double t, double f, double *x, double *y, double *z) {
  *x = r * sin(t) * cos(f);
  *y = r * sin(t) * sin(f);
  *z = r * cos(t);
}

GOP_HD void gop_cart_vec_to_sph(double x, double y, double z, double vx, double vy, double vz,
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

/* the spherical loop's potential: A_z = amp (R - d) for d < R about the axis
 * through (loop[0], loop[1]) along z, projected on (r, theta, phi) */
GOP_HD void gop_loops_a(const gop_problem *p, double x1, double x2, double x3, double a[3]) {
  double x, y, z;
  gop_sph_to_cart(x1, x2, x3, &x, &y, &z);
  double d = sqrt((x - p->loop[0]) * (x - p->loop[0]) + (y - p->loop[1]) * (y - p->loop[1]));
  double az = d < p->loop[2] ? p->loop[3] * (p->loop[2] - d) : 0.0;
  gop_cart_vec_to_sph(x, y, z, 0.0, 0.0, az, &a[0], &a[1], &a[2]);
}

/* component c of problem p's vector potential at (x1, x2, x3) */
GOP_HD double gop_potential(const gop_problem *p, int c, double x1, double x2, double x3) {
  if (p->kind == GOP_PROBLEM_OT) return c == 2 ? gop_ot_az(x1, x2) : 0.0;
  if (p->kind == GOP_PROBLEM_LOOP_CART) return c == 2 ? gop_loopc_az(x1, x2, x3) : 0.0;
  if (p->kind == GOP_PROBLEM_LOOP_SPH) {
    double a[3];
    gop_loops_a(p, x1, x2, x3, a);
    return a[c];
  }
  return 0.0;
}

/* mean of potential component c on the segment a -> b by 12-point
 * Gauss-Legendre quadrature (GaussianLineIntegral, src/solver_func.c:97-125:
 * the 10-digit abscissas and weights of the reference) */
GOP_HD double gop_line_mean(const gop_problem *p, int c, double xa, double ya, double za,
                            double xb, double yb, double zb) {
  const double node[6] = {0.1252334085, 0.3678314989, 0.5873179542,
                          0.7699026741, 0.9041172563, 0.9815606342};
  const double wt[6] = {0.2491470458, 0.2334925365, 0.2031674267,
                        0.1600783285, 0.1069393259, 0.0471753363};
  double hx = (xb - xa) / 2.0, hy = (yb - ya) / 2.0, hz = (zb - za) / 2.0;
  double mx = (xa + xb) / 2.0, my = (ya + yb) / 2.0, mz = (za + zb) / 2.0;
  double s = 0;
  for (int k = 0; k < 6; k++)
    s += wt[k] * (gop_potential(p, c, mx + node[k] * hx, my + node[k] * hy, mz + node[k] * hz) +
                  gop_potential(p, c, mx - node[k] * hx, my - node[k] * hy, mz - node[k] * hz));
  s /= 2.0;
  return s;
}

/* edge length (axis a) and face area (normal a) of the reference geometry
 * (set_geometry_arrays of cartesian_general.c / spherical_general.c) at the
 * point (i, j, k) of the face coordinates x1, x2, x3 */
GOP_HD double gop_edge_len(const double *x1, const double *x2, const double *x3, int sph, int a,
                           int i, int j, int k) {
  if (a == 0) return x1[i + 1] - x1[i];
  if (a == 1) return sph ? x1[i] * (x2[j + 1] - x2[j]) : x2[j + 1] - x2[j];
  return sph ? x1[i] * sin(x2[j]) * (x3[k + 1] - x3[k]) : x3[k + 1] - x3[k];
}

GOP_HD double gop_face_area(const double *x1, const double *x2, const double *x3, int sph, int a,
                            int i, int j, int k) {
  if (!sph) {  /* only the two spacings in the face (a = 0 reaches i = N-1) */
    if (a == 0) return (x2[j + 1] - x2[j]) * (x3[k + 1] - x3[k]);
    if (a == 1) return (x1[i + 1] - x1[i]) * (x3[k + 1] - x3[k]);
    return (x1[i + 1] - x1[i]) * (x2[j + 1] - x2[j]);
  }
  if (a == 0) return -x1[i] * x1[i] * (cos(x2[j + 1]) - cos(x2[j])) * (x3[k + 1] - x3[k]);
  if (a == 1)
    return 0.5 * (x1[i + 1] * x1[i + 1] - x1[i] * x1[i]) * sin(x2[j]) * (x3[k + 1] - x3[k]);
  return 0.5 * (x1[i + 1] * x1[i + 1] - x1[i] * x1[i]) * (x2[j + 1] - x2[j]);
}

/* line integral of potential component a along the edge from point
 * (i, j, k) in direction a (AinitB's LA arrays) */
GOP_HD double gop_edge_integral(const gop_problem *p, const double *x1, const double *x2,
                                const double *x3, int sph, int a, int i, int j, int k) {
  double m;
  if (a == 0) m = gop_line_mean(p, 0, x1[i + 1], x2[j], x3[k], x1[i], x2[j], x3[k]);
  else if (a == 1) m = gop_line_mean(p, 1, x1[i], x2[j + 1], x3[k], x1[i], x2[j], x3[k]);
  else m = gop_line_mean(p, 2, x1[i], x2[j], x3[k + 1], x1[i], x2[j], x3[k]);
  return gop_edge_len(x1, x2, x3, sph, a, i, j, k) * m;
}

/* volume centroid (x1ctr, x2ctr) of spherical cell (i, j)
 * (spherical_general.c:205-234) and the cell-centre phi */
GOP_HD void gop_sph_centroid(const double *x1, const double *x2, const double *x3, int i, int j,
                             int k, double *r, double *t, double *f) {
  double rc = 0.5 * (x1[i] + x1[i + 1]), dr = x1[i + 1] - x1[i];
  *r = rc + 2.0 * rc * dr * dr / (12.0 * rc * rc + dr * dr);
  *t = (sin(x2[j + 1]) - sin(x2[j]) - (x2[j + 1] * cos(x2[j + 1]) - x2[j] * cos(x2[j]))) /
       (-cos(x2[j + 1]) + cos(x2[j]));
  *f = 0.5 * (x3[k] + x3[k + 1]);
}

#endif /* GOP_FIELDS_H */

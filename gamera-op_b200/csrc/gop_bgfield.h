/*
 * Background magnetic field B0 routines shared by the host set-up
 * (host/gop_background.c, compiled as C by gcc) and the device set-up
 * (csrc/gop_bgdev.cu, compiled by nvcc): set_background_field
 * (src/solver_func.c:1851-2077) with g2int_ortho (src/solver_func.c:
 * 1623-1800) and GaussianLineIntegral (src/solver_func.c:97-125) for the
 * built-in backgrounds (uniform, the reference's unit dipole), in the
 * reference's evaluation order, so the host arrays equal the reference's bit
 * for bit and the device's differ only by the last bits of its pow, sin and
 * cos.
 */
#ifndef GOP_BGFIELD_H
#define GOP_BGFIELD_H

#include "gop_fields.h"

/* the background field, component c (B10/B20/B30 of src/common.c) */
GOP_HD double gop_b0_fn(const gop_background *bg, int c, double x, double y, double z) {
  if (bg->kind == GOP_BG_UNIFORM) return bg->b[c];
  double r_squared = x * x + y * y + z * z;
  double v;
  if (c == 0) v = (3 * x * z) / pow(r_squared, 2.5);
  else if (c == 1) v = (3 * y * z) / pow(r_squared, 2.5);
  else v = (2 * z * z - x * x - y * y) / pow(r_squared, 2.5);
  return bg->moment * v;
}

/* metric scale factors H1..H3 (src/cartesian/cartesian_general.c:30-40,
 * src/spherical/spherical_general.c:30-40) */
GOP_HD double gop_h_fn(int sph, int c, double x1, double x2) {
  if (!sph || c == 0) return 1.0;
  return c == 1 ? x1 : x1 * sin(x2);
}

/* the reference's 10-digit 12-point Gauss-Legendre abscissas and weights */
#define GOP_GAUSS12                                                                         \
  const double kA[12] = {0.1252334085,  0.3678314989,  0.5873179542,  0.7699026741,          \
                         0.9041172563,  0.9815606342,  -0.1252334085, -0.3678314989,         \
                         -0.5873179542, -0.7699026741, -0.9041172563, -0.9815606342};        \
  const double kW[12] = {0.2491470458, 0.2334925365, 0.2031674267, 0.1600783285,            \
                         0.1069393259, 0.0471753363, 0.2491470458, 0.2334925365,            \
                         0.2031674267, 0.1600783285, 0.1069393259, 0.0471753363}

/* mean of component c from point a to point b (GaussianLineIntegral) */
GOP_HD double gop_b0_line_mean(const gop_background *bg, int c, double xa, double ya, double za,
                               double xb, double yb, double zb) {
  GOP_GAUSS12;
  double hx = (xb - xa) / 2.0, hy = (yb - ya) / 2.0, hz = (zb - za) / 2.0;
  double mx = (xa + xb) / 2.0, my = (ya + yb) / 2.0, mz = (za + zb) / 2.0;
  double s = 0;
  for (int k = 0; k < 6; k++)
    s += kW[k] * (gop_b0_fn(bg, c, mx + kA[k] * hx, my + kA[k] * hy, mz + kA[k] * hz) +
                  gop_b0_fn(bg, c, mx - kA[k] * hx, my - kA[k] * hy, mz - kA[k] * hz));
  s /= 2.0;
  return s;
}

/* g2int_ortho: averages over the face with corners c[0..3] (coordinates
 * c[a][corner]) of b1..b3, |B|^2 and b_d * b1..b3 (d the face normal);
 * out = f1 f2 f3 fsq fn1 fn2 fn3 */
GOP_HD void gop_b0_face_average(const gop_background *bg, int sph, int dir, double area,
                                double c[3][4], double out[7]) {
  GOP_GAUSS12;
  double s1 = 0, s2 = 0, s3 = 0, ssq = 0, sn1 = 0, sn2 = 0, sn3 = 0;
  if (fabs(area) >= 1e-10) {
    for (int i = 0; i < 12; i++) {
      for (int j = 0; j < 12; j++) {
        double eta = 0.5 * (1.0 + kA[i]), psi = 0.5 * (1.0 + kA[j]), wt2 = kW[i] * kW[j];
        double x1 = c[0][0] + psi * (c[0][2] - c[0][0]) + eta * (c[0][1] - c[0][0]);
        double x2 = c[1][0] + psi * (c[1][2] - c[1][0]) + eta * (c[1][1] - c[1][0]);
        double x3 = c[2][0] + psi * (c[2][2] - c[2][0]) + eta * (c[2][1] - c[2][0]);
        double dx[3];
        for (int a = 0; a < 3; a++)
          dx[a] = fmax(fmax(fabs(c[a][1] - c[a][0]), fabs(c[a][2] - c[a][0])), fabs(c[a][3] - c[a][0]));
        double b1 = gop_b0_fn(bg, 0, x1, x2, x3), b2 = gop_b0_fn(bg, 1, x1, x2, x3),
               b3 = gop_b0_fn(bg, 2, x1, x2, x3);
        double h1 = gop_h_fn(sph, 0, x1, x2), h2 = gop_h_fn(sph, 1, x1, x2),
               h3 = gop_h_fn(sph, 2, x1, x2);
        double bn = dir == 0 ? b1 : (dir == 1 ? b2 : b3);
        double bsq = b1 * b1 + b2 * b2 + b3 * b3;
        double bn1 = bn * b1, bn2 = bn * b2, bn3 = bn * b3;
        /* the two spacings and scale factors in the face, in the
         * reference's product order */
        double da, db, ha, hb;
        if (dir == 0) { da = dx[1]; db = dx[2]; ha = h2; hb = h3; }
        else if (dir == 1) { da = dx[0]; db = dx[2]; ha = h1; hb = h3; }
        else { da = dx[0]; db = dx[1]; ha = h1; hb = h2; }
        s1 += 0.25 * da * db * wt2 * b1 * ha * hb;
        s2 += 0.25 * da * db * wt2 * b2 * ha * hb;
        s3 += 0.25 * da * db * wt2 * b3 * ha * hb;
        ssq += 0.25 * da * db * wt2 * bsq * ha * hb;
        sn1 += 0.25 * da * db * wt2 * bn1 * ha * hb;
        sn2 += 0.25 * da * db * wt2 * bn2 * ha * hb;
        sn3 += 0.25 * da * db * wt2 * bn3 * ha * hb;
      }
    }
    out[0] = s1 / area;
    out[1] = s2 / area;
    out[2] = s3 / area;
    out[3] = ssq / area;
    out[4] = sn1 / area;
    out[5] = sn2 / area;
    out[6] = sn3 / area;
    return;
  }
  /* a degenerate face: the mean along its diagonal */
  double f[3];
  for (int a = 0; a < 3; a++)
    f[a] = gop_b0_line_mean(bg, a, c[0][0], c[1][0], c[2][0], c[0][3], c[1][3], c[2][3]);
  out[0] = f[0];
  out[1] = f[1];
  out[2] = f[2];
  out[3] = f[0] * f[0] + f[1] * f[1] + f[2] * f[2];
  out[4] = f[dir] * f[0];
  out[5] = f[dir] * f[1];
  out[6] = f[dir] * f[2];
}

/* the corners of face (i, j, k) normal to dir, in the reference's order */
GOP_HD void gop_b0_face_corners(const double *x1, const double *x2, const double *x3, int dir,
                                int i, int j, int k, double c[3][4]) {
  int o[4][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  if (dir == 0) { o[1][1] = 1; o[2][2] = 1; o[3][1] = 1; o[3][2] = 1; }
  else if (dir == 1) { o[1][2] = 1; o[2][0] = 1; o[3][2] = 1; o[3][0] = 1; }
  else { o[1][0] = 1; o[2][1] = 1; o[3][0] = 1; o[3][1] = 1; }
  for (int q = 0; q < 4; q++) {
    c[0][q] = x1[i + o[q][0]];
    c[1][q] = x2[j + o[q][1]];
    c[2][q] = x3[k + o[q][2]];
  }
}

GOP_HD double gop_cell_volume(const double *x1, const double *x2, const double *x3, int sph, int i,
                              int j, int k) {
  if (!sph) return (x1[i + 1] - x1[i]) * (x2[j + 1] - x2[j]) * (x3[k + 1] - x3[k]);
  return fabs(1.0 / 3.0 * (pow(x1[i + 1], 3) - pow(x1[i], 3)) * (cos(x2[j + 1]) - cos(x2[j])) *
              (x3[k + 1] - x3[k]));
}

/* the Lorentz force of B0, component c, of cell (i, j, k) from the face
 * averages of |B0|^2 (bsq[dir]) and b_dir * b_c (bn[dir][c]) of its six
 * faces (lo: the cell's lower face of each axis, hi: its upper face) */
GOP_HD double gop_b0_lorentz(int c, const double bsq_lo[3], const double bsq_hi[3],
                             const double bn_lo[3], const double bn_hi[3], const double a_lo[3],
                             const double a_hi[3], double vol) {
  double s1[3], s0[3];
  for (int dir = 0; dir < 3; dir++) {
    s1[dir] = (dir == c ? 0.5 * bsq_hi[dir] : 0.0) - bn_hi[dir];
    s0[dir] = (dir == c ? 0.5 * bsq_lo[dir] : 0.0) - bn_lo[dir];
    if (dir != c) {  /* the reference's -bn (no 0.0 - bn) */
      s1[dir] = -bn_hi[dir];
      s0[dir] = -bn_lo[dir];
    }
  }
  return (s1[0] * a_hi[0] - s0[0] * a_lo[0] + s1[1] * a_hi[1] - s0[1] * a_lo[1] +
          s1[2] * a_hi[2] - s0[2] * a_lo[2]) /
             vol -
         0.0;
}

#endif /* GOP_BGFIELD_H */

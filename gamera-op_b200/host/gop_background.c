/*
 * Host-side set-up of a background magnetic field B0 for the built-in
 * backgrounds (uniform, the reference's unit dipole), following
 * set_background_field (src/solver_func.c:1851-2077) with its helpers
 * g2int_ortho (src/solver_func.c:1623-1800) and GaussianLineIntegral
 * (src/solver_func.c:97-125): B0 at the cell centroids, B0 averaged over
 * every face by 12x12-point Gauss quadrature with the metric scale factors
 * H1..H3 of the coordinate system (src/cartesian/cartesian_general.c:30-40,
 * src/spherical/spherical_general.c:30-40), averaged along every active edge
 * by 12-point Gauss quadrature, and the Lorentz force of B0 from the face
 * stresses.  No reference problem has a volume source for B0
 * (Source1_B0..3 are the zero default), so its volume quadrature adds zero
 * and is not evaluated.  The evaluation order is the reference's, so with
 * the same compiler flags the arrays agree with the reference's bit for bit.
 *
 * Arrays use the layout of gop_upload ([field][i][j][k], k fastest,
 * n + 9 points per axis).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "gamera_op.h"
#include "../csrc/gop_fields.h"

#define NG 4

typedef struct {
  int N[3];
  const double *x[3];
  int sph;
  const gop_background *bg;
} bgrid_t;

static size_t at3(const bgrid_t *g, int i, int j, int k) {
  return ((size_t)i * g->N[1] + j) * g->N[2] + k;
}

/* the background field, component c (B10/B20/B30) */
static double b0_fn(const gop_background *bg, int c, double x, double y, double z) {
  if (bg->kind == GOP_BG_UNIFORM) return bg->b[c];
  double r_squared = x * x + y * y + z * z;
  double v;
  if (c == 0) v = (3 * x * z) / pow(r_squared, 2.5);
  else if (c == 1) v = (3 * y * z) / pow(r_squared, 2.5);
  else v = (2 * z * z - x * x - y * y) / pow(r_squared, 2.5);
  return bg->moment * v;
}

/* metric scale factors H1..H3 */
static double h_fn(int sph, int c, double x1, double x2) {
  if (!sph || c == 0) return 1.0;
  return c == 1 ? x1 : x1 * sin(x2);
}

static const double kA[12] = {0.1252334085,  0.3678314989,  0.5873179542,  0.7699026741,
                              0.9041172563,  0.9815606342,  -0.1252334085, -0.3678314989,
                              -0.5873179542, -0.7699026741, -0.9041172563, -0.9815606342};
static const double kW[12] = {0.2491470458, 0.2334925365, 0.2031674267, 0.1600783285,
                              0.1069393259, 0.0471753363, 0.2491470458, 0.2334925365,
                              0.2031674267, 0.1600783285, 0.1069393259, 0.0471753363};

/* mean of component c from point a to point b (GaussianLineIntegral) */
static double line_mean_b0(const gop_background *bg, int c, double xa, double ya, double za,
                           double xb, double yb, double zb) {
  double hx = (xb - xa) / 2.0, hy = (yb - ya) / 2.0, hz = (zb - za) / 2.0;
  double mx = (xa + xb) / 2.0, my = (ya + yb) / 2.0, mz = (za + zb) / 2.0;
  double s = 0;
  for (int k = 0; k < 6; k++)
    s += kW[k] * (b0_fn(bg, c, mx + kA[k] * hx, my + kA[k] * hy, mz + kA[k] * hz) +
                  b0_fn(bg, c, mx - kA[k] * hx, my - kA[k] * hy, mz - kA[k] * hz));
  s /= 2.0;
  return s;
}

/* g2int_ortho: averages over the face with corners c[0..3] (coordinates
 * c[a][corner]) of b1..b3, |B|^2 and b_d * b1..b3 (d the face normal);
 * out = f1 f2 f3 fsq fn1 fn2 fn3 */
static void face_average(const bgrid_t *g, int dir, double area, double c[3][4], double out[7]) {
  const gop_background *bg = g->bg;
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
        double b1 = b0_fn(bg, 0, x1, x2, x3), b2 = b0_fn(bg, 1, x1, x2, x3),
               b3 = b0_fn(bg, 2, x1, x2, x3);
        double h1 = h_fn(g->sph, 0, x1, x2), h2 = h_fn(g->sph, 1, x1, x2),
               h3 = h_fn(g->sph, 2, x1, x2);
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
    f[a] = line_mean_b0(bg, a, c[0][0], c[1][0], c[2][0], c[0][3], c[1][3], c[2][3]);
  out[0] = f[0];
  out[1] = f[1];
  out[2] = f[2];
  out[3] = f[0] * f[0] + f[1] * f[1] + f[2] * f[2];
  out[4] = f[dir] * f[0];
  out[5] = f[dir] * f[1];
  out[6] = f[dir] * f[2];
}

static double cell_volume(const bgrid_t *g, int i, int j, int k) {
  const double *x1 = g->x[0], *x2 = g->x[1], *x3 = g->x[2];
  if (!g->sph) return (x1[i + 1] - x1[i]) * (x2[j + 1] - x2[j]) * (x3[k + 1] - x3[k]);
  return fabs(1.0 / 3.0 * (pow(x1[i + 1], 3) - pow(x1[i], 3)) * (cos(x2[j + 1]) - cos(x2[j])) *
              (x3[k + 1] - x3[k]));
}

int gop_background_init(const gop_desc *d, const gop_background *bg, double *b0, double *lorentz,
                        double *b0_face, double *b0_edge) {
  if (!d || !bg || !b0 || !lorentz || !b0_face || !b0_edge) return GOP_EINVAL;
  if (bg->kind != GOP_BG_UNIFORM && bg->kind != GOP_BG_DIPOLE) return GOP_EINVAL;
  bgrid_t g;
  g.N[0] = d->ni + 2 * NG + 1;
  g.N[1] = d->nj + 2 * NG + 1;
  g.N[2] = d->nk + 2 * NG + 1;
  g.x[0] = d->x1;
  g.x[1] = d->x2;
  g.x[2] = d->x3;
  g.sph = d->coord == GOP_COORD_SPHERICAL;
  g.bg = bg;
  const size_t n3 = (size_t)g.N[0] * g.N[1] * g.N[2];
  memset(b0, 0, 3 * n3 * sizeof(double));
  memset(lorentz, 0, 3 * n3 * sizeof(double));
  memset(b0_face, 0, 9 * n3 * sizeof(double));
  memset(b0_edge, 0, 9 * n3 * sizeof(double));
  /* |B0|^2 and b_d * b1..3 on the faces of each axis, for the Lorentz force */
  double *aux = (double *)calloc(12 * n3, sizeof(double));
  if (!aux) return GOP_ENOMEM;
  const double *x1 = g.x[0], *x2 = g.x[1], *x3 = g.x[2];
  const int ieg = g.N[0] - 2, jeg = g.N[1] - 2, keg = g.N[2] - 2;

  /* B0 at the cell centroids (x1ctr, x2ctr, x3ctr) */
  for (int i = 0; i <= ieg; i++)
    for (int j = 0; j <= jeg; j++)
      for (int k = 0; k <= keg; k++) {
        double r, t, f;
        if (g.sph) {
          gop_sph_centroid(x1, x2, x3, i, j, k, &r, &t, &f);
        } else {
          r = 0.5 * (x1[i] + x1[i + 1]);
          t = 0.5 * (x2[j] + x2[j + 1]);
          f = 0.5 * (x3[k] + x3[k + 1]);
        }
        for (int c = 0; c < 3; c++) b0[c * n3 + at3(&g, i, j, k)] = b0_fn(bg, c, r, t, f);
      }

  /* face averages: faces normal to axis d, corners in the reference's order */
  for (int dir = 0; dir < 3; dir++) {
    const int ni = dir == 0 ? ieg + 1 : ieg, nj = dir == 1 ? jeg + 1 : jeg,
              nk = dir == 2 ? keg + 1 : keg;
    for (int i = 0; i <= ni; i++)
      for (int j = 0; j <= nj; j++)
        for (int k = 0; k <= nk; k++) {
          /* corner offsets (di, dj, dk) of corners 1..3 */
          int o[4][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
          if (dir == 0) { o[1][1] = 1; o[2][2] = 1; o[3][1] = 1; o[3][2] = 1; }
          else if (dir == 1) { o[1][2] = 1; o[2][0] = 1; o[3][2] = 1; o[3][0] = 1; }
          else { o[1][0] = 1; o[2][1] = 1; o[3][0] = 1; o[3][1] = 1; }
          double c[3][4];
          for (int q = 0; q < 4; q++) {
            c[0][q] = x1[i + o[q][0]];
            c[1][q] = x2[j + o[q][1]];
            c[2][q] = x3[k + o[q][2]];
          }
          double out[7];
          face_average(&g, dir, gop_face_area(x1, x2, x3, g.sph, dir, i, j, k), c, out);
          const size_t p = at3(&g, i, j, k);
          for (int q = 0; q < 3; q++) b0_face[(3 * dir + q) * n3 + p] = out[q];
          for (int q = 0; q < 4; q++) aux[(4 * dir + q) * n3 + p] = out[3 + q];
        }
  }

  /* edge averages over the active range */
  const int is = NG, js = NG, ks = NG;
  const int ie = NG + d->ni - 1, je = NG + d->nj - 1, ke = NG + d->nk - 1;
  for (int dir = 0; dir < 3; dir++) {
    const int ni = dir == 0 ? ie : ie + 1, nj = dir == 1 ? je : je + 1, nk = dir == 2 ? ke : ke + 1;
    for (int i = is; i <= ni; i++)
      for (int j = js; j <= nj; j++)
        for (int k = ks; k <= nk; k++) {
          const int i1 = i + (dir == 0), j1 = j + (dir == 1), k1 = k + (dir == 2);
          for (int c = 0; c < 3; c++)
            b0_edge[(3 * dir + c) * n3 + at3(&g, i, j, k)] =
                line_mean_b0(bg, c, x1[i1], x2[j1], x3[k1], x1[i], x2[j], x3[k]);
        }
  }

  /* Lorentz force of B0 from the face stresses (dmagsf_G) */
  const double *bsq[3], *bn[3][3];
  for (int dir = 0; dir < 3; dir++) {
    bsq[dir] = aux + (4 * dir) * n3;
    for (int q = 0; q < 3; q++) bn[dir][q] = aux + (4 * dir + 1 + q) * n3;
  }
  const size_t si = (size_t)g.N[1] * g.N[2], sj = g.N[2];
  for (int i = 0; i <= ieg; i++)
    for (int j = 0; j <= jeg; j++)
      for (int k = 0; k <= keg; k++) {
        const size_t p = at3(&g, i, j, k);
        const double ai0 = gop_face_area(x1, x2, x3, g.sph, 0, i, j, k),
                     ai1 = gop_face_area(x1, x2, x3, g.sph, 0, i + 1, j, k),
                     aj0 = gop_face_area(x1, x2, x3, g.sph, 1, i, j, k),
                     aj1 = gop_face_area(x1, x2, x3, g.sph, 1, i, j + 1, k),
                     ak0 = gop_face_area(x1, x2, x3, g.sph, 2, i, j, k),
                     ak1 = gop_face_area(x1, x2, x3, g.sph, 2, i, j, k + 1);
        const double vol = cell_volume(&g, i, j, k);
        for (int c = 0; c < 3; c++) {
          /* stress of the faces normal to each axis, component c */
          double s1[3], s0[3];
          const size_t up[3] = {p + si, p + sj, p + 1};
          for (int dir = 0; dir < 3; dir++) {
            s1[dir] = (dir == c ? 0.5 * bsq[dir][up[dir]] : 0.0) - bn[dir][c][up[dir]];
            s0[dir] = (dir == c ? 0.5 * bsq[dir][p] : 0.0) - bn[dir][c][p];
            if (dir != c) {  /* the reference's -bn (no 0.0 - bn) */
              s1[dir] = -bn[dir][c][up[dir]];
              s0[dir] = -bn[dir][c][p];
            }
          }
          lorentz[c * n3 + p] = (s1[0] * ai1 - s0[0] * ai0 + s1[1] * aj1 - s0[1] * aj0 +
                                 s1[2] * ak1 - s0[2] * ak0) /
                                    vol -
                                0.0;
        }
      }
  free(aux);
  return GOP_OK;
}

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
#include "../csrc/gop_bgfield.h"

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
        for (int c = 0; c < 3; c++) b0[c * n3 + at3(&g, i, j, k)] = gop_b0_fn(bg, c, r, t, f);
      }

  /* face averages: faces normal to axis d, corners in the reference's order */
  for (int dir = 0; dir < 3; dir++) {
    const int ni = dir == 0 ? ieg + 1 : ieg, nj = dir == 1 ? jeg + 1 : jeg,
              nk = dir == 2 ? keg + 1 : keg;
    for (int i = 0; i <= ni; i++)
      for (int j = 0; j <= nj; j++)
        for (int k = 0; k <= nk; k++) {
          double c[3][4];
          gop_b0_face_corners(x1, x2, x3, dir, i, j, k, c);
          double out[7];
          gop_b0_face_average(bg, g.sph, dir, gop_face_area(x1, x2, x3, g.sph, dir, i, j, k), c, out);
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
                gop_b0_line_mean(bg, c, x1[i1], x2[j1], x3[k1], x1[i], x2[j], x3[k]);
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
        const double vol = gop_cell_volume(x1, x2, x3, g.sph, i, j, k);
        const double a_lo[3] = {ai0, aj0, ak0}, a_hi[3] = {ai1, aj1, ak1};
        const size_t up[3] = {p + si, p + sj, p + 1};
        for (int c = 0; c < 3; c++) {
          double q_lo[3], q_hi[3], n_lo[3], n_hi[3];
          for (int dir = 0; dir < 3; dir++) {
            q_lo[dir] = bsq[dir][p];
            q_hi[dir] = bsq[dir][up[dir]];
            n_lo[dir] = bn[dir][c][p];
            n_hi[dir] = bn[dir][c][up[dir]];
          }
          lorentz[c * n3 + p] = gop_b0_lorentz(c, q_lo, q_hi, n_lo, n_hi, a_lo, a_hi, vol);
        }
      }
  free(aux);
  return GOP_OK;
}

/*
 * gop_oracle.c -- CPU restatement of GAMERA-OP's single-domain MHD step.
 *
 * TEST INFRASTRUCTURE ONLY (the checker; see gop_oracle.h).  Every routine
 * names the reference file:line it restates.  Arithmetic is written in the
 * reference's evaluation order so that, built with the reference's strict
 * flags (-O2 -fno-fast-math -ffp-contract=off), results agree with the
 * reference binary to the last bit on the supported problems.
 */
#include "gop_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NG 4
#define GOP_PI 3.14159265358979323846

enum { RHO = 0, V1, V2, V3, PR, PS, NPRIM };

struct og {
  og_desc d;
  double gamma, cfl, ca, pdmb, rho_floor, p_floor;
  int n[3], N[3];
  size_t n3;
  long st[3];
  int lo[3], hi[3];   /* active range, inclusive */
  int gmax[3];        /* last ghost cell index n + 2*NG - 1 */
  int periodic[3];
  double *xs[3];      /* 1-D face coordinates */
  /* geometry, 3-D like the reference's geo[] / dx* / x*c / x*ctr arrays */
  double *dx[3], *xc[3], *xctr[3], *edge[3], *dl[3], *face[3], *vol;
  double *gff[3], *gfv[3], *volf[3];
  double *w[3][2][7]; /* rec[]: [dir][0 left,1 right][tap] */
  /* state and per-step work arrays */
  double *W[6], *Wh[6], *Wp[6];
  double *B[3], *Bh[3], *Bp[3];
  double *ms[3], *msh[3], *msp[3], *mt[3];
  double *U[6], *U0[6], *dU[6], *F[6];
  double *v0[3];
  double *L[6], *R[6], *mL[3], *mR[3];
  double *MF[3], *dMF[3], *SH[3], *SB[3];
  double *E[3];
  double *vil[3], *vir[3], *vin[3], *vav[3];
  double *bl[3], *br[3];
  double time, dt, dt0, divb;
  long steps;
  double *pool;
  size_t pool_used, pool_cap;
};

#define IX(g, i, j, k) (((size_t)(i) * (g)->N[1] + (size_t)(j)) * (g)->N[2] + (size_t)(k))
#define A3(a, i, j, k) (a)[IX(g, i, j, k)]
#define LOOP3(i, i0, i1, j, j0, j1, k, k0, k1)  \
  for (int i = (i0); i <= (i1); i++)            \
    for (int j = (j0); j <= (j1); j++)          \
      for (int k = (k0); k <= (k1); k++)

static double *take(og_t *g) {
  double *p = g->pool + g->pool_used * g->n3;
  g->pool_used++;
  return p;
}

/* ---------------------------------------------------------------- geometry */

/* Cartesian geometry, src/cartesian/cartesian_general.c:42-283 */
static void geometry_cartesian(og_t *g) {
  int NI = g->N[0], NJ = g->N[1], NK = g->N[2];
  const double *x1 = g->xs[0], *x2 = g->xs[1], *x3 = g->xs[2];
  LOOP3(i, 0, NI - 1, j, 0, NJ - 1, k, 0, NK - 1) {
    size_t c = IX(g, i, j, k);
    if (i < NI - 1) {
      g->dx[0][c] = x1[i + 1] - x1[i];
      g->xc[0][c] = 0.5 * (x1[i] + x1[i + 1]);
    }
    if (j < NJ - 1) {
      g->dx[1][c] = x2[j + 1] - x2[j];
      g->xc[1][c] = 0.5 * (x2[j] + x2[j + 1]);
    }
    if (k < NK - 1) {
      g->dx[2][c] = x3[k + 1] - x3[k];
      g->xc[2][c] = 0.5 * (x3[k] + x3[k + 1]);
    }
  }
  LOOP3(i, 0, NI - 1, j, 0, NJ - 1, k, 0, NK - 1) {
    size_t c = IX(g, i, j, k);
    for (int d = 0; d < 3; d++) {
      g->edge[d][c] = g->dx[d][c];
      g->dl[d][c] = g->dx[d][c];
      g->xctr[d][c] = g->xc[d][c];
    }
    g->face[0][c] = g->dx[1][c] * g->dx[2][c];
    g->face[1][c] = g->dx[0][c] * g->dx[2][c];
    g->face[2][c] = g->dx[0][c] * g->dx[1][c];
    g->vol[c] = g->dx[0][c] * g->dx[1][c] * g->dx[2][c];
    for (int d = 0; d < 3; d++) {
      g->gff[d][c] = g->face[d][c];
      g->gfv[d][c] = g->vol[c];
    }
  }
  /* face-averaged volumes with the 8-point stencil fac8th
   * (src/config.c:103-104, cartesian_general.c:203-241) */
  static const double f8[8] = {-3.0 / 840, 29.0 / 840, -139.0 / 840, 533.0 / 840,
                               533.0 / 840, -139.0 / 840, 29.0 / 840, -3.0 / 840};
  for (int d = 0; d < 3; d++) {
    int a = (d + 1) % 3, b = (d + 2) % 3;
    for (int f = g->lo[d]; f <= g->hi[d] + 1; f++)
      for (int p = 0; p <= g->gmax[a]; p++)
        for (int q = 0; q <= g->gmax[b]; q++) {
          int ijk[3];
          ijk[d] = f;
          ijk[a] = p;
          ijk[b] = q;
          size_t c = IX(g, ijk[0], ijk[1], ijk[2]);
          double s = 0.0;
          for (int o = -4; o <= 3; o++) s += g->vol[c + o * g->st[d]] * f8[o + 4];
          g->volf[d][c] = s;
        }
  }
  /* PDMU7 weights scaled by vol/vol_face (cartesian_general.c:286-358) */
  static const double fac[7] = {-1.0 / 140.0, 5.0 / 84.0, -101.0 / 420.0, 319.0 / 420.0,
                                107.0 / 210.0, -19.0 / 210.0, 1.0 / 105.0};
  for (int d = 0; d < 3; d++) {
    int a = (d + 1) % 3, b = (d + 2) % 3;
    for (int f = g->lo[d]; f <= g->hi[d] + 1; f++)
      for (int p = 0; p <= g->gmax[a]; p++)
        for (int q = 0; q <= g->gmax[b]; q++) {
          int ijk[3];
          ijk[d] = f;
          ijk[a] = p;
          ijk[b] = q;
          size_t c = IX(g, ijk[0], ijk[1], ijk[2]);
          /* left taps w1l..w7l = fac[0..6]; right taps are stored
           * w1r..w7r = fac[6..0] and applied reversed (wgt[t] = w(7-t)r),
           * so both sides apply fac[t] to their own 7-cell ordering */
          for (int t = 0; t < 7; t++) {
            g->w[d][0][t][c] = fac[t] * g->vol[c] / g->volf[d][c];
            g->w[d][1][t][c] = fac[t] * g->vol[c] / g->volf[d][c];
          }
        }
  }
}

/* Dense LU with partial pivoting and the matching solve; the textbook
 * Doolittle scheme that math_lib/lu_solver.c:10-104 implements. */
static int lu5(double a[5][5], const double b[5], double x[5]) {
  int perm[5];
  const int n = 5;
  for (int i = 0; i < n; i++) perm[i] = i;
  for (int k = 0; k < n - 1; k++) {
    double best = fabs(a[k][k]);
    int row = k;
    for (int i = k + 1; i < n; i++)
      if (fabs(a[i][k]) > best) {
        best = fabs(a[i][k]);
        row = i;
      }
    if (best < 1e-12) return -1;
    if (row != k) {
      for (int j = 0; j < n; j++) {
        double t = a[k][j];
        a[k][j] = a[row][j];
        a[row][j] = t;
      }
      int t = perm[k];
      perm[k] = perm[row];
      perm[row] = t;
    }
    for (int i = k + 1; i < n; i++) {
      double m = a[i][k] / a[k][k];
      a[i][k] = m;
      for (int j = k + 1; j < n; j++) a[i][j] -= m * a[k][j];
    }
  }
  if (fabs(a[n - 1][n - 1]) < 1e-12) return -1;
  double y[5];
  for (int i = 0; i < n; i++) {
    y[i] = b[perm[i]];
    for (int j = 0; j < i; j++) y[i] -= a[i][j] * y[j];
  }
  for (int i = n - 1; i >= 0; i--) {
    x[i] = y[i];
    for (int j = i + 1; j < n; j++) x[i] -= a[i][j] * x[j];
    x[i] /= a[i][i];
  }
  return 0;
}

static double fact(int k) {
  double r = 1.0;
  for (int i = 2; i <= k; ++i) r *= i;
  return r;
}

static double binom(int j, int k) {
  if (k < 0 || k > j) return 0.0;
  if (k == 0 || k == j) return 1.0;
  k = (k < j - k) ? k : j - k;
  double r = 1.0;
  for (int i = 1; i <= k; ++i) r *= (j - k + i) / (double)i;
  return r;
}

/* Spherical geometry and weights, src/spherical/spherical_general.c:42-594 */
static void geometry_spherical(og_t *g) {
  int NI = g->N[0], NJ = g->N[1], NK = g->N[2];
  const double *x1 = g->xs[0], *x2 = g->xs[1], *x3 = g->xs[2];
  LOOP3(i, 0, NI - 1, j, 0, NJ - 1, k, 0, NK - 1) {
    size_t c = IX(g, i, j, k);
    if (i < NI - 1) {
      g->xc[0][c] = 0.5 * (x1[i] + x1[i + 1]);
      g->dx[0][c] = x1[i + 1] - x1[i];
      g->edge[0][c] = g->dx[0][c];
    }
    if (j < NJ - 1) {
      g->xc[1][c] = 0.5 * (x2[j] + x2[j + 1]);
      g->dx[1][c] = x2[j + 1] - x2[j];
      g->edge[1][c] = x1[i] * g->dx[1][c];
    }
    if (k < NK - 1) {
      g->xc[2][c] = 0.5 * (x3[k] + x3[k + 1]);
      g->dx[2][c] = x3[k + 1] - x3[k];
      g->edge[2][c] = x1[i] * sin(x2[j]) * g->dx[2][c];
    }
  }
  LOOP3(i, 0, NI - 2, j, 0, NJ - 2, k, 0, NK - 2) {
    size_t c = IX(g, i, j, k);
    g->dl[0][c] = g->dx[0][c];
    g->dl[1][c] = g->xc[0][c] * g->dx[1][c];
    g->dl[2][c] = g->xc[0][c] * sin(g->xc[1][c]) * g->dx[2][c];
  }
  LOOP3(i, 0, NI - 1, j, 0, NJ - 2, k, 0, NK - 2) {
    size_t c = IX(g, i, j, k);
    g->face[0][c] = -x1[i] * x1[i] * (cos(x2[j + 1]) - cos(x2[j])) * g->dx[2][c];
    g->gff[0][c] = x1[i] * x1[i];
  }
  LOOP3(i, 0, NI - 2, j, 0, NJ - 1, k, 0, NK - 2) {
    size_t c = IX(g, i, j, k);
    g->face[1][c] = 0.5 * (x1[i + 1] * x1[i + 1] - x1[i] * x1[i]) * sin(x2[j]) * g->dx[2][c];
    g->gff[1][c] = sin(x2[j]);
  }
  LOOP3(i, 0, NI - 2, j, 0, NJ - 2, k, 0, NK - 1) {
    size_t c = IX(g, i, j, k);
    g->face[2][c] = 0.5 * (x1[i + 1] * x1[i + 1] - x1[i] * x1[i]) * g->dx[1][c];
    g->gff[2][c] = 1.0;
  }
  LOOP3(i, 0, NI - 2, j, 0, NJ - 2, k, 0, NK - 2) {
    size_t c = IX(g, i, j, k);
    g->vol[c] = fabs(1.0 / 3.0 * (pow(x1[i + 1], 3) - pow(x1[i], 3)) *
                     (cos(x2[j + 1]) - cos(x2[j])) * g->dx[2][c]);
    g->gfv[0][c] = 1.0 / 3.0 * (pow(x1[i + 1], 3) - pow(x1[i], 3));
    g->gfv[1][c] = -(cos(x2[j + 1]) - cos(x2[j]));
    g->gfv[2][c] = g->dx[2][c];
  }
  LOOP3(i, 0, NI - 2, j, 0, NJ - 1, k, 0, NK - 1) {
    size_t c = IX(g, i, j, k);
    double xc = g->xc[0][c], d1 = g->dx[0][c];
    g->xctr[0][c] = xc + 2.0 * xc * d1 * d1 / (12.0 * xc * xc + d1 * d1);
  }
  LOOP3(i, 0, NI - 1, j, 0, NJ - 2, k, 0, NK - 1) {
    size_t c = IX(g, i, j, k);
    g->xctr[1][c] = (sin(x2[j + 1]) - sin(x2[j]) -
                     (x2[j + 1] * cos(x2[j + 1]) - x2[j] * cos(x2[j]))) /
                    (-cos(x2[j + 1]) + cos(x2[j]));
  }
  LOOP3(i, 0, NI - 1, j, 0, NJ - 1, k, 0, NK - 2) {
    size_t c = IX(g, i, j, k);
    g->xctr[2][c] = g->xc[2][c];
  }

  /* radial weights: 5-point non-uniform reconstruction in r
   * (spherical_general.c:319-441); taps 1 and 7 are zero */
  const int m = 2;
  int n1 = g->n[0];
  double *xs = (double *)calloc((size_t)(n1 + 2 * NG + 1 + 2 * NG), sizeof(double));
  int ieg = g->gmax[0];
  for (int i = NG; i <= ieg + NG + 1; i++) xs[i] = x1[i - NG];
  for (int i = NG - 1; i >= 0; i--) xs[i] = xs[i + 1] - A3(g->dx[0], 0, 0, 0);
  for (int i = ieg + NG + 2; i <= ieg + 2 * NG + 1; i++) xs[i] = xs[i - 1] + A3(g->dx[0], ieg, 0, 0);
  for (int side = 0; side < 2; side++) {
    for (int idx = 0; idx <= ieg + 1; idx++) {
      double a[5][5], b[5], x[5];
      for (int i = -2; i <= 2; i++) {
        double xm = side == 0 ? xs[idx + NG + i - 1] : xs[idx + NG + i];
        double xp = side == 0 ? xs[idx + NG + i] : xs[idx + NG + i + 1];
        for (int j = 0; j <= 4; j++)
          a[j][i + 2] = (double)(m + 1) / (double)(j + m + 1) *
                        (pow(xp, j + m + 1) - pow(xm, j + m + 1)) /
                        (pow(xp, m + 1) - pow(xm, m + 1));
        b[i + 2] = pow(xs[idx + NG], i + 2);
      }
      double wv[7] = {0, 0, 0, 0, 0, 0, 0};
      if (lu5(a, b, x) == 0)
        for (int t = 0; t < 5; t++) wv[t + 1] = x[t];
      /* right-hand taps are stored w1r..w7r = wv[0..6]; applied reversed */
      for (int j = 0; j < NJ; j++)
        for (int k = 0; k < NK; k++)
          for (int t = 0; t < 7; t++)
            g->w[0][side][side == 0 ? t : 6 - t][IX(g, idx, j, k)] = wv[t];
    }
  }
  free(xs);

  /* polar weights (spherical_general.c:443-570); the right-hand loop stops
   * at jeg like the reference */
  int n2 = g->n[1];
  double *ts = (double *)calloc((size_t)(n2 + 2 * NG + 1 + 2 * NG), sizeof(double));
  int jeg = g->gmax[1];
  for (int j = NG; j <= jeg + NG + 1; j++) ts[j] = x2[j - NG];
  for (int j = NG - 1; j >= 0; j--) ts[j] = ts[j + 1] - A3(g->dx[1], 0, 0, 0);
  for (int j = jeg + NG + 2; j <= jeg + 2 * NG + 1; j++) ts[j] = ts[j - 1] + A3(g->dx[1], 0, jeg, 0);
  for (int side = 0; side < 2; side++) {
    int last = side == 0 ? jeg + 1 : jeg;
    for (int idx = 0; idx <= last; idx++) {
      double a[5][5], b[5], x[5];
      for (int i = -2; i <= 2; i++) {
        double xm = side == 0 ? ts[idx + NG + i - 1] : ts[idx + NG + i];
        double xp = side == 0 ? ts[idx + NG + i] : ts[idx + NG + i + 1];
        for (int j = 0; j <= 4; j++) {
          double sum = 0.0;
          for (int k = 0; k <= j; k++)
            sum = sum + fact(k) * binom(j, k) *
                            (pow(xm, j - k) * cos(xm + k * GOP_PI / 2.0) -
                             pow(xp, j - k) * cos(xp + k * GOP_PI / 2.0));
          a[j][i + 2] = sum / (cos(xm) - cos(xp));
        }
        b[i + 2] = pow(ts[idx + NG], i + 2);
      }
      double wv[7] = {0, 0, 0, 0, 0, 0, 0};
      if (lu5(a, b, x) == 0)
        for (int t = 0; t < 5; t++) wv[t + 1] = x[t];
      for (int i = 0; i < NI; i++)
        for (int k = 0; k < NK; k++)
          for (int t = 0; t < 7; t++)
            g->w[1][side][side == 0 ? t : 6 - t][IX(g, i, idx, k)] = wv[t];
    }
  }
  free(ts);

  /* azimuthal weights: fixed uniform 5-point (spherical_general.c:572-594) */
  static const double wl[7] = {0.0, 1.0 / 30.0, -13.0 / 60.0, 47.0 / 60.0,
                               9.0 / 20.0, -1.0 / 20.0, 0.0};
  static const double wr[7] = {0.0, -1.0 / 20.0, 9.0 / 20.0, 47.0 / 60.0,
                               -13.0 / 60.0, 1.0 / 30.0, 0.0};
  for (size_t c = 0; c < g->n3; c++)
    for (int t = 0; t < 7; t++) {
      g->w[2][0][t][c] = wl[t];
      g->w[2][1][6 - t][c] = wr[t];
    }
}

/* -------------------------------------------------------------- lifecycle */

og_t *og_create(const og_desc *d) {
  if (!d || d->ni < NG || d->nj < NG || d->nk < NG) return NULL;
  if (d->coord != 0 && d->coord != 2) return NULL;
  og_t *g = (og_t *)calloc(1, sizeof(og_t));
  g->d = *d;
  g->gamma = d->gamma;
  g->cfl = d->cfl;
  g->ca = d->ca;
  g->pdmb = d->pdmb;
  g->rho_floor = d->rho_floor;
  g->p_floor = d->p_floor;
  g->n[0] = d->ni;
  g->n[1] = d->nj;
  g->n[2] = d->nk;
  for (int a = 0; a < 3; a++) {
    g->N[a] = g->n[a] + 2 * NG + 1;
    g->lo[a] = NG;
    g->hi[a] = NG + g->n[a] - 1;
    g->gmax[a] = g->hi[a] + NG;
    g->periodic[a] = d->bc[2 * a] == 'p' && d->bc[2 * a + 1] == 'p';
  }
  g->st[0] = (long)g->N[1] * g->N[2];
  g->st[1] = g->N[2];
  g->st[2] = 1;
  g->n3 = (size_t)g->N[0] * g->N[1] * g->N[2];
  g->pool_cap = 240;
  g->pool = (double *)calloc(g->pool_cap * g->n3, sizeof(double));
  if (!g->pool) {
    free(g);
    return NULL;
  }
  for (int a = 0; a < 3; a++) {
    g->xs[a] = (double *)malloc(sizeof(double) * (size_t)g->N[a]);
    memcpy(g->xs[a], a == 0 ? d->x1 : a == 1 ? d->x2 : d->x3, sizeof(double) * (size_t)g->N[a]);
  }
  for (int a = 0; a < 3; a++) {
    g->dx[a] = take(g);
    g->xc[a] = take(g);
    g->xctr[a] = take(g);
    g->edge[a] = take(g);
    g->dl[a] = take(g);
    g->face[a] = take(g);
    g->gff[a] = take(g);
    g->gfv[a] = take(g);
    g->volf[a] = take(g);
    for (int s = 0; s < 2; s++)
      for (int t = 0; t < 7; t++) g->w[a][s][t] = take(g);
  }
  g->vol = take(g);
  for (int m = 0; m < 6; m++) {
    g->W[m] = take(g);
    g->Wh[m] = take(g);
    g->Wp[m] = take(g);
    g->U[m] = take(g);
    g->U0[m] = take(g);
    g->dU[m] = take(g);
    g->F[m] = take(g);
    g->L[m] = take(g);
    g->R[m] = take(g);
  }
  for (int a = 0; a < 3; a++) {
    g->B[a] = take(g);
    g->Bh[a] = take(g);
    g->Bp[a] = take(g);
    g->ms[a] = take(g);
    g->msh[a] = take(g);
    g->msp[a] = take(g);
    g->mt[a] = take(g);
    g->v0[a] = take(g);
    g->mL[a] = take(g);
    g->mR[a] = take(g);
    g->MF[a] = take(g);
    g->dMF[a] = take(g);
    g->SH[a] = take(g);
    g->SB[a] = take(g);
    g->E[a] = take(g);
    g->vil[a] = take(g);
    g->vir[a] = take(g);
    g->vin[a] = take(g);
    g->vav[a] = take(g);
    g->bl[a] = take(g);
    g->br[a] = take(g);
  }
  if (g->pool_used > g->pool_cap) abort();
  if (d->coord == 0)
    geometry_cartesian(g);
  else
    geometry_spherical(g);
  return g;
}

void og_destroy(og_t *g) {
  if (!g) return;
  for (int a = 0; a < 3; a++) free(g->xs[a]);
  free(g->pool);
  free(g);
}

/* ------------------------------------------------------- halo and ghosts */

/* Single-domain halo exchange, src/boundary_exchange.c:7-165 with the index
 * sets of src/setup_mpi.c:62-253: on a periodic axis the high ghosts take the
 * low active layers (shifted by onface for the face-normal field) and the low
 * ghosts take the high active layers.  Axes go in the order i, j, k over the
 * full transverse extent, so edges and corners wrap too. */
static void wrap(og_t *g, double *a, int axis, int onface) {
  int N = g->N[axis];
  int oa = (axis + 1) % 3, ob = (axis + 2) % 3;
  for (int p = 0; p < g->N[oa]; p++)
    for (int q = 0; q < g->N[ob]; q++) {
      int ijk[3];
      ijk[oa] = p;
      ijk[ob] = q;
      for (int t = 0; t < NG; t++) {
        ijk[axis] = NG + onface + t;
        double v = a[IX(g, ijk[0], ijk[1], ijk[2])];
        ijk[axis] = N - NG - 1 + onface + t;
        a[IX(g, ijk[0], ijk[1], ijk[2])] = v;
      }
      for (int t = 0; t < NG; t++) {
        ijk[axis] = N - 2 * NG - 1 + t;
        double v = a[IX(g, ijk[0], ijk[1], ijk[2])];
        ijk[axis] = t;
        a[IX(g, ijk[0], ijk[1], ijk[2])] = v;
      }
    }
}

/* One ghost-fill routine of src/boundary_conditions.c on one field.
 * kind: s symmetric, r reflective (sign flip of the normal velocity),
 * f fixed (constant), e extrapolated, n none.  flip: field is the normal
 * velocity; onface: field is face-centred along this axis. */
static void ghost_bc(og_t *g, double *a, int axis, int side, char kind, int onface,
                     int flip, int has_const, double cval) {
  int N = g->N[axis];
  int oa = (axis + 1) % 3, ob = (axis + 2) % 3;
  if (kind == 'n' || kind == 'p') return;
  if (kind == 'f' && !has_const) return;
  for (int p = 0; p < g->N[oa]; p++)
    for (int q = 0; q < g->N[ob]; q++) {
      int ijk[3];
      ijk[oa] = p;
      ijk[ob] = q;
      for (int t = 0; t < NG; t++) {
        int dst, src;
        if (side == 0) {
          dst = t;
          src = kind == 'e' ? NG : 2 * NG - 1 - t + onface;
        } else {
          dst = N - 1 - NG + t + onface;
          src = kind == 'e' ? N - 1 - NG - 1 + onface : N - 1 - NG - 1 - t;
        }
        if (kind == 'f') {
          ijk[axis] = side == 0 ? t : N - 1 - NG + t + onface;
          a[IX(g, ijk[0], ijk[1], ijk[2])] = cval;
          continue;
        }
        ijk[axis] = src;
        double v = a[IX(g, ijk[0], ijk[1], ijk[2])];
        if (kind == 'r' && flip) v = -v;
        ijk[axis] = dst;
        a[IX(g, ijk[0], ijk[1], ijk[2])] = v;
      }
    }
}

/* fixed-state constants of gas_bc_fixed_* (boundary_conditions.c:247-402) */
static int fixed_gas_value(int axis, int side, int m, double *v) {
  if (m == PS) return 0;
  if (m == V1 || m == V2 || m == V3) {
    *v = 0.0;
    return 1;
  }
  if (m == RHO) {
    *v = (axis == 1 && side == 0) ? 2.0 : 1.0;
    return 1;
  }
  *v = (axis == 1 && side == 1) ? 2.5 : 1.0; /* pressure */
  return 1;
}

/* halo exchange of gem and gas, then boundary_conditions()
 * (src/solver_solve.c:493-506); mags is exchanged but recomputed after */
static void fill_ghosts(og_t *g) {
  for (int axis = 0; axis < 3; axis++) {
    if (!g->periodic[axis]) continue;
    for (int c = 0; c < 3; c++) wrap(g, g->B[c], axis, c == axis);
    for (int c = 0; c < 3; c++) wrap(g, g->ms[c], axis, 0);
  }
  for (int axis = 0; axis < 3; axis++) {
    if (!g->periodic[axis])
      continue;
    for (int m = 0; m < 6; m++) wrap(g, g->W[m], axis, 0);
  }
  for (int face = 0; face < 6; face++) {
    int axis = face / 2, side = face % 2;
    char kind = g->d.bc[face];
    if (g->periodic[axis]) continue;
    for (int m = 0; m < 6; m++) {
      double cv = 0.0;
      int hc = kind == 'f' ? fixed_gas_value(axis, side, m, &cv) : 1;
      ghost_bc(g, g->W[m], axis, side, kind, 0, m == V1 + axis, hc, cv);
    }
    if (kind == 'r') continue; /* gem_bc_reflective_* are empty */
    for (int c = 0; c < 3; c++)
      ghost_bc(g, g->B[c], axis, side, kind, c == axis, 0, 1, 0.0);
    for (int c = 0; c < 3; c++)
      ghost_bc(g, g->ms[c], axis, side, kind, 0, 0, 1, 0.0);
  }
}

/* ------------------------------------------------------------- numerics */

static double sgn(double x) { return x > 0.0 ? 1.0 : (x < 0.0 ? -1.0 : 0.0); }

/* PDMU7, src/solver_func.c:215-253: 7-tap interpolation of the half-step
 * values, clamped to the two adjacent step-start values, then the PDM
 * limiter with its geometric reference slope. */
static double pdm7(const double fh[7], const double fp[7], const double wt[7],
                   double face_m1, double face_0, double vol, double dx, double pdmb) {
  double fi = 0.0;
  for (int t = 0; t < 7; t++) fi += fh[t] * wt[t];
  double hi = fmax(fp[3], fp[4]);
  double lo = fmin(fp[3], fp[4]);
  double f = fmax(lo, fmin(fi, hi));
  double d0 = pdmb * (fp[3] - fp[2]);
  double d1 = pdmb * (fp[4] - fp[3]);
  double s0 = sgn(d0), s1 = sgn(d1);
  d0 = fabs(d0);
  double q0 = fabs(s0 + s1);
  double dl = f - fp[3];
  double q = vol / dx;
  double e = 1.0 / (2 * pdmb + 1.0);
  double dc = fabs((q - e * face_0) / (e * face_0) * fp[3] +
                   (e * face_m1 - q) / (e * face_0) * fp[2]) / 2.0;
  double a1 = pdmb / (pdmb + 1.0);
  double a2 = 1.0 - a1;
  dc = a1 * dc + a2 * d0;
  return f - s1 * fmax(0, fabs(dl) - q0 * dc);
}

/* reconstruct_3dv_{i,j,k}, src/solver_func.c:503-649: left and right face
 * states along axis d, for faces lo..hi+1 along d and every ghost index
 * across.  fp is the limiter reference (fh itself for pdm_index 0). */
static void recon(og_t *g, int d, const double *fh, const double *fp, double *outl,
                  double *outr) {
  int a = (d + 1) % 3, b = (d + 2) % 3;
  long s = g->st[d];
  for (int f = g->lo[d]; f <= g->hi[d] + 1; f++)
    for (int p = 0; p <= g->gmax[a]; p++)
      for (int q = 0; q <= g->gmax[b]; q++) {
        int ijk[3];
        ijk[d] = f;
        ijk[a] = p;
        ijk[b] = q;
        size_t c = IX(g, ijk[0], ijk[1], ijk[2]);
        double h[7], r[7], wt[7];
        for (int t = 0; t < 7; t++) {
          h[t] = fh[c + (t - 4) * s];
          r[t] = fp[c + (t - 4) * s];
          wt[t] = g->w[d][0][t][c];
        }
        outl[c] = pdm7(h, r, wt, g->gff[d][c - s], g->gff[d][c], g->gfv[d][c - s],
                       g->dx[d][c - s], g->pdmb);
        for (int t = 0; t < 7; t++) {
          h[t] = fh[c + (3 - t) * s];
          r[t] = fp[c + (3 - t) * s];
          wt[t] = g->w[d][1][t][c];
        }
        outr[c] = pdm7(h, r, wt, g->gff[d][c + s], g->gff[d][c], g->gfv[d][c],
                       g->dx[d][c], g->pdmb);
      }
}

/* cell-centred field from the two faces, weighted by the centroid
 * (src/solver_func.c:311-322 and src/solver_solve.c:385-397) */
static void mags_from_faces(og_t *g, double *const *Bf, double **out, int i0, int i1,
                            int j0, int j1, int k0, int k1) {
  const double *x1 = g->xs[0], *x2 = g->xs[1], *x3 = g->xs[2];
  LOOP3(i, i0, i1, j, j0, j1, k, k0, k1) {
    size_t c = IX(g, i, j, k);
    out[0][c] = Bf[0][c] * (x1[i + 1] - g->xctr[0][c]) / g->dx[0][c] +
                Bf[0][c + g->st[0]] * (g->xctr[0][c] - x1[i]) / g->dx[0][c];
    out[1][c] = Bf[1][c] * (x2[j + 1] - g->xctr[1][c]) / g->dx[1][c] +
                Bf[1][c + g->st[1]] * (g->xctr[1][c] - x2[j]) / g->dx[1][c];
    out[2][c] = Bf[2][c] * (x3[k + 1] - g->xctr[2][c]) / g->dx[2][c] +
                Bf[2][c + g->st[2]] * (g->xctr[2][c] - x3[k]) / g->dx[2][c];
  }
}

/* get_derived_variables, src/solver_func.c:308-383 */
static void derived(og_t *g) {
  int *lo = g->lo, *hi = g->hi, *gm = g->gmax;
  mags_from_faces(g, g->B, g->ms, 0, gm[0], 0, gm[1], 0, gm[2]);
  double mx = 0.0;
  LOOP3(i, lo[0], hi[0], j, lo[1], hi[1], k, lo[2], hi[2]) {
    size_t c = IX(g, i, j, k);
    double db = (g->B[0][c + g->st[0]] * g->face[0][c + g->st[0]] - g->B[0][c] * g->face[0][c]) / g->vol[c] +
                (g->B[1][c + g->st[1]] * g->face[1][c + g->st[1]] - g->B[1][c] * g->face[1][c]) / g->vol[c] +
                (g->B[2][c + g->st[2]] * g->face[2][c + g->st[2]] - g->B[2][c] * g->face[2][c]) / g->vol[c];
    if (fabs(db) > mx) mx = fabs(db);
  }
  g->divb = mx;
  LOOP3(i, 0, gm[0], j, 0, gm[1], k, 0, gm[2]) {
    size_t c = IX(g, i, j, k);
    for (int a = 0; a < 3; a++) g->mt[a][c] = g->ms[a][c];
  }
  double gm1 = g->gamma - 1.0;
  LOOP3(i, lo[0], hi[0], j, lo[1], hi[1], k, lo[2], hi[2]) {
    size_t c = IX(g, i, j, k);
    double r = g->W[RHO][c], u = g->W[V1][c], v = g->W[V2][c], w = g->W[V3][c];
    g->U[0][c] = r;
    g->U[1][c] = r * u;
    g->U[2][c] = r * v;
    g->U[3][c] = r * w;
    g->U[4][c] = 0.5 * r * (u * u + v * v + w * w) + g->W[PR][c] / gm1;
    g->U[5][c] = g->W[PS][c] / pow(r, gm1);
  }
}

/* get_dt_normal, src/solver_func.c:255-298 */
static double cfl_dt(og_t *g) {
  double best = INFINITY;
  int *lo = g->lo, *hi = g->hi;
  LOOP3(i, lo[0], hi[0], j, lo[1], hi[1], k, lo[2], hi[2]) {
    size_t c = IX(g, i, j, k);
    double b2 = g->mt[0][c] * g->mt[0][c] + g->mt[1][c] * g->mt[1][c] + g->mt[2][c] * g->mt[2][c];
    double va = sqrt(b2 / g->W[RHO][c]);
    double vae = va * g->ca / (sqrt(va * va + g->ca * g->ca));
    double u = g->W[V1][c], v = g->W[V2][c], w = g->W[V3][c];
    double vf = sqrt(u * u + v * v + w * w);
    double vs = sqrt(g->gamma * g->W[PR][c] / g->W[RHO][c]);
    double vc = vf + sqrt(vs * vs + vae * vae);
    double dtc = g->cfl / (vc / g->dl[0][c] + vc / g->dl[1][c] + vc / g->dl[2][c]);
    best = fmin(best, dtc);
  }
  return best;
}

/* the AB2 predictor and history shift, src/solver_func.c:385-492 */
static void ab2(og_t *g) {
  int *gm = g->gmax;
  LOOP3(i, 0, gm[0], j, 0, gm[1], k, 0, gm[2]) {
    size_t c = IX(g, i, j, k);
    for (int m = 0; m < 6; m++)
      g->Wh[m][c] = g->W[m][c] + 0.5 * g->dt / g->dt0 * (g->W[m][c] - g->Wp[m][c]);
    for (int a = 0; a < 3; a++)
      g->msh[a][c] = g->ms[a][c] + 0.5 * g->dt / g->dt0 * (g->ms[a][c] - g->msp[a][c]);
  }
  for (int a = 0; a < 3; a++) {
    int e[3] = {gm[0], gm[1], gm[2]};
    e[a]++;
    LOOP3(i, 0, e[0], j, 0, e[1], k, 0, e[2]) {
      size_t c = IX(g, i, j, k);
      g->Bh[a][c] = g->B[a][c] + 0.5 * g->dt / g->dt0 * (g->B[a][c] - g->Bp[a][c]);
    }
  }
  LOOP3(i, 0, gm[0], j, 0, gm[1], k, 0, gm[2]) {
    size_t c = IX(g, i, j, k);
    for (int m = 0; m < 6; m++) g->Wp[m][c] = g->W[m][c];
    for (int a = 0; a < 3; a++) g->msp[a][c] = g->ms[a][c];
  }
  LOOP3(i, 0, gm[0] + 1, j, 0, gm[1] + 1, k, 0, gm[2] + 1) {
    size_t c = IX(g, i, j, k);
    for (int a = 0; a < 3; a++) g->Bp[a][c] = g->B[a][c];
  }
  g->dt0 = g->dt;
}

/* center2corner_{jk,ki,ij}, src/solver_func.c:686-778, for velocity
 * component vc: reconstruct along axis p (limiter on the step-start value),
 * average, reconstruct along axis q limiting against itself, average. */
static void center2corner(og_t *g, int p, int q, int vc) {
  int *lo = g->lo, *hi = g->hi, *gm = g->gmax;
  double *il = g->vil[vc], *ir = g->vir[vc], *in = g->vin[vc], *av = g->vav[vc];
  recon(g, p, g->Wh[V1 + vc], g->Wp[V1 + vc], il, ir);
  int r0[3], r1[3];
  for (int a = 0; a < 3; a++) {
    r0[a] = lo[a];
    r1[a] = hi[a];
  }
  r1[p] = hi[p] + 1;
  r0[q] = 0;
  r1[q] = gm[q];
  LOOP3(i, r0[0], r1[0], j, r0[1], r1[1], k, r0[2], r1[2]) {
    size_t c = IX(g, i, j, k);
    in[c] = 0.5 * (il[c] + ir[c]);
  }
  recon(g, q, in, in, il, ir);
  r0[q] = lo[q];
  r1[q] = hi[q] + 1;
  LOOP3(i, r0[0], r1[0], j, r0[1], r1[1], k, r0[2], r1[2]) {
    size_t c = IX(g, i, j, k);
    av[c] = 0.5 * (il[c] + ir[c]);
  }
}

/* get_e_fields_{i,j,k}, src/solver_func.c:779-902: edge EMF along axis d
 * from the corner velocity, the reconstructed transverse face fields and the
 * fast-speed diffusion term.  (p,q) = (d+1,d+2) cyclic. */
static void efield(og_t *g, int d) {
  int p = (d + 1) % 3, q = (d + 2) % 3;
  int *lo = g->lo, *hi = g->hi;
  /* the reference's centre-to-corner sweep order per edge direction */
  if (d == 0) {
    center2corner(g, 1, 2, 1);
    center2corner(g, 1, 2, 2);
  } else if (d == 1) {
    center2corner(g, 2, 0, 2);
    center2corner(g, 2, 0, 0);
  } else {
    center2corner(g, 0, 1, 0);
    center2corner(g, 0, 1, 1);
  }
  /* B_p reconstructed along q, B_q along p */
  recon(g, q, g->Bh[p], g->Bp[p], g->bl[p], g->br[p]);
  recon(g, p, g->Bh[q], g->Bp[q], g->bl[q], g->br[q]);
  int r0[3], r1[3];
  for (int a = 0; a < 3; a++) {
    r0[a] = lo[a];
    r1[a] = hi[a] + (a == d ? 0 : 1);
  }
  double *vp = g->vav[p], *vq = g->vav[q];
  long sp = g->st[p], sq = g->st[q];
  LOOP3(i, r0[0], r1[0], j, r0[1], r1[1], k, r0[2], r1[2]) {
    size_t c = IX(g, i, j, k);
    double bp = 0.5 * (g->bl[p][c] + g->br[p][c]);
    double bq = 0.5 * (g->bl[q][c] + g->br[q][c]);
    double e = -(vp[c] * bq - vq[c] * bp);
    const double *rh = g->Wh[RHO];
    double rho4;
    if (d == 0) /* (j-1,k-1) (j-1,k) (j,k-1) (j,k) */
      rho4 = rh[c - sp - sq] + rh[c - sp] + rh[c - sq] + rh[c];
    else if (d == 1) /* (i-1,k-1) (i-1,k) (i,k-1) (i,k): q = i, p = k */
      rho4 = rh[c - sq - sp] + rh[c - sq] + rh[c - sp] + rh[c];
    else /* (i-1,j-1) (i-1,j) (i,j-1) (i,j): p = i, q = j */
      rho4 = rh[c - sp - sq] + rh[c - sp] + rh[c - sq] + rh[c];
    double vz = sqrt((bp * bp + bq * bq) / (0.25 * rho4));
    vz = vz * g->ca / sqrt(vz * vz + g->ca * g->ca) + sqrt(vp[c] * vp[c] + vq[c] * vq[c]);
    /* J = b_{p,l} + b_{q,r} - b_{p,r} - b_{q,l} */
    e += 0.5 * vz * (g->bl[p][c] + g->br[q][c] - g->br[p][c] - g->bl[q][c]);
    g->E[d][c] = e;
  }
}

/* get_fluid_flux_rusanov_*, src/solver_func.c:934-1266 and
 * get_magnetic_stress_rusanov_*, 1268-1529, at faces normal to axis d */
static void fluxes(og_t *g, int d) {
  int *lo = g->lo, *hi = g->hi;
  int r1[3] = {hi[0], hi[1], hi[2]};
  r1[d] = hi[d] + 1;
  double gm = g->gamma, gm1 = g->gamma - 1.0, ca = g->ca;
  LOOP3(i, lo[0], r1[0], j, lo[1], r1[1], k, lo[2], r1[2]) {
    size_t c = IX(g, i, j, k);
    double rl = g->L[RHO][c], rr = g->R[RHO][c];
    double pl = g->L[PR][c], pr = g->R[PR][c];
    double sl = g->L[PS][c], sr = g->R[PS][c];
    double vl[3] = {g->L[V1][c], g->L[V2][c], g->L[V3][c]};
    double vr[3] = {g->R[V1][c], g->R[V2][c], g->R[V3][c]};
    double ml[3] = {g->mL[0][c], g->mL[1][c], g->mL[2][c]};
    double mr[3] = {g->mR[0][c], g->mR[1][c], g->mR[2][c]};
    double csl = sqrt(gm * pl / rl), csr = sqrt(gm * pr / rr);
    double csel = sqrt(gm * sl / rl), cser = sqrt(gm * sr / rr);
    double btl = ml[0] * ml[0] + ml[1] * ml[1] + ml[2] * ml[2];
    double btr = mr[0] * mr[0] + mr[1] * mr[1] + mr[2] * mr[2];
    double val = sqrt(btl / rl), var = sqrt(btr / rr);
    double vel = val * ca / (sqrt(val * val + ca * ca));
    double ver = var * ca / (sqrt(var * var + ca * ca));
    double vnl = vl[d], vnr = vr[d];
    double vf = fmax(fabs(vnl) + sqrt(csl * csl + vel * vel), fabs(vnr) + sqrt(csr * csr + ver * ver));
    double vfe = fmax(fabs(vnl) + sqrt(csel * csel + vel * vel), fabs(vnr) + sqrt(cser * cser + ver * ver));
    double mol[3], mor[3];
    for (int a = 0; a < 3; a++) {
      mol[a] = rl * vl[a];
      mor[a] = rr * vr[a];
    }
    double el = 0.5 * rl * (vl[0] * vl[0] + vl[1] * vl[1] + vl[2] * vl[2]) + pl / gm1;
    double er = 0.5 * rr * (vr[0] * vr[0] + vr[1] * vr[1] + vr[2] * vr[2]) + pr / gm1;
    double Sl = sl / pow(rl, gm1), Sr = sr / pow(rr, gm1);
    g->F[0][c] = 0.5 * (mol[d] + mor[d] - vf * (rr - rl));
    for (int a = 0; a < 3; a++) {
      if (a == d)
        g->F[1 + a][c] = 0.5 * (mol[a] * vnl + pl + mor[a] * vnr + pr - vf * (mor[a] - mol[a]));
      else
        g->F[1 + a][c] = 0.5 * (mol[a] * vnl + mor[a] * vnr - vf * (mor[a] - mol[a]));
    }
    g->F[4][c] = 0.5 * (el * vnl + pl * vnl + er * vnr + pr * vnr - vf * (er - el));
    g->F[5][c] = 0.5 * (Sl * vnl + Sr * vnr - vfe * (Sr - Sl));
    /* Maxwell stress with the step-start normal face field */
    double bn = g->B[d][c];
    double bsl = ml[0] * ml[0] + ml[1] * ml[1] + ml[2] * ml[2];
    double bsr = mr[0] * mr[0] + mr[1] * mr[1] + mr[2] * mr[2];
    for (int a = 0; a < 3; a++) {
      double tl, tr;
      if (a == d) {
        tl = 0.5 * (0.5 * bsl - ml[a] * bn);
        tr = 0.5 * (0.5 * bsr - mr[a] * bn);
      } else {
        tl = 0.5 * (-ml[a] * bn);
        tr = 0.5 * (-mr[a] * bn);
      }
      g->MF[a][c] = tl + tr;
    }
    double bq = (btl + btr) / 4 / ca;
    for (int a = 0; a < 3; a++) g->MF[a][c] = g->MF[a][c] - bq * (vr[a] - vl[a]);
  }
}

/* Source_Term_i / Source_Term_j, src/spherical/spherical_general.c:605-681 */
static void sources_spherical(og_t *g, int d) {
  int *lo = g->lo, *hi = g->hi;
  const double *x2 = g->xs[1];
  if (d == 0) {
    LOOP3(i, lo[0], hi[0], j, lo[1], hi[1], k, lo[2], hi[2]) {
      size_t c = IX(g, i, j, k), ci = c + g->st[0], cj = c + g->st[1];
      double m22 = g->Wh[PR][c] + g->Wh[RHO][c] * g->Wh[V2][c] * g->Wh[V2][c];
      double m33 = g->Wh[PR][c] + g->Wh[RHO][c] * g->Wh[V3][c] * g->Wh[V3][c];
      double fi0 = g->face[0][c], fi1 = g->face[0][ci], vol = g->vol[c];
      double dr = g->dx[0][c], rc = g->xc[0][c];
      g->SH[0][c] = 0.5 * (m22 + m33) * (fi1 - fi0) / vol;
      double s21 = -(g->F[2][c] * fi0 + g->F[2][ci] * fi1) * dr / rc / 2.0 / vol;
      double s22 = (g->face[1][cj] - g->face[1][c]) / vol * m33;
      g->SH[1][c] = s21 + s22;
      g->SH[2][c] = -(g->F[3][c] * fi0 + g->F[3][ci] * fi1) * dr / rc / 2.0 / vol;
      double b1 = g->msh[0][c], b2 = g->msh[1][c], b3 = g->msh[2][c];
      double bsq = b1 * b1 + b2 * b2 + b3 * b3;
      double n22 = (0.5 * bsq - b2 * b2);
      double n33 = (0.5 * bsq - b3 * b3);
      g->SB[0][c] = 0.5 * (n22 + n33) * (fi1 - fi0) / vol;
      double t21 = -(g->MF[1][c] * fi0 + g->MF[1][ci] * fi1) * dr / rc / 2.0 / vol;
      double t22 = (g->face[1][cj] - g->face[1][c]) / vol * n33;
      g->SB[1][c] = t21 + t22;
      g->SB[2][c] = -(g->MF[2][c] * fi0 + g->MF[2][ci] * fi1) * dr / rc / 2.0 / vol;
    }
  } else if (d == 1) {
    LOOP3(i, lo[0], hi[0], j, lo[1], hi[1], k, lo[2], hi[2]) {
      size_t c = IX(g, i, j, k), cj = c + g->st[1];
      double fj0 = g->face[1][c], fj1 = g->face[1][cj], vol = g->vol[c];
      double sd = sin(x2[j + 1]) - sin(x2[j]), ss = sin(x2[j + 1]) + sin(x2[j]);
      g->SH[2][c] += -(g->F[3][c] * fj0 + g->F[3][cj] * fj1) * sd / ss / vol;
      g->SB[2][c] += -(g->MF[2][c] * fj0 + g->MF[2][cj] * fj1) * sd / ss / vol;
    }
  }
}

/* one pass of the time loop, src/solver_solve.c:103-508 */
static void step(og_t *g) {
  int *lo = g->lo, *hi = g->hi;
  g->dt = cfl_dt(g);
  g->time += g->dt;
  ab2(g);
  LOOP3(i, lo[0], hi[0], j, lo[1], hi[1], k, lo[2], hi[2]) {
    size_t c = IX(g, i, j, k);
    for (int m = 0; m < 6; m++) g->U0[m][c] = g->U[m][c];
    for (int a = 0; a < 3; a++) g->v0[a][c] = g->W[V1 + a][c];
  }
  for (int d = 0; d < 3; d++) efield(g, d);

  for (int d = 0; d < 3; d++) {
    for (int m = 0; m < 6; m++) recon(g, d, g->Wh[m], g->Wp[m], g->L[m], g->R[m]);
    for (int a = 0; a < 3; a++) recon(g, d, g->msh[a], g->msp[a], g->mL[a], g->mR[a]);
    fluxes(g, d);
    if (g->d.coord == 2) sources_spherical(g, d);
    long s = g->st[d];
    LOOP3(i, lo[0], hi[0], j, lo[1], hi[1], k, lo[2], hi[2]) {
      size_t c = IX(g, i, j, k);
      for (int m = 0; m < 6; m++) {
        double v = (g->F[m][c + s] * g->face[d][c + s] - g->F[m][c] * g->face[d][c]) / g->vol[c];
        g->dU[m][c] = d == 0 ? v : g->dU[m][c] + v;
      }
      for (int a = 0; a < 3; a++) {
        double v = (g->MF[a][c + s] * g->face[d][c + s] - g->MF[a][c] * g->face[d][c]) / g->vol[c];
        g->dMF[a][c] = d == 0 ? v : g->dMF[a][c] + v;
      }
    }
  }

  /* constrained transport, src/solver_solve.c:263-306 */
  double dt = g->dt;
  for (int a = 0; a < 3; a++) {
    int p = (a + 1) % 3, q = (a + 2) % 3;
    int r1[3] = {hi[0], hi[1], hi[2]};
    r1[a] = hi[a] + 1;
    long sp = g->st[p], sq = g->st[q];
    LOOP3(i, lo[0], r1[0], j, lo[1], r1[1], k, lo[2], r1[2]) {
      size_t c = IX(g, i, j, k);
      double cq = g->E[q][c + sp] * g->edge[q][c + sp] - g->E[q][c] * g->edge[q][c];
      double cp = g->E[p][c + sq] * g->edge[p][c + sq] - g->E[p][c] * g->edge[p][c];
      g->B[a][c] -= dt * (cq - cp) / g->face[a][c];
    }
  }

  /* conservative update, cons -> prim, floors (src/solver_solve.c:326-382,
   * src/solver_func.c:2117-2135) */
  double gm1 = g->gamma - 1.0;
  LOOP3(i, lo[0], hi[0], j, lo[1], hi[1], k, lo[2], hi[2]) {
    size_t c = IX(g, i, j, k);
    g->U[0][c] -= dt * g->dU[0][c];
    for (int a = 0; a < 3; a++)
      g->U[1 + a][c] = g->U[1 + a][c] - dt * g->dU[1 + a][c] + dt * g->SH[a][c];
    g->U[4][c] -= dt * g->dU[4][c];
    g->U[5][c] -= dt * g->dU[5][c];
    g->W[RHO][c] = g->U[0][c];
    for (int a = 0; a < 3; a++) g->W[V1 + a][c] = g->U[1 + a][c] / g->U[0][c];
    double u = g->W[V1][c], v = g->W[V2][c], w = g->W[V3][c];
    g->W[PR][c] = (g->U[4][c] - 0.5 * (u * u + v * v + w * w) * g->W[RHO][c]) * gm1;
    g->W[PS][c] = g->U[5][c] * pow(g->U[0][c], gm1);
    if (g->W[RHO][c] < g->rho_floor) {
      g->W[RHO][c] = g->rho_floor;
      g->W[PR][c] = g->p_floor;
    }
    if (g->W[PR][c] < g->p_floor) g->W[PR][c] = g->p_floor;
  }
  mags_from_faces(g, g->B, g->ms, lo[0], hi[0], lo[1], hi[1], lo[2], hi[2]);
  /* time-centred field and the Alfven / Boris momentum correction
   * (src/solver_solve.c:399-484) */
  double ca2 = g->ca * g->ca;
  LOOP3(i, lo[0], hi[0], j, lo[1], hi[1], k, lo[2], hi[2]) {
    size_t c = IX(g, i, j, k);
    double mt[3];
    for (int a = 0; a < 3; a++) {
      mt[a] = 0.5 * (g->ms[a][c] + g->msp[a][c]);
      g->mt[a][c] = mt[a];
    }
    double alf = (mt[0] * mt[0] + mt[1] * mt[1] + mt[2] * mt[2]) / g->W[RHO][c] / (ca2);
    double perp = 1 / (1 + alf);
    double drho = -dt * g->dU[0][c];
    double dva = alf * drho;
    double tv[3];
    for (int a = 0; a < 3; a++)
      tv[a] = alf * (-dt * g->dU[1 + a][c] + dt * g->SH[a][c] - drho * g->v0[a][c]);
    double bdv = mt[0] * tv[0] + mt[1] * tv[1] + mt[2] * tv[2];
    bdv = bdv / (mt[0] * mt[0] + mt[1] * mt[1] + mt[2] * mt[2] + 1e-10);
    for (int a = 0; a < 3; a++) {
      g->U[1 + a][c] = g->U0[1 + a][c] +
                       perp * ((-dt * g->dU[1 + a][c] + dt * g->SH[a][c]) +
                               (-dt * g->dMF[a][c] + dt * g->SB[a][c]) + dva * g->v0[a][c] +
                               mt[a] * bdv);
    }
    for (int a = 0; a < 3; a++) g->W[V1 + a][c] = g->U[1 + a][c] / g->U[0][c];
  }
  fill_ghosts(g);
  derived(g);
  g->steps++;
}

int og_set_state(og_t *g, const double *W, const double *B, const double *Wp,
                 const double *Bp, double time, double dt0) {
  for (int m = 0; m < 6; m++) {
    memcpy(g->W[m], W + (size_t)m * g->n3, sizeof(double) * g->n3);
    if (Wp) memcpy(g->Wp[m], Wp + (size_t)m * g->n3, sizeof(double) * g->n3);
  }
  for (int a = 0; a < 3; a++) {
    memcpy(g->B[a], B + (size_t)a * g->n3, sizeof(double) * g->n3);
    if (Bp) memcpy(g->Bp[a], Bp + (size_t)a * g->n3, sizeof(double) * g->n3);
  }
  g->time = time;
  g->dt0 = dt0;
  g->steps = 0;
  return 0;
}

int og_prepare(og_t *g, int restart) {
  fill_ghosts(g);
  derived(g);
  if (restart) {
    /* mags_p of a restart is the interpolation of the stored B_p */
    mags_from_faces(g, g->Bp, g->msp, 0, g->gmax[0], 0, g->gmax[1], 0, g->gmax[2]);
    return 0;
  }
  int *gm = g->gmax;
  LOOP3(i, 0, gm[0], j, 0, gm[1], k, 0, gm[2]) {
    size_t c = IX(g, i, j, k);
    for (int m = 0; m < 6; m++) g->Wp[m][c] = g->W[m][c];
    for (int a = 0; a < 3; a++) g->msp[a][c] = g->ms[a][c];
  }
  LOOP3(i, 0, gm[0] + 1, j, 0, gm[1] + 1, k, 0, gm[2] + 1) {
    size_t c = IX(g, i, j, k);
    for (int a = 0; a < 3; a++) g->Bp[a][c] = g->B[a][c];
  }
  g->dt0 = cfl_dt(g);
  return 0;
}

int og_run(og_t *g, int nsteps) {
  for (int n = 0; n < nsteps; n++) step(g);
  return 0;
}

int og_get_state(og_t *g, double *W, double *B, double *Wp, double *Bp, double *scal) {
  for (int m = 0; m < 6; m++) {
    if (W) memcpy(W + (size_t)m * g->n3, g->W[m], sizeof(double) * g->n3);
    if (Wp) memcpy(Wp + (size_t)m * g->n3, g->Wp[m], sizeof(double) * g->n3);
  }
  for (int a = 0; a < 3; a++) {
    if (B) memcpy(B + (size_t)a * g->n3, g->B[a], sizeof(double) * g->n3);
    if (Bp) memcpy(Bp + (size_t)a * g->n3, g->Bp[a], sizeof(double) * g->n3);
  }
  if (scal) {
    scal[0] = g->time;
    scal[1] = g->dt;
    scal[2] = g->dt0;
    scal[3] = g->divb;
    scal[4] = (double)g->steps;
  }
  return 0;
}

int og_get_stage(og_t *g, double *Wh, double *Bh, double *E) {
  for (int m = 0; m < 6; m++)
    if (Wh) memcpy(Wh + (size_t)m * g->n3, g->Wh[m], sizeof(double) * g->n3);
  for (int a = 0; a < 3; a++) {
    if (Bh) memcpy(Bh + (size_t)a * g->n3, g->Bh[a], sizeof(double) * g->n3);
    if (E) memcpy(E + (size_t)a * g->n3, g->E[a], sizeof(double) * g->n3);
  }
  return 0;
}

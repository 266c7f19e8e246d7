// C ABI of the B200 MHD step (include/gamera_op.h): instance lifecycle,
// geometry / PDM-weight tables, host<->device layout conversion and the
// step sequence.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "gamera_op.h"
#include "gop_device.cuh"
#include "gop_internal.h"
#include "gop_kernels.h"

using namespace gop;

namespace {

thread_local char g_err[512] = "";

int fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

#define CK(call)                                                                  \
  do {                                                                            \
    cudaError_t e_ = (call);                                                      \
    if (e_ != cudaSuccess)                                                        \
      return fail(GOP_ECUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                  __LINE__);                                                      \
  } while (0)

// reference physics constants (src/config.c:82-90)
constexpr double kGamma = 5.0 / 3.0, kCfl = 0.3, kCa = 10.0, kPdmb = 1.0;
constexpr double kRhoFloor = 0.00316227, kPFloor = 0.000316227;

// Dense 5x5 LU with partial pivoting and solve (the scheme of
// math_lib/lu_solver.c:10-104, used by the spherical weights)
bool lu_solve5(double a[5][5], const double b[5], double x[5]) {
  int perm[5] = {0, 1, 2, 3, 4};
  for (int k = 0; k < 4; k++) {
    int piv = k;
    double best = std::fabs(a[k][k]);
    for (int i = k + 1; i < 5; i++)
      if (std::fabs(a[i][k]) > best) {
        best = std::fabs(a[i][k]);
        piv = i;
      }
    if (best < 1e-12) return false;
    if (piv != k) {
      for (int j = 0; j < 5; j++) std::swap(a[k][j], a[piv][j]);
      std::swap(perm[k], perm[piv]);
    }
    for (int i = k + 1; i < 5; i++) {
      double m = a[i][k] / a[k][k];
      a[i][k] = m;
      for (int j = k + 1; j < 5; j++) a[i][j] -= m * a[k][j];
    }
  }
  if (std::fabs(a[4][4]) < 1e-12) return false;
  double y[5];
  for (int i = 0; i < 5; i++) {
    y[i] = b[perm[i]];
    for (int j = 0; j < i; j++) y[i] -= a[i][j] * y[j];
  }
  for (int i = 4; i >= 0; i--) {
    x[i] = y[i];
    for (int j = i + 1; j < 5; j++) x[i] -= a[i][j] * x[j];
    x[i] /= a[i][i];
  }
  return true;
}

double factorial(int k) {
  double r = 1.0;
  for (int i = 2; i <= k; ++i) r *= i;
  return r;
}
double choose(int j, int k) {
  if (k < 0 || k > j) return 0.0;
  if (k == 0 || k == j) return 1.0;
  k = std::min(k, j - k);
  double r = 1.0;
  for (int i = 1; i <= k; ++i) r *= (j - k + i) / (double)i;
  return r;
}

// stride of the per-axis tables: longest axis + 1, rounded up to a multiple
// of 4 so the packed face records stay 16-byte aligned
int table_stride(const int N[3]) { return (std::max(N[0], std::max(N[1], N[2])) + 1 + 3) / 4 * 4; }

struct Tables {
  int tmax;
  std::vector<double> v;
  double& at(int axis, int t, int idx) { return v[((size_t)axis * NTAB + t) * tmax + idx]; }
};

// Per-axis geometry, mags interpolation weights, PDM weights and PDM limiter
// coefficients.  Cartesian formulas: src/cartesian/cartesian_general.c:42-358
// (the weights scale facPDMU7 by vol/vol_face; on the reference's uniform
// grid they depend on the transverse position only through round-off, so the
// tables use the first active transverse cell).  Spherical formulas:
// src/spherical/spherical_general.c:42-594.
void build_tables(const gop_desc& d, Tables& T) {
  const int n[3] = {d.ni, d.nj, d.nk};
  const double* xs[3] = {d.x1, d.x2, d.x3};
  int N[3];
  for (int a = 0; a < 3; a++) N[a] = n[a] + 2 * NGH + 1;
  T.tmax = table_stride(N);
  T.v.assign(tab_elems(T.tmax), 0.0);
  const bool sph = d.coord == GOP_COORD_SPHERICAL;
  std::vector<double> xctr[3], dxv[3], xcv[3];
  for (int a = 0; a < 3; a++) {
    const double* x = xs[a];
    dxv[a].assign(N[a], 0.0);
    xcv[a].assign(N[a], 0.0);
    xctr[a].assign(N[a], 0.0);
    for (int f = 0; f < N[a]; f++) T.at(a, T_X, f) = x[f];
    for (int c = 0; c + 1 < N[a]; c++) {
      dxv[a][c] = x[c + 1] - x[c];
      xcv[a][c] = 0.5 * (x[c] + x[c + 1]);
      T.at(a, T_DX, c) = dxv[a][c];
      double xc = xcv[a][c], dx = dxv[a][c];
      if (sph && a == 0)
        xctr[a][c] = xc + 2.0 * xc * dx * dx / (12.0 * xc * xc + dx * dx);
      else if (sph && a == 1)
        xctr[a][c] = (std::sin(x[c + 1]) - std::sin(x[c]) -
                      (x[c + 1] * std::cos(x[c + 1]) - x[c] * std::cos(x[c]))) /
                     (-std::cos(x[c + 1]) + std::cos(x[c]));
      else
        xctr[a][c] = xc;
      T.at(a, T_MA, c) = (x[c + 1] - xctr[a][c]) / dx;
      T.at(a, T_MB, c) = (xctr[a][c] - x[c]) / dx;
    }
  }
  if (sph) {
    const double* r = xs[0];
    const double* t = xs[1];
    for (int i = 0; i < N[0]; i++) {
      T.at(0, T_G0, i) = -r[i] * r[i];
      if (i + 1 < N[0]) {
        T.at(0, T_G1, i) = 1.0 / 3.0 * (std::pow(r[i + 1], 3) - std::pow(r[i], 3));
        T.at(0, T_G2, i) = 0.5 * (r[i + 1] * r[i + 1] - r[i] * r[i]);
        T.at(0, T_G3, i) = xcv[0][i];
      }
    }
    for (int j = 0; j < N[1]; j++) {
      T.at(1, T_G1, j) = std::sin(t[j]);
      if (j + 1 < N[1]) {
        T.at(1, T_G0, j) = std::cos(t[j + 1]) - std::cos(t[j]);
        T.at(1, T_G2, j) = std::sin(xcv[1][j]);
        T.at(1, T_G3, j) = std::sin(t[j + 1]) - std::sin(t[j]);
        T.at(1, T_G4, j) = std::sin(t[j + 1]) + std::sin(t[j]);
      }
    }
  }

  // PDM geometric factors GF_face / GF_vol along each axis
  auto gff = [&](int a, int f) -> double {
    if (!sph) {
      int o1 = (a + 1) % 3, o2 = (a + 2) % 3;
      int lo = std::min(o1, o2), hi = std::max(o1, o2);
      return dxv[lo][NGH] * dxv[hi][NGH];
    }
    if (a == 0) return xs[0][f] * xs[0][f];
    if (a == 1) return std::sin(xs[1][f]);
    return 1.0;
  };
  auto gfv = [&](int a, int f) -> double {
    if (!sph) {
      double v[3] = {dxv[0][NGH], dxv[1][NGH], dxv[2][NGH]};
      v[a] = dxv[a][f];
      return v[0] * v[1] * v[2];
    }
    if (a == 0) return 1.0 / 3.0 * (std::pow(xs[0][f + 1], 3) - std::pow(xs[0][f], 3));
    if (a == 1) return -(std::cos(xs[1][f + 1]) - std::cos(xs[1][f]));
    return dxv[2][f];
  };
  const double e = 1.0 / (2 * kPdmb + 1.0);
  static const double fac[7] = {-1.0 / 140.0, 5.0 / 84.0, -101.0 / 420.0, 319.0 / 420.0,
                                107.0 / 210.0, -19.0 / 210.0, 1.0 / 105.0};
  static const double f8[8] = {-3.0 / 840, 29.0 / 840, -139.0 / 840, 533.0 / 840,
                               533.0 / 840, -139.0 / 840, 29.0 / 840, -3.0 / 840};
  for (int a = 0; a < 3; a++) {
    for (int f = NGH; f <= NGH + n[a]; f++) {
      // limiter coefficients of the left (cell f-1) and right (cell f) states
      double q = gfv(a, f - 1) / dxv[a][f - 1], f0 = gff(a, f), fm = gff(a, f - 1);
      T.at(a, T_CL1, f) = (q - e * f0) / (e * f0);
      T.at(a, T_CL2, f) = (e * fm - q) / (e * f0);
      q = gfv(a, f) / dxv[a][f];
      fm = gff(a, f + 1);
      T.at(a, T_CR1, f) = (q - e * f0) / (e * f0);
      T.at(a, T_CR2, f) = (e * fm - q) / (e * f0);
      double wl[7], wr[7];
      if (!sph) {
        double vf = 0.0;
        for (int o = -4; o <= 3; o++) vf += gfv(a, f + o) * f8[o + 4];
        for (int t = 0; t < 7; t++) wl[t] = wr[t] = fac[t] * gfv(a, f) / vf;
      } else if (a == 2) {
        static const double pl[7] = {0.0, 1.0 / 30.0, -13.0 / 60.0, 47.0 / 60.0,
                                     9.0 / 20.0, -1.0 / 20.0, 0.0};
        static const double pr[7] = {0.0, -1.0 / 20.0, 9.0 / 20.0, 47.0 / 60.0,
                                     -13.0 / 60.0, 1.0 / 30.0, 0.0};
        for (int t = 0; t < 7; t++) {
          wl[t] = pl[t];
          wr[t] = pr[6 - t];  // stored w1r..w7r, applied in reverse
        }
      } else {
        // 5-point non-uniform reconstruction from cell averages: radial
        // moments of r^2 dr, polar moments of sin(theta) dtheta
        const double* x = xs[a];
        auto xs_ext = [&](int s) -> double {  // x_s[s] = x[s-4] with linear extension
          int idx = s - NGH;
          if (idx < 0) return x[0] + idx * dxv[a][0];
          if (idx > N[a] - 1) return x[N[a] - 1] + (idx - (N[a] - 1)) * dxv[a][N[a] - 2];
          return x[idx];
        };
        for (int side = 0; side < 2; side++) {
          double A[5][5], b[5], sol[5];
          for (int i = -2; i <= 2; i++) {
            double xm = side == 0 ? xs_ext(f + NGH + i - 1) : xs_ext(f + NGH + i);
            double xp = side == 0 ? xs_ext(f + NGH + i) : xs_ext(f + NGH + i + 1);
            for (int j = 0; j <= 4; j++) {
              if (a == 0) {
                const int m = 2;
                A[j][i + 2] = (double)(m + 1) / (double)(j + m + 1) *
                              (std::pow(xp, j + m + 1) - std::pow(xm, j + m + 1)) /
                              (std::pow(xp, m + 1) - std::pow(xm, m + 1));
              } else {
                double sum = 0.0;
                for (int k = 0; k <= j; k++)
                  sum = sum + factorial(k) * choose(j, k) *
                                  (std::pow(xm, j - k) * std::cos(xm + k * M_PI / 2.0) -
                                   std::pow(xp, j - k) * std::cos(xp + k * M_PI / 2.0));
                A[j][i + 2] = sum / (std::cos(xm) - std::cos(xp));
              }
            }
            b[i + 2] = std::pow(xs_ext(f + NGH), i + 2);
          }
          double wv[7] = {0, 0, 0, 0, 0, 0, 0};
          if (lu_solve5(A, b, sol))
            for (int t = 0; t < 5; t++) wv[t + 1] = sol[t];
          for (int t = 0; t < 7; t++) {
            if (side == 0) wl[t] = wv[t];
            else wr[t] = wv[6 - t];
          }
        }
      }
      for (int t = 0; t < 7; t++) {
        T.at(a, T_WL0 + t, f) = wl[t];
        T.at(a, T_WR0 + t, f) = wr[t];
      }
    }
  }
  // the same weights and coefficients packed per face (see FW)
  for (int a = 0; a < 3; a++) {
    for (int f = 0; f < T.tmax; f++) {
      double* r = T.v.data() + fw_offset(T.tmax) + ((size_t)a * T.tmax + f) * FW;
      for (int t = 0; t < 7; t++) {
        r[t] = T.at(a, T_WL0 + t, f);
        r[7 + t] = T.at(a, T_WR0 + t, f);
      }
      r[14] = T.at(a, T_CL1, f);
      r[15] = T.at(a, T_CL2, f);
      r[16] = T.at(a, T_CR1, f);
      r[17] = T.at(a, T_CR2, f);
    }
  }
}

}  // namespace

int gop::set_error(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

int gop::check_desc(const gop_desc* d) {
  if (!d) return fail(GOP_EINVAL, "desc is NULL");
  if (d->ni < NGH || d->nj < NGH || d->nk < NGH)
    return fail(GOP_EINVAL, "each axis needs at least %d active cells", NGH);
  if ((long long)d->ni * d->nj * d->nk > (1LL << 31))
    return fail(GOP_EINVAL, "grid too large");
  if (d->coord != GOP_COORD_CARTESIAN && d->coord != GOP_COORD_SPHERICAL)
    return fail(GOP_EINVAL, "coord must be GOP_COORD_CARTESIAN or GOP_COORD_SPHERICAL");
  if (!d->x1 || !d->x2 || !d->x3) return fail(GOP_EINVAL, "coordinate arrays are NULL");
  for (int a = 0; a < 3; a++) {
    char lo = d->bc[2 * a], hi = d->bc[2 * a + 1];
    // the pole fill only on the theta faces of a ring-averaged spherical grid
    const char* kinds = (a == 1 && d->ring_average) ? "psrfeno" : "psrfen";
    if (!strchr(kinds, lo) || !strchr(kinds, hi) || lo == 0 || hi == 0)
      return fail(GOP_EINVAL, "bad boundary kind on axis %d", a);
    if ((lo == 'p') != (hi == 'p'))
      return fail(GOP_EINVAL, "axis %d: periodic must be set on both faces", a);
    for (int s = 0; s < 2; s++) {
      char g = d->gem_bc[2 * a + s], b = d->bc[2 * a + s];
      if (g == 0) continue;
      if (!strchr(kinds, g)) return fail(GOP_EINVAL, "bad face-field boundary kind on axis %d", a);
      if ((g == 'p') != (b == 'p'))
        return fail(GOP_EINVAL, "axis %d: gas and face field disagree on periodicity", a);
    }
  }
  if (d->precision != GOP_PREC_FP64 && d->precision != GOP_PREC_MIXED)
    return fail(GOP_EINVAL, "precision must be GOP_PREC_FP64 or GOP_PREC_MIXED");
  if (d->ring_average) {
    RingSetup r;
    if (ring_setup(d, r) != GOP_OK) return GOP_EINVAL;
  }
  return GOP_OK;
}

// set_RingAverage_config (src/spherical/spherical_RingAverage.c:54-150) for
// one domain: the phi blocks of each ring row by nk, which poles the theta
// range reaches, the ring rows per pole
int gop::ring_setup(const gop_desc* d, RingSetup& r) {
  r = RingSetup{};
  if (d->coord != GOP_COORD_SPHERICAL) return fail(GOP_EINVAL, "the ring average needs a spherical grid");
  static const int t256[16] = {8, 16, 32, 32, 64, 64, 64, 64, 128, 128, 128, 128, 128, 128, 128, 128};
  int navr = 0;
  switch (d->nk) {
    case 256: navr = 16; break;
    case 128: navr = 8; break;
    case 64: navr = 4; break;
    case 32: navr = 2; break;
    default: return fail(GOP_EINVAL, "the ring average needs nk = 32, 64, 128 or 256");
  }
  for (int t = 0; t < navr; t++) r.nchunk[t] = t256[t];
  if (d->bc[4] != 'p') return fail(GOP_EINVAL, "the ring average needs periodic k faces");
  const double pi = 3.14159265358979323846;
  if (fabs(d->x2[NGH]) < 1e-10) r.poles |= 1;
  if (fabs(d->x2[NGH + d->nj] - pi) < 1e-10) r.poles |= 2;
  r.jmax = d->nj - 1 < navr ? d->nj - 1 : navr - 1;
  // the bands of the two poles (E rows jmax + 2 deep) must not meet
  const int need = (r.poles == 3 ? 2 : 1) * (r.jmax + 2) + 1;
  if (r.poles && d->nj < need)
    return fail(GOP_EINVAL, "the ring average needs nj >= %d here", need);
  return GOP_OK;
}

namespace {

struct Layout {
  int N[3];
  int pitch;
  long long fs;
};

Layout layout_of(const gop_desc* d) {
  Layout L;
  L.N[0] = d->ni + 2 * NGH + 1;
  L.N[1] = d->nj + 2 * NGH + 1;
  L.N[2] = d->nk + 2 * NGH + 1;
  L.pitch = (L.N[0] + 7) / 8 * 8;
  L.fs = (long long)L.pitch * L.N[1] * L.N[2];
  return L;
}

}  // namespace

struct gop_instance {
  gop_desc d;
  Params P;
  cudaStream_t own = nullptr;  // the instance's own non-blocking stream
  cudaStream_t st = nullptr;   // where its work goes (own, or the caller's)
  double* state = nullptr;   // 2 x (6 + 3) fields
  void* work = nullptr;      // WORK_FIELDS x R
  double* tab = nullptr;
  float* tabf = nullptr;     // FP32 copy of the tables (mixed path)
  double* scal = nullptr;
  double* staging = nullptr; // reference-layout scratch, 6 x NI*NJ*NK
  double* bg = nullptr;      // background field block (BG_NF fields), if set
  double* ringtab = nullptr; // pole ring average tables (Params::ringtab)
  double* hscal = nullptr;   // host copy of the scalars
  Work<double> wd;
  Work<float> wf;
  Tune tune;
  SweepSet* sweep = nullptr;  // tensor maps of the tile-staged flux sweeps
  cudaGraphExec_t step_graph = nullptr;  // one captured step (replayed by gop_step)
  uint64_t gen = 0;                      // bumped whenever a step's launches change
  int64_t step_nodes = 0;
  size_t bytes = 0;
  bool prepared = false;
  bool fresh = false;  // prepared without restart and not stepped: history == state
  // per-kernel-group event timing (gop_set_profiling)
  bool prof = false;
  std::vector<cudaEvent_t> pool;
  struct Rec {
    int group;
    cudaEvent_t a, b;
  };
  std::vector<Rec> recs;
  cudaEvent_t open_ev[NGROUP] = {};
  double prof_ms[NGROUP] = {};
  int64_t prof_n[NGROUP] = {};
};

// the background block (BG_NF fields of doubles), allocated at first use and
// zeroed
static int alloc_background(gop_instance* h) {
  const Params& P = h->P;
  if (!h->bg) {
    cudaError_t e = cudaMallocAsync((void**)&h->bg, (size_t)P.fs * BG_NF * sizeof(double), h->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
    if (e != cudaSuccess) {
      cudaGetLastError();
      h->bg = nullptr;
      return fail(GOP_ENOMEM, "background allocation failed: %s", cudaGetErrorString(e));
    }
    h->bytes += (size_t)P.fs * BG_NF * sizeof(double);
  }
  CK(cudaMemsetAsync(h->bg, 0, (size_t)P.fs * BG_NF * sizeof(double), h->st));
  return GOP_OK;
}

static cudaEvent_t take_event(gop_instance* h) {
  cudaEvent_t e = nullptr;
  if (!h->pool.empty()) {
    e = h->pool.back();
    h->pool.pop_back();
  } else {
    cudaEventCreate(&e);
  }
  return e;
}

static void prof_mark(void* ctx, int group, int start) {
  gop_instance* h = (gop_instance*)ctx;
  cudaEvent_t e = take_event(h);
  cudaEventRecord(e, h->st);
  if (start) {
    h->open_ev[group] = e;
  } else {
    h->recs.push_back({group, h->open_ev[group], e});
    h->open_ev[group] = nullptr;
  }
}

static void prof_collect(gop_instance* h) {
  for (auto& r : h->recs) {
    float ms = 0.f;
    if (cudaEventSynchronize(r.b) == cudaSuccess && cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
      h->prof_ms[r.group] += ms;
      h->prof_n[r.group] += 1;
    }
    h->pool.push_back(r.a);
    h->pool.push_back(r.b);
  }
  h->recs.clear();
}

// the launches of one step changed (kernel set, block shapes): the captured
// step goes, and batches holding this instance capture theirs again
static void drop_step_graph(gop_instance* h) {
  if (h->step_graph) cudaGraphExecDestroy(h->step_graph);
  h->step_graph = nullptr;
  h->gen++;
}

extern "C" {

const char* gop_last_error(void) { return g_err; }

int64_t gop_kernel_launches(void) { return gop::launches(); }

size_t gop_footprint(const gop_desc* d) {
  if (check_desc(d) != GOP_OK) return 0;
  Layout L = layout_of(d);
  size_t rsize = d->precision == GOP_PREC_MIXED ? sizeof(float) : sizeof(double);
  size_t ref = (size_t)L.N[0] * L.N[1] * L.N[2];
  const size_t tab = tab_elems(table_stride(L.N));
  const bool mixed = d->precision == GOP_PREC_MIXED;
  return (size_t)L.fs * (18 * sizeof(double) + work_fields(mixed) * rsize) +
         6 * ref * sizeof(double) + tab * (sizeof(double) + (mixed ? sizeof(float) : 0)) +
         NSCAL * sizeof(double);
}

int gop_create(const gop_desc* desc, gop_instance** out) {
  if (!out) return fail(GOP_EINVAL, "out is NULL");
  *out = nullptr;
  int rc = check_desc(desc);
  if (rc) return rc;
  int dev = 0, count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
    return fail(GOP_ENODEV, "no CUDA device");
  CK(cudaGetDevice(&dev));
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, dev));
  if (prop.major < 10) return fail(GOP_ENODEV, "device is sm_%d%d; sm_100 required", prop.major, prop.minor);

  gop_instance* h = new (std::nothrow) gop_instance();
  if (!h) return fail(GOP_ENOMEM, "host allocation failed");
  h->d = *desc;
  gop_desc& d = h->d;
  for (int f = 0; f < 6; f++)
    if (d.gem_bc[f] == 0) d.gem_bc[f] = d.bc[f];
  if (d.gamma == 0) d.gamma = kGamma;
  if (d.cfl == 0) d.cfl = kCfl;
  if (d.ca == 0) d.ca = kCa;
  if (d.rho_floor == 0) d.rho_floor = kRhoFloor;
  if (d.p_floor == 0) d.p_floor = kPFloor;

  Tables T;
  build_tables(d, T);
  Layout L = layout_of(&d);
  Params& P = h->P;
  P.n[0] = d.ni;
  P.n[1] = d.nj;
  P.n[2] = d.nk;
  for (int a = 0; a < 3; a++) P.N[a] = L.N[a];
  P.pitch = L.pitch;
  P.coord = d.coord;
  P.sj = L.pitch;
  P.sk = (long long)L.pitch * L.N[1];
  P.fs = L.fs;
  P.tmax = T.tmax;
  P.gamma = d.gamma;
  P.gm1 = d.gamma - 1.0;
  P.cfl = d.cfl;
  P.ca = d.ca;
  P.ca2 = d.ca * d.ca;
  P.rho_floor = d.rho_floor;
  P.p_floor = d.p_floor;
  P.pdm_a1 = kPdmb / (kPdmb + 1.0);
  P.pdm_a2 = 1.0 - P.pdm_a1;
  P.inv_gm1 = 1.0 / P.gm1;
  P.q_ca = 0.25 / d.ca;

  size_t rsize = d.precision == GOP_PREC_MIXED ? sizeof(float) : sizeof(double);
  size_t ref = (size_t)L.N[0] * L.N[1] * L.N[2];
  // Every instance works on its own non-blocking stream with stream-ordered
  // allocations, so creating, using and destroying one instance never waits
  // for another instance or a batch (the legacy default stream would).
  cudaError_t e = cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking);
  h->st = h->own;
  auto alloc = [&](void** p, size_t bytes) {
    if (e == cudaSuccess) {
      e = cudaMallocAsync(p, bytes, h->st);
      if (e == cudaSuccess) h->bytes += bytes;
    }
  };
  const bool mixed = d.precision == GOP_PREC_MIXED;
  const int nwork = work_fields(mixed);
  alloc((void**)&h->state, (size_t)L.fs * 18 * sizeof(double));
  alloc(&h->work, (size_t)L.fs * nwork * rsize);
  alloc((void**)&h->tab, T.v.size() * sizeof(double));
  if (mixed) alloc((void**)&h->tabf, T.v.size() * sizeof(float));
  alloc((void**)&h->scal, NSCAL * sizeof(double));
  alloc((void**)&h->staging, 6 * ref * sizeof(double));
  if (e == cudaSuccess) {
    h->hscal = new (std::nothrow) double[NSCAL];
    if (!h->hscal) e = cudaErrorMemoryAllocation;
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
  if (e != cudaSuccess) {
    cudaGetLastError();
    gop_destroy(h);
    return fail(GOP_ENOMEM, "device allocation of %zu bytes failed: %s", gop_footprint(&d),
                cudaGetErrorString(e));
  }
  cudaMemsetAsync(h->state, 0, (size_t)L.fs * 18 * sizeof(double), h->st);
  cudaMemsetAsync(h->work, 0, (size_t)L.fs * nwork * rsize, h->st);
  cudaMemcpyAsync(h->tab, T.v.data(), T.v.size() * sizeof(double), cudaMemcpyHostToDevice, h->st);
  std::vector<float> tf;
  if (mixed) {
    tf.assign(T.v.begin(), T.v.end());
    cudaMemcpyAsync(h->tabf, tf.data(), tf.size() * sizeof(float), cudaMemcpyHostToDevice, h->st);
  }
  cudaMemsetAsync(h->scal, 0, NSCAL * sizeof(double), h->st);
  P.tab = h->tab;
  P.scal = h->scal;
  P.Wbuf[0] = h->state;
  P.Bbuf[0] = h->state + 6 * L.fs;
  P.Wbuf[1] = h->state + 9 * L.fs;
  P.Bbuf[1] = h->state + 15 * L.fs;
  if (d.precision == GOP_PREC_MIXED) {
    float* w = (float*)h->work;
    h->wf = Work<float>{w, w + 6 * L.fs, w + 9 * L.fs, w + 12 * L.fs, w + 15 * L.fs,
                        w + 21 * L.fs, w + 24 * L.fs, w + 51 * L.fs, w + 57 * L.fs, h->tabf,
                        h->tabf + fw_offset(T.tmax)};
  } else {
    double* w = (double*)h->work;
    h->wd = Work<double>{w, w + 6 * L.fs, w + 9 * L.fs, w + 12 * L.fs, w + 15 * L.fs,
                         w + 21 * L.fs, w + 24 * L.fs, nullptr, nullptr, h->tab,
                         h->tab + fw_offset(T.tmax)};
  }
  P.ring = 0;
  P.ps_live = 1;  // until gop_prepare has looked
  if (d.ring_average) {
    RingSetup r;
    ring_setup(&d, r);  // validated by check_desc
    const int nk = d.nk, n1 = L.N[1];
    std::vector<double> rt(2 * nk + n1, 1.0);
    const double pi = 3.14159265358979323846, dtheta = 2.0 * pi / nk;
    for (int q = 0; q < nk; q++) {  // FilterBaseMode's phi angles
      const double theta = dtheta * (q + 0.5);
      rt[q] = std::cos(theta);
      rt[nk + q] = std::sin(theta);
    }
    // dxk_ring = (nk / nchunk) dxk on the ring rows, negative pole last
    for (int rr = 0; rr <= r.jmax; rr++) {
      if (r.poles & 1) rt[2 * nk + NGH + rr] = (double)(nk / r.nchunk[rr]);
      if (r.poles & 2) rt[2 * nk + NGH + d.nj - 1 - rr] = (double)(nk / r.nchunk[rr]);
    }
    alloc((void**)&h->ringtab, rt.size() * sizeof(double));
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(h->ringtab, rt.data(), rt.size() * sizeof(double), cudaMemcpyHostToDevice, h->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
    P.ring = r.poles;
    P.ring_jmax = r.jmax;
    for (int t = 0; t < 16; t++) P.nchunk[t] = r.nchunk[t];
    P.ringtab = h->ringtab;
  }
  // the tile-staged flux sweeps read the work and state arrays through
  // tensor maps made once here; without them the per-face kernels run
  h->sweep = mixed ? sweep_create<float>(P, h->wf) : sweep_create<double>(P, h->wd);
  // FP32 edge EMFs: the per-edge kernel measured faster on B200 (blast 256^3:
  // 1.09 vs 1.26 ms per step), FP64 the sweep (2.06 vs 2.25 ms); the
  // autotuner decides per launch
  if (mixed)
    for (int d = 0; d < 3; d++) h->tune.emf_sweep[d] = false;
  cudaError_t le = e != cudaSuccess ? e : cudaStreamSynchronize(h->st);
  if (le == cudaSuccess) le = cudaGetLastError();
  if (le != cudaSuccess) {
    gop_destroy(h);
    return fail(GOP_ECUDA, "initialisation failed: %s", cudaGetErrorString(le));
  }
  *out = h;
  return GOP_OK;
}

int gop_destroy(gop_instance* h) {
  if (!h) return GOP_OK;
  if (h->st) cudaStreamSynchronize(h->st);
  drop_step_graph(h);
  for (void* p : {(void*)h->state, h->work, (void*)h->tab, (void*)h->tabf, (void*)h->scal,
                  (void*)h->staging, (void*)h->bg, (void*)h->ringtab})
    if (p) cudaFreeAsync(p, h->st);
  if (h->own) cudaStreamDestroy(h->own);  // released once the frees have run
  sweep_destroy(h->sweep);
  delete[] h->hscal;
  prof_collect(h);
  for (cudaEvent_t e : h->pool) cudaEventDestroy(e);
  delete h;
  return GOP_OK;
}

int gop_set_stream(gop_instance* h, void* stream) {
  if (!h) return fail(GOP_EINVAL, "instance is NULL");
  CK(cudaStreamSynchronize(h->st));
  h->st = stream ? (cudaStream_t)stream : h->own;
  return GOP_OK;
}

int gop_upload(gop_instance* h, const double* gas, const double* face_b, const double* gas_p,
               const double* face_b_p, double time, double dt0) {
  if (!h || !gas || !face_b) return fail(GOP_EINVAL, "NULL argument");
  if ((gas_p == nullptr) != (face_b_p == nullptr))
    return fail(GOP_EINVAL, "gas_p and face_b_p go together");
  const Params& P = h->P;
  size_t ref = (size_t)P.N[0] * P.N[1] * P.N[2];
  // the current state goes to buffer 0, the history to buffer 1
  CK(cudaMemcpyAsync(h->staging, gas, 6 * ref * sizeof(double), cudaMemcpyHostToDevice, h->st));
  launch_from_ref(P, 6, h->staging, P.Wbuf[0], h->st);
  CK(cudaMemcpyAsync(h->staging, face_b, 3 * ref * sizeof(double), cudaMemcpyHostToDevice, h->st));
  launch_from_ref(P, 3, h->staging, P.Bbuf[0], h->st);
  if (gas_p) {
    CK(cudaMemcpyAsync(h->staging, gas_p, 6 * ref * sizeof(double), cudaMemcpyHostToDevice, h->st));
    launch_from_ref(P, 6, h->staging, P.Wbuf[1], h->st);
    CK(cudaMemcpyAsync(h->staging, face_b_p, 3 * ref * sizeof(double), cudaMemcpyHostToDevice, h->st));
    launch_from_ref(P, 3, h->staging, P.Bbuf[1], h->st);
  }
  double* s = h->hscal;
  CK(cudaStreamSynchronize(h->st));
  for (int t = 0; t < NSCAL; t++) s[t] = 0.0;
  s[S_TIME] = time;
  s[S_DT0] = dt0;
  s[S_PAR] = 0.0;
  CK(cudaMemcpyAsync(h->scal, s, NSCAL * sizeof(double), cudaMemcpyHostToDevice, h->st));
  CK(cudaStreamSynchronize(h->st));
  h->prepared = false;
  return GOP_OK;
}

int gop_set_background(gop_instance* h, const double* b0, const double* lorentz,
                       const double* b0_face, const double* b0_edge) {
  if (!h) return fail(GOP_EINVAL, "instance is NULL");
  const int given = (b0 != nullptr) + (lorentz != nullptr) + (b0_face != nullptr) + (b0_edge != nullptr);
  if (given != 0 && given != 4) return fail(GOP_EINVAL, "the four background arrays go together");
  Params& P = h->P;
  drop_step_graph(h);  // the captured step has the other kernel set
  h->prepared = false;
  if (given == 0) {
    if (h->bg) cudaFreeAsync(h->bg, h->st);
    h->bg = nullptr;
    P.bg = nullptr;
    CK(cudaStreamSynchronize(h->st));
    return GOP_OK;
  }
  int rc = alloc_background(h);
  if (rc) return rc;
  const size_t ref = (size_t)P.N[0] * P.N[1] * P.N[2];
  // through the staging buffer (6 fields) in groups of 3
  const double* src[8] = {b0, lorentz, b0_face, b0_face + 3 * ref, b0_face + 6 * ref,
                          b0_edge, b0_edge + 3 * ref, b0_edge + 6 * ref};
  const int dst[8] = {BG_B0, BG_LOR, BG_FACE, BG_FACE + 3, BG_FACE + 6,
                      BG_EDGE, BG_EDGE + 3, BG_EDGE + 6};
  for (int g = 0; g < 8; g++) {
    CK(cudaMemcpyAsync(h->staging, src[g], 3 * ref * sizeof(double), cudaMemcpyHostToDevice, h->st));
    launch_from_ref(P, 3, h->staging, h->bg + (size_t)dst[g] * P.fs, h->st);
  }
  CK(cudaStreamSynchronize(h->st));
  CK(cudaGetLastError());
  P.bg = h->bg;
  return GOP_OK;
}

int gop_set_background_device(gop_instance* h, const gop_background* bg) {
  if (!h || !bg) return fail(GOP_EINVAL, "NULL argument");
  if (bg->kind != GOP_BG_UNIFORM && bg->kind != GOP_BG_DIPOLE)
    return fail(GOP_EINVAL, "unknown background kind %d", bg->kind);
  Params& P = h->P;
  drop_step_graph(h);  // the captured step has the other kernel set
  h->prepared = false;
  int rc = alloc_background(h);
  if (rc) return rc;
  // the work arrays (>= 12 fields of doubles) are free until gop_prepare
  launch_background(P, *bg, h->d.coord == GOP_COORD_SPHERICAL ? 1 : 0, h->bg, (double*)h->work,
                    h->st);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(h->st));
  P.bg = h->bg;
  return GOP_OK;
}

int gop_get_background(gop_instance* h, double* b0, double* lorentz, double* b0_face,
                       double* b0_edge) {
  if (!h) return fail(GOP_EINVAL, "instance is NULL");
  if (!h->bg) return fail(GOP_ESTATE, "the instance has no background field");
  const Params& P = h->P;
  const size_t ref = (size_t)P.N[0] * P.N[1] * P.N[2];
  double* dst[8] = {b0, lorentz, b0_face, b0_face ? b0_face + 3 * ref : nullptr,
                    b0_face ? b0_face + 6 * ref : nullptr, b0_edge,
                    b0_edge ? b0_edge + 3 * ref : nullptr, b0_edge ? b0_edge + 6 * ref : nullptr};
  const int src[8] = {BG_B0, BG_LOR, BG_FACE, BG_FACE + 3, BG_FACE + 6,
                      BG_EDGE, BG_EDGE + 3, BG_EDGE + 6};
  for (int g = 0; g < 8; g++) {
    if (!dst[g]) continue;
    launch_to_ref(P, 3, h->bg + (size_t)src[g] * P.fs, h->staging, h->st);
    CK(cudaMemcpyAsync(dst[g], h->staging, 3 * ref * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  }
  CK(cudaStreamSynchronize(h->st));
  return GOP_OK;
}

int gop_problem_init_device(gop_instance* h, const gop_problem* p) {
  if (!h || !p) return fail(GOP_EINVAL, "NULL argument");
  const bool sph = h->d.coord == GOP_COORD_SPHERICAL;
  switch (p->kind) {
    case GOP_PROBLEM_OT:
    case GOP_PROBLEM_BLAST:
    case GOP_PROBLEM_LOOP_CART:
      if (sph) return fail(GOP_EINVAL, "problem %d needs a Cartesian grid", p->kind);
      break;
    case GOP_PROBLEM_LOOP_SPH:
      if (!sph) return fail(GOP_EINVAL, "problem %d needs a spherical grid", p->kind);
      break;
    default:
      return fail(GOP_EINVAL, "unknown problem kind %d", p->kind);
  }
  const Params& P = h->P;
  // the state goes to buffer 0 (as gop_upload puts it), zero where the
  // problem leaves it; the work arrays (>= 3 fields of doubles) are free
  // until gop_prepare and hold the edge integrals
  CK(cudaMemsetAsync(P.Wbuf[0], 0, (size_t)P.fs * 6 * sizeof(double), h->st));
  CK(cudaMemsetAsync(P.Bbuf[0], 0, (size_t)P.fs * 3 * sizeof(double), h->st));
  launch_problem_init(P, *p, sph ? 1 : 0, (double*)h->work, h->st);
  CK(cudaGetLastError());
  double* s = h->hscal;
  CK(cudaStreamSynchronize(h->st));
  for (int t = 0; t < NSCAL; t++) s[t] = 0.0;
  CK(cudaMemcpyAsync(h->scal, s, NSCAL * sizeof(double), cudaMemcpyHostToDevice, h->st));
  CK(cudaStreamSynchronize(h->st));
  h->prepared = false;
  return GOP_OK;
}

int gop_prepare(gop_instance* h, int restart) {
  if (!h) return fail(GOP_EINVAL, "instance is NULL");
  const Params& P = h->P;
  // halo + boundary fill of the current state (src/solver_solve.c:25-40),
  // every field: the state may be new
  Params Pall = P;
  Pall.ps_live = 1;
  launch_ghosts(Pall, h->d.bc, h->d.gem_bc, 1, h->st);
  if (!restart) {
    // AB2 history <- current state (src/solver_solve.c:55-92)
    CK(cudaMemcpyAsync(P.Wbuf[1], P.Wbuf[0], (size_t)P.fs * 6 * sizeof(double),
                       cudaMemcpyDeviceToDevice, h->st));
    CK(cudaMemcpyAsync(P.Bbuf[1], P.Bbuf[0], (size_t)P.fs * 3 * sizeof(double),
                       cudaMemcpyDeviceToDevice, h->st));
  }
  double* s = h->hscal;
  CK(cudaMemcpyAsync(s, h->scal, NSCAL * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  s[S_NEXT_DT] = DBL_MAX;
  s[S_DIVB] = 0.0;
  s[S_STOP] = 0.0;
  s[S_STEPS] = 0.0;
  s[S_FLAGS] = 0.0;
  s[S_PAR] = 0.0;
  s[S_PSNZ] = 0.0;
  CK(cudaMemcpyAsync(h->scal, s, NSCAL * sizeof(double), cudaMemcpyHostToDevice, h->st));
  // CFL dt and div B of the initial state (src/solver_solve.c:94-98)
  launch_dt(P, h->d.coord, h->d.precision == GOP_PREC_MIXED, h->st);
  // is the entropy channel live?  A p_S that is zero in the state and its
  // history stays zero in every later step, and the flux kernels skip it
  launch_ps_check(P, h->st);
  CK(cudaMemcpyAsync(s, h->scal, NSCAL * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  const int live = s[S_PSNZ] != 0.0 ? 1 : 0;
  if (live != h->P.ps_live) {
    drop_step_graph(h);
    h->P.ps_live = live;
  }
  if (!restart) s[S_DT0] = s[S_NEXT_DT];
  CK(cudaMemcpyAsync(h->scal, s, NSCAL * sizeof(double), cudaMemcpyHostToDevice, h->st));
  CK(cudaStreamSynchronize(h->st));
  CK(cudaGetLastError());
  if (!(s[S_NEXT_DT] > 0.0) || s[S_NEXT_DT] >= DBL_MAX)
    return fail(GOP_ENUMERIC, "initial CFL dt is not positive (%g)", s[S_NEXT_DT]);
  h->prepared = true;
  h->fresh = !restart;
  return GOP_OK;
}

}  // extern "C"

// thread-block shapes the autotuners choose from (at most 256 threads)
static const dim3 kBlockCandidates[] = {dim3(32, 4, 2), dim3(32, 8, 1), dim3(32, 1, 8),
                                        dim3(32, 2, 4),  dim3(64, 2, 2), dim3(64, 4, 1),
                                        dim3(64, 1, 4),  dim3(128, 2, 1), dim3(128, 1, 2),
                                        dim3(32, 4, 1),  dim3(64, 2, 1), dim3(256, 1, 1),
                                        dim3(8, 32, 1),  dim3(8, 4, 8)};
static const int kNumBlockCandidates = sizeof(kBlockCandidates) / sizeof(kBlockCandidates[0]);

// one step's launches: begin, the stages, the ghost fill, end
static void enqueue_one_step(gop_instance* h, cudaStream_t st, const Hook& hook) {
  const Params& P = h->P;
  hook(G_BEGIN, 1);
  launch_begin(P, st);
  hook(G_BEGIN, 0);
  if (h->d.precision == GOP_PREC_MIXED)
    launch_step_body<float>(P, h->d.coord, h->wf, st, h->tune, h->sweep, hook);
  else
    launch_step_body<double>(P, h->d.coord, h->wd, st, h->tune, h->sweep, hook);
  hook(G_GHOST, 1);
  launch_ghosts(P, h->d.bc, h->d.gem_bc, 0, st);
  hook(G_GHOST, 0);
  hook(G_END, 1);
  launch_end(P, st);
  hook(G_END, 0);
}

// Captures one step as a CUDA graph: every launch reads dt, the AB2
// coefficient, the buffer parity and the stop flag from device memory, so
// the same graph replays every step.
static int capture_step(gop_instance* h) {
  if (h->step_graph) return GOP_OK;
  CK(cudaStreamSynchronize(h->own));
  cudaGraph_t g = nullptr;
  const int64_t before = launches();
  CK(cudaStreamBeginCapture(h->own, cudaStreamCaptureModeThreadLocal));
  enqueue_one_step(h, h->own, Hook());
  cudaError_t e = cudaStreamEndCapture(h->own, &g);
  h->step_nodes = launches() - before;
  count_launches(-h->step_nodes);  // counted when replayed
  if (e == cudaSuccess) e = cudaGraphInstantiate(&h->step_graph, g, 0);
  if (g) cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    h->step_graph = nullptr;
    return fail(GOP_ECUDA, "step graph capture failed: %s", cudaGetErrorString(e));
  }
  return GOP_OK;
}

// steps between looks at the stop flag when gop_step runs to a stop time
static const int kStopCheck = 256;

static int enqueue_steps(gop_instance* h, int nsteps, double time_stop) {
  const Params& P = h->P;
  if (nsteps > 0) h->fresh = false;
  Hook hook;
  if (h->prof) {
    hook.mark = prof_mark;
    hook.ctx = h;
  }
  launch_arm(P, time_stop, (double)nsteps, h->st);
  // inside a caller's stream capture the launches go straight into it
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  CK(cudaStreamIsCapturing(h->st, &cap));
  if (!h->prof && nsteps >= 1 && cap == cudaStreamCaptureStatusNone) {  // replay the captured step
    int rc = capture_step(h);
    if (rc) return rc;
    // with a stop time and many steps, look at the stop flag between
    // chunks instead of queueing steps that would all return at once
    const bool check = time_stop < 1e299 && nsteps > kStopCheck;
    for (int n = 0; n < nsteps; n++) {
      CK(cudaGraphLaunch(h->step_graph, h->st));
      count_launches(h->step_nodes);
      if (check && (n + 1) % kStopCheck == 0) {
        CK(cudaMemcpyAsync(h->hscal, h->scal, NSCAL * sizeof(double), cudaMemcpyDeviceToHost, h->st));
        CK(cudaStreamSynchronize(h->st));
        if (h->hscal[S_STOP] != 0.0) break;
      }
    }
    CK(cudaGetLastError());
    return GOP_OK;
  }
  for (int n = 0; n < nsteps; n++) enqueue_one_step(h, h->st, hook);
  CK(cudaGetLastError());
  return GOP_OK;
}

extern "C" {

int gop_step(gop_instance* h, int nsteps, double time_stop, double* time_out) {
  if (!h) return fail(GOP_EINVAL, "instance is NULL");
  if (!h->prepared) return fail(GOP_ESTATE, "gop_prepare must run before gop_step");
  if (nsteps < 0) return fail(GOP_EINVAL, "nsteps < 0");
  int rc = enqueue_steps(h, nsteps, time_stop);
  if (rc) return rc;
  if (time_out) {
    CK(cudaMemcpyAsync(h->hscal, h->scal, NSCAL * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    *time_out = h->hscal[S_TIME];
    if (h->hscal[S_FLAGS] == 2.0)
      return fail(GOP_ECUDA, "a tile pipeline wait on the device timed out");
    if (h->hscal[S_FLAGS] != 0.0) return fail(GOP_ENUMERIC, "non-finite or non-positive state");
  }
  return GOP_OK;
}

}  // extern "C"

static int download_field(gop_instance* h, int nf, const double* dev, double* host) {
  const Params& P = h->P;
  size_t ref = (size_t)P.N[0] * P.N[1] * P.N[2];
  launch_to_ref(P, nf, dev, h->staging, h->st);
  CK(cudaMemcpyAsync(host, h->staging, nf * ref * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  return GOP_OK;
}

template <typename R>
static int download_work(gop_instance* h, int nf, const R* dev, double* host) {
  // widen the FP32 work array into a temporary FP64 array first
  const Params& P = h->P;
  double* tmp = nullptr;
  CK(cudaMallocAsync((void**)&tmp, (size_t)P.fs * nf * sizeof(double), h->st));
  launch_widen<R>(P, nf, dev, tmp, h->st);
  int rc = download_field(h, nf, tmp, host);
  cudaFreeAsync(tmp, h->st);
  CK(cudaStreamSynchronize(h->st));
  return rc;
}

extern "C" {

int gop_download(gop_instance* h, double* gas, double* face_b, double* gas_h, double* gas_p,
                 double* face_b_h, double* face_b_p, double* mags, double* mags_h,
                 double* mags_p) {
  if (!h) return fail(GOP_EINVAL, "instance is NULL");
  const Params& P = h->P;
  double* s = h->hscal;
  CK(cudaMemcpyAsync(s, h->scal, NSCAL * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  int cur = s[S_PAR] != 0.0 ? 1 : 0;
  int rc = GOP_OK;
  if (gas && (rc = download_field(h, 6, P.Wbuf[cur], gas))) return rc;
  if (face_b && (rc = download_field(h, 3, P.Bbuf[cur], face_b))) return rc;
  if (gas_p && (rc = download_field(h, 6, P.Wbuf[1 - cur], gas_p))) return rc;
  if (face_b_p && (rc = download_field(h, 3, P.Bbuf[1 - cur], face_b_p))) return rc;
  if (mags) {
    double* tmp = nullptr;
    CK(cudaMallocAsync((void**)&tmp, (size_t)P.fs * 3 * sizeof(double), h->st));
    CK(cudaMemsetAsync(tmp, 0, (size_t)P.fs * 3 * sizeof(double), h->st));
    launch_mags(P, P.Bbuf[cur], tmp, h->st);
    rc = download_field(h, 3, tmp, mags);
    cudaFreeAsync(tmp, h->st);
    if (rc) return rc;
  }
  bool mixed = h->d.precision == GOP_PREC_MIXED;
  if (gas_h) rc = mixed ? download_work<float>(h, 6, h->wf.Wh, gas_h) : download_field(h, 6, h->wd.Wh, gas_h);
  if (rc) return rc;
  if (face_b_h) rc = mixed ? download_work<float>(h, 3, h->wf.Bh, face_b_h) : download_field(h, 3, h->wd.Bh, face_b_h);
  if (rc) return rc;
  if (mags_h) rc = mixed ? download_work<float>(h, 3, h->wf.Msh, mags_h) : download_field(h, 3, h->wd.Msh, mags_h);
  if (rc) return rc;
  if (mags_p) rc = mixed ? download_work<float>(h, 3, h->wf.Ms, mags_p) : download_field(h, 3, h->wd.Ms, mags_p);
  CK(cudaGetLastError());
  return rc;
}

// Project-written autotuner: for each tunable kernel, time a set of block
// shapes on the instance's current state (these kernels are pure functions of
// the current buffers, so re-running them does not change the state) and
// keep the fastest.  The prepared state must be valid (after gop_prepare).
int gop_autotune(gop_instance* h, int reps, int* chosen) {
  if (!h) return fail(GOP_EINVAL, "instance is NULL");
  if (!h->prepared) return fail(GOP_ESTATE, "gop_prepare must run before gop_autotune");
  if (reps <= 0) reps = 3;
  const dim3* cand = kBlockCandidates;
  const int ncand = kNumBlockCandidates;
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  // k_update writes the next state into the history buffers: keep a copy of
  // them and of the device scalars, and put both back afterwards
  const Params& P = h->P;
  int cur = 0;
  CK(cudaMemcpyAsync(h->hscal, h->scal, NSCAL * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  std::vector<double> saved_scal(h->hscal, h->hscal + NSCAL);
  cur = saved_scal[S_PAR] != 0.0 ? 1 : 0;
  double* hist = nullptr;
  const size_t wbytes = (size_t)P.fs * 6 * sizeof(double), bbytes = (size_t)P.fs * 3 * sizeof(double);
  CK(cudaMallocAsync((void**)&hist, wbytes + bbytes, h->st));
  CK(cudaMemcpyAsync(hist, P.Wbuf[1 - cur], wbytes, cudaMemcpyDeviceToDevice, h->st));
  CK(cudaMemcpyAsync(hist + 6 * P.fs, P.Bbuf[1 - cur], bbytes, cudaMemcpyDeviceToDevice, h->st));
  const bool mixed = h->d.precision == GOP_PREC_MIXED;
  for (int slot = 0; slot < NTUNE; slot++) {
    float best = 1e30f;
    int best_c = 0;
    // the flux and EMF slots also try the tile-staged sweep kernel
    // (candidate ncand)
    const bool flux = slot >= K_FLUX0 && slot <= K_FLUX2;
    const bool emf = slot >= K_EMF0 && slot <= K_EMF2;
    const bool try_sweep = h->sweep && (emf || (flux && !P.ps_live));
    for (int c = 0; c < ncand + (try_sweep ? 1 : 0); c++) {
      const bool sw = c == ncand;
      if (!sw && cand[c].x * cand[c].y * cand[c].z > 256) continue;
      const dim3 blk = sw ? h->tune.blk[slot] : cand[c];
      // warm-up launch, then reps timed launches
      for (int r = 0; r <= reps; r++) {
        if (r == 1) cudaEventRecord(a, h->st);
        if (mixed) launch_slot<float>(h->P, h->d.coord, h->wf, slot, blk, h->st, sw ? h->sweep : nullptr);
        else launch_slot<double>(h->P, h->d.coord, h->wd, slot, blk, h->st, sw ? h->sweep : nullptr);
      }
      cudaEventRecord(b, h->st);
      CK(cudaEventSynchronize(b));
      float ms = 0.f;
      cudaEventElapsedTime(&ms, a, b);
      if (ms < best) {
        best = ms;
        best_c = c;
      }
    }
    if (best_c < ncand) h->tune.blk[slot] = cand[best_c];
    if (flux) h->tune.flux_sweep[slot - K_FLUX0] = best_c == ncand;
    if (emf) h->tune.emf_sweep[slot - K_EMF0] = best_c == ncand;
    if (chosen) chosen[slot] = best_c;
    drop_step_graph(h);  // the captured step has the old shapes
  }
  // The order of the three flux launches and of the three EMF launches
  // (independent launches: the order changes no result, only what L2 holds
  // from one launch to the next): two whole steps timed per rotation of
  // each, the whole state and its scalars restored after every trial.
  for (int t = 0; t < NSCAL; t++) h->hscal[t] = saved_scal[t];
  CK(cudaMemcpyAsync(h->scal, h->hscal, NSCAL * sizeof(double), cudaMemcpyHostToDevice, h->st));
  CK(cudaMemcpyAsync(P.Wbuf[1 - cur], hist, wbytes, cudaMemcpyDeviceToDevice, h->st));
  CK(cudaMemcpyAsync(P.Bbuf[1 - cur], hist + 6 * P.fs, bbytes, cudaMemcpyDeviceToDevice, h->st));
  {
    double* full = nullptr;
    const size_t sbytes = (size_t)P.fs * 18 * sizeof(double);
    if (cudaMallocAsync((void**)&full, sbytes, h->st) == cudaSuccess) {
      CK(cudaMemcpyAsync(full, h->state, sbytes, cudaMemcpyDeviceToDevice, h->st));
      for (int which = 0; which < 2; which++) {
        int* ord = which == 0 ? h->tune.flux_order : h->tune.emf_order;
        const int base[3] = {ord[0], ord[1], ord[2]};
        float best = 1e30f;
        int best_r = 0;
        for (int r = 0; r < 3; r++) {
          for (int n = 0; n < 3; n++) ord[n] = base[(n + r) % 3];
          launch_arm(P, 1e300, 3.0, h->st);
          enqueue_one_step(h, h->st, Hook());  // warm-up
          cudaEventRecord(a, h->st);
          enqueue_one_step(h, h->st, Hook());
          enqueue_one_step(h, h->st, Hook());
          cudaEventRecord(b, h->st);
          CK(cudaEventSynchronize(b));
          float ms = 0.f;
          cudaEventElapsedTime(&ms, a, b);
          CK(cudaMemcpyAsync(h->state, full, sbytes, cudaMemcpyDeviceToDevice, h->st));
          CK(cudaMemcpyAsync(h->scal, h->hscal, NSCAL * sizeof(double), cudaMemcpyHostToDevice, h->st));
          if (ms < best) {
            best = ms;
            best_r = r;
          }
        }
        for (int n = 0; n < 3; n++) ord[n] = base[(n + best_r) % 3];
      }
      CK(cudaStreamSynchronize(h->st));
      cudaFreeAsync(full, h->st);
      drop_step_graph(h);
    } else {
      cudaGetLastError();  // no room for the copy: the orders stay as they are
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  CK(cudaMemcpyAsync(P.Wbuf[1 - cur], hist, wbytes, cudaMemcpyDeviceToDevice, h->st));
  CK(cudaMemcpyAsync(P.Bbuf[1 - cur], hist + 6 * P.fs, bbytes, cudaMemcpyDeviceToDevice, h->st));
  for (int t = 0; t < NSCAL; t++) h->hscal[t] = saved_scal[t];
  CK(cudaMemcpyAsync(h->scal, h->hscal, NSCAL * sizeof(double), cudaMemcpyHostToDevice, h->st));
  CK(cudaStreamSynchronize(h->st));
  cudaFreeAsync(hist, h->st);
  CK(cudaStreamSynchronize(h->st));
  CK(cudaGetLastError());
  return GOP_OK;
}

int gop_get_launch_order(gop_instance* h, int* flux_order, int* emf_order) {
  if (!h) return fail(GOP_EINVAL, "instance is NULL");
  for (int d = 0; d < 3; d++) {
    if (flux_order) flux_order[d] = h->tune.flux_order[d];
    if (emf_order) emf_order[d] = h->tune.emf_order[d];
  }
  return GOP_OK;
}

int gop_set_sweep(gop_instance* h, int on) {
  if (!h) return fail(GOP_EINVAL, "instance is NULL");
  if (on && !h->sweep) return fail(GOP_ENODEV, "the tile-staged sweep kernels are not available");
  CK(cudaStreamSynchronize(h->st));
  for (int d = 0; d < 3; d++) h->tune.flux_sweep[d] = h->tune.emf_sweep[d] = on != 0;
  drop_step_graph(h);
  return GOP_OK;
}

int gop_set_profiling(gop_instance* h, int on) {
  if (!h) return fail(GOP_EINVAL, "instance is NULL");
  CK(cudaStreamSynchronize(h->st));
  prof_collect(h);
  for (int g = 0; g < NGROUP; g++) {
    h->prof_ms[g] = 0.0;
    h->prof_n[g] = 0;
  }
  h->prof = on != 0;
  return GOP_OK;
}

int gop_get_profile(gop_instance* h, double* ms, int64_t* count) {
  if (!h || !ms || !count) return fail(GOP_EINVAL, "NULL argument");
  CK(cudaStreamSynchronize(h->st));
  prof_collect(h);
  for (int g = 0; g < NGROUP; g++) {
    ms[g] = h->prof_ms[g];
    count[g] = h->prof_n[g];
  }
  return GOP_OK;
}

int gop_get_stats(gop_instance* h, gop_stats* out) {
  if (!h || !out) return fail(GOP_EINVAL, "NULL argument");
  double* s = h->hscal;
  CK(cudaMemcpyAsync(s, h->scal, NSCAL * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  out->time = s[S_TIME];
  out->dt = s[S_DT];
  out->dt0 = s[S_DT0];
  out->divb_max = s[S_DIVB];
  out->steps = (int64_t)s[S_STEPS];
  out->flags = s[S_FLAGS] == 2.0 ? 2 : (s[S_FLAGS] != 0.0 ? 1 : 0);
  out->reserved = 0;
  out->device_bytes = h->bytes;
  return GOP_OK;
}


// ----------------------------------------------------------------- batch

}  // extern "C"

// A batch advances many independent grids as one CUDA graph per step.  The
// graph holds every member's own step -- its single-instance launch
// sequence, with its parameters as kernel arguments -- on up to kBranches
// parallel branches (members placed largest first on the branch with the
// fewest cells so far), so small grids that could not fill the GPU alone
// run side by side, and the launches of one grid's memory-bound stages
// overlap other grids' compute-bound ones.  Each member keeps its own
// device scalars (dt, time, AB2 coefficient, step budget); the graph is
// replayed max(steps) times and a member whose budget is spent returns at
// once from every launch.
static const int kBranches = 16;

struct gop_batch {
  std::vector<gop_instance*> m;
  int64_t nodes = 0;           // kernels in one replay of the graph
  cudaStream_t own = nullptr;  // capture stream
  cudaStream_t st = nullptr;   // launch stream (own, or the caller's)
  std::vector<cudaStream_t> br;  // branch streams (used while capturing)
  std::vector<cudaEvent_t> ev;   // fork and join events of the capture
  cudaGraphExec_t graph = nullptr;
  std::vector<uint64_t> gen;     // the members' generations the graph holds
};

static void batch_release(gop_batch* b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  b->graph = nullptr;
}

// captures one step of every member into the batch graph
static int batch_build(gop_batch* b) {
  batch_release(b);
  const int nb = (int)b->br.size();
  std::vector<int> order(b->m.size());
  for (size_t i = 0; i < order.size(); i++) order[i] = (int)i;
  auto cells = [&](int i) {
    const gop_desc& d = b->m[i]->d;
    return (long long)d.ni * d.nj * d.nk;
  };
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cells(x) > cells(y); });
  std::vector<long long> load(nb, 0);
  std::vector<int> branch(b->m.size(), 0);
  for (int i : order) {
    const int k = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    branch[i] = k;
    load[k] += cells(i);
  }
  CK(cudaStreamSynchronize(b->own));
  cudaGraph_t g = nullptr;
  const int64_t before = launches();
  CK(cudaStreamBeginCapture(b->own, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = cudaEventRecord(b->ev[0], b->own);
  for (int k = 0; k < nb && e == cudaSuccess; k++) e = cudaStreamWaitEvent(b->br[k], b->ev[0], 0);
  if (e == cudaSuccess)
    for (int i : order) enqueue_one_step(b->m[i], b->br[branch[i]], Hook());
  for (int k = 0; k < nb && e == cudaSuccess; k++) {
    e = cudaEventRecord(b->ev[1 + k], b->br[k]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(b->own, b->ev[1 + k], 0);
  }
  cudaError_t e2 = cudaStreamEndCapture(b->own, &g);
  if (e == cudaSuccess) e = e2;
  // captured launches run at each replay, not now
  b->nodes = launches() - before;
  count_launches(-b->nodes);
  b->gen.resize(b->m.size());
  for (size_t i = 0; i < b->m.size(); i++) b->gen[i] = b->m[i]->gen;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&b->graph, g, 0);
  if (g) cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    cudaGetLastError();
    b->graph = nullptr;
    return fail(GOP_ECUDA, "batch graph capture failed: %s", cudaGetErrorString(e));
  }
  return GOP_OK;
}

// The sweep kernels were picked per class with each grid stepping alone.
// In the batch the members' launches run side by side on parallel branches,
// and a persistent sweep grid (sized for the whole GPU) then shares the SMs
// with the other branches' kernels.  Times replays of the batch step with
// the per-class picks and with every member on the per-point kernels, the
// member states and scalars restored after each trial, and keeps the
// faster.  Without device memory for the copies of the states the picks
// stay as they are.
static int batch_pick_sweeps(gop_batch* b) {
  bool any = false;
  for (gop_instance* h : b->m)
    for (int d = 0; d < 3; d++) any = any || h->tune.flux_sweep[d] || h->tune.emf_sweep[d];
  if (!any || !b->graph) return GOP_OK;
  const size_t nm = b->m.size();
  std::vector<double*> saved(nm, nullptr);
  std::vector<double> scal(nm * NSCAL);
  bool ok = true;
  for (size_t i = 0; i < nm && ok; i++) {
    gop_instance* h = b->m[i];
    const size_t bytes = (size_t)h->P.fs * 18 * sizeof(double);
    ok = cudaMallocAsync((void**)&saved[i], bytes, b->st) == cudaSuccess &&
         cudaMemcpyAsync(saved[i], h->state, bytes, cudaMemcpyDeviceToDevice, b->st) == cudaSuccess &&
         cudaMemcpyAsync(&scal[i * NSCAL], h->scal, NSCAL * sizeof(double), cudaMemcpyDeviceToHost,
                         b->st) == cudaSuccess;
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  ok = ok && cudaEventCreate(&e0) == cudaSuccess && cudaEventCreate(&e1) == cudaSuccess &&
       cudaStreamSynchronize(b->st) == cudaSuccess;
  int rc = GOP_OK;
  // two timed replays after a warm-up one, then every member put back
  auto trial = [&](float* ms) {
    for (gop_instance* h : b->m) launch_arm(h->P, 1e300, 3.0, b->st);
    cudaGraphLaunch(b->graph, b->st);
    cudaEventRecord(e0, b->st);
    cudaGraphLaunch(b->graph, b->st);
    cudaGraphLaunch(b->graph, b->st);
    cudaEventRecord(e1, b->st);
    count_launches(3 * b->nodes);
    cudaError_t e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(ms, e0, e1);
    for (size_t i = 0; i < nm && e == cudaSuccess; i++) {
      gop_instance* h = b->m[i];
      e = cudaMemcpyAsync(h->state, saved[i], (size_t)h->P.fs * 18 * sizeof(double),
                          cudaMemcpyDeviceToDevice, b->st);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(h->scal, &scal[i * NSCAL], NSCAL * sizeof(double),
                            cudaMemcpyHostToDevice, b->st);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->st);
    if (e != cudaSuccess) rc = fail(GOP_ECUDA, "batch sweep trial failed: %s", cudaGetErrorString(e));
  };
  if (ok) {
    float t_pick = 0.f, t_off = 0.f;
    trial(&t_pick);
    std::vector<Tune> pick(nm);
    for (size_t i = 0; i < nm; i++) pick[i] = b->m[i]->tune;
    for (gop_instance* h : b->m) {
      for (int d = 0; d < 3; d++) h->tune.flux_sweep[d] = h->tune.emf_sweep[d] = false;
      drop_step_graph(h);
    }
    if (rc == GOP_OK) rc = batch_build(b);
    if (rc == GOP_OK) trial(&t_off);
    if (rc != GOP_OK || t_pick <= t_off) {
      for (size_t i = 0; i < nm; i++) {
        b->m[i]->tune = pick[i];
        drop_step_graph(b->m[i]);
      }
      const int rc2 = batch_build(b);
      if (rc == GOP_OK) rc = rc2;
    }
  } else {
    cudaGetLastError();  // no room for the copies: the picks stay
  }
  cudaStreamSynchronize(b->st);
  for (double* p : saved)
    if (p) cudaFreeAsync(p, b->st);
  cudaStreamSynchronize(b->st);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  return rc;
}

extern "C" {

int gop_batch_create(gop_instance* const* members, int count, gop_batch** out) {
  if (!members || count <= 0 || !out) return fail(GOP_EINVAL, "bad batch arguments");
  if (count > 0xffff) return fail(GOP_EINVAL, "at most 65535 members per batch");
  *out = nullptr;
  for (int i = 0; i < count; i++) {
    if (!members[i]) return fail(GOP_EINVAL, "member %d is NULL", i);
    if (!members[i]->prepared) return fail(GOP_ESTATE, "member %d is not prepared", i);
    for (int k = 0; k < i; k++)
      if (members[k] == members[i]) return fail(GOP_EINVAL, "member %d appears twice", i);
  }
  gop_batch* b = new (std::nothrow) gop_batch();
  if (!b) return fail(GOP_ENOMEM, "host allocation failed");
  b->m.assign(members, members + count);
  const int nb = std::min(count, kBranches);
  cudaError_t e = cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking);
  for (int k = 0; k < nb && e == cudaSuccess; k++) {
    cudaStream_t s = nullptr;
    e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e == cudaSuccess) b->br.push_back(s);
  }
  for (int k = 0; k <= nb && e == cudaSuccess; k++) {
    cudaEvent_t ev = nullptr;
    e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e == cudaSuccess) b->ev.push_back(ev);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    gop_batch_destroy(b);
    return fail(GOP_ENOMEM, "batch set-up failed: %s", cudaGetErrorString(e));
  }
  b->st = b->own;
  int rc = batch_build(b);
  if (rc) {
    gop_batch_destroy(b);
    return rc;
  }
  *out = b;
  return GOP_OK;
}

int gop_batch_destroy(gop_batch* b) {
  if (!b) return GOP_OK;
  if (b->st) cudaStreamSynchronize(b->st);
  batch_release(b);
  for (cudaStream_t s : b->br) cudaStreamDestroy(s);
  for (cudaEvent_t ev : b->ev) cudaEventDestroy(ev);
  if (b->own) cudaStreamDestroy(b->own);
  delete b;
  return GOP_OK;
}

int gop_batch_set_stream(gop_batch* b, void* stream) {
  if (!b) return fail(GOP_EINVAL, "batch is NULL");
  CK(cudaStreamSynchronize(b->st));
  b->st = stream ? (cudaStream_t)stream : b->own;
  return GOP_OK;
}

// Batch autotuner: members of the same grid shape, geometry and precision
// share block shapes; gop_autotune chooses them on the first member of each
// such class (restoring its state afterwards), the others copy them, and the
// batch graph is captured again.  `chosen` receives the choice of the class
// with the most cells.
int gop_batch_autotune(gop_batch* b, int reps, int* chosen) {
  if (!b) return fail(GOP_EINVAL, "batch is NULL");
  CK(cudaStreamSynchronize(b->st));
  std::vector<int> rep(b->m.size(), -1);
  long long most = -1;
  for (size_t i = 0; i < b->m.size(); i++) {
    const gop_desc& d = b->m[i]->d;
    for (size_t k = 0; k < i && rep[i] < 0; k++) {
      const gop_desc& e = b->m[k]->d;
      if (d.ni == e.ni && d.nj == e.nj && d.nk == e.nk && d.coord == e.coord &&
          d.precision == e.precision)
        rep[i] = rep[k];
    }
    if (rep[i] >= 0) {
      b->m[i]->tune = b->m[rep[i]]->tune;
      drop_step_graph(b->m[i]);
      continue;
    }
    rep[i] = (int)i;
    int pick[NTUNE];
    const int rc = gop_autotune(b->m[i], reps, pick);
    if (rc) return rc;
    const long long cells = (long long)d.ni * d.nj * d.nk;
    if (chosen && cells > most) {
      most = cells;
      for (int t = 0; t < NTUNE; t++) chosen[t] = pick[t];
    }
  }
  const int rc = batch_build(b);
  return rc ? rc : batch_pick_sweeps(b);
}

int gop_batch_launch(gop_batch* b, const int* steps) {
  if (!b || !steps) return fail(GOP_EINVAL, "NULL argument");
  int most = 0;
  for (size_t i = 0; i < b->m.size(); i++) {
    if (steps[i] < 0) return fail(GOP_EINVAL, "negative step count");
    most = std::max(most, steps[i]);
  }
  // members' own streams may still hold work on their state
  for (gop_instance* h : b->m) CK(cudaStreamSynchronize(h->st));
  CK(cudaStreamSynchronize(b->st));  // the previous launch of this batch is done
  // a member prepared again with another kernel set, background or block
  // shapes: capture the step of all members again
  for (size_t i = 0; i < b->m.size(); i++) {
    if (!b->m[i]->prepared) return fail(GOP_ESTATE, "member %d is not prepared", (int)i);
    if (b->m[i]->gen != b->gen[i]) {
      const int rc = batch_build(b);
      if (rc) return rc;
      break;
    }
  }
  for (size_t i = 0; i < b->m.size(); i++) launch_arm(b->m[i]->P, 1e300, (double)steps[i], b->st);
  for (int n = 0; n < most; n++) CK(cudaGraphLaunch(b->graph, b->st));
  count_launches((int64_t)most * b->nodes);
  for (size_t i = 0; i < b->m.size(); i++)
    if (steps[i] > 0) b->m[i]->fresh = false;
  CK(cudaGetLastError());
  return GOP_OK;
}

int gop_batch_wait(gop_batch* b) {
  if (!b) return fail(GOP_EINVAL, "NULL argument");
  CK(cudaStreamSynchronize(b->st));
  CK(cudaGetLastError());
  for (gop_instance* h : b->m) {
    double* sc = h->hscal;
    CK(cudaMemcpyAsync(sc, h->scal, NSCAL * sizeof(double), cudaMemcpyDeviceToHost, b->st));
    CK(cudaStreamSynchronize(b->st));
    if (sc[S_FLAGS] == 2.0) return fail(GOP_ECUDA, "a tile pipeline wait on the device timed out");
    if (sc[S_FLAGS] != 0.0) return fail(GOP_ENUMERIC, "non-finite or non-positive state in a member");
  }
  return GOP_OK;
}

int gop_batch_step(gop_batch* b, const int* steps) {
  const int rc = gop_batch_launch(b, steps);
  return rc ? rc : gop_batch_wait(b);
}

}  // extern "C"

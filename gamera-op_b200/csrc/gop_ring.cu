// Pole treatment of spherical grids whose theta range reaches a pole
// (doRingAverage, src/spherical/spherical_RingAverage.c): the E and B fields
// on the pole faces and, after every update, averages in phi over the
// rings of cells nearest each pole.
//
//   pole_emf     tackle_Efield_pole (spherical_RingAverage.c:154-203): E_i on
//                the pole edges -> its phi mean, E_k on them -> 0
//   ring_hydro   HydroRingAverage_base (:235-376): rho and p block-averaged
//                in phi with a parabolic profile (RingBlockAvg); the
//                velocities the same after removing their mean and first
//                Fourier mode (FilterBaseMode)
//   ring_emf     MagneticRingAverage_base (:379-541): the face fluxes B_j A_j
//                and B_i A_i of each ring averaged the same way; their
//                change, summed along each block, is an EMF-like field
//   ring_curl    (:543-577) its curl updates B_i, B_j, B_k (E_k = 0)
//   ring_pole    (:579-627) B_j on the pole face <- its neighbour, the phi
//                mean of B_k in the pole rows removed
//
// Each ring line (one i, one j, all nk phi cells) is one thread: the work is
// a few thousand lines per step.  The line arithmetic uses explicitly
// rounded operations (no fused multiply-adds) and the host's cos/sin table,
// so it follows the reference's evaluation order operation for operation
// (FilterBaseMode, RingBlockAvg and PPM, src/solver_func.c:2136-2260).
#include "gop_device.cuh"
#include "gop_kernels.h"

namespace gop {

namespace {

constexpr int MAXNK = 256;

__device__ __forceinline__ double dsgn(double x) { return x > 0.0 ? 1.0 : (x < 0.0 ? -1.0 : 0.0); }

__device__ __forceinline__ double minmod(double x, double y) {
  return __dmul_rn(__dmul_rn(0.5, __dadd_rn(dsgn(x), dsgn(y))), fmin(fabs(x), fabs(y)));
}

// PPM edge values of cell f from its neighbours (src/solver_func.c:2141-2186)
__device__ void ppm(double fm2, double fm1, double f, double fp1, double fp2, double* vm,
                    double* vp) {
  const double dvm2 = __dsub_rn(fm1, fm2), dvm1 = __dsub_rn(f, fm1);
  const double dvp1 = __dsub_rn(fp1, f), dvp2 = __dsub_rn(fp2, fp1);
  double dvc = __dmul_rn(0.5, __dadd_rn(dvm2, dvm1));
  double SM = __dmul_rn(2.0, minmod(dvm2, dvm1));
  const double Sm1 = minmod(dvc, SM);
  dvc = __dmul_rn(0.5, __dadd_rn(dvm1, dvp1));
  SM = __dmul_rn(2.0, minmod(dvm1, dvp1));
  const double Sp1 = minmod(dvc, SM);
  dvc = __dmul_rn(0.5, __dadd_rn(dvp2, dvp1));
  SM = __dmul_rn(2.0, minmod(dvp2, dvp1));
  const double Sp2 = minmod(dvc, SM);
  double p = __dsub_rn(__dmul_rn(0.5, __dadd_rn(f, fp1)), __ddiv_rn(__dsub_rn(Sp2, Sp1), 6.0));
  double m = __dsub_rn(__dmul_rn(0.5, __dadd_rn(f, fm1)), __ddiv_rn(__dsub_rn(Sp1, Sm1), 6.0));
  double ap = __dsub_rn(p, f), am = __dsub_rn(m, f);
  if (__dmul_rn(ap, am) >= 0.0) {
    ap = 0.0;
    am = 0.0;
  } else {
    if (fabs(ap) >= __dmul_rn(2.0, fabs(am))) ap = __dmul_rn(-2.0, am);
    if (fabs(am) >= __dmul_rn(2.0, fabs(ap))) am = __dmul_rn(-2.0, ap);
  }
  *vp = __dadd_rn(f, ap);
  *vm = __dadd_rn(f, am);
}

// Q <- Q minus its mean and first phi Fourier mode, which go to Q0
// (FilterBaseMode); cs: cos then sin of (k + 1/2) 2 pi / N
__device__ void filter_base(double* Q, int N, double* Q0, const double* __restrict__ cs) {
  const double scl = 2.0 / N;
  double a0 = 0.0, a1 = 0.0, b1 = 0.0;
  for (int i = 0; i < N; i++) {
    a0 = __dadd_rn(a0, Q[i]);
    a1 = __dadd_rn(a1, __dmul_rn(Q[i], cs[i]));
    b1 = __dadd_rn(b1, __dmul_rn(Q[i], cs[N + i]));
  }
  a1 = __dmul_rn(a1, scl);
  b1 = __dmul_rn(b1, scl);
  a0 = __dmul_rn(a0, __dmul_rn(0.5, scl));
  for (int i = 0; i < N; i++) {
    Q0[i] = __dadd_rn(__dadd_rn(a0, __dmul_rn(a1, cs[i])), __dmul_rn(b1, cs[N + i]));
    Q[i] = __dsub_rn(Q[i], Q0[i]);
  }
}

// Q <- the parabolic profile of its nchunk block averages, periodic in phi
// (RingBlockAvg)
__device__ void block_avg(double* Q, int N, int nchunk) {
  const int ncell = N / nchunk;
  double ext[MAXNK / 2 + 4];  // nchunk <= N / 2 block averages + 4 wrapped
  for (int ib = 0; ib < nchunk; ib++) {
    double sum = 0.0;
    for (int ic = 0; ic < ncell; ic++) sum = __dadd_rn(sum, Q[ib * ncell + ic]);
    ext[ib + 2] = __ddiv_rn(sum, (double)ncell);
  }
  ext[0] = ext[nchunk];      // blk_avg[nchunk - 2]
  ext[1] = ext[nchunk + 1];  // blk_avg[nchunk - 1]
  ext[nchunk + 2] = ext[2];
  ext[nchunk + 3] = ext[3];
  for (int ib = 2; ib < nchunk + 2; ib++) {
    const int ig = (ib - 2) * ncell;
    double fL, fR;
    ppm(ext[ib - 2], ext[ib - 1], ext[ib], ext[ib + 1], ext[ib + 2], &fL, &fR);
    const double a = __dmul_rn(3.0, __dsub_rn(__dadd_rn(fL, fR), __dmul_rn(2.0, ext[ib])));
    const double b = __dmul_rn(2.0, __dsub_rn(__dsub_rn(__dmul_rn(3.0, ext[ib]), fR), __dmul_rn(2.0, fL)));
    const double c = fL;
    const double nc = (double)ncell;
    const double a3 = __ddiv_rn(__ddiv_rn(__ddiv_rn(a, 3.0), nc), nc);
    for (int ic = 0; ic < ncell; ic++) {
      const double kl = (double)ic + 1.0;
      const double poly = __dadd_rn(__dsub_rn(__dmul_rn(__dmul_rn(3.0, kl), kl), __dmul_rn(3.0, kl)), 1.0);
      const double lin = __ddiv_rn(__dmul_rn(__dmul_rn(0.5, b), __dsub_rn(__dmul_rn(2.0, kl), 1.0)), nc);
      Q[ig + ic] = __dadd_rn(__dadd_rn(__dmul_rn(a3, poly), lin), c);
    }
  }
}

// ring row r (0 .. jmax) of pole `pole` (0: theta = 0, 1: theta = pi):
// its cell row j and the chunk count of the ring
__device__ __forceinline__ int ring_row(const Params& P, int pole, int r) {
  return pole == 0 ? NGH + r : NGH + P.n[1] - 1 - r;
}

// --- E and B on the pole faces ----------------------------------------------

template <typename R>
__global__ void k_pole_emf(Params P, R* __restrict__ E) {
  if (P.scal[S_STOP] != 0.0) return;
  const int i = NGH + blockIdx.x * blockDim.x + threadIdx.x;
  const int pole = blockIdx.y;
  if (!(P.ring & (1 << pole)) || i > NGH + P.n[0]) return;
  const int jp = pole == 0 ? NGH : NGH + P.n[1];  // the pole's j face
  const int nk = P.n[2];
  const size_t fs = P.fs;
  if (i < NGH + P.n[0]) {  // E_i of the active cells: phi mean over nk + 1 edges
    double m = 0.0;
    for (int k = NGH; k <= NGH + nk; k++) m = m + (double)E[lin(P, i, jp, k)];
    m = m / (nk + 1);
    for (int k = NGH; k <= NGH + nk; k++) E[lin(P, i, jp, k)] = (R)m;
  }
  for (int k = NGH; k < NGH + nk; k++) E[2 * fs + lin(P, i, jp, k)] = R(0);
}

// --- averages over the rings -------------------------------------------------

// thread: (i, ring row r, pole); rho, v1..3, p of the new state
__global__ void k_ring_hydro(Params P) {
  if (P.scal[S_STOP] != 0.0) return;
  const int i = NGH + blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y, pole = blockIdx.z;
  if (!(P.ring & (1 << pole)) || i >= NGH + P.n[0] || r > P.ring_jmax) return;
  double* W = P.Wbuf[1 - cur_buf(P)];  // written by this step's update
  const int j = ring_row(P, pole, r), nk = P.n[2], nch = P.nchunk[r];
  const size_t fs = P.fs;
  const long long sk = P.sk, x0 = lin(P, i, j, NGH);
  double Q[MAXNK], base[MAXNK], rem[MAXNK];
  for (int f = 0; f < 5; f++) {  // rho v1 v2 v3 p (p_S is left alone)
    double* a = W + (size_t)f * fs + x0;
    for (int k = 0; k < nk; k++) Q[k] = a[k * sk];
    if (f == 0 || f == 4) {
      block_avg(Q, nk, nch);
    } else {
      filter_base(Q, nk, base, P.ringtab);
      for (int k = 0; k < nk; k++) rem[k] = Q[k];
      block_avg(rem, nk, nch);
      for (int k = 0; k < nk; k++) Q[k] = __dadd_rn(rem[k], base[k]);
    }
    for (int k = 0; k < nk; k++) a[k * sk] = Q[k];
  }
}

// thread: (i, ring row r, pole, which flux): the EMF-like fields of one ring
// line into scr (E_i at field 0, E_j at field 1), every k of the line
__global__ void k_ring_emf(Params P, double* __restrict__ scr) {
  if (P.scal[S_STOP] != 0.0) return;
  const int i = NGH + blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y, pole = blockIdx.z >> 1, which = blockIdx.z & 1;
  if (!(P.ring & (1 << pole)) || r > P.ring_jmax) return;
  // which 0: B_j flux on the j faces inside the band -> E_i (cells along i)
  // which 1: B_i flux on the i faces of the ring rows -> E_j (faces along i)
  if (i >= NGH + P.n[0] + which) return;
  const double* B = P.Bbuf[1 - cur_buf(P)];
  const int nk = P.n[2], nch = P.nchunk[r];
  const int j = which == 0 ? (pole == 0 ? NGH + r + 1 : NGH + P.n[1] - 1 - r)
                           : ring_row(P, pole, r);
  const size_t fs = P.fs;
  const long long sk = P.sk;
  const int a = which == 0 ? 1 : 0;  // the face field's axis
  const double* b = B + (size_t)a * fs;
  double flux[MAXNK], base[MAXNK], rem[MAXNK];
  for (int k = 0; k < nk; k++)
    flux[k] = __dmul_rn(b[lin(P, i, j, NGH + k)], Geo<2>::face(P, a, i, j, NGH + k));
  filter_base(flux, nk, base, P.ringtab);
  for (int k = 0; k < nk; k++) rem[k] = flux[k];
  block_avg(rem, nk, nch);
  double* e = scr + (size_t)(which == 0 ? 0 : 1) * fs + lin(P, i, j, 0);
  for (int k = 0; k < P.N[2]; k++) e[k * sk] = 0.0;
  const int ncell = nk / nch;
  for (int blk = 0; blk < nch; blk++) {
    const int start = blk * ncell;
    double sum = 0.0;
    for (int m = 0; m < ncell - 1; m++) {
      sum = __dadd_rn(sum, __dsub_rn(rem[start + m], flux[start + m]));
      e[(start + NGH + 1 + m) * sk] = which == 0 ? -sum : sum;
    }
  }
}

// E_i / E_j of the band at (i, j, k), zero outside it
__device__ __forceinline__ bool in_ei(const Params& P, int j) {
  const int jm = P.ring_jmax;
  return ((P.ring & 1) && j >= NGH + 1 && j <= NGH + jm + 1) ||
         ((P.ring & 2) && j >= NGH + P.n[1] - 1 - jm && j <= NGH + P.n[1] - 1);
}
__device__ __forceinline__ bool in_ej(const Params& P, int j) {
  const int jm = P.ring_jmax;
  return ((P.ring & 1) && j >= NGH && j <= NGH + jm) ||
         ((P.ring & 2) && j >= NGH + P.n[1] - 1 - jm && j <= NGH + P.n[1] - 1);
}
__device__ __forceinline__ double ei_at(const Params& P, const double* scr, int i, int j, int k) {
  return in_ei(P, j) ? scr[lin(P, i, j, k)] : 0.0;
}
__device__ __forceinline__ double ej_at(const Params& P, const double* scr, int i, int j, int k) {
  return in_ej(P, j) ? scr[P.fs + lin(P, i, j, k)] : 0.0;
}

// thread: (i, band row, k); B -= curl E / area on the faces the band touches
__global__ void k_ring_curl(Params P, const double* __restrict__ scr) {
  if (P.scal[S_STOP] != 0.0) return;
  const int i = NGH + blockIdx.x * blockDim.x + threadIdx.x;
  const int k = NGH + blockIdx.z * blockDim.z + threadIdx.z;
  const int slot = blockIdx.y * blockDim.y + threadIdx.y;
  const int jm = P.ring_jmax, nrow = jm + 2, pole = slot / nrow, rr = slot % nrow;
  if (pole > 1 || !(P.ring & (1 << pole)) || i > NGH + P.n[0] || k > NGH + P.n[2]) return;
  // band rows: theta = 0: j = NGH .. NGH+jm+1; theta = pi: NGH+nj-2-jm .. NGH+nj-1
  const int j = pole == 0 ? NGH + rr : NGH + P.n[1] - 2 - jm + rr;
  const int ie = NGH + P.n[0] - 1, ke = NGH + P.n[2] - 1;
  double* B = P.Bbuf[1 - cur_buf(P)];
  const size_t fs = P.fs;
  const long long c = lin(P, i, j, k);
  // B_i: i faces of rows with E_j
  if (k <= ke && in_ej(P, j)) {
    const double ce = 1.0 * ((0.0 - 0.0) - (ej_at(P, scr, i, j, k + 1) - ej_at(P, scr, i, j, k)));
    B[c] -= ce / Geo<2>::face(P, 0, i, j, k);
  }
  if (i > ie) return;
  // B_j: j faces carrying E_i
  if (k <= ke && in_ei(P, j)) {
    const double ce = 1.0 * ((ei_at(P, scr, i, j, k + 1) - ei_at(P, scr, i, j, k)) - (0.0 - 0.0));
    B[fs + c] -= ce / Geo<2>::face(P, 1, i, j, k);
  }
  // B_k: k faces next to E_i or E_j
  if (in_ej(P, j) || in_ei(P, j) || in_ei(P, j + 1)) {
    const double ce = 1.0 * ((ej_at(P, scr, i + 1, j, k) - ej_at(P, scr, i, j, k)) -
                             (ei_at(P, scr, i, j + 1, k) - ei_at(P, scr, i, j, k)));
    B[2 * fs + c] -= ce / Geo<2>::face(P, 2, i, j, k);
  }
}

// thread: (i, pole): B_j on the pole face, the phi mean of B_k in the pole row
__global__ void k_ring_pole(Params P) {
  if (P.scal[S_STOP] != 0.0) return;
  const int i = NGH + blockIdx.x * blockDim.x + threadIdx.x;
  const int pole = blockIdx.y;
  if (!(P.ring & (1 << pole)) || i >= NGH + P.n[0]) return;
  double* B = P.Bbuf[1 - cur_buf(P)];
  const size_t fs = P.fs;
  const int nk = P.n[2];
  const int jf = pole == 0 ? NGH : NGH + P.n[1];           // the pole face
  const int jn = pole == 0 ? NGH + 1 : NGH + P.n[1] - 1;   // its neighbour face
  const int jc = pole == 0 ? NGH : NGH + P.n[1] - 1;       // the pole cell row
  for (int k = NGH; k < NGH + nk; k++) B[fs + lin(P, i, jf, k)] = B[fs + lin(P, i, jn, k)];
  double m = 0.0;
  for (int k = NGH; k <= NGH + nk; k++) m += B[2 * fs + lin(P, i, jc, k)];
  m = m / (nk + 1);
  for (int k = NGH; k <= NGH + nk; k++) B[2 * fs + lin(P, i, jc, k)] -= m;
}

}  // namespace

template <typename R>
void launch_pole_emf(const Params& P, const Work<R>& w, cudaStream_t st) {
  if (!P.ring) return;
  const int n = P.n[0] + 1;
  k_pole_emf<R><<<dim3((n + 63) / 64, 2), 64, 0, st>>>(P, w.E);
  count_launches(1);
}
template void launch_pole_emf<double>(const Params&, const Work<double>&, cudaStream_t);
template void launch_pole_emf<float>(const Params&, const Work<float>&, cudaStream_t);

void launch_ring_average(const Params& P, double* scratch, cudaStream_t st) {
  if (!P.ring) return;
  const int jm = P.ring_jmax;
  const int n = P.n[0] + 1;
  k_ring_hydro<<<dim3((n + 31) / 32, jm + 1, 2), 32, 0, st>>>(P);
  k_ring_emf<<<dim3((n + 31) / 32, jm + 1, 4), 32, 0, st>>>(P, scratch);
  const dim3 blk(32, 2, 4);
  k_ring_curl<<<dim3((n + 31) / 32, (2 * (jm + 2) + 1) / 2, (P.n[2] + 1 + 3) / 4), blk, 0, st>>>(P, scratch);
  k_ring_pole<<<dim3((n + 63) / 64, 2), 64, 0, st>>>(P);
  count_launches(4);
}

}  // namespace gop

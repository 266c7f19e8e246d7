// CUDA kernels of the GAMERA-OP single-domain MHD step for B200 (sm_100a).
//
// One step (src/solver_solve.c:103-508) is a fixed sequence of launches on
// one stream, all reading dt and the AB2 coefficient from device memory so
// the sequence can be captured in a CUDA graph and replayed without host
// synchronisation:
//
//   begin     dt <- running CFL minimum, time += dt, c = dt/(2 dt0)
//   ab2       W_h, mags, mags_h, B_h over the ghost-extended grid
//   c2c       centre-to-edge velocity, first sweep (3 edge directions)
//   emf       centre-to-edge second sweep, face-B reconstruction, edge EMF
//   flux      PDM reconstruction + Rusanov flux + Maxwell stress per face
//   update    divergence, sources, constrained transport, cons->prim,
//             floors, Alfven/Boris correction, next CFL dt, max|div B|
//   ghost     periodic wrap and boundary fills of the new state
//
// R is the arithmetic type of the reconstruction / flux / EMF stages
// (double: plain path; float: mixed path).  The state, the AB2
// extrapolation, the conservative update and the pressure recovery are FP64
// in both.
#include "gop_device.cuh"
#include "gop_kernels.h"

#include <cfloat>

namespace gop {

enum { RHO = 0, V1, V2, V3, PR, PS };

// ------------------------------------------------------------------ utils

__device__ __forceinline__ bool stopped(const Params& P) { return P.scal[S_STOP] != 0.0; }

__device__ __forceinline__ void atomic_min_pos(double* slot, double v) {
  // positive doubles order like their bit patterns
  atomicMin(reinterpret_cast<unsigned long long*>(slot), (unsigned long long)__double_as_longlong(v));
}
__device__ __forceinline__ void atomic_max_pos(double* slot, double v) {
  atomicMax(reinterpret_cast<unsigned long long*>(slot), (unsigned long long)__double_as_longlong(v));
}

__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// block-wide min and max of (a, b); thread 0 commits them with one atomic each
__device__ __forceinline__ void block_commit(double a, double b, double* smin, double* smax) {
  __shared__ double sa[32], sb[32];
  int lane = threadIdx.x & 31;
  int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  int nw = (blockDim.x * blockDim.y * blockDim.z + 31) / 32;
  int w = tid / 32;
  lane = tid & 31;
  a = warp_min(a);
  b = warp_max(b);
  if (lane == 0) {
    sa[w] = a;
    sb[w] = b;
  }
  __syncthreads();
  if (w == 0) {
    a = lane < nw ? sa[lane] : DBL_MAX;
    b = lane < nw ? sb[lane] : 0.0;
    a = warp_min(a);
    b = warp_max(b);
    if (lane == 0) {
      if (a < DBL_MAX) atomic_min_pos(smin, a);
      if (b > 0.0) atomic_max_pos(smax, b);
    }
  }
}

// CFL time step of one cell (src/solver_func.c:255-298)
template <int COORD>
__device__ __forceinline__ double cfl_cell(const Params& P, int i, int j, int k, double rho,
                                           double u, double v, double w, double p, double b1,
                                           double b2, double b3) {
  double bsq = b1 * b1 + b2 * b2 + b3 * b3;
  double va = sqrt(bsq / rho);
  double vae = va * P.ca / sqrt(va * va + P.ca2);
  double vf = sqrt(u * u + v * v + w * w);
  double vs = sqrt(P.gamma * p / rho);
  double vc = vf + sqrt(vs * vs + vae * vae);
  double t = vc / Geo<COORD>::dl(P, 0, i, j, k) + vc / Geo<COORD>::dl(P, 1, i, j, k) +
             vc / Geo<COORD>::dl(P, 2, i, j, k);
  return P.cfl / t;
}

// cell-centred B from the two faces along each axis (src/solver_func.c:311-322)
__device__ __forceinline__ double mags_at(const Params& P, const double* B, int a, int i, int j,
                                          int k) {
  long long c = lin(P, i, j, k);
  int idx = a == 0 ? i : (a == 1 ? j : k);
  const double* f = B + (size_t)a * P.fs;
  return f[c] * tb(P, a, T_MA, idx) + f[c + stride(P, a)] * tb(P, a, T_MB, idx);
}

// ------------------------------------------------------------ begin / dt

// one thread: open the step (src/solver_solve.c:103-107, solver_func.c:385-491)
__global__ void k_begin(Params P) {
  double* s = P.scal;
  if (s[S_STOP] != 0.0) return;
  if (s[S_TIME] > s[S_TSTOP]) {
    s[S_STOP] = 1.0;
    return;
  }
  double dt = __longlong_as_double((long long)__double_as_longlong(s[S_NEXT_DT]));
  if (!(dt > 0.0) || !isfinite(dt)) s[S_FLAGS] = 1.0;
  s[S_DT] = dt;
  s[S_TIME] = s[S_TIME] + dt;
  s[S_CAB2] = 0.5 * dt / s[S_DT0];
  s[S_DT0] = dt;
  s[S_NEXT_DT] = DBL_MAX;
  s[S_DIVB] = 0.0;
  s[S_STEPS] = s[S_STEPS] + 1.0;
}

// one thread: arm a gop_step call with its stop time
__global__ void k_arm(Params P, double tstop) {
  P.scal[S_TSTOP] = tstop;
  P.scal[S_STOP] = 0.0;
}

// one thread: close the step -- the buffer written by this step becomes
// the current state
__global__ void k_end(Params P) {
  if (P.scal[S_STOP] != 0.0) return;
  P.scal[S_PAR] = P.scal[S_PAR] != 0.0 ? 0.0 : 1.0;
}

// CFL dt and max|div B| of the current state (used by prepare)
template <int COORD>
__global__ void k_dt(Params P) {
  const double* __restrict__ W = P.Wbuf[cur_buf(P)];
  const double* __restrict__ B = P.Bbuf[cur_buf(P)];
  int i = NGH + blockIdx.x * blockDim.x + threadIdx.x;
  int j = NGH + blockIdx.y * blockDim.y + threadIdx.y;
  int k = NGH + blockIdx.z * blockDim.z + threadIdx.z;
  double dtc = DBL_MAX, db = 0.0;
  if (i < NGH + P.n[0] && j < NGH + P.n[1] && k < NGH + P.n[2]) {
    long long c = lin(P, i, j, k);
    double b1 = mags_at(P, B, 0, i, j, k), b2 = mags_at(P, B, 1, i, j, k),
           b3 = mags_at(P, B, 2, i, j, k);
    dtc = cfl_cell<COORD>(P, i, j, k, W[c], W[c + P.fs], W[c + 2 * P.fs], W[c + 3 * P.fs],
                          W[c + 4 * P.fs], b1, b2, b3);
    double vol = Geo<COORD>::vol(P, i, j, k), d = 0.0;
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const double* f = B + (size_t)a * P.fs;
      long long s = stride(P, a);
      int i1 = i + (a == 0), j1 = j + (a == 1), k1 = k + (a == 2);
      d += (f[c + s] * Geo<COORD>::face(P, a, i1, j1, k1) - f[c] * Geo<COORD>::face(P, a, i, j, k)) /
           vol;
    }
    db = fabs(d);
  }
  block_commit(dtc, db, P.scal + S_NEXT_DT, P.scal + S_DIVB);
}

// ------------------------------------------------------------------- AB2

// W_h = W + c (W - W_old), mags and mags_h from the faces, B_h on faces
// (src/solver_func.c:385-449) over the whole ghost-extended grid
template <typename R>
__global__ void k_ab2(Params P, Work<R> w) {
  if (stopped(P)) return;
  const int cb = cur_buf(P);
  const double* __restrict__ W = P.Wbuf[cb];
  const double* __restrict__ Wo = P.Wbuf[1 - cb];
  const double* __restrict__ B = P.Bbuf[cb];
  const double* __restrict__ Bo = P.Bbuf[1 - cb];
  R* __restrict__ Wh = w.Wh;
  R* __restrict__ Ms = w.Ms;
  R* __restrict__ Msh = w.Msh;
  R* __restrict__ Bh = w.Bh;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= P.N[0] || j >= P.N[1] || k >= P.N[2]) return;
  const double c = P.scal[S_CAB2];
  long long x = lin(P, i, j, k);
  bool ci = i < P.N[0] - 1, cj = j < P.N[1] - 1, ck = k < P.N[2] - 1;
  if (ci && cj && ck) {
#pragma unroll
    for (int m = 0; m < 6; m++) {
      double w = W[x + m * P.fs], wo = Wo[x + m * P.fs];
      Wh[x + m * P.fs] = (R)(w + c * (w - wo));
    }
#pragma unroll
    for (int a = 0; a < 3; a++) {
      double ms = mags_at(P, B, a, i, j, k), mo = mags_at(P, Bo, a, i, j, k);
      Ms[x + a * P.fs] = (R)ms;
      Msh[x + a * P.fs] = (R)(ms + c * (ms - mo));
    }
  }
#pragma unroll
  for (int a = 0; a < 3; a++) {
    bool ok = (a == 0 || ci) && (a == 1 || cj) && (a == 2 || ck);
    if (ok) {
      double b = B[x + a * P.fs], bo = Bo[x + a * P.fs];
      Bh[x + a * P.fs] = (R)(b + c * (b - bo));
    }
  }
}

// ------------------------------------------------------------- edge EMF

// load v[0..7] = field at cells f-4..f+3 along axis s from x (x at cell f)
template <typename R, typename T>
__device__ __forceinline__ void line8(const T* __restrict__ a, long long x, long long s, R v[8]) {
#pragma unroll
  for (int t = 0; t < 8; t++) v[t] = (R)a[x + (t - 4) * s];
}

// First centre-to-edge sweep of center2corner_{jk,ki,ij}
// (src/solver_func.c:686-778): for edge direction d, velocity components
// p=(d+1)%3 and q=(d+2)%3 reconstructed along p (limiter on the step-start
// velocity) and averaged.  Points: d active, p faces lo..hi+1, q all ghosts.
template <typename R>
__global__ void k_c2c(Params P, int d, Work<R> wk) {
  if (stopped(P)) return;
  const double* __restrict__ W = P.Wbuf[cur_buf(P)];
  const R* __restrict__ Wh = wk.Wh;
  R* __restrict__ Vint = wk.V;
  int p = (d + 1) % 3, q = (d + 2) % 3;
  int t0 = blockIdx.x * blockDim.x + threadIdx.x;
  int t1 = blockIdx.y * blockDim.y + threadIdx.y;
  int t2 = blockIdx.z * blockDim.z + threadIdx.z;
  int ijk[3] = {t0, t1, t2};
  // ranges: axis d [NGH, NGH+n-1], axis p [NGH, NGH+n], axis q [0, n+2*NGH-1]
  int lo[3], cnt[3];
  lo[d] = NGH; cnt[d] = P.n[d];
  lo[p] = NGH; cnt[p] = P.n[p] + 1;
  lo[q] = 0;   cnt[q] = P.n[q] + 2 * NGH;
  if (ijk[0] >= cnt[0] || ijk[1] >= cnt[1] || ijk[2] >= cnt[2]) return;
  int i = ijk[0] + lo[0], j = ijk[1] + lo[1], k = ijk[2] + lo[2];
  int f = p == 0 ? i : (p == 1 ? j : k);
  long long x = lin(P, i, j, k), s = stride(P, p);
  FaceWeights<R> Wt;
  load_weights<R>(P, p, f, Wt);
  const R a1 = (R)P.pdm_a1, a2 = (R)P.pdm_a2;
#pragma unroll
  for (int cc = 0; cc < 2; cc++) {
    int comp = cc == 0 ? p : q;
    R v[8], lim[4], L, Rr;
    line8<R, R>(Wh + (size_t)(V1 + comp) * P.fs, x, s, v);
#pragma unroll
    for (int t = 0; t < 4; t++) lim[t] = (R)W[x + (V1 + comp) * P.fs + (t - 2) * s];
    recon_lr<R>(v, lim, Wt, a1, a2, L, Rr);
    Vint[x + (size_t)(2 * d + cc) * P.fs] = R(0.5) * (L + Rr);
  }
}

// Second sweep, face-field reconstruction and the edge EMF
// (src/solver_func.c:779-902) for edges along d: d active, p and q faces.
template <typename R>
__global__ void k_emf(Params P, int d, Work<R> wk) {
  if (stopped(P)) return;
  const double* __restrict__ B = P.Bbuf[cur_buf(P)];
  const R* __restrict__ Bh = wk.Bh;
  const R* __restrict__ Wh = wk.Wh;
  const R* __restrict__ Vint = wk.V;
  R* __restrict__ E = wk.E;
  int p = (d + 1) % 3, q = (d + 2) % 3;
  int ijk[3] = {(int)(blockIdx.x * blockDim.x + threadIdx.x),
                (int)(blockIdx.y * blockDim.y + threadIdx.y),
                (int)(blockIdx.z * blockDim.z + threadIdx.z)};
  int cnt[3];
  cnt[d] = P.n[d];
  cnt[p] = P.n[p] + 1;
  cnt[q] = P.n[q] + 1;
  if (ijk[0] >= cnt[0] || ijk[1] >= cnt[1] || ijk[2] >= cnt[2]) return;
  int i = ijk[0] + NGH, j = ijk[1] + NGH, k = ijk[2] + NGH;
  int pos[3] = {i, j, k};
  long long x = lin(P, i, j, k), sp = stride(P, p), sq = stride(P, q);
  const R a1 = (R)P.pdm_a1, a2 = (R)P.pdm_a2;
  R vav[2];
  {
    FaceWeights<R> Wt;
    load_weights<R>(P, q, pos[q], Wt);
#pragma unroll
    for (int cc = 0; cc < 2; cc++) {
      R v[8], lim[4], L, Rr;
      line8<R, R>(Vint + (size_t)(2 * d + cc) * P.fs, x, sq, v);
#pragma unroll
      for (int t = 0; t < 4; t++) lim[t] = v[t + 2];
      recon_lr<R>(v, lim, Wt, a1, a2, L, Rr);
      vav[cc] = R(0.5) * (L + Rr);
    }
  }
  // B_p along q and B_q along p
  R bpl, bpr, bql, bqr;
  {
    FaceWeights<R> Wt;
    load_weights<R>(P, q, pos[q], Wt);
    R v[8], lim[4];
    line8<R, R>(Bh + (size_t)p * P.fs, x, sq, v);
#pragma unroll
    for (int t = 0; t < 4; t++) lim[t] = (R)B[x + p * P.fs + (t - 2) * sq];
    recon_lr<R>(v, lim, Wt, a1, a2, bpl, bpr);
  }
  {
    FaceWeights<R> Wt;
    load_weights<R>(P, p, pos[p], Wt);
    R v[8], lim[4];
    line8<R, R>(Bh + (size_t)q * P.fs, x, sp, v);
#pragma unroll
    for (int t = 0; t < 4; t++) lim[t] = (R)B[x + q * P.fs + (t - 2) * sp];
    recon_lr<R>(v, lim, Wt, a1, a2, bql, bqr);
  }
  R bp = R(0.5) * (bpl + bpr), bq = R(0.5) * (bql + bqr);
  R vp = vav[0], vq = vav[1];
  R e = -(vp * bq - vq * bp);
  const R* rh = Wh;  // density slot
  R rho4 = rh[x - sp - sq] + rh[x - sp] + rh[x - sq] + rh[x];
  if (d == 1) rho4 = rh[x - sq - sp] + rh[x - sq] + rh[x - sp] + rh[x];
  R ca = (R)P.ca;
  R vz = sqrt((bp * bp + bq * bq) / (R(0.25) * rho4));
  vz = vz * ca / sqrt(vz * vz + ca * ca) + sqrt(vp * vp + vq * vq);
  e += R(0.5) * vz * (bpl + bqr - bpr - bql);
  E[x + (size_t)d * P.fs] = e;
}

// ------------------------------------------------------------ face flux

// Rusanov hydro flux and Maxwell stress at faces normal to d
// (src/solver_func.c:934-1529).  F[9] = mass, 3 momenta, energy, entropy,
// 3 stress components.
template <typename R>
__global__ void k_flux(Params P, int d, Work<R> wk) {
  if (stopped(P)) return;
  const double* __restrict__ W = P.Wbuf[cur_buf(P)];
  const double* __restrict__ B = P.Bbuf[cur_buf(P)];
  const R* __restrict__ Wh = wk.Wh;
  const R* __restrict__ Ms = wk.Ms;
  const R* __restrict__ Msh = wk.Msh;
  R* __restrict__ F = wk.F;
  int ijk[3] = {(int)(blockIdx.x * blockDim.x + threadIdx.x),
                (int)(blockIdx.y * blockDim.y + threadIdx.y),
                (int)(blockIdx.z * blockDim.z + threadIdx.z)};
  int cnt[3] = {P.n[0], P.n[1], P.n[2]};
  cnt[d] += 1;
  if (ijk[0] >= cnt[0] || ijk[1] >= cnt[1] || ijk[2] >= cnt[2]) return;
  int i = ijk[0] + NGH, j = ijk[1] + NGH, k = ijk[2] + NGH;
  int f = d == 0 ? i : (d == 1 ? j : k);
  long long x = lin(P, i, j, k), s = stride(P, d);
  FaceWeights<R> Wt;
  load_weights<R>(P, d, f, Wt);
  const R a1 = (R)P.pdm_a1, a2 = (R)P.pdm_a2;
  R L[6], Rt[6], mL[3], mR[3];
#pragma unroll
  for (int m = 0; m < 6; m++) {
    R v[8], lim[4];
    line8<R, R>(Wh + (size_t)m * P.fs, x, s, v);
#pragma unroll
    for (int t = 0; t < 4; t++) lim[t] = (R)W[x + m * P.fs + (t - 2) * s];
    recon_lr<R>(v, lim, Wt, a1, a2, L[m], Rt[m]);
  }
#pragma unroll
  for (int a = 0; a < 3; a++) {
    R v[8], lim[4];
    line8<R, R>(Msh + (size_t)a * P.fs, x, s, v);
#pragma unroll
    for (int t = 0; t < 4; t++) lim[t] = Ms[x + a * P.fs + (t - 2) * s];
    recon_lr<R>(v, lim, Wt, a1, a2, mL[a], mR[a]);
  }
  const R gm = (R)P.gamma, gm1 = (R)P.gm1, ca = (R)P.ca;
  R rl = L[RHO], rr = Rt[RHO], pl = L[PR], pr = Rt[PR], sl = L[PS], sr = Rt[PS];
  R csl = sqrt(gm * pl / rl), csr = sqrt(gm * pr / rr);
  R csel = sqrt(gm * sl / rl), cser = sqrt(gm * sr / rr);
  R btl = mL[0] * mL[0] + mL[1] * mL[1] + mL[2] * mL[2];
  R btr = mR[0] * mR[0] + mR[1] * mR[1] + mR[2] * mR[2];
  R val = sqrt(btl / rl), var = sqrt(btr / rr);
  R vel = val * ca / sqrt(val * val + ca * ca);
  R ver = var * ca / sqrt(var * var + ca * ca);
  R vnl = L[V1 + d], vnr = Rt[V1 + d];
  R vf = fmax(fabs(vnl) + sqrt(csl * csl + vel * vel), fabs(vnr) + sqrt(csr * csr + ver * ver));
  R vfe = fmax(fabs(vnl) + sqrt(csel * csel + vel * vel), fabs(vnr) + sqrt(cser * cser + ver * ver));
  R mol[3], mor[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    mol[a] = rl * L[V1 + a];
    mor[a] = rr * Rt[V1 + a];
  }
  R el = R(0.5) * rl * (L[V1] * L[V1] + L[V2] * L[V2] + L[V3] * L[V3]) + pl / gm1;
  R er = R(0.5) * rr * (Rt[V1] * Rt[V1] + Rt[V2] * Rt[V2] + Rt[V3] * Rt[V3]) + pr / gm1;
  R Sl = sl / pow(rl, gm1), Sr = sr / pow(rr, gm1);
  const size_t fs = P.fs;
  R* o = F + (size_t)(9 * d) * fs + x;
  o[0] = R(0.5) * (mol[d] + mor[d] - vf * (rr - rl));
#pragma unroll
  for (int a = 0; a < 3; a++) {
    R t = mol[a] * vnl + mor[a] * vnr - vf * (mor[a] - mol[a]);
    if (a == d) t = mol[a] * vnl + pl + mor[a] * vnr + pr - vf * (mor[a] - mol[a]);
    o[(1 + a) * fs] = R(0.5) * t;
  }
  o[4 * fs] = R(0.5) * (el * vnl + pl * vnl + er * vnr + pr * vnr - vf * (er - el));
  o[5 * fs] = R(0.5) * (Sl * vnl + Sr * vnr - vfe * (Sr - Sl));
  R bn = (R)B[x + d * fs];
  R bq = (btl + btr) / R(4) / ca;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    R tl, tr;
    if (a == d) {
      tl = R(0.5) * (R(0.5) * btl - mL[a] * bn);
      tr = R(0.5) * (R(0.5) * btr - mR[a] * bn);
    } else {
      tl = R(0.5) * (-mL[a] * bn);
      tr = R(0.5) * (-mR[a] * bn);
    }
    o[(6 + a) * fs] = (tl + tr) - bq * (Rt[V1 + a] - L[V1 + a]);
  }
}

// --------------------------------------------------------------- update

// new face field of component a at face (i,j,k) by constrained transport
// (src/solver_solve.c:263-306)
template <int COORD, typename R>
__device__ __forceinline__ double ct_face(const Params& P, const double* __restrict__ B,
                                          const R* __restrict__ E, int a, int i, int j, int k,
                                          double dt) {
  int p = (a + 1) % 3, q = (a + 2) % 3;
  long long x = lin(P, i, j, k), sp = stride(P, p), sq = stride(P, q);
  int ip = i + (p == 0), jp = j + (p == 1), kp = k + (p == 2);
  int iq = i + (q == 0), jq = j + (q == 1), kq = k + (q == 2);
  const size_t fs = P.fs;
  double cq = (double)E[x + sp + q * fs] * Geo<COORD>::edge(P, q, ip, jp, kp) -
              (double)E[x + q * fs] * Geo<COORD>::edge(P, q, i, j, k);
  double cp = (double)E[x + sq + p * fs] * Geo<COORD>::edge(P, p, iq, jq, kq) -
              (double)E[x + p * fs] * Geo<COORD>::edge(P, p, i, j, k);
  return B[x + a * fs] - dt * (cq - cp) / Geo<COORD>::face(P, a, i, j, k);
}

template <int COORD, typename R>
__global__ void k_update(Params P, Work<R> wk) {
  if (stopped(P)) return;
  const int cb = cur_buf(P);
  const double* __restrict__ W = P.Wbuf[cb];
  const double* __restrict__ B = P.Bbuf[cb];
  double* __restrict__ Wn = P.Wbuf[1 - cb];
  double* __restrict__ Bn = P.Bbuf[1 - cb];
  const R* __restrict__ Wh = wk.Wh;
  const R* __restrict__ Msh = wk.Msh;
  const R* __restrict__ F = wk.F;
  const R* __restrict__ E = wk.E;
  int i = NGH + blockIdx.x * blockDim.x + threadIdx.x;
  int j = NGH + blockIdx.y * blockDim.y + threadIdx.y;
  int k = NGH + blockIdx.z * blockDim.z + threadIdx.z;
  double dtc = DBL_MAX, dbmax = 0.0;
  bool inside = i < NGH + P.n[0] && j < NGH + P.n[1] && k < NGH + P.n[2];
  if (inside) {
    const size_t fs = P.fs;
    const double dt = P.scal[S_DT];
    long long x = lin(P, i, j, k);
    const double vol = Geo<COORD>::vol(P, i, j, k);
    double du[6], dm[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      long long s = stride(P, d);
      int i1 = i + (d == 0), j1 = j + (d == 1), k1 = k + (d == 2);
      double f0 = Geo<COORD>::face(P, d, i, j, k), f1 = Geo<COORD>::face(P, d, i1, j1, k1);
      const R* Fd = F + (size_t)(9 * d) * fs;
#pragma unroll
      for (int m = 0; m < 6; m++) {
        double v = ((double)Fd[x + s + m * fs] * f1 - (double)Fd[x + m * fs] * f0) / vol;
        du[m] = d == 0 ? v : du[m] + v;
      }
#pragma unroll
      for (int a = 0; a < 3; a++) {
        double v = ((double)Fd[x + s + (6 + a) * fs] * f1 - (double)Fd[x + (6 + a) * fs] * f0) / vol;
        dm[a] = d == 0 ? v : dm[a] + v;
      }
    }
    // spherical geometric sources (src/spherical/spherical_general.c:605-681)
    double sh[3] = {0.0, 0.0, 0.0}, sb[3] = {0.0, 0.0, 0.0};
    if (COORD == 2) {
      long long si = 1, sjj = P.sj;
      double fi0 = Geo<COORD>::face(P, 0, i, j, k), fi1 = Geo<COORD>::face(P, 0, i + 1, j, k);
      double fj0 = Geo<COORD>::face(P, 1, i, j, k), fj1 = Geo<COORD>::face(P, 1, i, j + 1, k);
      double dr = tb(P, 0, T_DX, i), rc = tb(P, 0, T_G3, i);
      double ph = Wh[x + PR * fs], rh = Wh[x + RHO * fs], v2h = Wh[x + V2 * fs], v3h = Wh[x + V3 * fs];
      double m22 = ph + rh * v2h * v2h, m33 = ph + rh * v3h * v3h;
      const R* Fi = F;
      const R* Fj = F + (size_t)9 * fs;
      sh[0] = 0.5 * (m22 + m33) * (fi1 - fi0) / vol;
      double s21 = -((double)Fi[x + 2 * fs] * fi0 + (double)Fi[x + si + 2 * fs] * fi1) * dr / rc / 2.0 / vol;
      sh[1] = s21 + (fj1 - fj0) / vol * m33;
      sh[2] = -((double)Fi[x + 3 * fs] * fi0 + (double)Fi[x + si + 3 * fs] * fi1) * dr / rc / 2.0 / vol;
      double sd = tb(P, 1, T_G3, j), ss = tb(P, 1, T_G4, j);
      sh[2] += -((double)Fj[x + 3 * fs] * fj0 + (double)Fj[x + sjj + 3 * fs] * fj1) * sd / ss / vol;
      double b1 = Msh[x], b2 = Msh[x + fs], b3 = Msh[x + 2 * fs];
      double bsq = b1 * b1 + b2 * b2 + b3 * b3;
      double n22 = 0.5 * bsq - b2 * b2, n33 = 0.5 * bsq - b3 * b3;
      sb[0] = 0.5 * (n22 + n33) * (fi1 - fi0) / vol;
      double t21 = -((double)Fi[x + 7 * fs] * fi0 + (double)Fi[x + si + 7 * fs] * fi1) * dr / rc / 2.0 / vol;
      sb[1] = t21 + (fj1 - fj0) / vol * n33;
      sb[2] = -((double)Fi[x + 8 * fs] * fi0 + (double)Fi[x + si + 8 * fs] * fi1) * dr / rc / 2.0 / vol;
      sb[2] += -((double)Fj[x + 8 * fs] * fj0 + (double)Fj[x + sjj + 8 * fs] * fj1) * sd / ss / vol;
    }
    // new face fields: this cell's lower faces and (for mags) the upper faces
    double bl[3], bu[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      bl[a] = ct_face<COORD, R>(P, B, E, a, i, j, k, dt);
      bu[a] = ct_face<COORD, R>(P, B, E, a, i + (a == 0), j + (a == 1), k + (a == 2), dt);
      Bn[x + a * fs] = bl[a];
      int pos = a == 0 ? i : (a == 1 ? j : k);
      if (pos == NGH + P.n[a] - 1) Bn[x + stride(P, a) + a * fs] = bu[a];
    }
    // U^n from W^n (src/solver_func.c:356-382)
    const double gm1 = P.gm1;
    double r0 = W[x], u0 = W[x + fs], v0 = W[x + 2 * fs], w0 = W[x + 3 * fs], p0 = W[x + 4 * fs],
           ps0 = W[x + 5 * fs];
    double U[6];
    U[0] = r0;
    U[1] = r0 * u0;
    U[2] = r0 * v0;
    U[3] = r0 * w0;
    U[4] = 0.5 * r0 * (u0 * u0 + v0 * v0 + w0 * w0) + p0 / gm1;
    U[5] = ps0 / pow(r0, gm1);
    double U0[3] = {U[1], U[2], U[3]};
    // conservative update and cons->prim (src/solver_solve.c:326-377)
    U[0] -= dt * du[0];
#pragma unroll
    for (int a = 0; a < 3; a++) U[1 + a] = U[1 + a] - dt * du[1 + a] + dt * sh[a];
    U[4] -= dt * du[4];
    U[5] -= dt * du[5];
    double rho = U[0];
    double vv[3] = {U[1] / U[0], U[2] / U[0], U[3] / U[0]};
    double p = (U[4] - 0.5 * (vv[0] * vv[0] + vv[1] * vv[1] + vv[2] * vv[2]) * rho) * gm1;
    double pS = U[5] * pow(U[0], gm1);
    // positivity floors (src/solver_func.c:2117-2135)
    if (rho < P.rho_floor) {
      rho = P.rho_floor;
      p = P.p_floor;
    }
    if (p < P.p_floor) p = P.p_floor;
    // mags^{n+1}, time-centred field, Alfven/Boris correction
    // (src/solver_solve.c:385-484)
    double mt[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      int idx = a == 0 ? i : (a == 1 ? j : k);
      double msn = bl[a] * tb(P, a, T_MA, idx) + bu[a] * tb(P, a, T_MB, idx);
      double mso = mags_at(P, B, a, i, j, k);
      mt[a] = 0.5 * (msn + mso);
      bu[a] = msn;  // keep mags^{n+1} for the next dt
    }
    double bsq = mt[0] * mt[0] + mt[1] * mt[1] + mt[2] * mt[2];
    double alf = bsq / rho / P.ca2;
    double perp = 1.0 / (1.0 + alf);
    double drho = -dt * du[0];
    double dva = alf * drho;
    double tv[3];
#pragma unroll
    for (int a = 0; a < 3; a++) tv[a] = alf * (-dt * du[1 + a] + dt * sh[a] - drho * W[x + (1 + a) * fs]);
    double bdv = mt[0] * tv[0] + mt[1] * tv[1] + mt[2] * tv[2];
    bdv = bdv / (bsq + 1e-10);
#pragma unroll
    for (int a = 0; a < 3; a++) {
      double mom = U0[a] + perp * ((-dt * du[1 + a] + dt * sh[a]) + (-dt * dm[a] + dt * sb[a]) +
                                   dva * W[x + (1 + a) * fs] + mt[a] * bdv);
      vv[a] = mom / U[0];
    }
    Wn[x] = rho;
    Wn[x + fs] = vv[0];
    Wn[x + 2 * fs] = vv[1];
    Wn[x + 3 * fs] = vv[2];
    Wn[x + 4 * fs] = p;
    Wn[x + 5 * fs] = pS;
    // CFL dt of the new state (magtot = mags^{n+1}) and max|div B^{n+1}|
    dtc = cfl_cell<COORD>(P, i, j, k, rho, vv[0], vv[1], vv[2], p, bu[0], bu[1], bu[2]);
    double dvb = 0.0;
#pragma unroll
    for (int a = 0; a < 3; a++) {
      int i1 = i + (a == 0), j1 = j + (a == 1), k1 = k + (a == 2);
      // bu was overwritten with mags; recompute the upper face
      double up = ct_face<COORD, R>(P, B, E, a, i1, j1, k1, dt);
      dvb += (up * Geo<COORD>::face(P, a, i1, j1, k1) - bl[a] * Geo<COORD>::face(P, a, i, j, k)) / vol;
    }
    dbmax = fabs(dvb);
    if (!(dtc > 0.0) || !isfinite(p) || !isfinite(rho) || !isfinite(vv[0] + vv[1] + vv[2]))
      P.scal[S_FLAGS] = 1.0;
  }
  block_commit(dtc, dbmax, P.scal + S_NEXT_DT, P.scal + S_DIVB);
}

// ---------------------------------------------------------------- ghosts

// Periodic wrap of one axis for all 9 state fields (src/boundary_exchange.c,
// index sets of src/setup_mpi.c:62-253), over the full transverse extent.
__global__ void k_wrap(Params P, int axis, int which) {
  if (stopped(P)) return;
  const int bsel = which ? cur_buf(P) : 1 - cur_buf(P);
  double* __restrict__ W = P.Wbuf[bsel];
  double* __restrict__ B = P.Bbuf[bsel];
  int oa = (axis + 1) % 3, ob = (axis + 2) % 3;
  int t = blockIdx.x * blockDim.x + threadIdx.x;  // transverse index a
  int u = blockIdx.y * blockDim.y + threadIdx.y;  // transverse index b
  int g = blockIdx.z;                             // 0..2*NGH-1
  if (t >= P.N[oa] || u >= P.N[ob]) return;
  int N = P.N[axis];
  int side = g / NGH, l = g % NGH;
  int ijk[3];
  ijk[oa] = t;
  ijk[ob] = u;
  for (int f = 0; f < 9; f++) {
    int onface = (f >= 6 && f - 6 == axis) ? 1 : 0;
    double* a = f < 6 ? W + (size_t)f * P.fs : B + (size_t)(f - 6) * P.fs;
    int src, dst;
    if (side == 0) {  // high ghosts <- low active
      src = NGH + onface + l;
      dst = N - NGH - 1 + onface + l;
    } else {          // low ghosts <- high active
      src = N - 2 * NGH - 1 + l;
      dst = l;
    }
    ijk[axis] = src;
    double v = a[lin(P, ijk[0], ijk[1], ijk[2])];
    ijk[axis] = dst;
    a[lin(P, ijk[0], ijk[1], ijk[2])] = v;
  }
}

// One face of the ghost-fill library (src/boundary_conditions.c): the 6 gas
// primitives with kind `kind` (gas_bc_*) and the 3 face fields with kind
// `gkind` (gem_bc_*); 0 skips that group.
__global__ void k_bcface(Params P, int axis, int side, int kind, int gkind, int which) {
  if (stopped(P)) return;
  const int bsel = which ? cur_buf(P) : 1 - cur_buf(P);
  double* __restrict__ W = P.Wbuf[bsel];
  double* __restrict__ B = P.Bbuf[bsel];
  int oa = (axis + 1) % 3, ob = (axis + 2) % 3;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int u = blockIdx.y * blockDim.y + threadIdx.y;
  int l = blockIdx.z;
  if (t >= P.N[oa] || u >= P.N[ob]) return;
  int N = P.N[axis];
  int ijk[3];
  ijk[oa] = t;
  ijk[ob] = u;
  for (int f = 0; f < 9; f++) {
    bool gas = f < 6;
    int kd = gas ? kind : gkind;
    if (kd == 0 || kd == 'n' || kd == 'p') continue;
    if (!gas && kd == 'r') continue;  // gem_bc_reflective_* are empty
    int onface = (!gas && f - 6 == axis) ? 1 : 0;
    double* a = gas ? W + (size_t)f * P.fs : B + (size_t)(f - 6) * P.fs;
    int dst = side == 0 ? l : N - 1 - NGH + l + onface;
    double v;
    if (kd == 'f') {
      if (gas) {
        if (f == PS) continue;
        if (f == RHO) v = (axis == 1 && side == 0) ? 2.0 : 1.0;
        else if (f == PR) v = (axis == 1 && side == 1) ? 2.5 : 1.0;
        else v = 0.0;
      } else {
        v = 0.0;
      }
    } else {
      int src;
      if (kd == 'e') src = side == 0 ? NGH : N - 1 - NGH - 1 + onface;
      else src = side == 0 ? 2 * NGH - 1 - l + onface : N - 1 - NGH - 1 - l;
      ijk[axis] = src;
      v = a[lin(P, ijk[0], ijk[1], ijk[2])];
      if (kd == 'r' && gas && f == V1 + axis) v = -v;
    }
    ijk[axis] = dst;
    a[lin(P, ijk[0], ijk[1], ijk[2])] = v;
  }
}

// ------------------------------------------------------ layout transposes

// reference layout [f][i][j][k] (k fastest) <-> device layout
__global__ void k_from_ref(Params P, int nf, const double* __restrict__ src, double* __restrict__ dst) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int kf = blockIdx.z;
  int k = kf % P.N[2], f = kf / P.N[2];
  if (i >= P.N[0] || j >= P.N[1] || f >= nf) return;
  size_t r = (((size_t)f * P.N[0] + i) * P.N[1] + j) * P.N[2] + k;
  dst[(size_t)f * P.fs + lin(P, i, j, k)] = src[r];
}

__global__ void k_to_ref(Params P, int nf, const double* __restrict__ src, double* __restrict__ dst) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int kf = blockIdx.z;
  int k = kf % P.N[2], f = kf / P.N[2];
  if (i >= P.N[0] || j >= P.N[1] || f >= nf) return;
  size_t r = (((size_t)f * P.N[0] + i) * P.N[1] + j) * P.N[2] + k;
  dst[r] = src[(size_t)f * P.fs + lin(P, i, j, k)];
}

template <typename R>
__global__ void k_widen(Params P, int nf, const R* __restrict__ src, double* __restrict__ dst) {
  size_t n = (size_t)nf * P.fs;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
    dst[t] = (double)src[t];
}

// mags over the ghost range from face fields (for downloads)
__global__ void k_mags(Params P, const double* __restrict__ B, double* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= P.N[0] - 1 || j >= P.N[1] - 1 || k >= P.N[2] - 1) return;
  long long x = lin(P, i, j, k);
  for (int a = 0; a < 3; a++) out[x + a * P.fs] = mags_at(P, B, a, i, j, k);
}

// ----------------------------------------------------------- launchers

static int64_t g_launches = 0;
int64_t launches() { return g_launches; }

static dim3 grid3(int a, int b, int c, dim3 blk) {
  return dim3((a + blk.x - 1) / blk.x, (b + blk.y - 1) / blk.y, (c + blk.z - 1) / blk.z);
}

#define LAUNCH(kern, grd, blk, st, ...)            \
  do {                                             \
    kern<<<grd, blk, 0, st>>>(__VA_ARGS__);        \
    g_launches++;                                  \
  } while (0)

void launch_begin(const Params& P, cudaStream_t st) { LAUNCH(k_begin, 1, 1, st, P); }
void launch_end(const Params& P, cudaStream_t st) { LAUNCH(k_end, 1, 1, st, P); }
void launch_arm(const Params& P, double tstop, cudaStream_t st) { LAUNCH(k_arm, 1, 1, st, P, tstop); }

void launch_dt(const Params& P, int coord, cudaStream_t st) {
  dim3 blk(32, 4, 2);
  dim3 g = grid3(P.n[0], P.n[1], P.n[2], blk);
  if (coord == 0) LAUNCH(k_dt<0>, g, blk, st, P);
  else LAUNCH(k_dt<2>, g, blk, st, P);
}

template <typename R>
void launch_step_body(const Params& P, int coord, const Work<R>& w, cudaStream_t st,
                      const Hook& hook) {
  dim3 blk(32, 4, 2);
  hook(G_AB2, 1);
  LAUNCH(k_ab2<R>, grid3(P.N[0], P.N[1], P.N[2], blk), blk, st, P, w);
  hook(G_AB2, 0);
  hook(G_C2C, 1);
  for (int d = 0; d < 3; d++) {
    int p = (d + 1) % 3, q = (d + 2) % 3;
    int cnt[3];
    cnt[d] = P.n[d];
    cnt[p] = P.n[p] + 1;
    cnt[q] = P.n[q] + 2 * NGH;
    LAUNCH(k_c2c<R>, grid3(cnt[0], cnt[1], cnt[2], blk), blk, st, P, d, w);
  }
  hook(G_C2C, 0);
  hook(G_EMF, 1);
  for (int d = 0; d < 3; d++) {
    int p = (d + 1) % 3, q = (d + 2) % 3;
    int cnt[3];
    cnt[d] = P.n[d];
    cnt[p] = P.n[p] + 1;
    cnt[q] = P.n[q] + 1;
    LAUNCH(k_emf<R>, grid3(cnt[0], cnt[1], cnt[2], blk), blk, st, P, d, w);
  }
  hook(G_EMF, 0);
  hook(G_FLUX, 1);
  for (int d = 0; d < 3; d++) {
    int cnt[3] = {P.n[0], P.n[1], P.n[2]};
    cnt[d] += 1;
    LAUNCH(k_flux<R>, grid3(cnt[0], cnt[1], cnt[2], blk), blk, st, P, d, w);
  }
  hook(G_FLUX, 0);
  hook(G_UPDATE, 1);
  dim3 ub(32, 4, 2);
  if (coord == 0)
    LAUNCH((k_update<0, R>), grid3(P.n[0], P.n[1], P.n[2], ub), ub, st, P, w);
  else
    LAUNCH((k_update<2, R>), grid3(P.n[0], P.n[1], P.n[2], ub), ub, st, P, w);
  hook(G_UPDATE, 0);
}

template void launch_step_body<double>(const Params&, int, const Work<double>&, cudaStream_t,
                                       const Hook&);
template void launch_step_body<float>(const Params&, int, const Work<float>&, cudaStream_t,
                                      const Hook&);

void launch_ghosts(const Params& P, const char bc[6], const char gem_bc[6], int which,
                   cudaStream_t st) {
  dim3 blk(32, 8, 1);
  bool periodic[3];
  for (int a = 0; a < 3; a++) periodic[a] = bc[2 * a] == 'p' && bc[2 * a + 1] == 'p';
  for (int a = 0; a < 3; a++) {
    if (!periodic[a]) continue;
    int oa = (a + 1) % 3, ob = (a + 2) % 3;
    dim3 g((P.N[oa] + blk.x - 1) / blk.x, (P.N[ob] + blk.y - 1) / blk.y, 2 * NGH);
    // both sides in one launch: sources (active layers) and destinations
    // (ghost layers) are disjoint for n >= NGH
    LAUNCH(k_wrap, g, blk, st, P, a, which);
  }
  for (int face = 0; face < 6; face++) {
    int a = face / 2, side = face % 2;
    char kind = bc[face], gkind = gem_bc[face];
    if (periodic[a]) continue;
    bool gas_work = kind != 'n';
    bool gem_work = gkind != 'n' && gkind != 'r';
    if (!gas_work && !gem_work) continue;
    int oa = (a + 1) % 3, ob = (a + 2) % 3;
    dim3 g((P.N[oa] + blk.x - 1) / blk.x, (P.N[ob] + blk.y - 1) / blk.y, NGH);
    LAUNCH(k_bcface, g, blk, st, P, a, side, (int)kind, (int)gkind, which);
  }
}

void launch_from_ref(const Params& P, int nf, const double* src, double* dst, cudaStream_t st) {
  dim3 blk(32, 8, 1);
  dim3 g((P.N[0] + 31) / 32, (P.N[1] + 7) / 8, P.N[2] * nf);
  LAUNCH(k_from_ref, g, blk, st, P, nf, src, dst);
}

void launch_to_ref(const Params& P, int nf, const double* src, double* dst, cudaStream_t st) {
  dim3 blk(32, 8, 1);
  dim3 g((P.N[0] + 31) / 32, (P.N[1] + 7) / 8, P.N[2] * nf);
  LAUNCH(k_to_ref, g, blk, st, P, nf, src, dst);
}

template <typename R>
void launch_widen(const Params& P, int nf, const R* src, double* dst, cudaStream_t st) {
  LAUNCH(k_widen<R>, 1184, 256, st, P, nf, src, dst);
}
template void launch_widen<double>(const Params&, int, const double*, double*, cudaStream_t);
template void launch_widen<float>(const Params&, int, const float*, double*, cudaStream_t);

void launch_mags(const Params& P, const double* B, double* out, cudaStream_t st) {
  dim3 blk(32, 4, 2);
  LAUNCH(k_mags, grid3(P.N[0], P.N[1], P.N[2], blk), blk, st, P, B, out);
}

}  // namespace gop

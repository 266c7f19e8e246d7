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
//   end       the written buffer becomes the current state
//
// Every stage is a per-point body function of a kernel whose launch grid
// covers one grid; a batch of grids captures each member's launches on
// parallel branches of one CUDA graph.
//
// R is the arithmetic type of the reconstruction / flux / EMF stages
// (double: plain path; float: mixed path).  The state, the AB2
// extrapolation, the conservative update and the pressure recovery are FP64
// in both.
#include "gop_device.cuh"
#include "gop_kernels.h"
#include "gop_stage.cuh"

#include <algorithm>
#include <type_traits>
#include <atomic>
#include <cfloat>

namespace gop {

// Options of the mixed path's Cartesian update (0: FP32 as documented): run
// the flux divergence, the Alfven/Boris correction or the CFL estimate in
// FP64 instead
#ifndef GOP_MX_DIV64
#define GOP_MX_DIV64 0
#endif
#ifndef GOP_MX_ALF64
#define GOP_MX_ALF64 0
#endif
#ifndef GOP_MX_CFL64
#define GOP_MX_CFL64 0
#endif

// ------------------------------------------------------------------ utils


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

// block-wide min and max of (a, b); one thread commits them with one atomic each
__device__ __forceinline__ void block_commit(double a, double b, double* smin, double* smax) {
  __shared__ double sa[32], sb[32];
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nw = (blockDim.x * blockDim.y * blockDim.z + 31) / 32;
  const int w = tid / 32, lane = tid & 31;
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

// CFL time step of one cell (src/solver_func.c:255-298), in T arithmetic
// (FP32 for the mixed path's estimate)
template <int COORD, typename T = double>
__device__ __forceinline__ double cfl_cell(const Params& P, int i, int j, int k, double rho,
                                           double u, double v, double w, double p, double b1,
                                           double b2, double b3) {
  const T r = (T)rho, x1 = (T)b1, x2 = (T)b2, x3 = (T)b3, ut = (T)u, vt = (T)v, wt = (T)w;
  T bsq = x1 * x1 + x2 * x2 + x3 * x3;
  T va = sqrt(bsq / r);
  T vae = va * (T)P.ca / sqrt(va * va + (T)P.ca2);
  T vf = sqrt(ut * ut + vt * vt + wt * wt);
  T vs = sqrt((T)P.gamma * (T)p / r);
  T vc = vf + sqrt(vs * vs + vae * vae);
  T dk = (T)Geo<COORD>::dl(P, 2, i, j, k);
  // the phi length of the pole rings is nk / nchunk times longer (dxk_ring,
  // spherical_RingAverage.c:110-138; get_dt_ring, spherical_general.c:700-743)
  if (COORD == 2 && P.ring) dk = (T)P.ringtab[2 * P.n[2] + j] * dk;
  T t = vc / (T)Geo<COORD>::dl(P, 0, i, j, k) + vc / (T)Geo<COORD>::dl(P, 1, i, j, k) + vc / dk;
  return (double)((T)P.cfl / t);
}

// rows of cells whose state or face field the pole ring average changes
// (the ring rows and the rows of the faces its EMF-like field touches)
__device__ __forceinline__ bool ring_band_row(const Params& P, int j) {
  const int jm = P.ring_jmax;
  return ((P.ring & 1) && j >= NGH && j <= NGH + jm + 1) ||
         ((P.ring & 2) && j >= NGH + P.n[1] - 2 - jm && j <= NGH + P.n[1] - 1);
}

// cell-centred B from the two faces along each axis (src/solver_func.c:311-322)
__device__ __forceinline__ double mags_at(const Params& P, const double* B, int a, int i, int j,
                                          int k) {
  long long c = lin(P, i, j, k);
  int idx = a == 0 ? i : (a == 1 ? j : k);
  const double* f = B + (size_t)a * P.fs;
  return f[c] * tb(P, a, T_MA, idx) + f[c + stride(P, a)] * tb(P, a, T_MB, idx);
}

template <int AX>
__device__ __forceinline__ long long sd(const Params& P) {
  return AX == 0 ? 1LL : (AX == 1 ? P.sj : P.sk);
}

// v[0..7] = a[(t-4)*s]: cells f-4..f+3 along stride s, a pointing at cell f
template <typename R, typename T>
__device__ __forceinline__ void line8(const T* __restrict__ a, long long s, R v[8]) {
#pragma unroll
  for (int t = 0; t < 8; t++) v[t] = (R)a[(t - 4) * s];
}



// thread coordinates in a launch space
struct Pos {
  int x, y, z;
};
__device__ __forceinline__ Pos grid_pos() {
  return {(int)(blockIdx.x * blockDim.x + threadIdx.x), (int)(blockIdx.y * blockDim.y + threadIdx.y),
          (int)(blockIdx.z * blockDim.z + threadIdx.z)};
}
// ---------------------------------------------------------- step control

// open the step (src/solver_solve.c:103-107, src/solver_func.c:385-491):
// dt from the running CFL minimum, time, AB2 coefficient; stop once the
// previous step passed time_stop or the step budget is spent
__device__ __forceinline__ void begin_body(const Params& P) {
  double* s = P.scal;
  if (s[S_STOP] != 0.0) return;
  if (s[S_TIME] > s[S_TSTOP] || s[S_BUDGET] <= 0.0) {
    s[S_STOP] = 1.0;
    return;
  }
  s[S_BUDGET] = s[S_BUDGET] - 1.0;
  const double dt = s[S_NEXT_DT];
  if (!(dt > 0.0) || !isfinite(dt)) s[S_FLAGS] = 1.0;
  s[S_DT] = dt;
  s[S_TIME] = s[S_TIME] + dt;
  s[S_CAB2] = 0.5 * dt / s[S_DT0];
  s[S_DT0] = dt;
  s[S_NEXT_DT] = DBL_MAX;
  s[S_DIVB] = 0.0;
  s[S_STEPS] = s[S_STEPS] + 1.0;
}

// close the step: the buffer written by this step becomes the current state
__device__ __forceinline__ void end_body(const Params& P) {
  if (P.scal[S_STOP] != 0.0) return;
  P.scal[S_PAR] = P.scal[S_PAR] != 0.0 ? 0.0 : 1.0;
}

__device__ __forceinline__ void arm_body(const Params& P, double tstop, double budget) {
  P.scal[S_TSTOP] = tstop;
  P.scal[S_BUDGET] = budget;
  P.scal[S_STOP] = 0.0;
}

// ------------------------------------------------------------------- AB2

// W_h = W + c (W - W_old), mags and mags_h from the faces, B_h on faces
// (src/solver_func.c:385-449) over the whole ghost-extended grid; PSL false:
// p_S and its extrapolation stay zero (Params::ps_live) and are not touched
template <typename R, bool PSL>
__device__ __forceinline__ void ab2_body(const Params& P, const Work<R>& w, Pos t) {
  const int i = t.x, j = t.y, k = t.z;
  if (i >= P.N[0] || j >= P.N[1] || k >= P.N[2]) return;
  const int cb = cur_buf(P);
  const double* __restrict__ W = P.Wbuf[cb];
  const double* __restrict__ Wo = P.Wbuf[1 - cb];
  const double* __restrict__ B = P.Bbuf[cb];
  const double* __restrict__ Bo = P.Bbuf[1 - cb];
  const double c = P.scal[S_CAB2];
  const long long x = lin(P, i, j, k);
  const size_t fs = P.fs;
  const bool ci = i < P.N[0] - 1, cj = j < P.N[1] - 1, ck = k < P.N[2] - 1;
  // all loads first, then the stores: with FP64 work arrays the compiler
  // cannot tell them from the state, and a store between two loads would
  // keep the second from being issued ahead
  constexpr int NW = PSL ? 6 : 5;
  const bool inner = ci && cj && ck;
  double v[NW], vo[NW], ms[3], mo[3], b[3], bo[3];
  bool ok[3];
  if (inner) {
#pragma unroll
    for (int m = 0; m < NW; m++) {
      v[m] = W[x + m * fs];
      vo[m] = Wo[x + m * fs];
    }
#pragma unroll
    for (int a = 0; a < 3; a++) {
      ms[a] = mags_at(P, B, a, i, j, k);
      mo[a] = mags_at(P, Bo, a, i, j, k);
    }
  }
#pragma unroll
  for (int a = 0; a < 3; a++) {
    ok[a] = (a == 0 || ci) && (a == 1 || cj) && (a == 2 || ck);
    if (ok[a]) {
      b[a] = B[x + a * fs];
      bo[a] = Bo[x + a * fs];
    }
  }
  if (inner) {
#pragma unroll
    for (int m = 0; m < NW; m++) {
      w.Wh[x + m * fs] = (R)(v[m] + c * (v[m] - vo[m]));
      if constexpr (sizeof(R) == 4) w.Wl[x + m * fs] = (R)v[m];
    }
#pragma unroll
    for (int a = 0; a < 3; a++) {
      w.Ms[x + a * fs] = (R)ms[a];
      w.Msh[x + a * fs] = (R)(ms[a] + c * (ms[a] - mo[a]));
    }
  }
#pragma unroll
  for (int a = 0; a < 3; a++) {
    if (ok[a]) {
      w.Bh[x + a * fs] = (R)(b[a] + c * (b[a] - bo[a]));
      if constexpr (sizeof(R) == 4) w.Bl[x + a * fs] = (R)b[a];
    }
  }
}

// ------------------------------------------------------------- edge EMF

// First centre-to-edge sweep of center2corner_{jk,ki,ij}
// (src/solver_func.c:686-778): for edges along D, velocity components
// p=(D+1)%3 and q=(D+2)%3 reconstructed along p (limiter on the step-start
// velocity) and averaged, at D active, p faces lo..hi+1, q over all cells
// including ghosts.  Over the active q range these are exactly the
// velocity states the face flux along p reconstructs (same inputs, same
// weights), so the flux stage writes them there and this kernel covers only
// the 2*NGH ghost layers of q.
template <typename R, int D>
__device__ __forceinline__ void c2c_body(const Params& P, const Work<R>& wk, Pos t) {
  constexpr int p = (D + 1) % 3, q = (D + 2) % 3;
  int ijk[3] = {t.x, t.y, t.z};
  int cnt[3], lo[3];
  lo[D] = NGH; cnt[D] = P.n[D];
  lo[p] = NGH; cnt[p] = P.n[p] + 1;
  lo[q] = 0;   cnt[q] = 2 * NGH;
  if (ijk[0] >= cnt[0] || ijk[1] >= cnt[1] || ijk[2] >= cnt[2]) return;
  if (ijk[q] >= NGH) ijk[q] += P.n[q];  // upper ghost layers
  const int i = ijk[0] + lo[0], j = ijk[1] + lo[1], k = ijk[2] + lo[2];
  const int f = p == 0 ? i : (p == 1 ? j : k);
  const long long x = lin(P, i, j, k), s = sd<p>(P);
  const size_t fs = P.fs;
  const R* __restrict__ W = lim_w<R>(P, wk) + x;
  FaceWeights<R> Wt;
  load_face_weights<p, R>(wk.tab, wk.fw, P.tmax, f, Wt);
  const R a1h = (R)(0.5 * P.pdm_a1), a2 = (R)P.pdm_a2;
#pragma unroll
  for (int cc = 0; cc < 2; cc++) {
    const int comp = cc == 0 ? p : q;
    R v[8], lim[4], L, Rr;
    line8<R, R>(wk.Wh + (size_t)(V1 + comp) * fs + x, s, v);
#pragma unroll
    for (int u = 0; u < 4; u++) lim[u] = W[(V1 + comp) * fs + (u - 2) * s];
    recon_lr<R>(v, lim, Wt, a1h, a2, L, Rr);
    wk.V[x + (size_t)(2 * D + cc) * fs] = R(0.5) * (L + Rr);
  }
}

// Second sweep, face-field reconstruction and the edge EMF
// (src/solver_func.c:779-902) for edges along D: D active, p and q faces.
template <typename R, int D, bool BG>
__device__ __forceinline__ void emf_body(const Params& P, const Work<R>& wk, Pos t) {
  constexpr int p = (D + 1) % 3, q = (D + 2) % 3;
  const int ijk[3] = {t.x, t.y, t.z};
  int cnt[3];
  cnt[D] = P.n[D];
  cnt[p] = P.n[p] + 1;
  cnt[q] = P.n[q] + 1;
  if (ijk[0] >= cnt[0] || ijk[1] >= cnt[1] || ijk[2] >= cnt[2]) return;
  const int i = ijk[0] + NGH, j = ijk[1] + NGH, k = ijk[2] + NGH;
  const int pos[3] = {i, j, k};
  const long long x = lin(P, i, j, k), sp = sd<p>(P), sq = sd<q>(P);
  const size_t fs = P.fs;
  const R* __restrict__ B = lim_b<R>(P, wk) + x;
  const R a1h = (R)(0.5 * P.pdm_a1), a2 = (R)P.pdm_a2;
  R vav[2], bpl, bpr, bql, bqr;
  {
    FaceWeights<R> Wt;
    load_face_weights<q, R>(wk.tab, wk.fw, P.tmax, pos[q], Wt);
#pragma unroll
    for (int cc = 0; cc < 2; cc++) {
      R v[8], lim[4], L, Rr;
      line8<R, R>(wk.V + (size_t)(2 * D + cc) * fs + x, sq, v);
#pragma unroll
      for (int u = 0; u < 4; u++) lim[u] = v[u + 2];
      recon_lr<R>(v, lim, Wt, a1h, a2, L, Rr);
      vav[cc] = R(0.5) * (L + Rr);
    }
    // B_p along q
    R v[8], lim[4];
    line8<R, R>(wk.Bh + (size_t)p * fs + x, sq, v);
#pragma unroll
    for (int u = 0; u < 4; u++) lim[u] = B[p * fs + (u - 2) * sq];
    recon_lr<R>(v, lim, Wt, a1h, a2, bpl, bpr);
  }
  {
    // B_q along p
    FaceWeights<R> Wt;
    load_face_weights<p, R>(wk.tab, wk.fw, P.tmax, pos[p], Wt);
    R v[8], lim[4];
    line8<R, R>(wk.Bh + (size_t)q * fs + x, sp, v);
#pragma unroll
    for (int u = 0; u < 4; u++) lim[u] = B[q * fs + (u - 2) * sp];
    recon_lr<R>(v, lim, Wt, a1h, a2, bql, bqr);
  }
  R b0p = R(0), b0q = R(0);
  if constexpr (BG) {  // B0 averaged along the edge (B0Aedge*)
    b0p = (R)P.bg[(size_t)(BG_EDGE + 3 * D + p) * fs + x];
    b0q = (R)P.bg[(size_t)(BG_EDGE + 3 * D + q) * fs + x];
  }
  const R* rh = wk.Wh + x;  // density slot
  // the reference sums the four densities around the edge in (i,j,k) order
  const R rho4 = D == 1 ? rh[-sq - sp] + rh[-sq] + rh[-sp] + rh[0]
                        : rh[-sp - sq] + rh[-sp] + rh[-sq] + rh[0];
  const R e = emf_finish<R, BG>(P, vav[0], vav[1], bpl, bpr, bql, bqr, b0p, b0q, rho4);
  wk.E[x + (size_t)D * fs] = e;
}

// ------------------------------------------------------------ face flux


// PDM reconstruction of the 9 face states, then flux_out: one thread per face
// (PSL: the entropy channel p_S is live, Params::ps_live)
template <typename R, int D, bool BG, bool PSL>
__device__ __forceinline__ void flux_body(const Params& P, const Work<R>& wk, Pos t) {
  const int i = NGH + t.x, j = NGH + t.y, k = NGH + t.z;
  if (i >= NGH + P.n[0] + (D == 0) || j >= NGH + P.n[1] + (D == 1) ||
      k >= NGH + P.n[2] + (D == 2))
    return;
  const int f = D == 0 ? i : (D == 1 ? j : k);
  const long long x = lin(P, i, j, k), s = sd<D>(P);
  const size_t fs = P.fs;
  const R* __restrict__ W = lim_w<R>(P, wk) + x;
  FaceWeights<R> Wt;
  load_face_weights<D, R>(wk.tab, wk.fw, P.tmax, f, Wt);
  const R a1h = (R)(0.5 * P.pdm_a1), a2 = (R)P.pdm_a2;
  R L[6], Rt[6], mL[3], mR[3];
  // PSL false: p_S is identically zero (Params::ps_live), its face states
  // are zero and flux_out's zero path gives the zero entropy flux that
  // reconstructing the zero line would give
  L[PS] = Rt[PS] = R(0);
#pragma unroll
  for (int m = 0; m < 6; m++) {
    if (m == PS && !PSL) continue;
    R v[8], lim[4];
    line8<R, R>(wk.Wh + (size_t)m * fs + x, s, v);
#pragma unroll
    for (int u = 0; u < 4; u++) lim[u] = W[m * fs + (u - 2) * s];
    recon_lr<R>(v, lim, Wt, a1h, a2, L[m], Rt[m]);
  }
#pragma unroll
  for (int a = 0; a < 3; a++) {
    R v[8], lim[4];
    line8<R, R>(wk.Msh + (size_t)a * fs + x, s, v);
    const R* ms = wk.Ms + (size_t)a * fs + x;
#pragma unroll
    for (int u = 0; u < 4; u++) lim[u] = ms[(u - 2) * s];
    recon_lr<R>(v, lim, Wt, a1h, a2, mL[a], mR[a]);
  }
  flux_out<R, D, BG, PSL>(P, wk, x, L, Rt, mL, mR, lim_b<R>(P, wk)[x + D * fs]);
}

// --------------------------------------------------------------- update

// new face field of component A at face (i,j,k) by constrained transport
// (src/solver_solve.c:263-306)
template <int COORD, int A, typename R>
__device__ __forceinline__ double ct_face(const Params& P, const double* __restrict__ B,
                                          const R* __restrict__ E, int i, int j, int k,
                                          double dt) {
  constexpr int p = (A + 1) % 3, q = (A + 2) % 3;
  const long long x = lin(P, i, j, k), sp = sd<p>(P), sq = sd<q>(P);
  const int ip = i + (p == 0), jp = j + (p == 1), kp = k + (p == 2);
  const int iq = i + (q == 0), jq = j + (q == 1), kq = k + (q == 2);
  const size_t fs = P.fs;
  const double cq = (double)E[x + sp + q * fs] * Geo<COORD>::edge(P, q, ip, jp, kp) -
                    (double)E[x + q * fs] * Geo<COORD>::edge(P, q, i, j, k);
  const double cp = (double)E[x + sq + p * fs] * Geo<COORD>::edge(P, p, iq, jq, kq) -
                    (double)E[x + p * fs] * Geo<COORD>::edge(P, p, i, j, k);
  return B[x + A * fs] - dt * (cq - cp) / Geo<COORD>::face(P, A, i, j, k);
}

// One active cell of a Cartesian grid (src/solver_solve.c:263-484 with the
// Cartesian geometry of src/cartesian/cartesian_general.c): every face of
// the cell has the area of its axis, every edge along axis a the length
// dx_a, and the geometric sources vanish, so the whole cell needs dx_i,
// dx_j, dx_k and one division.  Face fields, constrained transport, the
// conservative update and the pressure recovery are FP64; with R = float
// the flux divergence, the Alfven/Boris correction and the CFL estimate are
// FP32.  Returns the cell's CFL dt and |div B| of the new state.
template <typename R, bool BG, bool PSL>
__device__ __forceinline__ void update_cart(const Params& P, const Work<R>& wk, Pos t,
                                            double& dtc, double& dbmax) {
  // arithmetic of the stages the mixed path runs in FP32 (FP64 when their
  // option is on, and always on the plain path)
  using RD = typename std::conditional<sizeof(R) == 8 || GOP_MX_DIV64, double, R>::type;
  using RA = typename std::conditional<sizeof(R) == 8 || GOP_MX_ALF64, double, R>::type;
  using RC = typename std::conditional<sizeof(R) == 8 || GOP_MX_CFL64, double, R>::type;
  const int i = NGH + t.x, j = NGH + t.y, k = NGH + t.z;
  if (i >= NGH + P.n[0] || j >= NGH + P.n[1] || k >= NGH + P.n[2]) return;
  const size_t fs = P.fs;
  const double dt = P.scal[S_DT];
  const int cb = cur_buf(P);
  const double* __restrict__ W = P.Wbuf[cb];
  const double* __restrict__ B = P.Bbuf[cb];
  double* __restrict__ Wn = P.Wbuf[1 - cb];
  double* __restrict__ Bn = P.Bbuf[1 - cb];
  const long long x = lin(P, i, j, k), sj = P.sj, sk = P.sk;
  const double dx[3] = {tb(P, 0, T_DX, i), tb(P, 1, T_DX, j), tb(P, 2, T_DX, k)};
  const double A[3] = {dx[1] * dx[2], dx[0] * dx[2], dx[0] * dx[1]};
  const double ivol = 1.0 / (dx[0] * dx[1] * dx[2]);
  const double iA[3] = {dx[0] * ivol, dx[1] * ivol, dx[2] * ivol};  // 1/A_a
  const double il[3] = {A[0] * ivol, A[1] * ivol, A[2] * ivol};     // 1/dx_a

  // constrained transport: face A gets -dt (curl E)_A, from FP64 products
  // of the edge EMFs and edge lengths (src/solver_solve.c:263-306)
  const R* __restrict__ E = wk.E + x;
  auto ed = [&](int a, long long off) { return (double)E[a * fs + off] * dx[a]; };
  const double e0 = ed(0, 0), e1 = ed(1, 0), e2 = ed(2, 0);
  const double e0j = ed(0, sj), e0k = ed(0, sk), e1i = ed(1, 1), e1k = ed(1, sk);
  const double e2i = ed(2, 1), e2j = ed(2, sj);
  double bl[3], bu[3], mo[3];
  bl[0] = B[x] - dt * ((e2j - e2) - (e1k - e1)) * iA[0];
  bl[1] = B[x + fs] - dt * ((e0k - e0) - (e2i - e2)) * iA[1];
  bl[2] = B[x + 2 * fs] - dt * ((e1i - e1) - (e0j - e0)) * iA[2];
  {
    const double e1ik = ed(1, 1 + sk), e2ij = ed(2, 1 + sj), e0jk = ed(0, sj + sk);
    bu[0] = B[x + 1] - dt * ((e2ij - e2i) - (e1ik - e1i)) * iA[0];
    bu[1] = B[x + sj + fs] - dt * ((e0jk - e0j) - (e2ij - e2j)) * iA[1];
    bu[2] = B[x + sk + 2 * fs] - dt * ((e1ik - e1k) - (e0jk - e0k)) * iA[2];
  }
  // mags^n for the time-centred field
  mo[0] = B[x] * tb(P, 0, T_MA, i) + B[x + 1] * tb(P, 0, T_MB, i);
  mo[1] = B[x + fs] * tb(P, 1, T_MA, j) + B[x + sj + fs] * tb(P, 1, T_MB, j);
  mo[2] = B[x + 2 * fs] * tb(P, 2, T_MA, k) + B[x + sk + 2 * fs] * tb(P, 2, T_MB, k);
  // (stored here: keeping the six face values until after the flux loads
  // measured 8 % slower on B200, FP64 256^3, from the registers it holds)
  Bn[x] = bl[0];
  Bn[x + fs] = bl[1];
  Bn[x + 2 * fs] = bl[2];
  if (i == NGH + P.n[0] - 1) Bn[x + 1] = bu[0];
  if (j == NGH + P.n[1] - 1) Bn[x + sj + fs] = bu[1];
  if (k == NGH + P.n[2] - 1) Bn[x + sk + 2 * fs] = bu[2];
  if constexpr (BG) {  // div of B + B0 (face-normal B0, src/solver_func.c:324-343)
    const double* f0 = P.bg + (size_t)BG_FACE * fs + x;
    const double* f1 = P.bg + (size_t)(BG_FACE + 4) * fs + x;
    const double* f2 = P.bg + (size_t)(BG_FACE + 8) * fs + x;
    const double dvb = ((bu[0] + f0[1]) * A[0] - (bl[0] + f0[0]) * A[0]) * ivol +
                       ((bu[1] + f1[sj]) * A[1] - (bl[1] + f1[0]) * A[1]) * ivol +
                       ((bu[2] + f2[sk]) * A[2] - (bl[2] + f2[0]) * A[2]) * ivol;
    dbmax = fabs(dvb);
  } else {
    const double dvb = (bu[0] * A[0] - bl[0] * A[0]) * ivol + (bu[1] * A[1] - bl[1] * A[1]) * ivol +
                       (bu[2] * A[2] - bl[2] * A[2]) * ivol;
    dbmax = fabs(dvb);
  }
  // cell-centred B0 (magtot = mags + B0)
  double c0[3] = {0.0, 0.0, 0.0};
  if constexpr (BG) {
#pragma unroll
    for (int a = 0; a < 3; a++) c0[a] = P.bg[(size_t)(BG_B0 + a) * fs + x];
  }
  double mn[3], mt[3];
  mn[0] = bl[0] * tb(P, 0, T_MA, i) + bu[0] * tb(P, 0, T_MB, i);
  mn[1] = bl[1] * tb(P, 1, T_MA, j) + bu[1] * tb(P, 1, T_MB, j);
  mn[2] = bl[2] * tb(P, 2, T_MA, k) + bu[2] * tb(P, 2, T_MB, k);
#pragma unroll
  for (int a = 0; a < 3; a++) mt[a] = BG ? 0.5 * (mn[a] + mo[a]) + c0[a] : 0.5 * (mn[a] + mo[a]);

  // flux divergence: 6 hydro and 3 stress components (FP32 arithmetic on
  // the mixed path; the reference's F_u A - F_l A over the volume otherwise)
  RD du[6], dm[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const long long s = d == 0 ? 1LL : (d == 1 ? sj : sk);
    const R* __restrict__ Fd = wk.F + (size_t)(9 * d) * fs + x;
#pragma unroll
    for (int m = 0; m < 9; m++) {
      if (m == PS && !PSL) continue;
      RD v;
      if constexpr (sizeof(RD) == 4) {
        v = (Fd[s + m * fs] - Fd[m * fs]) * (R)il[d];
      } else {
        v = ((double)Fd[s + m * fs] * A[d] - (double)Fd[m * fs] * A[d]) * ivol;
      }
      if (m < 6) du[m] = d == 0 ? v : du[m] + v;
      else dm[m - 6] = d == 0 ? v : dm[m - 6] + v;
    }
  }
  if constexpr (BG) {  // + the Lorentz force of B0 (src/solver_solve.c:312-324)
#pragma unroll
    for (int a = 0; a < 3; a++) dm[a] += (RD)P.bg[(size_t)(BG_LOR + a) * fs + x];
  }

  // U^n from W^n, conservative update, cons->prim in FP64
  // (src/solver_func.c:356-382, src/solver_solve.c:326-377)
  const double gm1 = P.gm1;
  const double r0 = W[x], u0 = W[x + fs], v0 = W[x + 2 * fs], w0 = W[x + 3 * fs],
               p0 = W[x + 4 * fs];
  const double U0[3] = {r0 * u0, r0 * v0, r0 * w0};
  const double E0 = 0.5 * r0 * (u0 * u0 + v0 * v0 + w0 * w0) + p0 * P.inv_gm1;
  const double Ur = r0 - dt * (double)du[0];
  double Um[3];
#pragma unroll
  for (int a = 0; a < 3; a++) Um[a] = U0[a] - dt * (double)du[1 + a];
  const double Ue = E0 - dt * (double)du[4];
  double rho = Ur;
  const double irho = 1.0 / Ur;
  double vv[3] = {Um[0] * irho, Um[1] * irho, Um[2] * irho};
  double p = (Ue - 0.5 * (vv[0] * vv[0] + vv[1] * vv[1] + vv[2] * vv[2]) * rho) * gm1;
  double pS = 0.0;
  if constexpr (PSL) {  // entropy S = p_S / rho^(gamma-1), updated and back
    const double ps0 = W[x + 5 * fs];
    const double S0 = (ps0 == 0.0 && r0 > 0.0) ? ps0 : ps0 / pow(r0, gm1);
    const double Us = S0 - dt * (double)du[5];
    pS = (Us == 0.0 && Ur > 0.0) ? Us : Us * pow(Ur, gm1);
  }
  // positivity floors (src/solver_func.c:2117-2135)
  if (rho < P.rho_floor) {
    rho = P.rho_floor;
    p = P.p_floor;
  }
  if (p < P.p_floor) p = P.p_floor;

  // Alfven/Boris correction of the momentum (src/solver_solve.c:385-484)
  {
    const RA bsq = (RA)(mt[0] * mt[0] + mt[1] * mt[1] + mt[2] * mt[2]);
    const RA alf = bsq / ((RA)rho * (RA)P.ca2);
    const RA perp = RA(1) / (RA(1) + alf);
    const RA rdt = (RA)dt;
    const RA drho = -rdt * (RA)du[0];
    const RA dva = alf * drho;
    RA tv[3], wv[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      wv[a] = (RA)W[x + (1 + a) * fs];
      tv[a] = alf * (-rdt * (RA)du[1 + a] - drho * wv[a]);
    }
    RA bdv = (RA)mt[0] * tv[0] + (RA)mt[1] * tv[1] + (RA)mt[2] * tv[2];
    bdv = bdv / (bsq + RA(1e-10));
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const RA inc = perp * ((-rdt * (RA)du[1 + a]) + (-rdt * (RA)dm[a]) + dva * wv[a] + (RA)mt[a] * bdv);
      vv[a] = (U0[a] + (double)inc) * irho;
    }
  }
  Wn[x] = rho;
  Wn[x + fs] = vv[0];
  Wn[x + 2 * fs] = vv[1];
  Wn[x + 3 * fs] = vv[2];
  Wn[x + 4 * fs] = p;
  if constexpr (PSL) Wn[x + 5 * fs] = pS;  // else it stays zero in both buffers

  // CFL dt of the new state with magtot = mags^{n+1} (src/solver_func.c:255-298)
  {
    const RC r = (RC)rho, u = (RC)vv[0], v = (RC)vv[1], w = (RC)vv[2];
    const double t0 = mn[0] + c0[0], t1 = mn[1] + c0[1], t2 = mn[2] + c0[2];
    const RC bsq = BG ? (RC)(t0 * t0 + t1 * t1 + t2 * t2) : (RC)(mn[0] * mn[0] + mn[1] * mn[1] + mn[2] * mn[2]);
    const RC va = sqrt(bsq / r);
    const RC vae = va * (RC)P.ca / sqrt(va * va + (RC)P.ca2);
    const RC vf = sqrt(u * u + v * v + w * w);
    const RC vs = sqrt((RC)P.gamma * (RC)p / r);
    const RC vc = vf + sqrt(vs * vs + vae * vae);
    dtc = (double)((RC)P.cfl / (vc * (RC)il[0] + vc * (RC)il[1] + vc * (RC)il[2]));
  }
  if (!(dtc > 0.0) || !isfinite(p) || !isfinite(rho) || !isfinite(vv[0] + vv[1] + vv[2]))
    P.scal[S_FLAGS] = 1.0;
}

// Constrained transport of a curvilinear grid (src/solver_solve.c:263-306),
// its own launch before the update: every active cell writes its three lower
// faces, the last cell along an axis also the upper boundary face, so each
// face (with its division by the face area) is computed once
template <int COORD, typename R>
__device__ __forceinline__ void ct_body(const Params& P, const Work<R>& wk, Pos t) {
  const int i = NGH + t.x, j = NGH + t.y, k = NGH + t.z;
  if (i >= NGH + P.n[0] || j >= NGH + P.n[1] || k >= NGH + P.n[2]) return;
  const size_t fs = P.fs;
  const double dt = P.scal[S_DT];
  const int cb = cur_buf(P);
  const double* __restrict__ B = P.Bbuf[cb];
  double* __restrict__ Bn = P.Bbuf[1 - cb];
  const R* __restrict__ E = wk.E;
  const long long x = lin(P, i, j, k);
  const bool last[3] = {i == NGH + P.n[0] - 1, j == NGH + P.n[1] - 1, k == NGH + P.n[2] - 1};
  double bl[3], bu[3] = {0.0, 0.0, 0.0};
  bl[0] = ct_face<COORD, 0, R>(P, B, E, i, j, k, dt);
  bl[1] = ct_face<COORD, 1, R>(P, B, E, i, j, k, dt);
  bl[2] = ct_face<COORD, 2, R>(P, B, E, i, j, k, dt);
  if (last[0]) bu[0] = ct_face<COORD, 0, R>(P, B, E, i + 1, j, k, dt);
  if (last[1]) bu[1] = ct_face<COORD, 1, R>(P, B, E, i, j + 1, k, dt);
  if (last[2]) bu[2] = ct_face<COORD, 2, R>(P, B, E, i, j, k + 1, dt);
  if (COORD == 2 && P.ring) {
    // B_j on a pole face (zero area) from the face next to it and the one
    // half a turn away in phi (tackle_Magfield_pole,
    // spherical_RingAverage.c:205-233)
    const int ko = NGH + (k - NGH + P.n[2] / 2) % P.n[2];
    if ((P.ring & 1) && j == NGH)
      bl[1] = 0.5 * (ct_face<COORD, 1, R>(P, B, E, i, j + 1, k, dt) -
                     ct_face<COORD, 1, R>(P, B, E, i, j + 1, ko, dt));
    if ((P.ring & 2) && last[1])
      bu[1] = 0.5 * (bl[1] - ct_face<COORD, 1, R>(P, B, E, i, j, ko, dt));
  }
#pragma unroll
  for (int a = 0; a < 3; a++) {
    Bn[x + a * fs] = bl[a];
    if (last[a]) Bn[x + stride(P, a) + a * fs] = bu[a];
  }
}

// one active cell: returns its CFL dt and |div B| of the new state.  The
// flux divergence, the geometric sources, the Alfven/Boris correction and
// the CFL estimate are in R (FP32 on the mixed path); the face fields, the
// conservative update and the pressure recovery are FP64.
template <int COORD, typename R, bool BG, bool PSL>
__device__ __forceinline__ void update_body(const Params& P, const Work<R>& wk, Pos t,
                                            double& dtc, double& dbmax) {
  if constexpr (COORD == 0) {
    update_cart<R, BG, PSL>(P, wk, t, dtc, dbmax);
    return;
  }
  const int i = NGH + t.x, j = NGH + t.y, k = NGH + t.z;
  if (i >= NGH + P.n[0] || j >= NGH + P.n[1] || k >= NGH + P.n[2]) return;
  const size_t fs = P.fs;
  const double dt = P.scal[S_DT];
  const int cb = cur_buf(P);
  const double* __restrict__ W = P.Wbuf[cb];
  const double* __restrict__ B = P.Bbuf[cb];
  double* __restrict__ Wn = P.Wbuf[1 - cb];
  double* __restrict__ Bn = P.Bbuf[1 - cb];
  const R* __restrict__ F = wk.F;
  const long long x = lin(P, i, j, k);
  const double vol = Geo<COORD>::vol(P, i, j, k);
  const double ivol = 1.0 / vol;
  const R rivol = (R)ivol;
  R du[6], dm[3];
  double fl[3], fu[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const long long s = stride(P, d);
    const int i1 = i + (d == 0), j1 = j + (d == 1), k1 = k + (d == 2);
    fl[d] = Geo<COORD>::face(P, d, i, j, k);
    fu[d] = Geo<COORD>::face(P, d, i1, j1, k1);
    const R* Fd = F + (size_t)(9 * d) * fs + x;
#pragma unroll
    for (int m = 0; m < 6; m++) {
      if (m == PS && !PSL) continue;
      const R v = ((R)Fd[s + m * fs] * (R)fu[d] - (R)Fd[m * fs] * (R)fl[d]) * rivol;
      du[m] = d == 0 ? v : du[m] + v;
    }
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const R v = ((R)Fd[s + (6 + a) * fs] * (R)fu[d] - (R)Fd[(6 + a) * fs] * (R)fl[d]) * rivol;
      dm[a] = d == 0 ? v : dm[a] + v;
    }
  }
  if constexpr (BG) {  // + the Lorentz force of B0 (src/solver_solve.c:312-324)
#pragma unroll
    for (int a = 0; a < 3; a++) dm[a] += (R)P.bg[(size_t)(BG_LOR + a) * fs + x];
  }
  // spherical geometric sources (src/spherical/spherical_general.c:605-681)
  R sh[3] = {R(0), R(0), R(0)}, sb[3] = {R(0), R(0), R(0)};
  if (COORD == 2) {
    const long long si = 1, sjj = P.sj;
    const R fi0 = (R)fl[0], fi1 = (R)fu[0], fj0 = (R)fl[1], fj1 = (R)fu[1];
    const R dr = (R)tb(P, 0, T_DX, i), rc = (R)tb(P, 0, T_G3, i);
    const R* Wh = wk.Wh + x;
    const R ph = (R)Wh[PR * fs], rh = (R)Wh[RHO * fs], v2h = (R)Wh[V2 * fs], v3h = (R)Wh[V3 * fs];
    const R m22 = ph + rh * v2h * v2h, m33 = ph + rh * v3h * v3h;
    const R* Fi = F + x;
    const R* Fj = F + (size_t)9 * fs + x;
    const R geo = dr / rc / R(2) * rivol;
    sh[0] = R(0.5) * (m22 + m33) * (fi1 - fi0) * rivol;
    sh[1] = -((R)Fi[2 * fs] * fi0 + (R)Fi[si + 2 * fs] * fi1) * geo + (fj1 - fj0) * rivol * m33;
    sh[2] = -((R)Fi[3 * fs] * fi0 + (R)Fi[si + 3 * fs] * fi1) * geo;
    const R sr = (R)tb(P, 1, T_G3, j) / (R)tb(P, 1, T_G4, j) * rivol;
    sh[2] += -((R)Fj[3 * fs] * fj0 + (R)Fj[sjj + 3 * fs] * fj1) * sr;
    const R* Msh = wk.Msh + x;
    const R b1 = (R)Msh[0], b2 = (R)Msh[fs], b3 = (R)Msh[2 * fs];
    R bsq = b1 * b1 + b2 * b2 + b3 * b3;
    R n22 = R(0.5) * bsq - b2 * b2, n33 = R(0.5) * bsq - b3 * b3;
    if constexpr (BG) {  // with the B0 cross terms (spherical_general.c:634-638)
      const double* c0 = P.bg + (size_t)BG_B0 * fs + x;
      const R g1 = (R)c0[0], g2 = (R)c0[fs], g3 = (R)c0[2 * fs];
      bsq = b1 * b1 + b2 * b2 + b3 * b3 + R(2) * (b1 * g1 + b2 * g2 + b3 * g3);
      n22 = R(0.5) * bsq - (b2 + g2) * b2 - b2 * g2;
      n33 = R(0.5) * bsq - (b3 + g3) * b3 - b3 * g3;
    }
    sb[0] = R(0.5) * (n22 + n33) * (fi1 - fi0) * rivol;
    sb[1] = -((R)Fi[7 * fs] * fi0 + (R)Fi[si + 7 * fs] * fi1) * geo + (fj1 - fj0) * rivol * n33;
    sb[2] = -((R)Fi[8 * fs] * fi0 + (R)Fi[si + 8 * fs] * fi1) * geo;
    sb[2] += -((R)Fj[8 * fs] * fj0 + (R)Fj[sjj + 8 * fs] * fj1) * sr;
  }
  // the new face fields of this cell's lower and upper faces, written by
  // k_ct before this launch
  double bl[3], bu[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    bl[a] = Bn[x + a * fs];
    bu[a] = Bn[x + stride(P, a) + a * fs];
  }
  // U^n from W^n (src/solver_func.c:356-382)
  const double gm1 = P.gm1;
  const double r0 = W[x], u0 = W[x + fs], v0 = W[x + 2 * fs], w0 = W[x + 3 * fs],
               p0 = W[x + 4 * fs];
  double U[6];
  U[0] = r0;
  U[1] = r0 * u0;
  U[2] = r0 * v0;
  U[3] = r0 * w0;
  U[4] = 0.5 * r0 * (u0 * u0 + v0 * v0 + w0 * w0) + p0 * P.inv_gm1;
  U[5] = 0.0;
  if constexpr (PSL) {
    const double ps0 = W[x + 5 * fs];
    U[5] = (ps0 == 0.0 && r0 > 0.0) ? ps0 : ps0 / pow(r0, gm1);
  }
  const double U0[3] = {U[1], U[2], U[3]};
  // conservative update and cons->prim (src/solver_solve.c:326-377)
  U[0] -= dt * (double)du[0];
#pragma unroll
  for (int a = 0; a < 3; a++) U[1 + a] = U[1 + a] - dt * (double)du[1 + a] + dt * (double)sh[a];
  U[4] -= dt * (double)du[4];
  double rho = U[0];
  const double irho = 1.0 / U[0];
  double vv[3] = {U[1] * irho, U[2] * irho, U[3] * irho};
  double p = (U[4] - 0.5 * (vv[0] * vv[0] + vv[1] * vv[1] + vv[2] * vv[2]) * rho) * gm1;
  double pS = 0.0;
  if constexpr (PSL) {
    U[5] -= dt * (double)du[5];
    pS = (U[5] == 0.0 && U[0] > 0.0) ? U[5] : U[5] * pow(U[0], gm1);
  }
  // positivity floors (src/solver_func.c:2117-2135)
  if (rho < P.rho_floor) {
    rho = P.rho_floor;
    p = P.p_floor;
  }
  if (p < P.p_floor) p = P.p_floor;
  // mags^{n+1}, time-centred field, Alfven/Boris correction
  // (src/solver_solve.c:385-484)
  double mt[3], mn[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const int idx = a == 0 ? i : (a == 1 ? j : k);
    mn[a] = bl[a] * tb(P, a, T_MA, idx) + bu[a] * tb(P, a, T_MB, idx);
    mt[a] = 0.5 * (mn[a] + mags_at(P, B, a, i, j, k));
    if constexpr (BG) {  // magtot = mags + B0
      const double c0 = P.bg[(size_t)(BG_B0 + a) * fs + x];
      mt[a] += c0;
      mn[a] += c0;  // the next step's magtot, for its CFL dt
    }
  }
  const R mr[3] = {(R)mt[0], (R)mt[1], (R)mt[2]};
  const R bsq = mr[0] * mr[0] + mr[1] * mr[1] + mr[2] * mr[2];
  const R alf = bsq / (R)rho / (R)P.ca2;
  const R perp = R(1) / (R(1) + alf);
  const R rdt = (R)dt;
  const R drho = -rdt * du[0];
  const R dva = alf * drho;
  R tv[3], wv[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    wv[a] = (R)W[x + (1 + a) * fs];
    tv[a] = alf * (-rdt * du[1 + a] + rdt * sh[a] - drho * wv[a]);
  }
  R bdv = mr[0] * tv[0] + mr[1] * tv[1] + mr[2] * tv[2];
  bdv = bdv / (bsq + R(1e-10));
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const R inc = perp * ((-rdt * du[1 + a] + rdt * sh[a]) + (-rdt * dm[a] + rdt * sb[a]) +
                          dva * wv[a] + mr[a] * bdv);
    vv[a] = (U0[a] + (double)inc) * irho;
  }
  Wn[x] = rho;
  Wn[x + fs] = vv[0];
  Wn[x + 2 * fs] = vv[1];
  Wn[x + 3 * fs] = vv[2];
  Wn[x + 4 * fs] = p;
  if constexpr (PSL) Wn[x + 5 * fs] = pS;
  // CFL dt of the new state (magtot = mags^{n+1}) and max|div B^{n+1}|
  dtc = cfl_cell<COORD, R>(P, i, j, k, rho, vv[0], vv[1], vv[2], p, mn[0], mn[1], mn[2]);
  double b0l[3] = {0.0, 0.0, 0.0}, b0u[3] = {0.0, 0.0, 0.0};
  if constexpr (BG) {  // div of B + B0 (face-normal B0, src/solver_func.c:324-343)
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const double* f = P.bg + (size_t)(BG_FACE + 4 * a) * fs + x;
      b0l[a] = f[0];
      b0u[a] = f[stride(P, a)];
    }
  }
  const double dvb = ((bu[0] + b0u[0]) * fu[0] - (bl[0] + b0l[0]) * fl[0]) * ivol +
                     ((bu[1] + b0u[1]) * fu[1] - (bl[1] + b0l[1]) * fl[1]) * ivol +
                     ((bu[2] + b0u[2]) * fu[2] - (bl[2] + b0l[2]) * fl[2]) * ivol;
  dbmax = fabs(dvb);
  if (!(dtc > 0.0) || !isfinite(p) || !isfinite(rho) || !isfinite(vv[0] + vv[1] + vv[2]))
    P.scal[S_FLAGS] = 1.0;
  if (COORD == 2 && P.ring && ring_band_row(P, j)) {
    // the ring average still changes this row: k_ring_dt takes its CFL dt
    // and div B afterwards
    dtc = DBL_MAX;
    dbmax = 0.0;
  }
}

// CFL dt and |div B| of one cell of the current state (prepare).  The dt
// takes the form and arithmetic R of the step's own estimate (the
// Cartesian update's 1/dx from the face area over the volume; the FP32
// estimate on the mixed path; FP64 in the rows of the pole ring average),
// so a restarted run takes exactly the step the uninterrupted one would.
template <int COORD, bool BG, typename R>
__device__ __forceinline__ void dt_body(const Params& P, Pos t, double& dtc, double& db) {
  const int i = NGH + t.x, j = NGH + t.y, k = NGH + t.z;
  if (i >= NGH + P.n[0] || j >= NGH + P.n[1] || k >= NGH + P.n[2]) return;
  const double* __restrict__ W = P.Wbuf[cur_buf(P)];
  const double* __restrict__ B = P.Bbuf[cur_buf(P)];
  const long long c = lin(P, i, j, k);
  double b1 = mags_at(P, B, 0, i, j, k), b2 = mags_at(P, B, 1, i, j, k),
         b3 = mags_at(P, B, 2, i, j, k);
  if constexpr (BG) {  // magtot = mags + B0 (src/solver_func.c:345-353)
    b1 += P.bg[(size_t)BG_B0 * P.fs + c];
    b2 += P.bg[(size_t)(BG_B0 + 1) * P.fs + c];
    b3 += P.bg[(size_t)(BG_B0 + 2) * P.fs + c];
  }
  if constexpr (COORD == 0) {  // as update_cart
    using RC = typename std::conditional<sizeof(R) == 8 || GOP_MX_CFL64, double, R>::type;
    const double dx[3] = {tb(P, 0, T_DX, i), tb(P, 1, T_DX, j), tb(P, 2, T_DX, k)};
    const double A[3] = {dx[1] * dx[2], dx[0] * dx[2], dx[0] * dx[1]};
    const double ivol = 1.0 / (dx[0] * dx[1] * dx[2]);
    const double il[3] = {A[0] * ivol, A[1] * ivol, A[2] * ivol};
    const RC r = (RC)W[c], u = (RC)W[c + P.fs], v = (RC)W[c + 2 * P.fs], w = (RC)W[c + 3 * P.fs];
    const RC p = (RC)W[c + 4 * P.fs];
    const RC bsq = (RC)(b1 * b1 + b2 * b2 + b3 * b3);
    const RC va = sqrt(bsq / r);
    const RC vae = va * (RC)P.ca / sqrt(va * va + (RC)P.ca2);
    const RC vf = sqrt(u * u + v * v + w * w);
    const RC vs = sqrt((RC)P.gamma * p / r);
    const RC vc = vf + sqrt(vs * vs + vae * vae);
    dtc = (double)((RC)P.cfl / (vc * (RC)il[0] + vc * (RC)il[1] + vc * (RC)il[2]));
  } else if (P.ring && ring_band_row(P, j)) {  // as k_ring_dt
    dtc = cfl_cell<COORD>(P, i, j, k, W[c], W[c + P.fs], W[c + 2 * P.fs], W[c + 3 * P.fs],
                          W[c + 4 * P.fs], b1, b2, b3);
  } else {  // as the curvilinear update
    dtc = cfl_cell<COORD, R>(P, i, j, k, W[c], W[c + P.fs], W[c + 2 * P.fs], W[c + 3 * P.fs],
                             W[c + 4 * P.fs], b1, b2, b3);
  }
  const double vol = Geo<COORD>::vol(P, i, j, k);
  double d = 0.0;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const double* f = B + (size_t)a * P.fs;
    const long long s = stride(P, a);
    const int i1 = i + (a == 0), j1 = j + (a == 1), k1 = k + (a == 2);
    double bu = f[c + s], bl = f[c];
    if constexpr (BG) {
      const double* g = P.bg + (size_t)(BG_FACE + 4 * a) * P.fs;
      bu += g[c + s];
      bl += g[c];
    }
    d += (bu * Geo<COORD>::face(P, a, i1, j1, k1) - bl * Geo<COORD>::face(P, a, i, j, k)) / vol;
  }
  db = fabs(d);
}

// ---------------------------------------------------------------- ghosts

// Periodic wrap of one axis for all 9 state fields (src/boundary_exchange.c,
// index sets of src/setup_mpi.c:62-253), over the full transverse extent.
// Space: (N[oa], N[ob], 2*NGH); sources (active layers) and destinations
// (ghost layers) are disjoint for n >= NGH, so both sides go in one launch.
__device__ __forceinline__ void wrap_body(const Params& P, int axis, int which, Pos t) {
  // t = (i, j, k) with the component along `axis` replaced by the ghost
  // layer 0..2*NGH-1, so lanes run along i (along the layers for axis 0)
  int ijk[3] = {t.x, t.y, t.z};
  const int lay = ijk[axis];
  for (int a = 0; a < 3; a++)
    if (ijk[a] >= (a == axis ? 2 * NGH : P.N[a])) return;
  const int bsel = which ? cur_buf(P) : 1 - cur_buf(P);
  double* __restrict__ W = P.Wbuf[bsel];
  double* __restrict__ B = P.Bbuf[bsel];
  const int N = P.N[axis];
  const int side = lay / NGH, l = lay % NGH;
  // the sources are active cells and the destinations ghost cells, so no
  // thread writes what another reads: all 9 loads go out before the stores
  long long src[2], dst[2];  // [0]: cell-centred fields, [1]: the face field along axis
  for (int onface = 0; onface < 2; onface++) {
    if (side == 0) {  // high ghosts <- low active
      ijk[axis] = NGH + onface + l;
      src[onface] = lin(P, ijk[0], ijk[1], ijk[2]);
      ijk[axis] = N - NGH - 1 + onface + l;
    } else {          // low ghosts <- high active
      ijk[axis] = N - 2 * NGH - 1 + l;
      src[onface] = lin(P, ijk[0], ijk[1], ijk[2]);
      ijk[axis] = l;
    }
    dst[onface] = lin(P, ijk[0], ijk[1], ijk[2]);
  }
  const bool ps = P.ps_live != 0;  // p_S zero everywhere stays so: skipped
  double v[9];
#pragma unroll
  for (int f = 0; f < 9; f++) {
    const int o = (f >= 6 && f - 6 == axis) ? 1 : 0;
    const double* a = f < 6 ? W + (size_t)f * P.fs : B + (size_t)(f - 6) * P.fs;
    if (f != PS || ps) v[f] = a[src[o]];
  }
#pragma unroll
  for (int f = 0; f < 9; f++) {
    const int o = (f >= 6 && f - 6 == axis) ? 1 : 0;
    double* a = f < 6 ? W + (size_t)f * P.fs : B + (size_t)(f - 6) * P.fs;
    if (f != PS || ps) a[dst[o]] = v[f];
  }
}

// All three axes periodic: the three wraps above in one launch.  The three
// in turn leave at every ghost point the value of the active point reached
// by wrapping each of its ghost coordinates (x + n below the active range,
// x - n above it): each later wrap copies what the earlier ones wrote, edges
// and corners included.  Thread g runs over three slabs, axis a's 9 layers
// (4 ghost layers below, 5 points above: the cell fields' 4 ghost layers
// and the padding point, or the upper boundary face and the face field's 4
// ghost layers) times all points of the other two axes; a (point, field)
// pair is written by the slab of its lowest ghost axis only, so once, and
// no thread writes a point that another reads (sources have no ghost
// coordinate).
__device__ __forceinline__ void wrap3_body(const Params& P, int which, long long g) {
  const long long N0 = P.N[0], N1 = P.N[1], N2 = P.N[2];
  const long long s0 = 9 * N1 * N2, s1 = N0 * 9 * N2, s2 = N0 * N1 * 9;
  int a, x[3];
  if (g < s0) {
    a = 0;
    x[0] = (int)(g % 9);
    const long long r = g / 9;
    x[1] = (int)(r % N1);
    x[2] = (int)(r / N1);
  } else if (g < s0 + s1) {
    a = 1;
    const long long r = g - s0;
    x[0] = (int)(r % N0);
    x[1] = (int)((r / N0) % 9);
    x[2] = (int)(r / N0 / 9);
  } else if (g < s0 + s1 + s2) {
    a = 2;
    const long long r = g - s0 - s1;
    x[0] = (int)(r % N0);
    x[1] = (int)((r / N0) % N1);
    x[2] = (int)(r / N0 / N1);
  } else {
    return;
  }
  if (x[a] >= NGH) x[a] += P.n[a];  // the 5 points above the active range
  const int bsel = which ? cur_buf(P) : 1 - cur_buf(P);
  double* __restrict__ W = P.Wbuf[bsel];
  double* __restrict__ B = P.Bbuf[bsel];
  const bool ps = P.ps_live != 0;  // p_S zero everywhere stays so: skipped
  long long src[9], dst[9];
  bool on[9];
#pragma unroll
  for (int f = 0; f < 9; f++) {
    int y[3] = {x[0], x[1], x[2]};
    int low = 3;  // lowest ghost axis of this field at this point
#pragma unroll
    for (int b = 2; b >= 0; b--) {
      const int o = (f >= 6 && f - 6 == b) ? 1 : 0;  // the face field along b
      if (y[b] < NGH) {
        y[b] += P.n[b];
        low = b;
      } else if (y[b] >= NGH + P.n[b] + o && y[b] < 2 * NGH + P.n[b] + o) {
        y[b] -= P.n[b];
        low = b;
      }
    }
    on[f] = low == a && (f != PS || ps);
    src[f] = lin(P, y[0], y[1], y[2]);
    dst[f] = lin(P, x[0], x[1], x[2]);
  }
  double v[9];
#pragma unroll
  for (int f = 0; f < 9; f++) {
    const double* q = f < 6 ? W + (size_t)f * P.fs : B + (size_t)(f - 6) * P.fs;
    if (on[f]) v[f] = q[src[f]];
  }
#pragma unroll
  for (int f = 0; f < 9; f++) {
    double* q = f < 6 ? W + (size_t)f * P.fs : B + (size_t)(f - 6) * P.fs;
    if (on[f]) q[dst[f]] = v[f];
  }
}

// One face of the ghost-fill library (src/boundary_conditions.c): the 6 gas
// primitives with kind `kind` (gas_bc_*) and the 3 face fields with kind
// `gkind` (gem_bc_*); 0 skips that group.  t = (i, j, k) with the
// component along `axis` replaced by the ghost layer 0..NGH-1.
__device__ __forceinline__ void bcface_body(const Params& P, int axis, int side, int kind,
                                            int gkind, int which, Pos t) {
  int ijk[3] = {t.x, t.y, t.z};
  const int l = ijk[axis];
  for (int a = 0; a < 3; a++)
    if (ijk[a] >= (a == axis ? NGH : P.N[a])) return;
  const int bsel = which ? cur_buf(P) : 1 - cur_buf(P);
  double* __restrict__ W = P.Wbuf[bsel];
  double* __restrict__ B = P.Bbuf[bsel];
  const int N = P.N[axis];
  for (int f = 0; f < 9; f++) {
    if (f == PS && !P.ps_live) continue;  // zero everywhere, and stays so
    const bool gas = f < 6;
    const int kd = gas ? kind : gkind;
    if (kd == 0 || kd == 'n' || kd == 'p') continue;
    if (!gas && kd == 'r') continue;  // gem_bc_reflective_* are empty
    const int onface = (!gas && f - 6 == axis) ? 1 : 0;
    double* a = gas ? W + (size_t)f * P.fs : B + (size_t)(f - 6) * P.fs;
    const int dst = side == 0 ? l : N - 1 - NGH + l + onface;
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
      const int k0 = ijk[2];
      // pole ('o', j faces): mirrored across the axis half a turn away in
      // phi, the theta and phi components negated
      // (src/spherical/spherical_boundary.c:23-138)
      if (kd == 'o') ijk[2] = NGH + (k0 - NGH + P.n[2] / 2) % P.n[2];
      v = a[lin(P, ijk[0], ijk[1], ijk[2])];
      ijk[2] = k0;
      if (kd == 'r' && gas && f == V1 + axis) v = -v;
      if (kd == 'o' && (gas ? (f == V2 || f == V3) : f != 6)) v = -v;
    }
    ijk[axis] = dst;
    a[lin(P, ijk[0], ijk[1], ijk[2])] = v;
  }
}

// ------------------------------------------------- single-instance kernels

// 1: a fully periodic grid fills its ghosts in one launch (k_wrap3) instead
// of one per axis
#ifndef GOP_WRAP3
#define GOP_WRAP3 1
#endif

// Resident 256-thread blocks per SM each kernel is compiled for (caps its
// registers at 65536 / (256 * n)), per stage and arithmetic type; the
// defaults are the fastest of 1..4 timed on B200 (blast 256^3).
#ifndef GOP_MINB_AB2_F64
#define GOP_MINB_AB2_F64 1
#endif
#ifndef GOP_MINB_AB2_F32
#define GOP_MINB_AB2_F32 1
#endif
#ifndef GOP_MINB_C2C_F64
#define GOP_MINB_C2C_F64 3
#endif
#ifndef GOP_MINB_C2C_F32
#define GOP_MINB_C2C_F32 4
#endif
#ifndef GOP_MINB_EMF_F64
#define GOP_MINB_EMF_F64 2
#endif
#ifndef GOP_MINB_EMF_F32
#define GOP_MINB_EMF_F32 4
#endif
#ifndef GOP_MINB_FLUX_F64
#define GOP_MINB_FLUX_F64 2
#endif
#ifndef GOP_MINB_FLUX_F32
#define GOP_MINB_FLUX_F32 4
#endif
#ifndef GOP_MINB_UPDATE_F64
#define GOP_MINB_UPDATE_F64 2
#endif
#ifndef GOP_MINB_UPDATE_F32
#define GOP_MINB_UPDATE_F32 4
#endif
#ifndef GOP_MINB_UPDATE_SPH_F64
#define GOP_MINB_UPDATE_SPH_F64 2
#endif
#ifndef GOP_MINB_UPDATE_SPH_F32
#define GOP_MINB_UPDATE_SPH_F32 2
#endif
#ifndef GOP_MINB_CT
#define GOP_MINB_CT 4
#endif
#define GOP_MINB(STAGE, R) (sizeof(R) == 8 ? GOP_MINB_##STAGE##_F64 : GOP_MINB_##STAGE##_F32)
#define GOP_UPD_MINB(COORD, R) ((COORD) == 0 ? GOP_MINB(UPDATE, R) : GOP_MINB(UPDATE_SPH, R))

__global__ void k_begin(Params P) {
  pdl_enter();
  begin_body(P);
}
__global__ void k_end(Params P) {
  pdl_enter();
  end_body(P);
}
__global__ void k_arm(Params P, double tstop, double budget) {
  pdl_enter();
  arm_body(P, tstop, budget);
}

// S_PSNZ <- 1 if p_S of either state buffer is nonzero at a point the AB2
// stage reads (every point but the last plane of each axis)
__global__ void k_ps_check(Params P) {
  pdl_enter();
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
  bool nz = false;
  if (i < P.N[0] - 1 && j < P.N[1] - 1 && k < P.N[2] - 1) {
    const long long x = lin(P, i, j, k) + (long long)PS * P.fs;
    nz = P.Wbuf[0][x] != 0.0 || P.Wbuf[1][x] != 0.0;
  }
  if (__any_sync(0xffffffffu, nz) && (threadIdx.x & 31) == 0) P.scal[S_PSNZ] = 1.0;
}

template <int COORD, bool BG, typename R>
__global__ void k_dt(Params P) {
  pdl_enter();
  double dtc = DBL_MAX, db = 0.0;
  dt_body<COORD, BG, R>(P, grid_pos(), dtc, db);
  block_commit(dtc, db, P.scal + S_NEXT_DT, P.scal + S_DIVB);
}

// CFL dt and |div B| of the ring band rows of the new state, after the pole
// ring average (get_derived_variables and get_dt_ring of the next step,
// src/solver_func.c:308-343, src/spherical/spherical_general.c:700-743);
// thread (i, band row, k)
__global__ void k_ring_dt(Params P) {
  pdl_enter();
  double dtc = DBL_MAX, db = 0.0;
  const int i = NGH + blockIdx.x * blockDim.x + threadIdx.x;
  const int k = NGH + blockIdx.z * blockDim.z + threadIdx.z;
  const int slot = blockIdx.y * blockDim.y + threadIdx.y;
  const int jm = P.ring_jmax, nrow = jm + 2, pole = slot / nrow, rr = slot % nrow;
  const int j = pole == 0 ? NGH + rr : NGH + P.n[1] - 2 - jm + rr;
  if (!stopped(P) && pole <= 1 && (P.ring & (1 << pole)) && i < NGH + P.n[0] &&
      k < NGH + P.n[2]) {
    const int nb = 1 - cur_buf(P);  // this step's result
    const double* __restrict__ W = P.Wbuf[nb];
    const double* __restrict__ B = P.Bbuf[nb];
    const long long c = lin(P, i, j, k);
    double b[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      b[a] = mags_at(P, B, a, i, j, k);
      if (P.bg) b[a] += P.bg[(size_t)(BG_B0 + a) * P.fs + c];
    }
    dtc = cfl_cell<2>(P, i, j, k, W[c], W[c + P.fs], W[c + 2 * P.fs], W[c + 3 * P.fs],
                      W[c + 4 * P.fs], b[0], b[1], b[2]);
    const double vol = Geo<2>::vol(P, i, j, k);
    double d = 0.0;
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const double* f = B + (size_t)a * P.fs;
      const long long s = stride(P, a);
      double bu = f[c + s], bl = f[c];
      if (P.bg) {
        const double* g = P.bg + (size_t)(BG_FACE + 4 * a) * P.fs;
        bu += g[c + s];
        bl += g[c];
      }
      const int i1 = i + (a == 0), j1 = j + (a == 1), k1 = k + (a == 2);
      d += (bu * Geo<2>::face(P, a, i1, j1, k1) - bl * Geo<2>::face(P, a, i, j, k)) / vol;
    }
    db = fabs(d);
  }
  block_commit(dtc, db, P.scal + S_NEXT_DT, P.scal + S_DIVB);
}

template <typename R, bool PSL>
__global__ void __launch_bounds__(256, GOP_MINB(AB2, R)) k_ab2(Params P, Work<R> w) {
  pdl_enter();
  if (stopped(P)) return;
  ab2_body<R, PSL>(P, w, grid_pos());
}
template <typename R, int D>
__global__ void __launch_bounds__(256, GOP_MINB(C2C, R)) k_c2c(Params P, Work<R> w) {
  pdl_enter();
  if (stopped(P)) return;
  c2c_body<R, D>(P, w, grid_pos());
}
// BG: with the background-field terms (Params::bg set)
template <typename R, int D, bool BG>
__global__ void __launch_bounds__(256, GOP_MINB(EMF, R)) k_emf(Params P, Work<R> w) {
  pdl_enter();
  if (stopped(P)) return;
  emf_body<R, D, BG>(P, w, grid_pos());
}
template <typename R, int D, bool BG, bool PSL>
__global__ void __launch_bounds__(256, GOP_MINB(FLUX, R)) k_flux(Params P, Work<R> w) {
  pdl_enter();
  if (stopped(P)) return;
  flux_body<R, D, BG, PSL>(P, w, grid_pos());
}
// The faces i = NGH + n0 (the upper boundary face of every i row) of the
// flux along i, one thread per (j, k) row: the i sweep leaves them out when
// 32 divides n0 (a ninth tile of 32 lanes per row would run with one live
// lane per warp)
template <typename R, bool BG>
__global__ void __launch_bounds__(256) k_flux_col(Params P, Work<R> w) {
  pdl_enter();
  if (stopped(P)) return;
  const int tj = blockIdx.x * blockDim.x + threadIdx.x, tk = blockIdx.y * blockDim.y + threadIdx.y;
  flux_body<R, 0, BG, false>(P, w, Pos{P.n[0], tj, tk});
}
template <int COORD, typename R>
__global__ void __launch_bounds__(256, GOP_MINB_CT) k_ct(Params P, Work<R> w) {
  pdl_enter();
  if (stopped(P)) return;
  ct_body<COORD, R>(P, w, grid_pos());
}
template <int COORD, typename R, bool BG, bool PSL>
__global__ void __launch_bounds__(256, GOP_UPD_MINB(COORD, R)) k_update(Params P, Work<R> w) {
  pdl_enter();
  if (stopped(P)) return;
  double dtc = DBL_MAX, db = 0.0;
  update_body<COORD, R, BG, PSL>(P, w, grid_pos(), dtc, db);
  block_commit(dtc, db, P.scal + S_NEXT_DT, P.scal + S_DIVB);
}
__global__ void k_wrap(Params P, int axis, int which) {
  pdl_enter();
  if (stopped(P)) return;
  wrap_body(P, axis, which, grid_pos());
}
__global__ void k_wrap3(Params P, int which) {
  pdl_enter();
  if (stopped(P)) return;
  wrap3_body(P, which, (long long)blockIdx.x * blockDim.x + threadIdx.x);
}
__global__ void k_bcface(Params P, int axis, int side, int kind, int gkind, int which) {
  pdl_enter();
  if (stopped(P)) return;
  bcface_body(P, axis, side, kind, gkind, which, grid_pos());
}

// ------------------------------------------------------ layout transposes

// reference layout [f][i][j][k] (k fastest) <-> device layout
__global__ void k_from_ref(Params P, int nf, const double* __restrict__ src, double* __restrict__ dst) {
  pdl_enter();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int kf = blockIdx.z;
  const int k = kf % P.N[2], f = kf / P.N[2];
  if (i >= P.N[0] || j >= P.N[1] || f >= nf) return;
  const size_t r = (((size_t)f * P.N[0] + i) * P.N[1] + j) * P.N[2] + k;
  dst[(size_t)f * P.fs + lin(P, i, j, k)] = src[r];
}

__global__ void k_to_ref(Params P, int nf, const double* __restrict__ src, double* __restrict__ dst) {
  pdl_enter();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int kf = blockIdx.z;
  const int k = kf % P.N[2], f = kf / P.N[2];
  if (i >= P.N[0] || j >= P.N[1] || f >= nf) return;
  const size_t r = (((size_t)f * P.N[0] + i) * P.N[1] + j) * P.N[2] + k;
  dst[r] = src[(size_t)f * P.fs + lin(P, i, j, k)];
}

template <typename R>
__global__ void k_widen(Params P, int nf, const R* __restrict__ src, double* __restrict__ dst) {
  pdl_enter();
  const size_t n = (size_t)nf * P.fs;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
    dst[t] = (double)src[t];
}

// mags over the ghost range from face fields (for downloads)
__global__ void k_mags(Params P, const double* __restrict__ B, double* __restrict__ out) {
  pdl_enter();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= P.N[0] - 1 || j >= P.N[1] - 1 || k >= P.N[2] - 1) return;
  const long long x = lin(P, i, j, k);
  for (int a = 0; a < 3; a++) out[x + a * P.fs] = mags_at(P, B, a, i, j, k);
}

// ----------------------------------------------------------- launchers

// launches by this process (any host thread)
static std::atomic<int64_t> g_launches{0};
int64_t launches() { return g_launches.load(); }
void count_launches(int64_t n) { g_launches += n; }

static dim3 grid3(int a, int b, int c, dim3 blk) {
  return dim3((a + blk.x - 1) / blk.x, (b + blk.y - 1) / blk.y, (c + blk.z - 1) / blk.z);
}

// 1: step kernels go out with programmatic dependent launch
#ifndef GOP_PDL
#define GOP_PDL 1
#endif
// 1: also the first kernel after the tile-staged flux sweeps.  Off: placed
// early, its blocks (and the blocks launched early after them) start on SMs
// still configured for the sweep's 213 KB of shared memory, with a short
// L1, and the L1-bound edge-EMF stage slows down (blast 256^3 FP64 step
// 9.49 vs 8.09 ms on B200)
#ifndef GOP_PDL_AFTER_SWEEP
#define GOP_PDL_AFTER_SWEEP 0
#endif

#define LAUNCH_PDL(pdl, kern, grd, blk, st, ...)                                 \
  do {                                                                           \
    cudaLaunchAttribute at_[1];                                                  \
    at_[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;              \
    at_[0].val.programmaticStreamSerializationAllowed = 1;                       \
    cudaLaunchConfig_t cfg_ = {};                                                \
    cfg_.gridDim = dim3(grd);                                                    \
    cfg_.blockDim = dim3(blk);                                                   \
    cfg_.stream = st;                                                            \
    cfg_.attrs = at_;                                                            \
    cfg_.numAttrs = (GOP_PDL && (pdl)) ? 1 : 0;                                  \
    cudaLaunchKernelEx(&cfg_, kern, __VA_ARGS__);                                \
    g_launches++;                                                                \
  } while (0)
#define LAUNCH(kern, grd, blk, st, ...) LAUNCH_PDL(true, kern, grd, blk, st, __VA_ARGS__)

Tune::Tune() {
  // defaults: warps along i; the sweeps of D=1 / D=2 kernels run along the
  // block's longer transverse side so neighbouring rows share L1 lines
  for (int t = 0; t < NTUNE; t++) blk[t] = dim3(32, 4, 2);
  blk[K_EMF1] = blk[K_FLUX1] = dim3(32, 8, 1);
  blk[K_C2C2] = blk[K_EMF2] = blk[K_FLUX2] = dim3(32, 1, 8);
  // the first edge sweep of edges along j covers only the 8 ghost layers of i
  blk[K_C2C1] = dim3(8, 32, 1);
  for (int d = 0; d < 3; d++) {
    flux_sweep[d] = emf_sweep[d] = true;
    flux_order[d] = emf_order[d] = d;
  }
}

dim3 launch_space(const Params& P, int slot) {
  if (slot == K_AB2) return dim3(P.N[0], P.N[1], P.N[2]);
  if (slot == K_UPDATE) return dim3(P.n[0], P.n[1], P.n[2]);
  if (slot >= K_WRAP0 && slot <= K_BC5) {  // (i, j, k) with the ghost layers along the axis
    const bool wrap = slot <= K_WRAP2;
    const int a = wrap ? slot - K_WRAP0 : (slot - K_BC0) / 2;
    int e[3] = {P.N[0], P.N[1], P.N[2]};
    e[a] = wrap ? 2 * NGH : NGH;
    return dim3(e[0], e[1], e[2]);
  }
  const int stage = (slot - K_C2C0) / 3, D = (slot - K_C2C0) % 3;
  const int p = (D + 1) % 3, q = (D + 2) % 3;
  int cnt[3];
  if (stage == 0) {  // ghost layers of q only (the flux stage covers the rest)
    cnt[D] = P.n[D];
    cnt[p] = P.n[p] + 1;
    cnt[q] = 2 * NGH;
  } else if (stage == 1) {
    cnt[D] = P.n[D];
    cnt[p] = P.n[p] + 1;
    cnt[q] = P.n[q] + 1;
  } else {
    cnt[0] = P.n[0];
    cnt[1] = P.n[1];
    cnt[2] = P.n[2];
    cnt[D] += 1;
  }
  return dim3(cnt[0], cnt[1], cnt[2]);
}

void launch_begin(const Params& P, cudaStream_t st) { LAUNCH(k_begin, 1, 1, st, P); }
void launch_end(const Params& P, cudaStream_t st) { LAUNCH(k_end, 1, 1, st, P); }
void launch_arm(const Params& P, double tstop, double budget, cudaStream_t st) {
  LAUNCH(k_arm, 1, 1, st, P, tstop, budget);
}

void launch_ps_check(const Params& P, cudaStream_t st) {
  const int nx = (P.N[0] - 1 + 31) / 32 * 32;
  const dim3 blk(std::min(nx, 256), 1, 1);
  LAUNCH(k_ps_check, dim3((nx + blk.x - 1) / blk.x, P.N[1] - 1, P.N[2] - 1), blk, st, P);
}

template <typename R>
static void launch_dt_r(const Params& P, int coord, cudaStream_t st) {
  const dim3 blk(32, 4, 2);
  const dim3 g = grid3(P.n[0], P.n[1], P.n[2], blk);
  const bool bg = P.bg != nullptr;
  if (coord == 0) {
    if (bg) LAUNCH((k_dt<0, true, R>), g, blk, st, P);
    else LAUNCH((k_dt<0, false, R>), g, blk, st, P);
  } else {
    if (bg) LAUNCH((k_dt<2, true, R>), g, blk, st, P);
    else LAUNCH((k_dt<2, false, R>), g, blk, st, P);
  }
}

void launch_dt(const Params& P, int coord, bool mixed, cudaStream_t st) {
  if (mixed) launch_dt_r<float>(P, coord, st);
  else launch_dt_r<double>(P, coord, st);
}

template <typename R, bool BG>
static void launch_slot_bg(const Params& P, int coord, const Work<R>& w, int slot, dim3 blk,
                           cudaStream_t st, const SweepSet* sw, bool pdl) {
  if (slot >= K_FLUX0 && slot <= K_FLUX2 && launch_flux_sweep<R>(sw, P, w, slot - K_FLUX0, st)) return;
  if (slot >= K_EMF0 && slot <= K_EMF2 && launch_emf_sweep<R>(sw, P, w, slot - K_EMF0, st)) return;
  const dim3 sp = launch_space(P, slot);
  const dim3 g = grid3(sp.x, sp.y, sp.z, blk);
  switch (slot) {
    case K_AB2:
      if (P.ps_live) LAUNCH((k_ab2<R, true>), g, blk, st, P, w);
      else LAUNCH((k_ab2<R, false>), g, blk, st, P, w);
      break;
    case K_C2C0: LAUNCH_PDL(pdl, (k_c2c<R, 0>), g, blk, st, P, w); break;
    case K_C2C1: LAUNCH((k_c2c<R, 1>), g, blk, st, P, w); break;
    case K_C2C2: LAUNCH((k_c2c<R, 2>), g, blk, st, P, w); break;
    case K_EMF0: LAUNCH((k_emf<R, 0, BG>), g, blk, st, P, w); break;
    case K_EMF1: LAUNCH((k_emf<R, 1, BG>), g, blk, st, P, w); break;
    case K_EMF2: LAUNCH((k_emf<R, 2, BG>), g, blk, st, P, w); break;
    case K_FLUX0:
      if (P.ps_live) LAUNCH((k_flux<R, 0, BG, true>), g, blk, st, P, w);
      else LAUNCH((k_flux<R, 0, BG, false>), g, blk, st, P, w);
      break;
    case K_FLUX1:
      if (P.ps_live) LAUNCH((k_flux<R, 1, BG, true>), g, blk, st, P, w);
      else LAUNCH((k_flux<R, 1, BG, false>), g, blk, st, P, w);
      break;
    case K_FLUX2:
      if (P.ps_live) LAUNCH((k_flux<R, 2, BG, true>), g, blk, st, P, w);
      else LAUNCH((k_flux<R, 2, BG, false>), g, blk, st, P, w);
      break;
    case K_UPDATE:
      if (coord == 0) {
        if (P.ps_live) LAUNCH_PDL(pdl, (k_update<0, R, BG, true>), g, blk, st, P, w);
        else LAUNCH_PDL(pdl, (k_update<0, R, BG, false>), g, blk, st, P, w);
      } else {
        if (P.ps_live) LAUNCH_PDL(pdl, (k_update<2, R, BG, true>), g, blk, st, P, w);
        else LAUNCH_PDL(pdl, (k_update<2, R, BG, false>), g, blk, st, P, w);
      }
      break;
    default: break;
  }
}

template <typename R>
void launch_flux_col(const Params& P, const Work<R>& w, cudaStream_t st) {
  const dim3 blk(32, 8, 1);
  const dim3 g((P.n[1] + 31) / 32, (P.n[2] + 7) / 8, 1);
  // right after a sweep: no early launch (see launch_step_body)
  if (P.bg) LAUNCH_PDL(false, (k_flux_col<R, true>), g, blk, st, P, w);
  else LAUNCH_PDL(false, (k_flux_col<R, false>), g, blk, st, P, w);
}
template void launch_flux_col<double>(const Params&, const Work<double>&, cudaStream_t);
template void launch_flux_col<float>(const Params&, const Work<float>&, cudaStream_t);

template <typename R>
void launch_slot(const Params& P, int coord, const Work<R>& w, int slot, dim3 blk,
                 cudaStream_t st, const SweepSet* sw, bool pdl) {
  if (P.bg) launch_slot_bg<R, true>(P, coord, w, slot, blk, st, sw, pdl);
  else launch_slot_bg<R, false>(P, coord, w, slot, blk, st, sw, pdl);
}

template void launch_slot<double>(const Params&, int, const Work<double>&, int, dim3, cudaStream_t,
                                  const SweepSet*, bool);
template void launch_slot<float>(const Params&, int, const Work<float>&, int, dim3, cudaStream_t,
                                 const SweepSet*, bool);

template <typename R>
void launch_step_body(const Params& P, int coord, const Work<R>& w, cudaStream_t st,
                      const Tune& tune, const SweepSet* sw, const Hook& hook) {
  hook(G_AB2, 1);
  launch_slot<R>(P, coord, w, K_AB2, tune.blk[K_AB2], st);
  hook(G_AB2, 0);
  // flux first: it also writes the edge velocities of the active range
  // the three launches of a stage are independent (each axis writes its own
  // fluxes, edge velocities or EMFs), so their order (Tune) changes no result
  const int last_flux = tune.flux_order[2], last_emf = tune.emf_order[2];
  for (int stage : {2, 0, 1}) {
    const int g = stage == 0 ? G_C2C : (stage == 1 ? G_EMF : G_FLUX);
    hook(g, 1);
    for (int n = 0; n < 3; n++) {
      const int d = stage == 2 ? tune.flux_order[n] : (stage == 1 ? tune.emf_order[n] : n);
      const int slot = K_C2C0 + 3 * stage + d;
      const bool sweep = sw && ((stage == 2 && tune.flux_sweep[d]) || (stage == 1 && tune.emf_sweep[d]));
      // the launch after a persistent sweep grid waits for it to finish
      // instead of being placed early on SMs still configured for the
      // sweep's shared memory (and its short L1)
      const bool pdl = !(stage == 0 && n == 0 && sw && tune.flux_sweep[last_flux]) || GOP_PDL_AFTER_SWEEP;
      launch_slot<R>(P, coord, w, slot, tune.blk[slot], st, sweep ? sw : nullptr, pdl);
    }
    hook(g, 0);
  }
  hook(G_UPDATE, 1);
  const bool after_emf_sweep = sw && tune.emf_sweep[last_emf] && !GOP_PDL_AFTER_SWEEP;
  launch_pole_emf<R>(P, w, st);  // pole ring average only
  if (coord != 0) {  // curvilinear: the face fields in their own launch
    const dim3 blk = tune.blk[K_UPDATE];
    LAUNCH_PDL(!after_emf_sweep, (k_ct<2, R>), grid3(P.n[0], P.n[1], P.n[2], blk), blk, st, P, w);
  }
  launch_slot<R>(P, coord, w, K_UPDATE, tune.blk[K_UPDATE], st, nullptr,
                 coord != 0 || !after_emf_sweep);
  // the work arrays are free after the update: 2 fields of doubles of scratch
  if (P.ring) {
    launch_ring_average(P, reinterpret_cast<double*>(w.Wh), st);
    const int jm = P.ring_jmax;
    const dim3 blk(32, 2, 4);
    LAUNCH(k_ring_dt, grid3(P.n[0], 2 * (jm + 2), P.n[2], blk), blk, st, P);
  }
  hook(G_UPDATE, 0);
}

template void launch_step_body<double>(const Params&, int, const Work<double>&, cudaStream_t,
                                       const Tune&, const SweepSet*, const Hook&);
template void launch_step_body<float>(const Params&, int, const Work<float>&, cudaStream_t,
                                      const Tune&, const SweepSet*, const Hook&);

dim3 ghost_block(int slot) {
  if (slot == K_WRAP0) return dim3(8, 16, 2);               // 8 layers along i
  if (slot == K_BC0 || slot == K_BC1) return dim3(4, 32, 2);  // 4 layers along i
  return dim3(32, 8, 1);
}

void launch_ghosts(const Params& P, const char bc[6], const char gem_bc[6], int which,
                   cudaStream_t st) {
  bool periodic[3];
  for (int a = 0; a < 3; a++) periodic[a] = bc[2 * a] == 'p' && bc[2 * a + 1] == 'p';
  if (periodic[0] && periodic[1] && periodic[2] && GOP_WRAP3) {
    const long long N0 = P.N[0], N1 = P.N[1], N2 = P.N[2];
    const long long pts = 9 * (N1 * N2 + N0 * N2 + N0 * N1);
    LAUNCH(k_wrap3, dim3((unsigned)((pts + 255) / 256)), dim3(256), st, P, which);
    return;
  }
  for (int a = 0; a < 3; a++) {
    if (!periodic[a]) continue;
    const dim3 sp = launch_space(P, K_WRAP0 + a), blk = ghost_block(K_WRAP0 + a);
    LAUNCH(k_wrap, grid3(sp.x, sp.y, sp.z, blk), blk, st, P, a, which);
  }
  for (int face = 0; face < 6; face++) {
    const int a = face / 2, side = face % 2;
    const char kind = bc[face], gkind = gem_bc[face];
    if (periodic[a]) continue;
    const bool gas_work = kind != 'n';
    const bool gem_work = gkind != 'n' && gkind != 'r';
    if (!gas_work && !gem_work) continue;
    const dim3 sp = launch_space(P, K_BC0 + face), blk = ghost_block(K_BC0 + face);
    LAUNCH(k_bcface, grid3(sp.x, sp.y, sp.z, blk), blk, st, P, a, side, (int)kind, (int)gkind, which);
  }
}

void launch_from_ref(const Params& P, int nf, const double* src, double* dst, cudaStream_t st) {
  const dim3 blk(32, 8, 1);
  const dim3 g((P.N[0] + 31) / 32, (P.N[1] + 7) / 8, P.N[2] * nf);
  LAUNCH(k_from_ref, g, blk, st, P, nf, src, dst);
}

void launch_to_ref(const Params& P, int nf, const double* src, double* dst, cudaStream_t st) {
  const dim3 blk(32, 8, 1);
  const dim3 g((P.N[0] + 31) / 32, (P.N[1] + 7) / 8, P.N[2] * nf);
  LAUNCH(k_to_ref, g, blk, st, P, nf, src, dst);
}

template <typename R>
void launch_widen(const Params& P, int nf, const R* src, double* dst, cudaStream_t st) {
  LAUNCH(k_widen<R>, 1184, 256, st, P, nf, src, dst);
}
template void launch_widen<double>(const Params&, int, const double*, double*, cudaStream_t);
template void launch_widen<float>(const Params&, int, const float*, double*, cudaStream_t);

void launch_mags(const Params& P, const double* B, double* out, cudaStream_t st) {
  const dim3 blk(32, 4, 2);
  LAUNCH(k_mags, grid3(P.N[0], P.N[1], P.N[2], blk), blk, st, P, B, out);
}

}  // namespace gop

// Device-side data layout, geometry and per-face numerics of the GAMERA-OP
// MHD step on B200 (sm_100a).
//
// Layout in HBM: structure of arrays, one 3-D array per field, i fastest,
// each axis ghost-extended exactly like the reference (n + 2*4 + 1 points,
// active cells at 4..n+3, the extra point holds the upper boundary face).
// Rows are padded to a multiple of 8 doubles so every row starts on a
// 64-byte boundary and warps along i issue coalesced loads.
//
// Geometry is separable in both supported coordinate systems, so the device
// never stores 3-D geometry: face areas, volumes and edge lengths are
// products of per-axis 1-D tables evaluated in the reference's
// multiplication order (src/cartesian/cartesian_general.c:42-283,
// src/spherical/spherical_general.c:42-316).  PDM weights and the PDM
// limiter's geometric coefficients are per-face 1-D tables.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gop {

constexpr int NGH = 4;

// per-axis 1-D tables (index = position along the axis)
enum Tab : int {
  T_X = 0,     // face coordinate x[f]
  T_DX,        // x[f+1] - x[f]
  T_MA,        // (x[c+1] - xctr[c]) / dx[c]: weight of the lower face in mags
  T_MB,        // (xctr[c] - x[c]) / dx[c]: weight of the upper face
  T_WL0,       // 7 left PDM weights at face f (applied to cells f-4..f+2)
  T_WR0 = T_WL0 + 7,  // 7 right weights (applied to cells f+3..f-3)
  T_CL1 = T_WR0 + 7,  // PDM limiter coefficients of the left state
  T_CL2,
  T_CR1,       // ... of the right state
  T_CR2,
  T_G0,        // coordinate-specific factors (see Geo below)
  T_G1,
  T_G2,
  T_G3,
  T_G4,
  NTAB
};

// The PDM weights and limiter coefficients of one face packed together
// after the per-axis tables: fw[(axis * tmax + f) * FW + t], t = 0..6 left
// weights, 7..13 right weights, 14..17 cl1 cl2 cr1 cr2, 18..19 zero, so one
// face's 18 values come in five 16-byte loads (FP32) from one address.
// tmax is a multiple of 4, which keeps every face record 16-byte aligned.
constexpr int FW = 20;
__host__ __device__ constexpr size_t fw_offset(int tmax) { return (size_t)3 * NTAB * tmax; }
__host__ __device__ constexpr size_t tab_elems(int tmax) { return (size_t)3 * (NTAB + FW) * tmax; }

// device scalars (one double slot each)
enum Scal : int {
  S_DT = 0,      // dt of the current step
  S_DT0,         // dt of the previous step (AB2)
  S_TIME,        // time_sim
  S_CAB2,        // 0.5*dt/dt0 of the current step
  S_NEXT_DT,     // bit pattern of the running CFL minimum (uint64 atomicMin)
  S_DIVB,        // bit pattern of max|div B| (uint64 atomicMax)
  S_STEPS,       // steps taken (as double)
  S_STOP,        // nonzero: time_stop reached, kernels return at once
  S_TSTOP,       // time_stop of the current gop_step call
  S_FLAGS,       // bit 0: non-finite / non-positive state seen
  S_PAR,         // which of the two state buffers holds the current state
  S_BUDGET,      // steps left in the current gop_step call
  S_PSNZ,        // gop_prepare's check: nonzero if some p_S of the state or
                 // of its AB2 history is nonzero
  NSCAL
};

struct Params {
  int n[3];           // active cells
  int N[3];           // ghost-extended points
  int pitch;          // row pitch (elements)
  int coord;          // 0: Cartesian, 2: spherical (batched kernels select on it)
  long long sj, sk;   // strides of j and k (stride of i is 1)
  long long fs;       // stride between fields
  const double* tab;  // [3][NTAB][tmax]
  int tmax;
  double gamma, gm1, cfl, ca, ca2, rho_floor, p_floor;
  double pdm_a1, pdm_a2;  // PDMB/(PDMB+1), 1-a1
  double inv_gm1;         // 1/(gamma-1)
  double q_ca;            // 1/(4 CA): Boris diffusion coefficient of the stress
  double* scal;           // device scalars
  double* Wbuf[2];        // two 6-field primitive buffers (current / next)
  double* Bbuf[2];        // two 3-field face-B buffers
  const double* bg;       // background field block (BG_NF fields) or null
  // 1 if p_S (the entropy channel) is nonzero somewhere in the state or its
  // AB2 history; 0 keeps it zero for good (zero states give a zero entropy
  // flux and every fill copies), and the flux kernels skip it
  int ps_live;
  // pole ring average (spherical): bit 0 a pole at theta = 0 (j face NGH),
  // bit 1 at theta = pi (j face NGH + nj); 0 off
  int ring;
  int ring_jmax;          // ring rows per pole - 1
  int nchunk[16];         // phi blocks of ring row r
  const double* ringtab;  // cos, sin of (k + 1/2) 2 pi / nk; then per j the
                          // factor of the CFL length in phi (N[1] values)
};

// Background field B0 (src/solver_func.c:1851-2077), BG_NF fields of the
// state's layout: B0 at the cell centre (B0_b1..3), the Lorentz force of B0
// (dmagsf_G), B0 averaged over the faces normal to axis d (B0Aface*_b1..3,
// field BG_FACE + 3d + c) and along the edges of axis d (B0Aedge*_b1..3,
// field BG_EDGE + 3d + c).
enum BgField : int { BG_B0 = 0, BG_LOR = 3, BG_FACE = 6, BG_EDGE = 15, BG_NF = 24 };

__device__ __forceinline__ int cur_buf(const Params& P) { return P.scal[S_PAR] != 0.0 ? 1 : 0; }

__device__ __forceinline__ double tb(const Params& P, int axis, int t, int idx) {
  return __ldg(P.tab + ((size_t)axis * NTAB + t) * P.tmax + idx);
}

__device__ __forceinline__ long long lin(const Params& P, int i, int j, int k) {
  return (long long)k * P.sk + (long long)j * P.sj + i;
}

__device__ __forceinline__ long long stride(const Params& P, int axis) {
  return axis == 0 ? 1LL : (axis == 1 ? P.sj : P.sk);
}

// Geometry policy.  Cartesian: the reference's uniform-grid arrays
// (dx_a, face_i = dx2*dx3, vol = dx1*dx2*dx3).  Spherical (r, theta, phi):
// G0..G4 of axis 0 = -r^2, (r1^3-r0^3)/3, (r1^2-r0^2)/2, r_c;
// of axis 1 = cos(t1)-cos(t0), sin(t), sin(t_c), sin(t1)-sin(t0),
// sin(t1)+sin(t0).
template <int COORD>
struct Geo {
  __device__ static __forceinline__ double face(const Params& P, int a, int i, int j, int k) {
    if (COORD == 0) {
      if (a == 0) return tb(P, 1, T_DX, j) * tb(P, 2, T_DX, k);
      if (a == 1) return tb(P, 0, T_DX, i) * tb(P, 2, T_DX, k);
      return tb(P, 0, T_DX, i) * tb(P, 1, T_DX, j);
    } else {
      if (a == 0) return tb(P, 0, T_G0, i) * tb(P, 1, T_G0, j) * tb(P, 2, T_DX, k);
      if (a == 1) return tb(P, 0, T_G2, i) * tb(P, 1, T_G1, j) * tb(P, 2, T_DX, k);
      return tb(P, 0, T_G2, i) * tb(P, 1, T_DX, j);
    }
  }
  __device__ static __forceinline__ double vol(const Params& P, int i, int j, int k) {
    if (COORD == 0) return tb(P, 0, T_DX, i) * tb(P, 1, T_DX, j) * tb(P, 2, T_DX, k);
    return fabs(tb(P, 0, T_G1, i) * tb(P, 1, T_G0, j) * tb(P, 2, T_DX, k));
  }
  // edge length of the edge along axis a at (i,j,k)
  __device__ static __forceinline__ double edge(const Params& P, int a, int i, int j, int k) {
    if (COORD == 0 || a == 0) return tb(P, a, T_DX, a == 0 ? i : (a == 1 ? j : k));
    if (a == 1) return tb(P, 0, T_X, i) * tb(P, 1, T_DX, j);
    return tb(P, 0, T_X, i) * tb(P, 1, T_G1, j) * tb(P, 2, T_DX, k);
  }
  // CFL length of cell (i,j,k) along axis a (geo[dxi..dxk])
  __device__ static __forceinline__ double dl(const Params& P, int a, int i, int j, int k) {
    if (COORD == 0 || a == 0) return tb(P, a, T_DX, a == 0 ? i : (a == 1 ? j : k));
    if (a == 1) return tb(P, 0, T_G3, i) * tb(P, 1, T_DX, j);
    return tb(P, 0, T_G3, i) * tb(P, 1, T_G2, j) * tb(P, 2, T_DX, k);
  }
};

template <typename R>
__device__ __forceinline__ R sgn(R x) {
  return x > R(0) ? R(1) : (x < R(0) ? R(-1) : R(0));
}

// Left and right states at face f of a line v[0..7] = cells f-4..f+3, with
// the limiter on lim[0..3] = cells f-2..f+1.
template <typename R>
struct FaceWeights {
  R wl[7], wr[7], cl1, cl2, cr1, cr2;
};

// tab: the per-axis tables in the stage type R (layout of Params::tab)
template <typename R>
__device__ __forceinline__ void load_weights(const R* __restrict__ tab, int tmax, int axis, int f,
                                             FaceWeights<R>& W) {
  const R* t0 = tab + (size_t)axis * NTAB * tmax + f;
#pragma unroll
  for (int t = 0; t < 7; t++) {
    W.wl[t] = __ldg(t0 + (size_t)(T_WL0 + t) * tmax);
    W.wr[t] = __ldg(t0 + (size_t)(T_WR0 + t) * tmax);
  }
  W.cl1 = __ldg(t0 + (size_t)T_CL1 * tmax);
  W.cl2 = __ldg(t0 + (size_t)T_CL2 * tmax);
  W.cr1 = __ldg(t0 + (size_t)T_CR1 * tmax);
  W.cr2 = __ldg(t0 + (size_t)T_CR2 * tmax);
}

// the same from the packed face records (fw = the packed region): one
// address and five (FP32) or nine (FP64) vector loads per face
__device__ __forceinline__ void load_fw(const float* __restrict__ fw, int tmax, int axis, int f,
                                        FaceWeights<float>& W) {
  const float4* p = reinterpret_cast<const float4*>(fw + ((size_t)axis * tmax + f) * FW);
  const float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2), d = __ldg(p + 3), e = __ldg(p + 4);
  W.wl[0] = a.x; W.wl[1] = a.y; W.wl[2] = a.z; W.wl[3] = a.w;
  W.wl[4] = b.x; W.wl[5] = b.y; W.wl[6] = b.z; W.wr[0] = b.w;
  W.wr[1] = c.x; W.wr[2] = c.y; W.wr[3] = c.z; W.wr[4] = c.w;
  W.wr[5] = d.x; W.wr[6] = d.y; W.cl1 = d.z; W.cl2 = d.w;
  W.cr1 = e.x; W.cr2 = e.y;
}
__device__ __forceinline__ void load_fw(const double* __restrict__ fw, int tmax, int axis, int f,
                                        FaceWeights<double>& W) {
  const double2* p = reinterpret_cast<const double2*>(fw + ((size_t)axis * tmax + f) * FW);
  double v[18];
#pragma unroll
  for (int t = 0; t < 9; t++) {
    const double2 q = __ldg(p + t);
    v[2 * t] = q.x;
    v[2 * t + 1] = q.y;
  }
#pragma unroll
  for (int t = 0; t < 7; t++) {
    W.wl[t] = v[t];
    W.wr[t] = v[7 + t];
  }
  W.cl1 = v[14]; W.cl2 = v[15]; W.cr1 = v[16]; W.cr2 = v[17];
}

// Both states of a face (two evaluations of PDMU7, src/solver_func.c:215-253:
// a 7-tap interpolation of the half-step values, clamped to the two
// step-start values adjacent to the face, then the PDM limiter with the
// geometric reference slope |c1*p0 + c2*pm1|/2 blended with |p0 - pm1|)
// from the half-step line
// v[0..7] = cells f-4..f+3 and the step-start values lim[0..3] = cells
// f-2..f+1.  With D(g) = lim(g) - lim(g-1) the limiter of the left state
// needs sgn D(f-1), |D(f-1)| and sgn D(f); the right one (its differences
// taken in the mirrored direction, lim(f) - lim(f+1) = -D(f+1) exactly)
// needs sgn D(f+1), |D(f+1)| and sgn D(f), so the caller passes
// s1 = sgn D(f), q0l = |sgn D(f-1) + s1| and q0r = |sgn D(f+1) + s1|.
// a1h = a1/2: the reference's |c1 p0 + c2 pm1| * 0.5 * a1 with the exact
// factor 1/2 moved into a1.  Every other operation is the reference's, in
// its order.
// hi, lo: the larger and the smaller of lim[1], lim[2] (the clamp bounds)
template <typename R>
__device__ __forceinline__ void pdm_pair(const R v[8], const R lim[4], const FaceWeights<R>& W,
                                         R a1h, R a2, R s1, R q0l, R q0r, R L_ad0, R R_ad0,
                                         R hi, R lo, R& L, R& Rr) {
  {
    // left: cells f-4..f+2, limiter cells f-2 (im1), f-1 (i0), f (ip1)
    R fi = v[0] * W.wl[0];
#pragma unroll
    for (int t = 1; t < 7; t++) fi = fma(v[t], W.wl[t], fi);
    const R f = fmax(lo, fmin(fi, hi));
    const R dl = f - lim[1];
    const R dc = a1h * fabs(W.cl1 * lim[1] + W.cl2 * lim[0]) + a2 * L_ad0;
    L = f - s1 * fmax(R(0), fabs(dl) - q0l * dc);
  }
  {
    // right: cells f+3..f-3, limiter cells f+1 (im1), f (i0), f-1 (ip1);
    // its direction sign is -s1
    R fi = v[7] * W.wr[0];
#pragma unroll
    for (int t = 1; t < 7; t++) fi = fma(v[7 - t], W.wr[t], fi);
    const R f = fmax(lo, fmin(fi, hi));
    const R dl = f - lim[2];
    const R dc = a1h * fabs(W.cr1 * lim[2] + W.cr2 * lim[3]) + a2 * R_ad0;
    Rr = f + s1 * fmax(R(0), fabs(dl) - q0r * dc);
  }
}

// the same from a record in shared memory (16-byte aligned; the whole warp
// reads one record)
__device__ __forceinline__ void load_fw_smem(const float* rec, FaceWeights<float>& W) {
  const float4* p = reinterpret_cast<const float4*>(rec);
  const float4 a = p[0], b = p[1], c = p[2], d = p[3], e = p[4];
  W.wl[0] = a.x; W.wl[1] = a.y; W.wl[2] = a.z; W.wl[3] = a.w;
  W.wl[4] = b.x; W.wl[5] = b.y; W.wl[6] = b.z; W.wr[0] = b.w;
  W.wr[1] = c.x; W.wr[2] = c.y; W.wr[3] = c.z; W.wr[4] = c.w;
  W.wr[5] = d.x; W.wr[6] = d.y; W.cl1 = d.z; W.cl2 = d.w;
  W.cr1 = e.x; W.cr2 = e.y;
}
__device__ __forceinline__ void load_fw_smem(const double* rec, FaceWeights<double>& W) {
  const double2* p = reinterpret_cast<const double2*>(rec);
  double v[18];
#pragma unroll
  for (int t = 0; t < 9; t++) {
    const double2 q = p[t];
    v[2 * t] = q.x;
    v[2 * t + 1] = q.y;
  }
#pragma unroll
  for (int t = 0; t < 7; t++) {
    W.wl[t] = v[t];
    W.wr[t] = v[7 + t];
  }
  W.cl1 = v[14]; W.cl2 = v[15]; W.cr1 = v[16]; W.cr2 = v[17];
}

// one face on its own: the three differences of lim computed here
template <typename R>
__device__ __forceinline__ void recon_lr(const R v[8], const R lim[4], const FaceWeights<R>& W,
                                         R a1h, R a2, R& L, R& Rr) {
  const R dm = lim[1] - lim[0], d1 = lim[2] - lim[1], dp = lim[3] - lim[2];
  const R s1 = sgn(d1);
  pdm_pair<R>(v, lim, W, a1h, a2, s1, fabs(sgn(dm) + s1), fabs(sgn(dp) + s1), fabs(dm),
              fabs(dp), fmax(lim[1], lim[2]), fmin(lim[1], lim[2]), L, Rr);
}

// Weights of face f on axis AX for a warp whose lanes run along i: along
// i every lane has its own face, and the tap-major tables give coalesced
// loads; along j or k the whole warp shares one face record.
template <int AX, typename R>
__device__ __forceinline__ void load_face_weights(const R* __restrict__ tab, const R* __restrict__ fw,
                                                  int tmax, int f, FaceWeights<R>& W) {
  if constexpr (AX == 0) load_weights<R>(tab, tmax, 0, f, W);
  else load_fw(fw, tmax, AX, f, W);
}

}  // namespace gop

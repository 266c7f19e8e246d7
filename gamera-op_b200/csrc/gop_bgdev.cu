// Background magnetic field B0 built on the device (set_background_field,
// src/solver_func.c:1851-2077, for the built-in uniform and dipole
// backgrounds): the host port in host/gop_background.c runs its 12x12-point
// face quadratures point by point on one CPU core -- O(1728) field
// evaluations per cell, seconds for a large dipole grid, on the admission
// path of every served request -- while here one thread per face, edge or
// cell evaluates the same source (csrc/gop_bgfield.h), straight into the
// instance's background block in the device layout:
//
//   centroid  B0 at the cell centroids (BG_B0)
//   face      the 12x12 Gauss face averages of b1..b3 (BG_FACE), with |B0|^2
//             and b_d * b1..b3 of the face into a 12-field scratch
//   edge      the 12-point edge averages over the active edges (BG_EDGE)
//   lorentz   the Lorentz force of B0 from the six face stresses (BG_LOR)
//
// Points outside each stage's range stay zero, as the host arrays leave
// them.  The results differ from the host's only by the last bits of the
// device's pow, sin and cos and of fused multiply-adds.
#include "gop_bgfield.h"
#include "gop_device.cuh"
#include "gop_kernels.h"

namespace gop {

namespace {

struct X3 {
  const double *x1, *x2, *x3;  // face coordinates (the T_X tables)
};
__device__ __forceinline__ X3 face_coords(const Params& P) {
  return {P.tab + ((size_t)0 * NTAB + T_X) * P.tmax, P.tab + ((size_t)1 * NTAB + T_X) * P.tmax,
          P.tab + ((size_t)2 * NTAB + T_X) * P.tmax};
}

__global__ void k_bg_centroid(Params P, gop_background bg, int sph, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y,
            k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i > P.N[0] - 2 || j > P.N[1] - 2 || k > P.N[2] - 2) return;
  const X3 X = face_coords(P);
  double r, t, f;
  if (sph) {
    gop_sph_centroid(X.x1, X.x2, X.x3, i, j, k, &r, &t, &f);
  } else {
    r = 0.5 * (X.x1[i] + X.x1[i + 1]);
    t = 0.5 * (X.x2[j] + X.x2[j + 1]);
    f = 0.5 * (X.x3[k] + X.x3[k + 1]);
  }
  const long long p = lin(P, i, j, k);
  for (int c = 0; c < 3; c++) out[(size_t)(BG_B0 + c) * P.fs + p] = gop_b0_fn(&bg, c, r, t, f);
}

// faces normal to dir: up to N-1 along dir, N-2 across
__global__ void k_bg_face(Params P, gop_background bg, int sph, int dir, double* out, double* aux) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y,
            k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i > P.N[0] - 2 + (dir == 0) || j > P.N[1] - 2 + (dir == 1) || k > P.N[2] - 2 + (dir == 2))
    return;
  const X3 X = face_coords(P);
  double c[3][4], o[7];
  gop_b0_face_corners(X.x1, X.x2, X.x3, dir, i, j, k, c);
  gop_b0_face_average(&bg, sph, dir, gop_face_area(X.x1, X.x2, X.x3, sph, dir, i, j, k), c, o);
  const long long p = lin(P, i, j, k);
  for (int q = 0; q < 3; q++) out[(size_t)(BG_FACE + 3 * dir + q) * P.fs + p] = o[q];
  for (int q = 0; q < 4; q++) aux[(size_t)(4 * dir + q) * P.fs + p] = o[3 + q];
}

// active edges along dir: the active cells along dir, the faces across
__global__ void k_bg_edge(Params P, gop_background bg, int dir, double* out) {
  const int i = NGH + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = NGH + blockIdx.y * blockDim.y + threadIdx.y;
  const int k = NGH + blockIdx.z * blockDim.z + threadIdx.z;
  if (i > NGH + P.n[0] - (dir == 0) || j > NGH + P.n[1] - (dir == 1) || k > NGH + P.n[2] - (dir == 2))
    return;
  const X3 X = face_coords(P);
  const int i1 = i + (dir == 0), j1 = j + (dir == 1), k1 = k + (dir == 2);
  const long long p = lin(P, i, j, k);
  for (int c = 0; c < 3; c++)
    out[(size_t)(BG_EDGE + 3 * dir + c) * P.fs + p] =
        gop_b0_line_mean(&bg, c, X.x1[i1], X.x2[j1], X.x3[k1], X.x1[i], X.x2[j], X.x3[k]);
}

__global__ void k_bg_lorentz(Params P, int sph, const double* aux, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y,
            k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i > P.N[0] - 2 || j > P.N[1] - 2 || k > P.N[2] - 2) return;
  const X3 X = face_coords(P);
  const long long p = lin(P, i, j, k);
  const long long up[3] = {p + 1, p + P.sj, p + P.sk};
  const double a_lo[3] = {gop_face_area(X.x1, X.x2, X.x3, sph, 0, i, j, k),
                          gop_face_area(X.x1, X.x2, X.x3, sph, 1, i, j, k),
                          gop_face_area(X.x1, X.x2, X.x3, sph, 2, i, j, k)};
  const double a_hi[3] = {gop_face_area(X.x1, X.x2, X.x3, sph, 0, i + 1, j, k),
                          gop_face_area(X.x1, X.x2, X.x3, sph, 1, i, j + 1, k),
                          gop_face_area(X.x1, X.x2, X.x3, sph, 2, i, j, k + 1)};
  const double vol = gop_cell_volume(X.x1, X.x2, X.x3, sph, i, j, k);
  for (int c = 0; c < 3; c++) {
    double q_lo[3], q_hi[3], n_lo[3], n_hi[3];
    for (int dir = 0; dir < 3; dir++) {
      const double* bsq = aux + (size_t)(4 * dir) * P.fs;
      const double* bn = aux + (size_t)(4 * dir + 1 + c) * P.fs;
      q_lo[dir] = bsq[p];
      q_hi[dir] = bsq[up[dir]];
      n_lo[dir] = bn[p];
      n_hi[dir] = bn[up[dir]];
    }
    out[(size_t)(BG_LOR + c) * P.fs + p] = gop_b0_lorentz(c, q_lo, q_hi, n_lo, n_hi, a_lo, a_hi, vol);
  }
}

dim3 grid_of(int a, int b, int c, dim3 blk) {
  return dim3((a + blk.x - 1) / blk.x, (b + blk.y - 1) / blk.y, (c + blk.z - 1) / blk.z);
}

}  // namespace

void launch_background(const Params& P, const gop_background& bg, int sph, double* out, double* aux,
                       cudaStream_t st) {
  const dim3 blk(32, 4, 2);
  const int N0 = P.N[0], N1 = P.N[1], N2 = P.N[2];
  k_bg_centroid<<<grid_of(N0 - 1, N1 - 1, N2 - 1, blk), blk, 0, st>>>(P, bg, sph, out);
  for (int dir = 0; dir < 3; dir++)
    k_bg_face<<<grid_of(N0 - 1 + (dir == 0), N1 - 1 + (dir == 1), N2 - 1 + (dir == 2), blk), blk, 0,
                st>>>(P, bg, sph, dir, out, aux);
  for (int dir = 0; dir < 3; dir++)
    k_bg_edge<<<grid_of(P.n[0] + (dir != 0), P.n[1] + (dir != 1), P.n[2] + (dir != 2), blk), blk, 0,
                st>>>(P, bg, dir, out);
  k_bg_lorentz<<<grid_of(N0 - 1, N1 - 1, N2 - 1, blk), blk, 0, st>>>(P, sph, aux, out);
  count_launches(8);
}

}  // namespace gop

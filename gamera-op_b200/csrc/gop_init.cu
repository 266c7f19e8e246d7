// Device-side initial conditions: the problem states of host/gop_problems.c
// built directly in an instance's device state (current buffer, i-fastest
// layout), so a large grid or a served request needs no host-side set-up
// and no upload of the state.  Per point the arithmetic is the host's
// (csrc/gop_fields.h is shared by both); the results differ from the host's
// only by the last-bit differences of the device's sin, cos, exp, acos and
// atan2 and of fused multiply-adds.
//
//   cells   primitives of every cell the host writes (problem_init of the
//           reference problems, e.g. src/problem_test_OT_cartesion.c:50-130)
//   edges   AinitB's line integrals of A along every edge
//           (src/solver_func.c:15-60), into a scratch array of 3 fields
//   faces   face B = circulation around the face / face area
//           (src/solver_func.c:60-95)
#include "gop_device.cuh"
#include "gop_fields.h"
#include "gop_kernels.h"

namespace gop {

namespace {

struct Coords {
  const double* x[3];  // face coordinates per axis (the T_X tables)
};

__device__ __forceinline__ Coords coords(const Params& P) {
  Coords c;
  for (int a = 0; a < 3; a++) c.x[a] = P.tab + ((size_t)a * NTAB + T_X) * P.tmax;
  return c;
}

__global__ void k_init_cells(Params P, gop_problem p, int sph) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y,
            k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= P.N[0] || j >= P.N[1] || k >= P.N[2]) return;
  const Coords X = coords(P);
  const double *x1 = X.x[0], *x2 = X.x[1], *x3 = X.x[2];
  double* W = P.Wbuf[0];
  double* B = P.Bbuf[0];
  const size_t fs = P.fs;
  const long long c = lin(P, i, j, k);
  const bool act = i >= NGH && i < NGH + P.n[0] && j >= NGH && j < NGH + P.n[1] && k >= NGH &&
                   k < NGH + P.n[2];
  if (p.kind == GOP_PROBLEM_OT) {
    if (!act) return;
    const double xc = 0.5 * (x1[i] + x1[i + 1]), yc = 0.5 * (x2[j] + x2[j + 1]);
    W[c] = 25.0 / (GOP_PI * 36.0);
    W[c + 4 * fs] = 5.0 / (GOP_PI * 12.0);
    W[c + fs] = -sin(2 * GOP_PI * yc);
    W[c + 2 * fs] = sin(2 * GOP_PI * xc);
  } else if (p.kind == GOP_PROBLEM_LOOP_CART) {
    if (!act) return;
    W[c] = p.rho;
    W[c + fs] = p.v[0];
    W[c + 2 * fs] = p.v[1];
    W[c + 3 * fs] = p.v[2];
    W[c + 4 * fs] = p.p_out;
  } else if (p.kind == GOP_PROBLEM_LOOP_SPH) {
    if (i > P.N[0] - 2 || j > P.N[1] - 2 || k > P.N[2] - 2) return;
    double r, t, f, x, y, z, v1, v2, v3;
    gop_sph_centroid(x1, x2, x3, i, j, k, &r, &t, &f);
    gop_sph_to_cart(r, t, f, &x, &y, &z);
    gop_cart_vec_to_sph(x, y, z, p.v[0], p.v[1], p.v[2], &v1, &v2, &v3);
    W[c] = p.rho;
    W[c + fs] = v1;
    W[c + 2 * fs] = v2;
    W[c + 3 * fs] = v3;
    W[c + 4 * fs] = p.p_out;
  } else if (p.kind == GOP_PROBLEM_BLAST) {
    // cells and the uniform face field on the active faces of each axis
    const int lo = NGH, hi[3] = {NGH + P.n[0] - 1, NGH + P.n[1] - 1, NGH + P.n[2] - 1};
    const int q[3] = {i, j, k};
    for (int a = 0; a < 3; a++) {
      bool in = true;
      for (int d = 0; d < 3; d++) in = in && q[d] >= lo && q[d] <= hi[d] + (d == a);
      if (in) B[c + a * fs] = p.b[a];
    }
    if (!act) return;
    const double dx = 0.5 * (x1[i] + x1[i + 1]) - p.center[0];
    const double dy = 0.5 * (x2[j] + x2[j + 1]) - p.center[1];
    const double dz = 0.5 * (x3[k] + x3[k + 1]) - p.center[2];
    const double rr = sqrt(dx * dx + dy * dy + dz * dz);
    W[c] = p.rho;
    W[c + 4 * fs] = rr < p.radius ? p.p_in : p.p_out;
  }
}

// LA[a] at (i, j, k): the line integral along the edge of axis a; z runs
// over k and the three axes
__global__ void k_init_edges(Params P, gop_problem p, int sph, double* __restrict__ LA) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y,
            z = blockIdx.z * blockDim.z + threadIdx.z;
  const int a = z / P.N[2], k = z % P.N[2];
  if (a >= 3 || i >= P.N[0] || j >= P.N[1]) return;
  // AinitB's ranges: 0..ieg along the edge's axis, 0..ieg+1 across it
  if ((a == 0 && i > P.N[0] - 2) || (a == 1 && j > P.N[1] - 2) || (a == 2 && k > P.N[2] - 2))
    return;
  const Coords X = coords(P);
  LA[(size_t)a * P.fs + lin(P, i, j, k)] =
      gop_edge_integral(&p, X.x[0], X.x[1], X.x[2], sph, a, i, j, k);
}

// face B from the edge integrals (Stokes); z runs over k and the three axes
__global__ void k_init_faces(Params P, int sph, const double* __restrict__ LA) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y,
            z = blockIdx.z * blockDim.z + threadIdx.z;
  const int a = z / P.N[2], k = z % P.N[2];
  if (a >= 3 || i >= P.N[0] || j >= P.N[1]) return;
  // 0..ieg+1 along the face normal, 0..ieg across it
  if ((a != 0 && i > P.N[0] - 2) || (a != 1 && j > P.N[1] - 2) || (a != 2 && k > P.N[2] - 2))
    return;
  const Coords X = coords(P);
  const size_t fs = P.fs;
  const long long c = lin(P, i, j, k), sj = P.sj, sk = P.sk;
  const double *Li = LA, *Lj = LA + fs, *Lk = LA + 2 * fs;
  const double f = gop_face_area(X.x[0], X.x[1], X.x[2], sph, a, i, j, k);
  double b;
  if (a == 0) b = (Lj[c] - Lj[c + sk] + Lk[c + sj] - Lk[c]) / f;
  else if (a == 1) b = -(Li[c] - Li[c + sk] + Lk[c + 1] - Lk[c]) / f;
  else b = (Li[c] - Li[c + sj] + Lj[c + 1] - Lj[c]) / f;
  P.Bbuf[0][c + a * fs] = f < 1e-10 ? 0.0 : b;
}

dim3 grid_of(int a, int b, int c, dim3 blk) {
  return dim3((a + blk.x - 1) / blk.x, (b + blk.y - 1) / blk.y, (c + blk.z - 1) / blk.z);
}

}  // namespace

void launch_problem_init(const Params& P, const gop_problem& p, int sph, double* scratch,
                         cudaStream_t st) {
  const dim3 blk(32, 4, 2);
  k_init_cells<<<grid_of(P.N[0], P.N[1], P.N[2], blk), blk, 0, st>>>(P, p, sph);
  count_launches(1);
  if (p.kind == GOP_PROBLEM_BLAST) return;
  k_init_edges<<<grid_of(P.N[0], P.N[1], 3 * P.N[2], blk), blk, 0, st>>>(P, p, sph, scratch);
  k_init_faces<<<grid_of(P.N[0], P.N[1], 3 * P.N[2], blk), blk, 0, st>>>(P, sph, scratch);
  count_launches(2);
}

}  // namespace gop

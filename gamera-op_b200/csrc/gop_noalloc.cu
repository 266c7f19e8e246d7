// CFL time step and max|div B| of a caller-owned device state, computed
// without allocating any memory.
//
// Who needs this: a host that already keeps its grid in device memory and
// has to ask "what dt does this state allow?" where it may not allocate --
// a serving loop whose device memory was reserved once at start-up and may
// not grow (an allocation there can fail, or wait for the whole device,
// since cudaMalloc and cudaFree synchronise with running work), or a host
// program that owns all of its device buffers and hands the library only
// pointers.  The instance API (gop_create / gop_prepare) needs its own
// buffers; this entry point needs none.
//
// Its only scratch is g_cfl_scratch below: a file-scope device array of
// GOP_NOALLOC_SCRATCH_DOUBLES doubles (64 KiB) that every GPU loading this
// library holds until the process exits.  It stores the three coordinate
// arrays of the call (at most GOP_NOALLOC_MAX_N active cells per axis) and
// one (dt, div B) partial per block of the reduction.  Every call overwrites
// what it reads, so nothing has to start at zero; but all calls share the
// one array, so two calls whose kernels overlap on the GPU (different
// streams, or different host threads) race on it.
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <mutex>

#include "gamera_op.h"
#include "gop_internal.h"

namespace {

constexpr int kMaxN = GOP_NOALLOC_MAX_N;               // active cells per axis
constexpr int kStride = kMaxN + 16;                    // coordinate slot length
constexpr int kMaxBlocks = 2048;                       // reduction partials
constexpr int kScratch = GOP_NOALLOC_SCRATCH_DOUBLES;  // 3 slots + 2 * blocks
static_assert(3 * kStride + 2 * kMaxBlocks <= kScratch, "scratch layout");

__device__ __align__(256) double g_cfl_scratch[kScratch];

constexpr int NG = 4;
constexpr int kThreads = 256;

struct Args {
  int n[3], N[3];
  int sph;
  double gamma, cfl, ca, ca2;
  const double* gas;  // [6][NI][NJ][NK], k fastest (reference layout)
  const double* fb;   // [3][NI][NJ][NK]
  const double* b0;   // background field at the cell centroid [3][NI][NJ][NK], or null
  const double* b0f;  // background field averaged over the faces [9][NI][NJ][NK], or null
  double* scratch;    // device address of g_cfl_scratch on this device
  double* out;        // out[0] = dt, out[1] = max|div B|
  int nblocks;
};

__device__ __forceinline__ const double* coord(const Args& A, int a) {
  return A.scratch + (size_t)a * kStride;
}

// position of the volume centroid along axis a in cell c (x1ctr / x2ctr /
// x3ctr of src/cartesian/cartesian_general.c:190-201 and
// src/spherical/spherical_general.c:205-234)
__device__ double centroid(const Args& A, int a, int c) {
  const double* x = coord(A, a);
  double x0 = x[c], x1 = x[c + 1], xc = 0.5 * (x0 + x1), dx = x1 - x0;
  if (!A.sph || a == 2) return xc;
  if (a == 0) return xc + 2.0 * xc * dx * dx / (12.0 * xc * xc + dx * dx);
  return (sin(x1) - sin(x0) - (x1 * cos(x1) - x0 * cos(x0))) / (-cos(x1) + cos(x0));
}

__device__ double face_area(const Args& A, int a, int i, int j, int k) {
  const double *x1 = coord(A, 0), *x2 = coord(A, 1), *x3 = coord(A, 2);
  double d1 = x1[i + 1] - x1[i], d2 = x2[j + 1] - x2[j], d3 = x3[k + 1] - x3[k];
  if (!A.sph) return a == 0 ? d2 * d3 : (a == 1 ? d1 * d3 : d1 * d2);
  if (a == 0) return -x1[i] * x1[i] * (cos(x2[j + 1]) - cos(x2[j])) * d3;
  double h = 0.5 * (x1[i + 1] * x1[i + 1] - x1[i] * x1[i]);
  return a == 1 ? h * sin(x2[j]) * d3 : h * d2;
}

__device__ void cell_dt_divb(const Args& A, int i, int j, int k, double& dt, double& divb) {
  const double *x1 = coord(A, 0), *x2 = coord(A, 1), *x3 = coord(A, 2);
  size_t s1 = (size_t)A.N[1] * A.N[2], s2 = A.N[2];
  size_t c = (size_t)i * s1 + (size_t)j * s2 + k, n3 = (size_t)A.N[0] * s1;
  const double* g = A.gas;
  const double* b = A.fb;
  double d1 = x1[i + 1] - x1[i], d2 = x2[j + 1] - x2[j], d3 = x3[k + 1] - x3[k];
  // cell-centred field from the faces (src/solver_func.c:311-322)
  double xc[3] = {centroid(A, 0, i), centroid(A, 1, j), centroid(A, 2, k)};
  double m1 = b[c] * (x1[i + 1] - xc[0]) / d1 + b[c + s1] * (xc[0] - x1[i]) / d1;
  double m2 = b[n3 + c] * (x2[j + 1] - xc[1]) / d2 + b[n3 + c + s2] * (xc[1] - x2[j]) / d2;
  double m3 = b[2 * n3 + c] * (x3[k + 1] - xc[2]) / d3 + b[2 * n3 + c + 1] * (xc[2] - x3[k]) / d3;
  // magtot = mags + B0 (src/solver_func.c:345-353)
  if (A.b0) {
    m1 += A.b0[c];
    m2 += A.b0[n3 + c];
    m3 += A.b0[2 * n3 + c];
  }
  // get_dt_normal (src/solver_func.c:255-298)
  double rho = g[c], u = g[n3 + c], v = g[2 * n3 + c], w = g[3 * n3 + c], p = g[4 * n3 + c];
  double va = sqrt((m1 * m1 + m2 * m2 + m3 * m3) / rho);
  double vae = va * A.ca / sqrt(va * va + A.ca2);
  double vf = sqrt(u * u + v * v + w * w);
  double vs = sqrt(A.gamma * p / rho);
  double vc = vf + sqrt(vs * vs + vae * vae);
  double l1 = d1, l2 = d2, l3 = d3;
  if (A.sph) {
    double rc = 0.5 * (x1[i] + x1[i + 1]), tc = 0.5 * (x2[j] + x2[j + 1]);
    l2 = rc * d2;
    l3 = rc * sin(tc) * d3;
  }
  dt = A.cfl / (vc / l1 + vc / l2 + vc / l3);
  // div B over the cell (src/solver_func.c:324-343)
  double vol = A.sph ? fabs(1.0 / 3.0 * (pow(x1[i + 1], 3) - pow(x1[i], 3)) *
                            (cos(x2[j + 1]) - cos(x2[j])) * d3)
                     : d1 * d2 * d3;
  // face-normal field, plus the face-averaged background normal component
  // (B0AfaceI/J/K_bn, src/solver_func.c:324-343)
  double bl[3] = {b[c], b[n3 + c], b[2 * n3 + c]};
  double bu[3] = {b[c + s1], b[n3 + c + s2], b[2 * n3 + c + 1]};
  if (A.b0f) {
    const double* f0 = A.b0f;            // faces normal to i, component i
    const double* f1 = A.b0f + 4 * n3;   // faces normal to j, component j
    const double* f2 = A.b0f + 8 * n3;   // faces normal to k, component k
    bl[0] += f0[c];
    bu[0] += f0[c + s1];
    bl[1] += f1[c];
    bu[1] += f1[c + s2];
    bl[2] += f2[c];
    bu[2] += f2[c + 1];
  }
  double db = (bu[0] * face_area(A, 0, i + 1, j, k) - bl[0] * face_area(A, 0, i, j, k)) / vol +
              (bu[1] * face_area(A, 1, i, j + 1, k) - bl[1] * face_area(A, 1, i, j, k)) / vol +
              (bu[2] * face_area(A, 2, i, j, k + 1) - bl[2] * face_area(A, 2, i, j, k)) / vol;
  divb = fabs(db);
}

// per-block (min dt, max |div B|) into the scratch partials
__global__ void __launch_bounds__(kThreads) k_cfl_partial(Args A) {
  __shared__ double sdt[kThreads / 32], sdb[kThreads / 32];
  long long cells = (long long)A.n[0] * A.n[1] * A.n[2];
  double dt = DBL_MAX, db = 0.0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < cells;
       t += (long long)gridDim.x * blockDim.x) {
    int k = (int)(t % A.n[2]);
    long long r = t / A.n[2];
    int j = (int)(r % A.n[1]);
    int i = (int)(r / A.n[1]);
    double c_dt, c_db;
    cell_dt_divb(A, i + NG, j + NG, k + NG, c_dt, c_db);
    dt = fmin(dt, c_dt);
    db = fmax(db, c_db);
  }
  for (int o = 16; o > 0; o >>= 1) {
    dt = fmin(dt, __shfl_xor_sync(0xffffffffu, dt, o));
    db = fmax(db, __shfl_xor_sync(0xffffffffu, db, o));
  }
  if ((threadIdx.x & 31) == 0) {
    sdt[threadIdx.x / 32] = dt;
    sdb[threadIdx.x / 32] = db;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kThreads / 32; w++) {
      dt = fmin(dt, sdt[w]);
      db = fmax(db, sdb[w]);
    }
    double* part = A.scratch + 3 * kStride;
    part[2 * blockIdx.x] = dt;
    part[2 * blockIdx.x + 1] = db;
  }
}

// one block folds the partials written by this call into out[0..1]
__global__ void __launch_bounds__(kThreads) k_cfl_final(Args A) {
  __shared__ double sdt[kThreads / 32], sdb[kThreads / 32];
  const double* part = A.scratch + 3 * kStride;
  double dt = DBL_MAX, db = 0.0;
  for (int t = threadIdx.x; t < A.nblocks; t += blockDim.x) {
    dt = fmin(dt, part[2 * t]);
    db = fmax(db, part[2 * t + 1]);
  }
  for (int o = 16; o > 0; o >>= 1) {
    dt = fmin(dt, __shfl_xor_sync(0xffffffffu, dt, o));
    db = fmax(db, __shfl_xor_sync(0xffffffffu, db, o));
  }
  if ((threadIdx.x & 31) == 0) {
    sdt[threadIdx.x / 32] = dt;
    sdb[threadIdx.x / 32] = db;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kThreads / 32; w++) {
      dt = fmin(dt, sdt[w]);
      db = fmax(db, sdb[w]);
    }
    A.out[0] = dt;
    A.out[1] = db;
  }
}

// device address of g_cfl_scratch, looked up once per device
std::mutex g_mu;
double* g_addr[64] = {};

}  // namespace

extern "C" int gop_cfl_dt_noalloc(const gop_desc* desc, const double* gas, const double* face_b,
                                  const double* b0, const double* b0_face, double* out,
                                  void* stream) {
  int rc = gop::check_desc(desc);
  if (rc) return rc;
  if (!gas || !face_b || !out) return gop::set_error(GOP_EINVAL, "gop_cfl_dt_noalloc: NULL array");
  if ((b0 == nullptr) != (b0_face == nullptr))
    return gop::set_error(GOP_EINVAL, "gop_cfl_dt_noalloc: b0 and b0_face go together");
  // ring-averaged grids take the CFL length of their pole rows from the
  // ring average (get_dt_ring), which this call does not compute
  if (desc->ring_average)
    return gop::set_error(GOP_EINVAL, "gop_cfl_dt_noalloc: grids with the pole ring average are not supported");
  if (desc->ni > kMaxN || desc->nj > kMaxN || desc->nk > kMaxN)
    return gop::set_error(GOP_EINVAL,
                          "gop_cfl_dt_noalloc: grid %dx%dx%d exceeds the static scratch limit of %d "
                          "active cells per axis",
                          desc->ni, desc->nj, desc->nk, kMaxN);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 64)
    return gop::set_error(GOP_ECUDA, "gop_cfl_dt_noalloc: cudaGetDevice: %s", cudaGetErrorString(e));
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
      // first call on this device: resolve the array's device address
      e = cudaGetSymbolAddress((void**)&g_addr[dev], g_cfl_scratch);
      if (e != cudaSuccess) {
        g_addr[dev] = nullptr;
        return gop::set_error(GOP_ECUDA, "gop_cfl_dt_noalloc: cudaGetSymbolAddress: %s",
                              cudaGetErrorString(e));
      }
    }
    scratch = g_addr[dev];
  }
  cudaStream_t st = (cudaStream_t)stream;
  Args A;
  A.n[0] = desc->ni;
  A.n[1] = desc->nj;
  A.n[2] = desc->nk;
  for (int a = 0; a < 3; a++) A.N[a] = A.n[a] + 2 * NG + 1;
  A.sph = desc->coord == GOP_COORD_SPHERICAL;
  A.gamma = desc->gamma != 0 ? desc->gamma : 5.0 / 3.0;
  A.cfl = desc->cfl != 0 ? desc->cfl : 0.3;
  A.ca = desc->ca != 0 ? desc->ca : 10.0;
  A.ca2 = A.ca * A.ca;
  A.gas = gas;
  A.fb = face_b;
  A.b0 = b0;
  A.b0f = b0_face;
  A.scratch = scratch;
  A.out = out;
  const double* xs[3] = {desc->x1, desc->x2, desc->x3};
  for (int a = 0; a < 3; a++) {
    e = cudaMemcpyAsync(scratch + (size_t)a * kStride, xs[a], sizeof(double) * A.N[a],
                        cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess)
      return gop::set_error(GOP_ECUDA, "gop_cfl_dt_noalloc: coordinate copy: %s", cudaGetErrorString(e));
  }
  long long cells = (long long)A.n[0] * A.n[1] * A.n[2];
  long long want = (cells + kThreads - 1) / kThreads;
  A.nblocks = (int)(want < kMaxBlocks ? want : kMaxBlocks);
  k_cfl_partial<<<A.nblocks, kThreads, 0, st>>>(A);
  k_cfl_final<<<1, kThreads, 0, st>>>(A);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return gop::set_error(GOP_ECUDA, "gop_cfl_dt_noalloc: launch: %s", cudaGetErrorString(e));
  return GOP_OK;
}

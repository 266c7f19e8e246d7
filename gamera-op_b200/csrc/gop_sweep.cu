// Tile-staged flux sweeps of the MHD step for B200 (sm_100a).
//
// The face flux along axis D (PDM reconstruction of the 8 face states,
// Rusanov flux and Maxwell stress, src/solver_func.c:215-253,503-685,
// 934-1529) is the step's largest stage.  Its per-face form (k_flux in
// gop_kernels.cu) gathers each face's 8-point stencils of 16 input fields
// with ~100 global loads through L1; the loads' 64-bit address arithmetic
// and their latency, not the FP64 arithmetic, bound it.  Here each block is
// persistent and runs a copy pipeline:
//
//   copies   one elected thread streams tiles into a ring of STAGES
//            shared-memory slots with cp.async.bulk.tensor (one TMA box per
//            input array and tile), completing on the slot's "full"
//            mbarrier;
//   compute  8 warps compute one face per thread from shared memory (every
//            stencil tap is a load at a compile-time offset from one
//            per-thread base) and release the slot on its "empty"
//            mbarrier.
//
// So the global-memory latency of tile n+1 overlaps the arithmetic of tile
// n, and the stencil re-reads come from shared memory instead of L1.  The
// per-face arithmetic is the per-face kernel's own (recon_lr, flux_out), in
// the same order, so both kernels give the same results.
//
// Tiles (x = i, y = j, z = k; one box per array, field extent nf):
//   D = 0  32 faces along i (lanes) x 8 rows along j (warps) x 1 plane
//          box (40, 8, 1) from (f0 - 4, j0, k): stencil and limiter alike
//   D = 1  32 cells along i (lanes) x 8 faces along j (warps) x 1 plane
//          stencil box (32, 15, 1) from (i0, f0 - 4, k),
//          limiter box (32, 11, 1) from (i0, f0 - 2, k)
//   D = 2  32 cells along i x 1 row x 8 faces along k (warps)
//          stencil box (32, 1, 15) from (i0, j, f0 - 4),
//          limiter box (32, 1, 11) from (i0, j, f0 - 2)
// Every box starts at an x of f0 - 4 = 32 t or i0 = 4 + 32 t, so x times
// the element size is a multiple of 16 bytes (the TMA's alignment rule).
// Tiles are numbered with the x tile fastest, then the tile along the
// sweep, so the blocks in flight at any time share their halo rows in L2.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "gop_stage.cuh"
#include "gop_tma.cuh"

namespace gop {

constexpr int kConsumerWarps = 8;
constexpr int kSweepThreads = 32 * kConsumerWarps;

// shared-memory ring and residency per arithmetic type: two 53 KB slots
// and two blocks per SM in FP64, two 26 KB slots and three blocks in FP32
#ifndef GOP_SWEEP_STAGES_F64
#define GOP_SWEEP_STAGES_F64 2
#endif
#ifndef GOP_SWEEP_STAGES_F32
#define GOP_SWEEP_STAGES_F32 2
#endif
#ifndef GOP_SWEEP_CTAS_F64
#define GOP_SWEEP_CTAS_F64 2
#endif
#ifndef GOP_SWEEP_CTAS_F32
#define GOP_SWEEP_CTAS_F32 3
#endif
// 1: the sweeps go out with programmatic dependent launch like the other
// step kernels.  Off: a sweep grid placed early onto SMs that still run the
// previous kernel (persistent blocks, no room to spare) measured 2-20 %
// slower on B200 (blast 256^3: FP32 flux 2.47 vs 2.06 ms per step)
#ifndef GOP_SWEEP_PDL
#define GOP_SWEEP_PDL 0
#endif
template <typename R>
struct SweepCfg {
  static constexpr int STAGES = sizeof(R) == 8 ? GOP_SWEEP_STAGES_F64 : GOP_SWEEP_STAGES_F32;
  static constexpr int CTAS = sizeof(R) == 8 ? GOP_SWEEP_CTAS_F64 : GOP_SWEEP_CTAS_F32;
};

template <int D>
struct FluxTile {
  static constexpr int SX = D == 0 ? 40 : 32;
  static constexpr int SY = D == 0 ? 8 : (D == 1 ? 15 : 1);
  static constexpr int SZ = D == 2 ? 15 : 1;
  static constexpr int LX = SX;
  static constexpr int LY = D == 1 ? 11 : SY;
  static constexpr int LZ = D == 2 ? 11 : 1;
  static constexpr int SB = SX * SY * SZ;  // elements per field, stencil box
  static constexpr int LB = LX * LY * LZ;  // elements per field, limiter box
  static constexpr int NG = 5;             // gas fields (the entropy channel is off)
  // PDM weights of the tile's faces: D = 0 the 18 tap-major tables of the
  // 32 faces (box (32, 18) of the per-axis tables), else the 8 packed face
  // records (box (FW, 8))
  static constexpr int WB = D == 0 ? 18 * 32 : FW * 8;
  static constexpr int BNB = 256;          // step-start face field normal to the faces
  // slot layout in elements of R: W_h, limiter W, mags_h, mags, weights, B_n
  static constexpr int OFF_WH = 0;
  static constexpr int OFF_WL = OFF_WH + NG * SB;
  static constexpr int OFF_MSH = OFF_WL + NG * LB;
  static constexpr int OFF_MS = OFF_MSH + 3 * SB;
  static constexpr int OFF_W = OFF_MS + 3 * LB;
  static constexpr int OFF_BN = OFF_W + WB;
  static constexpr int ELEMS = OFF_BN + BNB;
};

template <typename R, int D>
__host__ __device__ constexpr int slot_bytes() {
  return FluxTile<D>::ELEMS * (int)sizeof(R);
}
template <typename R, int D>
__host__ __device__ constexpr int sweep_smem() {
  return SweepCfg<R>::STAGES * slot_bytes<R, D>() + 2 * SweepCfg<R>::STAGES * 8 + 128;
}

// every TMA destination must start on a 128-byte boundary
template <typename R, int D>
constexpr bool slots_aligned() {
  using T = FluxTile<D>;
  constexpr int e = sizeof(R);
  return (T::OFF_WL * e) % 128 == 0 && (T::OFF_MSH * e) % 128 == 0 && (T::OFF_MS * e) % 128 == 0 &&
         (T::OFF_W * e) % 128 == 0 && (T::OFF_BN * e) % 128 == 0 && (T::ELEMS * e) % 128 == 0;
}
static_assert(slots_aligned<double, 0>() && slots_aligned<double, 1>() && slots_aligned<double, 2>(),
              "FP64 slot layout");
static_assert(slots_aligned<float, 0>() && slots_aligned<float, 1>() && slots_aligned<float, 2>(),
              "FP32 slot layout");
static_assert(sweep_smem<double, 1>() * SweepCfg<double>::CTAS <= 228 * 1024, "FP64 blocks per SM");
static_assert(sweep_smem<float, 1>() * SweepCfg<float>::CTAS <= 228 * 1024, "FP32 blocks per SM");

struct alignas(64) FluxMaps {
  CUtensorMap wh;     // W_h, stencil box
  CUtensorMap wl[2];  // limiter reference: FP64 the state buffer of each parity, FP32 its copy
  CUtensorMap msh;    // mags_h, stencil box
  CUtensorMap ms;     // mags, limiter box
  CUtensorMap wt;     // PDM weights of the tile's faces
  CUtensorMap bn[2];  // step-start face field (as wl: per parity in FP64)
  int nt[3];          // tiles: x, along the sweep (D = 0: rows of j), third axis
};

struct SweepSet {
  FluxMaps flux[3];
  int sms = 0;
};

// tile t of the sweep along D: TMA origin of the stencil and limiter boxes
// and the cell / face of (warp, lane)
template <int D>
struct TileAt {
  int sx, sy, sz;  // stencil box origin
  int ly, lz;      // limiter box origin (x as the stencil's)
  int i, j, k;     // this thread's face (index along D) and transverse cell
};

template <int D>
__device__ __forceinline__ TileAt<D> tile_at(const int nt[3], int t, int warp, int lane) {
  const int a = t % nt[0], r = t / nt[0], b = r % nt[1], c = r / nt[1];
  TileAt<D> T;
  if constexpr (D == 0) {
    T.sx = 32 * a;
    T.sy = NGH + 8 * b;
    T.sz = NGH + c;
    T.ly = T.sy;
    T.lz = T.sz;
    T.i = NGH + 32 * a + lane;
    T.j = NGH + 8 * b + warp;
    T.k = NGH + c;
  } else if constexpr (D == 1) {
    T.sx = NGH + 32 * a;
    T.sy = 8 * b;
    T.sz = NGH + c;
    T.ly = 8 * b + 2;
    T.lz = T.sz;
    T.i = NGH + 32 * a + lane;
    T.j = NGH + 8 * b + warp;
    T.k = NGH + c;
  } else {
    T.sx = NGH + 32 * a;
    T.sy = NGH + c;
    T.sz = 8 * b;
    T.ly = T.sy;
    T.lz = 8 * b + 2;
    T.i = NGH + 32 * a + lane;
    T.j = NGH + c;
    T.k = NGH + 8 * b + warp;
  }
  return T;
}

// the faces of one tile from a filled slot (one face per consumer thread)
template <typename R, int D, bool BG>
__device__ __forceinline__ void flux_tile(const Params& P, const Work<R>& wk, const R* __restrict__ s,
                                          const TileAt<D>& T, int warp, int lane) {
  using F = FluxTile<D>;
  const bool on = T.i < NGH + P.n[0] + (D == 0) && T.j < NGH + P.n[1] + (D == 1) &&
                  T.k < NGH + P.n[2] + (D == 2);
  if (!on) return;
  // per-thread bases: tap t of field m is then at a compile-time offset
  const R* wh;
  const R* wl;
  const R* msh;
  const R* ms;
  if constexpr (D == 0) {
    const int b = warp * F::SX + lane;
    wh = s + F::OFF_WH + b;
    wl = s + F::OFF_WL + b + 2;  // the limiter cells f-2..f+1 start 2 cells in
    msh = s + F::OFF_MSH + b;
    ms = s + F::OFF_MS + b + 2;
  } else {
    const int b = warp * 32 + lane;
    wh = s + F::OFF_WH + b;
    wl = s + F::OFF_WL + b;
    msh = s + F::OFF_MSH + b;
    ms = s + F::OFF_MS + b;
  }
  constexpr int TS = D == 0 ? 1 : 32;  // stride of one stencil tap in the slot
  FaceWeights<R> Wt;
  if constexpr (D == 0) {  // this lane's face in the 18 tap-major rows
    const R* w = s + F::OFF_W + lane;
#pragma unroll
    for (int t = 0; t < 7; t++) {
      Wt.wl[t] = w[t * 32];
      Wt.wr[t] = w[(7 + t) * 32];
    }
    Wt.cl1 = w[14 * 32];
    Wt.cl2 = w[15 * 32];
    Wt.cr1 = w[16 * 32];
    Wt.cr2 = w[17 * 32];
  } else {  // the warp's face record (one broadcast address)
    load_fw_smem(s + F::OFF_W + warp * FW, Wt);
  }
  const R bn = s[F::OFF_BN + warp * 32 + lane];
  const R a1h = (R)(0.5 * P.pdm_a1), a2 = (R)P.pdm_a2;
  R L[6], Rt[6], mL[3], mR[3];
  L[PS] = Rt[PS] = R(0);
#pragma unroll
  for (int m = 0; m < F::NG; m++) {
    R v[8], lim[4];
#pragma unroll
    for (int t = 0; t < 8; t++) v[t] = wh[m * F::SB + t * TS];
#pragma unroll
    for (int u = 0; u < 4; u++) lim[u] = wl[m * F::LB + u * TS];
    recon_lr<R>(v, lim, Wt, a1h, a2, L[m], Rt[m]);
  }
#pragma unroll
  for (int a = 0; a < 3; a++) {
    R v[8], lim[4];
#pragma unroll
    for (int t = 0; t < 8; t++) v[t] = msh[a * F::SB + t * TS];
#pragma unroll
    for (int u = 0; u < 4; u++) lim[u] = ms[a * F::LB + u * TS];
    recon_lr<R>(v, lim, Wt, a1h, a2, mL[a], mR[a]);
  }
  flux_out<R, D, BG, false>(P, wk, lin(P, T.i, T.j, T.k), L, Rt, mL, mR, bn);
}

// Persistent flux sweep along D (entropy channel off).  Lane 0 of warp 0
// also feeds the ring: it fills the first STAGES slots, and after each tile
// waits until all 8 warps have released that tile's slot, then issues the
// tile STAGES ahead into it; the other warps meanwhile compute the next
// tile, whose copies were issued a tile earlier.
template <typename R, int D, bool BG>
__global__ void __launch_bounds__(kSweepThreads, SweepCfg<R>::CTAS)
    k_flux_sweep(Params P, Work<R> wk, const __grid_constant__ FluxMaps maps) {
  pdl_enter();
  // stop flag, or an earlier pipeline wait that timed out: do nothing
  if (stopped(P) || P.scal[S_FLAGS] == 2.0) return;
  using F = FluxTile<D>;
  constexpr int S = SweepCfg<R>::STAGES;
  extern __shared__ unsigned char smem_dyn[];
  // TMA destinations on 128-byte boundaries (the launch adds 128 bytes)
  unsigned char* smem_raw = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_dyn) + 127) & ~static_cast<uintptr_t>(127));
  R* slots = reinterpret_cast<R*>(smem_raw);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + S * slot_bytes<R, D>());
  uint64_t* empty = full + S;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool feeder = threadIdx.x == 0;
  const int ntiles = maps.nt[0] * maps.nt[1] * maps.nt[2];
  const int par = sizeof(R) == 8 ? cur_buf(P) : 0;
  const CUtensorMap* wl = &maps.wl[par];
  const CUtensorMap* bnm = &maps.bn[par];
  // issues the copies of the n-th tile of this block (tile index t) into its slot
  auto issue = [&](int n, int t) {
    const int q = n % S;
    const TileAt<D> T = tile_at<D>(maps.nt, t, 0, 0);
    R* s = slots + (size_t)q * F::ELEMS;
    mbar_arrive_expect_tx(&full[q], slot_bytes<R, D>());
    tma_load_4d(s + F::OFF_WH, &maps.wh, &full[q], T.sx, T.sy, T.sz, 0);
    tma_load_4d(s + F::OFF_WL, wl, &full[q], T.sx, T.ly, T.lz, 0);
    tma_load_4d(s + F::OFF_MSH, &maps.msh, &full[q], T.sx, T.sy, T.sz, 0);
    tma_load_4d(s + F::OFF_MS, &maps.ms, &full[q], T.sx, T.ly, T.lz, 0);
    // weights: D = 0 rows T_WL0.. of the faces f0..f0+31 of axis 0; else the
    // records of faces f0..f0+7 of axis D
    const int f0 = D == 0 ? T.sx + NGH : (D == 1 ? T.sy + NGH : T.sz + NGH);
    if constexpr (D == 0) tma_load_4d(s + F::OFF_W, &maps.wt, &full[q], f0, T_WL0, 0, 0);
    else tma_load_4d(s + F::OFF_W, &maps.wt, &full[q], 0, D * P.tmax + f0, 0, 0);
    // B_n at the tile's faces
    if constexpr (D == 0) tma_load_4d(s + F::OFF_BN, bnm, &full[q], f0, T.sy, T.sz, 0);
    else if constexpr (D == 1) tma_load_4d(s + F::OFF_BN, bnm, &full[q], T.sx, f0, T.sz, 1);
    else tma_load_4d(s + F::OFF_BN, bnm, &full[q], T.sx, T.sy, f0, 2);
  };
  int issued = 0;  // feeder only: tiles whose copies were issued
  if (feeder) {
    for (int q = 0; q < S; q++) {
      mbar_init(&full[q], 1);
      mbar_init(&empty[q], kConsumerWarps);
    }
    fence_mbar_init();
    for (int t = blockIdx.x; t < ntiles && issued < S; t += gridDim.x) issue(issued++, t);
  }
  __syncthreads();
  bool ok = true;
  int n = 0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x, n++) {
    const int q = n % S;
    const uint32_t ph = (n / S) & 1;
    if (!mbar_wait(&full[q], ph)) {
      ok = false;
      break;
    }
    const TileAt<D> T = tile_at<D>(maps.nt, t, warp, lane);
    flux_tile<R, D, BG>(P, wk, slots + (size_t)q * F::ELEMS, T, warp, lane);
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[q]);
    if (feeder) {
      const int tn = t + S * (int)gridDim.x;
      if (tn < ntiles) {
        // every warp has released this slot: refill it with the tile S ahead
        if (!mbar_wait(&empty[q], ph)) {
          ok = false;
          break;
        }
        issue(issued++, tn);
      }
    }
  }
  if (feeder) {
    // the copies of the tiles issued last must land before the block exits
    for (int m = issued > S ? issued - S : 0; m < issued; m++)
      if (!mbar_wait(&full[m % S], (m / S) & 1)) ok = false;
  }
  if (!ok) P.scal[S_FLAGS] = 2.0;
}

// ------------------------------------------------------------------ host

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

// a 4-D map (i, j, k, field) over nf fields of one array in the state's
// layout, read in boxes of bx x by x bz x bf elements
template <typename R>
static bool make_map(CUtensorMap* m, const R* base, int nf, const Params& P, int bx, int by, int bz,
                     int bf) {
  EncodeTiledFn fn = encode_fn();
  if (!fn || !base) return false;
  const cuuint64_t es = sizeof(R);
  const cuuint64_t dims[4] = {(cuuint64_t)P.N[0], (cuuint64_t)P.N[1], (cuuint64_t)P.N[2], (cuuint64_t)nf};
  const cuuint64_t strides[3] = {(cuuint64_t)P.pitch * es, (cuuint64_t)P.sk * es, (cuuint64_t)P.fs * es};
  const cuuint32_t box[4] = {(cuuint32_t)bx, (cuuint32_t)by, (cuuint32_t)bz, (cuuint32_t)bf};
  const cuuint32_t el[4] = {1, 1, 1, 1};
  const CUresult r =
      fn(m, sizeof(R) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
         const_cast<R*>(base), dims, strides, box, el, CU_TENSOR_MAP_INTERLEAVE_NONE,
         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// a 4-D map over a plain array of dims d[0..3] (elements, d[0] fastest)
template <typename R>
static bool make_map_dims(CUtensorMap* m, const R* base, const cuuint64_t d[4], const int box[4]) {
  EncodeTiledFn fn = encode_fn();
  if (!fn || !base) return false;
  const cuuint64_t es = sizeof(R);
  const cuuint64_t strides[3] = {d[0] * es, d[0] * d[1] * es, d[0] * d[1] * d[2] * es};
  const cuuint32_t bx[4] = {(cuuint32_t)box[0], (cuuint32_t)box[1], (cuuint32_t)box[2], (cuuint32_t)box[3]};
  const cuuint32_t el[4] = {1, 1, 1, 1};
  const CUresult r =
      fn(m, sizeof(R) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
         const_cast<R*>(base), d, strides, bx, el, CU_TENSOR_MAP_INTERLEAVE_NONE,
         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

template <typename R, int D>
static bool make_flux_maps(FluxMaps& m, const Params& P, const Work<R>& w) {
  using F = FluxTile<D>;
  bool ok = make_map<R>(&m.wh, w.Wh, 6, P, F::SX, F::SY, F::SZ, F::NG) &&
            make_map<R>(&m.msh, w.Msh, 3, P, F::SX, F::SY, F::SZ, 3) &&
            make_map<R>(&m.ms, w.Ms, 3, P, F::LX, F::LY, F::LZ, 3);
  // face field normal to the faces: box (32, 8, 1), (32, 8, 1) or (32, 1, 8)
  const int bx = 32, by = D == 2 ? 1 : 8, bz = D == 2 ? 8 : 1;
  for (int b = 0; b < 2 && ok; b++) {
    const R* lim = sizeof(R) == 8 ? reinterpret_cast<const R*>(P.Wbuf[b]) : w.Wl;
    const R* fb = sizeof(R) == 8 ? reinterpret_cast<const R*>(P.Bbuf[b]) : w.Bl;
    ok = make_map<R>(&m.wl[b], lim, 6, P, F::LX, F::LY, F::LZ, F::NG) &&
         make_map<R>(&m.bn[b], fb, 3, P, bx, by, bz, 1);
  }
  if (ok) {
    const cuuint64_t tm = (cuuint64_t)P.tmax;
    if (D == 0) {  // the per-axis tables [axis][NTAB][tmax]
      const cuuint64_t d[4] = {tm, (cuuint64_t)NTAB, 3, 1};
      const int box[4] = {32, 18, 1, 1};
      ok = make_map_dims<R>(&m.wt, w.tab, d, box);
    } else {       // the packed face records [axis * tmax + f][FW]
      const cuuint64_t d[4] = {(cuuint64_t)FW, 3 * tm, 1, 1};
      const int box[4] = {FW, 8, 1, 1};
      ok = make_map_dims<R>(&m.wt, w.fw, d, box);
    }
  }
  const int n0 = P.n[0], n1 = P.n[1], n2 = P.n[2];
  if (D == 0) {
    m.nt[0] = (n0 + 1 + 31) / 32;
    m.nt[1] = (n1 + 7) / 8;
    m.nt[2] = n2;
  } else if (D == 1) {
    m.nt[0] = (n0 + 31) / 32;
    m.nt[1] = (n1 + 1 + 7) / 8;
    m.nt[2] = n2;
  } else {
    m.nt[0] = (n0 + 31) / 32;
    m.nt[1] = (n2 + 1 + 7) / 8;
    m.nt[2] = n1;
  }
  return ok;
}

template <typename R, int D, bool BG>
static cudaError_t allow_smem() {
  return cudaFuncSetAttribute(k_flux_sweep<R, D, BG>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              sweep_smem<R, D>());
}

template <typename R>
SweepSet* sweep_create(const Params& P, const Work<R>& w) {
  SweepSet* s = new (std::nothrow) SweepSet();
  if (!s) return nullptr;
  int dev = 0;
  bool ok = cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess;
  ok = ok && make_flux_maps<R, 0>(s->flux[0], P, w) && make_flux_maps<R, 1>(s->flux[1], P, w) &&
       make_flux_maps<R, 2>(s->flux[2], P, w);
  ok = ok && allow_smem<R, 0, false>() == cudaSuccess && allow_smem<R, 1, false>() == cudaSuccess &&
       allow_smem<R, 2, false>() == cudaSuccess && allow_smem<R, 0, true>() == cudaSuccess &&
       allow_smem<R, 1, true>() == cudaSuccess && allow_smem<R, 2, true>() == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    delete s;
    return nullptr;
  }
  return s;
}
template SweepSet* sweep_create<double>(const Params&, const Work<double>&);
template SweepSet* sweep_create<float>(const Params&, const Work<float>&);

void sweep_destroy(SweepSet* s) { delete s; }

template <typename R, int D, bool BG>
static void launch_sweep_d(const SweepSet* sw, const Params& P, const Work<R>& w, cudaStream_t st) {
  const FluxMaps& m = sw->flux[D];
  const int ntiles = m.nt[0] * m.nt[1] * m.nt[2];
  const int grid = std::max(1, std::min(ntiles, sw->sms * SweepCfg<R>::CTAS));
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kSweepThreads);
  cfg.dynamicSmemBytes = sweep_smem<R, D>();
  cfg.stream = st;
  cfg.attrs = at;
  cfg.numAttrs = GOP_SWEEP_PDL ? 1 : 0;
  cudaLaunchKernelEx(&cfg, k_flux_sweep<R, D, BG>, P, w, m);
  count_launches(1);
}

template <typename R>
bool launch_flux_sweep(const SweepSet* sw, const Params& P, const Work<R>& w, int D,
                       cudaStream_t st) {
  if (!sw || P.ps_live) return false;  // the entropy channel runs the per-face kernels
  const bool bg = P.bg != nullptr;
  switch (D) {
    case 0: bg ? launch_sweep_d<R, 0, true>(sw, P, w, st) : launch_sweep_d<R, 0, false>(sw, P, w, st); break;
    case 1: bg ? launch_sweep_d<R, 1, true>(sw, P, w, st) : launch_sweep_d<R, 1, false>(sw, P, w, st); break;
    default: bg ? launch_sweep_d<R, 2, true>(sw, P, w, st) : launch_sweep_d<R, 2, false>(sw, P, w, st); break;
  }
  return true;
}
template bool launch_flux_sweep<double>(const SweepSet*, const Params&, const Work<double>&, int,
                                        cudaStream_t);
template bool launch_flux_sweep<float>(const SweepSet*, const Params&, const Work<float>&, int,
                                       cudaStream_t);

}  // namespace gop

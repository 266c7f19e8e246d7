// Tile-staged sweeps of the MHD step for B200 (sm_100a): the face flux and
// the edge EMF, the step's two stencil stages, computed from shared-memory
// tiles that the Tensor Memory Accelerator streams in ahead of the
// arithmetic.
//
// Face flux along axis D: PDM reconstruction of the 8 face states, Rusanov
// flux and Maxwell stress (src/solver_func.c:215-253,503-685,934-1529).
// Edge EMF along axis D: the second centre-to-edge sweep, the two face-field
// reconstructions and the EMF (src/solver_func.c:686-902).  Their per-point
// forms (k_flux, k_emf in gop_kernels.cu) gather each output's 8-point
// stencils with dozens of global loads through L1; the loads' 64-bit
// address arithmetic and latency, not the FP64 arithmetic, bound them.
// Here each block is persistent and runs a copy pipeline:
//
//   copies   one elected thread streams tiles into a ring of 2-4
//            shared-memory slots (as many as fit the SM at the kernel's
//            residency) with cp.async.bulk.tensor (one TMA box per
//            input array and tile: stencil windows, limiter windows, PDM
//            weights), completing on the slot's "full" mbarrier;
//   compute  8 warps compute one face or edge per thread from shared memory
//            (every stencil tap is a load at a compile-time offset from one
//            per-thread base) and release the slot on its "empty" mbarrier;
//            the feeding thread refills a released slot with the next tile
//            not yet issued, a ring's length ahead.
//
// So the global-memory latency of tile n+1 overlaps the arithmetic of tile
// n, and the stencil re-reads come from shared memory instead of L1.  The
// per-point arithmetic is the per-point kernels' own (recon_lr, flux_out,
// emf_finish), in the same order, so both forms give the same bits.
//
// Lanes always run along i (x, the TMA box's contiguous axis); a tile is 32
// lanes x 8 warps, one warp per row along the stage's sweep axis or its
// third axis.  Every box starts at an x of 32 t or 4 + 32 t, so x times the
// element size is a multiple of 16 bytes (the TMA's alignment rule); no
// coordinate is negative.  Boxes reaching past the grid are filled with
// zeros by the TMA and only feed threads outside the grid, which store
// nothing.  Tiles are numbered with the x tile fastest, then the tile along
// the warps, so the blocks in flight at any time share their halo rows in
// L2.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "gop_stage.cuh"
#include "gop_tma.cuh"

namespace gop {

constexpr int kWarps = 8;
constexpr int kSweepThreads = 32 * kWarps;

// shared-memory ring and residency per arithmetic type: at least two slots;
// two blocks per SM in FP64 (128 registers), three in FP32 (the flux; the
// EMF below)
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
// blocks per SM of the edge-EMF sweeps (smaller slots than the flux
// sweeps); FP32: four (64 registers, no spills) measured 1.06 ms per 256^3
// step on B200 against 1.13 ms with three
#ifndef GOP_SWEEP_EMF_CTAS_F64
#define GOP_SWEEP_EMF_CTAS_F64 GOP_SWEEP_CTAS_F64
#endif
#ifndef GOP_SWEEP_EMF_CTAS_F32
#define GOP_SWEEP_EMF_CTAS_F32 4
#endif
// 1: the sweeps go out with programmatic dependent launch like the other
// step kernels.  Off: a sweep grid placed early onto SMs that still run the
// previous kernel (persistent blocks, no room to spare) measured 2-20 %
// slower on B200 (blast 256^3: FP32 flux 2.47 vs 2.06 ms per step)
#ifndef GOP_SWEEP_PDL
#define GOP_SWEEP_PDL 0
#endif
template <typename R, bool EMF>
struct SweepCfg {
  // the least number of slots; a kernel whose slots are small takes more
  // (ring_slots below)
  static constexpr int STAGES = sizeof(R) == 8 ? GOP_SWEEP_STAGES_F64 : GOP_SWEEP_STAGES_F32;
  static constexpr int CTAS = EMF ? (sizeof(R) == 8 ? GOP_SWEEP_EMF_CTAS_F64 : GOP_SWEEP_EMF_CTAS_F32)
                                  : (sizeof(R) == 8 ? GOP_SWEEP_CTAS_F64 : GOP_SWEEP_CTAS_F32);
};
#ifndef GOP_SWEEP_MAX_STAGES
#define GOP_SWEEP_MAX_STAGES 4
#endif

// a box of the slot: extents (x, y, z, fields) and elements, rounded up to
// 32 so every box starts on a 128-byte boundary in FP32 and FP64
struct Box {
  int x, y, z, f;
  __host__ __device__ constexpr int elems() const { return x * y * z * f; }
  __host__ __device__ constexpr int padded() const { return (elems() + 31) / 32 * 32; }
};
constexpr Box kRec8{FW, 8, 1, 1};    // 8 packed face records
constexpr Box kRec1{FW, 1, 1, 1};    // 1 packed face record
// tap-major weights (T_WL0..T_CR2) of the 32 faces of a warp row, and of
// the face after them (the edge-EMF sweeps on i faces, below)
constexpr Box kTap32{32, 18, 1, 1};
constexpr Box kTap40{40, 18, 1, 1};

// The edge-EMF sweeps whose lanes run along i over the n+1 faces of an i
// row (the EMFs along j and k) tile the row in ceil(n/32) tiles of 32
// faces; when 32 divides n the last face of the row, the upper boundary
// face, is left over.  The last tile of the row then computes it too, in
// one extra pass of one warp whose lanes take the tile's 8 rows (its boxes
// are 40 wide along i, so that face's stencil is in the slot), where a
// ninth tile would cost eight warp passes with one live lane each: 1.6 %
// off the FP64 EMF stage at 256^3 on B200.  The flux sweep along i keeps
// its ninth tile: the same pass made it 1 % slower there (FP32 3.5 %).
__device__ __forceinline__ bool row_end_face(const Params& P, int x0) { return x0 + 32 == NGH + P.n[0]; }
// 1: the FP64 flux sweep along i leaves the row-end faces (32 dividing n)
// to a one-column launch of the per-face arithmetic (k_flux_col) instead
// of a ninth tile per row: FP64 step 7.26 -> 7.20 ms at 256^3 on B200; the
// FP32 step measured 1.5 % slower that way and keeps the ninth tile
#ifndef GOP_FLUX_COL
#define GOP_FLUX_COL 1
#endif
template <typename R>
constexpr bool flux_col() {
  return GOP_FLUX_COL && sizeof(R) == 8;
}
// the warp that takes it: rotates over the row sets (kWarps a power of 2)
template <class T>
__device__ __forceinline__ int row_end_warp(const int nt[3], const T& t) {
  return (t.b + nt[1] * t.c) & (kWarps - 1);
}

// the weights of one face of the tile (tap-major rows of X faces in shared
// memory)
template <int X, typename R>
__device__ __forceinline__ void load_tap(const R* w, FaceWeights<R>& W) {
#pragma unroll
  for (int u = 0; u < 7; u++) {
    W.wl[u] = w[u * X];
    W.wr[u] = w[(7 + u) * X];
  }
  W.cl1 = w[14 * X];
  W.cl2 = w[15 * X];
  W.cr1 = w[16 * X];
  W.cr2 = w[17 * X];
}

// ------------------------------------------------------------------ flux

template <int D>
struct FluxTile {
  static constexpr int NG = 5;  // gas fields (the entropy channel is off)
  // stencil and limiter windows of the tile's faces
  static constexpr Box S = D == 0 ? Box{40, 8, 1, 1} : (D == 1 ? Box{32, 15, 1, 1} : Box{32, 1, 15, 1});
  static constexpr Box L = D == 0 ? Box{40, 8, 1, 1} : (D == 1 ? Box{32, 11, 1, 1} : Box{32, 1, 11, 1});
  static constexpr Box WT = D == 0 ? kTap32 : kRec8;
  static constexpr Box BN = D == 2 ? Box{32, 1, 8, 1} : Box{32, 8, 1, 1};
  static constexpr int SB = S.elems(), LB = L.elems();
  // slot layout in elements: W_h, limiter W, mags_h, mags, weights, B_n
  static constexpr int OFF_WH = 0;
  static constexpr int OFF_WL = OFF_WH + NG * SB;
  static constexpr int OFF_MSH = OFF_WL + NG * LB;
  static constexpr int OFF_MS = OFF_MSH + 3 * SB;
  static constexpr int OFF_W = OFF_MS + 3 * LB;
  static constexpr int OFF_BN = OFF_W + WT.padded();
  static constexpr int ELEMS = OFF_BN + BN.padded();
  // elements the TMA delivers into a slot (the barrier's transaction count)
  static constexpr int TX = NG * SB + NG * LB + 3 * SB + 3 * LB + WT.elems() + BN.elems();
  static_assert((NG * SB) % 32 == 0 && (NG * LB) % 32 == 0 && (3 * SB) % 32 == 0 &&
                    (3 * LB) % 32 == 0,
                "flux boxes on 128-byte boundaries");
};

struct alignas(64) FluxMaps {
  CUtensorMap wh;     // W_h, stencil box
  CUtensorMap wl[2];  // limiter reference: FP64 the state buffer of each parity, FP32 its copy
  CUtensorMap msh;    // mags_h, stencil box
  CUtensorMap ms;     // mags, limiter box
  CUtensorMap wt;     // PDM weights of the tile's faces
  CUtensorMap bn[2];  // step-start face field (as wl: per parity in FP64)
  int nt[3];          // tiles: x, along the warps, third axis
};

// tile t of the flux sweep along D: its first cell / face on each axis
struct TileAt {
  int x0, y0, z0;
};
// A tile index t = a + nt[0] * (b + nt[1] * c) as its three digits.  The
// blocks walk the tiles in steps of the grid size, and adding the step's
// digits with carries replaces the divisions by nt of every tile (about a
// hundred integer instructions per thread and tile).
struct Tile {
  int a, b, c;
};
__device__ __forceinline__ Tile tile_of(const int nt[3], int t) {
  const int r = t / nt[0];
  return {t % nt[0], r % nt[1], r / nt[1]};
}
// p += s (s's digits below nt: one carry per digit at most)
__device__ __forceinline__ void tile_add(Tile& p, const Tile& s, const int nt[3]) {
  p.a += s.a;
  int carry = p.a >= nt[0];
  if (carry) p.a -= nt[0];
  p.b += s.b + carry;
  carry = p.b >= nt[1];
  if (carry) p.b -= nt[1];
  p.c += s.c + carry;
}
template <int D>
__device__ __forceinline__ TileAt flux_at(const Tile& p) {
  const int a = p.a, b = p.b, c = p.c;
  TileAt T;
  T.x0 = NGH + 32 * a;
  if constexpr (D == 2) {  // warps: faces along k, one row j
    T.y0 = NGH + c;
    T.z0 = NGH + 8 * b;
  } else {  // warps: rows along j (D = 0) or faces along j (D = 1), one plane k
    T.y0 = NGH + 8 * b;
    T.z0 = NGH + c;
  }
  return T;
}

template <typename R, int D, bool BG>
struct FluxStage {
  static constexpr bool EMF = false;
  using F = FluxTile<D>;
  using Maps = FluxMaps;
  static constexpr int ELEMS = F::ELEMS;
  static constexpr int TX = F::TX;

  __device__ static void issue(const Params& P, const Maps& m, int par, const Tile& t, R* s,
                               uint64_t* bar) {
    const TileAt T = flux_at<D>(t);
    const int f0 = D == 0 ? T.x0 : (D == 1 ? T.y0 : T.z0);  // first face along D
    // stencil windows start 4 cells before the first face, limiter windows
    // 2 (along i both start 4 before, keeping x aligned)
    const int sx = D == 0 ? T.x0 - 4 : T.x0, sy = D == 1 ? T.y0 - 4 : T.y0, sz = D == 2 ? T.z0 - 4 : T.z0;
    const int ly = D == 1 ? T.y0 - 2 : T.y0, lz = D == 2 ? T.z0 - 2 : T.z0;
    tma_load_4d(s + F::OFF_WH, &m.wh, bar, sx, sy, sz, 0);
    tma_load_4d(s + F::OFF_WL, &m.wl[par], bar, sx, ly, lz, 0);
    tma_load_4d(s + F::OFF_MSH, &m.msh, bar, sx, sy, sz, 0);
    tma_load_4d(s + F::OFF_MS, &m.ms, bar, sx, ly, lz, 0);
    if constexpr (D == 0) tma_load_4d(s + F::OFF_W, &m.wt, bar, f0, T_WL0, 0, 0);
    else tma_load_4d(s + F::OFF_W, &m.wt, bar, 0, D * P.tmax + f0, 0, 0);
    tma_load_4d(s + F::OFF_BN, &m.bn[par], bar, T.x0, T.y0, T.z0, D);
  }

  // one face per thread
  __device__ static void compute(const Params& P, const Work<R>& wk, const Maps& m, const R* s,
                                 const Tile& t, int warp, int lane) {
    const TileAt T = flux_at<D>(t);
    const int row = warp, col = lane;
    const int i = T.x0 + col, j = T.y0 + (D == 2 ? 0 : row), k = T.z0 + (D == 2 ? row : 0);
    if (!(i < NGH + P.n[0] + (D == 0) && j < NGH + P.n[1] + (D == 1) && k < NGH + P.n[2] + (D == 2)))
      return;
    // per-thread bases: tap u of field f is then at a compile-time offset
    const R *wh, *wl, *msh, *ms;
    if constexpr (D == 0) {
      const int b = row * 40 + col;
      wh = s + F::OFF_WH + b;
      wl = s + F::OFF_WL + b + 2;  // the limiter cells f-2..f+1 start 2 cells in
      msh = s + F::OFF_MSH + b;
      ms = s + F::OFF_MS + b + 2;
    } else {
      const int b = row * 32 + col;
      wh = s + F::OFF_WH + b;
      wl = s + F::OFF_WL + b;
      msh = s + F::OFF_MSH + b;
      ms = s + F::OFF_MS + b;
    }
    constexpr int TS = D == 0 ? 1 : 32;  // stride of one stencil tap in the slot
    FaceWeights<R> Wt;
    if constexpr (D == 0) load_tap<32>(s + F::OFF_W + col, Wt);
    else load_fw_smem(s + F::OFF_W + row * FW, Wt);
    const R bn = s[F::OFF_BN + row * F::BN.x + col];
    const R a1h = (R)(0.5 * P.pdm_a1), a2 = (R)P.pdm_a2;
    R L[6], Rt[6], mL[3], mR[3];
    L[PS] = Rt[PS] = R(0);
#pragma unroll
    for (int f = 0; f < F::NG; f++) {
      R v[8], lim[4];
#pragma unroll
      for (int u = 0; u < 8; u++) v[u] = wh[f * F::SB + u * TS];
#pragma unroll
      for (int u = 0; u < 4; u++) lim[u] = wl[f * F::LB + u * TS];
      recon_lr<R>(v, lim, Wt, a1h, a2, L[f], Rt[f]);
    }
#pragma unroll
    for (int a = 0; a < 3; a++) {
      R v[8], lim[4];
#pragma unroll
      for (int u = 0; u < 8; u++) v[u] = msh[a * F::SB + u * TS];
#pragma unroll
      for (int u = 0; u < 4; u++) lim[u] = ms[a * F::LB + u * TS];
      recon_lr<R>(v, lim, Wt, a1h, a2, mL[a], mR[a]);
    }
    flux_out<R, D, BG, false>(P, wk, lin(P, i, j, k), L, Rt, mL, mR, bn);
  }
};

// ------------------------------------------------------------------- EMF

// Edge EMF along D, p = D+1, q = D+2 (mod 3).  Inputs per edge: the two
// first-sweep velocities along q (V, 8 cells; limited against themselves),
// B_p along q (8 half-step, 4 step-start values), B_q along p (8 + 4), the
// four half-step densities around the edge, the weights of its q and p faces.
//   D = 0 (p = j, q = k): lanes cells along i, warps k faces, one j face
//   D = 1 (p = k, q = i): lanes i faces, warps k faces, one j cell
//   D = 2 (p = i, q = j): lanes i faces, warps j faces, one k cell
template <int D>
struct EmfTile {
  static constexpr Box V = D == 0 ? Box{32, 1, 15, 2} : (D == 1 ? Box{40, 1, 8, 2} : Box{40, 15, 1, 2});
  static constexpr Box BHP = D == 0 ? Box{32, 1, 15, 1} : (D == 1 ? Box{40, 1, 8, 1} : Box{40, 15, 1, 1});
  static constexpr Box BLP = D == 0 ? Box{32, 1, 11, 1} : (D == 1 ? Box{40, 1, 8, 1} : Box{40, 11, 1, 1});
  static constexpr Box BHQ = D == 0 ? Box{32, 8, 8, 1} : (D == 1 ? Box{40, 1, 15, 1} : Box{40, 8, 1, 1});
  static constexpr Box BLQ = D == 0 ? Box{32, 4, 8, 1} : (D == 1 ? Box{40, 1, 11, 1} : Box{40, 8, 1, 1});
  static constexpr Box RHO = D == 0 ? Box{32, 2, 9, 1} : (D == 1 ? Box{40, 1, 9, 1} : Box{40, 9, 1, 1});
  static constexpr Box WQ = D == 1 ? kTap40 : kRec8;
  static constexpr Box WP = D == 0 ? kRec1 : (D == 1 ? kRec8 : kTap40);
  static constexpr int VF = V.x * V.y * V.z;  // elements of one V field
  static constexpr int OFF_V = 0;
  static constexpr int OFF_BHP = OFF_V + V.padded();
  static constexpr int OFF_BLP = OFF_BHP + BHP.padded();
  static constexpr int OFF_BHQ = OFF_BLP + BLP.padded();
  static constexpr int OFF_BLQ = OFF_BHQ + BHQ.padded();
  static constexpr int OFF_RHO = OFF_BLQ + BLQ.padded();
  static constexpr int OFF_WQ = OFF_RHO + RHO.padded();
  static constexpr int OFF_WP = OFF_WQ + WQ.padded();
  static constexpr int ELEMS = OFF_WP + WP.padded();
  // elements the TMA delivers into a slot (the barrier's transaction count)
  static constexpr int TX = V.elems() + BHP.elems() + BLP.elems() + BHQ.elems() + BLQ.elems() +
                            RHO.elems() + WQ.elems() + WP.elems();
};

struct alignas(64) EmfMaps {
  CUtensorMap v;       // first-sweep velocities V (2 of its 6 fields)
  CUtensorMap bhp;     // B_h, component p, window along q
  CUtensorMap blp[2];  // step-start B (per parity in FP64), component p
  CUtensorMap bhq;     // B_h, component q, window along p
  CUtensorMap blq[2];  // step-start B, component q
  CUtensorMap rho;     // W_h density around the edges
  CUtensorMap wq;      // weights of the q faces
  CUtensorMap wp;      // weights of the p faces
  int nt[3];
};

template <int D>
__device__ __forceinline__ TileAt emf_at(const Tile& p) {
  const int a = p.a, b = p.b, c = p.c;
  TileAt T;
  T.x0 = NGH + 32 * a;
  if constexpr (D == 2) {  // warps: faces along j, one plane k
    T.y0 = NGH + 8 * b;
    T.z0 = NGH + c;
  } else {  // warps: faces along k, one row j
    T.y0 = NGH + c;
    T.z0 = NGH + 8 * b;
  }
  return T;
}

template <typename R, int D, bool BG>
struct EmfStage {
  static constexpr bool EMF = true;
  using E = EmfTile<D>;
  using Maps = EmfMaps;
  static constexpr int ELEMS = E::ELEMS;
  static constexpr int TX = E::TX;
  static constexpr int p = (D + 1) % 3, q = (D + 2) % 3;

  __device__ static void issue(const Params& P, const Maps& m, int par, const Tile& t, R* s,
                               uint64_t* bar) {
    const TileAt T = emf_at<D>(t);
    const int x0 = T.x0, y0 = T.y0, z0 = T.z0;
    if constexpr (D == 0) {  // i cells, j face y0, k faces z0..
      tma_load_4d(s + E::OFF_V, &m.v, bar, x0, y0, z0 - 4, 0);
      tma_load_4d(s + E::OFF_BHP, &m.bhp, bar, x0, y0, z0 - 4, 1);
      tma_load_4d(s + E::OFF_BLP, &m.blp[par], bar, x0, y0, z0 - 2, 1);
      tma_load_4d(s + E::OFF_BHQ, &m.bhq, bar, x0, y0 - 4, z0, 2);
      tma_load_4d(s + E::OFF_BLQ, &m.blq[par], bar, x0, y0 - 2, z0, 2);
      tma_load_4d(s + E::OFF_RHO, &m.rho, bar, x0, y0 - 1, z0 - 1, 0);
      tma_load_4d(s + E::OFF_WQ, &m.wq, bar, 0, 2 * P.tmax + z0, 0, 0);
      tma_load_4d(s + E::OFF_WP, &m.wp, bar, 0, P.tmax + y0, 0, 0);
    } else if constexpr (D == 1) {  // i faces, j cell y0, k faces z0..
      tma_load_4d(s + E::OFF_V, &m.v, bar, x0 - 4, y0, z0, 2);
      tma_load_4d(s + E::OFF_BHP, &m.bhp, bar, x0 - 4, y0, z0, 2);
      tma_load_4d(s + E::OFF_BLP, &m.blp[par], bar, x0 - 4, y0, z0, 2);
      tma_load_4d(s + E::OFF_BHQ, &m.bhq, bar, x0, y0, z0 - 4, 0);
      tma_load_4d(s + E::OFF_BLQ, &m.blq[par], bar, x0, y0, z0 - 2, 0);
      tma_load_4d(s + E::OFF_RHO, &m.rho, bar, x0 - 4, y0, z0 - 1, 0);
      tma_load_4d(s + E::OFF_WQ, &m.wq, bar, x0, T_WL0, 0, 0);
      tma_load_4d(s + E::OFF_WP, &m.wp, bar, 0, 2 * P.tmax + z0, 0, 0);
    } else {  // i faces, j faces y0.., k cell z0
      tma_load_4d(s + E::OFF_V, &m.v, bar, x0, y0 - 4, z0, 4);
      tma_load_4d(s + E::OFF_BHP, &m.bhp, bar, x0, y0 - 4, z0, 0);
      tma_load_4d(s + E::OFF_BLP, &m.blp[par], bar, x0, y0 - 2, z0, 0);
      tma_load_4d(s + E::OFF_BHQ, &m.bhq, bar, x0 - 4, y0, z0, 1);
      tma_load_4d(s + E::OFF_BLQ, &m.blq[par], bar, x0 - 4, y0, z0, 1);
      tma_load_4d(s + E::OFF_RHO, &m.rho, bar, x0 - 4, y0 - 1, z0, 0);
      tma_load_4d(s + E::OFF_WQ, &m.wq, bar, 0, P.tmax + y0, 0, 0);
      tma_load_4d(s + E::OFF_WP, &m.wp, bar, x0, T_WL0, 0, 0);
    }
  }

  // one edge per thread; the edges along j and k (lanes on i faces) take
  // the row's upper boundary face in the last tile of a row when 32
  // divides n (row_end_face)
  __device__ static void compute(const Params& P, const Work<R>& wk, const Maps& m, const R* s,
                                 const Tile& t, int warp, int lane) {
    const TileAt T = emf_at<D>(t);
    edge(P, wk, s, T, warp, lane);
    if constexpr (D != 0)
      if (row_end_face(P, T.x0) && warp == row_end_warp(m.nt, t) && lane < kWarps)
        row_end(P, wk, s, T, lane);
  }
  __device__ __forceinline__ static void row_end(const Params& P, const Work<R>& wk, const R* s,
                                                const TileAt T, int row) {
    edge(P, wk, s, T, row, 32);
  }

  // the edge in tile row `row` (a warp's row), column `col` (a lane's edge)
  __device__ static void edge(const Params& P, const Work<R>& wk, const R* s, const TileAt& T,
                              int row, int col) {
    const int warp = row, lane = col;
    const int i = T.x0 + lane, j = T.y0 + (D == 2 ? warp : 0), k = T.z0 + (D == 2 ? 0 : warp);
    if (!(i < NGH + P.n[0] + (D != 0) && j < NGH + P.n[1] + (D != 1) && k < NGH + P.n[2] + (D != 2)))
      return;
    const R a1h = (R)(0.5 * P.pdm_a1), a2 = (R)P.pdm_a2;
    // stencil bases and tap strides of the windows along q and along p (the
    // boxes whose rows run along i on i faces are 40 wide)
    const R *v0, *bp, *bpl, *bq, *bql;
    constexpr int tq = D == 1 ? 1 : (D == 2 ? 40 : 32);  // slot stride of one tap along q
    constexpr int tp = D == 2 ? 1 : (D == 1 ? 40 : 32);  // ... along p
    R rho4;
    const R* rh = s + E::OFF_RHO;
    FaceWeights<R> Wq, Wp;
    if constexpr (D == 0) {  // q = k rows of 32; p = j rows of 32 in the warp's k face
      v0 = s + E::OFF_V + warp * 32 + lane;
      bp = s + E::OFF_BHP + warp * 32 + lane;
      bpl = s + E::OFF_BLP + warp * 32 + lane;
      bq = s + E::OFF_BHQ + warp * 8 * 32 + lane;
      bql = s + E::OFF_BLQ + warp * 4 * 32 + lane;
      // (j-1,k-1) + (j-1,k) + (j,k-1) + (j,k); box rows [k][j]
      const R* r = rh + lane;
      rho4 = r[(warp * 2 + 0) * 32] + r[((warp + 1) * 2 + 0) * 32] + r[(warp * 2 + 1) * 32] +
             r[((warp + 1) * 2 + 1) * 32];
      load_fw_smem(s + E::OFF_WQ + warp * FW, Wq);
      load_fw_smem(s + E::OFF_WP, Wp);
    } else if constexpr (D == 1) {  // q = i in a row of 40; p = k rows of 40
      v0 = s + E::OFF_V + warp * 40 + lane;
      bp = s + E::OFF_BHP + warp * 40 + lane;
      bpl = s + E::OFF_BLP + warp * 40 + lane + 2;
      bq = s + E::OFF_BHQ + warp * 40 + lane;
      bql = s + E::OFF_BLQ + warp * 40 + lane;
      // (i-1,k-1) + (i-1,k) + (i,k-1) + (i,k); box rows of 40 along k
      const R* r = rh + lane + 3;
      rho4 = r[warp * 40] + r[(warp + 1) * 40] + r[warp * 40 + 1] + r[(warp + 1) * 40 + 1];
      load_tap<40>(s + E::OFF_WQ + lane, Wq);
      load_fw_smem(s + E::OFF_WP + warp * FW, Wp);
    } else {  // q = j rows of 40; p = i in a row of 40
      v0 = s + E::OFF_V + warp * 40 + lane;
      bp = s + E::OFF_BHP + warp * 40 + lane;
      bpl = s + E::OFF_BLP + warp * 40 + lane;
      bq = s + E::OFF_BHQ + warp * 40 + lane;
      bql = s + E::OFF_BLQ + warp * 40 + lane + 2;
      // (i-1,j-1) + (i-1,j) + (i,j-1) + (i,j); box rows of 40 along j
      const R* r = rh + lane + 3;
      rho4 = r[warp * 40] + r[(warp + 1) * 40] + r[warp * 40 + 1] + r[(warp + 1) * 40 + 1];
      load_fw_smem(s + E::OFF_WQ + warp * FW, Wq);
      load_tap<40>(s + E::OFF_WP + lane, Wp);
    }
    R vav[2], bpL, bpR, bqL, bqR;
#pragma unroll
    for (int cc = 0; cc < 2; cc++) {  // second sweep along q, limited against itself
      R v[8], lim[4], L, Rr;
#pragma unroll
      for (int u = 0; u < 8; u++) v[u] = v0[cc * E::VF + u * tq];
#pragma unroll
      for (int u = 0; u < 4; u++) lim[u] = v[u + 2];
      recon_lr<R>(v, lim, Wq, a1h, a2, L, Rr);
      vav[cc] = R(0.5) * (L + Rr);
    }
    {  // B_p along q
      R v[8], lim[4];
#pragma unroll
      for (int u = 0; u < 8; u++) v[u] = bp[u * tq];
#pragma unroll
      for (int u = 0; u < 4; u++) lim[u] = bpl[u * tq];
      recon_lr<R>(v, lim, Wq, a1h, a2, bpL, bpR);
    }
    {  // B_q along p
      R v[8], lim[4];
#pragma unroll
      for (int u = 0; u < 8; u++) v[u] = bq[u * tp];
#pragma unroll
      for (int u = 0; u < 4; u++) lim[u] = bql[u * tp];
      recon_lr<R>(v, lim, Wp, a1h, a2, bqL, bqR);
    }
    const long long x = lin(P, i, j, k);
    const size_t fs = P.fs;
    R b0p = R(0), b0q = R(0);
    if constexpr (BG) {  // B0 averaged along the edge (B0Aedge*)
      b0p = (R)P.bg[(size_t)(BG_EDGE + 3 * D + p) * fs + x];
      b0q = (R)P.bg[(size_t)(BG_EDGE + 3 * D + q) * fs + x];
    }
    wk.E[x + (size_t)D * fs] =
        emf_finish<R, BG>(P, vav[0], vav[1], bpL, bpR, bqL, bqR, b0p, b0q, rho4);
  }
};

// ------------------------------------------------------------- pipeline

template <class Stage, typename R>
__host__ __device__ constexpr int slot_bytes() {
  return Stage::ELEMS * (int)sizeof(R);
}
// Slots in a block's ring: as many as fit the SM's 228 KB of shared memory
// at SweepCfg::CTAS blocks per SM (each block also reserves 1 KB), at least
// SweepCfg::STAGES, at most GOP_SWEEP_MAX_STAGES.  The small slots of the
// edge-EMF sweeps get 3-4: their tiles compute for less time than the
// copies of the next take to land.
template <class Stage, typename R>
__host__ __device__ constexpr int ring_slots() {
  using Cfg = SweepCfg<R, Stage::EMF>;
  constexpr int per_block = 228 * 1024 / Cfg::CTAS - 1024 - 128 - 64;
  constexpr int fit = per_block / slot_bytes<Stage, R>();
  return fit < Cfg::STAGES ? Cfg::STAGES
                                   : (fit > GOP_SWEEP_MAX_STAGES ? GOP_SWEEP_MAX_STAGES : fit);
}
template <class Stage, typename R>
__host__ __device__ constexpr int sweep_smem() {
  return ring_slots<Stage, R>() * slot_bytes<Stage, R>() + 2 * ring_slots<Stage, R>() * 8 + 128;
}

// Persistent sweep: lane 0 of warp 0 also feeds the ring.  It fills the
// first S slots, and after each tile waits until all 8 warps have released
// that tile's slot, then issues the tile S ahead into it; the
// other warps meanwhile compute the next tile, whose copies were issued a
// tile earlier.  Every wait is bounded; a block that gives up records the
// failure in S_FLAGS (2) and drains its copies in flight before it exits.
template <class Stage, typename R>
__device__ __forceinline__ void sweep_run(const Params& P, const Work<R>& wk,
                                          const typename Stage::Maps& maps) {
  // stop flag, or an earlier pipeline wait that timed out: do nothing
  if (stopped(P) || P.scal[S_FLAGS] == 2.0) return;
  constexpr int S = ring_slots<Stage, R>();
  constexpr int SLOT = slot_bytes<Stage, R>();
  constexpr int TXB = Stage::TX * (int)sizeof(R);  // bytes the copies of one tile deliver
  static_assert(TXB <= SLOT, "slot holds its boxes");
  extern __shared__ unsigned char smem_dyn[];
  // TMA destinations on 128-byte boundaries (the launch adds 128 bytes)
  unsigned char* base = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_dyn) + 127) & ~static_cast<uintptr_t>(127));
  R* slots = reinterpret_cast<R*>(base);
  uint64_t* full = reinterpret_cast<uint64_t*>(base + S * SLOT);
  uint64_t* empty = full + S;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool feeder = threadIdx.x == 0;
  const int nt2 = maps.nt[2];  // tiles run out when the third digit reaches it
  const int par = sizeof(R) == 8 ? cur_buf(P) : 0;
  auto issue = [&](int n, const Tile& t) {
    const int q = n % S;
    mbar_arrive_expect_tx(&full[q], TXB);
    Stage::issue(P, maps, par, t, slots + (size_t)q * Stage::ELEMS, &full[q]);
  };
  const Tile step = tile_of(maps.nt, gridDim.x);
  Tile next = tile_of(maps.nt, blockIdx.x);  // feeder only: the first tile not yet issued
  int issued = 0;                            // feeder only: tiles whose copies were issued
  if (feeder) {
    for (int q = 0; q < S; q++) {
      mbar_init(&full[q], 1);
      mbar_init(&empty[q], kWarps);
    }
    fence_mbar_init();
    for (; next.c < nt2 && issued < S; tile_add(next, step, maps.nt)) issue(issued++, next);
  }
  __syncthreads();
  bool ok = true;
  int n = 0;
  for (Tile t = tile_of(maps.nt, blockIdx.x); t.c < nt2; tile_add(t, step, maps.nt), n++) {
    const int q = n % S;
    const uint32_t ph = (n / S) & 1;
    if (!mbar_wait(&full[q], ph)) {
      ok = false;
      break;
    }
    Stage::compute(P, wk, maps, slots + (size_t)q * Stage::ELEMS, t, warp, lane);
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[q]);
    if (feeder && next.c < nt2) {
      // every warp has released this slot: refill it with the tile S ahead
      if (!mbar_wait(&empty[q], ph)) {
        ok = false;
        break;
      }
      issue(issued++, next);
      tile_add(next, step, maps.nt);
    }
  }
  if (feeder) {
    // the copies of the tiles issued last must land before the block exits
    for (int k = issued > S ? issued - S : 0; k < issued; k++)
      if (!mbar_wait(&full[k % S], (k / S) & 1)) ok = false;
  }
  if (!ok) P.scal[S_FLAGS] = 2.0;
}

template <typename R, int D, bool BG>
__global__ void __launch_bounds__(kSweepThreads, (SweepCfg<R, false>::CTAS))
    k_flux_sweep(Params P, Work<R> wk, const __grid_constant__ FluxMaps maps) {
  pdl_enter();
  sweep_run<FluxStage<R, D, BG>, R>(P, wk, maps);
}

template <typename R, int D, bool BG>
__global__ void __launch_bounds__(kSweepThreads, (SweepCfg<R, true>::CTAS))
    k_emf_sweep(Params P, Work<R> wk, const __grid_constant__ EmfMaps maps) {
  pdl_enter();
  sweep_run<EmfStage<R, D, BG>, R>(P, wk, maps);
}

template <typename R, int D>
constexpr bool smem_fits() {
  return (size_t)sweep_smem<FluxStage<R, D, false>, R>() * SweepCfg<R, false>::CTAS <= 228 * 1024 &&
         (size_t)sweep_smem<EmfStage<R, D, false>, R>() * SweepCfg<R, true>::CTAS <= 228 * 1024;
}
static_assert(smem_fits<double, 0>() && smem_fits<double, 1>() && smem_fits<double, 2>(),
              "FP64 sweep blocks per SM");
static_assert(smem_fits<float, 0>() && smem_fits<float, 1>() && smem_fits<float, 2>(),
              "FP32 sweep blocks per SM");

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

// a 4-D map over a dense array of dims d[0..3] (elements, d[0] fastest;
// strides in bytes), read in boxes b
template <typename R>
static bool encode(CUtensorMap* m, const R* base, const cuuint64_t d[4], const cuuint64_t st[3],
                   const Box& b) {
  EncodeTiledFn fn = encode_fn();
  if (!fn || !base) return false;
  const cuuint32_t bx[4] = {(cuuint32_t)b.x, (cuuint32_t)b.y, (cuuint32_t)b.z, (cuuint32_t)b.f};
  const cuuint32_t el[4] = {1, 1, 1, 1};
  const CUresult r =
      fn(m, sizeof(R) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
         const_cast<R*>(base), d, st, bx, el, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// nf fields of one array in the state's layout (i, j, k, field)
template <typename R>
static bool field_map(CUtensorMap* m, const R* base, int nf, const Params& P, const Box& b) {
  const cuuint64_t es = sizeof(R);
  const cuuint64_t d[4] = {(cuuint64_t)P.N[0], (cuuint64_t)P.N[1], (cuuint64_t)P.N[2], (cuuint64_t)nf};
  const cuuint64_t st[3] = {(cuuint64_t)P.pitch * es, (cuuint64_t)P.sk * es, (cuuint64_t)P.fs * es};
  return encode<R>(m, base, d, st, b);
}

// PDM weights: the per-axis tables [axis][NTAB][tmax] for tap-major boxes,
// the packed face records [axis * tmax + f][FW] otherwise
template <typename R>
static bool weight_map(CUtensorMap* m, const Work<R>& w, const Params& P, const Box& b) {
  const cuuint64_t es = sizeof(R), tm = (cuuint64_t)P.tmax;
  if (b.y == kTap32.y && (b.x == kTap32.x || b.x == kTap40.x)) {
    const cuuint64_t d[4] = {tm, (cuuint64_t)NTAB, 3, 1};
    const cuuint64_t st[3] = {tm * es, tm * NTAB * es, tm * NTAB * 3 * es};
    return encode<R>(m, w.tab, d, st, b);
  }
  const cuuint64_t d[4] = {(cuuint64_t)FW, 3 * tm, 1, 1};
  const cuuint64_t st[3] = {FW * es, FW * 3 * tm * es, FW * 3 * tm * es};
  return encode<R>(m, w.fw, d, st, b);
}

// the limiters' step-start references: FP64 the state buffer of parity b,
// FP32 its copy (the same for both parities)
template <typename R>
static const R* lim_state(const Params& P, const Work<R>& w, int b) {
  return sizeof(R) == 8 ? reinterpret_cast<const R*>(P.Wbuf[b]) : w.Wl;
}
template <typename R>
static const R* lim_face(const Params& P, const Work<R>& w, int b) {
  return sizeof(R) == 8 ? reinterpret_cast<const R*>(P.Bbuf[b]) : w.Bl;
}

template <typename R, int D>
static bool make_flux_maps(FluxMaps& m, const Params& P, const Work<R>& w) {
  using F = FluxTile<D>;
  const Box S5{F::S.x, F::S.y, F::S.z, F::NG}, L5{F::L.x, F::L.y, F::L.z, F::NG};
  const Box S3{F::S.x, F::S.y, F::S.z, 3}, L3{F::L.x, F::L.y, F::L.z, 3};
  bool ok = field_map<R>(&m.wh, w.Wh, 6, P, S5) && field_map<R>(&m.msh, w.Msh, 3, P, S3) &&
            field_map<R>(&m.ms, w.Ms, 3, P, L3) && weight_map<R>(&m.wt, w, P, F::WT);
  for (int b = 0; b < 2 && ok; b++)
    ok = field_map<R>(&m.wl[b], lim_state<R>(P, w, b), 6, P, L5) &&
         field_map<R>(&m.bn[b], lim_face<R>(P, w, b), 3, P, F::BN);
  const int n0 = P.n[0], n1 = P.n[1], n2 = P.n[2];
  if (D == 0) {  // i-face tiles (the row-end faces by k_flux_col), j-row tiles, k planes
    m.nt[0] = flux_col<R>() ? (n0 + 31) / 32 : (n0 + 1 + 31) / 32;
    m.nt[1] = (n1 + 7) / 8;
    m.nt[2] = n2;
  } else if (D == 1) {  // i tiles, j-face tiles, k planes
    m.nt[0] = (n0 + 31) / 32;
    m.nt[1] = (n1 + 1 + 7) / 8;
    m.nt[2] = n2;
  } else {  // i tiles, k-face tiles, j rows
    m.nt[0] = (n0 + 31) / 32;
    m.nt[1] = (n2 + 1 + 7) / 8;
    m.nt[2] = n1;
  }
  return ok;
}

template <typename R, int D>
static bool make_emf_maps(EmfMaps& m, const Params& P, const Work<R>& w) {
  using E = EmfTile<D>;
  bool ok = field_map<R>(&m.v, w.V, 6, P, E::V) && field_map<R>(&m.bhp, w.Bh, 3, P, E::BHP) &&
            field_map<R>(&m.bhq, w.Bh, 3, P, E::BHQ) && field_map<R>(&m.rho, w.Wh, 6, P, E::RHO) &&
            weight_map<R>(&m.wq, w, P, E::WQ) && weight_map<R>(&m.wp, w, P, E::WP);
  for (int b = 0; b < 2 && ok; b++)
    ok = field_map<R>(&m.blp[b], lim_face<R>(P, w, b), 3, P, E::BLP) &&
         field_map<R>(&m.blq[b], lim_face<R>(P, w, b), 3, P, E::BLQ);
  const int n0 = P.n[0], n1 = P.n[1], n2 = P.n[2];
  if (D == 0) {  // i-cell tiles, k-face tiles, j faces
    m.nt[0] = (n0 + 31) / 32;
    m.nt[1] = (n2 + 1 + 7) / 8;
    m.nt[2] = n1 + 1;
  } else if (D == 1) {  // i-face tiles (the row-end face in the last), k-face tiles, j cells
    m.nt[0] = (n0 + 31) / 32;
    m.nt[1] = (n2 + 1 + 7) / 8;
    m.nt[2] = n1;
  } else {  // i-face tiles (the row-end face in the last), j-face tiles, k cells
    m.nt[0] = (n0 + 31) / 32;
    m.nt[1] = (n1 + 1 + 7) / 8;
    m.nt[2] = n2;
  }
  return ok;
}

struct SweepSet {
  FluxMaps flux[3];
  EmfMaps emf[3];
  int sms = 0;
};

template <typename R, int D, bool BG>
static cudaError_t allow_smem() {
  cudaError_t e = cudaFuncSetAttribute(k_flux_sweep<R, D, BG>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       sweep_smem<FluxStage<R, D, BG>, R>());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_emf_sweep<R, D, BG>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             sweep_smem<EmfStage<R, D, BG>, R>());
  return e;
}

template <typename R>
SweepSet* sweep_create(const Params& P, const Work<R>& w) {
  SweepSet* s = new (std::nothrow) SweepSet();
  if (!s) return nullptr;
  int dev = 0;
  bool ok = cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess;
  ok = ok && make_flux_maps<R, 0>(s->flux[0], P, w) && make_flux_maps<R, 1>(s->flux[1], P, w) &&
       make_flux_maps<R, 2>(s->flux[2], P, w) && make_emf_maps<R, 0>(s->emf[0], P, w) &&
       make_emf_maps<R, 1>(s->emf[1], P, w) && make_emf_maps<R, 2>(s->emf[2], P, w);
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

template <class Stage, typename R, class Maps, class K>
static void launch_persistent(K kern, const SweepSet* sw, const Params& P, const Work<R>& w,
                              const Maps& m, cudaStream_t st) {
  const int ntiles = m.nt[0] * m.nt[1] * m.nt[2];
  const int grid = std::max(1, std::min(ntiles, sw->sms * SweepCfg<R, Stage::EMF>::CTAS));
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kSweepThreads);
  cfg.dynamicSmemBytes = sweep_smem<Stage, R>();
  cfg.stream = st;
  cfg.attrs = at;
  cfg.numAttrs = GOP_SWEEP_PDL ? 1 : 0;
  cudaLaunchKernelEx(&cfg, kern, P, w, m);
  count_launches(1);
}

template <typename R, int D, bool BG>
static void launch_flux_d(const SweepSet* sw, const Params& P, const Work<R>& w, cudaStream_t st) {
  launch_persistent<FluxStage<R, D, BG>, R>(k_flux_sweep<R, D, BG>, sw, P, w, sw->flux[D], st);
}
template <typename R, int D, bool BG>
static void launch_emf_d(const SweepSet* sw, const Params& P, const Work<R>& w, cudaStream_t st) {
  launch_persistent<EmfStage<R, D, BG>, R>(k_emf_sweep<R, D, BG>, sw, P, w, sw->emf[D], st);
}

template <typename R>
bool launch_flux_sweep(const SweepSet* sw, const Params& P, const Work<R>& w, int D,
                       cudaStream_t st) {
  if (!sw || P.ps_live) return false;  // the entropy channel runs the per-face kernels
  const bool bg = P.bg != nullptr;
  switch (D) {
    case 0:
      bg ? launch_flux_d<R, 0, true>(sw, P, w, st) : launch_flux_d<R, 0, false>(sw, P, w, st);
      if (flux_col<R>() && P.n[0] % 32 == 0) launch_flux_col<R>(P, w, st);
      break;
    case 1: bg ? launch_flux_d<R, 1, true>(sw, P, w, st) : launch_flux_d<R, 1, false>(sw, P, w, st); break;
    default: bg ? launch_flux_d<R, 2, true>(sw, P, w, st) : launch_flux_d<R, 2, false>(sw, P, w, st); break;
  }
  return true;
}
template bool launch_flux_sweep<double>(const SweepSet*, const Params&, const Work<double>&, int,
                                        cudaStream_t);
template bool launch_flux_sweep<float>(const SweepSet*, const Params&, const Work<float>&, int,
                                       cudaStream_t);

template <typename R>
bool launch_emf_sweep(const SweepSet* sw, const Params& P, const Work<R>& w, int D, cudaStream_t st) {
  if (!sw) return false;
  const bool bg = P.bg != nullptr;
  switch (D) {
    case 0: bg ? launch_emf_d<R, 0, true>(sw, P, w, st) : launch_emf_d<R, 0, false>(sw, P, w, st); break;
    case 1: bg ? launch_emf_d<R, 1, true>(sw, P, w, st) : launch_emf_d<R, 1, false>(sw, P, w, st); break;
    default: bg ? launch_emf_d<R, 2, true>(sw, P, w, st) : launch_emf_d<R, 2, false>(sw, P, w, st); break;
  }
  return true;
}
template bool launch_emf_sweep<double>(const SweepSet*, const Params&, const Work<double>&, int,
                                       cudaStream_t);
template bool launch_emf_sweep<float>(const SweepSet*, const Params&, const Work<float>&, int,
                                      cudaStream_t);

}  // namespace gop

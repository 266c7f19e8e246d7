// Host-side launchers of the step kernels (implemented in gop_kernels.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "gamera_op.h"
#include "gop_device.cuh"

namespace gop {

// per-step work arrays, each field fs elements, element type R
template <typename R>
struct Work {
  R* Wh;   // 6 half-step primitives
  R* Ms;   // 3 cell-centred B at step start (PDM limiter reference)
  R* Msh;  // 3 half-step cell-centred B
  R* Bh;   // 3 half-step face fields
  R* V;    // 6 centre-to-edge first-sweep velocities (2 per edge direction)
  R* E;    // 3 edge EMFs
  R* F;    // 27 face fluxes (9 per direction)
  R* Wl;   // FP32 path: 6 step-start primitives in R (the limiters' reference)
  R* Bl;   // FP32 path: 3 step-start face fields in R
  const R* tab;  // the per-axis tables in R (same layout as Params::tab)
  const R* fw;   // the packed face records in R (tab + fw_offset(tmax))
};
constexpr int WORK_FIELDS = 6 + 3 + 3 + 3 + 6 + 3 + 27;
// the FP32 path adds the R copies of the step-start state (Wl, Bl)
constexpr int work_fields(bool mixed) { return WORK_FIELDS + (mixed ? 9 : 0); }

int64_t launches();
void count_launches(int64_t n);  // kernels run by graph replays

// kernel groups of one step, for event timing
enum Group : int { G_BEGIN = 0, G_AB2, G_C2C, G_EMF, G_FLUX, G_UPDATE, G_GHOST, G_END, NGROUP };

// launch shapes of the tunable kernels: AB2, C2C x3, EMF x3, FLUX x3,
// UPDATE; then the ghost launches (periodic wrap per axis, boundary fill
// per face), whose shapes are fixed (ghost_block)
enum TuneSlot : int { K_AB2 = 0, K_C2C0, K_C2C1, K_C2C2, K_EMF0, K_EMF1, K_EMF2,
                      K_FLUX0, K_FLUX1, K_FLUX2, K_UPDATE, NTUNE,
                      K_WRAP0 = NTUNE, K_WRAP1, K_WRAP2, K_BC0, K_BC1, K_BC2, K_BC3, K_BC4,
                      K_BC5, NSLOT };
struct Tune {
  dim3 blk[NTUNE];
  // flux of axis d / EMF of the edges along d from the tile-staged sweep
  // kernels (gop_sweep.cu) instead of the per-point kernels, where the
  // sweeps apply
  bool flux_sweep[3];
  bool emf_sweep[3];
  // order of the three (independent) launches of the flux and EMF stages
  int flux_order[3];
  int emf_order[3];
  Tune();
};

// Tensor maps and launch data of an instance's tile-staged flux sweeps
// (gop_sweep.cu); null when they could not be made (the per-face kernels run)
struct SweepSet;
template <typename R>
SweepSet* sweep_create(const Params& P, const Work<R>& w);
void sweep_destroy(SweepSet* s);
// the flux of axis D by the sweep kernel; false (nothing launched) where the
// sweep does not apply (no maps, or the entropy channel is live)
template <typename R>
bool launch_flux_sweep(const SweepSet* sw, const Params& P, const Work<R>& w, int D,
                       cudaStream_t st);
// the row-end faces of the flux along i that its sweep leaves out (32
// dividing n0), by the per-face arithmetic
template <typename R>
void launch_flux_col(const Params& P, const Work<R>& w, cudaStream_t st);
// the EMF of the edges along D by the sweep kernel; false without maps
template <typename R>
bool launch_emf_sweep(const SweepSet* sw, const Params& P, const Work<R>& w, int D,
                      cudaStream_t st);

// points covered by the launch of one slot (x, y, z extents)
dim3 launch_space(const Params& P, int slot);
// thread-block shape of a ghost-fill slot (K_WRAP*, K_BC*)
dim3 ghost_block(int slot);

// launches one tunable kernel alone (for the autotuner); a flux or EMF slot
// with sw set runs the sweep kernel instead (blk unused); pdl false:
// without programmatic dependent launch
template <typename R>
void launch_slot(const Params& P, int coord, const Work<R>& w, int slot, dim3 blk,
                 cudaStream_t st, const SweepSet* sw = nullptr, bool pdl = true);

// optional timing hook: mark(ctx, group, start) records an event on the stream
struct Hook {
  void (*mark)(void* ctx, int group, int start) = nullptr;
  void* ctx = nullptr;
  void operator()(int g, int s) const {
    if (mark) mark(ctx, g, s);
  }
};
void launch_begin(const Params& P, cudaStream_t st);
void launch_end(const Params& P, cudaStream_t st);
// arm a gop_step call: stop after time tstop or after `budget` steps
void launch_arm(const Params& P, double tstop, double budget, cudaStream_t st);
// CFL dt (in the form and arithmetic of the step's own estimate) and
// max|div B| of the current state
void launch_dt(const Params& P, int coord, bool mixed, cudaStream_t st);
// P.scal[S_PSNZ] <- 1 if p_S is nonzero in either state buffer (it must be 0 before)
void launch_ps_check(const Params& P, cudaStream_t st);
template <typename R>
void launch_step_body(const Params& P, int coord, const Work<R>& w, cudaStream_t st,
                      const Tune& tune, const SweepSet* sw, const Hook& hook = Hook());
// which = 0: the buffer being written this step; 1: the current state
void launch_ghosts(const Params& P, const char bc[6], const char gem_bc[6], int which,
                   cudaStream_t st);
void launch_from_ref(const Params& P, int nf, const double* src, double* dst, cudaStream_t st);
void launch_to_ref(const Params& P, int nf, const double* src, double* dst, cudaStream_t st);
template <typename R>
void launch_widen(const Params& P, int nf, const R* src, double* dst, cudaStream_t st);
void launch_mags(const Params& P, const double* B, double* out, cudaStream_t st);
// pole ring average (spherical grids reaching a pole): the pole-edge EMFs
// before the update; the ring averages of the new state after it (scratch:
// 2 fields of doubles)
template <typename R>
void launch_pole_emf(const Params& P, const Work<R>& w, cudaStream_t st);
void launch_ring_average(const Params& P, double* scratch, cudaStream_t st);
// background field B0 of a built-in kind into the background block out
// (BG_NF fields, zero beforehand); aux: 12 fields of doubles of scratch
void launch_background(const Params& P, const gop_background& bg, int sph, double* out, double* aux,
                       cudaStream_t st);
// problem p's initial state in buffer 0 (cells, face field; ghosts left for
// the ghost fill); scratch: 3 fields of doubles for the edge integrals
void launch_problem_init(const Params& P, const gop_problem& p, int sph, double* scratch,
                         cudaStream_t st);

}  // namespace gop

// Device-side pieces of the step shared by the per-point kernels
// (gop_kernels.cu) and the tile-staged sweep kernels (gop_sweep.cu): the
// state slot names, launch plumbing, the limiter references of each path and
// the Rusanov face flux with the Maxwell stress.
#pragma once

#include "gop_device.cuh"
#include "gop_kernels.h"

namespace gop {

enum { RHO = 0, V1, V2, V3, PR, PS };

__device__ __forceinline__ bool stopped(const Params& P) { return P.scal[S_STOP] != 0.0; }

// Programmatic dependent launch: LAUNCH lets each kernel start launching
// while its predecessor on the stream is still running.  Every kernel it
// launches first waits here until that predecessor has completed and its
// writes are visible, then lets its own successor start launching, so only
// launch latency and block scheduling overlap, never the work.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

__device__ __forceinline__ double rsq(double x) { return rsqrt(x); }
__device__ __forceinline__ float rsq(float x) { return rsqrtf(x); }

// The step-start state the PDM limiters compare against, in the stage type:
// the FP64 state itself on the plain path, its FP32 copy (written by the
// AB2 stage) on the mixed path.
template <typename R>
__device__ __forceinline__ const R* lim_w(const Params& P, const Work<R>& wk) {
  if constexpr (sizeof(R) == 8) return reinterpret_cast<const R*>(P.Wbuf[cur_buf(P)]);
  else return wk.Wl;
}
template <typename R>
__device__ __forceinline__ const R* lim_b(const Params& P, const Work<R>& wk) {
  if constexpr (sizeof(R) == 8) return reinterpret_cast<const R*>(P.Bbuf[cur_buf(P)]);
  else return wk.Bl;
}

// Rusanov hydro flux and Maxwell stress at the face normal to D at cell x
// from the reconstructed states (src/solver_func.c:934-1529) and bn, the
// step-start face field normal to the face.  F[9] = mass, 3 momenta,
// energy, entropy, 3 stress components.  Also writes the first
// centre-to-edge sweep of edges along (D+2)%3 (see c2c_body).
template <typename R, int D, bool BG, bool PSL>
__device__ __forceinline__ void flux_out(const Params& P, const Work<R>& wk, long long x,
                                         const R L[6], const R Rt[6], const R mL[3],
                                         const R mR[3], const R bn) {
  const size_t fs = P.fs;
  // background field averaged over this face (B0Aface*_b1..3; the normal
  // component is B0Aface*_bn)
  R b0[3] = {R(0), R(0), R(0)};
  if constexpr (BG) {
#pragma unroll
    for (int a = 0; a < 3; a++) b0[a] = (R)P.bg[(size_t)(BG_FACE + 3 * D + a) * fs + x];
  }
  const R gm = (R)P.gamma, gm1 = (R)P.gm1, ca = (R)P.ca, ca2 = (R)P.ca2;
  const R rl = L[RHO], rr = Rt[RHO], pl = L[PR], pr = Rt[PR], sl = L[PS], sr = Rt[PS];
  const R irl = R(1) / rl, irr = R(1) / rr;
  const R csl = sqrt(gm * pl * irl), csr = sqrt(gm * pr * irr);
  // entropy channel: p_S = 0 everywhere unless a problem sets it; the
  // zero test only skips exact zeros

  const R btl = mL[0] * mL[0] + mL[1] * mL[1] + mL[2] * mL[2];
  const R btr = mR[0] * mR[0] + mR[1] * mR[1] + mR[2] * mR[2];
  // |B + B0|^2 of either state: the Alfven speed and the Boris term see the
  // total field
  R ttl = btl, ttr = btr;
  if constexpr (BG) {
    ttl = (mL[0] + b0[0]) * (mL[0] + b0[0]) + (mL[1] + b0[1]) * (mL[1] + b0[1]) +
          (mL[2] + b0[2]) * (mL[2] + b0[2]);
    ttr = (mR[0] + b0[0]) * (mR[0] + b0[0]) + (mR[1] + b0[1]) * (mR[1] + b0[1]) +
          (mR[2] + b0[2]) * (mR[2] + b0[2]);
  }
  const R val = sqrt(ttl * irl), var = sqrt(ttr * irr);
  const R vel = val * ca * rsq(val * val + ca2);
  const R ver = var * ca * rsq(var * var + ca2);
  const R vnl = L[V1 + D], vnr = Rt[V1 + D];
  const R vf = fmax(fabs(vnl) + sqrt(csl * csl + vel * vel), fabs(vnr) + sqrt(csr * csr + ver * ver));
  R mol[3], mor[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    mol[a] = rl * L[V1 + a];
    mor[a] = rr * Rt[V1 + a];
  }
  const R igm1 = (R)P.inv_gm1;
  const R el = R(0.5) * rl * (L[V1] * L[V1] + L[V2] * L[V2] + L[V3] * L[V3]) + pl * igm1;
  const R er = R(0.5) * rr * (Rt[V1] * Rt[V1] + Rt[V2] * Rt[V2] + Rt[V3] * Rt[V3]) + pr * igm1;

  // the first centre-to-edge sweep for edges along E = (D+2)%3: velocity
  // components D and (D+1)%3 along D, averaged (see c2c_body)
  {
    constexpr int E = (D + 2) % 3, c1 = (D + 1) % 3;
    wk.V[x + (size_t)(2 * E) * fs] = R(0.5) * (L[V1 + D] + Rt[V1 + D]);
    wk.V[x + (size_t)(2 * E + 1) * fs] = R(0.5) * (L[V1 + c1] + Rt[V1 + c1]);
  }
  R* o = wk.F + (size_t)(9 * D) * fs + x;
  o[0] = R(0.5) * (mol[D] + mor[D] - vf * (rr - rl));
#pragma unroll
  for (int a = 0; a < 3; a++) {
    R u = mol[a] * vnl + mor[a] * vnr - vf * (mor[a] - mol[a]);
    if (a == D) u = mol[a] * vnl + pl + mor[a] * vnr + pr - vf * (mor[a] - mol[a]);
    o[(1 + a) * fs] = R(0.5) * u;
  }
  o[4 * fs] = R(0.5) * (el * vnl + pl * vnl + er * vnr + pr * vnr - vf * (er - el));
  // entropy channel (p_S = 0 unless a problem sets it): with zero left and
  // right states its flux is zero and the update leaves p_S at +0 either way
  R fS = R(0);
  if (sl != R(0) || sr != R(0)) {
    const R csel = sl == R(0) ? R(0) : sqrt(gm * sl * irl);
    const R cser = sr == R(0) ? R(0) : sqrt(gm * sr * irr);
    const R vfe = fmax(fabs(vnl) + sqrt(csel * csel + vel * vel), fabs(vnr) + sqrt(cser * cser + ver * ver));
    const R Sl = (sl == R(0) && rl > R(0)) ? sl : sl / pow(rl, gm1);
    const R Sr = (sr == R(0) && rr > R(0)) ? sr : sr / pow(rr, gm1);
    fS = R(0.5) * (Sl * vnl + Sr * vnr - vfe * (Sr - Sl));
  }
  if constexpr (PSL) o[5 * fs] = fS;  // else the update takes a zero divergence
  const R bq = (ttl + ttr) * (R)P.q_ca;
  if constexpr (BG) {
    // stress of B^2 + 2 B.B0 with the B0 cross terms
    // (src/solver_func.c:1268-1333)
    const R bsl = btl + R(2) * (mL[0] * b0[0] + mL[1] * b0[1] + mL[2] * b0[2]);
    const R bsr = btr + R(2) * (mR[0] * b0[0] + mR[1] * b0[1] + mR[2] * b0[2]);
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const R pl = a == D ? R(0.5) * bsl : R(0), pr = a == D ? R(0.5) * bsr : R(0);
      const R tl = R(0.5) * (pl - (mL[a] + b0[a]) * bn - mL[a] * b0[D]);
      const R tr = R(0.5) * (pr - (mR[a] + b0[a]) * bn - mR[a] * b0[D]);
      o[(6 + a) * fs] = (tl + tr) - bq * (Rt[V1 + a] - L[V1 + a]);
    }
  } else {
#pragma unroll
    for (int a = 0; a < 3; a++) {
      R tl, tr;
      if (a == D) {
        tl = R(0.5) * (R(0.5) * btl - mL[a] * bn);
        tr = R(0.5) * (R(0.5) * btr - mR[a] * bn);
      } else {
        tl = R(0.5) * (-mL[a] * bn);
        tr = R(0.5) * (-mR[a] * bn);
      }
      o[(6 + a) * fs] = (tl + tr) - bq * (Rt[V1 + a] - L[V1 + a]);
    }
  }
}

// The edge EMF (src/solver_func.c:779-902) from the edge's reconstructions:
// vp, vq the second-sweep velocities, (bpl, bpr) B_p reconstructed along q,
// (bql, bqr) B_q along p, b0p / b0q the background field averaged along the
// edge (BG), rho4 the sum of the four half-step densities around the edge.
template <typename R, bool BG>
__device__ __forceinline__ R emf_finish(const Params& P, R vp, R vq, R bpl, R bpr, R bql, R bqr,
                                        R b0p, R b0q, R rho4) {
  R bp = R(0.5) * (bpl + bpr), bq = R(0.5) * (bql + bqr);
  if constexpr (BG) {
    bp += b0p;
    bq += b0q;
  }
  R e = -(vp * bq - vq * bp);
  const R ca = (R)P.ca;
  R vz = sqrt((bp * bp + bq * bq) / (R(0.25) * rho4));
  vz = vz * ca * rsq(vz * vz + ca * ca) + sqrt(vp * vp + vq * vq);
  e += R(0.5) * vz * (bpl + bqr - bpr - bql);
  return e;
}

}  // namespace gop

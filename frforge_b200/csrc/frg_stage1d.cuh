// Fused 1D FR stage kernel for sm_100a (FP64).
//
// Same phase structure as the 2D kernel: a CTA stages TX elements plus one
// halo element on each side, computes traces and the interface flux of every
// face once (compute_interface_fluxes!, src/fr/Residual.jl:24-115), the
// strong-form volume + g_DG lift (Residual.jl:187-208), the BR0 or D(Du)
// dissipation (src/capturing/PerssonAV.jl:203-351), the SSP-RK stage
// combination, and for the new state the Persson sensor (PerssonAV.jl:116-135),
// element viscosity (:158-177) and the CFL wave speed (SSP_RK3.jl:8-24).
#pragma once

#include "frg_control.cuh"
#include "frg_device.cuh"

namespace frg {

template <int NP>
struct Tile1D {
  static constexpr int TX = 64;
};

template <int NP, int TXV = Tile1D<NP>::TX>
struct Smem1D {
  static constexpr int NEQ = 3, TX = TXV, NSLOT = TX + 2;
  static constexpr int oU = 0;
  static constexpr int oF = oU + NSLOT * NEQ * NP;
  static constexpr int oG = oF + TX * NEQ * NP;
  static constexpr int oFace = oG + TX * NEQ * NP;  // [TX+1][8]: fhat[3], ghat[3]
  static constexpr int oSlot = oFace + (TX + 1) * 8;  // eps, J, dx
  static constexpr int oTr = oSlot + NSLOT * 3;       // [NSLOT][6]: overridden traces xi = -1, +1
  static constexpr int oRed = oTr + NSLOT * 6;
  static constexpr int nDoubles = oRed + 32;
  static constexpr int nInts = NSLOT * 2;
  static constexpr size_t bytes = nDoubles * sizeof(double) + nInts * sizeof(int);
};

// One tile of one stage; x0: first element of the tile; TXV elements per tile.
// COHERENT: the stage input was written earlier in the same launch by other
// CTAs (the cluster loop kernel), so it is read through L2 (ld.global.cg)
// instead of the non-coherent read-only path, which lies outside the memory
// model's ordering by the cluster barriers.
template <int NP, int FLUX, int AV, int TXV = Tile1D<NP>::TX, bool COHERENT = false>
__device__ __forceinline__ void stage1d_tile(const OpsT<NP>& ops, const Mesh1Dev& M, const Phys& P,
                                             const StageBufs& B, const int x0) {
  using S = Smem1D<NP, TXV>;
  constexpr int NEQ = 3, TX = S::TX, NSLOT = S::NSLOT;
  constexpr bool kBR0 = (AV == kAvBR0);
  constexpr bool kAV = (AV != kAvNone);
  extern __shared__ __align__(16) double smem[];
  double* sU = smem + S::oU;
  double* sF = smem + S::oF;
  double* sG = smem + S::oG;
  double* sFace = smem + S::oFace;
  double* sEps = smem + S::oSlot;
  double* sJ = sEps + NSLOT;
  double* sDx = sJ + NSLOT;
  double* sTr = smem + S::oTr;
  double* sRed = smem + S::oRed;
  int* sEl = reinterpret_cast<int*>(smem + S::nDoubles);
  int* sOwn = sEl + NSLOT;

  const int tid = threadIdx.x, nthr = blockDim.x;
  const int nel = M.nel;
  const size_t cs = (size_t)nel * NP;

  // the step's status words are loaded first and tested after the staging
  // below, so that their latency overlaps the staging loads; a skipped stage
  // has written nothing when it returns
  int sc_active = 1;
  unsigned sc_flags = 0u;
  double dt = 0.0, tstage = 0.0, sc_t0 = 0.0;
  if (B.use_sc) {
    sc_active = B.sc->active;
    sc_flags = B.sc->flags;
    dt = B.sc->dt;
    sc_t0 = B.sc->t0;
  } else if (B.sc) {
    tstage = B.sc->t;
    dt = B.sc->dt;
  }
  const bool prime = (B.mode == kModePrime) || (B.mode == kModeSense);

  for (int s = tid; s < NSLOT; s += nthr) {
    int g = x0 + s - 1, el = -1, own = 0;
    bool ok = true, wrap = false;
    if (g < 0) {
      if (M.periodic) { g += nel; wrap = true; } else ok = false;
    } else if (g >= nel) {
      if (g == nel && M.periodic) { g = 0; wrap = true; } else ok = false;
    }
    if (ok) {
      el = g;
      own = (s >= 1 && s <= TX && !wrap);
      if (prime && !own) el = -1;
    }
    if (el >= 0) {
      sJ[s] = M.J[el];
      sDx[s] = M.dx[el];
      sEps[s] = (kAV && !prime) ? B.eps_in[el] : 0.0;
    }
    sEl[s] = el;
    sOwn[s] = own;
  }
  __syncthreads();

  for (int idx = tid; idx < NEQ * NSLOT * NP; idx += nthr) {
    const int r = idx % (NSLOT * NP), c = idx / (NSLOT * NP);
    const int s = r / NP, k = r % NP;
    const int el = sEl[s];
    if (el >= 0) {
      const double* src = &(B.uw ? B.uw : B.us)[c * cs + (size_t)el * NP + k];
      sU[(s * NEQ + c) * NP + k] = COHERENT ? __ldcg(src) : __ldg(src);
    }
  }
  __syncthreads();
  if (B.use_sc) {
    if (!sc_active || (sc_flags & (B.stage == 1 ? 0u : (B.stage == 2 ? 1u : 5u)))) return;
    tstage = (B.stage == 1) ? sc_t0 : (B.stage == 2 ? sc_t0 + dt : sc_t0 + dt / 2.0);
  }
  (void)tstage;

  // extrapolate_interface override (residual!, Residual.jl:175): both traces
  // of every staged element, for the numerical fluxes; the BR0 terms keep
  // the Lagrange traces, as apply_dissipation_br0! computes its own
  const bool trh = !prime && P.trace_hook != 0;
  if (trh) {
    double ws = 0.0;
#pragma unroll
    for (int i = 0; i < NP; ++i) ws += ops.w[i];
    for (int s = tid; s < NSLOT; s += nthr) {
      if (sEl[s] < 0) continue;
      double m[3], tl[3], tr[3];
#pragma unroll
      for (int c = 0; c < NEQ; ++c) {
        double a = 0.0, l = 0.0, r = 0.0;
#pragma unroll
        for (int i = 0; i < NP; ++i) {
          const double v = sU[(s * NEQ + c) * NP + i];
          a += ops.w[i] * v;
          l += ops.lL[i] * v;
          r += ops.lR[i] * v;
        }
        m[c] = a / ws;
        tl[c] = l;
        tr[c] = r;
      }
      trace_override1(P.trace_hook, P.trace_p0, P.trace_p1, P.g1, m, tl, tr);
#pragma unroll
      for (int c = 0; c < NEQ; ++c) {
        sTr[s * 6 + c] = tl[c];
        sTr[s * 6 + 3 + c] = tr[c];
      }
    }
    __syncthreads();
  }

  if (!prime) {
    // P1: physical flux at own solution points
    for (int idx = tid; idx < TX * NP; idx += nthr) {
      const int k = idx % NP, o = idx / NP, s = o + 1;
      if (!sOwn[s]) continue;
      double U[3], F[3];
#pragma unroll
      for (int c = 0; c < NEQ; ++c) U[c] = sU[(s * NEQ + c) * NP + k];
      flux1(P.g1, U, F);
#pragma unroll
      for (int c = 0; c < NEQ; ++c) sF[(o * NEQ + c) * NP + k] = F[c];
    }
    // P2: faces f = 0..TX between slots f and f+1
    for (int f = tid; f < TX + 1; f += nthr) {
      const int sA = f, sB = f + 1;
      double* out = sFace + f * 8;
      if (!(sOwn[sA] || sOwn[sB])) continue;
      const int eA = sEl[sA], eB = sEl[sB];
      double uA[3], uB[3], gA[3], gB[3];
      if (eA >= 0) {
#pragma unroll
        for (int c = 0; c < NEQ; ++c) {
          double su = 0.0, sg = 0.0;
          const double vc = sU[(sA * NEQ + c) * NP + NP / 2];
#pragma unroll
          for (int i = 0; i < NP; ++i) {
            const double v = sU[(sA * NEQ + c) * NP + i];
            su += ops.lR[i] * v;
            if (kBR0) sg += ops.lRD[i] * (v - vc);
          }
          uA[c] = su;
          gA[c] = sg;
        }
      }
      if (eB >= 0) {
#pragma unroll
        for (int c = 0; c < NEQ; ++c) {
          double su = 0.0, sg = 0.0;
          const double vc = sU[(sB * NEQ + c) * NP + NP / 2];
#pragma unroll
          for (int i = 0; i < NP; ++i) {
            const double v = sU[(sB * NEQ + c) * NP + i];
            su += ops.lL[i] * v;
            if (kBR0) sg += ops.lLD[i] * (v - vc);
          }
          uB[c] = su;
          gB[c] = sg;
        }
      }
      // the numerical flux's traces: the override's, or the Lagrange ones
      double fA[3], fB[3];
#pragma unroll
      for (int c = 0; c < NEQ; ++c) {
        fA[c] = (trh && eA >= 0) ? sTr[sA * 6 + 3 + c] : uA[c];
        fB[c] = (trh && eB >= 0) ? sTr[sB * 6 + c] : uB[c];
      }
      double fh[3], gh[3] = {0.0, 0.0, 0.0};
      if (eA >= 0 && eB >= 0) {
        iflux1<FLUX>(P.gamma, P.g1, fA, fB, fh, P.flux_alpha);
        if (kBR0) {
          const double sa = sEps[sA] / sJ[sA], sb = sEps[sB] / sJ[sB];
          const double tau = br0_tau(sEps[sA], sEps[sB], sDx[sA], sDx[sB], P.p);
#pragma unroll
          for (int c = 0; c < NEQ; ++c) gh[c] = 0.5 * (sa * gA[c] + sb * gB[c]) - tau * (uB[c] - uA[c]);
        }
      } else if (eB >= 0) {  // domain left end (Residual.jl:63-89)
        double ug[3];
        exterior1(M.bc[0], fB, -1.0, ug);
        iflux1<FLUX>(P.gamma, P.g1, ug, fB, fh, P.flux_alpha);
        if (kBR0) {
          const double sb = sEps[sB] / sJ[sB];
#pragma unroll
          for (int c = 0; c < NEQ; ++c) gh[c] = sb * gB[c];
        }
      } else {  // domain right end (Residual.jl:91-112)
        double ug[3];
        exterior1(M.bc[1], fA, 1.0, ug);
        iflux1<FLUX>(P.gamma, P.g1, fA, ug, fh, P.flux_alpha);
        if (kBR0) {
          const double sa = sEps[sA] / sJ[sA];
#pragma unroll
          for (int c = 0; c < NEQ; ++c) gh[c] = sa * gA[c];
        }
      }
#pragma unroll
      for (int c = 0; c < NEQ; ++c) {
        out[c] = fh[c];
        out[4 + c] = gh[c];
      }
    }
    __syncthreads();
    // P3: volume + lift (+ dissipation) per (element, component)
    for (int idx = tid; idx < TX * NEQ; idx += nthr) {
      const int c = idx % NEQ, o = idx / NEQ, s = o + 1;
      if (!sOwn[s]) continue;
      // shifted lines: Dt 1 = -(gL + gR), DtD 1 = DD 1 = 0 (exact identities)
      double Fl[NP], Ul[NP];
      const double fc = sF[(o * NEQ + c) * NP + NP / 2], uc = sU[(s * NEQ + c) * NP + NP / 2];
#pragma unroll
      for (int k = 0; k < NP; ++k) {
        Fl[k] = sF[(o * NEQ + c) * NP + k] - fc;
        Ul[k] = sU[(s * NEQ + c) * NP + k] - uc;
      }
      const double fL = sFace[o * 8 + c] - fc, fR = sFace[(o + 1) * 8 + c] - fc;
      const double gLh = kBR0 ? sFace[o * 8 + 4 + c] : 0.0;
      const double gRh = kBR0 ? sFace[(o + 1) * 8 + 4 + c] : 0.0;
      const double J = sJ[s], rJ = 1.0 / J;
      const double ev = kAV ? sEps[s] / (J * J) : 0.0;
#pragma unroll
      for (int j = 0; j < NP; ++j) {
        double acc = ops.gL[j] * fL + ops.gR[j] * fR;
#pragma unroll
        for (int k = 0; k < NP; ++k) acc += ops.Dt[j][k] * Fl[k];
        double r = -acc * rJ;
        if (kBR0) {
          double av = 0.0;
#pragma unroll
          for (int m = 0; m < NP; ++m) av += ops.DtD[j][m] * Ul[m];
          r += ev * av + (ops.gL[j] * gLh + ops.gR[j] * gRh) * rJ;
        } else if (AV == kAvDD) {
          double av = 0.0;
#pragma unroll
          for (int m = 0; m < NP; ++m) av += ops.DD[j][m] * Ul[m];
          r += ev * av;
        }
        sG[(o * NEQ + c) * NP + j] = r;
      }
    }
    __syncthreads();
    // P5: stage combination
    int bad_du = 0, bad_u = 0;
    const double cdt = B.c * dt;
    for (int idx = tid; idx < NEQ * TX * NP; idx += nthr) {
      const int r = idx % (TX * NP), c = idx / (TX * NP);
      const int o = r / NP, k = r % NP, s = o + 1;
      if (!sOwn[s]) continue;
      const double du = sG[(o * NEQ + c) * NP + k];
      const size_t gi = c * cs + (size_t)sEl[s] * NP + k;
      if (B.mode == kModeResidual) {
        B.du_out[gi] = du;
        bad_du |= !isfinite(du);
        continue;
      }
      const double us = B.uw ? __ldcg(&B.us[gi]) : sU[(s * NEQ + c) * NP + k];
      const double u0 = (B.stage == 1) ? us : B.u0[gi];
      const double un = (B.a * u0 + B.b * us) + cdt * du;
      B.uout[gi] = un;
      sF[(o * NEQ + c) * NP + k] = un;
      bad_du |= !isfinite(du);
      bad_u |= !isfinite(un);
    }
    // one barrier that also votes on non-finite values; only a tile with one
    // tells the residual and the state apart
    if (__syncthreads_or(bad_du | bad_u)) {
      const int any_du = __syncthreads_or(bad_du);
      const int any_u = __syncthreads_or(bad_u);
      if (tid == 0 && B.sc)
        atomicOr(&B.sc->flags, ((any_du ? 1u : 0u) | (any_u ? 2u : 0u)) << (2 * (B.stage - 1)));
    }
    if (B.mode == kModeResidual) return;
  } else {
    for (int idx = tid; idx < TX * NEQ * NP; idx += nthr) {
      const int o = idx / (NEQ * NP), s = o + 1;
      if (sOwn[s]) sF[idx] = sU[(s * NEQ) * NP + (idx - o * NEQ * NP)];
    }
    __syncthreads();
  }

  // P6: sensor, eps and CFL wave speed of the new state
  if (!(kAV || B.want_lambda || B.mode == kModeSense)) return;
  double lmax = 0.0;
  double* sWS = sG;
  for (int idx = tid; idx < TX * NP; idx += nthr) {
    const int k = idx % NP, o = idx / NP, s = o + 1;
    if (!sOwn[s]) continue;
    double U[3];
#pragma unroll
    for (int c = 0; c < NEQ; ++c) U[c] = sF[(o * NEQ + c) * NP + k];
    const double w = wave_speed1(P.gamma, P.g1, U);
    sWS[o * NP + k] = w;
    lmax = jmax(lmax, w);
  }
  if (B.want_lambda) {
    for (int off = 16; off > 0; off >>= 1) lmax = jmax(lmax, __shfl_xor_sync(0xffffffffu, lmax, off));
    if ((tid & 31) == 0) sRed[tid >> 5] = lmax;
  }
  __syncthreads();
  if (B.want_lambda && tid < 32) {
    double v = (tid < (nthr >> 5)) ? sRed[tid] : 0.0;
    for (int off = 16; off > 0; off >>= 1) v = jmax(v, __shfl_xor_sync(0xffffffffu, v, off));
    if (tid == 0 && B.sc) atomic_max_nonneg(&B.sc->lam_bits, v);
  }
  if (!(kAV || B.mode == kModeSense)) return;
  for (int o = tid; o < TX; o += nthr) {
    const int s = o + 1;
    if (!sOwn[s]) continue;
    const int el = sEl[s];
    double rho[NP];
#pragma unroll
    for (int k = 0; k < NP; ++k) rho[k] = sF[(o * NEQ) * NP + k];
    double etot = 0.0, ehigh = 0.0;
#pragma unroll
    for (int i = 0; i < NP; ++i) {
      double a = 0.0;
#pragma unroll
      for (int k = 0; k < NP; ++k) a += ops.Vinv[i][k] * rho[k];
      etot += a * a;
      if (i == NP - 1) ehigh = a * a;
    }
    const double sig = persson_sigma(ehigh, etot + P.eps_floor, P.s0, P.kappa, P.eps_floor);
    if (B.mode == kModeSense) {
      B.sigma_out[el] = sig;
      continue;
    }
    double lam = 0.0;
#pragma unroll
    for (int k = 0; k < NP; ++k) lam = jmax(lam, sWS[o * NP + k]);
    lam = jmax(lam, kEps);
    B.eps_out[el] = (sig > 0.0) ? P.c_av * sig * (sDx[s] / (double)P.pm) * lam : 0.0;
  }
}

// Single solve: the grid covers the mesh with tiles.
template <int NP, int FLUX, int AV>
__global__ void __launch_bounds__(256)
    stage1d_kernel(const OpsT<NP> ops, const Mesh1Dev M, const Phys P, const StageBufs B) {
  stage1d_tile<NP, FLUX, AV>(ops, M, P, B, blockIdx.x * Tile1D<NP>::TX);
}

// All threads of the cluster: prior global and shared writes of every CTA
// become visible to every CTA of the cluster (release / acquire).
FRG_DEV void cluster_barrier() {
  asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;\n" ::: "memory");
}

// Small 1D solves: one thread-block cluster covers the whole mesh, one tile
// of LTX elements per CTA, and runs `nsteps` passes of the ssp_rk3!/ssp_rk2! loop body (the
// top, the stages, the bottom) with cluster barriers between them, instead of
// five kernel launches per step.  Every CTA runs the same tile function on the
// same tile as stage1d_kernel, reading its stage input through L2.  The
// compiler fuses a few multiply-adds differently when the tile function is
// inlined here, so the steps agree with the launched path to a few ulps of
// the state (not bit for bit), with the same step count, time and status.
// The CTAs take the same barriers in the same order; a tile whose step is
// inactive returns from the tile function, not from the kernel.
template <int NP, int FLUX, int AV, int LTX>
__global__ void __launch_bounds__(256)
    loop1d_kernel(const OpsT<NP> ops, const Mesh1Dev M, const Phys P, const Loop1DBufs L, DevScalars* sc,
                  int nsteps) {
  const int x0 = blockIdx.x * LTX;
  const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
  if (lead) step_begin_device(sc);
  cluster_barrier();
  for (int n = 0; n < nsteps; ++n) {
    for (int s = 0; s < L.nstages; ++s) {
      stage1d_tile<NP, FLUX, AV, LTX, true>(ops, M, P, L.st[s], x0);
      cluster_barrier();
    }
    // the bottom of this pass and the top of the next, by the same thread
    if (lead) {
      step_end_device(sc, L.nstages);
      if (n + 1 < nsteps) step_begin_device(sc);
    }
    cluster_barrier();
  }
}

}  // namespace frg

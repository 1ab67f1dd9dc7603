// Fused 2D FR stage kernel for sm_100a (FP64).
//
// A CTA owns a TX x TY tile of elements and stages the tile plus a
// one-element halo ring (no corners) of the stage input in shared memory.
// Everything a stage needs happens on chip:
//   P0  cp.async copies of the tile: u_s (tile + halo), the step-start state
//       u0 of the tile and the per-slot mesh values (eps, Jx, Jy, 1/Jx,
//       1/Jy, h_char); every other per-element factor is a product of these
//   P1  physical fluxes -> contravariant F~, G~ at every own solution point
//       (Residual2D.jl:342-352)
//   P2  every face point of the tile once: u traces of both sides
//       (face_trace!, Residual2D.jl:9-48), for BR0 the g traces and the
//       averaged viscous flux g^ (PerssonAV2D.jl:228-350), then one
//       Rusanov/HLLC evaluation on the interior pair or on a trace and its
//       wall / boundary ghost state, times sJ (Residual2D.jl:173-334)
//   P3  xi-direction divergence + g_DG lift (Residual2D.jl:354-374) and the
//       BR0 / D(Du) x-terms (PerssonAV2D.jl:135-194, :352-375)
//   P4  eta-direction terms (Residual2D.jl:376-396, PerssonAV2D.jl:376-395),
//       independent of P3; the epilogue adds the two directions
//   P5  SSP-RK stage combination (SSP_RK3.jl:135-164) written straight to
//       HBM -- du never leaves the chip -- plus non-finite flags
//   P6  sensor of the NEW state (sense!, PerssonAV2D.jl:20-59), element
//       viscosity eps for the next stage (element_viscosities_2d,
//       PerssonAV2D.jl:89-109) and the CFL wave speed (compute_dt,
//       SSP_RK3.jl:126-133) as one atomic max per tile of its elements'
//       maxima.
// Halo values come from the neighbouring tiles' own loads, so they are
// L2 hits; DRAM traffic per stage is the algorithmic u_s + u0 + u_out.
//
// The single-solve kernel and the batched kernels run one tile per CTA
// through the same phases (tile_slots / tile_issue / tile_compute); tile
// variants differ in tile shape, threads per CTA (256, 384 or 512) and CTAs
// per SM, and the single-solve kernel has affine and curved instantiations.
// A persistent variant that copied each CTA's next tile into a second buffer
// while computing the current one measured slower on a B200: the other
// resident CTAs already cover the load latency.
//
// Shared-memory blocks use odd strides (in doubles) between elements and
// lanes walk over elements first, so a warp's 8-byte accesses spread over
// all banks.
#pragma once

#include "frg_device.cuh"

namespace frg {

template <int NP>
struct Tile2D;
// Default tile shapes (elements) of stage2d_kernel<..> without explicit
// tile arguments.
template <>
struct Tile2D<2> {
  static constexpr int TX = 8, TY = 8;
};
template <>
struct Tile2D<3> {
  static constexpr int TX = 8, TY = 6;
};
template <>
struct Tile2D<4> {
  static constexpr int TX = 8, TY = 4;
};
template <>
struct Tile2D<5> {
  static constexpr int TX = 4, TY = 4;
};
template <>
struct Tile2D<6> {
  static constexpr int TX = 4, TY = 3;
};

constexpr int odd_up(int n) { return (n % 2) ? n : n + 1; }

// Element stride (doubles) of a staged element, NEQ * NP2 padded so that the
// warps' 8-byte shared loads of P1-P5 spread over the 16 bank pairs: picked
// per tile shape with a model of the phases' address patterns (wavefronts =
// most distinct words on one bank pair) -- e.g. 3.07 -> 2.60 wavefronts per
// load on the 4x4 P=3 tile, 2.68 -> 2.38 on the 8x2 one; on a B200 the 512^2
// P=3 stage kernel gained 5.7 % (64.7 -> 68.4 G DOF-stage/s), with the
// vertical face order below.
constexpr int stage_es(int np, int tx, int ty) {
  return np == 2 ? (tx == 16 ? (ty == 8 ? 17 : 19) : 23)  // 16x8: 19 would not fit two CTAs
       : np == 3 ? 41
       : np == 4 ? ((tx == 8 && ty == 4) ? 65 : 67)
       : np == 5 ? 105
       : np == 6 ? (tx == 6 ? 151 : 153)
       : odd_up(4 * np * np);
}

// Shared-memory layout.  U0S: stage the step-start state u0 in shared memory
// (copied with the tile); otherwise the epilogue reads it from global memory.
template <int NP, int TX, int TY, bool U0S = true, int MINB = 2, int NTHR = 256>
struct Smem2D {
  static constexpr int NT = NTHR;  // threads per CTA
  static constexpr int NEQ = 4, NP2 = NP * NP;
  static constexpr int BX = TX + 2, BY = TY + 2, NSLOT = BX * BY, NOWN = TX * TY;
  static constexpr int NFV = (TX + 1) * TY, NFH = TX * (TY + 1);
  static constexpr int ES = stage_es(NP, TX, TY);  // element stride (doubles)
  static constexpr int FS = odd_up(NP * 8);     // face stride: NP points x (fhat[4], ghat[4])
  // one tile buffer (doubles): u_s of tile + halo, u0 of the tile, per-slot
  // mesh values [6][NSLOT] = eps, Jx, Jy, 1/Jx, 1/Jy, h_char
  static constexpr int bU = 0;
  static constexpr int bU0 = bU + NSLOT * ES;
  static constexpr int bRaw = bU0 + (U0S ? NOWN * ES : 0);
  static constexpr int bDoubles = bRaw + 6 * NSLOT;
  static constexpr int oF = bDoubles;               // [NOWN][ES]
  static constexpr int oG = oF + NOWN * ES;         // [NOWN][ES]
  static constexpr int oFV = oG + NOWN * ES;        // [NFV][FS]
  static constexpr int oFH = oFV + NFV * FS;        // [NFH][FS]
  static constexpr int oRed = oFH + NFH * FS;       // reduction scratch
  static constexpr int nDoubles = oRed + 32;
  static constexpr int nInts = NSLOT * 2 + 8;  // element ids, flags
  static_assert(NOWN <= NTHR, "the viscosity pass covers a tile with one pass of the block");
  static constexpr size_t bytes = nDoubles * sizeof(double) + nInts * sizeof(int);
  // 1 KB reserved per CTA plus the batched kernels' static descriptors
  static_assert(MINB * (bytes + 1024 + kBatchStaticSmem) <= 228 * 1024,
                "MINB CTAs must fit in one SM's shared memory");
};

constexpr int kStageThreads = 256;

// slot flag bits
enum : int { kSlotOwn = 1, kSlotWrap = 2, kSlotSolid = 4 };

FRG_DEV void cp_async8(double* dst, const double* src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(src) : "memory");
}
FRG_DEV void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
FRG_DEV void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// One tile buffer in shared memory.
struct TileBuf {
  double* U;    // [NSLOT][ES]
  double* U0;   // [NOWN][ES]
  double* raw;  // [6][NSLOT]
  int* el;      // [NSLOT]
  int* flag;    // [NSLOT]
};

template <class S>
FRG_DEV TileBuf tile_buf(double* smem) {
  TileBuf t;
  t.U = smem + S::bU;
  t.U0 = smem + S::bU0;
  t.raw = smem + S::bRaw;
  t.el = reinterpret_cast<int*>(smem + S::nDoubles);
  t.flag = t.el + S::NSLOT;
  return t;
}

// Stage-wide control values, the same for every tile of the launch.
struct StageCtl {
  double dt, tstage;
  bool prime, need_u0;
};

// false: the stage is skipped (the step is inactive or an earlier stage
// flagged a non-finite value).
FRG_DEV bool stage_control(const StageBufs& B, StageCtl& c) {
  c.dt = 0.0;
  c.tstage = 0.0;
  if (B.use_sc) {
    if (!B.sc->active || (B.sc->flags & (B.stage == 1 ? 0u : (B.stage == 2 ? 1u : 5u)))) return false;
    c.dt = B.sc->dt;
    const double t0 = B.sc->t0;
    c.tstage = (B.stage == 1) ? t0 : (B.stage == 2 ? t0 + c.dt : t0 + c.dt / 2.0);
  } else if (B.sc) {
    c.tstage = B.sc->t;
    c.dt = B.sc->dt;
  }
  c.prime = (B.mode == kModePrime) || (B.mode == kModeSense);
  c.need_u0 = (B.mode == kModeStage) && (B.stage != 1);
  return true;
}

// Slots of a tile: element id (-1: none) and flags of every tile + halo slot.
template <class S>
FRG_DEV void tile_slots(const Mesh2Dev& M, const TileBuf& tb, const int tx0, const int ty0, const bool prime) {
  constexpr int BX = S::BX, BY = S::BY, NSLOT = S::NSLOT, TX = S::BX - 2, TY = S::BY - 2;
  const int nx = M.nx, ny = M.ny;
  for (int s = threadIdx.x; s < NSLOT; s += S::NT) {
    const int bx = s % BX, by = s / BX;
    const bool corner = (bx == 0 || bx == BX - 1) && (by == 0 || by == BY - 1);
    int gx = tx0 + bx - 1, gy = ty0 + by - 1;
    int el = -1, fl = 0;
    if (!corner) {
      const bool ownpos = (bx >= 1 && bx <= TX && by >= 1 && by <= TY);
      bool ok = true, wrap = false;
      if (gx < 0) {
        if (M.px) { gx += nx; wrap = true; } else ok = false;
      } else if (gx >= nx) {
        if (gx == nx && M.px) { gx = 0; wrap = true; } else ok = false;
      }
      if (gy < 0) {
        if (M.py) { gy += ny; wrap = true; } else ok = false;
      } else if (gy >= ny) {
        if (gy == ny && M.py) { gy = 0; wrap = true; } else ok = false;
      }
      if (ok) {
        el = gy * nx + gx;
        if (ownpos && !wrap) fl |= kSlotOwn;
        if (wrap) fl |= kSlotWrap;
        if (prime && !(fl & kSlotOwn)) el = -1;  // prime/sense: own elements only
        if (el >= 0 && M.solid && M.solid[el]) fl |= kSlotSolid;
      }
    }
    tb.el[s] = el;
    tb.flag[s] = fl;
  }
}

// P0: issue the cp.async copies of a tile (one commit group); the slots of
// the buffer must be visible to every thread.
// PRE: a preprocess_state hook is active; the tile stages the work state
// B.uw (the residual's input) instead of the stage state B.us.
template <int NP, int AV, class S, bool PRE = false>
FRG_DEV void tile_issue(const Mesh2Dev& M, const StageBufs& B, const TileBuf& tb, const StageCtl& c) {
  constexpr int NEQ = 4, NP2 = NP * NP, ES = S::ES, BX = S::BX, BY = S::BY, NSLOT = S::NSLOT;
  constexpr int TX = BX - 2, TY = BY - 2;
  constexpr int NT = S::NT;
  constexpr bool U0S = (S::bRaw != S::bU0);
  const int tid = threadIdx.x;
  const size_t cs = (size_t)M.nel * NP2;  // component stride
  // Thread (e, k): solution point k of every EL-th slot, all components.
  // Per copy only the two addresses advance; a warp covers whole elements,
  // which are contiguous per component in global memory.
  constexpr int EL = NT / NP2;
  const int k = tid % NP2, e = tid / NP2;
  if (e < EL) {
    for (int s = e; s < NSLOT; s += EL) {
      const int el = tb.el[s];
      if (el < 0) continue;
      double* dst = tb.U + s * ES + k;
      const double* src = (PRE ? B.uw : B.us) + (size_t)el * NP2 + k;
#pragma unroll
      for (int cc = 0; cc < NEQ; ++cc) cp_async8(dst + cc * NP2, src + cc * cs);
    }
    if (U0S && c.need_u0) {
      for (int o = e; o < TX * TY; o += EL) {
        const int s = (o / TX + 1) * BX + (o % TX) + 1;
        if (!(tb.flag[s] & kSlotOwn)) continue;
        double* dst = tb.U0 + o * ES + k;
        const double* src = B.u0 + (size_t)tb.el[s] * NP2 + k;
#pragma unroll
        for (int cc = 0; cc < NEQ; ++cc) cp_async8(dst + cc * NP2, src + cc * cs);
      }
    }
  }
  // per-slot mesh values
  for (int s = tid; s < NSLOT; s += NT) {
    const int el = tb.el[s];
    if (el < 0) continue;
    const int gx = el % M.nx, gy = el / M.nx;
    if (AV != kAvNone && !c.prime) cp_async8(&tb.raw[s], &B.eps_in[el]);
    cp_async8(&tb.raw[NSLOT + s], &M.Jx[gx]);
    cp_async8(&tb.raw[2 * NSLOT + s], &M.Jy[gy]);
    cp_async8(&tb.raw[3 * NSLOT + s], &M.rJx[gx]);
    cp_async8(&tb.raw[4 * NSLOT + s], &M.rJy[gy]);
    if (AV != kAvNone && (tb.flag[s] & kSlotOwn)) cp_async8(&tb.raw[5 * NSLOT + s], &M.hchar[el]);
  }
  cp_async_commit();
}

// P1-P6 of one tile whose copies are in tb.  WAIT: cp.async groups that may
// still be pending when the tile starts.
// CURV: 0 affine mesh, 1 curved mesh, -1 read from the descriptor.
// INT: an interior tile of an affine mesh (tile_is_interior): every slot
// holds an element, the tile positions are its own elements, there is no
// solid element and every face is an interior face, so no slot flag is read
// and no boundary or wall case is compiled.
// PRE: the staged state is the work state of a preprocess_state hook; the
// stage combination reads the stage state itself from global memory.
template <int NP, int FLUX, int AV, class S, int WAIT, int CURV = -1, bool INT = false, bool PRE = false>
FRG_DEV void tile_compute(const OpsT<NP>& ops, const Mesh2Dev& M, const Phys& P, const StageBufs& B,
                          const TileBuf& tb, double* smem, const StageCtl& ctl) {
  static_assert(!INT || CURV == 0, "interior tiles are affine");
  const bool curved = CURV < 0 ? (M.curved != 0) : (CURV == 1);
  constexpr int NEQ = 4, NP2 = NP * NP, ES = S::ES, FS = S::FS;
  constexpr int BX = S::BX, NSLOT = S::NSLOT, NOWN = S::NOWN;
  constexpr int TX = S::BX - 2, TY = S::BY - 2;
  constexpr int NFV = S::NFV, NFH = S::NFH;
  constexpr int NT = S::NT;
  constexpr bool kBR0 = (AV == kAvBR0);
  constexpr bool kAV = (AV != kAvNone);
  constexpr bool U0S = (S::bRaw != S::bU0);

  double* sU = tb.U;
  double* sU0 = tb.U0;
  const int* sEl = tb.el;
  int* sFlag = tb.flag;
  const double* sEps = tb.raw;
  const double* sJx = tb.raw + NSLOT;
  const double* sJy = tb.raw + 2 * NSLOT;
  const double* sRjx = tb.raw + 3 * NSLOT;  // 1/Jx
  const double* sRjy = tb.raw + 4 * NSLOT;  // 1/Jy
  const double* sHc = tb.raw + 5 * NSLOT;
  double* sF = smem + S::oF;
  double* sG = smem + S::oG;
  double* sFV = smem + S::oFV;
  double* sFH = smem + S::oFH;
  double* sRed = smem + S::oRed;

  const int tid = threadIdx.x;
  const int nx = M.nx;
  const size_t cs = (size_t)M.nel * NP2;  // component stride
  const bool prime = ctl.prime;
  const double dt = ctl.dt, tstage = ctl.tstage;

  cp_async_wait<WAIT>();
  __syncthreads();

  // wave speeds of the new state (P5 in a stage, P6 in prime / sense), in the
  // face-array space, which is free once P3 and P4 are done
  constexpr int WS = odd_up(NP2);
  double* sWS = sFV;  // [NOWN][WS]
  const bool need_ws = kAV || B.want_lambda || B.mode == kModeSense;
  double lmax = 0.0;

  if (!prime) {
    // ------------------------------------------------------- P1 fluxes
    // item = k + NP2*o: lanes walk over the points of an element, so a warp's
    // loads of the staged state are consecutive words (no bank conflicts)
    for (int idx = tid; idx < NOWN * NP2; idx += NT) {
      const int k = idx % NP2, o = idx / NP2;
      const int s = (o / TX + 1) * BX + (o % TX) + 1;
      if (!INT && (!(sFlag[s] & kSlotOwn) || (sFlag[s] & kSlotSolid))) continue;
      double U[4], F[4], G[4];
#pragma unroll
      for (int c = 0; c < NEQ; ++c) U[c] = sU[s * ES + c * NP2 + k];
      flux_xy(P.g1, U, F, G);
      double* fo = sF + o * ES + k;
      double* go = sG + o * ES + k;
      if (curved) {
        const size_t m = (size_t)sEl[s] * NP2 + k;
        const double xxi = M.m_xxi[m], xeta = M.m_xeta[m], yxi = M.m_yxi[m], yeta = M.m_yeta[m];
#pragma unroll
        for (int c = 0; c < NEQ; ++c) {
          fo[c * NP2] = yeta * F[c] - xeta * G[c];
          go[c * NP2] = -yxi * F[c] + xxi * G[c];
        }
      } else {
        const double jy = sJy[s], jx = sJx[s];
#pragma unroll
        for (int c = 0; c < NEQ; ++c) {
          fo[c * NP2] = jy * F[c];
          go[c * NP2] = jx * G[c];
        }
      }
    }

    // ------------------------------------------------------- P2 faces
    for (int idx = tid; idx < (NFV + NFH) * NP; idx += NT) {
      const bool vert = idx < NFV * NP;
      const int id2 = vert ? idx : idx - NFV * NP;
      int f, q, sA, sB;
      if (vert) {
        // lanes walk over the points of a face and then the faces of a row
        // (P = 3, 4), or over the faces of a row (fewer bank conflicts there)
        int fx, fy;
        if (NP == 4 || NP == 5) {
          q = id2 % NP;
          const int r = id2 / NP;
          fx = r % (TX + 1);
          fy = r / (TX + 1);
        } else {
          fx = id2 % (TX + 1);
          const int r = id2 / (TX + 1);
          q = r % NP;
          fy = r / NP;
        }
        f = fy * (TX + 1) + fx;
        sA = (fy + 1) * BX + fx;
        sB = sA + 1;
      } else {
        const int fx = id2 % TX, r = id2 / TX;
        q = r % NP;
        const int fy = r / NP;
        f = fy * TX + fx;
        sA = fy * BX + fx + 1;
        sB = sA + BX;
      }
      const int flA = INT ? kSlotOwn : sFlag[sA], flB = INT ? kSlotOwn : sFlag[sB];
      if (!INT && !((flA | flB) & kSlotOwn)) continue;
      double* out = (vert ? sFV : sFH) + f * FS + q * 8;
      const int eA = INT ? 0 : sEl[sA], eB = INT ? 0 : sEl[sB];
      // the face line inside A (its east/north end) and B (west/south end)
      const int lstride = vert ? 1 : NP;
      const int lbase = vert ? NP * q : q;
      double uA[4], uB[4], gA[4], gB[4];
      // g traces use l^T D, whose entries sum to zero: shifting the line by
      // one of its values removes the cancellation of large terms exactly.
      if (INT || eA >= 0) {
#pragma unroll
        for (int c = 0; c < NEQ; ++c) {
          const double* a = sU + sA * ES + c * NP2 + lbase;
          const double vc = a[(NP / 2) * lstride];
          double su = 0.0, sg = 0.0;
#pragma unroll
          for (int i = 0; i < NP; ++i) {
            const double v = a[i * lstride];
            su += ops.lR[i] * v;
            if (kBR0) sg += ops.lRD[i] * (v - vc);
          }
          uA[c] = su;
          gA[c] = sg;
        }
      }
      if (INT || eB >= 0) {
#pragma unroll
        for (int c = 0; c < NEQ; ++c) {
          const double* b = sU + sB * ES + c * NP2 + lbase;
          const double vc = b[(NP / 2) * lstride];
          double su = 0.0, sg = 0.0;
#pragma unroll
          for (int i = 0; i < NP; ++i) {
            const double v = b[i * lstride];
            su += ops.lL[i] * v;
            if (kBR0) sg += ops.lLD[i] * (v - vc);
          }
          uB[c] = su;
          gB[c] = sg;
        }
      }
      // BR0 averaged viscous flux first, so that the g traces are dead
      // before the numerical flux
      if (kBR0) {
        double gh[4];
        if (INT || (eA >= 0 && eB >= 0)) {
          // eps/J of both sides; element widths 2 J (exact)
          const double sa = sEps[sA] * (vert ? sRjx[sA] : sRjy[sA]);
          const double sb = sEps[sB] * (vert ? sRjx[sB] : sRjy[sB]);
          const double tau = br0_tau(sEps[sA], sEps[sB], 2.0 * (vert ? sJx[sA] : sJy[sA]),
                                     2.0 * (vert ? sJx[sB] : sJy[sB]), P.p);
#pragma unroll
          for (int c = 0; c < NEQ; ++c) gh[c] = 0.5 * (sa * gA[c] + sb * gB[c]) - tau * (uB[c] - uA[c]);
        } else {
          const bool haveB = eB >= 0;
          const int s = haveB ? sB : sA;
          const double sc = sEps[s] * (vert ? sRjx[s] : sRjy[s]);
#pragma unroll
          for (int c = 0; c < NEQ; ++c) gh[c] = sc * (haveB ? gB[c] : gA[c]);
        }
#pragma unroll
        for (int c = 0; c < NEQ; ++c) out[4 + c] = gh[c];
      }
      double fh[4] = {0.0, 0.0, 0.0, 0.0};
      const int fE = vert ? 1 : 3, fW = vert ? 0 : 2;  // face slots E/N and W/S
      // The two states and the normal of the numerical flux: the interior
      // pair, or an element's trace and its ghost state (wall or domain
      // boundary).  One flux evaluation serves every case.
      double fL[4], fR[4], fnx = 0.0, fny = 0.0, fsJ = 0.0;
      bool doflux = false;
      if (INT) {
        // interior pair, affine unit normal
        fnx = vert ? 1.0 : 0.0;
        fny = vert ? 0.0 : 1.0;
        fsJ = vert ? sJy[sA] : sJx[sA];
#pragma unroll
        for (int c = 0; c < NEQ; ++c) {
          fL[c] = uA[c];
          fR[c] = uB[c];
        }
        doflux = true;
      } else if (eA >= 0 && eB >= 0) {
        const bool solA = flA & kSlotSolid, solB = flB & kSlotSolid;
        const bool wrapf = (flA | flB) & kSlotWrap;
        if (wrapf && (solA || solB)) {
          // the reference never writes these slots (Residual2D.jl:220, :302)
        } else if (solA && solB) {
        } else if (solA || solB) {
          // wall between a solid and a fluid element (Residual2D.jl:186-200)
          const bool fluidB = solA;
          const int e = fluidB ? eB : eA;
          const int face = fluidB ? fW : fE;
          double nxo, nyo, sJ;
          if (curved) {
            nxo = M.f_nx[face][(size_t)e * NP + q];
            nyo = M.f_ny[face][(size_t)e * NP + q];
            sJ = M.f_sJ[face][(size_t)e * NP + q];
          } else {
            nxo = vert ? (fluidB ? -1.0 : 1.0) : 0.0;
            nyo = vert ? 0.0 : (fluidB ? -1.0 : 1.0);
            sJ = vert ? sJy[fluidB ? sB : sA] : sJx[fluidB ? sB : sA];
          }
          double ui[4], ug[4];
#pragma unroll
          for (int c = 0; c < NEQ; ++c) ui[c] = fluidB ? uB[c] : uA[c];
          reflect2(ui, nxo, nyo, ug);
#pragma unroll
          for (int c = 0; c < NEQ; ++c) {
            fL[c] = fluidB ? ug[c] : ui[c];
            fR[c] = fluidB ? ui[c] : ug[c];
          }
          fnx = fluidB ? -nxo : nxo;
          fny = fluidB ? -nyo : nyo;
          fsJ = sJ;
          doflux = true;
        } else {
          if (curved) {
            fnx = M.f_nx[fE][(size_t)eA * NP + q];
            fny = M.f_ny[fE][(size_t)eA * NP + q];
            fsJ = M.f_sJ[fE][(size_t)eA * NP + q];
          } else {
            fnx = vert ? 1.0 : 0.0;
            fny = vert ? 0.0 : 1.0;
            fsJ = vert ? sJy[sA] : sJx[sA];
          }
#pragma unroll
          for (int c = 0; c < NEQ; ++c) {
            fL[c] = uA[c];
            fR[c] = uB[c];
          }
          doflux = true;
        }
      } else {
        // domain boundary: A missing (left/bottom) or B missing (right/top)
        const bool haveB = eB >= 0;
        const int s = haveB ? sB : sA;
        const int e = haveB ? eB : eA;
        const int fl = haveB ? flB : flA;
        const int face = haveB ? fW : fE;
        const BCDev& bc = M.bc[vert ? (haveB ? 0 : 1) : (haveB ? 2 : 3)];
        if (!(fl & kSlotSolid)) {
          double nxo, nyo, sJ;
          if (curved) {
            nxo = M.f_nx[face][(size_t)e * NP + q];
            nyo = M.f_ny[face][(size_t)e * NP + q];
            sJ = M.f_sJ[face][(size_t)e * NP + q];
          } else {
            nxo = vert ? (haveB ? -1.0 : 1.0) : 0.0;
            nyo = vert ? 0.0 : (haveB ? -1.0 : 1.0);
            sJ = vert ? sJy[s] : sJx[s];
          }
          // face point coordinates (physical_xy, MeshMetrics2D.jl:49-74)
          const int gx = e % nx, gy = e / nx;
          double X, Y;
          if (vert) {
            X = M.xc[gx] + M.Jx[gx] * (haveB ? -1.0 : 1.0);
            Y = M.yc[gy] + M.Jy[gy] * ops.xi[q];
          } else {
            X = M.xc[gx] + M.Jx[gx] * ops.xi[q];
            Y = M.yc[gy] + M.Jy[gy] * (haveB ? -1.0 : 1.0);
          }
          if (M.wavy) X = X + M.amp * sin(6.283185307179586 * Y) * sin(3.141592653589793 * X);
          double ui[4], ug[4];
#pragma unroll
          for (int c = 0; c < NEQ; ++c) ui[c] = haveB ? uB[c] : uA[c];
          exterior<4>(bc, ui, nxo, nyo, X, tstage, ug);
#pragma unroll
          for (int c = 0; c < NEQ; ++c) {
            fL[c] = haveB ? ug[c] : ui[c];
            fR[c] = haveB ? ui[c] : ug[c];
          }
          fnx = haveB ? -nxo : nxo;
          fny = haveB ? -nyo : nyo;
          fsJ = sJ;
          doflux = true;
        }
      }
      if (doflux) {
        iflux2<FLUX>(P.gamma, P.g1, fL, fR, fnx, fny, fh, !curved);
#pragma unroll
        for (int c = 0; c < NEQ; ++c) fh[c] *= fsJ;
      }
#pragma unroll
      for (int c = 0; c < NEQ; ++c) out[c] = fh[c];
    }
    __syncthreads();

    // u0 of this thread's epilogue points, from global memory when it is not
    // staged: issued here so that P3 and P4 cover the load latency
    constexpr int EL5 = NT / NP2, NIT5 = (NOWN + EL5 - 1) / EL5;
    double u0r[NIT5][NEQ];
    if (!U0S && ctl.need_u0) {
      const int k = tid % NP2, e = tid / NP2;
#pragma unroll
      for (int it = 0; it < NIT5; ++it) {
        const int o = e + it * EL5;
        if (e < EL5 && o < NOWN) {
          const int s = (o / TX + 1) * BX + (o % TX) + 1;
          if (INT || (sFlag[s] & kSlotOwn)) {
            const size_t g0 = (size_t)sEl[s] * NP2 + k;
#pragma unroll
            for (int c = 0; c < NEQ; ++c) u0r[it][c] = __ldg(&B.u0[c * cs + g0]);
          }
        }
      }
    }

    // ------------------------------------------------ P3 xi-direction
    // item = o + NOWN*(j + NP*c): lanes walk over elements
    for (int idx = tid; idx < NOWN * NP * NEQ; idx += NT) {
      const int o = idx % NOWN, t = idx / NOWN;
      const int j = t % NP, c = t / NP;
      const int ox = o % TX, oy = o / TX;
      const int s = (oy + 1) * BX + ox + 1;
      if (!INT && !(sFlag[s] & kSlotOwn)) continue;
      double* Fo = sF + o * ES + c * NP2 + NP * j;
      if (!INT && (sFlag[s] & kSlotSolid)) {
#pragma unroll
        for (int i = 0; i < NP; ++i) Fo[i] = 0.0;
        continue;
      }
      const double* Uo = sU + s * ES + c * NP2 + NP * j;
      // Dt 1 = -(gL + gR) and DtD 1 = DD 1 = 0: every line is shifted by its
      // middle value so the folded operators never cancel large terms.
      double Fl[NP], Ul[NP];
      const double fc = Fo[NP / 2], uc = Uo[NP / 2];
#pragma unroll
      for (int k = 0; k < NP; ++k) {
        Fl[k] = Fo[k] - fc;
        Ul[k] = Uo[k] - uc;
      }
      const int fWi = oy * (TX + 1) + ox;
      const double* fw = sFV + fWi * FS + j * 8 + c;
      const double fhW = fw[0] - fc;
      const double fhE = fw[FS] - fc;
      const double ghW = kBR0 ? fw[4] : 0.0;
      const double ghE = kBR0 ? fw[FS + 4] : 0.0;
      const double rjx = sRjx[s];
      const double ev = kAV ? (sEps[s] * rjx) * rjx : 0.0;
      if (!curved) {
        // affine: the element factors -1/J, eps/J^2 and 1/Jx are folded into
        // the line data; each output is two short chains (lifts and fluxes,
        // dissipation) and one add
        const double sj = -(rjx * sRjy[s]);
#pragma unroll
        for (int k = 0; k < NP; ++k) {
          Fl[k] *= sj;
          if (kAV) Ul[k] *= ev;
        }
        const double LW = kBR0 ? sj * fhW + rjx * ghW : sj * fhW;
        const double LE = kBR0 ? sj * fhE + rjx * ghE : sj * fhE;
#pragma unroll
        for (int i = 0; i < NP; ++i) {
          double r = ops.gL[i] * LW + ops.gR[i] * LE;
#pragma unroll
          for (int k = 0; k < NP; ++k) r += ops.Dt[i][k] * Fl[k];
          double d = 0.0;
          if (kBR0) {
#pragma unroll
            for (int m = 0; m < NP; ++m) d += ops.DtD[i][m] * Ul[m];
          } else if (AV == kAvDD) {
#pragma unroll
            for (int m = 0; m < NP; ++m) d += ops.DD[i][m] * Ul[m];
          }
          Fo[i] = kAV ? r + d : r;
        }
        continue;
      }
      const size_t mrow = (size_t)sEl[s] * NP2 + NP * j;
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        double acc = ops.gL[i] * fhW + ops.gR[i] * fhE;
#pragma unroll
        for (int k = 0; k < NP; ++k) acc += ops.Dt[i][k] * Fl[k];
        const double rJ = M.m_rJ[mrow + i];
        double r = -acc * rJ;
        if (kBR0) {
          double av = 0.0;
#pragma unroll
          for (int m = 0; m < NP; ++m) av += ops.DtD[i][m] * Ul[m];
          r += ev * av + (ops.gL[i] * ghW + ops.gR[i] * ghE) * rjx;
        } else if (AV == kAvDD) {
          double av = 0.0;
#pragma unroll
          for (int m = 0; m < NP; ++m) av += ops.DD[i][m] * Ul[m];
          r += ev * av;
        }
        Fo[i] = r;
      }
    }

    // ----------------------------------------------- P4 eta-direction
    // independent of P3 (it writes only sG): the two share one barrier
    // interval and the epilogue adds the two directions
    for (int idx = tid; idx < NOWN * NP * NEQ; idx += NT) {
      const int o = idx % NOWN, t = idx / NOWN;
      const int i = t % NP, c = t / NP;
      const int ox = o % TX, oy = o / TX;
      const int s = (oy + 1) * BX + ox + 1;
      if (!INT && !(sFlag[s] & kSlotOwn)) continue;
      double* Go = sG + o * ES + c * NP2 + i;
      if (!INT && (sFlag[s] & kSlotSolid)) {
#pragma unroll
        for (int j = 0; j < NP; ++j) Go[NP * j] = 0.0;
        continue;
      }
      const double* Uo = sU + s * ES + c * NP2 + i;
      double Gl[NP], Ul[NP];
      const double gc = Go[NP * (NP / 2)], uc = Uo[NP * (NP / 2)];
#pragma unroll
      for (int k = 0; k < NP; ++k) {
        Gl[k] = Go[NP * k] - gc;
        Ul[k] = Uo[NP * k] - uc;
      }
      const int fSi = oy * TX + ox;
      const double* fs = sFH + fSi * FS + i * 8 + c;
      const double fhS = fs[0] - gc;
      const double fhN = fs[TX * FS] - gc;
      const double ghS = kBR0 ? fs[4] : 0.0;
      const double ghN = kBR0 ? fs[TX * FS + 4] : 0.0;
      const double rjy = sRjy[s];
      const double ev = kAV ? (sEps[s] * rjy) * rjy : 0.0;
      if (!curved) {
        // affine: element factors folded into the line data (as in P3)
        const double sj = -(sRjx[s] * rjy);
#pragma unroll
        for (int k = 0; k < NP; ++k) {
          Gl[k] *= sj;
          if (kAV) Ul[k] *= ev;
        }
        const double LS = kBR0 ? sj * fhS + rjy * ghS : sj * fhS;
        const double LN = kBR0 ? sj * fhN + rjy * ghN : sj * fhN;
#pragma unroll
        for (int j = 0; j < NP; ++j) {
          double r = ops.gL[j] * LS + ops.gR[j] * LN;
#pragma unroll
          for (int k = 0; k < NP; ++k) r += ops.Dt[j][k] * Gl[k];
          double d = 0.0;
          if (kBR0) {
#pragma unroll
            for (int m = 0; m < NP; ++m) d += ops.DtD[j][m] * Ul[m];
          } else if (AV == kAvDD) {
#pragma unroll
            for (int m = 0; m < NP; ++m) d += ops.DD[j][m] * Ul[m];
          }
          Go[NP * j] = kAV ? r + d : r;
        }
        continue;
      }
      const size_t mbase = (size_t)sEl[s] * NP2 + i;
#pragma unroll
      for (int j = 0; j < NP; ++j) {
        double acc = ops.gL[j] * fhS + ops.gR[j] * fhN;
#pragma unroll
        for (int k = 0; k < NP; ++k) acc += ops.Dt[j][k] * Gl[k];
        const double rJ = M.m_rJ[mbase + NP * j];
        double r = -acc * rJ;
        if (kBR0) {
          double av = 0.0;
#pragma unroll
          for (int m = 0; m < NP; ++m) av += ops.DtD[j][m] * Ul[m];
          r += ev * av + (ops.gL[j] * ghS + ops.gR[j] * ghN) * rjy;
        } else if (AV == kAvDD) {
          double av = 0.0;
#pragma unroll
          for (int m = 0; m < NP; ++m) av += ops.DD[j][m] * Ul[m];
          r += ev * av;
        }
        Go[NP * j] = r;
      }
    }
    __syncthreads();

    // --------------------------------------------------- P5 epilogue
    // thread (e, k): solution point k of every EL-th own element, all
    // components (coalesced stores of whole elements).  Non-finite values
    // are caught by accumulating v * 0, which is NaN for an infinite or NaN v.
    {
      constexpr int EL = NT / NP2;
      const int k = tid % NP2, e = tid / NP2;
      double chk_du = 0.0, chk_u = 0.0;
      const double cdt = B.c * dt;
      if (e < EL) {
#pragma unroll
        for (int it = 0; it < NIT5; ++it) {
          const int o = e + it * EL;
          if (o >= NOWN) break;
          const int s = (o / TX + 1) * BX + (o % TX) + 1;
          if (!INT && !(sFlag[s] & kSlotOwn)) continue;
          const size_t g0 = (size_t)sEl[s] * NP2 + k;
          double unv[NEQ];
#pragma unroll
          for (int c = 0; c < NEQ; ++c) {
            const int li = o * ES + c * NP2 + k;
            const double du = sF[li] + sG[li];
            const size_t gi = c * cs + g0;
            chk_du = fma(du, 0.0, chk_du);
            if (B.mode == kModeResidual) {
              B.du_out[gi] = du;
              continue;
            }
            // with a preprocess_state hook the residual's input is the work
            // state; the stage combination takes the stage state itself
            const double us = PRE ? __ldcg(&B.us[gi]) : sU[s * ES + c * NP2 + k];
            const double u0 = (B.stage == 1) ? us : (U0S ? sU0[li] : u0r[it][c]);
            const double un = (B.a * u0 + B.b * us) + cdt * du;
            B.uout[gi] = un;
            if (c == 0) sF[li] = un;  // the sensor reads the new density
            unv[c] = un;
            chk_u = fma(un, 0.0, chk_u);
          }
          // wave speed of the new state at this point (P6 uses it)
          if (B.mode != kModeResidual && need_ws) {
            const double w = wave_speed2(P.gamma, P.g1, unv);
            sWS[o * WS + k] = w;
            lmax = jmax(lmax, w);
          }
        }
      }
      // one barrier (P6 reads what P5 wrote) that also votes on non-finite
      // values; only a tile with one tells the residual and the state apart
      const bool bad_du = chk_du != chk_du, bad_u = chk_u != chk_u;
      if (__syncthreads_or(bad_du || bad_u)) {
        const int any_du = __syncthreads_or(bad_du);
        const int any_u = __syncthreads_or(bad_u);
        if (tid == 0 && B.sc)
          atomicOr(&B.sc->flags, ((any_du ? 1u : 0u) | (any_u ? 2u : 0u)) << (2 * (B.stage - 1)));
      }
    }
    if (B.mode == kModeResidual) return;
  } else {
    // prime / sense: the "new" state is the loaded state
    for (int idx = tid; idx < NOWN * NEQ * NP2; idx += NT) {
      const int o = idx % NOWN, r = idx / NOWN;
      const int s = (o / TX + 1) * BX + (o % TX) + 1;
      if (INT || (sFlag[s] & kSlotOwn)) sF[o * ES + r] = sU[s * ES + r];
    }
    __syncthreads();
  }

  // ------------------------------------------ P6 sensor / eps / lambda
  if (!(kAV || B.want_lambda || B.mode == kModeSense)) return;
  {
    constexpr int PS = odd_up(2 * NP);
    double* sX = sG;                 // [NOWN][WS] V^{-1} rho
    double* sPart = sX + NOWN * WS;  // [NOWN][PS] row energies
    // in a stage the epilogue computed the wave speeds
    for (int idx = tid; prime && idx < NOWN * NP2; idx += NT) {
      const int o = idx % NOWN, k = idx / NOWN;
      const int s = (o / TX + 1) * BX + (o % TX) + 1;
      if (!INT && !(sFlag[s] & kSlotOwn)) continue;
      double U[4];
#pragma unroll
      for (int c = 0; c < NEQ; ++c) U[c] = sF[o * ES + c * NP2 + k];
      const double w = wave_speed2(P.gamma, P.g1, U);
      sWS[o * WS + k] = w;
      lmax = jmax(lmax, w);
    }
    if (kAV || B.mode == kModeSense) {
      // X = V^{-1} rho, column by column
      for (int idx = tid; idx < NOWN * NP; idx += NT) {
        const int o = idx % NOWN, j = idx / NOWN;
        const int s = (o / TX + 1) * BX + (o % TX) + 1;
        if (!INT && !(sFlag[s] & kSlotOwn)) continue;
        const double* rho = sF + o * ES + NP * j;
        double col[NP];
#pragma unroll
        for (int k = 0; k < NP; ++k) col[k] = rho[k];
#pragma unroll
        for (int i = 0; i < NP; ++i) {
          double a = 0.0;
#pragma unroll
          for (int k = 0; k < NP; ++k) a += ops.Vinv[i][k] * col[k];
          sX[o * WS + i + NP * j] = a;
        }
      }
    }
    // The CFL wave speed (compute_dt) of the tile: with the viscosity pass
    // below, the maximum over its elements' maxima (taken there); otherwise a
    // block maximum of the points' wave speeds.  One atomic per tile or warp.
    const bool lam_blk = B.want_lambda && !(kAV && B.mode != kModeSense);
    if (lam_blk) {
      for (int off = 16; off > 0; off >>= 1) lmax = jmax(lmax, __shfl_xor_sync(0xffffffffu, lmax, off));
      if ((tid & 31) == 0) sRed[tid >> 5] = lmax;
    }
    __syncthreads();
    if (lam_blk && tid < 32) {
      double v = (tid < (NT >> 5)) ? sRed[tid] : 0.0;
      for (int off = 16; off > 0; off >>= 1) v = jmax(v, __shfl_xor_sync(0xffffffffu, v, off));
      if (tid == 0 && B.sc) atomic_max_nonneg(&B.sc->lam_bits, v);
    }
    if (!(kAV || B.mode == kModeSense)) return;
    // Uhat = X V^{-T}: row i energies
    for (int idx = tid; idx < NOWN * NP; idx += NT) {
      const int o = idx % NOWN, i = idx / NOWN;
      const int s = (o / TX + 1) * BX + (o % TX) + 1;
      if (!INT && !(sFlag[s] & kSlotOwn)) continue;
      double row[NP];
#pragma unroll
      for (int k = 0; k < NP; ++k) row[k] = sX[o * WS + i + NP * k];
      double etot = 0.0, ehigh = 0.0;
#pragma unroll
      for (int j = 0; j < NP; ++j) {
        double a = 0.0;
#pragma unroll
        for (int k = 0; k < NP; ++k) a += row[k] * ops.Vinv[j][k];
        const double a2 = a * a;
        etot += a2;
        if (i == NP - 1 || j == NP - 1) ehigh += a2;
      }
      sPart[o * PS + 2 * i + 0] = etot;
      sPart[o * PS + 2 * i + 1] = ehigh;
    }
    __syncthreads();
    double lcta = 0.0;
    for (int o = tid; o < NOWN; o += NT) {
      const int s = (o / TX + 1) * BX + (o % TX) + 1;
      if (!INT && !(sFlag[s] & kSlotOwn)) continue;
      const int el = sEl[s];
      double etot = 0.0, ehigh = 0.0, lam = 0.0;
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        etot += sPart[o * PS + 2 * i + 0];
        ehigh += sPart[o * PS + 2 * i + 1];
      }
      {
        // pairwise (depth log2 NP2): the same maximum, a shorter chain
        double w[NP2];
#pragma unroll
        for (int k = 0; k < NP2; ++k) w[k] = sWS[o * WS + k];
#pragma unroll
        for (int h = 1; h < NP2; h *= 2)
#pragma unroll
          for (int k = 0; k + h < NP2; k += 2 * h) w[k] = jmax(w[k], w[k + h]);
        lam = jmax(lam, w[0]);
      }
      lcta = jmax(lcta, lam);
      lam = jmax(lam, kEps);
      const double sig = persson_sigma(ehigh, etot + P.eps_floor, P.s0, P.kappa, P.eps_floor);
      if (B.mode == kModeSense) {
        B.sigma_out[el] = (!INT && (sFlag[s] & kSlotSolid)) ? 0.0 : sig;
        continue;
      }
      double ev = 0.0;
      if ((INT || !(sFlag[s] & kSlotSolid)) && sig > 0.0) ev = P.c_av * sig * (sHc[s] * frcp((double)P.pm)) * lam;
      B.eps_out[el] = ev;
    }
    // the warps that hold elements (NOWN <= NT)
    if (B.want_lambda && B.mode != kModeSense && tid < ((NOWN + 31) & ~31)) {
      for (int off = 16; off > 0; off >>= 1) lcta = jmax(lcta, __shfl_xor_sync(0xffffffffu, lcta, off));
      if ((tid & 31) == 0 && B.sc) atomic_max_nonneg(&B.sc->lam_bits, lcta);
    }
  }
}

// A full tile of an affine mesh without solid elements whose one-element
// halo ring exists on all four sides (inside the mesh or across a periodic
// boundary): every face of its elements is an interior face.
template <int TX, int TY>
FRG_DEV bool tile_is_interior(const Mesh2Dev& M, const int tx0, const int ty0) {
  if (M.curved || M.solid) return false;
  if (tx0 + TX > M.nx || ty0 + TY > M.ny) return false;
  if (!M.px && (tx0 < 1 || tx0 + TX >= M.nx)) return false;
  if (!M.py && (ty0 < 1 || ty0 + TY >= M.ny)) return false;
  return true;
}

// One tile of one stage (single buffer).  tx0, ty0: first element of the
// tile.  Used by stage2d_kernel and by the batched kernels.
template <int NP, int FLUX, int AV, int TX, int TY, int MINB, bool U0S, int NTHR = kStageThreads,
          int CURV = -1, bool PRE = false>
__device__ __forceinline__ void stage2d_tile(const OpsT<NP>& ops, const Mesh2Dev& M, const Phys& P,
                                             const StageBufs& B, const int tx0, const int ty0) {
  using S = Smem2D<NP, TX, TY, U0S, MINB, NTHR>;
  extern __shared__ __align__(16) double smem[];
  StageCtl ctl;
  ctl.prime = (B.mode == kModePrime) || (B.mode == kModeSense);
  ctl.need_u0 = (B.mode == kModeStage) && (B.stage != 1);
  const TileBuf tb = tile_buf<S>(smem);
  tile_slots<S>(M, tb, tx0, ty0, ctl.prime);
  __syncthreads();
  // the copies go out before the step's status is read, so that the status
  // load overlaps them; a skipped stage waits for its copies and writes nothing
  tile_issue<NP, AV, S, PRE>(M, B, tb, ctl);
  if (!stage_control(B, ctl)) {
    cp_async_wait<0>();
    return;
  }
  // interior tiles of P >= 4 (NP >= 5) run the general body: the interior
  // body does not fit their 64 registers per thread and spills (measured on
  // a B200: P = 4 and 5 are 11-17 % faster without it, P = 1..3 11-21 %
  // faster with it)
  if (CURV != 1 && NP <= 4 && tile_is_interior<TX, TY>(M, tx0, ty0))
    tile_compute<NP, FLUX, AV, S, 0, 0, true, PRE>(ops, M, P, B, tb, smem, ctl);
  else
    tile_compute<NP, FLUX, AV, S, 0, CURV, false, PRE>(ops, M, P, B, tb, smem, ctl);
}

// Single solve, one tile per CTA: the grid covers the mesh with tiles.
template <int NP, int FLUX, int AV, int TX = Tile2D<NP>::TX, int TY = Tile2D<NP>::TY, int MINB = 2,
          bool U0S = true, int NTHR = kStageThreads, int CURV = -1, bool PRE = false>
__global__ void __launch_bounds__(NTHR, MINB)
    stage2d_kernel(const OpsT<NP> ops, const Mesh2Dev M, const Phys P, const StageBufs B) {
  stage2d_tile<NP, FLUX, AV, TX, TY, MINB, U0S, NTHR, CURV, PRE>(ops, M, P, B, blockIdx.x * TX,
                                                                 blockIdx.y * TY);
}

}  // namespace frg

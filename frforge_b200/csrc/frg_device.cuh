// Device-side Euler physics, numerical fluxes and boundary ghosts (FP64).
//
// Restates, for sm_100a, the point-wise functions of FRForge:
//   pressure / fluxes          src/equations/Euler.jl:18-128, Euler2D.jl:14-150
//   Rusanov                    src/flux/Rusanov.jl:10-25, Euler2D.jl:114-150
//   HLLC (Toro, Davis speeds)  src/flux/HLLC.jl:9-148
//   exterior_state / reflect   src/mesh/BoundaryConditions.jl:43-134
// Branch structure and floors follow the reference; reciprocals replace
// repeated divisions by the same density and the compiler may fuse
// multiply-adds, so results agree with the reference to rounding.
#pragma once

#include <cuda_runtime.h>

#include "frg_internal.h"

namespace frg {

#define FRG_DEV __device__ __forceinline__

// Floor max(x, c) for a finite constant c with Julia's NaN propagation:
// fmax drops a NaN operand, and adding x - x (0 for finite x, NaN otherwise)
// puts it back.
FRG_DEV double jfloor(double x, double c) { return fmax(x, c) + (x - x); }

// NaN-propagating max/min (Julia semantics for Float64).
FRG_DEV double jmax(double a, double b) {
  double r = fmax(a, b);
  return (a != a) ? a : ((b != b) ? b : r);
}
FRG_DEV double jmin(double a, double b) {
  double r = fmin(a, b);
  return (a != a) ? a : ((b != b) ? b : r);
}

// 1/x for the flux kernels: the hardware estimate of PTX rcp.approx.ftz.f64
// refined by two Newton-Raphson steps y <- y + y (1 - x y), each of which
// about doubles the number of correct bits (Markstein, IBM J. Res. Dev. 34
// (1990) 111-119); the result is within 1 ulp of the correctly rounded 1/x
// for finite x with 2^-1022 <= |x| < 2^1022 (checked against CUDA's division
// by tests/test_gpu_reciprocal.py).  It replaces the divisions of the flux
// and wave-speed formulas, whose operands are floored densities or guarded
// denominators; x = 0 gives NaN where the exact division gives an infinity,
// and either is caught as non-finite by the stage kernels.
FRG_DEV double frcp(double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  double e = fma(-x, y, 1.0);
  y = fma(y, e, y);
  e = fma(-x, y, 1.0);
  return fma(y, e, y);
}

// sqrt(x) for the sound speeds of the flux kernels: Goldschmidt's coupled
// iteration for g -> sqrt(x) and h -> 1/(2 sqrt(x)) (r = 1/2 - g h;
// g += g r; h += h r; Goldschmidt 1964, as in Markstein, "IA-64 and
// Elementary Functions", 2000), started from the PTX rsqrt.approx.ftz.f64
// estimate, two iterations and one residual correction g + (x - g^2) h.
// Within 1 ulp of CUDA's correctly rounded sqrt for positive normal x
// (tests/test_gpu_reciprocal.py); the operands are gamma p / rho with p and
// rho floored at eps, so always positive.  x = 0 gives NaN.
FRG_DEV double fsqrt(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  double h = 0.5 * y;
  double g = x * y;
  double r = fma(-g, h, 0.5);
  g = fma(g, r, g);
  h = fma(h, r, h);
  r = fma(-g, h, 0.5);
  g = fma(g, r, g);
  h = fma(h, r, h);
  const double d = fma(-g, g, x);
  return fma(d, h, g);
}

// ---------------------------------------------------------------- 2D Euler

// Physical fluxes F(U), G(U): physical_flux_x!/y!, Euler2D.jl:54-79.
FRG_DEV void flux_xy(double g1, const double U[4], double F[4], double G[4]) {
  const double r = jfloor(U[0], kEps);
  const double ri = frcp(r);
  const double u = U[1] * ri, v = U[2] * ri;
  const double p = g1 * (U[3] - 0.5 * r * (u * u + v * v));
  F[0] = U[1];
  F[1] = U[1] * u + p;
  F[2] = U[2] * u;
  F[3] = (U[3] + p) * u;
  G[0] = U[2];
  G[1] = U[1] * v;
  G[2] = U[2] * v + p;
  G[3] = (U[3] + p) * v;
}

// max(|u|+c, |v|+c) at one state: max_wave_speed, Euler2D.jl:92-105.
FRG_DEV double wave_speed2(double gamma, double g1, const double U[4]) {
  const double r = jfloor(U[0], kEps);
  const double ri = frcp(r);
  const double u = U[1] * ri, v = U[2] * ri;
  const double p = jfloor(g1 * (U[3] - 0.5 * r * (u * u + v * v)), kEps);
  const double c = fsqrt(gamma * p * ri);
  return jmax(fabs(u) + c, fabs(v) + c);
}

// Rusanov normal flux, numerical_flux_n!, Euler2D.jl:114-150.
FRG_DEV void rusanov2(double gamma, double g1, const double uL[4], const double uR[4],
                      double nx, double ny, double out[4]) {
  const double rL = jfloor(uL[0], kEps), riL = frcp(rL);
  const double uLv = uL[1] * riL, vLv = uL[2] * riL;
  const double pL = g1 * (uL[3] - 0.5 * rL * (uLv * uLv + vLv * vLv));
  const double rR = jfloor(uR[0], kEps), riR = frcp(rR);
  const double uRv = uR[1] * riR, vRv = uR[2] * riR;
  const double pR = g1 * (uR[3] - 0.5 * rR * (uRv * uRv + vRv * vRv));
  const double unL = uLv * nx + vLv * ny, unR = uRv * nx + vRv * ny;
  const double fL0 = uL[1] * nx + uL[2] * ny;
  const double fL1 = (uL[1] * uLv + pL) * nx + (uL[1] * vLv) * ny;
  const double fL2 = (uL[2] * uLv) * nx + (uL[2] * vLv + pL) * ny;
  const double fL3 = (uL[3] + pL) * unL;
  const double fR0 = uR[1] * nx + uR[2] * ny;
  const double fR1 = (uR[1] * uRv + pR) * nx + (uR[1] * vRv) * ny;
  const double fR2 = (uR[2] * uRv) * nx + (uR[2] * vRv + pR) * ny;
  const double fR3 = (uR[3] + pR) * unR;
  const double cL = fsqrt(gamma * jfloor(pL, kEps) * riL);
  const double cR = fsqrt(gamma * jfloor(pR, kEps) * riR);
  const double lam = jmax(fabs(unL) + cL, fabs(unR) + cR);
  const double hl = 0.5 * lam;
  out[0] = 0.5 * (fL0 + fR0) - hl * (uR[0] - uL[0]);
  out[1] = 0.5 * (fL1 + fR1) - hl * (uR[1] - uL[1]);
  out[2] = 0.5 * (fL2 + fR2) - hl * (uR[2] - uL[2]);
  out[3] = 0.5 * (fL3 + fR3) - hl * (uR[3] - uL[3]);
}

// HLLC normal flux, hllc_flux_n, src/flux/HLLC.jl:72-148.  `unit` skips the
// renormalisation of an exactly unit normal (affine faces: (+-1,0), (0,+-1)).
FRG_DEV void hllc2(double gamma, double g1, const double uL[4], const double uR[4], double nxi,
                   double nyi, double out[4], bool unit = false) {
  double nx = nxi, ny = nyi;
  if (!unit) {
    const double nrm = sqrt(nxi * nxi + nyi * nyi);
    if (nrm < kEps) {
      rusanov2(gamma, g1, uL, uR, nxi, nyi, out);
      return;
    }
    const double rn = 1.0 / nrm;
    nx = nxi * rn;
    ny = nyi * rn;
  }
  const double rL = jfloor(uL[0], kEps), riL = frcp(rL);
  const double rR = jfloor(uR[0], kEps), riR = frcp(rR);
  const double uLv = uL[1] * riL, vLv = uL[2] * riL;
  const double uRv = uR[1] * riR, vRv = uR[2] * riR;
  const double pLu = g1 * (uL[3] - 0.5 * rL * (uLv * uLv + vLv * vLv));
  const double pRu = g1 * (uR[3] - 0.5 * rR * (uRv * uRv + vRv * vRv));
  const double pL = jfloor(pLu, kEps), pR = jfloor(pRu, kEps);
  const double unL = uLv * nx + vLv * ny, unR = uRv * nx + vRv * ny;
  const double cL = fsqrt(gamma * pL * riL), cR = fsqrt(gamma * pR * riR);
  const double SL = jmin(unL - cL, unR - cR);
  const double SR = jmax(unL + cL, unR + cR);
  const double num = pR - pL + rL * unL * (SL - unL) - rR * unR * (SR - unR);
  const double den = rL * (SL - unL) - rR * (SR - unR);
  const double SM = fabs(den) < kEps ? 0.5 * (unL + unR) : num * frcp(den);
  // F.n with the unfloored pressure of physical_flux_x!/y!
  if (0.0 <= SL) {
    out[0] = uL[1] * nx + uL[2] * ny;
    out[1] = (uL[1] * uLv + pLu) * nx + (uL[1] * vLv) * ny;
    out[2] = (uL[2] * uLv) * nx + (uL[2] * vLv + pLu) * ny;
    out[3] = (uL[3] + pLu) * uLv * nx + (uL[3] + pLu) * vLv * ny;
    return;
  }
  if (0.0 >= SR) {
    out[0] = uR[1] * nx + uR[2] * ny;
    out[1] = (uR[1] * uRv + pRu) * nx + (uR[1] * vRv) * ny;
    out[2] = (uR[2] * uRv) * nx + (uR[2] * vRv + pRu) * ny;
    out[3] = (uR[3] + pRu) * uRv * nx + (uR[3] + pRu) * vRv * ny;
    return;
  }
  const bool left = (SL <= 0.0) && (0.0 <= SM);
  const double* U = left ? uL : uR;
  const double r = left ? rL : rR, ri = left ? riL : riR;
  const double u = left ? uLv : uRv, v = left ? vLv : vRv;
  const double p = left ? pL : pR, pu = left ? pLu : pRu;
  const double un = left ? unL : unR, S = left ? SL : SR;
  const double F0 = U[1] * nx + U[2] * ny;
  const double F1 = (U[1] * u + pu) * nx + (U[1] * v) * ny;
  const double F2 = (U[2] * u) * nx + (U[2] * v + pu) * ny;
  const double F3 = (U[3] + pu) * u * nx + (U[3] + pu) * v * ny;
  const double ustar = (u - un * nx) + SM * nx;
  const double vstar = (v - un * ny) + SM * ny;
  const double Sun = S - un;
  // the two remaining divisions are independent reciprocals
  const double rB = frcp(S - SM), rA = frcp(r * Sun);
  const double factor = r * Sun * rB;
  const double estar = U[3] * ri + (SM - un) * (SM + p * rA);
  out[0] = F0 + S * (factor - U[0]);
  out[1] = F1 + S * (factor * ustar - U[1]);
  out[2] = F2 + S * (factor * vstar - U[2]);
  out[3] = F3 + S * (factor * estar - U[3]);
}

template <int FLUX>
FRG_DEV void iflux2(double gamma, double g1, const double uL[4], const double uR[4], double nx,
                    double ny, double out[4], bool unit = false) {
  if (FLUX == FRG_FLUX_HLLC)
    hllc2(gamma, g1, uL, uR, nx, ny, out, unit);
  else
    rusanov2(gamma, g1, uL, uR, nx, ny, out);
}

// The normal fluxes above for the unit normals (1, 0) (X = true) and (0, 1)
// of the faces of an affine mesh: the same formulas with the zero normal
// component dropped (for finite states the general forms give these values:
// every term multiplied by the zero component vanishes and the one
// multiplied by 1 is unchanged), written in the rotated frame
// (n = normal velocity index, t = tangential).
template <bool X>
FRG_DEV void rusanov2_axis(double gamma, double g1, const double uL[4], const double uR[4], double out[4]) {
  constexpr int n = X ? 1 : 2, t = X ? 2 : 1;
  const double rL = jfloor(uL[0], kEps), riL = frcp(rL);
  const double uLv = uL[1] * riL, vLv = uL[2] * riL;
  const double pL = g1 * (uL[3] - 0.5 * rL * (uLv * uLv + vLv * vLv));
  const double rR = jfloor(uR[0], kEps), riR = frcp(rR);
  const double uRv = uR[1] * riR, vRv = uR[2] * riR;
  const double pR = g1 * (uR[3] - 0.5 * rR * (uRv * uRv + vRv * vRv));
  const double unL = X ? uLv : vLv, unR = X ? uRv : vRv;
  double fL[4], fR[4];
  fL[0] = uL[n];
  fL[n] = uL[n] * unL + pL;
  fL[t] = uL[t] * unL;
  fL[3] = (uL[3] + pL) * unL;
  fR[0] = uR[n];
  fR[n] = uR[n] * unR + pR;
  fR[t] = uR[t] * unR;
  fR[3] = (uR[3] + pR) * unR;
  const double cL = fsqrt(gamma * jfloor(pL, kEps) * riL);
  const double cR = fsqrt(gamma * jfloor(pR, kEps) * riR);
  const double lam = jmax(fabs(unL) + cL, fabs(unR) + cR);
  const double hl = 0.5 * lam;
#pragma unroll
  for (int c = 0; c < 4; ++c) out[c] = 0.5 * (fL[c] + fR[c]) - hl * (uR[c] - uL[c]);
}

template <bool X>
FRG_DEV void hllc2_axis(double gamma, double g1, const double uL[4], const double uR[4], double out[4]) {
  constexpr int n = X ? 1 : 2, t = X ? 2 : 1;
  const double rL = jfloor(uL[0], kEps), riL = frcp(rL);
  const double rR = jfloor(uR[0], kEps), riR = frcp(rR);
  const double uLv = uL[1] * riL, vLv = uL[2] * riL;
  const double uRv = uR[1] * riR, vRv = uR[2] * riR;
  const double pLu = g1 * (uL[3] - 0.5 * rL * (uLv * uLv + vLv * vLv));
  const double pRu = g1 * (uR[3] - 0.5 * rR * (uRv * uRv + vRv * vRv));
  const double pL = jfloor(pLu, kEps), pR = jfloor(pRu, kEps);
  const double unL = X ? uLv : vLv, unR = X ? uRv : vRv;
  const double cL = fsqrt(gamma * pL * riL), cR = fsqrt(gamma * pR * riR);
  const double SL = jmin(unL - cL, unR - cR);
  const double SR = jmax(unL + cL, unR + cR);
  const double num = pR - pL + rL * unL * (SL - unL) - rR * unR * (SR - unR);
  const double den = rL * (SL - unL) - rR * (SR - unR);
  const double SM = fabs(den) < kEps ? 0.5 * (unL + unR) : num * frcp(den);
  if (0.0 <= SL) {
    out[0] = uL[n];
    out[n] = uL[n] * unL + pLu;
    out[t] = uL[t] * unL;
    out[3] = (uL[3] + pLu) * unL;
    return;
  }
  if (0.0 >= SR) {
    out[0] = uR[n];
    out[n] = uR[n] * unR + pRu;
    out[t] = uR[t] * unR;
    out[3] = (uR[3] + pRu) * unR;
    return;
  }
  const bool left = (SL <= 0.0) && (0.0 <= SM);
  const double* U = left ? uL : uR;
  const double r = left ? rL : rR, ri = left ? riL : riR;
  const double un = left ? unL : unR;
  const double p = left ? pL : pR, pu = left ? pLu : pRu;
  const double S = left ? SL : SR;
  double F[4], ust[4];
  F[0] = U[n];
  F[n] = U[n] * un + pu;
  F[t] = U[t] * un;
  F[3] = (U[3] + pu) * un;
  ust[n] = SM;                // normal velocity of the star state
  ust[t] = U[t] * ri;         // tangential velocity, unchanged
  const double Sun = S - un;
  const double rB = frcp(S - SM), rA = frcp(r * Sun);
  const double factor = r * Sun * rB;
  const double estar = U[3] * ri + (SM - un) * (SM + p * rA);
  out[0] = F[0] + S * (factor - U[0]);
  out[n] = F[n] + S * (factor * ust[n] - U[n]);
  out[t] = F[t] + S * (factor * ust[t] - U[t]);
  out[3] = F[3] + S * (factor * estar - U[3]);
}

template <int FLUX, bool X>
FRG_DEV void iflux2_axis(double gamma, double g1, const double uL[4], const double uR[4], double out[4]) {
  if (FLUX == FRG_FLUX_HLLC)
    hllc2_axis<X>(gamma, g1, uL, uR, out);
  else
    rusanov2_axis<X>(gamma, g1, uL, uR, out);
}

// reflect_conserved (2D), BoundaryConditions.jl:43-60
FRG_DEV void reflect2(const double U[4], double nx, double ny, double out[4]) {
  const double r = jfloor(U[0], kEps), ri = 1.0 / r;
  const double u = U[1] * ri, v = U[2] * ri;
  const double un = u * nx + v * ny;
  out[0] = r;
  out[1] = r * (u - 2.0 * un * nx);
  out[2] = r * (v - 2.0 * un * ny);
  out[3] = U[3];
}

// exterior_state, BoundaryConditions.jl:67-134 (+ x-split GhostStateBC)
template <int NEQ>
FRG_DEV void exterior(const BCDev& bc, const double* ui, double nx, double ny, double x, double t,
                      double* ug);

template <>
FRG_DEV void exterior<4>(const BCDev& bc, const double* ui, double nx, double ny, double x, double t,
                         double* ug) {
  switch (bc.kind) {
    case FRG_BC_REFLECTING:
      reflect2(ui, nx, ny, ug);
      return;
    case FRG_BC_DIRICHLET:
#pragma unroll
      for (int c = 0; c < 4; ++c) ug[c] = bc.st[c];
      return;
    case FRG_BC_XSPLIT: {
      const double xs = bc.x0 + (bc.s0 + bc.s1 * t) / bc.sdiv;
      if (x < xs) {
#pragma unroll
        for (int c = 0; c < 4; ++c) ug[c] = bc.st[c];
      } else if (bc.mode == 0) {
        reflect2(ui, nx, ny, ug);
      } else {
#pragma unroll
        for (int c = 0; c < 4; ++c) ug[c] = bc.stb[c];
      }
      return;
    }
    default:  // transmissive
#pragma unroll
      for (int c = 0; c < 4; ++c) ug[c] = ui[c];
  }
}

// ---------------------------------------------------------------- 1D Euler

// physical_flux!, Euler.jl:88-99 (velocity from the unfloored density)
FRG_DEV void flux1(double g1, const double U[3], double F[3]) {
  const double rs = jmax(U[0], kEps);
  const double us = U[1] / rs;
  const double p = g1 * (U[2] - 0.5 * rs * us * us);
  const double u = U[1] / U[0];
  F[0] = U[1];
  F[1] = U[1] * u + p;
  F[2] = (U[2] + p) * u;
}

// |u| + c, Euler.jl:107-124 / element_max_wavespeed (PerssonAV.jl:138-155)
FRG_DEV double wave_speed1(double gamma, double g1, const double U[3]) {
  const double r = jmax(U[0], kEps), ri = 1.0 / r;
  const double u = U[1] * ri;
  const double p = jmax(g1 * (U[2] - 0.5 * r * u * u), kEps);
  return fabs(u) + sqrt(gamma * p * ri);
}

// rusanov_flux, Rusanov.jl:10-25 with max_wave_speed Euler.jl:107-113
// alpha scales the dissipation (a numerical_flux_method override); alpha = 1
// is the reference's flux exactly.
FRG_DEV void rusanov1(double gamma, double g1, const double uL[3], const double uR[3], double out[3],
                      double alpha = 1.0) {
  double fL[3], fR[3];
  flux1(g1, uL, fL);
  flux1(g1, uR, fR);
  const double lam = alpha * jmax(wave_speed1(gamma, g1, uL), wave_speed1(gamma, g1, uR));
  const double hl = 0.5 * lam;
#pragma unroll
  for (int c = 0; c < 3; ++c) out[c] = 0.5 * (fL[c] + fR[c]) - hl * (uR[c] - uL[c]);
}

// hllc_flux, HLLC.jl:9-69
FRG_DEV void hllc1(double gamma, double g1, const double uL[3], const double uR[3], double out[3]) {
  const double rL = jmax(uL[0], kEps), rR = jmax(uR[0], kEps);
  const double riL = 1.0 / rL, riR = 1.0 / rR;
  const double vL = uL[1] * riL, vR = uR[1] * riR;
  const double pL = jmax(g1 * (uL[2] - 0.5 * rL * vL * vL), kEps);
  const double pR = jmax(g1 * (uR[2] - 0.5 * rR * vR * vR), kEps);
  const double cL = sqrt(gamma * pL * riL), cR = sqrt(gamma * pR * riR);
  const double SL = jmin(vL - cL, vR - cR);
  const double SR = jmax(vL + cL, vR + cR);
  const double num = pR - pL + rL * vL * (SL - vL) - rR * vR * (SR - vR);
  const double den = rL * (SL - vL) - rR * (SR - vR);
  const double SM = fabs(den) < kEps ? 0.5 * (vL + vR) : num / den;
  double FL[3], FR[3];
  if (0.0 <= SL) {
    flux1(g1, uL, out);
    return;
  }
  if (0.0 >= SR) {
    flux1(g1, uR, out);
    return;
  }
  const bool left = (SL <= 0.0) && (0.0 <= SM);
  const double* U = left ? uL : uR;
  flux1(g1, U, FL);
  (void)FR;
  const double r = left ? rL : rR, ri = left ? riL : riR;
  const double v = left ? vL : vR, p = left ? pL : pR, S = left ? SL : SR;
  const double Sv = S - v;
  const double factor = r * Sv / (S - SM);
  const double eint = U[2] * ri + (SM - v) * (SM + p / (r * Sv));
  out[0] = FL[0] + S * (factor - U[0]);
  out[1] = FL[1] + S * (factor * SM - U[1]);
  out[2] = FL[2] + S * (factor * eint - U[2]);
}

template <int FLUX>
FRG_DEV void iflux1(double gamma, double g1, const double uL[3], const double uR[3], double out[3],
                    double alpha = 1.0) {
  if (FLUX == FRG_FLUX_HLLC)
    hllc1(gamma, g1, uL, uR, out);
  else
    rusanov1(gamma, g1, uL, uR, out, alpha);
}

// 1D exterior state for the domain ends (Residual.jl:63-112): transmissive
// or Dirichlet; reflecting uses reflect_conserved with n = -1 / +1.
FRG_DEV void exterior1(const BCDev& bc, const double* ui, double nx, double* ug) {
  if (bc.kind == FRG_BC_DIRICHLET) {
#pragma unroll
    for (int c = 0; c < 3; ++c) ug[c] = bc.st[c];
  } else if (bc.kind == FRG_BC_REFLECTING) {
    const double r = jmax(ui[0], kEps);
    const double u = ui[1] / r;
    const double un = u * nx;
    ug[0] = r;
    ug[1] = r * (u - 2.0 * un * nx);
    ug[2] = ui[2];
  } else {
#pragma unroll
    for (int c = 0; c < 3; ++c) ug[c] = ui[c];
  }
}

// Persson logistic indicator, SharedAV.jl:9-21
FRG_DEV double persson_sigma(double e_high, double e_tot, double s0, double kappa, double ef) {
  // the quotients by frcp: one warp finishes a tile's elements here, so its
  // latency is the tile's tail
  const double se = log10(e_high * frcp(e_tot) + ef);
  return frcp(1.0 + exp(-kappa * (se - s0)));
}

// BR0 interior penalty and average, SharedAV.jl:29-42
FRG_DEV double br0_tau(double em, double ep, double hm, double hp, int p) {
  const double eb = 0.5 * (em + ep);
  const double hb = 0.5 * (hm + hp);
  return 2.0 * eb * (double)(p + 1) * frcp(jmax(hb, kEps));
}

// smallest root in [0, 1] of a t^2 + b t + c with c > 0 >= a + b + c (the
// pressure quadratic of the Zhang-Shu scaling)
FRG_DEV double root01(double a, double b, double c) {
  if (fabs(a) < 1e-300) return b != 0.0 ? fmin(fmax(-c / b, 0.0), 1.0) : 0.0;
  const double disc = fmax(b * b - 4.0 * a * c, 0.0);
  const double q = -0.5 * (b + copysign(sqrt(disc), b));
  double r1 = q / a, r2 = q != 0.0 ? c / q : 2.0;
  double t = 1.0;
  if (r1 >= 0.0 && r1 <= 1.0) t = fmin(t, r1);
  if (r2 >= 0.0 && r2 <= 1.0) t = fmin(t, r2);
  return t;
}

// extrapolate_interface override of a 1D element (Interfaces.jl:49-71 is the
// default, "Override for hybrid reconstruction"): given the element mean m
// and its Lagrange traces tl (xi = -1) and tr (xi = +1) of (rho, rho u, E),
// kind kHookTraceMean pulls both toward the mean, t = m + p0 (t - m);
// kind kHookTracePositivity applies the Zhang-Shu scaling to the two traces
// (density >= p0 first, then pressure >= p1 by the pressure quadratic's root
// along m + theta (t - m)), and leaves an element whose mean is not
// admissible as it is.
FRG_DEV void trace_override1(int kind, double p0, double p1, double g1, const double* m, double* tl, double* tr) {
  if (kind == kHookTraceMean) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      tl[c] = m[c] + p0 * (tl[c] - m[c]);
      tr[c] = m[c] + p0 * (tr[c] - m[c]);
    }
    return;
  }
  if (kind != kHookTracePositivity) return;
  const double er = p0, ep = p1;
  const double pbar = g1 * (m[2] - 0.5 * m[1] * m[1] / m[0]);
  if (!(m[0] > er) || !(pbar > ep)) return;
  const double rmin = fmin(tl[0], tr[0]);
  if (rmin < er) {
    const double th = (m[0] - er) / (m[0] - rmin);
    tl[0] = m[0] + th * (tl[0] - m[0]);
    tr[0] = m[0] + th * (tr[0] - m[0]);
  }
  double theta = 1.0;
#pragma unroll
  for (int side = 0; side < 2; ++side) {
    const double* U = side == 0 ? tl : tr;
    const double pk = g1 * (U[2] - 0.5 * U[1] * U[1] / U[0]);
    if (pk >= ep) continue;
    const double d0 = U[0] - m[0], d1 = U[1] - m[1], d2 = U[2] - m[2];
    const double a = g1 * (d2 * d0 - 0.5 * d1 * d1);
    const double b = g1 * (m[2] * d0 + m[0] * d2 - m[1] * d1) - ep * d0;
    const double cc = m[0] * (pbar - ep);
    theta = fmin(theta, root01(a, b, cc));
  }
  if (theta < 1.0) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      tl[c] = m[c] + theta * (tl[c] - m[c]);
      tr[c] = m[c] + theta * (tr[c] - m[c]);
    }
  }
}

// atomic max of a non-negative double via its bit pattern (NaN sorts high)
FRG_DEV void atomic_max_nonneg(unsigned long long* addr, double v) {
  atomicMax(addr, (unsigned long long)__double_as_longlong(v));
}

}  // namespace frg

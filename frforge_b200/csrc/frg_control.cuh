// Device-side time-loop control shared by the single-solve runtime and the
// batched engine: the top and the bottom of the ssp_rk3!/ssp_rk2! loop body.
#pragma once

#include "frg_device.cuh"
#include "frg_internal.h"

namespace frg {

// Top of the ssp_rk3!/ssp_rk2! loop body (SSP_RK3.jl:185-189): loop test,
// dt from the CFL wave speed of the current state, last-step clipping.
__device__ __forceinline__ void step_begin_device(DevScalars* sc) {
  sc->stepped_ok = 0;
  if (sc->status != kRunning) {
    sc->active = 0;
    return;
  }
  if (!(sc->t < sc->t_final - 10 * kEps)) {
    sc->status = kFinished;
    sc->active = 0;
    return;
  }
  double dt;
  if (sc->fixed_dt > 0.0) {
    dt = sc->fixed_dt;
  } else {
    double lam = __longlong_as_double((long long)sc->lam_bits);
    lam = jmax(jmax(lam, kEps), kEps);
    dt = sc->cfl * sc->hmin / ((double)sc->two_p1 * lam);
  }
  if (sc->t + dt > sc->t_final) dt = sc->t_final - sc->t;
  sc->dt = dt;
  sc->t0 = sc->t;
  sc->flags = 0u;
  sc->lam_bits = 0ull;
  sc->active = 1;
}

// Bottom of the loop body: step count, status and the time of the state.
__device__ __forceinline__ void step_end_device(DevScalars* sc, int nstages) {
  if (!sc->active) return;
  sc->active = 0;
  sc->n_steps += 1;
  const unsigned f = sc->flags;
  int div_stage = 0;
  for (int s = 1; s <= nstages; ++s)
    if (f & (1u << (2 * (s - 1)))) {
      div_stage = s;
      break;
    }
  if (!div_stage && (f & (2u << (2 * (nstages - 1))))) div_stage = 4;
  const double t0 = sc->t0, dt = sc->dt;
  sc->residual_evals += div_stage && div_stage <= nstages ? div_stage : nstages;
  if (div_stage) {
    sc->status = FRG_DIVERGED;
    sc->diverged_stage = div_stage;
    // state.t at the moment ssp_rk3_step! returned :diverged
    if (div_stage == 1)
      sc->t = t0;
    else if (div_stage == 2 || div_stage == 4)
      sc->t = t0 + dt;
    else
      sc->t = t0 + dt / 2.0;
    return;
  }
  sc->t = t0 + dt;
  sc->stepped_ok = 1;
  if (sc->n_steps >= sc->max_steps) sc->status = FRG_MAX_STEPS;
}

}  // namespace frg

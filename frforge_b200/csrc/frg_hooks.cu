// Device hook registry: compiled implementations of capturing-method hooks
// that a method selects by name, so that a method overriding a hook can run
// on the GPU instead of being rejected with FRG_ERR_UNSUPPORTED_HOOK.  The
// reference's hooks are Julia functions dispatched on the method type
// (src/capturing/Interfaces.jl:43-92); a solve here carries at most one
// implementation per hook slot, chosen with frg_solve_set_hook.
//
// Registered implementations:
//   numerical_flux_method "flux_rusanov"  (1D) the Rusanov flux with its
//       dissipation scaled by alpha: 1/2 (F(uL) + F(uR)) - 1/2 alpha lambda
//       (uR - uL), lambda the larger |u| + c (Rusanov.jl:10-25 at alpha = 1);
//       params: alpha (default 1).
//   numerical_flux_method "flux_hllc"  (1D) the HLLC flux (HLLC.jl:9-69)
//       whatever the scheme's flux.
//       Both replace the interface flux of every 1D interface, boundary
//       interfaces included, as the reference's _resolve_flux does
//       (src/fr/Residual.jl:9-15, :36-46); the 2D residual never consults
//       the override (Residual2D.jl calls interface_flux_n! directly), so on a
//       2D solve the slot is accepted and has no effect, as there.
//   extrapolate_interface "traces_toward_mean"  (1D) the traces of every
//       element's numerical fluxes pulled toward its mean, ubar + theta
//       (ell . u - ubar) (theta = 1: the Lagrange traces of the default
//       extrapolate_interface!, Interfaces.jl:49-71; theta = 0: first-order
//       traces); params: theta in [0, 1] (default 1).
//   extrapolate_interface "traces_positivity_zhang_shu"  (1D) the
//       Zhang-Shu scaling (below) applied to an element's two traces; params:
//       eps_rho, eps_p (defaults 1e-13).
//       Both feed only compute_interface_fluxes! (Residual.jl:175-184); the
//       BR0 dissipation keeps the Lagrange traces, as apply_dissipation_br0!
//       computes its own (PerssonAV.jl:249-300).  The 2D residual never calls
//       extrapolate_interface!, so on a 2D solve the slot has no effect.
//   preprocess_state "preprocess_positivity_zhang_shu"  the same scaling
//       (below) applied to the work state u_work that the residual is
//       evaluated on (preprocess_state!, Interfaces.jl:41-46; called first in
//       residual!, Residual.jl:172, Residual2D.jl:148): before every stage a
//       kernel writes u_work = the limited copy of the stage state, the
//       element viscosity is recomputed from it (sense! and the dissipation
//       take u_work) and the stage kernel evaluates the residual on it, while
//       the SSP-RK combination, compute_dt and post_step! keep the stage
//       state itself.  params: eps_rho, eps_p (defaults 1e-13).  Single
//       solves only: the batched engine refuses it.
//   post_step "positivity_zhang_shu"  the positivity-preserving scaling of
//       Zhang & Shu (J. Comput. Phys. 229 (2010) 8918-8934): per element,
//       the density at every solution point is pulled toward the element
//       mean until it is >= eps_rho, then all components are pulled toward
//       the mean by the largest theta in [0, 1] that keeps the pressure
//       >= eps_p at every point (the exact root of the pressure quadratic
//       along u_mean + t (u_k - u_mean)).  Element means use the quadrature
//       weights w_i w_j |J|, so the element integrals -- and the discrete
//       mass -- are unchanged.  Elements whose mean is not admissible are
//       left as they are.  params: eps_rho, eps_p (defaults 1e-13).
//
// Time-loop placement (ssp_rk3_step!, SSP_RK3.jl:135-164): post_step! runs
// after every step that did not diverge, before the next compute_dt; here
// the hook kernel runs after the step's end kernel when the step completed,
// and a prime pass recomputes the element viscosity and the CFL wave speed
// of the limited state.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "frg_device.cuh"
#include "frg_runtime.h"

namespace frg {
namespace {

struct HookEntry {
  const char* name;
  int slot;
  int id;
  int nparams;
};
const HookEntry kHooks[] = {
    {"positivity_zhang_shu", FRG_HOOK_POST_STEP, kHookPositivity, 2},
    {"flux_rusanov", FRG_HOOK_NUMERICAL_FLUX, kHookFluxRusanov, 1},
    {"flux_hllc", FRG_HOOK_NUMERICAL_FLUX, kHookFluxHLLC, 0},
    {"preprocess_positivity_zhang_shu", FRG_HOOK_PREPROCESS_STATE, kHookPrePositivity, 2},
    {"traces_toward_mean", FRG_HOOK_EXTRAPOLATE_INTERFACE, kHookTraceMean, 1},
    {"traces_positivity_zhang_shu", FRG_HOOK_EXTRAPOLATE_INTERFACE, kHookTracePositivity, 2},
};
constexpr int kNumHooks = (int)(sizeof(kHooks) / sizeof(kHooks[0]));

struct Weights {
  double w[kMaxNp];
};

template <int NEQ>
__device__ void zs_element(double* u, size_t n, size_t base, int npts, const double* ww, double g1, double er,
                           double ep) {
  double mean[NEQ], wsum = 0.0;
  for (int c = 0; c < NEQ; ++c) mean[c] = 0.0;
  for (int k = 0; k < npts; ++k) {
    wsum += ww[k];
    for (int c = 0; c < NEQ; ++c) mean[c] += ww[k] * u[c * n + base + k];
  }
  for (int c = 0; c < NEQ; ++c) mean[c] /= wsum;
  const double mm2 = NEQ == 4 ? mean[1] * mean[1] + mean[2] * mean[2] : mean[1] * mean[1];
  const double pbar = g1 * (mean[NEQ - 1] - 0.5 * mm2 / mean[0]);
  if (!(mean[0] > er) || !(pbar > ep)) return;  // mean not admissible
  // density
  double rmin = mean[0];
  for (int k = 0; k < npts; ++k) rmin = fmin(rmin, u[base + k]);
  if (rmin < er) {
    const double th = (mean[0] - er) / (mean[0] - rmin);
    for (int k = 0; k < npts; ++k) u[base + k] = mean[0] + th * (u[base + k] - mean[0]);
  }
  // pressure
  double theta = 1.0;
  for (int k = 0; k < npts; ++k) {
    double U[NEQ];
    for (int c = 0; c < NEQ; ++c) U[c] = u[c * n + base + k];
    const double m2 = NEQ == 4 ? U[1] * U[1] + U[2] * U[2] : U[1] * U[1];
    const double pk = g1 * (U[NEQ - 1] - 0.5 * m2 / U[0]);
    if (pk >= ep) continue;
    double d[NEQ];
    for (int c = 0; c < NEQ; ++c) d[c] = U[c] - mean[c];
    const double dm2 = NEQ == 4 ? d[1] * d[1] + d[2] * d[2] : d[1] * d[1];
    const double mdm = NEQ == 4 ? mean[1] * d[1] + mean[2] * d[2] : mean[1] * d[1];
    // rho(t) (p(t) - eps_p) = a t^2 + b t + c along mean + t d
    const double a = g1 * (d[NEQ - 1] * d[0] - 0.5 * dm2);
    const double b = g1 * (mean[NEQ - 1] * d[0] + mean[0] * d[NEQ - 1] - mdm) - ep * d[0];
    const double cc = mean[0] * (pbar - ep);
    theta = fmin(theta, root01(a, b, cc));
  }
  if (theta < 1.0)
    for (int k = 0; k < npts; ++k)
      for (int c = 0; c < NEQ; ++c) {
        double& v = u[c * n + base + k];
        v = mean[c] + theta * (v - mean[c]);
      }
}

// Zhang-Shu scaling of 2D element e (quadrature weights w_i w_j |J|)
__device__ void zs_element_2d(double* u, const Mesh2Dev& M, const Weights& W, int np, double g1, double er,
                              double ep, int e) {
  if (M.solid && M.solid[e]) return;
  const int np2 = np * np;
  const size_t n = (size_t)M.nel * np2, base = (size_t)e * np2;
  double ww[kMaxNp * kMaxNp];
  const int gx = e % M.nx, gy = e / M.nx;
  for (int k = 0; k < np2; ++k) {
    const double absJ = M.curved ? fabs(1.0 / M.m_rJ[base + k]) : fabs(M.Jx[gx] * M.Jy[gy]);
    ww[k] = W.w[k % np] * W.w[k / np] * absJ;
  }
  zs_element<4>(u, n, base, np2, ww, g1, er, ep);
}

__device__ void zs_element_1d(double* u, const Mesh1Dev& M, const Weights& W, int np, double g1, double er,
                              double ep, int e) {
  const size_t n = (size_t)M.nel * np, base = (size_t)e * np;
  double ww[kMaxNp];
  for (int k = 0; k < np; ++k) ww[k] = W.w[k] * M.J[e];
  zs_element<3>(u, n, base, np, ww, g1, er, ep);
}

// one count per launch that passed its gate (the HookProbeMethod counters of
// the reference's test/test_capturing.jl:5-41, kept on the device so graph
// replays count too)
__device__ __forceinline__ void count_call(DevScalars* sc, int slot) {
  if (sc && blockIdx.x == 0 && threadIdx.x == 0) sc->hook_calls[slot] += 1;
}

// one thread per element; `force` ignores the step's completion flag
__global__ void zs_limiter_2d(double* u, const Mesh2Dev M, Weights W, int np, double g1, double er, double ep,
                              DevScalars* sc, int force) {
  if (!force && !(sc && sc->stepped_ok)) return;
  if (!force && blockIdx.x == 0 && threadIdx.x == 0) sc->lam_bits = 0ull;  // the prime pass recomputes it
  count_call(sc, FRG_HOOK_POST_STEP);
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= M.nel) return;
  zs_element_2d(u, M, W, np, g1, er, ep, e);
}

__global__ void zs_limiter_1d(double* u, const Mesh1Dev M, Weights W, int np, double g1, double er, double ep,
                              DevScalars* sc, int force) {
  if (!force && !(sc && sc->stepped_ok)) return;
  if (!force && blockIdx.x == 0 && threadIdx.x == 0) sc->lam_bits = 0ull;
  count_call(sc, FRG_HOOK_POST_STEP);
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= M.nel) return;
  zs_element_1d(u, M, W, np, g1, er, ep, e);
}

// preprocess_state: u_work = the limited copy of the stage state, one thread
// per element; gated like the stage it precedes (skipped when the step is
// inactive or an earlier stage flagged a non-finite value: stage_mask as in
// stage_control), unless `gated` is 0.
__global__ void zs_preprocess_2d(const double* __restrict__ us, double* __restrict__ uw, const Mesh2Dev M,
                                 Weights W, int np, double g1, double er, double ep, DevScalars* sc,
                                 unsigned stage_mask, int gated) {
  if (gated && (!sc->active || (sc->flags & stage_mask))) return;
  count_call(sc, FRG_HOOK_PREPROCESS_STATE);
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= M.nel) return;
  const int np2 = np * np;
  const size_t n = (size_t)M.nel * np2, base = (size_t)e * np2;
  for (int c = 0; c < 4; ++c)
    for (int k = 0; k < np2; ++k) uw[c * n + base + k] = us[c * n + base + k];
  zs_element_2d(uw, M, W, np, g1, er, ep, e);
}

__global__ void zs_preprocess_1d(const double* __restrict__ us, double* __restrict__ uw, const Mesh1Dev M,
                                 Weights W, int np, double g1, double er, double ep, DevScalars* sc,
                                 unsigned stage_mask, int gated) {
  if (gated && (!sc->active || (sc->flags & stage_mask))) return;
  count_call(sc, FRG_HOOK_PREPROCESS_STATE);
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= M.nel) return;
  const size_t n = (size_t)M.nel * np, base = (size_t)e * np;
  for (int c = 0; c < 3; ++c)
    for (int k = 0; k < np; ++k) uw[c * n + base + k] = us[c * n + base + k];
  zs_element_1d(uw, M, W, np, g1, er, ep, e);
}

// Batched groups: one CTA per TX x TY tile of the group's tile list, one
// thread per element of the tile; instances whose step did not complete, or
// that carry no hook, are left alone.  The CTA of an instance's first tile
// clears its CFL wave speed, which the group's prime pass recomputes.
__global__ void zs_limiter_batch(const BatchInst* __restrict__ insts, const BatchTile* __restrict__ tiles,
                                 Weights W, int np, int tx, int ty) {
  const BatchTile t = tiles[blockIdx.x];
  const BatchInst& I = insts[t.inst];
  if (I.hook != kHookPositivity || !(I.sc && I.sc->stepped_ok)) return;
  if (t.x0 == 0 && t.y0 == 0 && threadIdx.x == 0) {
    I.sc->lam_bits = 0ull;
    I.sc->hook_calls[FRG_HOOK_POST_STEP] += 1;
  }
  const double er = I.hook_params[0], ep = I.hook_params[1];
  for (int k = threadIdx.x; k < tx * ty; k += blockDim.x) {
    const int x = t.x0 + k % tx, y = t.y0 + k / tx;
    if (I.dim == 2) {
      if (x < I.M2.nx && y < I.M2.ny) zs_element_2d(I.U[0], I.M2, W, np, I.P.g1, er, ep, y * I.M2.nx + x);
    } else if (x < I.M1.nel) {
      zs_element_1d(I.U[0], I.M1, W, np, I.P.g1, er, ep, x);
    }
  }
}

Weights weights_of(const HostOps& ops) {
  Weights W;
  std::memset(&W, 0, sizeof(W));
  for (int i = 0; i < ops.np; ++i) W.w[i] = ops.w[i];
  return W;
}

}  // namespace

// Enqueue the post-step hook of a solve on stream `st` (no-op without one):
// the hook kernel, then the prime pass of the limited state.  force: run even
// if no step just completed.
int enqueue_post_step_on(frg_solve* s, bool force, cudaStream_t st) {
  if (s->post_step_id != kHookPositivity) return FRG_OK;
  const Weights W = weights_of(s->ops);
  const int threads = 128, blocks = (s->nel + threads - 1) / threads;
  const double er = s->post_step_params[0], ep = s->post_step_params[1];
  if (s->dim == 2)
    zs_limiter_2d<<<blocks, threads, 0, st>>>(s->U[0], s->L2.mesh, W, s->np, s->L2.phys.g1, er, ep, s->sc,
                                               force ? 1 : 0);
  else
    zs_limiter_1d<<<blocks, threads, 0, st>>>(s->U[0], s->L1.mesh, W, s->np, s->L1.phys.g1, er, ep, s->sc,
                                               force ? 1 : 0);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return rt::cuda_err(s->ctx, e, "post-step hook");
  return rt::prime_on(s, 0, true, st);
}
int enqueue_post_step(frg_solve* s, bool force) { return enqueue_post_step_on(s, force, s->ctx->stream); }

// Enqueue the preprocess_state hook of a solve for the residual of stage
// `stage` (0: an ungated evaluation outside the time loop) on the state `us`:
// the work-state kernel, then the element viscosity of the work state into
// `eps` (the eps the stage kernel reads).  No-op without a hook.
int enqueue_preprocess(frg_solve* s, const double* us, double* eps, int stage) {
  if (s->pre_id != kHookPrePositivity) return FRG_OK;
  cudaStream_t st = s->ctx->stream;
  const Weights W = weights_of(s->ops);
  const int threads = 128, blocks = (s->nel + threads - 1) / threads;
  const double er = s->pre_params[0], ep = s->pre_params[1];
  const unsigned mask = stage <= 1 ? 0u : (stage == 2 ? 1u : 5u);
  const int gated = stage > 0 ? 1 : 0;
  if (s->dim == 2)
    zs_preprocess_2d<<<blocks, threads, 0, st>>>(us, s->Uw, s->L2.mesh, W, s->np, s->L2.phys.g1, er, ep, s->sc,
                                                  mask, gated);
  else
    zs_preprocess_1d<<<blocks, threads, 0, st>>>(us, s->Uw, s->L1.mesh, W, s->np, s->L1.phys.g1, er, ep, s->sc,
                                                  mask, gated);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return rt::cuda_err(s->ctx, e, "preprocess hook");
  if (s->method != FRG_METHOD_PERSSON) return FRG_OK;
  StageBufs b{};
  b.us = s->Uw;
  b.eps_out = eps;
  b.mode = kModePrime;
  b.sc = s->sc;
  b.use_sc = gated;
  b.stage = stage > 0 ? stage : 1;
  return rt::launch(s, b);
}

int enqueue_batch_post_step(const HostOps& ops, int tx, int ty, const BatchInst* insts, const BatchTile* tiles,
                            int ntiles, cudaStream_t st) {
  if (ntiles < 1) return (int)cudaSuccess;
  zs_limiter_batch<<<ntiles, 128, 0, st>>>(insts, tiles, weights_of(ops), ops.np, tx, ty);
  return (int)cudaGetLastError();
}

}  // namespace frg

using namespace frg;
using namespace frg::rt;

extern "C" {

int frg_hook_count(void) { return kNumHooks; }

int frg_hook_info(int i, const char** name, int* slot, int* id, int* nparams) {
  if (i < 0 || i >= kNumHooks) return FRG_ERR_INVALID_ARG;
  if (name) *name = kHooks[i].name;
  if (slot) *slot = kHooks[i].slot;
  if (id) *id = kHooks[i].id;
  if (nparams) *nparams = kHooks[i].nparams;
  return FRG_OK;
}

int frg_hook_lookup(const char* name, int* slot, int* id) {
  if (!name) return FRG_ERR_INVALID_ARG;
  for (int i = 0; i < kNumHooks; ++i)
    if (std::strcmp(name, kHooks[i].name) == 0) {
      if (slot) *slot = kHooks[i].slot;
      if (id) *id = kHooks[i].id;
      return FRG_OK;
    }
  return FRG_ERR_UNSUPPORTED_HOOK;
}

// numerical_flux_method slot: the 1D interface flux of the solve (the 2D
// residual ignores overrides, as the reference's does)
static int set_flux_hook(frg_solve* s, int id, const double* params, int nparams) {
  int found = -1;
  for (int i = 0; i < kNumHooks; ++i)
    if (kHooks[i].slot == FRG_HOOK_NUMERICAL_FLUX && kHooks[i].id == id) found = i;
  if (id != 0 && found < 0) return set_err(s->ctx, FRG_ERR_UNSUPPORTED_HOOK, "unknown hook implementation");
  if (id != 0 && (nparams < 0 || nparams > kHooks[found].nparams || (nparams > 0 && !params)))
    return set_err(s->ctx, FRG_ERR_INVALID_ARG, "hook parameters");
  double alpha = 1.0;
  if (id == kHookFluxRusanov && nparams > 0) alpha = params[0];
  if (!(alpha >= 0.0) || !std::isfinite(alpha)) return set_err(s->ctx, FRG_ERR_INVALID_ARG, "alpha must be >= 0");
  s->flux_hook_id = id;
  s->flux_hook_alpha = alpha;
  if (s->dim == 1) {
    s->L1.flux = id == kHookFluxRusanov ? FRG_FLUX_RUSANOV : (id == kHookFluxHLLC ? FRG_FLUX_HLLC : s->scheme_flux);
    s->L1.phys.flux_alpha = id == kHookFluxRusanov ? alpha : 1.0;
  }
  return FRG_OK;
}

// extrapolate_interface slot: the traces of the 1D numerical fluxes (the 2D
// residual never calls extrapolate_interface!, so a 2D solve ignores it)
static int set_trace_hook(frg_solve* s, int id, const double* params, int nparams) {
  if (id != 0 && id != kHookTraceMean && id != kHookTracePositivity)
    return set_err(s->ctx, FRG_ERR_UNSUPPORTED_HOOK, "unknown hook implementation");
  const int maxp = id == kHookTraceMean ? 1 : 2;
  if (id != 0 && (nparams < 0 || nparams > maxp || (nparams > 0 && !params)))
    return set_err(s->ctx, FRG_ERR_INVALID_ARG, "hook parameters");
  double p[2] = {id == kHookTraceMean ? 1.0 : 1e-13, 1e-13};
  for (int k = 0; k < nparams; ++k) p[k] = params[k];
  if (id == kHookTraceMean && !(p[0] >= 0.0 && p[0] <= 1.0))
    return set_err(s->ctx, FRG_ERR_INVALID_ARG, "theta must be in [0, 1]");
  if (id == kHookTracePositivity && (!(p[0] > 0.0) || !(p[1] > 0.0) || !std::isfinite(p[0]) || !std::isfinite(p[1])))
    return set_err(s->ctx, FRG_ERR_INVALID_ARG, "eps_rho, eps_p must be > 0");
  s->trace_id = id;
  s->trace_params[0] = id ? p[0] : 0.0;
  s->trace_params[1] = id ? p[1] : 0.0;
  if (s->dim == 1) {
    s->L1.phys.trace_hook = id;
    s->L1.phys.trace_p0 = s->trace_params[0];
    s->L1.phys.trace_p1 = s->trace_params[1];
  }
  return FRG_OK;
}

// preprocess_state slot: the work state's buffer is allocated on selection
static int set_pre_hook(frg_solve* s, int id, const double* params, int nparams) {
  if (id != 0 && id != kHookPrePositivity)
    return set_err(s->ctx, FRG_ERR_UNSUPPORTED_HOOK, "unknown hook implementation");
  if (id != 0 && (nparams < 0 || nparams > 2 || (nparams > 0 && !params)))
    return set_err(s->ctx, FRG_ERR_INVALID_ARG, "hook parameters");
  double p[2] = {1e-13, 1e-13};
  for (int k = 0; k < nparams; ++k) p[k] = params[k];
  if (id != 0 && (!(p[0] > 0.0) || !(p[1] > 0.0)))
    return set_err(s->ctx, FRG_ERR_INVALID_ARG, "eps_rho, eps_p must be > 0");
  if (id != 0 && !s->Uw) {
    cudaSetDevice(s->ctx->device);
    const int rc = alloc_doubles(s, &s->Uw, s->ndof);
    if (rc) return rc;
  }
  s->pre_id = id;
  s->pre_params[0] = p[0];
  s->pre_params[1] = p[1];
  return FRG_OK;
}

int frg_solve_set_hook(frg_solve* s, int slot, int id, const double* params, int nparams) {
  if (!s) return FRG_ERR_INVALID_ARG;
  if (slot == FRG_HOOK_PREPROCESS_STATE) {
    const int rc = set_pre_hook(s, id, params, nparams);
    if (rc) return rc;
    if (s->graph) {  // captured step graphs do not contain the hook
      cudaGraphExecDestroy(s->graph);
      s->graph = nullptr;
    }
    return FRG_OK;
  }
  if (slot == FRG_HOOK_EXTRAPOLATE_INTERFACE) {
    const int rc = set_trace_hook(s, id, params, nparams);
    if (rc) return rc;
    if (s->graph) {  // captured step graphs bake the kernel parameters in
      cudaGraphExecDestroy(s->graph);
      s->graph = nullptr;
    }
    return FRG_OK;
  }
  if (slot == FRG_HOOK_NUMERICAL_FLUX) {
    const int rc = set_flux_hook(s, id, params, nparams);
    if (rc) return rc;
    if (s->graph) {  // captured step graphs bake the flux kernels in
      cudaGraphExecDestroy(s->graph);
      s->graph = nullptr;
    }
    return FRG_OK;
  }
  if (slot != FRG_HOOK_POST_STEP) return set_err(s->ctx, FRG_ERR_UNSUPPORTED_HOOK, "unknown hook slot");
  if (id == 0) {
    s->post_step_id = 0;
  } else {
    int found = -1;
    for (int i = 0; i < kNumHooks; ++i)
      if (kHooks[i].slot == slot && kHooks[i].id == id) found = i;
    if (found < 0) return set_err(s->ctx, FRG_ERR_UNSUPPORTED_HOOK, "unknown hook implementation");
    if (nparams < 0 || nparams > kHooks[found].nparams || (nparams > 0 && !params))
      return set_err(s->ctx, FRG_ERR_INVALID_ARG, "hook parameters");
    double p[2] = {1e-13, 1e-13};
    for (int k = 0; k < nparams; ++k) p[k] = params[k];
    if (!(p[0] > 0.0) || !(p[1] > 0.0)) return set_err(s->ctx, FRG_ERR_INVALID_ARG, "eps_rho, eps_p must be > 0");
    s->post_step_id = id;
    s->post_step_params[0] = p[0];
    s->post_step_params[1] = p[1];
  }
  // captured step graphs do not contain the hook (or contain the old one)
  if (s->graph) {
    cudaGraphExecDestroy(s->graph);
    s->graph = nullptr;
  }
  return FRG_OK;
}

int frg_apply_post_step(frg_solve* s) {
  if (!s) return FRG_ERR_INVALID_ARG;
  if (!s->have_state) return set_err(s->ctx, FRG_ERR_STATE, "no state uploaded");
  cudaSetDevice(s->ctx->device);
  int rc = make_current_canonical(s);
  if (rc) return rc;
  if ((rc = enqueue_post_step(s, true))) return rc;
  return cuda_err(s->ctx, cudaStreamSynchronize(s->ctx->stream), "post-step hook");
}

int frg_solve_hook_calls(frg_solve* s, int64_t* counts, int n) {
  if (!s || !counts || n < 1 || n > 4) return FRG_ERR_INVALID_ARG;
  cudaSetDevice(s->ctx->device);
  long long c[4] = {0, 0, 0, 0};
  cudaError_t e = cudaMemcpyAsync(c, s->sc->hook_calls, sizeof(c), cudaMemcpyDeviceToHost, s->ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->ctx->stream);
  if (e != cudaSuccess) return cuda_err(s->ctx, e, "hook counters");
  for (int i = 0; i < n; ++i) counts[i] = c[i];
  // the flux and trace overrides run inline in every interface pass: no launch of their own to count
  if (n > FRG_HOOK_NUMERICAL_FLUX) counts[FRG_HOOK_NUMERICAL_FLUX] = -1;
  if (n > FRG_HOOK_EXTRAPOLATE_INTERFACE) counts[FRG_HOOK_EXTRAPOLATE_INTERFACE] = -1;
  return FRG_OK;
}

}  // extern "C"

// Runtime internals shared by the single-solve ABI (frforge_cuda.cu) and the
// batched / served engine (frg_batch.cu).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "frg_internal.h"

using frg::DevScalars;
using frg::HostOps;
using frg::Launch1D;
using frg::Launch2D;

struct frg_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
};

struct frg_solve {
  frg_ctx* ctx = nullptr;
  int dim = 2, np = 0, nel = 0, neq = 4, nx = 0, ny = 1;
  size_t ndof = 0;
  int time_scheme = FRG_TIME_SSP_RK3;
  int method = FRG_METHOD_NULL;
  HostOps ops;
  Launch2D L2{};
  Launch1D L1{};
  double* U[3] = {nullptr, nullptr, nullptr};
  double* E[3] = {nullptr, nullptr, nullptr};
  double* du = nullptr;
  double* sigma = nullptr;
  DevScalars* sc = nullptr;
  DevScalars* hsc = nullptr;  // pinned host mirror
  std::vector<void*> allocs;
  size_t bytes = 0;
  bool have_state = false;
  int cur = 0;  // buffer index of the current state
  double t = 0.0;
  cudaGraphExec_t graph = nullptr;
  int graph_steps = 0;
  bool graph_lambda = false;
  int64_t residual_evals = 0, steps = 0;
  double hmin = 0.0;
  int post_step_id = 0;  // device post-step hook (frg_hooks.cu), 0 = none
  double post_step_params[2] = {0.0, 0.0};
  int scheme_flux = 0;     // the scheme's flux (FRG_FLUX_*)
  int flux_hook_id = 0;    // numerical_flux_method override (frg_hooks.cu), 0 = none
  double flux_hook_alpha = 1.0;
  int trace_id = 0;        // extrapolate_interface hook (frg_hooks.cu), 0 = none
  double trace_params[2] = {0.0, 0.0};
  int pre_id = 0;          // preprocess_state hook (frg_hooks.cu), 0 = none
  double pre_params[2] = {0.0, 0.0};
  double* Uw = nullptr;    // the work state u_work of a preprocess_state hook
};


namespace frg {
namespace rt {
int set_err(frg_ctx* c, int code, const std::string& msg);
// a device buffer of n doubles owned by the solve (freed with it)
int alloc_doubles(frg_solve* s, double** p, size_t n);
// the descriptor checks of frg_solve_create (c may be null)
int validate_desc(frg_ctx* c, const frg_solve_desc* d);
int cuda_err(frg_ctx* c, cudaError_t e, const char* what);
int push_scalars(frg_solve* s);
int pull_scalars(frg_solve* s);
int launch(frg_solve* s, const StageBufs& b);
int prime(frg_solve* s, int buf, bool want_lambda);
int prime_on(frg_solve* s, int buf, bool want_lambda, cudaStream_t st);
int finish_run(frg_solve* s);
int make_current_canonical(frg_solve* s);
void init_run_scalars(frg_solve* s, double t_final, double cfl, double fixed_dt, int64_t max_steps);
StageBufs stage_bufs(const frg_solve* s, int stage, bool want_lambda);
}  // namespace rt
// post-step hook of a solve and the prime pass of its result (frg_hooks.cu),
// on the solve's stream or on `st`
int enqueue_post_step(frg_solve* s, bool force);
// preprocess_state hook of a solve for the residual of stage `stage` (0: an
// ungated evaluation) on state us: u_work into s->Uw and its element
// viscosity into eps (frg_hooks.cu); no-op without a hook
int enqueue_preprocess(frg_solve* s, const double* us, double* eps, int stage);
int enqueue_post_step_on(frg_solve* s, bool force, cudaStream_t st);
// post-step hook of the instances of a batched group whose step completed,
// one CTA per TX x TY tile of the group's tile list (frg_hooks.cu); the
// caller follows it with the group's prime pass
int enqueue_batch_post_step(const HostOps& ops, int tx, int ty, const BatchInst* insts, const BatchTile* tiles,
                            int ntiles, cudaStream_t st);
__global__ void step_begin_kernel(DevScalars* sc);
__global__ void step_end_kernel(DevScalars* sc, int nstages);
}  // namespace frg

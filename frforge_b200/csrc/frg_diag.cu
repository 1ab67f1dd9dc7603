// Device-side diagnostics of a solve's state: the scoring-harness
// reductions of the reference, computed where the state lives so that a
// served solve reports them without downloading the state.
//
//   discrete_mass(state, c)       SolutionState.jl:80-90, SolutionState2D.jl:85-97
//   l2_error(state, uexact, c)    SolutionState.jl:93-107, SolutionState2D.jl:98-111
//   positivity_ok(eq, state)      Euler.jl:62-77, Euler2D.jl:153-163
//   has_nonfinite(u)              Residual.jl:219-226 (as a count)
//   minimum / maximum of density  Cases2D_Riemann.jl:111-116
//
// Exact solutions available to l2_error on the device: the isentropic vortex
// (isentropic_vortex_primitives, Cases2D_Riemann.jl:163-186), the smooth 2D
// order-test wave (Cases2D_Smooth.jl:124-135), the 1D density wave
// (euler_density_wave_conserved, Cases.jl:404-414), or a reference state in
// device memory.
//
// One grid-stride pass over the solution points accumulates per-thread
// partials; every block reduces them in a fixed-order tree and a one-block
// kernel reduces the block partials in order, so results do not depend on
// scheduling.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "frg_device.cuh"
#include "frg_runtime.h"

namespace frg {
namespace {

constexpr int kDiagThreads = 256;
constexpr int kDiagMaxBlocks = 1184;  // 8 x 148 SMs

struct DiagPart {
  double mass[4];
  double rmin, rmax, pmin, l2;
  double nonfinite;  // count (exact in double up to 2^53)
  double posfail;    // count of points failing positivity
};

struct DiagTables {
  double w[kMaxNp], xi[kMaxNp];
};

__device__ __forceinline__ void part_init(DiagPart& p) {
  for (int c = 0; c < 4; ++c) p.mass[c] = 0.0;
  p.rmin = INFINITY;
  p.rmax = -INFINITY;
  p.pmin = INFINITY;
  p.l2 = 0.0;
  p.nonfinite = 0.0;
  p.posfail = 0.0;
}

__device__ __forceinline__ void part_merge(DiagPart& a, const DiagPart& b) {
  for (int c = 0; c < 4; ++c) a.mass[c] += b.mass[c];
  a.rmin = jmin(a.rmin, b.rmin);
  a.rmax = jmax(a.rmax, b.rmax);
  a.pmin = jmin(a.pmin, b.pmin);
  a.l2 += b.l2;
  a.nonfinite += b.nonfinite;
  a.posfail += b.posfail;
}

// fixed-order tree over the block; result in s[0]
__device__ void block_reduce(DiagPart* s, DiagPart mine) {
  const int t = threadIdx.x;
  s[t] = mine;
  __syncthreads();
  for (int h = kDiagThreads / 2; h > 0; h >>= 1) {
    if (t < h) {
      DiagPart a = s[t];
      part_merge(a, s[t + h]);
      s[t] = a;
    }
    __syncthreads();
  }
}

// exact solutions (conserved), gamma of the solve
__device__ void exact_vortex(double g, double x, double y, double t, double* U) {
  const double beta = 5.0, x0 = 5.0, y0 = 5.0, uinf = 1.0, vinf = 1.0, gv = 1.4;
  const double xd = x - x0 - uinf * t, yd = y - y0 - vinf * t;
  const double r2 = xd * xd + yd * yd;
  const double ef = exp(0.5 * (1.0 - r2));
  const double b2pi = beta / 6.283185307179586;
  const double du = -b2pi * ef * yd, dv = b2pi * ef * xd;
  const double pi2 = 3.141592653589793 * 3.141592653589793;
  double T = 1.0 - (gv - 1.0) * (beta * beta) / (8.0 * gv * pi2) * exp(1.0 - r2);
  T = jmax(T, 1e-14);
  const double r = pow(T, 1.0 / (gv - 1.0));
  const double p = pow(r, gv);
  const double u = uinf + du, v = vinf + dv;
  U[0] = r;
  U[1] = r * u;
  U[2] = r * v;
  U[3] = p / (g - 1.0) + 0.5 * r * (u * u + v * v);
}
__device__ void exact_smooth2d(double g, double x, double y, double t, double* U) {
  const double r = 1.0 + 0.2 * sin(6.283185307179586 * (x - t)) * sin(6.283185307179586 * (y - t));
  U[0] = r;
  U[1] = r;
  U[2] = r;
  U[3] = 1.0 / (g - 1.0) + 0.5 * r * 2.0;
}
__device__ void exact_density_wave1d(double g, double x, double t, double* U) {
  const double r = 1.0 + 0.2 * sin(6.283185307179586 * (x - 1.0 * t));
  U[0] = r;
  U[1] = r;
  U[2] = 1.0 / (g - 1.0) + 0.5 * r;
}

__global__ void __launch_bounds__(kDiagThreads)
    diag2d_kernel(const double* __restrict__ u, const Mesh2Dev M, const DiagTables T, int np, double g1,
                  int exact, const double* __restrict__ ref, double texact, int cl2, DiagPart* part) {
  __shared__ DiagPart s[kDiagThreads];
  const int np2 = np * np;
  const size_t n = (size_t)M.nel * np2;
  DiagPart p;
  part_init(p);
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
    const int e = (int)(idx / np2), k = (int)(idx % np2);
    const int i = k % np, j = k / np;
    const int gx = e % M.nx, gy = e / M.nx;
    double U[4];
    for (int c = 0; c < 4; ++c) U[c] = u[c * n + idx];
    const double absJ = M.curved ? fabs(1.0 / M.m_rJ[idx]) : fabs(M.Jx[gx] * M.Jy[gy]);
    const double ww = T.w[i] * T.w[j] * absJ;
    for (int c = 0; c < 4; ++c) {
      p.mass[c] += ww * U[c];
      p.nonfinite += isfinite(U[c]) ? 0.0 : 1.0;
    }
    // pressure(eq, U), Euler2D.jl:14-19
    const double r = jfloor(U[0], kEps);
    const double uu = U[1] / r, vv = U[2] / r;
    const double pr = g1 * (U[3] - 0.5 * r * (uu * uu + vv * vv));
    p.rmin = jmin(p.rmin, U[0]);
    p.rmax = jmax(p.rmax, U[0]);
    p.pmin = jmin(p.pmin, pr);
    if (!(U[0] > 0.0 && pr > 0.0 && isfinite(U[0]) && isfinite(pr))) p.posfail += 1.0;
    if (exact) {
      double E[4];
      if (exact == FRG_EXACT_STATE) {
        for (int c = 0; c < 4; ++c) E[c] = ref[c * n + idx];
      } else {
        // physical_xy, MeshMetrics2D.jl:49-74
        const double X = M.xc[gx] + M.Jx[gx] * T.xi[i], Y = M.yc[gy] + M.Jy[gy] * T.xi[j];
        double x = X, y = Y;
        if (M.wavy) {
          x = X + M.amp * sin(6.283185307179586 * Y) * sin(3.141592653589793 * X);
          y = Y + M.amp * sin(6.283185307179586 * X) * sin(3.141592653589793 * Y);
        }
        if (exact == FRG_EXACT_VORTEX_2D)
          exact_vortex(g1 + 1.0, x, y, texact, E);
        else
          exact_smooth2d(g1 + 1.0, x, y, texact, E);
      }
      const double err = U[cl2] - E[cl2];
      p.l2 += ww * err * err;
    }
  }
  block_reduce(s, p);
  if (threadIdx.x == 0) part[blockIdx.x] = s[0];
}

__global__ void __launch_bounds__(kDiagThreads)
    diag1d_kernel(const double* __restrict__ u, const Mesh1Dev M, const DiagTables T, int np, double g1,
                  int exact, const double* __restrict__ ref, double texact, int cl2, DiagPart* part) {
  __shared__ DiagPart s[kDiagThreads];
  const size_t n = (size_t)M.nel * np;
  DiagPart p;
  part_init(p);
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
    const int e = (int)(idx / np), j = (int)(idx % np);
    double U[3];
    for (int c = 0; c < 3; ++c) U[c] = u[c * n + idx];
    const double ww = T.w[j] * M.J[e];
    for (int c = 0; c < 3; ++c) {
      p.mass[c] += ww * U[c];
      p.nonfinite += isfinite(U[c]) ? 0.0 : 1.0;
    }
    // pressure(eq, U), Euler.jl:19-24
    const double r = jfloor(U[0], kEps);
    const double uu = U[1] / r;
    const double pr = g1 * (U[2] - 0.5 * r * uu * uu);
    p.rmin = jmin(p.rmin, U[0]);
    p.rmax = jmax(p.rmax, U[0]);
    p.pmin = jmin(p.pmin, pr);
    if (!(U[0] > 0.0 && pr > 0.0 && isfinite(U[0]) && isfinite(pr))) p.posfail += 1.0;
    if (exact) {
      double E[3];
      if (exact == FRG_EXACT_STATE) {
        for (int c = 0; c < 3; ++c) E[c] = ref[c * n + idx];
      } else {
        exact_density_wave1d(g1 + 1.0, M.xc[e] + M.J[e] * T.xi[j], texact, E);
      }
      const double err = U[cl2] - E[cl2];
      p.l2 += ww * err * err;
    }
  }
  block_reduce(s, p);
  if (threadIdx.x == 0) part[blockIdx.x] = s[0];
}

// one block: the block partials in order
__global__ void __launch_bounds__(kDiagThreads) diag_final_kernel(const DiagPart* part, int nparts, DiagPart* out) {
  __shared__ DiagPart s[kDiagThreads];
  DiagPart p;
  part_init(p);
  for (int b = threadIdx.x; b < nparts; b += blockDim.x) part_merge(p, part[b]);
  block_reduce(s, p);
  if (threadIdx.x == 0) *out = s[0];
}

}  // namespace
}  // namespace frg

using namespace frg;
using namespace frg::rt;

extern "C" int frg_diagnostics_compute(frg_solve* s, int exact, const double* ref_dev, double t_exact, int c,
                                       frg_diagnostics* out) {
  if (!s || !out) return FRG_ERR_INVALID_ARG;
  if (!s->have_state) return set_err(s->ctx, FRG_ERR_STATE, "no state uploaded");
  if (c < 0 || c >= s->neq) return set_err(s->ctx, FRG_ERR_INVALID_ARG, "component out of range");
  const bool is2 = s->dim == 2;
  switch (exact) {
    case FRG_EXACT_NONE:
      break;
    case FRG_EXACT_STATE:
      if (!ref_dev) return set_err(s->ctx, FRG_ERR_INVALID_ARG, "reference state pointer is NULL");
      break;
    case FRG_EXACT_VORTEX_2D:
    case FRG_EXACT_SMOOTH_2D:
      if (!is2) return set_err(s->ctx, FRG_ERR_INVALID_ARG, "2D exact solution on a 1D solve");
      if (s->L2.mesh.curved && !s->L2.mesh.wavy)
        return set_err(s->ctx, FRG_ERR_INVALID_ARG, "exact solution needs point coordinates (caller metrics)");
      break;
    case FRG_EXACT_DENSITY_WAVE_1D:
      if (is2) return set_err(s->ctx, FRG_ERR_INVALID_ARG, "1D exact solution on a 2D solve");
      break;
    default:
      return set_err(s->ctx, FRG_ERR_INVALID_ARG, "unknown exact solution");
  }
  cudaSetDevice(s->ctx->device);
  cudaStream_t st = s->ctx->stream;
  DiagTables T;
  std::memset(&T, 0, sizeof(T));
  for (int i = 0; i < s->np; ++i) {
    T.w[i] = s->ops.w[i];
    T.xi[i] = s->ops.xi[i];
  }
  const size_t npts = s->ndof / s->neq;
  const int blocks = (int)std::min<size_t>((npts + kDiagThreads - 1) / kDiagThreads, (size_t)kDiagMaxBlocks);
  DiagPart* d = nullptr;
  cudaError_t e = cudaMallocAsync((void**)&d, sizeof(DiagPart) * (blocks + 1), st);
  if (e != cudaSuccess) return cuda_err(s->ctx, e, "diagnostics scratch");
  const double* u = s->U[s->cur];
  const double g1 = s->dim == 2 ? s->L2.phys.g1 : s->L1.phys.g1;
  if (is2)
    diag2d_kernel<<<blocks, kDiagThreads, 0, st>>>(u, s->L2.mesh, T, s->np, g1, exact, ref_dev, t_exact, c, d);
  else
    diag1d_kernel<<<blocks, kDiagThreads, 0, st>>>(u, s->L1.mesh, T, s->np, g1, exact, ref_dev, t_exact, c, d);
  diag_final_kernel<<<1, kDiagThreads, 0, st>>>(d, blocks, d + blocks);
  DiagPart h;
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, d + blocks, sizeof(h), cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(d, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_err(s->ctx, e, "diagnostics");
  std::memset(out, 0, sizeof(*out));
  for (int k = 0; k < 4; ++k) out->mass[k] = k < s->neq ? h.mass[k] : 0.0;
  out->rho_min = h.rmin;
  out->rho_max = h.rmax;
  out->p_min = h.pmin;
  out->nonfinite = (int64_t)h.nonfinite;
  out->positivity_ok = h.posfail == 0.0 ? 1 : 0;
  out->l2_error = exact ? std::sqrt(h.l2) : 0.0;
  out->t = s->t;
  return FRG_OK;
}

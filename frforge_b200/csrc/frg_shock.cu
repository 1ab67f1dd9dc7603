// 1D shock-capturing scores of a solve's density, computed on the device:
// the scoring fields of the reference's discontinuous 1D cases (Sod and
// Shu-Osher reports, Cases.jl:987-1021, :1100-1122) without downloading the
// state.
//
//   sample_solution_1d(state, eq; :density)   Metrics.jl:95-123
//       The samples sorted by x are the density block of the state in
//       (element, point) order: elements run left to right and the GL nodes
//       ascend inside each, so the sort is the identity.  x = mid + J xi is
//       evaluated without contraction, as the reference does.
//   overshoot_metric                          Metrics.jl:81-87
//   shock_thickness_sp                        Metrics.jl:138-200 (plateaus
//       from the window medians; the variant with given jump bounds is not
//       used by the reference's reports)
//   smooth_region_mask + excess_dissipation   Metrics.jl:208-255, against a
//       reference density on the same samples (the mask is the reference's)
//   relative L1 against the reference         Cases.jl:1021
//
// Pass 1 (each thread a contiguous run of samples, fixed-order block trees,
// then one block over the block partials in order): the steepest density
// gradient (first index on ties),
// the density extrema, the largest reference gradient and the unmasked L1
// sums.  Pass 2: the masked sums.  A one-thread kernel then walks the shock
// window.  Every result is independent of scheduling.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "frg_device.cuh"
#include "frg_runtime.h"

namespace frg {
namespace {

constexpr int kShockThreads = 256;
constexpr int kShockMaxBlocks = 592;  // 4 x 148 SMs
constexpr int kMaxWindowSp = 1024;

struct ShockPart {
  double gmax;    // steepest |d rho / dx|
  long long imax;  // its sample index (>= 1)
  double rmin, rmax;
  double gref;    // largest reference gradient
  double l1n, l1d;  // sum |rho - ref|, sum |ref|
  double exn, exd;  // the same over the smooth-region mask
};

struct ShockGeom {
  const double* xc;  // [nel] element mid points
  const double* J;   // [nel]
  double xi[kMaxNp];
  int np;
};

struct ShockArgs {
  double ref_min, ref_max, grad_frac;
  int window_sp, n_exclude;
  double exclude[4][2];
};

// x of sample i: mid + J xi without fused multiply-add
__device__ __forceinline__ double sample_x(const ShockGeom& G, long long i) {
  const long long e = i / G.np;
  const int j = (int)(i % G.np);
  return __dadd_rn(G.xc[e], __dmul_rn(G.J[e], G.xi[j]));
}

// |v_i - v_{i-1}| / max(|x_i - x_{i-1}|, 1e-30), i >= 1
__device__ __forceinline__ double grad_at(const double* v, const ShockGeom& G, long long i) {
  const double dx = fabs(sample_x(G, i) - sample_x(G, i - 1));
  return fabs(v[i] - v[i - 1]) / jmax(dx, 1e-30);
}

__device__ __forceinline__ void part_init(ShockPart& p) {
  p.gmax = 0.0;
  p.imax = 1;
  p.rmin = INFINITY;
  p.rmax = -INFINITY;
  p.gref = -INFINITY;
  p.l1n = p.l1d = p.exn = p.exd = 0.0;
}

// a holds lower sample indices than b (first-index tie rule of the scan)
__device__ __forceinline__ void part_merge(ShockPart& a, const ShockPart& b) {
  if (b.gmax > a.gmax || (b.gmax == a.gmax && b.imax < a.imax)) {
    a.gmax = b.gmax;
    a.imax = b.imax;
  }
  a.rmin = jmin(a.rmin, b.rmin);
  a.rmax = jmax(a.rmax, b.rmax);
  a.gref = jmax(a.gref, b.gref);
  a.l1n += b.l1n;
  a.l1d += b.l1d;
  a.exn += b.exn;
  a.exd += b.exd;
}

__device__ void block_reduce(ShockPart* s, const ShockPart& mine) {
  const int t = threadIdx.x;
  s[t] = mine;
  __syncthreads();
  for (int h = kShockThreads / 2; h > 0; h >>= 1) {
    if (t < h) {
      ShockPart a = s[t];
      part_merge(a, s[t + h]);
      s[t] = a;
    }
    __syncthreads();
  }
}

// Each thread covers one contiguous run of samples, so a scan of it meets
// the indices in increasing order and the tree merges runs left to right.
__device__ __forceinline__ void thread_run(long long n, long long* i0, long long* i1) {
  const long long nthr = (long long)gridDim.x * blockDim.x;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long per = (n + nthr - 1) / nthr;
  *i0 = t * per;
  *i1 = min(n, *i0 + per);
}

__global__ void __launch_bounds__(kShockThreads)
    shock_pass1(const double* __restrict__ rho, const double* __restrict__ ref, ShockGeom G, long long n,
                ShockPart* part) {
  __shared__ ShockPart s[kShockThreads];
  ShockPart p;
  part_init(p);
  long long i0, i1;
  thread_run(n, &i0, &i1);
  for (long long i = i0; i < i1; ++i) {
    const double r = rho[i];
    p.rmin = jmin(p.rmin, r);
    p.rmax = jmax(p.rmax, r);
    if (i >= 1) {
      const double g = grad_at(rho, G, i);
      if (g > p.gmax) {
        p.gmax = g;
        p.imax = i;
      }
    }
    if (ref) {
      p.l1n += fabs(r - ref[i]);
      p.l1d += fabs(ref[i]);
      // g[1] = g[2] adds no new value to the maximum
      if (i >= 1) p.gref = jmax(p.gref, grad_at(ref, G, i));
    }
  }
  block_reduce(s, p);
  if (threadIdx.x == 0) part[blockIdx.x] = s[0];
}

__global__ void __launch_bounds__(kShockThreads)
    shock_pass2(const double* __restrict__ rho, const double* __restrict__ ref, ShockGeom G, long long n,
                ShockArgs A, const ShockPart* acc, ShockPart* part) {
  __shared__ ShockPart s[kShockThreads];
  ShockPart p;
  part_init(p);
  const double thr = A.grad_frac * acc->gref;
  long long i0, i1;
  thread_run(n, &i0, &i1);
  for (long long i = i0; i < i1; ++i) {
    const double g = grad_at(ref, G, i >= 1 ? i : 1);
    bool keep = !(g > thr);
    const double x = sample_x(G, i);
    for (int w = 0; w < A.n_exclude; ++w)
      if (A.exclude[w][0] <= x && x <= A.exclude[w][1]) keep = false;
    if (keep) {
      p.exn += fabs(rho[i] - ref[i]);
      p.exd += fabs(ref[i]);
    }
  }
  block_reduce(s, p);
  if (threadIdx.x == 0) part[blockIdx.x] = s[0];
}

__global__ void __launch_bounds__(kShockThreads) shock_final(const ShockPart* part, int nparts, ShockPart* out) {
  __shared__ ShockPart s[kShockThreads];
  // thread t takes a contiguous run of the partials (index order kept)
  ShockPart p;
  part_init(p);
  const int per = (nparts + kShockThreads - 1) / kShockThreads;
  for (int b = threadIdx.x * per; b < min(nparts, (int)(threadIdx.x + 1) * per); ++b) part_merge(p, part[b]);
  block_reduce(s, p);
  if (threadIdx.x == 0) *out = s[0];
}

// Julia isless on Float64: NaN after everything, -0.0 before 0.0
__device__ __forceinline__ bool jl_isless(double a, double b) {
  if (isnan(a)) return false;
  if (isnan(b)) return true;
  if (a < b) return true;
  if (a > b) return false;
  return signbit(a) && !signbit(b);
}

// the k-th smallest (0-based) of v[0..n), n <= kMaxWindowSp
__device__ double sorted_at(const double* v, int n, int k) {
  // rank selection: the element with exactly k smaller ones (ties by index)
  for (int a = 0; a < n; ++a) {
    int below = 0;
    for (int b = 0; b < n; ++b)
      if (jl_isless(v[b], v[a]) || (!jl_isless(v[a], v[b]) && b < a)) ++below;
    if (below == k) return v[a];
  }
  return NAN;
}

// shock_thickness_sp (Metrics.jl:138-200) from the steepest-gradient index;
// out[0] = thickness, out[1] = x of the steepest gradient
__global__ void shock_thickness(const double* __restrict__ rho, ShockGeom G, long long n, ShockArgs A,
                                const ShockPart* acc, double* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  out[1] = sample_x(G, acc->imax);
  if (n < 4) {
    out[0] = NAN;
    return;
  }
  // 1-based indices as in the reference
  const long long imax = acc->imax + 1;
  const long long i0 = max(1ll, imax - A.window_sp);
  const long long i1 = min(n, imax + A.window_sp);
  const long long w = i1 - i0 + 1;
  const int nL = (int)max(1ll, w / 3);
  const double rL = sorted_at(rho + (i0 - 1), nL, max(1, nL / 2) - 1);
  const double rR = sorted_at(rho + (i1 - nL), nL, max(1, nL / 2) - 1);
  const double rmin = jmin(rL, rR), rmax = jmax(rL, rR);
  const double D = rmax - rmin;
  if (fabs(D) < 1e-14) {
    out[0] = NAN;
    return;
  }
  const double lo = __dadd_rn(rmin, __dmul_rn(0.1, D));
  const double hi = __dadd_rn(rmin, __dmul_rn(0.9, D));
  const bool rising = rR >= rL;
  long long i10 = imax, i90 = imax;
  auto R = [&](long long i) { return rho[i - 1]; };
  if (rising) {
    while (i10 > i0 && R(i10) > lo) --i10;
    while (i90 < i1 && R(i90) < hi) ++i90;
  } else {
    while (i10 < i1 && R(i10) > lo) ++i10;
    while (i90 > i0 && R(i90) < hi) --i90;
  }
  const double dx = fabs(sample_x(G, i90 - 1) - sample_x(G, i10 - 1));
  const double mean = (sample_x(G, n - 1) - sample_x(G, 0)) / (double)(n - 1);
  out[0] = dx / mean;
}

}  // namespace
}  // namespace frg

using namespace frg;
using namespace frg::rt;

extern "C" int frg_shock_metrics_1d(frg_solve* s, const frg_shock_params* prm, const double* ref_host,
                                    const frg_solve* ref_solve, frg_shock_metrics* out) {
  if (!s || !prm || !out) return FRG_ERR_INVALID_ARG;
  if (s->dim != 1) return set_err(s->ctx, FRG_ERR_INVALID_ARG, "shock metrics are defined for 1D solves");
  if (!s->have_state) return set_err(s->ctx, FRG_ERR_STATE, "no state uploaded");
  if (ref_host && ref_solve) return set_err(s->ctx, FRG_ERR_INVALID_ARG, "give one reference, not two");
  if (prm->n_exclude < 0 || prm->n_exclude > 4) return set_err(s->ctx, FRG_ERR_INVALID_ARG, "at most 4 windows");
  if (prm->window_sp < 1 || prm->window_sp > kMaxWindowSp / 2)
    return set_err(s->ctx, FRG_ERR_INVALID_ARG, "window_sp out of range");
  const long long n = (long long)s->nel * s->np;
  if (ref_solve) {
    if (ref_solve->dim != 1 || ref_solve->nel != s->nel || ref_solve->np != s->np)
      return set_err(s->ctx, FRG_ERR_INVALID_ARG, "reference solve has other samples");
    if (!ref_solve->have_state) return set_err(s->ctx, FRG_ERR_STATE, "reference solve has no state");
    if (ref_solve->ctx->device != s->ctx->device)
      return set_err(s->ctx, FRG_ERR_INVALID_ARG, "reference solve is on another device");
  }
  cudaSetDevice(s->ctx->device);
  cudaStream_t st = s->ctx->stream;
  int rc = make_current_canonical(s);
  if (rc) return rc;
  if (ref_solve) {
    // the reference's pending work (its own stream) comes first
    cudaError_t e = cudaStreamSynchronize(ref_solve->ctx->stream);
    if (e != cudaSuccess) return cuda_err(s->ctx, e, "reference solve");
  }
  ShockGeom G;
  std::memset(&G, 0, sizeof(G));
  G.xc = s->L1.mesh.xc;
  G.J = s->L1.mesh.J;
  G.np = s->np;
  for (int i = 0; i < s->np; ++i) G.xi[i] = s->ops.xi[i];
  ShockArgs A;
  std::memset(&A, 0, sizeof(A));
  A.ref_min = prm->ref_min;
  A.ref_max = prm->ref_max;
  A.grad_frac = prm->grad_frac;
  A.window_sp = prm->window_sp;
  A.n_exclude = prm->n_exclude;
  for (int w = 0; w < prm->n_exclude; ++w) {
    A.exclude[w][0] = prm->exclude[w][0];
    A.exclude[w][1] = prm->exclude[w][1];
  }
  const int blocks = (int)std::min<long long>((n + kShockThreads - 1) / kShockThreads, (long long)kShockMaxBlocks);
  // scratch: block partials, two accumulators, thickness and shock x, a host reference copy
  const size_t part_bytes = sizeof(ShockPart) * (blocks + 2) + 16;
  const size_t ref_bytes = ref_host ? sizeof(double) * (size_t)n : 0;
  char* d = nullptr;
  cudaError_t e = cudaMallocAsync((void**)&d, part_bytes + 16 + ref_bytes, st);
  // layout: partials | thickness, x (16 B) | pad | reference
  if (e != cudaSuccess) return cuda_err(s->ctx, e, "shock metrics scratch");
  ShockPart* part = reinterpret_cast<ShockPart*>(d);
  ShockPart* acc1 = part + blocks;
  ShockPart* acc2 = part + blocks + 1;
  double* thick = reinterpret_cast<double*>(d + part_bytes - 16);
  const double* ref = nullptr;
  if (ref_host) {
    double* r = reinterpret_cast<double*>(d + part_bytes + 16);
    e = cudaMemcpyAsync(r, ref_host, ref_bytes, cudaMemcpyHostToDevice, st);
    ref = r;
  } else if (ref_solve) {
    ref = ref_solve->U[ref_solve->cur];  // density block
  }
  const double* rho = s->U[s->cur];
  if (e == cudaSuccess) {
    shock_pass1<<<blocks, kShockThreads, 0, st>>>(rho, ref, G, n, part);
    shock_final<<<1, kShockThreads, 0, st>>>(part, blocks, acc1);
    if (ref) {
      shock_pass2<<<blocks, kShockThreads, 0, st>>>(rho, ref, G, n, A, acc1, part);
      shock_final<<<1, kShockThreads, 0, st>>>(part, blocks, acc2);
    }
    shock_thickness<<<1, 32, 0, st>>>(rho, G, n, A, acc1, thick);
    e = cudaGetLastError();
  }
  ShockPart h1, h2;
  double th[2] = {NAN, NAN};
  std::memset(&h1, 0, sizeof(h1));
  std::memset(&h2, 0, sizeof(h2));
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h1, acc1, sizeof(h1), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && ref) e = cudaMemcpyAsync(&h2, acc2, sizeof(h2), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(th, thick, sizeof(th), cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(d, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_err(s->ctx, e, "shock metrics");
  std::memset(out, 0, sizeof(*out));
  out->n_samples = n;
  out->rho_min = h1.rmin;
  out->rho_max = h1.rmax;
  out->shock_index = h1.imax;
  out->shock_x = th[1];
  out->shock_thickness = th[0];
  // overshoot_metric (Metrics.jl:81-87); max(0.0, NaN) is NaN as in Julia
  const double D = std::fmax(std::fabs(prm->ref_max - prm->ref_min), 2.220446049250313e-16);
  auto jl_max0 = [](double v) { return std::isnan(v) ? v : std::fmax(0.0, v); };
  out->overshoot_over = jl_max0(h1.rmax - prm->ref_max) / D;
  out->overshoot_under = jl_max0(prm->ref_min - h1.rmin) / D;
  out->overshoot = (std::isnan(out->overshoot_over) || std::isnan(out->overshoot_under))
                       ? NAN
                       : std::fmax(out->overshoot_over, out->overshoot_under);
  out->has_reference = ref ? 1 : 0;
  out->excess_dissipation = ref ? h2.exn / (h2.exd + 1e-30) : NAN;
  out->l1_rel = ref ? h1.l1n / (h1.l1d + 1e-30) : NAN;
  return FRG_OK;
}

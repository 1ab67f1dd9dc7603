// Allocation-free 2D residual evaluation.
//
// frg_residual2d_noalloc evaluates the same residual as frg_residual (the FR
// residual with its capturing hooks) but never allocates device memory: the
// caller passes the state and the output as device pointers it already
// owns, and every piece of scratch the kernels need -- the per-element
// artificial viscosity, the mesh spacing arrays and the small status block --
// lives in one file-scope __device__ array of fixed size.  It is meant for
// callers that cannot call cudaMalloc at the point they need a residual:
// host frameworks whose device memory is owned by their own pool or budget
// (a foreign cudaMalloc would bypass it or fail against a hard limit), and
// code paths where a device allocation is not allowed at call time.
//
// Limits and sharing:
//   - at most FRG_NOALLOC_MAX_ELEMENTS elements and FRG_NOALLOC_MAX_SIDE
//     elements per mesh side; larger meshes are rejected with
//     FRG_ERR_INVALID_ARG;
//   - every GPU that loads the library holds the array (about 4.2 MB) until
//     the process exits;
//   - the first call on a device resolves the array's device address with
//     cudaGetSymbolAddress (device-specific set-up); make that first call
//     before any stream capture on that device;
//   - all calls share the array and it keeps the last call's contents: every
//     call rewrites what it reads, but calls that overlap on the GPU (two
//     streams, or two host threads) race on it and must be serialised by the
//     caller.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>

#include "frg_internal.h"

namespace frg {

// layout of the scratch array, in doubles
constexpr int kNaMaxEl = FRG_NOALLOC_MAX_ELEMENTS;
constexpr int kNaMaxSide = FRG_NOALLOC_MAX_SIDE;
constexpr size_t kNaEps = 0;                            // [kNaMaxEl] eps
constexpr size_t kNaHchar = kNaEps + kNaMaxEl;          // [kNaMaxEl] h_char
constexpr size_t kNaCols = kNaHchar + kNaMaxEl;         // 3 x [kNaMaxSide]: xc, Jx, 1/Jx
constexpr size_t kNaRows = kNaCols + 3 * kNaMaxSide;    // 3 x [kNaMaxSide]: yc, Jy, 1/Jy
constexpr size_t kNaScalars = kNaRows + 3 * kNaMaxSide;  // DevScalars
constexpr size_t kNaDoubles = kNaScalars + (sizeof(DevScalars) + 7) / 8;

static __device__ __align__(256) double g_noalloc_scratch[kNaDoubles];

namespace {

std::mutex g_na_mu;
double* g_na_ptr[64] = {nullptr};  // device address of the scratch array, per device

// Host staging for the mesh arrays (no allocation at call time).
struct NaHost {
  double cols[3 * kNaMaxSide];
  double rows[3 * kNaMaxSide];
  double hchar[kNaMaxEl];
  double xv[kNaMaxSide + 1], yv[kNaMaxSide + 1];
};
NaHost g_na_host;

}  // namespace
}  // namespace frg

using namespace frg;

extern "C" int frg_residual2d_noalloc(const frg_solve_desc* d, const double* u, double* du, double t,
                                      void* stream) {
  if (!d || !u || !du) return FRG_ERR_INVALID_ARG;
  if (d->dim != 2 || d->p < 1 || d->p > FRG_MAX_NP - 1) return FRG_ERR_INVALID_ARG;
  if (d->nx < 1 || d->ny < 1 || d->nx > kNaMaxSide || d->ny > kNaMaxSide ||
      (long long)d->nx * d->ny > kNaMaxEl)
    return FRG_ERR_INVALID_ARG;  // beyond the fixed scratch size
  if (d->geometry != FRG_GEOM_AFFINE || d->solid) return FRG_ERR_INVALID_ARG;
  if (d->method != FRG_METHOD_NULL && d->method != FRG_METHOD_PERSSON) return FRG_ERR_UNSUPPORTED_HOOK;
  if ((d->bc[0].kind == FRG_BC_PERIODIC) != (d->bc[1].kind == FRG_BC_PERIODIC) ||
      (d->bc[2].kind == FRG_BC_PERIODIC) != (d->bc[3].kind == FRG_BC_PERIODIC))
    return FRG_ERR_INVALID_ARG;
  if (!d->x_vertices && !(d->x_right > d->x_left)) return FRG_ERR_INVALID_ARG;
  if (!d->y_vertices && !(d->y_top > d->y_bottom)) return FRG_ERR_INVALID_ARG;

  std::lock_guard<std::mutex> lock(g_na_mu);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return FRG_ERR_CUDA;
  if (!g_na_ptr[dev]) {
    // once per device, with that device current
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return FRG_ERR_CUDA;
    g_na_ptr[dev] = (double*)p;
  }
  double* base = g_na_ptr[dev];
  cudaStream_t st = (cudaStream_t)stream;

  HostOps ops;
  int rc = d->ops ? host_ops_from_caller(d->ops, &ops) : build_host_ops(d->p, d->points, &ops);
  if (rc) return rc;

  const int nx = d->nx, ny = d->ny, nel = nx * ny;
  NaHost& h = g_na_host;
  if (d->x_vertices)
    std::memcpy(h.xv, d->x_vertices, sizeof(double) * (nx + 1));
  else
    julia_linspace(d->x_left, d->x_right, nx + 1, h.xv);
  if (d->y_vertices)
    std::memcpy(h.yv, d->y_vertices, sizeof(double) * (ny + 1));
  else
    julia_linspace(d->y_bottom, d->y_top, ny + 1, h.yv);
  for (int i = 0; i < nx; ++i) {
    h.cols[i] = (h.xv[i] + h.xv[i + 1]) / 2.0;
    h.cols[kNaMaxSide + i] = (h.xv[i + 1] - h.xv[i]) / 2.0;
    h.cols[2 * kNaMaxSide + i] = 1.0 / h.cols[kNaMaxSide + i];
  }
  for (int i = 0; i < ny; ++i) {
    h.rows[i] = (h.yv[i] + h.yv[i + 1]) / 2.0;
    h.rows[kNaMaxSide + i] = (h.yv[i + 1] - h.yv[i]) / 2.0;
    h.rows[2 * kNaMaxSide + i] = 1.0 / h.rows[kNaMaxSide + i];
  }
  for (int e = 0; e < nel; ++e)
    h.hchar[e] = std::fmin(h.xv[e % nx + 1] - h.xv[e % nx], h.yv[e / nx + 1] - h.yv[e / nx]);
  DevScalars sc;
  std::memset(&sc, 0, sizeof(sc));
  sc.t = t;
  sc.two_p1 = 2 * d->p + 1;

  cudaError_t e = cudaMemcpyAsync(base + kNaCols, h.cols, sizeof(h.cols), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(base + kNaRows, h.rows, sizeof(h.rows), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(base + kNaHchar, h.hchar, sizeof(double) * nel, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(base + kNaScalars, &sc, sizeof(sc), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return FRG_ERR_CUDA;

  Launch2D L{};
  L.ops = &ops;
  Mesh2Dev& M = L.mesh;
  M.nx = nx;
  M.ny = ny;
  M.nel = nel;
  M.px = d->bc[0].kind == FRG_BC_PERIODIC;
  M.py = d->bc[2].kind == FRG_BC_PERIODIC;
  M.xc = base + kNaCols;
  M.Jx = base + kNaCols + kNaMaxSide;
  M.rJx = base + kNaCols + 2 * kNaMaxSide;
  M.yc = base + kNaRows;
  M.Jy = base + kNaRows + kNaMaxSide;
  M.rJy = base + kNaRows + 2 * kNaMaxSide;
  M.hchar = base + kNaHchar;
  for (int k = 0; k < 4; ++k) {
    const frg_bc& b = d->bc[k];
    BCDev& o = M.bc[k];
    o.kind = b.kind;
    o.mode = b.mode;
    for (int c = 0; c < 4; ++c) {
      o.st[c] = b.state[c];
      o.stb[c] = b.state_b[c];
    }
    o.x0 = b.x0;
    o.s0 = b.s0;
    o.s1 = b.s1;
    o.sdiv = b.sdiv == 0.0 ? 1.0 : b.sdiv;
  }
  Phys& P = L.phys;
  P.gamma = d->gamma;
  P.g1 = d->gamma - 1.0;
  P.c_av = d->c_av;
  P.kappa = d->kappa;
  P.eps_floor = d->eps_floor;
  P.p = d->p;
  P.pm = d->p > 1 ? d->p : 1;
  P.s0 = d->s0_factor * std::log10((double)P.pm);
  L.flux = d->flux;
  L.av = d->method == FRG_METHOD_PERSSON ? (d->av_form == FRG_AV_LOCAL_DD ? kAvDD : kAvBR0) : kAvNone;
  L.variant = 0;

  DevScalars* dsc = reinterpret_cast<DevScalars*>(base + kNaScalars);
  double* eps = base + kNaEps;
  if (L.av != kAvNone) {
    // element viscosity of the state (every element is written)
    StageBufs b{};
    b.us = u;
    b.eps_out = eps;
    b.mode = kModePrime;
    b.sc = dsc;
    if (launch_stage2d(L, b, st)) return FRG_ERR_CUDA;
  }
  StageBufs b{};
  b.us = u;
  b.eps_in = eps;
  b.du_out = du;
  b.mode = kModeResidual;
  b.stage = 1;
  b.sc = dsc;
  if (launch_stage2d(L, b, st)) return FRG_ERR_CUDA;
  if (cudaGetLastError() != cudaSuccess) return FRG_ERR_CUDA;
  return FRG_OK;
}

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
//     cudaGetSymbolAddress (device-specific set-up);
//   - all calls share the array and it keeps the last call's contents: every
//     call rewrites what it reads, but calls that overlap on the GPU (two
//     streams, or two host threads) race on it and must be serialised by the
//     caller.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>

#include "frg_runtime.h"

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

// Host staging for the row and column arrays (no allocation at call time).
struct NaHost {
  double cols[3 * kNaMaxSide];
  double rows[3 * kNaMaxSide];
  double xv[kNaMaxSide + 1], yv[kNaMaxSide + 1];
};
NaHost g_na_host;

// Element sizes h_char = min(dx, dy) (Mesh2D.jl:35-91) from the column and
// row half-widths (2 Jx = dx exactly), and the status block of one residual
// evaluation: O(nel) work on the device instead of a host loop and copy.
__global__ void noalloc_setup_kernel(int nx, int ny, const double* Jx, const double* Jy, double* hchar,
                                     DevScalars* sc, double t, int two_p1) {
  const int nel = nx * ny;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nel; e += gridDim.x * blockDim.x)
    hchar[e] = fmin(2.0 * Jx[e % nx], 2.0 * Jy[e / nx]);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    DevScalars z = {};
    z.t = t;
    z.two_p1 = two_p1;
    *sc = z;
  }
}

}  // namespace
}  // namespace frg

using namespace frg;

extern "C" int frg_residual2d_noalloc(const frg_solve_desc* d, const double* u, double* du, double t,
                                      void* stream) {
  if (!d || !u || !du) return FRG_ERR_INVALID_ARG;
  // the checks of frg_solve_create, then the limits of this entry point
  const int vrc = rt::validate_desc(nullptr, d);
  if (vrc) return vrc;
  if (d->dim != 2) return FRG_ERR_INVALID_ARG;
  if (d->nx > kNaMaxSide || d->ny > kNaMaxSide || (long long)d->nx * d->ny > kNaMaxEl)
    return FRG_ERR_INVALID_ARG;  // beyond the fixed scratch size
  if (d->geometry != FRG_GEOM_AFFINE || d->solid) return FRG_ERR_INVALID_ARG;

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
  // xc, Jx, 1/Jx packed at stride nx (yc, Jy, 1/Jy at stride ny), so one
  // copy of 3 nx (3 ny) doubles moves what the mesh uses
  for (int i = 0; i < nx; ++i) {
    h.cols[i] = (h.xv[i] + h.xv[i + 1]) / 2.0;
    h.cols[nx + i] = (h.xv[i + 1] - h.xv[i]) / 2.0;
    h.cols[2 * nx + i] = 1.0 / h.cols[nx + i];
  }
  for (int i = 0; i < ny; ++i) {
    h.rows[i] = (h.yv[i] + h.yv[i + 1]) / 2.0;
    h.rows[ny + i] = (h.yv[i + 1] - h.yv[i]) / 2.0;
    h.rows[2 * ny + i] = 1.0 / h.rows[ny + i];
  }
  double* cols = base + kNaCols;
  double* rows = base + kNaRows;
  DevScalars* dsc = reinterpret_cast<DevScalars*>(base + kNaScalars);
  cudaError_t e = cudaMemcpyAsync(cols, h.cols, sizeof(double) * 3 * nx, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(rows, h.rows, sizeof(double) * 3 * ny, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return FRG_ERR_CUDA;
  {
    const int blocks = (nel + 255) / 256 < 1184 ? (nel + 255) / 256 : 1184;
    noalloc_setup_kernel<<<blocks, 256, 0, st>>>(nx, ny, cols + nx, rows + ny, base + kNaHchar, dsc, t,
                                                  2 * d->p + 1);
    if (cudaGetLastError() != cudaSuccess) return FRG_ERR_CUDA;
  }

  Launch2D L{};
  L.ops = &ops;
  Mesh2Dev& M = L.mesh;
  M.nx = nx;
  M.ny = ny;
  M.nel = nel;
  M.px = d->bc[0].kind == FRG_BC_PERIODIC;
  M.py = d->bc[2].kind == FRG_BC_PERIODIC;
  M.xc = cols;
  M.Jx = cols + nx;
  M.rJx = cols + 2 * nx;
  M.yc = rows;
  M.Jy = rows + ny;
  M.rJy = rows + 2 * ny;
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
  P.flux_alpha = 1.0;
  P.trace_hook = 0;
  P.trace_p0 = 0.0;
  P.trace_p1 = 0.0;
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

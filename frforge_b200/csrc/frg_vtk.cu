// VTU point data on the device: the high-order VTK writer's node values,
// evaluated where the state lives.
//
// The reference's writer (src/io/VTKHighOrder.jl:325-535) places (p+1)^d
// equispaced VTK Lagrange nodes in every element (VTK node order, given by
// the caller), interpolates the solution from the Gauss points with the
// Lagrange basis (gl_to_equi_interp, :8-41, and its tensor product in 2D),
// maps the nodes with physical_xy (src/mesh/MeshMetrics2D.jl:49-74, the
// analytic wavy map included) and writes the Euler point fields
//   2D: rho, u, v, p, rho_u, rho_v, E     1D: rho, u, p, rho_u, E
// with u = rho_u / max(rho, eps) and p from the floored density
// (pressure, src/equations/Euler.jl:18-24, Euler2D.jl:14-19).
//
// frg_vtk_point_data runs one thread per node: Lagrange weights of the node
// on the solution points, the interpolated conserved state, the fields and
// the coordinates, written field-major ([field][element * n_per + node])
// for the writer.  Only the node data crosses to the host; the solve's state
// stays on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "frg_device.cuh"
#include "frg_runtime.h"

namespace frg {
namespace {

constexpr int kVtkMaxNodes = kMaxNp * kMaxNp;

struct VtkNodes {
  double xi[kMaxNp];            // solution points
  double a[kVtkMaxNodes];       // node xi (VTK order)
  double b[kVtkMaxNodes];       // node eta (2D)
  int np, n_per;
};

// Lagrange basis on the solution points at x (lagrange_at, src/fr/Points.jl:65-76)
FRG_DEV void lagrange_weights(const VtkNodes& N, double x, double* l) {
  for (int j = 0; j < N.np; ++j) {
    double v = 1.0;
    for (int m = 0; m < N.np; ++m)
      if (m != j) v *= (x - N.xi[m]) / (N.xi[j] - N.xi[m]);
    l[j] = v;
  }
}

__global__ void vtk_points_2d(const double* __restrict__ u, const Mesh2Dev M, const VtkNodes N, double gamma,
                              double* __restrict__ xy, double* __restrict__ f) {
  const size_t npts = (size_t)M.nel * N.n_per;
  const size_t cs = (size_t)M.nel * N.np * N.np;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < npts; idx += (size_t)gridDim.x * blockDim.x) {
    const int e = (int)(idx / N.n_per), a = (int)(idx % N.n_per);
    double lx[kMaxNp], ly[kMaxNp];
    lagrange_weights(N, N.a[a], lx);
    lagrange_weights(N, N.b[a], ly);
    double U[4] = {0.0, 0.0, 0.0, 0.0};
    const size_t base = (size_t)e * N.np * N.np;
    for (int j = 0; j < N.np; ++j)
      for (int i = 0; i < N.np; ++i) {
        const double w = lx[i] * ly[j];
        for (int c = 0; c < 4; ++c) U[c] += w * u[c * cs + base + i + N.np * j];
      }
    const double r = fmax(U[0], kEps);
    const double uu = U[1] / r, vv = U[2] / r;
    f[0 * npts + idx] = U[0];
    f[1 * npts + idx] = uu;
    f[2 * npts + idx] = vv;
    f[3 * npts + idx] = (gamma - 1.0) * (U[3] - 0.5 * r * (uu * uu + vv * vv));
    f[4 * npts + idx] = U[1];
    f[5 * npts + idx] = U[2];
    f[6 * npts + idx] = U[3];
    const int gx = e % M.nx, gy = e / M.nx;
    double X = M.xc[gx] + M.Jx[gx] * N.a[a];
    double Y = M.yc[gy] + M.Jy[gy] * N.b[a];
    if (M.wavy) {
      const double X0 = X;
      X = X0 + M.amp * sin(2.0 * M_PI * Y) * sin(M_PI * X0);
      Y = Y + M.amp * sin(2.0 * M_PI * X0) * sin(M_PI * Y);
    }
    xy[idx] = X;
    xy[npts + idx] = Y;
  }
}

__global__ void vtk_points_1d(const double* __restrict__ u, const Mesh1Dev M, const VtkNodes N, double gamma,
                              double* __restrict__ xy, double* __restrict__ f) {
  const size_t npts = (size_t)M.nel * N.n_per;
  const size_t cs = (size_t)M.nel * N.np;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < npts; idx += (size_t)gridDim.x * blockDim.x) {
    const int e = (int)(idx / N.n_per), a = (int)(idx % N.n_per);
    double l[kMaxNp];
    lagrange_weights(N, N.a[a], l);
    double U[3] = {0.0, 0.0, 0.0};
    for (int k = 0; k < N.np; ++k)
      for (int c = 0; c < 3; ++c) U[c] += l[k] * u[c * cs + (size_t)e * N.np + k];
    const double r = fmax(U[0], kEps);
    const double uu = U[1] / r;
    f[0 * npts + idx] = U[0];
    f[1 * npts + idx] = uu;
    f[2 * npts + idx] = (gamma - 1.0) * (U[2] - 0.5 * r * uu * uu);
    f[3 * npts + idx] = U[1];
    f[4 * npts + idx] = U[2];
    xy[idx] = M.xc[e] + M.J[e] * N.a[a];
  }
}

}  // namespace
}  // namespace frg

using namespace frg;
using namespace frg::rt;

extern "C" int frg_vtk_point_data(frg_solve* s, int n_per, const double* node_xi, const double* node_eta,
                                  double* xy, double* fields, size_t n_points) {
  if (!s || !node_xi || !xy || !fields) return FRG_ERR_INVALID_ARG;
  if (!s->have_state) return set_err(s->ctx, FRG_ERR_STATE, "no state uploaded");
  const bool is2 = s->dim == 2;
  const int want = is2 ? s->np * s->np : s->np;
  if (n_per != want || (is2 && !node_eta))
    return set_err(s->ctx, FRG_ERR_INVALID_ARG, "n_per must be (p+1)^dim with eta nodes in 2D");
  if (n_points != (size_t)s->nel * n_per) return set_err(s->ctx, FRG_ERR_INVALID_ARG, "n_points != nel * n_per");
  if (is2 && s->L2.mesh.curved && !s->L2.mesh.wavy)
    return set_err(s->ctx, FRG_ERR_INVALID_ARG, "node coordinates need an affine or analytic wavy mesh");
  VtkNodes N;
  std::memset(&N, 0, sizeof(N));
  N.np = s->np;
  N.n_per = n_per;
  for (int i = 0; i < s->np; ++i) N.xi[i] = s->ops.xi[i];
  for (int k = 0; k < n_per; ++k) {
    N.a[k] = node_xi[k];
    N.b[k] = is2 ? node_eta[k] : 0.0;
  }
  cudaSetDevice(s->ctx->device);
  cudaStream_t st = s->ctx->stream;
  const int nf = is2 ? 7 : 5, nc = is2 ? 2 : 1;
  double* d = nullptr;
  cudaError_t e = cudaMallocAsync((void**)&d, sizeof(double) * n_points * (nf + nc), st);
  if (e != cudaSuccess) return cuda_err(s->ctx, e, "vtk point data");
  double* dxy = d;
  double* df = d + n_points * nc;
  const int blocks = (int)std::min<size_t>((n_points + 255) / 256, (size_t)4 * 148 * 8);
  const double* u = s->U[s->cur];
  if (is2)
    vtk_points_2d<<<blocks, 256, 0, st>>>(u, s->L2.mesh, N, s->L2.phys.gamma, dxy, df);
  else
    vtk_points_1d<<<blocks, 256, 0, st>>>(u, s->L1.mesh, N, s->L1.phys.gamma, dxy, df);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(xy, dxy, sizeof(double) * n_points * nc, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(fields, df, sizeof(double) * n_points * nf, cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(d, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return cuda_err(s->ctx, e, "vtk point data");
}

// Device-side set-up of a solve: analytic wavy-mesh metrics and the
// reference's case initial conditions, evaluated where the state lives, so
// that admitting a large request costs no host loop over its points and no
// upload of its state.
//
//   build_mesh_metrics_analytic_wavy   MeshMetrics2D.jl:327-442
//   wavy_physical / wavy_partials      MeshMetrics2D.jl:299-318
//   set_initial_condition!             SolutionState.jl:59-73, SolutionState2D.jl:58-82
//   sod_ic / shu_osher_ic              Cases.jl:930-946
//   euler_density_wave_conserved       Cases.jl:404-414
//   riemann2d_ic (quadrant rule)       Cases2D_Riemann.jl:33-51
//   isentropic_vortex_primitives       Cases2D_Riemann.jl:163-186
//   smooth order-test wave             Cases2D_Smooth.jl:124-135
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "frg_device.cuh"
#include "frg_runtime.h"

namespace frg {
namespace {

constexpr int kSetupThreads = 256;
constexpr double kTwoPi = 6.283185307179586, kPi = 3.141592653589793;

struct NodeTable {
  double xi[kMaxNp];
};

__device__ __forceinline__ void wavy_partials_dev(double X, double Y, double a, double* xX, double* xY, double* yX,
                                                  double* yY) {
  *xX = 1.0 + a * sin(kTwoPi * Y) * kPi * cos(kPi * X);
  *xY = a * kTwoPi * cos(kTwoPi * Y) * sin(kPi * X);
  *yX = a * kTwoPi * cos(kTwoPi * X) * sin(kPi * Y);
  *yY = 1.0 + a * sin(kTwoPi * X) * kPi * cos(kPi * Y);
}

// metric fields at the solution points, element-major [e][i + np j]
__global__ void wavy_sp_kernel(int nel, int nx, int np, const double* xc, const double* Jx, const double* yc,
                               const double* Jy, NodeTable T, double amp, double* xxi, double* xeta, double* yxi,
                               double* yeta, double* rJ) {
  const size_t n = (size_t)nel * np * np;
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    const int e = (int)(k / (np * np)), r = (int)(k % (np * np));
    const int i = r % np, j = r / np;
    const int jx = e % nx, jy = e / nx;
    const double X = xc[jx] + Jx[jx] * T.xi[i], Y = yc[jy] + Jy[jy] * T.xi[j];
    double a, b, c2, d2;
    wavy_partials_dev(X, Y, amp, &a, &b, &c2, &d2);
    const double vxx = a * Jx[jx], vxe = b * Jy[jy], vyx = c2 * Jx[jx], vye = d2 * Jy[jy];
    xxi[k] = vxx;
    xeta[k] = vxe;
    yxi[k] = vyx;
    yeta[k] = vye;
    rJ[k] = 1.0 / (vxx * vye - vxe * vyx);
  }
}

// unit normals and surface Jacobians at the face points [e][q], faces W E S N
struct FaceOut {
  double* nx[4];
  double* ny[4];
  double* sJ[4];
};

__global__ void wavy_face_kernel(int nel, int nx, int np, const double* xc, const double* Jx, const double* yc,
                                 const double* Jy, NodeTable T, double amp, FaceOut F) {
  const size_t n = (size_t)nel * np;
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    const int e = (int)(k / np), q = (int)(k % np);
    const int jx = e % nx, jy = e / nx;
    const double Y = yc[jy] + Jy[jy] * T.xi[q], X = xc[jx] + Jx[jx] * T.xi[q];
    double a, b, c2, d2;
    // west / east: n ~ (-y_eta, x_eta) / (y_eta, -x_eta)
    for (int side = 0; side < 2; ++side) {
      wavy_partials_dev(xc[jx] + Jx[jx] * (side ? 1.0 : -1.0), Y, amp, &a, &b, &c2, &d2);
      const double xe = b * Jy[jy], ye = d2 * Jy[jy];
      const double sJ = fmax(sqrt(ye * ye + xe * xe), kEps);
      F.nx[side][k] = side ? ye / sJ : -ye / sJ;
      F.ny[side][k] = side ? -xe / sJ : xe / sJ;
      F.sJ[side][k] = sJ;
    }
    // south / north: n ~ (y_xi, -x_xi) / (-y_xi, x_xi)
    for (int side = 0; side < 2; ++side) {
      wavy_partials_dev(X, yc[jy] + Jy[jy] * (side ? 1.0 : -1.0), amp, &a, &b, &c2, &d2);
      const double xx = a * Jx[jx], yx = c2 * Jx[jx];
      const double sJ = fmax(sqrt(yx * yx + xx * xx), kEps);
      F.nx[2 + side][k] = side ? -yx / sJ : yx / sJ;
      F.ny[2 + side][k] = side ? xx / sJ : -xx / sJ;
      F.sJ[2 + side][k] = sJ;
    }
  }
}

// ------------------------------------------------------------------ ICs
struct IcDev {
  int kind;
  double x0, y0, amp, phase, t;
  double prim[4][4];
};

__device__ __forceinline__ void prim2cons2_dev(double g, const double* P, double* U) {
  const double r = P[0], u = P[1], v = P[2], p = P[3];
  U[0] = r;
  U[1] = r * u;
  U[2] = r * v;
  U[3] = p / (g - 1.0) + 0.5 * r * (u * u + v * v);
}
__device__ __forceinline__ void prim2cons1_dev(double g, const double* P, double* U) {
  const double r = P[0], u = P[1], p = P[2];
  U[0] = r;
  U[1] = r * u;
  U[2] = p / (g - 1.0) + 0.5 * r * u * u;
}

__device__ void ic2d(const IcDev& c, double g, double x, double y, double* U) {
  double P[4];
  switch (c.kind) {
    case FRG_IC_TWO_STATE: {
      const double* s = x < c.x0 ? c.prim[0] : c.prim[1];
      for (int k = 0; k < 4; ++k) P[k] = s[k];
      break;
    }
    case FRG_IC_FOUR_QUADRANT: {
      const double* s;
      if (x >= c.x0 && y >= c.y0)
        s = c.prim[0];  // ne
      else if (x < c.x0 && y >= c.y0)
        s = c.prim[1];  // nw
      else if (x < c.x0 && y < c.y0)
        s = c.prim[2];  // sw
      else
        s = c.prim[3];  // se
      for (int k = 0; k < 4; ++k) P[k] = s[k];
      break;
    }
    case FRG_IC_DENSITY_WAVE:
      for (int k = 0; k < 4; ++k) P[k] = c.prim[0][k];
      P[0] = c.prim[0][0] + c.amp * sin(kTwoPi * (x + y - c.t) + c.phase);
      break;
    case FRG_IC_VORTEX: {
      const double beta = 5.0, x0 = 5.0, y0 = 5.0, uinf = 1.0, vinf = 1.0, gv = 1.4;
      const double xd = x - x0 - uinf * c.t, yd = y - y0 - vinf * c.t;
      const double r2 = xd * xd + yd * yd;
      const double ef = exp(0.5 * (1.0 - r2));
      const double b2pi = beta / kTwoPi;
      const double du = -b2pi * ef * yd, dv = b2pi * ef * xd;
      double T = 1.0 - (gv - 1.0) * (beta * beta) / (8.0 * gv * (kPi * kPi)) * exp(1.0 - r2);
      T = jmax(T, 1e-14);
      P[0] = pow(T, 1.0 / (gv - 1.0));
      P[1] = uinf + du;
      P[2] = vinf + dv;
      P[3] = pow(P[0], gv);
      break;
    }
    case FRG_IC_SMOOTH_2D:
      P[0] = 1.0 + 0.2 * sin(kTwoPi * (x - c.t)) * sin(kTwoPi * (y - c.t));
      P[1] = 1.0;
      P[2] = 1.0;
      P[3] = 1.0;
      break;
    default:  // uniform
      for (int k = 0; k < 4; ++k) P[k] = c.prim[0][k];
  }
  prim2cons2_dev(g, P, U);
}

__device__ void ic1d(const IcDev& c, double g, double x, double* U) {
  double P[3];
  switch (c.kind) {
    case FRG_IC_TWO_STATE: {
      const double* s = x < c.x0 ? c.prim[0] : c.prim[1];
      for (int k = 0; k < 3; ++k) P[k] = s[k];
      break;
    }
    case FRG_IC_DENSITY_WAVE:
      for (int k = 0; k < 3; ++k) P[k] = c.prim[0][k];
      P[0] = c.prim[0][0] + c.amp * sin(kTwoPi * (x - c.t) + c.phase);
      break;
    case FRG_IC_SHU_OSHER:
      if (x < 1.0) {
        P[0] = 3.857143;
        P[1] = 2.629369;
        P[2] = 10.33333;
      } else {
        P[0] = 1.0 + 0.2 * sin(5.0 * (x - 5.0));
        P[1] = 0.0;
        P[2] = 1.0;
      }
      break;
    default:  // uniform
      for (int k = 0; k < 3; ++k) P[k] = c.prim[0][k];
  }
  prim2cons1_dev(g, P, U);
}

__global__ void ic2d_kernel(double* u, const Mesh2Dev M, NodeTable T, int np, double g, IcDev c) {
  const size_t n = (size_t)M.nel * np * np;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
    const int e = (int)(idx / (np * np)), r = (int)(idx % (np * np));
    const int i = r % np, j = r / np;
    const int gx = e % M.nx, gy = e / M.nx;
    // physical_xy, MeshMetrics2D.jl:49-74
    const double X = M.xc[gx] + M.Jx[gx] * T.xi[i], Y = M.yc[gy] + M.Jy[gy] * T.xi[j];
    double x = X, y = Y;
    if (M.wavy) {
      x = X + M.amp * sin(kTwoPi * Y) * sin(kPi * X);
      y = Y + M.amp * sin(kTwoPi * X) * sin(kPi * Y);
    }
    double U[4];
    ic2d(c, g, x, y, U);
    for (int k = 0; k < 4; ++k) u[k * n + idx] = U[k];
  }
}

__global__ void ic1d_kernel(double* u, const Mesh1Dev M, NodeTable T, int np, double g, IcDev c) {
  const size_t n = (size_t)M.nel * np;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
    const int e = (int)(idx / np), j = (int)(idx % np);
    double U[3];
    ic1d(c, g, M.xc[e] + M.J[e] * T.xi[j], U);
    for (int k = 0; k < 3; ++k) u[k * n + idx] = U[k];
  }
}

int grid_for(size_t n) {
  const size_t b = (n + kSetupThreads - 1) / kSetupThreads;
  return (int)(b < 4096 ? (b ? b : 1) : 4096);
}

}  // namespace

int launch_wavy_metrics(int nel, int nx, int np, const double* xc, const double* Jx, const double* yc,
                        const double* Jy, const double* xi, double amp, double* xxi, double* xeta, double* yxi,
                        double* yeta, double* rJ, double* const fnx[4], double* const fny[4],
                        double* const fsJ[4], void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  NodeTable T;
  std::memset(&T, 0, sizeof(T));
  for (int i = 0; i < np; ++i) T.xi[i] = xi[i];
  FaceOut F;
  for (int f = 0; f < 4; ++f) {
    F.nx[f] = fnx[f];
    F.ny[f] = fny[f];
    F.sJ[f] = fsJ[f];
  }
  wavy_sp_kernel<<<grid_for((size_t)nel * np * np), kSetupThreads, 0, st>>>(nel, nx, np, xc, Jx, yc, Jy, T, amp, xxi,
                                                                          xeta, yxi, yeta, rJ);
  wavy_face_kernel<<<grid_for((size_t)nel * np), kSetupThreads, 0, st>>>(nel, nx, np, xc, Jx, yc, Jy, T, amp, F);
  return (int)cudaGetLastError();
}

}  // namespace frg

using namespace frg;
using namespace frg::rt;

extern "C" int frg_set_initial_condition(frg_solve* s, const frg_ic* ic) {
  if (!s || !ic) return FRG_ERR_INVALID_ARG;
  const bool is2 = s->dim == 2;
  switch (ic->kind) {
    case FRG_IC_UNIFORM:
    case FRG_IC_TWO_STATE:
    case FRG_IC_DENSITY_WAVE:
      break;
    case FRG_IC_FOUR_QUADRANT:
    case FRG_IC_VORTEX:
    case FRG_IC_SMOOTH_2D:
      if (!is2) return set_err(s->ctx, FRG_ERR_INVALID_ARG, "2D initial condition on a 1D solve");
      break;
    case FRG_IC_SHU_OSHER:
      if (is2) return set_err(s->ctx, FRG_ERR_INVALID_ARG, "1D initial condition on a 2D solve");
      break;
    default:
      return set_err(s->ctx, FRG_ERR_INVALID_ARG, "unknown initial condition");
  }
  if (is2 && s->L2.mesh.curved && !s->L2.mesh.wavy)
    return set_err(s->ctx, FRG_ERR_INVALID_ARG, "initial condition needs point coordinates (caller metrics)");
  cudaSetDevice(s->ctx->device);
  IcDev c;
  std::memset(&c, 0, sizeof(c));
  c.kind = ic->kind;
  c.x0 = ic->x0;
  c.y0 = ic->y0;
  c.amp = ic->amp;
  c.phase = ic->phase;
  c.t = ic->t;
  std::memcpy(c.prim, ic->prim, sizeof(c.prim));
  NodeTable T;
  std::memset(&T, 0, sizeof(T));
  for (int i = 0; i < s->np; ++i) T.xi[i] = s->ops.xi[i];
  const size_t npts = s->ndof / s->neq;
  cudaStream_t st = s->ctx->stream;
  if (is2)
    ic2d_kernel<<<grid_for(npts), kSetupThreads, 0, st>>>(s->U[0], s->L2.mesh, T, s->np, s->L2.phys.gamma, c);
  else
    ic1d_kernel<<<grid_for(npts), kSetupThreads, 0, st>>>(s->U[0], s->L1.mesh, T, s->np, s->L1.phys.gamma, c);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_err(s->ctx, e, "initial condition");
  // set_initial_condition! resets the time (SolutionState.jl:71)
  s->t = 0.0;
  s->cur = 0;
  s->have_state = true;
  s->hsc->t = 0.0;
  return push_scalars(s);
}

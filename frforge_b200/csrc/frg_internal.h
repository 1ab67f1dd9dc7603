// Internal structures shared by the host runtime and the sm_100a kernels.
#pragma once

#include <cstddef>
#include <cstdint>

#include "../../include/frforge_cuda.h"

namespace frg {

constexpr double kEps = 2.220446049250313e-16;  // Julia eps(Float64)
constexpr int kMaxNp = FRG_MAX_NP;

// Boundary condition as seen by the kernels.
struct BCDev {
  int kind;
  int mode;
  double st[4];
  double stb[4];
  double x0, s0, s1, sdiv;
};

// Reference-element tables, derived on the host from FROperators.
//   Dt  = D - gL_xi l_L^T - gR_xi l_R^T   (divergence with the g_DG lift folded in)
//   DtD = Dt * D                           (BR0 volume term acting on u)
//   DD  = D * D                            (element-local D(Du) dissipation)
//   lLD = l_L^T D, lRD = l_R^T D           (face traces of D u)
//   Vinv = V^{-1}                           (modal coefficients of the sensor)
// Row-major [i][k] so that a thread computing output i reads a contiguous row.
template <int NP>
struct OpsT {
  double Dt[NP][NP];
  double DtD[NP][NP];
  double DD[NP][NP];
  double Vinv[NP][NP];
  double lL[NP], lR[NP], lLD[NP], lRD[NP], gL[NP], gR[NP];
  double xi[NP];
  double w[NP];  // quadrature weights (element means)
};

// Host copy of all tables for one (p, points) pair (NP <= kMaxNp).
struct HostOps {
  int p = 0, np = 0, points = 0;
  double xi[kMaxNp], w[kMaxNp];
  double D[kMaxNp][kMaxNp];  // row-major D[i][k]
  double lL[kMaxNp], lR[kMaxNp], gLxi[kMaxNp], gRxi[kMaxNp], gL[kMaxNp], gR[kMaxNp];
  double V[kMaxNp][kMaxNp];  // V[j][k] = P_k(xi_j)
  // derived
  double Dt[kMaxNp][kMaxNp], DtD[kMaxNp][kMaxNp], DD[kMaxNp][kMaxNp], Vinv[kMaxNp][kMaxNp];
  double lLD[kMaxNp], lRD[kMaxNp];
};

// 2D mesh on the device.  Affine meshes keep only per-column / per-row
// spacing; curved meshes add per-solution-point metric fields and
// per-face-point normals (the MeshMetrics2D arrays).
struct Mesh2Dev {
  int nx, ny, nel;
  int px, py;  // periodic in x / y
  const double* xc;  // [nx] column centres (xL+xR)/2
  const double* Jx;   // [nx] dx/2
  const double* rJx;  // [nx] 1/Jx
  const double* yc;
  const double* Jy;
  const double* rJy;  // [ny] 1/Jy
  const double* hchar;  // [nel]
  int curved;
  const double* m_xxi;  // [nel*np2] per SP, element-major
  const double* m_xeta;
  const double* m_yxi;
  const double* m_yeta;
  const double* m_rJ;     // 1/J
  const double* f_nx[4];  // [nel*np] per face point; faces W,E,S,N
  const double* f_ny[4];
  const double* f_sJ[4];
  const unsigned char* solid;  // [nel] or null
  int wavy;
  double amp;
  BCDev bc[4];  // left right bottom top
};

struct Mesh1Dev {
  int nel;
  int periodic;
  const double* xc;  // [nel] element centres
  const double* J;   // [nel] dx/2
  const double* dx;  // [nel]
  BCDev bc[2];
};

// Per-solve device scalars: time, dt, loop control and status word.
struct DevScalars {
  double t;        // time of the state in buffer 0
  double t0;       // step start time
  double dt;       // dt of the step in flight
  double t_final;
  double cfl;
  double fixed_dt;  // > 0: fixed step
  double hmin;      // 2D: min h_char; 1D: min dx
  unsigned long long lam_bits;  // max wave speed of the current state (non-negative double bits)
  unsigned int flags;           // bit0: du non-finite, bit1: state non-finite
  int status;                   // 0 running, FRG_DIVERGED, FRG_MAX_STEPS, 3 finished
  int active;                   // the step in flight runs
  int diverged_stage;           // 1..3, 4 = end-of-step state check
  int two_p1;                   // 2p+1
  int stepped_ok;               // the last step ran and did not diverge (post-step hooks)
  long long n_steps;
  long long max_steps;
  long long residual_evals;
  // launches of each hook slot's kernel that passed their gate (indexed by
  // FRG_HOOK_*); counted on the device and never overwritten from the host
  long long hook_calls[4];
};

enum : int { kRunning = 0, kFinished = 3 };

// device hook implementations (frg_hooks.cu)
enum : int {
  kHookNone = 0,
  kHookPositivity = 1,       // post_step: Zhang-Shu positivity scaling
  kHookFluxRusanov = 2,      // numerical_flux: Rusanov, dissipation scaled by a parameter
  kHookFluxHLLC = 3,         // numerical_flux: HLLC
  kHookPrePositivity = 4,    // preprocess_state: Zhang-Shu scaling of the work state
  kHookTraceMean = 5,        // extrapolate_interface: traces pulled toward the element mean
  kHookTracePositivity = 6,  // extrapolate_interface: Zhang-Shu scaling of the traces
};

// Stage kernel launch parameters (shared by the 1D and 2D kernels).
struct StageBufs {
  const double* us;   // stage input state
  const double* u0;   // step-start state (stages 2, 3)
  double* uout;       // output state (may alias u0)
  double* du_out;     // residual-only output
  const double* eps_in;
  double* eps_out;
  double a, b, c;  // u_new = a*u0 + b*us + (c*dt)*du
  int stage;       // 1..3 (time offset 0, dt, dt/2 for RK3; 0, dt for RK2)
  int mode;        // kModeStage / kModeResidual / kModePrime / kModeSense
  int rk2;
  int want_lambda;  // accumulate the CFL wave speed of the output state
  int want_eps;     // compute the element viscosity of the output state
  int use_sc;       // honour DevScalars active/flags (graph execution)
  DevScalars* sc;
  double* sigma_out;  // kModeSense
  // residual input when a preprocess_state hook is selected (the work state
  // u_work); null: the residual is evaluated on us itself
  const double* uw;
};

enum : int { kModeStage = 0, kModeResidual = 1, kModePrime = 2, kModeSense = 3 };

struct Phys {
  double gamma, g1;  // gamma, gamma-1
  double c_av, kappa, s0, eps_floor;
  // 1D interface flux: dissipation scale of the Rusanov flux (1 except under
  // a numerical_flux_method override that scales it)
  double flux_alpha;
  // 1D interface traces: extrapolate_interface override (kHookTrace*, 0:
  // the Lagrange traces) and its two parameters
  double trace_p0, trace_p1;
  int trace_hook;
  int p, pm;  // p, max(p,1)
};

enum : int { kAvNone = 0, kAvBR0 = 1, kAvDD = 2 };

// static shared memory the batched stage kernels hold for their descriptors
constexpr int kBatchStaticSmem = 1024;

// One instance of a batch, as the batched kernels see it.
struct BatchInst {
  Mesh2Dev M2;  // dim == 2
  Mesh1Dev M1;  // dim == 1
  Phys P;
  double* U[3];
  double* E[3];
  DevScalars* sc;
  int rk2;
  int dim;
  int hook;              // post-step hook id (kHookNone: none)
  int hook_pad;
  double hook_params[2];  // kHookPositivity: eps_rho, eps_p
};
// A tile of one instance: first element (x0, y0) of a TX x TY tile.
struct BatchTile {
  int inst, x0, y0, pad;
};
// Per-instance outcome gathered for the host in one copy.
struct BatchStatus {
  int status;
  int active;
  long long n_steps;
  double t;
};

// ---- device set-up (frg_setup.cu) ----
// analytic wavy metrics (MeshMetrics2D.jl:327-442) into device arrays;
// returns 0 or a CUDA error code
int launch_wavy_metrics(int nel, int nx, int np, const double* xc, const double* Jx, const double* yc,
                        const double* Jy, const double* xi, double amp, double* xxi, double* xeta, double* yxi,
                        double* yeta, double* rJ, double* const fnx[4], double* const fny[4],
                        double* const fsJ[4], void* stream);

// ---- host helpers (frg_host.cpp) ----
int build_host_ops(int p, int points, HostOps* out);
int host_ops_from_caller(const frg_operators* in, HostOps* out);
void derive_tables(HostOps* o);
void julia_linspace(double a, double b, int len, double* out);

// ---- kernel launchers (frg_launch_np*.cu) ----
struct Launch2D {
  const HostOps* ops;
  Mesh2Dev mesh;
  Phys phys;
  int flux;     // FRG_FLUX_*
  int av;       // kAv*
  int variant;  // tile variant (autotuned)
};
struct Launch1D {
  const HostOps* ops;
  Mesh1Dev mesh;
  Phys phys;
  int flux;
  int av;
};
// The stage buffers of one SSP-RK step, for the whole-solve 1D loop kernel.
struct Loop1DBufs {
  StageBufs st[3];
  int nstages;
  int pad;
};
// Largest 1D mesh, in tiles, that one thread-block cluster steps by itself
// (one tile per CTA; 8 is the portable cluster size).
constexpr int kLoop1DMaxTiles = 8;
// Largest cluster of the narrowest 1D loop tiles (a non-portable size, used
// only where the device can schedule it).
constexpr int kLoop1DMaxCluster = 16;
// Returns 0 or a CUDA error code.
int launch_stage2d(const Launch2D& L, const StageBufs& b, void* stream);
// batched stage launch over a group's tile list (same NP, flux, AV, tables)
int launch_batch2d(const HostOps* ops, int flux, int av, int variant, const BatchInst* insts,
                   const BatchTile* tiles, int ntiles, int stage, int mode, void* stream);
int launch_batch1d(const HostOps* ops, int flux, int av, const BatchInst* insts,
                   const BatchTile* tiles, int ntiles, int stage, int mode, void* stream);
// Tile shape of the batched kernels; returns their CTAs per SM (2D), 1 (1D)
// or -1 (unsupported NP).
int batch_tile_shape(int dim, int np, int variant, int* tx, int* ty);
int launch_stage1d(const Launch1D& L, const StageBufs& b, void* stream);
int stage2d_variants(int np);
// persisted autotune table (frg_autotune.cpp), keyed by (p, FRG_FLUX_*,
// kAv*, curved): lookup returns 1 and the variant if present
int autotune_table_lookup(int p, int flux, int av, int curved, int* variant);
void autotune_table_record(int p, int flux, int av, int curved, int variant, double ms);

}  // namespace frg

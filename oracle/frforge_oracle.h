/*
 * FRForge CPU oracle -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C FP64 restatement of FRForge's FR residual + SSP-RK time-step path
 * (Julia sources: src/fr, src/flux, src/capturing, src/equations, src/mesh,
 * src/solvestate, src/time).  Loop order and arithmetic order follow the
 * Julia code; the build uses -ffp-contract=off so no multiply-add is fused,
 * matching Julia's default (non-@fastmath) Float64 semantics.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
 * this library, and only as the checker / the timed CPU baseline.  The
 * product path (frforge_b200) never links or calls it.
 *
 * Parity pins: see tests/test_oracle_golden.py (golden values recorded in
 * the reference's own tests and fixtures, test/test_2d.jl:316-321,
 * the snapshot_fixture JSON files and test/data/shu_osher_ref.csv).
 */
#ifndef FRFORGE_ORACLE_H
#define FRFORGE_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAXNP 8

/* scheme axes (src/scheme/SchemeConfig.jl:15-31) */
enum { ORC_POINTS_GL = 0, ORC_POINTS_GLL = 1 };
enum { ORC_FLUX_RUSANOV = 0, ORC_FLUX_HLLC = 1 };
enum { ORC_TIME_SSP_RK3 = 0, ORC_TIME_SSP_RK2 = 1 };
/* boundary conditions (src/mesh/BoundaryConditions.jl) */
enum {
  ORC_BC_PERIODIC = 0,
  ORC_BC_TRANSMISSIVE = 1,
  ORC_BC_DIRICHLET = 2,
  ORC_BC_REFLECTING = 3,
  /* GhostStateBC restricted to the x-split form used by the double-Mach case
     (src/verification/Cases2D_Optional.jl:72-84): ghost = A for
     x < x0 + (s0 + s1*t), else (mode 0: reflect interior, mode 1: state B) */
  ORC_BC_XSPLIT = 4
};
/* capturing methods (src/capturing/Interfaces.jl, PerssonAV.jl) */
enum { ORC_METHOD_NULL = 0, ORC_METHOD_PERSSON = 1 };
enum { ORC_AV_BR0 = 0, ORC_AV_LOCAL_DD = 1 };
/* step status (src/time/SSP_RK3.jl:44-64, :110-117) */
enum { ORC_OK = 0, ORC_DIVERGED = 1, ORC_MAX_STEPS = 2 };

typedef struct {
  int p, np, points;
  double xi[ORC_MAXNP], w[ORC_MAXNP];
  double D[ORC_MAXNP * ORC_MAXNP]; /* column-major: D[i + np*k] = D[i,k] */
  double lL[ORC_MAXNP], lR[ORC_MAXNP];
  double gLxi[ORC_MAXNP], gRxi[ORC_MAXNP];
  double gL[ORC_MAXNP], gR[ORC_MAXNP];
  double V[ORC_MAXNP * ORC_MAXNP]; /* V[j + np*k] = P_k(xi_j) */
} orc_ops;

typedef struct {
  int kind;          /* ORC_BC_* */
  int mode;          /* x-split right side: 0 reflect interior, 1 state B */
  double state[4];   /* Dirichlet state / x-split state A */
  double state_b[4]; /* x-split state B */
  /* x-split position: x_split(t) = x0 + (s0 + s1*t) / sdiv */
  double x0, s0, s1, sdiv;
} orc_bc;

typedef struct orc_solver orc_solver;

int orc_build_operators(int p, int points, orc_ops* out);

/* 1D solver on a uniform mesh [xl, xr] with nel elements (src/mesh/Mesh1D.jl:23-42) */
orc_solver* orc_create_1d(int p, int points, int nel, double xl, double xr,
                          const orc_bc* left, const orc_bc* right, double gamma,
                          int flux, int time_scheme, int method, int av_form,
                          double kappa, double s0_factor, double eps_floor,
                          double c_av);
/* 2D solver on a structured nx x ny mesh (src/mesh/Mesh2D.jl:98-154), optional
   analytic wavy metrics (src/mesh/MeshMetrics2D.jl:327-442) when wavy != 0 */
orc_solver* orc_create_2d(int p, int points, int nx, int ny, double xl,
                          double xr, double yb, double yt, const orc_bc* bcs4,
                          const unsigned char* solid, int wavy, double amp,
                          double gamma, int flux, int time_scheme, int method,
                          int av_form, double kappa, double s0_factor,
                          double eps_floor, double c_av);
void orc_destroy(orc_solver* s);

void orc_get_ops(const orc_solver* s, orc_ops* out);
size_t orc_ndof(const orc_solver* s);
double* orc_state(orc_solver* s); /* u, Julia column-major layout */
double orc_get_time(const orc_solver* s);
void orc_set_time(orc_solver* s, double t);
/* 2D metric arrays; name in {"x","y","x_xi","x_eta","y_xi","y_eta","J",
   "nx_W","ny_W","sJ_W",... "sJ_N","h_char"}; returns NULL if unknown */
const double* orc_metric(const orc_solver* s, const char* name);
void orc_physical_coords(const orc_solver* s, double* x, double* y);

void orc_set_threads(int n);

void orc_residual(orc_solver* s, double* du);
void orc_sense(orc_solver* s, double* sigma);
double orc_compute_dt(orc_solver* s, double cfl);
int orc_step(orc_solver* s, double dt);
int orc_integrate(orc_solver* s, double t_final, double cfl, double fixed_dt,
                  int64_t max_steps, int64_t* n_steps);

/* diagnostics (src/solvestate, src/equations, src/verification/Metrics.jl) */
double orc_discrete_mass(const orc_solver* s, int c);
int orc_positivity_ok(const orc_solver* s);
int orc_has_nonfinite(const double* a, size_t n);
void orc_solution_extrema(const orc_solver* s, int c, double* umin,
                          double* umax);

/* reference initial conditions */
void orc_ic_sod(orc_solver* s);
void orc_ic_shu_osher(orc_solver* s);
void orc_ic_density_wave_1d(orc_solver* s, double t);
void orc_ic_two_state_1d(orc_solver* s, double x0, const double* primL,
                         const double* primR);
void orc_ic_vortex_2d(orc_solver* s, double t);
void orc_ic_smooth_2d(orc_solver* s);
void orc_ic_four_quadrant_2d(orc_solver* s, double x0, double y0,
                             const double* ne, const double* nw,
                             const double* sw, const double* se);
void orc_ic_uniform(orc_solver* s, const double* prim);
double orc_l2_error_vortex(const orc_solver* s, double t);
double orc_l2_error_smooth_2d(const orc_solver* s, double t);
double orc_l2_error_density_wave_1d(const orc_solver* s, double t);

/* numerical_flux_method override of the 1D residual: kind -1 none,
   ORC_FLUX_RUSANOV (dissipation scaled by alpha) or ORC_FLUX_HLLC */
void orc_set_flux_override(orc_solver* s, int kind, double alpha);
/* A 1D method's extrapolate_interface! override: ORC_TRACE_NONE (0) clears
   it; ORC_TRACE_MEAN (p0 = theta) pulls each element's traces toward its
   mean; ORC_TRACE_POSITIVITY (p0 = eps_rho, p1 = eps_p) scales them
   (Zhang-Shu).  Only the interface fluxes use the traces. */
enum { ORC_TRACE_NONE = 0, ORC_TRACE_MEAN = 1, ORC_TRACE_POSITIVITY = 2 };
void orc_set_trace_override(orc_solver* s, int kind, double p0, double p1);
/* 1D: the traces the last orc_residual's interface fluxes used, [nel,3] each */
void orc_get_traces_1d(const orc_solver* s, double* trL, double* trR);

/* single-interface fluxes (unit checks) */
void orc_hllc_1d(double gamma, const double* uL, const double* uR, double* out);
void orc_rusanov_1d(double gamma, const double* uL, const double* uR,
                    double* out);
void orc_hllc_2d(double gamma, const double* uL, const double* uR, double nx,
                 double ny, double* out);
void orc_rusanov_2d(double gamma, const double* uL, const double* uR,
                    double nx, double ny, double* out);

#ifdef __cplusplus
}
#endif
#endif

/*
 * frforge_cuda.h -- C ABI of the B200 (sm_100a) FR residual + SSP-RK library.
 *
 * This is the drop-in boundary for FRForge's hot path.  Each entry point
 * names the Julia function it replaces (paths are relative to the FRForge
 * source tree).  Conventions:
 *   - every function returns an int status (frg_status); numerical outcomes
 *     of a time integration (ok / diverged / max_steps) are reported in
 *     frg_result.status exactly like the Symbol returned by ssp_rk3!
 *     (src/time/SSP_RK3.jl:110-117); configuration errors map to
 *     FRG_ERR_INVALID_ARG (Julia's ArgumentError, src/scheme/SchemeConfig.jl:26-29);
 *   - arrays use FRForge's Julia layout: u[j,e,c] (1D) / u[i,j,e,c] (2D),
 *     column-major, FP64 -- so upload/download are plain copies;
 *   - the library owns all device memory of a solve; host buffers are owned
 *     by the caller and only read/written during the call;
 *   - calls on one solve are serialised on that solve's CUDA stream; one
 *     frg_ctx per host thread.
 */
#ifndef FRFORGE_CUDA_H
#define FRFORGE_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FRG_ABI_VERSION 1
#define FRG_MAX_NP 6 /* P <= 5 */
/* size limits of frg_residual2d_noalloc's fixed device scratch */
#define FRG_NOALLOC_MAX_ELEMENTS 262144
#define FRG_NOALLOC_MAX_SIDE 4096

/* Status codes.  Numerical statuses mirror :ok / :diverged / :max_steps
   (src/time/SSP_RK3.jl:44-64, :110-117). */
typedef enum {
  FRG_OK = 0,
  FRG_DIVERGED = 1,
  FRG_MAX_STEPS = 2,
  FRG_RUNNING = 3,               /* batched instance still advancing */
  FRG_CANCELLED = 4,             /* served request cancelled */
  FRG_ERR_INVALID_ARG = -1,      /* ArgumentError in the reference */
  FRG_ERR_UNSUPPORTED_HOOK = -2, /* a capturing hook with no GPU implementation */
  FRG_ERR_OOM = -3,              /* device allocation / admission budget */
  FRG_ERR_CUDA = -4,             /* CUDA runtime failure; see frg_last_error */
  FRG_ERR_TIMEOUT = -5,          /* reserved: no entry point waits on the device
                                    with a bound today, so none returns it */
  FRG_ERR_STATE = -6             /* call order (e.g. no state uploaded) */
} frg_status;

/* Scheme axes, src/scheme/SchemeConfig.jl:15-31 */
enum { FRG_POINTS_GL = 0, FRG_POINTS_GLL = 1 };
enum { FRG_FLUX_RUSANOV = 0, FRG_FLUX_HLLC = 1 };
enum { FRG_TIME_SSP_RK3 = 0, FRG_TIME_SSP_RK2 = 1 };

/* Boundary conditions, src/mesh/BoundaryConditions.jl:9-134.  XSPLIT is the
   GhostStateBC shape used by the double-Mach case
   (src/verification/Cases2D_Optional.jl:72-84): ghost = state for
   x < x0 + (s0 + s1*t)/sdiv, else (mode 0) the reflected interior state or
   (mode 1) state_b. */
enum {
  FRG_BC_PERIODIC = 0,
  FRG_BC_TRANSMISSIVE = 1,
  FRG_BC_DIRICHLET = 2,
  FRG_BC_REFLECTING = 3,
  FRG_BC_XSPLIT = 4
};

/* Capturing methods: NullCapturing (src/capturing/Interfaces.jl:21-26) and
   PerssonAVMethod (src/capturing/PerssonAV.jl:53-77); scaled_persson
   (src/methods/ScaledPersson.jl) is PERSSON with c_av = 0.5. */
enum { FRG_METHOD_NULL = 0, FRG_METHOD_PERSSON = 1 };
enum { FRG_AV_BR0 = 0, FRG_AV_LOCAL_DD = 1 };

/* Geometry (2D): affine Cartesian mesh (build_mesh_metrics,
   src/mesh/MeshMetrics2D.jl:82-218), analytic wavy map
   (build_mesh_metrics_analytic_wavy, :327-442), or caller metrics. */
enum { FRG_GEOM_AFFINE = 0, FRG_GEOM_WAVY = 1, FRG_GEOM_METRICS = 2 };

typedef struct {
  int kind; /* FRG_BC_* */
  int mode; /* XSPLIT: 0 reflect interior, 1 state_b */
  double state[4];
  double state_b[4];
  double x0, s0, s1, sdiv;
} frg_bc;

/* Reference-element tables of FROperators (src/fr/Operators.jl:62-77).
   Matrices are np x np column-major (Julia layout). */
typedef struct {
  int p;
  int points;
  const double* xi;    /* np */
  const double* w;     /* np */
  const double* D;     /* np*np, D[i + np*k] = D[i,k] */
  const double* l_L;   /* np */
  const double* l_R;   /* np */
  const double* gL_xi; /* np */
  const double* gR_xi; /* np */
  const double* V;     /* np*np Legendre Vandermonde */
} frg_operators;

/* Per-solve metrics (MeshMetrics2D, src/mesh/MeshMetrics2D.jl:15-39), used
   with FRG_GEOM_METRICS.  SP fields are [np,np,nel]; face fields [np,nel]. */
typedef struct {
  const double *x_xi, *x_eta, *y_xi, *y_eta, *J;
  const double *nx_W, *ny_W, *sJ_W, *nx_E, *ny_E, *sJ_E;
  const double *nx_S, *ny_S, *sJ_S, *nx_N, *ny_N, *sJ_N;
  const double* h_char; /* [nel] */
} frg_metrics2d;

/* Solve descriptor: SchemeConfig + Mesh1D/Mesh2D + metrics + method params. */
typedef struct {
  int dim; /* 1 or 2 */
  int p;
  int points;      /* FRG_POINTS_* */
  int flux;        /* FRG_FLUX_* */
  int time_scheme; /* FRG_TIME_* */
  double gamma;
  int nx, ny; /* 1D: nx = n_elements, ny = 1 */
  double x_left, x_right, y_bottom, y_top;
  const double* x_vertices; /* optional nx+1 (overrides x_left/x_right) */
  const double* y_vertices; /* optional ny+1 */
  frg_bc bc[4];             /* left, right, bottom, top (1D: left, right) */
  const unsigned char* solid; /* optional [nel] solid-element mask (2D) */
  int geometry;               /* FRG_GEOM_* (2D) */
  double wavy_amp;
  const frg_metrics2d* metrics; /* FRG_GEOM_METRICS */
  const frg_operators* ops;     /* optional caller tables (NULL: built here) */
  int method;                   /* FRG_METHOD_* */
  int av_form;                  /* FRG_AV_* */
  double kappa, s0_factor, eps_floor, c_av;
} frg_solve_desc;

typedef struct {
  int status; /* FRG_OK / FRG_DIVERGED / FRG_MAX_STEPS */
  int64_t n_steps;
  double t;
} frg_result;

typedef struct {
  size_t ndof;   /* state length (doubles) */
  int nel, np, neq;
  size_t device_bytes; /* HBM held by this solve */
  int64_t residual_evals; /* residual (stage) evaluations so far */
  int64_t steps;          /* completed time steps so far */
} frg_solve_info;

typedef struct frg_ctx frg_ctx;
typedef struct frg_solve frg_solve;
typedef struct frg_batch frg_batch;
typedef struct frg_server frg_server;

/* ---- library / context ---------------------------------------------- */
int frg_abi_version(void);
const char* frg_version(void);
const char* frg_status_string(int status);

/* Host construction of FROperators: replaces build_operators
   (src/fr/Operators.jl:85-104) for callers without their own tables.  Any
   output pointer may be NULL.  Matrices are column-major. */
int frg_build_operators(int p, int points, double* xi, double* w, double* D,
                        double* l_L, double* l_R, double* gL_xi, double* gR_xi,
                        double* gL, double* gR, double* V);

int frg_ctx_create(int device, frg_ctx** out);
int frg_ctx_destroy(frg_ctx* ctx);
const char* frg_last_error(const frg_ctx* ctx);
/* The cudaStream_t every solve of this context is launched on (for event
   timing and interop); no reference counterpart. */
int frg_ctx_get_stream(frg_ctx* ctx, void** stream);

/* ---- single solve ------------------------------------------------------ */
/* allocate_state + build_mesh_metrics + method selection
   (src/solvestate/SolutionState2D.jl:137-160, SolutionState.jl:25-39) */
int frg_solve_create(frg_ctx* ctx, const frg_solve_desc* desc, frg_solve** out);
int frg_solve_destroy(frg_solve* s);
int frg_solve_get_info(const frg_solve* s, frg_solve_info* info);

/* state.u / state.t upload and download (copies, Julia layout) */
int frg_upload_state(frg_solve* s, const double* u, size_t n, double t);
int frg_download_state(frg_solve* s, double* u, size_t n, double* t);

/* residual!(du, state, eq, method): src/fr/Residual.jl:161-214 (1D),
   src/fr/Residual2D.jl:131-416 (2D), including the sense! /
   apply_dissipation! hooks of the method.  du is a host array of n doubles. */
int frg_residual(frg_solve* s, double* du, size_t n);

/* sense! (src/capturing/PerssonAV.jl:116-135, PerssonAV2D.jl:20-59): the
   element sensor sigma of the current state; sigma has nel entries. */
int frg_sense(frg_solve* s, double* sigma, size_t nel);

/* compute_dt(state, eq; cfl): src/time/SSP_RK3.jl:8-24 (1D), :126-133 (2D) */
int frg_compute_dt(frg_solve* s, double cfl, double* dt);

/* ssp_rk3_step! / ssp_rk2_step! with the given dt (src/time/SSP_RK3.jl:29-65,
   :135-164; src/time/SSP_RK2.jl:14-68).  *step_status receives FRG_OK or
   FRG_DIVERGED. */
int frg_step(frg_solve* s, double dt, int* step_status);

/* integrate! / ssp_rk3! / ssp_rk2! (src/time/Integrate.jl:9-43,
   src/time/SSP_RK3.jl:75-118, :166-211, src/time/SSP_RK2.jl:70-132):
   advance to t_final with the CFL dt (fixed_dt <= 0) or a fixed dt; the last
   step is clipped to t_final; max_steps caps the step count.  The whole loop
   runs on the device (CUDA graphs of several steps); the host only polls the
   device status word between graph launches. */
int frg_advance(frg_solve* s, double t_final, double cfl, double fixed_dt,
                int64_t max_steps, frg_result* out);

/* Stage-kernel tile variants (elements per CTA, threads per CTA, CTAs per
   SM, u0 staging), no reference counterpart.  frg_autotune times every variant on the
   solve's current state (scratch buffers only; the state is untouched) with
   `reps` launches each, selects the fastest and returns it in *best; ms (may
   be NULL) receives the mean launch time of each variant. */
int frg_get_variant(const frg_solve* s, int* variant, int* n_variants);
int frg_set_variant(frg_solve* s, int variant);
int frg_autotune(frg_solve* s, int reps, int* best, double* ms);

/* Persisted autotune table (no reference counterpart): the tile variant of
   the 2D stage kernels per key (p, flux FRG_FLUX_*, av 0 none / 1 BR0 /
   2 element-local DD, curved 0 affine / 1 curved geometry), shared by the
   whole process.  frg_autotune records its choice under the solve's key;
   frg_solve_create starts a 2D solve from its key's variant; the batched
   engine runs each group of instances with its key's variant (else a fixed
   default tile).  save writes the table as JSON, load merges a file written
   by save (FRG_ERR_INVALID_ARG and nothing merged if the file is malformed or
   names an unknown variant).  get returns FRG_ERR_STATE for an absent key. */
int frg_autotune_table_load(const char* path);
int frg_autotune_table_save(const char* path);
int frg_autotune_table_set(int p, int flux, int av, int curved, int variant);
int frg_autotune_table_get(int p, int flux, int av, int curved, int* variant);
int frg_autotune_table_clear(void);
int frg_autotune_table_size(void);

/* Allocation-free residual evaluation (no counterpart in the reference).
   Same result as frg_residual for a 2D affine mesh without solid mask, for
   callers that cannot call cudaMalloc when they need a residual -- e.g. a
   host framework whose device memory is owned by its own pool or budget.
   u (input state) and du (output) are DEVICE pointers of ndof doubles in
   the Julia layout, owned by the caller; t is the state time; stream is a
   cudaStream_t (NULL: legacy default stream).  All scratch lives in one
   fixed __device__ array (at most FRG_NOALLOC_MAX_ELEMENTS elements,
   FRG_NOALLOC_MAX_SIDE per side; larger meshes return FRG_ERR_INVALID_ARG).
   The first call on a device resolves that array's address
   (cudaGetSymbolAddress).  Calls share the array: calls that overlap on the
   GPU race and must be serialised by the caller.  Returns after enqueueing. */
int frg_residual2d_noalloc(const frg_solve_desc* desc, const double* u, double* du,
                           double t, void* stream);

/* Instrumented frg_advance for profiling (no reference counterpart): runs
   nsteps steps with direct launches and times every stage kernel with CUDA
   events on the solve's stream; stage_ms[k] = mean duration (ms) of the
   stage-(k+1) kernel, k = 0..2 (stage 3 unused for SSP-RK2). */
int frg_time_stages(frg_solve* s, int64_t nsteps, double cfl, double fixed_dt,
                    double* stage_ms, frg_result* out);

/* ---------------------------------------------------------------- batches
   Many independent solves advanced together on one GPU (no counterpart in
   the reference, whose callers -- case sweeps, robustness matrices, the
   invent/confirm loop (src/invent/Robustness.jl:245, src/invent/Confirm.jl:35)
   -- call integrate! (src/time/Integrate.jl:9) once per case, one after the
   other).  Every instance is an ordinary solve with its own state, mesh,
   tables, dt, time and status.  An instance's results do not depend on the
   mix: they are bit-identical to the same instance alone in a batch.  Against
   the same solve advanced alone with frg_advance they agree to rounding
   (the batched kernels read their descriptors from shared memory and the
   compiler fuses a few multiply-adds differently): within 1e-10 relative,
   with identical status and step counts.  An instance large enough to run
   through the single-solve kernels (a solo group) is bit-identical to
   frg_advance.  Each stage launches one kernel per
   group of instances that share (dim, P, flux, dissipation form, tables),
   over the ragged list of that group's tiles; K steps are captured in one
   CUDA graph.  Adding or removing instances takes effect at the next
   frg_batch_run (continuous batching). */

/* capacity: instance slots; hbm_budget: admission limit in bytes on the
   instances' device memory (0 = none). */
int frg_batch_create(frg_ctx* ctx, int capacity, size_t hbm_budget, frg_batch** out);
int frg_batch_destroy(frg_batch* b); /* destroys its instances too */
/* Create an instance in a free slot (*slot).  FRG_ERR_OOM when the batch is
   full or the HBM budget would be exceeded.  The instance is idle until
   frg_batch_start. */
int frg_batch_add(frg_batch* b, const frg_solve_desc* desc, int* slot);
int frg_batch_remove(frg_batch* b, int slot);
/* Scheduling: lockstep (0, default: every instance takes one step per round)
   or multirate (1: a group of instances whose step is cheaper takes up to 32
   steps per round, so cheap solves that need many steps keep pace).  Results
   do not depend on the mode; max_steps of frg_batch_run counts rounds. */
int frg_batch_set_multirate(frg_batch* b, int on);
/* The instance's solve: frg_upload_state / frg_download_state /
   frg_residual work on it while it is not running. */
int frg_batch_get_solve(frg_batch* b, int slot, frg_solve** s);
/* The group an instance ran in at the last frg_batch_run (no reference
   counterpart): *variant is the tile variant of its batched kernels (the
   autotune table's entry for its key, or -1 for the default tile) and *solo
   whether it runs alone through the single-solve kernels.  FRG_ERR_STATE
   before its first run. */
int frg_batch_slot_group(frg_batch* b, int slot, int* variant, int* solo);
/* Start an instance's run with integrate!'s arguments (as frg_advance). */
int frg_batch_start(frg_batch* b, int slot, double t_final, double cfl, double fixed_dt,
                    int64_t max_steps);
/* Advance every running instance by up to max_steps steps, or until none
   runs.  results (capacity entries, may be NULL): per slot FRG_OK /
   FRG_DIVERGED / FRG_MAX_STEPS when the run ended, FRG_RUNNING while it
   goes on, FRG_ERR_STATE for an empty slot; n_steps and t of the run. */
int frg_batch_run(frg_batch* b, int64_t max_steps, frg_result* results, int* n_running);
/* Upper bound of the device bytes a solve of this descriptor holds (the
   admission test of a served batch). */
int frg_solve_bytes(const frg_solve_desc* desc, size_t* bytes);

/* ----------------------------------------------------------------- server
   A request queue in front of a batch (no counterpart in the reference,
   whose case runners, src/cli/run.jl:267, solve one request at a time).
   frg_server_pump admits queued requests in arrival order into free slots
   while their footprint fits the HBM budget, advances the batch by up to
   steps_per_pump rounds (multirate) and delivers finished requests (final
   state copied to u_out, slot freed and refilled at once).  The caller's loop
   drives the server; there is no internal thread. */
int frg_server_create(frg_ctx* ctx, int slots, size_t hbm_budget, int64_t steps_per_pump,
                      frg_server** out);
int frg_server_destroy(frg_server* s);
/* Queue one solve.  desc and every array it points to, u0 (ndof doubles,
   host) and u_out (ndof doubles, host, written on completion; NULL: the
   final state is not downloaded, only its diagnostics are kept) must stay
   valid until the request completes.  FRG_ERR_OOM if the request alone
   exceeds the budget. */
int frg_server_submit(frg_server* s, const frg_solve_desc* desc, const double* u0, double t0,
                      double t_final, double cfl, double fixed_dt, int64_t max_steps,
                      double* u_out, int64_t* request_id);
/* Cancel a queued or running request (result FRG_CANCELLED). */
int frg_server_cancel(frg_server* s, int64_t request_id);
/* One scheduling round; counts of requests completed by this call, still
   queued and running. */
int frg_server_pump(frg_server* s, int* n_done, int* n_queued, int* n_active);
/* *done = 1 once the request completed; r = its status, steps and time. */
int frg_server_result(frg_server* s, int64_t request_id, int* done, frg_result* r);
/* Up to cap request ids completed since the last call, in completion order. */
int frg_server_take_completed(frg_server* s, int64_t* ids, int cap, int* n);

/* ------------------------------------------------------------ diagnostics
   The scoring-harness reductions of the reference on the device state, so a
   caller gets them without downloading the state:
     mass[c]        discrete_mass(state, c+1)  (SolutionState.jl:80-90,
                    SolutionState2D.jl:85-97)
     rho_min/max    minimum / maximum of the density (Cases2D_Riemann.jl:111-116)
     p_min          minimum pressure(eq, U)
     nonfinite      number of non-finite entries (has_nonfinite, Residual.jl:219)
     positivity_ok  positivity_ok(eq, state) (Euler.jl:62-77, Euler2D.jl:153-163)
     l2_error       l2_error(state, uexact, c+1) (SolutionState.jl:93-107,
                    SolutionState2D.jl:98-111) against an exact solution
   Sums are reduced in a fixed order (deterministic), not in the reference's
   sequential order, so they agree with it to rounding. */
enum {
  FRG_EXACT_NONE = 0,
  FRG_EXACT_STATE = 1,           /* a reference state in device memory, the solve's layout */
  FRG_EXACT_VORTEX_2D = 2,       /* isentropic_vortex_primitives, Cases2D_Riemann.jl:163-186 */
  FRG_EXACT_SMOOTH_2D = 3,       /* the smooth order-test wave, Cases2D_Smooth.jl:124-135 */
  FRG_EXACT_DENSITY_WAVE_1D = 4  /* euler_density_wave_conserved, Cases.jl:404-414 */
};
typedef struct frg_diagnostics {
  double mass[4]; /* per component; entries beyond neq are 0 */
  double rho_min, rho_max, p_min;
  int64_t nonfinite;
  int positivity_ok;
  int pad;
  double l2_error; /* 0 when exact == FRG_EXACT_NONE */
  double t;        /* time of the state */
} frg_diagnostics;
/* exact: FRG_EXACT_*; ref_dev: device pointer for FRG_EXACT_STATE (else
   ignored); t_exact: time of the exact solution; c: 0-based component of
   l2_error.  2D exact solutions need point coordinates: affine or analytic
   wavy meshes, not caller metrics. */
int frg_diagnostics_compute(frg_solve* s, int exact, const double* ref_dev, double t_exact, int c,
                            frg_diagnostics* out);

/* Point data of the high-order VTU writer (write_vtu_high_order,
   src/io/VTKHighOrder.jl:325-535) evaluated on the device from the current
   state: n_per = (p+1)^dim VTK Lagrange nodes per element given as reference
   coordinates node_xi / node_eta (eta: 2D only) in VTK node order; the state
   is interpolated from the solution points with the Lagrange basis at each
   node.  Host outputs, field-major over n_points = nel * n_per nodes
   (element-major): xy = x (and y in 2D) from physical_xy including the
   analytic wavy map; fields = rho, u, v, p, rho_u, rho_v, E (2D) or rho, u,
   p, rho_u, E (1D).  2D meshes with caller metrics (no node coordinates)
   are rejected with FRG_ERR_INVALID_ARG. */
int frg_vtk_point_data(frg_solve* s, int n_per, const double* node_xi, const double* node_eta,
                       double* xy, double* fields, size_t n_points);

/* Device-side diagnostics of a delivered server request's final state (see
   frg_diagnostics_compute; no exact solution).  FRG_ERR_STATE before the
   request completed successfully. */
int frg_server_diagnostics(frg_server* s, int64_t request_id, frg_diagnostics* out);

/* 1D shock-capturing scores of a solve's density on the device: the scoring
   fields of the reference's discontinuous 1D case reports (Cases.jl:987-1021)
   from src/verification/Metrics.jl, over the density samples in x order
   (sample_solution_1d, :95-123):
     shock_thickness   shock_thickness_sp(x, rho) (:138-200), in mean
                       solution-point spacings; NaN as the reference
     shock_index/_x    0-based sample index and x of the steepest gradient
     overshoot*        overshoot_metric(rho_min, rho_max, ref_min, ref_max)
                       (:81-87)
     excess_dissipation  excess_dissipation(x, rho, ref; mask =
                       smooth_region_mask(x, ref; grad_frac, exclude))
                       (:208-255); NaN without a reference
     l1_rel            sum|rho - ref| / (sum|ref| + 1e-30) (Cases.jl:1021)
   The reference density is either ref_host (n_samples doubles, host memory,
   x order) or the current state of ref_solve (a 1D solve on the same
   samples, e.g. the NullCapturing run of the same case), or neither.
   Indices and the thickness are exact; sums are reduced in a fixed order. */
typedef struct frg_shock_params {
  double ref_min, ref_max; /* overshoot bounds (Sod: 0.125, 1.0) */
  double grad_frac;        /* smooth_region_mask gradient fraction */
  int window_sp;           /* shock_thickness_sp window, 1..512 (reference: 30) */
  int n_exclude;           /* excluded x windows of the mask, 0..4 */
  double exclude[4][2];    /* [a, b] windows (closed) */
} frg_shock_params;
typedef struct frg_shock_metrics {
  double shock_thickness;
  int64_t shock_index;
  double shock_x;
  double overshoot, overshoot_over, overshoot_under;
  double rho_min, rho_max;
  double excess_dissipation;
  double l1_rel;
  int64_t n_samples;
  int has_reference;
  int pad;
} frg_shock_metrics;
int frg_shock_metrics_1d(frg_solve* s, const frg_shock_params* params, const double* ref_host,
                         const frg_solve* ref_solve, frg_shock_metrics* out);

/* ------------------------------------------------------ initial conditions
   set_initial_condition! (SolutionState.jl:59-73, SolutionState2D.jl:58-82)
   for the reference's case initial conditions, evaluated on the device at
   the solution points (physical_xy, MeshMetrics2D.jl:49-74, including the
   analytic wavy map), so a request needs no host evaluation or upload of
   its state.  Sets the state time to 0.  prim rows are primitive states
   (rho, u, v, p) in 2D, (rho, u, p) in 1D:
     UNIFORM        prim[0]
     TWO_STATE      x < x0 ? prim[0] : prim[1]  (sod_ic, Cases.jl:940-946)
     FOUR_QUADRANT  riemann2d_ic quadrant rule at (x0, y0), prim = ne, nw, sw, se
                    (Cases2D_Riemann.jl:33-51)
     DENSITY_WAVE   prim[0] with rho = prim[0][0] + amp sin(2 pi (x [+ y] - t) + phase)
                    (euler_density_wave_conserved, Cases.jl:404-414)
     VORTEX         isentropic_vortex_primitives at time t (Cases2D_Riemann.jl:163-186)
     SMOOTH_2D      the smooth order-test wave at time t (Cases2D_Smooth.jl:124-135)
     SHU_OSHER      shu_osher_ic (Cases.jl:930-938), 1D */
enum {
  FRG_IC_UNIFORM = 0,
  FRG_IC_TWO_STATE = 1,
  FRG_IC_FOUR_QUADRANT = 2,
  FRG_IC_DENSITY_WAVE = 3,
  FRG_IC_VORTEX = 4,
  FRG_IC_SMOOTH_2D = 5,
  FRG_IC_SHU_OSHER = 6
};
typedef struct frg_ic {
  int kind; /* FRG_IC_* */
  int pad;
  double x0, y0, amp, phase, t;
  double prim[4][4];
} frg_ic;
int frg_set_initial_condition(frg_solve* s, const frg_ic* ic);
/* frg_server_submit with the initial state evaluated on the device at
   admission (frg_set_initial_condition) instead of uploaded; the state time
   starts at 0. */
int frg_server_submit_ic(frg_server* s, const frg_solve_desc* desc, const frg_ic* ic, double t_final,
                         double cfl, double fixed_dt, int64_t max_steps, double* u_out,
                         int64_t* request_id);

/* --------------------------------------------------------- device hooks
   A registry of compiled implementations of capturing-method hooks, chosen
   by name, so a method that overrides a hook can still run on the GPU
   (no counterpart in the reference, whose hooks are Julia methods:
   src/capturing/Interfaces.jl:43-92).  Slots: post_step (called after every
   completed step, before the next compute_dt, as post_step! in
   ssp_rk3_step!, SSP_RK3.jl:162); numerical_flux_method (the flux of every
   1D interface, boundary interfaces included, as _resolve_flux,
   src/fr/Residual.jl:9-15; the 2D residual ignores it, as the reference's
   does); preprocess_state (the state the residual is evaluated on);
   extrapolate_interface (the element traces the 1D interface fluxes use, as
   extrapolate_interface! in residual!, Residual.jl:175; the 2D residual
   never calls it, and a 2D solve ignores the slot).
   Implementations:
     "positivity_zhang_shu"  post_step: the positivity-preserving scaling of
        Zhang & Shu (J. Comput. Phys. 229, 2010) toward the element mean,
        density >= params[0], pressure >= params[1] (default 1e-13 each);
        element integrals are unchanged.
     "flux_rusanov"  numerical_flux_method: Rusanov with its dissipation
        scaled by params[0] = alpha >= 0 (default 1, the reference's flux).
     "flux_hllc"  numerical_flux_method: HLLC whatever the scheme's flux.
     "preprocess_positivity_zhang_shu"  preprocess_state: the residual is
        evaluated on the work state u_work = the Zhang & Shu scaling of the
        stage state (params as "positivity_zhang_shu"), its element viscosity
        included, while the SSP-RK combination, compute_dt and post_step keep
        the stage state (preprocess_state!, Interfaces.jl:41-46, called first
        in residual!).  Single solves only: frg_batch_start and
        frg_server_set_hook refuse it with FRG_ERR_UNSUPPORTED_HOOK.
     "traces_toward_mean"  extrapolate_interface: each element's two traces
        pulled toward its mean (quadrature weights), ubar + theta (t - ubar),
        params[0] = theta in [0, 1] (default 1: the Lagrange traces, to
        rounding; 0: first-order traces).
     "traces_positivity_zhang_shu"  extrapolate_interface: the Zhang & Shu
        scaling (as "positivity_zhang_shu") applied to an element's two
        traces, density >= params[0], pressure >= params[1] (defaults 1e-13).
        Both change only the numerical fluxes' inputs; the BR0 dissipation
        keeps the Lagrange traces (apply_dissipation_br0!, PerssonAV.jl:249).
   Batched instances run their hooks too: set one on the slot's solve
   (frg_batch_get_solve) before frg_batch_start, or on a queued request with
   frg_server_set_hook; the batch groups instances by hook and steps them
   to the same results as a single solve. */
enum {
  FRG_HOOK_POST_STEP = 0,
  FRG_HOOK_NUMERICAL_FLUX = 1,
  FRG_HOOK_PREPROCESS_STATE = 2,
  FRG_HOOK_EXTRAPOLATE_INTERFACE = 3
};
int frg_hook_count(void);
int frg_hook_info(int index, const char** name, int* slot, int* id, int* nparams);
/* FRG_ERR_UNSUPPORTED_HOOK if no implementation has that name. */
int frg_hook_lookup(const char* name, int* slot, int* id);
/* id 0 removes the slot's hook. */
int frg_solve_set_hook(frg_solve* s, int slot, int id, const double* params, int nparams);
/* Apply the post-step hook once to the current state (host-driven loops). */
int frg_apply_post_step(frg_solve* s);
/* Invocation counts of the solve's hooks since frg_solve_create, counted on
   the device (graph replays and batched steps included), as the counters of
   HookProbeMethod (test/test_capturing.jl:5-41): counts[FRG_HOOK_POST_STEP]
   = post-step passes run (one per completed step, plus each
   frg_apply_post_step), counts[FRG_HOOK_PREPROCESS_STATE] = work states made
   (one per residual evaluation: stage, frg_residual, frg_sense).  The flux
   and trace overrides run inline in every interface pass, with no launch of
   their own: counts[FRG_HOOK_NUMERICAL_FLUX] =
   counts[FRG_HOOK_EXTRAPOLATE_INTERFACE] = -1 (frg_solve_info.residual_evals
   counts the residuals that used them).  n: entries to fill, 1..4. */
int frg_solve_hook_calls(frg_solve* s, int64_t* counts, int n);
/* Select hook `id` of `slot` for a request that is still queued (id 0
   removes it); applied to the request's solve at admission.  FRG_ERR_STATE
   once the request was admitted or completed. */
int frg_server_set_hook(frg_server* s, int64_t request_id, int slot, int id, const double* params,
                        int nparams);

#ifdef __cplusplus
}
#endif
#endif

/*
 * FRForge CPU oracle -- TEST INFRASTRUCTURE ONLY (see frforge_oracle.h).
 *
 * Plain-C FP64 restatement of the reference's FR residual + SSP-RK path.
 * Each function names the Julia function (file:line) it restates.  The
 * arithmetic order of every expression follows the Julia source (Julia
 * evaluates a*b*c as (a*b)*c and a+b+c as (a+b)+c and never contracts
 * a*b+c into an fma); the build passes -ffp-contract=off.
 *
 * Third-party arithmetic the reference takes from LAPACK (OpenBLAS 0.3.27 via
 * Julia LinearAlgebra, Manifest.toml:52-55) is restated from the published
 * algorithms: the Golub-Welsch eigen-solve uses the implicit symmetric QL
 * method with Wilkinson shifts; `V \ u` uses LU with partial pivoting
 * (dgetf2 form) followed by unit-lower / upper triangular solves (dtrsm
 * column form).  Those two pieces agree with LAPACK to rounding, not bitwise.
 */
#include "frforge_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define EPS DBL_EPSILON /* Julia eps(Float64) */
#define TWO_PI 6.283185307179586 /* Julia 2π (Float64) */
#define PI_F64 3.141592653589793

/* ---------------------------------------------------------------- helpers */

/* Julia max/min for Float64: NaN-propagating, max(-0.0,0.0) == 0.0 */
static inline double jmax(double a, double b) {
  if (a != a || b != b) return a + b;
  if (a > b) return a;
  if (b > a) return b;
  return signbit(a) ? b : a;
}
static inline double jmin(double a, double b) {
  if (a != a || b != b) return a + b;
  if (a < b) return a;
  if (b < a) return b;
  return signbit(a) ? a : b;
}

void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

/* ------------------------------------------------------------- operators */

/* legendre_P, src/fr/Correction.jl:8-24 */
static double legendre_P(int k, double x) {
  if (k == 0) return 1.0;
  if (k == 1) return x;
  double pkm2 = 1.0, pkm1 = x, pk = pkm1;
  for (int m = 2; m <= k; ++m) {
    pk = (((double)(2 * m - 1) * x * pkm1) - ((double)(m - 1) * pkm2)) / (double)m;
    pkm2 = pkm1;
    pkm1 = pk;
  }
  return pk;
}

/* legendre_P_prime, src/fr/Correction.jl:32-45 */
static double legendre_P_prime(int k, double x) {
  if (k == 0) return 0.0;
  if (x >= 1.0 - 1000 * EPS) return (double)(k * (k + 1)) / 2.0;
  if (x <= -1.0 + 1000 * EPS)
    return ((k % 2 == 1) ? 1.0 : -1.0) * (double)(k * (k + 1)) / 2.0;
  double pk = legendre_P(k, x);
  double pkm1 = legendre_P(k - 1, x);
  return ((double)k * pkm1 - (double)k * x * pk) / (1.0 - x * x);
}

/* Symmetric tridiagonal eigen-solve by the implicit QL method with Wilkinson
   shifts (published algorithm; replaces LAPACK in eigen(Symmetric(J))).
   d: diagonal (in: n, out: eigenvalues); e: sub-diagonal e[0..n-2];
   z: n x n eigenvectors, column-major (z[r + n*c] = component r of vector c). */
static void tridiag_ql(int n, double* d, double* e_in, double* z) {
  double e[ORC_MAXNP + 1];
  for (int i = 0; i < n - 1; ++i) e[i] = e_in[i];
  e[n - 1] = 0.0;
  for (int r = 0; r < n; ++r)
    for (int c = 0; c < n; ++c) z[r + n * c] = (r == c) ? 1.0 : 0.0;
  for (int l = 0; l < n; ++l) {
    int iter = 0;
    int m;
    do {
      for (m = l; m < n - 1; ++m) {
        double dd = fabs(d[m]) + fabs(d[m + 1]);
        if (fabs(e[m]) <= EPS * dd) break;
      }
      if (m != l) {
        if (++iter > 60) break;
        double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
        double r = hypot(g, 1.0);
        g = d[m] - d[l] + e[l] / (g + (g >= 0.0 ? fabs(r) : -fabs(r)));
        double s = 1.0, c = 1.0, p = 0.0;
        int i;
        for (i = m - 1; i >= l; --i) {
          double f = s * e[i];
          double b = c * e[i];
          r = hypot(f, g);
          e[i + 1] = r;
          if (r == 0.0) {
            d[i + 1] -= p;
            e[m] = 0.0;
            break;
          }
          s = f / r;
          c = g / r;
          g = d[i + 1] - p;
          r = (d[i] - g) * s + 2.0 * c * b;
          p = s * r;
          d[i + 1] = g + p;
          g = c * r - b;
          for (int k = 0; k < n; ++k) {
            f = z[k + n * (i + 1)];
            z[k + n * (i + 1)] = s * z[k + n * i] + c * f;
            z[k + n * i] = c * z[k + n * i] - s * f;
          }
        }
        if (r == 0.0 && i >= l) continue;
        d[l] -= p;
        e[l] = g;
        e[m] = 0.0;
      }
    } while (m != l);
  }
}

/* gauss_legendre_nodes_weights, src/fr/Points.jl:10-34 */
static void gauss_legendre(int n, double* xi, double* w) {
  if (n == 1) {
    xi[0] = 0.0;
    w[0] = 2.0;
    return;
  }
  double d[ORC_MAXNP], e[ORC_MAXNP], z[ORC_MAXNP * ORC_MAXNP];
  for (int i = 0; i < n; ++i) d[i] = 0.0;
  for (int k = 1; k <= n - 1; ++k) e[k - 1] = (double)k / sqrt((double)(4 * k * k - 1));
  tridiag_ql(n, d, e, z);
  int perm[ORC_MAXNP];
  for (int i = 0; i < n; ++i) perm[i] = i;
  for (int i = 1; i < n; ++i) { /* stable insertion sort (sortperm) */
    int pi = perm[i], j = i - 1;
    while (j >= 0 && d[perm[j]] > d[pi]) {
      perm[j + 1] = perm[j];
      --j;
    }
    perm[j + 1] = pi;
  }
  double sw = 0.0;
  for (int i = 0; i < n; ++i) {
    xi[i] = d[perm[i]];
    double v = z[0 + n * perm[i]];
    w[i] = 2 * (v * v);
  }
  for (int i = 0; i < n; ++i) sw += w[i];
  double scale = 2.0 / sw;
  for (int i = 0; i < n; ++i) w[i] *= scale;
}

static void sort_asc(int n, double* a) {
  for (int i = 1; i < n; ++i) {
    double v = a[i];
    int j = i - 1;
    while (j >= 0 && a[j] > v) {
      a[j + 1] = a[j];
      --j;
    }
    a[j + 1] = v;
  }
}

/* gauss_lobatto_legendre_nodes_weights, src/fr/Operators.jl:10-59 */
static void gauss_lobatto(int n, double* xi, double* w) {
  if (n == 1) {
    xi[0] = 0.0;
    w[0] = 2.0;
    return;
  }
  int p = n - 1;
  xi[0] = -1.0;
  xi[n - 1] = 1.0;
  for (int j = 2; j <= n - 1; ++j) {
    double x = cos(PI_F64 * (double)(j - 1) / (double)p);
    for (int it = 0; it < 80; ++it) {
      double Pp = legendre_P(p, x);
      double dPp = legendre_P_prime(p, x);
      double one_m_x2 = 1.0 - x * x;
      if (fabs(one_m_x2) < 1000 * EPS) break;
      double d2Pp = (2.0 * x * dPp - (double)(p * (p + 1)) * Pp) / one_m_x2;
      if (fabs(d2Pp) < EPS) break;
      double xnew = x - dPp / d2Pp;
      xnew = jmin(jmax(xnew, -1.0 + 10 * EPS), 1.0 - 10 * EPS);
      if (fabs(xnew - x) < 10 * EPS) {
        x = xnew;
        break;
      }
      x = xnew;
    }
    xi[j - 1] = x;
  }
  sort_asc(n, xi);
  xi[0] = -1.0;
  xi[n - 1] = 1.0;
  double sw = 0.0;
  for (int i = 0; i < n; ++i) {
    double Pp = legendre_P(p, xi[i]);
    double den = (double)p * (double)(p + 1) * Pp * Pp;
    w[i] = 2.0 / jmax(den, EPS);
  }
  for (int i = 0; i < n; ++i) sw += w[i];
  double scale = 2.0 / sw;
  for (int i = 0; i < n; ++i) w[i] *= scale;
}

/* lagrange_at, src/fr/Points.jl:65-76 */
static void lagrange_at(int n, const double* xi, double x, double* l) {
  for (int j = 0; j < n; ++j) {
    l[j] = 1.0;
    for (int k = 0; k < n; ++k)
      if (k != j) l[j] *= (x - xi[k]) / (xi[j] - xi[k]);
  }
}

/* differentiation_matrix, src/fr/Points.jl:83-104 */
static void differentiation_matrix(int n, const double* xi, double* D) {
  for (int i = 0; i < n; ++i) {
    for (int j = 0; j < n; ++j) {
      D[i + n * j] = 0.0;
      if (i != j) {
        double num = 1.0;
        double den = xi[j] - xi[i];
        for (int k = 0; k < n; ++k)
          if (k != i && k != j) num *= (xi[i] - xi[k]) / (xi[j] - xi[k]);
        D[i + n * j] = num / den;
      }
    }
    /* -sum(D[i,k] for k != i): generator sum starts from the first term */
    double s = 0.0;
    int first = 1;
    for (int k = 0; k < n; ++k) {
      if (k == i) continue;
      if (first) {
        s = D[i + n * k];
        first = 0;
      } else {
        s += D[i + n * k];
      }
    }
    D[i + n * i] = -s;
  }
}

/* build_operators, src/fr/Operators.jl:85-104; g_DG_values_and_derivs,
   src/fr/Correction.jl:57-90; legendre_vandermonde, Correction.jl:93-101 */
int orc_build_operators(int p, int points, orc_ops* o) {
  if (p < 0 || p + 1 > ORC_MAXNP) return -1;
  if (points != ORC_POINTS_GL && points != ORC_POINTS_GLL) return -1;
  memset(o, 0, sizeof(*o));
  int n = p + 1;
  o->p = p;
  o->np = n;
  o->points = points;
  if (points == ORC_POINTS_GL)
    gauss_legendre(n, o->xi, o->w);
  else
    gauss_lobatto(n, o->xi, o->w);
  differentiation_matrix(n, o->xi, o->D);
  lagrange_at(n, o->xi, -1.0, o->lL);
  lagrange_at(n, o->xi, 1.0, o->lR);
  double rR_m1 = legendre_P(p + 1, -1.0) - legendre_P(p, -1.0);
  double rL_p1 = legendre_P(p + 1, 1.0) + legendre_P(p, 1.0);
  for (int i = 0; i < n; ++i) {
    double x = o->xi[i];
    double Pp = legendre_P(p, x), Pp1 = legendre_P(p + 1, x);
    o->gL[i] = (Pp1 - Pp) / rR_m1;
    o->gR[i] = (Pp1 + Pp) / rL_p1;
    double dPp = legendre_P_prime(p, x), dPp1 = legendre_P_prime(p + 1, x);
    o->gLxi[i] = (dPp1 - dPp) / rR_m1;
    o->gRxi[i] = (dPp1 + dPp) / rL_p1;
  }
  for (int j = 0; j < n; ++j)
    for (int k = 0; k < n; ++k) o->V[j + n * k] = legendre_P(k, o->xi[j]);
  return 0;
}

/* ------------------------------------------- Julia range (linspace) values */

/* Base.rat: continued-fraction rational approximation (Float64 -> narrow
   Float32 maxintfloat = 2^24) */
static void julia_rat(double x, long long* num, long long* den) {
  double y = x;
  long long a = 1, d = 1, b = 0, c = 0;
  const double m = 16777216.0;
  while (fabs(y) <= m) {
    long long f = (long long)trunc(y);
    y -= (double)f;
    long long na = f * a + c, nc = a;
    long long nb = f * b + d, nd = b;
    a = na;
    c = nc;
    b = nb;
    d = nd;
    if (!(llabs(a) <= (long long)m && llabs(b) <= (long long)m)) {
      *num = c;
      *den = d;
      return;
    }
    if ((double)a / (double)b == x) break;
    y = 1.0 / y;
  }
  *num = a;
  *den = b;
}
static long long gcdll(long long a, long long b) {
  a = llabs(a);
  b = llabs(b);
  while (b) {
    long long t = a % b;
    a = b;
    b = t;
  }
  return a;
}

/* collect(range(a, b; length=len)): Julia expresses both ends as integer
   ratios over a common denominator and rounds each element of the exact
   rational progression once (Base.range_start_stop_length / _linspace). */
static void julia_linspace(double a, double b, int len, double* out) {
  long long an, ad, bn, bd;
  julia_rat(a, &an, &ad);
  julia_rat(b, &bn, &bd);
  if (ad != 0 && bd != 0) {
    long long den = ad / gcdll(ad, bd) * bd;
    double m = 9007199254740992.0;
    if (den != 0 && fabs((double)den * a) <= m && fabs((double)den * b) <= m) {
      long long sn = llround((double)den * a), en = llround((double)den * b);
      if ((double)sn / (double)den == a && (double)en / (double)den == b) {
        for (int i = 1; i <= len; ++i) {
          long double numr = (long double)(len - i) * sn + (long double)(i - 1) * en;
          long double denr = (long double)(len - 1) * den;
          /* numerator and denominator are exact integers: one rounding */
          out[i - 1] = (double)(numr / denr);
          if (fabsl(numr) < 9007199254740992.0L && fabsl(denr) < 9007199254740992.0L)
            out[i - 1] = (double)numr / (double)denr;
        }
        return;
      }
    }
  }
  for (int i = 1; i <= len; ++i)
    out[i - 1] = (double)((long double)a + ((long double)b - a) * (i - 1) / (len - 1));
}

/* ---------------------------------------------------------------- solver */

struct orc_solver {
  int dim, np, nel, nx, ny, neq;
  orc_ops ops;
  double gamma;
  int flux, time_scheme, method, av_form;
  double kappa, s0_factor, eps_floor, c_av;
  int flux_override;  /* numerical_flux_method override (1D): -1 none, else ORC_FLUX_* */
  double flux_alpha;  /* its Rusanov dissipation scale */
  int trace_override; /* extrapolate_interface override (1D): 0 none, ORC_TRACE_* */
  double trace_p0, trace_p1;
  orc_bc bc[4]; /* 1D: [0]=left [1]=right; 2D: left right bottom top */
  double t;
  /* 1D mesh */
  double *xv, *dx, *J1;
  /* 2D mesh + metrics */
  double *xv2, *yv2, *dx2, *dy2, *Jx, *Jy;
  int wavy;
  double amp;
  double *mx, *my, *x_xi, *x_eta, *y_xi, *y_eta, *J2;
  double *nx_W, *ny_W, *sJ_W, *nx_E, *ny_E, *sJ_E;
  double *nx_S, *ny_S, *sJ_S, *nx_N, *ny_N, *sJ_N;
  double* h_char;
  unsigned char* solid;
  /* state + RK work */
  double *u, *du, *u0, *u1, *u2, *u_work;
  /* residual workspace */
  double *trL, *trR, *fL, *fR; /* 1D traces / interface fluxes [nel,neq] */
  double *trW, *trE, *trS, *trN;
  double *fhW, *fhE, *fhS, *fhN; /* 2D [np,neq,nel] */
  double* sigma;
  double* eps_e;
  /* BR0 */
  double *g, *gx, *gy;
  double *bW, *bE, *bS, *bN;     /* u traces [np,nel,neq] (2D) / [nel,neq] (1D) */
  double *gW, *gE, *gS, *gN;     /* g traces */
  double *ghW, *ghE, *ghS, *ghN; /* ghat */
};

size_t orc_ndof(const orc_solver* s) {
  return (size_t)s->nel * (size_t)(s->dim == 1 ? s->np : s->np * s->np) * (size_t)s->neq;
}
double* orc_state(orc_solver* s) { return s->u; }
double orc_get_time(const orc_solver* s) { return s->t; }
void orc_set_time(orc_solver* s, double t) { s->t = t; }
void orc_get_ops(const orc_solver* s, orc_ops* out) { *out = s->ops; }

static double* dalloc(size_t n) {
  double* p = (double*)calloc(n ? n : 1, sizeof(double));
  return p;
}

static void common_alloc(orc_solver* s) {
  size_t n = orc_ndof(s);
  s->u = dalloc(n);
  s->du = dalloc(n);
  s->u0 = dalloc(n);
  s->u1 = dalloc(n);
  s->u2 = dalloc(n);
  s->u_work = dalloc(n);
  s->sigma = dalloc(s->nel);
  s->eps_e = dalloc(s->nel);
}

/* Mesh1D, src/mesh/Mesh1D.jl:23-42 */
orc_solver* orc_create_1d(int p, int points, int nel, double xl, double xr,
                          const orc_bc* left, const orc_bc* right, double gamma,
                          int flux, int time_scheme, int method, int av_form,
                          double kappa, double s0_factor, double eps_floor,
                          double c_av) {
  if (nel < 1 || !(xr > xl)) return NULL;
  if ((left->kind == ORC_BC_PERIODIC) != (right->kind == ORC_BC_PERIODIC)) return NULL;
  orc_solver* s = (orc_solver*)calloc(1, sizeof(orc_solver));
  if (orc_build_operators(p, points, &s->ops) != 0) {
    free(s);
    return NULL;
  }
  s->dim = 1;
  s->np = p + 1;
  s->nel = nel;
  s->nx = nel;
  s->ny = 1;
  s->neq = 3;
  s->gamma = gamma;
  s->flux = flux;
  s->flux_override = -1;
  s->flux_alpha = 1.0;
  s->trace_override = 0;
  s->trace_p0 = 0.0;
  s->trace_p1 = 0.0;
  s->time_scheme = time_scheme;
  s->method = method;
  s->av_form = av_form;
  s->kappa = kappa;
  s->s0_factor = s0_factor;
  s->eps_floor = eps_floor;
  s->c_av = c_av;
  s->bc[0] = *left;
  s->bc[1] = *right;
  s->xv = dalloc(nel + 1);
  s->dx = dalloc(nel);
  s->J1 = dalloc(nel);
  julia_linspace(xl, xr, nel + 1, s->xv);
  for (int e = 0; e < nel; ++e) {
    s->dx[e] = s->xv[e + 1] - s->xv[e];
    s->J1[e] = s->dx[e] / 2.0;
  }
  common_alloc(s);
  int nq = nel * 3;
  s->trL = dalloc(nq);
  s->trR = dalloc(nq);
  s->fL = dalloc(nq);
  s->fR = dalloc(nq);
  s->g = dalloc(orc_ndof(s));
  s->bW = dalloc(nq);
  s->bE = dalloc(nq);
  s->gW = dalloc(nq);
  s->gE = dalloc(nq);
  s->ghW = dalloc(nq);
  s->ghE = dalloc(nq);
  return s;
}

/* wavy_physical / wavy_partials, src/mesh/MeshMetrics2D.jl:299-318 */
static void wavy_physical(double X, double Y, double a, double* x, double* y) {
  *x = X + a * sin(TWO_PI * Y) * sin(PI_F64 * X);
  *y = Y + a * sin(TWO_PI * X) * sin(PI_F64 * Y);
}
static void wavy_partials(double X, double Y, double a, double* xX, double* xY,
                          double* yX, double* yY) {
  *xX = 1.0 + a * sin(TWO_PI * Y) * PI_F64 * cos(PI_F64 * X);
  *xY = a * TWO_PI * cos(TWO_PI * Y) * sin(PI_F64 * X);
  *yX = a * TWO_PI * cos(TWO_PI * X) * sin(PI_F64 * Y);
  *yY = 1.0 + a * sin(TWO_PI * X) * PI_F64 * cos(PI_F64 * Y);
}

/* physical_xy, src/mesh/MeshMetrics2D.jl:49-74 (affine or analytic wavy) */
static void physical_xy(const orc_solver* s, int e, double xi, double eta,
                        double* x, double* y) {
  int jx = e % s->nx, jy = e / s->nx;
  double xL = s->xv2[jx], xR = s->xv2[jx + 1];
  double yB = s->yv2[jy], yT = s->yv2[jy + 1];
  double X = (xL + xR) / 2.0 + s->Jx[jx] * xi;
  double Y = (yB + yT) / 2.0 + s->Jy[jy] * eta;
  if (s->wavy) {
    wavy_physical(X, Y, s->amp, x, y);
    return;
  }
  *x = X;
  *y = Y;
}

#define IX3(i, j, e, np) ((size_t)(i) + (size_t)(np) * ((size_t)(j) + (size_t)(np) * (size_t)(e)))
#define IX2(q, e, np) ((size_t)(q) + (size_t)(np) * (size_t)(e))

/* build_mesh_metrics, src/mesh/MeshMetrics2D.jl:82-218 (affine and, for
   wavy==2, D-differentiated isoparametric geometry) */
static void build_metrics_discrete(orc_solver* s, int curved) {
  int np = s->np, nel = s->nel;
  const double* D = s->ops.D;
  const double* xi = s->ops.xi;
  for (int e = 0; e < nel; ++e) {
    for (int j = 0; j < np; ++j)
      for (int i = 0; i < np; ++i)
        physical_xy(s, e, xi[i], xi[j], &s->mx[IX3(i, j, e, np)], &s->my[IX3(i, j, e, np)]);
    for (int j = 0; j < np; ++j)
      for (int i = 0; i < np; ++i) {
        double dxxi = 0, dyxi = 0, dxeta = 0, dyeta = 0;
        for (int k = 0; k < np; ++k) {
          dxxi += D[i + np * k] * s->mx[IX3(k, j, e, np)];
          dyxi += D[i + np * k] * s->my[IX3(k, j, e, np)];
          dxeta += D[j + np * k] * s->mx[IX3(i, k, e, np)];
          dyeta += D[j + np * k] * s->my[IX3(i, k, e, np)];
        }
        size_t id = IX3(i, j, e, np);
        s->x_xi[id] = dxxi;
        s->y_xi[id] = dyxi;
        s->x_eta[id] = dxeta;
        s->y_eta[id] = dyeta;
        s->J2[id] = dxxi * dyeta - dxeta * dyxi;
      }
  }
  const double *lL = s->ops.lL, *lR = s->ops.lR;
  for (int e = 0; e < nel; ++e) {
    for (int j = 0; j < np; ++j) {
      double xeW = 0, yeW = 0, xeE = 0, yeE = 0;
      for (int i = 0; i < np; ++i) {
        xeW += lL[i] * s->x_eta[IX3(i, j, e, np)];
        yeW += lL[i] * s->y_eta[IX3(i, j, e, np)];
        xeE += lR[i] * s->x_eta[IX3(i, j, e, np)];
        yeE += lR[i] * s->y_eta[IX3(i, j, e, np)];
      }
      double sE = sqrt(yeE * yeE + xeE * xeE);
      sE = jmax(sE, EPS);
      s->sJ_E[IX2(j, e, np)] = sE;
      s->nx_E[IX2(j, e, np)] = yeE / sE;
      s->ny_E[IX2(j, e, np)] = -xeE / sE;
      double sW = sqrt(yeW * yeW + xeW * xeW);
      sW = jmax(sW, EPS);
      s->sJ_W[IX2(j, e, np)] = sW;
      s->nx_W[IX2(j, e, np)] = -yeW / sW;
      s->ny_W[IX2(j, e, np)] = xeW / sW;
    }
    for (int i = 0; i < np; ++i) {
      double xxS = 0, yxS = 0, xxN = 0, yxN = 0;
      for (int j = 0; j < np; ++j) {
        xxS += lL[j] * s->x_xi[IX3(i, j, e, np)];
        yxS += lL[j] * s->y_xi[IX3(i, j, e, np)];
        xxN += lR[j] * s->x_xi[IX3(i, j, e, np)];
        yxN += lR[j] * s->y_xi[IX3(i, j, e, np)];
      }
      double sN = sqrt(yxN * yxN + xxN * xxN);
      sN = jmax(sN, EPS);
      s->sJ_N[IX2(i, e, np)] = sN;
      s->nx_N[IX2(i, e, np)] = -yxN / sN;
      s->ny_N[IX2(i, e, np)] = xxN / sN;
      double sS = sqrt(yxS * yxS + xxS * xxS);
      sS = jmax(sS, EPS);
      s->sJ_S[IX2(i, e, np)] = sS;
      s->nx_S[IX2(i, e, np)] = yxS / sS;
      s->ny_S[IX2(i, e, np)] = -xxS / sS;
    }
  }
  for (int e = 0; e < nel; ++e) {
    double area = 0.0;
    for (int j = 0; j < np; ++j)
      for (int i = 0; i < np; ++i)
        area += s->ops.w[i] * s->ops.w[j] * fabs(s->J2[IX3(i, j, e, np)]);
    double h_area = sqrt(jmax(area, EPS));
    double h_face = INFINITY;
    for (int q = 0; q < np; ++q) {
      double m = jmin(h_face, s->sJ_W[IX2(q, e, np)]);
      m = jmin(m, s->sJ_E[IX2(q, e, np)]);
      m = jmin(m, s->sJ_S[IX2(q, e, np)]);
      h_face = jmin(m, s->sJ_N[IX2(q, e, np)]);
    }
    s->h_char[e] = jmin(h_area, 2.0 * h_face);
    if (!curved) {
      int jx = e % s->nx, jy = e / s->nx;
      s->h_char[e] = jmin(s->dx2[jx], s->dy2[jy]);
    }
  }
}

/* build_mesh_metrics_analytic_wavy, src/mesh/MeshMetrics2D.jl:327-442 */
static void build_metrics_wavy(orc_solver* s) {
  int np = s->np, nel = s->nel;
  double a = s->amp;
  const double* xi = s->ops.xi;
  for (int e = 0; e < nel; ++e) {
    int jx = e % s->nx, jy = e / s->nx;
    double Jx = s->Jx[jx], Jy = s->Jy[jy];
    double xL = s->xv2[jx], xR = s->xv2[jx + 1], yB = s->yv2[jy], yT = s->yv2[jy + 1];
    for (int j = 0; j < np; ++j)
      for (int i = 0; i < np; ++i) {
        double X = (xL + xR) / 2.0 + Jx * xi[i];
        double Y = (yB + yT) / 2.0 + Jy * xi[j];
        size_t id = IX3(i, j, e, np);
        wavy_physical(X, Y, a, &s->mx[id], &s->my[id]);
        double xX, xY, yX, yY;
        wavy_partials(X, Y, a, &xX, &xY, &yX, &yY);
        s->x_xi[id] = xX * Jx;
        s->x_eta[id] = xY * Jy;
        s->y_xi[id] = yX * Jx;
        s->y_eta[id] = yY * Jy;
        s->J2[id] = s->x_xi[id] * s->y_eta[id] - s->x_eta[id] * s->y_xi[id];
      }
  }
  for (int e = 0; e < nel; ++e) {
    int jx = e % s->nx, jy = e / s->nx;
    double Jx = s->Jx[jx], Jy = s->Jy[jy];
    double xL = s->xv2[jx], xR = s->xv2[jx + 1], yB = s->yv2[jy], yT = s->yv2[jy + 1];
    for (int j = 0; j < np; ++j) {
      double Y = (yB + yT) / 2.0 + Jy * xi[j];
      double xX, xY, yX, yY;
      double Xw = (xL + xR) / 2.0 + Jx * (-1.0);
      wavy_partials(Xw, Y, a, &xX, &xY, &yX, &yY);
      double xe = xY * Jy, ye = yY * Jy;
      double sW = jmax(sqrt(ye * ye + xe * xe), EPS);
      s->sJ_W[IX2(j, e, np)] = sW;
      s->nx_W[IX2(j, e, np)] = -ye / sW;
      s->ny_W[IX2(j, e, np)] = xe / sW;
      double Xe = (xL + xR) / 2.0 + Jx * (1.0);
      wavy_partials(Xe, Y, a, &xX, &xY, &yX, &yY);
      xe = xY * Jy;
      ye = yY * Jy;
      double sE = jmax(sqrt(ye * ye + xe * xe), EPS);
      s->sJ_E[IX2(j, e, np)] = sE;
      s->nx_E[IX2(j, e, np)] = ye / sE;
      s->ny_E[IX2(j, e, np)] = -xe / sE;
    }
    for (int i = 0; i < np; ++i) {
      double X = (xL + xR) / 2.0 + Jx * xi[i];
      double xX, xY, yX, yY;
      double Ys = (yB + yT) / 2.0 + Jy * (-1.0);
      wavy_partials(X, Ys, a, &xX, &xY, &yX, &yY);
      double xx = xX * Jx, yx = yX * Jx;
      double sS = jmax(sqrt(yx * yx + xx * xx), EPS);
      s->sJ_S[IX2(i, e, np)] = sS;
      s->nx_S[IX2(i, e, np)] = yx / sS;
      s->ny_S[IX2(i, e, np)] = -xx / sS;
      double Yn = (yB + yT) / 2.0 + Jy * (1.0);
      wavy_partials(X, Yn, a, &xX, &xY, &yX, &yY);
      xx = xX * Jx;
      yx = yX * Jx;
      double sN = jmax(sqrt(yx * yx + xx * xx), EPS);
      s->sJ_N[IX2(i, e, np)] = sN;
      s->nx_N[IX2(i, e, np)] = -yx / sN;
      s->ny_N[IX2(i, e, np)] = xx / sN;
    }
  }
  for (int e = 0; e < nel; ++e) {
    int jx = e % s->nx, jy = e / s->nx;
    s->h_char[e] = jmin(s->dx2[jx], s->dy2[jy]);
  }
}

/* Mesh2D, src/mesh/Mesh2D.jl:98-154; metrics per allocate_state,
   src/solvestate/SolutionState2D.jl:152-158 */
orc_solver* orc_create_2d(int p, int points, int nx, int ny, double xl,
                          double xr, double yb, double yt, const orc_bc* bcs4,
                          const unsigned char* solid, int wavy, double amp,
                          double gamma, int flux, int time_scheme, int method,
                          int av_form, double kappa, double s0_factor,
                          double eps_floor, double c_av) {
  if (nx < 1 || ny < 1 || !(xr > xl) || !(yt > yb)) return NULL;
  if ((bcs4[0].kind == ORC_BC_PERIODIC) != (bcs4[1].kind == ORC_BC_PERIODIC)) return NULL;
  if ((bcs4[2].kind == ORC_BC_PERIODIC) != (bcs4[3].kind == ORC_BC_PERIODIC)) return NULL;
  orc_solver* s = (orc_solver*)calloc(1, sizeof(orc_solver));
  if (orc_build_operators(p, points, &s->ops) != 0) {
    free(s);
    return NULL;
  }
  s->dim = 2;
  s->np = p + 1;
  s->nx = nx;
  s->ny = ny;
  s->nel = nx * ny;
  s->neq = 4;
  s->gamma = gamma;
  s->flux = flux;
  s->flux_override = -1;
  s->flux_alpha = 1.0;
  s->trace_override = 0;
  s->trace_p0 = 0.0;
  s->trace_p1 = 0.0;
  s->time_scheme = time_scheme;
  s->method = method;
  s->av_form = av_form;
  s->kappa = kappa;
  s->s0_factor = s0_factor;
  s->eps_floor = eps_floor;
  s->c_av = c_av;
  for (int k = 0; k < 4; ++k) s->bc[k] = bcs4[k];
  s->xv2 = dalloc(nx + 1);
  s->yv2 = dalloc(ny + 1);
  s->dx2 = dalloc(nx);
  s->dy2 = dalloc(ny);
  s->Jx = dalloc(nx);
  s->Jy = dalloc(ny);
  julia_linspace(xl, xr, nx + 1, s->xv2);
  julia_linspace(yb, yt, ny + 1, s->yv2);
  for (int i = 0; i < nx; ++i) {
    s->dx2[i] = s->xv2[i + 1] - s->xv2[i];
    s->Jx[i] = s->dx2[i] / 2.0;
  }
  for (int i = 0; i < ny; ++i) {
    s->dy2[i] = s->yv2[i + 1] - s->yv2[i];
    s->Jy[i] = s->dy2[i] / 2.0;
  }
  s->wavy = wavy;
  s->amp = amp;
  int np = s->np, nel = s->nel;
  size_t nsp = (size_t)np * np * nel, nfp = (size_t)np * nel;
  s->mx = dalloc(nsp);
  s->my = dalloc(nsp);
  s->x_xi = dalloc(nsp);
  s->x_eta = dalloc(nsp);
  s->y_xi = dalloc(nsp);
  s->y_eta = dalloc(nsp);
  s->J2 = dalloc(nsp);
  double** fa[12] = {&s->nx_W, &s->ny_W, &s->sJ_W, &s->nx_E, &s->ny_E, &s->sJ_E,
                     &s->nx_S, &s->ny_S, &s->sJ_S, &s->nx_N, &s->ny_N, &s->sJ_N};
  for (int k = 0; k < 12; ++k) *fa[k] = dalloc(nfp);
  s->h_char = dalloc(nel);
  if (wavy == 1)
    build_metrics_wavy(s);
  else
    build_metrics_discrete(s, wavy == 2);
  if (solid) {
    s->solid = (unsigned char*)calloc(nel, 1);
    memcpy(s->solid, solid, nel);
  }
  common_alloc(s);
  size_t ntr = (size_t)np * 4 * nel;
  double** ta[8] = {&s->trW, &s->trE, &s->trS, &s->trN, &s->fhW, &s->fhE, &s->fhS, &s->fhN};
  for (int k = 0; k < 8; ++k) *ta[k] = dalloc(ntr);
  s->gx = dalloc(orc_ndof(s));
  s->gy = dalloc(orc_ndof(s));
  double** ba[12] = {&s->bW, &s->bE, &s->bS, &s->bN, &s->gW, &s->gE,
                     &s->gS, &s->gN, &s->ghW, &s->ghE, &s->ghS, &s->ghN};
  for (int k = 0; k < 12; ++k) *ba[k] = dalloc(ntr);
  return s;
}

void orc_destroy(orc_solver* s) {
  if (!s) return;
  double* ptrs[] = {s->xv, s->dx, s->J1, s->xv2, s->yv2, s->dx2, s->dy2, s->Jx,
                    s->Jy, s->mx, s->my, s->x_xi, s->x_eta, s->y_xi, s->y_eta,
                    s->J2, s->nx_W, s->ny_W, s->sJ_W, s->nx_E, s->ny_E, s->sJ_E,
                    s->nx_S, s->ny_S, s->sJ_S, s->nx_N, s->ny_N, s->sJ_N,
                    s->h_char, s->u, s->du, s->u0, s->u1, s->u2, s->u_work,
                    s->trL, s->trR, s->fL, s->fR, s->trW, s->trE, s->trS, s->trN,
                    s->fhW, s->fhE, s->fhS, s->fhN, s->sigma, s->eps_e, s->g,
                    s->gx, s->gy, s->bW, s->bE, s->bS, s->bN, s->gW, s->gE,
                    s->gS, s->gN, s->ghW, s->ghE, s->ghS, s->ghN};
  for (size_t k = 0; k < sizeof(ptrs) / sizeof(ptrs[0]); ++k) free(ptrs[k]);
  free(s->solid);
  free(s);
}

const double* orc_metric(const orc_solver* s, const char* name) {
  if (s->dim != 2) return NULL;
  struct {
    const char* n;
    const double* p;
  } tab[] = {{"x", s->mx},        {"y", s->my},       {"x_xi", s->x_xi},
             {"x_eta", s->x_eta}, {"y_xi", s->y_xi},  {"y_eta", s->y_eta},
             {"J", s->J2},        {"nx_W", s->nx_W},  {"ny_W", s->ny_W},
             {"sJ_W", s->sJ_W},   {"nx_E", s->nx_E},  {"ny_E", s->ny_E},
             {"sJ_E", s->sJ_E},   {"nx_S", s->nx_S},  {"ny_S", s->ny_S},
             {"sJ_S", s->sJ_S},   {"nx_N", s->nx_N},  {"ny_N", s->ny_N},
             {"sJ_N", s->sJ_N},   {"h_char", s->h_char}};
  for (size_t k = 0; k < sizeof(tab) / sizeof(tab[0]); ++k)
    if (strcmp(tab[k].n, name) == 0) return tab[k].p;
  return NULL;
}

/* physical_coords (src/mesh/Mesh1D.jl:45-52) / physical_coords_2d
   (src/mesh/Mesh2D.jl:172-185), solution-point order of the state */
void orc_physical_coords(const orc_solver* s, double* x, double* y) {
  int np = s->np;
  if (s->dim == 1) {
    for (int e = 0; e < s->nel; ++e) {
      double mid = (s->xv[e] + s->xv[e + 1]) / 2.0;
      for (int j = 0; j < np; ++j) x[j + np * e] = mid + s->J1[e] * s->ops.xi[j];
    }
    return;
  }
  for (int e = 0; e < s->nel; ++e)
    for (int j = 0; j < np; ++j)
      for (int i = 0; i < np; ++i)
        physical_xy(s, e, s->ops.xi[i], s->ops.xi[j], &x[IX3(i, j, e, np)],
                    &y[IX3(i, j, e, np)]);
}

/* ------------------------------------------------------------- Euler 1D */

/* pressure, src/equations/Euler.jl:18-22 */
static inline double pressure1(double g, const double* U) {
  double rs = jmax(U[0], EPS);
  double u = U[1] / rs;
  return (g - 1.0) * (U[2] - 0.5 * rs * u * u);
}
/* sound_speed, Euler.jl:37-41 */
static inline double sound1(double g, const double* U) {
  double r = jmax(U[0], EPS);
  double p = jmax(pressure1(g, U), EPS);
  return sqrt(g * p / r);
}
static inline double velocity1(const double* U) { return U[1] / jmax(U[0], EPS); }
/* physical_flux!, Euler.jl:88-99 (divides by the unfloored density) */
static inline void pflux1(double g, const double* U, double* f) {
  double r = U[0], ru = U[1], E = U[2];
  double u = ru / r;
  double p = pressure1(g, U);
  f[0] = ru;
  f[1] = ru * u + p;
  f[2] = (E + p) * u;
}
/* rusanov_flux, src/flux/Rusanov.jl:10-25 with max_wave_speed Euler.jl:107-113;
   alpha scales the dissipation (1 for the reference's flux, exactly) */
static void rusanov_1d_scaled(double g, const double* uL, const double* uR, double alpha, double* out) {
  double fl[3], fr[3];
  pflux1(g, uL, fl);
  pflux1(g, uR, fr);
  double lam = jmax(fabs(velocity1(uL)) + sound1(g, uL), fabs(velocity1(uR)) + sound1(g, uR));
  lam = alpha * lam;
  for (int c = 0; c < 3; ++c) out[c] = 0.5 * (fl[c] + fr[c]) - 0.5 * lam * (uR[c] - uL[c]);
}
void orc_rusanov_1d(double g, const double* uL, const double* uR, double* out) {
  rusanov_1d_scaled(g, uL, uR, 1.0, out);
}
/* hllc_flux, src/flux/HLLC.jl:9-69 */
void orc_hllc_1d(double g, const double* uL, const double* uR, double* out) {
  double rL = jmax(uL[0], EPS), rR = jmax(uR[0], EPS);
  double vL = uL[1] / rL, vR = uR[1] / rR;
  double pL = jmax(pressure1(g, uL), EPS), pR = jmax(pressure1(g, uR), EPS);
  double cL = sqrt(g * pL / rL), cR = sqrt(g * pR / rR);
  double SL = jmin(vL - cL, vR - cR);
  double SR = jmax(vL + cL, vR + cR);
  double num = pR - pL + rL * vL * (SL - vL) - rR * vR * (SR - vR);
  double den = rL * (SL - vL) - rR * (SR - vR);
  double SM = (fabs(den) < EPS) ? 0.5 * (vL + vR) : num / den;
  double FL[3], FR[3];
  pflux1(g, uL, FL);
  pflux1(g, uR, FR);
  if (0.0 <= SL) {
    for (int c = 0; c < 3; ++c) out[c] = FL[c];
    return;
  } else if (0.0 >= SR) {
    for (int c = 0; c < 3; ++c) out[c] = FR[c];
    return;
  }
  const double *U, *F;
  double r, v, p, S;
  if (SL <= 0.0 && 0.0 <= SM) {
    U = uL; F = FL; r = rL; v = vL; p = pL; S = SL;
  } else {
    U = uR; F = FR; r = rR; v = vR; p = pR; S = SR;
  }
  double factor = r * (S - v) / (S - SM);
  double e_int = U[2] / r + (SM - v) * (SM + p / (r * (S - v)));
  double Us[3] = {factor, factor * SM, factor * e_int};
  for (int c = 0; c < 3; ++c) out[c] = F[c] + S * (Us[c] - U[c]);
}
/* _resolve_flux (src/fr/Residual.jl:9-15): the method's numerical_flux_method
   override when it has one, else the scheme's interface_flux */
static inline void iflux1(const orc_solver* s, const double* um, const double* up, double* out) {
  const int kind = s->flux_override >= 0 ? s->flux_override : s->flux;
  if (kind == ORC_FLUX_HLLC)
    orc_hllc_1d(s->gamma, um, up, out);
  else
    rusanov_1d_scaled(s->gamma, um, up, s->flux_override >= 0 ? s->flux_alpha : 1.0, out);
}

/* A 1D method's numerical_flux_method override (plugin fluxes of the
   checker): kind -1 clears it; ORC_FLUX_RUSANOV with its dissipation scaled
   by alpha; ORC_FLUX_HLLC.  The 2D residual ignores overrides, as the
   reference's does. */
void orc_set_flux_override(orc_solver* s, int kind, double alpha) {
  s->flux_override = kind;
  s->flux_alpha = alpha;
}

/* ------------------------------------------------------------- Euler 2D */

/* pressure, src/equations/Euler2D.jl:14-19 */
static inline double pressure2(double g, const double* U) {
  double r = jmax(U[0], EPS);
  double u = U[1] / r, v = U[2] / r;
  return (g - 1.0) * (U[3] - 0.5 * r * (u * u + v * v));
}
static inline double sound2(double g, const double* U) {
  double r = jmax(U[0], EPS);
  double p = jmax(pressure2(g, U), EPS);
  return sqrt(g * p / r);
}
/* physical_flux_x! / physical_flux_y!, Euler2D.jl:54-79 */
static inline void pflux_x(double g, const double* U, double* f) {
  double u = U[1] / jmax(U[0], EPS);
  double p = pressure2(g, U);
  f[0] = U[1];
  f[1] = U[1] * u + p;
  f[2] = U[2] * u;
  f[3] = (U[3] + p) * u;
}
static inline void pflux_y(double g, const double* U, double* f) {
  double v = U[2] / jmax(U[0], EPS);
  double p = pressure2(g, U);
  f[0] = U[2];
  f[1] = U[1] * v;
  f[2] = U[2] * v + p;
  f[3] = (U[3] + p) * v;
}
/* max_wave_speed_n, Euler2D.jl:81-90 */
static inline double spd_n(double g, const double* U, double nx, double ny) {
  double r = jmax(U[0], EPS);
  double u = U[1] / r, v = U[2] / r;
  double un = u * nx + v * ny;
  return fabs(un) + sound2(g, U);
}
/* numerical_flux_n!, Euler2D.jl:114-150 */
void orc_rusanov_2d(double g, const double* uL, const double* uR, double nx,
                    double ny, double* out) {
  double rL = jmax(uL[0], EPS);
  double uL_ = uL[1] / rL, vL_ = uL[2] / rL;
  double pL = pressure2(g, uL);
  double rR = jmax(uR[0], EPS);
  double uR_ = uR[1] / rR, vR_ = uR[2] / rR;
  double pR = pressure2(g, uR);
  double fL1 = uL[1] * nx + uL[2] * ny;
  double fL2 = (uL[1] * uL_ + pL) * nx + (uL[1] * vL_) * ny;
  double fL3 = (uL[2] * uL_) * nx + (uL[2] * vL_ + pL) * ny;
  double fL4 = (uL[3] + pL) * (uL_ * nx + vL_ * ny);
  double fR1 = uR[1] * nx + uR[2] * ny;
  double fR2 = (uR[1] * uR_ + pR) * nx + (uR[1] * vR_) * ny;
  double fR3 = (uR[2] * uR_) * nx + (uR[2] * vR_ + pR) * ny;
  double fR4 = (uR[3] + pR) * (uR_ * nx + vR_ * ny);
  double lam = jmax(spd_n(g, uL, nx, ny), spd_n(g, uR, nx, ny));
  double h = 0.5;
  out[0] = h * (fL1 + fR1) - h * lam * (uR[0] - uL[0]);
  out[1] = h * (fL2 + fR2) - h * lam * (uR[1] - uL[1]);
  out[2] = h * (fL3 + fR3) - h * lam * (uR[2] - uL[2]);
  out[3] = h * (fL4 + fR4) - h * lam * (uR[3] - uL[3]);
}
/* hllc_flux_n, src/flux/HLLC.jl:72-148 */
void orc_hllc_2d(double g, const double* uL, const double* uR, double nx_in,
                 double ny_in, double* out) {
  double nrm = hypot(nx_in, ny_in);
  if (nrm < EPS) {
    orc_rusanov_2d(g, uL, uR, nx_in, ny_in, out);
    return;
  }
  double nx = nx_in / nrm, ny = ny_in / nrm;
  double rL = jmax(uL[0], EPS), rR = jmax(uR[0], EPS);
  double uL_ = uL[1] / rL, vL_ = uL[2] / rL, uR_ = uR[1] / rR, vR_ = uR[2] / rR;
  double pL = jmax(pressure2(g, uL), EPS), pR = jmax(pressure2(g, uR), EPS);
  double unL = uL_ * nx + vL_ * ny, unR = uR_ * nx + vR_ * ny;
  double cL = sqrt(g * pL / rL), cR = sqrt(g * pR / rR);
  double SL = jmin(unL - cL, unR - cR);
  double SR = jmax(unL + cL, unR + cR);
  double num = pR - pL + rL * unL * (SL - unL) - rR * unR * (SR - unR);
  double den = rL * (SL - unL) - rR * (SR - unR);
  double SM = fabs(den) < EPS ? 0.5 * (unL + unR) : num / den;
  double fxL[4], gyL[4], fxR[4], gyR[4], fL[4], fR[4];
  pflux_x(g, uL, fxL);
  pflux_y(g, uL, gyL);
  pflux_x(g, uR, fxR);
  pflux_y(g, uR, gyR);
  for (int c = 0; c < 4; ++c) {
    fL[c] = fxL[c] * nx + gyL[c] * ny;
    fR[c] = fxR[c] * nx + gyR[c] * ny;
  }
  if (0.0 <= SL) {
    for (int c = 0; c < 4; ++c) out[c] = fL[c];
    return;
  } else if (0.0 >= SR) {
    for (int c = 0; c < 4; ++c) out[c] = fR[c];
    return;
  }
  const double *U, *F;
  double r, u, v, p, un, S;
  if (SL <= 0.0 && 0.0 <= SM) {
    U = uL; F = fL; r = rL; u = uL_; v = vL_; p = pL; un = unL; S = SL;
  } else {
    U = uR; F = fR; r = rR; u = uR_; v = vR_; p = pR; un = unR; S = SR;
  }
  double ut_x = u - un * nx, ut_y = v - un * ny;
  double u_star = ut_x + SM * nx, v_star = ut_y + SM * ny;
  double factor = r * (S - un) / (S - SM);
  double e_star = U[3] / r + (SM - un) * (SM + p / (r * (S - un)));
  double Us[4] = {factor, factor * u_star, factor * v_star, factor * e_star};
  for (int c = 0; c < 4; ++c) out[c] = F[c] + S * (Us[c] - U[c]);
}
/* interface_flux_n!, src/flux/HLLC.jl:182-200 */
static inline void iflux2(const orc_solver* s, const double* um, const double* up,
                          double nx, double ny, double* out) {
  if (s->flux == ORC_FLUX_HLLC)
    orc_hllc_2d(s->gamma, um, up, nx, ny, out);
  else
    orc_rusanov_2d(s->gamma, um, up, nx, ny, out);
}

/* reflect_conserved, src/mesh/BoundaryConditions.jl:43-60 */
static void reflect_conserved(int neq, const double* U, double nx, double ny, double* out) {
  double r = jmax(U[0], EPS);
  double u = U[1] / r;
  double v = neq >= 3 ? U[2] / r : 0.0;
  if (neq == 3) v = 0.0; /* 1D Euler: no y-momentum */
  double un = u * nx + v * ny;
  double ug = u - 2 * un * nx;
  double vg = v - 2 * un * ny;
  if (neq == 3) {
    out[0] = r;
    out[1] = r * ug;
    out[2] = U[2];
  } else {
    out[0] = r;
    out[1] = r * ug;
    out[2] = r * vg;
    out[3] = U[3];
  }
}

/* exterior_state, src/mesh/BoundaryConditions.jl:67-134 (x-split = the
   double-Mach GhostStateBC closures, src/verification/Cases2D_Optional.jl:72-84) */
static void exterior_state(const orc_bc* bc, int neq, const double* ui, double nx,
                           double ny, double x, double t, double* ug) {
  switch (bc->kind) {
    case ORC_BC_TRANSMISSIVE:
      for (int c = 0; c < neq; ++c) ug[c] = ui[c];
      return;
    case ORC_BC_REFLECTING:
      reflect_conserved(neq, ui, nx, ny, ug);
      return;
    case ORC_BC_DIRICHLET:
      for (int c = 0; c < neq; ++c) ug[c] = bc->state[c];
      return;
    case ORC_BC_XSPLIT: {
      double xs = bc->x0 + (bc->s0 + bc->s1 * t) / bc->sdiv;
      if (x < xs) {
        for (int c = 0; c < neq; ++c) ug[c] = bc->state[c];
      } else if (bc->mode == 0) {
        reflect_conserved(neq, ui, nx, ny, ug);
      } else {
        for (int c = 0; c < neq; ++c) ug[c] = bc->state_b[c];
      }
      return;
    }
    default:
      for (int c = 0; c < neq; ++c) ug[c] = NAN;
  }
}

/* --------------------------------------------------- Persson sensor / LU */

/* LU with partial pivoting (dgetf2 form: first max-|a| pivot, reciprocal
   scaling of the column, rank-1 update); in place, column-major */
static void lu_factor(int n, double* A, int* piv) {
  for (int j = 0; j < n; ++j) {
    int p = j;
    double amax = fabs(A[j + n * j]);
    for (int i = j + 1; i < n; ++i)
      if (fabs(A[i + n * j]) > amax) {
        amax = fabs(A[i + n * j]);
        p = i;
      }
    piv[j] = p;
    if (p != j)
      for (int k = 0; k < n; ++k) {
        double tmp = A[j + n * k];
        A[j + n * k] = A[p + n * k];
        A[p + n * k] = tmp;
      }
    if (A[j + n * j] != 0.0) {
      if (fabs(A[j + n * j]) >= DBL_MIN) {
        double r = 1.0 / A[j + n * j];
        for (int i = j + 1; i < n; ++i) A[i + n * j] *= r;
      } else {
        for (int i = j + 1; i < n; ++i) A[i + n * j] /= A[j + n * j];
      }
    }
    for (int k = j + 1; k < n; ++k) {
      double akj = A[j + n * k];
      if (akj != 0.0)
        for (int i = j + 1; i < n; ++i) A[i + n * k] -= A[i + n * j] * akj;
    }
  }
}
/* row interchanges, then dtrsm (lower unit) and dtrsm (upper) column forms */
static void lu_solve(int n, const double* LU, const int* piv, double* b) {
  for (int j = 0; j < n; ++j)
    if (piv[j] != j) {
      double tmp = b[j];
      b[j] = b[piv[j]];
      b[piv[j]] = tmp;
    }
  for (int k = 0; k < n; ++k)
    if (b[k] != 0.0)
      for (int i = k + 1; i < n; ++i) b[i] -= b[k] * LU[i + n * k];
  for (int k = n - 1; k >= 0; --k)
    if (b[k] != 0.0) {
      b[k] /= LU[k + n * k];
      for (int i = 0; i < k; ++i) b[i] -= b[k] * LU[i + n * k];
    }
}

/* persson_s0 / persson_sigma, src/capturing/SharedAV.jl:9-21 */
static inline double persson_s0(int p, double s0f) { return s0f * log10((double)(p > 1 ? p : 1)); }
static inline double persson_sigma(double eh, double et, double s0, double kappa, double ef) {
  double se = log10(eh / et + ef);
  return 1.0 / (1.0 + exp(-kappa * (se - s0)));
}
/* sum(abs2, x): first two terms, then left-to-right */
static double sum_abs2(int n, const double* x) {
  if (n == 1) return x[0] * x[0];
  double v = x[0] * x[0] + x[1] * x[1];
  for (int i = 2; i < n; ++i) v += x[i] * x[i];
  return v;
}

/* sense! 1D, src/capturing/PerssonAV.jl:116-135 */
static void sense_1d(orc_solver* s, const double* uw, double* sigma) {
  int np = s->np, nel = s->nel;
  double LU[ORC_MAXNP * ORC_MAXNP];
  int piv[ORC_MAXNP];
  memcpy(LU, s->ops.V, sizeof(double) * np * np);
  lu_factor(np, LU, piv);
  double s0 = persson_s0(s->ops.p, s->s0_factor);
#pragma omp parallel for schedule(static)
  for (int e = 0; e < nel; ++e) {
    double uh[ORC_MAXNP];
    for (int j = 0; j < np; ++j) uh[j] = uw[j + np * e]; /* density */
    lu_solve(np, LU, piv, uh);
    double e_high = uh[np - 1] * uh[np - 1];
    double e_tot = sum_abs2(np, uh) + s->eps_floor;
    sigma[e] = persson_sigma(e_high, e_tot, s0, s->kappa, s->eps_floor);
  }
}

/* sense! 2D, src/capturing/PerssonAV2D.jl:20-59: Uhat = (V \ U) / V' */
static void sense_2d(orc_solver* s, const double* uw, double* sigma) {
  int np = s->np, nel = s->nel;
  double LU[ORC_MAXNP * ORC_MAXNP];
  int piv[ORC_MAXNP];
  memcpy(LU, s->ops.V, sizeof(double) * np * np);
  lu_factor(np, LU, piv);
  double s0 = persson_s0(s->ops.p, s->s0_factor);
#pragma omp parallel for schedule(static)
  for (int e = 0; e < nel; ++e) {
    double X[ORC_MAXNP * ORC_MAXNP], Y[ORC_MAXNP * ORC_MAXNP], Uh[ORC_MAXNP * ORC_MAXNP] = {0};
    for (int j = 0; j < np; ++j)
      for (int i = 0; i < np; ++i) X[i + np * j] = uw[IX3(i, j, e, np)];
    for (int j = 0; j < np; ++j) lu_solve(np, LU, piv, &X[np * j]);
    /* Xhat / V' == (V \ Xhat')' */
    for (int j = 0; j < np; ++j)
      for (int i = 0; i < np; ++i) Y[i + np * j] = X[j + np * i];
    for (int j = 0; j < np; ++j) lu_solve(np, LU, piv, &Y[np * j]);
    for (int j = 0; j < np; ++j)
      for (int i = 0; i < np; ++i) Uh[i + np * j] = Y[j + np * i];
    double e_tot = sum_abs2(np * np, Uh) + s->eps_floor;
    double e_high = 0.0;
    for (int j = 0; j < np; ++j) e_high += Uh[(np - 1) + np * j] * Uh[(np - 1) + np * j];
    for (int i = 0; i < np - 1; ++i) e_high += Uh[i + np * (np - 1)] * Uh[i + np * (np - 1)];
    sigma[e] = persson_sigma(e_high, e_tot, s0, s->kappa, s->eps_floor);
  }
}

/* element_viscosities (1D) src/capturing/PerssonAV.jl:138-177 */
static void element_viscosities_1d(orc_solver* s, const double* uw, const double* sigma,
                                   double* eps_e) {
  int np = s->np, nel = s->nel;
  int p = s->ops.p > 1 ? s->ops.p : 1;
  size_t cs = (size_t)np * nel;
  for (int e = 0; e < nel; ++e) {
    eps_e[e] = 0.0;
    double se = sigma[e];
    if (se <= 0.0) continue;
    double h = s->dx[e];
    double m = 0.0;
    for (int j = 0; j < np; ++j) {
      double U[3] = {uw[j + np * e], uw[j + np * e + cs], uw[j + np * e + 2 * cs]};
      m = jmax(m, fabs(velocity1(U)) + sound1(s->gamma, U));
    }
    double lam = jmax(m, EPS);
    eps_e[e] = s->c_av * se * (h / (double)p) * lam;
  }
}

/* element_viscosities_2d, src/capturing/PerssonAV2D.jl:62-109 */
static void element_viscosities_2d(orc_solver* s, const double* uw, const double* sigma,
                                   double* eps_e) {
  int np = s->np, nel = s->nel;
  int p = s->ops.p > 1 ? s->ops.p : 1;
  size_t cs = (size_t)np * np * nel;
#pragma omp parallel for schedule(static)
  for (int e = 0; e < nel; ++e) {
    eps_e[e] = 0.0;
    double se = sigma[e];
    if (se <= 0.0) continue;
    double h = s->h_char[e];
    double m = 0.0;
    for (int j = 0; j < np; ++j)
      for (int i = 0; i < np; ++i) {
        size_t id = IX3(i, j, e, np);
        double U[4] = {uw[id], uw[id + cs], uw[id + 2 * cs], uw[id + 3 * cs]};
        double r = jmax(U[0], EPS);
        double u = U[1] / r, v = U[2] / r;
        double c = sound2(s->gamma, U);
        m = jmax(jmax(m, fabs(u) + c), fabs(v) + c);
      }
    double lam = jmax(m, EPS);
    eps_e[e] = s->c_av * se * (h / (double)p) * lam;
  }
}

/* br0_tau_1d / br0_avg_flux, src/capturing/SharedAV.jl:29-42 */
static inline double br0_tau(double em, double ep, double hm, double hp, int p) {
  double eb = 0.5 * (em + ep);
  double hb = 0.5 * (hm + hp);
  return 2.0 * eb * (double)(p + 1) / jmax(hb, EPS);
}
static inline double br0_avg(double gm, double gp, double um, double up, double tau) {
  return 0.5 * (gm + gp) - tau * (up - um);
}

/* ------------------------------------------------------------ 1D residual */

/* apply_dissipation_br0!, src/capturing/PerssonAV.jl:249-351 */
static void br0_1d(orc_solver* s, double* du, const double* uw) {
  int np = s->np, nel = s->nel, neq = 3, p = s->ops.p;
  const double *D = s->ops.D, *lL = s->ops.lL, *lR = s->ops.lR;
  const double *gLx = s->ops.gLxi, *gRx = s->ops.gRxi;
  double* eps = s->eps_e;
  element_viscosities_1d(s, uw, s->sigma, eps);
  size_t cs = (size_t)np * nel;
  double *g = s->g, *uL = s->bW, *uR = s->bE, *gL = s->gW, *gR = s->gE;
  double *ghL = s->ghW, *ghR = s->ghE;
  for (int e = 0; e < nel; ++e) {
    double J = s->J1[e], ee = eps[e];
    for (int c = 0; c < neq; ++c) {
      const double* ue = uw + c * cs + (size_t)np * e;
      double* ge = g + c * cs + (size_t)np * e;
      for (int j = 0; j < np; ++j) {
        double dq = 0.0;
        for (int k = 0; k < np; ++k) dq += D[j + np * k] * ue[k];
        ge[j] = ee * dq / J;
      }
      double suL = 0, suR = 0, sgL = 0, sgR = 0;
      for (int j = 0; j < np; ++j) {
        suL += lL[j] * ue[j];
        suR += lR[j] * ue[j];
        sgL += lL[j] * ge[j];
        sgR += lR[j] * ge[j];
      }
      uL[e + nel * c] = suL;
      uR[e + nel * c] = suR;
      gL[e + nel * c] = sgL;
      gR[e + nel * c] = sgR;
    }
  }
#define BR0F(el, er, c)                                                           \
  br0_avg(gR[(el) + nel * (c)], gL[(er) + nel * (c)], uR[(el) + nel * (c)],       \
          uL[(er) + nel * (c)], br0_tau(eps[el], eps[er], s->dx[el], s->dx[er], p))
  for (int e = 0; e < nel - 1; ++e)
    for (int c = 0; c < neq; ++c) {
      double gh = BR0F(e, e + 1, c);
      ghR[e + nel * c] = gh;
      ghL[e + 1 + nel * c] = gh;
    }
  if (s->bc[0].kind == ORC_BC_PERIODIC) {
    for (int c = 0; c < neq; ++c) {
      double gh = BR0F(nel - 1, 0, c);
      ghR[nel - 1 + nel * c] = gh;
      ghL[0 + nel * c] = gh;
    }
  } else {
    for (int c = 0; c < neq; ++c) {
      ghL[0 + nel * c] = gL[0 + nel * c];
      ghR[nel - 1 + nel * c] = gR[nel - 1 + nel * c];
    }
  }
#undef BR0F
  for (int e = 0; e < nel; ++e) {
    double J = s->J1[e];
    for (int c = 0; c < neq; ++c) {
      const double* ge = g + c * cs + (size_t)np * e;
      for (int j = 0; j < np; ++j) {
        double vol = 0.0;
        for (int k = 0; k < np; ++k) vol += D[j + np * k] * ge[k];
        double corr = (ghL[e + nel * c] - gL[e + nel * c]) * gLx[j] +
                      (ghR[e + nel * c] - gR[e + nel * c]) * gRx[j];
        du[c * cs + (size_t)np * e + j] += (vol + corr) / J;
      }
    }
  }
}

/* apply_dissipation_local_DD!, src/capturing/PerssonAV.jl:203-240 */
static void local_dd_1d(orc_solver* s, double* du, const double* uw) {
  int np = s->np, nel = s->nel, neq = 3;
  const double* D = s->ops.D;
  double* eps = s->eps_e;
  element_viscosities_1d(s, uw, s->sigma, eps);
  size_t cs = (size_t)np * nel;
  double v[ORC_MAXNP];
  for (int e = 0; e < nel; ++e) {
    double ee = eps[e];
    if (ee <= 0.0) continue;
    double J = s->J1[e];
    double scale = ee / (J * J);
    for (int c = 0; c < neq; ++c) {
      const double* ue = uw + c * cs + (size_t)np * e;
      for (int j = 0; j < np; ++j) {
        double a = 0.0;
        for (int k = 0; k < np; ++k) a += D[j + np * k] * ue[k];
        v[j] = a;
      }
      for (int j = 0; j < np; ++j) {
        double a = 0.0;
        for (int k = 0; k < np; ++k) a += D[j + np * k] * v[k];
        du[c * cs + (size_t)np * e + j] += scale * a;
      }
    }
  }
}

/* smallest root in [0, 1] of a t^2 + b t + c with c > 0 >= a + b + c, the
   stable quadratic formula (the pressure condition of the Zhang & Shu
   positivity-preserving scaling, J. Comput. Phys. 229 (2010) 8918-8934) */
static double root01(double a, double b, double c) {
  if (fabs(a) < 1e-300) return b != 0.0 ? fmin(fmax(-c / b, 0.0), 1.0) : 0.0;
  double disc = fmax(b * b - 4.0 * a * c, 0.0);
  double q = -0.5 * (b + copysign(sqrt(disc), b));
  double r1 = q / a, r2 = q != 0.0 ? c / q : 2.0;
  double t = 1.0;
  if (r1 >= 0.0 && r1 <= 1.0) t = fmin(t, r1);
  if (r2 >= 0.0 && r2 <= 1.0) t = fmin(t, r2);
  return t;
}

/* A method's extrapolate_interface! override (Interfaces.jl:49-71 is the
   default, "Override for hybrid reconstruction") applied to one element's
   traces tl (xi = -1) and tr (xi = +1) given its mean m: ORC_TRACE_MEAN
   pulls them toward the mean by p0 in [0, 1]; ORC_TRACE_POSITIVITY scales
   them toward it until density >= p0 and then pressure >= p1 (Zhang & Shu),
   an element with an inadmissible mean left as it is. */
static void trace_override_1d(const orc_solver* s, const double* m, double* tl, double* tr) {
  const double g1 = s->gamma - 1.0;
  if (s->trace_override == ORC_TRACE_MEAN) {
    for (int c = 0; c < 3; ++c) {
      tl[c] = m[c] + s->trace_p0 * (tl[c] - m[c]);
      tr[c] = m[c] + s->trace_p0 * (tr[c] - m[c]);
    }
    return;
  }
  if (s->trace_override != ORC_TRACE_POSITIVITY) return;
  const double er = s->trace_p0, ep = s->trace_p1;
  const double pbar = g1 * (m[2] - 0.5 * m[1] * m[1] / m[0]);
  if (!(m[0] > er) || !(pbar > ep)) return;
  const double rmin = fmin(tl[0], tr[0]);
  if (rmin < er) {
    const double th = (m[0] - er) / (m[0] - rmin);
    tl[0] = m[0] + th * (tl[0] - m[0]);
    tr[0] = m[0] + th * (tr[0] - m[0]);
  }
  double theta = 1.0;
  for (int side = 0; side < 2; ++side) {
    const double* U = side == 0 ? tl : tr;
    const double pk = g1 * (U[2] - 0.5 * U[1] * U[1] / U[0]);
    if (pk >= ep) continue;
    const double d0 = U[0] - m[0], d1 = U[1] - m[1], d2 = U[2] - m[2];
    const double a = g1 * (d2 * d0 - 0.5 * d1 * d1);
    const double b = g1 * (m[2] * d0 + m[0] * d2 - m[1] * d1) - ep * d0;
    const double cc = m[0] * (pbar - ep);
    theta = fmin(theta, root01(a, b, cc));
  }
  if (theta < 1.0)
    for (int c = 0; c < 3; ++c) {
      tl[c] = m[c] + theta * (tl[c] - m[c]);
      tr[c] = m[c] + theta * (tr[c] - m[c]);
    }
}

void orc_set_trace_override(orc_solver* s, int kind, double p0, double p1) {
  s->trace_override = kind;
  s->trace_p0 = p0;
  s->trace_p1 = p1;
}

/* the 1D traces the last residual's interface fluxes used, [nel, 3] each
   (Julia layout: trL[e + nel*c]) */
void orc_get_traces_1d(const orc_solver* s, double* trL, double* trR) {
  const size_t n = (size_t)s->nel * 3;
  memcpy(trL, s->trL, n * sizeof(double));
  memcpy(trR, s->trR, n * sizeof(double));
}

/* residual! 1D, src/fr/Residual.jl:161-214 (interface fluxes :24-115,
   default extrapolate_interface! src/capturing/Interfaces.jl:49-71) */
static void residual_1d(orc_solver* s, double* du) {
  int np = s->np, nel = s->nel, neq = 3;
  size_t n = orc_ndof(s), cs = (size_t)np * nel;
  double* uw = s->u_work;
  memcpy(uw, s->u, n * sizeof(double));
  const double *lL = s->ops.lL, *lR = s->ops.lR, *D = s->ops.D;
  for (int e = 0; e < nel; ++e)
    for (int c = 0; c < neq; ++c) {
      double sL = 0, sR = 0;
      for (int j = 0; j < np; ++j) {
        sL += lL[j] * uw[c * cs + (size_t)np * e + j];
        sR += lR[j] * uw[c * cs + (size_t)np * e + j];
      }
      s->trL[e + nel * c] = sL;
      s->trR[e + nel * c] = sR;
    }
  if (s->trace_override) {
    double wsum = 0.0;
    for (int j = 0; j < np; ++j) wsum += s->ops.w[j];
    for (int e = 0; e < nel; ++e) {
      double m[3], tl[3], tr[3];
      for (int c = 0; c < neq; ++c) {
        double a = 0.0;
        for (int j = 0; j < np; ++j) a += s->ops.w[j] * uw[c * cs + (size_t)np * e + j];
        m[c] = a / wsum;
        tl[c] = s->trL[e + nel * c];
        tr[c] = s->trR[e + nel * c];
      }
      trace_override_1d(s, m, tl, tr);
      for (int c = 0; c < neq; ++c) {
        s->trL[e + nel * c] = tl[c];
        s->trR[e + nel * c] = tr[c];
      }
    }
  }
  double um[3], up[3], ft[3];
  for (int e = 0; e < nel - 1; ++e) {
    for (int c = 0; c < neq; ++c) {
      um[c] = s->trR[e + nel * c];
      up[c] = s->trL[e + 1 + nel * c];
    }
    iflux1(s, um, up, ft);
    for (int c = 0; c < neq; ++c) {
      s->fR[e + nel * c] = ft[c];
      s->fL[e + 1 + nel * c] = ft[c];
    }
  }
  for (int c = 0; c < neq; ++c) up[c] = s->trL[0 + nel * c];
  const orc_bc* lb = &s->bc[0];
  if (lb->kind == ORC_BC_PERIODIC) {
    for (int c = 0; c < neq; ++c) um[c] = s->trR[nel - 1 + nel * c];
  } else if (lb->kind == ORC_BC_TRANSMISSIVE) {
    for (int c = 0; c < neq; ++c) um[c] = s->trL[0 + nel * c];
  } else {
    for (int c = 0; c < neq; ++c) um[c] = lb->state[c];
  }
  iflux1(s, um, up, ft);
  for (int c = 0; c < neq; ++c) {
    s->fL[0 + nel * c] = ft[c];
    if (lb->kind == ORC_BC_PERIODIC) s->fR[nel - 1 + nel * c] = ft[c];
  }
  const orc_bc* rb = &s->bc[1];
  if (rb->kind != ORC_BC_PERIODIC) {
    for (int c = 0; c < neq; ++c) um[c] = s->trR[nel - 1 + nel * c];
    if (rb->kind == ORC_BC_TRANSMISSIVE) {
      for (int c = 0; c < neq; ++c) up[c] = s->trR[nel - 1 + nel * c];
    } else {
      for (int c = 0; c < neq; ++c) up[c] = rb->state[c];
    }
    iflux1(s, um, up, ft);
    for (int c = 0; c < neq; ++c) s->fR[nel - 1 + nel * c] = ft[c];
  }
  memset(du, 0, n * sizeof(double));
  for (int e = 0; e < nel; ++e) {
    double f[ORC_MAXNP][3];
    for (int j = 0; j < np; ++j) {
      double U[3] = {uw[(size_t)np * e + j], uw[cs + (size_t)np * e + j],
                     uw[2 * cs + (size_t)np * e + j]};
      pflux1(s->gamma, U, f[j]);
    }
    double fLe[3], fRe[3];
    for (int c = 0; c < neq; ++c) {
      double a = 0, b = 0;
      for (int j = 0; j < np; ++j) a += lL[j] * f[j][c];
      for (int j = 0; j < np; ++j) b += lR[j] * f[j][c];
      fLe[c] = a;
      fRe[c] = b;
    }
    double Je = s->J1[e];
    for (int c = 0; c < neq; ++c)
      for (int j = 0; j < np; ++j) {
        double vol = 0.0;
        for (int k = 0; k < np; ++k) vol += D[j + np * k] * f[k][c];
        double corr = (s->fL[e + nel * c] - fLe[c]) * s->ops.gLxi[j] +
                      (s->fR[e + nel * c] - fRe[c]) * s->ops.gRxi[j];
        du[c * cs + (size_t)np * e + j] = -(vol + corr) / Je;
      }
  }
  if (s->method == ORC_METHOD_PERSSON) {
    sense_1d(s, uw, s->sigma);
    if (s->av_form == ORC_AV_BR0)
      br0_1d(s, du, uw);
    else
      local_dd_1d(s, du, uw);
  } else {
    for (int e = 0; e < nel; ++e) s->sigma[e] = 0.0;
  }
}

/* ------------------------------------------------------------ 2D residual */

static inline int is_solid(const orc_solver* s, int e) { return s->solid && s->solid[e]; }

/* face_trace!, src/fr/Residual2D.jl:9-48 */
static void face_traces_2d(orc_solver* s, const double* uw, int e) {
  int np = s->np, nel = s->nel;
  size_t cs = (size_t)np * np * nel;
  const double *lL = s->ops.lL, *lR = s->ops.lR;
  for (int j = 0; j < np; ++j)
    for (int c = 0; c < 4; ++c) {
      double a = 0, b = 0;
      for (int i = 0; i < np; ++i) a += lL[i] * uw[c * cs + IX3(i, j, e, np)];
      for (int i = 0; i < np; ++i) b += lR[i] * uw[c * cs + IX3(i, j, e, np)];
      s->trW[j + np * (c + 4 * (size_t)e)] = a;
      s->trE[j + np * (c + 4 * (size_t)e)] = b;
    }
  for (int i = 0; i < np; ++i)
    for (int c = 0; c < 4; ++c) {
      double a = 0, b = 0;
      for (int j = 0; j < np; ++j) a += lL[j] * uw[c * cs + IX3(i, j, e, np)];
      for (int j = 0; j < np; ++j) b += lR[j] * uw[c * cs + IX3(i, j, e, np)];
      s->trS[i + np * (c + 4 * (size_t)e)] = a;
      s->trN[i + np * (c + 4 * (size_t)e)] = b;
    }
}

#define TR(arr, q, c, e) (arr)[(q) + np * ((c) + 4 * (size_t)(e))]

/* boundary_fhat!, src/fr/Residual2D.jl:63-94 */
static void boundary_fhat(orc_solver* s, double* fh_face, int q, int e, const orc_bc* bc,
                          const double* ui, double nxo, double nyo, double sJ, double x,
                          double y, int into_domain) {
  int np = s->np;
  (void)y;
  double ug[4], fh[4];
  exterior_state(bc, 4, ui, nxo, nyo, x, s->t, ug);
  if (into_domain)
    iflux2(s, ug, ui, -nxo, -nyo, fh);
  else
    iflux2(s, ui, ug, nxo, nyo, fh);
  for (int c = 0; c < 4; ++c) TR(fh_face, q, c, e) = fh[c] * sJ;
}

/* apply_dissipation_br0_2d!, src/capturing/PerssonAV2D.jl:203-398 */
static void br0_2d(orc_solver* s, double* du, const double* uw) {
  int np = s->np, nel = s->nel, nx = s->nx, ny = s->ny, p = s->ops.p;
  size_t cs = (size_t)np * np * nel;
  const double *D = s->ops.D, *lL = s->ops.lL, *lR = s->ops.lR;
  const double *gLx = s->ops.gLxi, *gRx = s->ops.gRxi;
  double* eps = s->eps_e;
  element_viscosities_2d(s, uw, s->sigma, eps);
  double *gx = s->gx, *gy = s->gy;
  double *uW = s->bW, *uE = s->bE, *uS = s->bS, *uN = s->bN;
  double *gxW = s->gW, *gxE = s->gE, *gyS = s->gS, *gyN = s->gN;
  double *ghW = s->ghW, *ghE = s->ghE, *ghS = s->ghS, *ghN = s->ghN;
  /* br0 face arrays are [np, nel, neq] */
#define FB(arr, q, e, c) (arr)[(q) + np * ((size_t)(e) + (size_t)nel * (c))]
#pragma omp parallel for schedule(static)
  for (int e = 0; e < nel; ++e) {
    int jx = e % nx, jy = e / nx;
    double Jx = s->Jx[jx], Jy = s->Jy[jy], ee = eps[e];
    for (int c = 0; c < 4; ++c) {
      const double* U = uw + c * cs;
      for (int j = 0; j < np; ++j)
        for (int i = 0; i < np; ++i) {
          double dxi = 0, deta = 0;
          for (int k = 0; k < np; ++k) {
            dxi += D[i + np * k] * U[IX3(k, j, e, np)];
            deta += D[j + np * k] * U[IX3(i, k, e, np)];
          }
          gx[c * cs + IX3(i, j, e, np)] = ee * dxi / Jx;
          gy[c * cs + IX3(i, j, e, np)] = ee * deta / Jy;
        }
      for (int j = 0; j < np; ++j) {
        double suW = 0, suE = 0, sgW = 0, sgE = 0;
        for (int i = 0; i < np; ++i) {
          suW += lL[i] * U[IX3(i, j, e, np)];
          suE += lR[i] * U[IX3(i, j, e, np)];
          sgW += lL[i] * gx[c * cs + IX3(i, j, e, np)];
          sgE += lR[i] * gx[c * cs + IX3(i, j, e, np)];
        }
        FB(uW, j, e, c) = suW;
        FB(uE, j, e, c) = suE;
        FB(gxW, j, e, c) = sgW;
        FB(gxE, j, e, c) = sgE;
      }
      for (int i = 0; i < np; ++i) {
        double suS = 0, suN = 0, sgS = 0, sgN = 0;
        for (int j = 0; j < np; ++j) {
          suS += lL[j] * U[IX3(i, j, e, np)];
          suN += lR[j] * U[IX3(i, j, e, np)];
          sgS += lL[j] * gy[c * cs + IX3(i, j, e, np)];
          sgN += lR[j] * gy[c * cs + IX3(i, j, e, np)];
        }
        FB(uS, i, e, c) = suS;
        FB(uN, i, e, c) = suN;
        FB(gyS, i, e, c) = sgS;
        FB(gyN, i, e, c) = sgN;
      }
    }
  }
#define BR0X(eL, eR, q, c)                                                        \
  br0_avg(FB(gxE, q, eL, c), FB(gxW, q, eR, c), FB(uE, q, eL, c), FB(uW, q, eR, c), \
          br0_tau(eps[eL], eps[eR], s->dx2[(eL) % nx], s->dx2[(eR) % nx], p))
#define BR0Y(eB, eT, q, c)                                                        \
  br0_avg(FB(gyN, q, eB, c), FB(gyS, q, eT, c), FB(uN, q, eB, c), FB(uS, q, eT, c), \
          br0_tau(eps[eB], eps[eT], s->dy2[(eB) / nx], s->dy2[(eT) / nx], p))
#pragma omp parallel for schedule(static)
  for (int jy = 0; jy < ny; ++jy)
    for (int jx = 0; jx < nx - 1; ++jx) {
      int eL = jy * nx + jx, eR = eL + 1;
      for (int q = 0; q < np; ++q)
        for (int c = 0; c < 4; ++c) {
          double gh = BR0X(eL, eR, q, c);
          FB(ghE, q, eL, c) = gh;
          FB(ghW, q, eR, c) = gh;
        }
    }
  for (int jy = 0; jy < ny; ++jy) {
    int eL = jy * nx, eR = jy * nx + nx - 1;
    for (int q = 0; q < np; ++q)
      for (int c = 0; c < 4; ++c) {
        if (s->bc[0].kind == ORC_BC_PERIODIC) {
          double gh = BR0X(eR, eL, q, c);
          FB(ghE, q, eR, c) = gh;
          FB(ghW, q, eL, c) = gh;
        } else {
          FB(ghW, q, eL, c) = FB(gxW, q, eL, c);
          FB(ghE, q, eR, c) = FB(gxE, q, eR, c);
        }
      }
  }
#pragma omp parallel for schedule(static)
  for (int jy = 0; jy < ny - 1; ++jy)
    for (int jx = 0; jx < nx; ++jx) {
      int eB = jy * nx + jx, eT = eB + nx;
      for (int q = 0; q < np; ++q)
        for (int c = 0; c < 4; ++c) {
          double gh = BR0Y(eB, eT, q, c);
          FB(ghN, q, eB, c) = gh;
          FB(ghS, q, eT, c) = gh;
        }
    }
  for (int jx = 0; jx < nx; ++jx) {
    int eB = jx, eT = (ny - 1) * nx + jx;
    for (int q = 0; q < np; ++q)
      for (int c = 0; c < 4; ++c) {
        if (s->bc[2].kind == ORC_BC_PERIODIC) {
          double gh = BR0Y(eT, eB, q, c);
          FB(ghN, q, eT, c) = gh;
          FB(ghS, q, eB, c) = gh;
        } else {
          FB(ghS, q, eB, c) = FB(gyS, q, eB, c);
          FB(ghN, q, eT, c) = FB(gyN, q, eT, c);
        }
      }
  }
#undef BR0X
#undef BR0Y
#pragma omp parallel for schedule(static)
  for (int e = 0; e < nel; ++e) {
    int jx = e % nx, jy = e / nx;
    double Jx = s->Jx[jx], Jy = s->Jy[jy];
    for (int c = 0; c < 4; ++c) {
      const double* GX = gx + c * cs;
      const double* GY = gy + c * cs;
      double* DU = du + c * cs;
      for (int j = 0; j < np; ++j) {
        double gLf = 0, gRf = 0;
        for (int i = 0; i < np; ++i) {
          gLf += lL[i] * GX[IX3(i, j, e, np)];
          gRf += lR[i] * GX[IX3(i, j, e, np)];
        }
        for (int i = 0; i < np; ++i) {
          double vol = 0;
          for (int k = 0; k < np; ++k) vol += D[i + np * k] * GX[IX3(k, j, e, np)];
          double corr = (FB(ghW, j, e, c) - gLf) * gLx[i] + (FB(ghE, j, e, c) - gRf) * gRx[i];
          DU[IX3(i, j, e, np)] += (vol + corr) / Jx;
        }
      }
      for (int i = 0; i < np; ++i) {
        double gSf = 0, gNf = 0;
        for (int j = 0; j < np; ++j) {
          gSf += lL[j] * GY[IX3(i, j, e, np)];
          gNf += lR[j] * GY[IX3(i, j, e, np)];
        }
        for (int j = 0; j < np; ++j) {
          double vol = 0;
          for (int k = 0; k < np; ++k) vol += D[j + np * k] * GY[IX3(i, k, e, np)];
          double corr = (FB(ghS, i, e, c) - gSf) * gLx[j] + (FB(ghN, i, e, c) - gNf) * gRx[j];
          DU[IX3(i, j, e, np)] += (vol + corr) / Jy;
        }
      }
    }
  }
#undef FB
}

/* apply_dissipation_local_DD_2d!, src/capturing/PerssonAV2D.jl:135-194 */
static void local_dd_2d(orc_solver* s, double* du, const double* uw) {
  int np = s->np, nel = s->nel, nx = s->nx;
  size_t cs = (size_t)np * np * nel;
  const double* D = s->ops.D;
  double* eps = s->eps_e;
  element_viscosities_2d(s, uw, s->sigma, eps);
#pragma omp parallel for schedule(static)
  for (int e = 0; e < nel; ++e) {
    double ee = eps[e];
    if (ee <= 0.0) continue;
    int jx = e % nx, jy = e / nx;
    double Jx = s->Jx[jx], Jy = s->Jy[jy];
    double sx = ee / (Jx * Jx), sy = ee / (Jy * Jy);
    double v[ORC_MAXNP];
    for (int c = 0; c < 4; ++c) {
      const double* U = uw + c * cs;
      double* DU = du + c * cs;
      for (int j = 0; j < np; ++j) {
        for (int i = 0; i < np; ++i) {
          double a = 0;
          for (int k = 0; k < np; ++k) a += D[i + np * k] * U[IX3(k, j, e, np)];
          v[i] = a;
        }
        for (int i = 0; i < np; ++i) {
          double a = 0;
          for (int k = 0; k < np; ++k) a += D[i + np * k] * v[k];
          DU[IX3(i, j, e, np)] += sx * a;
        }
      }
      for (int i = 0; i < np; ++i) {
        for (int j = 0; j < np; ++j) {
          double a = 0;
          for (int k = 0; k < np; ++k) a += D[j + np * k] * U[IX3(i, k, e, np)];
          v[j] = a;
        }
        for (int j = 0; j < np; ++j) {
          double a = 0;
          for (int k = 0; k < np; ++k) a += D[j + np * k] * v[k];
          DU[IX3(i, j, e, np)] += sy * a;
        }
      }
    }
  }
}

/* residual! 2D, src/fr/Residual2D.jl:131-416 */
static void residual_2d(orc_solver* s, double* du) {
  int np = s->np, nel = s->nel, nx = s->nx, ny = s->ny;
  size_t n = orc_ndof(s), cs = (size_t)np * np * nel;
  double* uw = s->u_work;
  memcpy(uw, s->u, n * sizeof(double));
  memset(du, 0, n * sizeof(double));
  const int has_solid = s->solid != NULL;
  const double* xi = s->ops.xi;
  orc_bc wall;
  memset(&wall, 0, sizeof(wall));
  wall.kind = ORC_BC_REFLECTING;
  double *trW = s->trW, *trE = s->trE, *trS = s->trS, *trN = s->trN;
  double *fhW = s->fhW, *fhE = s->fhE, *fhS = s->fhS, *fhN = s->fhN;

#pragma omp parallel for schedule(static)
  for (int e = 0; e < nel; ++e) {
    if (has_solid && is_solid(s, e)) continue;
    face_traces_2d(s, uw, e);
  }
  /* interior vertical faces */
#pragma omp parallel for schedule(static)
  for (int iface = 0; iface < ny * (nx - 1); ++iface) {
    int jy = iface / (nx - 1), jx = iface % (nx - 1);
    int eL = jy * nx + jx, eR = eL + 1;
    int sL = has_solid && is_solid(s, eL), sR = has_solid && is_solid(s, eR);
    if (sL && sR) continue;
    double um[4], up[4], fh[4];
    for (int q = 0; q < np; ++q) {
      double nnx = s->nx_E[IX2(q, eL, np)], nny = s->ny_E[IX2(q, eL, np)];
      double sJ = s->sJ_E[IX2(q, eL, np)];
      if (sL && !sR) {
        for (int c = 0; c < 4; ++c) um[c] = TR(trW, q, c, eR);
        double x, y;
        physical_xy(s, eR, -1.0, xi[q], &x, &y);
        boundary_fhat(s, fhW, q, eR, &wall, um, s->nx_W[IX2(q, eR, np)],
                      s->ny_W[IX2(q, eR, np)], s->sJ_W[IX2(q, eR, np)], x, y, 1);
      } else if (sR && !sL) {
        for (int c = 0; c < 4; ++c) um[c] = TR(trE, q, c, eL);
        double x, y;
        physical_xy(s, eL, 1.0, xi[q], &x, &y);
        boundary_fhat(s, fhE, q, eL, &wall, um, nnx, nny, sJ, x, y, 0);
      } else {
        for (int c = 0; c < 4; ++c) {
          um[c] = TR(trE, q, c, eL);
          up[c] = TR(trW, q, c, eR);
        }
        iflux2(s, um, up, nnx, nny, fh);
        for (int c = 0; c < 4; ++c) {
          double val = fh[c] * sJ;
          TR(fhE, q, c, eL) = val;
          TR(fhW, q, c, eR) = val;
        }
      }
    }
  }
  /* domain left/right */
  for (int jy = 0; jy < ny; ++jy) {
    int eL = jy * nx, eR = jy * nx + nx - 1;
    double um[4], up[4], fh[4];
    for (int q = 0; q < np; ++q) {
      if (s->bc[0].kind == ORC_BC_PERIODIC) {
        if (!(has_solid && (is_solid(s, eL) || is_solid(s, eR)))) {
          for (int c = 0; c < 4; ++c) {
            um[c] = TR(trE, q, c, eR);
            up[c] = TR(trW, q, c, eL);
          }
          double nnx = s->nx_E[IX2(q, eR, np)], nny = s->ny_E[IX2(q, eR, np)];
          double sJ = s->sJ_E[IX2(q, eR, np)];
          iflux2(s, um, up, nnx, nny, fh);
          for (int c = 0; c < 4; ++c) {
            double val = fh[c] * sJ;
            TR(fhE, q, c, eR) = val;
            TR(fhW, q, c, eL) = val;
          }
        }
      } else {
        if (!(has_solid && is_solid(s, eL))) {
          for (int c = 0; c < 4; ++c) um[c] = TR(trW, q, c, eL);
          double x, y;
          physical_xy(s, eL, -1.0, xi[q], &x, &y);
          boundary_fhat(s, fhW, q, eL, &s->bc[0], um, s->nx_W[IX2(q, eL, np)],
                        s->ny_W[IX2(q, eL, np)], s->sJ_W[IX2(q, eL, np)], x, y, 1);
        }
        if (!(has_solid && is_solid(s, eR))) {
          for (int c = 0; c < 4; ++c) up[c] = TR(trE, q, c, eR);
          double x, y;
          physical_xy(s, eR, 1.0, xi[q], &x, &y);
          boundary_fhat(s, fhE, q, eR, &s->bc[1], up, s->nx_E[IX2(q, eR, np)],
                        s->ny_E[IX2(q, eR, np)], s->sJ_E[IX2(q, eR, np)], x, y, 0);
        }
      }
    }
  }
  /* interior horizontal faces */
#pragma omp parallel for schedule(static)
  for (int iface = 0; iface < (ny - 1) * nx; ++iface) {
    int jy = iface / nx, jx = iface % nx;
    int eB = jy * nx + jx, eT = eB + nx;
    int sB = has_solid && is_solid(s, eB), sT = has_solid && is_solid(s, eT);
    if (sB && sT) continue;
    double um[4], up[4], fh[4];
    for (int q = 0; q < np; ++q) {
      double nnx = s->nx_N[IX2(q, eB, np)], nny = s->ny_N[IX2(q, eB, np)];
      double sJ = s->sJ_N[IX2(q, eB, np)];
      if (sB && !sT) {
        for (int c = 0; c < 4; ++c) um[c] = TR(trS, q, c, eT);
        double x, y;
        physical_xy(s, eT, xi[q], -1.0, &x, &y);
        boundary_fhat(s, fhS, q, eT, &wall, um, s->nx_S[IX2(q, eT, np)],
                      s->ny_S[IX2(q, eT, np)], s->sJ_S[IX2(q, eT, np)], x, y, 1);
      } else if (sT && !sB) {
        for (int c = 0; c < 4; ++c) um[c] = TR(trN, q, c, eB);
        double x, y;
        physical_xy(s, eB, xi[q], 1.0, &x, &y);
        boundary_fhat(s, fhN, q, eB, &wall, um, nnx, nny, sJ, x, y, 0);
      } else {
        for (int c = 0; c < 4; ++c) {
          um[c] = TR(trN, q, c, eB);
          up[c] = TR(trS, q, c, eT);
        }
        iflux2(s, um, up, nnx, nny, fh);
        for (int c = 0; c < 4; ++c) {
          double val = fh[c] * sJ;
          TR(fhN, q, c, eB) = val;
          TR(fhS, q, c, eT) = val;
        }
      }
    }
  }
  /* domain bottom/top */
  for (int jx = 0; jx < nx; ++jx) {
    int eB = jx, eT = (ny - 1) * nx + jx;
    double um[4], up[4], fh[4];
    for (int q = 0; q < np; ++q) {
      if (s->bc[2].kind == ORC_BC_PERIODIC) {
        if (!(has_solid && (is_solid(s, eB) || is_solid(s, eT)))) {
          for (int c = 0; c < 4; ++c) {
            um[c] = TR(trN, q, c, eT);
            up[c] = TR(trS, q, c, eB);
          }
          double nnx = s->nx_N[IX2(q, eT, np)], nny = s->ny_N[IX2(q, eT, np)];
          double sJ = s->sJ_N[IX2(q, eT, np)];
          iflux2(s, um, up, nnx, nny, fh);
          for (int c = 0; c < 4; ++c) {
            double val = fh[c] * sJ;
            TR(fhN, q, c, eT) = val;
            TR(fhS, q, c, eB) = val;
          }
        }
      } else {
        if (!(has_solid && is_solid(s, eB))) {
          for (int c = 0; c < 4; ++c) um[c] = TR(trS, q, c, eB);
          double x, y;
          physical_xy(s, eB, xi[q], -1.0, &x, &y);
          boundary_fhat(s, fhS, q, eB, &s->bc[2], um, s->nx_S[IX2(q, eB, np)],
                        s->ny_S[IX2(q, eB, np)], s->sJ_S[IX2(q, eB, np)], x, y, 1);
        }
        if (!(has_solid && is_solid(s, eT))) {
          for (int c = 0; c < 4; ++c) up[c] = TR(trN, q, c, eT);
          double x, y;
          physical_xy(s, eT, xi[q], 1.0, &x, &y);
          boundary_fhat(s, fhN, q, eT, &s->bc[3], up, s->nx_N[IX2(q, eT, np)],
                        s->ny_N[IX2(q, eT, np)], s->sJ_N[IX2(q, eT, np)], x, y, 0);
        }
      }
    }
  }
  /* volume residual */
  const double *D = s->ops.D, *lL = s->ops.lL, *lR = s->ops.lR;
  const double *gL = s->ops.gLxi, *gR = s->ops.gRxi;
#pragma omp parallel for schedule(static)
  for (int e = 0; e < nel; ++e) {
    if (has_solid && is_solid(s, e)) continue;
    double Ft[ORC_MAXNP][ORC_MAXNP][4], Gt[ORC_MAXNP][ORC_MAXNP][4];
    for (int j = 0; j < np; ++j)
      for (int i = 0; i < np; ++i) {
        size_t id = IX3(i, j, e, np);
        double U[4] = {uw[id], uw[id + cs], uw[id + 2 * cs], uw[id + 3 * cs]};
        double Fx[4], Gy[4];
        pflux_x(s->gamma, U, Fx);
        pflux_y(s->gamma, U, Gy);
        double xxi = s->x_xi[id], xeta = s->x_eta[id], yxi = s->y_xi[id], yeta = s->y_eta[id];
        for (int c = 0; c < 4; ++c) {
          Ft[i][j][c] = yeta * Fx[c] - xeta * Gy[c];
          Gt[i][j][c] = -yxi * Fx[c] + xxi * Gy[c];
        }
      }
    for (int j = 0; j < np; ++j)
      for (int c = 0; c < 4; ++c) {
        double fLs = 0, fRs = 0;
        for (int i = 0; i < np; ++i) {
          fLs += lL[i] * Ft[i][j][c];
          fRs += lR[i] * Ft[i][j][c];
        }
        for (int i = 0; i < np; ++i) {
          double vol = 0;
          for (int k = 0; k < np; ++k) vol += D[i + np * k] * Ft[k][j][c];
          double corr = (TR(fhW, j, c, e) - fLs) * gL[i] + (TR(fhE, j, c, e) - fRs) * gR[i];
          double Je = s->J2[IX3(i, j, e, np)];
          du[c * cs + IX3(i, j, e, np)] -= (vol + corr) / Je;
        }
      }
    for (int i = 0; i < np; ++i)
      for (int c = 0; c < 4; ++c) {
        double gSs = 0, gNs = 0;
        for (int j = 0; j < np; ++j) {
          gSs += lL[j] * Gt[i][j][c];
          gNs += lR[j] * Gt[i][j][c];
        }
        for (int j = 0; j < np; ++j) {
          double vol = 0;
          for (int k = 0; k < np; ++k) vol += D[j + np * k] * Gt[i][k][c];
          double corr = (TR(fhS, i, c, e) - gSs) * gL[j] + (TR(fhN, i, c, e) - gNs) * gR[j];
          double Je = s->J2[IX3(i, j, e, np)];
          du[c * cs + IX3(i, j, e, np)] -= (vol + corr) / Je;
        }
      }
  }
  if (s->method == ORC_METHOD_PERSSON) {
    sense_2d(s, uw, s->sigma);
    if (has_solid)
      for (int e = 0; e < nel; ++e)
        if (is_solid(s, e)) s->sigma[e] = 0.0;
    if (s->av_form == ORC_AV_BR0)
      br0_2d(s, du, uw);
    else
      local_dd_2d(s, du, uw);
  } else {
    for (int e = 0; e < nel; ++e) s->sigma[e] = 0.0;
  }
  if (has_solid)
    for (int e = 0; e < nel; ++e)
      if (is_solid(s, e))
        for (int c = 0; c < 4; ++c)
          for (int k = 0; k < np * np; ++k) du[c * cs + (size_t)np * np * e + k] = 0.0;
}
#undef TR

void orc_residual(orc_solver* s, double* du) {
  if (s->dim == 1)
    residual_1d(s, s->du);
  else
    residual_2d(s, s->du);
  if (du) memcpy(du, s->du, orc_ndof(s) * sizeof(double));
}

void orc_sense(orc_solver* s, double* sigma) {
  memcpy(s->u_work, s->u, orc_ndof(s) * sizeof(double));
  if (s->dim == 1)
    sense_1d(s, s->u_work, sigma);
  else
    sense_2d(s, s->u_work, sigma);
}

/* ----------------------------------------------------------- time stepping */

/* has_nonfinite, src/fr/Residual.jl:219-226 */
int orc_has_nonfinite(const double* a, size_t n) {
  int bad = 0;
#pragma omp parallel for reduction(| : bad) schedule(static)
  for (long i = 0; i < (long)n; ++i)
    if (!isfinite(a[i])) bad = 1;
  return bad;
}

/* compute_dt, src/time/SSP_RK3.jl:8-24 (1D) and :126-133 (2D) with
   max_wave_speed Euler.jl:115-124 / Euler2D.jl:92-105 */
double orc_compute_dt(orc_solver* s, double cfl) {
  int np = s->np, nel = s->nel, p = s->ops.p;
  double m = 0.0;
  if (s->dim == 1) {
    size_t cs = (size_t)np * nel;
    for (int e = 0; e < nel; ++e)
      for (int j = 0; j < np; ++j) {
        double U[3] = {s->u[(size_t)np * e + j], s->u[cs + (size_t)np * e + j],
                       s->u[2 * cs + (size_t)np * e + j]};
        m = jmax(m, fabs(velocity1(U)) + sound1(s->gamma, U));
      }
    double lam = jmax(jmax(m, EPS), EPS);
    double dt = INFINITY;
    for (int e = 0; e < nel; ++e)
      dt = jmin(dt, cfl * s->dx[e] / ((double)(2 * p + 1) * lam));
    return dt;
  }
  size_t cs = (size_t)np * np * nel;
#pragma omp parallel for reduction(max : m) schedule(static)
  for (long id = 0; id < (long)cs; ++id) {
    double U[4] = {s->u[id], s->u[id + cs], s->u[id + 2 * cs], s->u[id + 3 * cs]};
    double r = jmax(U[0], EPS);
    double u = U[1] / r, v = U[2] / r;
    double c = sound2(s->gamma, U);
    double a = fabs(u) + c, b = fabs(v) + c;
    double mm = a > b ? a : b;
    if (mm > m) m = mm;
    if (mm != mm) m = mm; /* NaN poisons the maximum as in Julia */
  }
  double lam = jmax(jmax(m, EPS), EPS);
  double hmin = INFINITY;
  for (int e = 0; e < nel; ++e) hmin = jmin(hmin, s->h_char[e]);
  return cfl * hmin / ((double)(2 * p + 1) * lam);
}

/* ssp_rk3_step! (src/time/SSP_RK3.jl:29-65, :135-164) and ssp_rk2_step!
   (src/time/SSP_RK2.jl:14-68) */
int orc_step(orc_solver* s, double dt) {
  size_t n = orc_ndof(s);
  double *u = s->u, *du = s->du, *u0 = s->u0, *u1 = s->u1, *u2 = s->u2;
  memcpy(u0, u, n * sizeof(double));
  double t0 = s->t;
  orc_residual(s, NULL);
  if (orc_has_nonfinite(du, n)) return ORC_DIVERGED;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)n; ++i) u[i] = u0[i] + dt * du[i];
  s->t = t0 + dt;
  orc_residual(s, NULL);
  if (orc_has_nonfinite(du, n)) return ORC_DIVERGED;
  if (s->time_scheme == ORC_TIME_SSP_RK2) {
    const double h = 1.0 / 2.0;
    memcpy(u1, u, n * sizeof(double));
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; ++i) u[i] = h * u0[i] + h * u1[i] + h * dt * du[i];
    s->t = t0 + dt;
  } else {
    const double a = 3.0 / 4.0, b = 1.0 / 4.0;
    memcpy(u1, u, n * sizeof(double));
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; ++i) u[i] = a * u0[i] + b * u1[i] + b * dt * du[i];
    s->t = t0 + dt / 2.0;
    orc_residual(s, NULL);
    if (orc_has_nonfinite(du, n)) return ORC_DIVERGED;
    const double c13 = 1.0 / 3.0, c23 = 2.0 / 3.0;
    memcpy(u2, u, n * sizeof(double));
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; ++i) u[i] = c13 * u0[i] + c23 * u2[i] + c23 * dt * du[i];
    s->t = t0 + dt;
  }
  if (orc_has_nonfinite(u, n)) return ORC_DIVERGED;
  return ORC_OK; /* post_step! default is a no-op (Interfaces.jl:90-92) */
}

/* ssp_rk3! / ssp_rk2! drivers, src/time/SSP_RK3.jl:75-118 / SSP_RK2.jl:70-132 */
int orc_integrate(orc_solver* s, double t_final, double cfl, double fixed_dt,
                  int64_t max_steps, int64_t* n_steps_out) {
  int64_t n_steps = 0;
  int status = ORC_OK;
  while (s->t < t_final - 10 * EPS) {
    double step_dt = fixed_dt > 0 ? fixed_dt : orc_compute_dt(s, cfl);
    if (s->t + step_dt > t_final) step_dt = t_final - s->t;
    status = orc_step(s, step_dt);
    n_steps += 1;
    if (status != ORC_OK) break;
    if (n_steps >= max_steps) {
      status = ORC_MAX_STEPS;
      break;
    }
  }
  if (n_steps_out) *n_steps_out = n_steps;
  return status;
}

/* ------------------------------------------------------------ diagnostics */

/* discrete_mass, src/solvestate/SolutionState.jl:80-90 / SolutionState2D.jl:85-97 */
double orc_discrete_mass(const orc_solver* s, int c) {
  int np = s->np, nel = s->nel;
  double m = 0.0;
  if (s->dim == 1) {
    size_t cs = (size_t)np * nel;
    for (int e = 0; e < nel; ++e)
      for (int j = 0; j < np; ++j) m += s->ops.w[j] * s->J1[e] * s->u[c * cs + (size_t)np * e + j];
    return m;
  }
  size_t cs = (size_t)np * np * nel;
  for (int e = 0; e < nel; ++e)
    for (int j = 0; j < np; ++j)
      for (int i = 0; i < np; ++i)
        m += s->ops.w[i] * s->ops.w[j] * fabs(s->J2[IX3(i, j, e, np)]) *
             s->u[c * cs + IX3(i, j, e, np)];
  return m;
}

/* positivity_ok, src/equations/Euler.jl:62-77 / Euler2D.jl:153-163 */
int orc_positivity_ok(const orc_solver* s) {
  int np = s->np, nel = s->nel;
  if (s->dim == 1) {
    size_t cs = (size_t)np * nel;
    for (int e = 0; e < nel; ++e)
      for (int j = 0; j < np; ++j) {
        size_t id = (size_t)np * e + j;
        double U[3] = {s->u[id], s->u[id + cs], s->u[id + 2 * cs]};
        double p = pressure1(s->gamma, U);
        if (!(U[0] > 0.0 && p > 0.0 && isfinite(U[0]) && isfinite(p))) return 0;
      }
    return 1;
  }
  size_t cs = (size_t)np * np * nel;
  for (size_t id = 0; id < cs; ++id) {
    double U[4] = {s->u[id], s->u[id + cs], s->u[id + 2 * cs], s->u[id + 3 * cs]};
    double p = pressure2(s->gamma, U);
    if (!(U[0] > 0.0 && p > 0.0 && isfinite(U[0]) && isfinite(p))) return 0;
  }
  return 1;
}

/* solution_extrema, src/verification/Metrics.jl:64-73 */
void orc_solution_extrema(const orc_solver* s, int c, double* umin, double* umax) {
  size_t per = (size_t)s->nel * (s->dim == 1 ? s->np : s->np * s->np);
  double lo = INFINITY, hi = -INFINITY;
  for (size_t i = 0; i < per; ++i) {
    double v = s->u[c * per + i];
    lo = jmin(lo, v);
    hi = jmax(hi, v);
  }
  *umin = lo;
  *umax = hi;
}

/* ------------------------------------------------------------------- ICs */

/* primitives_to_conserved, Euler.jl:45-51 and Euler2D.jl:21-25 */
static void prim2cons1(double g, double r, double u, double p, double* U) {
  double E = p / (g - 1.0) + 0.5 * r * u * u;
  U[0] = r;
  U[1] = r * u;
  U[2] = E;
}
static void prim2cons2(double g, double r, double u, double v, double p, double* U) {
  double E = p / (g - 1.0) + 0.5 * r * (u * u + v * v);
  U[0] = r;
  U[1] = r * u;
  U[2] = r * v;
  U[3] = E;
}

static void set_ic_1d(orc_solver* s, void (*f)(const orc_solver*, double, const void*, double*),
                      const void* ctx) {
  int np = s->np, nel = s->nel;
  size_t cs = (size_t)np * nel;
  for (int e = 0; e < nel; ++e) {
    double mid = (s->xv[e] + s->xv[e + 1]) / 2.0;
    for (int j = 0; j < np; ++j) {
      double x = mid + s->J1[e] * s->ops.xi[j];
      double U[3];
      f(s, x, ctx, U);
      for (int c = 0; c < 3; ++c) s->u[c * cs + (size_t)np * e + j] = U[c];
    }
  }
  s->t = 0.0;
}

/* sod_ic, src/verification/Cases.jl:940-946 */
static void f_sod(const orc_solver* s, double x, const void* ctx, double* U) {
  (void)ctx;
  if (x < 0.5)
    prim2cons1(s->gamma, 1.0, 0.0, 1.0, U);
  else
    prim2cons1(s->gamma, 0.125, 0.0, 0.1, U);
}
void orc_ic_sod(orc_solver* s) { set_ic_1d(s, f_sod, NULL); }

/* shu_osher_ic, src/verification/Cases.jl:930-938 */
static void f_shu(const orc_solver* s, double x, const void* ctx, double* U) {
  (void)ctx;
  if (x < 1.0) {
    prim2cons1(s->gamma, 3.857143, 2.629369, 10.33333, U);
  } else {
    double xc = x - 5.0;
    double r = 1.0 + 0.2 * sin(5.0 * xc);
    prim2cons1(s->gamma, r, 0.0, 1.0, U);
  }
}
void orc_ic_shu_osher(orc_solver* s) { set_ic_1d(s, f_shu, NULL); }

/* euler_density_wave_conserved, src/verification/Cases.jl:404-414 */
static void f_dw(const orc_solver* s, double x, const void* ctx, double* U) {
  double t = *(const double*)ctx;
  double r = 1.0 + 0.2 * sin(TWO_PI * (x - 1.0 * t));
  prim2cons1(s->gamma, r, 1.0, 1.0, U);
}
void orc_ic_density_wave_1d(orc_solver* s, double t) { set_ic_1d(s, f_dw, &t); }

struct two_state {
  double x0;
  const double *L, *R;
};
static void f_two(const orc_solver* s, double x, const void* ctx, double* U) {
  const struct two_state* ts = (const struct two_state*)ctx;
  const double* P = x < ts->x0 ? ts->L : ts->R;
  prim2cons1(s->gamma, P[0], P[1], P[2], U);
}
void orc_ic_two_state_1d(orc_solver* s, double x0, const double* primL, const double* primR) {
  struct two_state ts = {x0, primL, primR};
  set_ic_1d(s, f_two, &ts);
}

static void set_ic_2d(orc_solver* s,
                      void (*f)(const orc_solver*, double, double, const void*, double*),
                      const void* ctx) {
  int np = s->np, nel = s->nel;
  size_t cs = (size_t)np * np * nel;
  for (int e = 0; e < nel; ++e)
    for (int jy = 0; jy < np; ++jy)
      for (int jx = 0; jx < np; ++jx) {
        double x, y, U[4];
        physical_xy(s, e, s->ops.xi[jx], s->ops.xi[jy], &x, &y);
        f(s, x, y, ctx, U);
        for (int c = 0; c < 4; ++c) s->u[c * cs + IX3(jx, jy, e, np)] = U[c];
      }
  s->t = 0.0;
}

/* isentropic_vortex_primitives, src/verification/Cases2D_Riemann.jl:163-186
   (defaults γ=1.4, β=5, center (5,5), u∞=v∞=1) */
static void vortex_prims(double x, double y, double t, double* P) {
  const double g = 1.4, beta = 5.0, x0 = 5.0, y0 = 5.0, uinf = 1.0, vinf = 1.0;
  double xd = x - x0 - uinf * t;
  double yd = y - y0 - vinf * t;
  double r2 = xd * xd + yd * yd;
  double expf_ = exp(0.5 * (1.0 - r2));
  double b2pi = beta / TWO_PI;
  double du = -b2pi * expf_ * yd;
  double dv = b2pi * expf_ * xd;
  double pi2 = PI_F64 * PI_F64;
  double T = 1.0 - (g - 1.0) * (beta * beta) / (8.0 * g * pi2) * exp(1.0 - r2);
  T = jmax(T, 1e-14);
  double r = pow(T, 1.0 / (g - 1.0));
  double p = pow(r, g);
  P[0] = r;
  P[1] = uinf + du;
  P[2] = vinf + dv;
  P[3] = p;
}
static void f_vortex(const orc_solver* s, double x, double y, const void* ctx, double* U) {
  double t = *(const double*)ctx;
  double P[4];
  vortex_prims(x, y, t, P);
  prim2cons2(s->gamma, P[0], P[1], P[2], P[3], U);
}
void orc_ic_vortex_2d(orc_solver* s, double t) { set_ic_2d(s, f_vortex, &t); }

/* run_euler2d_smooth_order IC, src/verification/Cases2D_Smooth.jl:124-135 */
static void f_smooth(const orc_solver* s, double x, double y, const void* ctx, double* U) {
  double t = ctx ? *(const double*)ctx : 0.0;
  double r = 1.0 + 0.2 * sin(TWO_PI * (x - t)) * sin(TWO_PI * (y - t));
  prim2cons2(s->gamma, r, 1.0, 1.0, 1.0, U);
}
void orc_ic_smooth_2d(orc_solver* s) { set_ic_2d(s, f_smooth, NULL); }

struct quad_states {
  double x0, y0;
  const double *ne, *nw, *sw, *se;
};
/* riemann2d_ic, src/verification/Cases2D_Riemann.jl:33-51 */
static void f_quad(const orc_solver* s, double x, double y, const void* ctx, double* U) {
  const struct quad_states* q = (const struct quad_states*)ctx;
  const double* P;
  if (x >= q->x0 && y >= q->y0)
    P = q->ne;
  else if (x < q->x0 && y >= q->y0)
    P = q->nw;
  else if (x < q->x0 && y < q->y0)
    P = q->sw;
  else
    P = q->se;
  prim2cons2(s->gamma, P[0], P[1], P[2], P[3], U);
}
void orc_ic_four_quadrant_2d(orc_solver* s, double x0, double y0, const double* ne,
                             const double* nw, const double* sw, const double* se) {
  struct quad_states q = {x0, y0, ne, nw, sw, se};
  set_ic_2d(s, f_quad, &q);
}

static void f_uniform2(const orc_solver* s, double x, double y, const void* ctx, double* U) {
  (void)x;
  (void)y;
  const double* P = (const double*)ctx;
  prim2cons2(s->gamma, P[0], P[1], P[2], P[3], U);
}
static void f_uniform1(const orc_solver* s, double x, const void* ctx, double* U) {
  (void)x;
  const double* P = (const double*)ctx;
  prim2cons1(s->gamma, P[0], P[1], P[2], U);
}
void orc_ic_uniform(orc_solver* s, const double* prim) {
  if (s->dim == 1)
    set_ic_1d(s, f_uniform1, prim);
  else
    set_ic_2d(s, f_uniform2, prim);
}

/* l2_error (density), src/solvestate/SolutionState2D.jl:98-111 */
static double l2_2d(const orc_solver* s,
                    void (*f)(const orc_solver*, double, double, const void*, double*),
                    const void* ctx) {
  int np = s->np, nel = s->nel;
  double acc = 0.0;
  for (int e = 0; e < nel; ++e)
    for (int j = 0; j < np; ++j)
      for (int i = 0; i < np; ++i) {
        double x, y, U[4];
        physical_xy(s, e, s->ops.xi[i], s->ops.xi[j], &x, &y);
        f(s, x, y, ctx, U);
        double err = s->u[IX3(i, j, e, np)] - U[0];
        acc += s->ops.w[i] * s->ops.w[j] * fabs(s->J2[IX3(i, j, e, np)]) * err * err;
      }
  return sqrt(acc);
}
double orc_l2_error_vortex(const orc_solver* s, double t) { return l2_2d(s, f_vortex, &t); }
double orc_l2_error_smooth_2d(const orc_solver* s, double t) { return l2_2d(s, f_smooth, &t); }

/* l2_error (density), src/solvestate/SolutionState.jl:93-107 */
double orc_l2_error_density_wave_1d(const orc_solver* s, double t) {
  int np = s->np, nel = s->nel;
  double acc = 0.0;
  for (int e = 0; e < nel; ++e) {
    double mid = (s->xv[e] + s->xv[e + 1]) / 2.0;
    for (int j = 0; j < np; ++j) {
      double x = mid + s->J1[e] * s->ops.xi[j];
      double U[3];
      f_dw(s, x, &t, U);
      double err = s->u[(size_t)np * e + j] - U[0];
      acc += s->ops.w[j] * s->J1[e] * err * err;
    }
  }
  return sqrt(acc);
}

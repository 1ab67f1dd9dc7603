// Host-side set-up of the reference-element tables.
//
// build_operators (src/fr/Operators.jl:85-104) is restated here for callers
// that do not pass their own FROperators tables.  Gauss-Legendre nodes come
// from Newton iteration on P_n (the reference uses the Golub-Welsch
// eigen-solve; both converge to the same nodes to rounding), Gauss-Lobatto
// nodes from Newton on P'_p as in Operators.jl:10-59.  D, l_L/l_R, g_DG and
// the Legendre Vandermonde follow Points.jl:65-104 and Correction.jl:57-101.
#include <cmath>
#include <cstring>

#include "frg_internal.h"

namespace frg {

namespace {

double legendre_P(int k, double x) {
  if (k == 0) return 1.0;
  if (k == 1) return x;
  double pm2 = 1.0, pm1 = x, pk = x;
  for (int m = 2; m <= k; ++m) {
    pk = ((double)(2 * m - 1) * x * pm1 - (double)(m - 1) * pm2) / (double)m;
    pm2 = pm1;
    pm1 = pk;
  }
  return pk;
}

// P_k'(x) with the closed endpoint values (Correction.jl:32-45)
double legendre_dP(int k, double x) {
  if (k == 0) return 0.0;
  const double e = 2.220446049250313e-16;
  if (x >= 1.0 - 1000 * e) return (double)(k * (k + 1)) / 2.0;
  if (x <= -1.0 + 1000 * e) return ((k % 2) ? 1.0 : -1.0) * (double)(k * (k + 1)) / 2.0;
  return ((double)k * legendre_P(k - 1, x) - (double)k * x * legendre_P(k, x)) / (1.0 - x * x);
}

void gauss_legendre_newton(int n, double* xi, double* w) {
  if (n == 1) {
    xi[0] = 0.0;
    w[0] = 2.0;
    return;
  }
  const double pi = 3.141592653589793;
  for (int i = 0; i < n; ++i) {
    // roots in descending order from the classical cosine guess
    double x = std::cos(pi * (i + 0.75) / (n + 0.5));
    for (int it = 0; it < 100; ++it) {
      const double p = legendre_P(n, x);
      const double dp = (double)n * (legendre_P(n - 1, x) - x * p) / (1.0 - x * x);
      const double dx = p / dp;
      x -= dx;
      if (std::fabs(dx) <= 1e-17) break;
    }
    xi[n - 1 - i] = x;
  }
  double sw = 0.0;
  for (int i = 0; i < n; ++i) {
    const double x = xi[i];
    const double dp = (double)n * (legendre_P(n - 1, x) - x * legendre_P(n, x)) / (1.0 - x * x);
    w[i] = 2.0 / ((1.0 - x * x) * dp * dp);
    sw += w[i];
  }
  for (int i = 0; i < n; ++i) w[i] *= 2.0 / sw;
}

void gauss_lobatto_newton(int n, double* xi, double* w) {
  if (n == 1) {
    xi[0] = 0.0;
    w[0] = 2.0;
    return;
  }
  const int p = n - 1;
  const double e = 2.220446049250313e-16;
  xi[0] = -1.0;
  xi[n - 1] = 1.0;
  for (int j = 2; j <= n - 1; ++j) {
    double x = std::cos(3.141592653589793 * (double)(j - 1) / (double)p);
    for (int it = 0; it < 80; ++it) {
      const double Pp = legendre_P(p, x), dPp = legendre_dP(p, x);
      const double omx2 = 1.0 - x * x;
      if (std::fabs(omx2) < 1000 * e) break;
      const double d2 = (2.0 * x * dPp - (double)(p * (p + 1)) * Pp) / omx2;
      if (std::fabs(d2) < e) break;
      double xn = x - dPp / d2;
      xn = std::fmin(std::fmax(xn, -1.0 + 10 * e), 1.0 - 10 * e);
      const bool done = std::fabs(xn - x) < 10 * e;
      x = xn;
      if (done) break;
    }
    xi[j - 1] = x;
  }
  for (int i = 1; i < n; ++i)  // ascending
    for (int k = i; k > 0 && xi[k - 1] > xi[k]; --k) std::swap(xi[k - 1], xi[k]);
  xi[0] = -1.0;
  xi[n - 1] = 1.0;
  double sw = 0.0;
  for (int i = 0; i < n; ++i) {
    const double Pp = legendre_P(p, xi[i]);
    w[i] = 2.0 / std::fmax((double)p * (double)(p + 1) * Pp * Pp, e);
    sw += w[i];
  }
  for (int i = 0; i < n; ++i) w[i] *= 2.0 / sw;
}

void lagrange_at(int n, const double* xi, double x, double* l) {
  for (int j = 0; j < n; ++j) {
    l[j] = 1.0;
    for (int k = 0; k < n; ++k)
      if (k != j) l[j] *= (x - xi[k]) / (xi[j] - xi[k]);
  }
}

// Gauss-Jordan inverse with partial pivoting (n <= kMaxNp)
bool invert(int n, const double A[kMaxNp][kMaxNp], double R[kMaxNp][kMaxNp]) {
  double M[kMaxNp][2 * kMaxNp];
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < 2 * n; ++j) M[i][j] = j < n ? A[i][j] : (j - n == i ? 1.0 : 0.0);
  for (int c = 0; c < n; ++c) {
    int piv = c;
    for (int r = c + 1; r < n; ++r)
      if (std::fabs(M[r][c]) > std::fabs(M[piv][c])) piv = r;
    if (M[piv][c] == 0.0) return false;
    if (piv != c)
      for (int j = 0; j < 2 * n; ++j) std::swap(M[c][j], M[piv][j]);
    const double d = M[c][c];
    for (int j = 0; j < 2 * n; ++j) M[c][j] /= d;
    for (int r = 0; r < n; ++r) {
      if (r == c) continue;
      const double f = M[r][c];
      if (f == 0.0) continue;
      for (int j = 0; j < 2 * n; ++j) M[r][j] -= f * M[c][j];
    }
  }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) R[i][j] = M[i][n + j];
  return true;
}

long long gcdll(long long a, long long b) {
  a = a < 0 ? -a : a;
  b = b < 0 ? -b : b;
  while (b) {
    long long t = a % b;
    a = b;
    b = t;
  }
  return a;
}

// continued-fraction rational form of x (numerator, denominator <= 2^24)
void rational_of(double x, long long* num, long long* den) {
  double y = x;
  long long a = 1, d = 1, b = 0, c = 0;
  const double m = 16777216.0;
  while (std::fabs(y) <= m) {
    const long long f = (long long)std::trunc(y);
    y -= (double)f;
    const long long na = f * a + c, nb = f * b + d;
    c = a;
    d = b;
    a = na;
    b = nb;
    if (!(std::llabs(a) <= (long long)m && std::llabs(b) <= (long long)m)) {
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

}  // namespace

// Element vertices of Mesh1D/Mesh2D: collect(range(a, b; length=len)).  The
// reference's range writes both ends as ratios of integers over a common
// denominator and rounds each exact element once; we do the same.
void julia_linspace(double a, double b, int len, double* out) {
  if (len == 1) {
    out[0] = a;
    return;
  }
  long long an, ad, bn, bd;
  rational_of(a, &an, &ad);
  rational_of(b, &bn, &bd);
  if (ad != 0 && bd != 0) {
    const long long den = ad / gcdll(ad, bd) * bd;
    const double lim = 9007199254740992.0;
    if (std::fabs((double)den * a) <= lim && std::fabs((double)den * b) <= lim) {
      const long long sn = std::llround((double)den * a), en = std::llround((double)den * b);
      if ((double)sn / (double)den == a && (double)en / (double)den == b) {
        for (int i = 1; i <= len; ++i) {
          const long double num = (long double)(len - i) * sn + (long double)(i - 1) * en;
          const long double dd = (long double)(len - 1) * den;
          if (std::fabs((double)num) < lim && std::fabs((double)dd) < lim)
            out[i - 1] = (double)num / (double)dd;
          else
            out[i - 1] = (double)(num / dd);
        }
        return;
      }
    }
  }
  for (int i = 1; i <= len; ++i)
    out[i - 1] = (double)((long double)a + ((long double)b - a) * (i - 1) / (len - 1));
}

void derive_tables(HostOps* o) {
  const int n = o->np;
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < n; ++k) o->Dt[i][k] = o->D[i][k] - o->gLxi[i] * o->lL[k] - o->gRxi[i] * o->lR[k];
  for (int i = 0; i < n; ++i)
    for (int m = 0; m < n; ++m) {
      double a = 0.0, b = 0.0;
      for (int k = 0; k < n; ++k) {
        a += o->Dt[i][k] * o->D[k][m];
        b += o->D[i][k] * o->D[k][m];
      }
      o->DtD[i][m] = a;
      o->DD[i][m] = b;
    }
  for (int m = 0; m < n; ++m) {
    double a = 0.0, b = 0.0;
    for (int k = 0; k < n; ++k) {
      a += o->lL[k] * o->D[k][m];
      b += o->lR[k] * o->D[k][m];
    }
    o->lLD[m] = a;
    o->lRD[m] = b;
  }
  if (!invert(n, o->V, o->Vinv)) std::memset(o->Vinv, 0, sizeof(o->Vinv));
}

int build_host_ops(int p, int points, HostOps* o) {
  if (p < 1 || p + 1 > kMaxNp) return FRG_ERR_INVALID_ARG;
  if (points != FRG_POINTS_GL && points != FRG_POINTS_GLL) return FRG_ERR_INVALID_ARG;
  std::memset(o, 0, sizeof(*o));
  const int n = p + 1;
  o->p = p;
  o->np = n;
  o->points = points;
  if (points == FRG_POINTS_GL)
    gauss_legendre_newton(n, o->xi, o->w);
  else
    gauss_lobatto_newton(n, o->xi, o->w);
  // differentiation matrix, Points.jl:83-104
  for (int i = 0; i < n; ++i) {
    double diag = 0.0;
    for (int j = 0; j < n; ++j) {
      if (i == j) continue;
      double num = 1.0;
      for (int k = 0; k < n; ++k)
        if (k != i && k != j) num *= (o->xi[i] - o->xi[k]) / (o->xi[j] - o->xi[k]);
      o->D[i][j] = num / (o->xi[j] - o->xi[i]);
      diag += o->D[i][j];
    }
    o->D[i][i] = -diag;
  }
  lagrange_at(n, o->xi, -1.0, o->lL);
  lagrange_at(n, o->xi, 1.0, o->lR);
  const double rRm1 = legendre_P(p + 1, -1.0) - legendre_P(p, -1.0);
  const double rLp1 = legendre_P(p + 1, 1.0) + legendre_P(p, 1.0);
  for (int i = 0; i < n; ++i) {
    const double x = o->xi[i];
    const double Pp = legendre_P(p, x), Pp1 = legendre_P(p + 1, x);
    o->gL[i] = (Pp1 - Pp) / rRm1;
    o->gR[i] = (Pp1 + Pp) / rLp1;
    const double d0 = legendre_dP(p, x), d1 = legendre_dP(p + 1, x);
    o->gLxi[i] = (d1 - d0) / rRm1;
    o->gRxi[i] = (d1 + d0) / rLp1;
  }
  for (int j = 0; j < n; ++j)
    for (int k = 0; k < n; ++k) o->V[j][k] = legendre_P(k, o->xi[j]);
  derive_tables(o);
  return FRG_OK;
}

int host_ops_from_caller(const frg_operators* in, HostOps* o) {
  if (!in || in->p < 1 || in->p + 1 > kMaxNp) return FRG_ERR_INVALID_ARG;
  if (!in->xi || !in->D || !in->l_L || !in->l_R || !in->gL_xi || !in->gR_xi)
    return FRG_ERR_INVALID_ARG;
  HostOps base;
  const int rc = build_host_ops(in->p, in->points, &base);  // w, V fallbacks
  if (rc != FRG_OK) return rc;
  *o = base;
  const int n = in->p + 1;
  for (int i = 0; i < n; ++i) {
    o->xi[i] = in->xi[i];
    if (in->w) o->w[i] = in->w[i];
    o->lL[i] = in->l_L[i];
    o->lR[i] = in->l_R[i];
    o->gLxi[i] = in->gL_xi[i];
    o->gRxi[i] = in->gR_xi[i];
    for (int k = 0; k < n; ++k) {
      o->D[i][k] = in->D[i + n * k];  // column-major in
      if (in->V) o->V[i][k] = in->V[i + n * k];
    }
  }
  derive_tables(o);
  return FRG_OK;
}

}  // namespace frg

extern "C" int frg_build_operators(int p, int points, double* xi, double* w, double* D, double* l_L,
                                   double* l_R, double* gL_xi, double* gR_xi, double* gL,
                                   double* gR, double* V) {
  frg::HostOps o;
  const int rc = frg::build_host_ops(p, points, &o);
  if (rc != FRG_OK) return rc;
  const int n = o.np;
  for (int i = 0; i < n; ++i) {
    if (xi) xi[i] = o.xi[i];
    if (w) w[i] = o.w[i];
    if (l_L) l_L[i] = o.lL[i];
    if (l_R) l_R[i] = o.lR[i];
    if (gL_xi) gL_xi[i] = o.gLxi[i];
    if (gR_xi) gR_xi[i] = o.gRxi[i];
    if (gL) gL[i] = o.gL[i];
    if (gR) gR[i] = o.gR[i];
    for (int k = 0; k < n; ++k) {
      if (D) D[i + n * k] = o.D[i][k];
      if (V) V[i + n * k] = o.V[i][k];
    }
  }
  return FRG_OK;
}

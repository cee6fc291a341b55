// Host-side 1-D discretisation tables for the B200 engine.
//
// Gauss-Lobatto-Legendre (GLL) and Gauss-Legendre points and weights, the GLL
// collocation derivative, the orthonormal Legendre basis sampled on both point
// sets, and the two side interpolation operators DGM uses:
//   GL2G: GLL element points -> Gauss side points  (src/Hex.cpp:866-884)
//   G2GL: Gauss side points  -> GLL element points (src/Hex.cpp:866-884)
// The point sets come from the Jacobi-polynomial Newton iteration with
// deflation published with Polylib (Karniadakis & Sherwin, appendix B), the
// algorithm src/Polylib.tpp:351-478 implements, so the tables agree with the
// reference's to the last few ulps.  The basis is orthonormal because the
// reference is built with DGM_BASIS_NORM (src/Basis.hpp:55).
#include <cmath>
#include <vector>

#include "dgmx_internal.hpp"

namespace dgmx {
namespace {

// P_n^{(al,be)}(x) by the normalised three-term recurrence.
double jacobi(int n, double al, double be, double x) {
  if (n == 0) return 1.0;
  double p0 = 1.0, p1 = 0.5 * (al - be + (al + be + 2.0) * x);
  const double s = al + be;
  for (int k = 2; k <= n; ++k) {
    const double a1 = 2.0 * k * (k + s) * (2.0 * k + s - 2.0);
    const double a2 = (2.0 * k + s - 1.0) * (al * al - be * be) / a1;
    const double a3 = (2.0 * k + s - 2.0) * (2.0 * k + s - 1.0) * (2.0 * k + s) / a1;
    const double a4 = 2.0 * (k + al - 1.0) * (k + be - 1.0) * (2.0 * k + s) / a1;
    const double p2 = (a2 + a3 * x) * p1 - a4 * p0;
    p0 = p1;
    p1 = p2;
  }
  return p1;
}

double jacobi_deriv(int n, double al, double be, double x) {
  if (n == 0) return 0.0;
  return 0.5 * (al + be + n + 1.0) * jacobi(n - 1, al + 1.0, be + 1.0, x);
}

// Zeros of P_n^{(al,be)}: Chebyshev-Gauss guesses, each refined by Newton's
// method on P_n divided by the zeros already found.
void jacobi_roots(int n, double al, double be, double *z) {
  double prev = 0.0;
  for (int k = 0; k < n; ++k) {
    double r = -std::cos((2.0 * k + 1.0) * M_PI / (2.0 * n));
    if (k) r = 0.5 * (r + prev);
    for (int it = 1; it < 30; ++it) {
      const double p = jacobi(n, al, be, r);
      const double dp = jacobi_deriv(n, al, be, r);
      double defl = 0.0;
      for (int i = 0; i < k; ++i) defl += 1.0 / (r - z[i]);
      const double step = -p / (dp - defl * p);
      r += step;
      if (std::fabs(step) < 1.0e-12) break;
    }
    z[k] = r;
    prev = r;
  }
}

}  // namespace

void gll_points(int Q, double *z, double *w) {
  if (Q == 1) { z[0] = 0.0; w[0] = 2.0; return; }
  z[0] = -1.0;
  z[Q - 1] = 1.0;
  jacobi_roots(Q - 2, 1.0, 1.0, z + 1);
  for (int i = 0; i < Q; ++i) {
    const double p = jacobi(Q - 1, 0.0, 0.0, z[i]);
    w[i] = 2.0 / (Q * (Q - 1.0)) / (p * p);
  }
}

void gauss_points(int G, double *z, double *w) {
  jacobi_roots(G, 0.0, 0.0, z);
  for (int i = 0; i < G; ++i) {
    const double dp = jacobi_deriv(G, 0.0, 0.0, z[i]);
    w[i] = 2.0 / (dp * dp * (1.0 - z[i] * z[i]));
  }
}

Tables1D make_tables(int L, int Q, int G) {
  Tables1D t;
  t.L = L; t.Q = Q; t.G = G;
  t.z.resize(Q); t.w.resize(Q); t.zg.resize(G); t.wg.resize(G);
  gll_points(Q, t.z.data(), t.w.data());
  gauss_points(G, t.zg.data(), t.wg.data());
  // collocation derivative on GLL points: D[i][j] = l_j'(z_i), using
  // l_j'(z_i) = c_i / (c_j (z_i - z_j)) with c_i = (1-z_i^2) P'_{Q-1}(z_i)
  // in the interior and the closed forms at the end points.
  t.D.assign(Q * Q, 0.0);
  std::vector<double> c(Q);
  for (int i = 0; i < Q; ++i) {
    if (i == 0) c[i] = (Q % 2 == 0 ? 2.0 : -2.0) * (Q - 1.0);
    else if (i == Q - 1) c[i] = -2.0 * (Q - 1.0);
    else c[i] = (1.0 - t.z[i] * t.z[i]) * jacobi_deriv(Q - 2, 1.0, 1.0, t.z[i]);
  }
  for (int i = 0; i < Q; ++i)
    for (int j = 0; j < Q; ++j) {
      double v;
      if (i != j) v = c[i] / (c[j] * (t.z[i] - t.z[j]));
      else if (i == 0) v = -0.25 * (Q - 1.0) * Q;
      else if (i == Q - 1) v = 0.25 * (Q - 1.0) * Q;
      else v = 0.0;
      t.D[i * Q + j] = v;
    }
  // orthonormal Legendre on GLL and on Gauss points
  t.B.resize(L * Q);
  t.Bg.resize(L * G);
  for (int a = 0; a < L; ++a) {
    const double s = std::sqrt(0.5 * (2.0 * a + 1.0));
    for (int i = 0; i < Q; ++i) t.B[a * Q + i] = s * jacobi(a, 0.0, 0.0, t.z[i]);
    for (int g = 0; g < G; ++g) t.Bg[a * G + g] = s * jacobi(a, 0.0, 0.0, t.zg[g]);
  }
  // GL2G[g][i]: GLL Lagrange polynomial i evaluated at Gauss point g,
  //   l_i(x) = (1-x^2) P'_{Q-1}(x) / (((1-z_i^2) P'_{Q-1}(z_i))' (x - z_i))
  // G2GL[i][g]: Gauss Lagrange polynomial g evaluated at GLL point i,
  //   h_g(x) = P_G(x) / (P_G'(zg_g) (x - zg_g))
  t.gl2g.resize(G * Q);
  for (int g = 0; g < G; ++g)
    for (int i = 0; i < Q; ++i) {
      const double zi = t.z[i], x = t.zg[g], dx = x - zi;
      double v;
      if (std::fabs(dx) < 1.0e-12) v = 1.0;
      else {
        const double den = (1.0 - zi * zi) * jacobi_deriv(Q - 2, 1.0, 1.0, zi) -
                           2.0 * zi * jacobi(Q - 2, 1.0, 1.0, zi);
        v = (1.0 - x * x) * jacobi(Q - 2, 1.0, 1.0, x) / (den * dx);
      }
      t.gl2g[g * Q + i] = v;
    }
  t.g2gl.resize(Q * G);
  for (int i = 0; i < Q; ++i)
    for (int g = 0; g < G; ++g) {
      const double zg = t.zg[g], x = t.z[i], dx = x - zg;
      double v;
      if (std::fabs(dx) < 1.0e-12) v = 1.0;
      else v = jacobi(G, 0.0, 0.0, x) / (jacobi_deriv(G, 0.0, 0.0, zg) * dx);
      t.g2gl[i * G + g] = v;
    }
  return t;
}

}  // namespace dgmx

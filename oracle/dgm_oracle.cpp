// =============================================================================
// dgm_oracle.cpp -- CPU FP64 restatement of DGM's DG residual and RK stage.
//
// TEST INFRASTRUCTURE ONLY.  This file is the correctness oracle: it is loaded
// by tests/, by __graft_entry__.smoke() and by bench.py's cpu_baseline and
// reference arms, and by nothing in the product (dgm_b200/).  It restates,
// operation for operation, the algorithm of the reference DGM code for
//   Domain::time_derivative of Euler (2-D/3-D), Navier-Stokes (2-D/3-D, BR1)
//   and shallow water on affine Quad/Hex elements, and the RK4, TVD-RK3 and
//   LSRK14 stage updates that consume it.
// Citations are path:line inside the reference project (sandialabs/dgm).
//
// Parity status: pinned against the reference's own golden restart files
// runs/vhex.ref, runs/vquad.ref, runs/vortex.ref and runs/chan/chan.ref
// (tests/golden/, checked by tests/test_oracle_golden.py and
// tests/test_restart.py).  runs/nvortex.ref uses NodalQuad elements, which
// this oracle does not restate, so it pins nothing here.
// =============================================================================
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace ora {

typedef std::vector<double> vec;

// -----------------------------------------------------------------------------
// Gauss-Jacobi quadrature, derivative and interpolation operators.
// Restates the published Polylib algorithms that src/Polylib.tpp implements
// (Karniadakis & Sherwin, "Spectral/hp Element Methods", appendix B).
// -----------------------------------------------------------------------------
static const double kNewtonTol = 1.0e-12;   // src/Polylib.tpp:201
static const int kNewtonMax = 30;           // src/Polylib.tpp:197

// Jacobi polynomial P_n^{(a,b)} at np points, normalised three-term
// recurrence (src/Polylib.tpp:1434-1488).
static void jacobi_values(int np, const double *z, double *poly, int n,
                          double a, double b) {
  if (np <= 0) return;
  if (n == 0) { for (int i = 0; i < np; ++i) poly[i] = 1.0; return; }
  if (n == 1) {
    for (int i = 0; i < np; ++i) poly[i] = 0.5 * (a - b + (a + b + 2.0) * z[i]);
    return;
  }
  vec pm1(np), pm2(np);
  for (int i = 0; i < np; ++i) {
    pm2[i] = 1.0;
    pm1[i] = 0.5 * (a - b + (a + b + 2.0) * z[i]);
  }
  const double ab = a + b;
  for (int k = 2; k <= n; ++k) {
    double c1 = 2.0 * k * (k + ab) * (2.0 * k + ab - 2.0);
    double c2 = (2.0 * k + ab - 1.0) * (a * a - b * b);
    double c3 = (2.0 * k + ab - 2.0) * (2.0 * k + ab - 1.0) * (2.0 * k + ab);
    double c4 = 2.0 * (k + a - 1.0) * (k + b - 1.0) * (2.0 * k + ab);
    c2 /= c1; c3 /= c1; c4 /= c1;
    for (int i = 0; i < np; ++i) {
      poly[i] = (c2 + c3 * z[i]) * pm1[i] - c4 * pm2[i];
      pm2[i] = pm1[i];
      pm1[i] = poly[i];
    }
  }
}

// d/dz P_n^{(a,b)} = 0.5 (a+b+n+1) P_{n-1}^{(a+1,b+1)} (src/Polylib.tpp:1496-1507)
static void jacobi_derivs(int np, const double *z, double *pd, int n,
                          double a, double b) {
  if (n == 0) { for (int i = 0; i < np; ++i) pd[i] = 0.0; return; }
  jacobi_values(np, z, pd, n - 1, a + 1.0, b + 1.0);
  for (int i = 0; i < np; ++i) pd[i] *= 0.5 * (a + b + (double)n + 1.0);
}

// Value and derivative at one point, unnormalised recurrence used by the
// Newton root finder (src/Polylib.tpp:279-314).
static void jacobi_point(double z, double *p, double *pd, int n, double a,
                         double b) {
  if (n == 0) { *p = 1.0; *pd = 0.0; return; }
  if (n == 1) { *p = 0.5 * (a - b + (a + b + 2.0) * z); *pd = 0.5 * (a + b + 2.0); return; }
  const double ab = a + b;
  double q2 = 1.0, q1 = 0.5 * (a - b + (ab + 2.0) * z);
  for (int k = 2; k <= n; ++k) {
    double c1 = 2.0 * k * (k + ab) * (2.0 * k + ab - 2.0);
    double c2 = (2.0 * k + ab - 1.0) * (a * a - b * b);
    double c3 = (2.0 * k + ab - 2.0) * (2.0 * k + ab - 1.0) * (2.0 * k + ab);
    double c4 = 2.0 * (k + a - 1.0) * (k + b - 1.0) * (2.0 * k + ab);
    *p = ((c2 + c3 * z) * q1 - c4 * q2) / c1;
    q2 = q1;
    q1 = *p;
  }
  double prev = q2;
  *pd = n * (a - b - (2.0 * n + a + b) * z) * (*p);
  *pd += 2.0 * (n + a) * (n + b) * prev;
  *pd /= (2.0 * n + a + b) * (1.0 - z * z);
}

// Gamma function on integers and half integers (src/Polylib.tpp:322-345).
static double gamma_int_half(double x) {
  double g = 1.0;
  if (x == -0.5) return -2.0 * std::sqrt(M_PI);
  if (x == 0.0) return g;
  if ((x - (long long)x) == 0.5) {
    long long n = (long long)x;
    double t = x;
    g = std::sqrt(M_PI);
    while (n--) { t -= 1.0; g *= t; }
  } else {
    long long n = (long long)x;
    double t = x;
    while (--n) { t -= 1.0; g *= t; }
  }
  return g;
}

// Zeros of P_n^{(a,b)}: Chebyshev initial guesses, Newton with deflation
// (src/Polylib.tpp:351-381).
static void jacobi_zeros(int n, double *z, double a, double b) {
  if (!n) return;
  const double dth = M_PI / (2.0 * n);
  double rlast = 0.0;
  for (int k = 0; k < n; ++k) {
    double r = -std::cos((2.0 * k + 1.0) * dth);
    if (k) r = 0.5 * (r + rlast);
    for (int it = 1; it < kNewtonMax; ++it) {
      double p = 0, pd = 0;
      jacobi_point(r, &p, &pd, n, a, b);
      double s = 0.0;
      for (int i = 0; i < k; ++i) s += 1.0 / (r - z[i]);
      double dr = -p / (pd - s * p);
      r += dr;
      if (std::fabs(dr) < kNewtonTol) break;
    }
    z[k] = r;
    rlast = r;
  }
}

// Gauss-Legendre points/weights (src/Polylib.tpp:388-404 with a=b=0).
static void gauss_legendre(int np, double *z, double *w) {
  jacobi_zeros(np, z, 0.0, 0.0);
  jacobi_derivs(np, z, w, np, 0.0, 0.0);
  for (int i = 0; i < np; ++i) w[i] = 2.0 / (w[i] * w[i] * (1.0 - z[i] * z[i]));
}

// Gauss-Lobatto-Legendre points/weights (src/Polylib.tpp:451-478, a=b=0).
static void gauss_lobatto_legendre(int np, double *z, double *w) {
  if (np == 1) { z[0] = 0.0; w[0] = 2.0; return; }
  z[0] = -1.0;
  z[np - 1] = 1.0;
  jacobi_zeros(np - 2, z + 1, 1.0, 1.0);
  jacobi_values(np, z, w, np - 1, 0.0, 0.0);
  const double fac = 2.0 / (double)(np * (np - 1));
  for (int i = 0; i < np; ++i) w[i] = fac / (w[i] * w[i]);
}

// Collocation derivative matrix on GLL points, d[i*np+j] = d l_j/dz (z_i)
// (src/Polylib.tpp:1008-1049 with a=b=0).
static void gll_derivative(int np, const double *z, double *d) {
  if (np <= 1) { d[0] = 0.0; return; }
  vec pd(np);
  pd[0] = 2.0 * std::pow(-1.0, np) * gamma_int_half(np + 0.0);
  pd[0] /= gamma_int_half(np - 1.0) * gamma_int_half(2.0);
  jacobi_derivs(np - 2, z + 1, pd.data() + 1, np - 2, 1.0, 1.0);
  for (int i = 1; i < np - 1; ++i) pd[i] *= (1.0 - z[i] * z[i]);
  pd[np - 1] = -2.0 * gamma_int_half(np + 0.0);
  pd[np - 1] /= gamma_int_half(np - 1.0) * gamma_int_half(2.0);
  for (int i = 0; i < np; ++i)
    for (int j = 0; j < np; ++j) {
      double v;
      if (i != j) v = pd[i] / (pd[j] * (z[i] - z[j]));
      else if (i == 0) v = (0.0 - (np - 1) * (np + 0.0)) / (2.0 * 2.0);
      else if (i == np - 1) v = -(0.0 - (np - 1) * (np + 0.0)) / (2.0 * 2.0);
      else v = 0.0 / (2.0 * (1.0 - z[i] * z[i]));
      d[i * np + j] = v;
    }
}

// Lagrange interpolant through np GLL points (src/Polylib.tpp:1339-1360).
static double lagrange_gll(int i, double z, const double *zg, int np) {
  const double zi = zg[i];
  const double dz = z - zi;
  if (std::fabs(dz) < kNewtonTol) return 1.0;
  double p, pd;
  jacobi_values(1, &zi, &p, np - 2, 1.0, 1.0);
  jacobi_derivs(1, &zi, &pd, np - 2, 1.0, 1.0);
  double h = (1.0 - zi * zi) * pd - 2.0 * zi * p;
  jacobi_values(1, &z, &p, np - 2, 1.0, 1.0);
  return (1.0 - z * z) * p / (h * dz);
}

// Lagrange interpolant through np Gauss points (src/Polylib.tpp:1296-1309).
static double lagrange_gauss(int i, double z, const double *zg, int np) {
  const double zi = zg[i];
  const double dz = z - zi;
  if (std::fabs(dz) < kNewtonTol) return 1.0;
  double p, pd;
  jacobi_derivs(1, &zi, &pd, np, 0.0, 0.0);
  jacobi_values(1, &z, &p, np, 0.0, 0.0);
  return p / (pd * dz);
}

// -----------------------------------------------------------------------------
// 1-D tables: GLL points, weights, collocation derivative and the
// orthonormal Legendre basis sampled on GLL points (DGM_BASIS_NORM is
// defined in src/Basis.hpp:55, so rows are scaled by sqrt((2l+1)/2),
// src/Basis.cpp:97-101).
// -----------------------------------------------------------------------------
struct Table1D {
  int L = 0, Q = 0;
  vec z, w;   // GLL points and weights (Q)
  vec D;      // Q x Q collocation derivative, D[i*Q+j]
  vec B;      // L x Q orthonormal Legendre, B[l*Q+i]
};

struct Interp {
  int qto = 0, qfrom = 0;
  vec m;      // qto x qfrom
};

static std::mutex g_tab_mutex;
static std::map<std::pair<int, int>, std::shared_ptr<Table1D>> g_tables;
static std::map<std::tuple<int, int, int>, std::shared_ptr<Interp>> g_interps;

static std::shared_ptr<Table1D> table(int L, int Q) {
  std::lock_guard<std::mutex> lk(g_tab_mutex);
  auto key = std::make_pair(L, Q);
  auto it = g_tables.find(key);
  if (it != g_tables.end()) return it->second;
  auto t = std::make_shared<Table1D>();
  t->L = L; t->Q = Q;
  t->z.resize(Q); t->w.resize(Q); t->D.resize(Q * Q); t->B.resize(L * Q);
  gauss_lobatto_legendre(Q, t->z.data(), t->w.data());
  gll_derivative(Q, t->z.data(), t->D.data());
  for (int l = 0; l < L; ++l) {
    jacobi_values(Q, t->z.data(), &t->B[l * Q], l, 0.0, 0.0);
    const double s = std::sqrt(0.5 * (2.0 * l + 1.0));
    for (int i = 0; i < Q; ++i) t->B[l * Q + i] *= s;
  }
  g_tables[key] = t;
  return t;
}

// type 0: GL2G (GLL qfrom -> Gauss qto); type 1: G2GL (Gauss qfrom -> GLL qto)
// (src/Quad.cpp:863-882, src/Hex.cpp:866-889)
static std::shared_ptr<Interp> interp(int type, int qto, int qfrom) {
  std::lock_guard<std::mutex> lk(g_tab_mutex);
  auto key = std::make_tuple(type, qto, qfrom);
  auto it = g_interps.find(key);
  if (it != g_interps.end()) return it->second;
  auto r = std::make_shared<Interp>();
  r->qto = qto; r->qfrom = qfrom; r->m.resize(qto * qfrom);
  vec zt(qto), wt(qto), zf(qfrom), wf(qfrom);
  if (type == 0) {
    gauss_lobatto_legendre(qfrom, zf.data(), wf.data());
    gauss_legendre(qto, zt.data(), wt.data());
    for (int i = 0; i < qto; ++i)
      for (int j = 0; j < qfrom; ++j)
        r->m[i * qfrom + j] = lagrange_gll(j, zt[i], zf.data(), qfrom);
  } else {
    gauss_legendre(qfrom, zf.data(), wf.data());
    gauss_lobatto_legendre(qto, zt.data(), wt.data());
    for (int i = 0; i < qto; ++i)
      for (int j = 0; j < qfrom; ++j)
        r->m[i * qfrom + j] = lagrange_gauss(j, zt[i], zf.data(), qfrom);
  }
  g_interps[key] = r;
  return r;
}

// -----------------------------------------------------------------------------
// Elements and sides (affine Quad / Hex).
// -----------------------------------------------------------------------------
struct Side {
  int id = 0;
  int q1 = 0, q2 = 1, qtot = 0;  // Gauss points per direction (q2=1 in 2-D)
  bool master = false;
  int link_e = -1, link_s = -1;
  int bc = -1;                    // boundary: index of the boundary record / ghost side
  bool flip_a = false, flip_b = false, transp = false;
  size_t off = 0;                 // offset into one field's side storage
  vec nx, ny, nz, J;              // J = surface Jacobian / interior Jacobian
  std::shared_ptr<Interp> to1, to2, from1, from2;  // GL2G / G2GL per direction
};

struct Elem {
  int dim = 2, L = 0, Q = 0, qtot = 0, nmodes = 0, nsides = 0;
  double X[8][3];
  double rx = 0, ry = 0, rz = 0, sx = 0, sy = 0, sz = 0, tx = 0, ty = 0, tz = 0;
  double J = 0;
  vec wJ, cx, cy, cz;
  size_t off = 0;                 // offset into one field's interior storage
  Side side[6];
  std::shared_ptr<Table1D> T;
};

// Hex face vertices (src/Hex.cpp:68-69)
static const int kHexFaceVerts[6][4] = {{0, 1, 2, 3}, {0, 1, 5, 4}, {1, 2, 6, 5},
                                        {3, 2, 6, 7}, {0, 3, 7, 4}, {4, 5, 6, 7}};
// Quad edge-flip table (src/Field.cpp:87-90)
static const int kQuadFlip[4][4] = {{1, 1, 0, 0}, {1, 1, 0, 0}, {0, 0, 1, 1}, {0, 0, 1, 1}};

// Quad side extraction (src/Quad.cpp:767-790); point (i,j) -> i*qb+j
static void quad_get_side(const Elem &E, const double *f, int s, double *to) {
  const int qa = E.Q, qb = E.Q;
  switch (s) {
    case 0: for (int p = 0; p < qa; ++p) to[p] = f[0 + p * qb]; break;
    case 1: for (int q = 0; q < qb; ++q) to[q] = f[q + (qa - 1) * qb]; break;
    case 2: for (int p = 0; p < qa; ++p) to[p] = f[(qb - 1) + p * qb]; break;
    case 3: for (int q = 0; q < qb; ++q) to[q] = f[q + 0 * qb]; break;
  }
}

// Hex side extraction (src/Hex.cpp:815-865); point (i,j,k) -> (i*qb+j)*qc+k
static void hex_get_side(const Elem &E, const double *f, int s, double *to) {
  const int qa = E.Q, qb = E.Q, qc = E.Q;
  auto F = [&](int i, int j, int k) { return f[(i * qb + j) * qc + k]; };
  switch (s) {
    case 0: for (int i = 0; i < qa; ++i) for (int j = 0; j < qb; ++j) to[i * qb + j] = F(i, j, 0); break;
    case 1: for (int i = 0; i < qa; ++i) for (int k = 0; k < qc; ++k) to[i * qc + k] = F(i, 0, k); break;
    case 2: for (int j = 0; j < qb; ++j) for (int k = 0; k < qc; ++k) to[j * qc + k] = F(qa - 1, j, k); break;
    case 3: for (int i = 0; i < qa; ++i) for (int k = 0; k < qc; ++k) to[i * qc + k] = F(i, qb - 1, k); break;
    case 4: for (int j = 0; j < qb; ++j) for (int k = 0; k < qc; ++k) to[j * qc + k] = F(0, j, k); break;
    case 5: for (int i = 0; i < qa; ++i) for (int j = 0; j < qb; ++j) to[i * qb + j] = F(i, j, qc - 1); break;
  }
}

static void get_side(const Elem &E, const double *f, int s, double *to) {
  if (E.dim == 2) quad_get_side(E, f, s, to); else hex_get_side(E, f, s, to);
}

// GLL side values -> Gauss side values (src/Quad.cpp:884-905 mvmult;
// src/Hex.cpp:1294-1318 two matmults)
static void interpolate_to_side(const Elem &E, int s, const double *from, double *to) {
  const Side &S = E.side[s];
  if (E.dim == 2) {
    const Interp *im = S.to1.get();
    for (int i = 0; i < S.q1; ++i) {
      double acc = 0.0;
      for (int j = 0; j < E.Q; ++j) acc += im->m[i * E.Q + j] * from[j];
      to[i] = acc;
    }
  } else {
    const int q1 = E.Q, q2 = E.Q;
    const Interp *im1 = S.to1.get(), *im2 = S.to2.get();
    vec wk(S.q1 * q2);
    for (int i = 0; i < S.q1; ++i)
      for (int j = 0; j < q2; ++j) {
        double acc = 0.0;
        for (int m = 0; m < q1; ++m) acc += im1->m[i * q1 + m] * from[m * q2 + j];
        wk[i * q2 + j] = acc;
      }
    for (int i = 0; i < S.q1; ++i)
      for (int j = 0; j < S.q2; ++j) {
        double acc = 0.0;
        for (int m = 0; m < q2; ++m) acc += wk[i * q2 + m] * im2->m[j * q2 + m];
        to[i * S.q2 + j] = acc;
      }
  }
}

// Gauss side values -> GLL side values (src/Quad.cpp:1988-1991;
// src/Hex.cpp:1320-1341)
static void interpolate_from_side(const Elem &E, int s, const double *from, double *to) {
  const Side &S = E.side[s];
  if (E.dim == 2) {
    const Interp *im = S.from1.get();
    for (int i = 0; i < E.Q; ++i) {
      double acc = 0.0;
      for (int j = 0; j < S.q1; ++j) acc += im->m[i * S.q1 + j] * from[j];
      to[i] = acc;
    }
  } else {
    const int q1 = E.Q, q2 = E.Q;
    const Interp *im1 = S.from1.get(), *im2 = S.from2.get();
    vec wk(q1 * S.q2);
    for (int i = 0; i < q1; ++i)
      for (int j = 0; j < S.q2; ++j) {
        double acc = 0.0;
        for (int m = 0; m < S.q1; ++m) acc += im1->m[i * S.q1 + m] * from[m * S.q2 + j];
        wk[i * S.q2 + j] = acc;
      }
    for (int i = 0; i < q1; ++i)
      for (int j = 0; j < q2; ++j) {
        double acc = 0.0;
        for (int m = 0; m < S.q2; ++m) acc += wk[i * S.q2 + m] * im2->m[j * S.q2 + m];
        to[i * q2 + j] = acc;
      }
  }
}

// side quadrature index map with flips/transpose (src/BaseQuad.hpp:53-57,
// src/BaseHex.hpp:291-308)
static int side_map(int dim, const Side &s, int ql) {
  if (dim == 2) return s.flip_a ? (s.q1 - 1) - ql : ql;
  const int il = ql / s.q2, jl = ql % s.q2;
  int i, j;
  if (s.transp) {
    j = il; i = jl;
    if (s.flip_a) j = (s.q1 - 1) - j;
    if (s.flip_b) i = (s.q2 - 1) - i;
  } else {
    i = il; j = jl;
    if (s.flip_a) i = (s.q1 - 1) - i;
    if (s.flip_b) j = (s.q2 - 1) - j;
  }
  return j + s.q2 * i;
}

// Collocation gradient along one physical direction
// (src/Quad.cpp:2308-2330, src/Hex.cpp:2030-2071)
static void gradient_dir(const Elem &E, const double *f, double *df, char dir) {
  const int Q = E.Q;
  const double *D = E.T->D.data();
  if (E.dim == 2) {
    vec fr(E.qtot), fs(E.qtot);
    for (int i = 0; i < Q; ++i)
      for (int j = 0; j < Q; ++j) {
        double a = 0.0, b = 0.0;
        for (int m = 0; m < Q; ++m) a += D[i * Q + m] * f[m * Q + j];
        for (int m = 0; m < Q; ++m) b += f[i * Q + m] * D[j * Q + m];
        fr[i * Q + j] = a;
        fs[i * Q + j] = b;
      }
    double c1 = dir == 'x' ? E.rx : E.ry;
    double c2 = dir == 'x' ? E.sx : E.sy;
    for (int i = 0; i < E.qtot; ++i) { df[i] = c1 * fr[i]; df[i] = c2 * fs[i] + df[i]; }
  } else {
    vec fr(E.qtot), fs(E.qtot), ft(E.qtot);
    const int Q2 = Q * Q;
    for (int i = 0; i < Q; ++i)
      for (int jk = 0; jk < Q2; ++jk) {
        double a = 0.0;
        for (int m = 0; m < Q; ++m) a += D[i * Q + m] * f[m * Q2 + jk];
        fr[i * Q2 + jk] = a;
      }
    for (int i = 0; i < Q; ++i)
      for (int j = 0; j < Q; ++j)
        for (int k = 0; k < Q; ++k) {
          double a = 0.0;
          for (int m = 0; m < Q; ++m) a += D[j * Q + m] * f[i * Q2 + m * Q + k];
          fs[i * Q2 + j * Q + k] = a;
        }
    for (int ij = 0; ij < Q2; ++ij)
      for (int k = 0; k < Q; ++k) {
        double a = 0.0;
        for (int m = 0; m < Q; ++m) a += f[ij * Q + m] * D[k * Q + m];
        ft[ij * Q + k] = a;
      }
    double c1, c2, c3;
    if (dir == 'x') { c1 = E.rx; c2 = E.sx; c3 = E.tx; }
    else if (dir == 'y') { c1 = E.ry; c2 = E.sy; c3 = E.ty; }
    else { c1 = E.rz; c2 = E.sz; c3 = E.tz; }
    for (int i = 0; i < E.qtot; ++i) {
      df[i] = c1 * fr[i];
      df[i] = c2 * fs[i] + df[i];
      df[i] = c3 * ft[i] + df[i];
    }
  }
}

// Fill all sides of one element with GLL->Gauss traces (src/Quad.cpp:884-905,
// src/Hex.cpp:933-947).  sb = base of this field's side storage.
static void fill_sides(const Elem &E, const double *f, double *sb) {
  vec wk(E.Q * E.Q);
  for (int s = 0; s < E.nsides; ++s) {
    get_side(E, f, s, wk.data());
    interpolate_to_side(E, s, wk.data(), sb + E.side[s].off);
  }
}

// Normal-flux version: side = n . (fx,fy[,fz]) at Gauss points
// (src/Quad.cpp:930-970, src/Hex.cpp:950-972)
static void fill_sides_flux(const Elem &E, const double *fx, const double *fy,
                            const double *fz, double *sb) {
  vec wk(E.Q * E.Q), tmp(64 * 64);
  for (int s = 0; s < E.nsides; ++s) {
    const Side &S = E.side[s];
    double *u = sb + S.off;
    get_side(E, fx, s, wk.data());
    interpolate_to_side(E, s, wk.data(), u);
    for (int q = 0; q < S.qtot; ++q) u[q] = S.nx[q] * u[q];
    get_side(E, fy, s, wk.data());
    interpolate_to_side(E, s, wk.data(), tmp.data());
    for (int q = 0; q < S.qtot; ++q) u[q] = S.ny[q] * tmp[q] + u[q];
    if (E.dim == 3) {
      get_side(E, fz, s, wk.data());
      interpolate_to_side(E, s, wk.data(), tmp.data());
      for (int q = 0; q < S.qtot; ++q) u[q] = S.nz[q] * tmp[q] + u[q];
    }
  }
}

// Lift (F^ - F) J n_dir onto the element's boundary GLL points scaled by the
// inverse end weight (Quad: src/Quad.cpp:1971-2038 + 2189-2232;
// Hex: src/Hex.cpp:1768-1952).  fsb = flux-field sides, usb = state sides.
static void lift(const Elem &E, const double *fsb, const double *usb, double *in, char dir) {
  const int Q = E.Q;
  const vec &w = E.T->w;
  if (E.dim == 2) {
    vec f(64), fi(64);
    for (int e = 0; e < 4; ++e) {
      const Side &S = E.side[e];
      const double *Fs = fsb + S.off, *Us = usb + S.off;
      for (int q = 0; q < S.qtot; ++q) f[q] = Fs[q] - Us[q];
      for (int q = 0; q < S.qtot; ++q) f[q] = S.J[q] * f[q];
      if (dir == 'x') for (int q = 0; q < S.qtot; ++q) f[q] = S.nx[q] * f[q];
      else if (dir == 'y') for (int q = 0; q < S.qtot; ++q) f[q] = S.ny[q] * f[q];
      interpolate_from_side(E, e, f.data(), fi.data());
      double sc;
      switch (e) {
        case 0: sc = 1.0 / w[0]; for (int i = 0; i < Q; ++i) fi[i] = sc * fi[i];
                for (int i = 0; i < Q; ++i) in[i * Q + 0] = fi[i] + in[i * Q + 0]; break;
        case 1: sc = 1.0 / w[Q - 1]; for (int i = 0; i < Q; ++i) fi[i] = sc * fi[i];
                for (int j = 0; j < Q; ++j) in[(Q - 1) * Q + j] = fi[j] + in[(Q - 1) * Q + j]; break;
        case 2: sc = 1.0 / w[Q - 1]; for (int i = 0; i < Q; ++i) fi[i] = sc * fi[i];
                for (int i = 0; i < Q; ++i) in[i * Q + (Q - 1)] = fi[i] + in[i * Q + (Q - 1)]; break;
        case 3: sc = 1.0 / w[0]; for (int i = 0; i < Q; ++i) fi[i] = sc * fi[i];
                for (int j = 0; j < Q; ++j) in[0 * Q + j] = fi[j] + in[0 * Q + j]; break;
      }
    }
  } else {
    const double W[6] = {1.0 / w[0], 1.0 / w[0], 1.0 / w[Q - 1],
                         1.0 / w[Q - 1], 1.0 / w[0], 1.0 / w[Q - 1]};
    vec f(64 * 64), fi(64 * 64);
    const int Q2 = Q * Q;
    for (int s = 0; s < 6; ++s) {
      const Side &S = E.side[s];
      const double *Fs = fsb + S.off, *Us = usb + S.off;
      for (int q = 0; q < S.qtot; ++q) f[q] = Fs[q] - Us[q];
      for (int q = 0; q < S.qtot; ++q) f[q] = S.J[q] * f[q];
      if (dir == 'x') for (int q = 0; q < S.qtot; ++q) f[q] = S.nx[q] * f[q];
      else if (dir == 'y') for (int q = 0; q < S.qtot; ++q) f[q] = S.ny[q] * f[q];
      else if (dir == 'z') for (int q = 0; q < S.qtot; ++q) f[q] = S.nz[q] * f[q];
      interpolate_from_side(E, s, f.data(), fi.data());
      const double a = W[s];
      switch (s) {
        case 0: for (int ij = 0; ij < Q2; ++ij) in[ij * Q + 0] = a * fi[ij] + in[ij * Q + 0]; break;
        case 1: for (int i = 0; i < Q; ++i) for (int k = 0; k < Q; ++k)
                  in[i * Q2 + 0 * Q + k] = a * fi[i * Q + k] + in[i * Q2 + 0 * Q + k]; break;
        case 2: for (int jk = 0; jk < Q2; ++jk) in[(Q - 1) * Q2 + jk] = a * fi[jk] + in[(Q - 1) * Q2 + jk]; break;
        case 3: for (int i = 0; i < Q; ++i) for (int k = 0; k < Q; ++k)
                  in[i * Q2 + (Q - 1) * Q + k] = a * fi[i * Q + k] + in[i * Q2 + (Q - 1) * Q + k]; break;
        case 4: for (int jk = 0; jk < Q2; ++jk) in[jk] = a * fi[jk] + in[jk]; break;
        case 5: for (int ij = 0; ij < Q2; ++ij) in[ij * Q + (Q - 1)] = a * fi[ij] + in[ij * Q + (Q - 1)]; break;
      }
    }
  }
}

// Inner product against the basis with wJ (f is scaled in place as in the
// reference) followed by the diagonal inverse mass 1/J
// (src/Quad.cpp:632-662, :286-305; src/Hex.cpp:652-685, :289-301).
static void forward_transform(const Elem &E, double *f, double *fh) {
  const int Q = E.Q, L = E.L;
  const double *B = E.T->B.data();
  for (int i = 0; i < E.qtot; ++i) f[i] = E.wJ[i] * f[i];
  if (E.dim == 2) {
    vec wk(L * Q);
    for (int a = 0; a < L; ++a)
      for (int j = 0; j < Q; ++j) {
        double acc = 0.0;
        for (int i = 0; i < Q; ++i) acc += B[a * Q + i] * f[i * Q + j];
        wk[a * Q + j] = acc;
      }
    for (int a = 0; a < L; ++a)
      for (int b = 0; b < L; ++b) {
        double acc = 0.0;
        for (int j = 0; j < Q; ++j) acc += wk[a * Q + j] * B[b * Q + j];
        fh[a * L + b] = acc;
      }
  } else {
    const int Q2 = Q * Q;
    vec H(L * Q2), Ha(L * L * Q);
    for (int a = 0; a < L; ++a)
      for (int jk = 0; jk < Q2; ++jk) {
        double acc = 0.0;
        for (int i = 0; i < Q; ++i) acc += B[a * Q + i] * f[i * Q2 + jk];
        H[a * Q2 + jk] = acc;
      }
    for (int a = 0; a < L; ++a)
      for (int b = 0; b < L; ++b)
        for (int k = 0; k < Q; ++k) {
          double acc = 0.0;
          for (int j = 0; j < Q; ++j) acc += B[b * Q + j] * H[a * Q2 + j * Q + k];
          Ha[(a * L + b) * Q + k] = acc;
        }
    for (int ab = 0; ab < L * L; ++ab)
      for (int c = 0; c < L; ++c) {
        double acc = 0.0;
        for (int k = 0; k < Q; ++k) acc += Ha[ab * Q + k] * B[c * Q + k];
        fh[ab * L + c] = acc;
      }
  }
  const double m = 1.0 / E.J;   // DGM_BASIS_NORM mass matrix (src/Hex.cpp:200-205)
  for (int i = 0; i < E.nmodes; ++i) fh[i] *= m;
}

// Modal -> GLL values (src/Quad.cpp:740-764, src/Hex.cpp:795-812)
static void backward_transform(const Elem &E, const double *fh, double *f) {
  const int Q = E.Q, L = E.L;
  const double *B = E.T->B.data();
  if (E.dim == 2) {
    vec wk(Q * L);
    for (int i = 0; i < Q; ++i)
      for (int b = 0; b < L; ++b) {
        double acc = 0.0;
        for (int a = 0; a < L; ++a) acc += B[a * Q + i] * fh[a * L + b];
        wk[i * L + b] = acc;
      }
    for (int i = 0; i < Q; ++i)
      for (int j = 0; j < Q; ++j) {
        double acc = 0.0;
        for (int b = 0; b < L; ++b) acc += wk[i * L + b] * B[b * Q + j];
        f[i * Q + j] = acc;
      }
  } else {
    const int L2 = L * L;
    vec H(Q * L2), Ha(Q * Q * L);
    for (int i = 0; i < Q; ++i)
      for (int bc = 0; bc < L2; ++bc) {
        double acc = 0.0;
        for (int a = 0; a < L; ++a) acc += B[a * Q + i] * fh[a * L2 + bc];
        H[i * L2 + bc] = acc;
      }
    for (int i = 0; i < Q; ++i)
      for (int j = 0; j < Q; ++j)
        for (int c = 0; c < L; ++c) {
          double acc = 0.0;
          for (int b = 0; b < L; ++b) acc += B[b * Q + j] * H[i * L2 + b * L + c];
          Ha[(i * Q + j) * L + c] = acc;
        }
    for (int ij = 0; ij < Q * Q; ++ij)
      for (int k = 0; k < Q; ++k) {
        double acc = 0.0;
        for (int c = 0; c < L; ++c) acc += Ha[ij * L + c] * B[c * Q + k];
        f[ij * Q + k] = acc;
      }
  }
}

// Element::project (src/Element.hpp:427-437)
static void project(const Elem &E, double *x) {
  vec xh(E.nmodes);
  forward_transform(E, x, xh.data());
  backward_transform(E, xh.data(), x);
}

// -----------------------------------------------------------------------------
// Problem: mesh, connectivity, geometry, fields and physics.
// -----------------------------------------------------------------------------
enum Physics { EULER2D = 1, NS2D = 2, EULER3D = 8, NS3D = 9, SHALLOW = 30 };
enum Flux { LAX_FRIEDRICHS = 0, ROE = 1, STEGER_WARMING = 2, VAN_LEER = 3 };

struct Problem {
  int dim = 2, ne = 0, nf = 4, physics = EULER2D, flux = LAX_FRIEDRICHS;
  double gamma = 1.4, vis = 0.0, Pr = 0.72;
  bool sw_balance = true;          // REO_SHALLOW_ENFORCE_BALANCE (src/Shallow.cpp:251)
  bool sw_first = true;
  std::vector<Elem> el;
  size_t ntot = 0, nstot = 0;
  int err = 0;                     // non-physical state seen (density/pressure)
  // work fields: interior [nf][ntot] and sides [nf][nstot]
  vec Us_s, Uf_s, Uv_u, Uv_s, Usrc;
  vec S;                           // source field at the GLL points [nf][ntot] (empty: none)
  double t = 0.0;                  // Domain::t, set per stage by the integrators
  bool pulse = false;              // Shallow::GaussianSource time factor on S
  double pulse_t0 = 0.0, pulse_s2t2i = 0.0;
  vec U, Ut, R0, R1;               // integrator registers
  // boundary sides (src/Boundary.cpp:25-75, src/Field.cpp:4426-4460): the
  // record names the element side, the BC kind and its two parameters; the
  // ghost side gs[b] is the clone that holds the boundary state
  struct BCRec { int e, s, kind; double a, b, v[5]; };   // a, b = v[0], v[1]
  std::vector<BCRec> bcs;
  std::vector<Side> gs;
  bool hold_bulk = false;          // Channel::holdBulkMassFlow (src/Channel.hpp:116-163)
};

// BC kinds: the Euler 3-D slip wall (Euler3d::WallBC, src/Euler3d.cpp:875-903)
// and the Navier-Stokes 3-D isothermal wall (slip-wall state in the inviscid
// flux, Navier_Stokes3d::Isothermal_WallBC in the viscous terms,
// src/Navier_Stokes3d.cpp:472-513)
enum BCKind { BC_SLIP_WALL = 1, BC_ISOTHERMAL_WALL = 2, BC_STATE = 3, BC_SUBSONIC_OUTFLOW = 4,
              BC_SUPERSONIC_OUTFLOW = 5 };

// The side a master side is paired with: the neighbour's side, or for a
// boundary side its ghost clone (src/Field.cpp:4451).
static inline const Side &link(const Problem &P, const Side &S) {
  return S.bc >= 0 ? P.gs[S.bc] : P.el[S.link_e].side[S.link_s];
}

static void elem_setup(Problem &P, Elem &E) {
  const int Q = E.Q;
  E.T = table(E.L, Q);
  E.nmodes = (E.dim == 2) ? E.L * E.L : E.L * E.L * E.L;
  E.qtot = (E.dim == 2) ? Q * Q : Q * Q * Q;
  const vec &z = E.T->z, &w = E.T->w;
  // coordinates of GLL points from vertex (bilinear / trilinear) modes
  // (src/Quad.cpp:996-1020, src/Hex.cpp:990-1029)
  E.cx.assign(E.qtot, 0.0); E.cy.assign(E.qtot, 0.0); E.cz.assign(E.qtot, 0.0);
  if (E.dim == 2) {
    static const int va[4] = {0, 1, 1, 0}, vb[4] = {0, 0, 1, 1};
    for (int n = 0; n < 4; ++n)
      for (int i = 0; i < Q; ++i)
        for (int j = 0; j < Q; ++j) {
          double pa = va[n] ? 0.5 * (1.0 + z[i]) : 0.5 * (1.0 - z[i]);
          double pb = vb[n] ? 0.5 * (1.0 + z[j]) : 0.5 * (1.0 - z[j]);
          double phi = pa * pb;
          E.cx[i * Q + j] += E.X[n][0] * phi;
          E.cy[i * Q + j] += E.X[n][1] * phi;
        }
    // affine geometry (src/Quad.cpp:1227-1285)
    double xr = (E.X[1][0] - E.X[0][0]) * 0.5, xs = (E.X[3][0] - E.X[0][0]) * 0.5;
    double yr = (E.X[1][1] - E.X[0][1]) * 0.5, ys = (E.X[3][1] - E.X[0][1]) * 0.5;
    double detJ = xr * ys - xs * yr;
    if (detJ <= 0.0) throw std::runtime_error("non-positive Jacobian");
    E.J = detJ;
    E.rx = ys / detJ; E.ry = -xs / detJ; E.sx = -yr / detJ; E.sy = xr / detJ;
    E.wJ.assign(E.qtot, detJ);
    for (int j = 0; j < Q; ++j) for (int i = 0; i < Q; ++i) E.wJ[i * Q + j] *= w[i];
    for (int i = 0; i < Q; ++i) for (int j = 0; j < Q; ++j) E.wJ[i * Q + j] *= w[j];
  } else {
    static const int va[8] = {0, 1, 1, 0, 0, 1, 1, 0}, vb[8] = {0, 0, 1, 1, 0, 0, 1, 1},
                     vc[8] = {0, 0, 0, 0, 1, 1, 1, 1};
    for (int n = 0; n < 8; ++n)
      for (int i = 0; i < Q; ++i)
        for (int j = 0; j < Q; ++j)
          for (int k = 0; k < Q; ++k) {
            double pa = va[n] ? 0.5 * (1.0 + z[i]) : 0.5 * (1.0 - z[i]);
            double pb = vb[n] ? 0.5 * (1.0 + z[j]) : 0.5 * (1.0 - z[j]);
            double pc = vc[n] ? 0.5 * (1.0 + z[k]) : 0.5 * (1.0 - z[k]);
            double phi = pa * pb * pc;
            int q = k + j * Q + i * Q * Q;
            E.cx[q] += E.X[n][0] * phi;
            E.cy[q] += E.X[n][1] * phi;
            E.cz[q] += E.X[n][2] * phi;
          }
    // affine geometry (src/Hex.cpp:1130-1280)
    double xr = (E.X[1][0] - E.X[0][0]) * 0.5, xs = (E.X[3][0] - E.X[0][0]) * 0.5, xt = (E.X[4][0] - E.X[0][0]) * 0.5;
    double yr = (E.X[1][1] - E.X[0][1]) * 0.5, ys = (E.X[3][1] - E.X[0][1]) * 0.5, yt = (E.X[4][1] - E.X[0][1]) * 0.5;
    double zr = (E.X[1][2] - E.X[0][2]) * 0.5, zs = (E.X[3][2] - E.X[0][2]) * 0.5, zt = (E.X[4][2] - E.X[0][2]) * 0.5;
    double detJ = xr * ys * zt + yr * zs * xt + zr * xs * yt - xt * ys * zr - zt * xs * yr - xr * zs * yt;
    if (detJ <= 0.0) throw std::runtime_error("non-positive Jacobian");
    E.J = detJ;
    E.rx = (ys * zt - yt * zs) / detJ;  E.ry = -(xs * zt - xt * zs) / detJ; E.rz = (xs * yt - xt * ys) / detJ;
    E.sx = -(yr * zt - yt * zr) / detJ; E.sy = (xr * zt - xt * zr) / detJ;  E.sz = -(xr * yt - xt * yr) / detJ;
    E.tx = (yr * zs - ys * zr) / detJ;  E.ty = -(xr * zs - xs * zr) / detJ; E.tz = (xr * ys - xs * yr) / detJ;
    E.wJ.assign(E.qtot, detJ);
    const int Q2 = Q * Q;
    for (int i = 0; i < Q; ++i) {
      for (int k = 0; k < Q; ++k) for (int j = 0; j < Q; ++j) E.wJ[i * Q2 + j * Q + k] *= w[j];
      for (int j = 0; j < Q; ++j) for (int k = 0; k < Q; ++k) E.wJ[i * Q2 + j * Q + k] *= w[k];
    }
    for (int jk = 0; jk < Q2; ++jk) for (int i = 0; i < Q; ++i) E.wJ[i * Q2 + jk] *= w[i];
  }
}

// Side normals and the side/interior Jacobian ratio (src/Quad.cpp:1367-1455,
// src/Hex.cpp:1385-1497).  Constant metric fields are interpolated exactly as
// the reference does so the Gauss-point values carry the same rounding.
static void side_geometry(Elem &E) {
  const int Q = E.Q;
  const double *D = E.T->D.data();
  for (int s = 0; s < E.nsides; ++s) {
    Side &S = E.side[s];
    S.nx.assign(S.qtot, 0.0); S.ny.assign(S.qtot, 0.0); S.nz.assign(S.qtot, 0.0); S.J.assign(S.qtot, 0.0);
    vec full(E.qtot), wk(Q * Q), ij(S.qtot), tmp(S.qtot);
    if (E.dim == 2) {
      double X = (s == 0 || s == 2) ? E.sx : E.rx;
      double Y = (s == 0 || s == 2) ? E.sy : E.ry;
      std::fill(full.begin(), full.end(), X);
      get_side(E, full.data(), s, wk.data()); interpolate_to_side(E, s, wk.data(), S.nx.data());
      std::fill(full.begin(), full.end(), Y);
      get_side(E, full.data(), s, wk.data()); interpolate_to_side(E, s, wk.data(), S.ny.data());
      if (s == 0 || s == 3) for (int q = 0; q < S.qtot; ++q) { S.nx[q] *= -1.0; S.ny[q] *= -1.0; }
      std::fill(full.begin(), full.end(), E.J);
      get_side(E, full.data(), s, wk.data()); interpolate_to_side(E, s, wk.data(), ij.data());
      for (int q = 0; q < S.qtot; ++q) {
        double len = std::sqrt(S.nx[q] * S.nx[q] + S.ny[q] * S.ny[q]);
        S.nx[q] /= len; S.ny[q] /= len;
      }
      vec x(Q), y(Q), gx(Q), gy(Q), g(Q);
      get_side(E, E.cx.data(), s, x.data());
      get_side(E, E.cy.data(), s, y.data());
      for (int i = 0; i < Q; ++i) {
        double a = 0.0, b = 0.0;
        for (int m = 0; m < Q; ++m) { a += D[i * Q + m] * x[m]; b += D[i * Q + m] * y[m]; }
        gx[i] = a; gy[i] = b;
      }
      for (int i = 0; i < Q; ++i) { gx[i] = gx[i] * gx[i]; gx[i] = gy[i] * gy[i] + gx[i]; g[i] = std::sqrt(gx[i]); }
      interpolate_to_side(E, s, g.data(), S.J.data());
      for (int q = 0; q < S.qtot; ++q) S.J[q] = S.J[q] / ij[q];
    } else {
      double N[3];
      if (s == 0 || s == 5) { N[0] = E.tx; N[1] = E.ty; N[2] = E.tz; }
      else if (s == 1 || s == 3) { N[0] = E.sx; N[1] = E.sy; N[2] = E.sz; }
      else { N[0] = E.rx; N[1] = E.ry; N[2] = E.rz; }
      vec *dst[3] = {&S.nx, &S.ny, &S.nz};
      for (int c = 0; c < 3; ++c) {
        std::fill(full.begin(), full.end(), N[c]);
        get_side(E, full.data(), s, wk.data());
        interpolate_to_side(E, s, wk.data(), dst[c]->data());
      }
      if (s == 0 || s == 1 || s == 4)
        for (int q = 0; q < S.qtot; ++q) { S.nx[q] *= -1.0; S.ny[q] *= -1.0; S.nz[q] *= -1.0; }
      std::fill(full.begin(), full.end(), E.J);
      get_side(E, full.data(), s, wk.data()); interpolate_to_side(E, s, wk.data(), ij.data());
      for (int q = 0; q < S.qtot; ++q) {
        tmp[q] = S.nx[q] * S.nx[q];
        tmp[q] = S.ny[q] * S.ny[q] + tmp[q];
        tmp[q] = S.nz[q] * S.nz[q] + tmp[q];
        tmp[q] = std::sqrt(tmp[q]);
        S.nx[q] = S.nx[q] / tmp[q]; S.ny[q] = S.ny[q] / tmp[q]; S.nz[q] = S.nz[q] / tmp[q];
      }
      const int n = Q * Q;
      vec x(n), y(n), z(n), xr(n), xs(n), yr(n), ys(n), zr(n), zs(n), g(n);
      get_side(E, E.cx.data(), s, x.data());
      get_side(E, E.cy.data(), s, y.data());
      get_side(E, E.cz.data(), s, z.data());
      auto dr = [&](const vec &a, vec &o) {
        for (int i = 0; i < Q; ++i) for (int j = 0; j < Q; ++j) {
          double acc = 0.0; for (int m = 0; m < Q; ++m) acc += D[i * Q + m] * a[m * Q + j];
          o[i * Q + j] = acc; }
      };
      auto ds = [&](const vec &a, vec &o) {
        for (int i = 0; i < Q; ++i) for (int j = 0; j < Q; ++j) {
          double acc = 0.0; for (int m = 0; m < Q; ++m) acc += a[i * Q + m] * D[j * Q + m];
          o[i * Q + j] = acc; }
      };
      dr(x, xr); ds(x, xs); dr(y, yr); ds(y, ys); dr(z, zr); ds(z, zs);
      for (int i = 0; i < n; ++i) {
        double cxv = yr[i] * zs[i]; cxv = cxv - zr[i] * ys[i];
        double cyv = zr[i] * xs[i]; cyv = cyv - xr[i] * zs[i];
        double czv = xr[i] * ys[i]; czv = czv - xs[i] * yr[i];
        double a = cxv * cxv; a = cyv * cyv + a; a = czv * czv + a;
        g[i] = std::sqrt(a);
      }
      interpolate_to_side(E, s, g.data(), S.J.data());
      for (int q = 0; q < S.qtot; ++q) S.J[q] = S.J[q] / ij[q];
    }
  }
}

// 3-D master-side orientation flags (src/Field.cpp:596-680)
static void set_flip3(Problem &P, int e, int s) {
  Side &S = P.el[e].side[s];
  const Elem &A = P.el[e];
  const Elem &B = P.el[S.link_e];
  auto unit = [](const double *p, const double *q, double *o) {
    o[0] = p[0] - q[0]; o[1] = p[1] - q[1]; o[2] = p[2] - q[2];
    double n = std::sqrt(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]);
    o[0] /= n; o[1] /= n; o[2] /= n;
  };
  auto dot = [](const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
  const int *f0 = kHexFaceVerts[s], *f1 = kHexFaceVerts[S.link_s];
  double a0[3], b0[3], a1[3], b1[3], a1p[3];
  unit(A.X[f0[1]], A.X[f0[0]], a0);
  unit(A.X[f0[3]], A.X[f0[0]], b0);
  unit(B.X[f1[1]], B.X[f1[0]], a1);
  unit(B.X[f1[3]], B.X[f1[0]], b1);
  unit(B.X[f1[2]], B.X[f1[3]], a1p);
  S.transp = S.flip_a = S.flip_b = false;
  const double a0a1 = dot(a0, a1), a0a1p = dot(a0, a1p);
  auto near1 = [](double v) { return std::fabs(std::fabs(v) - 1.0) < 1e-8; };
  if (near1(a0a1) || near1(a0a1p)) {
    if (a0a1 < 0) S.flip_a = true;
    if (dot(b0, b1) < 0) S.flip_b = true;
  } else {
    S.transp = true;
    if (dot(b0, a1) < 0) S.flip_a = true;
    if (dot(a0, b1) < 0) S.flip_b = true;
  }
}

static Problem *build(int dim, int ne, const double *verts, const int *porder,
                      const int *qorder, int ncon, const int *con, int physics,
                      int flux, double gamma, double vis, double Pr) {
  auto *P = new Problem();
  P->dim = dim; P->ne = ne; P->physics = physics; P->flux = flux;
  P->gamma = gamma; P->vis = vis; P->Pr = Pr;
  P->nf = (physics == SHALLOW) ? 3 : (dim == 2 ? 4 : 5);
  const int nv = dim == 2 ? 4 : 8;
  P->el.resize(ne);
  for (int e = 0; e < ne; ++e) {
    Elem &E = P->el[e];
    E.dim = dim; E.L = porder[e] + 1; E.Q = qorder[e];
    E.nsides = dim == 2 ? 4 : 6;
    for (int v = 0; v < nv; ++v)
      for (int c = 0; c < 3; ++c) E.X[v][c] = verts[(e * nv + v) * 3 + c];
    for (int s = 0; s < E.nsides; ++s) {
      E.side[s].id = s;
      E.side[s].q1 = E.Q - 1;
      E.side[s].q2 = dim == 2 ? 1 : E.Q - 1;
    }
  }
  // connectivity: first line mentioning a pair makes that side master
  // (src/Field.cpp:3478-3540)
  for (int c = 0; c < ncon; ++c) {
    int e = con[4 * c], s = con[4 * c + 1], le = con[4 * c + 2], ls = con[4 * c + 3];
    Side &nb = P->el[le].side[ls];
    if (nb.master) continue;   // link already set from the other direction
    Side &me = P->el[e].side[s];
    me.master = true; me.link_e = le; me.link_s = ls;
    nb.master = false; nb.link_e = e; nb.link_s = s;
  }
  // side quadrature matching (src/Side.cpp:106-117)
  for (int e = 0; e < ne; ++e)
    for (int s = 0; s < P->el[e].nsides; ++s) {
      Side &S = P->el[e].side[s];
      if (!S.master) continue;
      Side &R = P->el[S.link_e].side[S.link_s];
      S.q1 = R.q1 = std::max(S.q1, R.q1);
      S.q2 = R.q2 = std::max(S.q2, R.q2);
    }
  size_t off = 0, soff = 0;
  for (int e = 0; e < ne; ++e) {
    Elem &E = P->el[e];
    elem_setup(*P, E);
    E.off = off; off += E.qtot;
    for (int s = 0; s < E.nsides; ++s) {
      Side &S = E.side[s];
      S.qtot = S.q1 * S.q2;
      S.off = soff; soff += S.qtot;
      S.to1 = interp(0, S.q1, E.Q);
      S.from1 = interp(1, E.Q, S.q1);
      if (dim == 3) { S.to2 = interp(0, S.q2, E.Q); S.from2 = interp(1, E.Q, S.q2); }
    }
  }
  P->ntot = off; P->nstot = soff;
  for (int e = 0; e < ne; ++e)
    for (int s = 0; s < P->el[e].nsides; ++s) {
      Side &S = P->el[e].side[s];
      if (!S.master) continue;
      if (dim == 2) S.flip_a = kQuadFlip[s][S.link_s] != 0;
      else set_flip3(*P, e, s);
    }
  for (int e = 0; e < ne; ++e) side_geometry(P->el[e]);
  const size_t nf = P->nf;
  P->Us_s.assign(nf * P->nstot, 0.0); P->Uf_s.assign(nf * P->nstot, 0.0);
  P->Uv_u.assign(nf * P->ntot, 0.0);  P->Uv_s.assign(nf * P->nstot, 0.0);
  P->U.assign(nf * P->ntot, 0.0); P->Ut.assign(nf * P->ntot, 0.0);
  P->R0.assign(nf * P->ntot, 0.0); P->R1.assign(nf * P->ntot, 0.0);
  return P;
}

// ---------------------------------------------------------------- helpers
static inline double *fld(Problem &P, vec &v, int n) { return v.data() + (size_t)n * P.ntot; }
static inline double *sfld(Problem &P, vec &v, int n) { return v.data() + (size_t)n * P.nstot; }

static void fill_all_sides(Problem &P, double *Ubase) {
  const int nf = P.nf;
#pragma omp parallel for schedule(static)
  for (int e = 0; e < P.ne; ++e)
    for (int n = 0; n < nf; ++n) {
      const Elem &E = P.el[e];
      fill_sides(E, Ubase + (size_t)n * P.ntot + E.off, sfld(P, P.Us_s, n));
    }
}

static void lift_all(Problem &P, double *Fbase, int nfirst) {
#pragma omp parallel for schedule(static)
  for (int e = 0; e < P.ne; ++e)
    for (int n = nfirst; n < P.nf; ++n) {
      const Elem &E = P.el[e];
      lift(E, sfld(P, P.Uf_s, n), sfld(P, P.Us_s, n), Fbase + (size_t)n * P.ntot + E.off, 0);
    }
}

// Boundary states on the ghost sides from the element sides' traces
// (Domain::enforce_bc looping BC::apply).  Navier_Stokes3d keeps a second BC
// database beside the Domain's (src/Navier_Stokes3d.hpp:83): the inviscid
// flux calls Euler3d::enforce_bc (src/Euler3d.cpp:476), which reads the
// Domain's database where every "*wall*" code is Euler3d::WallBC
// (src/Euler3d.cpp:862-866), while the viscous terms call
// Navier_Stokes3d::enforce_bc (src/Navier_Stokes3d.cpp:192, :457-461) and see
// the isothermal wall.  So in 3-D `viscous` selects the database.  The 2-D
// inviscid flux calls the virtual enforce_bc (src/Euler.cpp:313-316, no
// USE_EULER_BC in any build), so Navier-Stokes 2-D walls are isothermal in
// both phases and Euler 2-D walls are Euler::WallBC (src/EulerBC.hpp:43-62):
//   slip wall       B = (r, m - (m.n) n, rE - |m|^2/2r + |m_t|^2/2r)
//                   (src/Euler3d.cpp:875-903)
//   isothermal wall B = (r, 0, 0, 0, (Eref - 1/2) r Tw)
//                   (src/Navier_Stokes3d.cpp:472-494; a = Tw, b = Eref)
// and in every database: the fixed state B = v (StateBC), and in 2-D the
// outflows (B = S; or the pressure set from Mach Mref = v[0]).
static void enforce_bc(Problem &P, bool viscous) {
  for (size_t b = 0; b < P.bcs.size(); ++b) {
    const Problem::BCRec &R = P.bcs[b];
    const Side &S = P.el[R.e].side[R.s];
    const Side &G = P.gs[b];
    double *s[5], *g[5];
    for (int n = 0; n < P.nf; ++n) { s[n] = sfld(P, P.Us_s, n) + S.off; g[n] = sfld(P, P.Us_s, n) + G.off; }
    for (int i = 0; i < S.qtot; ++i) {
      if (P.physics == SHALLOW) {              // Shallow::WallBC, src/ShallowBC.hpp:45-61
        const double nx = S.nx[i], ny = S.ny[i];
        g[0][i] = s[0][i];
        g[1][i] = (s[1][i] * ny - s[2][i] * nx) * ny;
        g[2][i] = (s[2][i] * nx - s[1][i] * ny) * nx;
      } else if (R.kind == BC_STATE) {                // StateBC::apply, src/BC.cpp:17-28
        for (int n = 0; n < P.nf; ++n) g[n][i] = R.v[n];
      } else if (R.kind == BC_SUPERSONIC_OUTFLOW) {   // src/EulerBC.hpp:214-241
        for (int n = 0; n < P.nf; ++n) g[n][i] = s[n][i];
      } else if (R.kind == BC_SUBSONIC_OUTFLOW) {     // src/EulerBC.hpp:138-167 (gamma 1.4 fixed)
        const double gam = 1.4, Mref = R.v[0];
        const double Eref = 1.0 / (gam * (gam - 1.0) * std::pow(Mref, 2)) + 0.5;
        const double pref = (gam - 1.0) * (Eref - 0.5 * (1.0 - 0.0));
        const double rl = s[0][i], ml = s[1][i], nl = s[2][i];
        const double ul = ml / rl, vl = nl / rl;
        g[0][i] = rl; g[1][i] = ml; g[2][i] = nl;
        g[3][i] = pref / (gam - 1.0) + 0.5 * (ml * ul + nl * vl);
      } else if (P.dim == 2) {
        if (R.kind == BC_ISOTHERMAL_WALL) {   // src/Navier_StokesBC.hpp:47-65
          g[0][i] = s[0][i];
          g[1][i] = 0.0; g[2][i] = 0.0;
          g[3][i] = (R.b - 0.5) * g[0][i] * R.a;
        } else {                               // src/EulerBC.hpp:43-62
          const double nx = S.nx[i], ny = S.ny[i];
          g[0][i] = s[0][i];
          g[1][i] = (s[1][i] * ny - s[2][i] * nx) * ny;
          g[2][i] = (s[2][i] * nx - s[1][i] * ny) * nx;
          g[3][i] = s[3][i] - 0.5 * (s[1][i] * s[1][i] + s[2][i] * s[2][i]) / s[0][i] +
                    0.5 * (g[1][i] * g[1][i] + g[2][i] * g[2][i]) / g[0][i];
        }
      } else if (viscous && R.kind == BC_ISOTHERMAL_WALL) {
        g[0][i] = s[0][i];
        g[1][i] = 0.0; g[2][i] = 0.0; g[3][i] = 0.0;
        g[4][i] = (R.b - 0.5) * g[0][i] * R.a;
      } else {
        double up = s[1][i], vp = s[2][i], wp = s[3][i];
        const double dot = up * S.nx[i] + vp * S.ny[i] + wp * S.nz[i];
        up = up - dot * S.nx[i]; vp = vp - dot * S.ny[i]; wp = wp - dot * S.nz[i];
        g[0][i] = s[0][i]; g[1][i] = up; g[2][i] = vp; g[3][i] = wp;
        g[4][i] = s[4][i] - 0.5 * (s[1][i] * s[1][i] + s[2][i] * s[2][i] + s[3][i] * s[3][i]) / s[0][i] +
                  0.5 * (g[1][i] * g[1][i] + g[2][i] * g[2][i] + g[3][i] * g[3][i]) / g[0][i];
      }
    }
  }
}

// Boundary viscous fluxes (Domain::enforce_flux_bc, BC::apply_flux): the
// isothermal wall mirrors every field, B = -S, so that average_flux('-')
// returns the element's own viscous flux (src/Navier_Stokes3d.cpp:496-513).
static void enforce_flux_bc(Problem &P) {
  for (size_t b = 0; b < P.bcs.size(); ++b) {
    const Problem::BCRec &R = P.bcs[b];
    const Side &S = P.el[R.e].side[R.s];
    const Side &G = P.gs[b];
    for (int n = 0; n < P.nf; ++n) {
      const double *s = sfld(P, P.Us_s, n) + S.off;
      double *g = sfld(P, P.Us_s, n) + G.off;
      for (int i = 0; i < S.qtot; ++i) g[i] = -s[i];
    }
  }
}

// Channel::holdBulkMassFlow (src/Channel.hpp:116-163): subtract the volume
// mean of the density, x-momentum and energy rates from every point.
static void hold_bulk_mass_flow(Problem &P, double *Fb) {
  double sum[5] = {0, 0, 0, 0, 0}, vol = 0.0;
  for (int e = 0; e < P.ne; ++e) {
    const Elem &E = P.el[e];
    double lvol = 0.0;
    for (int i = 0; i < E.qtot; ++i) lvol += E.wJ[i];
    for (int n = 0; n < 5; ++n) {
      const double *f = Fb + (size_t)n * P.ntot + E.off;
      double acc = 0.0;
      for (int i = 0; i < E.qtot; ++i) acc += E.wJ[i] * f[i];
      sum[n] += acc;
    }
    vol += lvol;
  }
  const int held[3] = {0, 1, 4};
  for (int h = 0; h < 3; ++h) {
    const int n = held[h];
    const double m = sum[n] / vol;
    double *f = Fb + (size_t)n * P.ntot;
    for (size_t i = 0; i < P.ntot; ++i) f[i] -= m;
  }
}

// positivity threshold aepsM = eps^(2/3) (src/Constants.hpp:27, :43)
static const double kAeps = std::pow(2.220446049250313e-16, 0.6666666666666666667);
static void report_bad(Problem &P) { P.err = 1; }

// ------------------------------------------------------------ Euler 2-D flux
// src/Euler.cpp:399-757 (LF, Steger-Warming, van Leer, Roe)
static void euler2d_flux(Problem &P) {
  const double gamma = P.gamma, gm1 = gamma - 1.0;
#pragma omp parallel for schedule(static)
  for (int e = 0; e < P.ne; ++e) {
    const Elem &E = P.el[e];
    for (int i = 0; i < 4; ++i) {
      const Side &S = E.side[i];
      if (!S.master) continue;
      const Side &SR = link(P, S);
      double *sl[4], *sr[4], *fl[4], *fr[4];
      for (int n = 0; n < 4; ++n) {
        sl[n] = sfld(P, P.Us_s, n) + S.off;  sr[n] = sfld(P, P.Us_s, n) + SR.off;
        fl[n] = sfld(P, P.Uf_s, n) + S.off;  fr[n] = sfld(P, P.Uf_s, n) + SR.off;
      }
      for (int q = 0; q < S.qtot; ++q) {
        const int ql = side_map(2, S, q), qr = side_map(2, SR, q);
        const double nxl = S.nx[ql], nyl = S.ny[ql];
        double Ul[4], Ur[4], Fpl[4], Fmr[4], Fh[4], Gh[4], lam[4], alpha[4];
        for (int n = 0; n < 4; ++n) Ul[n] = sl[n][ql];
        double rl = Ul[0], rul = Ul[1] * nxl + Ul[2] * nyl, rvl = Ul[2] * nxl - Ul[1] * nyl, rEl = Ul[3];
        const double irl = 1.0 / rl;
        double ul = irl * rul, vl = irl * rvl;
        double pl = gm1 * (rEl - 0.5 * (rul * ul + rvl * vl));
        double Hl = irl * (rEl + pl);
        if (rl < kAeps || pl < kAeps) report_bad(P);
        sl[0][ql] = Fpl[0] = rul;
        sl[1][ql] = Fpl[1] = (rul * ul + pl) * nxl - (rvl * ul) * nyl;
        sl[2][ql] = Fpl[2] = (rul * ul + pl) * nyl + (rvl * ul) * nxl;
        sl[3][ql] = Fpl[3] = ul * (rEl + pl);
        for (int n = 0; n < 4; ++n) Ur[n] = sr[n][qr];
        double rr = Ur[0], rur = Ur[1] * nxl + Ur[2] * nyl, rvr = Ur[2] * nxl - Ur[1] * nyl, rEr = Ur[3];
        const double irr = 1.0 / rr;
        double ur = irr * rur, vr = irr * rvr;
        double pr = gm1 * (rEr - 0.5 * (rur * ur + rvr * vr));
        double Hr = irr * (rEr + pr);
        if (rr < kAeps || pr < kAeps) report_bad(P);
        sr[0][qr] = Fmr[0] = rr * ur;
        sr[1][qr] = Fmr[1] = (rur * ur + pr) * nxl - (rvr * ur) * nyl;
        sr[2][qr] = Fmr[2] = (rur * ur + pr) * nyl + (rvr * ur) * nxl;
        sr[3][qr] = Fmr[3] = ur * (rEr + pr);
        switch (P.flux) {
          case LAX_FRIEDRICHS: {
            double lmax = 0.0;
            const double al = std::sqrt(gm1 * (Hl - 0.5 * (ul * ul + vl * vl)));
            lam[0] = ul - al; lam[1] = ul; lam[2] = ul; lam[3] = ul + al;
            for (int n = 0; n < 4; ++n) lmax = std::max(lmax, std::fabs(lam[n]));
            const double ar = std::sqrt(gm1 * (Hr - 0.5 * (ur * ur + vr * vr)));
            lam[0] = ur - ar; lam[1] = ur; lam[2] = ur; lam[3] = ur + ar;
            for (int n = 0; n < 4; ++n) lmax = std::max(lmax, std::fabs(lam[n]));
            for (int n = 0; n < 4; ++n) Fh[n] = 0.5 * (Fpl[n] + Fmr[n] + lmax * (Ul[n] - Ur[n]));
            break;
          }
          case STEGER_WARMING: {
            {
              const double r = rl, u = ul, v = vl, H = Hl;
              const double a = std::sqrt((gamma - 1.0) * (H - 0.5 * (u * u + v * v)));
              lam[0] = std::max(u - a, 0.0); lam[1] = std::max(u, 0.0); lam[2] = std::max(u, 0.0); lam[3] = std::max(u + a, 0.0);
              const double c1 = 0.5 * r / gamma, c2 = 2.0 * (gamma - 1.0);
              Fpl[0] = c1 * (lam[0] + c2 * lam[1] + lam[3]);
              Fpl[1] = c1 * ((u - a) * lam[0] + c2 * u * lam[1] + (u + a) * lam[3]);
              Fpl[2] = c1 * (v * lam[0] + c2 * v * lam[1] + v * lam[3]);
              Fpl[3] = c1 * ((H - u * a) * lam[0] + (gamma - 1.0) * (u * u + v * v) * lam[1] + (H + u * a) * lam[3]);
            }
            {
              const double r = rr, u = ur, v = vr, H = Hr;
              const double a = std::sqrt((gamma - 1.0) * (H - 0.5 * (u * u + v * v)));
              lam[0] = std::min(u - a, 0.0); lam[1] = std::min(u, 0.0); lam[2] = std::min(u, 0.0); lam[3] = std::min(u + a, 0.0);
              const double c1 = 0.5 * r / gamma, c2 = 2.0 * (gamma - 1.0);
              Fmr[0] = c1 * (lam[0] + c2 * lam[1] + lam[3]);
              Fmr[1] = c1 * ((u - a) * lam[0] + c2 * u * lam[1] + (u + a) * lam[3]);
              Fmr[2] = c1 * (v * lam[0] + c2 * v * lam[1] + v * lam[3]);
              Fmr[3] = c1 * ((H - u * a) * lam[0] + (gamma - 1.0) * (u * u + v * v) * lam[1] + (H + u * a) * lam[3]);
            }
            for (int n = 0; n < 4; ++n) Gh[n] = Fpl[n] + Fmr[n];
            Fh[0] = Gh[0]; Fh[1] = Gh[1] * nxl - Gh[2] * nyl; Fh[2] = Gh[1] * nyl + Gh[2] * nxl; Fh[3] = Gh[3];
            break;
          }
          case VAN_LEER: {
            const double al = std::sqrt((gamma - 1.0) * (Hl - 0.5 * (ul * ul + vl * vl)));
            const double Ml = ul / al;
            const double c1l = 0.25 * rl * al * (1.0 + Ml) * (1.0 + Ml);
            const double c2l = 0.5 * (gamma - 1.0) * Ml + 1.0;
            const double ig = 1.0 / gamma;
            Fpl[0] = c1l; Fpl[1] = c1l * 2.0 * al * ig * c2l; Fpl[2] = c1l * vl;
            Fpl[3] = c1l * (2.0 * al * al / (gamma * gamma - 1.0) * c2l * c2l + 0.5 * vl * vl);
            const double ar = std::sqrt((gamma - 1.0) * (Hr - 0.5 * (ur * ur + vr * vr)));
            const double Mr = ur / ar;
            const double c1r = -0.25 * rr * ar * (1.0 - Mr) * (1.0 - Mr);
            const double c2r = 0.5 * (gamma - 1.0) * Mr - 1.0;
            Fmr[0] = c1r; Fmr[1] = c1r * 2.0 * ar / gamma * c2r; Fmr[2] = c1r * vr;
            Fmr[3] = c1r * (2.0 * ar * ar / (gamma * gamma - 1.0) * c2r * c2r + 0.5 * vr * vr);
            for (int n = 0; n < 4; ++n) Gh[n] = Fpl[n] + Fmr[n];
            Fh[0] = Gh[0]; Fh[1] = Gh[1] * nxl - Gh[2] * nyl; Fh[2] = Gh[1] * nyl + Gh[2] * nxl; Fh[3] = Gh[3];
            break;
          }
          case ROE: default: {
            const double R = std::sqrt(rr / rl);
            const double iRp1 = 1.0 / (1.0 + R);
            const double u = (ul + R * ur) * iRp1, v = (vl + R * vr) * iRp1, H = (Hl + R * Hr) * iRp1;
            const double a2 = gm1 * (H - 0.5 * (u * u + v * v));
            const double a = std::sqrt(a2), ainv = 1.0 / a;
            const double c1 = gm1 * ainv * ainv, c1inv = 1.0 / c1;
            alpha[2] = (rvr - rvl) - v * (rr - rl);
            alpha[1] = (gamma - 1.0) * ainv * ainv * ((rr - rl) * (H - u * u) + u * (rur - rul) -
                                                      ((rEr - rEl) - ((rvr - rvl) - v * (rr - rl)) * v));
            alpha[0] = 0.5 * ainv * ((rr - rl) * (u + a) - (rur - rul) - a * alpha[1]);
            alpha[3] = (rr - rl) - (alpha[0] + alpha[1]);
            lam[0] = std::min(u - a, 0.0); lam[1] = std::min(u, 0.0); lam[2] = std::min(u, 0.0); lam[3] = std::min(u + a, 0.0);
            Gh[0] = lam[0] * alpha[0]; Gh[1] = lam[0] * (u - a) * alpha[0];
            Gh[2] = lam[0] * v * alpha[0]; Gh[3] = lam[0] * (H - u * a) * alpha[0];
            Gh[0] += lam[1] * alpha[1]; Gh[1] += lam[1] * u * alpha[1];
            Gh[2] += lam[1] * v * alpha[1]; Gh[3] += lam[1] * (H - c1inv) * alpha[1];
            Gh[2] += lam[2] * alpha[2]; Gh[3] += lam[2] * v * alpha[2];
            Gh[0] += lam[3] * alpha[3]; Gh[1] += lam[3] * (u + a) * alpha[3];
            Gh[2] += lam[3] * v * alpha[3]; Gh[3] += lam[3] * (H + u * a) * alpha[3];
            Fh[0] = Fpl[0] + Gh[0];
            Fh[1] = Fpl[1] + Gh[1] * nxl - Gh[2] * nyl;
            Fh[2] = Fpl[2] + Gh[1] * nyl + Gh[2] * nxl;
            Fh[3] = Fpl[3] + Gh[3];
            break;
          }
        }
        for (int n = 0; n < 4; ++n) {
          sr[n][qr] *= -1.0;
          fl[n][ql] = Fh[n];
          fr[n][qr] = -Fh[n];
        }
      }
    }
  }
}

// Roe flux in a rotated (n,s,t) frame: the 3-D extension of the 2-D Roe
// average (src/Euler.cpp:682-741).  The reference's Euler3d has no Roe
// branch (src/Euler3d.cpp:803-805); this is checked against the 2-D Roe by a
// quasi-2-D test.
static void roe3(double gamma, const double *Ln, const double *Rn, double *G) {
  // Ln/Rn: rho, rho un, rho us, rho ut, rhoE in the rotated frame
  const double gm1 = gamma - 1.0;
  const double rl = Ln[0], rr = Rn[0];
  const double ul = Ln[1] / rl, vl = Ln[2] / rl, wl = Ln[3] / rl;
  const double ur = Rn[1] / rr, vr = Rn[2] / rr, wr = Rn[3] / rr;
  const double pl = gm1 * (Ln[4] - 0.5 * (Ln[1] * ul + Ln[2] * vl + Ln[3] * wl));
  const double pr = gm1 * (Rn[4] - 0.5 * (Rn[1] * ur + Rn[2] * vr + Rn[3] * wr));
  const double Hl = (Ln[4] + pl) / rl, Hr = (Rn[4] + pr) / rr;
  const double R = std::sqrt(rr / rl), iRp1 = 1.0 / (1.0 + R);
  const double u = (ul + R * ur) * iRp1, v = (vl + R * vr) * iRp1, w = (wl + R * wr) * iRp1;
  const double H = (Hl + R * Hr) * iRp1;
  const double a2 = gm1 * (H - 0.5 * (u * u + v * v + w * w));
  const double a = std::sqrt(a2), ainv = 1.0 / a;
  const double c1inv = a2 / gm1;
  const double dr = rr - rl, dru = Rn[1] - Ln[1], drv = Rn[2] - Ln[2], drw = Rn[3] - Ln[3], drE = Rn[4] - Ln[4];
  double al[5];
  al[2] = drv - v * dr;
  al[3] = drw - w * dr;
  al[1] = gm1 * ainv * ainv * (dr * (H - u * u) + u * dru - ((drE - al[2] * v - al[3] * w)));
  al[0] = 0.5 * ainv * (dr * (u + a) - dru - a * al[1]);
  al[4] = dr - (al[0] + al[1]);
  const double lam0 = std::min(u - a, 0.0), lam1 = std::min(u, 0.0), lam4 = std::min(u + a, 0.0);
  G[0] = lam0 * al[0]; G[1] = lam0 * (u - a) * al[0]; G[2] = lam0 * v * al[0]; G[3] = lam0 * w * al[0];
  G[4] = lam0 * (H - u * a) * al[0];
  G[0] += lam1 * al[1]; G[1] += lam1 * u * al[1]; G[2] += lam1 * v * al[1]; G[3] += lam1 * w * al[1];
  G[4] += lam1 * (H - c1inv) * al[1];
  G[2] += lam1 * al[2]; G[4] += lam1 * v * al[2];
  G[3] += lam1 * al[3]; G[4] += lam1 * w * al[3];
  G[0] += lam4 * al[4]; G[1] += lam4 * (u + a) * al[4]; G[2] += lam4 * v * al[4]; G[3] += lam4 * w * al[4];
  G[4] += lam4 * (H + u * a) * al[4];
}

// ------------------------------------------------------------ Euler 3-D flux
// src/Euler3d.cpp:584-817 (LF); Roe is the extension above.
static void euler3d_flux(Problem &P) {
  const double gm1 = P.gamma - 1.0;
#pragma omp parallel for schedule(static)
  for (int e = 0; e < P.ne; ++e) {
    const Elem &E = P.el[e];
    for (int i = 0; i < 6; ++i) {
      const Side &S = E.side[i];
      if (!S.master) continue;
      const Side &SR = link(P, S);
      double *sl[5], *sr[5], *fl[5], *fr[5];
      for (int n = 0; n < 5; ++n) {
        sl[n] = sfld(P, P.Us_s, n) + S.off;  sr[n] = sfld(P, P.Us_s, n) + SR.off;
        fl[n] = sfld(P, P.Uf_s, n) + S.off;  fr[n] = sfld(P, P.Uf_s, n) + SR.off;
      }
      for (int q = 0; q < S.qtot; ++q) {
        const int ql = side_map(3, S, q), qr = side_map(3, SR, q);
        const double nx = S.nx[ql], ny = S.ny[ql], nz = S.nz[ql];
        double sx = ny, sy = nz, sz = nx;
        const double sdn = nx * sx + ny * sy + nz * sz;
        sx -= sdn * nx; sy -= sdn * ny; sz -= sdn * nz;
        const double sni = 1.0 / std::sqrt(sx * sx + sy * sy + sz * sz);
        sx *= sni; sy *= sni; sz *= sni;
        double tx = ny * sz - sy * nz, ty = nz * sx - sz * nx, tz = nx * sy - sx * ny;
        const double tni = 1.0 / std::sqrt(tx * tx + ty * ty + tz * tz);
        tx *= tni; ty *= tni; tz *= tni;
        const double detA = (nx * sy * tz + sx * ty * nz + tx * sz * ny) - (nz * sy * tx + sz * ty * nx + tz * sx * ny);
        const double idetA = 1.0 / detA;
        const double xn = (sy * tz - sz * ty) * idetA, yn = -(sx * tz - sz * tx) * idetA, zn = (sx * ty - sy * tx) * idetA;
        const double xs = -(ny * tz - nz * ty) * idetA, ys = (nx * tz - nz * tx) * idetA, zs = -(nx * ty - ny * tx) * idetA;
        const double xt = (ny * sz - nz * sy) * idetA, yt = -(nx * sz - nz * sx) * idetA, zt = (nx * sy - ny * sx) * idetA;
        double Ul[5], Ur[5], Fpl[5], Fmr[5], Fh[5], lam[5];
        for (int n = 0; n < 5; ++n) Ul[n] = sl[n][ql];
        double rl = Ul[0];
        double rul = Ul[1] * nx + Ul[2] * ny + Ul[3] * nz;
        double rvl = Ul[1] * sx + Ul[2] * sy + Ul[3] * sz;
        double rwl = Ul[1] * tx + Ul[2] * ty + Ul[3] * tz;
        double rEl = Ul[4];
        const double irl = 1.0 / rl;
        double ul = irl * rul, vl = irl * rvl, wl = irl * rwl;
        double pl = gm1 * (rEl - 0.5 * (rul * ul + rvl * vl + rwl * wl));
        double Hl = irl * (rEl + pl);
        if (rl < kAeps || pl < kAeps) report_bad(P);
        sl[0][ql] = Fpl[0] = rl * ul;
        sl[1][ql] = Fpl[1] = (rul * ul + pl) * xn + (rvl * ul) * xs + (rwl * ul) * xt;
        sl[2][ql] = Fpl[2] = (rul * ul + pl) * yn + (rvl * ul) * ys + (rwl * ul) * yt;
        sl[3][ql] = Fpl[3] = (rul * ul + pl) * zn + (rvl * ul) * zs + (rwl * ul) * zt;
        sl[4][ql] = Fpl[4] = ul * (rEl + pl);
        for (int n = 0; n < 5; ++n) Ur[n] = sr[n][qr];
        double rr = Ur[0];
        double rur = Ur[1] * nx + Ur[2] * ny + Ur[3] * nz;
        double rvr = Ur[1] * sx + Ur[2] * sy + Ur[3] * sz;
        double rwr = Ur[1] * tx + Ur[2] * ty + Ur[3] * tz;
        double rEr = Ur[4];
        const double irr = 1.0 / rr;
        double ur = irr * rur, vr = irr * rvr, wr = irr * rwr;
        double pr = gm1 * (rEr - 0.5 * (rur * ur + rvr * vr + rwr * wr));
        double Hr = irr * (rEr + pr);
        if (rr < kAeps || pr < kAeps) report_bad(P);
        sr[0][qr] = Fmr[0] = rr * ur;
        sr[1][qr] = Fmr[1] = (rur * ur + pr) * xn + (rvr * ur) * xs + (rwr * ur) * xt;
        sr[2][qr] = Fmr[2] = (rur * ur + pr) * yn + (rvr * ur) * ys + (rwr * ur) * yt;
        sr[3][qr] = Fmr[3] = (rur * ur + pr) * zn + (rvr * ur) * zs + (rwr * ur) * zt;
        sr[4][qr] = Fmr[4] = ur * (rEr + pr);
        if (P.flux == ROE) {
          const double Ln[5] = {rl, rul, rvl, rwl, rEl}, Rn[5] = {rr, rur, rvr, rwr, rEr};
          double G[5];
          roe3(P.gamma, Ln, Rn, G);
          const double Gn = G[1], Gs = G[2], Gt = G[3];
          Fh[0] = Fpl[0] + G[0];
          Fh[1] = Fpl[1] + Gn * xn + Gs * xs + Gt * xt;
          Fh[2] = Fpl[2] + Gn * yn + Gs * ys + Gt * yt;
          Fh[3] = Fpl[3] + Gn * zn + Gs * zs + Gt * zt;
          Fh[4] = Fpl[4] + G[4];
        } else {
          double lmax = 0.0;
          const double al = std::sqrt(gm1 * (Hl - 0.5 * (ul * ul + vl * vl + wl * wl)));
          lam[0] = ul - al; lam[1] = ul; lam[2] = ul; lam[3] = ul; lam[4] = ul + al;
          for (int n = 0; n < 5; ++n) lmax = std::max(lmax, std::fabs(lam[n]));
          const double ar = std::sqrt(gm1 * (Hr - 0.5 * (ur * ur + vr * vr + wr * wr)));
          lam[0] = ur - ar; lam[1] = ur; lam[2] = ur; lam[3] = ur; lam[4] = ur + ar;
          for (int n = 0; n < 5; ++n) lmax = std::max(lmax, std::fabs(lam[n]));
          for (int n = 0; n < 5; ++n) Fh[n] = 0.5 * (Fpl[n] + Fmr[n] + lmax * (Ul[n] - Ur[n]));
        }
        for (int n = 0; n < 5; ++n) {
          sr[n][qr] *= -1.0;
          fl[n][ql] = Fh[n];
          fr[n][qr] = -Fh[n];
        }
      }
    }
  }
}

// ------------------------------------------------------- shallow water flux
// src/Shallow.cpp:357-534
static void shallow_flux(Problem &P) {
#pragma omp parallel for schedule(static)
  for (int e = 0; e < P.ne; ++e) {
    const Elem &E = P.el[e];
    for (int i = 0; i < 4; ++i) {
      const Side &S = E.side[i];
      if (!S.master) continue;
      const Side &SR = link(P, S);
      double *sl[3], *sr[3], *fl[3], *fr[3];
      for (int n = 0; n < 3; ++n) {
        sl[n] = sfld(P, P.Us_s, n) + S.off;  sr[n] = sfld(P, P.Us_s, n) + SR.off;
        fl[n] = sfld(P, P.Uf_s, n) + S.off;  fr[n] = sfld(P, P.Uf_s, n) + SR.off;
      }
      for (int q = 0; q < S.qtot; ++q) {
        const int ql = side_map(2, S, q), qr = side_map(2, SR, q);
        const double nxl = S.nx[ql], nyl = S.ny[ql];
        double Ul[3], Ur[3], Fpl[3], Fmr[3], Fh[3], lam[3];
        for (int n = 0; n < 3; ++n) Ul[n] = sl[n][ql];
        double phil = Ul[0], uphil = Ul[1] * nxl + Ul[2] * nyl, vphil = Ul[2] * nxl - Ul[1] * nyl;
        const double iphil = 1.0 / phil;
        double ul = iphil * uphil, pl = 0.5 * phil * phil;
        if (phil < kAeps || pl < kAeps) report_bad(P);
        sl[0][ql] = Fpl[0] = uphil;
        sl[1][ql] = Fpl[1] = (uphil * ul + pl) * nxl - (vphil * ul) * nyl;
        sl[2][ql] = Fpl[2] = (uphil * ul + pl) * nyl + (vphil * ul) * nxl;
        for (int n = 0; n < 3; ++n) Ur[n] = sr[n][qr];
        double phir = Ur[0], uphir = Ur[1] * nxl + Ur[2] * nyl, vphir = Ur[2] * nxl - Ur[1] * nyl;
        const double iphir = 1.0 / phir;
        double ur = iphir * uphir, pr = 0.5 * phir * phir;
        if (phir < kAeps || pr < kAeps) report_bad(P);
        sr[0][qr] = Fmr[0] = uphir;
        sr[1][qr] = Fmr[1] = (uphir * ur + pr) * nxl - (vphir * ur) * nyl;
        sr[2][qr] = Fmr[2] = (uphir * ur + pr) * nyl + (vphir * ur) * nxl;
        double lmax = 0.0;
        const double al = std::sqrt(phil);
        lam[0] = ul - al; lam[1] = ul; lam[2] = ul + al;
        for (int n = 0; n < 3; ++n) lmax = std::max(lmax, std::fabs(lam[n]));
        const double ar = std::sqrt(phir);
        lam[0] = ur - ar; lam[1] = ur; lam[2] = ur + ar;
        for (int n = 0; n < 3; ++n) lmax = std::max(lmax, std::fabs(lam[n]));
        for (int n = 0; n < 3; ++n) Fh[n] = 0.5 * (Fpl[n] + Fmr[n] + lmax * (Ul[n] - Ur[n]));
        for (int n = 0; n < 3; ++n) {
          sr[n][qr] *= -1.0;
          fl[n][ql] = Fh[n];
          fr[n][qr] = -Fh[n];
        }
      }
    }
  }
}

// ---------------------------------------------------- convection (volume)
// Euler 2-D: src/Euler.cpp:296-390
static void euler2d_volume(Problem &P, const double *Ub, double *Fb) {
  const double gm1 = P.gamma - 1.0, m5g = -0.5 * gm1;
#pragma omp parallel for schedule(static)
  for (int e = 0; e < P.ne; ++e) {
    const Elem &E = P.el[e];
    const int n = E.qtot;
    const double *r = Ub + E.off, *ru = Ub + P.ntot + E.off, *rv = Ub + 2 * P.ntot + E.off, *rE = Ub + 3 * P.ntot + E.off;
    double *F0 = Fb + E.off, *F1 = Fb + P.ntot + E.off, *F2 = Fb + 2 * P.ntot + E.off, *F3 = Fb + 3 * P.ntot + E.off;
    vec u(n), v(n), p(n), d(n), d1(n);
    for (int i = 0; i < n; ++i) { u[i] = ru[i] / r[i]; v[i] = rv[i] / r[i]; }
    for (int i = 0; i < n; ++i) { p[i] = u[i] * ru[i]; d[i] = v[i] * rv[i]; p[i] = d[i] + p[i]; p[i] = m5g * p[i]; p[i] = gm1 * rE[i] + p[i]; }
    gradient_dir(E, ru, F0, 'x'); gradient_dir(E, rv, d.data(), 'y');
    for (int i = 0; i < n; ++i) F0[i] = d[i] + F0[i];
    for (int i = 0; i < n; ++i) { d[i] = ru[i] * u[i]; d[i] = p[i] + d[i]; }
    gradient_dir(E, d.data(), F1, 'x');
    for (int i = 0; i < n; ++i) d[i] = ru[i] * v[i];
    gradient_dir(E, d.data(), d1.data(), 'y');
    for (int i = 0; i < n; ++i) F1[i] = d1[i] + F1[i];
    for (int i = 0; i < n; ++i) d[i] = rv[i] * u[i];
    gradient_dir(E, d.data(), F2, 'x');
    for (int i = 0; i < n; ++i) { d[i] = rv[i] * v[i]; d[i] = p[i] + d[i]; }
    gradient_dir(E, d.data(), d1.data(), 'y');
    for (int i = 0; i < n; ++i) F2[i] = d1[i] + F2[i];
    for (int i = 0; i < n; ++i) p[i] = rE[i] + p[i];
    for (int i = 0; i < n; ++i) d[i] = u[i] * p[i];
    gradient_dir(E, d.data(), F3, 'x');
    for (int i = 0; i < n; ++i) d[i] = v[i] * p[i];
    gradient_dir(E, d.data(), d1.data(), 'y');
    for (int i = 0; i < n; ++i) F3[i] = d1[i] + F3[i];
  }
}

// Euler 3-D: src/Euler3d.cpp:468-575
static void euler3d_volume(Problem &P, const double *Ub, double *Fb) {
  const double gm1 = P.gamma - 1.0, m5g = -0.5 * gm1;
  const size_t N = P.ntot;
#pragma omp parallel for schedule(static)
  for (int e = 0; e < P.ne; ++e) {
    const Elem &E = P.el[e];
    const int n = E.qtot;
    const double *r = Ub + E.off, *ru = Ub + N + E.off, *rv = Ub + 2 * N + E.off, *rw = Ub + 3 * N + E.off, *rE = Ub + 4 * N + E.off;
    double *F[5];
    for (int k = 0; k < 5; ++k) F[k] = Fb + k * N + E.off;
    vec u(n), v(n), w(n), p(n), d(n), d1(n);
    for (int i = 0; i < n; ++i) { u[i] = ru[i] / r[i]; v[i] = rv[i] / r[i]; w[i] = rw[i] / r[i]; }
    for (int i = 0; i < n; ++i) {
      p[i] = u[i] * ru[i]; p[i] = v[i] * rv[i] + p[i]; p[i] = w[i] * rw[i] + p[i];
      p[i] = m5g * p[i]; p[i] = gm1 * rE[i] + p[i];
    }
    gradient_dir(E, ru, F[0], 'x');
    gradient_dir(E, rv, d.data(), 'y'); for (int i = 0; i < n; ++i) F[0][i] = d[i] + F[0][i];
    gradient_dir(E, rw, d.data(), 'z'); for (int i = 0; i < n; ++i) F[0][i] = d[i] + F[0][i];
    for (int i = 0; i < n; ++i) d[i] = ru[i] * u[i] + p[i];
    gradient_dir(E, d.data(), F[1], 'x');
    for (int i = 0; i < n; ++i) d[i] = ru[i] * v[i];
    gradient_dir(E, d.data(), d1.data(), 'y'); for (int i = 0; i < n; ++i) F[1][i] = d1[i] + F[1][i];
    for (int i = 0; i < n; ++i) d[i] = ru[i] * w[i];
    gradient_dir(E, d.data(), d1.data(), 'z'); for (int i = 0; i < n; ++i) F[1][i] = d1[i] + F[1][i];
    for (int i = 0; i < n; ++i) d[i] = rv[i] * u[i];
    gradient_dir(E, d.data(), F[2], 'x');
    for (int i = 0; i < n; ++i) d[i] = rv[i] * v[i] + p[i];
    gradient_dir(E, d.data(), d1.data(), 'y'); for (int i = 0; i < n; ++i) F[2][i] = d1[i] + F[2][i];
    for (int i = 0; i < n; ++i) d[i] = rv[i] * w[i];
    gradient_dir(E, d.data(), d1.data(), 'z'); for (int i = 0; i < n; ++i) F[2][i] = d1[i] + F[2][i];
    for (int i = 0; i < n; ++i) d[i] = rw[i] * u[i];
    gradient_dir(E, d.data(), F[3], 'x');
    for (int i = 0; i < n; ++i) d[i] = rw[i] * v[i];
    gradient_dir(E, d.data(), d1.data(), 'y'); for (int i = 0; i < n; ++i) F[3][i] = d1[i] + F[3][i];
    for (int i = 0; i < n; ++i) d[i] = rw[i] * w[i] + p[i];
    gradient_dir(E, d.data(), d1.data(), 'z'); for (int i = 0; i < n; ++i) F[3][i] = d1[i] + F[3][i];
    for (int i = 0; i < n; ++i) p[i] = rE[i] + p[i];
    for (int i = 0; i < n; ++i) d[i] = u[i] * p[i];
    gradient_dir(E, d.data(), F[4], 'x');
    for (int i = 0; i < n; ++i) d[i] = v[i] * p[i];
    gradient_dir(E, d.data(), d1.data(), 'y'); for (int i = 0; i < n; ++i) F[4][i] = d1[i] + F[4][i];
    for (int i = 0; i < n; ++i) d[i] = w[i] * p[i];
    gradient_dir(E, d.data(), d1.data(), 'z'); for (int i = 0; i < n; ++i) F[4][i] = d1[i] + F[4][i];
  }
}

// Shallow water: src/Shallow.cpp:276-351
static void shallow_volume(Problem &P, const double *Ub, double *Fb) {
  const size_t N = P.ntot;
#pragma omp parallel for schedule(static)
  for (int e = 0; e < P.ne; ++e) {
    const Elem &E = P.el[e];
    const int n = E.qtot;
    const double *phi = Ub + E.off, *uphi = Ub + N + E.off, *vphi = Ub + 2 * N + E.off;
    double *F0 = Fb + E.off, *F1 = Fb + N + E.off, *F2 = Fb + 2 * N + E.off;
    vec u(n), v(n), p(n), d(n), d1(n);
    for (int i = 0; i < n; ++i) { u[i] = uphi[i] / phi[i]; v[i] = vphi[i] / phi[i]; }
    for (int i = 0; i < n; ++i) { p[i] = phi[i] * phi[i]; p[i] = 0.5 * p[i]; }
    gradient_dir(E, uphi, F0, 'x'); gradient_dir(E, vphi, d.data(), 'y');
    for (int i = 0; i < n; ++i) F0[i] = d[i] + F0[i];
    for (int i = 0; i < n; ++i) d[i] = uphi[i] * u[i] + p[i];
    gradient_dir(E, d.data(), F1, 'x');
    for (int i = 0; i < n; ++i) d[i] = uphi[i] * v[i];
    gradient_dir(E, d.data(), d1.data(), 'y'); for (int i = 0; i < n; ++i) F1[i] = d1[i] + F1[i];
    for (int i = 0; i < n; ++i) d[i] = vphi[i] * u[i];
    gradient_dir(E, d.data(), F2, 'x');
    for (int i = 0; i < n; ++i) d[i] = vphi[i] * v[i] + p[i];
    gradient_dir(E, d.data(), d1.data(), 'y'); for (int i = 0; i < n; ++i) F2[i] = d1[i] + F2[i];
  }
}

// ----------------------------------------------- BR1 viscous terms (NS)
// primitive side values (src/Euler.cpp:1420-1452, src/Euler3d.cpp:1162-1199)
static void primitive_sides(Problem &P) {
  const int nvel = P.dim;
#pragma omp parallel for schedule(static)
  for (int e = 0; e < P.ne; ++e) {
    const Elem &E = P.el[e];
    for (int i = 0; i < E.nsides; ++i) {
      const Side &S = E.side[i];
      if (!S.master) continue;
      const Side &SR = link(P, S);
      for (int pass = 0; pass < 2; ++pass) {
        const Side &X = pass == 0 ? S : SR;
        double *r = sfld(P, P.Us_s, 0) + X.off;
        double *m[3];
        for (int c = 0; c < nvel; ++c) m[c] = sfld(P, P.Us_s, 1 + c) + X.off;
        double *en = sfld(P, P.Us_s, 1 + nvel) + X.off;
        for (int q = 0; q < X.qtot; ++q) {
          for (int c = 0; c < nvel; ++c) m[c][q] = m[c][q] / r[q];
          en[q] = en[q] / r[q];
          double wk = m[0][q] * m[0][q];
          for (int c = 1; c < nvel; ++c) wk = m[c][q] * m[c][q] + wk;
          en[q] = -0.5 * wk + en[q];
        }
      }
    }
  }
}

// average_flux (src/Domain.cpp:1883-1937): F sides = 0.5 (U_l + fact U_r)
static void average_flux(Problem &P, double fact) {
#pragma omp parallel for schedule(static)
  for (int e = 0; e < P.ne; ++e)
    for (int n = 0; n < P.nf; ++n) {
      const Elem &E = P.el[e];
      for (int i = 0; i < E.nsides; ++i) {
        const Side &S = E.side[i];
        if (!S.master) continue;
        const Side &SR = link(P, S);
        double *us = sfld(P, P.Us_s, n), *fs = sfld(P, P.Uv_s, n);
        for (int q = 0; q < S.qtot; ++q) {
          const int ql = side_map(P.dim, S, q), qr = side_map(P.dim, SR, q);
          fs[S.off + ql] = 0.5 * (us[S.off + ql] + fact * us[SR.off + qr]);
          fs[SR.off + qr] = fact * fs[S.off + ql];
        }
      }
    }
}

// lifted, projected gradient (src/Euler.cpp:1406-1417, src/Euler3d.cpp:1144-1159)
static void lifted_gradient(Problem &P, const Elem &E, int n, const double *u,
                            double *gx, double *gy, double *gz) {
  const double *fsb = sfld(P, P.Uv_s, n), *usb = sfld(P, P.Us_s, n);
  gradient_dir(E, u, gx, 'x');
  gradient_dir(E, u, gy, 'y');
  if (E.dim == 3) gradient_dir(E, u, gz, 'z');
  lift(E, fsb, usb, gx, 'x'); project(E, gx);
  lift(E, fsb, usb, gy, 'y'); project(E, gy);
  if (E.dim == 3) { lift(E, fsb, usb, gz, 'z'); project(E, gz); }
}

// Navier-Stokes 2-D diffusion (src/Navier_Stokes.cpp:113-252)
static void ns2d_diffusion(Problem &P, const double *Ub, double *Rb) {
  const size_t N = P.ntot;
  const double gPr = P.gamma / P.Pr, mu = P.vis;
  fill_all_sides(P, const_cast<double *>(Ub));
  if (!P.bcs.empty()) enforce_bc(P, true);   // src/Navier_Stokes.cpp:124-125
  primitive_sides(P);
  average_flux(P, 1.0);
#pragma omp parallel for schedule(static)
  for (int k = 0; k < P.ne; ++k) {
    const Elem &E = P.el[k];
    const int n = E.qtot;
    const double *r = Ub + E.off, *ru = Ub + N + E.off, *rv = Ub + 2 * N + E.off, *rE = Ub + 3 * N + E.off;
    vec u(n), v(n), e(n), wk(n), ux(n), uy(n), vx(n), vy(n), t11(n), t12(n), t22(n);
    for (int i = 0; i < n; ++i) {
      u[i] = ru[i] / r[i]; v[i] = rv[i] / r[i]; e[i] = rE[i] / r[i];
      wk[i] = u[i] * u[i]; wk[i] = v[i] * v[i] + wk[i]; e[i] = -0.5 * wk[i] + e[i];
    }
    lifted_gradient(P, E, 1, u.data(), ux.data(), uy.data(), nullptr);
    lifted_gradient(P, E, 2, v.data(), vx.data(), vy.data(), nullptr);
    for (int i = 0; i < n; ++i) {
      wk[i] = mu;
      t12[i] = uy[i] + vx[i]; t12[i] = wk[i] * t12[i];
      t11[i] = 2.0 * ux[i] - vy[i]; t11[i] = (2.0 / 3.0) * t11[i]; t11[i] = wk[i] * t11[i];
      t22[i] = 2.0 * vy[i] - ux[i]; t22[i] = (2.0 / 3.0) * t22[i]; t22[i] = wk[i] * t22[i];
    }
    double *F1 = P.Uv_u.data() + N + E.off, *F2 = P.Uv_u.data() + 2 * N + E.off, *F3 = P.Uv_u.data() + 3 * N + E.off;
    fill_sides_flux(E, t11.data(), t12.data(), nullptr, sfld(P, P.Us_s, 1));
    gradient_dir(E, t11.data(), ux.data(), 'x'); gradient_dir(E, t12.data(), wk.data(), 'y');
    for (int i = 0; i < n; ++i) F1[i] = ux[i] + wk[i];
    fill_sides_flux(E, t12.data(), t22.data(), nullptr, sfld(P, P.Us_s, 2));
    gradient_dir(E, t12.data(), ux.data(), 'x'); gradient_dir(E, t22.data(), wk.data(), 'y');
    for (int i = 0; i < n; ++i) F2[i] = ux[i] + wk[i];
    for (int i = 0; i < n; ++i) {
      ux[i] = t11[i] * u[i]; ux[i] = t12[i] * v[i] + ux[i];
      uy[i] = t12[i] * u[i]; uy[i] = t22[i] * v[i] + uy[i];
    }
    lifted_gradient(P, E, 3, e.data(), vx.data(), vy.data(), nullptr);
    for (int i = 0; i < n; ++i) {
      wk[i] = mu;
      vx[i] = wk[i] * vx[i]; ux[i] = gPr * vx[i] + ux[i];
      vy[i] = wk[i] * vy[i]; uy[i] = gPr * vy[i] + uy[i];
    }
    fill_sides_flux(E, ux.data(), uy.data(), nullptr, sfld(P, P.Us_s, 3));
    gradient_dir(E, ux.data(), wk.data(), 'x'); gradient_dir(E, uy.data(), ux.data(), 'y');
    for (int i = 0; i < n; ++i) F3[i] = wk[i] + ux[i];
  }
  if (!P.bcs.empty()) enforce_flux_bc(P);
  average_flux(P, -1.0);
#pragma omp parallel for schedule(static)
  for (int k = 0; k < P.ne; ++k)
    for (int n = 1; n < P.nf; ++n) {
      const Elem &E = P.el[k];
      lift(E, sfld(P, P.Uv_s, n), sfld(P, P.Us_s, n), P.Uv_u.data() + n * N + E.off, 0);
    }
  for (int n = 1; n < P.nf; ++n)
    for (size_t i = 0; i < N; ++i) {
      double x = -1.0 * P.Uv_u[n * N + i];
      Rb[n * N + i] = x + Rb[n * N + i];
    }
}

// Navier-Stokes 3-D diffusion (src/Navier_Stokes3d.cpp:182-391, DNS branch)
static void ns3d_diffusion(Problem &P, const double *Ub, double *Rb) {
  const size_t N = P.ntot;
  const double gPr = P.gamma / P.Pr, muv = P.vis;
  fill_all_sides(P, const_cast<double *>(Ub));
  if (!P.bcs.empty()) enforce_bc(P, true);
  primitive_sides(P);
  average_flux(P, 1.0);
#pragma omp parallel for schedule(static)
  for (int k = 0; k < P.ne; ++k) {
    const Elem &E = P.el[k];
    const int n = E.qtot;
    const double *r = Ub + E.off, *ru = Ub + N + E.off, *rv = Ub + 2 * N + E.off, *rw = Ub + 3 * N + E.off, *rE = Ub + 4 * N + E.off;
    vec u(n), v(n), w(n), e(n), mu(n), wk(n);
    vec ux(n), uy(n), uz(n), vx(n), vy(n), vz(n), wx(n), wy(n), wz(n);
    vec t11(n), t12(n), t13(n), t22(n), t23(n), t33(n);
    for (int i = 0; i < n; ++i) {
      u[i] = ru[i] / r[i]; v[i] = rv[i] / r[i]; w[i] = rw[i] / r[i]; e[i] = rE[i] / r[i];
      wk[i] = u[i] * u[i]; wk[i] = v[i] * v[i] + wk[i]; wk[i] = w[i] * w[i] + wk[i];
      e[i] = -0.5 * wk[i] + e[i];
    }
    lifted_gradient(P, E, 1, u.data(), ux.data(), uy.data(), uz.data());
    lifted_gradient(P, E, 2, v.data(), vx.data(), vy.data(), vz.data());
    lifted_gradient(P, E, 3, w.data(), wx.data(), wy.data(), wz.data());
    for (int i = 0; i < n; ++i) {
      mu[i] = muv;
      t12[i] = uy[i] + vx[i]; t12[i] = mu[i] * t12[i];
      t13[i] = uz[i] + wx[i]; t13[i] = mu[i] * t13[i];
      t23[i] = vz[i] + wy[i]; t23[i] = mu[i] * t23[i];
      wk[i] = 2.0 * ux[i] - vy[i]; t11[i] = 1.0 * wk[i] - wz[i]; t11[i] = (2.0 / 3.0) * t11[i]; t11[i] = mu[i] * t11[i];
      wk[i] = 2.0 * vy[i] - ux[i]; t22[i] = 1.0 * wk[i] - wz[i]; t22[i] = (2.0 / 3.0) * t22[i]; t22[i] = mu[i] * t22[i];
      wk[i] = 2.0 * wz[i] - ux[i]; t33[i] = 1.0 * wk[i] - vy[i]; t33[i] = (2.0 / 3.0) * t33[i]; t33[i] = mu[i] * t33[i];
    }
    double *F[5];
    for (int c = 0; c < 5; ++c) F[c] = P.Uv_u.data() + c * N + E.off;
    fill_sides_flux(E, t11.data(), t12.data(), t13.data(), sfld(P, P.Us_s, 1));
    gradient_dir(E, t11.data(), ux.data(), 'x'); gradient_dir(E, t12.data(), wk.data(), 'y');
    for (int i = 0; i < n; ++i) F[1][i] = ux[i] + wk[i];
    gradient_dir(E, t13.data(), wk.data(), 'z'); for (int i = 0; i < n; ++i) F[1][i] = wk[i] + F[1][i];
    fill_sides_flux(E, t12.data(), t22.data(), t23.data(), sfld(P, P.Us_s, 2));
    gradient_dir(E, t12.data(), ux.data(), 'x'); gradient_dir(E, t22.data(), wk.data(), 'y');
    for (int i = 0; i < n; ++i) F[2][i] = ux[i] + wk[i];
    gradient_dir(E, t23.data(), wk.data(), 'z'); for (int i = 0; i < n; ++i) F[2][i] = wk[i] + F[2][i];
    fill_sides_flux(E, t13.data(), t23.data(), t33.data(), sfld(P, P.Us_s, 3));
    gradient_dir(E, t13.data(), ux.data(), 'x'); gradient_dir(E, t23.data(), wk.data(), 'y');
    for (int i = 0; i < n; ++i) F[3][i] = ux[i] + wk[i];
    gradient_dir(E, t33.data(), wk.data(), 'z'); for (int i = 0; i < n; ++i) F[3][i] = wk[i] + F[3][i];
    for (int i = 0; i < n; ++i) {
      ux[i] = t11[i] * u[i]; ux[i] = t12[i] * v[i] + ux[i]; ux[i] = t13[i] * w[i] + ux[i];
      uy[i] = t12[i] * u[i]; uy[i] = t22[i] * v[i] + uy[i]; uy[i] = t23[i] * w[i] + uy[i];
      uz[i] = t13[i] * u[i]; uz[i] = t23[i] * v[i] + uz[i]; uz[i] = t33[i] * w[i] + uz[i];
    }
    lifted_gradient(P, E, 4, e.data(), vx.data(), vy.data(), vz.data());
    for (int i = 0; i < n; ++i) {
      vx[i] = mu[i] * vx[i]; ux[i] = gPr * vx[i] + ux[i];
      vy[i] = mu[i] * vy[i]; uy[i] = gPr * vy[i] + uy[i];
      vz[i] = mu[i] * vz[i]; uz[i] = gPr * vz[i] + uz[i];
    }
    fill_sides_flux(E, ux.data(), uy.data(), uz.data(), sfld(P, P.Us_s, 4));
    gradient_dir(E, ux.data(), wk.data(), 'x'); gradient_dir(E, uy.data(), ux.data(), 'y');
    for (int i = 0; i < n; ++i) F[4][i] = wk[i] + ux[i];
    gradient_dir(E, uz.data(), wk.data(), 'z'); for (int i = 0; i < n; ++i) F[4][i] = wk[i] + F[4][i];
  }
  if (!P.bcs.empty()) enforce_flux_bc(P);
  average_flux(P, -1.0);
#pragma omp parallel for schedule(static)
  for (int k = 0; k < P.ne; ++k)
    for (int n = 1; n < P.nf; ++n) {
      const Elem &E = P.el[k];
      lift(E, sfld(P, P.Uv_s, n), sfld(P, P.Us_s, n), P.Uv_u.data() + n * N + E.off, 0);
    }
  for (int n = 1; n < P.nf; ++n)
    for (size_t i = 0; i < N; ++i) {
      double x = -1.0 * P.Uv_u[n * N + i];
      Rb[n * N + i] = x + Rb[n * N + i];
    }
}

static void project_all(Problem &P, double *Fb) {
#pragma omp parallel for schedule(static)
  for (int e = 0; e < P.ne; ++e)
    for (int n = 0; n < P.nf; ++n) {
      const Elem &E = P.el[e];
      project(E, Fb + (size_t)n * P.ntot + E.off);
    }
}

// Domain::time_derivative (F = -dU/dt; src/Euler.cpp:282-287,
// src/Euler3d.cpp:455-458, src/Navier_Stokes.cpp:95-100,
// src/Navier_Stokes3d.cpp:135-161, src/Shallow.cpp:255-267)
static void time_derivative(Problem &P, const double *Ub, double *Fb) {
  fill_all_sides(P, const_cast<double *>(Ub));
  if (!P.bcs.empty()) enforce_bc(P, false);
  switch (P.physics) {
    case EULER2D: case NS2D: euler2d_volume(P, Ub, Fb); euler2d_flux(P); break;
    case EULER3D: case NS3D: euler3d_volume(P, Ub, Fb); euler3d_flux(P); break;
    case SHALLOW: shallow_volume(P, Ub, Fb); shallow_flux(P); break;
  }
  lift_all(P, Fb, 0);
  if (P.physics == NS2D) ns2d_diffusion(P, Ub, Fb);
  if (P.physics == NS3D) ns3d_diffusion(P, Ub, Fb);
  // add_source (src/Euler.cpp:1297-1302, src/Navier_Stokes.cpp:375-381,
  // src/Shallow.cpp:851-856): ConstSource / FileSource apply, F -= S
  if (!P.S.empty() && P.dim == 2) {
    // GaussianSource: value = dx^2/(2sx^2) + dy^2/(2sy^2) + (t-t0)^2/(2st^2),
    // S = hamp exp(-value) (src/Shallow.hpp:720-730), as S(x) exp(-dt^2/(2st^2))
    const double dtp = P.t - P.pulse_t0;
    const double g = P.pulse ? std::exp(-(dtp * dtp * P.pulse_s2t2i)) : 1.0;
    for (size_t i = 0; i < P.S.size(); ++i) Fb[i] = Fb[i] - g * P.S[i];
  }
  project_all(P, Fb);
  if (P.physics == NS3D && P.hold_bulk) hold_bulk_mass_flow(P, Fb);
  if (P.physics == SHALLOW && P.sw_balance) {
    const size_t M = (size_t)P.nf * P.ntot;
    if (P.sw_first) { P.Usrc.assign(Fb, Fb + M); P.sw_first = false; }
    for (size_t i = 0; i < M; ++i) Fb[i] = -1.0 * P.Usrc[i] + Fb[i];
  }
}

// ------------------------------------------------------------ integrators
// RK4 (src/TimeInt.cpp:204-209, :266-302)
static void rk4_step(Problem &P, double dt) {
  static const double a[3] = {0.5, 0.5, 1.0};
  static const double b[4] = {0.16666666666666667, 0.33333333333333333,
                              0.33333333333333333, 0.16666666666666667};
  const size_t M = (size_t)P.nf * P.ntot;
  double *U = P.U.data(), *Ut = P.Ut.data(), *R0 = P.R0.data(), *R1 = P.R1.data();
  const double tn = P.t;
  time_derivative(P, U, R0);
  for (size_t i = 0; i < M; ++i) Ut[i] = (-a[0] * dt) * R0[i] + U[i];
  for (size_t i = 0; i < M; ++i) R0[i] = -b[0] * R0[i];
  P.t = tn + 0.5 * dt;
  time_derivative(P, Ut, R1);
  for (size_t i = 0; i < M; ++i) Ut[i] = (-a[1] * dt) * R1[i] + U[i];
  for (size_t i = 0; i < M; ++i) R0[i] = -b[1] * R1[i] + R0[i];
  time_derivative(P, Ut, R1);
  for (size_t i = 0; i < M; ++i) Ut[i] = (-a[2] * dt) * R1[i] + U[i];
  for (size_t i = 0; i < M; ++i) R0[i] = -b[2] * R1[i] + R0[i];
  P.t = tn + dt;
  time_derivative(P, Ut, R1);
  for (size_t i = 0; i < M; ++i) R0[i] = -b[3] * R1[i] + R0[i];
  for (size_t i = 0; i < M; ++i) U[i] = dt * R0[i] + U[i];
}

// TVD-RK3 (src/TimeInt.cpp:738-741, :826-860)
static void tvd3_step(Problem &P, double dt) {
  static const double a[3] = {0.0, 3.0 / 4.0, 1.0 / 3.0};
  static const double b[3] = {1.0, 1.0 / 4.0, 2.0 / 3.0};
  const size_t M = (size_t)P.nf * P.ntot;
  double *U = P.U.data(), *Ut = P.Ut.data(), *R0 = P.R0.data();
  const double tn = P.t;   // stage times tn + c dt, c = 0, 1, 1/2 (src/TimeInt.cpp:740)
  time_derivative(P, U, R0);
  for (size_t i = 0; i < M; ++i) Ut[i] = -dt * R0[i] + U[i];
  P.t = tn + 1.0 * dt;
  time_derivative(P, Ut, R0);
  for (size_t i = 0; i < M; ++i) R0[i] = -dt * R0[i] + Ut[i];
  for (size_t i = 0; i < M; ++i) { Ut[i] = b[1] * R0[i]; Ut[i] = a[1] * U[i] + Ut[i]; }
  P.t = tn + 0.5 * dt;
  time_derivative(P, Ut, R0);
  for (size_t i = 0; i < M; ++i) R0[i] = -dt * R0[i] + Ut[i];
  for (size_t i = 0; i < M; ++i) { U[i] = a[2] * U[i]; U[i] = b[2] * R0[i] + U[i]; }
  P.t = tn + dt;
}

// LSRK14 (src/TimeInt.cpp:1870-1917 coefficients, :1989-2013 advance)
static const double kLsrkA[14] = {
    0.0, -0.7188012108672410, -0.7785331173421570, -0.0053282796654044,
    -0.8552979934029281, -3.9564138245774565, -1.5780575380587385,
    -2.0837094552574054, -0.7483334182761610, -0.7032861106563359,
    0.0013917096117681, -0.0932075369637460, -0.9514200470875948,
    -7.1151571693922548};
static const double kLsrkB[14] = {
    0.0367762454319673, 0.3136296607553959, 0.1531848691869027,
    0.0030097086818182, 0.3326293790646110, 0.2440251405350864,
    0.3718879239592277, 0.6204126221582444, 0.1524043173028741,
    0.0760894927419266, 0.0077604214040978, 0.0024647284755382,
    0.0780348340049386, 5.5059777270269628};

static void lsrk14_step(Problem &P, double dt) {
  const size_t M = (size_t)P.nf * P.ntot;
  double *U = P.U.data(), *Ut = P.Ut.data(), *R0 = P.R0.data();
  static const double c[14] = {0.0, 0.0367762454319673, 0.1249685262725025, 0.2446177702277698,
                               0.2476149531070420, 0.2969311120382472, 0.3978149645802642,
                               0.5270854589440328, 0.6981269994175695, 0.8190890835352128,
                               0.8527059887098624, 0.8604711817462826, 0.8627060376969976,
                               0.8734213127600976};
  const double tn = P.t;   // t = tn + c_s dt per stage, tn + dt after (src/TimeInt.cpp:1999-2011)
  for (int s = 0; s < 14; ++s) {
    P.t = tn + c[s] * dt;
    time_derivative(P, U, R0);
    for (size_t i = 0; i < M; ++i) { double t = kLsrkA[s] * Ut[i]; Ut[i] = -dt * R0[i] + t; }
    for (size_t i = 0; i < M; ++i) U[i] = kLsrkB[s] * Ut[i] + U[i];
  }
  P.t = tn + dt;
}

}  // namespace ora

// =============================================================================
// C ABI used by tests/ and bench.py (ctypes).
// =============================================================================
using namespace ora;
extern "C" {

void *ora_create(int dim, int ne, const double *verts, const int *porder,
                 const int *qorder, int ncon, const int *con, int physics,
                 int flux, double gamma, double vis, double Pr) {
  try {
    return build(dim, ne, verts, porder, qorder, ncon, con, physics, flux, gamma, vis, Pr);
  } catch (...) {
    return nullptr;
  }
}
void ora_free(void *h) { delete (Problem *)h; }
// Boundary sides: nbc records (element, side, kind) with five
// parameters each (isothermal wall: Tw, Eref; state: the conserved values;
// subsonic outflow: Mref).  A record replaces the side's connectivity link; a
// linked partner must be named too.  Returns 0, or -1 on a bad record.
// Call once, before any state is set.
int ora_set_bc(void *h, int nbc, const int *es_kind, const double *par) {
  auto *P = (Problem *)h;
  if (!P->bcs.empty()) return -1;
  const int nsides = P->dim == 2 ? 4 : 6;
  size_t off = P->nstot;
  for (int b = 0; b < nbc; ++b) {
    const int e = es_kind[3 * b], s = es_kind[3 * b + 1], kind = es_kind[3 * b + 2];
    if (e < 0 || e >= P->ne || s < 0 || s >= nsides) return -1;
    if (kind < BC_SLIP_WALL || kind > BC_SUPERSONIC_OUTFLOW) return -1;
    if (P->physics == SHALLOW && kind != BC_SLIP_WALL) return -1;
    if (kind == BC_ISOTHERMAL_WALL && P->physics != NS3D && P->physics != NS2D) return -1;
    if (kind == BC_SLIP_WALL && P->physics != EULER3D && P->physics != EULER2D && P->physics != SHALLOW) return -1;
    if ((kind == BC_SUBSONIC_OUTFLOW || kind == BC_SUPERSONIC_OUTFLOW) && P->dim != 2) return -1;
    Side &S = P->el[e].side[s];
    if (S.bc >= 0) return -1;
    S.master = true; S.bc = b;
    S.flip_a = S.flip_b = S.transp = false;
    Side G = S;
    G.master = false; G.bc = -1; G.off = off; off += S.qtot;
    P->gs.push_back(G);
    Problem::BCRec rec{e, s, kind, par[5 * b], par[5 * b + 1], {}};
    for (int k = 0; k < 5; ++k) rec.v[k] = par[5 * b + k];
    P->bcs.push_back(rec);
  }
  // a boundary record replaces the side's connectivity link
  // (src/Field.cpp:4451); its former partner must be a boundary side too
  for (auto &R : P->bcs) {
    Side &S = P->el[R.e].side[R.s];
    if (S.link_e >= 0 && P->el[S.link_e].side[S.link_s].bc < 0) return -1;
  }
  for (auto &R : P->bcs) { Side &S = P->el[R.e].side[R.s]; S.link_e = S.link_s = -1; }
  for (auto &G : P->gs) G.link_e = G.link_s = -1;
  const size_t nf = P->nf;
  P->nstot = off;
  P->Us_s.assign(nf * P->nstot, 0.0); P->Uf_s.assign(nf * P->nstot, 0.0);
  P->Uv_s.assign(nf * P->nstot, 0.0);
  return 0;
}
// Channel forcing: hold the bulk density, x-momentum and energy (NS 3-D).
void ora_set_hold_bulk(void *h, int on) { ((Problem *)h)->hold_bulk = on != 0; }

long ora_ntot(void *h) { return (long)((Problem *)h)->ntot; }
int ora_nfields(void *h) { return ((Problem *)h)->nf; }
int ora_error(void *h) { return ((Problem *)h)->err; }
// Source field S (GLL values [nf][ntot]), or none when S is null.
void ora_set_source(void *h, const double *S) {
  auto *P = (Problem *)h;
  if (!S) { P->S.clear(); return; }
  P->S.assign(S, S + (size_t)P->nf * P->ntot);
}

void ora_set_time(void *h, double t) { ((Problem *)h)->t = t; }
double ora_get_time(void *h) { return ((Problem *)h)->t; }
void ora_set_source_pulse(void *h, double t0, double sigma_t) {
  auto *P = (Problem *)h;
  P->pulse = sigma_t > 0.0;
  P->pulse_t0 = t0;
  P->pulse_s2t2i = P->pulse ? 1.0 / (2.0 * sigma_t * sigma_t) : 0.0;
}

// The LSRK14 2N-storage coefficients (A: register decay, B: update weight).
void ora_lsrk14_coefficients(double *A, double *B) {
  for (int k = 0; k < 14; ++k) { A[k] = kLsrkA[k]; B[k] = kLsrkB[k]; }
}

void ora_set_threads(int n) {
#ifdef _OPENMP
  omp_set_num_threads(n);
#else
  (void)n;
#endif
}
void ora_set_sw_balance(void *h, int on) { auto *P = (Problem *)h; P->sw_balance = on != 0; P->sw_first = true; }

// GLL coordinates, wJ (per point) and element offsets
void ora_coords(void *h, double *x, double *y, double *z) {
  auto *P = (Problem *)h;
  for (auto &E : P->el)
    for (int i = 0; i < E.qtot; ++i) {
      x[E.off + i] = E.cx[i]; y[E.off + i] = E.cy[i]; z[E.off + i] = E.cz[i];
    }
}
void ora_wj(void *h, double *wj) {
  auto *P = (Problem *)h;
  for (auto &E : P->el) for (int i = 0; i < E.qtot; ++i) wj[E.off + i] = E.wJ[i];
}
void ora_set_state(void *h, const double *U) {
  auto *P = (Problem *)h;
  std::memcpy(P->U.data(), U, sizeof(double) * P->U.size());
  std::fill(P->Ut.begin(), P->Ut.end(), 0.0);
}
void ora_get_state(void *h, double *U) {
  auto *P = (Problem *)h;
  std::memcpy(U, P->U.data(), sizeof(double) * P->U.size());
}
// project every field of U in place (Field::project)
void ora_project(void *h, double *U) {
  auto *P = (Problem *)h;
  project_all(*P, U);
}
// modal coefficients per field per element (restart layout, src/vField.cpp:1102-1179)
void ora_forward(void *h, const double *U, double *Uh) {
  auto *P = (Problem *)h;
  size_t mo = 0;
  for (int n = 0; n < P->nf; ++n)
    for (auto &E : P->el) {
      vec f(U + (size_t)n * P->ntot + E.off, U + (size_t)n * P->ntot + E.off + E.qtot);
      forward_transform(E, f.data(), Uh + mo);
      mo += E.nmodes;
    }
}
void ora_backward(void *h, const double *Uh, double *U) {
  auto *P = (Problem *)h;
  size_t mo = 0;
  for (int n = 0; n < P->nf; ++n)
    for (auto &E : P->el) {
      backward_transform(E, Uh + mo, U + (size_t)n * P->ntot + E.off);
      mo += E.nmodes;
    }
}
long ora_nmodes(void *h) {
  auto *P = (Problem *)h;
  long m = 0;
  for (auto &E : P->el) m += E.nmodes;
  return m;
}
// F = -dU/dt
void ora_rhs(void *h, const double *U, double *F) {
  auto *P = (Problem *)h;
  time_derivative(*P, U, F);
}
// inttype: 3 = TVD-RK3, 4 = RK4, 14 = LSRK14 (src/TimeInt.hpp:62-85)
int ora_advance(void *h, int inttype, double dt, int nsteps) {
  auto *P = (Problem *)h;
  for (int s = 0; s < nsteps; ++s) {
    if (inttype == 3) tvd3_step(*P, dt);
    else if (inttype == 4) rk4_step(*P, dt);
    else if (inttype == 14) lsrk14_step(*P, dt);
    else return -1;
  }
  return P->err;
}
// 1-D tables for tests: z, w (Q), D (QxQ), B (LxQ), GL2G (GxQ), G2GL (QxG)
void ora_tables(int L, int Q, int G, double *z, double *w, double *D, double *B,
                double *gl2g, double *g2gl) {
  auto t = table(L, Q);
  std::memcpy(z, t->z.data(), sizeof(double) * Q);
  std::memcpy(w, t->w.data(), sizeof(double) * Q);
  std::memcpy(D, t->D.data(), sizeof(double) * Q * Q);
  std::memcpy(B, t->B.data(), sizeof(double) * L * Q);
  auto a = interp(0, G, Q), b = interp(1, Q, G);
  std::memcpy(gl2g, a->m.data(), sizeof(double) * G * Q);
  std::memcpy(g2gl, b->m.data(), sizeof(double) * Q * G);
}
void ora_gauss(int np, double *z, double *w) { gauss_legendre(np, z, w); }
// side orientation flags for tests: per element per side (master, link_e,
// link_s, flip_a, flip_b, transp)
void ora_sides(void *h, int *out) {
  auto *P = (Problem *)h;
  int k = 0;
  for (auto &E : P->el)
    for (int s = 0; s < E.nsides; ++s) {
      const Side &S = E.side[s];
      out[k++] = S.master; out[k++] = S.link_e; out[k++] = S.link_s;
      out[k++] = S.flip_a; out[k++] = S.flip_b; out[k++] = S.transp;
    }
}
}

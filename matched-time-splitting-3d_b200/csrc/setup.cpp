// Host-side problem setup; see setup.h.  Compiled without FMA contraction so
// that every floating-point operation rounds as in the reference build.
#include "setup.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <thread>

namespace mts {
namespace {

const double TOL_SETUP = 1.0e-12;   // src/constant.h:10
const double TOL_RTSAFE = 1.0e-14;  // src/constant.h:11

// ---------------------------------------------------------------------------
// Surfaces

// Ellipsoid with centre.  With a zero centre every expression is the one of
// Surface_Ellipsoid (src/surface/surface_ellipsoid.cc:60-168), since x - 0.0
// is x exactly.
class Ellipsoid : public Surface {
 public:
  explicit Ellipsoid(const double* p) : a(p[0]), b(p[1]), c(p[2]), r(p[3]), cx(p[4]), cy(p[5]), cz(p[6]) {}
  double set_node(double x, double y, double z) const override {
    double X = x - cx, Y = y - cy, Z = z - cz;
    return X * X / (a * a) + Y * Y / (b * b) + Z * Z / (c * c) - r * r + TOL_SETUP;
  }
  double func(double x, double y, double z) const override {
    double X = x - cx, Y = y - cy, Z = z - cz;
    return X * X / (a * a) + Y * Y / (b * b) + Z * Z / (c * c) - r * r;
  }
  double dfx(double x, double, double) const override { return 2 * (x - cx) / (a * a); }
  double dfy(double, double y, double) const override { return 2 * (y - cy) / (b * b); }
  double dfz(double, double, double z) const override { return 2 * (z - cz) / (c * c); }
  void normal(double x, double y, double z, double n[3]) const override {
    double X = x - cx, Y = y - cy, Z = z - cz;
    double total = std::sqrt(std::pow(2 * X / (a * a), 2) + std::pow(2 * Y / (b * b), 2) +
                             std::pow(2 * Z / (c * c), 2));
    n[0] = 2 * X / (a * a) / total;
    n[1] = 2 * Y / (b * b) / total;
    n[2] = 2 * Z / (c * c) / total;
  }

 private:
  double a, b, c, r, cx, cy, cz;
};

// Torus about the z axis, Surface_Torus (src/surface/surface_torus.cc:15-150).
class Torus : public Surface {
 public:
  explicit Torus(const double* p) : a(p[0]), b(p[1]) {}
  double set_node(double x, double y, double z) const override {
    return std::pow((a - std::sqrt(x * x + y * y)), 2) + z * z - b * b + TOL_SETUP;
  }
  double func(double x, double y, double z) const override {
    return std::pow((a - std::sqrt(x * x + y * y)), 2) + z * z - b * b;
  }
  double dfx(double x, double y, double) const override {
    return (-2.0 * a * x) / (std::sqrt(x * x + y * y)) + 2.0 * x;
  }
  double dfy(double x, double y, double) const override {
    return (-2.0 * a * y) / (std::sqrt(x * x + y * y)) + 2.0 * y;
  }
  double dfz(double, double, double z) const override { return 2.0 * z; }
  void normal(double x, double y, double z, double n[3]) const override {
    double total = std::sqrt(std::pow((-2.0 * a * x) / (std::sqrt(x * x + y * y)) + 2.0 * x, 2) +
                             std::pow((-2.0 * a * y) / (std::sqrt(x * x + y * y)) + 2.0 * y, 2) +
                             std::pow(2.0 * z, 2));
    n[0] = ((-2.0 * a * x) / (std::sqrt(x * x + y * y)) + 2.0 * x) / total;
    n[1] = ((-2.0 * a * y) / (std::sqrt(x * x + y * y)) + 2.0 * y) / total;
    n[2] = (2.0 * z) / total;
  }

 private:
  double a, b;
};

// Newton-Raphson with bisection fallback along one axis: Rtsafe_x/y/z
// (src/surface/surface_cartesian.cc:157-373), the Numerical-Recipes rtsafe.
// axis selects which coordinate varies; q holds the other two fixed values.
struct Root {
  bool ok;
  double value;
};

Root rtsafe(const Surface& s, int axis, double v1, double v2, double p, double q) {
  auto F = [&](double v) {
    return axis == 0 ? s.func(v, p, q) : axis == 1 ? s.func(p, v, q) : s.func(p, q, v);
  };
  auto DF = [&](double v) {
    return axis == 0 ? s.dfx(v, p, q) : axis == 1 ? s.dfy(p, v, q) : s.dfz(p, q, v);
  };
  const int MAXIT = 100;
  double fl, fh, xh, xl, rts, dxold, dx, f, df, temp;
  fl = F(v1);
  fh = F(v2);
  if ((fl > 0.0 && fh > 0.0) || (fl < 0.0 && fh < 0.0)) return {false, 0};
  if (fl == 0.0) return {true, v1};
  if (fh == 0.0) return {true, v2};
  if (fl < 0.0) {
    xl = v1;
    xh = v2;
  } else {
    xh = v1;
    xl = v2;
  }
  rts = 0.5 * (v1 + v2);
  dxold = std::abs(v2 - v1);
  dx = dxold;
  f = F(rts);
  df = DF(rts);
  for (int j = 0; j < MAXIT; j++) {
    if ((((rts - xh) * df - f) * ((rts - xl) * df - f) > 0.0) || (std::abs(2.0 * f) > std::abs(dxold * df))) {
      dxold = dx;
      dx = 0.5 * (xh - xl);
      rts = xl + dx;
      if (xl == rts) return {true, rts};
    } else {
      dxold = dx;
      dx = f / df;
      temp = rts;
      rts -= dx;
      if (temp == rts) return {true, rts};
    }
    if (std::abs(dx) < TOL_RTSAFE) return {true, rts};
    f = F(rts);
    df = DF(rts);
    if (f < 0.0)
      xl = rts;
    else
      xh = rts;
  }
  return {false, 0};
}

// Gamma_x/y/z (src/surface/surface_cartesian.cc:23-131).
Root gamma_root(const Surface& s, int axis, double v1, double v2, double p, double q) {
  if (!(v1 > v2) && !(v1 < v2)) return {false, 0};
  if (std::abs(v1 - v2) < TOL_RTSAFE) return {true, (v1 + v2) / 2};
  return rtsafe(s, axis, v1, v2, p, q);
}

// ---------------------------------------------------------------------------
// Dense LU with implicit pivoting: LU::LU, LU::solve, LU::det
// (src/decomposition/lu.cc:15-115, 164-173), the Numerical-Recipes ludcmp.
class Lu {
 public:
  Lu(const std::vector<double>& a, int n) : n_(n), lu_(a), indx_(n) {
    const double TINY = 1.0e-40;
    int i, imax = 0, j, k;
    double big, temp;
    std::vector<double> vv(n);
    d_ = 1.0;
    ok_ = true;
    for (i = 0; i < n; i++) {
      big = 0.0;
      for (j = 0; j < n; j++)
        if ((temp = std::abs(at(i, j))) > big) big = temp;
      if (big == 0.0) {
        ok_ = false;
        return;
      }
      vv[i] = 1.0 / big;
    }
    for (k = 0; k < n; k++) {
      big = 0.0;
      for (i = k; i < n; i++) {
        temp = vv[i] * std::abs(at(i, k));
        if (temp > big) {
          big = temp;
          imax = i;
        }
      }
      if (k != imax) {
        for (j = 0; j < n; j++) {
          temp = at(imax, j);
          at(imax, j) = at(k, j);
          at(k, j) = temp;
        }
        d_ = -d_;
        vv[imax] = vv[k];
      }
      indx_[k] = imax;
      if (at(k, k) == 0.0) at(k, k) = TINY;
      for (i = k + 1; i < n; i++) {
        temp = at(i, k) /= at(k, k);
        for (j = k + 1; j < n; j++) at(i, j) -= temp * at(k, j);
      }
    }
  }
  bool ok() const { return ok_; }
  void solve(const std::vector<double>& b, std::vector<double>& x) {
    int i, ii = 0, ip, j;
    double sum;
    for (i = 0; i < n_; i++) x[i] = b[i];
    for (i = 0; i < n_; i++) {
      ip = indx_[i];
      sum = x[ip];
      x[ip] = x[i];
      if (ii != 0)
        for (j = ii - 1; j < i; j++) sum -= at(i, j) * x[j];
      else if (sum != 0.0)
        ii = i + 1;
      x[i] = sum;
    }
    for (i = n_ - 1; i >= 0; i--) {
      sum = x[i];
      for (j = i + 1; j < n_; j++) sum -= at(i, j) * x[j];
      x[i] = sum / at(i, i);
    }
  }
  double det() const {
    double dd = d_;
    for (int i = 0; i < n_; i++) dd *= lu_[(size_t)i * n_ + i];
    return dd;
  }

 private:
  double& at(int i, int j) { return lu_[(size_t)i * n_ + j]; }
  int n_;
  std::vector<double> lu_;
  std::vector<int> indx_;
  double d_;
  bool ok_;
};

// Fornberg finite-difference weights, Intersections::Weights
// (src/spatial/intersection.cc:5093-5130).  c is n x (m+1), row major.
void fd_weights(double z, const double* x, int n, int m, double* c) {
  double c1, c2, c3, c4, c5;
  int mn;
  const int w = m + 1;
  c1 = 1;
  c4 = x[0] - z;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < m + 1; j++) c[i * w + j] = 0;
  c[0] = 1;
  for (int i = 1; i < n; i++) {
    mn = i < m ? i : m;
    c2 = 1;
    c5 = c4;
    c4 = x[i] - z;
    for (int j = 0; j < i; j++) {
      c3 = x[i] - x[j];
      c2 = c2 * c3;
      if (j == i - 1) {
        for (int k = mn; k > 0; k--) c[i * w + k] = c1 * (k * c[(i - 1) * w + k - 1] - c5 * c[(i - 1) * w + k]) / c2;
        c[i * w + 0] = -c1 * c5 * c[(i - 1) * w + 0] / c2;
      }
      for (int k = mn; k > 0; k--) c[j * w + k] = (c4 * c[j * w + k] - k * c[j * w + k - 1]) / c3;
      c[j * w + 0] = c4 * c[j * w + 0] / c3;
    }
    c1 = c2;
  }
}

// wei[order][j] = temp[j][order] for the two-order (value, first derivative)
// tables the MIB solves use.
struct Wei2 {
  double w[2][4];
};
Wei2 weights_table(double z, const double* v, int n) {
  double temp[4 * 2];
  fd_weights(z, v, n, 1, temp);
  Wei2 r;
  for (int i = 0; i < 2; i++)
    for (int j = 0; j < n; j++) r.w[i][j] = temp[j * 2 + i];
  return r;
}

struct SolveResult {
  bool ok;
  bool singular;
};

SolveResult lu_solve(std::vector<double>& A, int n, std::vector<double>& B, std::vector<double>& x) {
  Lu lu(A, n);
  if (!lu.ok()) return {false, false};
  lu.solve(B, x);
  return {true, std::abs(lu.det()) < TOL_SETUP};
}

// Working copy of one crossing during setup.
struct Xing {
  mts_crossing c;
  double inside, outside;
};

// MIB_L1 (src/spatial/intersection.cc:930-1066): 8x8 system for the two
// fictitious points of one crossing.
SolveResult mib_l1(const Xing& q, double dv, std::vector<double>& x) {
  const int one = 4, tot = 8;
  std::vector<double> A(tot * tot, 0.0), B(tot, 0.0);
  double v[2] = {0, dv};
  Wei2 wt = weights_table(q.c.gamma, v, 2);
  auto& wei = wt.w;
  bool even = std::abs(q.c.id) % 2 == 0;
  int order = 0;
  B[0] = -wei[order][0];
  B[1] = wei[order][1];
  for (int i = 0; i < one; i++) {
    A[i * tot + i] = -wei[order][0];
    A[i * tot + one + i] = wei[order][1];
  }
  if (even)
    B[one - 2] += -1;
  else
    B[one - 2] += 1;
  order = 1;
  double coefl, coefr;
  if (even) {
    coefr = q.inside;
    coefl = q.outside;
  } else {
    coefr = q.outside;
    coefl = q.inside;
  }
  B[one + 0] = -wei[order][0] * coefr;
  B[one + 1] = wei[order][1] * coefl;
  for (int i = 0; i < one; i++) {
    A[(one + i) * tot + i] = -wei[order][0] * coefl;
    A[(one + i) * tot + one + i] = wei[order][1] * coefr;
  }
  if (even)
    B[tot - 1] += -1;
  else
    B[tot - 1] += 1;
  x.assign(tot, 0.0);
  return lu_solve(A, tot, B, x);
}

// Irregular_MIB_L1 (intersection.cc:1076-1122).
SolveResult irregular_l1(Xing& q, double dv) {
  std::vector<double> x;
  SolveResult r = mib_l1(q, dv, x);
  if (!r.ok) return r;
  q.c.nwei = 6;
  std::memset(q.c.weil, 0, sizeof q.c.weil);
  std::memset(q.c.weir, 0, sizeof q.c.weir);
  q.c.weil[1] = x[0];
  q.c.weil[2] = x[1];
  q.c.weil[4] = x[2];
  q.c.weil[5] = x[3];
  q.c.weir[1] = x[4];
  q.c.weir[2] = x[5];
  q.c.weir[4] = x[6];
  q.c.weir[5] = x[7];
  return r;
}

// Corner_MIB_L1 (intersection.cc:1128-1200): each crossing of the pair on
// its own, placed in the 9-wide corner layout.
SolveResult corner_l1(Xing& l, Xing& r, double dv) {
  std::vector<double> x;
  SolveResult s1 = mib_l1(l, dv, x);
  if (!s1.ok) return s1;
  l.c.nwei = 9;
  r.c.nwei = 9;
  std::memset(l.c.weil, 0, sizeof l.c.weil);
  std::memset(l.c.weir, 0, sizeof l.c.weir);
  std::memset(r.c.weil, 0, sizeof r.c.weil);
  std::memset(r.c.weir, 0, sizeof r.c.weir);
  l.c.weil[1] = x[0];
  l.c.weil[2] = x[1];
  l.c.weil[5] = x[2];
  l.c.weil[6] = x[3];
  l.c.weir[1] = x[4];
  l.c.weir[2] = x[5];
  l.c.weir[5] = x[6];
  l.c.weir[6] = x[7];
  SolveResult s2 = mib_l1(r, dv, x);
  if (!s2.ok) return s2;
  r.c.weil[2] = x[0];
  r.c.weil[3] = x[1];
  r.c.weil[7] = x[2];
  r.c.weil[8] = x[3];
  r.c.weir[2] = x[4];
  r.c.weir[3] = x[5];
  r.c.weir[7] = x[6];
  r.c.weir[8] = x[7];
  return {true, s1.singular || s2.singular};
}

// Irregular_MIB_L2 + Irregular_MIB_L2_Recursive + Get_irr_weights
// (intersection.cc:1207-1395, 1424-1470) at second order: one pass, 3-point
// stencils (2 real points + 1 fictitious point per side), 12x12 system.
SolveResult irregular_l2(Xing& q, double dv) {
  const int accuracy = 2;
  const int one = accuracy * 2 + 2;  // 6
  const int st = accuracy + 1;       // 3
  const int side = accuracy;         // 2
  const int tot = 2 * one;           // 12
  std::vector<double> A(tot * tot, 0.0), B(tot, 0.0), x(tot, 0.0);
  // Get_irr_weights
  double vr[3], vl[3];
  for (int i = 0; i < st; i++) {
    vr[i] = -(side - 1) * dv + i * dv;
    vl[i] = (side - st + 1) * dv + i * dv;
  }
  Wei2 wr = weights_table(q.c.gamma, vr, st);
  Wei2 wl = weights_table(q.c.gamma, vl, st);
  auto& weir = wr.w;
  auto& weil = wl.w;
  bool even = std::abs(q.c.id) % 2 == 0;
  int order = 0;
  for (int i = 0; i < side; i++) {
    B[i] += -weir[order][i];
    B[side + i] += weil[order][st - side + i];
  }
  for (int i = 0; i < one; i++) {
    A[i * tot + i] = -weil[order][0];
    A[i * tot + one + i] = weir[order][st - 1];
  }
  if (even)
    B[one - 2] += -1;
  else
    B[one - 2] += 1;
  order = 1;
  double coefl, coefr;
  if (even) {
    coefr = q.inside;
    coefl = q.outside;
  } else {
    coefr = q.outside;
    coefl = q.inside;
  }
  for (int i = 0; i < side; i++) {
    B[one + i] += -weir[order][i] * coefr;
    B[one + side + i] += weil[order][st - side + i] * coefl;
  }
  for (int i = 0; i < one; i++) {
    A[(one + i) * tot + one + i] = weir[order][st - 1] * coefr;
    A[(one + i) * tot + i] = -weil[order][0] * coefl;
  }
  if (even)
    B[tot - 1] += -1;
  else
    B[tot - 1] += 1;
  SolveResult r = lu_solve(A, tot, B, x);
  if (!r.ok) return r;
  q.c.nwei = one;
  std::memset(q.c.weil, 0, sizeof q.c.weil);
  std::memset(q.c.weir, 0, sizeof q.c.weir);
  for (int j = 0; j < one; j++) {
    q.c.weil[j] = x[j];
    q.c.weir[j] = x[one + j];
  }
  return r;
}

// Corner_MIB_L2_2nd + Get_cor_weights (intersection.cc:1479-1704,
// 1752-1830): four fictitious points, 36x36 system.
SolveResult corner_l2(Xing& L, Xing& R, double dv) {
  const int one = 5 + 2 * 2;  // 9
  const int tot = 4 * one;    // 36
  const int ns = 4;           // stencil length
  std::vector<double> A(tot * tot, 0.0), B(tot, 0.0), x(tot, 0.0);
  auto a = [&](int i, int j) -> double& { return A[(size_t)i * tot + j]; };
  double gl = L.c.gamma, gr = R.c.gamma;
  double lvo[4], lvi[4], rvo[4], rvi[4];
  for (int i = 0; i < ns; i++) {
    lvo[i] = -dv + i * dv;
    rvo[i] = i * dv;
  }
  for (int i = 0; i < ns; i++) lvi[i] = i * dv;
  if ((dv - gl) > gr) lvi[ns - 1] = -dv;
  for (int i = 0; i < ns; i++) rvi[i] = lvi[i];
  Wei2 lo = weights_table(gl, lvo, ns);
  Wei2 li = weights_table(gl, lvi, ns);
  Wei2 ro = weights_table(dv + gr, rvo, ns);
  Wei2 ri = weights_table(dv + gr, rvi, ns);
  auto& lwo = lo.w;
  auto& lwi = li.w;
  auto& rwo = ro.w;
  auto& rwi = ri.w;
  bool even = std::abs(L.c.id) % 2 == 0;

  // left interface, zero order
  int order = 0;
  B[0] = -lwo[order][0];
  B[1] = -lwo[order][1];
  B[2] = lwi[order][1];
  B[3] = -lwo[order][3];
  for (int i = 0; i < one; i++) {
    a(i, i) = -lwi[order][0];
    a(i, one + i) = lwo[order][2];
    a(i, one * 2 + i) = -lwi[order][2];
    a(i, one * 3 + i) = -lwi[order][3];
  }
  B[5] = even ? -1 : 1;
  // left interface, first order
  order = 1;
  double cin, cout_;
  if (even) {
    cin = L.outside;
    cout_ = L.inside;
  } else {
    cin = L.inside;
    cout_ = L.outside;
  }
  B[one + 0] = -lwo[order][0] * cout_;
  B[one + 1] = -lwo[order][1] * cout_;
  B[one + 2] = lwi[order][1] * cin;
  B[one + 3] = -lwo[order][3] * cout_;
  for (int i = 0; i < one; i++) {
    a(one + i, i) = -lwi[order][0] * cin;
    a(one + i, one + i) = lwo[order][2] * cout_;
    a(one + i, one * 2 + i) = -lwi[order][2] * cin;
    a(one + i, one * 3 + i) = -lwi[order][3] * cin;
  }
  B[one + 6] = even ? -1 : 1;
  // right interface, zero order
  order = 0;
  B[one * 2 + 1] = -rwo[order][0];
  B[one * 2 + 2] = rwi[order][1];
  B[one * 2 + 3] = -rwo[order][2];
  B[one * 2 + 4] = -rwo[order][3];
  for (int i = 0; i < one; i++) {
    a(one * 2 + i, i) = -rwi[order][0];
    a(one * 2 + i, one + i) = rwo[order][1];
    a(one * 2 + i, one * 2 + i) = -rwi[order][2];
    a(one * 2 + i, one * 3 + i) = -rwi[order][3];
  }
  B[one * 2 + 7] = even ? -1 : 1;
  // right interface, first order (the reference keys the sides on the left
  // crossing's ID parity here too)
  order = 1;
  if (even) {
    cin = R.outside;
    cout_ = R.inside;
  } else {
    cin = R.inside;
    cout_ = R.outside;
  }
  B[one * 3 + 1] = -rwo[order][0] * cout_;
  B[one * 3 + 2] = rwi[order][1] * cin;
  B[one * 3 + 3] = -rwo[order][2] * cout_;
  B[one * 3 + 4] = -rwo[order][3] * cout_;
  for (int i = 0; i < one; i++) {
    a(one * 3 + i, i) = -rwi[order][0] * cin;
    a(one * 3 + i, one + i) = rwo[order][1] * cout_;
    a(one * 3 + i, one * 2 + i) = -rwi[order][2] * cin;
    a(one * 3 + i, one * 3 + i) = -rwi[order][3] * cin;
  }
  B[one * 3 + 8] = even ? -1 : 1;

  SolveResult r = lu_solve(A, tot, B, x);
  if (!r.ok) return r;
  L.c.nwei = one;
  R.c.nwei = one;
  for (int j = 0; j < one; j++) {
    L.c.weil[j] = x[j];
    L.c.weir[j] = x[one + j];
    R.c.weil[j] = x[one + j];
    R.c.weir[j] = x[one * 2 + j];
  }
  return r;
}

// Pmatrix_Setup_x/y/z (intersection.cc:2503-2598).
void frame(int dir, const double a[3], double p[9]) {
  for (int i = 0; i < 3; i++) p[i] = a[i];
  if (dir == 0) {
    p[3] = a[2] / std::sqrt(a[0] * a[0] + a[2] * a[2]);
    p[4] = 0;
    p[5] = -a[0] / std::sqrt(a[0] * a[0] + a[2] * a[2]);
    p[6] = a[1] / std::sqrt(a[0] * a[0] + a[1] * a[1]);
    p[7] = -a[0] / std::sqrt(a[0] * a[0] + a[1] * a[1]);
    p[8] = 0;
  } else if (dir == 1) {
    p[3] = 0;
    p[4] = a[2] / std::sqrt(a[1] * a[1] + a[2] * a[2]);
    p[5] = -a[1] / std::sqrt(a[1] * a[1] + a[2] * a[2]);
    p[6] = a[1] / std::sqrt(a[0] * a[0] + a[1] * a[1]);
    p[7] = -a[0] / std::sqrt(a[0] * a[0] + a[1] * a[1]);
    p[8] = 0;
  } else {
    p[3] = 0;
    p[4] = a[2] / std::sqrt(a[1] * a[1] + a[2] * a[2]);
    p[5] = -a[1] / std::sqrt(a[1] * a[1] + a[2] * a[2]);
    p[6] = a[2] / std::sqrt(a[0] * a[0] + a[2] * a[2]);
    p[7] = 0;
    p[8] = -a[0] / std::sqrt(a[0] * a[0] + a[2] * a[2]);
  }
}

}  // namespace

Grid make_grid(const mts_grid& in) {
  Grid g;
  g.nx = in.nx;
  g.ny = in.ny;
  g.nz = in.nz;
  g.xl = in.xl;
  g.xr = in.xr;
  g.yl = in.yl;
  g.yr = in.yr;
  g.zl = in.zl;
  g.zr = in.zr;
  g.dx = (g.xr - g.xl) / (g.nx - 1.0);
  g.dy = (g.yr - g.yl) / (g.ny - 1.0);
  g.dz = (g.zr - g.zl) / (g.nz - 1.0);
  g.x.resize(g.nx);
  g.y.resize(g.ny);
  g.z.resize(g.nz);
  for (int i = 0; i < g.nx; i++) g.x[i] = g.xl + i * g.dx;
  for (int i = 0; i < g.ny; i++) g.y[i] = g.yl + i * g.dy;
  for (int i = 0; i < g.nz; i++) g.z[i] = g.zl + i * g.dz;
  return g;
}

Surface* make_surface(const mts_surface& s) {
  if (s.kind == MTS_SURFACE_ELLIPSOID) return new Ellipsoid(s.params);
  if (s.kind == MTS_SURFACE_TORUS) return new Torus(s.params);
  return nullptr;
}

namespace {

// Host threads of a setup: one per 2^20 nodes, up to the cores (MTS_SETUP_THREADS
// overrides), so that small problems, which servers set up many at a time on
// their own pools, stay on one thread.
int setup_threads(long long nodes) {
  int t = (int)std::min<long long>(64, std::max<long long>(1, nodes >> 20));
  const unsigned hw = std::thread::hardware_concurrency();
  if (hw > 0) t = std::min(t, (int)hw);
  if (const char* e = std::getenv("MTS_SETUP_THREADS")) {
    const int v = std::atoi(e);
    if (v > 0) t = v;
  }
  return t;
}

// Runs body(k) for k in [0, parts) on up to `threads` threads.
template <class F>
void run_parts(int parts, int threads, F body) {
  threads = std::max(1, std::min(threads, parts));
  if (threads == 1) {
    for (int k = 0; k < parts; k++) body(k);
    return;
  }
  std::vector<std::thread> pool;
  for (int w = 0; w < threads; w++)
    pool.emplace_back([&, w] {
      for (int k = w; k < parts; k += threads) body(k);
    });
  for (auto& th : pool) th.join();
}

}  // namespace

mts_status build_tags(const Grid& g, const Surface& s, std::vector<int8_t>& tags) {
  tags.assign((size_t)g.nodes(), 0);
  // planes in parallel; the first failing plane in order decides the status,
  // as in one pass
  std::vector<mts_status> st(g.nz, MTS_OK);
  run_parts(g.nz, setup_threads(g.nodes()), [&](int iz) {
    for (int iy = 0; iy < g.ny; iy++)
      for (int ix = 0; ix < g.nx; ix++) {
        double v = s.set_node(g.x[ix], g.y[iy], g.z[iz]);
        int8_t t;
        if (v > TOL_SETUP)
          t = 1;
        else if (v < TOL_SETUP)
          t = -1;
        else {
          st[iz] = MTS_ERR_SETUP;  // "Interface on grid, reset the mesh!"
          return;
        }
        tags[(size_t)g.index(ix, iy, iz)] = t;
      }
  });
  for (mts_status e : st)
    if (e) return e;
  return MTS_OK;
}

bool frame_inverse_col0(const double p[9], int row, double* out) {
  std::vector<double> a(p, p + 9);
  Lu lu(a, 3);
  if (!lu.ok()) return false;
  // LU::inverse solves for each identity column; column 0 suffices.
  std::vector<double> e(3, 0.0), x(3);
  e[0] = 1.0;
  lu.solve(e, x);
  *out = x[row];
  return true;
}

namespace {

// The crossings of the d-lines with i1 in [i1a, i1b), in line order, into
// out; the first failure stops the range and is returned.
mts_status crossings_of_lines(const Grid& g, const std::vector<int8_t>& tags, const Surface& s, double beta_in,
                              double beta_out, int mib, int d, int i1a, int i1b, std::vector<mts_crossing>& out,
                              SetupReport& rep) {
  const int n[3] = {g.nx, g.ny, g.nz};
  const double h[3] = {g.dx, g.dy, g.dz};
  const std::vector<double>* ax[3] = {&g.x, &g.y, &g.z};
  // fixed axes of a d-line in the reference's (indx1, indx2) convention
  const int a1 = d == 0 ? 1 : 0;
  const int a2 = d == 2 ? 1 : 2;
  for (int i1 = i1a; i1 < i1b; i1++)
    for (int i2 = 1; i2 < n[a2] - 1; i2++) {
      int idx3[3];
      idx3[a1] = i1;
      idx3[a2] = i2;
      auto tag = [&](int j) {
        idx3[d] = j;
        return (double)tags[(size_t)g.index(idx3[0], idx3[1], idx3[2])];
      };
      auto point = [&](int j, double v, double c[3]) {
        idx3[d] = j;
        c[0] = g.x[idx3[0]];
        c[1] = g.y[idx3[1]];
        c[2] = g.z[idx3[2]];
        c[d] = v;
      };
      // fixed coordinates for the root search along d
      double fp = (*ax[a1])[i1], fq = (*ax[a2])[i2];
      auto locate = [&](int j, Xing& q, int id) -> mts_status {
        const std::vector<double>& v = *ax[d];
        Root rt;
        if (d == 0)
          rt = gamma_root(s, 0, v[j], v[j + 1], fp, fq);
        else if (d == 1)
          rt = gamma_root(s, 1, v[j], v[j + 1], fp, fq);
        else
          rt = gamma_root(s, 2, v[j], v[j + 1], fp, fq);
        if (!rt.ok) return MTS_ERR_NONFINITE;
        std::memset(&q.c, 0, sizeof q.c);
        q.c.dir = d;
        q.c.indx1 = i1;
        q.c.indx2 = i2;
        q.c.id = id;
        q.c.left_loc = j;
        point(j, rt.value, q.c.coord);
        q.c.gamma = q.c.coord[d] - v[j];
        q.inside = beta_in;
        q.outside = beta_out;
        s.normal(q.c.coord[0], q.c.coord[1], q.c.coord[2], q.c.normal);
        frame(d, q.c.normal, q.c.p);
        return MTS_OK;
      };
      // Setup_Intersections scan (intersection.cc:79-291)
      int ifp = 0;
      int j = 1;
      while (j < n[d] - 1) {
        if (tag(j) * tag(j + 1) < 0) {
          if (j + 2 >= n[d]) return MTS_ERR_SETUP;  // crossing in the last cell
          if (tag(j + 1) * tag(j + 2) > 0) {
            ifp += 1;
            Xing q;
            mts_status st = locate(j, q, ifp);
            if (st) return st;
            SolveResult r = mib == 1 ? irregular_l1(q, h[d]) : irregular_l2(q, h[d]);
            if (!r.ok) return MTS_ERR_SETUP;
            rep.singular_warnings += r.singular;
            out.push_back(q.c);
            j += 2;
          } else {
            if (j + 3 >= n[d] || tag(j + 2) * tag(j + 3) < 0) return MTS_ERR_SETUP;  // coherent corners
            ifp += 1;
            Xing l, r;
            mts_status st = locate(j, l, -ifp);
            if (st) return st;
            ifp += 1;
            st = locate(j + 1, r, -ifp);
            if (st) return st;
            SolveResult sr = mib == 1 ? corner_l1(l, r, h[d]) : corner_l2(l, r, h[d]);
            if (!sr.ok) return MTS_ERR_SETUP;
            rep.singular_warnings += sr.singular;
            rep.corner_pairs += 1;
            out.push_back(l.c);
            out.push_back(r.c);
            j += 3;
          }
        } else {
          j += 1;
        }
      }
      if (ifp % 2 == 1) return MTS_ERR_SETUP;  // open surface
    }
  return MTS_OK;
}

}  // namespace

mts_status build_crossings(const Grid& g, const std::vector<int8_t>& tags, const Surface& s,
                           double beta_in, double beta_out, int mib,
                           std::vector<mts_crossing>& out, SetupReport* report) {
  out.clear();
  if (mib != 1 && mib != 2) return MTS_ERR_ARG;
  const int n[3] = {g.nx, g.ny, g.nz};
  // Every line's crossings and weights depend on that line alone: ranges of
  // lines run on their own threads into their own lists, which are joined in
  // line order (direction, i1, i2), the order of one pass.  The first failing
  // range in that order decides the status, as in one pass.
  struct Range {
    int d, a, b;
    std::vector<mts_crossing> out;
    SetupReport rep;
    mts_status st = MTS_OK;
  };
  std::vector<Range> ranges;
  const int threads = setup_threads(g.nodes());
  for (int d = 0; d < 3; d++) {
    const int a1 = d == 0 ? 1 : 0;
    const int lo = 1, hi = n[a1] - 1;
    const int per = std::max(1, (hi - lo + 4 * threads - 1) / (4 * threads));
    for (int a = lo; a < hi; a += per) ranges.push_back(Range{d, a, std::min(hi, a + per), {}, {}, MTS_OK});
  }
  run_parts((int)ranges.size(), threads, [&](int k) {
    Range& r = ranges[k];
    r.st = crossings_of_lines(g, tags, s, beta_in, beta_out, mib, r.d, r.a, r.b, r.out, r.rep);
  });
  SetupReport rep;
  size_t total = 0;
  for (const Range& r : ranges) {
    if (r.st) return r.st;
    total += r.out.size();
  }
  out.reserve(total);
  for (const Range& r : ranges) {
    out.insert(out.end(), r.out.begin(), r.out.end());
    rep.singular_warnings += r.rep.singular_warnings;
    rep.corner_pairs += r.rep.corner_pairs;
  }
  if (report) *report = rep;
  return MTS_OK;
}

}  // namespace mts

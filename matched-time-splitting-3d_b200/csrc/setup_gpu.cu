// Problem setup on the device: the node tags (Mesh::Mesh, src/mesh/mesh.cc:57-69),
// the crossing scan with rtsafe root finding (Setup_Intersections,
// src/spatial/intersection.cc:79-291; Rtsafe_x/y/z,
// src/surface/surface_cartesian.cc:134-372) and the MIB-L1/L2 weight solves
// with their LU (intersection.cc:930-1830, src/decomposition/lu.cc:15-115).
//
// The host restatement in setup.cpp is the specification: the same routines,
// the same operand order, compiled without FMA contraction, so every +, -, *,
// / and sqrt rounds as there (IEEE double, round to nearest).  One operation
// differs: where the reference (and setup.cpp) square with glibc's
// pow(v, 2), this file multiplies v * v, the correctly rounded square; glibc's
// pow misses it in about 1 of 1200 operands by one unit in the last place.  A
// root or a normal computed from such a square can differ from the host's in
// its last bits, and with it that crossing's weights.
//
// Kernels, in order:
//   k_su_tags    one thread per node: level set, tag +1 / -1;
//   k_su_count   one thread per grid line: the scan, crossings per line;
//   k_su_scan    exclusive sum of the counts (one CTA), the list offsets;
//   k_su_cross   one thread per line with crossings: roots, normals, local
//                frames, and the weights of single crossings and MIB-L1
//                corner pairs, written at the line's offset, in the host's
//                order (direction, line, left_loc);
//   k_su_corner  one thread per MIB-L2 corner pair: the 36x36 system.
// Each thread solves its systems in a slot of shared memory (LU updates are
// serial chains of loads and stores, so they must not wait on L2).
#include <cuda_runtime.h>

#include <cstring>
#include <string>
#include <vector>

#include "setup.h"

namespace mts {
namespace {

constexpr double kTolSetup = 1.0e-12;   // src/constant.h:10
constexpr double kTolRtsafe = 1.0e-14;  // src/constant.h:11
// An LU slot of order N holds, in doubles: A (N x N), B, x, the pivot
// scales (N each) and the pivot rows (N ints); everything an LU works on
// sits there, so the kernels keep no arrays of their own in local memory.
template <int N>
constexpr int slot_doubles() {
  return (N * N + 3 * N + (N + 1) / 2 + 7) / 8 * 8;
}
constexpr int kSlotL1 = slot_doubles<8>();
constexpr int kSlotL2 = slot_doubles<12>();
constexpr int kSlotCorner = slot_doubles<36>();
template <int N>
__device__ __forceinline__ double* slot_b(double* s) { return s + N * N; }
template <int N>
__device__ __forceinline__ double* slot_x(double* s) { return s + N * N + N; }

struct SurfD {
  int kind;
  double p[7];
};

// Stands for the reference's pow(v, 2).
__device__ __forceinline__ double sqr(double v) { return v * v; }

__device__ __forceinline__ double lv_func(const SurfD& s, double x, double y, double z) {
  if (s.kind == MTS_SURFACE_ELLIPSOID) {
    const double a = s.p[0], b = s.p[1], c = s.p[2], r = s.p[3];
    const double X = x - s.p[4], Y = y - s.p[5], Z = z - s.p[6];
    return X * X / (a * a) + Y * Y / (b * b) + Z * Z / (c * c) - r * r;
  }
  const double a = s.p[0], b = s.p[1];
  return sqr(a - sqrt(x * x + y * y)) + z * z - b * b;
}

__device__ __forceinline__ double lv_df(const SurfD& s, int axis, double x, double y, double z) {
  if (s.kind == MTS_SURFACE_ELLIPSOID) {
    if (axis == 0) return 2 * (x - s.p[4]) / (s.p[0] * s.p[0]);
    if (axis == 1) return 2 * (y - s.p[5]) / (s.p[1] * s.p[1]);
    return 2 * (z - s.p[6]) / (s.p[2] * s.p[2]);
  }
  const double a = s.p[0];
  if (axis == 0) return (-2.0 * a * x) / (sqrt(x * x + y * y)) + 2.0 * x;
  if (axis == 1) return (-2.0 * a * y) / (sqrt(x * x + y * y)) + 2.0 * y;
  return 2.0 * z;
}

__device__ __forceinline__ void lv_normal(const SurfD& s, double x, double y, double z, double* n) {
  if (s.kind == MTS_SURFACE_ELLIPSOID) {
    const double a = s.p[0], b = s.p[1], c = s.p[2];
    const double X = x - s.p[4], Y = y - s.p[5], Z = z - s.p[6];
    const double total = sqrt(sqr(2 * X / (a * a)) + sqr(2 * Y / (b * b)) + sqr(2 * Z / (c * c)));
    n[0] = 2 * X / (a * a) / total;
    n[1] = 2 * Y / (b * b) / total;
    n[2] = 2 * Z / (c * c) / total;
    return;
  }
  const double a = s.p[0];
  const double total = sqrt(sqr((-2.0 * a * x) / (sqrt(x * x + y * y)) + 2.0 * x) +
                            sqr((-2.0 * a * y) / (sqrt(x * x + y * y)) + 2.0 * y) + sqr(2.0 * z));
  n[0] = ((-2.0 * a * x) / (sqrt(x * x + y * y)) + 2.0 * x) / total;
  n[1] = ((-2.0 * a * y) / (sqrt(x * x + y * y)) + 2.0 * y) / total;
  n[2] = (2.0 * z) / total;
}

// The level set along one axis, the other two coordinates fixed at (p, q)
// in axis order (x: (y, z); y: (x, z); z: (x, y)).
__device__ __forceinline__ double along_f(const SurfD& s, int axis, double v, double p, double q) {
  return axis == 0 ? lv_func(s, v, p, q) : axis == 1 ? lv_func(s, p, v, q) : lv_func(s, p, q, v);
}
__device__ __forceinline__ double along_df(const SurfD& s, int axis, double v, double p, double q) {
  return axis == 0 ? lv_df(s, 0, v, p, q) : axis == 1 ? lv_df(s, 1, p, v, q) : lv_df(s, 2, p, q, v);
}

// Newton-Raphson safeguarded by bisection (Numerical Recipes rtsafe, as
// Rtsafe_x/y/z); false when the bracket holds no sign change or 100
// iterations do not converge.
__device__ __forceinline__ bool rtsafe(const SurfD& s, int axis, double v1, double v2, double p, double q, double* root) {
  double fl = along_f(s, axis, v1, p, q);
  double fh = along_f(s, axis, v2, p, q);
  if ((fl > 0.0 && fh > 0.0) || (fl < 0.0 && fh < 0.0)) return false;
  if (fl == 0.0) {
    *root = v1;
    return true;
  }
  if (fh == 0.0) {
    *root = v2;
    return true;
  }
  double xl, xh;
  if (fl < 0.0) {
    xl = v1;
    xh = v2;
  } else {
    xh = v1;
    xl = v2;
  }
  double rts = 0.5 * (v1 + v2);
  double dxold = fabs(v2 - v1);
  double dx = dxold;
  double f = along_f(s, axis, rts, p, q);
  double df = along_df(s, axis, rts, p, q);
  for (int it = 0; it < 100; it++) {
    if ((((rts - xh) * df - f) * ((rts - xl) * df - f) > 0.0) || (fabs(2.0 * f) > fabs(dxold * df))) {
      dxold = dx;
      dx = 0.5 * (xh - xl);
      rts = xl + dx;
      if (xl == rts) {
        *root = rts;
        return true;
      }
    } else {
      dxold = dx;
      dx = f / df;
      const double temp = rts;
      rts -= dx;
      if (temp == rts) {
        *root = rts;
        return true;
      }
    }
    if (fabs(dx) < kTolRtsafe) {
      *root = rts;
      return true;
    }
    f = along_f(s, axis, rts, p, q);
    df = along_df(s, axis, rts, p, q);
    if (f < 0.0)
      xl = rts;
    else
      xh = rts;
  }
  return false;
}

// Gamma_x/y/z (surface_cartesian.cc:23-131).
__device__ __forceinline__ bool gamma_root(const SurfD& s, int axis, double v1, double v2, double p, double q, double* root) {
  if (!(v1 > v2) && !(v1 < v2)) return false;
  if (fabs(v1 - v2) < kTolRtsafe) {
    *root = (v1 + v2) / 2;
    return true;
  }
  return rtsafe(s, axis, v1, v2, p, q, root);
}

// LU with implicit partial pivoting (Numerical Recipes ludcmp / lubksb, as
// LU::LU, LU::solve and LU::det), on an N x N row-major matrix in place.
template <int N>
struct LuD {
  double* a;     // N x N, row major, factored in place
  double* vv;    // N pivot scales
  int* indx;     // N pivot rows
  double d;

  __device__ __forceinline__ bool factor() {
    const double TINY = 1.0e-40;
    d = 1.0;
    for (int i = 0; i < N; i++) {
      double big = 0.0, temp;
      for (int j = 0; j < N; j++)
        if ((temp = fabs(a[i * N + j])) > big) big = temp;
      if (big == 0.0) return false;
      vv[i] = 1.0 / big;
    }
    int imax = 0;
    for (int k = 0; k < N; k++) {
      double big = 0.0;
      for (int i = k; i < N; i++) {
        const double temp = vv[i] * fabs(a[i * N + k]);
        if (temp > big) {
          big = temp;
          imax = i;
        }
      }
      if (k != imax) {
        for (int j = 0; j < N; j++) {
          const double t = a[imax * N + j];
          a[imax * N + j] = a[k * N + j];
          a[k * N + j] = t;
        }
        d = -d;
        vv[imax] = vv[k];
      }
      indx[k] = imax;
      if (a[k * N + k] == 0.0) a[k * N + k] = TINY;
      for (int i = k + 1; i < N; i++) {
        const double temp = a[i * N + k] /= a[k * N + k];
        for (int j = k + 1; j < N; j++) a[i * N + j] -= temp * a[k * N + j];
      }
    }
    return true;
  }
  __device__ __forceinline__ void solve(const double* b, double* x) const {
    int ii = 0;
    for (int i = 0; i < N; i++) x[i] = b[i];
    for (int i = 0; i < N; i++) {
      const int ip = indx[i];
      double sum = x[ip];
      x[ip] = x[i];
      if (ii != 0)
        for (int j = ii - 1; j < i; j++) sum -= a[i * N + j] * x[j];
      else if (sum != 0.0)
        ii = i + 1;
      x[i] = sum;
    }
    for (int i = N - 1; i >= 0; i--) {
      double sum = x[i];
      for (int j = i + 1; j < N; j++) sum -= a[i * N + j] * x[j];
      x[i] = sum / a[i * N + i];
    }
  }
  __device__ double det() const {
    double dd = d;
    for (int i = 0; i < N; i++) dd *= a[i * N + i];
    return dd;
  }
};

// Solves A x = B of the slot (x into the slot); returns 0 (no pivot row),
// 1 (solved) or 2 (solved, |det| < TOL_SETUP: the reference's
// singular-matrix warning).
template <int N>
__device__ __forceinline__ int lu_solve(double* slot) {
  LuD<N> lu;
  lu.a = slot;
  lu.vv = slot + N * N + 2 * N;
  lu.indx = (int*)(slot + N * N + 3 * N);
  if (!lu.factor()) return 0;
  lu.solve(slot_b<N>(slot), slot_x<N>(slot));
  return fabs(lu.det()) < kTolSetup ? 2 : 1;
}

// Fornberg's finite-difference weights (Intersections::Weights,
// intersection.cc:5093-5130) for m = 1 on n points: c is n x 2, row major.
template <int n>
__device__ __forceinline__ void fd_weights(double z, const double* x, double* c) {
  const int m = 1, w = 2;
  double c1 = 1, c2, c3, c4 = x[0] - z, c5;
#pragma unroll
  for (int i = 0; i < n; i++)
#pragma unroll
    for (int j = 0; j < m + 1; j++) c[i * w + j] = 0;
  c[0] = 1;
#pragma unroll
  for (int i = 1; i < n; i++) {
    const int mn = i < m ? i : m;
    c2 = 1;
    c5 = c4;
    c4 = x[i] - z;
#pragma unroll
    for (int j = 0; j < i; j++) {
      c3 = x[i] - x[j];
      c2 = c2 * c3;
      if (j == i - 1) {
#pragma unroll
        for (int k = mn; k > 0; k--) c[i * w + k] = c1 * (k * c[(i - 1) * w + k - 1] - c5 * c[(i - 1) * w + k]) / c2;
        c[i * w + 0] = -c1 * c5 * c[(i - 1) * w + 0] / c2;
      }
#pragma unroll
      for (int k = mn; k > 0; k--) c[j * w + k] = (c4 * c[j * w + k] - k * c[j * w + k - 1]) / c3;
      c[j * w + 0] = c4 * c[j * w + 0] / c3;
    }
    c1 = c2;
  }
}

// w[order][j] for orders 0 (value) and 1 (first derivative).
struct Wei2 {
  double w[2][4];
};
template <int n>
__device__ __forceinline__ Wei2 weights_table(double z, const double* v) {
  double temp[4 * 2];
  fd_weights<n>(z, v, temp);
  Wei2 r;
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) r.w[i][j] = j < n ? temp[j * 2 + i] : 0.0;
  return r;
}

// MIB_L1 (intersection.cc:930-1066): the 8x8 system of one crossing.
__device__ __forceinline__ int mib_l1(double gamma, int id, double bi, double bo, double dv, double* slot) {
  const int one = 4, tot = 8;
  double* A = slot;
  double* B = slot_b<tot>(slot);
  for (int i = 0; i < tot * tot; i++) A[i] = 0.0;
  for (int i = 0; i < tot; i++) B[i] = 0.0;
  const double v[2] = {0, dv};
  const Wei2 wt = weights_table<2>(gamma, v);
  const bool even = abs(id) % 2 == 0;
  int order = 0;
  B[0] = -wt.w[order][0];
  B[1] = wt.w[order][1];
  for (int i = 0; i < one; i++) {
    A[i * tot + i] = -wt.w[order][0];
    A[i * tot + one + i] = wt.w[order][1];
  }
  if (even)
    B[one - 2] += -1;
  else
    B[one - 2] += 1;
  order = 1;
  const double coefr = even ? bi : bo;
  const double coefl = even ? bo : bi;
  B[one + 0] = -wt.w[order][0] * coefr;
  B[one + 1] = wt.w[order][1] * coefl;
  for (int i = 0; i < one; i++) {
    A[(one + i) * tot + i] = -wt.w[order][0] * coefl;
    A[(one + i) * tot + one + i] = wt.w[order][1] * coefr;
  }
  if (even)
    B[tot - 1] += -1;
  else
    B[tot - 1] += 1;
  return lu_solve<8>(slot);
}

// Irregular_MIB_L2 at second order (intersection.cc:1207-1395,
// 1424-1470): the 12x12 system of one crossing.
__device__ __forceinline__ int mib_l2(double gamma, int id, double bi, double bo, double dv, double* slot) {
  const int side = 2, st = 3, one = 6, tot = 12;
  double* A = slot;
  double* B = slot_b<tot>(slot);
  for (int i = 0; i < tot * tot; i++) A[i] = 0.0;
  for (int i = 0; i < tot; i++) B[i] = 0.0;
  double vr[3], vl[3];
  for (int i = 0; i < st; i++) {
    vr[i] = -(side - 1) * dv + i * dv;
    vl[i] = (side - st + 1) * dv + i * dv;
  }
  const Wei2 wr = weights_table<st>(gamma, vr);
  const Wei2 wl = weights_table<st>(gamma, vl);
  const bool even = abs(id) % 2 == 0;
  int order = 0;
  for (int i = 0; i < side; i++) {
    B[i] += -wr.w[order][i];
    B[side + i] += wl.w[order][st - side + i];
  }
  for (int i = 0; i < one; i++) {
    A[i * tot + i] = -wl.w[order][0];
    A[i * tot + one + i] = wr.w[order][st - 1];
  }
  if (even)
    B[one - 2] += -1;
  else
    B[one - 2] += 1;
  order = 1;
  const double coefr = even ? bi : bo;
  const double coefl = even ? bo : bi;
  for (int i = 0; i < side; i++) {
    B[one + i] += -wr.w[order][i] * coefr;
    B[one + side + i] += wl.w[order][st - side + i] * coefl;
  }
  for (int i = 0; i < one; i++) {
    A[(one + i) * tot + one + i] = wr.w[order][st - 1] * coefr;
    A[(one + i) * tot + i] = -wl.w[order][0] * coefl;
  }
  if (even)
    B[tot - 1] += -1;
  else
    B[tot - 1] += 1;
  return lu_solve<12>(slot);
}

// Corner_MIB_L2_2nd + Get_cor_weights (intersection.cc:1479-1704,
// 1752-1830): the 36x36 system of a corner pair L, R (consecutive
// crossings of one line).
__device__ __forceinline__ int corner_l2(const mts_crossing& L, const mts_crossing& R, double bi, double bo, double dv,
                         double* slot) {
  const int one = 9, tot = 36, ns = 4;
  double* A = slot;
  double* B = slot_b<tot>(slot);
  for (int i = 0; i < tot * tot; i++) A[i] = 0.0;
  for (int i = 0; i < tot; i++) B[i] = 0.0;
  auto a = [&](int i, int j) -> double& { return A[i * tot + j]; };
  const double gl = L.gamma, gr = R.gamma;
  double lvo[4], lvi[4], rvo[4], rvi[4];
  for (int i = 0; i < ns; i++) {
    lvo[i] = -dv + i * dv;
    rvo[i] = i * dv;
  }
  for (int i = 0; i < ns; i++) lvi[i] = i * dv;
  if ((dv - gl) > gr) lvi[ns - 1] = -dv;
  for (int i = 0; i < ns; i++) rvi[i] = lvi[i];
  const Wei2 lo = weights_table<ns>(gl, lvo);
  const Wei2 li = weights_table<ns>(gl, lvi);
  const Wei2 ro = weights_table<ns>(dv + gr, rvo);
  const Wei2 ri = weights_table<ns>(dv + gr, rvi);
  const bool even = abs(L.id) % 2 == 0;
  // left interface, zero order
  int order = 0;
  B[0] = -lo.w[order][0];
  B[1] = -lo.w[order][1];
  B[2] = li.w[order][1];
  B[3] = -lo.w[order][3];
  for (int i = 0; i < one; i++) {
    a(i, i) = -li.w[order][0];
    a(i, one + i) = lo.w[order][2];
    a(i, one * 2 + i) = -li.w[order][2];
    a(i, one * 3 + i) = -li.w[order][3];
  }
  B[5] = even ? -1 : 1;
  // left interface, first order
  order = 1;
  double cin = even ? bo : bi, cout_ = even ? bi : bo;
  B[one + 0] = -lo.w[order][0] * cout_;
  B[one + 1] = -lo.w[order][1] * cout_;
  B[one + 2] = li.w[order][1] * cin;
  B[one + 3] = -lo.w[order][3] * cout_;
  for (int i = 0; i < one; i++) {
    a(one + i, i) = -li.w[order][0] * cin;
    a(one + i, one + i) = lo.w[order][2] * cout_;
    a(one + i, one * 2 + i) = -li.w[order][2] * cin;
    a(one + i, one * 3 + i) = -li.w[order][3] * cin;
  }
  B[one + 6] = even ? -1 : 1;
  // right interface, zero order
  order = 0;
  B[one * 2 + 1] = -ro.w[order][0];
  B[one * 2 + 2] = ri.w[order][1];
  B[one * 2 + 3] = -ro.w[order][2];
  B[one * 2 + 4] = -ro.w[order][3];
  for (int i = 0; i < one; i++) {
    a(one * 2 + i, i) = -ri.w[order][0];
    a(one * 2 + i, one + i) = ro.w[order][1];
    a(one * 2 + i, one * 2 + i) = -ri.w[order][2];
    a(one * 2 + i, one * 3 + i) = -ri.w[order][3];
  }
  B[one * 2 + 7] = even ? -1 : 1;
  // right interface, first order (sides keyed on the left crossing's ID
  // parity, as in the reference)
  order = 1;
  cin = even ? bo : bi;
  cout_ = even ? bi : bo;
  B[one * 3 + 1] = -ro.w[order][0] * cout_;
  B[one * 3 + 2] = ri.w[order][1] * cin;
  B[one * 3 + 3] = -ro.w[order][2] * cout_;
  B[one * 3 + 4] = -ro.w[order][3] * cout_;
  for (int i = 0; i < one; i++) {
    a(one * 3 + i, i) = -ri.w[order][0] * cin;
    a(one * 3 + i, one + i) = ro.w[order][1] * cout_;
    a(one * 3 + i, one * 2 + i) = -ri.w[order][2] * cin;
    a(one * 3 + i, one * 3 + i) = -ri.w[order][3] * cin;
  }
  B[one * 3 + 8] = even ? -1 : 1;
  return lu_solve<36>(slot);
}

// Pmatrix_Setup_x/y/z (intersection.cc:2503-2598): the local frame, row
// major, with the normal as its first row.
__device__ __forceinline__ void frame(int dir, const double* a, double* p) {
  for (int i = 0; i < 3; i++) p[i] = a[i];
  if (dir == 0) {
    p[3] = a[2] / sqrt(a[0] * a[0] + a[2] * a[2]);
    p[4] = 0;
    p[5] = -a[0] / sqrt(a[0] * a[0] + a[2] * a[2]);
    p[6] = a[1] / sqrt(a[0] * a[0] + a[1] * a[1]);
    p[7] = -a[0] / sqrt(a[0] * a[0] + a[1] * a[1]);
    p[8] = 0;
  } else if (dir == 1) {
    p[3] = 0;
    p[4] = a[2] / sqrt(a[1] * a[1] + a[2] * a[2]);
    p[5] = -a[1] / sqrt(a[1] * a[1] + a[2] * a[2]);
    p[6] = a[1] / sqrt(a[0] * a[0] + a[1] * a[1]);
    p[7] = -a[0] / sqrt(a[0] * a[0] + a[1] * a[1]);
    p[8] = 0;
  } else {
    p[3] = 0;
    p[4] = a[2] / sqrt(a[1] * a[1] + a[2] * a[2]);
    p[5] = -a[1] / sqrt(a[1] * a[1] + a[2] * a[2]);
    p[6] = a[2] / sqrt(a[0] * a[0] + a[2] * a[2]);
    p[7] = 0;
    p[8] = -a[0] / sqrt(a[0] * a[0] + a[2] * a[2]);
  }
}

// Everything the kernels share.
struct SetupArgs {
  SurfD s;
  int n[3];
  double h[3];
  const double* ax[3];  // node coordinates per axis
  int8_t* tags;
  long long lines[3];   // lines per direction (interior lines only)
  int* counts;          // crossings per line, in line order
  uint8_t* lerr;        // the scan of this line fails
  int* offs;            // exclusive sum of counts; offs[total lines] = all
  mts_crossing* out;
  int* corner_list;     // offsets of the left crossings of MIB-L2 pairs
  int* ctrl;            // [0] node on the interface, [1] corner pairs, [2] L2 pairs listed,
                        // [3] first failing line (INT_MAX: none), [4] its status
  unsigned long long* singular;
  double bi, bo;
  int mib;
};

constexpr int kCtrlTagErr = 0, kCtrlCorners = 1, kCtrlListed = 2, kCtrlFirstBad = 3;
constexpr int kCtrlInts = 8;

__global__ void k_su_tags(const SetupArgs A) {
  const long long N = (long long)A.n[0] * A.n[1] * A.n[2];
  for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < N; m += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(m % A.n[0]);
    const long long r = m / A.n[0];
    const int iy = (int)(r % A.n[1]);
    const int iz = (int)(r / A.n[1]);
    const double v = lv_func(A.s, A.ax[0][ix], A.ax[1][iy], A.ax[2][iz]) + kTolSetup;
    int8_t t = 0;
    if (v > kTolSetup)
      t = 1;
    else if (v < kTolSetup)
      t = -1;
    else
      atomicExch(&A.ctrl[kCtrlTagErr], 1);  // "Interface on grid, reset the mesh!"
    A.tags[m] = t;
  }
}

// Line l (global order: direction, then i1, then i2) as (d, i1, i2).
__device__ __forceinline__ void line_of(const SetupArgs& A, long long l, int& d, int& i1, int& i2) {
  d = 0;
  while (d < 2 && l >= A.lines[d]) l -= A.lines[d++];
  const int a2 = d == 2 ? 1 : 2;
  const int w = A.n[a2] - 2;
  i1 = 1 + (int)(l / w);
  i2 = 1 + (int)(l % w);
}

// Node indices of row j of line (d, i1, i2): the line's fixed axes are
// (y, z) for x lines, (x, z) for y lines and (x, y) for z lines.
__device__ __forceinline__ void node_ijk(int d, int i1, int i2, int j, int& ix, int& iy, int& iz) {
  ix = d == 0 ? j : i1;
  iy = d == 0 ? i1 : d == 1 ? j : i2;
  iz = d == 2 ? j : i2;
}

__device__ __forceinline__ long long node_of(const SetupArgs& A, int d, int i1, int i2, int j) {
  int ix, iy, iz;
  node_ijk(d, i1, i2, j, ix, iy, iz);
  return (long long)ix + (long long)A.n[0] * ((long long)iy + (long long)A.n[1] * iz);
}

__global__ void k_su_count(const SetupArgs A, long long total_lines) {
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < total_lines;
       l += (long long)gridDim.x * blockDim.x) {
    int d, i1, i2;
    line_of(A, l, d, i1, i2);
    const long long s0 = node_of(A, d, i1, i2, 0);
    const long long st = node_of(A, d, i1, i2, 1) - s0;
    auto tag = [&](int j) { return (int)A.tags[s0 + st * j]; };
    const int nd = A.n[d];
    int cnt = 0, ifp = 0, pairs = 0;
    bool bad = false;
    int j = 1;
    while (j < nd - 1) {
      if (tag(j) * tag(j + 1) < 0) {
        if (j + 2 >= nd) {
          bad = true;
          break;
        }
        if (tag(j + 1) * tag(j + 2) > 0) {
          ifp += 1;
          cnt += 1;
          j += 2;
        } else {
          if (j + 3 >= nd || tag(j + 2) * tag(j + 3) < 0) {
            bad = true;
            break;
          }
          ifp += 2;
          cnt += 2;
          pairs += 1;
          j += 3;
        }
      } else {
        j += 1;
      }
    }
    if (!bad && ifp % 2 == 1) bad = true;
    A.counts[l] = cnt;
    A.lerr[l] = bad;
    if (pairs) atomicAdd(&A.ctrl[kCtrlCorners], pairs);
  }
}

// Exclusive sum of counts[0..n) into offs[0..n], one CTA of 1024 threads,
// each over a contiguous chunk.
__global__ void __launch_bounds__(1024) k_su_scan(const int* __restrict__ counts, int* __restrict__ offs, long long n) {
  __shared__ long long part[1024];
  const long long per = (n + 1023) / 1024;
  const long long a = threadIdx.x * per, b = a + per < n ? a + per : n;
  long long s = 0;
  for (long long i = a; i < b; i++) s += counts[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    const long long v = threadIdx.x >= off ? part[threadIdx.x - off] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  long long run = part[threadIdx.x] - s;
  for (long long i = a; i < b; i++) {
    offs[i] = (int)run;
    run += counts[i];
  }
  if (threadIdx.x == 1023) offs[n] = (int)part[1023];
}

__device__ __forceinline__ void note_failure(const SetupArgs& A, long long l, int status) {
  // the first failing line in line order decides the status, as in one pass
  const int prev = atomicMin(&A.ctrl[kCtrlFirstBad], (int)l);
  (void)prev;
  A.lerr[l] = (uint8_t)status;
}

// Root, coordinates, normal and frame of the crossing in cell [j, j+1] of
// line (d, i1, i2); the record's other fields stay zero.
__device__ __forceinline__ bool locate(const SetupArgs& A, int d, int i1, int i2, int j, int id, mts_crossing* c) {
  const double* v = d == 0 ? A.ax[0] : d == 1 ? A.ax[1] : A.ax[2];
  const double fp = d == 0 ? A.ax[1][i1] : A.ax[0][i1];
  const double fq = d == 2 ? A.ax[1][i2] : A.ax[2][i2];
  double root;
  if (!gamma_root(A.s, d, v[j], v[j + 1], fp, fq, &root)) return false;
  int ix, iy, iz;
  node_ijk(d, i1, i2, j, ix, iy, iz);
  c->dir = d;
  c->indx1 = i1;
  c->indx2 = i2;
  c->id = id;
  c->left_loc = j;
  const double cx = d == 0 ? root : A.ax[0][ix];
  const double cy = d == 1 ? root : A.ax[1][iy];
  const double cz = d == 2 ? root : A.ax[2][iz];
  c->coord[0] = cx;
  c->coord[1] = cy;
  c->coord[2] = cz;
  c->gamma = root - v[j];
  double nrm[3], p[9];
  lv_normal(A.s, cx, cy, cz, nrm);
  frame(d, nrm, p);
  for (int k = 0; k < 3; k++) c->normal[k] = nrm[k];
  for (int k = 0; k < 9; k++) c->p[k] = p[k];
  return true;
}

__device__ __forceinline__ void count_singular(const SetupArgs& A, int r) {
  if (r == 2) atomicAdd(A.singular, 1ULL);
}

constexpr int kCrossThreads = 32;  // x one LU slot of shared memory each: 48 KB at MIB-L2

__global__ void __launch_bounds__(kCrossThreads) k_su_cross(const SetupArgs A, long long total_lines) {
  extern __shared__ double su_smem[];
  double* const M = su_smem + threadIdx.x * (A.mib == 1 ? kSlotL1 : kSlotL2);
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < total_lines;
       l += (long long)gridDim.x * blockDim.x) {
    if (A.counts[l] == 0 && !A.lerr[l]) continue;
    int d, i1, i2;
    line_of(A, l, d, i1, i2);
    const long long s0 = node_of(A, d, i1, i2, 0);
    const long long st = node_of(A, d, i1, i2, 1) - s0;
    auto tag = [&](int j) { return (int)A.tags[s0 + st * j]; };
    const int nd = A.n[d];
    const double dv = A.h[d];
    int k = A.offs[l];
    int ifp = 0, j = 1, status = 0;
    while (j < nd - 1) {
      if (tag(j) * tag(j + 1) < 0) {
        if (j + 2 >= nd) {
          status = MTS_ERR_SETUP;  // a crossing in the last cell
          break;
        }
        if (tag(j + 1) * tag(j + 2) > 0) {
          ifp += 1;
          mts_crossing* c = A.out + k;
          if (!locate(A, d, i1, i2, j, ifp, c)) {
            status = MTS_ERR_NONFINITE;
            break;
          }
          if (A.mib == 1) {
            const int r = mib_l1(c->gamma, c->id, A.bi, A.bo, dv, M);
            const double* x = slot_x<8>(M);
            if (!r) {
              status = MTS_ERR_SETUP;
              break;
            }
            count_singular(A, r);
            c->nwei = 6;
            c->weil[1] = x[0];
            c->weil[2] = x[1];
            c->weil[4] = x[2];
            c->weil[5] = x[3];
            c->weir[1] = x[4];
            c->weir[2] = x[5];
            c->weir[4] = x[6];
            c->weir[5] = x[7];
          } else {
            const int r = mib_l2(c->gamma, c->id, A.bi, A.bo, dv, M);
            const double* x = slot_x<12>(M);
            if (!r) {
              status = MTS_ERR_SETUP;
              break;
            }
            count_singular(A, r);
            c->nwei = 6;
            for (int q = 0; q < 6; q++) {
              c->weil[q] = x[q];
              c->weir[q] = x[6 + q];
            }
          }
          k += 1;
          j += 2;
        } else {
          if (j + 3 >= nd || tag(j + 2) * tag(j + 3) < 0) {
            status = MTS_ERR_SETUP;  // corners that do not pair up
            break;
          }
          mts_crossing* L = A.out + k;
          mts_crossing* R = L + 1;
          ifp += 1;
          if (!locate(A, d, i1, i2, j, -ifp, L)) {
            status = MTS_ERR_NONFINITE;
            break;
          }
          ifp += 1;
          if (!locate(A, d, i1, i2, j + 1, -ifp, R)) {
            status = MTS_ERR_NONFINITE;
            break;
          }
          if (A.mib == 1) {
            // Corner_MIB_L1 (intersection.cc:1128-1200): each crossing alone
            const int r1 = mib_l1(L->gamma, L->id, A.bi, A.bo, dv, M);
            const double* x = slot_x<8>(M);
            if (!r1) {
              status = MTS_ERR_SETUP;
              break;
            }
            L->nwei = 9;
            R->nwei = 9;
            L->weil[1] = x[0];
            L->weil[2] = x[1];
            L->weil[5] = x[2];
            L->weil[6] = x[3];
            L->weir[1] = x[4];
            L->weir[2] = x[5];
            L->weir[5] = x[6];
            L->weir[6] = x[7];
            const int r2 = mib_l1(R->gamma, R->id, A.bi, A.bo, dv, M);
            if (!r2) {
              status = MTS_ERR_SETUP;
              break;
            }
            R->weil[2] = x[0];
            R->weil[3] = x[1];
            R->weil[7] = x[2];
            R->weil[8] = x[3];
            R->weir[2] = x[4];
            R->weir[3] = x[5];
            R->weir[7] = x[6];
            R->weir[8] = x[7];
            count_singular(A, (r1 == 2 || r2 == 2) ? 2 : 1);
          } else {
            A.corner_list[atomicAdd(&A.ctrl[kCtrlListed], 1)] = k;  // the 36x36 solve runs next
          }
          k += 2;
          j += 3;
        }
      } else {
        j += 1;
      }
    }
    if (!status && ifp % 2 == 1) status = MTS_ERR_SETUP;  // an open surface
    if (status) note_failure(A, l, status);
  }
}

// One thread per CTA, its 36x36 slot (11.4 KB) in shared memory.
__global__ void __launch_bounds__(1) k_su_corner(const SetupArgs A) {
  extern __shared__ double su_smem[];
  const int i = blockIdx.x;
  if (i >= A.ctrl[kCtrlListed]) return;
  const int k = A.corner_list[i];
  mts_crossing* L = A.out + k;
  mts_crossing* R = L + 1;
  double* M = su_smem;
  const int r = corner_l2(*L, *R, A.bi, A.bo, A.h[L->dir], M);
  const double* x = slot_x<36>(M);
  if (!r) {
    const int d = L->dir;
    long long l = (long long)(L->indx1 - 1) * (A.n[d == 2 ? 1 : 2] - 2) + (L->indx2 - 1);
    for (int e = 0; e < d; e++) l += A.lines[e];
    note_failure(A, l, MTS_ERR_SETUP);
    return;
  }
  count_singular(A, r);
  L->nwei = 9;
  R->nwei = 9;
  for (int q = 0; q < 9; q++) {
    L->weil[q] = x[q];
    L->weir[q] = x[9 + q];
    R->weil[q] = x[9 + q];
    R->weir[q] = x[18 + q];
  }
}

int grid_for(long long work, int threads) {
  long long b = (work + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > 148LL * 64) b = 148LL * 64;
  return (int)b;
}

}  // namespace

mts_status setup_on_device(const Grid& g, const mts_surface& surf, double beta_in, double beta_out, int mib,
                           void* stream, std::vector<int8_t>& tags, std::vector<mts_crossing>& out,
                           SetupReport* report, std::string* why) {
  cudaStream_t st = (cudaStream_t)stream;
  std::vector<void*> owned;
  auto release = [&] {
    for (void* p : owned) cudaFreeAsync(p, st);
    cudaStreamSynchronize(st);
    owned.clear();
  };
  auto cuda_fail = [&](cudaError_t e, const char* what) {
    if (why) *why = std::string("device setup, ") + what + ": " + cudaGetErrorString(e);
    release();
    return e == cudaErrorMemoryAllocation ? MTS_ERR_OOM : MTS_ERR_CUDA;
  };
  auto alloc = [&](size_t bytes, void** p) {
    *p = nullptr;
    cudaError_t e = cudaMallocAsync(p, bytes > 0 ? bytes : 16, st);
    if (e == cudaSuccess) owned.push_back(*p);
    return e;
  };
#define SU_TRY(call, what)                  \
  do {                                      \
    cudaError_t e_ = (call);                \
    if (e_ != cudaSuccess) return cuda_fail(e_, what); \
  } while (0)

  if (mib != 1 && mib != 2) return MTS_ERR_ARG;
  SetupArgs A;
  std::memset(&A, 0, sizeof A);
  A.s.kind = surf.kind;
  for (int k = 0; k < 7; k++) A.s.p[k] = surf.params[k];
  A.n[0] = g.nx;
  A.n[1] = g.ny;
  A.n[2] = g.nz;
  A.h[0] = g.dx;
  A.h[1] = g.dy;
  A.h[2] = g.dz;
  long long total_lines = 0;
  for (int d = 0; d < 3; d++) {
    const int a1 = d == 0 ? 1 : 0, a2 = d == 2 ? 1 : 2;
    A.lines[d] = (long long)(A.n[a1] - 2) * (A.n[a2] - 2);
    total_lines += A.lines[d];
  }
  A.bi = beta_in;
  A.bo = beta_out;
  A.mib = mib;
  const long long N = g.nodes();

  // first allocation: coordinates, tags, per-line counts, offsets, flags, control
  const size_t ncoord = (size_t)g.nx + g.ny + g.nz;
  const size_t off_tags = ncoord * 8;
  const size_t off_counts = (off_tags + (size_t)N + 15) / 16 * 16;
  const size_t off_offs = off_counts + (size_t)total_lines * 4;
  const size_t off_lerr = (off_offs + ((size_t)total_lines + 1) * 4 + 15) / 16 * 16;
  const size_t off_ctrl = (off_lerr + (size_t)total_lines + 15) / 16 * 16;
  const size_t bytes1 = off_ctrl + kCtrlInts * 4 + 8;
  char* base = nullptr;
  SU_TRY(alloc(bytes1, (void**)&base), "allocation");
  double* coords = (double*)base;
  A.ax[0] = coords;
  A.ax[1] = coords + g.nx;
  A.ax[2] = coords + g.nx + g.ny;
  A.tags = (int8_t*)(base + off_tags);
  A.counts = (int*)(base + off_counts);
  A.offs = (int*)(base + off_offs);
  A.lerr = (uint8_t*)(base + off_lerr);
  A.ctrl = (int*)(base + off_ctrl);
  A.singular = (unsigned long long*)(base + off_ctrl + kCtrlInts * 4);
  int ctrl0[kCtrlInts + 2] = {0, 0, 0, 0x7fffffff, 0, 0, 0, 0, 0, 0};
  SU_TRY(cudaMemcpyAsync(A.ctrl, ctrl0, sizeof ctrl0, cudaMemcpyHostToDevice, st), "control upload");
  SU_TRY(cudaMemcpyAsync((void*)A.ax[0], g.x.data(), g.nx * 8, cudaMemcpyHostToDevice, st), "coordinate upload");
  SU_TRY(cudaMemcpyAsync((void*)A.ax[1], g.y.data(), g.ny * 8, cudaMemcpyHostToDevice, st), "coordinate upload");
  SU_TRY(cudaMemcpyAsync((void*)A.ax[2], g.z.data(), g.nz * 8, cudaMemcpyHostToDevice, st), "coordinate upload");

  k_su_tags<<<grid_for(N, 256), 256, 0, st>>>(A);
  k_su_count<<<grid_for(total_lines, 128), 128, 0, st>>>(A, total_lines);
  k_su_scan<<<1, 1024, 0, st>>>(A.counts, A.offs, total_lines);
  SU_TRY(cudaGetLastError(), "launch");
  int ctrl[kCtrlInts];
  int total = 0;
  SU_TRY(cudaMemcpyAsync(ctrl, A.ctrl, sizeof ctrl, cudaMemcpyDeviceToHost, st), "control read");
  SU_TRY(cudaMemcpyAsync(&total, A.offs + total_lines, 4, cudaMemcpyDeviceToHost, st), "count read");
  SU_TRY(cudaStreamSynchronize(st), "scan");
  if (ctrl[kCtrlTagErr]) {
    if (why) *why = "a grid node lies on the interface";
    release();
    return MTS_ERR_SETUP;
  }
  const int corners = ctrl[kCtrlCorners];

  // second allocation: the records and the list of MIB-L2 corner pairs
  const size_t b_out = ((size_t)total * sizeof(mts_crossing) + 255) / 256 * 256;
  const size_t ncs = mib == 2 ? (size_t)corners : 0;
  char* base2 = nullptr;
  SU_TRY(alloc(b_out + ncs * 4, (void**)&base2), "allocation");
  A.out = (mts_crossing*)base2;
  A.corner_list = (int*)(base2 + b_out);
  SU_TRY(cudaMemsetAsync(A.out, 0, (size_t)total * sizeof(mts_crossing), st), "clear");
  const size_t cross_smem = (size_t)kCrossThreads * (mib == 1 ? kSlotL1 : kSlotL2) * sizeof(double);
  k_su_cross<<<grid_for(total_lines, kCrossThreads), kCrossThreads, cross_smem, st>>>(A, total_lines);
  if (mib == 2 && corners > 0) k_su_corner<<<corners, 1, kSlotCorner * sizeof(double), st>>>(A);
  SU_TRY(cudaGetLastError(), "launch");
  unsigned long long singular = 0;
  SU_TRY(cudaMemcpyAsync(ctrl, A.ctrl, sizeof ctrl, cudaMemcpyDeviceToHost, st), "control read");
  SU_TRY(cudaMemcpyAsync(&singular, A.singular, 8, cudaMemcpyDeviceToHost, st), "control read");
  SU_TRY(cudaStreamSynchronize(st), "crossings");
  if (ctrl[kCtrlFirstBad] != 0x7fffffff) {
    uint8_t s8 = 0;
    SU_TRY(cudaMemcpyAsync(&s8, A.lerr + ctrl[kCtrlFirstBad], 1, cudaMemcpyDeviceToHost, st), "status read");
    SU_TRY(cudaStreamSynchronize(st), "status read");
    if (why) *why = "interface setup failed (root finding, coherent corners, open surface or singular LU)";
    release();
    return s8 == MTS_ERR_NONFINITE ? MTS_ERR_NONFINITE : MTS_ERR_SETUP;
  }
  tags.resize((size_t)N);
  out.resize((size_t)total);
  SU_TRY(cudaMemcpyAsync(tags.data(), A.tags, (size_t)N, cudaMemcpyDeviceToHost, st), "tag read");
  if (total > 0)
    SU_TRY(cudaMemcpyAsync(out.data(), A.out, (size_t)total * sizeof(mts_crossing), cudaMemcpyDeviceToHost, st),
           "crossing read");
  SU_TRY(cudaStreamSynchronize(st), "read back");
  release();
  if (report) {
    report->corner_pairs = corners;
    report->singular_warnings = (int64_t)singular;
  }
#undef SU_TRY
  return MTS_OK;
}

}  // namespace mts

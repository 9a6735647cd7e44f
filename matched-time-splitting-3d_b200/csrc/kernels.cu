// Time-stepping kernels for sm_100a.
//
// Each directional pass is one kernel with one thread per grid line: the
// thread builds the right-hand side of its line on the fly (3-point stencils,
// exact-solution source/boundary data, MIB fictitious-point rows), runs the
// Thomas forward elimination with the line's MIB row blocks spliced in, and
// back-substitutes.  Lines along y and z are handled by consecutive threads at
// consecutive x, so every load and store of a warp is one contiguous 256-byte
// segment.  The forward factors c_{j-1}/bet go to a scratch field and the
// partial solutions d'_j to the output field; both are read back by the same
// thread microseconds later, from L2.
//
// The file is compiled with -fmad=false: every product and sum is rounded on
// its own, in the operand order of the reference statement it restates, which
// makes the plain FP64 path bit-identical to the reference CPU build.
#include <cuda_runtime.h>

#include "device.h"

namespace mts {
namespace {

constexpr int TPB = 128;

enum Kind { K_ADI_X = 0, K_COPY = 1, K_ADI_Z = 2, K_LOD = 3, K_TS_Z = 4 };

struct SweepIO {
  const double* stin;  // field the stencil of the explicit part reads
  const double* add;   // field added to the explicit part (or copied)
  double* out;         // result field (holds d'_j during the forward pass)
  double e1;           // exp(-t_next): boundary data, source, jumps
  double e0;           // exp(-t_prev) (TS source of the first half step)
  int jumps;           // implicit MIB rows carry jump terms (LOD, TS)
  int cn;              // LOD: Crank-Nicolson explicit part
  int last;            // LOD: epilogue adds dt*f(t_next)
};

// ---------------------------------------------------------------------------
// Exact solutions (eq 0: src/equation/eq_0.cc; eq 8: see oracle/ref_harness.cc
// Eq8 for the operand order).

__device__ __forceinline__ double outer_u(const Dev& P, double E, int ix, int iy, int iz) {
  if (P.eq == 0) return 100.0;
  double x = P.ax[0][ix], y = P.ax[1][iy], z = P.ax[2][iz];
  return ((x * x + y * y) + z * z) * E;
}
__device__ __forceinline__ double inner_u(const Dev& P, double E, int ix, int iy, int iz) {
  if (P.eq == 0) return 80.0;
  return ((P.s2[0][ix] * P.c2[1][iy]) * P.s2[2][iz]) * E;
}
__device__ __forceinline__ double source(const Dev& P, double E, bool out, int ix, int iy, int iz) {
  if (P.eq == 0) return 0.0;
  if (out) return -outer_u(P, E, ix, iy, iz) - P.c6bo * E;
  return P.kin * inner_u(P, E, ix, iy, iz);
}

// ---------------------------------------------------------------------------
// Line geometry.  Direction D lines are indexed (i1, i2) as in the reference
// (src/constant.h:83-89): x -> (iy, iz), y -> (ix, iz), z -> (ix, iy); the
// thread index runs over i1 fastest.

struct Line {
  long long base, s;
  int n, lid, i1, i2;
  bool boundary;
};

template <int D>
__device__ __forceinline__ bool decode_line(const Dev& P, long long t, Line& L) {
  int n1 = D == 0 ? P.ny : P.nx;
  int n2 = D == 2 ? P.ny : P.nz;
  if (t >= (long long)n1 * n2) return false;
  L.i1 = (int)(t % n1);
  L.i2 = (int)(t / n1);
  L.lid = L.i1 * n2 + L.i2;
  if (D == 0) {
    L.base = (long long)P.nx * (L.i1 + (long long)P.ny * L.i2);
    L.s = 1;
    L.n = P.nx;
  } else if (D == 1) {
    L.base = L.i1 + (long long)P.nx * P.ny * L.i2;
    L.s = P.nx;
    L.n = P.ny;
  } else {
    L.base = L.i1 + (long long)P.nx * L.i2;
    L.s = (long long)P.nx * P.ny;
    L.n = P.nz;
  }
  L.boundary = L.i1 == 0 || L.i1 == n1 - 1 || L.i2 == 0 || L.i2 == n2 - 1;
  return true;
}

template <int D>
__device__ __forceinline__ void node_of(const Line& L, int j, int& ix, int& iy, int& iz) {
  if (D == 0) {
    ix = j;
    iy = L.i1;
    iz = L.i2;
  } else if (D == 1) {
    ix = L.i1;
    iy = j;
    iz = L.i2;
  } else {
    ix = L.i1;
    iy = L.i2;
    iz = j;
  }
}

// ---------------------------------------------------------------------------
// MIB rows

__device__ __forceinline__ double corner_jumps(const double* w, double2 l, double2 r) {
  return l.x * w[5] + l.y * w[6] + r.x * w[7] + r.y * w[8];
}

// Explicit 3-point sum of row r of block b with fictitious points, before the
// dt factor: the MIB branches of douglas_adi.cc:112-210 (jumps = 0) and
// lod.cc:337-496 (jumps = 1).
__device__ double mib_sum(const MibBlock& b, int r, const double* in, long long base, long long s,
                          const double* vd, bool jumps, const double2* jv) {
  const int L = b.L;
#define U(j) in[base + (long long)(j) * s]
  double sum = 0.0;
  if (b.kind == 2) {
    if (r == 0) {
      sum += vd[0] * U(L - 1);
      sum += vd[1] * U(L);
      for (int i = 0; i < 4; i++) sum += vd[2] * U(L - 1 + i) * b.w[1][i];
      if (jumps) {
        double2 J = jv[b.c0];
        sum += vd[2] * (J.x * b.w[1][4] + J.y * b.w[1][5]);
      }
    } else {
      sum += vd[1] * U(L + 1);
      sum += vd[2] * U(L + 2);
      for (int i = 0; i < 4; i++) sum += vd[0] * U(L - 1 + i) * b.w[0][i];
      if (jumps) {
        double2 J = jv[b.c0];
        sum += vd[0] * (J.x * b.w[0][4] + J.y * b.w[0][5]);
      }
    }
  } else {
    double2 Jl = make_double2(0, 0), Jr = make_double2(0, 0);
    if (jumps) {
      Jl = jv[b.c0];
      Jr = jv[b.c1];
    }
    if (r == 0) {
      sum += vd[0] * U(L - 1);
      sum += vd[1] * U(L);
      for (int i = 0; i < 5; i++) sum += vd[2] * U(L - 1 + i) * b.w[1][i];
      if (jumps) sum += vd[2] * corner_jumps(b.w[1], Jl, Jr);
    } else if (r == 1) {
      for (int i = 0; i < 5; i++) sum += vd[0] * U(L - 1 + i) * b.w[0][i];
      if (jumps) sum += vd[0] * corner_jumps(b.w[0], Jl, Jr);
      sum += vd[1] * U(L + 1);
      for (int i = 0; i < 5; i++) sum += vd[2] * U(L - 1 + i) * b.w[3][i];
      if (jumps) sum += vd[2] * corner_jumps(b.w[3], Jl, Jr);
    } else {
      sum += vd[1] * U(L + 2);
      sum += vd[2] * U(L + 3);
      for (int i = 0; i < 5; i++) sum += vd[0] * U(L - 1 + i) * b.w[2][i];
      if (jumps) sum += vd[0] * corner_jumps(b.w[2], Jl, Jr);
    }
  }
#undef U
  return sum;
}

// Douglas-ADI source jump terms of row r (Src_2nd, douglas_adi.cc:1156-1427).
__device__ __forceinline__ double adi_src_add(double src, const MibBlock& b, int r, const double* vd,
                                              const double2* jv) {
  if (b.kind == 2) {
    double2 J = jv[b.c0];
    if (r == 0) return src + vd[2] * (J.x * b.w[1][4] + J.y * b.w[1][5]);
    return src + vd[0] * (J.x * b.w[0][4] + J.y * b.w[0][5]);
  }
  double2 Jl = jv[b.c0], Jr = jv[b.c1];
  if (r == 0) return src + vd[2] * corner_jumps(b.w[1], Jl, Jr);
  if (r == 1) {
    src = src + vd[0] * corner_jumps(b.w[0], Jl, Jr);
    return src + vd[2] * corner_jumps(b.w[3], Jl, Jr);
  }
  return src + vd[0] * corner_jumps(b.w[2], Jl, Jr);
}

// LOD/TS: jump terms on the right-hand side of the implicit MIB rows
// (D_xx_l, lod.cc:960-1097), then the Convert2Tri row operations.
__device__ __forceinline__ void implicit_rows(const Dev& P, const MibBlock& b, double* r,
                                              const double (*vd)[3], bool jumps, const double2* jv) {
  const double cdt = P.cdt;
  if (jumps) {
    if (b.kind == 2) {
      double2 J = jv[b.c0];
      r[0] = r[0] + cdt * vd[0][2] * (J.x * b.w[1][4] + J.y * b.w[1][5]);
      r[1] = r[1] + cdt * vd[1][0] * (J.x * b.w[0][4] + J.y * b.w[0][5]);
    } else {
      double2 Jl = jv[b.c0], Jr = jv[b.c1];
      r[0] = r[0] + cdt * vd[0][2] * corner_jumps(b.w[1], Jl, Jr);
      r[1] = r[1] + cdt * vd[1][0] * corner_jumps(b.w[0], Jl, Jr);
      r[1] += cdt * vd[1][2] * corner_jumps(b.w[3], Jl, Jr);
      r[2] = r[2] + cdt * vd[2][0] * corner_jumps(b.w[2], Jl, Jr);
    }
  }
  if (b.kind == 2) {
    r[1] -= b.rate[0] * r[0];
    r[0] -= b.rate[1] * r[1];
  } else {
    r[1] -= b.rate[0] * r[0];
    r[2] -= b.rate[1] * r[0];
    r[0] -= b.rate[2] * r[2];
    r[1] -= b.rate[3] * r[2];
    r[2] -= b.rate[4] * r[1];
    r[0] -= b.rate[5] * r[1];
  }
}

template <int DD>
__device__ __forceinline__ const MibBlock* find_block(const Dev& P, int lid, int j, int& row) {
  int be = P.bstart[DD][lid + 1];
  for (int k = P.bstart[DD][lid]; k < be; k++) {
    const MibBlock* b = &P.blk[DD][k];
    if (j >= b->L && j < b->L + b->kind) {
      row = j - b->L;
      return b;
    }
  }
  row = 0;
  return nullptr;
}

// ---------------------------------------------------------------------------
// Right-hand sides

// Douglas-ADI first stage at node (ix,iy,iz) (douglas_adi.cc:89-359):
//   ((dt*D_yy u + dt*D_zz u) + u) + dt*src,  src = f + x, y, z jump terms.
// xb/xr: the node's row in an x block of the thread's own line (or null).
__device__ double adi_x_rhs(const Dev& P, const SweepIO& io, int ix, int iy, int iz, long long m,
                            const MibBlock* xb, int xr, double& ydt) {
  const double* un = io.stin;
  const uint8_t tg = P.tag[m];
  const int side = tg & TAG_OUT;
  const double dt = P.dt;
  const long long sy = P.nx, sz = (long long)P.nx * P.ny;
  const double* vdy = P.vd[1][side];
  const double* vdz = P.vd[2][side];
  const MibBlock* yb = nullptr;
  const MibBlock* zb = nullptr;
  int yr = 0, zr = 0;
  double sum;
  if (tg & TAG_MIBY) yb = find_block<1>(P, ix * P.nz + iz, iy, yr);
  if (yb) {
    sum = mib_sum(*yb, yr, un, ix + sz * iz, sy, vdy, false, P.jv);
    ydt = sum * dt;
  } else {
    sum = 0.0;
    sum += un[m - sy] * vdy[0];
    sum += un[m] * vdy[1];
    sum += un[m + sy] * vdy[2];
    ydt = dt * sum;
  }
  double zdt;
  if (tg & TAG_MIBZ) zb = find_block<2>(P, ix * P.ny + iy, iz, zr);
  if (zb) {
    sum = mib_sum(*zb, zr, un, ix + (long long)P.nx * iy, sz, vdz, false, P.jv);
    zdt = sum * dt;
  } else {
    sum = 0.0;
    sum += un[m - sz] * vdz[0];
    sum += un[m] * vdz[1];
    sum += un[m + sz] * vdz[2];
    zdt = dt * sum;
  }
  double src = source(P, io.e1, side, ix, iy, iz);
  if (xb) src = adi_src_add(src, *xb, xr, P.vd[0][side], P.jv);
  if (yb) src = adi_src_add(src, *yb, yr, vdy, P.jv);
  if (zb) src = adi_src_add(src, *zb, zr, vdz, P.jv);
  double r = ydt + zdt;
  r += un[m];
  r += dt * src;
  return r;
}

// Own-line explicit part value before the additive field: k * sum.
template <int D>
__device__ __forceinline__ double own_explicit(const Dev& P, const Line& L, int j, long long m, int side,
                                               const double* in, const MibBlock* b, int r, bool jumps,
                                               double k) {
  const double* vd = P.vd[D][side];
  double sum;
  if (b) {
    sum = mib_sum(*b, r, in, L.base, L.s, vd, jumps, P.jv);
  } else {
    sum = 0.0;
    sum += in[m - L.s] * vd[0];
    sum += in[m] * vd[1];
    sum += in[m + L.s] * vd[2];
  }
  return k * sum;
}

// Right-hand side of interior row j of the line (b/r: the row's own block).
template <int D, int KIND>
__device__ __forceinline__ double line_rhs(const Dev& P, const SweepIO& io, const Line& L, int j,
                                           const MibBlock* b, int r) {
  int ix, iy, iz;
  node_of<D>(L, j, ix, iy, iz);
  const long long m = L.base + (long long)j * L.s;
  const int side = P.tag[m] & TAG_OUT;
  if (KIND == K_COPY) {
    return io.add[m];
  } else if (KIND == K_ADI_X) {
    double ydt;
    double v = adi_x_rhs(P, io, ix, iy, iz, m, b, r, ydt);
    P.ydt[m] = ydt;
    return v;
  } else if (KIND == K_ADI_Z) {
    // uh1 = -dt * D_zz u^n + u**  (douglas_adi.cc:811-940)
    return own_explicit<D>(P, L, j, m, side, io.stin, b, r, false, -P.dt) + io.add[m];
  } else if (KIND == K_LOD) {
    if (!io.cn) return io.add[m];
    return own_explicit<D>(P, L, j, m, side, io.stin, b, r, true, P.kex) + io.add[m];
  } else {  // K_TS_Z: explicit z half step, then the two half-step sources
    double v = own_explicit<D>(P, L, j, m, side, io.stin, b, r, true, P.kex) + io.add[m];
    v = v + P.hdt * source(P, io.e0, side, ix, iy, iz);
    v = v + P.hdt * source(P, io.e1, side, ix, iy, iz);
    return v;
  }
}

template <int D, int KIND>
__device__ __forceinline__ double boundary_value(const Dev& P, const SweepIO& io, const Line& L, int j) {
  int ix, iy, iz;
  node_of<D>(L, j, ix, iy, iz);
  if (KIND == K_COPY) return io.add[L.base + (long long)j * L.s];
  return outer_u(P, io.e1, ix, iy, iz);
}

// ---------------------------------------------------------------------------
// The sweep kernel: one implicit line solve per thread.

template <int D, int KIND>
__global__ void __launch_bounds__(TPB) k_sweep(const Dev P, const SweepIO io) {
  Line L;
  long long t = (long long)blockIdx.x * TPB + threadIdx.x;
  if (!decode_line<D>(P, t, L)) return;
  const int n = L.n;
  if (L.boundary) {
    if (KIND == K_COPY) return;  // in place: boundary faces already hold Outer_u
    for (int j = 0; j < n; j++) {
      int ix, iy, iz;
      node_of<D>(L, j, ix, iy, iz);
      long long m = L.base + (long long)j * L.s;
      double v = outer_u(P, io.e1, ix, iy, iz);
      if (KIND == K_LOD && io.last) v = v + P.dt * source(P, io.e1, P.tag[m] & TAG_OUT, ix, iy, iz);
      io.out[m] = v;
    }
    return;
  }
  double* __restrict__ out = io.out;
  double* __restrict__ gam = P.gam;
  const MibBlock* blocks = P.blk[D];
  int bk = P.bstart[D][L.lid];
  const int bend = P.bstart[D][L.lid + 1];
  int nextL = bk < bend ? blocks[bk].L : 0x7fffffff;
  bool zero_pivot = false;

  // TDMA (douglas_adi.cc:1784-1807), row 0 is the Dirichlet identity row.
  double bet = 1.0;
  double dprev = boundary_value<D, KIND>(P, io, L, 0) / bet;
  double cprev = 0.0;
  out[L.base] = dprev;
  int j = 1;
  while (j < n) {
    if (j == nextL) {
      const MibBlock& b = blocks[bk];
      double r[3], vdr[3][3];
      for (int q = 0; q < b.kind; q++) {
        long long m = L.base + (long long)(j + q) * L.s;
        int side = P.tag[m] & TAG_OUT;
        for (int k = 0; k < 3; k++) vdr[q][k] = P.vd[D][side][k];
        r[q] = (j + q == n - 1) ? boundary_value<D, KIND>(P, io, L, j + q) : line_rhs<D, KIND>(P, io, L, j + q, &b, q);
      }
      implicit_rows(P, b, r, vdr, io.jumps, P.jv);
      for (int q = 0; q < b.kind; q++) {
        long long m = L.base + (long long)(j + q) * L.s;
        double g = cprev / bet;
        bet = b.ib[q] - b.ia[q] * g;
        zero_pivot |= (bet == 0.0);
        double d = (r[q] - b.ia[q] * dprev) / bet;
        gam[m] = g;
        out[m] = d;
        dprev = d;
        cprev = b.ic[q];
      }
      j += b.kind;
      bk++;
      nextL = bk < bend ? blocks[bk].L : 0x7fffffff;
    } else if (j == n - 1) {
      long long m = L.base + (long long)j * L.s;
      const double a = 0.0, bb = 1.0;
      double rr = boundary_value<D, KIND>(P, io, L, j);
      double g = cprev / bet;
      bet = bb - a * g;
      zero_pivot |= (bet == 0.0);
      double d = (rr - a * dprev) / bet;
      gam[m] = g;
      out[m] = d;
      dprev = d;
      cprev = 0.0;
      j++;
    } else {
      long long m = L.base + (long long)j * L.s;
      int side = P.tag[m] & TAG_OUT;
      double a = P.ia[D][side], bb = P.ib[D][side], c = P.ic[D][side];
      double rr = line_rhs<D, KIND>(P, io, L, j, nullptr, 0);
      double g = cprev / bet;
      bet = bb - a * g;
      zero_pivot |= (bet == 0.0);
      double d = (rr - a * dprev) / bet;
      gam[m] = g;
      out[m] = d;
      dprev = d;
      cprev = c;
      j++;
    }
  }
  if (zero_pivot) atomicOr(P.status, 1);

  // Back substitution and the pass epilogue.
  double unext = 0.0;
  for (j = n - 1; j >= 0; j--) {
    long long m = L.base + (long long)j * L.s;
    double u;
    if (j == n - 1) {
      u = out[m];
    } else {
      u = out[m];
      u -= gam[m + L.s] * unext;
    }
    unext = u;
    double v = u;
    if (KIND == K_ADI_X) {
      // uhss = -dt * D_yy u^n + u*  (douglas_adi.cc:516-640); faces keep Outer_u
      if (j > 0 && j < n - 1) v = -P.ydt[m] + u;
    } else if (KIND == K_LOD) {
      if (io.last) {
        int ix, iy, iz;
        node_of<D>(L, j, ix, iy, iz);
        v = u + P.dt * source(P, io.e1, P.tag[m] & TAG_OUT, ix, iy, iz);
      }
    }
    out[m] = v;
  }
}

// TS explicit half step along D = x or y (TS::D_xx_r / D_yy_r, which are the
// LOD Crank-Nicolson operators, trapezoidal.cc:319-895), followed by Set_bc
// at t_half.
template <int D>
__global__ void __launch_bounds__(TPB) k_ts_explicit(const Dev P, const double* in, double* out, double eh,
                                                     double e1) {
  Line L;
  long long t = (long long)blockIdx.x * TPB + threadIdx.x;
  if (!decode_line<D>(P, t, L)) return;
  const int n = L.n;
  int ix, iy, iz;
  if (L.boundary) {
    for (int j = 0; j < n; j++) {
      node_of<D>(L, j, ix, iy, iz);
      out[L.base + (long long)j * L.s] = outer_u(P, eh, ix, iy, iz);
    }
    return;
  }
  node_of<D>(L, 0, ix, iy, iz);
  out[L.base] = outer_u(P, eh, ix, iy, iz);
  node_of<D>(L, n - 1, ix, iy, iz);
  out[L.base + (long long)(n - 1) * L.s] = outer_u(P, eh, ix, iy, iz);
  int bk = P.bstart[D][L.lid];
  const int bend = P.bstart[D][L.lid + 1];
  for (int j = 1; j < n - 1; j++) {
    long long m = L.base + (long long)j * L.s;
    int side = P.tag[m] & TAG_OUT;
    const MibBlock* b = nullptr;
    int r = 0;
    while (bk < bend && P.blk[D][bk].L + P.blk[D][bk].kind <= j) bk++;
    if (bk < bend && j >= P.blk[D][bk].L) {
      b = &P.blk[D][bk];
      r = j - b->L;
    }
    out[m] = own_explicit<D>(P, L, j, m, side, in, b, r, true, P.kex) + in[m];
  }
  (void)e1;
}

// Refresh_Jump (intersection.cc:2294-2490): [u] and u_dir per crossing.
__global__ void __launch_bounds__(TPB) k_jumps(const Dev P, double E) {
  int c = blockIdx.x * TPB + threadIdx.x;
  if (c >= P.ncross) return;
  const CrossConst q = P.cc[c];
  double ju, jb[3];
  if (P.eq == 0) {
    ju = 100.0 - 80.0;
    for (int d = 0; d < 3; d++) jb[d] = P.bi * 0.0 - P.bo * 0.0;
  } else {
    ju = q.R2 * E - q.S * E;
    const double xyz[3] = {q.x, q.y, q.z};
    for (int d = 0; d < 3; d++) jb[d] = P.bo * ((2.0 * xyz[d]) * E) - P.bi * (q.D[d] * E);
  }
  double bxi = q.p[0] * jb[0] + q.p[1] * jb[1] + q.p[2] * jb[2];
  P.jv[c] = make_double2(ju, q.pinv * bxi);
}

__global__ void __launch_bounds__(256) k_init(const Dev P, double E, double* u) {
  long long m = (long long)blockIdx.x * 256 + threadIdx.x;
  if (m >= P.nn) return;
  int ix = (int)(m % P.nx);
  long long q = m / P.nx;
  int iy = (int)(q % P.ny);
  int iz = (int)(q / P.ny);
  u[m] = (P.tag[m] & TAG_OUT) ? outer_u(P, E, ix, iy, iz) : inner_u(P, E, ix, iy, iz);
}

// Error norms: block partials of (max |e|, first argmax key, sum e^2), the key
// being the position in the reference's [ix][iy][iz] loop order.
constexpr int NB_TPB = 256;

__device__ __forceinline__ void better(double& v, long long& k, double v2, long long k2) {
  if (v2 > v || (v2 == v && k2 < k)) {
    v = v2;
    k = k2;
  }
}

__global__ void __launch_bounds__(NB_TPB) k_norms_partial(const Dev P, double E, const double* u, double* part) {
  __shared__ double smax[NB_TPB], ssum[NB_TPB];
  __shared__ long long skey[NB_TPB];
  double vmax = 0.0, vsum = 0.0;
  long long vkey = 0x7fffffffffffffffLL;
  for (long long m = (long long)blockIdx.x * NB_TPB + threadIdx.x; m < P.nn; m += (long long)gridDim.x * NB_TPB) {
    int ix = (int)(m % P.nx);
    long long q = m / P.nx;
    int iy = (int)(q % P.ny);
    int iz = (int)(q / P.ny);
    double ex = (P.tag[m] & TAG_OUT) ? outer_u(P, E, ix, iy, iz) : inner_u(P, E, ix, iy, iz);
    double e = fabs(u[m] - ex);
    long long key = ((long long)ix * P.ny + iy) * P.nz + iz;
    better(vmax, vkey, e, key);
    vsum += e * e;
  }
  smax[threadIdx.x] = vmax;
  skey[threadIdx.x] = vkey;
  ssum[threadIdx.x] = vsum;
  __syncthreads();
  for (int w = NB_TPB / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      better(smax[threadIdx.x], skey[threadIdx.x], smax[threadIdx.x + w], skey[threadIdx.x + w]);
      ssum[threadIdx.x] += ssum[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[3 * blockIdx.x + 0] = smax[0];
    part[3 * blockIdx.x + 1] = (double)skey[0];
    part[3 * blockIdx.x + 2] = ssum[0];
  }
}

__global__ void __launch_bounds__(NB_TPB) k_norms_final(const Dev P, const double* part, int nb, double* out3) {
  __shared__ double smax[NB_TPB], ssum[NB_TPB];
  __shared__ long long skey[NB_TPB];
  double vmax = 0.0, vsum = 0.0;
  long long vkey = 0x7fffffffffffffffLL;
  for (int i = threadIdx.x; i < nb; i += NB_TPB) {
    better(vmax, vkey, part[3 * i], (long long)part[3 * i + 1]);
    vsum += part[3 * i + 2];
  }
  smax[threadIdx.x] = vmax;
  skey[threadIdx.x] = vkey;
  ssum[threadIdx.x] = vsum;
  __syncthreads();
  for (int w = NB_TPB / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      better(smax[threadIdx.x], skey[threadIdx.x], smax[threadIdx.x + w], skey[threadIdx.x + w]);
      ssum[threadIdx.x] += ssum[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out3[0] = smax[0];
    out3[1] = smax[0] > 0.0 ? (double)skey[0] : 0.0;
    out3[2] = sqrt(ssum[0] / (1.0 * P.nx * P.ny * P.nz));
  }
}

template <int D>
long long nlines(const Dev& P) {
  int n1 = D == 0 ? P.ny : P.nx;
  int n2 = D == 2 ? P.ny : P.nz;
  return (long long)n1 * n2;
}

template <int D, int KIND>
void sweep(const Dev& P, const SweepIO& io, cudaStream_t st) {
  long long nl = nlines<D>(P);
  k_sweep<D, KIND><<<(unsigned)((nl + TPB - 1) / TPB), TPB, 0, st>>>(P, io);
}

}  // namespace

int launch_initialize(const Dev& P, double E, double* u, cudaStream_t st) {
  k_init<<<(unsigned)((P.nn + 255) / 256), 256, 0, st>>>(P, E, u);
  return 1;
}

int norms_blocks(const Dev& P) {
  long long nb = (P.nn + NB_TPB * 8 - 1) / (NB_TPB * 8);
  if (nb > 4096) nb = 4096;
  if (nb < 1) nb = 1;
  return (int)nb;
}

int launch_norms(const Dev& P, double E, const double* u, double* partial, int nb, double* out3, cudaStream_t st) {
  k_norms_partial<<<nb, NB_TPB, 0, st>>>(P, E, u, partial);
  k_norms_final<<<1, NB_TPB, 0, st>>>(P, partial, nb, out3);
  return 2;
}

// One time step.  u0 holds u^n on entry and u^{n+1} on return (the two
// pointers are swapped when the result lands in the other buffer).
int launch_step(const Dev& P, const StepTimes& T, double*& u0, double*& u1, cudaStream_t st, cudaEvent_t* ev) {
  int launches = 0;
  int slot = 0;
  auto mark = [&](int k) {
    if (ev) cudaEventRecord(ev[2 * slot + k], st);
    if (k == 1) slot++;
  };
  mark(0);
  if (P.ncross > 0) {
    k_jumps<<<(P.ncross + TPB - 1) / TPB, TPB, 0, st>>>(P, T.e_next);
    launches++;
  }
  mark(1);
  SweepIO io{};
  io.e1 = T.e_next;
  io.e0 = T.e_prev;
  if (P.method == 0) {
    // Douglas-ADI: x sweep writes uhss = -dt D_yy u^n + u*; y sweep in place
    // gives u**; z sweep in place gives u^{n+1}.
    io.stin = u0;
    io.add = u0;
    io.out = u1;
    io.jumps = 0;
    mark(0);
    sweep<0, K_ADI_X>(P, io, st);
    mark(1);
    io.add = u1;
    io.out = u1;
    mark(0);
    sweep<1, K_COPY>(P, io, st);
    mark(1);
    io.stin = u0;
    io.add = u1;
    io.out = u1;
    mark(0);
    sweep<2, K_ADI_Z>(P, io, st);
    mark(1);
    launches += 3;
    double* tmp = u0;
    u0 = u1;
    u1 = tmp;
  } else if (P.method == 1 || P.method == 2) {
    io.jumps = 1;
    io.cn = P.method == 2;
    io.stin = u0;
    io.add = u0;
    io.out = u1;
    io.last = 0;
    mark(0);
    sweep<0, K_LOD>(P, io, st);
    mark(1);
    io.stin = u1;
    io.add = u1;
    io.out = u0;
    mark(0);
    sweep<1, K_LOD>(P, io, st);
    mark(1);
    io.stin = u0;
    io.add = u0;
    io.out = u1;
    io.last = 1;
    mark(0);
    sweep<2, K_LOD>(P, io, st);
    mark(1);
    launches += 3;
    double* tmp = u0;
    u0 = u1;
    u1 = tmp;
  } else {
    // TS: explicit x and y half steps, fused explicit z + sources + implicit
    // z, then implicit y and x in place.
    long long nx_l = nlines<0>(P), ny_l = nlines<1>(P);
    mark(0);
    k_ts_explicit<0><<<(unsigned)((nx_l + TPB - 1) / TPB), TPB, 0, st>>>(P, u0, u1, T.e_half, T.e_next);
    mark(1);
    mark(0);
    k_ts_explicit<1><<<(unsigned)((ny_l + TPB - 1) / TPB), TPB, 0, st>>>(P, u1, u0, T.e_half, T.e_next);
    mark(1);
    io.jumps = 1;
    io.stin = u0;
    io.add = u0;
    io.out = u1;
    mark(0);
    sweep<2, K_TS_Z>(P, io, st);
    mark(1);
    io.add = u1;
    io.out = u1;
    mark(0);
    sweep<1, K_COPY>(P, io, st);
    mark(1);
    mark(0);
    sweep<0, K_COPY>(P, io, st);
    mark(1);
    launches += 5;
    double* tmp = u0;
    u0 = u1;
    u1 = tmp;
  }
  return launches;
}

}  // namespace mts

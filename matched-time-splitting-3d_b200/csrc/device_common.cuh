// Device helpers shared by the plain FP64 kernels (kernels.cu) and the mixed
// precision kernels (mixed.cu): the exact solutions, line geometry, cp.async
// staging, the MIB row sums and the Convert2Tri row operations.
#pragma once

#include <cuda_runtime.h>

#include "device.h"

namespace mts {
namespace {

constexpr int TPB = 128;                // pointwise kernels and small kernels
constexpr int kMaxSweepSmem = 232448;  // 227 KB: the sm_100 per-CTA limit

enum Kind { K_COPY = 0, K_STENCIL = 1, K_TS_Z = 2 };

struct SweepIO {
  const double* stin;  // field the explicit stencil reads
  const double* add;   // field added to the explicit part (or copied)
  double* out;         // result field (may alias stin/add: a line is read
                       // completely before any of it is written)
  double e1;           // exp(-t_next): boundary data, source, jumps
  double e0;           // exp(-t_prev): TS source of the first half step
  double k;            // explicit factor: -dt (ADI), 0.5*dt (LOD-CN, TS)
  int jumps;           // MIB rows carry jump terms (LOD, TS)
  int bmode;           // boundary lines: 0 keep, 1 Outer_u(t_next), 2 + dt*f
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
__device__ __forceinline__ double source(const Dev& P, double E, int out, int ix, int iy, int iz) {
  if (P.eq == 0) return 0.0;
  if (out) return -outer_u(P, E, ix, iy, iz) - P.c6bo * E;
  return P.kin * inner_u(P, E, ix, iy, iz);
}

// CTAs of a persistent line sweep: one per SM at most, no more than nl lines
// of nt threads need.
inline unsigned sweep_grid(const Dev& P, long long nl, int nt) {
  const long long b = (nl + nt - 1) / nt;
  return (unsigned)(b < P.sweep_blocks ? (b > 0 ? b : 1) : P.sweep_blocks);
}

// The step's time factor k (0: exp(-t_prev), 1: exp(-t_half), 2: exp(-t_next)):
// the launch argument, or the step table of a replayed graph.
__device__ __forceinline__ double step_e(const Dev& P, double given, int k) {
  return P.tsched ? P.tsched[3 * (*P.tstep) + k] : given;
}

// The exact jumps at crossing q for time factor E: [u] (Equation::Jump_u) and
// [beta u_x], [beta u_y], [beta u_z] (the Eq's Jump_betau_x/y/z), with the
// operations of src/equation/eq_0.cc and of the measured problem in their
// order.
__device__ __forceinline__ void exact_jumps(const Dev& P, const CrossConst& q, double E, double& ju, double jb[3]) {
  if (P.eq == 0) {
    ju = 100.0 - 80.0;
    for (int d = 0; d < 3; d++) jb[d] = P.bi * 0.0 - P.bo * 0.0;
  } else {
    ju = q.R2 * E - q.S * E;
    const double xyz[3] = {q.x, q.y, q.z};
    for (int d = 0; d < 3; d++) jb[d] = P.bo * ((2.0 * xyz[d]) * E) - P.bi * (q.D[d] * E);
  }
}

// ---------------------------------------------------------------------------
// Line geometry.  Direction D lines are indexed (i1, i2) as in the reference
// (src/constant.h:83-89): x -> (iy, iz), y -> (ix, iz), z -> (ix, iy); the
// line number runs over i1 fastest.

struct Line {
  long long base, s;
  int n, lid, i1, i2;
  bool boundary;
};

template <int D>
__host__ __device__ __forceinline__ long long nlines(const Dev& P) {
  int n1 = D == 0 ? P.ny : P.nx;
  int n2 = D == 2 ? P.ny : P.nz;
  return (long long)n1 * n2;
}

template <int D>
__device__ __forceinline__ void decode_line(const Dev& P, long long t, Line& L) {
  int n1 = D == 0 ? P.ny : P.nx;
  int n2 = D == 2 ? P.ny : P.nz;
  // a direction has n1*n2 < 2^31 lines: 32-bit division
  L.i1 = (int)t % n1;
  L.i2 = (int)t / n1;
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

__device__ __forceinline__ void node_xyz(const Dev& P, long long m, int& ix, int& iy, int& iz) {
  ix = (int)(m % P.nx);
  long long q = m / P.nx;
  iy = (int)(q % P.ny);
  iz = (int)(q / P.ny);
}

// ---------------------------------------------------------------------------
// cp.async (8-byte, L1-allocating) staging

__device__ __forceinline__ void cp_async8(double* smem_dst, const double* gsrc) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// ---------------------------------------------------------------------------
// MIB rows

__device__ __forceinline__ double corner_jumps(const double* w, double2 l, double2 r) {
  return l.x * w[5] + l.y * w[6] + r.x * w[7] + r.y * w[8];
}

// Explicit 3-point sum of row r of block b with fictitious points, before the
// dt factor: the MIB branches of douglas_adi.cc:112-210 (jumps = 0) and
// lod.cc:337-496 (jumps = 1).  U(j) returns the field at row j of the line.
template <class UF>
__device__ double mib_sum(const MibBlock& b, int r, UF U, const double* vd, bool jumps, const double2* jv) {
  const int L = b.L;
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
                                              const double* vd0, const double* vd1, const double* vd2,
                                              bool jumps, const double2* jv) {
  const double cdt = P.cdt;
  if (jumps) {
    if (b.kind == 2) {
      double2 J = jv[b.c0];
      r[0] = r[0] + cdt * vd0[2] * (J.x * b.w[1][4] + J.y * b.w[1][5]);
      r[1] = r[1] + cdt * vd1[0] * (J.x * b.w[0][4] + J.y * b.w[0][5]);
    } else {
      double2 Jl = jv[b.c0], Jr = jv[b.c1];
      r[0] = r[0] + cdt * vd0[2] * corner_jumps(b.w[1], Jl, Jr);
      r[1] = r[1] + cdt * vd1[0] * corner_jumps(b.w[0], Jl, Jr);
      r[1] += cdt * vd1[2] * corner_jumps(b.w[3], Jl, Jr);
      r[2] = r[2] + cdt * vd2[0] * corner_jumps(b.w[2], Jl, Jr);
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


// Rows of the pointwise passes: a warp takes one x-row (iy, iz) at a time and
// covers it in groups of G x 32 nodes (ROW_G, or 2 for the five-load ADI
// RHS).  All loads of a group are issued before any of them is used, so each
// warp keeps G rows' worth of DRAM reads in flight; the exact-solution parts
// fixed along the row are computed once.
constexpr int ROW_G = 4;

struct RowExact {
  double y2, z2;   // y*y, z*z
  double c2y, s2z; // cos 2y, sin 2z
};
__device__ __forceinline__ RowExact row_exact(const Dev& P, int iy, int iz) {
  const double y = P.ax[1][iy], z = P.ax[2][iz];
  return {y * y, z * z, P.c2[1][iy], P.s2[2][iz]};
}
// outer_u and source in the operand order of outer_u / inner_u / source
__device__ __forceinline__ double row_outer(const Dev& P, const RowExact& q, int ix, double E) {
  if (P.eq == 0) return 100.0;
  const double x = P.ax[0][ix];
  return ((x * x + q.y2) + q.z2) * E;
}
__device__ __forceinline__ double row_source(const Dev& P, const RowExact& q, int ix, double E, int out) {
  if (P.eq == 0) return 0.0;
  if (out) return -row_outer(P, q, ix, E) - P.c6bo * E;
  return P.kin * (((P.s2[0][ix] * q.c2y) * q.s2z) * E);
}

template <bool B>
struct BoolC {
  static constexpr bool value = B;
};
template <int I>
struct IntC {
  static constexpr int value = I;
};

// The CTA's item and its problem's record, copied into shared memory.
#define BATCH_PROLOGUE                                                                \
  __shared__ __align__(16) long long sdev_[(sizeof(Dev) + 7) / 8];                    \
  const BatchItem w = items[blockIdx.x];                                              \
  {                                                                                   \
    const long long* src_ = reinterpret_cast<const long long*>(Ps + w.p);             \
    for (int i_ = threadIdx.x; i_ < (int)((sizeof(Dev) + 7) / 8); i_ += blockDim.x) \
      sdev_[i_] = src_[i_];                                                           \
  }                                                                                   \
  __syncthreads();                                                                    \
  const Dev& P = *reinterpret_cast<const Dev*>(sdev_);                                \
  if (*P.tstep >= P.tstop) return; /* this problem's steps of the batch are done */


}  // namespace
}  // namespace mts

// Time-stepping kernels for sm_100a.
//
// Implicit line sweeps (the Thomas solves, douglas_adi.cc:1784-1807 and the
// LOD/TS copies) run as one persistent CTA of 128 threads per SM; each thread
// solves one grid line at a time, lines of a warp being consecutive in the
// fast index.  Per line:
//   * forward: the inputs of the line are staged into a 4-chunk shared-memory
//     ring with cp.async, 2-3 chunks (32-48 rows) ahead of use; the
//     right-hand side of chunk k+1 is built from the ring (3-point stencil,
//     MIB fictitious-point rows, source terms) while chunk k runs the
//     elimination recurrence; the MIB row blocks of chunk k are mixed in
//     (Convert2Tri row operations replayed on the right-hand side) just
//     before their rows are eliminated;
//   * the factors c_{j-1}/bet and partial solutions d'_j go to per-thread
//     scratch laid out [row][thread] (coalesced in every direction, reused
//     line after line, so it lives in L2);
//   * backward: the scratch is staged back through the same ring and the
//     solution is written once.
// The inside/outside side of a node, which selects the stencil weights and
// the source, changes along a line only at its recorded crossings, so it is
// tracked from the line's block list instead of being read per node.
//
// Pointwise passes (the Douglas-ADI first right-hand side and the TS explicit
// half steps) are plain grid-stride kernels.
//
// The file is compiled with -fmad=false: every product and sum is rounded on
// its own, in the operand order of the reference statement it restates, which
// makes the plain FP64 path bit-identical to the reference CPU build.
#include <cuda_runtime.h>

#include "device.h"

namespace mts {
namespace {

constexpr int TPB = 128;  // pointwise kernels and small kernels

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

// ---------------------------------------------------------------------------
// Pointwise passes

// Douglas-ADI first right-hand side (douglas_adi.cc:89-359):
//   uhs = ((dt*D_yy u + dt*D_zz u) + u) + dt*src,  src = f + x, y, z jump
// terms; Outer_u(t_next) on the faces.
// Pointwise kernels run one warp per grid row (iy, iz), lanes over ix.
#define FOR_EACH_NODE(P)                                                                          \
  for (int row_ = blockIdx.x * (TPB / 32) + (threadIdx.x >> 5); row_ < (P).ny * (P).nz;          \
       row_ += gridDim.x * (TPB / 32))                                                            \
    for (int ix = threadIdx.x & 31, iy = row_ % (P).ny, iz = row_ / (P).ny; ix < (P).nx; ix += 32) \
      if (long long m = ix + (long long)(P).nx * row_; true)

__global__ void __launch_bounds__(TPB) k_adi_rhs(const Dev P, const double* __restrict__ un,
                                                 double* __restrict__ R, double E) {
  const long long sy = P.nx, sz = (long long)P.nx * P.ny;
  FOR_EACH_NODE(P) {
    if (ix == 0 || iy == 0 || iz == 0 || ix == P.nx - 1 || iy == P.ny - 1 || iz == P.nz - 1) {
      R[m] = outer_u(P, E, ix, iy, iz);
      continue;
    }
    const uint8_t tg = P.tag[m];
    const int side = tg & TAG_OUT;
    const double dt = P.dt;
    const double* vdy = P.vd[1][side];
    const double* vdz = P.vd[2][side];
    const MibBlock* xb = nullptr;
    const MibBlock* yb = nullptr;
    const MibBlock* zb = nullptr;
    int xr = 0, yr = 0, zr = 0;
    double sum, ydt, zdt;
    if (tg & TAG_MIBY) yb = find_block<1>(P, ix * P.nz + iz, iy, yr);
    if (yb) {
      const long long base = ix + sz * iz;
      sum = mib_sum(*yb, yr, [&](int j) { return un[base + (long long)j * sy]; }, vdy, false, P.jv);
      ydt = sum * dt;
    } else {
      sum = 0.0;
      sum += un[m - sy] * vdy[0];
      sum += un[m] * vdy[1];
      sum += un[m + sy] * vdy[2];
      ydt = dt * sum;
    }
    if (tg & TAG_MIBZ) zb = find_block<2>(P, ix * P.ny + iy, iz, zr);
    if (zb) {
      const long long base = ix + (long long)P.nx * iy;
      sum = mib_sum(*zb, zr, [&](int j) { return un[base + (long long)j * sz]; }, vdz, false, P.jv);
      zdt = sum * dt;
    } else {
      sum = 0.0;
      sum += un[m - sz] * vdz[0];
      sum += un[m] * vdz[1];
      sum += un[m + sz] * vdz[2];
      zdt = dt * sum;
    }
    double src = source(P, E, side, ix, iy, iz);
    if (tg & TAG_MIBX) xb = find_block<0>(P, iy * P.nz + iz, ix, xr);
    if (xb) src = adi_src_add(src, *xb, xr, P.vd[0][side], P.jv);
    if (yb) src = adi_src_add(src, *yb, yr, vdy, P.jv);
    if (zb) src = adi_src_add(src, *zb, zr, vdz, P.jv);
    double r = ydt + zdt;
    r += un[m];
    r += dt * src;
    R[m] = r;
  }
}

// TS explicit half step along D = x or y (TS::D_xx_r / D_yy_r, the LOD
// Crank-Nicolson operators, trapezoidal.cc:319-895), then Set_bc at t_half.
template <int D>
__global__ void __launch_bounds__(TPB) k_ts_explicit(const Dev P, const double* __restrict__ in,
                                                     double* __restrict__ out, double eh) {
  const long long s = D == 0 ? 1 : (long long)P.nx;
  const uint8_t flag = D == 0 ? TAG_MIBX : TAG_MIBY;
  FOR_EACH_NODE(P) {
    if (ix == 0 || iy == 0 || iz == 0 || ix == P.nx - 1 || iy == P.ny - 1 || iz == P.nz - 1) {
      out[m] = outer_u(P, eh, ix, iy, iz);
      continue;
    }
    const uint8_t tg = P.tag[m];
    const double* vd = P.vd[D][tg & TAG_OUT];
    const MibBlock* b = nullptr;
    int r = 0;
    if (tg & flag) b = D == 0 ? find_block<0>(P, iy * P.nz + iz, ix, r) : find_block<1>(P, ix * P.nz + iz, iy, r);
    double sum;
    if (b) {
      const long long base = D == 0 ? m - ix : m - (long long)iy * P.nx;
      sum = mib_sum(*b, r, [&](int j) { return in[base + (long long)j * s]; }, vd, true, P.jv);
    } else {
      sum = 0.0;
      sum += in[m - s] * vd[0];
      sum += in[m] * vd[1];
      sum += in[m + s] * vd[2];
    }
    out[m] = P.kex * sum + in[m];
  }
}

// ---------------------------------------------------------------------------
// The persistent line sweep.  Shape: CH rows per staged chunk, NS chunks in
// the ring (both powers of two), NT threads per CTA (one CTA per SM).
//
// Shared memory per thread column: three staged fields [NS*CH] (forward:
// stencil field, added field, bet from the first MIB row on; backward: d'_j,
// gam_{j+1}) and the right-hand sides of two chunks [2*CH].

struct BlockHead {
  int L, kind, sides;
  double a0, a1, a2;
};

__device__ __forceinline__ void load_head(const MibBlock* blk, int k, int end, BlockHead& h) {
  if (k < end) {
    const MibBlock& b = blk[k];
    h.L = b.L;
    h.kind = b.kind;
    h.sides = b.sides;
    h.a0 = b.ia[0];
    h.a1 = b.ia[1];
    h.a2 = b.ia[2];
  } else {
    h.L = 0x7fffffff;
    h.kind = 0;
    h.sides = 0;
  }
}

template <int CH, int NS, int NT>
constexpr size_t shape_smem() {
  return sizeof(double) * (size_t)(3 * NS * CH * NT + 2 * CH * NT);
}

template <int D, int KIND, int CH, int NS, int NT>
__global__ void __launch_bounds__(NT, 1) k_sweep(const Dev P, const SweepIO io) {
  static_assert((CH & (CH - 1)) == 0 && (NS & (NS - 1)) == 0 && NS >= 4 && CH >= 4, "shape");
  constexpr int RING = NS * CH;
  extern __shared__ double sm[];
  const int tid = threadIdx.x;
  double* const sA = sm + tid;                  // [RING][NT]
  double* const sB = sm + RING * NT + tid;      // [RING][NT]
  double* const sC = sm + 2 * RING * NT + tid;  // [RING][NT]
  double* const rb = sm + 3 * RING * NT + tid;  // [2*CH][NT]
#define SA(j) sA[((j) & (RING - 1)) * NT]
#define SB(j) sB[((j) & (RING - 1)) * NT]
#define SC(j) sC[((j) & (RING - 1)) * NT]
#define RB(j) rb[((j) & (2 * CH - 1)) * NT]
  const long long T = (long long)gridDim.x * NT;
  const long long gt = (long long)blockIdx.x * NT + tid;
  double* const dp = P.dp + gt;
  const long long nl = nlines<D>(P);
  const MibBlock* __restrict__ blk = P.blk[D];
  const double* __restrict__ fbet = P.fbet[D];
  const double* __restrict__ fgam = P.fgam[D];
  const double E1 = io.e1;
  const double kx = io.k;
  // per-direction constants by side (0 inside, 1 outside), in registers
  const double v0i = P.vd[D][0][0], v0o = P.vd[D][1][0];
  const double v1i = P.vd[D][0][1], v1o = P.vd[D][1][1];
  const double v2i = P.vd[D][0][2], v2o = P.vd[D][1][2];
  const double cai = P.ia[D][0], cao = P.ia[D][1];

  for (long long t = gt; t < nl; t += T) {
    Line L;
    decode_line<D>(P, t, L);
    const int n = L.n;
    if (L.boundary) {
      if (io.bmode) {
        for (int j = 0; j < n; j++) {
          int ix, iy, iz;
          node_of<D>(L, j, ix, iy, iz);
          long long m = L.base + (long long)j * L.s;
          double v = outer_u(P, E1, ix, iy, iz);
          if (io.bmode == 2) v = v + P.dt * source(P, E1, P.tag[m] & TAG_OUT, ix, iy, iz);
          io.out[m] = v;
        }
      }
      continue;
    }
    const int nch = (n + CH - 1) / CH;
    const int ls = P.lside[D][L.lid];
    const int bfirst = P.bstart[D][L.lid];
    const int bend = P.bstart[D][L.lid + 1];
    const int L1 = bfirst < bend ? blk[bfirst].L : n;  // first MIB row
    const double* __restrict__ pt = P.ptab[D][(ls >> 1) & 1];
    // field A = the stencil field (or the copied field), field B = the added field
    const double* fA = KIND == K_COPY ? io.add : io.stin;
    const double* fB = io.add;
    const bool two = KIND != K_COPY && io.add != io.stin;

    auto stage = [&](int c) {
      if (c < nch) {
        long long off = L.base + (long long)c * CH * L.s;
#pragma unroll
        for (int r = 0; r < CH; r++) {
          const int j = c * CH + r;
          if (j < n) {
            cp_async8(&SA(j), fA + off);
            if (two) cp_async8(&SB(j), fB + off);
            if (j >= L1) cp_async8(&SC(j), fbet + off);
          }
          off += L.s;
        }
      }
      cp_async_commit();
    };

    // right-hand side of chunk c into RB; r-pass block cursor and side
    int rbk = bfirst;
    int rbL = L1 < n ? L1 : 0x7fffffff;
    int rside = (ls >> 1) & 1;
    auto compute_r = [&](int c) {
#pragma unroll 2
      for (int rr = 0; rr < CH; rr++) {
        const int j = c * CH + rr;
        if (j >= n) break;
        double r;
        if (j == 0 || j == n - 1) {
          int ix, iy, iz;
          node_of<D>(L, j, ix, iy, iz);
          r = outer_u(P, E1, ix, iy, iz);
        } else if (j < rbL) {
          // regular row
          if (KIND == K_COPY) {
            r = SA(j);
          } else {
            double sum = 0.0;
            sum += SA(j - 1) * (rside ? v0o : v0i);
            sum += SA(j) * (rside ? v1o : v1i);
            sum += SA(j + 1) * (rside ? v2o : v2i);
            r = kx * sum + (two ? SB(j) : SA(j));
            if (KIND == K_TS_Z) {
              int ix, iy, iz;
              node_of<D>(L, j, ix, iy, iz);
              r = r + P.hdt * source(P, io.e0, rside, ix, iy, iz);
              r = r + P.hdt * source(P, E1, rside, ix, iy, iz);
            }
          }
        } else {
          // a MIB row of the line's next block
          const MibBlock& b = blk[rbk];
          const int q = j - rbL;
          const int side = (b.sides >> q) & 1;
          if (KIND == K_COPY) {
            r = SA(j);
          } else {
            const double* vd = P.vd[D][side];
            double sum = mib_sum(b, q, [&](int jj) { return SA(jj); }, vd, io.jumps, P.jv);
            r = kx * sum + (two ? SB(j) : SA(j));
            if (KIND == K_TS_Z) {
              int ix, iy, iz;
              node_of<D>(L, j, ix, iy, iz);
              r = r + P.hdt * source(P, io.e0, side, ix, iy, iz);
              r = r + P.hdt * source(P, E1, side, ix, iy, iz);
            }
          }
          if (q == b.kind - 1) {
            rside = side;
            rbk++;
            rbL = rbk < bend ? blk[rbk].L : 0x7fffffff;
          }
        }
        RB(j) = r;
      }
    };

    // MIB row mixing for the blocks that start in chunk c
    int xb = bfirst;
    auto mix = [&](int c) {
      while (xb < bend && blk[xb].L < (c + 1) * CH) {
        const MibBlock& b = blk[xb];
        double r[3];
        for (int q = 0; q < b.kind; q++) r[q] = RB(b.L + q);
        implicit_rows(P, b, r, P.vd[D][b.sides & 1], P.vd[D][(b.sides >> 1) & 1], P.vd[D][(b.sides >> 2) & 1],
                      io.jumps, P.jv);
        for (int q = 0; q < b.kind; q++) RB(b.L + q) = r[q];
        xb++;
      }
    };

    // forward substitution with the precomputed factors (TDMA,
    // douglas_adi.cc:1794-1800): d'_j = (r_j - a_j d'_{j-1}) / bet_j
    int mb = bfirst;
    BlockHead hb;
    load_head(blk, mb, bend, hb);
    int mside = (ls >> 1) & 1;
    double dprev = 0.0;
    double* dq = dp;
    auto forward = [&](int c) {
#pragma unroll 2
      for (int rr = 0; rr < CH; rr++) {
        const int j = c * CH + rr;
        if (j >= n) break;
        const double r = RB(j);
        double d;
        if (j == 0) {
          d = r / pt[0];
        } else {
          double a;
          if (j >= hb.L) {
            const int q = j - hb.L;
            a = q == 0 ? hb.a0 : q == 1 ? hb.a1 : hb.a2;
            if (q == hb.kind - 1) {
              mside = (hb.sides >> q) & 1;
              mb++;
              load_head(blk, mb, bend, hb);
            }
          } else if (j == n - 1) {
            a = 0.0;
          } else {
            a = mside ? cao : cai;
          }
          const double bet = j >= L1 ? SC(j) : pt[2 * j];
          d = (r - a * dprev) / bet;
        }
        *dq = d;
        dq += T;
        dprev = d;
      }
    };

    for (int c = 0; c < NS - 1; c++) stage(c);
    cp_async_wait<NS - 3>();
    compute_r(0);
    for (int c = 0; c < nch; c++) {
      stage(c + NS - 1);
      cp_async_wait<NS - 3>();
      if (c + 1 < nch) compute_r(c + 1);
      mix(c);
      forward(c);
    }

    // back substitution u_j = d'_j - gam_{j+1} u_{j+1} (douglas_adi.cc:
    // 1805-1806), staged back through the ring: field A = d'_j, field B =
    // gam_{j+1} where it comes from the per-node factors.  The fence orders
    // this thread's d' stores before the asynchronous copies that read them.
    __threadfence_block();
    auto bstage = [&](int c) {
      if (c >= 0) {
#pragma unroll
        for (int r = 0; r < CH; r++) {
          const int j = c * CH + r;
          if (j < n) {
            cp_async8(&SA(j), dp + (long long)j * T);
            if (j + 1 < n && j + 1 >= L1) cp_async8(&SB(j), fgam + L.base + (long long)(j + 1) * L.s);
          }
        }
      }
      cp_async_commit();
    };
    // side tracking downwards (only the LOD epilogue needs it): below a block
    // the side is that of the block's first row, above the last block that of
    // its last row.
    int db = bend - 1;
    int dbL = db >= bfirst ? blk[db].L : -1, dbK = db >= bfirst ? blk[db].kind : 0;
    int dbS = db >= bfirst ? blk[db].sides : 0;
    int dside = db >= bfirst ? (dbS >> (dbK - 1)) & 1 : (ls >> 1) & 1;
    double unext = 0.0;
    for (int c = nch - 1; c > nch - NS; c--) bstage(c);
    for (int c = nch - 1; c >= 0; c--) {
      bstage(c - NS + 1);
      cp_async_wait<NS - 1>();
#pragma unroll 2
      for (int rr = CH - 1; rr >= 0; rr--) {
        const int j = c * CH + rr;
        if (j >= n) continue;
        double u = SA(j);
        if (j != n - 1) {
          const double gm = j + 1 >= L1 ? SB(j) : pt[2 * (j + 1) + 1];
          u -= gm * unext;
        }
        unext = u;
        double v = u;
        if (io.last) {
          int side;
          if (j == 0) {
            side = ls & 1;
          } else if (j == n - 1) {
            side = (ls >> 2) & 1;
          } else if (j >= dbL && j < dbL + dbK) {
            side = (dbS >> (j - dbL)) & 1;
            if (j == dbL) {
              dside = dbS & 1;
              db--;
              if (db >= bfirst) {
                dbL = blk[db].L;
                dbK = blk[db].kind;
                dbS = blk[db].sides;
              } else {
                dbL = -1;
                dbK = 0;
              }
            }
          } else {
            side = dside;
          }
          int ix, iy, iz;
          node_of<D>(L, j, ix, iy, iz);
          v = u + P.dt * source(P, E1, side, ix, iy, iz);
        }
        io.out[L.base + (long long)j * L.s] = v;
      }
    }
    cp_async_wait<0>();
  }
#undef SA
#undef SB
#undef SC
#undef RB
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

__global__ void __launch_bounds__(TPB) k_init(const Dev P, double E, double* u) {
  FOR_EACH_NODE(P) { u[m] = (P.tag[m] & TAG_OUT) ? outer_u(P, E, ix, iy, iz) : inner_u(P, E, ix, iy, iz); }
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
    int ix, iy, iz;
    node_xyz(P, m, ix, iy, iz);
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

unsigned pointwise_blocks(const Dev& P) {
  long long rows = (long long)P.ny * P.nz;
  long long b = (rows + TPB / 32 - 1) / (TPB / 32);
  long long cap = (long long)P.sweep_blocks * 32;
  return (unsigned)(b < cap ? b : cap);
}

// Sweep shapes (rows per chunk, ring chunks, threads per CTA), selected per
// sweep of a step by Dev::shape (mts_set_sweep_shape / mts_autotune).
#define MTS_SHAPES(X) X(0, 16, 4, 128) X(1, 8, 8, 128) X(2, 8, 4, 256) X(3, 4, 8, 256) X(4, 8, 4, 192)

template <int D, int KIND, int CH, int NS, int NT>
void sweep_shape(const Dev& P, const SweepIO& io, cudaStream_t st) {
  k_sweep<D, KIND, CH, NS, NT><<<P.sweep_blocks, NT, shape_smem<CH, NS, NT>(), st>>>(P, io);
}

template <int D, int KIND>
void sweep(const Dev& P, const SweepIO& io, int shape, cudaStream_t st) {
  switch (shape) {
#define MTS_CASE(id, ch, ns, nt) \
  case id:                       \
    sweep_shape<D, KIND, ch, ns, nt>(P, io, st); \
    break;
    MTS_SHAPES(MTS_CASE)
#undef MTS_CASE
    default:
      sweep_shape<D, KIND, 16, 4, 128>(P, io, st);
  }
}

template <int D, int KIND>
void set_smem_attr() {
#define MTS_ATTR(id, ch, ns, nt)                                                             \
  cudaFuncSetAttribute(k_sweep<D, KIND, ch, ns, nt>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                       (int)shape_smem<ch, ns, nt>());
  MTS_SHAPES(MTS_ATTR)
#undef MTS_ATTR
}

}  // namespace

int sweep_shape_count() { return 5; }
int sweep_shape_max_threads() { return 256; }

void configure_kernels() {
  set_smem_attr<0, K_COPY>();
  set_smem_attr<1, K_COPY>();
  set_smem_attr<2, K_COPY>();
  set_smem_attr<0, K_STENCIL>();
  set_smem_attr<1, K_STENCIL>();
  set_smem_attr<2, K_STENCIL>();
  set_smem_attr<2, K_TS_Z>();
}

int launch_initialize(const Dev& P, double E, double* u, cudaStream_t st) {
  k_init<<<pointwise_blocks(P), TPB, 0, st>>>(P, E, u);
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
    // Douglas-ADI.  u1 <- uhs (pointwise); x sweep in place gives u*; y sweep
    // builds uhss = -dt D_yy u^n + u* and solves in place (u**); z sweep builds
    // uh1 = -dt D_zz u^n + u** and solves in place (u^{n+1}).
    mark(0);
    k_adi_rhs<<<pointwise_blocks(P), TPB, 0, st>>>(P, u0, u1, T.e_next);
    mark(1);
    io.stin = u1;
    io.add = u1;
    io.out = u1;
    io.jumps = 0;
    io.bmode = 0;
    mark(0);
    sweep<0, K_COPY>(P, io, P.shape[0], st);
    mark(1);
    io.stin = u0;
    io.k = -P.dt;
    mark(0);
    sweep<1, K_STENCIL>(P, io, P.shape[1], st);
    mark(1);
    mark(0);
    sweep<2, K_STENCIL>(P, io, P.shape[2], st);
    mark(1);
    launches += 4;
    double* tmp = u0;
    u0 = u1;
    u1 = tmp;
  } else if (P.method == 1 || P.method == 2) {
    // LOD, in place on u0.
    io.jumps = 1;
    io.k = P.kex;
    io.stin = u0;
    io.add = u0;
    io.out = u0;
    io.bmode = 1;
    mark(0);
    if (P.method == 2)
      sweep<0, K_STENCIL>(P, io, P.shape[0], st);
    else
      sweep<0, K_COPY>(P, io, P.shape[0], st);
    mark(1);
    mark(0);
    if (P.method == 2)
      sweep<1, K_STENCIL>(P, io, P.shape[1], st);
    else
      sweep<1, K_COPY>(P, io, P.shape[1], st);
    mark(1);
    io.last = 1;
    io.bmode = 2;
    mark(0);
    if (P.method == 2)
      sweep<2, K_STENCIL>(P, io, P.shape[2], st);
    else
      sweep<2, K_COPY>(P, io, P.shape[2], st);
    mark(1);
    launches += 3;
  } else {
    // TS: explicit x (u0 -> u1) and y (u1 -> u0) half steps, fused explicit
    // z + sources + implicit z in place on u0, then implicit y and x in place.
    mark(0);
    k_ts_explicit<0><<<pointwise_blocks(P), TPB, 0, st>>>(P, u0, u1, T.e_half);
    mark(1);
    mark(0);
    k_ts_explicit<1><<<pointwise_blocks(P), TPB, 0, st>>>(P, u1, u0, T.e_half);
    mark(1);
    io.jumps = 1;
    io.k = P.kex;
    io.stin = u0;
    io.add = u0;
    io.out = u0;
    io.bmode = 1;
    mark(0);
    sweep<2, K_TS_Z>(P, io, P.shape[0], st);
    mark(1);
    io.bmode = 0;
    mark(0);
    sweep<1, K_COPY>(P, io, P.shape[1], st);
    mark(1);
    mark(0);
    sweep<0, K_COPY>(P, io, P.shape[2], st);
    mark(1);
    launches += 5;
  }
  return launches;
}

}  // namespace mts

// Time-stepping kernels for sm_100a.
//
// Implicit line sweeps (the Thomas solves, douglas_adi.cc:1784-1807 and the
// LOD/TS copies) run as one persistent CTA of 128-512 threads per SM (the
// sweep shape); each thread solves one grid line at a time, lines of a warp
// being consecutive in the fast index.  The Thomas factors (bet, gam) are
// computed once at setup.  Per line:
//   * forward: the inputs of the line (and its per-node factors from its
//     first MIB row on) are staged into a shared-memory ring with cp.async,
//     chunks ahead of use; each row's right-hand side is built from the ring
//     (3-point stencil, source terms), the MIB row blocks' right-hand sides
//     come from the block pre-pass (Convert2Tri row operations replayed on
//     them), and the elimination recurrence runs over the chunk;
//   * the partial solutions d'_j go to per-thread scratch laid out
//     [row][thread] (coalesced in every direction, reused line after line);
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

#include "device_common.cuh"

namespace mts {
namespace {

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

// RHS1 of a node that is a MIB row of some x, y or z block: the general form.
__device__ __forceinline__ double adi_rhs_mib(const Dev& P, const double* __restrict__ un, double E, long long m,
                                              int ix, int iy, int iz, int tg) {
  const long long sy = P.nx, sz = (long long)P.nx * P.ny;
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
  return r;
}

template <int G>
__device__ __forceinline__ void k_adi_rhs_body(const Dev& P, unsigned cta_, unsigned ncta_,
                                               const double* __restrict__ un, double* __restrict__ R, double E) {
  E = step_e(P, E, 2);
  const int lane = threadIdx.x & 31;
  const int nx = P.nx, nrows = P.ny * P.nz;
  const long long sy = nx, sz = (long long)nx * P.ny;
  const double dt = P.dt;
  // a node's side selects one of two specialised bodies (uniform over a warp
  // away from the interface), whose stencil weights are fixed kernel
  // parameters (constant-bank operands) instead of weights indexed per node
  for (int row = cta_ * (TPB / 32) + (threadIdx.x >> 5); row < nrows; row += ncta_ * (TPB / 32)) {
    const int iy = row % P.ny, iz = row / P.ny;
    const long long m0 = (long long)nx * row;
    const RowExact q = row_exact(P, iy, iz);
    double* const Rr = R + m0;
    if (iy == 0 || iz == 0 || iy == P.ny - 1 || iz == P.nz - 1) {
      for (int ix = lane; ix < nx; ix += 32) Rr[ix] = row_outer(P, q, ix, E);
      continue;
    }
    // the row's two face nodes, then its interior in groups of G x 32
    if (lane < 2) {
      const int ix = lane ? nx - 1 : 0;
      Rr[ix] = row_outer(P, q, ix, E);
    }
    const double* const uc_r = un + m0;
    const double* const uym_r = uc_r - sy;
    const double* const uyp_r = uc_r + sy;
    const double* const uzm_r = uc_r - sz;
    const double* const uzp_r = uc_r + sz;
    const uint8_t* const tg_r = P.tag + m0;
    for (int ix0 = 1; ix0 < nx - 1; ix0 += 32 * G) {
      double uc[G], uym[G], uyp[G], uzm[G], uzp[G];
      int tg[G];
#pragma unroll
      for (int g = 0; g < G; g++) {
        const int ix = ix0 + 32 * g + lane;
        if (ix < nx - 1) {
          tg[g] = tg_r[ix];
          uc[g] = uc_r[ix];
          uym[g] = uym_r[ix];
          uyp[g] = uyp_r[ix];
          uzm[g] = uzm_r[ix];
          uzp[g] = uzp_r[ix];
        }
      }
#pragma unroll
      for (int g = 0; g < G; g++) {
        const int ix = ix0 + 32 * g + lane;
        if (ix >= nx - 1) break;
        if (tg[g] & (TAG_MIBX | TAG_MIBY | TAG_MIBZ)) continue;  // a MIB row: k_adi_rhs_mib writes it
        auto node = [&](auto S) {
          constexpr int sd = decltype(S)::value;
          double sum = 0.0;
          sum += uym[g] * P.vd[1][sd][0];
          sum += uc[g] * P.vd[1][sd][1];
          sum += uyp[g] * P.vd[1][sd][2];
          const double ydt = dt * sum;
          sum = 0.0;
          sum += uzm[g] * P.vd[2][sd][0];
          sum += uc[g] * P.vd[2][sd][1];
          sum += uzp[g] * P.vd[2][sd][2];
          const double zdt = dt * sum;
          const double src = row_source(P, q, ix, E, sd);
          double r = ydt + zdt;
          r += uc[g];
          r += dt * src;
          return r;
        };
        Rr[ix] = (tg[g] & TAG_OUT) ? node(IntC<1>{}) : node(IntC<0>{});
      }
    }
  }
}

template <int G>
__global__ void __launch_bounds__(TPB, 8) k_adi_rhs(const __grid_constant__ Dev P, const double* __restrict__ un,
                                                 double* __restrict__ R, double E) {
  k_adi_rhs_body<G>(P, blockIdx.x, gridDim.x, un, R, E);
}

// The MIB rows of RHS1, one thread per listed node.
__device__ __forceinline__ void k_adi_rhs_mib_body(const Dev& P, unsigned cta_, unsigned ncta_,
                                                   const double* __restrict__ un, double* __restrict__ R, double E) {
  const int k = cta_ * TPB + threadIdx.x;
  if (k >= P.nmibnode) return;
  E = step_e(P, E, 2);
  const long long m = P.mibnode[k];
  int ix, iy, iz;
  node_xyz(P, m, ix, iy, iz);
  R[m] = adi_rhs_mib(P, un, E, m, ix, iy, iz, P.tag[m]);
}

__global__ void __launch_bounds__(TPB) k_adi_rhs_mib(const __grid_constant__ Dev P, const double* __restrict__ un,
                                                     double* __restrict__ R, double E) {
  k_adi_rhs_mib_body(P, blockIdx.x, gridDim.x, un, R, E);
}

// TS explicit half step along D = x or y (TS::D_xx_r / D_yy_r, the LOD
// Crank-Nicolson operators, trapezoidal.cc:319-895), then Set_bc at t_half.
template <int D>
__device__ __forceinline__ double ts_explicit_mib(const Dev& P, const double* __restrict__ in, long long m, int ix,
                                               int iy, int iz, int tg) {
  const long long s = D == 0 ? 1 : (long long)P.nx;
  const double* vd = P.vd[D][tg & TAG_OUT];
  int r = 0;
  const MibBlock* b = D == 0 ? find_block<0>(P, iy * P.nz + iz, ix, r) : find_block<1>(P, ix * P.nz + iz, iy, r);
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
  return P.kex * sum + in[m];
}

template <int D>
__device__ __forceinline__ void k_ts_explicit_mib_body(const Dev& P, unsigned cta_, unsigned ncta_,
                                                       const double* __restrict__ in, double* __restrict__ out) {
  const int k = cta_ * TPB + threadIdx.x;
  if (k >= P.nmibnode) return;
  const long long m = P.mibnode[k];
  const int tg = P.tag[m];
  if (!(tg & (D == 0 ? TAG_MIBX : TAG_MIBY))) return;
  int ix, iy, iz;
  node_xyz(P, m, ix, iy, iz);
  out[m] = ts_explicit_mib<D>(P, in, m, ix, iy, iz, tg);
}

template <int D>
__global__ void __launch_bounds__(TPB) k_ts_explicit_mib(const __grid_constant__ Dev P,
                                                         const double* __restrict__ in, double* __restrict__ out) {
  k_ts_explicit_mib_body<D>(P, blockIdx.x, gridDim.x, in, out);
}

template <int D>
__device__ __forceinline__ void k_ts_explicit_body(const Dev& P, unsigned cta_, unsigned ncta_,
                                                   const double* __restrict__ in, double* __restrict__ out,
                                                   double eh) {
  eh = step_e(P, eh, 1);
  const long long s = D == 0 ? 1 : (long long)P.nx;
  const int flag = D == 0 ? TAG_MIBX : TAG_MIBY;
  const int lane = threadIdx.x & 31;
  const int nrows = P.ny * P.nz;
  const double kex = P.kex;
  const double w0i = P.vd[D][0][0], w1i = P.vd[D][0][1], w2i = P.vd[D][0][2];
  const double w0o = P.vd[D][1][0], w1o = P.vd[D][1][1], w2o = P.vd[D][1][2];
  for (int row = cta_ * (TPB / 32) + (threadIdx.x >> 5); row < nrows; row += ncta_ * (TPB / 32)) {
    const int iy = row % P.ny, iz = row / P.ny;
    const long long m0 = (long long)P.nx * row;
    const RowExact q = row_exact(P, iy, iz);
    if (iy == 0 || iz == 0 || iy == P.ny - 1 || iz == P.nz - 1) {
      for (int ix = lane; ix < P.nx; ix += 32) out[m0 + ix] = row_outer(P, q, ix, eh);
      continue;
    }
    for (int ix0 = 0; ix0 < P.nx; ix0 += 32 * ROW_G) {
      double um[ROW_G], uc[ROW_G], up[ROW_G];
      int tg[ROW_G];
#pragma unroll
      for (int g = 0; g < ROW_G; g++) {
        const int ix = ix0 + 32 * g + lane;
        if (ix < P.nx) {
          const long long m = m0 + ix;
          tg[g] = P.tag[m];
          uc[g] = in[m];
          um[g] = in[m - s];
          up[g] = in[m + s];
        }
      }
#pragma unroll
      for (int g = 0; g < ROW_G; g++) {
        const int ix = ix0 + 32 * g + lane;
        if (ix >= P.nx) break;
        const long long m = m0 + ix;
        double v;
        if (ix == 0 || ix == P.nx - 1) {
          v = row_outer(P, q, ix, eh);
        } else if (!(tg[g] & flag)) {
          const int side = tg[g] & TAG_OUT;
          double sum = 0.0;
          sum += um[g] * (side ? w0o : w0i);
          sum += uc[g] * (side ? w1o : w1i);
          sum += up[g] * (side ? w2o : w2i);
          v = kex * sum + uc[g];
        } else {
          continue;  // a MIB row of a D block: k_ts_explicit_mib writes it
        }
        out[m] = v;
      }
    }
  }
}

template <int D>
__global__ void __launch_bounds__(TPB) k_ts_explicit(const __grid_constant__ Dev P, const double* __restrict__ in,
                                                     double* __restrict__ out, double eh) {
  k_ts_explicit_body<D>(P, blockIdx.x, gridDim.x, in, out, eh);
}

// ---------------------------------------------------------------------------
// The persistent line sweep.  Shape: CH rows per staged chunk, NS chunks in
// the ring (both powers of two), NT threads per CTA (one CTA per SM).
//
// Shared memory per thread column: three staged fields of NS*CH rows
// (forward: stencil field, added field, bet from the first MIB row on;
// backward: d'_j, gam_{j+1}).  Whole chunks are staged without per-row bound
// checks: every field the sweep reads (the solution fields, the per-node
// factors, the d' scratch) carries kRowPad rows of slack past its last row,
// so the rows of a line's last chunk beyond n are readable (and never used).
// The forward pass handles a chunk of regular rows (no MIB row, no line end)
// with a fully unrolled loop at compile-time shared-memory offsets whose
// stencil window slides in registers; chunks that hold a MIB block or a line
// end take the row-by-row path.  The backward pass does the same for chunks
// without the line end (and without the LOD epilogue).

struct BlockHead {
  int L, kind, sides;
  double a0, a1, a2;  // sub-diagonal of the block's rows after Convert2Tri
  double r0, r1, r2;  // their right-hand sides this sweep (block pre-pass)
};

__device__ __forceinline__ void load_head(const MibBlock* blk, const double* rblk, int k, int end,
                                          BlockHead& h) {
  if (k < end) {
    const MibBlock& b = blk[k];
    h.L = b.L;
    h.kind = b.kind;
    h.sides = b.sides;
    h.a0 = b.ia[0];
    h.a1 = b.ia[1];
    h.a2 = b.ia[2];
    h.r0 = rblk[3 * k];
    h.r1 = rblk[3 * k + 1];
    h.r2 = rblk[3 * k + 2];
  } else {
    h.L = 0x7fffffff;
    h.kind = 0;
    h.sides = 0;
  }
}

// Block pre-pass of a sweep: one thread per MIB block of direction D computes
// the right-hand sides of the block's rows exactly as the sweep would (the
// explicit MIB stencil of douglas_adi.cc:112-210 / lod.cc:337-496, the jump
// terms of D_xx_l lod.cc:960-1097, the Convert2Tri row operations) and stores
// them for the sweep, which then spends no time on MIB data.
template <int D, int KIND>
__device__ __forceinline__ void k_block_rhs_body(const Dev& P, unsigned cta_, unsigned ncta_, const SweepIO io,
                                                 int nblk) {
  const int k = cta_ * TPB + threadIdx.x;
  if (k >= nblk) return;
  const MibBlock& b = P.blk[D][k];
  const int n2 = D == 2 ? P.ny : P.nz;
  Line L;
  decode_line<D>(P, (long long)(b.line % n2) * (D == 0 ? P.ny : P.nx) + b.line / n2, L);
  const double* stin = KIND == K_COPY ? io.add : io.stin;
  const double e0 = step_e(P, io.e0, 0), e1 = step_e(P, io.e1, 2);
  auto U = [&](int j) { return stin[L.base + (long long)j * L.s]; };
  double r[3] = {0.0, 0.0, 0.0};
  for (int q = 0; q < b.kind; q++) {
    const int jj = b.L + q;
    const int side = (b.sides >> q) & 1;
    const double av = io.add[L.base + (long long)jj * L.s];
    if (KIND == K_COPY) {
      r[q] = av;
    } else {
      double sum = mib_sum(b, q, U, P.vd[D][side], io.jumps, P.jv);
      double v = io.k * sum + av;
      if (KIND == K_TS_Z) {
        int ix, iy, iz;
        node_of<D>(L, jj, ix, iy, iz);
        v = v + P.hdt * source(P, e0, side, ix, iy, iz);
        v = v + P.hdt * source(P, e1, side, ix, iy, iz);
      }
      r[q] = v;
    }
  }
  implicit_rows(P, b, r, P.vd[D][b.sides & 1], P.vd[D][(b.sides >> 1) & 1], P.vd[D][(b.sides >> 2) & 1], io.jumps,
                P.jv);
  for (int q = 0; q < 3; q++) P.rblk[D][3 * k + q] = r[q];
}

template <int D, int KIND>
__global__ void __launch_bounds__(TPB) k_block_rhs(const __grid_constant__ Dev P, const SweepIO io, int nblk) {
  k_block_rhs_body<D, KIND>(P, blockIdx.x, gridDim.x, io, nblk);
}

// Exact-solution parts along a line: the fixed axes are read once per line,
// the sweep axis from shared memory.  S = (sin2x cos2y) sin2z and
// R2 = (x*x + y*y) + z*z keep the operand order of the exact-solution code,
// so S*E and R2*E are the inner and outer solutions bit for bit.
struct LineExact {
  double x, y, z, s2x, c2y, s2z;
};

template <int D>
__device__ __forceinline__ void line_exact(const Dev& P, const Line& L, LineExact& f) {
  int ix, iy, iz;
  node_of<D>(L, 0, ix, iy, iz);
  f.x = P.ax[0][ix];
  f.y = P.ax[1][iy];
  f.z = P.ax[2][iz];
  f.s2x = P.s2[0][ix];
  f.c2y = P.c2[1][iy];
  f.s2z = P.s2[2][iz];
}

// sX: [coordinate | sin 2x | cos 2x] of the sweep axis, nd rows each.
template <int D>
__device__ __forceinline__ void row_parts(const LineExact& f, const double* sX, int nd, int j, double& S,
                                          double& R2) {
  if (D == 0) {
    const double x = sX[j];
    S = (sX[nd + j] * f.c2y) * f.s2z;
    R2 = (x * x + f.y * f.y) + f.z * f.z;
  } else if (D == 1) {
    const double y = sX[j];
    S = (f.s2x * sX[2 * nd + j]) * f.s2z;
    R2 = (f.x * f.x + y * y) + f.z * f.z;
  } else {
    const double z = sX[j];
    S = (f.s2x * f.c2y) * sX[nd + j];
    R2 = (f.x * f.x + f.y * f.y) + z * z;
  }
}
__device__ __forceinline__ double outer_from(const Dev& P, double R2, double E) {
  return P.eq == 0 ? 100.0 : R2 * E;
}
__device__ __forceinline__ double source_from(const Dev& P, double S, double R2, double E, int out) {
  if (P.eq == 0) return 0.0;
  if (out) return -(R2 * E) - P.c6bo * E;
  return P.kin * (S * E);
}

// Shared memory of a shape: the staging ring, the two prefix factor tables
// of the sweep direction (2 sides x 2 values x n rows) and its exact-solution
// tables (3 x n).
template <int CH, int NS, int NT, int D = 0>
constexpr size_t shape_smem(int n) {
  // D = 0 pads each ring row by 4 doubles (the x sweeps' cooperative staging);
  // the default D = 0 is the largest, used for the fit check
  return sizeof(double) * ((size_t)3 * NS * CH * (D == 0 ? NT + 4 : NT) + (size_t)7 * n);
}


template <int D, int KIND, int CH, int NS, int NT>
__device__ __forceinline__ void k_sweep_body(const Dev& P, unsigned cta_, unsigned ncta_, const SweepIO io) {
  static_assert((CH & (CH - 1)) == 0 && (NS & (NS - 1)) == 0 && NS >= 4 && CH >= 4, "shape");
  static_assert(CH <= kRowPad, "chunk rows past a line end must stay within the fields' slack");
  constexpr int RING = NS * CH;    // rows in a field's ring
  // x lines (kCoop, below) are staged by the warp together, with 4 doubles of
  // padding per ring row so that a copy instruction's lanes, which write
  // CH rows of 32/CH columns, fall on distinct banks in pairs
  constexpr int RS = D == 0 ? NT + 4 : NT;  // doubles per ring row
  constexpr int SLOT = CH * RS;    // doubles per chunk slot
  extern __shared__ double sm[];
  const int tid = threadIdx.x;
  double* const sA = sm + tid;             // [NS][CH][NT]
  double* const sB = sA + NS * SLOT;       // [NS][CH][NT]
  double* const sC = sB + NS * SLOT;       // [NS][CH][NT]
#define SA(j) sA[((j) & (RING - 1)) * RS]
#define SB(j) sB[((j) & (RING - 1)) * RS]
#define SC(j) sC[((j) & (RING - 1)) * RS]
  const long long T = (long long)ncta_ * NT;
  const long long gt = (long long)cta_ * NT + tid;
  double* const dp = P.dp + gt;
  const long long nl = nlines<D>(P);
  const MibBlock* __restrict__ blk = P.blk[D];
  const double* __restrict__ fbet = P.fbet[D];
  const double* __restrict__ fgam = P.fgam[D];
  const double* __restrict__ rblk = P.rblk[D];
  const double E1 = step_e(P, io.e1, 2);
  const double E0 = step_e(P, io.e0, 0);
  const double kx = io.k;
  // per-direction constants by side (0 inside, 1 outside), in registers
  const double v0i = P.vd[D][0][0], v0o = P.vd[D][1][0];
  const double v1i = P.vd[D][0][1], v1o = P.vd[D][1][1];
  const double v2i = P.vd[D][0][2], v2o = P.vd[D][1][2];
  const double cai = P.ia[D][0], cao = P.ia[D][1];
  // prefix factor tables [side][row][bet, gam] and exact-solution tables of
  // the sweep axis [coordinate | sin 2x | cos 2x] into shared memory (they sit
  // on the recurrence chain; the staging stream would evict them from L1)
  const int nd = D == 0 ? P.nx : D == 1 ? P.ny : P.nz;
  double* const sP = sm + 3 * NS * SLOT;
  double* const sX = sP + 4 * nd;
  for (int i = tid; i < 4 * nd; i += NT) sP[i] = i < 2 * nd ? P.ptab[D][0][i] : P.ptab[D][1][i - 2 * nd];
  for (int i = tid; i < nd; i += NT) {
    sX[i] = P.ax[D][i];
    sX[nd + i] = P.s2[D][i];
    sX[2 * nd + i] = P.c2[D][i];
  }
  __syncthreads();

  // x lines are contiguous in memory and 2 KB apart, so a thread staging its
  // own line would touch 32 segments per warp instruction.  There the warp
  // stages and stores its 32 lines together (kCoop): lane e of copy q moves
  // row e % CH of line e / CH, so runs of CH lanes read one line's
  // consecutive rows, into that line's column of the ring.  The warp then
  // walks its lines' chunks in step, including lanes whose line is a face
  // line or past the end, which only help with the copies.
  constexpr bool kCoop = D == 0;
  const int lane = tid & 31;
  double* const sAw = sm + (tid - lane);  // the warp's first column of ring A
  const long long nxl = P.nx;

  for (long long t0 = gt - (kCoop ? lane : 0); t0 < nl; t0 += T) {
    const long long t = kCoop ? t0 + lane : t0;
    const bool act = t < nl;
    Line L;
    decode_line<D>(P, act ? t : nl - 1, L);
    const int n = L.n;
    const long long s = L.s;
    LineExact fx;
    line_exact<D>(P, L, fx);
    if (L.boundary && act) {
      if (io.bmode) {
        for (int j = 0; j < n; j++) {
          long long m = L.base + (long long)j * s;
          double S, R2;
          row_parts<D>(fx, sX, nd, j, S, R2);
          double v = outer_from(P, R2, E1);
          if (io.bmode == 2) v = v + P.dt * source_from(P, S, R2, E1, P.tag[m] & TAG_OUT);
          io.out[m] = v;
        }
      }
    }
    const bool solve = act && !L.boundary;
    if (!kCoop && !solve) continue;
    unsigned solvers = 0;
    if (kCoop) {
      __syncwarp();
      solvers = __ballot_sync(0xffffffffu, solve);
      if (!solvers) continue;
    }
    const int nch = (n + CH - 1) / CH;
    const int ls = P.lside[D][L.lid];
    const int bfirst = P.bstart[D][L.lid];
    const int bend = P.bstart[D][L.lid + 1];
    const int L1 = bfirst < bend ? blk[bfirst].L : n;  // first MIB row
    const double* pt = sP + ((ls >> 1) & 1) * 2 * nd;
    const bool two = KIND != K_COPY && io.add != io.stin;
    // row j of a field: g[j*s]; rows up to nch*CH-1 are readable (the fields
    // carry one chunk of slack past their end)
    const double* gA = (KIND == K_COPY ? io.add : io.stin) + L.base;
    const double* gB = io.add + L.base;
    const double* gC = fbet + L.base;
    // kCoop: the first MIB row of the line each of this lane's copies serves
    int L1q[CH];
    long long gq[CH];  // start of the line each copy serves, or -1 past the end
    if (kCoop) {
#pragma unroll
      for (int q = 0; q < CH; q++) {
        const int l = (q * 32 + lane) / CH;
        L1q[q] = __shfl_sync(0xffffffffu, L1, l);
        gq[q] = t0 + l < nl ? (t0 + l) * nxl + (q * 32 + lane) % CH : -1;
      }
    }
    auto stage = [&](int c) {
      if (kCoop) {
        if (c < nch) {
          const double* fA = KIND == K_COPY ? io.add : io.stin;
          double* aw = sAw + (c & (NS - 1)) * SLOT;
          double* bw = aw + NS * SLOT;
          double* cw = bw + NS * SLOT;
#pragma unroll
          for (int q = 0; q < CH; q++) {
            const int e = q * 32 + lane, l = e / CH, r = e % CH;
            if (gq[q] >= 0) {
              const long long g = gq[q] + (long long)c * CH;
              cp_async8(aw + r * RS + l, fA + g);
              if (two) cp_async8(bw + r * RS + l, io.add + g);
              if ((c + 1) * CH > L1q[q] && L1q[q] < n) cp_async8(cw + r * RS + l, fbet + g);
            }
          }
        }
        cp_async_commit();
        return;
      }
      if (c < nch) {
        const long long off = (long long)c * CH * s;
        double* a = sA + (c & (NS - 1)) * SLOT;
#pragma unroll
        for (int r = 0; r < CH; r++) cp_async8(a + r * RS, gA + off + r * s);
        if (two) {
          double* b = sB + (c & (NS - 1)) * SLOT;
#pragma unroll
          for (int r = 0; r < CH; r++) cp_async8(b + r * RS, gB + off + r * s);
        }
        if ((c + 1) * CH > L1 && L1 < n) {  // per-node factors exist only for lines with blocks
          double* cc = sC + (c & (NS - 1)) * SLOT;
#pragma unroll
          for (int r = 0; r < CH; r++) cp_async8(cc + r * RS, gC + off + r * s);
        }
      }
      cp_async_commit();
    };
    auto outer_at = [&](int j) -> double {
      double S, R2;
      row_parts<D>(fx, sX, nd, j, S, R2);
      return outer_from(P, R2, E1);
    };
    // right-hand side of a regular row from its stencil values
    auto rhs = [&](int j, double xm, double x0, double xp, double addv, double w0, double w1, double w2,
                   int side) -> double {
      if (KIND == K_COPY) return x0;
      double sum = 0.0;
      sum += xm * w0;
      sum += x0 * w1;
      sum += xp * w2;
      double r = kx * sum + addv;
      if (KIND == K_TS_Z) {
        double S, R2;
        row_parts<D>(fx, sX, nd, j, S, R2);
        r = r + P.hdt * source_from(P, S, R2, E0, side);
        r = r + P.hdt * source_from(P, S, R2, E1, side);
      }
      return r;
    };

    // ---- forward substitution with the precomputed factors (TDMA,
    // douglas_adi.cc:1794-1800): d'_j = (r_j - a_j d'_{j-1}) / bet_j
    for (int c = 0; c < NS - 2; c++) stage(c);
    int mb = bfirst;
    BlockHead hb, hb2;  // the next block and the one after (prefetched)
    load_head(blk, rblk, mb, bend, hb);
    load_head(blk, rblk, mb + 1, bend, hb2);
    int mside = (ls >> 1) & 1;
    double dprev = 0.0;
    int j = 1;
    for (int c = 0; c < nch; c++) {
      if (kCoop) __syncwarp();  // every lane is done with the slot restaged next
      stage(c + NS - 2);
      cp_async_wait<NS - 3>();  // chunks c-1, c, c+1 resident
      if (kCoop) {
        __syncwarp();  // and the other lanes' copies into this lane's column visible
        if (!solve) continue;
      }
      if (c == 0) {
        dprev = outer_at(0) / pt[0];
        dp[0] = dprev;
      }
      const int c0 = c * CH;
      const int cend = min(c0 + CH, n - 1);
      if (j >= cend) continue;
      if (j == c0 && cend == c0 + CH && hb.L >= cend && (cend <= L1 || c0 >= L1)) {
        // a chunk of regular rows, same side, factors from one source
        const double w0 = mside ? v0o : v0i, w1 = mside ? v1o : v1i, w2 = mside ? v2o : v2i;
        const double ac = mside ? cao : cai;
        const double* a = sA + (c & (NS - 1)) * SLOT;
        const double* ap = sA + ((c - 1) & (NS - 1)) * SLOT;
        const double* an = sA + ((c + 1) & (NS - 1)) * SLOT;
        const double* b = sB + (c & (NS - 1)) * SLOT;
        double* q = dp + (long long)c0 * T;
        auto run = [&](auto tag) {
          // tag: bet from the staged per-node factors, else from the prefix table
          constexpr bool kField = decltype(tag)::value;
          const double* bt = kField ? sC + (c & (NS - 1)) * SLOT : pt + 2 * c0;
          double xm = ap[(CH - 1) * RS];
          double x0 = a[0];
#pragma unroll
          for (int rr = 0; rr < CH; rr++) {
            const double xp = rr == CH - 1 ? an[0] : a[(rr + 1) * RS];
            const double r = rhs(c0 + rr, xm, x0, xp, two ? b[rr * RS] : x0, w0, w1, w2, mside);
            const double bet = kField ? bt[rr * RS] : bt[2 * rr];
            const double d = (r - ac * dprev) / bet;
            q[rr * T] = d;
            dprev = d;
            xm = x0;
            x0 = xp;
          }
        };
        if (c0 >= L1)
          run(BoolC<true>{});
        else
          run(BoolC<false>{});
        j = cend;
      } else {
        while (j < cend) {
          const double bet = j >= L1 ? SC(j) : pt[2 * j];
          if (j == hb.L) {
            // a MIB block: its rows' right-hand sides come mixed from the
            // block pre-pass (k_block_rhs); substitute them
            double d = (hb.r0 - hb.a0 * dprev) / bet;
            dp[(long long)j * T] = d;
            dprev = d;
            d = (hb.r1 - hb.a1 * dprev) / SC(j + 1);
            dp[(long long)(j + 1) * T] = d;
            dprev = d;
            if (hb.kind == 3) {
              d = (hb.r2 - hb.a2 * dprev) / SC(j + 2);
              dp[(long long)(j + 2) * T] = d;
              dprev = d;
            }
            mside = (hb.sides >> (hb.kind - 1)) & 1;
            j += hb.kind;
            mb++;
            hb = hb2;
            load_head(blk, rblk, mb + 1, bend, hb2);
          } else {
            const double r = rhs(j, SA(j - 1), SA(j), SA(j + 1), two ? SB(j) : SA(j), mside ? v0o : v0i,
                                 mside ? v1o : v1i, mside ? v2o : v2i, mside);
            const double d = (r - (mside ? cao : cai) * dprev) / bet;
            dp[(long long)j * T] = d;
            dprev = d;
            j++;
          }
        }
      }
    }
    if (solve) {
      // last row: the Dirichlet identity row (a = 0)
      const double r = outer_at(n - 1);
      const double a = 0.0;
      const double bet = n - 1 >= L1 ? SC(n - 1) : pt[2 * (n - 1)];
      dp[(long long)(n - 1) * T] = (r - a * dprev) / bet;
    }
    cp_async_wait<0>();

    // ---- back substitution u_j = d'_j - gam_{j+1} u_{j+1} (douglas_adi.cc:
    // 1805-1806), staged back through the ring: field A = d'_j, field B =
    // gam_{j+1} where it comes from the per-node factors.  The fence orders
    // this thread's d' stores before the asynchronous copies that read them.
    __threadfence_block();
    const double* gG = fgam + L.base;
    auto bstage = [&](int c) {
      if (c >= 0) {
        double* a = sA + (c & (NS - 1)) * SLOT;
        const double* g = dp + (long long)c * CH * T;
#pragma unroll
        for (int r = 0; r < CH; r++) cp_async8(a + r * RS, g + r * T);
        if ((c + 1) * CH >= L1 && L1 < n) {
          double* b = sB + (c & (NS - 1)) * SLOT;
          const long long off = ((long long)c * CH + 1) * s;
#pragma unroll
          for (int r = 0; r < CH; r++) cp_async8(b + r * RS, gG + off + r * s);
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
      if (kCoop) __syncwarp();  // the previous chunk's stores have read its slot
      bstage(c - NS + 1);
      cp_async_wait<NS - 1>();
      const int c0 = c * CH;
      // kCoop: results go to this lane's column of the slot, then the warp
      // stores its lines' rows together
      double* const aslot = sA + (c & (NS - 1)) * SLOT;
      if (!solve) {
      } else if (!io.last && c0 + CH <= n - 1 && (c0 + CH < L1 || c0 + 1 >= L1)) {
        // every row has a successor; gam_{j+1} from one source
        double* a = aslot;
        double* o = io.out + L.base + (long long)c0 * s;
        auto run = [&](auto tag) {
          // tag: gam_{j+1} from the staged per-node factors, else from the
          // prefix table (pt + 2*c0 + 3 is gam of row c0 + 1)
          constexpr bool kField = decltype(tag)::value;
          const double* gb = kField ? sB + (c & (NS - 1)) * SLOT : pt + 2 * c0 + 3;
#pragma unroll
          for (int rr = CH - 1; rr >= 0; rr--) {
            const double gm = kField ? gb[rr * RS] : gb[2 * rr];
            double u = a[rr * RS];
            u -= gm * unext;
            unext = u;
            if (kCoop)
              a[rr * RS] = u;
            else
              o[rr * s] = u;
          }
        };
        if (c0 + 1 >= L1)
          run(BoolC<true>{});
        else
          run(BoolC<false>{});
      } else {
        for (int rr = CH - 1; rr >= 0; rr--) {
          const int jj = c0 + rr;
          if (jj >= n) continue;
          double u = SA(jj);
          if (jj != n - 1) u -= (jj + 1 >= L1 ? SB(jj) : pt[2 * (jj + 1) + 1]) * unext;
          unext = u;
          double v = u;
          if (io.last) {
            int side;
            if (jj == 0) {
              side = ls & 1;
            } else if (jj == n - 1) {
              side = (ls >> 2) & 1;
            } else if (jj >= dbL && jj < dbL + dbK) {
              side = (dbS >> (jj - dbL)) & 1;
              if (jj == dbL) {
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
            double S, R2;
            row_parts<D>(fx, sX, nd, jj, S, R2);
            v = u + P.dt * source_from(P, S, R2, E1, side);
          }
          if (kCoop)
            SA(jj) = v;
          else
            io.out[L.base + (long long)jj * s] = v;
        }
      }
      if (kCoop) {
        __syncwarp();
        const double* aw = sAw + (c & (NS - 1)) * SLOT;
#pragma unroll
        for (int q = 0; q < CH; q++) {
          const int e = q * 32 + lane, l = e / CH, r = e % CH;
          if (((solvers >> l) & 1u) && c0 + r < n) io.out[gq[q] + c0] = aw[r * RS + l];
        }
      }
    }
    cp_async_wait<0>();
  }
#undef SA
#undef SB
#undef SC
}

template <int D, int KIND, int CH, int NS, int NT>
__global__ void __launch_bounds__(NT, 1) k_sweep(const __grid_constant__ Dev P, const SweepIO io) {
  k_sweep_body<D, KIND, CH, NS, NT>(P, blockIdx.x, gridDim.x, io);
}

// Thomas factors of the lines that cross the interface (the factor half of
// TDMA, douglas_adi.cc:1790-1798: gam_j = c_{j-1}/bet, bet = b_j - a_j*gam_j,
// the same IEEE operations as the host's prefix tables), once at setup, one
// thread per line.  A line's rows are the identity on its faces, the regular
// three-point rows of the node's side elsewhere, and the Convert2Tri rows of
// its blocks; from the first MIB row on, bet and gam are stored per node in
// FP64 (fbet, fgam) and as 1/bet and gam in FP32 (fib32, fgam32).  A zero
// pivot sets *zero_pivot.
template <int D>
__global__ void __launch_bounds__(TPB) k_factor_lines(const __grid_constant__ Dev P, int* zero_pivot) {
  const long long t = (long long)blockIdx.x * TPB + threadIdx.x;
  if (t >= nlines<D>(P)) return;
  Line L;
  decode_line<D>(P, t, L);
  if (L.boundary) return;
  const int bfirst = P.bstart[D][L.lid], bend = P.bstart[D][L.lid + 1];
  if (bfirst == bend) return;
  const MibBlock* const blk = P.blk[D];
  const int n = L.n;
  const int L1 = blk[bfirst].L;
  int b = bfirst;
  double bet = 1.0;   // row 0: b = 1
  double cprev = 0.0; // c of the previous row
  for (int j = 1; j < n; j++) {
    double aj, bj, cj;
    if (j == n - 1) {
      aj = 0.0;
      bj = 1.0;
      cj = 0.0;
    } else if (b < bend && j >= blk[b].L) {
      const int q = j - blk[b].L;
      aj = blk[b].ia[q];
      bj = blk[b].ib[q];
      cj = blk[b].ic[q];
      if (q == blk[b].kind - 1) b++;
    } else {
      const int side = (P.tag[L.base + (long long)j * L.s] & TAG_OUT) ? 1 : 0;
      aj = P.ia[D][side];
      bj = P.ib[D][side];
      cj = P.ic[D][side];
    }
    const double gm = cprev / bet;
    bet = bj - aj * gm;
    if (bet == 0.0) {
      atomicOr(zero_pivot, 1);
      return;
    }
    if (j >= L1) {
      // (the factor fields are read-only to the step kernels; setup fills them here)
      const long long m = L.base + (long long)j * L.s;
      const_cast<double*>(P.fbet[D])[m] = bet;
      const_cast<double*>(P.fgam[D])[m] = gm;
      const_cast<float*>(P.fib32[D])[m] = (float)(1.0 / bet);
      const_cast<float*>(P.fgam32[D])[m] = (float)gm;
    }
    cprev = cj;
  }
}

// Refresh_Jump (intersection.cc:2294-2490): [u] and u_dir per crossing.
__device__ __forceinline__ void k_jumps_body(const Dev& P, unsigned cta_, unsigned ncta_, double E) {
  int c = cta_ * TPB + threadIdx.x;
  if (c >= P.ncross) return;
  E = step_e(P, E, 2);
  const CrossConst q = P.cc[c];
  double ju, jb[3];
  exact_jumps(P, q, E, ju, jb);
  double bxi = q.p[0] * jb[0] + q.p[1] * jb[1] + q.p[2] * jb[2];
  P.jv[c] = make_double2(ju, q.pinv * bxi);
}

__global__ void __launch_bounds__(TPB) k_jumps(const __grid_constant__ Dev P, double E) {
  k_jumps_body(P, blockIdx.x, gridDim.x, E);
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
#define MTS_SHAPES(X)                                                                        \
  X(0, 8, 8, 128) X(1, 4, 16, 128) X(2, 4, 8, 256) X(3, 8, 4, 256) X(4, 4, 8, 192) X(5, 4, 8, 288) \
  X(6, 4, 4, 384) X(7, 4, 4, 512) X(8, 4, 4, 448) X(9, 4, 4, 128)

template <int D, int KIND, int CH, int NS, int NT>
void sweep_shape(const Dev& P, const SweepIO& io, cudaStream_t st) {
  // persistent CTAs, one per SM at most, no more than the lines need
  const int nd = D == 0 ? P.nx : D == 1 ? P.ny : P.nz;
  k_sweep<D, KIND, CH, NS, NT><<<sweep_grid(P, nlines<D>(P), NT), NT, shape_smem<CH, NS, NT, D>(nd), st>>>(P, io);
}

template <int D, int KIND>
void sweep(const Dev& P, const SweepIO& io, int shape, cudaStream_t st) {
  if (P.nblk[D] > 0) k_block_rhs<D, KIND><<<(P.nblk[D] + TPB - 1) / TPB, TPB, 0, st>>>(P, io, P.nblk[D]);
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
                       kMaxSweepSmem);
  MTS_SHAPES(MTS_ATTR)
#undef MTS_ATTR
}

}  // namespace

int sweep_shape_count() { return 10; }

bool sweep_shape_fits(int shape, int nmax) {
  switch (shape) {
#define MTS_FITS(id, ch, ns, nt) \
  case id:                       \
    return shape_smem<ch, ns, nt>(nmax) <= (size_t)kMaxSweepSmem;
    MTS_SHAPES(MTS_FITS)
#undef MTS_FITS
    default:
      return false;
  }
}
int sweep_shape_max_threads() { return 512; }

void configure_kernels() {
  set_smem_attr<0, K_COPY>();
  set_smem_attr<1, K_COPY>();
  set_smem_attr<2, K_COPY>();
  set_smem_attr<0, K_STENCIL>();
  set_smem_attr<1, K_STENCIL>();
  set_smem_attr<2, K_STENCIL>();
  set_smem_attr<2, K_TS_Z>();
}

__global__ void k_tick(int* step) { ++*step; }

void launch_tick(const Dev& P, cudaStream_t st) { k_tick<<<1, 1, 0, st>>>(P.tstep); }

void launch_jumps(const Dev& P, double E, cudaStream_t st) {
  k_jumps<<<(P.ncross + TPB - 1) / TPB, TPB, 0, st>>>(P, E);
}

unsigned pointwise_rows_grid(const Dev& P) { return pointwise_blocks(P); }

int launch_factor_lines(const Dev& P, int* zero_pivot, cudaStream_t st) {
  int launches = 0;
  if (P.nblk[0] > 0) {
    k_factor_lines<0><<<(unsigned)((nlines<0>(P) + TPB - 1) / TPB), TPB, 0, st>>>(P, zero_pivot);
    launches++;
  }
  if (P.nblk[1] > 0) {
    k_factor_lines<1><<<(unsigned)((nlines<1>(P) + TPB - 1) / TPB), TPB, 0, st>>>(P, zero_pivot);
    launches++;
  }
  if (P.nblk[2] > 0) {
    k_factor_lines<2><<<(unsigned)((nlines<2>(P) + TPB - 1) / TPB), TPB, 0, st>>>(P, zero_pivot);
    launches++;
  }
  return launches;
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
int launch_step(const Dev& P, const StepTimes& T, double*& u0, double*& u1, cudaStream_t st, cudaEvent_t* ev,
                const SideStream* side) {
  int launches = 0;
  int slot = 0;
  auto mark = [&](int k) {
    if (ev) cudaEventRecord(ev[2 * slot + k], st);
    if (k == 1) slot++;
  };
  // Douglas-ADI: the jumps and the MIB rows of the first right-hand side
  // (which read the jumps) run on the side stream beside its pointwise pass;
  // the two passes write disjoint nodes and read only u^n.
  const bool fork = side && side->stream && P.method == 0 && (P.ncross > 0 || P.nmibnode > 0);
  cudaStream_t sst = fork ? side->stream : st;
  if (fork) {
    cudaEventRecord(side->fork, st);
    cudaStreamWaitEvent(sst, side->fork, 0);
  }
  if (ev) cudaEventRecord(ev[0], sst);
  if (P.ncross > 0) {
    k_jumps<<<(P.ncross + TPB - 1) / TPB, TPB, 0, sst>>>(P, T.e_next);
    launches++;
  }
  if (ev) cudaEventRecord(ev[1], sst);
  slot = 1;
  SweepIO io{};
  io.e1 = T.e_next;
  io.e0 = T.e_prev;
  if (P.method == 0) {
    // Douglas-ADI.  u1 <- uhs (pointwise); x sweep in place gives u*; y sweep
    // builds uhss = -dt D_yy u^n + u* and solves in place (u**); z sweep builds
    // uh1 = -dt D_zz u^n + u** and writes u^{n+1} over u^n in u0 (a z line
    // reads only its own nodes of u^n; its faces get Outer_u(t_next), the
    // value u** holds there).  The state stays in u0, u1 is scratch.
    mark(0);
    if (P.nmibnode > 0) {
      k_adi_rhs_mib<<<(P.nmibnode + TPB - 1) / TPB, TPB, 0, sst>>>(P, u0, u1, T.e_next);
      launches++;
    }
    k_adi_rhs<2><<<pointwise_blocks(P), TPB, 0, st>>>(P, u0, u1, T.e_next);
    if (fork) {
      cudaEventRecord(side->join, sst);
      cudaStreamWaitEvent(st, side->join, 0);
    }
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
    io.out = u0;
    io.bmode = 1;
    mark(0);
    sweep<2, K_STENCIL>(P, io, P.shape[2], st);
    mark(1);
    launches += 4;
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
    if (P.nmibnode > 0) {
      k_ts_explicit_mib<0><<<(P.nmibnode + TPB - 1) / TPB, TPB, 0, st>>>(P, u0, u1);
      launches++;
    }
    mark(1);
    mark(0);
    k_ts_explicit<1><<<pointwise_blocks(P), TPB, 0, st>>>(P, u1, u0, T.e_half);
    if (P.nmibnode > 0) {
      k_ts_explicit_mib<1><<<(P.nmibnode + TPB - 1) / TPB, TPB, 0, st>>>(P, u1, u0);
      launches++;
    }
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
  // every method sweeps each direction once; each sweep with MIB blocks is
  // preceded by its block pre-pass
  for (int d = 0; d < 3; d++) launches += P.nblk[d] > 0;
  return launches;
}

// ---------------------------------------------------------------------------
// Error norms with no allocation (mts_norms_noalloc).  A caller that cannot
// allocate device memory still needs somewhere for the per-block partials of
// the reduction, so they live in one statically sized module array instead
// of a buffer owned by a handle.  Layout, in doubles:
//   [0]        ticket counter (read as unsigned): MUST be zero when the
//              kernel starts; the host clears it before each launch and the
//              last block leaves it at zero
//   [32..34]   the result triple (max |e|, argmax key, L2)
//   [64 ..)    3 doubles of partials per block, kNoAllocMaxBlocks blocks
// Every call on a device uses the same array, so calls that overlap in time
// on one device (two handles, two streams, two host threads) race.

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

cudaError_t noalloc_scratch_address(double** p) { return cudaGetSymbolAddress((void**)p, g_noalloc_scratch); }

namespace {

// One launch: each block reduces its share exactly as k_norms_partial does;
// the block that takes the last ticket then combines the partials exactly as
// k_norms_final does, so the triple is bit-identical to launch_norms' with
// the same block count.
__global__ void __launch_bounds__(NB_TPB) k_norms_noalloc(const Dev P, double E, const double* u, double* scratch) {
  __shared__ double smax[NB_TPB], ssum[NB_TPB];
  __shared__ long long skey[NB_TPB];
  __shared__ int last;
  unsigned* const ticket = reinterpret_cast<unsigned*>(scratch);
  double* const res = scratch + 32;
  double* const part = scratch + 64;
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
    __threadfence();  // the partial is visible device-wide before the ticket
    last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  const int nb = gridDim.x;
  vmax = 0.0;
  vsum = 0.0;
  vkey = 0x7fffffffffffffffLL;
  for (int i = threadIdx.x; i < nb; i += NB_TPB) {
    // other blocks wrote these: read through L2, past this SM's L1
    better(vmax, vkey, __ldcg(part + 3 * i), (long long)__ldcg(part + 3 * i + 1));
    vsum += __ldcg(part + 3 * i + 2);
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
    res[0] = smax[0];
    res[1] = smax[0] > 0.0 ? (double)skey[0] : 0.0;
    res[2] = sqrt(ssum[0] / (1.0 * P.nx * P.ny * P.nz));
    *ticket = 0u;
  }
}

}  // namespace

int launch_norms_noalloc(const Dev& P, double E, const double* u, double* scratch, int nb, cudaStream_t st) {
  k_norms_noalloc<<<nb, NB_TPB, 0, st>>>(P, E, u, scratch);
  return 1;
}

// ---------------------------------------------------------------------------
// Batched plain steps: the kernels above, launched once for many problems.

namespace {

struct Roles {
  int stin, add, out;  // fields: 0 = u0, 1 = u1
  int ksel;            // explicit factor: 0 none, 1 -dt (ADI), 2 0.5*dt (LOD-CN, TS)
  int jumps, bmode, last;
};

__device__ __forceinline__ SweepIO make_io(const Dev& P, const Roles& r) {
  SweepIO io{};
  io.stin = r.stin ? P.u1 : P.u0;
  io.add = r.add ? P.u1 : P.u0;
  io.out = r.out ? P.u1 : P.u0;
  io.k = r.ksel == 1 ? -P.dt : r.ksel == 2 ? P.kex : 0.0;
  io.jumps = r.jumps;
  io.bmode = r.bmode;
  io.last = r.last;
  io.e0 = io.e1 = 0.0;  // from the step table
  return io;
}

__global__ void __launch_bounds__(TPB) kb_jumps(const Dev* __restrict__ Ps, const BatchItem* __restrict__ items) {
  BATCH_PROLOGUE
  k_jumps_body(P, w.cta, w.ncta, 0.0);
}

__global__ void __launch_bounds__(TPB) kb_adi_rhs(const Dev* __restrict__ Ps, const BatchItem* __restrict__ items) {
  BATCH_PROLOGUE
  k_adi_rhs_body<2>(P, w.cta, w.ncta, P.u0, P.u1, 0.0);
}

__global__ void __launch_bounds__(TPB) kb_adi_rhs_mib(const Dev* __restrict__ Ps,
                                                      const BatchItem* __restrict__ items) {
  BATCH_PROLOGUE
  k_adi_rhs_mib_body(P, w.cta, w.ncta, P.u0, P.u1, 0.0);
}

template <int D>
__global__ void __launch_bounds__(TPB) kb_ts_explicit(const Dev* __restrict__ Ps,
                                                      const BatchItem* __restrict__ items, int in) {
  BATCH_PROLOGUE
  k_ts_explicit_body<D>(P, w.cta, w.ncta, in ? P.u1 : P.u0, in ? P.u0 : P.u1, 0.0);
}

template <int D>
__global__ void __launch_bounds__(TPB) kb_ts_explicit_mib(const Dev* __restrict__ Ps,
                                                          const BatchItem* __restrict__ items, int in) {
  BATCH_PROLOGUE
  k_ts_explicit_mib_body<D>(P, w.cta, w.ncta, in ? P.u1 : P.u0, in ? P.u0 : P.u1);
}

template <int D, int KIND>
__global__ void __launch_bounds__(TPB) kb_block_rhs(const Dev* __restrict__ Ps, const BatchItem* __restrict__ items,
                                                    Roles r) {
  BATCH_PROLOGUE
  k_block_rhs_body<D, KIND>(P, w.cta, w.ncta, make_io(P, r), P.nblk[D]);
}

// the small-CTA shape (several CTAs per SM) for batches of small problems
constexpr int BCH = 4, BNS = 4, BNT = 128;

template <int D, int KIND>
__global__ void __launch_bounds__(BNT) kb_sweep(const Dev* __restrict__ Ps, const BatchItem* __restrict__ items,
                                                Roles r) {
  BATCH_PROLOGUE
  k_sweep_body<D, KIND, BCH, BNS, BNT>(P, w.cta, w.ncta, make_io(P, r));
}

__global__ void kb_tick(const Dev* __restrict__ Ps, int n) {
  const int i = blockIdx.x * TPB + threadIdx.x;
  if (i < n && *Ps[i].tstep < Ps[i].tstop) ++*Ps[i].tstep;
}

template <int D, int KIND>
void bsweep(const BatchPlan& b, const Roles& r, cudaStream_t st, int& launches) {
  if (b.nblk[D] > 0) {
    kb_block_rhs<D, KIND><<<b.nblk[D], TPB, 0, st>>>(b.Ps, b.blk[D], r);
    launches++;
  }
  if (b.nsw[D] > 0) {
    kb_sweep<D, KIND><<<b.nsw[D], BNT, shape_smem<BCH, BNS, BNT, D>(b.nmax), st>>>(b.Ps, b.sw[D], r);
    launches++;
  }
}

template <int D, int KIND>
void bsweep_attr() {
  cudaFuncSetAttribute(kb_sweep<D, KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       kMaxSweepSmem - (int)sizeof(Dev) - 64);
}

}  // namespace

int batch_sweep_threads() { return BNT; }

int launch_batch_jumps(const Dev* Ps, const BatchItem* items, int nitems, cudaStream_t st) {
  if (nitems <= 0) return 0;
  kb_jumps<<<nitems, TPB, 0, st>>>(Ps, items);
  return 1;
}

int launch_batch_tick(const Dev* Ps, int n, cudaStream_t st) {
  kb_tick<<<(n + TPB - 1) / TPB, TPB, 0, st>>>(Ps, n);
  return 1;
}

unsigned jumps_grid(const Dev& P) { return (unsigned)((P.ncross + TPB - 1) / TPB); }
unsigned mib_grid(const Dev& P) { return (unsigned)((P.nmibnode + TPB - 1) / TPB); }
unsigned block_grid(const Dev& P, int d) { return (unsigned)((P.nblk[d] + TPB - 1) / TPB); }
unsigned batch_sweep_grid(const Dev& P, int d) {
  return sweep_grid(P, d == 0 ? nlines<0>(P) : d == 1 ? nlines<1>(P) : nlines<2>(P), BNT);
}

void configure_batch_kernels() {
  bsweep_attr<0, K_COPY>();
  bsweep_attr<1, K_COPY>();
  bsweep_attr<2, K_COPY>();
  bsweep_attr<0, K_STENCIL>();
  bsweep_attr<1, K_STENCIL>();
  bsweep_attr<2, K_STENCIL>();
  bsweep_attr<2, K_TS_Z>();
}

// One step of every problem of the plan, the launch sequence of launch_step.
int launch_step_batch(const BatchPlan& b, cudaStream_t st) {
  int launches = 0;
  if (b.njumps > 0) {
    kb_jumps<<<b.njumps, TPB, 0, st>>>(b.Ps, b.jumps);
    launches++;
  }
  if (b.method == 0) {
    kb_adi_rhs<<<b.nrows, TPB, 0, st>>>(b.Ps, b.rows);
    launches++;
    if (b.nmib > 0) {
      kb_adi_rhs_mib<<<b.nmib, TPB, 0, st>>>(b.Ps, b.mib);
      launches++;
    }
    bsweep<0, K_COPY>(b, Roles{1, 1, 1, 0, 0, 0, 0}, st, launches);
    bsweep<1, K_STENCIL>(b, Roles{0, 1, 1, 1, 0, 0, 0}, st, launches);
    bsweep<2, K_STENCIL>(b, Roles{0, 1, 0, 1, 0, 1, 0}, st, launches);
  } else if (b.method == 1 || b.method == 2) {
    if (b.method == 2) {
      bsweep<0, K_STENCIL>(b, Roles{0, 0, 0, 2, 1, 1, 0}, st, launches);
      bsweep<1, K_STENCIL>(b, Roles{0, 0, 0, 2, 1, 1, 0}, st, launches);
      bsweep<2, K_STENCIL>(b, Roles{0, 0, 0, 2, 1, 2, 1}, st, launches);
    } else {
      bsweep<0, K_COPY>(b, Roles{0, 0, 0, 2, 1, 1, 0}, st, launches);
      bsweep<1, K_COPY>(b, Roles{0, 0, 0, 2, 1, 1, 0}, st, launches);
      bsweep<2, K_COPY>(b, Roles{0, 0, 0, 2, 1, 2, 1}, st, launches);
    }
  } else {
    kb_ts_explicit<0><<<b.nrows, TPB, 0, st>>>(b.Ps, b.rows, 0);
    launches++;
    if (b.nmib > 0) {
      kb_ts_explicit_mib<0><<<b.nmib, TPB, 0, st>>>(b.Ps, b.mib, 0);
      launches++;
    }
    kb_ts_explicit<1><<<b.nrows, TPB, 0, st>>>(b.Ps, b.rows, 1);
    launches++;
    if (b.nmib > 0) {
      kb_ts_explicit_mib<1><<<b.nmib, TPB, 0, st>>>(b.Ps, b.mib, 1);
      launches++;
    }
    bsweep<2, K_TS_Z>(b, Roles{0, 0, 0, 2, 1, 1, 0}, st, launches);
    bsweep<1, K_COPY>(b, Roles{0, 0, 0, 2, 1, 0, 0}, st, launches);
    bsweep<0, K_COPY>(b, Roles{0, 0, 0, 2, 1, 0, 0}, st, launches);
  }
  kb_tick<<<(b.n + TPB - 1) / TPB, TPB, 0, st>>>(b.Ps, b.n);
  return launches + 1;
}

}  // namespace mts

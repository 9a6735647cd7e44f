// Fast FP64 form of the Douglas-ADI step (precision = 2).
//
// The Douglas step (douglas_adi.cc:66-1110) written for the increments
// d* = u* - u^n, d** = u** - u^n and d = u^{n+1} - u^n reads
//   (I - A_x) d*  = rho = dt (A_x u^n + A_y u^n + A_z u^n + src)
//   (I - A_y) d** = d*
//   (I - A_z) d   = d**,      u^{n+1} = u^n + d,
// with d = Outer_u(t^{n+1}) - u^n on the faces (A_d = dt beta D_dd with the
// MIB rows, src = f plus the jump terms of Src_2nd, douglas_adi.cc:1123-1428).
// Everything here is FP64; the result differs from the reference's sequence
// of operations only by rounding.
//
// Lines are split by kind.  Most lines do not cross the interface: their
// Thomas factors are those of a line of one side, from a per-side row table,
// and their kernels carry no dependent memory reads.  The lines that cross
// the interface (a few tens of percent at most) have their own factors and
// MIB blocks; they are solved by separate kernels on a second stream, at the
// same time as the others.  A step is:
//
//   kf_mib  the right-hand side of every MIB row (the explicit MIB sums of
//           all three directions and the jump terms, one thread per node),
//           written into d at those nodes;
//   kf_xw   rho of the regular x lines (and d on the face lines), fused with
//           their solves: a CTA walks a column of planes for TY lines with
//           the stencil's planes in a shared-memory ring filled by bulk
//           copies (see the kernel);
//   kf_xc   the same for the x lines that cross the interface, their x
//           blocks' Convert2Tri row operations first (douglas_adi.cc:
//           1554-1675) (side stream);
//   kf_yt   the regular y lines, solved in place on d*, in tiles of NL
//           neighbouring lines (the same row of NL lines is NL consecutive
//           doubles) copied into shared memory with cp.async, double-buffered
//           so that the next tile's copy overlaps this tile's solves;
//   kf_yc   the y lines that cross the interface, one warp per line, their
//           Convert2Tri row operations first (side stream);
//   kf_yt / kf_yc for z, with the update u^{n+1} = u^n + d (u^n of a tile
//           is copied in while the tile is solved).
//
// Line solve: with the Thomas factors fixed (bet_j, gam_j of TDMA,
// douglas_adi.cc:1784-1807), both recurrences are first-order and linear:
//   forward   d_j = (r_j - a_j d_{j-1}) / bet_j = ib_j r_j + p_j d_{j-1}
//   backward  x_j = d_j - gam_{j+1} x_{j+1}    = d_j + q_j x_{j+1}
// with ib = 1/bet, p = -a/bet, q = -gam_{j+1} = -c_j/bet_j.  On every row
// that is not a MIB block row, a = c (the weights beta/h^2 on both sides of a
// node are the same number), so q = p exactly: the tables and the crossing
// lines' coefficients hold (ib, p) per row, and only block rows carry their
// own q.  Lane l of the warp takes the rows [l MX, l MX + MX); each lane runs
// its rows from a zero carry, the lanes' affine end maps are composed by a
// shuffle scan, and a second pass runs the rows again from the true carry.
#include <cuda_runtime.h>

#include <algorithm>

#include "device.h"
#include "device_common.cuh"

namespace mts {
namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int YZ_NL = 16;  // lines per tile of kf_yt (one warp each): rows of 128 bytes
constexpr int CW = 8;     // warps per CTA of the crossing-line kernels
constexpr int X_NFACE = 8;  // CTAs of kf_xw that fill the face lines
constexpr long long kWaitCycles = 1LL << 32;  // ~2 s of SM clock: a bulk copy that has not landed by then never will

// ---------------------------------------------------------------------------
// Bulk copies into shared memory with mbarrier completion

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_expect(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
// src and dst 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void bulk_copy(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for the phase of the given parity to complete, giving up after
// kWaitCycles clocks of this SM.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
  if (mbar_test(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_test(bar, parity))
    if (clock64() - t0 > kWaitCycles) return false;
  return true;
}
// Orders this thread's generic-proxy shared-memory accesses before later
// bulk copies into the same memory.
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// ---------------------------------------------------------------------------
// Jump data on the fly (Refresh_Jump, intersection.cc:2294-2490): [u] and
// u_dir of crossing c at the step's exp(-t), the values k_jumps stores.

__device__ __forceinline__ double2 jump_at(const Dev& P, int c, double E) {
  const CrossConst& q = P.cc[c];
  double ju, jb[3];
  if (P.eq == 0) {
    ju = 100.0 - 80.0;
    for (int d = 0; d < 3; d++) jb[d] = 0.0;
  } else {
    ju = q.R2 * E - q.S * E;
    const double xyz[3] = {q.x, q.y, q.z};
    for (int d = 0; d < 3; d++) jb[d] = P.bo * ((2.0 * xyz[d]) * E) - P.bi * (q.D[d] * E);
  }
  const double bxi = q.p[0] * jb[0] + q.p[1] * jb[1] + q.p[2] * jb[2];
  return make_double2(ju, q.pinv * bxi);
}

// Src_2nd's jump terms of row r of block b (douglas_adi.cc:1156-1427).
__device__ __forceinline__ double src_jumps(const Dev& P, double E, double src, const MibBlock& b, int r,
                                            const double* vd) {
  if (b.kind == 2) {
    const double2 J = jump_at(P, b.c0, E);
    if (r == 0) return src + vd[2] * (J.x * b.w[1][4] + J.y * b.w[1][5]);
    return src + vd[0] * (J.x * b.w[0][4] + J.y * b.w[0][5]);
  }
  const double2 Jl = jump_at(P, b.c0, E), Jr = jump_at(P, b.c1, E);
  if (r == 0) return src + vd[2] * corner_jumps(b.w[1], Jl, Jr);
  if (r == 1) {
    src = src + vd[0] * corner_jumps(b.w[0], Jl, Jr);
    return src + vd[2] * corner_jumps(b.w[3], Jl, Jr);
  }
  return src + vd[0] * corner_jumps(b.w[2], Jl, Jr);
}

// rho at a MIB node m = (ix, iy, iz): the explicit MIB sums of
// douglas_adi.cc:112-210 (no jumps) in every direction the node is a block
// row of, the regular three-point sums in the others, and the jump terms of
// Src_2nd.  ref: the node's block in x, y, z (-1: none).
__device__ __noinline__ double rho_mib(const Dev& P, const double* __restrict__ un, double E, long long m, int ix,
                                       int iy, int iz, int tg, int4 ref) {
  const int side = tg & TAG_OUT;
  const long long sy = P.nx, sz = (long long)P.nx * P.ny;
  const double* vdx = P.vd[0][side];
  const double* vdy = P.vd[1][side];
  const double* vdz = P.vd[2][side];
  const MibBlock* xb = ref.x >= 0 ? &P.blk[0][ref.x] : nullptr;
  const MibBlock* yb = ref.y >= 0 ? &P.blk[1][ref.y] : nullptr;
  const MibBlock* zb = ref.z >= 0 ? &P.blk[2][ref.z] : nullptr;
  double sx, sy_, sz_;
  if (xb) {
    const long long base = m - ix;
    sx = mib_sum(*xb, ix - xb->L, [&](int j) { return un[base + j]; }, vdx, false, P.jv);
  } else {
    sx = (un[m - 1] * vdx[0] + un[m] * vdx[1]) + un[m + 1] * vdx[2];
  }
  if (yb) {
    const long long base = ix + sz * iz;
    sy_ = mib_sum(*yb, iy - yb->L, [&](int j) { return un[base + (long long)j * sy]; }, vdy, false, P.jv);
  } else {
    sy_ = (un[m - sy] * vdy[0] + un[m] * vdy[1]) + un[m + sy] * vdy[2];
  }
  if (zb) {
    const long long base = ix + (long long)P.nx * iy;
    sz_ = mib_sum(*zb, iz - zb->L, [&](int j) { return un[base + (long long)j * sz]; }, vdz, false, P.jv);
  } else {
    sz_ = (un[m - sz] * vdz[0] + un[m] * vdz[1]) + un[m + sz] * vdz[2];
  }
  double src = source(P, E, side, ix, iy, iz);
  if (xb) src = src_jumps(P, E, src, *xb, ix - xb->L, vdx);
  if (yb) src = src_jumps(P, E, src, *yb, iy - yb->L, vdy);
  if (zb) src = src_jumps(P, E, src, *zb, iz - zb->L, vdz);
  return P.dt * (((sx + sy_) + sz_) + src);
}

// The Convert2Tri row operations of a line's blocks on its right-hand side
// in shared memory (buf: the line's rows, stride 1), and their rows' own q
// into qbuf; one lane per block.
template <int D>
__device__ __forceinline__ void block_rows(const Dev& P, double* buf, double* qbuf, int bfirst, int bend, int lane,
                                           bool ops) {
  for (int k = bfirst + lane; k < bend; k += 32) {
    const MibBlock& b = P.blk[D][k];
    const int L = b.L, kind = b.kind;
    const double* const bq = P.fbq[D] + 3 * (long long)k;
    double* r = buf + L;
    if (ops) {
      if (kind == 2) {
        double r0 = r[0], r1 = r[1];
        r1 -= b.rate[0] * r0;
        r0 -= b.rate[1] * r1;
        r[0] = r0;
        r[1] = r1;
      } else {
        double r0 = r[0], r1 = r[1], r2 = r[2];
        r1 -= b.rate[0] * r0;
        r2 -= b.rate[1] * r0;
        r0 -= b.rate[2] * r2;
        r1 -= b.rate[3] * r2;
        r2 -= b.rate[4] * r1;
        r0 -= b.rate[5] * r1;
        r[0] = r0;
        r[1] = r1;
        r[2] = r2;
      }
    }
    for (int q = 0; q < kind; q++) qbuf[L + q] = bq[q];
  }
}

// ---------------------------------------------------------------------------
// Segmented line solves on a line held in shared memory (buf[j], j < n:
// right-hand side in, solution out).  Lane l owns rows jb = l MX .. jb+MX-1.

// Inclusive scan of the maps c -> A c + B over the lanes (lane 0 first), and
// the carry into each lane: the composition over the lanes before it,
// applied to 0.
__device__ __forceinline__ double carry_up(double A, double B, int lane) {
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const double Ap = __shfl_up_sync(FULL, A, off), Bp = __shfl_up_sync(FULL, B, off);
    if (lane >= off) {
      B = fma(A, Bp, B);
      A = A * Ap;
    }
  }
  const double C = __shfl_up_sync(FULL, B, 1);
  return lane == 0 ? 0.0 : C;
}
// The same from the last lane down (suffix scan).
__device__ __forceinline__ double carry_down(double A, double B, int lane) {
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const double Ap = __shfl_down_sync(FULL, A, off), Bp = __shfl_down_sync(FULL, B, off);
    if (lane + off < 32) {
      B = fma(A, Bp, B);
      A = A * Ap;
    }
  }
  const double X = __shfl_down_sync(FULL, B, 1);
  return lane == 31 ? 0.0 : X;
}

// The segmented solve proper; IB(k), PP(k), QQ(k) give ib, p, q of the
// lane's row jb + k.
template <int MX, class FI, class FP, class FQ>
__device__ __forceinline__ void solve_seg(double* buf, int n, int lane, FI IB, FP PP, FQ QQ) {
  const int jb = lane * MX;
  double y[MX];
  double B = 0.0, A = 1.0;
#pragma unroll
  for (int k = 0; k < MX; k++) {
    const int j = jb + k;
    if (j < n) {
      const double p = PP(k);
      y[k] = IB(k) * buf[j];
      B = fma(p, B, y[k]);
      A *= p;
    }
  }
  double d = carry_up(A, B, lane);
#pragma unroll
  for (int k = 0; k < MX; k++) {
    if (jb + k < n) {
      d = fma(PP(k), d, y[k]);
      y[k] = d;
    }
  }
  B = 0.0;
  A = 1.0;
#pragma unroll
  for (int k = MX - 1; k >= 0; k--) {
    if (jb + k < n) {
      const double q = QQ(k);
      B = fma(q, B, y[k]);
      A *= q;
    }
  }
  double x = carry_down(A, B, lane);
#pragma unroll
  for (int k = MX - 1; k >= 0; k--) {
    const int j = jb + k;
    if (j < n) {
      x = fma(QQ(k), x, y[k]);
      buf[j] = x;
    }
  }
}

// The same with the lane's rows in registers (y: right-hand side in,
// solution out).
template <int MX, class FI, class FP, class FQ>
__device__ __forceinline__ void solve_reg(double (&y)[MX], int n, int lane, FI IB, FP PP, FQ QQ) {
  const int jb = lane * MX;
  double B = 0.0, A = 1.0;
#pragma unroll
  for (int k = 0; k < MX; k++) {
    if (jb + k < n) {
      const double p = PP(k);
      y[k] = IB(k) * y[k];
      B = fma(p, B, y[k]);
      A *= p;
    }
  }
  double d = carry_up(A, B, lane);
#pragma unroll
  for (int k = 0; k < MX; k++) {
    if (jb + k < n) {
      d = fma(PP(k), d, y[k]);
      y[k] = d;
    }
  }
  B = 0.0;
  A = 1.0;
#pragma unroll
  for (int k = MX - 1; k >= 0; k--) {
    if (jb + k < n) {
      const double q = QQ(k);
      B = fma(q, B, y[k]);
      A *= q;
    }
  }
  double x = carry_down(A, B, lane);
#pragma unroll
  for (int k = MX - 1; k >= 0; k--) {
    if (jb + k < n) {
      x = fma(QQ(k), x, y[k]);
      y[k] = x;
    }
  }
}

// Row table of one side of a direction, TABW(MX) doubles: ib[R], p[R] by
// row, then the multipliers of the two lane scans, fm[5][32] and bm[5][32].
// With q = p on every row of such a line, a lane's forward end map is
// c -> A c + B and its backward one X -> A X + B', with the same A (the
// product of its rows' p); step s of the Kogge-Stone scan over the lanes
// multiplies the value shuffled in from 2^s lanes away by the product of A
// over the lane's current window: fm[s][l] = prod A over (l - 2^s, l] (0
// when l < 2^s), bm[s][l] = prod A over [l, l + 2^s) (0 past lane 31).
// Those are constants of the side, so a scan step is two shuffles and one
// fused multiply-add.
template <int MX>
__host__ __device__ constexpr int tabw() {
  return 2 * 32 * MX + 320;
}

// The lane's rows of a line without crossings, in registers (y: right-hand
// side in, solution out; rows past the line end must hold 0).
template <int MX>
__device__ __forceinline__ void solve_lean(double (&y)[MX], const double* tab, int lane) {
  constexpr int R = 32 * MX;
  const int jb = lane * MX;
  const double* const fm = tab + 2 * R;
  const double* const bm = fm + 160;
  double p[MX];
  double B = 0.0;
#pragma unroll
  for (int k = 0; k < MX; k++) {
    p[k] = tab[R + jb + k];
    y[k] *= tab[jb + k];
    B = fma(p[k], B, y[k]);
  }
#pragma unroll
  for (int st = 0; st < 5; st++) {
    const double Bp = __shfl_up_sync(FULL, B, 1 << st);
    B = fma(fm[32 * st + lane], Bp, B);
  }
  double d = __shfl_up_sync(FULL, B, 1);
  if (lane == 0) d = 0.0;
#pragma unroll
  for (int k = 0; k < MX; k++) {
    d = fma(p[k], d, y[k]);
    y[k] = d;
  }
  B = 0.0;
#pragma unroll
  for (int k = MX - 1; k >= 0; k--) B = fma(p[k], B, y[k]);
#pragma unroll
  for (int st = 0; st < 5; st++) {
    const double Bp = __shfl_down_sync(FULL, B, 1 << st);
    B = fma(bm[32 * st + lane], Bp, B);
  }
  double x = __shfl_down_sync(FULL, B, 1);
  if (lane == 31) x = 0.0;
#pragma unroll
  for (int k = MX - 1; k >= 0; k--) {
    x = fma(p[k], x, y[k]);
    y[k] = x;
  }
}

// The same on a line held in shared memory (rows past the end hold 0).
template <int MX>
__device__ __forceinline__ void solve_tab(double* buf, const double* tab, int lane) {
  const int jb = lane * MX;
  double y[MX];
#pragma unroll
  for (int k = 0; k < MX; k++) y[k] = buf[jb + k];
  solve_lean<MX>(y, tab, lane);
#pragma unroll
  for (int k = 0; k < MX; k++) buf[jb + k] = y[k];
}

// A line that crosses the interface: the lane's rows of its own coefficients
// (cf: [ib, p][R] in global memory, zero past the line end), loaded into
// registers at once; q from qbuf (p, with the block rows' own q over it).
template <int MX>
struct LineCoef {
  double ib[MX], p[MX];
  // The line's (ib, p) by row: cf, its own, from its first MIB row L1 on;
  // before that the row table of the side of its row 1, tab (same layout),
  // which holds the same values (the factors up to L1 are the prefix
  // factors of that side) and stays in cache.
  __device__ __forceinline__ void load(const double* __restrict__ cf, const double* __restrict__ tab, int L1,
                                       int lane) {
    constexpr int R = 32 * MX;
    const int jb = lane * MX;
#pragma unroll
    for (int k = 0; k < MX; k++) {
      const double* const src = jb + k < L1 ? tab : cf;
      ib[k] = __ldg(src + jb + k);
      p[k] = __ldg(src + R + jb + k);
    }
  }
  // p as the q of the lane's rows, before the block rows' own go over it
  __device__ __forceinline__ void put_q(double* qbuf, int lane) const {
    const int jb = lane * MX;
#pragma unroll
    for (int k = 0; k < MX; k++) qbuf[jb + k] = p[k];
  }
};
template <int MX>
__device__ __forceinline__ void solve_cross(double* buf, const double* qbuf, const LineCoef<MX>& c, int n, int lane) {
  const int jb = lane * MX;
  solve_seg<MX>(
      buf, n, lane, [&](int k) { return c.ib[k]; }, [&](int k) { return c.p[k]; },
      [&](int k) { return qbuf[jb + k]; });
}

// Row tables [side][TABW] into shared memory.
__device__ __forceinline__ void load_tab(double* s, const double* g, int w2) {
  for (int i = threadIdx.x; i < w2; i += blockDim.x) s[i] = g[i];
}

// ---------------------------------------------------------------------------
// kf_mib: the MIB rows' right-hand sides of the x solve, into d.

__global__ void __launch_bounds__(TPB) kf_mib(const __grid_constant__ Dev P, const double* __restrict__ un,
                                              double* __restrict__ d, double E) {
  // every MIB row at once, one thread each (the rows of an x block too:
  // kf_xc applies their block's row operations when it solves the line)
  const long long k = (long long)blockIdx.x * TPB + threadIdx.x;
  if (k >= P.nmibnode) return;
  E = step_e(P, E, 2);
  const long long m = P.mibnode[k];
  int ix, iy, iz;
  node_xyz(P, m, ix, iy, iz);
  d[m] = rho_mib(P, un, E, m, ix, iy, iz, P.tag[m], P.mibref[k]);
}

// ---------------------------------------------------------------------------
// The x pass.

// Constants of rho along one x line.
struct XLine {
  double cx0, cy0, cz0, cx1, cy1, cz1;  // dt beta / h^2 of each direction, by side
  double kin, koa, kob, yzE;           // source and boundary parts fixed along the line
};
__device__ __forceinline__ XLine x_line(const Dev& P, int iy, int iz, double E) {
  XLine c;
  c.cx0 = P.dt * P.vd[0][0][0];
  c.cy0 = P.dt * P.vd[1][0][0];
  c.cz0 = P.dt * P.vd[2][0][0];
  c.cx1 = P.dt * P.vd[0][1][0];
  c.cy1 = P.dt * P.vd[1][1][0];
  c.cz1 = P.dt * P.vd[2][1][0];
  const double yv = P.ax[1][iy], zv = P.ax[2][iz];
  const double yz2 = yv * yv + zv * zv;
  const bool eq8 = P.eq != 0;
  // inside dt kin sin2x cos2y sin2z E; outside -dt E (x^2 + y^2 + z^2) -
  // dt 6 beta_out E; on the faces (x^2 + y^2 + z^2) E
  c.kin = eq8 ? P.dt * (P.kin * ((P.c2[1][iy] * P.s2[2][iz]) * E)) : 0.0;
  c.koa = eq8 ? -P.dt * E : 0.0;
  c.kob = eq8 ? -P.dt * E * yz2 - P.dt * (P.c6bo * E) : 0.0;
  c.yzE = yz2 * E;
  return c;
}

// rho of interior x line (iy, iz) into buf[j] (j = lane + 32 k, coalesced
// loads); MIB rows take kf_mib's value from d.
template <int MX>
__device__ __forceinline__ void x_rho(const Dev& P, const double* __restrict__ un, const double* __restrict__ d,
                                      double E, int iy, int iz, double* buf, int lane) {
  const int nx = P.nx;
  const long long sy = nx, sz = (long long)nx * P.ny;
  const long long m0 = (long long)nx * (iy + (long long)P.ny * iz);
  const XLine c = x_line(P, iy, iz, E);
  const bool eq8 = P.eq != 0;
  const double* const ur = un + m0;
  const unsigned char* const tr = P.tag + m0;
#pragma unroll 3
  for (int k = 0; k < MX; k++) {
    const int j = lane + 32 * k;
    if (j < nx) {
      // (an interior line: every neighbour index lies inside the field)
      const int t = tr[j];
      const double uc = ur[j], uxm = ur[j - 1], uxp = ur[j + 1];
      const double uym = ur[j - sy], uyp = ur[j + sy], uzm = ur[j - sz], uzp = ur[j + sz];
      const double x = P.ax[0][j], s2x = P.s2[0][j];
      double r;
      if (j == 0 || j == nx - 1) {
        r = (eq8 ? fma(x * x, E, c.yzE) : 100.0) - uc;
      } else if (t & (TAG_MIBX | TAG_MIBY | TAG_MIBZ)) {
        r = d[m0 + j];  // from kf_mib
      } else {
        const double lx = fma(-2.0, uc, uxm + uxp);
        const double ly = fma(-2.0, uc, uym + uyp);
        const double lz = fma(-2.0, uc, uzm + uzp);
        if (t & TAG_OUT)
          r = fma(c.cx1, lx, fma(c.cy1, ly, fma(c.cz1, lz, fma(c.koa, x * x, c.kob))));
        else
          r = fma(c.cx0, lx, fma(c.cy0, ly, fma(c.cz0, lz, c.kin * s2x)));
      }
      buf[j] = r;
    }
  }
}

// Shared memory of kf_xw: a ring of XS slabs of u^n (the TY+2 rows around
// the CTA's lines at one plane, from a 16-byte aligned start) and XS slabs
// of their tags (TY rows), {sin 2x, x^2} per column, the row tables.  Three
// slabs are in use at a plane (z-1, z, z+1) and one more is on its way.
constexpr int XS = 4;
struct XLayout {
  int slabd;  // doubles per u^n slab (even)
  int tagb;   // bytes per tag slab (multiple of 16)
  size_t o_tag, o_xt, o_tab, o_bar, total;
};
__host__ __device__ inline XLayout x_layout(int nx, int TY, int MX) {
  XLayout L;
  L.slabd = ((TY + 2) * nx + 2 + 1) & ~1;
  L.tagb = (TY * nx + 32 + 15) & ~15;
  L.o_tag = (size_t)XS * L.slabd * sizeof(double);
  L.o_xt = L.o_tag + (size_t)XS * L.tagb;
  L.o_tab = L.o_xt + (size_t)(nx + 1) * 2 * sizeof(double);
  L.o_bar = L.o_tab + (size_t)2 * (2 * 32 * MX + 320) * sizeof(double);
  L.total = L.o_bar + XS * sizeof(uint64_t);
  return L;
}

// The x lines that do not cross the interface, and the face lines.  A CTA
// owns TY neighbouring lines (rows iy0..iy0+TY-1) and walks a range of z
// planes.  Plane by plane it brings the TY+2 rows of u^n around its lines
// (one contiguous run of memory) and their tags into shared memory with one
// bulk copy each (cp.async.bulk, completion on an mbarrier), XS planes in a
// ring, so that the z-1, z and z+1 rows of the stencil all come from shared
// memory and the copy of plane z+2 is in flight while plane z is computed.
// Lane l of warp w forms rho of its rows l MX .. l MX + MX - 1 of line
// iy0 + w in registers; the MIB rows' values (from kf_mib) and the next
// line's flags are read one plane ahead.  The solved line goes out through
// the line's z-1 row in shared memory (no other warp reads it) as coalesced
// stores.
template <int TY, int MX>
__global__ void __launch_bounds__(32 * TY, 2) kf_xw(const __grid_constant__ Dev P, const double* __restrict__ un,
                                                    double* __restrict__ dst, double E, int nyt, int zchunk,
                                                    int ntiles) {
  constexpr int R = 32 * MX;
  E = step_e(P, E, 2);
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const bool eq8 = P.eq != 0;

  if ((int)blockIdx.x >= ntiles) {
    // face x lines (iy or iz on a face): d = Outer_u(t_next) - u^n
    const int nface = 2 * ny + 2 * (nz - 2);
    const int fw = (blockIdx.x - ntiles) * TY + w, fstride = (gridDim.x - ntiles) * TY;
    for (int f = fw; f < nface; f += fstride) {
      int iy, iz;
      if (f < 2 * ny) {
        iy = f % ny;
        iz = f < ny ? 0 : nz - 1;
      } else {
        iz = 1 + (f - 2 * ny) % (nz - 2);
        iy = (f - 2 * ny) < nz - 2 ? 0 : ny - 1;
      }
      const long long m0 = (long long)nx * (iy + (long long)ny * iz);
      const double y = P.ax[1][iy], z = P.ax[2][iz];
      const double yz2 = y * y + z * z;
      for (int ix = lane; ix < nx; ix += 32) {
        const double x = P.ax[0][ix];
        dst[m0 + ix] = (eq8 ? (x * x + yz2) * E : 100.0) - un[m0 + ix];
      }
    }
    return;
  }

  extern __shared__ __align__(16) unsigned char smx[];
  const XLayout LY = x_layout(nx, TY, MX);
  double* const slab = reinterpret_cast<double*>(smx);
  unsigned char* const tslab = smx + LY.o_tag;
  double2* const xt = reinterpret_cast<double2*>(smx + LY.o_xt);  // {sin 2x, x^2} per column
  double* const stab = reinterpret_cast<double*>(smx + LY.o_tab);
  uint64_t* const bar = reinterpret_cast<uint64_t*>(smx + LY.o_bar);

  const int ty = blockIdx.x % nyt, zc = blockIdx.x / nyt;
  const int y0 = 1 + ty * TY;
  const int z0 = 1 + zc * zchunk;
  const int z1 = min(z0 + zchunk, nz - 1);
  const int nplanes = z1 - z0;  // >= 1
  const int nslabs = nplanes + 2;

  // slab i holds plane z0 - 1 + i: where each copy starts, and the offset
  // (in elements) of the data within the aligned copy
  auto slab_src = [&](int i, int& shift) -> const double* {
    const double* g = un + (long long)nx * ((y0 - 1) + (long long)ny * (z0 - 1 + i));
    const uintptr_t a = reinterpret_cast<uintptr_t>(g);
    shift = (int)((a & 15) >> 3);
    return reinterpret_cast<const double*>(a & ~(uintptr_t)15);
  };
  auto tag_src = [&](int i, int& shift) -> const unsigned char* {
    const unsigned char* g = P.tag + (long long)nx * (y0 + (long long)ny * (z0 - 1 + i));
    const uintptr_t a = reinterpret_cast<uintptr_t>(g);
    shift = (int)(a & 15);
    return reinterpret_cast<const unsigned char*>(a & ~(uintptr_t)15);
  };
  const unsigned ubytes = (unsigned)((((size_t)(TY + 2) * nx + 1) * sizeof(double) + 15) & ~(size_t)15);
  const unsigned tbytes = (unsigned)((TY * nx + 15 + 15) & ~15);
  auto issue = [&](int i) {
    const int s = i % XS;
    int sh;
    const double* gu = slab_src(i, sh);
    const unsigned char* gt = tag_src(i, sh);
    mbar_expect(&bar[s], ubytes + tbytes);
    bulk_copy(slab + (size_t)s * LY.slabd, gu, ubytes, &bar[s]);
    bulk_copy(tslab + (size_t)s * LY.tagb, gt, tbytes, &bar[s]);
  };
  auto tags_of = [&](int i) -> const unsigned char* {  // this warp's tag row of slab i
    int sh;
    tag_src(i, sh);
    return tslab + (size_t)(i % XS) * LY.tagb + sh + (size_t)w * nx;
  };

  if (threadIdx.x == 0) {
    for (int s = 0; s < XS; s++) mbar_init(&bar[s]);
    mbar_init_fence();
  }
  __syncthreads();
  if (threadIdx.x == 0)
    for (int i = 0; i < XS - 1 && i < nslabs; i++) issue(i);
  for (int i = threadIdx.x; i < nx; i += blockDim.x) {
    const double x = P.ax[0][i];
    xt[i] = make_double2(P.s2[0][i], x * x);
  }
  load_tab(stab, P.ftab[0], 2 * tabw<MX>());
  __syncthreads();

  const double cx0 = P.dt * P.vd[0][0][0], cy0 = P.dt * P.vd[1][0][0], cz0 = P.dt * P.vd[2][0][0];
  const double cx1 = P.dt * P.vd[0][1][0], cy1 = P.dt * P.vd[1][1][0], cz1 = P.dt * P.vd[2][1][0];
  const int iy = y0 + w;
  const bool live = iy <= ny - 2;
  const double yv = P.ax[1][live ? iy : 1];
  const int jb = lane * MX;
  const uint8_t* const fl = P.fline[0];
  // flags of this warp's line at the plane in hand (a line not live, or one
  // that crosses the interface, is skipped: bit0)
  int fcur = live ? fl[(long long)iy * nz + z0] : 1;
  double mcur[MX];  // the MIB rows' values at the plane in hand
  bool mib_ready = false;
  bool bad = false;

  for (int pi = 0; pi < nplanes; pi++) {
    // (slab pi + XS - 1 goes into the slot of slab pi - 1, done with at the
    // last plane)
    if (threadIdx.x == 0 && pi + XS - 1 < nslabs) issue(pi + XS - 1);
    const int iz = z0 + pi;
    // slabs pi (z-1), pi+1 (z), pi+2 (z+1) must have landed
    bool ok = true;
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const int i = pi + k;
      ok = ok && mbar_wait(&bar[i % XS], (unsigned)((i / XS) & 1));
    }
    if (!ok) bad = true;
    const long long m0 = (long long)nx * (iy + (long long)ny * iz);
    if (ok && !mib_ready && !(fcur & 1)) {
      // the first plane: its MIB values now (later planes: a plane ahead)
      const unsigned char* const tg = tags_of(pi + 1);
#pragma unroll
      for (int k = 0; k < MX; k++) {
        const int j = jb + k;
        mcur[k] = (j > 0 && j < nx - 1 && (tg[j] & (TAG_MIBX | TAG_MIBY | TAG_MIBZ))) ? dst[m0 + j] : 0.0;
      }
    }
    // the next plane's flags and MIB values, read ahead
    int fnxt = 1;
    double mnxt[MX];
    if (ok && live && pi + 1 < nplanes) {
      fnxt = fl[(long long)iy * nz + iz + 1];
      if (!(fnxt & 1)) {
        const unsigned char* const tg = tags_of(pi + 2);
        const long long m1 = m0 + (long long)nx * ny;
#pragma unroll
        for (int k = 0; k < MX; k++) {
          const int j = jb + k;
          mnxt[k] = (j > 0 && j < nx - 1 && (tg[j] & (TAG_MIBX | TAG_MIBY | TAG_MIBZ))) ? dst[m1 + j] : 0.0;
        }
      }
    }
    if (ok && !(fcur & 1)) {
      int shm, shc, shp;
      slab_src(pi, shm);
      slab_src(pi + 1, shc);
      slab_src(pi + 2, shp);
      const double* const sc = slab + (size_t)((pi + 1) % XS) * LY.slabd + shc + (size_t)(w + 1) * nx;
      const double* const sym = sc - nx;
      const double* const syp = sc + nx;
      double* const szm = slab + (size_t)(pi % XS) * LY.slabd + shm + (size_t)(w + 1) * nx;
      const double* const szp = slab + (size_t)((pi + 2) % XS) * LY.slabd + shp + (size_t)(w + 1) * nx;
      const unsigned char* const tg = tags_of(pi + 1);
      const double zv = P.ax[2][iz];
      const double yz2 = yv * yv + zv * zv;
      // source constants of the line: inside dt kin sin2x cos2y sin2z E,
      // outside -dt E (x^2 + y^2 + z^2) - dt 6 beta_out E
      const double kin = eq8 ? P.dt * (P.kin * ((P.c2[1][iy] * P.s2[2][iz]) * E)) : 0.0;
      const double koa = eq8 ? -P.dt * E : 0.0;
      const double kob = eq8 ? -P.dt * E * yz2 - P.dt * (P.c6bo * E) : 0.0;
      // the lane's rows and the two beside them: x +- 1 from registers
      double uc[MX + 2];
#pragma unroll
      for (int k = 0; k < MX + 2; k++) {
        const int j = jb + k - 1;
        uc[k] = (j >= 0 && j < nx) ? sc[j] : 0.0;
      }
      double y[MX];
#pragma unroll
      for (int k = 0; k < MX; k++) {
        const int j = jb + k;
        double r = 0.0;
        if (j < nx) {
          const double2 q = xt[j];
          if (j == 0 || j == nx - 1) {
            r = (eq8 ? fma(q.y, E, yz2 * E) : 100.0) - uc[k + 1];
          } else {
            const int t = tg[j];
            if (t & (TAG_MIBX | TAG_MIBY | TAG_MIBZ)) {
              r = mcur[k];
            } else {
              const double c0 = uc[k + 1];
              const double lx = fma(-2.0, c0, uc[k] + uc[k + 2]);
              const double ly = fma(-2.0, c0, sym[j] + syp[j]);
              const double lz = fma(-2.0, c0, szm[j] + szp[j]);
              if (t & TAG_OUT)
                r = fma(cx1, lx, fma(cy1, ly, fma(cz1, lz, fma(koa, q.y, kob))));
              else
                r = fma(cx0, lx, fma(cy0, ly, fma(cz0, lz, kin * q.x)));
            }
          }
        }
        y[k] = r;
      }
      solve_lean<MX>(y, stab + ((fcur >> 1) & 1) * tabw<MX>(), lane);
      // out through the line's z-1 row (this warp alone reads it, and every
      // lane is done with it once the solve's shuffles are past)
#pragma unroll
      for (int k = 0; k < MX; k++)
        if (jb + k < nx) szm[jb + k] = y[k];
      __syncwarp();
      for (int j = lane; j < nx; j += 32) dst[m0 + j] = szm[j];
    }
    fcur = fnxt;
#pragma unroll
    for (int k = 0; k < MX; k++) mcur[k] = mnxt[k];
    mib_ready = true;
    // every thread's shared-memory accesses to the slot reloaded next are done
    fence_async_smem();
    if (__syncthreads_or(bad)) {
      if (threadIdx.x == 0) {
        atomicOr(P.status, 2);
        // let the copies still in flight land before the CTA leaves
        for (int i = pi + 3; i < nslabs && i < pi + XS; i++) mbar_wait(&bar[i % XS], (unsigned)((i / XS) & 1));
      }
      return;
    }
  }
}

template <int MX>
__host__ __device__ constexpr size_t cross_smem() {
  // per warp a line buffer and its q
  return sizeof(double) * (size_t)CW * 2 * 32 * MX;
}

// The x lines that cross the interface, one warp per line.
template <int MX>
__global__ void __launch_bounds__(32 * CW, 3) kf_xc(const __grid_constant__ Dev P, const double* __restrict__ un,
                                                    double* __restrict__ dst, double E) {
  constexpr int R = 32 * MX;
  extern __shared__ __align__(16) double smc[];
  E = step_e(P, E, 2);
  const int nx = P.nx, nz = P.nz;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double* const buf = smc + 2 * w * R;
  double* const qbuf = buf + R;
  const int nc = P.nfcross[0];
  for (int c = blockIdx.x * CW + w; c < nc; c += gridDim.x * CW) {
    const long long lid = P.fcross[0][c];
    const int iy = (int)(lid / nz), iz = (int)(lid % nz);
    const int bfirst = P.bstart[0][lid], bend = P.bstart[0][lid + 1];
    LineCoef<MX> cf;
    cf.load(P.fcoef[0] + (size_t)c * 2 * R, P.ftab[0] + (size_t)((P.lside[0][lid] >> 1) & 1) * tabw<MX>(),
            P.blk[0][bfirst].L, lane);
    x_rho<MX>(P, un, dst, E, iy, iz, buf, lane);
    cf.put_q(qbuf, lane);
    __syncwarp();
    block_rows<0>(P, buf, qbuf, bfirst, bend, lane, true);  // the x blocks' Convert2Tri row operations
    __syncwarp();
    solve_cross<MX>(buf, qbuf, cf, nx, lane);
    __syncwarp();
    const long long m0 = (long long)nx * (iy + (long long)P.ny * iz);
    for (int j = lane; j < nx; j += 32) dst[m0 + j] = buf[j];
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// The y and z passes.

template <int MX, bool ACC>
__host__ __device__ constexpr size_t yt_smem() {
  // row tables 2 TABW; two buffers of NL lines x (R + 2) doubles; ACC: one
  // buffer of u^n
  return sizeof(double) * ((size_t)2 * tabw<MX>() + (size_t)(ACC ? 3 : 2) * YZ_NL * (32 * MX + 2));
}

// The regular lines of direction D in tiles: y in place on d*; z (ACC) with
// the update of u, face lines included (their d** passes through).
template <int D, int MX, bool ACC>
__global__ void __launch_bounds__(32 * YZ_NL, ACC ? 1 : 2) kf_yt(const __grid_constant__ Dev P,
                                                                  double* __restrict__ f, double* __restrict__ u,
                                                                  int ntiles) {
  static_assert(D == 1 || D == 2, "y and z lines");
  constexpr int R = 32 * MX;
  // line stride 2 mod 16 doubles: a lane's stride-MX rows (MX odd) fall on
  // distinct bank pairs
  constexpr int LS = R + 2;
  extern __shared__ __align__(16) double smyz[];
  double* const stab = smyz;
  double* const bufs = smyz + 2 * tabw<MX>();
  double* const ubuf = bufs + 2 * YZ_NL * LS;  // (ACC)
  const int nx = P.nx;
  const int n = D == 1 ? P.ny : P.nz;
  const int n2 = D == 1 ? P.nz : P.ny;  // the second line index: iz (y lines) or iy (z lines)
  const long long s = D == 1 ? (long long)nx : (long long)nx * P.ny;   // row stride
  const long long s2 = D == 1 ? (long long)nx * P.ny : (long long)nx;  // stride of the second line index
  // y tiles cover the interior lines (face y lines keep d*); z tiles cover
  // every line (face z lines pass d** through to the update)
  const int i1lo = ACC ? 0 : 1, i1n = ACC ? nx : nx - 2;
  const int i2lo = ACC ? 0 : 1;
  const int tpr = (i1n + YZ_NL - 1) / YZ_NL;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int c = threadIdx.x % YZ_NL, jc = threadIdx.x / YZ_NL;  // this thread's copy share: line c, rows jc + 32 m
  const uint8_t* const fline = P.fline[D];

  load_tab(stab, P.ftab[D], 2 * tabw<MX>());
  // the rows past the line end stay 0 (the copies never write them)
  for (int i = threadIdx.x; i < 2 * YZ_NL * LS; i += blockDim.x) bufs[i] = 0.0;
  __syncthreads();

  struct Tile {
    int i1, i2;
    bool ok;
  };
  auto tile_of = [&](int t) -> Tile {
    Tile T;
    T.i2 = i2lo + t / tpr;
    T.i1 = i1lo + (t % tpr) * YZ_NL;
    T.ok = t < ntiles;
    return T;
  };
  // flags of line i of tile T (-1: no line there); bit0 crosses the
  // interface (left to kf_yc), bit1 side of row 1
  auto flags = [&](const Tile& T, int i) -> int {
    const int i1 = T.i1 + i;
    if (!T.ok || i1 >= i1lo + i1n) return -1;
    return fline[(long long)i1 * n2 + T.i2];
  };
  auto copy_rows = [&](const Tile& T, int fc, const double* src, double* buf) {
    if (fc >= 0 && !(fc & 1)) {
      const long long g0 = T.i1 + c + s2 * T.i2 + (long long)jc * s;
      double* const cb = buf + c * LS;
#pragma unroll
      for (int m = 0; m < MX; m++) {
        const int j = jc + 32 * m;
        if (j < n) cp_async8(cb + j, src + g0 + (long long)32 * m * s);
      }
    }
    cp_async_commit();
  };

  int t = blockIdx.x;
  Tile cur = tile_of(t);
  Tile nxt = tile_of(t + gridDim.x);
  // flags are read two tiles ahead: this thread's copy line (fc*) and this
  // warp's solve line (fw*)
  int fc0 = flags(cur, c), fc1 = flags(nxt, c);
  int fw0 = flags(cur, w), fw1 = flags(nxt, w);
  copy_rows(cur, fc0, f, bufs);
  for (int it = 0; cur.ok; it++) {
    const Tile nx2 = tile_of(t + 2 * gridDim.x);
    const int fc2 = flags(nx2, c), fw2 = flags(nx2, w);
    double* const buf = bufs + (size_t)(it & 1) * YZ_NL * LS;
    if (ACC) copy_rows(cur, fc0, u, ubuf);
    copy_rows(nxt, fc1, f, bufs + (size_t)((it + 1) & 1) * YZ_NL * LS);
    if (ACC)
      cp_async_wait<2>();
    else
      cp_async_wait<1>();
    __syncthreads();
    {
      const int i1 = cur.i1 + w;
      const bool interior = i1 >= 1 && i1 <= nx - 2 && cur.i2 >= 1 && cur.i2 <= n2 - 2;
      if (fw0 >= 0 && !(fw0 & 1) && interior) solve_tab<MX>(buf + w * LS, stab + ((fw0 >> 1) & 1) * tabw<MX>(), lane);
    }
    if (ACC) cp_async_wait<1>();
    __syncthreads();
    if (fc0 >= 0 && !(fc0 & 1)) {
      const long long g0 = cur.i1 + c + s2 * cur.i2 + (long long)jc * s;
      const double* const cb = buf + c * LS;
#pragma unroll
      for (int m = 0; m < MX; m++) {
        const int j = jc + 32 * m;
        if (j < n) {
          if (ACC)
            u[g0 + (long long)32 * m * s] = ubuf[c * LS + j] + cb[j];
          else
            f[g0 + (long long)32 * m * s] = cb[j];
        }
      }
    }
    t += gridDim.x;
    cur = nxt;
    nxt = nx2;
    fc0 = fc1;
    fc1 = fc2;
    fw0 = fw1;
    fw1 = fw2;
  }
  cp_async_wait<0>();
}

// The lines of direction D that cross the interface, in tiles of CW entries
// of their list (which is in memory order, so a tile's lines are mostly
// neighbours): the rows are copied in with cp.async, the next tile's while
// this one is solved, and warp w solves entry w with its own coefficients
// (loaded while the copy lands) and its blocks' Convert2Tri row operations.
// y in place on d*, z (ACC) with the update of u.
template <int MX, bool ACC>
__host__ __device__ constexpr size_t yc_smem() {
  // two buffers of CW lines x (R + 2), the lines' q (CW x R), ACC: u^n
  return sizeof(double) * ((size_t)(ACC ? 3 : 2) * CW * (32 * MX + 2) + (size_t)CW * 32 * MX);
}

template <int D, int MX, bool ACC>
__global__ void __launch_bounds__(32 * CW, 3) kf_yc(const __grid_constant__ Dev P, double* __restrict__ f,
                                                    double* __restrict__ u) {
  static_assert(D == 1 || D == 2, "y and z lines");
  constexpr int R = 32 * MX;
  constexpr int LS = R + 2;
  extern __shared__ __align__(16) double smc[];
  double* const bufs = smc;                      // [2][CW][LS]
  double* const qbufs = smc + 2 * CW * LS;       // [CW][R]
  double* const ubuf = qbufs + CW * R;           // [CW][LS] (ACC)
  const int nx = P.nx;
  const int n = D == 1 ? P.ny : P.nz;
  const int n2 = D == 1 ? P.nz : P.ny;
  const long long s = D == 1 ? (long long)nx : (long long)nx * P.ny;
  const long long s2 = D == 1 ? (long long)nx * P.ny : (long long)nx;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int c = threadIdx.x % CW, jc = threadIdx.x / CW;  // copy share: entry c, rows jc + 32 m
  const int nc = P.nfcross[D];
  const int ntile = (nc + CW - 1) / CW;
  const int32_t* const list = P.fcross[D];
  // the rows past the line end stay 0 (the copies never write them)
  for (int i = threadIdx.x; i < 2 * CW * LS; i += blockDim.x) bufs[i] = 0.0;
  __syncthreads();
  auto base_of = [&](long long lid) { return lid / n2 + s2 * (lid % n2); };
  // entry i of tile t: its line (-1: none)
  auto lid_of = [&](int t, int i) -> long long {
    const int e = t * CW + i;
    return (t < ntile && e < nc) ? (long long)list[e] : -1;
  };
  auto copy_rows = [&](long long lid, const double* src, double* cb) {
    if (lid >= 0) {
      const long long g0 = base_of(lid) + (long long)jc * s;
#pragma unroll
      for (int m = 0; m < MX; m++) {
        const int j = jc + 32 * m;
        if (j < n) cp_async8(cb + j, src + g0 + (long long)32 * m * s);
      }
    }
    cp_async_commit();
  };

  int t = blockIdx.x;
  long long lc0 = lid_of(t, c), lc1 = lid_of(t + gridDim.x, c);  // this thread's copy entry, two tiles
  long long lw0 = lid_of(t, w), lw1 = lid_of(t + gridDim.x, w);  // this warp's solve entry
  copy_rows(lc0, f, bufs + c * LS);
  for (int it = 0; t < ntile; it++) {
    const long long lc2 = lid_of(t + 2 * gridDim.x, c), lw2 = lid_of(t + 2 * gridDim.x, w);
    double* const buf = bufs + (size_t)(it & 1) * CW * LS;
    if (ACC) copy_rows(lc0, u, ubuf + c * LS);
    copy_rows(lc1, f, bufs + (size_t)((it + 1) & 1) * CW * LS + c * LS);
    // this warp's line: its coefficients and blocks, read while the rows land
    LineCoef<MX> cf;
    int bfirst = 0, bend = 0;
    if (lw0 >= 0) {
      bfirst = P.bstart[D][lw0];
      bend = P.bstart[D][lw0 + 1];
      cf.load(P.fcoef[D] + (size_t)(t * CW + w) * 2 * R,
              P.ftab[D] + (size_t)((P.lside[D][lw0] >> 1) & 1) * tabw<MX>(), P.blk[D][bfirst].L, lane);
    }
    if (ACC)
      cp_async_wait<2>();
    else
      cp_async_wait<1>();
    __syncthreads();
    if (lw0 >= 0) {
      double* const lb = buf + w * LS;
      double* const qb = qbufs + w * R;
      cf.put_q(qb, lane);
      __syncwarp();
      block_rows<D>(P, lb, qb, bfirst, bend, lane, true);
      __syncwarp();
      solve_cross<MX>(lb, qb, cf, n, lane);
    }
    if (ACC) cp_async_wait<1>();
    __syncthreads();
    if (lc0 >= 0) {
      const long long g0 = base_of(lc0) + (long long)jc * s;
      const double* const cb = buf + c * LS;
#pragma unroll
      for (int m = 0; m < MX; m++) {
        const int j = jc + 32 * m;
        if (j < n) {
          if (ACC)
            u[g0 + (long long)32 * m * s] = ubuf[c * LS + j] + cb[j];
          else
            f[g0 + (long long)32 * m * s] = cb[j];
        }
      }
    }
    t += gridDim.x;
    lc0 = lc1;
    lc1 = lc2;
    lw0 = lw1;
    lw1 = lw2;
  }
  cp_async_wait<0>();
}

// ---------------------------------------------------------------------------
// Set-up of the form (once per handle).

// Row tables of direction D: [side][TABW]: ib and p by row from the prefix
// factors of that side (ptab: bet_j, gam_j), zero past the line end.
template <int D>
__global__ void __launch_bounds__(TPB) kf_tab(const __grid_constant__ Dev P, double* tab, int R) {
  const int n = D == 0 ? P.nx : D == 1 ? P.ny : P.nz;
  const int i = blockIdx.x * TPB + threadIdx.x;
  if (i >= 2 * R) return;
  const int side = i / R, j = i % R;
  double ib = 0.0, p = 0.0;
  if (j < n) {
    const double bet = P.ptab[D][side][2 * j];
    const double a = (j == 0 || j == n - 1) ? 0.0 : P.ia[D][side];
    ib = 1.0 / bet;
    p = -(a / bet);
  }
  double* T = tab + (size_t)side * (2 * R + 320);
  T[j] = ib;
  T[R + j] = p;
}

// The scan multipliers of the row tables (after kf_tab), one thread per side.
__global__ void kf_tabscan(double* tab, int R, int n) {
  const int side = threadIdx.x;
  if (side >= 2) return;
  double* T = tab + (size_t)side * (2 * R + 320);
  const int MX = R / 32;
  double A[32];
  for (int l = 0; l < 32; l++) {
    double a = 1.0;
    for (int k = 0; k < MX; k++)
      if (l * MX + k < n) a *= T[R + l * MX + k];
    A[l] = a;
  }
  for (int st = 0; st < 5; st++) {
    const int o = 1 << st;
    for (int l = 0; l < 32; l++) {
      double f = 0.0, b = 0.0;
      if (l >= o) {
        f = 1.0;
        for (int m = l - o + 1; m <= l; m++) f *= A[m];
      }
      if (l + o <= 31) {
        b = 1.0;
        for (int m = l; m < l + o; m++) b *= A[m];
      }
      T[2 * R + 32 * st + l] = f;
      T[2 * R + 160 + 32 * st + l] = b;
    }
  }
}

// Per line of direction D: bit0 the line crosses the interface (has MIB
// blocks), bit1 the side of its row 1.  Face lines: 0.
template <int D>
__global__ void __launch_bounds__(TPB) kf_fline(const __grid_constant__ Dev P, uint8_t* fl) {
  const long long t = (long long)blockIdx.x * TPB + threadIdx.x;
  if (t >= nlines<D>(P)) return;
  Line L;
  decode_line<D>(P, t, L);
  uint8_t v = 0;
  if (!L.boundary) {
    v = (uint8_t)(((P.lside[D][L.lid] >> 1) & 1) << 1);
    if (P.bstart[D][L.lid + 1] > P.bstart[D][L.lid]) v |= 1;
  }
  fl[L.lid] = v;
}

// Line geometry from a line id (i1 * n2 + i2) of direction D.
template <int D>
__device__ __forceinline__ void line_at(const Dev& P, long long lid, long long& base, long long& s) {
  const int n2 = D == 2 ? P.ny : P.nz;
  const int i1 = (int)(lid / n2), i2 = (int)(lid % n2);
  if (D == 0) {
    base = (long long)P.nx * (i1 + (long long)P.ny * i2);
    s = 1;
  } else if (D == 1) {
    base = i1 + (long long)P.nx * P.ny * i2;
    s = P.nx;
  } else {
    base = i1 + (long long)P.nx * i2;
    s = (long long)P.nx * P.ny;
  }
}

// Coefficients (ib, p) of the crossing lines, one thread per listed line,
// walking the line as the sequential sweep does (the factors from the
// prefix table before the first MIB row and per node from it on; the regular
// rows' side from the line's start and after each block), into cf[c][2][R].
template <int D>
__global__ void __launch_bounds__(TPB) kf_coef(const __grid_constant__ Dev P, double* cf, int R) {
  const int c = blockIdx.x * TPB + threadIdx.x;
  if (c >= P.nfcross[D]) return;
  const long long lid = P.fcross[D][c];
  const int n = D == 0 ? P.nx : D == 1 ? P.ny : P.nz;
  long long base, s;
  line_at<D>(P, lid, base, s);
  const int bfirst = P.bstart[D][lid], bend = P.bstart[D][lid + 1];
  const MibBlock* const blk = P.blk[D];
  const int L1 = blk[bfirst].L;
  const int side1 = (P.lside[D][lid] >> 1) & 1;
  const double* const pt = P.ptab[D][side1];
  double* const o = cf + (size_t)c * 2 * R;
  int b = bfirst, side = side1;
  for (int j = 0; j < n; j++) {
    const double bet = j >= L1 ? P.fbet[D][base + (long long)j * s] : pt[2 * j];
    double a;
    if (j == 0 || j == n - 1) {
      a = 0.0;
    } else if (b < bend && j >= blk[b].L) {
      const int q = j - blk[b].L;
      a = blk[b].ia[q];
      if (q == blk[b].kind - 1) {
        side = (blk[b].sides >> q) & 1;
        b++;
      }
    } else {
      a = P.ia[D][side];
    }
    o[j] = 1.0 / bet;
    o[R + j] = -(a / bet);
  }
}

// q = -gam_{j+1} of the rows of each block of direction D (their c is not
// their a), from the per-node factors: bq[3 k + r].
template <int D>
__global__ void __launch_bounds__(TPB) kf_bq(const __grid_constant__ Dev P, double* bq) {
  const int k = blockIdx.x * TPB + threadIdx.x;
  if (k >= P.nblk[D]) return;
  const MibBlock& b = P.blk[D][k];
  long long base, s;
  line_at<D>(P, b.line, base, s);
  for (int r = 0; r < 3; r++)
    bq[3 * (long long)k + r] = r < b.kind ? -P.fgam[D][base + (long long)(b.L + r + 1) * s] : 0.0;
}

// Per MIB node: its block in each direction (-1: none).
__global__ void __launch_bounds__(TPB) kf_mibref(const __grid_constant__ Dev P, int4* ref) {
  const int k = blockIdx.x * TPB + threadIdx.x;
  if (k >= P.nmibnode) return;
  const long long m = P.mibnode[k];
  const int tg = P.tag[m];
  int ix, iy, iz;
  node_xyz(P, m, ix, iy, iz);
  int4 r = make_int4(-1, -1, -1, 0);
  int row = 0;
  if (tg & TAG_MIBX) {
    const MibBlock* b = find_block<0>(P, iy * P.nz + iz, ix, row);
    if (b) r.x = (int)(b - P.blk[0]);
  }
  if (tg & TAG_MIBY) {
    const MibBlock* b = find_block<1>(P, ix * P.nz + iz, iy, row);
    if (b) r.y = (int)(b - P.blk[1]);
  }
  if (tg & TAG_MIBZ) {
    const MibBlock* b = find_block<2>(P, ix * P.ny + iy, iz, row);
    if (b) r.z = (int)(b - P.blk[2]);
  }
  ref[k] = r;
}

// ---------------------------------------------------------------------------
// Launches

int fast_mx(int n) {
  const int c[6] = {1, 3, 5, 9, 13, 17};
  for (int k = 0; k < 6; k++)
    if (32 * c[k] >= n) return c[k];
  return 0;
}

template <class K>
int resident_grid(const Dev& P, K kernel, int threads, size_t smem, long long want) {
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
  if (per_sm < 1) per_sm = 1;
  return (int)std::max(1LL, std::min(want, (long long)per_sm * P.sweep_blocks));
}

template <int TY, int MX>
void launch_xw_ty(const Dev& P, const double* un, double* d, double E, cudaStream_t st) {
  const size_t smem = x_layout(P.nx, TY, MX).total;
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kf_xw<TY, MX>, 32 * TY, smem);
  if (per_sm < 1) per_sm = 1;
  const int nyt = (P.ny - 2 + TY - 1) / TY;
  const int target = std::max(1, per_sm * P.sweep_blocks - X_NFACE);
  int nzc = std::max(1, std::min(P.nz - 2, target / nyt));
  const int zchunk = (P.nz - 2 + nzc - 1) / nzc;
  nzc = (P.nz - 2 + zchunk - 1) / zchunk;
  const int ntiles = nyt * nzc;
  kf_xw<TY, MX><<<ntiles + X_NFACE, 32 * TY, smem, st>>>(P, un, d, E, nyt, zchunk, ntiles);
}
template <int MX>
void launch_xr(const Dev& P, const double* un, double* d, double E, cudaStream_t st) {
  if (x_layout(P.nx, 8, MX).total <= (size_t)113 * 1024)
    launch_xw_ty<8, MX>(P, un, d, E, st);
  else
    launch_xw_ty<4, MX>(P, un, d, E, st);
}
template <int MX>
void launch_xc(const Dev& P, const double* un, double* d, double E, cudaStream_t st) {
  const int grid = resident_grid(P, kf_xc<MX>, 32 * CW, cross_smem<MX>(), (P.nfcross[0] + CW - 1) / CW);
  kf_xc<MX><<<grid, 32 * CW, cross_smem<MX>(), st>>>(P, un, d, E);
}
template <int D, int MX, bool ACC>
void launch_yt(const Dev& P, double* f, double* u, cudaStream_t st) {
  const int i1n = ACC ? P.nx : P.nx - 2;
  const int n2 = D == 1 ? P.nz : P.ny;
  const int rows = ACC ? n2 : n2 - 2;
  const int ntiles = (i1n + YZ_NL - 1) / YZ_NL * rows;
  const int grid = resident_grid(P, kf_yt<D, MX, ACC>, 32 * YZ_NL, yt_smem<MX, ACC>(), ntiles);
  kf_yt<D, MX, ACC><<<grid, 32 * YZ_NL, yt_smem<MX, ACC>(), st>>>(P, f, u, ntiles);
}
template <int D, int MX, bool ACC>
void launch_yc(const Dev& P, double* f, double* u, cudaStream_t st) {
  const int grid = resident_grid(P, kf_yc<D, MX, ACC>, 32 * CW, yc_smem<MX, ACC>(), (P.nfcross[D] + CW - 1) / CW);
  kf_yc<D, MX, ACC><<<grid, 32 * CW, yc_smem<MX, ACC>(), st>>>(P, f, u);
}

#define MTS_FAST_MX(X) X(1) X(3) X(5) X(9) X(13) X(17)

// The regular (crossing = false) or crossing lines' launch of direction d,
// dispatched on its rows per lane.
void launch_dir(const Dev& P, int d, bool crossing, const double* un, double* f, double* u, double E,
                cudaStream_t st) {
  const int n = d == 0 ? P.nx : d == 1 ? P.ny : P.nz;
  switch (fast_mx(n)) {
#define MTS_CASE(mx)                                                     \
  case mx:                                                               \
    if (d == 0 && !crossing) launch_xr<mx>(P, un, f, E, st);             \
    if (d == 0 && crossing) launch_xc<mx>(P, un, f, E, st);              \
    if (d == 1 && !crossing) launch_yt<1, mx, false>(P, f, nullptr, st); \
    if (d == 1 && crossing) launch_yc<1, mx, false>(P, f, nullptr, st);  \
    if (d == 2 && !crossing) launch_yt<2, mx, true>(P, f, u, st);        \
    if (d == 2 && crossing) launch_yc<2, mx, true>(P, f, u, st);         \
    break;
    MTS_FAST_MX(MTS_CASE)
#undef MTS_CASE
  }
}

template <int MX>
void fast_attr() {
  cudaFuncSetAttribute(kf_xw<8, MX>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSweepSmem);
  cudaFuncSetAttribute(kf_xw<4, MX>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSweepSmem);
  cudaFuncSetAttribute(kf_xc<MX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cross_smem<MX>());
  cudaFuncSetAttribute(kf_yt<1, MX, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)yt_smem<MX, false>());
  cudaFuncSetAttribute(kf_yt<2, MX, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)yt_smem<MX, true>());
  cudaFuncSetAttribute(kf_yc<1, MX, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)yc_smem<MX, false>());
  cudaFuncSetAttribute(kf_yc<2, MX, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)yc_smem<MX, true>());
}

}  // namespace

void configure_fast_kernels() {
#define MTS_ATTR(mx) fast_attr<mx>();
  MTS_FAST_MX(MTS_ATTR)
#undef MTS_ATTR
}

int fast_rows_per_lane(int n) { return fast_mx(n); }

bool fast_fits(int nx, int ny, int nz) {
  const int mx = fast_mx(nx);
  return mx && fast_mx(ny) && fast_mx(nz) && x_layout(nx, 4, mx).total <= (size_t)kMaxSweepSmem;
}

int build_fast_lines(const Dev& P, uint8_t* const fline[3], cudaStream_t st) {
  kf_fline<0><<<(unsigned)((nlines<0>(P) + TPB - 1) / TPB), TPB, 0, st>>>(P, fline[0]);
  kf_fline<1><<<(unsigned)((nlines<1>(P) + TPB - 1) / TPB), TPB, 0, st>>>(P, fline[1]);
  kf_fline<2><<<(unsigned)((nlines<2>(P) + TPB - 1) / TPB), TPB, 0, st>>>(P, fline[2]);
  return 3;
}

int build_fast_tables(const Dev& P, cudaStream_t st) {
  int launches = 0;
  const int nd[3] = {P.nx, P.ny, P.nz};
  for (int d = 0; d < 3; d++) {
    const int R = 32 * fast_mx(nd[d]);
    const unsigned g = (unsigned)((2 * R + TPB - 1) / TPB);
    double* tab = const_cast<double*>(P.ftab[d]);
    if (d == 0) kf_tab<0><<<g, TPB, 0, st>>>(P, tab, R);
    if (d == 1) kf_tab<1><<<g, TPB, 0, st>>>(P, tab, R);
    if (d == 2) kf_tab<2><<<g, TPB, 0, st>>>(P, tab, R);
    kf_tabscan<<<1, 32, 0, st>>>(tab, R, nd[d]);
    launches += 2;
    if (P.nblk[d] == 0) continue;
    double* cf = const_cast<double*>(P.fcoef[d]);
    double* bq = const_cast<double*>(P.fbq[d]);
    const unsigned gc = (unsigned)((P.nfcross[d] + TPB - 1) / TPB);
    const unsigned gb = (unsigned)((P.nblk[d] + TPB - 1) / TPB);
    if (d == 0) {
      if (gc) kf_coef<0><<<gc, TPB, 0, st>>>(P, cf, R);
      kf_bq<0><<<gb, TPB, 0, st>>>(P, bq);
    }
    if (d == 1) {
      if (gc) kf_coef<1><<<gc, TPB, 0, st>>>(P, cf, R);
      kf_bq<1><<<gb, TPB, 0, st>>>(P, bq);
    }
    if (d == 2) {
      if (gc) kf_coef<2><<<gc, TPB, 0, st>>>(P, cf, R);
      kf_bq<2><<<gb, TPB, 0, st>>>(P, bq);
    }
    launches += 2;
  }
  if (P.nmibnode > 0) {
    kf_mibref<<<(unsigned)((P.nmibnode + TPB - 1) / TPB), TPB, 0, st>>>(P, const_cast<int4*>(P.mibref));
    launches++;
  }
  return launches;
}

int launch_step_fast(const Dev& P, const StepTimes& T, double* u, double* d, cudaStream_t st, cudaEvent_t* ev,
                     const SideStream* side) {
  int launches = 0;
  auto mark = [&](int k) {
    if (ev) cudaEventRecord(ev[k], st);
  };
  // The crossing lines' kernels run on the side stream beside the regular
  // lines' (the two write disjoint lines).
  const bool two = side && side->stream;
  auto pass = [&](int dir, const double* un, double* f, double* uu, double E) {
    const bool cross = P.nfcross[dir] > 0;
    if (cross && two) {
      cudaEventRecord(side->fork, st);
      cudaStreamWaitEvent(side->stream, side->fork, 0);
      launch_dir(P, dir, true, un, f, uu, E, side->stream);
    }
    launch_dir(P, dir, false, un, f, uu, E, st);
    if (cross && !two) launch_dir(P, dir, true, un, f, uu, E, st);
    if (cross && two) {
      cudaEventRecord(side->join, side->stream);
      cudaStreamWaitEvent(st, side->join, 0);
    }
    launches += cross ? 2 : 1;
  };
  mark(0);
  if (P.nmibnode > 0) {
    kf_mib<<<(unsigned)((P.nmibnode + TPB - 1) / TPB), TPB, 0, st>>>(P, u, d, T.e_next);
    launches++;
  }

  pass(0, u, d, nullptr, T.e_next);
  mark(1);
  mark(2);
  pass(1, nullptr, d, nullptr, 0.0);
  mark(3);
  mark(4);
  pass(2, nullptr, d, u, 0.0);
  mark(5);
  return launches;
}

}  // namespace mts

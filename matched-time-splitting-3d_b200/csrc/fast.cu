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
// of operations only by rounding.  A step is four launches:
//
//   kf_mib the right-hand side of every MIB row (the explicit MIB sums of all
//          three directions and the jump terms, one thread per node; the
//          Convert2Tri row operations of the x blocks, one thread per
//          block), written into the d field at those nodes.  Their
//          dependent table walks run here, spread over many threads, and not
//          inside the line solves.
//   kf_x   rho fused with the x line solves: warp w of a CTA takes one x
//          line at a time (the CTA's warps take a 4 x 2 block of lines, so
//          that a line's y and z neighbours are mostly its siblings' lines
//          and come from L1), forms rho of its rows from coalesced loads of
//          u^n (taking the MIB rows from kf_mib), solves the line in shared
//          memory and writes d*.
//   kf_yz  the y solve in place on d*, and the z solve with the accumulation
//          u^{n+1} = u^n + d.  A CTA copies NL neighbouring lines (the same
//          row of NL lines is NL consecutive doubles) into shared memory,
//          double-buffered so that the next tile's copy overlaps this tile's
//          solves, and warp w solves line w (the Convert2Tri row operations
//          of its blocks first, douglas_adi.cc:1554-1675).
//
// Line solve: with the Thomas factors fixed (bet_j, gam_j of TDMA,
// douglas_adi.cc:1784-1807), both recurrences are first-order and linear:
//   forward   d_j = (r_j - a_j d_{j-1}) / bet_j = ib_j r_j + p_j d_{j-1}
//   backward  x_j = d_j - gam_{j+1} x_{j+1}    = d_j + q_j x_{j+1}
// with ib = 1/bet, p = -a/bet, q = -gam_{j+1}.  Lane l of the warp takes the
// rows [l MX, l MX + MX); each lane runs its rows from a zero carry, the
// lanes' affine end maps are composed by a shuffle scan, and a second pass
// runs the rows again from the true carry.  Lines without crossings read
// (ib, p, q) from per-side row tables in shared memory; the lines that cross
// the interface read their own, stored line after line ([line][ib, p, q][row]),
// so that each lane loads its rows' 27 values in one round.
#include <cuda_runtime.h>

#include <algorithm>

#include "device.h"
#include "device_common.cuh"

namespace mts {
namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int YZ_NL = 8;     // lines per tile of kf_yz (one warp each)

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

// rho at a node that is a MIB row of some x, y or z block: the explicit MIB
// sums of douglas_adi.cc:112-210 (no jumps) and the jump terms of Src_2nd.
__device__ __noinline__ double rho_mib(const Dev& P, const double* __restrict__ un, double E, long long m, int ix,
                                       int iy, int iz, int tg) {
  const int side = tg & TAG_OUT;
  const long long sy = P.nx, sz = (long long)P.nx * P.ny;
  const double* vdx = P.vd[0][side];
  const double* vdy = P.vd[1][side];
  const double* vdz = P.vd[2][side];
  int xr = 0, yr = 0, zr = 0;
  const MibBlock* xb = (tg & TAG_MIBX) ? find_block<0>(P, iy * P.nz + iz, ix, xr) : nullptr;
  const MibBlock* yb = (tg & TAG_MIBY) ? find_block<1>(P, ix * P.nz + iz, iy, yr) : nullptr;
  const MibBlock* zb = (tg & TAG_MIBZ) ? find_block<2>(P, ix * P.ny + iy, iz, zr) : nullptr;
  double sx, sy_, sz_;
  if (xb) {
    const long long base = m - ix;
    sx = mib_sum(*xb, xr, [&](int j) { return un[base + j]; }, vdx, false, P.jv);
  } else {
    sx = (un[m - 1] * vdx[0] + un[m] * vdx[1]) + un[m + 1] * vdx[2];
  }
  if (yb) {
    const long long base = ix + sz * iz;
    sy_ = mib_sum(*yb, yr, [&](int j) { return un[base + (long long)j * sy]; }, vdy, false, P.jv);
  } else {
    sy_ = (un[m - sy] * vdy[0] + un[m] * vdy[1]) + un[m + sy] * vdy[2];
  }
  if (zb) {
    const long long base = ix + (long long)P.nx * iy;
    sz_ = mib_sum(*zb, zr, [&](int j) { return un[base + (long long)j * sz]; }, vdz, false, P.jv);
  } else {
    sz_ = (un[m - sz] * vdz[0] + un[m] * vdz[1]) + un[m + sz] * vdz[2];
  }
  double src = source(P, E, side, ix, iy, iz);
  if (xb) src = src_jumps(P, E, src, *xb, xr, vdx);
  if (yb) src = src_jumps(P, E, src, *yb, yr, vdy);
  if (zb) src = src_jumps(P, E, src, *zb, zr, vdz);
  return P.dt * (((sx + sy_) + sz_) + src);
}

// The Convert2Tri row operations of a line's blocks on its right-hand side
// in shared memory (buf: the line's rows, stride 1), one lane per block.
template <int D>
__device__ __forceinline__ void block_rows(const Dev& P, double* buf, int bfirst, int bend, int lane) {
  for (int k = bfirst + lane; k < bend; k += 32) {
    const MibBlock& b = P.blk[D][k];
    double* r = buf + b.L;
    if (b.kind == 2) {
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
// lane's row jb + k (zero past the line end).
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

// A line without crossings: (ib, p, q) from the row table of its side in
// shared memory, tab[0..R) = ib, tab[R..2R) = p, tab[2R..3R) = q.
template <int MX>
__device__ __forceinline__ void solve_tab(double* buf, const double* tab, int n, int lane) {
  constexpr int R = 32 * MX;
  const int jb = lane * MX;
  solve_seg<MX>(
      buf, n, lane, [&](int k) { return tab[jb + k]; }, [&](int k) { return tab[R + jb + k]; },
      [&](int k) { return tab[2 * R + jb + k]; });
}

// A line that crosses the interface: the lane's rows of its own coefficients
// (cf: [ib, p, q][R] in global memory, zero past the line end), loaded into
// registers at once.
template <int MX>
struct LineCoef {
  double ib[MX], p[MX], q[MX];
  __device__ __forceinline__ void load(const double* __restrict__ cf, int lane) {
    constexpr int R = 32 * MX;
    const int jb = lane * MX;
#pragma unroll
    for (int k = 0; k < MX; k++) {
      ib[k] = __ldg(cf + jb + k);
      p[k] = __ldg(cf + R + jb + k);
      q[k] = __ldg(cf + 2 * R + jb + k);
    }
  }
};
template <int MX>
__device__ __forceinline__ void solve_coef(double* buf, const LineCoef<MX>& c, int n, int lane) {
  solve_seg<MX>(
      buf, n, lane, [&](int k) { return c.ib[k]; }, [&](int k) { return c.p[k]; }, [&](int k) { return c.q[k]; });
}

// What a line's solve needs to know about it, loaded ahead of its data.
struct LineMeta {
  int bfirst, bend, side1, cidx;
};
template <int D>
__device__ __forceinline__ LineMeta line_meta(const Dev& P, long long lid) {
  LineMeta m;
  m.bfirst = P.bstart[D][lid];
  m.bend = P.bstart[D][lid + 1];
  m.side1 = (P.lside[D][lid] >> 1) & 1;
  m.cidx = P.fcidx[D] ? P.fcidx[D][lid] : -1;
  return m;
}

// Row tables [side][ib, p, q][R] into shared memory.
__device__ __forceinline__ void load_tab(double* s, const double* g, int R) {
  for (int i = threadIdx.x; i < 6 * R; i += blockDim.x) s[i] = g[i];
}

// ---------------------------------------------------------------------------
// kf_mib: the MIB rows' right-hand sides of the x solve, into d.

__global__ void __launch_bounds__(TPB) kf_mib(const __grid_constant__ Dev P, const double* __restrict__ un,
                                              double* __restrict__ d, double E) {
  const long long t = (long long)blockIdx.x * TPB + threadIdx.x;
  E = step_e(P, E, 2);
  const int nxb = P.nblk[0];
  if (t < nxb) {
    // an x block: rho of its rows, then the Convert2Tri row operations
    const MibBlock& b = P.blk[0][t];
    const int iy = b.line / P.nz, iz = b.line % P.nz;
    const long long m0 = (long long)P.nx * (iy + (long long)P.ny * iz);
    double r[3] = {0.0, 0.0, 0.0};
    for (int q = 0; q < b.kind; q++) {
      const long long m = m0 + b.L + q;
      r[q] = rho_mib(P, un, E, m, b.L + q, iy, iz, P.tag[m]);
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
    for (int q = 0; q < b.kind; q++) d[m0 + b.L + q] = r[q];
    return;
  }
  const long long k = t - nxb;
  if (k >= P.nmibnode) return;
  const long long m = P.mibnode[k];
  const int tg = P.tag[m];
  if (tg & TAG_MIBX) return;  // its x block's thread writes it
  int ix, iy, iz;
  node_xyz(P, m, ix, iy, iz);
  d[m] = rho_mib(P, un, E, m, ix, iy, iz, tg);
}

// ---------------------------------------------------------------------------
// kf_x: rho fused with the x solves.

constexpr int XW = 8;  // warps per CTA of kf_x: a 4 (y) x 2 (z) block of lines

template <int MX>
__host__ __device__ constexpr size_t x_smem() {
  // row tables 6 R, one line buffer of R doubles per warp
  return sizeof(double) * ((size_t)6 * 32 * MX + (size_t)XW * 32 * MX);
}

template <int MX>
__global__ void __launch_bounds__(32 * XW, 3) kf_x(const __grid_constant__ Dev P, const double* __restrict__ un,
                                                   double* __restrict__ dst, double E) {
  constexpr int R = 32 * MX;
  extern __shared__ __align__(16) double smx[];
  double* const stab = smx;
  load_tab(stab, P.ftab[0], R);
  __syncthreads();
  E = step_e(P, E, 2);
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double* const buf = smx + 6 * R + w * R;
  const bool eq8 = P.eq != 0;
  const long long sy = nx, sz = (long long)nx * ny;
  // dt beta / h^2 of each direction, by side
  const double cx0 = P.dt * P.vd[0][0][0], cy0 = P.dt * P.vd[1][0][0], cz0 = P.dt * P.vd[2][0][0];
  const double cx1 = P.dt * P.vd[0][1][0], cy1 = P.dt * P.vd[1][1][0], cz1 = P.dt * P.vd[2][1][0];
  const int nbY = (ny + 3) / 4, nbZ = (nz + 1) / 2;
  const long long nb = (long long)nbY * nbZ;
  for (long long blk = blockIdx.x; blk < nb; blk += gridDim.x) {
    const int iy = (int)(blk % nbY) * 4 + (w & 3), iz = (int)(blk / nbY) * 2 + (w >> 2);
    if (iy >= ny || iz >= nz) continue;  // (warp-uniform)
    const long long m0 = (long long)nx * (iy + (long long)ny * iz);
    const double yv = P.ax[1][iy], zv = P.ax[2][iz];
    const double yz2 = yv * yv + zv * zv;
    if (iy == 0 || iz == 0 || iy == ny - 1 || iz == nz - 1) {
      // face line: d = Outer_u(t_next) - u^n
      for (int j = lane; j < nx; j += 32) {
        const double x = P.ax[0][j];
        dst[m0 + j] = (eq8 ? (x * x + yz2) * E : 100.0) - un[m0 + j];
      }
      continue;
    }
    const long long lid = (long long)iy * nz + iz;
    const LineMeta lm = line_meta<0>(P, lid);
    // source constants of the line: inside dt kin sin2x cos2y sin2z E,
    // outside -dt E (x^2 + y^2 + z^2) - dt 6 beta_out E
    const double kin = eq8 ? P.dt * (P.kin * ((P.c2[1][iy] * P.s2[2][iz]) * E)) : 0.0;
    const double koa = eq8 ? -P.dt * E : 0.0;
    const double kob = eq8 ? -P.dt * E * yz2 - P.dt * (P.c6bo * E) : 0.0;
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
          r = (eq8 ? fma(x * x, E, yz2 * E) : 100.0) - uc;
        } else if (t & (TAG_MIBX | TAG_MIBY | TAG_MIBZ)) {
          r = dst[m0 + j];  // from kf_mib
        } else {
          const double lx = fma(-2.0, uc, uxm + uxp);
          const double ly = fma(-2.0, uc, uym + uyp);
          const double lz = fma(-2.0, uc, uzm + uzp);
          if (t & TAG_OUT)
            r = fma(cx1, lx, fma(cy1, ly, fma(cz1, lz, fma(koa, x * x, kob))));
          else
            r = fma(cx0, lx, fma(cy0, ly, fma(cz0, lz, kin * s2x)));
        }
        buf[j] = r;
      }
    }
    __syncwarp();
    if (lm.bend > lm.bfirst) {
      LineCoef<MX> c;
      c.load(P.fcoef[0] + (size_t)lm.cidx * 3 * R, lane);
      solve_coef<MX>(buf, c, nx, lane);
    } else {
      solve_tab<MX>(buf, stab + lm.side1 * 3 * R, nx, lane);
    }
    __syncwarp();
    for (int j = lane; j < nx; j += 32) dst[m0 + j] = buf[j];
    __syncwarp();  // the buffer is free for the next line
  }
}

// ---------------------------------------------------------------------------
// kf_yz: y solves in place on d*, z solves with the accumulation into u.

template <int MX>
__host__ __device__ constexpr size_t yz_smem() {
  // row tables 6 R, two buffers of NL lines x (R + 1) doubles
  return sizeof(double) * ((size_t)6 * 32 * MX + (size_t)2 * YZ_NL * (32 * MX + 1));
}

template <int D, int MX, bool ACC>
__global__ void __launch_bounds__(32 * YZ_NL, 3) kf_yz(const __grid_constant__ Dev P, double* __restrict__ f,
                                                        double* __restrict__ u, int ntiles) {
  static_assert(D == 1 || D == 2, "y and z lines");
  constexpr int R = 32 * MX;
  constexpr int LS = R + 1;  // odd: a copy's lines and a lane's stride-MX rows fall on distinct banks
  extern __shared__ __align__(16) double smyz[];
  double* const stab = smyz;
  double* const bufs = smyz + 6 * R;
  const int nx = P.nx;
  const int n = D == 1 ? P.ny : P.nz;
  const int n2 = D == 1 ? P.nz : P.ny;  // the second line index: iz (y lines) or iy (z lines)
  const long long s = D == 1 ? (long long)nx : (long long)nx * P.ny;   // row stride
  const long long s2 = D == 1 ? (long long)nx * P.ny : (long long)nx;  // stride of the second line index
  // y tiles cover the interior lines (face y lines keep d*); z tiles cover
  // every line (face z lines pass d** through to the accumulation)
  const int i1lo = ACC ? 0 : 1, i1n = ACC ? nx : nx - 2;
  const int i2lo = ACC ? 0 : 1;
  const int tpr = (i1n + YZ_NL - 1) / YZ_NL;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int c = threadIdx.x % YZ_NL, jc = threadIdx.x / YZ_NL;  // this thread's copy share: line c, rows jc + 32 m

  load_tab(stab, P.ftab[D], R);

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
  // line c of tile T: its first element
  auto copy_in = [&](const Tile& T, double* buf) {
    const int i1 = T.i1 + c;
    if (T.ok && i1 < i1lo + i1n) {
      const long long g0 = i1 + s2 * T.i2 + (long long)jc * s;
      double* const cb = buf + c * LS;
#pragma unroll
      for (int m = 0; m < MX; m++) {
        const int j = jc + 32 * m;
        if (j < n) cp_async8(cb + j, f + g0 + (long long)32 * m * s);
      }
    }
    cp_async_commit();
  };

  int t = blockIdx.x;
  Tile cur = tile_of(t);
  copy_in(cur, bufs);
  for (int it = 0; cur.ok; it++) {
    const Tile nxt = tile_of(t + gridDim.x);
    double* const buf = bufs + (size_t)(it & 1) * YZ_NL * LS;
    copy_in(nxt, bufs + (size_t)((it + 1) & 1) * YZ_NL * LS);
    // warp w's line of this tile: what its solve needs, loaded before the
    // tile's data has landed
    const int i1w = cur.i1 + w;
    const bool solve = i1w < i1lo + i1n && i1w >= 1 && i1w <= nx - 2 && cur.i2 >= 1 && cur.i2 <= n2 - 2;
    LineMeta lm{0, 0, 0, -1};
    const long long lid = (long long)i1w * n2 + cur.i2;
    if (solve) lm = line_meta<D>(P, lid);
    cp_async_wait<1>();
    __syncthreads();
    if (solve) {
      double* const lb = buf + w * LS;
      if (lm.bend > lm.bfirst) {
        LineCoef<MX> cf;
        cf.load(P.fcoef[D] + (size_t)lm.cidx * 3 * R, lane);
        block_rows<D>(P, lb, lm.bfirst, lm.bend, lane);
        __syncwarp();
        solve_coef<MX>(lb, cf, n, lane);
      } else {
        solve_tab<MX>(lb, stab + lm.side1 * 3 * R, n, lane);
      }
    }
    __syncthreads();
    {
      const int i1 = cur.i1 + c;
      if (i1 < i1lo + i1n) {
        const long long g0 = i1 + s2 * cur.i2 + (long long)jc * s;
        const double* const cb = buf + c * LS;
        if (ACC) {
          double uv[MX];
#pragma unroll
          for (int m = 0; m < MX; m++)
            if (jc + 32 * m < n) uv[m] = u[g0 + (long long)32 * m * s];
#pragma unroll
          for (int m = 0; m < MX; m++)
            if (jc + 32 * m < n) u[g0 + (long long)32 * m * s] = uv[m] + cb[jc + 32 * m];
        } else {
#pragma unroll
          for (int m = 0; m < MX; m++)
            if (jc + 32 * m < n) f[g0 + (long long)32 * m * s] = cb[jc + 32 * m];
        }
      }
    }
    t += gridDim.x;
    cur = nxt;
  }
  cp_async_wait<0>();
}

// ---------------------------------------------------------------------------
// Set-up of the form (once per handle).

// Row tables of direction D: [side][ib, p, q][R] from the prefix factors of
// that side (ptab: bet_j, gam_j); zero past the line end.
template <int D>
__global__ void __launch_bounds__(TPB) kf_tab(const __grid_constant__ Dev P, double* tab, int R) {
  const int n = D == 0 ? P.nx : D == 1 ? P.ny : P.nz;
  const int i = blockIdx.x * TPB + threadIdx.x;
  if (i >= 2 * R) return;
  const int side = i / R, j = i % R;
  double ib = 0.0, p = 0.0, q = 0.0;
  if (j < n) {
    const double* pt = P.ptab[D][side];
    const double a = (j == 0 || j == n - 1) ? 0.0 : P.ia[D][side];
    ib = 1.0 / pt[2 * j];
    p = -a * ib;
    q = j == n - 1 ? 0.0 : -pt[2 * (j + 1) + 1];
  }
  double* T = tab + (size_t)side * 3 * R;
  T[j] = ib;
  T[R + j] = p;
  T[2 * R + j] = q;
}

// Coefficients of the lines that cross the interface, one thread per line,
// walking the line as the sequential sweep does (the factors from the prefix
// table before the first MIB row and per node from it on; the regular rows'
// side from the line's start and after each block), into the line's slot c
// of cf: [c][ib, p, q][R].
template <int D>
__global__ void __launch_bounds__(TPB) kf_coef(const __grid_constant__ Dev P, double* cf, int R) {
  const long long t = (long long)blockIdx.x * TPB + threadIdx.x;
  if (t >= nlines<D>(P)) return;
  Line L;
  decode_line<D>(P, t, L);
  if (L.boundary) return;
  const int bfirst = P.bstart[D][L.lid], bend = P.bstart[D][L.lid + 1];
  if (bfirst == bend) return;
  const int n = L.n;
  const long long s = L.s;
  const MibBlock* const blk = P.blk[D];
  const int L1 = blk[bfirst].L;
  const int side1 = (P.lside[D][L.lid] >> 1) & 1;
  const double* const pt = P.ptab[D][side1];
  double* const c = cf + (size_t)P.fcidx[D][L.lid] * 3 * R;
  int b = bfirst, side = side1;
  for (int j = 0; j < n; j++) {
    const long long g = L.base + (long long)j * s;
    const double bet = j >= L1 ? P.fbet[D][g] : pt[2 * j];
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
    const double gn = j == n - 1 ? 0.0 : j + 1 >= L1 ? P.fgam[D][g + s] : pt[2 * (j + 1) + 1];
    c[j] = 1.0 / bet;
    c[R + j] = -(a / bet);
    c[2 * R + j] = -gn;
  }
}

// ---------------------------------------------------------------------------
// Launch shapes

int fast_mx(int n) {
  const int c[6] = {1, 3, 5, 9, 13, 17};
  for (int k = 0; k < 6; k++)
    if (32 * c[k] >= n) return c[k];
  return 0;
}

template <int MX>
void launch_x(const Dev& P, const double* un, double* d, double E, cudaStream_t st) {
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kf_x<MX>, 32 * XW, x_smem<MX>());
  if (per_sm < 1) per_sm = 1;
  const long long nb = (long long)((P.ny + 3) / 4) * ((P.nz + 1) / 2);
  const int grid = (int)std::max(1LL, std::min(nb, (long long)per_sm * P.sweep_blocks));
  kf_x<MX><<<grid, 32 * XW, x_smem<MX>(), st>>>(P, un, d, E);
}

template <int D, int MX, bool ACC>
void launch_yz(const Dev& P, double* f, double* u, cudaStream_t st) {
  const int i1n = ACC ? P.nx : P.nx - 2;
  const int n2 = D == 1 ? P.nz : P.ny;
  const int rows = ACC ? n2 : n2 - 2;
  const int ntiles = (i1n + YZ_NL - 1) / YZ_NL * rows;
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kf_yz<D, MX, ACC>, 32 * YZ_NL, yz_smem<MX>());
  if (per_sm < 1) per_sm = 1;
  const int grid = std::max(1, std::min(ntiles, per_sm * P.sweep_blocks));
  kf_yz<D, MX, ACC><<<grid, 32 * YZ_NL, yz_smem<MX>(), st>>>(P, f, u, ntiles);
}

#define MTS_FAST_MX(X) X(1) X(3) X(5) X(9) X(13) X(17)

template <int D, bool ACC>
void launch_yz_n(const Dev& P, double* f, double* u, cudaStream_t st) {
  const int n = D == 1 ? P.ny : P.nz;
  switch (fast_mx(n)) {
#define MTS_CASE(mx) \
  case mx:           \
    launch_yz<D, mx, ACC>(P, f, u, st); \
    break;
    MTS_FAST_MX(MTS_CASE)
#undef MTS_CASE
  }
}

void launch_x_n(const Dev& P, const double* un, double* d, double E, cudaStream_t st) {
  switch (fast_mx(P.nx)) {
#define MTS_CASE(mx) \
  case mx:           \
    launch_x<mx>(P, un, d, E, st); \
    break;
    MTS_FAST_MX(MTS_CASE)
#undef MTS_CASE
  }
}

template <int MX>
void fast_attr() {
  cudaFuncSetAttribute(kf_x<MX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)x_smem<MX>());
  cudaFuncSetAttribute(kf_yz<1, MX, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)yz_smem<MX>());
  cudaFuncSetAttribute(kf_yz<2, MX, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)yz_smem<MX>());
}

}  // namespace

void configure_fast_kernels() {
#define MTS_ATTR(mx) fast_attr<mx>();
  MTS_FAST_MX(MTS_ATTR)
#undef MTS_ATTR
}

int fast_rows_per_lane(int n) { return fast_mx(n); }

bool fast_fits(int nx, int ny, int nz) {
  const int mx = fast_mx(nx), my = fast_mx(ny), mz = fast_mx(nz);
  return mx && my && mz;
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
    launches++;
    if (P.nblk[d] == 0) continue;
    double* cf = const_cast<double*>(P.fcoef[d]);
    if (d == 0) kf_coef<0><<<(unsigned)((nlines<0>(P) + TPB - 1) / TPB), TPB, 0, st>>>(P, cf, R);
    if (d == 1) kf_coef<1><<<(unsigned)((nlines<1>(P) + TPB - 1) / TPB), TPB, 0, st>>>(P, cf, R);
    if (d == 2) kf_coef<2><<<(unsigned)((nlines<2>(P) + TPB - 1) / TPB), TPB, 0, st>>>(P, cf, R);
    launches++;
  }
  return launches;
}

int launch_step_fast(const Dev& P, const StepTimes& T, double* u, double* d, cudaStream_t st, cudaEvent_t* ev) {
  auto mark = [&](int k) {
    if (ev) cudaEventRecord(ev[k], st);
  };
  int launches = 3;
  mark(0);
  if (P.nblk[0] > 0 || P.nmibnode > 0) {
    const long long nt = (long long)P.nblk[0] + P.nmibnode;
    kf_mib<<<(unsigned)((nt + TPB - 1) / TPB), TPB, 0, st>>>(P, u, d, T.e_next);
    launches++;
  }
  launch_x_n(P, u, d, T.e_next, st);
  mark(1);
  mark(2);
  launch_yz_n<1, false>(P, d, nullptr, st);
  mark(3);
  mark(4);
  launch_yz_n<2, true>(P, d, u, st);
  mark(5);
  return launches;
}

}  // namespace mts

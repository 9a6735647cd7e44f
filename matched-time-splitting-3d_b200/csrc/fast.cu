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
// of operations only by rounding.  A step is three launches:
//
//   kf_x   the residual rho fused with the x line solves.  A CTA owns TY
//          neighbouring x lines (rows iy0..iy0+TY-1) and walks a range of z
//          planes.  Plane by plane it brings the TY+2 rows of u^n around its
//          lines (one contiguous run of memory) and their tags into shared
//          memory with one bulk copy each (cp.async.bulk, completion on an
//          mbarrier), four planes in a ring, so that the z-1, z and z+1 rows
//          of the stencil all come from shared memory and the copy of plane
//          z+2 is in flight while plane z is computed.  Warp w forms rho of
//          line iy0+w (the MIB rows with their fictitious-point sums and jump
//          terms included), applies the Convert2Tri row operations of the
//          line's blocks (douglas_adi.cc:1554-1675), solves the line and
//          writes d* to global memory.
//   kf_yz  the y solve in place on d*, and the z solve with the accumulation
//          u^{n+1} = u^n + d.  A CTA copies NL neighbouring lines (the same
//          row of NL lines is NL consecutive doubles) into shared memory,
//          double-buffered so that the next tile's copy overlaps this tile's
//          solves, and warp w solves line w.
//
// Line solve: with the Thomas factors fixed (bet_j, gam_j of TDMA,
// douglas_adi.cc:1784-1807), both recurrences are first-order and linear:
//   forward   d_j = (r_j - a_j d_{j-1}) / bet_j = ib_j r_j + p_j d_{j-1}
//   backward  x_j = d_j - gam_{j+1} x_{j+1}    = d_j + q_j x_{j+1}
// with ib = 1/bet, p = -a/bet, q = -gam_{j+1}.  Lane l of the warp takes the
// rows [l MX, l MX + MX); each lane runs its rows from a zero carry, the
// lanes' affine end maps are composed by a shuffle scan, and a second pass
// runs the rows again from the true carry.  Lines without crossings read
// (ib, p, q) from per-side row tables; a line that crosses the interface
// recomputes its factors from the block rows (bet_j = b_j + a_j q_{j-1},
// q_j = -c_j / bet_j), each lane starting from the stored bet of its first
// row, so no per-node factor field is read.
#include <cuda_runtime.h>

#include <algorithm>

#include "device.h"
#include "device_common.cuh"

namespace mts {
namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int X_NFACE = 8;   // CTAs of kf_x that fill the face lines
constexpr int YZ_NL = 8;     // lines per tile of kf_yz (one warp each)
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

// A line without crossings: (ib, p, q) from the row table of its side,
// tab[0..R) = ib, tab[R..2R) = p, tab[2R..3R) = q (zero past the line end).
template <int MX>
__device__ __forceinline__ void solve_tab(double* buf, const double* tab, int n, int lane) {
  constexpr int R = 32 * MX;
  const int jb = lane * MX;
  double y[MX];
  double B = 0.0, A = 1.0;
#pragma unroll
  for (int k = 0; k < MX; k++) {
    const int j = jb + k;
    if (j < n) {
      const double p = tab[R + j];
      y[k] = tab[j] * buf[j];
      B = fma(p, B, y[k]);
      A *= p;
    }
  }
  double d = carry_up(A, B, lane);
#pragma unroll
  for (int k = 0; k < MX; k++) {
    const int j = jb + k;
    if (j < n) {
      d = fma(tab[R + j], d, y[k]);
      y[k] = d;
    }
  }
  B = 0.0;
  A = 1.0;
#pragma unroll
  for (int k = MX - 1; k >= 0; k--) {
    const int j = jb + k;
    if (j < n) {
      const double q = tab[2 * R + j];
      B = fma(q, B, y[k]);
      A *= q;
    }
  }
  double x = carry_down(A, B, lane);
#pragma unroll
  for (int k = MX - 1; k >= 0; k--) {
    const int j = jb + k;
    if (j < n) {
      x = fma(tab[2 * R + j], x, y[k]);
      buf[j] = x;
    }
  }
}

// A line that crosses the interface: each lane recomputes the factors of its
// rows from the stored bet of its first row (the factor recurrence of TDMA,
// douglas_adi.cc:1790-1798): regular rows a, b, c of the node's side, the
// Convert2Tri rows of the blocks, identity rows on the faces.
template <int D, int MX>
__device__ __forceinline__ void solve_cross(const Dev& P, double* buf, const FastChk& ck, int bend, int n, int lane) {
  const int jb = lane * MX;
  const MibBlock* __restrict__ blk = P.blk[D];
  double y[MX], pk[MX], qk[MX];
  double bet = ck.bet;
  int side = ck.side;
  int kb = ck.blk;
  int Lk = kb < bend ? blk[kb].L : 0x7fffffff;
  double B = 0.0, A = 1.0, qprev = 0.0;
#pragma unroll
  for (int k = 0; k < MX; k++) {
    const int j = jb + k;
    pk[k] = 0.0;
    qk[k] = 0.0;
    if (j < n) {
      double a, b, c;
      if (j == 0 || j == n - 1) {
        a = 0.0;
        b = 1.0;
        c = 0.0;
      } else if (j >= Lk) {
        const MibBlock& bk = blk[kb];
        const int q = j - Lk;
        a = bk.ia[q];
        b = bk.ib[q];
        c = bk.ic[q];
        if (q == bk.kind - 1) {
          side = (bk.sides >> q) & 1;
          kb++;
          Lk = kb < bend ? blk[kb].L : 0x7fffffff;
        }
      } else {
        a = P.ia[D][side];
        b = P.ib[D][side];
        c = P.ic[D][side];
      }
      if (k > 0) bet = fma(a, qprev, b);
      const double ib = 1.0 / bet;
      const double p = -a * ib;
      qprev = -c * ib;
      pk[k] = p;
      qk[k] = qprev;
      y[k] = ib * buf[j];
      B = fma(p, B, y[k]);
      A *= p;
    }
  }
  double d = carry_up(A, B, lane);
#pragma unroll
  for (int k = 0; k < MX; k++) {
    if (jb + k < n) {
      d = fma(pk[k], d, y[k]);
      y[k] = d;
    }
  }
  B = 0.0;
  A = 1.0;
#pragma unroll
  for (int k = MX - 1; k >= 0; k--) {
    if (jb + k < n) {
      B = fma(qk[k], B, y[k]);
      A *= qk[k];
    }
  }
  double x = carry_down(A, B, lane);
#pragma unroll
  for (int k = MX - 1; k >= 0; k--) {
    const int j = jb + k;
    if (j < n) {
      x = fma(qk[k], x, y[k]);
      buf[j] = x;
    }
  }
}

// Solve line lid of direction D held in buf (after its block rows).
template <int D, int MX>
__device__ __forceinline__ void solve_line(const Dev& P, double* buf, const double* stab, long long lid, int n,
                                           int lane) {
  constexpr int R = 32 * MX;
  const int bfirst = P.bstart[D][lid], bend = P.bstart[D][lid + 1];
  if (bfirst == bend) {
    const int side1 = (P.lside[D][lid] >> 1) & 1;
    solve_tab<MX>(buf, stab + side1 * 3 * R, n, lane);
  } else {
    block_rows<D>(P, buf, bfirst, bend, lane);
    __syncwarp();
    const FastChk ck = P.fchk[D][lid * 32 + lane];
    solve_cross<D, MX>(P, buf, ck, bend, n, lane);
  }
}

// Row tables [side][ib, p, q][R] into shared memory.
__device__ __forceinline__ void load_tab(double* s, const double* g, int R) {
  for (int i = threadIdx.x; i < 6 * R; i += blockDim.x) s[i] = g[i];
}

// ---------------------------------------------------------------------------
// kf_x: rho fused with the x solves.

struct XLayout {
  int slabd;  // doubles per u^n slab (TY+2 rows, aligned start, even)
  int tagb;   // bytes per tag slab (TY rows, multiple of 16)
  size_t o_tag, o_xt, o_tab, o_bar, total;
};
__host__ __device__ inline XLayout x_layout(int nx, int TY, int R) {
  XLayout L;
  L.slabd = ((TY + 2) * nx + 2 + 1) & ~1;
  L.tagb = (TY * nx + 32 + 15) & ~15;
  L.o_tag = (size_t)4 * L.slabd * sizeof(double);
  L.o_xt = L.o_tag + (size_t)4 * L.tagb;
  L.o_tab = L.o_xt + (((size_t)2 * nx * sizeof(double) + 15) & ~(size_t)15);
  L.o_bar = L.o_tab + (size_t)6 * R * sizeof(double);
  L.total = L.o_bar + 4 * sizeof(uint64_t);
  return L;
}

template <int TY, int MX>
__global__ void __launch_bounds__(32 * TY, 2) kf_x(const __grid_constant__ Dev P, const double* __restrict__ un,
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
        const double out = eq8 ? (x * x + yz2) * E : 100.0;
        dst[m0 + ix] = out - un[m0 + ix];
      }
    }
    return;
  }

  extern __shared__ __align__(16) unsigned char smx[];
  const XLayout LY = x_layout(nx, TY, R);
  double* const slab = reinterpret_cast<double*>(smx);
  unsigned char* const tslab = smx + LY.o_tag;
  double* const xs2 = reinterpret_cast<double*>(smx + LY.o_xt);  // sin 2x
  double* const xxx = xs2 + nx;                                   // x^2
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
    const int s = i & 3;
    int sh;
    const double* gu = slab_src(i, sh);
    const unsigned char* gt = tag_src(i, sh);
    mbar_expect(&bar[s], ubytes + tbytes);
    bulk_copy(slab + (size_t)s * LY.slabd, gu, ubytes, &bar[s]);
    bulk_copy(tslab + (size_t)s * LY.tagb, gt, tbytes, &bar[s]);
  };

  if (threadIdx.x == 0) {
    for (int s = 0; s < 4; s++) mbar_init(&bar[s]);
    mbar_init_fence();
  }
  __syncthreads();
  if (threadIdx.x == 0)
    for (int i = 0; i < 3 && i < nslabs; i++) issue(i);
  for (int i = threadIdx.x; i < nx; i += blockDim.x) {
    xs2[i] = P.s2[0][i];
    const double x = P.ax[0][i];
    xxx[i] = x * x;
  }
  load_tab(stab, P.ftab[0], R);
  __syncthreads();

  // dt beta / h^2 of each direction, by side
  const double cx0 = P.dt * P.vd[0][0][0], cy0 = P.dt * P.vd[1][0][0], cz0 = P.dt * P.vd[2][0][0];
  const double cx1 = P.dt * P.vd[0][1][0], cy1 = P.dt * P.vd[1][1][0], cz1 = P.dt * P.vd[2][1][0];
  const int iy = y0 + w;
  const bool live = iy <= ny - 2;
  const double yv = P.ax[1][live ? iy : 1];
  const int jb = lane * MX;
  bool bad = false;

  for (int pi = 0; pi < nplanes; pi++) {
    if (threadIdx.x == 0 && pi + 3 < nslabs) issue(pi + 3);
    const int iz = z0 + pi;
    // slabs pi (z-1), pi+1 (z), pi+2 (z+1) must have landed
    bool ok = true;
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const int i = pi + k;
      ok = ok && mbar_wait(&bar[i & 3], (unsigned)((i >> 2) & 1));
    }
    if (!ok) bad = true;
    if (live && ok) {
      int shm, shc, shp, tsh;
      slab_src(pi, shm);
      slab_src(pi + 1, shc);
      slab_src(pi + 2, shp);
      tag_src(pi + 1, tsh);
      const double* const sc = slab + (size_t)((pi + 1) & 3) * LY.slabd + shc + (size_t)(w + 1) * nx;
      const double* const sym = sc - nx;
      const double* const syp = sc + nx;
      double* const szm = slab + (size_t)(pi & 3) * LY.slabd + shm + (size_t)(w + 1) * nx;
      const double* const szp = slab + (size_t)((pi + 2) & 3) * LY.slabd + shp + (size_t)(w + 1) * nx;
      const unsigned char* const tg = tslab + (size_t)((pi + 1) & 3) * LY.tagb + tsh + (size_t)w * nx;
      const double zv = P.ax[2][iz];
      const double yz2 = yv * yv + zv * zv;
      // source constants of the line: inside dt kin sin2x cos2y sin2z E,
      // outside -dt E (x^2 + y^2 + z^2) - dt 6 beta_out E
      const double kin = eq8 ? P.dt * (P.kin * ((P.c2[1][iy] * P.s2[2][iz]) * E)) : 0.0;
      const double koa = eq8 ? -P.dt * E : 0.0;
      const double kob = eq8 ? -P.dt * E * yz2 - P.dt * (P.c6bo * E) : 0.0;
      const long long m0 = (long long)nx * (iy + (long long)ny * iz);
      // rho into the line buffer: the z-1 row of this line, which no other
      // warp reads (each element is read before this lane overwrites it)
      double* const buf = szm;
#pragma unroll
      for (int k = 0; k < MX; k++) {
        const int j = jb + k;
        if (j < nx) {
          const double uc = sc[j];
          double r;
          if (j == 0 || j == nx - 1) {
            r = (eq8 ? fma(xxx[j], E, yz2 * E) : 100.0) - uc;
          } else {
            const int t = tg[j];
            if (t & (TAG_MIBX | TAG_MIBY | TAG_MIBZ)) {
              r = rho_mib(P, un, E, m0 + j, j, iy, iz, t);
            } else {
              const double lx = fma(-2.0, uc, sc[j - 1] + sc[j + 1]);
              const double ly = fma(-2.0, uc, sym[j] + syp[j]);
              const double lz = fma(-2.0, uc, buf[j] + szp[j]);
              if (t & TAG_OUT)
                r = fma(cx1, lx, fma(cy1, ly, fma(cz1, lz, fma(koa, xxx[j], kob))));
              else
                r = fma(cx0, lx, fma(cy0, ly, fma(cz0, lz, kin * xs2[j])));
            }
          }
          buf[j] = r;
        }
      }
      __syncwarp();
      solve_line<0, MX>(P, buf, stab, (long long)iy * nz + iz, nx, lane);
      __syncwarp();
      for (int j = lane; j < nx; j += 32) dst[m0 + j] = buf[j];
    }
    // every thread's shared-memory accesses to the slot reloaded next are done
    fence_async_smem();
    if (__syncthreads_or(bad)) {
      if (threadIdx.x == 0) {
        atomicOr(P.status, 2);
        // let the copies still in flight land before the CTA leaves
        for (int i = pi + 3; i < nslabs && i < pi + 4; i++) mbar_wait(&bar[i & 3], (unsigned)((i >> 2) & 1));
      }
      return;
    }
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
    cp_async_wait<1>();
    __syncthreads();
    {
      const int i1 = cur.i1 + w;
      const bool interior = i1 >= 1 && i1 <= nx - 2 && cur.i2 >= 1 && cur.i2 <= n2 - 2;
      if (i1 < i1lo + i1n && interior) {
        const long long lid = (long long)i1 * n2 + cur.i2;
        solve_line<D, MX>(P, buf + w * LS, stab, lid, n, lane);
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

// Checkpoints of the lines that cross the interface: for lane l, the bet of
// row l MX (the prefix table before the first MIB row, the per-node factors
// from it on), the side of the regular rows there and the first block that
// ends at or after it.
template <int D>
__global__ void __launch_bounds__(TPB) kf_chk(const __grid_constant__ Dev P, FastChk* chk, int MX) {
  const long long t = (long long)blockIdx.x * TPB + threadIdx.x;
  const long long line = t >> 5;
  const int l = (int)(t & 31);
  if (line >= nlines<D>(P)) return;
  Line L;
  decode_line<D>(P, line, L);
  if (L.boundary) return;
  const int bfirst = P.bstart[D][L.lid], bend = P.bstart[D][L.lid + 1];
  if (bfirst == bend) return;
  const int jb = l * MX;
  if (jb >= L.n) return;
  const MibBlock* blk = P.blk[D];
  const int L1 = blk[bfirst].L;
  const int side1 = (P.lside[D][L.lid] >> 1) & 1;
  FastChk c;
  c.bet = jb < L1 ? P.ptab[D][side1][2 * jb] : P.fbet[D][L.base + (long long)jb * L.s];
  int side = side1, k = bfirst;
  while (k < bend && blk[k].L + blk[k].kind - 1 < jb) {
    side = (blk[k].sides >> (blk[k].kind - 1)) & 1;
    k++;
  }
  c.side = side;
  c.blk = k;
  chk[(long long)L.lid * 32 + l] = c;
}

// ---------------------------------------------------------------------------
// Launch shapes

template <int TY, int MX>
size_t x_smem_of(int nx) {
  return x_layout(nx, TY, 32 * MX).total;
}

int fast_mx(int n) {
  const int c[6] = {1, 3, 5, 9, 13, 17};
  for (int k = 0; k < 6; k++)
    if (32 * c[k] >= n) return c[k];
  return 0;
}

// kf_x with TY lines per CTA: the z range of a CTA is chosen so that the
// tiles fill the resident CTAs of the GPU about once.
template <int TY, int MX>
void launch_x(const Dev& P, const double* un, double* d, double E, cudaStream_t st) {
  const size_t smem = x_smem_of<TY, MX>(P.nx);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kf_x<TY, MX>, 32 * TY, smem);
  if (per_sm < 1) per_sm = 1;
  const int nyt = (P.ny - 2 + TY - 1) / TY;
  const int target = std::max(1, per_sm * P.sweep_blocks - X_NFACE);
  int nzc = std::max(1, std::min(P.nz - 2, target / nyt));
  const int zchunk = (P.nz - 2 + nzc - 1) / nzc;
  nzc = (P.nz - 2 + zchunk - 1) / zchunk;
  const int ntiles = nyt * nzc;
  kf_x<TY, MX><<<ntiles + X_NFACE, 32 * TY, smem, st>>>(P, un, d, E, nyt, zchunk, ntiles);
}

template <int MX>
void launch_x_mx(const Dev& P, const double* un, double* d, double E, cudaStream_t st) {
  if (x_smem_of<8, MX>(P.nx) <= (size_t)113 * 1024)
    launch_x<8, MX>(P, un, d, E, st);
  else
    launch_x<4, MX>(P, un, d, E, st);
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
    launch_x_mx<mx>(P, un, d, E, st); \
    break;
    MTS_FAST_MX(MTS_CASE)
#undef MTS_CASE
  }
}

template <int TY, int MX>
void x_attr() {
  cudaFuncSetAttribute(kf_x<TY, MX>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSweepSmem);
}
template <int MX>
void fast_attr() {
  x_attr<8, MX>();
  x_attr<4, MX>();
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
  if (!mx || !my || !mz) return false;
  if (x_layout(nx, 4, 32 * mx).total > (size_t)kMaxSweepSmem) return false;
  return true;
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
    FastChk* chk = const_cast<FastChk*>(P.fchk[d]);
    const int mx = fast_mx(nd[d]);
    if (d == 0) kf_chk<0><<<(unsigned)((nlines<0>(P) * 32 + TPB - 1) / TPB), TPB, 0, st>>>(P, chk, mx);
    if (d == 1) kf_chk<1><<<(unsigned)((nlines<1>(P) * 32 + TPB - 1) / TPB), TPB, 0, st>>>(P, chk, mx);
    if (d == 2) kf_chk<2><<<(unsigned)((nlines<2>(P) * 32 + TPB - 1) / TPB), TPB, 0, st>>>(P, chk, mx);
    launches++;
  }
  return launches;
}

int launch_step_fast(const Dev& P, const StepTimes& T, double* u, double* d, cudaStream_t st, cudaEvent_t* ev) {
  auto mark = [&](int k) {
    if (ev) cudaEventRecord(ev[k], st);
  };
  mark(0);
  launch_x_n(P, u, d, T.e_next, st);
  mark(1);
  mark(2);
  launch_yz_n<1, false>(P, d, nullptr, st);
  mark(3);
  mark(4);
  launch_yz_n<2, true>(P, d, u, st);
  mark(5);
  return 3;
}

}  // namespace mts

// Mixed-precision form of the Douglas-ADI step (precision = 1).
//
// The Douglas step (douglas_adi.cc:66-1110) is three line solves,
//   (I - A_x) u*     = u^n + A_y u^n + A_z u^n + dt src
//   (I - A_y) u**    = u* - A_y u^n
//   (I - A_z) u^n+1  = u** - A_z u^n,
// with A_d = dt beta D_dd (MIB rows included) and src carrying f and the jump
// terms of Src_2nd.  Written for the increments d* = u* - u^n, d** = u** - u^n
// and d = u^{n+1} - u^n the same equations read
//   (I - A_x) d*  = rho = dt (A_x u^n + A_y u^n + A_z u^n + src)
//   (I - A_y) d** = d*
//   (I - A_z) d   = d**,      u^{n+1} = u^n + d,
// and on the faces d = Outer_u(t^{n+1}) - u^n.  The residual rho is formed in
// FP64 from the FP64 state, the three line solves run on FP32 increments
// (4-byte fields and scratch, FP32 factors), and the increment is added to the
// FP64 state after the last sweep.  The FP32 rounding thus touches only the
// increment of one step, never the accumulated solution.
#include <cuda_runtime.h>

#include <algorithm>

#include "device.h"
#include "device_common.cuh"

namespace mts {
namespace {

// ---------------------------------------------------------------------------
// Residual rho = dt (A_x u + A_y u + A_z u + src), FP64 in, FP32 out.

template <int G>
__device__ __forceinline__ void adi_resid_body(const Dev& P, unsigned cta_, unsigned ncta_,
                                               const double* __restrict__ un, float* __restrict__ rho, double E) {
  E = step_e(P, E, 2);
  const long long sy = P.nx, sz = (long long)P.nx * P.ny;
  const int lane = threadIdx.x & 31;
  const int nrows = P.ny * P.nz;
  const double dt = P.dt;
  // a node's side selects one of two specialised bodies (uniform over a
  // warp away from the interface), whose stencil weights are fixed kernel
  // parameters (constant-bank operands, no registers)
  for (int row = cta_ * (TPB / 32) + (threadIdx.x >> 5); row < nrows; row += ncta_ * (TPB / 32)) {
    const int iy = row % P.ny, iz = row / P.ny;
    const long long m0 = (long long)P.nx * row;
    const RowExact q = row_exact(P, iy, iz);
    if (iy == 0 || iz == 0 || iy == P.ny - 1 || iz == P.nz - 1) {
      for (int ix = lane; ix < P.nx; ix += 32) rho[m0 + ix] = (float)(row_outer(P, q, ix, E) - un[m0 + ix]);
      continue;
    }
    // the row and its four neighbour rows, indexed by ix (an interior row:
    // uc_r[-1] and uc_r[nx] lie inside the field)
    const double* const uc_r = un + m0;
    const double* const uym_r = uc_r - sy;
    const double* const uyp_r = uc_r + sy;
    const double* const uzm_r = uc_r - sz;
    const double* const uzp_r = uc_r + sz;
    const uint8_t* const tg_r = P.tag + m0;
    float* const rho_r = rho + m0;
    for (int ix0 = 0; ix0 < P.nx; ix0 += 32 * G) {
      double uc[G], uxm[G], uxp[G], uym[G], uyp[G], uzm[G], uzp[G];
      int tg[G];
#pragma unroll
      for (int g = 0; g < G; g++) {
        const int ix = ix0 + 32 * g + lane;
        if (ix < P.nx) {
          tg[g] = tg_r[ix];
          uc[g] = uc_r[ix];
          uxm[g] = uc_r[ix - 1];
          uxp[g] = uc_r[ix + 1];
          uym[g] = uym_r[ix];
          uyp[g] = uyp_r[ix];
          uzm[g] = uzm_r[ix];
          uzp[g] = uzp_r[ix];
        }
      }
#pragma unroll
      for (int g = 0; g < G; g++) {
        const int ix = ix0 + 32 * g + lane;
        if (ix >= P.nx) break;
        double r;
        if (ix == 0 || ix == P.nx - 1) {
          r = row_outer(P, q, ix, E) - uc[g];
        } else if (!(tg[g] & (TAG_MIBX | TAG_MIBY | TAG_MIBZ))) {
          auto node = [&](auto S) {
            constexpr int sd = decltype(S)::value;
            const double sx = (uxm[g] * P.vd[0][sd][0] + uc[g] * P.vd[0][sd][1]) + uxp[g] * P.vd[0][sd][2];
            const double sy_ = (uym[g] * P.vd[1][sd][0] + uc[g] * P.vd[1][sd][1]) + uyp[g] * P.vd[1][sd][2];
            const double sz_ = (uzm[g] * P.vd[2][sd][0] + uc[g] * P.vd[2][sd][1]) + uzp[g] * P.vd[2][sd][2];
            return dt * (((sx + sy_) + sz_) + row_source(P, q, ix, E, sd));
          };
          r = (tg[g] & TAG_OUT) ? node(IntC<1>{}) : node(IntC<0>{});
        } else {
          continue;  // a MIB row: k_adi_resid_mib writes it
        }
        rho_r[ix] = (float)r;
      }
    }
  }
}

template <int G>
__global__ void __launch_bounds__(TPB, 8) k_adi_resid(const __grid_constant__ Dev P, const double* __restrict__ un,
                                                   float* __restrict__ rho, double E) {
  adi_resid_body<G>(P, blockIdx.x, gridDim.x, un, rho, E);
}

// The MIB rows of rho, one thread per listed node: the explicit MIB sums of
// every direction the node is a MIB row of (douglas_adi.cc:112-210, without
// jumps) and the jump terms of Src_2nd (douglas_adi.cc:1156-1427).
__device__ __forceinline__ void adi_resid_mib_body(const Dev& P, unsigned cta_, const double* __restrict__ un,
                                                   float* __restrict__ rho, double E) {
  const int k = cta_ * TPB + threadIdx.x;
  if (k >= P.nmibnode) return;
  E = step_e(P, E, 2);
  const long long m = P.mibnode[k];
  int ix, iy, iz;
  node_xyz(P, m, ix, iy, iz);
  const int tg = P.tag[m];
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
  if (xb) src = adi_src_add(src, *xb, xr, vdx, P.jv);
  if (yb) src = adi_src_add(src, *yb, yr, vdy, P.jv);
  if (zb) src = adi_src_add(src, *zb, zr, vdz, P.jv);
  rho[m] = (float)(P.dt * (((sx + sy_) + sz_) + src));
}

__global__ void __launch_bounds__(TPB) k_adi_resid_mib(const __grid_constant__ Dev P, const double* __restrict__ un,
                                                       float* __restrict__ rho, double E) {
  adi_resid_mib_body(P, blockIdx.x, un, rho, E);
}

// ---------------------------------------------------------------------------
// FP32 line solves of the increments.

// Block pre-pass: the Convert2Tri row operations (douglas_adi.cc:1554-1675)
// on the right-hand sides of each block's rows, in FP64, stored in FP32.
// INPLACE (the segmented solves): the results replace the rows' right-hand
// sides in the field, else they go to rblk32 for the ring sweeps.
template <int D, bool INPLACE>
__device__ __forceinline__ void block_rhs32_body(const Dev& P, unsigned cta_, float* __restrict__ f, int nblk) {
  const int k = cta_ * TPB + threadIdx.x;
  if (k >= nblk) return;
  const MibBlock& b = P.blk[D][k];
  const int n2 = D == 2 ? P.ny : P.nz;
  Line L;
  decode_line<D>(P, (long long)(b.line % n2) * (D == 0 ? P.ny : P.nx) + b.line / n2, L);
  double r[3] = {0.0, 0.0, 0.0};
  for (int q = 0; q < b.kind; q++) r[q] = f[L.base + (long long)(b.L + q) * L.s];
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
  if (INPLACE)
    for (int q = 0; q < b.kind; q++) f[L.base + (long long)(b.L + q) * L.s] = (float)r[q];
  else
    for (int q = 0; q < 3; q++) P.rblk32[D][3 * k + q] = (float)r[q];
}

template <int D, bool INPLACE>
__global__ void __launch_bounds__(TPB) k_block_rhs32(const __grid_constant__ Dev P, float* __restrict__ f,
                                                     int nblk) {
  block_rhs32_body<D, INPLACE>(P, blockIdx.x, f, nblk);
}

struct BlockHead32 {
  int L, kind, sides;
  float a0, a1, a2;  // sub-diagonal of the block's rows after Convert2Tri
  float r0, r1, r2;  // their right-hand sides this sweep
};

__device__ __forceinline__ void load_head32(const MibBlock* blk, const float* rblk, int k, int end, BlockHead32& h) {
  if (k < end) {
    const MibBlock& b = blk[k];
    h.L = b.L;
    h.kind = b.kind;
    h.sides = b.sides;
    h.a0 = (float)b.ia[0];
    h.a1 = (float)b.ia[1];
    h.a2 = (float)b.ia[2];
    h.r0 = rblk[3 * k];
    h.r1 = rblk[3 * k + 1];
    h.r2 = rblk[3 * k + 2];
  } else {
    h.L = 0x7fffffff;
    h.kind = 0;
    h.sides = 0;
  }
}

__device__ __forceinline__ void cp_async4(float* smem_dst, const float* gsrc) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gsrc) : "memory");
}

// Shared memory of a shape: rings A and C and the two prefix factor tables
// (2 sides x 2 values x n rows), all FP32.
template <int CH, int NS, int NT>
constexpr size_t shape32_smem(int n) {
  // x sweeps pad each ring row by 4 floats; the size covers that case
  return sizeof(float) * ((size_t)2 * NS * CH * (NT + 4) + (size_t)4 * n);
}

// One thread per line, persistent CTAs, as the FP64 sweep (kernels.cu): f
// holds the right-hand side and receives the solution in place.  Ring A
// stages f (forward) and d' (backward); ring C stages 1/bet (forward) and gam
// (backward) of crossing lines from their first MIB row on.
template <int D, int CH, int NS, int NT>
__global__ void __launch_bounds__(NT, 1) k_sweep32(const __grid_constant__ Dev P, float* f) {
  static_assert((CH & (CH - 1)) == 0 && (NS & (NS - 1)) == 0 && NS >= 4 && CH >= 4 && CH <= kRowPad, "shape");
  constexpr int RING = NS * CH;
  // x lines are staged and stored by the warp together (as in the FP64 sweep),
  // with 4 floats of padding per ring row so that a copy's lanes (CH rows of
  // 32/CH columns) fall on 32 distinct banks
  constexpr bool kCoop = D == 0;
  constexpr int RS = kCoop ? NT + 4 : NT;  // floats per ring row
  constexpr int SLOT = CH * RS;
  extern __shared__ float sm32[];
  const int tid = threadIdx.x;
  float* const sA = sm32 + tid;
  float* const sC = sA + NS * SLOT;
#define RA(j) sA[((j) & (RING - 1)) * RS]
#define RC(j) sC[((j) & (RING - 1)) * RS]
  const long long T = (long long)gridDim.x * NT;
  const long long gt = (long long)blockIdx.x * NT + tid;
  float* const dp = P.dp32 + gt;
  const long long nl = nlines<D>(P);
  const MibBlock* __restrict__ blk = P.blk[D];
  const float* __restrict__ fib = P.fib32[D];
  const float* __restrict__ fgam = P.fgam32[D];
  const float* __restrict__ rblk = P.rblk32[D];
  const float ai = (float)P.ia[D][0], ao = (float)P.ia[D][1];
  const int nd = D == 0 ? P.nx : D == 1 ? P.ny : P.nz;
  float* const sP = sm32 + 2 * NS * SLOT;
  for (int i = tid; i < 4 * nd; i += NT) sP[i] = i < 2 * nd ? P.ptab32[D][0][i] : P.ptab32[D][1][i - 2 * nd];
  __syncthreads();
  const int lane = tid & 31;
  float* const sAw = sm32 + (tid - lane);  // the warp's first column of ring A
  const long long nxl = P.nx;

  for (long long t0 = gt - (kCoop ? lane : 0); t0 < nl; t0 += T) {
    const long long t = kCoop ? t0 + lane : t0;
    const bool act = t < nl;
    Line L;
    decode_line<D>(P, act ? t : nl - 1, L);
    const int n = L.n;
    const long long s = L.s;
    // face line: the solution is the right-hand side itself
    const bool solve = act && !L.boundary;
    if (!kCoop && !solve) continue;
    unsigned solvers = 0;
    if (kCoop) {
      solvers = __ballot_sync(0xffffffffu, solve);
      if (!solvers) continue;
    }
    const int nch = (n + CH - 1) / CH;
    const int ls = P.lside[D][L.lid];
    const int bfirst = P.bstart[D][L.lid];
    const int bend = P.bstart[D][L.lid + 1];
    const int L1 = bfirst < bend ? blk[bfirst].L : n;
    const float* pt = sP + ((ls >> 1) & 1) * 2 * nd;
    const float* gA = f + L.base;
    const float* gC = fib + L.base;
    int L1q[CH];
    long long gq[CH];  // start of the line each cooperative copy serves, -1 past the end
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
          float* aw = sAw + (c & (NS - 1)) * SLOT;
          float* cw = aw + NS * SLOT;
#pragma unroll
          for (int q = 0; q < CH; q++) {
            const int e = q * 32 + lane, l = e / CH, r = e % CH;
            if (gq[q] >= 0) {
              const long long g = gq[q] + (long long)c * CH;
              cp_async4(aw + r * RS + l, f + g);
              if ((c + 1) * CH > L1q[q] && L1q[q] < n) cp_async4(cw + r * RS + l, fib + g);
            }
          }
        }
        cp_async_commit();
        return;
      }
      if (c < nch) {
        const long long off = (long long)c * CH * s;
        float* a = sA + (c & (NS - 1)) * SLOT;
#pragma unroll
        for (int r = 0; r < CH; r++) cp_async4(a + r * RS, gA + off + r * s);
        if ((c + 1) * CH > L1 && L1 < n) {  // per-node factors exist only for lines with blocks
          float* cc = sC + (c & (NS - 1)) * SLOT;
#pragma unroll
          for (int r = 0; r < CH; r++) cp_async4(cc + r * RS, gC + off + r * s);
        }
      }
      cp_async_commit();
    };

    // forward: d'_j = (r_j - a_j d'_{j-1}) / bet_j
    for (int c = 0; c < NS - 2; c++) stage(c);
    int mb = bfirst;
    BlockHead32 hb, hb2;
    load_head32(blk, rblk, mb, bend, hb);
    load_head32(blk, rblk, mb + 1, bend, hb2);
    int mside = (ls >> 1) & 1;
    float dprev = 0.0f;
    int j = 1;
    for (int c = 0; c < nch; c++) {
      if (kCoop) __syncwarp();  // every lane is done with the slot restaged next
      stage(c + NS - 2);
      cp_async_wait<NS - 3>();
      if (kCoop) {
        __syncwarp();  // the other lanes' copies into this lane's column are visible
        if (!solve) continue;
      }
      if (c == 0) {
        dprev = RA(0) * pt[0];
        dp[0] = dprev;
      }
      const int c0 = c * CH;
      const int cend = min(c0 + CH, n - 1);
      if (j >= cend) continue;
      if (j == c0 && cend == c0 + CH && hb.L >= cend && (cend <= L1 || c0 >= L1)) {
        const float ac = mside ? ao : ai;
        const float* a = sA + (c & (NS - 1)) * SLOT;
        float* q = dp + (long long)c0 * T;
        auto run = [&](auto tag) {
          constexpr bool kField = decltype(tag)::value;
          const float* bt = kField ? sC + (c & (NS - 1)) * SLOT : pt + 2 * c0;
#pragma unroll
          for (int rr = 0; rr < CH; rr++) {
            const float ib = kField ? bt[rr * RS] : bt[2 * rr];
            const float d = __fmul_rn(__fmaf_rn(-ac, dprev, a[rr * RS]), ib);
            q[rr * T] = d;
            dprev = d;
          }
        };
        if (c0 >= L1)
          run(BoolC<true>{});
        else
          run(BoolC<false>{});
        j = cend;
      } else {
        while (j < cend) {
          const float ib = j >= L1 ? RC(j) : pt[2 * j];
          if (j == hb.L) {
            float d = __fmul_rn(__fmaf_rn(-hb.a0, dprev, hb.r0), ib);
            dp[(long long)j * T] = d;
            d = __fmul_rn(__fmaf_rn(-hb.a1, d, hb.r1), RC(j + 1));
            dp[(long long)(j + 1) * T] = d;
            if (hb.kind == 3) {
              d = __fmul_rn(__fmaf_rn(-hb.a2, d, hb.r2), RC(j + 2));
              dp[(long long)(j + 2) * T] = d;
            }
            dprev = d;
            mside = (hb.sides >> (hb.kind - 1)) & 1;
            j += hb.kind;
            mb++;
            hb = hb2;
            load_head32(blk, rblk, mb + 1, bend, hb2);
          } else {
            const float d = __fmul_rn(__fmaf_rn(-(mside ? ao : ai), dprev, RA(j)), ib);
            dp[(long long)j * T] = d;
            dprev = d;
            j++;
          }
        }
      }
    }
    if (solve) {
      // last row: the Dirichlet identity row (a = 0)
      const float ib = n - 1 >= L1 ? RC(n - 1) : pt[2 * (n - 1)];
      dp[(long long)(n - 1) * T] = __fmul_rn(RA(n - 1), ib);
    }
    cp_async_wait<0>();

    // backward: x_j = d'_j - gam_{j+1} x_{j+1}
    __threadfence_block();
    const float* gG = fgam + L.base;
    auto bstage = [&](int c) {
      if (c >= 0) {
        float* a = sA + (c & (NS - 1)) * SLOT;
        const float* g = dp + (long long)c * CH * T;
#pragma unroll
        for (int r = 0; r < CH; r++) cp_async4(a + r * RS, g + r * T);
        if ((c + 1) * CH >= L1 && L1 < n) {
          float* b = sC + (c & (NS - 1)) * SLOT;
          const long long off = ((long long)c * CH + 1) * s;
#pragma unroll
          for (int r = 0; r < CH; r++) cp_async4(b + r * RS, gG + off + r * s);
        }
      }
      cp_async_commit();
    };
    float xnext = 0.0f;
    for (int c = nch - 1; c > nch - NS; c--) bstage(c);
    for (int c = nch - 1; c >= 0; c--) {
      if (kCoop) __syncwarp();  // the previous chunk's stores have read its slot
      bstage(c - NS + 1);
      cp_async_wait<NS - 1>();
      const int c0 = c * CH;
      if (!solve) {
      } else if (c0 + CH <= n - 1 && (c0 + CH < L1 || c0 + 1 >= L1)) {
        float* a = sA + (c & (NS - 1)) * SLOT;
        auto run = [&](auto tag) {
          constexpr bool kField = decltype(tag)::value;
          const float* gb = kField ? sC + (c & (NS - 1)) * SLOT : pt + 2 * c0 + 3;
#pragma unroll
          for (int rr = CH - 1; rr >= 0; rr--) {
            const float gm = kField ? gb[rr * RS] : gb[2 * rr];
            const float x = __fmaf_rn(-gm, xnext, a[rr * RS]);
            xnext = x;
            if (kCoop)
              a[rr * RS] = x;
            else
              f[L.base + (long long)(c0 + rr) * s] = x;
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
          float x = RA(jj);
          if (jj != n - 1) x = __fmaf_rn(-(jj + 1 >= L1 ? RC(jj) : pt[2 * (jj + 1) + 1]), xnext, x);
          xnext = x;
          if (kCoop)
            RA(jj) = x;
          else
            f[L.base + (long long)jj * s] = x;
        }
      }
      if (kCoop) {
        __syncwarp();
        const float* aw = sAw + (c & (NS - 1)) * SLOT;
#pragma unroll
        for (int q = 0; q < CH; q++) {
          const int e = q * 32 + lane, l = e / CH, r = e % CH;
          if (((solvers >> l) & 1u) && c0 + r < n) f[gq[q] + c0] = aw[r * RS + l];
        }
      }
    }
    cp_async_wait<0>();
  }
#undef RA
#undef RC
}

// ---------------------------------------------------------------------------
// Segmented FP32 line solves.  With the factors fixed, both Thomas
// recurrences are first-order and linear:
//   forward   d_j = (r_j - a_j d_{j-1}) / bet_j = r_j ib_j + p_j d_{j-1}
//   backward  x_j = d_j - gam_{j+1} x_{j+1}    = d_j + q_j x_{j+1}
// with ib_j = 1/bet_j, p_j = -a_j/bet_j and q_j = -gam_{j+1} stored per node
// (Dev::cib/cp/cq; block rows carry their Convert2Tri sub-diagonal, face
// rows p = 0, the last row q = 0).  A line is cut into segments that run at
// once: each runs the recurrence from a zero carry while it multiplies up
// its multipliers (P_j, Q_j); the segments' end states (value, product)
// compose into the carry of every segment, and the true values are
//   d_j = d~_j + P_j C,   x_j = x~_j + Q_j X.
// The rounding differs from one sequential pass only within the FP32
// increment.  The block pre-pass writes the block rows' right-hand sides into
// the field in place first, so every row reads its right-hand side there.

// Coefficients of one direction, one thread per line that crosses the
// interface, walking the line as the sequential sweep does (side of the
// regular rows from the line's start and after each block, factors from the
// prefix tables up to the first MIB row and per node from there on).
template <int D>
__global__ void __launch_bounds__(TPB) k_coef32(const __grid_constant__ Dev P) {
  const long long t = (long long)blockIdx.x * TPB + threadIdx.x;
  if (t >= nlines<D>(P)) return;
  Line L;
  decode_line<D>(P, t, L);
  if (L.boundary) return;
  const int bfirst = P.bstart[D][L.lid], bend = P.bstart[D][L.lid + 1];
  if (bfirst == bend) return;  // no crossing: the line reads the row tables
  const int n = L.n;
  const long long s = L.s;
  const int ls = P.lside[D][L.lid];
  const MibBlock* const blk = P.blk[D];
  const int L1 = blk[bfirst].L;
  const double* const pt = P.ptab[D][(ls >> 1) & 1];
  int b = bfirst;
  int side = (ls >> 1) & 1;
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
    P.cib[D][g] = (float)(1.0 / bet);
    P.cp[D][g] = (float)(-(a / bet));
    P.cq[D][g] = (float)(-gn);
  }
}

// Row tables of the lines without crossings: [side][ib, p, q][row], from the
// prefix tables of that side.
template <int D>
__global__ void __launch_bounds__(TPB) k_ctab32(const __grid_constant__ Dev P) {
  const int n = D == 0 ? P.nx : D == 1 ? P.ny : P.nz;
  const int i = blockIdx.x * TPB + threadIdx.x;
  if (i >= 2 * n) return;
  const int side = i / n, j = i % n;
  const double* const pt = P.ptab[D][side];
  const double bet = pt[2 * j];
  const double a = j == 0 || j == n - 1 ? 0.0 : P.ia[D][side];
  const double gn = j == n - 1 ? 0.0 : pt[2 * (j + 1) + 1];
  float* const T = P.ctab[D] + (size_t)side * 3 * n;
  T[j] = (float)(1.0 / bet);
  T[n + j] = (float)(-(a / bet));
  T[2 * n + j] = (float)(-gn);
}

constexpr int WL_WARPS = 8;

template <int MX>
constexpr size_t xline_smem() {
  // row tables 2 x 3 x R, then per warp r, ib, p, q (R each) + 4 floats
  return sizeof(float) * ((size_t)6 * 32 * MX + (size_t)WL_WARPS * (4 * 32 * MX + 4));
}

// A warp solves one line held in shared memory: rows sr[j] (right-hand side
// in, solution out) with 1/bet, p, q in si, sp, sq (by row).  Lane l runs
// rows [l MX, l MX + MX) (MX odd: the lanes' stride falls on distinct
// banks); the segment carries are warp scans (shuffles) of the affine end
// maps.
template <int MX>
__device__ __forceinline__ void solve_line32(float* sr, const float* si, const float* sp, const float* sq, int n,
                                             int l) {
  constexpr unsigned FULL = 0xffffffffu;
  const int jb = l * MX;
  float d[MX], pm[MX];
  float dl = 0.0f, pl = 1.0f;
#pragma unroll
  for (int k = 0; k < MX; k++) {
    const int j = jb + k;
    if (j < n) {
      const float p = sp[j];
      dl = __fmaf_rn(p, dl, __fmul_rn(sr[j], si[j]));
      pl = __fmul_rn(pl, p);
      d[k] = dl;
      pm[k] = pl;
    }
  }
  // inclusive scan of the maps c -> pl c + dl over the lanes; the carry into
  // lane l is the composition over lanes < l applied to 0 (lane 0 starts at
  // face row 0, whose p = 0)
  float A = pl, B = dl;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const float Ap = __shfl_up_sync(FULL, A, off), Bp = __shfl_up_sync(FULL, B, off);
    if (l >= off) {
      B = __fmaf_rn(A, Bp, B);
      A = __fmul_rn(A, Ap);
    }
  }
  float C = __shfl_up_sync(FULL, B, 1);
  if (l == 0) C = 0.0f;
  float xl = 0.0f, ql = 1.0f;
#pragma unroll
  for (int k = MX - 1; k >= 0; k--) {
    const int j = jb + k;
    if (j < n) {
      const float q = sq[j];
      xl = __fmaf_rn(q, xl, __fmaf_rn(pm[k], C, d[k]));
      ql = __fmul_rn(ql, q);
      d[k] = xl;
      pm[k] = ql;
    }
  }
  // suffix scan of the maps X -> ql X + xl (the last row's q = 0)
  A = ql;
  B = xl;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const float Ap = __shfl_down_sync(FULL, A, off), Bp = __shfl_down_sync(FULL, B, off);
    if (l + off < 32) {
      B = __fmaf_rn(A, Bp, B);
      A = __fmul_rn(A, Ap);
    }
  }
  float X = __shfl_down_sync(FULL, B, 1);
  if (l == 31) X = 0.0f;
#pragma unroll
  for (int k = 0; k < MX; k++) {
    const int j = jb + k;
    if (j < n) sr[j] = __fmaf_rn(pm[k], X, d[k]);
  }
}

// Row tables into shared memory: [side][ib, p, q][R].
__device__ __forceinline__ void load_row_tables(float* tab, const float* ctab, int n, int R) {
  for (int i = threadIdx.x; i < 6 * n; i += blockDim.x) tab[(i / n) * R + i % n] = ctab[i];
}

// x lines: contiguous in memory, so a warp copies its own line in and out.
template <int MX>
__device__ __forceinline__ void xline32_body(const Dev& P, unsigned cta_, unsigned ncta_, float* __restrict__ f) {
  static_assert(MX & 1, "odd rows per lane");
  constexpr int R = 32 * MX;
  constexpr int LS = 4 * R + 4;
  extern __shared__ float sw[];
  const int n = P.nx;
  float* const tab = sw;  // [side][ib, p, q][R]
  load_row_tables(tab, P.ctab[0], n, R);
  __syncthreads();
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  float* const sr = sw + 6 * R + w * LS;
  const long long nl = nlines<0>(P);
  const float* __restrict__ cib = P.cib[0];
  const float* __restrict__ cpp = P.cp[0];
  const float* __restrict__ cqq = P.cq[0];
  for (long long t = (long long)cta_ * WL_WARPS + w; t < nl; t += (long long)ncta_ * WL_WARPS) {
    Line L;
    decode_line<0>(P, t, L);
    if (L.boundary) continue;  // face line: its right-hand side is its solution (warp-uniform)
    const bool cross = P.bstart[0][L.lid + 1] > P.bstart[0][L.lid];
    const int side0 = (P.lside[0][L.lid] >> 1) & 1;
    __syncwarp();  // the previous line's stores have read the rows
#pragma unroll
    for (int k = 0; k < MX; k++) {
      const int j = l + 32 * k;
      if (j < n) {
        const long long g = L.base + j;
        cp_async4(sr + j, f + g);
        if (cross) {
          cp_async4(sr + R + j, cib + g);
          cp_async4(sr + 2 * R + j, cpp + g);
          cp_async4(sr + 3 * R + j, cqq + g);
        }
      }
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncwarp();
    const float* const si = cross ? sr + R : tab + side0 * 3 * R;
    solve_line32<MX>(sr, si, si + R, si + 2 * R, n, l);
    __syncwarp();
#pragma unroll
    for (int k = 0; k < MX; k++) {
      const int j = l + 32 * k;
      if (j < n) f[L.base + j] = sr[j];
    }
  }
}

template <int MX>
__global__ void __launch_bounds__(32 * WL_WARPS) k_xline32(const __grid_constant__ Dev P, float* __restrict__ f) {
  xline32_body<MX>(P, blockIdx.x, gridDim.x, f);
}

// y and z lines: strided, so the CTA copies NL neighbouring lines together,
// NL neighbours (4 NL bytes) of a row at a time, and warp w solves line w:
// NL = 16 for y, 8 for z with the accumulation (whose FP64 state rows would
// leave room for only one CTA of 16 per SM).  (8 for the y lines of more than
// 288 rows too, for more CTAs per SM, measured slower at 385^3.)  (A
// second buffer, to copy the next 8 lines in while these are solved, was
// measured slower: it halves the CTAs an SM holds, and they already overlap
// one another's copies.)
// ACC (z): the FP64 state is copied in with the right-hand side and the
// increment is added to it instead of being stored, face lines included, so
// that u^{n+1} = u^n + d at every node.
template <bool ACC, int MX>
__host__ __device__ constexpr int yz_lines() { return ACC ? 8 : 16; }
// Padding of a line's rows so that a copy instruction's lanes (NL lines x
// 32/NL rows) fall on distinct banks: 32/NL floats per line of (r, ib, p, q)
// (line c starts at bank 32 c / NL), and 16/NL doubles per line of the FP64
// state (a half warp's 8-byte accesses: NL lines x 16/NL rows).
template <int NL>
__host__ __device__ constexpr int yz_pad() { return 32 / NL; }
template <int NL>
__host__ __device__ constexpr int yz_upad() { return 16 / NL; }

template <int MX, bool ACC>
constexpr size_t yzline_smem() {
  // row tables 2 x 3 x R; NL lines x (r, ib, p, q: R each + padding); ACC:
  // NL lines x (R + padding) doubles
  constexpr int NL = yz_lines<ACC, MX>();
  return sizeof(float) * ((size_t)6 * 32 * MX + (size_t)NL * (4 * 32 * MX + yz_pad<NL>())) +
         (ACC ? sizeof(double) * NL * (32 * MX + yz_upad<NL>()) : 0);
}

template <int D, int MX, bool ACC>
__device__ __forceinline__ void yzline32_body(const Dev& P, unsigned cta_, unsigned ncta_, float* __restrict__ f,
                                              double* __restrict__ u) {
  static_assert(MX & 1, "odd rows per lane");
  static_assert(D != 0 && (!ACC || D == 2), "y and z lines; accumulation after the z solve");
  constexpr int R = 32 * MX;
  constexpr int NL = yz_lines<ACC, MX>();
  constexpr int LS = 4 * R + yz_pad<NL>();
  constexpr int US = R + yz_upad<NL>();
  extern __shared__ float sw[];
  const int n = D == 1 ? P.ny : P.nz;
  float* const tab = sw;
  load_row_tables(tab, P.ctab[D], n, R);
  float* const buf0 = sw + 6 * R;  // [NL][LS]
  // (the float offset 6 R + NL LS = (6 + 4 NL) R + 32 is even: 8-byte aligned)
  double* const ubuf0 = reinterpret_cast<double*>(buf0 + NL * LS);  // [NL][US]
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  // this thread's share of a copy: line c, rows jc + 32 m
  const int c = threadIdx.x & (NL - 1), jc = threadIdx.x / NL;
  const long long nl = nlines<D>(P);
  const long long stride = (long long)ncta_ * NL;
  const float* __restrict__ cib = P.cib[D];
  const float* __restrict__ cpp = P.cp[D];
  const float* __restrict__ cqq = P.cq[D];

  // line c of the tile at t0: where it is and what to copy
  struct Copy {
    long long g0, s32;  // row jc of the line, 32 rows
    bool st, cross;
  };
  auto copy_in = [&](long long t0) -> Copy {
    Copy cp{0, 0, false, false};
    const long long tc = t0 + c;
    if (tc < nl) {
      Line Lc;
      decode_line<D>(P, tc, Lc);
      cp.st = !Lc.boundary || ACC;  // (ACC) face lines pass their right-hand side through
      cp.cross = !Lc.boundary && P.bstart[D][Lc.lid + 1] > P.bstart[D][Lc.lid];
      cp.g0 = Lc.base + (long long)jc * Lc.s;
      cp.s32 = 32 * Lc.s;
    }
    float* const cr = buf0 + c * LS;
    double* const cu = ubuf0 + c * US;
    if (cp.st) {
#pragma unroll
      for (int m = 0; m < MX; m++) {
        const int j = jc + 32 * m;
        if (j < n) {
          const long long g = cp.g0 + m * cp.s32;
          cp_async4(cr + j, f + g);
          if (ACC) cp_async8(cu + j, u + g);
          if (cp.cross) {
            cp_async4(cr + R + j, cib + g);
            cp_async4(cr + 2 * R + j, cpp + g);
            cp_async4(cr + 3 * R + j, cqq + g);
          }
        }
      }
    }
    cp_async_commit();
    return cp;
  };

  for (long long t0 = (long long)cta_ * NL; t0 < nl; t0 += stride) {
    // a thread copies into exactly the rows it stored from last time: no
    // barrier needed before the copy
    const Copy cur = copy_in(t0);
    cp_async_wait<0>();
    __syncthreads();  // every thread's copies are in
    // warp w: line t0 + w
    const long long t = t0 + w;
    if (t < nl) {
      Line L;
      decode_line<D>(P, t, L);
      if (!L.boundary) {
        const bool cross = P.bstart[D][L.lid + 1] > P.bstart[D][L.lid];
        const int side0 = (P.lside[D][L.lid] >> 1) & 1;
        float* const sr = buf0 + w * LS;
        const float* const si = cross ? sr + R : tab + side0 * 3 * R;
        solve_line32<MX>(sr, si, si + R, si + 2 * R, n, l);
      }
    }
    __syncthreads();
    if (cur.st) {
      const float* const cr = buf0 + c * LS;
      const double* const cu = ubuf0 + c * US;
#pragma unroll
      for (int m = 0; m < MX; m++) {
        const int j = jc + 32 * m;
        if (j < n) {
          const long long g = cur.g0 + m * cur.s32;
          if (ACC)
            u[g] = cu[j] + (double)cr[j];
          else
            f[g] = cr[j];
        }
      }
    }
  }
}

template <int D, int MX, bool ACC>
__global__ void __launch_bounds__(32 * yz_lines<ACC, MX>()) k_yzline32(const __grid_constant__ Dev P, float* __restrict__ f,
                                                          double* __restrict__ u) {
  yzline32_body<D, MX, ACC>(P, blockIdx.x, gridDim.x, f, u);
}

// u^{n+1} = u^n + d, four nodes per thread
__global__ void __launch_bounds__(256) k_accumulate(double* __restrict__ u, const float* __restrict__ d, long long n) {
  const long long stride = (long long)gridDim.x * 256;
  for (long long i = (long long)blockIdx.x * 256 + threadIdx.x; i < n; i += 4 * stride) {
    double a[4];
    float b[4];
#pragma unroll
    for (int k = 0; k < 4; k++)
      if (i + k * stride < n) {
        a[k] = u[i + k * stride];
        b[k] = d[i + k * stride];
      }
#pragma unroll
    for (int k = 0; k < 4; k++)
      if (i + k * stride < n) u[i + k * stride] = a[k] + (double)b[k];
  }
}

// Longest line of the segmented solves: 32 lanes of 17 rows.
constexpr int kSegMaxRows = 32 * 17;

// Shape of the FP32 ring sweeps (rows per chunk, ring chunks, threads per
// CTA), for lines longer than that: 448 threads on each of the 148 SMs
// cover the 66,049 lines of a 257^3 grid in one wave.
constexpr int S32_CH = 8, S32_NS = 4, S32_NT = 448;

template <int D, int MX>
void launch_wline(const Dev& P, float* f, double* u, cudaStream_t st) {
  const long long need = (nlines<D>(P) + WL_WARPS - 1) / WL_WARPS;
  if (D == 0) {
    constexpr size_t smem = xline_smem<MX>();
    const int per_sm = (int)std::max<size_t>(1, std::min<size_t>(8, 232448 / (smem + 1024)));
    const unsigned grid = (unsigned)std::min<long long>(need, (long long)P.sweep_blocks * per_sm);
    k_xline32<MX><<<grid, 32 * WL_WARPS, smem, st>>>(P, f);
    return;
  }
  const bool acc = D == 2 && u;
  const size_t smem = acc ? yzline_smem<MX, true>() : yzline_smem<MX, false>();
  const int per_sm = (int)std::max<size_t>(1, std::min<size_t>(8, 232448 / (smem + 1024)));
  const int nl_cta = acc ? yz_lines<true, MX>() : yz_lines<false, MX>();
  const long long tiles = (nlines<D>(P) + nl_cta - 1) / nl_cta;
  const unsigned grid = (unsigned)std::min<long long>(tiles, (long long)P.sweep_blocks * per_sm);
  if (acc)
    k_yzline32<2, MX, true><<<grid, 32 * nl_cta, smem, st>>>(P, f, u);
  else
    k_yzline32<D == 0 ? 1 : D, MX, false><<<grid, 32 * nl_cta, smem, st>>>(P, f, nullptr);
}

template <int D>
void launch_wline_n(const Dev& P, float* f, double* u, cudaStream_t st) {
  const int nd = D == 0 ? P.nx : D == 1 ? P.ny : P.nz;
  if (nd <= 32 * 3)
    launch_wline<D, 3>(P, f, u, st);
  else if (nd <= 32 * 5)
    launch_wline<D, 5>(P, f, u, st);
  else if (nd <= 32 * 9)
    launch_wline<D, 9>(P, f, u, st);
  else if (nd <= 32 * 13)
    launch_wline<D, 13>(P, f, u, st);
  else
    launch_wline<D, 17>(P, f, u, st);
}

// ---------------------------------------------------------------------------
// The mixed step inside multi-problem launches: one item per CTA (its
// problem, its CTA index in that problem's own launch, that launch's CTA
// count); the CTA runs the same body as the problem's own launch, so a
// problem computes the same bits alone or in a batch.  The step's time
// factors come from the step table (step_e).

__global__ void __launch_bounds__(TPB, 8) kbm_adi_resid(const Dev* __restrict__ Ps,
                                                        const BatchItem* __restrict__ items) {
  BATCH_PROLOGUE
  adi_resid_body<2>(P, w.cta, w.ncta, P.u0, P.r32, 0.0);
}

__global__ void __launch_bounds__(TPB) kbm_adi_resid_mib(const Dev* __restrict__ Ps,
                                                         const BatchItem* __restrict__ items) {
  BATCH_PROLOGUE
  adi_resid_mib_body(P, w.cta, P.u0, P.r32, 0.0);
}

template <int D>
__global__ void __launch_bounds__(TPB) kbm_block_rhs32(const Dev* __restrict__ Ps,
                                                       const BatchItem* __restrict__ items) {
  BATCH_PROLOGUE
  block_rhs32_body<D, true>(P, w.cta, P.r32, P.nblk[D]);
}

template <int MX>
__global__ void __launch_bounds__(32 * WL_WARPS) kbm_xline32(const Dev* __restrict__ Ps,
                                                             const BatchItem* __restrict__ items) {
  BATCH_PROLOGUE
  xline32_body<MX>(P, w.cta, w.ncta, P.r32);
}

template <int D, int MX, bool ACC>
__global__ void __launch_bounds__(32 * yz_lines<ACC, MX>()) kbm_yzline32(const Dev* __restrict__ Ps,
                                                                      const BatchItem* __restrict__ items) {
  BATCH_PROLOGUE
  yzline32_body<D, MX, ACC>(P, w.cta, w.ncta, P.r32, ACC ? P.u0 : nullptr);
}

// rows per lane of the batched classes
constexpr int kBatchMX[2] = {3, 5};

template <int D, int MX>
void launch_batch_lines(const BatchItem* items, int n, const Dev* Ps, cudaStream_t st) {
  if (n <= 0) return;
  if (D == 0)
    kbm_xline32<MX><<<n, 32 * WL_WARPS, xline_smem<MX>(), st>>>(Ps, items);
  else if (D == 1)
    kbm_yzline32<1, MX, false><<<n, 32 * yz_lines<false, MX>(), yzline_smem<MX, false>(), st>>>(Ps, items);
  else
    kbm_yzline32<2, MX, true><<<n, 32 * yz_lines<true, MX>(), yzline_smem<MX, true>(), st>>>(Ps, items);
}

template <int D>
int launch_batch_dir(const MixedBatchPlan& b, cudaStream_t st) {
  int launches = 0;
  if (b.nblk[D] > 0) {
    kbm_block_rhs32<D><<<b.nblk[D], TPB, 0, st>>>(b.Ps, b.blk[D]);
    launches++;
  }
  launch_batch_lines<D, kBatchMX[0]>(b.line[D][0], b.nline[D][0], b.Ps, st);
  launch_batch_lines<D, kBatchMX[1]>(b.line[D][1], b.nline[D][1], b.Ps, st);
  return launches + (b.nline[D][0] > 0) + (b.nline[D][1] > 0);
}

template <int D>
void sweep32(const Dev& P, float* f, double* u, cudaStream_t st) {
  const int nd = D == 0 ? P.nx : D == 1 ? P.ny : P.nz;
  const bool seg = P.cib[D] != nullptr;  // coefficients built: the lines fit the segmented solves
  if (P.nblk[D] > 0) {
    if (seg)
      k_block_rhs32<D, true><<<(P.nblk[D] + TPB - 1) / TPB, TPB, 0, st>>>(P, f, P.nblk[D]);
    else
      k_block_rhs32<D, false><<<(P.nblk[D] + TPB - 1) / TPB, TPB, 0, st>>>(P, f, P.nblk[D]);
  }
  if (seg) {
    launch_wline_n<D>(P, f, u, st);
    return;
  }
  k_sweep32<D, S32_CH, S32_NS, S32_NT>
      <<<sweep_grid(P, nlines<D>(P), S32_NT), S32_NT, shape32_smem<S32_CH, S32_NS, S32_NT>(nd), st>>>(P, f);
  if (D == 2 && u) {
    const long long nn = P.nn;
    k_accumulate<<<4 * P.sweep_blocks * 4, 256, 0, st>>>(u, f, nn);
  }
}

}  // namespace

template <int MX>
void allow_smem() {
  cudaFuncSetAttribute(k_xline32<MX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)xline_smem<MX>());
  cudaFuncSetAttribute(k_yzline32<1, MX, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)yzline_smem<MX, false>());
  cudaFuncSetAttribute(k_yzline32<2, MX, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)yzline_smem<MX, false>());
  cudaFuncSetAttribute(k_yzline32<2, MX, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)yzline_smem<MX, true>());
}

void configure_mixed_kernels() {
  constexpr int smem = 232448;
  cudaFuncSetAttribute(k_sweep32<0, S32_CH, S32_NS, S32_NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  cudaFuncSetAttribute(k_sweep32<1, S32_CH, S32_NS, S32_NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  cudaFuncSetAttribute(k_sweep32<2, S32_CH, S32_NS, S32_NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  allow_smem<3>();
  allow_smem<5>();
  allow_smem<9>();
  allow_smem<13>();
  allow_smem<17>();
}

int mixed_sweep_threads() { return S32_NT; }

bool mixed_shape_fits(int nmax) { return shape32_smem<S32_CH, S32_NS, S32_NT>(nmax) <= (size_t)232448; }

bool mixed_segments_fit(int n) { return n <= kSegMaxRows; }

int build_mixed_coefs(const Dev& P, cudaStream_t st) {
  k_coef32<0><<<(unsigned)((nlines<0>(P) + TPB - 1) / TPB), TPB, 0, st>>>(P);
  k_coef32<1><<<(unsigned)((nlines<1>(P) + TPB - 1) / TPB), TPB, 0, st>>>(P);
  k_coef32<2><<<(unsigned)((nlines<2>(P) + TPB - 1) / TPB), TPB, 0, st>>>(P);
  k_ctab32<0><<<(2 * P.nx + TPB - 1) / TPB, TPB, 0, st>>>(P);
  k_ctab32<1><<<(2 * P.ny + TPB - 1) / TPB, TPB, 0, st>>>(P);
  k_ctab32<2><<<(2 * P.nz + TPB - 1) / TPB, TPB, 0, st>>>(P);
  return 6;
}

int mixed_batch_class(const Dev& P, int d) {
  if (!P.cib[0] || !P.cib[1] || !P.cib[2]) return -1;  // no segmented coefficients
  const int nd = d == 0 ? P.nx : d == 1 ? P.ny : P.nz;
  for (int c = 0; c < 2; c++)
    if (nd <= 32 * kBatchMX[c]) return c;
  return -1;
}

unsigned mixed_line_ctas(const Dev& P, int d) {
  const int c = mixed_batch_class(P, d);
  const int mx = c >= 0 ? kBatchMX[c] : kBatchMX[1];
  if (d == 0) return (unsigned)((nlines<0>(P) + WL_WARPS - 1) / WL_WARPS);
  const int nl = d == 2 ? (mx == 3 ? yz_lines<true, 3>() : yz_lines<true, 5>())
                        : (mx == 3 ? yz_lines<false, 3>() : yz_lines<false, 5>());
  return (unsigned)(((d == 1 ? nlines<1>(P) : nlines<2>(P)) + nl - 1) / nl);
}

void configure_mixed_batch_kernels() {
  cudaFuncSetAttribute(kbm_xline32<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)xline_smem<3>());
  cudaFuncSetAttribute(kbm_xline32<5>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)xline_smem<5>());
  cudaFuncSetAttribute(kbm_yzline32<1, 3, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)yzline_smem<3, false>());
  cudaFuncSetAttribute(kbm_yzline32<1, 5, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)yzline_smem<5, false>());
  cudaFuncSetAttribute(kbm_yzline32<2, 3, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)yzline_smem<3, true>());
  cudaFuncSetAttribute(kbm_yzline32<2, 5, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)yzline_smem<5, true>());
}

int launch_step_batch_mixed(const MixedBatchPlan& b, cudaStream_t st) {
  int launches = launch_batch_jumps(b.Ps, b.jumps, b.njumps, st);
  if (b.nmib > 0) {
    kbm_adi_resid_mib<<<b.nmib, TPB, 0, st>>>(b.Ps, b.mib);
    launches++;
  }
  kbm_adi_resid<<<b.nrows, TPB, 0, st>>>(b.Ps, b.rows);
  launches++;
  launches += launch_batch_dir<0>(b, st);
  launches += launch_batch_dir<1>(b, st);
  launches += launch_batch_dir<2>(b, st);
  return launches + launch_batch_tick(b.Ps, b.n, st);
}

int launch_step_mixed(const Dev& P, const StepTimes& T, double* u, cudaStream_t st, cudaEvent_t* ev,
                      const SideStream* side) {
  int launches = 0;
  // The jumps and the residual's MIB rows (which read the jumps) run on the
  // side stream, beside the pointwise residual: the two passes write
  // disjoint nodes and read only the state.
  const bool fork = side && side->stream && (P.ncross > 0 || P.nmibnode > 0);
  cudaStream_t sst = fork ? side->stream : st;
  if (fork) {
    cudaEventRecord(side->fork, st);
    cudaStreamWaitEvent(sst, side->fork, 0);
  }
  if (ev) cudaEventRecord(ev[0], sst);
  if (P.ncross > 0) {
    launch_jumps(P, T.e_next, sst);
    launches++;
  }
  if (ev) cudaEventRecord(ev[1], sst);
  if (ev) cudaEventRecord(ev[2], st);
  if (P.nmibnode > 0) {
    k_adi_resid_mib<<<(P.nmibnode + TPB - 1) / TPB, TPB, 0, sst>>>(P, u, P.r32, T.e_next);
    launches++;
  }
  k_adi_resid<2><<<pointwise_rows_grid(P), TPB, 0, st>>>(P, u, P.r32, T.e_next);
  launches++;
  if (fork) {
    cudaEventRecord(side->join, sst);
    cudaStreamWaitEvent(st, side->join, 0);
  }
  if (ev) cudaEventRecord(ev[3], st);
  int slot = 2;
  auto mark = [&](int k) {
    if (ev) cudaEventRecord(ev[2 * slot + k], st);
    if (k == 1) slot++;
  };
  mark(0);
  sweep32<0>(P, P.r32, nullptr, st);
  mark(1);
  mark(0);
  sweep32<1>(P, P.r32, nullptr, st);
  mark(1);
  mark(0);
  sweep32<2>(P, P.r32, u, st);
  mark(1);
  launches += P.cib[2] ? 3 : 4;
  for (int d = 0; d < 3; d++) launches += P.nblk[d] > 0;
  return launches;
}

}  // namespace mts

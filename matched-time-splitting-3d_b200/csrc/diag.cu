// The error reports on the device.
//
// Fictitious points: Refresh_Fp
// (src/spatial/intersection.cc:1841-2281) evaluates, for every crossing, the
// MIB fictitious values that its weights give from the exact solution and
// the exact jumps, and their relative error against the exact solution of
// the other side at those nodes; Error_Fp (:4667-4771) reports their maximum
// and root mean square.
//
// One thread per single crossing or corner pair computes its two (pair:
// four) relative errors with the reference's operations in its order
// (compiled without FMA contraction): the same bits.  The host adds them up
// in Error_Fp's loop order (directions z, y, x; lines in loop order;
// crossings by position), so the maximum and the root mean square are the
// reference's bits too.
//
// Jumps: Refresh_Jump (:2294-2490) compares, per crossing, the u_dir it hands
// the solvers with the exact flux jump along the crossing's line; Error_Jump
// (:4594-4662) reports their maximum and root mean square, added up on the
// host in the same order.
#include <cuda_runtime.h>

#include "../../include/mts.h"
#include "device.h"
#include "device_common.cuh"

namespace mts {
namespace {

// Node (ix, iy, iz) of row j of the line (d, i1, i2): x lines are indexed
// (iy, iz), y lines (ix, iz), z lines (ix, iy).
__device__ __forceinline__ void line_node(int d, int i1, int i2, int j, int& ix, int& iy, int& iz) {
  ix = d == 0 ? j : i1;
  iy = d == 0 ? i1 : d == 1 ? j : i2;
  iz = d == 2 ? j : i2;
}

struct FpLine {
  const Dev& P;
  double E;
  int d, i1, i2;
  // the exact solution at row j on the node's own side (inv = false) or on
  // the other side (inv = true), Refresh_Fp's u and invu
  __device__ double u(int j, bool inv) const {
    int ix, iy, iz;
    line_node(d, i1, i2, j, ix, iy, iz);
    const long long m = (long long)ix + (long long)P.nx * ((long long)iy + (long long)P.ny * iz);
    const bool out = (P.tag[m] & TAG_OUT) != 0;
    return (out != inv) ? outer_u(P, E, ix, iy, iz) : inner_u(P, E, ix, iy, iz);
  }
  // Jump_u and Jump_betau along the line at crossing c (Equation::Jump_u,
  // the Eq's Jump_betau_x/y/z)
  __device__ void jumps(int c, double& ju, double& jb) const {
    double b[3];
    exact_jumps(P, P.cc[c], E, ju, b);
    jb = b[d];
  }
};

// role: 0 a single crossing, 1 the left crossing of a corner pair (the right
// one follows it), 2 the right one (done by the left one's thread).
// cr: the records sorted by (direction, line, position); ci: each one's index
// in the handle's crossing list (its jump constants P.cc[ci]).
__global__ void __launch_bounds__(TPB) k_fp_errors(const __grid_constant__ Dev P, const mts_crossing* __restrict__ cr,
                                                   const int32_t* __restrict__ ci, const int8_t* __restrict__ role,
                                                   int n, double E, double* __restrict__ err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || role[i] == 2) return;
  const mts_crossing& c = cr[i];
  const FpLine L{P, E, c.dir, c.indx1, c.indx2};
  const int j0 = c.left_loc;
  if (role[i] == 0) {
    const int nw = c.nwei - 2, one = nw / 2;
    double ju, jb;
    L.jumps(ci[i], ju, jb);
    double suml = 0, sumr = 0;
    suml += c.weil[nw] * ju;
    suml += c.weil[nw + 1] * jb;
    sumr += c.weir[nw] * ju;
    sumr += c.weir[nw + 1] * jb;
    for (int j = 0; j < nw; j++) {
      const double u = L.u(j0 - one + 1 + j, false);
      suml += c.weil[j] * u;
      sumr += c.weir[j] * u;
    }
    const double vl = L.u(j0, true), vr = L.u(j0 + 1, true);
    err[2 * i] = fabs((vl - suml) / vl);
    err[2 * i + 1] = fabs((vr - sumr) / vr);
    return;
  }
  const mts_crossing& R = cr[i + 1];
  const int nw = c.nwei - 4;
  double jul, jbl, jur, jbr;
  L.jumps(ci[i], jul, jbl);
  L.jumps(ci[i + 1], jur, jbr);
  double lsl = 0, lsr = 0, rsr = 0;
  lsl += c.weil[nw] * jul;
  lsl += c.weil[nw + 1] * jbl;
  lsl += c.weil[nw + 2] * jur;
  lsl += c.weil[nw + 3] * jbr;
  lsr += c.weir[nw] * jul;
  lsr += c.weir[nw + 1] * jbl;
  lsr += c.weir[nw + 2] * jur;
  lsr += c.weir[nw + 3] * jbr;
  rsr += R.weir[nw] * jul;
  rsr += R.weir[nw + 1] * jbl;
  rsr += R.weir[nw + 2] * jur;
  rsr += R.weir[nw + 3] * jbr;
  for (int k = 0; k < nw; k++) {
    const double u = L.u(j0 - 1 + k, false);
    lsl += c.weil[k] * u;
    lsr += c.weir[k] * u;
    rsr += R.weir[k] * u;
  }
  const double v0 = L.u(j0, true), v1 = L.u(j0 + 1, true), v2 = L.u(j0 + 2, true);
  const double el = fabs((v0 - lsl) / v0), er = fabs((v1 - lsr) / v1);
  err[2 * i] = el;
  err[2 * i + 1] = er;
  err[2 * i + 2] = er;  // the right crossing's left error is the left one's right error
  err[2 * i + 3] = fabs((v2 - rsr) / v2);
}

// Refresh_Jump's check of the jump data (intersection.cc:2294-2490): per
// crossing, u_dir = (P^-1)[d][0] [beta u_xi] against the exact [beta u_d]
// along its line, |u_dir - [beta u_d]| / [beta u_d] (the divisor's sign kept,
// as there).  Thread i takes record i of the sorted list; ci maps it to the
// handle's jump constants.
__global__ void __launch_bounds__(TPB) k_jump_errors(const __grid_constant__ Dev P, const mts_crossing* __restrict__ cr,
                                                     const int32_t* __restrict__ ci, int n, double E,
                                                     double* __restrict__ err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const CrossConst q = P.cc[ci[i]];
  double ju, jb[3];
  exact_jumps(P, q, E, ju, jb);
  const double bxi = q.p[0] * jb[0] + q.p[1] * jb[1] + q.p[2] * jb[2];
  const double udir = q.pinv * bxi;
  const double jd = jb[cr[i].dir];
  err[i] = fabs(udir - jd) / jd;
}

}  // namespace

int launch_jump_errors(const Dev& P, const mts_crossing* cr, const int32_t* ci, int n, double E, double* err,
                       cudaStream_t st) {
  if (n <= 0) return 0;
  k_jump_errors<<<(n + TPB - 1) / TPB, TPB, 0, st>>>(P, cr, ci, n, E, err);
  return 1;
}

int launch_fp_errors(const Dev& P, const mts_crossing* cr, const int32_t* ci, const int8_t* role, int n, double E,
                     double* err, cudaStream_t st) {
  if (n <= 0) return 0;
  k_fp_errors<<<(n + TPB - 1) / TPB, TPB, 0, st>>>(P, cr, ci, role, n, E, err);
  return 1;
}

}  // namespace mts

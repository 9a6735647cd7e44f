/* Test infrastructure only (the checker, never the product): a plain-C CPU
 * restatement of the reference's time step for the Douglas-ADI, LOD-IE,
 * LOD-CN and trapezoidal-splitting (TS) methods with MIB-L1/L2 interface rows.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
 *
 * Fields are flat float64 arrays, x fastest: idx = ix + nx*(iy + ny*iz), the
 * order of Mesh::To1d (src/mesh/mesh.cc:93-99).
 *
 * Parity is pinned against the reference binary built from the reference
 * sources by oracle/Makefile (tests/test_oracle_pin.py): same grid, tags and
 * crossing list in, bit-identical solution out.
 */
#ifndef MTS_ORACLE_H
#define MTS_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int32_t nx, ny, nz;
  double xl, xr, yl, yr, zl, zr; /* domain bounds */
  double beta_in, beta_out;      /* piecewise-constant beta */
  int32_t eq;                    /* 0: reference Eq_0, 8: e^{-t} trig/quadratic */
  int32_t pad;
  double dt;
} mts_oracle_problem;

/* One crossing, field meanings of Intersection_Data (src/constant.h:141-156):
 * dir 0/1/2 = x/y/z; (indx1, indx2) = the line's two fixed indices in the
 * reference's order; id = ID (>0 irregular, <0 corner pair); left_loc;
 * nwei = length of the weil/weir rows; p = the 3x3 local frame (row major). */
typedef struct {
  int32_t dir, indx1, indx2, id, left_loc, nwei;
  double coord[3], gamma, normal[3], p[9], weil[9], weir[9];
} mts_oracle_crossing;

enum { MTS_ORACLE_ADI = 0, MTS_ORACLE_LOD_IE = 1, MTS_ORACLE_LOD_CN = 2, MTS_ORACLE_TS = 3 };

/* Fill u with the exact solution at time t by node tag (Initialization,
 * src/temporal/douglas_adi.cc:1684-1714). */
int mts_oracle_init(const mts_oracle_problem* p, const int8_t* tags, double t, double* u);

/* Advance u by `steps` steps of `method` from time t0, with the time loop of
 * src/helper.h:199-238 (t += dt before each step).  Returns 0 on success,
 * 1 on a zero pivot in the line solve, 2 on a malformed crossing list. */
int mts_oracle_run(const mts_oracle_problem* p, const int8_t* tags, const mts_oracle_crossing* cr,
                   int32_t ncr, int32_t method, double t0, int32_t steps, double* u);

/* L-infinity (with first argmax in [ix][iy][iz] loop order) and L2 error of u
 * against the exact solution at t (Error, src/temporal/douglas_adi.cc:1723-1770). */
int mts_oracle_norms(const mts_oracle_problem* p, const int8_t* tags, double t, const double* u,
                     double* lmax, double* l2, int32_t* argmax3);

#ifdef __cplusplus
}
#endif
#endif

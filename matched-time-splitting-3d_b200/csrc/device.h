// Device-resident problem layout shared by the C ABI (capi.cu) and the
// kernels (kernels.cu).
//
// HBM layout of one problem (N = nx*ny*nz nodes, x fastest):
//   u0, u1   float64[N]   solution ping-pong (state + stage results)
//   gam      float64[N]   Thomas forward factors c_{j-1}/bet of the sweep in
//                         flight (scratch, rewritten every sweep)
//   ydt      float64[N]   Douglas-ADI: dt*D_yy u^n of the x sweep, read back
//                         in that sweep's back substitution (scratch)
//   tag      uint8[N]     bit0 outside, bit1/2/3 node is a MIB row of an
//                         x/y/z crossing block
//   per axis: coordinates, sin 2x, cos 2x (exact-solution tables)
//   per direction: CSR offsets over grid lines -> MIB row blocks
//   per crossing: time-invariant constants of its jump data, and the
//                 per-step ([u], [beta u_d]) pair
#pragma once

#include <cstdint>

namespace mts {

enum : uint8_t { TAG_OUT = 1, TAG_MIBX = 2, TAG_MIBY = 4, TAG_MIBZ = 8 };

// One irregular crossing (2 rows: L, L+1) or one corner pair (3 rows: L..L+2)
// on a grid line.  w[0]/w[1] are weil/weir of the (left) crossing, w[2]/w[3]
// those of the right crossing of a corner pair (Intersection_Data::wei,
// src/constant.h:119-122).  ia/ib/ic are the implicit rows after the
// Convert2Tri_irr/_cor elimination (src/temporal/douglas_adi.cc:1554-1675),
// rate[] the elimination multipliers to replay on the right-hand side.
struct MibBlock {
  int32_t line;
  int32_t L;
  int32_t kind;  // 2 or 3 rows
  int32_t c0, c1;
  int32_t pad;
  double w[4][9];
  double ia[3], ib[3], ic[3];
  double rate[6];
};

// Time-invariant constants of one crossing's jump data for the exact
// solutions supported on the device.  For eq 8 the per-step values are
//   [u]       = R2*E - S*E
//   [beta u_d]= beta_out*((2 x_d)*E) - beta_in*(D_d*E)
//   u_dir     = pinv * (p0*[bu_x] + p1*[bu_y] + p2*[bu_z])
// with E = exp(-t), the operand order of the exact-solution code.
struct CrossConst {
  double x, y, z;
  double R2, S;
  double D[3];
  double p[3];
  double pinv;
};

struct Dev {
  int nx, ny, nz;
  int eq, method;
  int ncross;
  long long nn;
  double dt;
  double kex;   // explicit Crank-Nicolson factor coef*dt, coef = 0.5
  double cdt;   // implicit factor: dt (ADI, LOD-IE) or 0.5*dt (LOD-CN, TS)
  double hdt;   // 0.5*dt (TS source halves)
  double bi, bo, kin, c6bo;  // beta_in, beta_out, 12*beta_in-1, 6*beta_out
  double vd[3][2][3];        // [dir][side] 3-point weights beta/h^2, -(2beta)/h^2, beta/h^2
  double ia[3][2], ib[3][2], ic[3][2];  // regular implicit rows
  const double* ax[3];  // node coordinates per axis
  const double* s2[3];  // sin(2 x_i) per axis
  const double* c2[3];  // cos(2 x_i) per axis
  const uint8_t* tag;
  const int32_t* bstart[3];
  const MibBlock* blk[3];
  const CrossConst* cc;
  double2* jv;  // per crossing ([u], u_dir) of the current step
  double* gam;
  double* ydt;
  int* status;  // bit0: zero pivot in a line solve
};

// Per-step exact-solution time factors.
struct StepTimes {
  double e_prev, e_half, e_next;  // exp(-t_prev), exp(-t_half), exp(-t_next)
};

// Host-side launchers (kernels.cu).  All enqueue on `stream` and return the
// number of kernel launches made.
int launch_initialize(const Dev& P, double E, double* u, cudaStream_t stream);
// ev: null, or 2 events per kernel slot recorded around each launch.
int launch_step(const Dev& P, const StepTimes& T, double*& u0, double*& u1, cudaStream_t stream,
                cudaEvent_t* ev);
constexpr int kProfileSlots = 8;
int launch_norms(const Dev& P, double E, const double* u, double* partial, int nblocks,
                 double* out3, cudaStream_t stream);
int norms_blocks(const Dev& P);

}  // namespace mts

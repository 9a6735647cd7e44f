// Device-resident problem layout shared by the C ABI (capi.cu) and the
// kernels (kernels.cu).
//
// HBM layout of one problem (N = nx*ny*nz nodes, x fastest):
//   u0, u1   float64[N]   solution ping-pong (state + stage results)
//   tag      uint8[N]     bit0 outside, bit1/2/3 node is a MIB row of an
//                         x/y/z crossing block
//   dp       float64[nmax x T]  partial solutions d'_j of the T = grid
//                         threads' lines in flight, row-major [row][thread]
//                         so every access is coalesced whatever the sweep
//                         direction; reused line after line (L2-resident:
//                         ~25 MB at 257 nodes and 148 x 256 threads)
//   fbet, fgam float64[N] per direction that has crossings: Thomas factors
//                         of crossing lines from their first MIB row on
//   u0, u1, dp, fbet, fgam carry kRowPad rows of slack (an x-y plane per row
//                         for the node fields) past their end: the sweeps
//                         stage whole chunks of rows without bound checks
//   lside    uint8 per line and direction: bit0 node 0, bit1 node 1, bit2
//                         node n-1 outside (the side changes only at crossings)
//   per axis: coordinates, sin 2x, cos 2x (exact-solution tables)
//   per direction: CSR offsets over grid lines -> MIB row blocks
//   per crossing: time-invariant constants of its jump data, and the
//                 per-step ([u], [beta u_d]) pair
#pragma once

#include <cstdint>

#include "../../include/mts.h"

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
  int32_t sides;  // bit q: row L+q is outside
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
  const uint8_t* lside[3];
  const int32_t* bstart[3];
  const MibBlock* blk[3];
  const CrossConst* cc;
  double2* jv;  // per crossing ([u], u_dir) of the current step
  // Thomas factorisation of every line, computed once (the matrices do not
  // change between steps): bet_j = b_j - a_j*gam_j, gam_j = c_{j-1}/bet_{j-1}.
  // Up to its first MIB row a line's factors depend only on the side of its
  // row 1, so they come from the per-direction prefix tables
  // ptab[d][side][2*j + {0: bet, 1: gam}]; from the first MIB row on they are
  // stored per node in fbet[d] / fgam[d] (field layout, written only for
  // lines that cross the interface).
  const double* ptab[3][2];
  const double* fbet[3];
  const double* fgam[3];
  // Per block, for the sweep in flight: the right-hand sides of its rows after
  // the jump terms and the Convert2Tri row operations, [3*block + q]
  // (written by the block pre-pass, read by the sweep).
  double* rblk[3];
  int nblk[3];
  double* dp;        // [nmax][sweep threads of the launch]: forward results d'_j
  int sweep_blocks;  // one persistent CTA per SM
  int shape[3];      // sweep shape of the first, second and third sweep of a step
  // Mixed precision (Douglas-ADI): the step is solved for its increment
  // delta = u^{n+1} - u^n in FP32 (residual in FP64, state accumulated in
  // FP64).  Factors as 1/bet and gam in FP32, laid out like ptab/fbet/fgam.
  float* r32;                 // residual in, increment out [N + slack]
  float* dp32;                // [nmax + slack][sweep threads]
  const float* ptab32[3][2];  // [2*j + {0: 1/bet, 1: gam}]
  const float* fib32[3];      // per node 1/bet of crossing lines from L1
  const float* fgam32[3];
  float* rblk32[3];           // block rows' right-hand sides after Convert2Tri
  // Dense per-node coefficients of the segmented FP32 solves, built on the
  // device when the mixed form is switched on (null before, and for grids
  // whose lines are too long for them): for row j of a direction-d line,
  //   cib = 1/bet_j,  cp = -a_j/bet_j (forward multiplier, 0 on face rows),
  //   cq = -gam_{j+1} (backward multiplier, 0 on the last row).
  // They are filled only for lines that cross the interface; every other
  // interior line takes its row's values from ctab[d][side][{ib, p, q}][row]
  // by the side of its row 1.
  float* cib[3];
  float* cp[3];
  float* cq[3];
  float* ctab[3];
  int precision;              // 0 plain FP64, 1 mixed, 2 fast FP64
  // Fast FP64 form (segmented line solves, fast.cu), built when the form is
  // switched on.  Per direction: the row tables [side][1/bet, -a/bet by row
  // (32 MX each), then 2 x 5 x 32 lane-scan multipliers] of the lines
  // without crossings; per line a flag byte (bit0 the line
  // crosses the interface, bit1 the side of its row 1); the crossing lines'
  // ids in memory order (fcross, nfcross of them) and their own rows
  // [c][1/bet, -a/bet][32 MX]; per block the -gam_{j+1} of its rows.  Per
  // MIB node its block in x, y, z (-1: none); per x block the MIB node
  // index of each of its rows.
  const double* ftab[3];
  const uint8_t* fline[3];
  const int32_t* fcross[3];
  int nfcross[3];
  const double* fcoef[3];
  const double* fbq[3];
  const int4* mibref;
  // Replayable steps (batches captured in a CUDA graph): when tsched is set,
  // kernels take the step's exp(-t) factors from tsched[3*(*tstep) + {0: t_prev,
  // 1: t_half, 2: t_next}] instead of their arguments; k_tick advances tstep.
  const double* tsched;
  int* tstep;
  int tstop;   // batched launches skip the problem once *tstep reaches it
  double* u0;  // the state (every method keeps it here)
  double* u1;  // scratch field
  const long long* mibnode;  // nodes with a MIB flag (any direction), ascending
  int nmibnode;
  int* status;       // reserved
};

// Persistent line-sweep shapes (rows per staged chunk, ring depth, threads
// per CTA); all give bit-identical results, they differ only in speed.
int sweep_shape_count();
int sweep_shape_max_threads();
bool sweep_shape_fits(int shape, int nmax);  // shared memory of the shape within the limit
void configure_kernels();

// Per-step exact-solution time factors.
struct StepTimes {
  double e_prev, e_half, e_next;  // exp(-t_prev), exp(-t_half), exp(-t_next)
};

// Host-side launchers (kernels.cu).  All enqueue on `stream` and return the
// number of kernel launches made.
int launch_initialize(const Dev& P, double E, double* u, cudaStream_t stream);
// Per-node Thomas factors of the lines with MIB blocks (once, at setup);
// *zero_pivot is set on a zero pivot.
int launch_factor_lines(const Dev& P, int* zero_pivot, cudaStream_t stream);
// ev: null, or 2 events per kernel slot recorded around each launch.
// A second stream with its fork and join events (timing off), for work of a
// step that can run beside the main stream's.
struct SideStream {
  cudaStream_t stream;
  cudaEvent_t fork, join;
};
int launch_step(const Dev& P, const StepTimes& T, double*& u0, double*& u1, cudaStream_t stream,
                cudaEvent_t* ev, const SideStream* side = nullptr);
// The mixed-precision Douglas-ADI step (mixed.cu), in place on u.
int launch_step_mixed(const Dev& P, const StepTimes& T, double* u, cudaStream_t stream, cudaEvent_t* ev,
                      const SideStream* side);
void configure_mixed_kernels();
int mixed_sweep_threads();            // threads per CTA of the FP32 sweeps
bool mixed_shape_fits(int nmax);      // their shared memory within the limit
bool mixed_segments_fit(int n);       // the segmented solves take lines of n rows (else the ring sweeps run)
// Fills Dev::cib/cp/cq (allocated by the caller) from the FP64 factors.
int build_mixed_coefs(const Dev& P, cudaStream_t stream);
// The fast FP64 Douglas-ADI step (fast.cu): u holds u^n on entry and
// u^{n+1} on return, d is scratch.  ev: null, or 6 events recorded around
// the three launches.
int launch_step_fast(const Dev& P, const StepTimes& T, double* u, double* d, cudaStream_t stream, cudaEvent_t* ev,
                     const SideStream* side);
void configure_fast_kernels();
int fast_rows_per_lane(int n);               // MX of a direction with n rows (0: lines too long)
bool fast_fits(int nx, int ny, int nz);      // the form takes this grid
int build_fast_lines(const Dev& P, uint8_t* const fline[3], cudaStream_t stream);  // the line flags
int build_fast_tables(const Dev& P, cudaStream_t stream);  // fills ftab, fcoef, fbq, mibref (allocated by the caller)
// Batched plain steps (kernels.cu): problems of one method advance together,
// one launch per kernel of the step for all of them.  A launch's CTAs are
// listed as items (problem, the CTA's index in that problem's own grid, the
// size of that grid), so every problem sees exactly the grid its own launch
// would have; the problems' Dev records live in device memory.
struct BatchItem {
  int32_t p, cta, ncta, pad;
};
struct BatchPlan {
  int method;         // MTS_ADI .. MTS_TS, shared by all problems
  int n;              // problems
  int nmax;           // longest line over the problems
  const Dev* Ps;      // [n] device records (tsched/tstep set)
  const BatchItem* jumps;
  int njumps;
  const BatchItem* rows;  // pointwise passes over grid rows
  int nrows;
  const BatchItem* mib;   // MIB node list passes
  int nmib;
  const BatchItem* blk[3];  // block pre-pass per direction
  int nblk[3];
  const BatchItem* sw[3];   // line sweeps per direction
  int nsw[3];
};
// The mixed form's batched step (ADI, lines of at most 160 rows): the
// mixed kernels' bodies, one item per CTA (mixed.cu).  line[d][c]: the line
// solves of direction d for the problems of rows-per-lane class c (3, 5).
struct MixedBatchPlan {
  int n;
  const Dev* Ps;
  const BatchItem* jumps;
  int njumps;
  const BatchItem* rows;
  int nrows;
  const BatchItem* mib;
  int nmib;
  const BatchItem* blk[3];
  int nblk[3];
  const BatchItem* line[3][2];
  int nline[3][2];
};
int mixed_batch_class(const Dev& P, int d);          // -1: not batchable
unsigned mixed_line_ctas(const Dev& P, int d);      // CTAs of the line solves of direction d
int launch_step_batch_mixed(const MixedBatchPlan& plan, cudaStream_t stream);  // one step + tick
void configure_mixed_batch_kernels();
int launch_batch_jumps(const Dev* Ps, const BatchItem* items, int nitems, cudaStream_t stream);
int launch_batch_tick(const Dev* Ps, int n, cudaStream_t stream);
int batch_sweep_threads();                 // threads per CTA of the batched sweeps
void configure_batch_kernels();
int launch_step_batch(const BatchPlan& plan, cudaStream_t stream);  // one step + tick
unsigned jumps_grid(const Dev& P);
unsigned mib_grid(const Dev& P);
unsigned block_grid(const Dev& P, int d);
unsigned batch_sweep_grid(const Dev& P, int d);

// Shared by both step forms (kernels.cu).
void launch_jumps(const Dev& P, double E, cudaStream_t stream);
void launch_tick(const Dev& P, cudaStream_t stream);  // ++(*P.tstep)
unsigned pointwise_rows_grid(const Dev& P);
constexpr int kProfileSlots = 8;
constexpr int kRowPad = 16;  // rows of slack after each staged field (>= chunk rows)
// The fictitious points' relative errors (Refresh_Fp): two per crossing
// into err, for the records cr sorted by (direction, line, position) whose
// indices in the handle's list are ci; role[i] 0 single, 1 left of a corner
// pair, 2 its right (diag.cu).
int launch_fp_errors(const Dev& P, const mts_crossing* cr, const int32_t* ci, const int8_t* role, int n, double E,
                     double* err, cudaStream_t stream);
// The jumps' relative errors (Refresh_Jump's jump.err): one per record of
// the same sorted list into err (diag.cu).
int launch_jump_errors(const Dev& P, const mts_crossing* cr, const int32_t* ci, int n, double E, double* err,
                       cudaStream_t stream);

int launch_norms(const Dev& P, double E, const double* u, double* partial, int nblocks,
                 double* out3, cudaStream_t stream);
int norms_blocks(const Dev& P);

// Error norms through a statically sized module array instead of handle
// buffers (mts_norms_noalloc).  The array holds the ticket counter, the
// result triple and the partials of at most kNoAllocMaxBlocks blocks, i.e.
// grids of at most kNoAllocMaxBlocks * 2048 nodes (norms_blocks).
constexpr int kNoAllocMaxBlocks = 2048;
constexpr int kNoAllocScratchDoubles = 64 + 3 * kNoAllocMaxBlocks;  // 48.5 KiB
cudaError_t noalloc_scratch_address(double** p);  // call with the device current
int launch_norms_noalloc(const Dev& P, double E, const double* u, double* scratch, int nb, cudaStream_t stream);

}  // namespace mts

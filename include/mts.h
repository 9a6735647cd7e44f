/* Matched-TS on B200: C ABI of the GPU time-stepping path.
 *
 * One handle = one parabolic interface problem resident on one GPU: grid,
 * node tags, the MIB crossing list with its fictitious-point weights, the
 * time-invariant line-solve coefficients and the solution field stay in
 * device memory for all time steps; per step only the time crosses the bus.
 *
 * Fields are float64, x fastest: index = ix + nx*(iy + ny*iz), the order of
 * Mesh::To1d in the reference (src/mesh/mesh.cc:93-99).  Every function
 * returns an mts_status; no function exits or throws.  Functions on one
 * handle are not thread-safe; distinct handles are independent (one CUDA
 * stream each).
 *
 * A handle lives on the CUDA device that was current when it was created.
 * Call the functions that take it with that device current (the usual one
 * process per GPU does so by construction); a batch takes handles of one
 * device.
 */
#ifndef MTS_H
#define MTS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  MTS_OK = 0,
  MTS_ERR_ARG = 1,           /* bad argument or unsupported option */
  MTS_ERR_SETUP = 2,         /* reference setup abort: interface on a grid node,
                                coherent corners, open surface, singular LU */
  MTS_ERR_ZERO_PIVOT = 3,    /* zero pivot in a line solve (TDMA "tridag" throw) */
  MTS_ERR_NONFINITE = 4,     /* root finding failed to bracket / converge */
  MTS_ERR_CUDA = 5,          /* CUDA runtime error (see mts_last_error) */
  MTS_ERR_NO_DEVICE = 6,     /* no CUDA device visible */
  MTS_ERR_OOM = 7            /* device allocation failed */
} mts_status;

typedef enum { MTS_ADI = 0, MTS_LOD_IE = 1, MTS_LOD_CN = 2, MTS_TS = 3 } mts_method;
typedef enum { MTS_SURFACE_ELLIPSOID = 0, MTS_SURFACE_TORUS = 1 } mts_surface_kind;

/* Uniform grid on [xl,xr]x[yl,yr]x[zl,zr] with nx*ny*nz nodes (Mesh ctor,
 * src/mesh/mesh.h:20). */
typedef struct {
  int32_t nx, ny, nz;
  int32_t pad;
  double xl, xr, yl, yr, zl, zr;
} mts_grid;

/* Level set.  Ellipsoid: params = {a, b, c, r, cx, cy, cz} for
 * (x-cx)^2/a^2 + (y-cy)^2/b^2 + (z-cz)^2/c^2 - r^2 (Surface_Ellipsoid,
 * src/surface/surface_ellipsoid.h with a centre); torus: params = {R, r} for
 * (R - sqrt(x^2+y^2))^2 + z^2 - r^2 (Surface_Torus, src/surface/surface_torus.h). */
typedef struct {
  int32_t kind;
  int32_t pad;
  double params[7];
} mts_surface;

/* Where mts_create builds the tags, crossings and MIB weights. */
typedef enum { MTS_SETUP_HOST = 0, MTS_SETUP_DEVICE = 1 } mts_setup_where;

/* Problem parameters.  beta is piecewise constant (beta_in inside, beta_out
 * outside).  eq selects the exact solution that supplies source, boundary and
 * jump data: 0 = the reference's Eq_0 (src/equation/eq_0.cc), 8 = inside
 * e^{-t} sin2x cos2y sin2z / outside e^{-t}(x^2+y^2+z^2).  mib is 1 (MIB-L1)
 * or 2 (MIB-L2) as in Intersections(..., mib_method, ...).  setup
 * (mts_setup_where) selects the host threads (0, the default) or the device
 * (1) for mts_create's setup; see mts_setup_device. */
typedef struct {
  double beta_in, beta_out;
  int32_t eq;
  int32_t method; /* mts_method */
  int32_t mib;
  int32_t setup;  /* mts_setup_where */
  double dt;
  double t0;
} mts_params;

/* One interface crossing, field by field the reference's Intersection_Data
 * (src/constant.h:141-156): dir 0/1/2 = x/y/z; (indx1, indx2) = the grid
 * line (x: iy,iz; y: ix,iz; z: ix,iy); id = ID (>0 irregular, <0 corner pair);
 * left_loc; nwei = length of wei.weil[0]/weir[0]; p = local frame, row major. */
typedef struct {
  int32_t dir, indx1, indx2, id, left_loc, nwei;
  double coord[3], gamma, normal[3], p[9], weil[9], weir[9];
} mts_crossing;

typedef struct mts_problem* mts_handle;

/* Builds the mesh tags, crossing list and MIB weights (on host threads, or
 * on the device when params->setup is MTS_SETUP_DEVICE) and places the
 * problem on the current CUDA device, all of its buffers in one block of the
 * device's stream-ordered pool.  Replaces the setup of
 *   Mesh::Mesh            src/mesh/mesh.cc:20-70
 *   Intersections ctor    src/spatial/intersection.cc:22-51 (crossings,
 *                         MIB-L1/L2 weights via LU, src/decomposition/lu.cc)
 * and the constructors Douglas_ADI / LOD / TS (src/temporal/douglas_adi.h:47,
 * lod.h:51, trapezoidal.h:48).  The time starts at params->t0. */
mts_status mts_create(const mts_grid* grid, const mts_surface* surface, const mts_params* params,
                      mts_handle* out);

/* Same, from a caller-supplied mesh and crossing list (the drop-in path: the
 * reference's Mesh::mesh_value and Intersections::ifpx/ifpy/ifpz, flattened).
 * tags: nx*ny*nz values in {+1, -1}, x fastest. */
mts_status mts_create_from_crossings(const mts_grid* grid, const int8_t* tags,
                                     const mts_crossing* crossings, int32_t ncrossings,
                                     const mts_params* params, mts_handle* out);

mts_status mts_destroy(mts_handle h);

/* The host half of mts_create alone (no device needed): node tags and the
 * crossing list with MIB weights.  tags may be NULL; when out is NULL or
 * capacity < *count only *count is set.  counts (may be NULL) receives
 * [corner pairs, singular-matrix warnings]. */
mts_status mts_setup_host(const mts_grid* grid, const mts_surface* surface, const mts_params* params,
                          int8_t* tags, mts_crossing* out, int32_t capacity, int32_t* count,
                          int64_t counts[2]);

/* The same setup on the current CUDA device, with the same arguments and
 * results: a thread per node for the tags, a thread per grid line for the
 * crossing scan, rtsafe and the MIB-L1/L2 weight solves, a thread per corner
 * pair for the MIB-L2 36x36 systems.  The tags equal mts_setup_host's; the
 * crossing records equal them bit for bit except where the reference's
 * pow(v, 2) (glibc) is not the correctly rounded square, which the device
 * computes: there a root, normal or weight can differ in its last bits.
 * Synchronous.  No reference counterpart beyond mts_setup_host's. */
mts_status mts_setup_device(const mts_grid* grid, const mts_surface* surface, const mts_params* params,
                            int8_t* tags, mts_crossing* out, int32_t capacity, int32_t* count,
                            int64_t counts[2]);

/* Initialization (douglas_adi.cc:1684-1714, lod/trapezoidal copies): the
 * exact solution at the current time, by node tag, written on the device. */
mts_status mts_initialize(mts_handle h);

/* Host <-> device copies of the solution field (nx*ny*nz doubles). */
mts_status mts_set_solution(mts_handle h, const double* u);
mts_status mts_get_solution(mts_handle h, double* u);

/* One step of the handle's method ending at t_next.  Replaces
 *   Douglas_ADI::Solve_2nd(eq(t_next), inter, uh, beta)   douglas_adi.cc:66-1110
 *   LOD::Solve_2nd(eq(t_next), inter, uh, beta, 'I'|'C')   lod.cc:44-205
 *   TS::Solve_2nd(eq(t_prev), eq(t_half), eq(t_next), ...)  trapezoidal.cc:46-272
 * t_prev and t_half are read by TS only.  Refresh_Jump (intersection.cc:
 * 2294-2490) runs on the device inside the step.  Asynchronous. */
mts_status mts_solve_2nd(mts_handle h, double t_prev, double t_half, double t_next);

/* nsteps steps of the time loop of src/helper.h:199-238 (t += dt before each
 * step; TS evaluates at t-dt, t-dt/2, t).  Asynchronous. */
mts_status mts_advance(mts_handle h, int32_t nsteps);

/* nsteps steps of each of n independent handles, run as one batch: the
 * plain-form handles of one method advance together, one kernel launch per
 * kernel of the step for all of them (each CTA carries its problem and its
 * place in that problem's grid), and so do the mixed-precision Douglas-ADI
 * handles whose lines have at most 160 rows, in a group of their own;
 * handles whose lines fill the GPU (256 per SM in every direction),
 * fast-form handles and longer-line mixed ones step on their own streams
 * alongside, and the groups run at once on their own streams.  Each
 * handle's result and time are those of mts_advance(h, nsteps), bit for
 * bit.  Handles must be distinct, on one
 * device, with profiling off.  Synchronous.  No counterpart in the
 * reference, which steps one problem per process (helper.h:199-426). */
mts_status mts_batch_advance(const mts_handle* handles, int32_t n, int32_t nsteps);

/* The same with a step count per handle (counts[i] steps for handles[i]):
 * the batched launches run for the longest count and skip each problem once
 * its own steps are done, so problems with different remaining work share
 * one batch.  Used by the continuous-batching server. */
mts_status mts_batch_advance_steps(const mts_handle* handles, const int32_t* counts, int32_t n);

/* The same loop with the caller's host field: u_in is uploaded, nsteps steps
 * run, the result is downloaded into u_out (which may equal u_in).  This is
 * the per-call cost of the reference's Solve_2nd(..., CubicDoub& uh, ...)
 * contract with the field in host memory. */
mts_status mts_advance_host(mts_handle h, const double* u_in, double* u_out, int32_t nsteps);

/* Error (douglas_adi.cc:1723-1770): L-infinity with its first argmax in
 * [ix][iy][iz] loop order, and L2 = sqrt(sum e^2 / (nx ny nz)), against the
 * exact solution at the current time.  Synchronous; on an error status the
 * outputs are left untouched. */
mts_status mts_norms(mts_handle h, double* lmax, double* l2, int32_t* argmax3);

/* The same norms with no allocation of any kind.  This entry point has no
 * counterpart in the reference.  It is for host programs that keep fields in
 * a device pool of their own (a framework's caching allocator holding most of
 * HBM, a process under a hard memory cap) and check their error mid-run,
 * where a cudaMalloc may fail and a cudaFree would synchronize the device.
 *
 * u_dev: a device field of nx*ny*nz doubles laid out like the solution,
 * evaluated against the exact solution at time t; NULL evaluates the handle's
 * own solution at the handle's time (t ignored).  The outputs equal
 * mts_norms' bit for bit.  Synchronous on the handle's stream.
 *
 * The reduction's scratch is one static device array of 48.5 KiB per device,
 * holding the partials of at most 2048 reduction blocks: grids of more than
 * 4194304 nodes (2048 x 2048) are rejected with MTS_ERR_ARG.  Its ticket
 * counter must be zero when the kernel starts; each call clears it first.
 * All calls on a device share the array, so calls that overlap in time on one
 * device (other handles, streams or host threads) race: serialise them.  Each
 * call looks the array's address up again, so a device reset between calls
 * is harmless; the first call on a device may load the module, so make it
 * before any stream capture begins on the device.  On an error status the
 * outputs are left untouched. */
mts_status mts_norms_noalloc(mts_handle h, const double* u_dev, double t, double* lmax, double* l2,
                             int32_t* argmax3);

/* The fictitious points' error report at the current time: Refresh_Fp
 * (src/spatial/intersection.cc:1841-2281) on the device, one thread per
 * crossing or corner pair, and Error_Fp's maximum and root mean square of
 * the relative errors (:4667-4771), added up on the host in its loop order:
 * the reference's values bit for bit (inf or NaN where the exact solution of
 * the other side is 0 at a fictitious point's node, as there).  The reference
 * prints them with 4 digits ("Lmax = ...", "L2   = ..."). */
mts_status mts_fp_errors(mts_handle h, double* lmax, double* l2);

/* The jumps' error report at the current time: Refresh_Jump's check
 * (src/spatial/intersection.cc:2294-2490) on the device, one thread per
 * crossing, the relative error |u_dir - [beta u_d]| / [beta u_d] of the
 * jump data the solvers are given against the exact flux jump along the
 * crossing's line (the divisor's sign kept), and Error_Jump's maximum and
 * root mean square (:4594-4662) added up on the host in its loop order: the
 * reference's values bit for bit (NaN for Eq_0, whose flux jumps are 0).
 * The report depends on the geometry and the time only, not on the
 * solution.  Printed as "Lmax = ...", "L2   = ..." with 4 digits. */
mts_status mts_jump_errors(mts_handle h, double* lmax, double* l2);

mts_status mts_get_time(mts_handle h, double* t);
mts_status mts_set_time(mts_handle h, double t);

/* Blocks until all work queued on the handle's stream is done; reports a
 * zero pivot met by any line solve since the last check. */
mts_status mts_synchronize(mts_handle h);

/* Counts: [0..2] crossings per direction, [3..5] MIB row blocks per
 * direction, [6] corner pairs, [7] singular-matrix warnings of the weight
 * solves (intersection.cc:1034-1057 prints these and carries on). */
mts_status mts_get_counts(mts_handle h, int64_t counts[8]);

/* Host copies of the setup products (for parity checks): node tags (+1/-1,
 * x fastest) and the crossing list in the reference's order (per direction
 * x, y, z; lines in loop order; crossings by left_loc). */
mts_status mts_export_tags(mts_handle h, int8_t* tags);
mts_status mts_export_crossings(mts_handle h, mts_crossing* out, int32_t capacity, int32_t* count);

/* Number of kernel launches the library has queued on this handle. */
mts_status mts_get_launch_count(mts_handle h, int64_t* launches);

/* Device memory the handle holds (the sum of its allocations), for callers
 * that admit problems against a memory budget.  No reference counterpart. */
mts_status mts_get_device_bytes(mts_handle h, int64_t* bytes);

/* The CUDA stream of the handle (a cudaStream_t), for callers that order
 * their own work against it. */
mts_status mts_get_stream(mts_handle h, void** stream);

/* Per-kernel timing with CUDA events recorded on the handle's stream around
 * every launch of a step (negligible overhead; off by default).  Slots, in
 * launch order: Douglas-ADI and LOD {0 jumps, 1 x sweep, 2 y sweep, 3 z sweep};
 * TS {0 jumps, 1 explicit x, 2 explicit y, 3 z sweep, 4 y sweep, 5 x sweep}.
 * mts_profile_read synchronizes, returns the summed milliseconds and launch
 * counts per slot since the last read, and resets them. */
mts_status mts_set_profiling(mts_handle h, int32_t on);
mts_status mts_profile_read(mts_handle h, double ms[8], int64_t launches[8]);

/* Launch shape of the persistent line-sweep kernels (rows staged per chunk,
 * staging-ring depth, threads per CTA), chosen separately for the first,
 * second and third implicit sweep of a step.  Every shape computes the same
 * bits; they differ only in speed.  mts_autotune times each compiled shape on
 * the handle's own problem for `steps` steps (the solution and time are
 * restored afterwards) and keeps the fastest per sweep; shapes[3] receives
 * the choice.  mts_sweep_shape_count gives the number of shapes. */
int32_t mts_sweep_shape_count(void);
mts_status mts_set_sweep_shape(mts_handle h, int32_t sweep, int32_t shape);
mts_status mts_autotune(mts_handle h, int32_t steps, int32_t shapes[3]);

/* Arithmetic of the step.  MTS_PRECISION_PLAIN (the default) is the FP64
 * drop-in, bit-identical to the reference.  MTS_PRECISION_MIXED (Douglas-ADI
 * only) solves each step for its increment u^{n+1} - u^n: the residual
 * dt (A_x + A_y + A_z) u^n + dt src is formed in FP64, the three line solves
 * of douglas_adi.cc:66-1110 run on the FP32 increment with FP32 factors, and
 * the increment is added to the FP64 state.  Results differ from the plain
 * form by the FP32 rounding of one step's increment per step; the error
 * against the exact solution stays that of the plain form.  Switching the
 * form on builds its per-node FP32 coefficients on the device once (3 x 4
 * bytes per node and direction, for lines of up to 544 rows).  No
 * counterpart in the reference, which computes in FP64 only.
 *
 * MTS_PRECISION_FAST (Douglas-ADI only, at most 544 nodes per axis) is the
 * same step in FP64 throughout, reorganised for the GPU: it is solved for the
 * increment as above, with the residual formed inside the x sweep, and every
 * line is solved by one warp whose lanes split the Thomas recurrences into
 * segments joined by shuffle scans.  The operations are those of the plain
 * form in another order, so results differ from it by rounding only (within
 * 1e-10 relative max-norm over the runs the tests cover).  Where setup has
 * reported near-singular MIB weight systems (mts_get_counts()[7] > 0) the
 * problem itself is that sensitive to rounding (the reference's own code
 * moves by ~1e-5 when compiled with fused multiply-adds) and only the plain
 * form reproduces the reference to 1e-10.  Switching it on
 * builds its row tables and, for each line that crosses the interface, its
 * per-row solve coefficients (3 x 8 bytes per row) on the device once.
 * Profiling slots of this form: {0 MIB rows + residual + x solve, 1 y solve,
 * 2 z solve + update}.
 * No counterpart in the reference, which computes in FP64 only. */
typedef enum { MTS_PRECISION_PLAIN = 0, MTS_PRECISION_MIXED = 1, MTS_PRECISION_FAST = 2 } mts_precision;
mts_status mts_set_precision(mts_handle h, int32_t precision);
mts_status mts_get_precision(mts_handle h, int32_t* precision);

/* Text of the last error on this thread. */
const char* mts_last_error(void);

/* ABI version (major*100 + minor). */
int32_t mts_version(void);

#ifdef __cplusplus
}
#endif
#endif /* MTS_H */

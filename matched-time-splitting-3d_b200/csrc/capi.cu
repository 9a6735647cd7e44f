// C ABI of the GPU path (include/mts.h): handle lifecycle, the one-time
// precompute of the time-invariant MIB row blocks, device residency, and the
// per-step launches.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/mts.h"
#include "device.h"
#include "setup.h"

namespace {

thread_local std::string g_last_error;

mts_status fail(mts_status s, const std::string& msg) {
  g_last_error = msg;
  return s;
}

#define CUDA_TRY(call)                                                             \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess) {                                                       \
      return fail(e_ == cudaErrorMemoryAllocation ? MTS_ERR_OOM : MTS_ERR_CUDA,    \
                  std::string(#call) + ": " + cudaGetErrorString(e_));             \
    }                                                                              \
  } while (0)

// Device memory comes from the device's stream-ordered pool (cudaMallocAsync
// on the handle's stream, cudaFreeAsync when the handle is destroyed): a
// server that creates and destroys problems continuously then neither
// synchronizes the device on every free nor returns memory to the driver in
// between (the pool keeps what it has, see configure_pool).  A handle takes
// its small buffers from a few shared slabs: a pool that holds many freed
// blocks makes every cudaMallocAsync slower (measured on B200: 512 handles
// of 40 buffers each took 14 s to allocate once the previous 512 had been
// freed, against 0.35 s with one block per handle).  Buffers of 64 KB or
// more get blocks of their own size, so the slabs waste at most their
// unused tail (under 1 MB).
constexpr size_t kOwnBlock = (size_t)64 << 10;
constexpr size_t kSlabFirst = (size_t)64 << 10;
constexpr size_t kSlabMax = (size_t)1 << 20;
constexpr size_t kAlign = 256;

}  // namespace

struct mts_problem {
  int device = 0;
  cudaStream_t stream = nullptr;
  mts::Grid g;
  mts_params prm{};
  std::vector<int8_t> tags;
  std::vector<mts_crossing> cross;
  mts::SetupReport rep;
  int64_t nblk[3] = {0, 0, 0};
  int64_t ncr[3] = {0, 0, 0};
  mts::Dev dev{};
  double* u0 = nullptr;
  double* u1 = nullptr;
  struct Slab {
    char* base;
    size_t size, used;
  };
  std::vector<Slab> slabs;
  int small_slab = -1;           // the slab small buffers are cut from
  size_t next_slab = kSlabFirst;  // size of the next small-buffer slab
  int64_t device_bytes = 0;       // sum of the slabs' sizes
  bool sizing = false;            // grab only adds up sizes (the plan pass of finish_create)
  size_t planned = 0;
  double* norm_part = nullptr;
  double* norm_out = nullptr;
  mts::SideStream side{nullptr, nullptr, nullptr};  // the mixed form's second stream
  // the fast and mixed forms' data are built on the first switch to the
  // form; a build that fails part way is done again on the next switch
  bool fast_built = false;
  bool mixed_built = false;
  // the error reports' tables (mts_fp_errors, mts_jump_errors), built on
  // first use
  mts_crossing* fp_cr = nullptr;
  int32_t* fp_ci = nullptr;
  int8_t* fp_role = nullptr;
  double* fp_err = nullptr;
  std::vector<int32_t> fp_perm;

  int norm_nb = 1;
  double t = 0;
  int64_t launches = 0;
  // per-kernel event timing (mts_set_profiling)
  bool profiling = false;
  std::vector<std::array<cudaEvent_t, 2 * mts::kProfileSlots>> ev_busy, ev_free;
  double prof_ms[mts::kProfileSlots] = {};
  int64_t prof_n[mts::kProfileSlots] = {};

  int slots() const {
    if (dev.precision == 2) return 3;
    return prm.method == MTS_TS ? 6 : prm.method == MTS_ADI ? 5 : 4;
  }

  ~mts_problem() {
    if (stream) cudaStreamSynchronize(stream);
    for (auto& a : ev_busy)
      for (cudaEvent_t e : a) cudaEventDestroy(e);
    for (auto& a : ev_free)
      for (cudaEvent_t e : a) cudaEventDestroy(e);
    for (const Slab& sl : slabs) cudaFreeAsync(sl.base, stream);
    if (stream) {
      cudaStreamSynchronize(stream);
      cudaStreamDestroy(stream);
    }
    // every step joins the side stream back into the main one before it ends
    if (side.stream) cudaStreamDestroy(side.stream);
    if (side.fork) cudaEventDestroy(side.fork);
    if (side.join) cudaEventDestroy(side.join);
  }
  // bytes of device memory, 256-byte aligned: a buffer of 64 KB or more
  // gets a block of its own size; smaller ones are cut from the current
  // small-buffer slab, and when that is full from a new one of twice its
  // size (64 KB, then up to 1 MB)
  cudaError_t grab(size_t bytes, void** out) {
    *out = nullptr;
    bytes = (bytes + kAlign - 1) / kAlign * kAlign;
    if (bytes == 0) bytes = kAlign;
    if (sizing) {
      planned += bytes;
      return cudaSuccess;
    }
    if (small_slab >= 0 && slabs[small_slab].size - slabs[small_slab].used >= bytes) {
      Slab& sl = slabs[small_slab];
      *out = sl.base + sl.used;
      sl.used += bytes;
      return cudaSuccess;
    }
    const bool own = bytes >= kOwnBlock;
    const size_t size = own ? bytes : next_slab;
    void* p = nullptr;
    cudaError_t e = cudaMallocAsync(&p, size, stream);
    if (e != cudaSuccess) return e;
    slabs.push_back(Slab{(char*)p, size, bytes});
    device_bytes += (int64_t)size;
    if (!own) {
      small_slab = (int)slabs.size() - 1;
      next_slab = std::min(kSlabMax, next_slab * 2);
    }
    *out = p;
    return cudaSuccess;
  }
  // one block of `bytes` that the next grabs are cut from, whatever their size
  cudaError_t reserve(size_t bytes) {
    if (bytes == 0) return cudaSuccess;
    void* p = nullptr;
    cudaError_t e = cudaMallocAsync(&p, bytes, stream);
    if (e != cudaSuccess) return e;
    slabs.push_back(Slab{(char*)p, bytes, 0});
    device_bytes += (int64_t)bytes;
    small_slab = (int)slabs.size() - 1;
    return cudaSuccess;
  }
  template <class T>
  cudaError_t put(T** dst, const T* src, size_t n) {
    if (n == 0) n = 1;
    cudaError_t e = grab(n * sizeof(T), (void**)dst);
    if (e != cudaSuccess || !src || sizing) return e;
    return cudaMemcpyAsync(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice, stream);
  }
  // n elements (uploaded from src when given) followed by `pad` zeroed
  // elements of slack that the sweep kernels may read but never use
  template <class T>
  cudaError_t put_padded(T** dst, const T* src, size_t n, size_t pad) {
    cudaError_t e = grab((n + pad) * sizeof(T), (void**)dst);
    if (e != cudaSuccess || sizing) return e;
    e = cudaMemsetAsync(*dst + (src ? n : 0), 0, (src ? pad : n + pad) * sizeof(T), stream);
    if (e != cudaSuccess || !src) return e;
    return cudaMemcpyAsync(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice, stream);
  }
};

namespace {

// Convert2Tri_irr / _cor (src/temporal/douglas_adi.cc:1554-1577, 1637-1675)
// applied to the matrix part of a MIB row block, once: the coefficients do
// not change between steps.  The multipliers are kept so that each step
// replays the same row operations on its right-hand side.
void precompute_block(mts::MibBlock& b, double cdt, const double vd[3][3]) {
  if (b.kind == 2) {
    double row[2][4];
    std::memset(row, 0, sizeof row);
    row[0][0] = -cdt * vd[0][0];
    row[0][1] = 1 - cdt * vd[0][1];
    for (int i = 0; i < 4; i++) row[0][i] += -cdt * vd[0][2] * b.w[1][i];
    row[1][2] = 1 - cdt * vd[1][1];
    row[1][3] = -cdt * vd[1][2];
    for (int i = 0; i < 4; i++) row[1][i] += -cdt * vd[1][0] * b.w[0][i];
    double rate = row[1][0] / row[0][0];
    for (int i = 0; i < 4; i++) row[1][i] -= rate * row[0][i];
    b.rate[0] = rate;
    rate = row[0][3] / row[1][3];
    for (int i = 0; i < 4; i++) row[0][i] -= rate * row[1][i];
    b.rate[1] = rate;
    for (int i = 0; i < 2; i++) {
      b.ia[i] = row[i][i];
      b.ib[i] = row[i][i + 1];
      b.ic[i] = row[i][i + 2];
    }
  } else {
    double row[3][5];
    std::memset(row, 0, sizeof row);
    row[0][0] = -cdt * vd[0][0];
    row[0][1] = 1 - cdt * vd[0][1];
    for (int i = 0; i < 5; i++) row[0][i] -= cdt * vd[0][2] * b.w[1][i];
    row[1][2] = 1 - cdt * vd[1][1];
    for (int i = 0; i < 5; i++) row[1][i] -= cdt * vd[1][0] * b.w[0][i];
    for (int i = 0; i < 5; i++) row[1][i] -= cdt * vd[1][2] * b.w[3][i];
    row[2][3] = 1 - cdt * vd[2][1];
    row[2][4] = -cdt * vd[2][2];
    for (int i = 0; i < 5; i++) row[2][i] -= cdt * vd[2][0] * b.w[2][i];
    double r1 = row[1][0] / row[0][0], r2 = row[2][0] / row[0][0];
    for (int i = 0; i < 5; i++) {
      row[1][i] -= r1 * row[0][i];
      row[2][i] -= r2 * row[0][i];
    }
    double r0b = row[0][4] / row[2][4], r1b = row[1][4] / row[2][4];
    for (int i = 0; i < 5; i++) {
      row[0][i] -= r0b * row[2][i];
      row[1][i] -= r1b * row[2][i];
    }
    double r2b = row[2][1] / row[1][1];
    for (int i = 0; i < 5; i++) row[2][i] -= r2b * row[1][i];
    double r0c = row[0][3] / row[1][3];
    for (int i = 0; i < 5; i++) row[0][i] -= r0c * row[1][i];
    b.rate[0] = r1;
    b.rate[1] = r2;
    b.rate[2] = r0b;
    b.rate[3] = r1b;
    b.rate[4] = r2b;
    b.rate[5] = r0c;
    for (int i = 0; i < 3; i++) {
      b.ia[i] = row[i][i];
      b.ib[i] = row[i][i + 1];
      b.ic[i] = row[i][i + 2];
    }
  }
}

int line_count(const mts::Grid& g, int d) {
  int n1 = d == 0 ? g.ny : g.nx;
  int n2 = d == 2 ? g.ny : g.nz;
  return n1 * n2;
}

// Douglas-ADI steps of a single handle run their jumps and MIB
// right-hand-side rows beside the pointwise pass, on a second stream that is
// made when such a step is first launched (handles that only step in batches
// never make one).
cudaError_t ensure_side_stream(mts_problem* h) {
  if (h->side.stream || h->prm.method != MTS_ADI) return cudaSuccess;
  cudaError_t e = cudaStreamCreateWithFlags(&h->side.stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->side.fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->side.join, cudaEventDisableTiming);
  return e;
}

// Builds every device-side table of a problem from its grid, tags and
// crossing list, and uploads them.
// The device's pool keeps freed memory for the next allocations instead of
// returning it to the driver at every synchronization (once per device,
// before the first allocation of a handle or a device setup).
void keep_pool(int device) {
  static std::atomic<bool> kept[64];
  if (device < 0 || device >= 64 || kept[device].exchange(true)) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
}

mts_status finish_create(mts_problem* h) {
  const mts::Grid& g = h->g;
  const mts_params& p = h->prm;
  const long long N = g.nodes();
  mts::Dev& D = h->dev;
  D.nx = g.nx;
  D.ny = g.ny;
  D.nz = g.nz;
  D.nn = N;
  D.eq = p.eq;
  D.method = p.method;
  D.dt = p.dt;
  D.kex = 0.5 * p.dt;
  const double coef = (p.method == MTS_LOD_CN || p.method == MTS_TS) ? 0.5 : 1;
  D.cdt = coef * p.dt;
  D.hdt = 0.5 * p.dt;
  D.bi = p.beta_in;
  D.bo = p.beta_out;
  D.kin = 12.0 * p.beta_in - 1.0;
  D.c6bo = 6.0 * p.beta_out;
  const double h3[3] = {g.dx, g.dy, g.dz};
  for (int d = 0; d < 3; d++)
    for (int side = 0; side < 2; side++) {
      double beta = side ? p.beta_out : p.beta_in;
      double hh = h3[d];
      D.vd[d][side][0] = beta / (hh * hh);
      D.vd[d][side][1] = -(beta + beta) / (hh * hh);
      D.vd[d][side][2] = beta / (hh * hh);
      D.ia[d][side] = -D.cdt * D.vd[d][side][0];
      D.ib[d][side] = 1 - D.cdt * D.vd[d][side][1];
      D.ic[d][side] = -D.cdt * D.vd[d][side][2];
    }

  // node tags with MIB-row flags; blocks per direction
  std::vector<uint8_t> tag8((size_t)N);
  for (long long m = 0; m < N; m++) tag8[m] = h->tags[m] == 1 ? mts::TAG_OUT : 0;
  std::vector<mts::MibBlock> blocks[3];
  std::vector<int32_t> bstart[3];
  std::vector<mts::CrossConst> cc(h->cross.size());
  // order crossings per direction by (line, left_loc), keeping pairs together
  std::vector<int> order(h->cross.size());
  for (size_t i = 0; i < order.size(); i++) order[i] = (int)i;
  auto lid = [&](const mts_crossing& c) {
    int n2 = c.dir == 2 ? g.ny : g.nz;
    return (long long)c.indx1 * n2 + c.indx2;
  };
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    const mts_crossing &A = h->cross[a], &B = h->cross[b];
    if (A.dir != B.dir) return A.dir < B.dir;
    long long la = lid(A), lb = lid(B);
    if (la != lb) return la < lb;
    return A.left_loc < B.left_loc;
  });
  for (int d = 0; d < 3; d++) bstart[d].assign((size_t)line_count(g, d) + 1, 0);
  const uint8_t flag[3] = {mts::TAG_MIBX, mts::TAG_MIBY, mts::TAG_MIBZ};
  for (size_t k = 0; k < order.size();) {
    const int ci = order[k];
    const mts_crossing& c = h->cross[ci];
    if (c.dir < 0 || c.dir > 2) return fail(MTS_ERR_ARG, "crossing direction out of range");
    const int d = c.dir;
    const int n[3] = {g.nx, g.ny, g.nz};
    const int a1 = d == 0 ? 1 : 0, a2 = d == 2 ? 1 : 2;
    if (c.indx1 < 1 || c.indx1 >= n[a1] - 1 || c.indx2 < 1 || c.indx2 >= n[a2] - 1 || c.left_loc < 1)
      return fail(MTS_ERR_ARG, "crossing outside the interior lines");
    mts::MibBlock b;
    std::memset(&b, 0, sizeof b);
    b.line = (int32_t)lid(c);
    b.L = c.left_loc;
    b.c0 = ci;
    if (c.id > 0) {
      b.kind = 2;
      b.c1 = ci;
      std::memcpy(b.w[0], c.weil, sizeof c.weil);
      std::memcpy(b.w[1], c.weir, sizeof c.weir);
      k += 1;
    } else {
      if (k + 1 >= order.size()) return fail(MTS_ERR_ARG, "corner crossing without its pair");
      const int cj = order[k + 1];
      const mts_crossing& r = h->cross[cj];
      if (r.id >= 0 || r.dir != d || lid(r) != lid(c) || r.left_loc != c.left_loc + 1)
        return fail(MTS_ERR_ARG, "corner crossing without its pair");
      b.kind = 3;
      b.c1 = cj;
      std::memcpy(b.w[0], c.weil, sizeof c.weil);
      std::memcpy(b.w[1], c.weir, sizeof c.weir);
      std::memcpy(b.w[2], r.weil, sizeof r.weil);
      std::memcpy(b.w[3], r.weir, sizeof r.weir);
      k += 2;
    }
    // the fictitious-point stencils read nodes L-1 .. L+kind: all must exist
    if (b.L + b.kind >= n[d]) return fail(MTS_ERR_ARG, "crossing block runs past the line end");
    if (!blocks[d].empty() && blocks[d].back().line == b.line && blocks[d].back().L + blocks[d].back().kind > b.L)
      return fail(MTS_ERR_ARG, "overlapping crossing blocks on one line");
    double vdr[3][3];
    for (int q = 0; q < b.kind; q++) {
      int idx3[3];
      idx3[a1] = c.indx1;
      idx3[a2] = c.indx2;
      idx3[d] = b.L + q;
      long long m = g.index(idx3[0], idx3[1], idx3[2]);
      int side = h->tags[m] == 1;
      for (int z = 0; z < 3; z++) vdr[q][z] = D.vd[d][side][z];
      tag8[m] |= flag[d];
      b.sides |= side << q;
    }
    precompute_block(b, D.cdt, vdr);
    blocks[d].push_back(b);
    bstart[d][b.line + 1]++;
  }
  for (int d = 0; d < 3; d++) {
    for (size_t l = 0; l + 1 < bstart[d].size(); l++) bstart[d][l + 1] += bstart[d][l];
    h->nblk[d] = (int64_t)blocks[d].size();
  }
  // Thomas factorisation (the factor half of TDMA, douglas_adi.cc:1790-1798:
  // gam_j = c_{j-1}/bet, bet = b_j - a_j*gam_j, same operations): prefix
  // tables per direction and row-1 side here; the per-node factors of the
  // lines that cross the interface, from their first MIB row on, are
  // computed on the device once the tables are there (launch_factor_lines).
  std::vector<double> ptab[3][2];
  {
    const int n[3] = {g.nx, g.ny, g.nz};
    std::vector<double> a, b, c;
    auto factor = [&](int len, std::vector<double>& bet_out, std::vector<double>& gam_out) -> bool {
      bet_out.resize(len);
      gam_out.resize(len);
      double bet = b[0];
      if (bet == 0.0) return false;
      bet_out[0] = bet;
      gam_out[0] = 0.0;
      for (int j = 1; j < len; j++) {
        double gm = c[j - 1] / bet;
        bet = b[j] - a[j] * gm;
        if (bet == 0.0) return false;
        gam_out[j] = gm;
        bet_out[j] = bet;
      }
      return true;
    };
    std::vector<double> lb, lg;
    for (int d = 0; d < 3; d++) {
      const int len = n[d];
      a.assign(len, 0.0);
      b.assign(len, 1.0);
      c.assign(len, 0.0);
      for (int side = 0; side < 2; side++) {
        for (int j = 1; j < len - 1; j++) {
          a[j] = D.ia[d][side];
          b[j] = D.ib[d][side];
          c[j] = D.ic[d][side];
        }
        a[len - 1] = 0.0;
        b[len - 1] = 1.0;
        c[len - 1] = 0.0;
        if (!factor(len, lb, lg)) return fail(MTS_ERR_ZERO_PIVOT, "zero pivot in a line factorisation");
        ptab[d][side].resize(2 * (size_t)len);
        for (int j = 0; j < len; j++) {
          ptab[d][side][2 * j] = lb[j];
          ptab[d][side][2 * j + 1] = lg[j];
        }
      }
    }
  }

  // per-line side bits: node 0, node 1, node n-1 outside
  std::vector<uint8_t> lside[3];
  {
    const int n[3] = {g.nx, g.ny, g.nz};
    for (int d = 0; d < 3; d++) {
      const int a1 = d == 0 ? 1 : 0, a2 = d == 2 ? 1 : 2;
      const int n2 = n[a2];
      lside[d].assign((size_t)line_count(g, d), 0);
      for (int i1 = 0; i1 < n[a1]; i1++)
        for (int i2 = 0; i2 < n[a2]; i2++) {
          int idx3[3];
          idx3[a1] = i1;
          idx3[a2] = i2;
          auto out_at = [&](int j) {
            idx3[d] = j;
            return h->tags[(size_t)g.index(idx3[0], idx3[1], idx3[2])] == 1 ? 1 : 0;
          };
          lside[d][(size_t)i1 * n2 + i2] = (uint8_t)(out_at(0) | (out_at(1) << 1) | (out_at(n[d] - 1) << 2));
        }
    }
  }
  for (size_t i = 0; i < h->cross.size(); i++) {
    const mts_crossing& c = h->cross[i];
    mts::CrossConst& q = cc[i];
    q.x = c.coord[0];
    q.y = c.coord[1];
    q.z = c.coord[2];
    q.R2 = (q.x * q.x + q.y * q.y) + q.z * q.z;
    q.S = (std::sin(2.0 * q.x) * std::cos(2.0 * q.y)) * std::sin(2.0 * q.z);
    q.D[0] = ((2.0 * std::cos(2.0 * q.x)) * std::cos(2.0 * q.y)) * std::sin(2.0 * q.z);
    q.D[1] = ((-2.0 * std::sin(2.0 * q.x)) * std::sin(2.0 * q.y)) * std::sin(2.0 * q.z);
    q.D[2] = ((2.0 * std::sin(2.0 * q.x)) * std::cos(2.0 * q.y)) * std::cos(2.0 * q.z);
    for (int k = 0; k < 3; k++) q.p[k] = c.p[k];
    if (!mts::frame_inverse_col0(c.p, c.dir, &q.pinv)) return fail(MTS_ERR_SETUP, "singular local frame");
    h->ncr[c.dir]++;
  }
  D.ncross = (int)h->cross.size();

  // axis tables
  std::vector<double> axv[3], s2v[3], c2v[3];
  const std::vector<double>* axes[3] = {&g.x, &g.y, &g.z};
  for (int d = 0; d < 3; d++) {
    axv[d] = *axes[d];
    s2v[d].resize(axv[d].size());
    c2v[d].resize(axv[d].size());
    for (size_t i = 0; i < axv[d].size(); i++) {
      s2v[d][i] = std::sin(2.0 * axv[d][i]);
      c2v[d][i] = std::cos(2.0 * axv[d][i]);
    }
  }

  keep_pool(h->device);
  static bool configured = false;
  if (!configured) {
    mts::configure_kernels();
    mts::configure_mixed_kernels();
    mts::configure_batch_kernels();
    mts::configure_fast_kernels();
    mts::configure_mixed_batch_kernels();
    configured = true;
  }
  int sms = 0;
  CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));
  D.sweep_blocks = sms > 0 ? sms : 1;
  // sweep threads of a launch: one CTA per SM at most and no more CTAs than
  // the lines of a direction need, so at most max lines + one CTA
  long long maxlines = 0;
  for (int d = 0; d < 3; d++) maxlines = std::max(maxlines, (long long)line_count(g, d));
  const size_t tmax = std::min((size_t)D.sweep_blocks * (size_t)mts::sweep_shape_max_threads(),
                               (size_t)maxlines + (size_t)mts::sweep_shape_max_threads());
  const int nmax = std::max(g.nx, std::max(g.ny, g.nz));
  {
    // default shapes: when the lines fill the GPU, 4 rows x 4 chunks with 384
    // threads for x and y lines and 448 for z lines (the shapes mts_autotune
    // picks at 257^3, 23 % faster per step than 8 x 4 x 256 there); the small
    // shape 9 (several CTAs per SM, for concurrent small problems) when they
    // do not; mts_autotune picks per problem.  TS runs its sweeps z, y, x.
    const bool large = maxlines >= (long long)D.sweep_blocks * 256;
    const int by_dir[3] = {large ? 6 : 9, large ? 6 : 9, large ? 8 : 9};  // x, y, z
    const int dir_of_sweep[3] = {p.method == MTS_TS ? 2 : 0, 1, p.method == MTS_TS ? 0 : 2};
    for (int k = 0; k < 3; k++) {
      const int want = by_dir[dir_of_sweep[k]];
      int def = -1;
      for (int s = mts::sweep_shape_count() - 1; s >= 0; s--)
        if (mts::sweep_shape_fits(s, nmax) && (def < 0 || s == want)) def = s;
      if (def < 0) return fail(MTS_ERR_ARG, "grid lines too long for the sweep kernels' shared memory");
      D.shape[k] = def;
    }
  }
  CUDA_TRY(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  // row slack of the fields the sweeps stage whole chunks of: kRowPad rows of
  // the largest stride (an x-y plane)
  const size_t fpad = (size_t)mts::kRowPad * (size_t)g.nx * (size_t)g.ny;
  // nodes that are a MIB row of some block: the pointwise passes leave them
  // to a per-node pass over this list
  std::vector<long long> mibn;
  for (long long m = 0; m < N; m++)
    if (tag8[(size_t)m] & (mts::TAG_MIBX | mts::TAG_MIBY | mts::TAG_MIBZ)) mibn.push_back(m);
  h->norm_nb = mts::norms_blocks(D);
  // Every buffer of the handle, placed twice: first only to add up their
  // sizes, then into the one pool block of that size.
  auto place_all = [&]() -> mts_status {
    CUDA_TRY(h->put_padded(&h->u0, (const double*)nullptr, (size_t)N, fpad));
    CUDA_TRY(h->put_padded(&h->u1, (const double*)nullptr, (size_t)N, fpad));
    D.u0 = h->u0;
    D.u1 = h->u1;
    CUDA_TRY(h->put_padded(&D.dp, (const double*)nullptr, (size_t)nmax * tmax, (size_t)mts::kRowPad * tmax));
    for (int d = 0; d < 3; d++) {
      for (int side = 0; side < 2; side++) {
        double* pt = nullptr;
        CUDA_TRY(h->put(&pt, ptab[d][side].data(), ptab[d][side].size()));
        D.ptab[d][side] = pt;
      }
      double* rbk = nullptr;
      CUDA_TRY(h->put(&rbk, (const double*)nullptr, 3 * blocks[d].size()));
      D.rblk[d] = rbk;
      D.nblk[d] = (int)blocks[d].size();
      // per-node factor fields of the crossing lines (zero elsewhere), FP64
      // and, for the mixed form, FP32 (1/bet and gam): filled on the device
      double *fb = nullptr, *fg = nullptr;
      float *fb32 = nullptr, *fg32 = nullptr;
      if (!blocks[d].empty()) {
        CUDA_TRY(h->put_padded(&fb, (const double*)nullptr, (size_t)N, fpad));
        CUDA_TRY(h->put_padded(&fg, (const double*)nullptr, (size_t)N, fpad));
        CUDA_TRY(h->put_padded(&fb32, (const float*)nullptr, (size_t)N, fpad));
        CUDA_TRY(h->put_padded(&fg32, (const float*)nullptr, (size_t)N, fpad));
      }
      D.fbet[d] = fb;
      D.fgam[d] = fg;
      D.fib32[d] = fb32;
      D.fgam32[d] = fg32;
      // the same factors in FP32 for the mixed-precision sweeps, as 1/bet and gam
      for (int side = 0; side < 2; side++) {
        std::vector<float> p32(ptab[d][side].size());
        for (size_t j = 0; j + 1 < p32.size(); j += 2) {
          p32[j] = (float)(1.0 / ptab[d][side][j]);
          p32[j + 1] = (float)ptab[d][side][j + 1];
        }
        float* pt = nullptr;
        CUDA_TRY(h->put(&pt, p32.data(), p32.size()));
        D.ptab32[d][side] = pt;
      }
      float* rb32 = nullptr;
      CUDA_TRY(h->put(&rb32, (const float*)nullptr, 3 * blocks[d].size()));
      D.rblk32[d] = rb32;
    }
    {
      const size_t t32 = std::min((size_t)D.sweep_blocks * (size_t)mts::mixed_sweep_threads(),
                                  (size_t)maxlines + (size_t)mts::mixed_sweep_threads());
      CUDA_TRY(h->put_padded(&D.r32, (const float*)nullptr, (size_t)N, fpad));
      CUDA_TRY(h->put_padded(&D.dp32, (const float*)nullptr, (size_t)nmax * t32, (size_t)mts::kRowPad * t32));
      D.precision = 0;
    }
    uint8_t* dtag = nullptr;
    // (slack past the end: the fast form's bulk copies of tag rows may run
    // past the last row of the last plane)
    CUDA_TRY(h->put_padded(&dtag, tag8.data(), tag8.size(), fpad));
    D.tag = dtag;
    {
      long long* dm = nullptr;
      CUDA_TRY(h->put(&dm, mibn.empty() ? nullptr : mibn.data(), mibn.size()));
      D.mibnode = dm;
      D.nmibnode = (int)mibn.size();
    }
    for (int d = 0; d < 3; d++) {
      uint8_t* ls = nullptr;
      CUDA_TRY(h->put(&ls, lside[d].data(), lside[d].size()));
      D.lside[d] = ls;
    }
    for (int d = 0; d < 3; d++) {
      double *a = nullptr, *s = nullptr, *c = nullptr;
      CUDA_TRY(h->put(&a, axv[d].data(), axv[d].size()));
      CUDA_TRY(h->put(&s, s2v[d].data(), s2v[d].size()));
      CUDA_TRY(h->put(&c, c2v[d].data(), c2v[d].size()));
      D.ax[d] = a;
      D.s2[d] = s;
      D.c2[d] = c;
      int32_t* bs = nullptr;
      mts::MibBlock* bl = nullptr;
      CUDA_TRY(h->put(&bs, bstart[d].data(), bstart[d].size()));
      CUDA_TRY(h->put(&bl, blocks[d].empty() ? nullptr : blocks[d].data(), blocks[d].size()));
      D.bstart[d] = bs;
      D.blk[d] = bl;
    }
    mts::CrossConst* dcc = nullptr;
    CUDA_TRY(h->put(&dcc, cc.empty() ? nullptr : cc.data(), cc.size()));
    D.cc = dcc;
    CUDA_TRY(h->put(&D.jv, (const double2*)nullptr, h->cross.size()));
    CUDA_TRY(h->put(&D.status, (const int*)nullptr, 1));
    CUDA_TRY(h->put(&h->norm_part, (const double*)nullptr, (size_t)3 * h->norm_nb));
    CUDA_TRY(h->put(&h->norm_out, (const double*)nullptr, 3));
    return MTS_OK;
  };
  h->sizing = true;
  h->planned = 0;
  mts_status placed = place_all();
  h->sizing = false;
  if (placed) return placed;
  CUDA_TRY(h->reserve(h->planned));
  placed = place_all();
  if (placed) return placed;
  CUDA_TRY(cudaMemsetAsync(D.status, 0, sizeof(int), h->stream));
  {
    // the crossing lines' per-node factors; a zero pivot raises D.status
    mts::launch_factor_lines(D, D.status, h->stream);
    CUDA_TRY(cudaGetLastError());
    int zero_pivot = 0;
    CUDA_TRY(cudaMemcpyAsync(&zero_pivot, D.status, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    if (zero_pivot) return fail(MTS_ERR_ZERO_PIVOT, "zero pivot in a line factorisation");
    CUDA_TRY(cudaMemsetAsync(D.status, 0, sizeof(int), h->stream));
  }
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->t = p.t0;
  return MTS_OK;
}

mts_status check_params(const mts_grid* grid, const mts_params* p) {
  if (!grid || !p) return fail(MTS_ERR_ARG, "null argument");
  if (grid->nx < 3 || grid->ny < 3 || grid->nz < 3) return fail(MTS_ERR_ARG, "grid needs at least 3 nodes per axis");
  if ((long long)grid->nx * grid->ny * grid->nz > (1LL << 40)) return fail(MTS_ERR_ARG, "grid too large");
  if (!(grid->xr > grid->xl) || !(grid->yr > grid->yl) || !(grid->zr > grid->zl))
    return fail(MTS_ERR_ARG, "empty domain");
  if (p->eq != 0 && p->eq != 8) return fail(MTS_ERR_ARG, "eq must be 0 or 8");
  if (p->method < MTS_ADI || p->method > MTS_TS) return fail(MTS_ERR_ARG, "unknown method");
  if (p->mib != 1 && p->mib != 2) return fail(MTS_ERR_ARG, "mib must be 1 or 2");
  if (!(p->dt > 0)) return fail(MTS_ERR_ARG, "dt must be positive");
  if (!(p->beta_in > 0) || !(p->beta_out > 0)) return fail(MTS_ERR_ARG, "beta must be positive");
  if (p->setup != MTS_SETUP_HOST && p->setup != MTS_SETUP_DEVICE) return fail(MTS_ERR_ARG, "setup must be 0 or 1");
  return MTS_OK;
}

// The device setup on a stream of its own (created and destroyed here).
mts_status device_setup(const mts::Grid& g, const mts_surface& surf, const mts_params& p, std::vector<int8_t>& tags,
                        std::vector<mts_crossing>& cross, mts::SetupReport* rep) {
  if (surf.kind != MTS_SURFACE_ELLIPSOID && surf.kind != MTS_SURFACE_TORUS)
    return fail(MTS_ERR_ARG, "unknown surface kind");
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  keep_pool(dev);
  cudaStream_t st = nullptr;
  CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  std::string why;
  mts_status r = mts::setup_on_device(g, surf, p.beta_in, p.beta_out, p.mib, st, tags, cross, rep, &why);
  cudaStreamDestroy(st);
  if (r) return fail(r, why);
  return MTS_OK;
}

mts_status check_device() {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) return fail(MTS_ERR_NO_DEVICE, "no CUDA device visible");
  return MTS_OK;
}

mts_status enqueue_step(mts_problem* h, double t_prev, double t_half, double t_next) {
  mts::StepTimes T;
  T.e_prev = std::exp(-t_prev);
  T.e_half = std::exp(-t_half);
  T.e_next = std::exp(-t_next);
  cudaEvent_t* ev = nullptr;
  if (h->profiling) {
    if (h->ev_free.empty()) {
      std::array<cudaEvent_t, 2 * mts::kProfileSlots> a;
      for (auto& e : a) {
        cudaError_t ce = cudaEventCreate(&e);
        if (ce != cudaSuccess) return fail(MTS_ERR_CUDA, std::string("cudaEventCreate: ") + cudaGetErrorString(ce));
      }
      h->ev_free.push_back(a);
    }
    h->ev_busy.push_back(h->ev_free.back());
    h->ev_free.pop_back();
    ev = h->ev_busy.back().data();
  }
  CUDA_TRY(ensure_side_stream(h));
  if (h->dev.precision == 2)
    h->launches += mts::launch_step_fast(h->dev, T, h->u0, h->u1, h->stream, ev, &h->side);
  else if (h->dev.precision == 1)
    h->launches += mts::launch_step_mixed(h->dev, T, h->u0, h->stream, ev, &h->side);
  else
    h->launches += mts::launch_step(h->dev, T, h->u0, h->u1, h->stream, ev, &h->side);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(MTS_ERR_CUDA, std::string("step launch: ") + cudaGetErrorString(e));
  h->t = t_next;
  return MTS_OK;
}

mts_status advance(mts_problem* h, int nsteps) {
  const double dt = h->prm.dt;
  for (int s = 0; s < nsteps; s++) {
    double t1 = h->t + dt;
    mts_status st = enqueue_step(h, t1 - dt, t1 - 0.5 * dt, t1);
    if (st) return st;
  }
  return MTS_OK;
}

mts_status sync_status(mts_problem* h) {
  int flag = 0;
  CUDA_TRY(cudaMemcpyAsync(&flag, h->dev.status, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  if (flag & 1) return fail(MTS_ERR_ZERO_PIVOT, "zero pivot in a line solve");
  return MTS_OK;
}

}  // namespace

extern "C" {

int32_t mts_version(void) { return 100; }

const char* mts_last_error(void) { return g_last_error.c_str(); }

mts_status mts_create(const mts_grid* grid, const mts_surface* surface, const mts_params* params,
                      mts_handle* out) {
  if (!out || !surface) return fail(MTS_ERR_ARG, "null argument");
  *out = nullptr;
  mts_status st = check_params(grid, params);
  if (st) return st;
  st = check_device();
  if (st) return st;
  std::unique_ptr<mts::Surface> surf(mts::make_surface(*surface));
  if (!surf) return fail(MTS_ERR_ARG, "unknown surface kind");
  std::unique_ptr<mts_problem> h(new mts_problem());
  cudaGetDevice(&h->device);
  h->g = mts::make_grid(*grid);
  h->prm = *params;
  if (params->setup == MTS_SETUP_DEVICE) {
    st = device_setup(h->g, *surface, *params, h->tags, h->cross, &h->rep);
    if (st) return st;
  } else {
    st = mts::build_tags(h->g, *surf, h->tags);
    if (st) return fail(st, "a grid node lies on the interface");
    st = mts::build_crossings(h->g, h->tags, *surf, params->beta_in, params->beta_out, params->mib, h->cross,
                              &h->rep);
    if (st) return fail(st, "interface setup failed (root finding, coherent corners, open surface or singular LU)");
  }
  st = finish_create(h.get());
  if (st) return st;
  *out = h.release();
  return MTS_OK;
}

mts_status mts_create_from_crossings(const mts_grid* grid, const int8_t* tags, const mts_crossing* crossings,
                                     int32_t ncrossings, const mts_params* params, mts_handle* out) {
  if (!out || !tags || (ncrossings > 0 && !crossings) || ncrossings < 0) return fail(MTS_ERR_ARG, "null argument");
  *out = nullptr;
  mts_status st = check_params(grid, params);
  if (st) return st;
  st = check_device();
  if (st) return st;
  std::unique_ptr<mts_problem> h(new mts_problem());
  cudaGetDevice(&h->device);
  h->g = mts::make_grid(*grid);
  h->prm = *params;
  h->tags.assign(tags, tags + h->g.nodes());
  for (int8_t v : h->tags)
    if (v != 1 && v != -1) return fail(MTS_ERR_ARG, "tags must be +1 or -1");
  h->cross.assign(crossings, crossings + ncrossings);
  for (const mts_crossing& c : h->cross) h->rep.corner_pairs += c.id < 0;
  h->rep.corner_pairs /= 2;
  st = finish_create(h.get());
  if (st) return st;
  *out = h.release();
  return MTS_OK;
}

mts_status mts_setup_host(const mts_grid* grid, const mts_surface* surface, const mts_params* params,
                          int8_t* tags, mts_crossing* out, int32_t capacity, int32_t* count, int64_t counts[2]) {
  if (!surface || !count) return fail(MTS_ERR_ARG, "null argument");
  mts_status st = check_params(grid, params);
  if (st) return st;
  std::unique_ptr<mts::Surface> surf(mts::make_surface(*surface));
  if (!surf) return fail(MTS_ERR_ARG, "unknown surface kind");
  mts::Grid g = mts::make_grid(*grid);
  std::vector<int8_t> tg;
  st = mts::build_tags(g, *surf, tg);
  if (st) return fail(st, "a grid node lies on the interface");
  std::vector<mts_crossing> cr;
  mts::SetupReport rep;
  st = mts::build_crossings(g, tg, *surf, params->beta_in, params->beta_out, params->mib, cr, &rep);
  if (st) return fail(st, "interface setup failed (root finding, coherent corners, open surface or singular LU)");
  if (tags) std::memcpy(tags, tg.data(), tg.size());
  *count = (int32_t)cr.size();
  if (out && capacity >= (int32_t)cr.size()) std::memcpy(out, cr.data(), cr.size() * sizeof(mts_crossing));
  if (counts) {
    counts[0] = rep.corner_pairs;
    counts[1] = rep.singular_warnings;
  }
  return MTS_OK;
}

mts_status mts_setup_device(const mts_grid* grid, const mts_surface* surface, const mts_params* params,
                            int8_t* tags, mts_crossing* out, int32_t capacity, int32_t* count, int64_t counts[2]) {
  if (!surface || !count) return fail(MTS_ERR_ARG, "null argument");
  mts_status st = check_params(grid, params);
  if (st) return st;
  st = check_device();
  if (st) return st;
  mts::Grid g = mts::make_grid(*grid);
  std::vector<int8_t> tg;
  std::vector<mts_crossing> cr;
  mts::SetupReport rep;
  st = device_setup(g, *surface, *params, tg, cr, &rep);
  if (st) return st;
  if (cr.size() > (size_t)INT32_MAX) return fail(MTS_ERR_ARG, "more crossings than an int32 count holds");
  if (tags) std::memcpy(tags, tg.data(), tg.size());
  *count = (int32_t)cr.size();
  if (out && capacity >= (int32_t)cr.size()) std::memcpy(out, cr.data(), cr.size() * sizeof(mts_crossing));
  if (counts) {
    counts[0] = rep.corner_pairs;
    counts[1] = rep.singular_warnings;
  }
  return MTS_OK;
}

mts_status mts_destroy(mts_handle h) {
  if (!h) return fail(MTS_ERR_ARG, "null handle");
  cudaStreamSynchronize(h->stream);
  delete h;
  return MTS_OK;
}

mts_status mts_initialize(mts_handle h) {
  if (!h) return fail(MTS_ERR_ARG, "null handle");
  h->launches += mts::launch_initialize(h->dev, std::exp(-h->t), h->u0, h->stream);
  CUDA_TRY(cudaGetLastError());
  return MTS_OK;
}

mts_status mts_set_solution(mts_handle h, const double* u) {
  if (!h || !u) return fail(MTS_ERR_ARG, "null argument");
  CUDA_TRY(cudaMemcpyAsync(h->u0, u, sizeof(double) * (size_t)h->g.nodes(), cudaMemcpyHostToDevice, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return MTS_OK;
}

mts_status mts_get_solution(mts_handle h, double* u) {
  if (!h || !u) return fail(MTS_ERR_ARG, "null argument");
  CUDA_TRY(cudaMemcpyAsync(u, h->u0, sizeof(double) * (size_t)h->g.nodes(), cudaMemcpyDeviceToHost, h->stream));
  return sync_status(h);
}

mts_status mts_solve_2nd(mts_handle h, double t_prev, double t_half, double t_next) {
  if (!h) return fail(MTS_ERR_ARG, "null handle");
  return enqueue_step(h, t_prev, t_half, t_next);
}

mts_status mts_advance(mts_handle h, int32_t nsteps) {
  if (!h || nsteps < 0) return fail(MTS_ERR_ARG, "bad argument");
  return advance(h, nsteps);
}

// Batched stepping.  Handles of the plain form are grouped by method; a
// group advances with one launch per kernel of the step for all its problems
// (mts::launch_step_batch: each CTA of a launch carries its problem and its
// place in that problem's own grid, so every problem computes exactly what
// its own launches would).  Mixed-precision handles step on their own
// streams.  Every handle reads its step's exp(-t) factors from a table
// computed here exactly as advance() computes them, indexed by a device step
// counter that each step advances, so batching changes no bit of any result.
mts_status mts_batch_advance(const mts_handle* hs, int32_t n, int32_t nsteps) {
  if (!hs || n < 1 || nsteps < 0) return fail(MTS_ERR_ARG, "bad argument");
  std::vector<int32_t> counts((size_t)n, nsteps);
  return mts_batch_advance_steps(hs, counts.data(), n);
}

mts_status mts_batch_advance_steps(const mts_handle* hs, const int32_t* counts, int32_t n) {
  if (!hs || !counts || n < 1) return fail(MTS_ERR_ARG, "bad argument");
  int32_t nsteps = 0;
  for (int i = 0; i < n; i++) {
    if (counts[i] < 0) return fail(MTS_ERR_ARG, "negative step count");
    nsteps = std::max(nsteps, counts[i]);
  }
  for (int i = 0; i < n; i++) {
    if (!hs[i]) return fail(MTS_ERR_ARG, "null handle in batch");
    for (int k = 0; k < i; k++)
      if (hs[k] == hs[i]) return fail(MTS_ERR_ARG, "a handle appears twice in the batch");
    if (hs[i]->device != hs[0]->device) return fail(MTS_ERR_ARG, "batch handles live on different devices");
    if (hs[i]->profiling) return fail(MTS_ERR_ARG, "profiling is on for a batch handle");
  }
  if (nsteps == 0) return MTS_OK;
  std::vector<void*> dev_alloc;  // freed at the end
  std::vector<cudaStream_t> streams;
  std::vector<double> t_end((size_t)n);
  mts_status st = MTS_OK;
  auto cleanup = [&]() {
    for (cudaStream_t q : streams) cudaStreamDestroy(q);
    for (void* q : dev_alloc) cudaFreeAsync(q, hs[0]->stream);
    for (int i = 0; i < n; i++) {
      hs[i]->dev.tsched = nullptr;
      hs[i]->dev.tstep = nullptr;
    }
  };
#define BATCH_TRY(call)                                                                          \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess) {                                                                     \
      st = fail(e_ == cudaErrorMemoryAllocation ? MTS_ERR_OOM : MTS_ERR_CUDA,                    \
                std::string(#call) + ": " + cudaGetErrorString(e_));                             \
      cleanup();                                                                                 \
      return st;                                                                                 \
    }                                                                                            \
  } while (0)
  auto dev_upload = [&](const void* src, size_t bytes, cudaStream_t q, void** out) -> cudaError_t {
    *out = nullptr;
    cudaError_t e = cudaMallocAsync(out, bytes ? bytes : 16, q);
    if (e != cudaSuccess) return e;
    dev_alloc.push_back(*out);
    return bytes ? cudaMemcpyAsync(*out, src, bytes, cudaMemcpyHostToDevice, q) : cudaSuccess;
  };
  // step tables and counters, one allocation each for the whole batch
  {
    std::vector<double> tab(3 * (size_t)nsteps * (size_t)n);
    for (int i = 0; i < n; i++) {
      mts_problem* h = hs[i];
      double t = h->t;
      const double dt = h->prm.dt;
      double* row = tab.data() + 3 * (size_t)nsteps * (size_t)i;
      for (int k = 0; k < counts[i]; k++) {
        const double t1 = t + dt;
        row[3 * (size_t)k] = std::exp(-(t1 - dt));
        row[3 * (size_t)k + 1] = std::exp(-(t1 - 0.5 * dt));
        row[3 * (size_t)k + 2] = std::exp(-t1);
        t = t1;
      }
      t_end[(size_t)i] = t;
      BATCH_TRY(cudaStreamSynchronize(h->stream));  // the handle's earlier work is done
    }
    std::vector<int> zeros((size_t)n, 0);
    void *tab_d = nullptr, *step_d = nullptr;
    cudaStream_t q0 = hs[0]->stream;
    BATCH_TRY(dev_upload(tab.data(), tab.size() * sizeof(double), q0, &tab_d));
    BATCH_TRY(dev_upload(zeros.data(), zeros.size() * sizeof(int), q0, &step_d));
    BATCH_TRY(cudaStreamSynchronize(q0));
    for (int i = 0; i < n; i++) {
      hs[i]->dev.tsched = (const double*)tab_d + 3 * (size_t)nsteps * (size_t)i;
      hs[i]->dev.tstep = (int*)step_d + i;
      hs[i]->dev.tstop = counts[i];
    }
  }
  // Problems whose lines fill the GPU by themselves (256 per SM or more in
  // every direction), and mixed-precision ones, step on their own streams
  // with their own launch shapes (in a batched launch a large grid would run
  // with the small shared-SM shape); the rest are batched per method.  Every
  // group and every solo problem is on its own stream, so they all run at
  // once; the results are those of stepping each problem alone either way.
  auto fills_gpu = [&](const mts_problem* h) {
    long long lines = line_count(h->g, 0);
    for (int d = 1; d < 3; d++) lines = std::min(lines, (long long)line_count(h->g, d));
    return lines >= 256LL * h->dev.sweep_blocks;
  };
  // mixed-form ADI problems whose lines fit the batched segmented solves
  // (at most 160 rows) batch in a group of their own
  auto mixed_batchable = [&](const mts_problem* h) {
    if (h->dev.precision != 1 || h->prm.method != MTS_ADI) return false;
    for (int d = 0; d < 3; d++)
      if (mts::mixed_batch_class(h->dev, d) < 0) return false;
    return true;
  };
  auto solo = [&](int i) {
    return fills_gpu(hs[i]) || (hs[i]->dev.precision != 0 && !mixed_batchable(hs[i]));
  };
  // plain handles by method: one batched launch sequence per group
  for (int method = 0; method < 4; method++) {
    std::vector<int> mem;
    for (int i = 0; i < n; i++)
      if (!solo(i) && hs[i]->dev.precision == 0 && hs[i]->prm.method == method) mem.push_back(i);
    if (mem.empty()) continue;
    cudaStream_t q = nullptr;
    BATCH_TRY(cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking));
    streams.push_back(q);
    std::vector<mts::Dev> recs;
    mts::BatchPlan plan{};
    plan.method = method;
    plan.n = (int)mem.size();
    std::vector<mts::BatchItem> jumps, rows, mib, blk[3], sw[3];
    auto add = [](std::vector<mts::BatchItem>& v, int p, unsigned ncta) {
      for (unsigned c = 0; c < ncta; c++) v.push_back(mts::BatchItem{p, (int32_t)c, (int32_t)ncta, 0});
    };
    for (int k = 0; k < (int)mem.size(); k++) {
      const mts::Dev& d = hs[mem[(size_t)k]]->dev;
      recs.push_back(d);
      plan.nmax = std::max(plan.nmax, std::max(d.nx, std::max(d.ny, d.nz)));
      if (d.ncross > 0) add(jumps, k, mts::jumps_grid(d));
      add(rows, k, mts::pointwise_rows_grid(d));
      if (d.nmibnode > 0) add(mib, k, mts::mib_grid(d));
      for (int dd = 0; dd < 3; dd++) {
        if (d.nblk[dd] > 0) add(blk[dd], k, mts::block_grid(d, dd));
        add(sw[dd], k, mts::batch_sweep_grid(d, dd));
      }
    }
    void* tmp = nullptr;
    BATCH_TRY(dev_upload(recs.data(), recs.size() * sizeof(mts::Dev), q, &tmp));
    plan.Ps = (const mts::Dev*)tmp;
    auto up = [&](std::vector<mts::BatchItem>& v, const mts::BatchItem** dst, int* cnt) -> cudaError_t {
      *cnt = (int)v.size();
      void* p = nullptr;
      cudaError_t e = dev_upload(v.data(), v.size() * sizeof(mts::BatchItem), q, &p);
      *dst = (const mts::BatchItem*)p;
      return e;
    };
    BATCH_TRY(up(jumps, &plan.jumps, &plan.njumps));
    BATCH_TRY(up(rows, &plan.rows, &plan.nrows));
    BATCH_TRY(up(mib, &plan.mib, &plan.nmib));
    for (int dd = 0; dd < 3; dd++) {
      BATCH_TRY(up(blk[dd], &plan.blk[dd], &plan.nblk[dd]));
      BATCH_TRY(up(sw[dd], &plan.sw[dd], &plan.nsw[dd]));
    }
    // the host vectors must outlive the asynchronous uploads
    BATCH_TRY(cudaStreamSynchronize(q));
    int gsteps = 0;  // the group's longest count: later steps skip finished problems
    for (int i : mem) gsteps = std::max(gsteps, counts[i]);
    int64_t launches = 0;
    for (int k = 0; k < gsteps; k++) launches += mts::launch_step_batch(plan, q);
    BATCH_TRY(cudaGetLastError());
    for (int i : mem) hs[i]->launches += launches;
  }
  // the mixed-form group: one batched launch sequence of the mixed step
  {
    std::vector<int> mem;
    for (int i = 0; i < n; i++)
      if (!solo(i) && hs[i]->dev.precision == 1) mem.push_back(i);
    if (!mem.empty()) {
      cudaStream_t q = nullptr;
      BATCH_TRY(cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking));
      streams.push_back(q);
      std::vector<mts::Dev> recs;
      mts::MixedBatchPlan plan{};
      plan.n = (int)mem.size();
      std::vector<mts::BatchItem> jumps, rows, mib, blk[3], line[3][2];
      auto add = [](std::vector<mts::BatchItem>& v, int p, unsigned ncta) {
        for (unsigned c = 0; c < ncta; c++) v.push_back(mts::BatchItem{p, (int32_t)c, (int32_t)ncta, 0});
      };
      for (int k = 0; k < (int)mem.size(); k++) {
        const mts::Dev& d = hs[mem[(size_t)k]]->dev;
        recs.push_back(d);
        if (d.ncross > 0) add(jumps, k, mts::jumps_grid(d));
        add(rows, k, mts::pointwise_rows_grid(d));
        if (d.nmibnode > 0) add(mib, k, mts::mib_grid(d));
        for (int dd = 0; dd < 3; dd++) {
          if (d.nblk[dd] > 0) add(blk[dd], k, mts::block_grid(d, dd));
          add(line[dd][mts::mixed_batch_class(d, dd)], k, mts::mixed_line_ctas(d, dd));
        }
      }
      void* tmp = nullptr;
      BATCH_TRY(dev_upload(recs.data(), recs.size() * sizeof(mts::Dev), q, &tmp));
      plan.Ps = (const mts::Dev*)tmp;
      auto up = [&](std::vector<mts::BatchItem>& v, const mts::BatchItem** dst, int* cnt) -> cudaError_t {
        *cnt = (int)v.size();
        void* p = nullptr;
        cudaError_t e = dev_upload(v.data(), v.size() * sizeof(mts::BatchItem), q, &p);
        *dst = (const mts::BatchItem*)p;
        return e;
      };
      BATCH_TRY(up(jumps, &plan.jumps, &plan.njumps));
      BATCH_TRY(up(rows, &plan.rows, &plan.nrows));
      BATCH_TRY(up(mib, &plan.mib, &plan.nmib));
      for (int dd = 0; dd < 3; dd++) {
        BATCH_TRY(up(blk[dd], &plan.blk[dd], &plan.nblk[dd]));
        for (int c = 0; c < 2; c++) BATCH_TRY(up(line[dd][c], &plan.line[dd][c], &plan.nline[dd][c]));
      }
      BATCH_TRY(cudaStreamSynchronize(q));  // the host vectors must outlive the uploads
      int gsteps = 0;
      for (int i : mem) gsteps = std::max(gsteps, counts[i]);
      int64_t launches = 0;
      for (int k = 0; k < gsteps; k++) launches += mts::launch_step_batch_mixed(plan, q);
      BATCH_TRY(cudaGetLastError());
      for (int i : mem) hs[i]->launches += launches;
    }
  }
  // solo problems: their own steps on their own streams
  for (int i = 0; i < n; i++) {
    mts_problem* h = hs[i];
    if (!solo(i)) continue;
    BATCH_TRY(ensure_side_stream(h));
    for (int k = 0; k < counts[i]; k++) {
      mts::StepTimes T{0, 0, 0};  // unused: the kernels read the table
      if (h->dev.precision == 2)
        h->launches += mts::launch_step_fast(h->dev, T, h->u0, h->u1, h->stream, nullptr, &h->side);
      else if (h->dev.precision == 1)
        h->launches += mts::launch_step_mixed(h->dev, T, h->u0, h->stream, nullptr, &h->side);
      else
        h->launches += mts::launch_step(h->dev, T, h->u0, h->u1, h->stream, nullptr, &h->side);
      mts::launch_tick(h->dev, h->stream);
      h->launches++;
    }
    BATCH_TRY(cudaGetLastError());
  }
  for (cudaStream_t q : streams) BATCH_TRY(cudaStreamSynchronize(q));
  for (int i = 0; i < n; i++) {
    mts_problem* h = hs[i];
    if (solo(i)) {
      mts_status s2 = sync_status(h);
      if (s2 && !st) st = s2;
    }
    h->t = t_end[(size_t)i];
  }
  cleanup();
#undef BATCH_TRY
  return st;
}

mts_status mts_advance_host(mts_handle h, const double* u_in, double* u_out, int32_t nsteps) {
  if (!h || !u_in || !u_out || nsteps < 0) return fail(MTS_ERR_ARG, "bad argument");
  const size_t bytes = sizeof(double) * (size_t)h->g.nodes();
  CUDA_TRY(cudaMemcpyAsync(h->u0, u_in, bytes, cudaMemcpyHostToDevice, h->stream));
  mts_status st = advance(h, nsteps);
  if (st) return st;
  CUDA_TRY(cudaMemcpyAsync(u_out, h->u0, bytes, cudaMemcpyDeviceToHost, h->stream));
  return sync_status(h);
}

mts_status mts_norms(mts_handle h, double* lmax, double* l2, int32_t* argmax3) {
  if (!h) return fail(MTS_ERR_ARG, "null handle");
  h->launches += mts::launch_norms(h->dev, std::exp(-h->t), h->u0, h->norm_part, h->norm_nb, h->norm_out, h->stream);
  CUDA_TRY(cudaGetLastError());
  double r[3] = {0.0, 0.0, 0.0};
  CUDA_TRY(cudaMemcpyAsync(r, h->norm_out, 3 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  mts_status st = sync_status(h);
  if (st != MTS_OK) return st;
  if (lmax) *lmax = r[0];
  if (l2) *l2 = r[2];
  if (argmax3) {
    long long key = (long long)r[1];
    argmax3[2] = (int32_t)(key % h->g.nz);
    key /= h->g.nz;
    argmax3[1] = (int32_t)(key % h->g.ny);
    argmax3[0] = (int32_t)(key / h->g.ny);
  }
  return st;
}

// Norms with no allocation.  Who needs it: a host program that keeps its own
// fields in a device pool it manages (a framework's caching allocator that
// has reserved most of HBM, a service under a hard memory cap) and checks
// their error mid-run, where a cudaMalloc may fail for want of free memory
// and a cudaFree would synchronize the whole device.  It reuses nothing the
// handle allocated for mts_norms: the reduction scratch is the module's
// static array, whose device address is looked up once per device, with that
// device current, and then cached.  The first call on a device therefore
// does one runtime lookup (which may load the module); make it before any
// stream capture starts on that device.
mts_status mts_norms_noalloc(mts_handle h, const double* u_dev, double t, double* lmax, double* l2,
                             int32_t* argmax3) {
  if (!h) return fail(MTS_ERR_ARG, "null handle");
  const int nb = mts::norms_blocks(h->dev);
  if (nb > mts::kNoAllocMaxBlocks)
    return fail(MTS_ERR_ARG, "mts_norms_noalloc: a grid of " + std::to_string(h->g.nodes()) + " nodes needs " +
                                 std::to_string(nb) + " reduction blocks; the static scratch holds " +
                                 std::to_string(mts::kNoAllocMaxBlocks) + " (grids of at most " +
                                 std::to_string((long long)mts::kNoAllocMaxBlocks * 2048) + " nodes)");
  // The scratch's address is looked up on every call (cheap once the module
  // is loaded), so a device reset or a new primary context between calls
  // never leaves a stale address behind.
  double* scratch = nullptr;
  {
    int cur = -1;
    CUDA_TRY(cudaGetDevice(&cur));
    if (cur != h->device) CUDA_TRY(cudaSetDevice(h->device));
    cudaError_t e = mts::noalloc_scratch_address(&scratch);
    if (cur != h->device) cudaSetDevice(cur);
    if (e != cudaSuccess)
      return fail(MTS_ERR_CUDA, std::string("cudaGetSymbolAddress(static norms scratch): ") + cudaGetErrorString(e));
  }
  const double* u = u_dev ? u_dev : h->u0;
  const double tt = u_dev ? t : h->t;
  // the ticket counter must start at zero
  CUDA_TRY(cudaMemsetAsync(scratch, 0, sizeof(unsigned), h->stream));
  h->launches += mts::launch_norms_noalloc(h->dev, std::exp(-tt), u, scratch, nb, h->stream);
  CUDA_TRY(cudaGetLastError());
  double r[3] = {0.0, 0.0, 0.0};
  CUDA_TRY(cudaMemcpyAsync(r, scratch + 32, sizeof r, cudaMemcpyDeviceToHost, h->stream));
  mts_status st = sync_status(h);
  if (st != MTS_OK) return st;
  if (lmax) *lmax = r[0];
  if (l2) *l2 = r[2];
  if (argmax3) {
    long long key = (long long)r[1];
    argmax3[2] = (int32_t)(key % h->g.nz);
    key /= h->g.nz;
    argmax3[1] = (int32_t)(key % h->g.ny);
    argmax3[0] = (int32_t)(key / h->g.ny);
  }
  return st;
}

// The crossing records sorted by (direction, line, position), the order of
// the report loops of Refresh_Fp / Error_Fp and Refresh_Jump / Error_Jump
// within a direction, on the device with their handle indices, corner-pair
// roles and an error buffer of two doubles per record; built on first use.
static mts_status report_tables(mts_handle h) {
  const int n = (int)h->cross.size();
  if (n > 0 && !h->fp_cr) {
    // the records sorted by (direction, line, position), the order of
    // Refresh_Fp's and Error_Fp's loops within a direction
    std::vector<int32_t>& perm = h->fp_perm;
    perm.resize((size_t)n);
    for (int i = 0; i < n; i++) perm[(size_t)i] = i;
    std::stable_sort(perm.begin(), perm.end(), [&](int32_t a, int32_t b) {
      const mts_crossing &x = h->cross[(size_t)a], &y = h->cross[(size_t)b];
      if (x.dir != y.dir) return x.dir < y.dir;
      if (x.indx1 != y.indx1) return x.indx1 < y.indx1;
      if (x.indx2 != y.indx2) return x.indx2 < y.indx2;
      return x.left_loc < y.left_loc;
    });
    std::vector<mts_crossing> rec((size_t)n);
    std::vector<int8_t> role((size_t)n, 0);
    for (int i = 0; i < n; i++) rec[(size_t)i] = h->cross[(size_t)perm[(size_t)i]];
    for (int i = 0; i < n;) {
      if (rec[(size_t)i].id > 0) {
        i += 1;
        continue;
      }
      if (i + 1 >= n || rec[(size_t)i + 1].id >= 0 || rec[(size_t)i + 1].dir != rec[(size_t)i].dir ||
          rec[(size_t)i + 1].indx1 != rec[(size_t)i].indx1 || rec[(size_t)i + 1].indx2 != rec[(size_t)i].indx2)
        return fail(MTS_ERR_SETUP, "a corner crossing without its pair on the same line");
      role[(size_t)i] = 1;
      role[(size_t)i + 1] = 2;
      i += 2;
    }
    // (the handle takes the buffers only once all of them are in place, so
    // a failed first call leaves nothing half built for the next one)
    mts_crossing* cr = nullptr;
    int32_t* ci = nullptr;
    int8_t* ro = nullptr;
    double* er = nullptr;
    CUDA_TRY(h->put(&cr, rec.data(), rec.size()));
    CUDA_TRY(h->put(&ci, perm.data(), perm.size()));
    CUDA_TRY(h->put(&ro, role.data(), role.size()));
    CUDA_TRY(h->put(&er, (const double*)nullptr, 2 * (size_t)n));
    CUDA_TRY(cudaStreamSynchronize(h->stream));  // the host vectors must outlive the uploads
    h->fp_cr = cr;
    h->fp_ci = ci;
    h->fp_role = ro;
    h->fp_err = er;
  }
  return MTS_OK;
}

mts_status mts_fp_errors(mts_handle h, double* lmax, double* l2) {
  if (!h) return fail(MTS_ERR_ARG, "null handle");
  const int n = (int)h->cross.size();
  mts_status ts = report_tables(h);
  if (ts != MTS_OK) return ts;
  std::vector<double> err(2 * (size_t)n);
  if (n > 0) {
    h->launches += mts::launch_fp_errors(h->dev, h->fp_cr, h->fp_ci, h->fp_role, n, std::exp(-h->t), h->fp_err,
                                         h->stream);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(err.data(), h->fp_err, err.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  }
  mts_status st = sync_status(h);
  if (st != MTS_OK) return st;
  // Error_Fp's loops: directions z, y, x; per crossing its left error, then
  // its right one
  double fmax = 0, sum = 0;
  long long no = 0;
  for (int d = 2; d >= 0; d--)
    for (int i = 0; i < n; i++) {
      if (h->cross[(size_t)h->fp_perm[(size_t)i]].dir != d) continue;
      const double el = err[2 * (size_t)i], er = err[2 * (size_t)i + 1];
      no += 2;
      sum += el * el;
      sum += er * er;
      if (std::abs(el) > fmax) fmax = std::abs(el);
      if (std::abs(er) > fmax) fmax = std::abs(er);
    }
  if (lmax) *lmax = fmax;
  if (l2) *l2 = std::sqrt(sum / (double)no);
  return MTS_OK;
}

mts_status mts_jump_errors(mts_handle h, double* lmax, double* l2) {
  if (!h) return fail(MTS_ERR_ARG, "null handle");
  const int n = (int)h->cross.size();
  mts_status ts = report_tables(h);
  if (ts != MTS_OK) return ts;
  std::vector<double> err((size_t)n);
  if (n > 0) {
    h->launches += mts::launch_jump_errors(h->dev, h->fp_cr, h->fp_ci, n, std::exp(-h->t), h->fp_err, h->stream);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(err.data(), h->fp_err, err.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  }
  mts_status st = sync_status(h);
  if (st != MTS_OK) return st;
  // Error_Jump's loops: directions z, y, x, one error per crossing
  double jmax = 0, sum = 0;
  long long no = 0;
  for (int d = 2; d >= 0; d--)
    for (int i = 0; i < n; i++) {
      if (h->cross[(size_t)h->fp_perm[(size_t)i]].dir != d) continue;
      const double e = err[(size_t)i];
      no += 1;
      sum += e * e;
      if (std::abs(e) > jmax) jmax = std::abs(e);
    }
  if (lmax) *lmax = jmax;
  if (l2) *l2 = std::sqrt(sum / (double)no);
  return MTS_OK;
}

mts_status mts_get_time(mts_handle h, double* t) {
  if (!h || !t) return fail(MTS_ERR_ARG, "null argument");
  *t = h->t;
  return MTS_OK;
}

mts_status mts_set_time(mts_handle h, double t) {
  if (!h) return fail(MTS_ERR_ARG, "null handle");
  h->t = t;
  return MTS_OK;
}

mts_status mts_synchronize(mts_handle h) {
  if (!h) return fail(MTS_ERR_ARG, "null handle");
  return sync_status(h);
}

mts_status mts_get_counts(mts_handle h, int64_t counts[8]) {
  if (!h || !counts) return fail(MTS_ERR_ARG, "null argument");
  for (int d = 0; d < 3; d++) {
    counts[d] = h->ncr[d];
    counts[3 + d] = h->nblk[d];
  }
  counts[6] = h->rep.corner_pairs;
  counts[7] = h->rep.singular_warnings;
  return MTS_OK;
}

mts_status mts_export_tags(mts_handle h, int8_t* tags) {
  if (!h || !tags) return fail(MTS_ERR_ARG, "null argument");
  std::memcpy(tags, h->tags.data(), h->tags.size());
  return MTS_OK;
}

mts_status mts_export_crossings(mts_handle h, mts_crossing* out, int32_t capacity, int32_t* count) {
  if (!h || !count) return fail(MTS_ERR_ARG, "null argument");
  *count = (int32_t)h->cross.size();
  if (out) {
    if (capacity < (int32_t)h->cross.size()) return fail(MTS_ERR_ARG, "capacity too small");
    std::memcpy(out, h->cross.data(), h->cross.size() * sizeof(mts_crossing));
  }
  return MTS_OK;
}

mts_status mts_get_launch_count(mts_handle h, int64_t* launches) {
  if (!h || !launches) return fail(MTS_ERR_ARG, "null argument");
  *launches = h->launches;
  return MTS_OK;
}

mts_status mts_get_device_bytes(mts_handle h, int64_t* bytes) {
  if (!h || !bytes) return fail(MTS_ERR_ARG, "null argument");
  *bytes = h->device_bytes;
  return MTS_OK;
}

mts_status mts_set_profiling(mts_handle h, int32_t on) {
  if (!h) return fail(MTS_ERR_ARG, "null handle");
  h->profiling = on != 0;
  return MTS_OK;
}

mts_status mts_profile_read(mts_handle h, double ms[8], int64_t launches[8]) {
  if (!h) return fail(MTS_ERR_ARG, "null handle");
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  for (auto& a : h->ev_busy) {
    for (int k = 0; k < h->slots(); k++) {
      float v = 0;
      CUDA_TRY(cudaEventElapsedTime(&v, a[2 * k], a[2 * k + 1]));
      h->prof_ms[k] += v;
      h->prof_n[k] += 1;
    }
    h->ev_free.push_back(a);
  }
  h->ev_busy.clear();
  for (int k = 0; k < mts::kProfileSlots; k++) {
    if (ms) ms[k] = h->prof_ms[k];
    if (launches) launches[k] = h->prof_n[k];
    h->prof_ms[k] = 0;
    h->prof_n[k] = 0;
  }
  return MTS_OK;
}

int32_t mts_sweep_shape_count(void) { return mts::sweep_shape_count(); }

mts_status mts_set_sweep_shape(mts_handle h, int32_t sweep, int32_t shape) {
  if (!h || sweep < 0 || sweep > 2 || shape < 0 || shape >= mts::sweep_shape_count())
    return fail(MTS_ERR_ARG, "bad sweep or shape index");
  if (!mts::sweep_shape_fits(shape, std::max(h->g.nx, std::max(h->g.ny, h->g.nz))))
    return fail(MTS_ERR_ARG, "shape needs more shared memory than this grid allows");
  h->dev.shape[sweep] = shape;
  return MTS_OK;
}

mts_status mts_set_precision(mts_handle h, int32_t precision) {
  if (!h) return fail(MTS_ERR_ARG, "null handle");
  if (precision != MTS_PRECISION_PLAIN && precision != MTS_PRECISION_MIXED && precision != MTS_PRECISION_FAST)
    return fail(MTS_ERR_ARG, "precision must be MTS_PRECISION_PLAIN, MTS_PRECISION_MIXED or MTS_PRECISION_FAST");
  if (precision == MTS_PRECISION_FAST) {
    if (h->prm.method != MTS_ADI) return fail(MTS_ERR_ARG, "the fast FP64 form is built for Douglas-ADI only");
    if (!mts::fast_fits(h->g.nx, h->g.ny, h->g.nz))
      return fail(MTS_ERR_ARG, "grid lines too long for the fast FP64 form (at most 544 nodes per axis)");
    if (!h->fast_built) {
      // row tables, line flags, the crossing lines' list and coefficients,
      // the block rows' q and the MIB nodes' block references, once per
      // handle
      mts::Dev& D = h->dev;
      const int nd[3] = {h->g.nx, h->g.ny, h->g.nz};
      uint8_t* fl[3] = {nullptr, nullptr, nullptr};
      for (int d = 0; d < 3; d++) {
        const size_t R = 32 * (size_t)mts::fast_rows_per_lane(nd[d]);
        double* tab = nullptr;
        CUDA_TRY(h->put(&tab, (const double*)nullptr, 2 * (2 * R + 320)));
        D.ftab[d] = tab;
        CUDA_TRY(h->put(&fl[d], (const uint8_t*)nullptr, (size_t)line_count(h->g, d)));
        D.fline[d] = fl[d];
      }
      mts::build_fast_lines(D, fl, h->stream);
      CUDA_TRY(cudaGetLastError());
      for (int d = 0; d < 3; d++) {
        const size_t R = 32 * (size_t)mts::fast_rows_per_lane(nd[d]);
        const size_t nl = (size_t)line_count(h->g, d);
        std::vector<uint8_t> hf(nl);
        CUDA_TRY(cudaMemcpyAsync(hf.data(), fl[d], nl, cudaMemcpyDeviceToHost, h->stream));
        CUDA_TRY(cudaStreamSynchronize(h->stream));
        // listed in memory order (the fast line index first), so that the
        // warps that take neighbouring entries read neighbouring lines
        const int n1 = d == 0 ? h->g.ny : h->g.nx, n2 = d == 2 ? h->g.ny : h->g.nz;
        std::vector<int32_t> list;
        for (int i2 = 0; i2 < n2; i2++)
          for (int i1 = 0; i1 < n1; i1++) {
            const size_t l = (size_t)i1 * n2 + i2;
            if (hf[l] & 1) list.push_back((int32_t)l);
          }
        int32_t* dl = nullptr;
        double *cf = nullptr, *bq = nullptr;
        if (!list.empty()) {
          CUDA_TRY(h->put(&dl, list.data(), list.size()));
          CUDA_TRY(h->put(&cf, (const double*)nullptr, 2 * R * list.size()));
          CUDA_TRY(cudaMemsetAsync(cf, 0, 2 * R * list.size() * sizeof(double), h->stream));
        }
        if (h->nblk[d] > 0) CUDA_TRY(h->put(&bq, (const double*)nullptr, 3 * (size_t)h->nblk[d]));
        D.fcross[d] = dl;
        D.nfcross[d] = (int)list.size();
        D.fcoef[d] = cf;
        D.fbq[d] = bq;
        // the host list must outlive the asynchronous upload
        CUDA_TRY(cudaStreamSynchronize(h->stream));
      }
      int4* ref = nullptr;
      if (D.nmibnode > 0) CUDA_TRY(h->put(&ref, (const int4*)nullptr, (size_t)D.nmibnode));
      D.mibref = ref;
      mts::build_fast_tables(h->dev, h->stream);
      CUDA_TRY(cudaGetLastError());
      CUDA_TRY(cudaStreamSynchronize(h->stream));
      h->fast_built = true;
    }
  }
  if (precision == MTS_PRECISION_MIXED) {
    if (h->prm.method != MTS_ADI) return fail(MTS_ERR_ARG, "the mixed-precision form is built for Douglas-ADI only");
    const int nmax = std::max(h->g.nx, std::max(h->g.ny, h->g.nz));
    if (!mts::mixed_shape_fits(nmax))
      return fail(MTS_ERR_ARG, "grid lines too long for the mixed-precision sweeps' shared memory");
    if (mts::mixed_segments_fit(nmax) && !h->mixed_built) {
      // the segmented solves' per-node coefficients, once per handle
      const size_t N = (size_t)h->g.nodes();
      const int nd[3] = {h->g.nx, h->g.ny, h->g.nz};
      for (int d = 0; d < 3; d++) {
        float *ib = nullptr, *p = nullptr, *q = nullptr, *tab = nullptr;
        CUDA_TRY(h->put(&ib, (const float*)nullptr, N));
        CUDA_TRY(h->put(&p, (const float*)nullptr, N));
        CUDA_TRY(h->put(&q, (const float*)nullptr, N));
        CUDA_TRY(h->put(&tab, (const float*)nullptr, (size_t)6 * nd[d]));
        h->dev.cib[d] = ib;
        h->dev.cp[d] = p;
        h->dev.cq[d] = q;
        h->dev.ctab[d] = tab;
      }
      mts::build_mixed_coefs(h->dev, h->stream);
      CUDA_TRY(cudaGetLastError());
      h->mixed_built = true;
    }

  }
  h->dev.precision = precision;
  return MTS_OK;
}

mts_status mts_get_precision(mts_handle h, int32_t* precision) {
  if (!h || !precision) return fail(MTS_ERR_ARG, "null argument");
  *precision = h->dev.precision;
  return MTS_OK;
}

mts_status mts_autotune(mts_handle h, int32_t steps, int32_t shapes[3]) {
  if (!h || steps < 1) return fail(MTS_ERR_ARG, "bad argument");
  if (h->dev.precision != MTS_PRECISION_PLAIN) {
    // the shapes are those of the bit-exact sweeps; the other forms have none
    if (shapes)
      for (int k = 0; k < 3; k++) shapes[k] = h->dev.shape[k];
    return MTS_OK;
  }
  const size_t bytes = sizeof(double) * (size_t)h->g.nodes();
  double* backup = nullptr;
  CUDA_TRY(cudaMalloc((void**)&backup, bytes));
  std::unique_ptr<double, decltype(&cudaFree)> guard(backup, &cudaFree);
  CUDA_TRY(cudaMemcpyAsync(backup, h->u0, bytes, cudaMemcpyDeviceToDevice, h->stream));
  const double t0 = h->t;
  const bool prof = h->profiling;
  // profile slots of the three implicit sweeps
  const int first = h->prm.method == MTS_ADI ? 2 : h->prm.method == MTS_TS ? 3 : 1;
  double best[3] = {1e300, 1e300, 1e300};
  int choice[3] = {0, 0, 0};
  mts_status st = MTS_OK;
  h->profiling = true;
  int choice0[3] = {h->dev.shape[0], h->dev.shape[1], h->dev.shape[2]};
  for (int k = 0; k < 3; k++) choice[k] = choice0[k];
  const int nmax = std::max(h->g.nx, std::max(h->g.ny, h->g.nz));
  for (int s = 0; s < mts::sweep_shape_count() && st == MTS_OK; s++) {
    if (!mts::sweep_shape_fits(s, nmax)) continue;
    for (int k = 0; k < 3; k++) h->dev.shape[k] = s;
    st = mts_profile_read(h, nullptr, nullptr);
    if (st) break;
    st = advance(h, steps);
    if (st) break;
    double ms[8];
    int64_t cnt[8];
    st = mts_profile_read(h, ms, cnt);
    if (st) break;
    for (int k = 0; k < 3; k++)
      if (ms[first + k] < best[k]) {
        best[k] = ms[first + k];
        choice[k] = s;
      }
    CUDA_TRY(cudaMemcpyAsync(h->u0, backup, bytes, cudaMemcpyDeviceToDevice, h->stream));
    h->t = t0;
  }
  h->profiling = prof;
  CUDA_TRY(cudaMemcpyAsync(h->u0, backup, bytes, cudaMemcpyDeviceToDevice, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->t = t0;
  for (int k = 0; k < 3; k++) {
    h->dev.shape[k] = choice[k];
    if (shapes) shapes[k] = choice[k];
  }
  return st;
}

mts_status mts_get_stream(mts_handle h, void** stream) {
  if (!h || !stream) return fail(MTS_ERR_ARG, "null argument");
  *stream = (void*)h->stream;
  return MTS_OK;
}

}  // extern "C"

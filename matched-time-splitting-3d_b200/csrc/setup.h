// Host-side problem setup: mesh tags, interface crossings and MIB
// fictitious-point weights.  Runs once per problem; its output is uploaded to
// the device by the C ABI (capi.cu).  Every routine restates the reference
// routine it cites with the same operand order, so the weights are the
// reference's bit for bit (checked by tests/test_setup_parity.py).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/mts.h"

namespace mts {

struct Grid {
  int nx = 0, ny = 0, nz = 0;
  double xl = 0, xr = 0, yl = 0, yr = 0, zl = 0, zr = 0;
  double dx = 0, dy = 0, dz = 0;
  std::vector<double> x, y, z;
  long long nodes() const { return (long long)nx * ny * nz; }
  long long index(int ix, int iy, int iz) const {
    return (long long)ix + (long long)nx * ((long long)iy + (long long)ny * iz);
  }
};

// Mesh::Mesh coordinates (src/mesh/mesh.cc:37-55).
Grid make_grid(const mts_grid& g);

// Level-set surface: value with and without the TOL_SETUP perturbation,
// partial derivatives and unit normal, in the expression shapes of the
// reference surface classes.
class Surface {
 public:
  virtual ~Surface() = default;
  virtual double set_node(double x, double y, double z) const = 0;
  virtual double func(double x, double y, double z) const = 0;
  virtual double dfx(double x, double y, double z) const = 0;
  virtual double dfy(double x, double y, double z) const = 0;
  virtual double dfz(double x, double y, double z) const = 0;
  virtual void normal(double x, double y, double z, double n[3]) const = 0;
};

// nullptr on an unknown kind.
Surface* make_surface(const mts_surface& s);

// Node tags +1 (outside) / -1 (inside), Mesh::Mesh src/mesh/mesh.cc:57-69.
// Returns MTS_ERR_SETUP when a node lies on the interface.
mts_status build_tags(const Grid& g, const Surface& s, std::vector<int8_t>& tags);

struct SetupReport {
  int64_t singular_warnings = 0;  // |det| < TOL_SETUP in a weight solve
  int64_t corner_pairs = 0;
};

// Crossing detection, crossing data and MIB weights: Setup_Intersections,
// Getdata_*, Pmatrix_Setup_*, Setup_MIB_L1/L2 (src/spatial/intersection.cc
// 79-291, 304-780, 789-1830, 2503-2598).  Output order: direction x, y, z;
// lines in the reference's loop order; crossings by left_loc.
mts_status build_crossings(const Grid& g, const std::vector<int8_t>& tags, const Surface& s,
                           double beta_in, double beta_out, int mib,
                           std::vector<mts_crossing>& out, SetupReport* report);

// build_tags + build_crossings on the current CUDA device (setup_gpu.cu),
// queued on `stream` (a cudaStream_t) and synchronized before returning: the
// same tags and crossing list, bit for bit except where the reference's
// pow(v, 2) is not the correctly rounded square.  On failure `why` (may be
// null) receives the reason.
mts_status setup_on_device(const Grid& g, const mts_surface& surf, double beta_in, double beta_out, int mib,
                           void* stream, std::vector<int8_t>& tags, std::vector<mts_crossing>& out,
                           SetupReport* report, std::string* why);

// (P^{-1})[row][0] of the 3x3 local frame via the reference LU inverse
// (src/decomposition/lu.cc:15-161); returns false on an all-zero row.
bool frame_inverse_col0(const double p[9], int row, double* out);

}  // namespace mts

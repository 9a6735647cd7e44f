// Drop-in stepper for the reference's time loop (C++, header only).
//
// mts::GpuStepper has the constructor and the methods that the reference's
// time loops call on Douglas_ADI, LOD and TS:
//   Douglas_ADI(Intersections&, Mesh&, Beta&, VecDoub_I time, Int_I accuracy)
//       (src/temporal/douglas_adi.h:48-52; LOD src/temporal/lod.h:52-56,
//       TS src/temporal/trapezoidal.h:48-53)
//   Initialization(Equation&, CubicDoub&), Solve_2nd(...), Error(...)
// so ADI_Solver / LOD_Solver / TS_Solver (src/helper.h:199-426) run on the
// GPU with the stepper in place of the reference class.  It is included
// after the reference's own headers (it uses their types) and linked with
// libmts_b200.so; oracle/ref_harness.cc built -DMTS_DROPIN is an example.
//
// The problem goes to the device once: the reference's own node tags
// (Mesh::mesh_value) and crossing list (Intersections::ifpx/ifpy/ifpz, with
// the MIB weights the reference computed) are flattened into the C ABI's
// records and handed to mts_create_from_crossings.  The handle keeps the
// time (t += dt per step, as the reference loops do) and the jump data, so a
// step reads neither the Equation nor the Intersections; the field uh goes
// to the device and back around every Solve_2nd, as the reference's contract
// (a CubicDoub in host memory) requires.
//
// beta must be piecewise constant: beta_in and beta_out are read from
// Beta::Inside / Beta::Outside at the origin.  The exact solution the device
// evaluates for source, boundary and jump data is selected by eq (0 for the
// reference's Eq_0, 8 for the measured e^{-t} solution).
#pragma once

#include <cmath>
#include <fstream>
#include <iomanip>
#include <stdexcept>
#include <string>
#include <vector>

#include "mts.h"

namespace mts {

class GpuStepper {
 public:
  // time = {t_start, t_end, dt}; accuracy = the spatial order the reference
  // passes (2; Douglas_ADI stores it and reads it nowhere); method =
  // MTS_ADI, MTS_LOD_IE, MTS_LOD_CN or MTS_TS.  The MIB level (L1 or L2) is
  // the one the Intersections were built with: it is carried by the crossing
  // weights, and mts_params.mib, only range-checked on this path, is set to 2.
  GpuStepper(Intersections& inter, Mesh& mesh, Beta& beta, VecDoub_I time, Int_I accuracy,
             int method = MTS_ADI, int eq = 8)
      : nx_(mesh.nx), ny_(mesh.ny), nz_(mesh.nz) {
    (void)accuracy;
    mts_grid g{nx_, ny_, nz_, 0, mesh.xi[0], mesh.xi[nx_ - 1], mesh.yi[0], mesh.yi[ny_ - 1],
               mesh.zi[0], mesh.zi[nz_ - 1]};
    mts_params p{beta.Inside(0, 0, 0), beta.Outside(0, 0, 0), eq, method, 2, 0, time[2], time[0]};
    std::vector<int8_t> tags(static_cast<size_t>(nx_) * ny_ * nz_);
    for (size_t m = 0; m < tags.size(); m++) tags[m] = mesh.mesh_value[m] > 0 ? 1 : -1;
    std::vector<mts_crossing> cr;
    flatten(inter.ifpx, ny_, nz_, cr);
    flatten(inter.ifpy, nx_, nz_, cr);
    flatten(inter.ifpz, nx_, ny_, cr);
    check(mts_create_from_crossings(&g, tags.data(), cr.empty() ? nullptr : cr.data(), (int32_t)cr.size(), &p,
                                    &h_));
    field_.resize(tags.size());
  }
  ~GpuStepper() { mts_destroy(h_); }
  GpuStepper(const GpuStepper&) = delete;
  GpuStepper& operator=(const GpuStepper&) = delete;

  void Initialization(Equation&, CubicDoub_I& uh) {
    check(mts_initialize(h_));
    download(uh);
  }
  // Douglas_ADI::Solve_2nd(eq, inter, uh, beta)
  void Solve_2nd(Equation&, Intersections&, CubicDoub_I& uh, Beta&) { step(uh); }
  // LOD::Solve_2nd(eq, inter, uh, beta, 'I' | 'C'); the variant is the
  // method given at construction
  void Solve_2nd(Equation&, Intersections&, CubicDoub_I& uh, Beta&, char&) { step(uh); }
  // TS::Solve_2nd(eq(t-dt), eq(t-dt/2), eq(t), inter, uh, beta)
  void Solve_2nd(Equation&, Equation&, Equation&, Intersections&, CubicDoub_I& uh, Beta&) { step(uh); }

  // Douglas_ADI::Error (src/temporal/douglas_adi.cc:1723-1770): L-infinity
  // with its argmax and L2 against the exact solution at the current time,
  // written to the report stream in the reference's format.  The norms come
  // from the device (mts_norms), bit-identical to the reference's loop.
  void Error(Equation&, CubicDoub_I&, std::ofstream& out) {
    double lmax, l2;
    int32_t am[3];
    check(mts_norms(h_, &lmax, &l2, am));
    out << std::setprecision(3) << std::scientific;
    out << "[Xmax,Ymax,Zmax] = [" << am[0] << "," << am[1] << "," << am[2] << "]" << std::endl;
    out << " Lmax = " << lmax << ";  L2 = " << l2 << std::endl;
    out << std::fixed << std::endl;
  }

  mts_handle handle() const { return h_; }

 private:
  void step(CubicDoub_I& uh) {
    upload(uh);
    check(mts_advance(h_, 1));
    download(uh);
  }
  // Intersections::ifpx/ifpy/ifpz, direction by direction, lines in their
  // (indx1, indx2) loop order, crossings in each line's order: the record of
  // Intersection_Data (src/constant.h:141-156) the C ABI takes.
  template <class C>
  static void flatten(C& ifp, int n1, int n2, std::vector<mts_crossing>& out) {
    for (int i1 = 1; i1 < n1 - 1; i1++)
      for (int i2 = 1; i2 < n2 - 1; i2++)
        for (const Intersection_Data& d : ifp[i1][i2]) {
          mts_crossing c{};
          c.dir = d.dir == 'x' ? 0 : d.dir == 'y' ? 1 : 2;
          c.indx1 = d.line.indx1;
          c.indx2 = d.line.indx2;
          c.id = d.ID;
          c.left_loc = d.left_loc;
          c.nwei = (int32_t)d.wei.weil[0].size();
          c.coord[0] = d.coord.x_value;
          c.coord[1] = d.coord.y_value;
          c.coord[2] = d.coord.z_value;
          c.gamma = d.gamma;
          for (int k = 0; k < 3; k++) c.normal[k] = d.local.normal[k];
          for (int r = 0; r < 3; r++)
            for (int k = 0; k < 3; k++) c.p[3 * r + k] = d.p[r][k];
          for (int k = 0; k < c.nwei && k < 9; k++) {
            c.weil[k] = d.wei.weil[0][k];
            c.weir[k] = d.wei.weir[0][k];
          }
          out.push_back(c);
        }
  }
  // CubicDoub is uh[ix][iy][iz]; the device field is x fastest.
  void upload(CubicDoub_I& uh) {
    for (int iz = 0; iz < nz_; iz++)
      for (int iy = 0; iy < ny_; iy++)
        for (int ix = 0; ix < nx_; ix++) field_[ix + (size_t)nx_ * (iy + (size_t)ny_ * iz)] = uh[ix][iy][iz];
    check(mts_set_solution(h_, field_.data()));
  }
  void download(CubicDoub_I& uh) {
    check(mts_get_solution(h_, field_.data()));
    uh.resize(nx_);
    for (int ix = 0; ix < nx_; ix++) {
      uh[ix].resize(ny_);
      for (int iy = 0; iy < ny_; iy++) uh[ix][iy].resize(nz_);
    }
    for (int iz = 0; iz < nz_; iz++)
      for (int iy = 0; iy < ny_; iy++)
        for (int ix = 0; ix < nx_; ix++) uh[ix][iy][iz] = field_[ix + (size_t)nx_ * (iy + (size_t)ny_ * iz)];
  }
  static void check(mts_status s) {
    if (s != MTS_OK) throw std::runtime_error(std::string("mts: ") + mts_last_error());
  }
  int nx_, ny_, nz_;
  mts_handle h_ = nullptr;
  std::vector<double> field_;
};

}  // namespace mts

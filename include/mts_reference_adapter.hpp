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
// The problem goes to the device once, at the first call that needs it
// (Initialization, normally): the reference's own node tags
// (Mesh::mesh_value) and crossing list (Intersections::ifpx/ifpy/ifpz, with
// the MIB weights the reference computed) are flattened into the C ABI's
// records and handed to mts_create_from_crossings.  The handle keeps the
// time (t += dt per step, as the reference loops do) and the jump data, so a
// step reads neither the Equation nor the Intersections; the field uh goes
// to the device and back around every Solve_2nd, as the reference's contract
// (a CubicDoub in host memory) requires.
//
// The device evaluates beta, source, boundary and jump data itself, so the
// stepper refuses plugins it would not reproduce, with std::invalid_argument
// and before any device work:
//   * beta must be piecewise constant (the reference's Beta_0 and the like;
//     Beta_1..4 of src/diffusion/ vary in space): the constructor samples
//     Beta::Inside / Outside and their derivatives on a lattice of mesh
//     nodes and requires one value per side and zero derivatives;
//   * the Equation handed to Initialization, Solve_2nd and Error must be the
//     exact solution that eq selects (0: the reference's Eq_0, piecewise
//     constant; 8: inside e^{-t} sin2x cos2y sin2z, outside e^{-t}(x^2+y^2+z^2));
//     its u, f and [beta u_d] are compared with that closed form on the same
//     lattice at the step's time (relative 1e-12), so Eq_1..Eq_7 of
//     src/helper.h:56-90 are refused.
#pragma once

#include <algorithm>
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
      : inter_(inter), mesh_(mesh), nx_(mesh.nx), ny_(mesh.ny), nz_(mesh.nz), method_(method), eq_(eq),
        t_(time[0]), dt_(time[2]) {
    (void)accuracy;
    if (eq != 0 && eq != 8) throw std::invalid_argument("mts::GpuStepper: eq must be 0 or 8");
    check_beta(mesh, beta, &bi_, &bo_);
  }
  ~GpuStepper() {
    if (h_) mts_destroy(h_);
  }
  GpuStepper(const GpuStepper&) = delete;
  GpuStepper& operator=(const GpuStepper&) = delete;

  void Initialization(Equation& e, CubicDoub_I& uh) {
    check_equation(mesh_, e, eq_, bi_, bo_, t_);
    create();
    check(mts_initialize(h_));
    download(uh);
  }
  // Douglas_ADI::Solve_2nd(eq, inter, uh, beta)
  void Solve_2nd(Equation& e, Intersections&, CubicDoub_I& uh, Beta&) {
    check_equation(mesh_, e, eq_, bi_, bo_, t_ + dt_);
    step(uh);
  }
  // LOD::Solve_2nd(eq, inter, uh, beta, 'I' | 'C'); the variant is the
  // method given at construction
  void Solve_2nd(Equation& e, Intersections&, CubicDoub_I& uh, Beta&, char&) {
    check_equation(mesh_, e, eq_, bi_, bo_, t_ + dt_);
    step(uh);
  }
  // TS::Solve_2nd(eq(t-dt), eq(t-dt/2), eq(t), inter, uh, beta)
  void Solve_2nd(Equation& e0, Equation& eh, Equation& e1, Intersections&, CubicDoub_I& uh, Beta&) {
    check_equation(mesh_, e0, eq_, bi_, bo_, t_);
    check_equation(mesh_, eh, eq_, bi_, bo_, t_ + 0.5 * dt_);
    check_equation(mesh_, e1, eq_, bi_, bo_, t_ + dt_);
    step(uh);
  }

  // Refuses a beta that is not piecewise constant (std::invalid_argument);
  // returns its two values (inside, outside) in *bi / *bo.
  static void check_beta(const Mesh& mesh, Beta& beta, double* bi, double* bo) {
    const double b_in = beta.Inside(mesh.xi[0], mesh.yi[0], mesh.zi[0]);
    const double b_out = beta.Outside(mesh.xi[0], mesh.yi[0], mesh.zi[0]);
    bool ok = b_in > 0 && b_out > 0;
    for_lattice(mesh, [&](double x, double y, double z) {
      ok = ok && beta.Inside(x, y, z) == b_in && beta.Outside(x, y, z) == b_out && beta.Inside_Dx(x, y, z) == 0 &&
           beta.Outside_Dx(x, y, z) == 0 && beta.Inside_Dy(x, y, z) == 0 && beta.Outside_Dy(x, y, z) == 0 &&
           beta.Inside_Dz(x, y, z) == 0 && beta.Outside_Dz(x, y, z) == 0;
    });
    if (!ok)
      throw std::invalid_argument(
          "mts::GpuStepper: beta must be piecewise constant and positive (one value inside, one outside); "
          "the device does not evaluate variable-coefficient Beta plugins");
    *bi = b_in;
    *bo = b_out;
  }

  // Refuses an Equation whose u, f or [beta u_d] at time t differ from the
  // closed form that eq selects (std::invalid_argument).
  static void check_equation(const Mesh& mesh, Equation& e, int eq, double bi, double bo, double t) {
    const double E = std::exp(-t);
    bool ok = true;
    auto near = [](double a, double b) { return std::fabs(a - b) <= 1e-12 * std::max(1.0, std::fabs(b)); };
    for_lattice(mesh, [&](double x, double y, double z) {
      double ui, uo, fi, fo, jb[3];
      if (eq == 0) {
        ui = 80.0;
        uo = 100.0;
        fi = fo = 0.0;
        jb[0] = jb[1] = jb[2] = 0.0;
      } else {
        const double s2x = std::sin(2.0 * x), c2x = std::cos(2.0 * x), s2y = std::sin(2.0 * y);
        const double c2y = std::cos(2.0 * y), s2z = std::sin(2.0 * z), c2z = std::cos(2.0 * z);
        ui = ((s2x * c2y) * s2z) * E;
        uo = ((x * x + y * y) + z * z) * E;
        fi = (12.0 * bi - 1.0) * ui;
        fo = -uo - (6.0 * bo) * E;
        jb[0] = bo * ((2.0 * x) * E) - bi * ((((2.0 * c2x) * c2y) * s2z) * E);
        jb[1] = bo * ((2.0 * y) * E) - bi * ((((-2.0 * s2x) * s2y) * s2z) * E);
        jb[2] = bo * ((2.0 * z) * E) - bi * ((((2.0 * s2x) * c2y) * c2z) * E);
      }
      ok = ok && near(e.Inner_u(x, y, z), ui) && near(e.Outer_u(x, y, z), uo) && near(e.Inner_f(x, y, z), fi) &&
           near(e.Outer_f(x, y, z), fo) && near(e.Jump_betau_x(x, y, z), jb[0]) &&
           near(e.Jump_betau_y(x, y, z), jb[1]) && near(e.Jump_betau_z(x, y, z), jb[2]);
    });
    if (!ok)
      throw std::invalid_argument(
          "mts::GpuStepper: the Equation is not the exact solution the device evaluates (eq " + std::to_string(eq) +
          ", beta " + std::to_string(bi) + "/" + std::to_string(bo) + ")");
  }

  // Douglas_ADI::Error (src/temporal/douglas_adi.cc:1723-1770): L-infinity
  // with its argmax and L2 against the exact solution at the current time,
  // written to the report stream in the reference's format.  The norms come
  // from the device (mts_norms), bit-identical to the reference's loop.
  void Error(Equation& e, CubicDoub_I&, std::ofstream& out) {
    check_equation(mesh_, e, eq_, bi_, bo_, t_);
    create();
    double lmax, l2;
    int32_t am[3];
    check(mts_norms(h_, &lmax, &l2, am));
    out << std::setprecision(3) << std::scientific;
    out << "[Xmax,Ymax,Zmax] = [" << am[0] << "," << am[1] << "," << am[2] << "]" << std::endl;
    out << " Lmax = " << lmax << ";  L2 = " << l2 << std::endl;
    out << std::fixed << std::endl;
  }

  // In place of the reference's report pair
  //   inter.Refresh_Fp(eq); inter.Error_Fp(out);   (helper.h:230-231)
  // the fictitious points' errors at the stepper's time, evaluated on the
  // device (mts_fp_errors), written in Error_Fp's text
  // (intersection.cc:4763-4770).
  void Error_Fp(Equation& e, std::ofstream& out) {
    check_equation(mesh_, e, eq_, bi_, bo_, t_);
    create();
    double lmax, l2;
    check(mts_fp_errors(h_, &lmax, &l2));
    out << "------------------------ Error of FPs ------------------------" << std::endl;
    out << std::setprecision(3) << std::scientific;
    out << "Lmax = " << lmax << std::endl;
    out << "L2   = " << l2 << std::endl;
    out << std::fixed << std::endl;
  }

  // In place of the reference's report pair
  //   inter.Refresh_Jump(eq, uh, beta); inter.Error_Jump(out);   (helper.h:233-234)
  // the jumps' errors at the stepper's time, evaluated on the device
  // (mts_jump_errors), written in Error_Jump's text (intersection.cc:4656-4661).
  void Error_Jump(Equation& e, std::ofstream& out) {
    check_equation(mesh_, e, eq_, bi_, bo_, t_);
    create();
    double lmax, l2;
    check(mts_jump_errors(h_, &lmax, &l2));
    out << "------------------------ Error of Jumps ------------------------" << std::endl;
    out << std::setprecision(3) << std::scientific;
    out << "Lmax = " << lmax << std::endl;
    out << "L2   = " << l2 << std::endl;
    out << std::fixed << std::endl;
  }

  mts_handle handle() const { return h_; }

 private:
  // Up to 9 nodes per axis, ends included.
  template <class F>
  static void for_lattice(const Mesh& mesh, F f) {
    auto pick = [](int n, int k) { return (int)((long long)(n - 1) * k / 8); };
    for (int a = 0; a <= 8; a++)
      for (int b = 0; b <= 8; b++)
        for (int c = 0; c <= 8; c++) f(mesh.xi[pick(mesh.nx, a)], mesh.yi[pick(mesh.ny, b)], mesh.zi[pick(mesh.nz, c)]);
  }
  void create() {
    if (h_) return;
    mts_grid g{nx_, ny_, nz_, 0, mesh_.xi[0], mesh_.xi[nx_ - 1], mesh_.yi[0], mesh_.yi[ny_ - 1],
               mesh_.zi[0], mesh_.zi[nz_ - 1]};
    mts_params p{bi_, bo_, eq_, method_, 2, 0, dt_, t_};
    std::vector<int8_t> tags(static_cast<size_t>(nx_) * ny_ * nz_);
    for (size_t m = 0; m < tags.size(); m++) tags[m] = mesh_.mesh_value[m] > 0 ? 1 : -1;
    std::vector<mts_crossing> cr;
    flatten(inter_.ifpx, ny_, nz_, cr);
    flatten(inter_.ifpy, nx_, nz_, cr);
    flatten(inter_.ifpz, nx_, ny_, cr);
    check(mts_create_from_crossings(&g, tags.data(), cr.empty() ? nullptr : cr.data(), (int32_t)cr.size(), &p,
                                    &h_));
    field_.resize(tags.size());
  }
  void step(CubicDoub_I& uh) {
    create();
    upload(uh);
    check(mts_advance(h_, 1));
    t_ += dt_;
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
  Intersections& inter_;
  Mesh& mesh_;
  int nx_, ny_, nz_;
  int method_, eq_;
  double t_, dt_;  // the time of uh, as the reference's loop advances it (t += dt per step)
  double bi_ = 0, bo_ = 0;
  mts_handle h_ = nullptr;
  std::vector<double> field_;
};

}  // namespace mts

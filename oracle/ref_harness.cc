// Test infrastructure only: a command-line driver around the reference's own
// classes (Mesh, Intersections, Douglas_ADI, LOD, TS), compiled from the
// reference sources where they lie.  It replaces the reference CLI
// (src/main.cc:26-133 and the time loops of src/helper.h:199-426) so that the
// problems this project measures can be posed without editing reference code:
//   * Eq8 — the exact solution of the measured problems (not shipped by the
//     reference; written here from its mathematics, see eq8 below),
//   * PiecewiseBeta — piecewise-constant (beta_in, beta_out) in the shape of
//     src/diffusion/beta_0.cc:19-42 with free constants,
//   * ShiftedEllipsoid — src/surface/surface_ellipsoid.cc with a centre.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg run it.
//
// Output: one JSON line on stdout; optional binary dumps of the solution
// (x-fastest, the order of Mesh::To1d, src/mesh/mesh.cc:93-99), the node tags
// and the crossing list (one fixed-size record per Intersection_Data).

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <memory>
#include <string>
#include <vector>

#include "constant.h"
#include "diffusion/beta.h"
#include "diffusion/beta_1.h"
#include "equation/eq_0.h"
#include "equation/eq_3.h"
#include "equation/equation.h"
#include "mesh/mesh.h"
#include "spatial/intersection.h"
#include "surface/surface_cartesian.h"
#include "surface/surface_ellipsoid.h"
#include "surface/surface_torus.h"
#include "temporal/douglas_adi.h"
#include "temporal/lod.h"
#include "temporal/trapezoidal.h"
#ifdef MTS_DROPIN
#include "mts_reference_adapter.hpp"
#endif

// The reference's Write_txt (ref_write_txt.cc).
void ref_write_txt(Intersections& inter, Mesh& mesh, Beta& beta, CubicDoub& uh, int equation, double t);


using namespace std;

namespace {

// Piecewise-constant diffusion coefficient; zero derivatives.
class PiecewiseBeta : public Beta {
 public:
  PiecewiseBeta(double bi, double bo) : bi_(bi), bo_(bo) {}
  double Inside(Doub_I, Doub_I, Doub_I) const override { return bi_; }
  double Outside(Doub_I, Doub_I, Doub_I) const override { return bo_; }
  double Inside_Dx(Doub_I, Doub_I, Doub_I) const override { return 0; }
  double Outside_Dx(Doub_I, Doub_I, Doub_I) const override { return 0; }
  double Inside_Dy(Doub_I, Doub_I, Doub_I) const override { return 0; }
  double Outside_Dy(Doub_I, Doub_I, Doub_I) const override { return 0; }
  double Inside_Dz(Doub_I, Doub_I, Doub_I) const override { return 0; }
  double Outside_Dz(Doub_I, Doub_I, Doub_I) const override { return 0; }

 private:
  double bi_, bo_;
};

// Exact solution of the measured problems:
//   inside  u = e^{-t} sin(2x) cos(2y) sin(2z),  outside u = e^{-t} (x^2+y^2+z^2)
// with u_t = div(beta grad u) + f, piecewise-constant beta.  The evaluation
// order of every expression is fixed (time factor E = exp(-t) multiplied last)
// so that a GPU evaluation from per-axis tables reproduces it bit for bit.
class Eq8 : public Equation {
 public:
  Eq8(double ti, double bi, double bo) : bi_(bi), bo_(bo) {
    t = ti;
    E_ = exp(-ti);
  }
  double Inner_u(Doub_I x, Doub_I y, Doub_I z) const override {
    return ((sin(2.0 * x) * cos(2.0 * y)) * sin(2.0 * z)) * E_;
  }
  double Outer_u(Doub_I x, Doub_I y, Doub_I z) const override {
    return ((x * x + y * y) + z * z) * E_;
  }
  double Inner_f(Doub_I x, Doub_I y, Doub_I z) const override {
    return (12.0 * bi_ - 1.0) * Inner_u(x, y, z);
  }
  double Outer_f(Doub_I x, Doub_I y, Doub_I z) const override {
    return -Outer_u(x, y, z) - (6.0 * bo_) * E_;
  }
  double Jump_betau_x(Doub_I x, Doub_I y, Doub_I z) const override {
    return bo_ * Outer_dux(x, y, z) - bi_ * Inner_dux(x, y, z);
  }
  double Jump_betau_y(Doub_I x, Doub_I y, Doub_I z) const override {
    return bo_ * Outer_duy(x, y, z) - bi_ * Inner_duy(x, y, z);
  }
  double Jump_betau_z(Doub_I x, Doub_I y, Doub_I z) const override {
    return bo_ * Outer_duz(x, y, z) - bi_ * Inner_duz(x, y, z);
  }

 private:
  double Inner_dux(Doub_I x, Doub_I y, Doub_I z) const override {
    return (((2.0 * cos(2.0 * x)) * cos(2.0 * y)) * sin(2.0 * z)) * E_;
  }
  double Inner_duy(Doub_I x, Doub_I y, Doub_I z) const override {
    return (((-2.0 * sin(2.0 * x)) * sin(2.0 * y)) * sin(2.0 * z)) * E_;
  }
  double Inner_duz(Doub_I x, Doub_I y, Doub_I z) const override {
    return (((2.0 * sin(2.0 * x)) * cos(2.0 * y)) * cos(2.0 * z)) * E_;
  }
  double Outer_dux(Doub_I x, Doub_I, Doub_I) const override { return (2.0 * x) * E_; }
  double Outer_duy(Doub_I, Doub_I y, Doub_I) const override { return (2.0 * y) * E_; }
  double Outer_duz(Doub_I, Doub_I, Doub_I z) const override { return (2.0 * z) * E_; }

  double bi_, bo_, E_;
};

// Ellipsoid (x-cx)^2/a^2 + (y-cy)^2/b^2 + (z-cz)^2/c^2 - r^2 with the
// expression shapes of src/surface/surface_ellipsoid.cc (Set_Node :60-66,
// func :79-85, dfx/dfy/dfz :97-140, normal :151-168).
class ShiftedEllipsoid : public Surface_Cartesian {
 public:
  explicit ShiftedEllipsoid(const vector<double>& p)
      : a(p[0]), b(p[1]), c(p[2]), r(p[3]), cx(p[4]), cy(p[5]), cz(p[6]) {}
  double Set_Node(Doub_I x, Doub_I y, Doub_I z) const override {
    return func(x, y, z) + TOL_SETUP;
  }
  void display() override {}
  VecDoub normal(Doub_I x, Doub_I y, Doub_I z) override {
    double X = x - cx, Y = y - cy, Z = z - cz;
    double total = sqrt(pow(2 * X / (a * a), 2) + pow(2 * Y / (b * b), 2) +
                        pow(2 * Z / (c * c), 2));
    VecDoub n;
    n.push_back(2 * X / (a * a) / total);
    n.push_back(2 * Y / (b * b) / total);
    n.push_back(2 * Z / (c * c) / total);
    return n;
  }
  double check(Doub_I x, Doub_I y, Doub_I z) override { return func(x, y, z); }

 private:
  double func(const Doub_I x, const Doub_I y, const Doub_I z) const override {
    double X = x - cx, Y = y - cy, Z = z - cz;
    return X * X / (a * a) + Y * Y / (b * b) + Z * Z / (c * c) - r * r;
  }
  double dfx(const Doub_I x, const Doub_I, const Doub_I) const override {
    return 2 * (x - cx) / (a * a);
  }
  double dfy(const Doub_I, const Doub_I y, const Doub_I) const override {
    return 2 * (y - cy) / (b * b);
  }
  double dfz(const Doub_I, const Doub_I, const Doub_I z) const override {
    return 2 * (z - cz) / (c * c);
  }
  double a, b, c, r, cx, cy, cz;
};

struct Args {
  int n[3] = {33, 33, 33};
  double dom[6] = {-1, 1, -1, 1, -1, 1};
  string surface = "ellipsoid";
  vector<double> sp = {1, 1, 1, 0.49, 0, 0, 0};
  double bi = 1, bo = 10;
  int eq = 8;
  string method = "adi";
  int mib = 1;
  double dt = 1.0 / 32, t0 = 0;
  int steps = -1;
  double t_end = 1.0;
  string dump_u, dump_tags, dump_mib, dump_u0;
  string report;     // --report F: the stepper's own Error() text at the end
  bool write_txt = false;  // --write-txt: the reference's Write_txt files (Eq_0..Eq_7) at the end
  string fp_errors;  // --fp-errors F: Refresh_Fp + Error_Fp at the end (values in binary, then the text)
  string jump_errors;  // --jump-errors F: Refresh_Jump + Error_Jump at the end (the same layout)
  bool gpu = false;  // --gpu: mts::GpuStepper in place of the reference's stepper
  int beta_plugin = -1;  // --beta-plugin 1: the reference's Beta_1 instead of the piecewise-constant beta
};

[[noreturn]] void usage() {
  fprintf(stderr,
          "mts_ref --n NX NY NZ --domain xl xr yl yr zl zr\n"
          "        --surface ellipsoid a b c r [cx cy cz] | torus R r\n"
          "        --beta bi bo [--beta-plugin 1] --eq 0|3|8 --method adi|lod-ie|lod-cn|ts --mib 1|2\n"
          "        --dt DT [--t0 T0] (--steps K | --t-end T)\n"
          "        [--dump-u F] [--dump-u0 F] [--dump-tags F] [--dump-mib F] [--report F] [--fp-errors F] [--jump-errors F]\n"
          "        [--write-txt]\n"
#ifdef MTS_DROPIN
          "        [--gpu]\n"
#endif
  );
  exit(2);
}

Args parse(int argc, char** argv) {
  Args a;
  for (int i = 1; i < argc; i++) {
    string k = argv[i];
    auto need = [&](int m) {
      if (i + m >= argc) usage();
    };
    if (k == "--n") {
      need(3);
      for (int d = 0; d < 3; d++) a.n[d] = atoi(argv[++i]);
    } else if (k == "--domain") {
      need(6);
      for (int d = 0; d < 6; d++) a.dom[d] = atof(argv[++i]);
    } else if (k == "--surface") {
      need(1);
      a.surface = argv[++i];
      a.sp.clear();
      while (i + 1 < argc && strncmp(argv[i + 1], "--", 2) != 0) a.sp.push_back(atof(argv[++i]));
    } else if (k == "--beta") {
      need(2);
      a.bi = atof(argv[++i]);
      a.bo = atof(argv[++i]);
    } else if (k == "--beta-plugin") {
      need(1);
      a.beta_plugin = atoi(argv[++i]);
    } else if (k == "--eq") {
      need(1);
      a.eq = atoi(argv[++i]);
    } else if (k == "--method") {
      need(1);
      a.method = argv[++i];
    } else if (k == "--mib") {
      need(1);
      a.mib = atoi(argv[++i]);
    } else if (k == "--dt") {
      need(1);
      a.dt = atof(argv[++i]);
    } else if (k == "--t0") {
      need(1);
      a.t0 = atof(argv[++i]);
    } else if (k == "--steps") {
      need(1);
      a.steps = atoi(argv[++i]);
    } else if (k == "--t-end") {
      need(1);
      a.t_end = atof(argv[++i]);
    } else if (k == "--dump-u") {
      need(1);
      a.dump_u = argv[++i];
    } else if (k == "--dump-u0") {
      need(1);
      a.dump_u0 = argv[++i];
    } else if (k == "--dump-tags") {
      need(1);
      a.dump_tags = argv[++i];
    } else if (k == "--dump-mib") {
      need(1);
      a.dump_mib = argv[++i];
    } else if (k == "--report") {
      need(1);
      a.report = argv[++i];
    } else if (k == "--write-txt") {
      a.write_txt = true;
    } else if (k == "--fp-errors") {
      need(1);
      a.fp_errors = argv[++i];
    } else if (k == "--jump-errors") {
      need(1);
      a.jump_errors = argv[++i];
#ifdef MTS_DROPIN
    } else if (k == "--gpu") {
      a.gpu = true;
#endif
    } else {
      usage();
    }
  }
  return a;
}

unique_ptr<Equation> make_eq(const Args& a, double t, Beta& beta) {
  if (a.eq == 8) return unique_ptr<Equation>(new Eq8(t, a.bi, a.bo));
  if (a.eq == 0) return unique_ptr<Equation>(new Eq_0(t, beta));
  if (a.eq == 3) return unique_ptr<Equation>(new Eq_3(t, beta));
  fprintf(stderr, "unsupported --eq %d\n", a.eq);
  exit(2);
}

void dump_field(const string& path, const CubicDoub& uh, int nx, int ny, int nz) {
  vector<double> buf((size_t)nx * ny * nz);
  for (int iz = 0; iz < nz; iz++)
    for (int iy = 0; iy < ny; iy++)
      for (int ix = 0; ix < nx; ix++) buf[(size_t)ix + (size_t)nx * (iy + (size_t)ny * iz)] = uh[ix][iy][iz];
  FILE* f = fopen(path.c_str(), "wb");
  if (!f) {
    perror(path.c_str());
    exit(3);
  }
  fwrite(buf.data(), sizeof(double), buf.size(), f);
  fclose(f);
}

// Fixed-size crossing record; field meanings follow Intersection_Data
// (src/constant.h:141-156).
struct CrossingRecord {
  int32_t dir, indx1, indx2, id, left_loc, nwei;
  double coord[3], gamma, normal[3], p[9], weil[9], weir[9];
};

void dump_crossings(const string& path, Intersections& inter, int nx, int ny, int nz) {
  FILE* f = fopen(path.c_str(), "wb");
  if (!f) {
    perror(path.c_str());
    exit(3);
  }
  auto emit = [&](const Intersection_Data& d) {
    CrossingRecord r;
    memset(&r, 0, sizeof r);
    r.dir = d.dir == 'x' ? 0 : d.dir == 'y' ? 1 : 2;
    r.indx1 = d.line.indx1;
    r.indx2 = d.line.indx2;
    r.id = d.ID;
    r.left_loc = d.left_loc;
    r.nwei = (int)d.wei.weil[0].size();
    r.coord[0] = d.coord.x_value;
    r.coord[1] = d.coord.y_value;
    r.coord[2] = d.coord.z_value;
    r.gamma = d.gamma;
    for (int i = 0; i < 3; i++) r.normal[i] = d.local.normal[i];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) r.p[3 * i + j] = d.p[i][j];
    for (int i = 0; i < r.nwei && i < 9; i++) {
      r.weil[i] = d.wei.weil[0][i];
      r.weir[i] = d.wei.weir[0][i];
    }
    fwrite(&r, sizeof r, 1, f);
  };
  for (int iy = 1; iy < ny - 1; iy++)
    for (int iz = 1; iz < nz - 1; iz++)
      for (auto& d : inter.ifpx[iy][iz]) emit(d);
  for (int ix = 1; ix < nx - 1; ix++)
    for (int iz = 1; iz < nz - 1; iz++)
      for (auto& d : inter.ifpy[ix][iz]) emit(d);
  for (int ix = 1; ix < nx - 1; ix++)
    for (int iy = 1; iy < ny - 1; iy++)
      for (auto& d : inter.ifpz[ix][iy]) emit(d);
  fclose(f);
}

}  // namespace

int main(int argc, char** argv) {
  Args a = parse(argc, argv);
  static_assert(sizeof(CrossingRecord) == 296, "record layout");

  unique_ptr<Surface_Cartesian> surf;
  if (a.surface == "ellipsoid") {
    if (a.sp.size() == 4) a.sp.insert(a.sp.end(), {0.0, 0.0, 0.0});
    if (a.sp.size() != 7) usage();
    if (a.sp[4] == 0 && a.sp[5] == 0 && a.sp[6] == 0)
      surf.reset(new Surface_Ellipsoid(VecDoub{a.sp[0], a.sp[1], a.sp[2], a.sp[3]}));
    else
      surf.reset(new ShiftedEllipsoid(a.sp));
  } else if (a.surface == "torus") {
    if (a.sp.size() != 2) usage();
    surf.reset(new Surface_Torus(VecDoub{a.sp[0], a.sp[1]}));
  } else {
    usage();
  }
  unique_ptr<Beta> beta_own;
  if (a.beta_plugin == 1)
    beta_own.reset(new Beta_1());
  else if (a.beta_plugin < 0)
    beta_own.reset(new PiecewiseBeta(a.bi, a.bo));
  else
    usage();
  Beta& beta = *beta_own;

  VecDoub domain(a.dom, a.dom + 6);
  VecInt size{a.n[0], a.n[1], a.n[2]};
  double t_finish = a.steps >= 0 ? a.t0 + a.steps * a.dt : a.t_end;
  VecDoub time{a.t0, t_finish, a.dt};
  // Same step count as helper.h:208 (loop = (int)(t_finish / dt) / NPRINT).
  int steps = a.steps >= 0 ? a.steps : (int)(t_finish / a.dt) / NPRINT;

  auto t_setup0 = chrono::steady_clock::now();
  Mesh mesh(domain, size, *surf);
  ofstream sink("/dev/null");
  Intersections inter(*surf, mesh, beta, 2, a.mib, sink);
  auto t_setup1 = chrono::steady_clock::now();
  int nx = mesh.nx, ny = mesh.ny, nz = mesh.nz;

  if (!a.dump_tags.empty()) {
    vector<int8_t> tags((size_t)nx * ny * nz);
    for (size_t i = 0; i < tags.size(); i++) tags[i] = (int8_t)mesh.mesh_value[i];
    FILE* f = fopen(a.dump_tags.c_str(), "wb");
    fwrite(tags.data(), 1, tags.size(), f);
    fclose(f);
  }
  if (!a.dump_mib.empty()) dump_crossings(a.dump_mib, inter, nx, ny, nz);

  size_t ncross[3] = {0, 0, 0};
  for (int iy = 1; iy < ny - 1; iy++)
    for (int iz = 1; iz < nz - 1; iz++) ncross[0] += inter.ifpx[iy][iz].size();
  for (int ix = 1; ix < nx - 1; ix++)
    for (int iz = 1; iz < nz - 1; iz++) ncross[1] += inter.ifpy[ix][iz].size();
  for (int ix = 1; ix < nx - 1; ix++)
    for (int iy = 1; iy < ny - 1; iy++) ncross[2] += inter.ifpz[ix][iy].size();

  CubicDoub uh;
  double t_now = a.t0;
  double step_seconds = 0;
  ofstream report("/dev/null");
  double lmax = 0, l2 = 0;
  int am[3] = {0, 0, 0};

  // Error() writes its norms to a stream; re-computing them here with the
  // same loop order (src/temporal/douglas_adi.cc:1723-1770) keeps the values
  // in binary instead of the 3-digit text of the report.
  auto norms = [&](Equation& eq) {
    lmax = 0;
    l2 = 0;
    for (int ix = 0; ix < nx; ix++)
      for (int iy = 0; iy < ny; iy++)
        for (int iz = 0; iz < nz; iz++) {
          int indx = iz * nx * ny + iy * nx + ix;
          double temp;
          if (mesh.mesh_value[indx] == 1)
            temp = fabs(uh[ix][iy][iz] - eq.Outer_u(mesh.xi[ix], mesh.yi[iy], mesh.zi[iz]));
          else
            temp = fabs(uh[ix][iy][iz] - eq.Inner_u(mesh.xi[ix], mesh.yi[iy], mesh.zi[iz]));
          if (temp > lmax) {
            lmax = temp;
            am[0] = ix;
            am[1] = iy;
            am[2] = iz;
          }
          l2 += temp * temp;
        }
    l2 = sqrt(l2 / (1.0 * nx * ny * nz));
  };

  // The reference's time loops (src/helper.h:199-426): Initialization at t0,
  // then one Solve_2nd per step with the exact solutions at the step's
  // times.  St is the reference's stepper or, with --gpu, mts::GpuStepper in
  // its place: the loop is the same code for both.
  auto run = [&](auto& st, auto&& solve) {
    st.Initialization(*make_eq(a, a.t0, beta), uh);
    if (!a.dump_u0.empty()) dump_field(a.dump_u0, uh, nx, ny, nz);
    auto s0 = chrono::steady_clock::now();
    for (int j = 0; j < steps; j++) {
      t_now += a.dt;
      solve(st);
    }
    step_seconds = chrono::duration<double>(chrono::steady_clock::now() - s0).count();
    if (!a.report.empty()) {
      ofstream rep(a.report);
      st.Error(*make_eq(a, t_now, beta), uh, rep);
    }
  };
  auto adi_step = [&](auto& st) {
    auto eq = make_eq(a, t_now, beta);
    st.Solve_2nd(*eq, inter, uh, beta);
  };
  char lod_m = a.method == "lod-ie" ? 'I' : 'C';
  auto lod_step = [&](auto& st) {
    auto eq = make_eq(a, t_now, beta);
    st.Solve_2nd(*eq, inter, uh, beta, lod_m);
  };
  auto ts_step = [&](auto& st) {
    auto e0 = make_eq(a, t_now - a.dt, beta);
    auto eh = make_eq(a, t_now - 0.5 * a.dt, beta);
    auto e1 = make_eq(a, t_now, beta);
    st.Solve_2nd(*e0, *eh, *e1, inter, uh, beta);
  };

  bool lod = a.method == "lod-ie" || a.method == "lod-cn";
  if (a.method != "adi" && !lod && a.method != "ts") usage();
#ifdef MTS_DROPIN
  if (a.gpu) {
    int method = a.method == "adi" ? MTS_ADI : a.method == "lod-ie" ? MTS_LOD_IE : a.method == "lod-cn" ? MTS_LOD_CN : MTS_TS;
    try {
      // (the stepper is told eq 8 for any Equation the loop builds other than
      // Eq_0: it must refuse the ones it does not evaluate)
      mts::GpuStepper st(inter, mesh, beta, time, 2, method, a.eq == 0 ? 0 : 8);
      if (a.method == "adi")
        run(st, adi_step);
      else if (lod)
        run(st, lod_step);
      else
        run(st, ts_step);
      if (!a.fp_errors.empty()) {
        // the device's fictitious-point report, beside the reference's below
        ofstream o(a.fp_errors + ".gpu");
        st.Error_Fp(*make_eq(a, t_now, beta), o);
      }
      if (!a.jump_errors.empty()) {
        ofstream o(a.jump_errors + ".gpu");
        st.Error_Jump(*make_eq(a, t_now, beta), o);
      }
    } catch (const std::exception& e) {
      fprintf(stderr, "mts_dropin: %s\n", e.what());
      return 3;
    }
  } else
#endif
  if (a.method == "adi") {
    Douglas_ADI st(inter, mesh, beta, time, 2);
    run(st, adi_step);
  } else if (lod) {
    LOD st(inter, mesh, beta, time);
    run(st, lod_step);
  } else {
    TS st(inter, mesh, beta, time);
    run(st, ts_step);
  }
  norms(*make_eq(a, t_now, beta));
  if (!a.dump_u.empty()) dump_field(a.dump_u, uh, nx, ny, nz);
  if (a.write_txt) {
    if (a.eq > 7) {
      fprintf(stderr, "--write-txt: the reference's Write_txt knows Eq_0..Eq_7 only\n");
      return 2;
    }
    ref_write_txt(inter, mesh, beta, uh, a.eq, t_now);
  }
  if (!a.fp_errors.empty()) {
    // The fictitious points' errors against the exact solution at the final
    // time, as the reference's time loops report them (helper.h:230-231):
    // Refresh_Fp, then Error_Fp's maximum and root mean square recomputed
    // here in its loop order (intersection.cc:4667-4771) so that the values
    // stay in binary, followed by Error_Fp's own text.
    inter.Refresh_Fp(*make_eq(a, t_now, beta));
    double fmax = 0, fsum = 0;
    long long fno = 0;
    auto add = [&](Intersection_Data& d) {
      for (size_t i = 0; i < d.err.errr.size(); i++) {
        fno += 2;
        fsum += d.err.errl[i] * d.err.errl[i];
        fsum += d.err.errr[i] * d.err.errr[i];
        if (fabs(d.err.errl[i]) > fmax) fmax = fabs(d.err.errl[i]);
        if (fabs(d.err.errr[i]) > fmax) fmax = fabs(d.err.errr[i]);
      }
    };
    for (int ix = 1; ix < nx - 1; ix++)
      for (int iy = 1; iy < ny - 1; iy++)
        for (auto& d : inter.ifpz[ix][iy])
          if (d.ID != 0) add(d);
    for (int ix = 1; ix < nx - 1; ix++)
      for (int iz = 1; iz < nz - 1; iz++)
        for (auto& d : inter.ifpy[ix][iz])
          if (d.ID != 0) add(d);
    for (int iy = 1; iy < ny - 1; iy++)
      for (int iz = 1; iz < nz - 1; iz++)
        for (auto& d : inter.ifpx[iy][iz])
          if (d.ID != 0) add(d);
    FILE* f = fopen(a.fp_errors.c_str(), "w");
    fprintf(f, "%.17g %.17g %.17g %lld\n", fmax, sqrt(fsum / fno), fsum, fno);
    fclose(f);
    ofstream txt(a.fp_errors, ios::app);
    inter.Error_Fp(txt);
  }
  if (!a.jump_errors.empty()) {
    // The jumps' errors at the final time (helper.h:233-234): Refresh_Jump,
    // then Error_Jump's maximum and root mean square recomputed here in its
    // loop order (intersection.cc:4594-4662), followed by its own text.  In
    // the noaux build Refresh_Jump's eta / tau estimates are 0, which
    // Error_Jump does not read.
    inter.Refresh_Jump(*make_eq(a, t_now, beta), uh, beta);
    double jmax = 0, jsum = 0;
    long long jno = 0;
    auto add = [&](Intersection_Data& d) {
      jno += 1;
      jsum += d.jump.err * d.jump.err;
      if (fabs(d.jump.err) > jmax) jmax = fabs(d.jump.err);
    };
    for (int ix = 1; ix < nx - 1; ix++)
      for (int iy = 1; iy < ny - 1; iy++)
        for (auto& d : inter.ifpz[ix][iy])
          if (d.ID != 0) add(d);
    for (int ix = 1; ix < nx - 1; ix++)
      for (int iz = 1; iz < nz - 1; iz++)
        for (auto& d : inter.ifpy[ix][iz])
          if (d.ID != 0) add(d);
    for (int iy = 1; iy < ny - 1; iy++)
      for (int iz = 1; iz < nz - 1; iz++)
        for (auto& d : inter.ifpx[iy][iz])
          if (d.ID != 0) add(d);
    FILE* f = fopen(a.jump_errors.c_str(), "w");
    fprintf(f, "%.17g %.17g %.17g %lld\n", jmax, sqrt(jsum / jno), jsum, jno);
    fclose(f);
    ofstream txt(a.jump_errors, ios::app);
    inter.Error_Jump(txt);
  }

  printf(
      "{\"nx\": %d, \"ny\": %d, \"nz\": %d, \"steps\": %d, \"t\": %.17g, \"lmax\": %.17g, "
      "\"l2\": %.17g, \"argmax\": [%d, %d, %d], \"ncross\": [%zu, %zu, %zu], "
      "\"setup_seconds\": %.6f, \"step_seconds\": %.6f}\n",
      nx, ny, nz, steps, t_now, lmax, l2, am[0], am[1], am[2], ncross[0], ncross[1], ncross[2],
      chrono::duration<double>(t_setup1 - t_setup0).count(), step_seconds);
  return 0;
}

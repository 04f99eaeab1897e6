// rs_run.cpp — the reference's host program (main(), fun.cu:344-530 ≡
// src/main.cu:156-240) rebuilt on the C-ABI of include/rs_b200.h.
//
// The loop body keeps the reference's order and cadences:
//   set_fields_output  every step_fields   (fun.cu:621-666)  data/c_<k>.txt, data/phi0_<k>.txt
//   set_tip_output     every step_tip      (fun.cu:3024-3072) tip row on stdout and tip.txt
//   set_check_point    every step_check_point and at the end (fun.cu:668-691)
//                      data/check_point_{c,phi}.bin, parameters.txt, check_point_temperature.bin
//   set_pull_back      every step_pull_back (fun.cu:693-742) coarse tip on the device, offset.txt
//   step               rs_step (pull_back + compute_phi + compute_psi + compute_c_CALPHAD)
//   TFC                rs_integrate_phi + rs_temperature_step (fun.cu:486-497)
//   l_offset_Vp       += Vp_ramp(step tau0 dt) dt tau0 / (S W0) (fun.cu:508-509)
// Restart (--load) reads parameters.txt and the checkpoints as the reference's
// if_load path does (fun.cu:587-603), with psi = phi (one orientation).
// Fields are FP64 in the reference layout by default; --precision f32 runs the
// FP32 path (c stored as c - cinf) and converts at every file boundary.
#include <cuda_runtime.h>

#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "rs_b200.h"

namespace {

void die(const char *what) {
  std::fprintf(stderr, "rs_run: %s: %s\n", what, rs_last_error());
  std::exit(1);
}
void check(int rc, const char *what) {
  if (rc != RS_OK) die(what);
}
void cuda_check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) {
    std::fprintf(stderr, "rs_run: %s: %s\n", what, cudaGetErrorString(e));
    std::exit(1);
  }
}

struct Options {
  int nx = 768, ny = 832, i_tip = -1;
  long long steps = -1;  // default: total_step of total_time_ns
  bool f32 = false, load = false, fields = true;
  int tfc = -1;
  double Vp = -1, GG = -1, noise = 0.0;
  long long seed = 3, planar_seed = -1;
  int tip_every = 0, fields_every = 0, check_every = 0;
  std::string out = ".";
};

void usage() {
  std::puts(
      "usage: rs_run [--nx N] [--ny N] [--i-tip N] [--steps K] [--precision f64|f32] [--tfc 0|1]\n"
      "              [--Vp m/s] [--GG K/nm] [--noise A] [--seed S] [--planar SEED] [--load]\n"
      "              [--tip-every N] [--fields-every N] [--check-every N] [--no-fields] [--out DIR]");
}

Options parse(int argc, char **argv) {
  Options o;
  for (int k = 1; k < argc; ++k) {
    const std::string a = argv[k];
    auto val = [&]() -> const char * {
      if (k + 1 >= argc) {
        usage();
        std::exit(2);
      }
      return argv[++k];
    };
    if (a == "--nx") o.nx = std::atoi(val());
    else if (a == "--ny") o.ny = std::atoi(val());
    else if (a == "--i-tip") o.i_tip = std::atoi(val());
    else if (a == "--steps") o.steps = std::atoll(val());
    else if (a == "--precision") o.f32 = std::string(val()) == "f32";
    else if (a == "--tfc") o.tfc = std::atoi(val());
    else if (a == "--Vp") o.Vp = std::atof(val());
    else if (a == "--GG") o.GG = std::atof(val());
    else if (a == "--noise") o.noise = std::atof(val());
    else if (a == "--seed") o.seed = std::atoll(val());
    else if (a == "--planar") o.planar_seed = std::atoll(val());
    else if (a == "--load") o.load = true;
    else if (a == "--tip-every") o.tip_every = std::atoi(val());
    else if (a == "--fields-every") o.fields_every = std::atoi(val());
    else if (a == "--check-every") o.check_every = std::atoi(val());
    else if (a == "--no-fields") o.fields = false;
    else if (a == "--out") o.out = val();
    else if (a == "-h" || a == "--help") {
      usage();
      std::exit(0);
    } else {
      std::fprintf(stderr, "rs_run: unknown option %s\n", a.c_str());
      usage();
      std::exit(2);
    }
  }
  return o;
}

void ensure_dir(const std::string &d) {
  if (mkdir(d.c_str(), 0755) != 0 && errno != EEXIST) {
    std::fprintf(stderr, "rs_run: cannot create %s\n", d.c_str());
    std::exit(1);
  }
}

// Device field set with host staging in the reference's FP64 layout.
struct Fields {
  rs_fields f{};
  size_t n = 0;
  bool f32 = false;
  double cinf = 0.0;
  void alloc(size_t cells, bool use_f32, double c_inf) {
    n = cells;
    f32 = use_f32;
    cinf = c_inf;
    const size_t es = f32 ? sizeof(float) : sizeof(double);
    cuda_check(cudaMalloc(&f.c, n * es), "cudaMalloc c");
    cuda_check(cudaMalloc(&f.psi, n * es), "cudaMalloc psi");
    f.phi = nullptr;
    f.precision = f32 ? RS_F32 : RS_F64;
    f.pitch = 0;
  }
  void release() {
    cudaFree(f.c);
    cudaFree(f.psi);
  }
  // c (true composition) and phi = clamp(psi) as doubles
  void download(std::vector<double> &c, std::vector<double> &phi, std::vector<double> *psi = nullptr) const {
    c.resize(n);
    phi.resize(n);
    std::vector<double> p(n);
    if (f32) {
      std::vector<float> cf(n), pf(n);
      cuda_check(cudaMemcpy(cf.data(), f.c, n * sizeof(float), cudaMemcpyDeviceToHost), "D2H c");
      cuda_check(cudaMemcpy(pf.data(), f.psi, n * sizeof(float), cudaMemcpyDeviceToHost), "D2H psi");
      for (size_t k = 0; k < n; ++k) {
        c[k] = cinf + (double)cf[k];
        p[k] = pf[k];
      }
    } else {
      cuda_check(cudaMemcpy(c.data(), f.c, n * sizeof(double), cudaMemcpyDeviceToHost), "D2H c");
      cuda_check(cudaMemcpy(p.data(), f.psi, n * sizeof(double), cudaMemcpyDeviceToHost), "D2H psi");
    }
    for (size_t k = 0; k < n; ++k) phi[k] = std::fmin(std::fmax(p[k], -1.0), 1.0);
    if (psi) *psi = p;
  }
  void upload(const std::vector<double> &c, const std::vector<double> &psi) {
    if (f32) {
      std::vector<float> cf(n), pf(n);
      for (size_t k = 0; k < n; ++k) {
        cf[k] = (float)(c[k] - cinf);
        pf[k] = (float)psi[k];
      }
      cuda_check(cudaMemcpy(f.c, cf.data(), n * sizeof(float), cudaMemcpyHostToDevice), "H2D c");
      cuda_check(cudaMemcpy(f.psi, pf.data(), n * sizeof(float), cudaMemcpyHostToDevice), "H2D psi");
    } else {
      cuda_check(cudaMemcpy(f.c, c.data(), n * sizeof(double), cudaMemcpyHostToDevice), "H2D c");
      cuda_check(cudaMemcpy(f.psi, psi.data(), n * sizeof(double), cudaMemcpyHostToDevice), "H2D psi");
    }
  }
};

}  // namespace

int main(int argc, char **argv) {
  const Options o = parse(argc, argv);
  if (rs_abi_version() != RS_ABI_VERSION) {
    std::fprintf(stderr, "rs_run: library ABI %d, header %d\n", rs_abi_version(), RS_ABI_VERSION);
    return 1;
  }
  ensure_dir(o.out);
  ensure_dir(o.out + "/data");

  // ---- parameters (set_parameters, fun.cu:1984-2058)
  rs_params p;
  check(rs_default_params(&p), "rs_default_params");
  p.nx_all = o.nx;
  p.ny_all = o.ny;
  p.i_tip_target = o.i_tip >= 0 ? o.i_tip : o.nx - 268;
  if (o.tfc >= 0) p.tfc = o.tfc;
  if (o.Vp > 0) p.Vp = o.Vp;
  if (o.GG > 0) p.GG = o.GG;
  p.noise_amplitude = o.noise;
  p.seed = (uint64_t)o.seed;

  rs_run_state rs{};
  if (o.load) {
    check(rs_read_parameters((o.out + "/parameters.txt").c_str(), p.tfc, &rs), "rs_read_parameters");
    // the loaded run continues from its dynamic state (load_parameters, fun.cu:2204-2388)
    p.delta_initial = rs.delta;
    p.i_offset_history_initial = rs.i_offset_history;
    p.l_offset_Vp_initial = rs.l_offset_Vp;
  }
  rs_ctx *ctx = nullptr;
  check(rs_create(&p, &ctx), "rs_create");
  rs_derived d;
  check(rs_get_derived(ctx, &d), "rs_get_derived");
  const int step_tip = o.tip_every > 0 ? o.tip_every : d.step_tip;
  const int step_fields = o.fields_every > 0 ? o.fields_every : d.step_fields;
  const int step_check = o.check_every > 0 ? o.check_every : d.step_check_point;
  const size_t cells = (size_t)p.nx_all * p.ny_all;

  Fields cur, nxt;
  cur.alloc(cells, o.f32, p.cinf);
  nxt.alloc(cells, o.f32, p.cinf);
  double *d_T = nullptr, *d_T_next = nullptr, *d_dphidt = nullptr, *d_T_fine = nullptr;
  const size_t cellsT = (size_t)d.NxT_all * d.NyT_all;
  if (p.tfc) {
    cuda_check(cudaMalloc(&d_T, cellsT * sizeof(double)), "cudaMalloc T");
    cuda_check(cudaMalloc(&d_T_next, cellsT * sizeof(double)), "cudaMalloc T_next");
    cuda_check(cudaMalloc(&d_dphidt, cellsT * sizeof(double)), "cudaMalloc dphidt");
    cuda_check(cudaMalloc(&d_T_fine, cells * sizeof(double)), "cudaMalloc T_fine");
  }
  int32_t *d_itip = nullptr;
  rs_tip *d_tip = nullptr;
  cuda_check(cudaMalloc(&d_itip, sizeof(int32_t)), "cudaMalloc itip");
  cuda_check(cudaMalloc(&d_tip, sizeof(rs_tip)), "cudaMalloc tip");

  // ---- state of the host loop (the constants struct fields the loop updates)
  long long initial_step = 0;
  int i_offset_history = p.i_offset_history_initial;
  double l_offset_Vp = p.l_offset_Vp_initial;
  double delta = p.delta_initial;
  double x_tip_history = p.i_tip_target * p.dx;  // set_parameters, fun.cu:1997
  int i_left_end = d.i_left_end_initial, i_left_end_T = d.i_left_end_initial;
  std::vector<double> hc, hphi, hpsi, hT;

  if (o.load) {  // if_load path (fun.cu:587-603)
    initial_step = rs.step;
    i_left_end = rs.i_left_end;
    i_left_end_T = rs.i_left_end;
    hc.resize(cells);
    hphi.resize(cells);
    check(rs_read_check_point((o.out + "/data/check_point_c.bin").c_str(), hc.data(), p.nx_all, p.ny_all),
          "check_point_c");
    check(rs_read_check_point((o.out + "/data/check_point_phi.bin").c_str(), hphi.data(), p.nx_all, p.ny_all),
          "check_point_phi");
    cur.upload(hc, hphi);  // psi = phi for one orientation (get_local_psi)
    if (p.tfc) {
      hT.assign(cellsT, 0.0);
      check(rs_read_check_point_temperature((o.out + "/data/check_point_temperature.bin").c_str(), hT.data(),
                                            d.NxT, d.NyT, d.NxT_all),
            "check_point_temperature");
      cuda_check(cudaMemcpy(d_T, hT.data(), cellsT * sizeof(double), cudaMemcpyHostToDevice), "H2D T");
    }
    std::printf("Load data finished!\n\n");
  } else {  // initial (fun.cu:559-571)
    if (o.planar_seed >= 0)
      check(rs_initial_planar(ctx, &cur.f, p.cinf, 0.8795504308633851, (uint64_t)o.planar_seed, nullptr),
            "rs_initial_planar");
    else
      check(rs_initial(ctx, &cur.f, nullptr), "rs_initial");
    if (p.tfc) check(rs_temperature_init(ctx, d_T, nullptr), "rs_temperature_init");
  }
  // --steps K runs K iterations (the reference loop runs step = initial .. total_step)
  const long long total_step = o.steps >= 0 ? initial_step + o.steps - 1 : d.total_step;
  const double tau0 = d.tau0, dt = d.dt;
  auto vp_ramp = [&](double t_ns) { return p.vp_ramp ? p.Vp + 0.0107587 * (t_ns * 0.001) : p.Vp; };
  auto get_delta = [&](int i) {  // fun.cu:1610-1619 (frozen temperature)
    return p.delta_initial +
           p.GG * (i - p.i_tip_target + i_offset_history - p.i_offset_history_initial) * p.dx * p.S * p.W0 / d.deltaT0 -
           p.GG * (l_offset_Vp - p.l_offset_Vp_initial) * p.S * p.W0 / d.deltaT0;
  };

  FILE *tipf = std::fopen((o.out + "/tip.txt").c_str(), o.load ? "a" : "w");
  FILE *offf = std::fopen((o.out + "/data/offset.txt").c_str(), o.load ? "a" : "w");
  if (!tipf || !offf) {
    std::fprintf(stderr, "rs_run: cannot open output files in %s\n", o.out.c_str());
    return 1;
  }
  if (!o.load)
    std::fprintf(tipf,
                 "(1)        (2)        (3)        (4)        (5)        (6)        (7)        (8)        (9)        "
                 "(10)       (11)\nstep       t[us]      Δtip       Ttip[K]    Vtip[m/s]  Vp[m/s]    tip.R[nm]  "
                 "tip.i      tip.j      tip.x      tip.y\n");

  auto save_check_point = [&](long long step) {  // set_check_point (fun.cu:668-691)
    cur.download(hc, hphi);
    check(rs_write_check_point((o.out + "/data/check_point_c.bin").c_str(), hc.data(), p.nx_all, p.ny_all),
          "check_point_c");
    check(rs_write_check_point((o.out + "/data/check_point_phi.bin").c_str(), hphi.data(), p.nx_all, p.ny_all),
          "check_point_phi");
    rs_run_state s{};
    s.step = step;
    s.i_offset_history = i_offset_history;
    s.l_offset_Vp = l_offset_Vp;
    s.delta = delta;
    s.i_left_end_initial = d.i_left_end_initial;
    s.i_left_end = i_left_end;
    check(rs_write_parameters((o.out + "/parameters.txt").c_str(), &p, &s), "rs_write_parameters");
    if (p.tfc) {
      hT.resize(cellsT);
      cuda_check(cudaMemcpy(hT.data(), d_T, cellsT * sizeof(double), cudaMemcpyDeviceToHost), "D2H T");
      check(rs_write_check_point_temperature((o.out + "/data/check_point_temperature.bin").c_str(), hT.data(),
                                             d.NxT, d.NyT, d.NxT_all),
            "check_point_temperature");
    }
  };

  std::printf("total steps for this simulation is: %lld\n", total_step);
  long long step;
  for (step = initial_step; step <= total_step; ++step) {
    // set_fields_output (fun.cu:621-666)
    if (o.fields && (step % step_fields == 0 || step == initial_step)) {
      cur.download(hc, hphi);
      const int index = (int)(step / step_fields);
      char name[512];
      std::snprintf(name, sizeof(name), "%s/data/c_%d.txt", o.out.c_str(), index);
      check(rs_write_field_text(name, hc.data(), p.nx_all, p.ny_all, 1, 1), "save_field c");
      std::snprintf(name, sizeof(name), "%s/data/phi0_%d.txt", o.out.c_str(), index);
      check(rs_write_field_text(name, hphi.data(), p.nx_all, p.ny_all, 1, 1), "save_field phi0");
    }
    // set_tip_output (fun.cu:3024-3072)
    if (step % step_tip == 0 || step == initial_step) {
      check(rs_precise_tip(ctx, &cur.f, d_tip, nullptr), "rs_precise_tip");
      rs_tip tip;
      cuda_check(cudaMemcpy(&tip, d_tip, sizeof(tip), cudaMemcpyDeviceToHost), "D2H tip");
      const double x_tip_now = (i_offset_history + tip.x) * p.dx;
      double V_tip = (x_tip_now - x_tip_history) * p.S * p.W0 / (step_tip * tau0 * dt);
      x_tip_history = x_tip_now;
      if (V_tip < 0.0) V_tip = 0.01;
      if (V_tip > 10.0) V_tip = 10.0;
      if (step == initial_step) V_tip = NAN;
      double T_tip;
      if (p.tfc) {
        check(rs_interpolate_temperature(ctx, d_T, d_T_fine, i_left_end, nullptr), "rs_interpolate_temperature");
        cuda_check(cudaMemcpy(&T_tip, d_T_fine + tip.i, sizeof(double), cudaMemcpyDeviceToHost), "D2H T_tip");
        delta = (T_tip - p.Tmelt) / d.deltaT0;
      } else {
        delta = get_delta(tip.i);
        T_tip = delta * d.deltaT0 + p.Tmelt;
      }
      char row[512];
      std::snprintf(row, sizeof(row), "%-10lld %-10e %-10e %-10e %-10e %-10e %-10e %-10d %-10d %-10e %-10e\n", step,
                    step * dt * tau0 * 1e-3, delta, T_tip, V_tip, vp_ramp(step * tau0 * dt), tip.R, tip.i, tip.j,
                    tip.x, tip.y);
      std::fputs(row, stdout);
      std::fputs(row, tipf);
      std::fflush(tipf);
    }
    // set_check_point (fun.cu:668-691)
    if (step % step_check == 0) save_check_point(step);

    rs_step_args a{};
    a.step = step;
    // set_pull_back (fun.cu:693-742): the shift is applied inside rs_step
    if (step % d.step_pull_back == 0) {
      check(rs_itip(ctx, &cur.f, d_itip, nullptr), "rs_itip");
      int32_t itip = 0;
      cuda_check(cudaMemcpy(&itip, d_itip, sizeof(itip), cudaMemcpyDeviceToHost), "D2H itip");
      a.pull_back = 1;
      a.i_offset = itip - p.i_tip_target;
      i_offset_history += a.i_offset;
      if (p.tfc) i_left_end = d.i_left_end_initial + i_offset_history - (int)(l_offset_Vp / p.dx);
      std::fprintf(offf, "%lld\t%d\t%d\t%d\n", step, a.i_offset, i_offset_history, d.step_pull_back);
    }
    a.i_offset_history = i_offset_history;
    a.l_offset_Vp = l_offset_Vp;
    if (p.tfc) {
      a.T_coarse = d_T;
      a.i_left_end = i_left_end;
      a.i_left_end_T = i_left_end_T;
    }
    check(rs_step(ctx, &cur.f, &nxt.f, &a, nullptr), "rs_step");
    if (p.tfc) {  // fun.cu:486-497
      check(rs_integrate_phi(ctx, &cur.f, &nxt.f, d_dphidt, i_left_end, nullptr), "rs_integrate_phi");
      check(rs_temperature_step(ctx, d_T, d_T_next, d_dphidt, step, nullptr), "rs_temperature_step");
      i_left_end_T = i_left_end;  // the fine T follows the interpolation at this i_left_end
    }
    std::swap(cur, nxt);
    l_offset_Vp += vp_ramp(step * tau0 * dt) * dt * tau0 / (p.S * p.W0);
  }
  save_check_point(step);  // final check point (fun.cu:516)
  check(rs_device_status(ctx, nullptr), "rs_device_status");
  std::fclose(tipf);
  std::fclose(offf);
  cur.release();
  nxt.release();
  cudaFree(d_T);
  cudaFree(d_T_next);
  cudaFree(d_dphidt);
  cudaFree(d_T_fine);
  cudaFree(d_itip);
  cudaFree(d_tip);
  rs_destroy(ctx);
  return 0;
}

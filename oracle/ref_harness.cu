// ref_harness.cu — drives the reference's own code (test infrastructure).
//
// Compiled by oracle/ref_build.sh together with a macro-patched copy of the
// reference's old-fun.cu (kernels fun.cu:1030-1492 equivalents, CALPHAD
// fun.cu:1628-1720, tip tracker fun.cu:2608-2954).  The reference's main() is
// renamed; this file supplies a small command-line front end that feeds the
// reference routines with caller-provided inputs, the same way the reference's
// restart path injects a checkpoint (load_check_point, fun.cu:1894-1918), and
// writes their raw FP64 outputs.
//
//   ref_harness calphad <in.bin> <out.bin>   host: Gl, Gs, Glc, Gsc on (T, c)
//   ref_harness tip <psi.bin>                host: get_itip_all_grain, get_precise_tip
//   ref_harness step <in_dir> <out_dir> <nsteps> <dt> <delta_initial>
//                    <pull_back_first:0|1> <i_offset|auto>
//                                            GPU: pull_back, compute_phi,
//                                            compute_psi, compute_c_CALPHAD
//   ref_harness bench <nsteps> <dt>          GPU: times the three step kernels
// Built from the coarse-temperature copy (ifTFC 1), the step modes give way to
//   ref_harness_tfc tfc <in_dir> <out_dir> <nsteps> <dt> <delta_initial> <step_pull_back>
//                                            GPU: the main() loop with TFC
#include REF_PATCHED
#undef main

#include <cstring>
#include <string>
#include <vector>

static std::vector<double> read_doubles(const std::string &path, size_t n) {
  std::vector<double> v(n);
  FILE *f = fopen(path.c_str(), "rb");
  if (!f) { fprintf(stderr, "cannot open %s\n", path.c_str()); exit(2); }
  if (fread(v.data(), sizeof(double), n, f) != n) { fprintf(stderr, "short read %s\n", path.c_str()); exit(2); }
  fclose(f);
  return v;
}

static void write_doubles(const std::string &path, const double *p, size_t n) {
  FILE *f = fopen(path.c_str(), "wb");
  if (!f) { fprintf(stderr, "cannot write %s\n", path.c_str()); exit(2); }
  fwrite(p, sizeof(double), n, f);
  fclose(f);
}

#define CK(x)                                                                 \
  do {                                                                        \
    cudaError_t e_ = (x);                                                     \
    if (e_ != cudaSuccess) {                                                  \
      fprintf(stderr, "CUDA %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, \
              __LINE__);                                                      \
      exit(3);                                                                \
    }                                                                         \
  } while (0)

static void fill_constants(constants *p, double dt, double delta_initial) {
  memset(p, 0, sizeof(*p));
  p->dt = dt;
  p->delta_initial = delta_initial;
  p->delta = delta_initial;
  p->i_offset_history_initial = 0;
  p->i_offset_history = 0;
  p->l_offset_Vp_initial = 0;
  p->l_offset_Vp = 0;
}

int main(int argc, char **argv) {
  if (argc < 2) { fprintf(stderr, "usage: see ref_harness.cu\n"); return 1; }
  const std::string mode = argv[1];
  const size_t N = (size_t)Nx_all * Ny_all;

  if (mode == "calphad") {
    FILE *f = fopen(argv[2], "rb");
    if (!f) return 2;
    double nd = 0;
    if (fread(&nd, sizeof(double), 1, f) != 1) return 2;
    size_t n = (size_t)nd;
    std::vector<double> T(n), c(n), out(4 * n);
    if (fread(T.data(), sizeof(double), n, f) != n) return 2;
    if (fread(c.data(), sizeof(double), n, f) != n) return 2;
    fclose(f);
    for (size_t k = 0; k < n; ++k) {
      out[4 * k + 0] = Gl(T[k], c[k]);
      out[4 * k + 1] = Gs(T[k], c[k]);
      out[4 * k + 2] = Glc(T[k], c[k]);
      out[4 * k + 3] = Gsc(T[k], c[k]);
    }
    write_doubles(argv[3], out.data(), out.size());
    return 0;
  }

  if (mode == "tip") {
    std::vector<double> psi = read_doubles(argv[2], N);
    int itip = get_itip_all_grain(psi.data());
    TIP tip;
    get_precise_tip(psi.data(), &tip, 0);
    printf("%d %d %d %.17g %.17g %.17g\n", itip, tip.i, tip.j, tip.x, tip.y, tip.R);
    return 0;
  }

#if (ifTFC)
  // The coarse-temperature loop of the reference's main() (old-fun.cu:386-440
  // with ifTFC 1): pull_back every step_pull_back steps with set_pull_back's
  // i_offset / i_left_end bookkeeping (old-fun.cu:606-616), compute_phi,
  // compute_psi, compute_c_CALPHAD on the interpolated T_fine, then
  // integrate_phi, ratio_dt_dtT x compute_temperature and
  // interpolate_temperature.  T starts from initial_temperature and
  // interpolate_temperature as set_initial does (old-fun.cu:491-492).
  //   ref_harness_tfc tfc <in_dir> <out_dir> <nsteps> <dt> <delta_initial> <step_pull_back>
  // in_dir holds c/phi/psi.bin; out_dir receives c/phi/psi/T/T_fine.bin and
  // the i_offset of every pull-back on stdout.
  if (mode == "tfc") {
    const std::string in_dir = argv[2], out_dir = argv[3];
    const long nsteps = atol(argv[4]);
    const double dt = atof(argv[5]);
    const double delta_initial = atof(argv[6]);
    const int step_pull_back = atoi(argv[7]);
    std::vector<double> h_c = read_doubles(in_dir + "/c.bin", N);
    std::vector<double> h_phi = read_doubles(in_dir + "/phi.bin", N);
    std::vector<double> h_psi = read_doubles(in_dir + "/psi.bin", N);
    constants h_para;
    memset(&h_para, 0, sizeof(h_para));
    set_parameters(&h_para);  // the reference's TFC geometry (NxT, NyT, Tcold, Thot, i_left_end_initial)
    // the harness time step replaces set_parameters' 0.6 factor; the coarse
    // sub-step count follows it by set_parameters' own rule
    h_para.dt = dt;
    {
      constexpr real DDT = DT * tau0 / pow2(SS * W0 * ratio_dxT_dx);
      constexpr real dtT = 0.9 * dx * dx / (4.0 * DDT);
      h_para.ratio_dt_dtT = 1;
      if (dtT < h_para.dt) h_para.ratio_dt_dtT = ceil(h_para.dt / dtT);
      h_para.dtT = h_para.dt / h_para.ratio_dt_dtT;
    }
    h_para.delta_initial = delta_initial;
    h_para.delta = delta_initial;
    h_para.step_pull_back = step_pull_back;
    printf("tfc NxT %d NyT %d NxT_all %d NyT_all %d ratio_dt_dtT %d i_left_end_initial %d\n", h_para.NxT,
           h_para.NyT, h_para.NxT_all, h_para.NyT_all, h_para.ratio_dt_dtT, h_para.i_left_end_initial);
    real h_orientation[num_axes * num_orientation];
    set_orientation(h_orientation, alpha0, beta0, gamma0);
    const size_t bytes = N * sizeof(real), bytesT = (size_t)h_para.NxT_all * h_para.NyT_all * sizeof(real);
    real *d_c, *d_phi, *d_psi, *d_c_next, *d_phi_next, *d_psi_next, *d_orientation, *d_temp;
    real *d_T, *d_T_next, *d_T_fine, *d_dphidt;
    constants *d_para;
    CK(cudaMalloc(&d_c, bytes));
    CK(cudaMalloc(&d_phi, bytes));
    CK(cudaMalloc(&d_psi, bytes));
    CK(cudaMalloc(&d_c_next, bytes));
    CK(cudaMalloc(&d_phi_next, bytes));
    CK(cudaMalloc(&d_psi_next, bytes));
    // compute_temperature reads its five-point stencil before testing the
    // interior (old-fun.cu:1379-1398), so threads on the array's border read
    // one row (NxT_all doubles) and one element outside it; each coarse
    // array gets a zeroed guard of NxT_all + 1 doubles on both sides, which
    // keeps those reads inside the allocation.  Their values only reach
    // threads that write nothing from them.
    const size_t guard = (size_t)h_para.NxT_all + 1;
    real *g_T, *g_T_next, *g_dphidt;
    CK(cudaMalloc(&g_T, bytesT + 2 * guard * sizeof(real)));
    CK(cudaMalloc(&g_T_next, bytesT + 2 * guard * sizeof(real)));
    CK(cudaMalloc(&g_dphidt, bytesT + 2 * guard * sizeof(real)));
    CK(cudaMemset(g_T, 0, bytesT + 2 * guard * sizeof(real)));
    CK(cudaMemset(g_T_next, 0, bytesT + 2 * guard * sizeof(real)));
    CK(cudaMemset(g_dphidt, 0, bytesT + 2 * guard * sizeof(real)));
    d_T = g_T + guard;
    d_T_next = g_T_next + guard;
    d_dphidt = g_dphidt + guard;
    CK(cudaMalloc(&d_T_fine, bytes));
    CK(cudaMalloc(&d_orientation, sizeof(h_orientation)));
    CK(cudaMalloc(&d_para, sizeof(constants)));
    CK(cudaMemset(d_c_next, 0, bytes));
    CK(cudaMemset(d_phi_next, 0, bytes));
    CK(cudaMemset(d_psi_next, 0, bytes));
    CK(cudaMemcpy(d_para, &h_para, sizeof(constants), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_orientation, h_orientation, sizeof(h_orientation), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_c, h_c.data(), bytes, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_phi, h_phi.data(), bytes, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_psi, h_psi.data(), bytes, cudaMemcpyHostToDevice));
    dim3 threadsPerBlock(BLOCK_SIZE_X, BLOCK_SIZE_Y);
    dim3 numBlocks(Nx_all / threadsPerBlock.x, Ny_all / threadsPerBlock.y);
    dim3 threadsPerBlockT(BLOCK_SIZE_T_X, BLOCK_SIZE_T_Y);
    dim3 numBlocksT(h_para.NxT_all / threadsPerBlockT.x, h_para.NyT_all / threadsPerBlockT.y);
    initial_temperature<<<numBlocksT, threadsPerBlockT>>>(d_T, d_para);
    interpolate_temperature<<<numBlocks, threadsPerBlock>>>(d_T, d_T_fine, d_para, h_para.i_left_end, 0);
    CK(cudaGetLastError());
    for (long step = 0; step < nsteps; ++step) {
      if (step % h_para.step_pull_back == 0) {
        CK(cudaMemcpy(h_psi.data(), d_psi, bytes, cudaMemcpyDeviceToHost));
        h_para.i_offset = get_itip_all_grain(h_psi.data()) - i_tip_target;
        h_para.i_offset_history += h_para.i_offset;
        h_para.i_left_end = h_para.i_left_end_initial + h_para.i_offset_history - int(h_para.l_offset_Vp / dx);
        CK(cudaMemcpy(d_para, &h_para, sizeof(constants), cudaMemcpyHostToDevice));
        printf("pull_back step %ld i_offset %d i_left_end %d\n", step, h_para.i_offset, h_para.i_left_end);
        pull_back<<<numBlocks, threadsPerBlock>>>(d_c, d_phi, d_psi, d_c_next, d_phi_next, d_psi_next,
                                                  h_para.i_offset, step);
        d_temp = d_c; d_c = d_c_next; d_c_next = d_temp;
        d_temp = d_phi; d_phi = d_phi_next; d_phi_next = d_temp;
        d_temp = d_psi; d_psi = d_psi_next; d_psi_next = d_temp;
      }
      compute_phi<<<numBlocks, threadsPerBlock>>>(d_c, d_phi, d_psi, d_T_fine, d_c_next, d_phi_next, d_psi_next,
                                                  d_orientation, NULL, d_para, step, h_para.i_offset_history,
                                                  h_para.l_offset_Vp);
      compute_psi<<<numBlocks, threadsPerBlock>>>(d_c, d_phi, d_psi, d_c_next, d_phi_next, d_psi_next,
                                                  d_orientation, NULL, d_para, step);
      compute_c_CALPHAD<<<numBlocks, threadsPerBlock>>>(d_c, d_phi, d_psi, d_T_fine, d_c_next, d_phi_next,
                                                        d_psi_next, d_orientation, NULL, d_para, step,
                                                        h_para.i_offset_history, h_para.l_offset_Vp);
      integrate_phi<<<numBlocksT, threadsPerBlockT>>>(d_dphidt, d_psi, d_psi_next, d_para, h_para.i_left_end, step);
      for (int sub_step = 0; sub_step < h_para.ratio_dt_dtT; sub_step++) {
        compute_temperature<<<numBlocksT, threadsPerBlockT>>>(d_T, d_T_next, d_dphidt, d_para, step, sub_step);
        d_temp = d_T; d_T = d_T_next; d_T_next = d_temp;
      }
      interpolate_temperature<<<numBlocks, threadsPerBlock>>>(d_T, d_T_fine, d_para, h_para.i_left_end, step);
      d_temp = d_c; d_c = d_c_next; d_c_next = d_temp;
      d_temp = d_phi; d_phi = d_phi_next; d_phi_next = d_temp;
      d_temp = d_psi; d_psi = d_psi_next; d_psi_next = d_temp;
      h_para.l_offset_Vp += Vp_ramp(step * tau0 * h_para.dt) * h_para.dt * tau0 / (SS * W0);
      CK(cudaGetLastError());
    }
    CK(cudaDeviceSynchronize());
    std::vector<double> h_T((size_t)h_para.NxT_all * h_para.NyT_all), h_Tf(N);
    CK(cudaMemcpy(h_c.data(), d_c, bytes, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(h_phi.data(), d_phi, bytes, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(h_psi.data(), d_psi, bytes, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(h_T.data(), d_T, bytesT, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(h_Tf.data(), d_T_fine, bytes, cudaMemcpyDeviceToHost));
    write_doubles(out_dir + "/c.bin", h_c.data(), N);
    write_doubles(out_dir + "/phi.bin", h_phi.data(), N);
    write_doubles(out_dir + "/psi.bin", h_psi.data(), N);
    write_doubles(out_dir + "/T.bin", h_T.data(), h_T.size());
    write_doubles(out_dir + "/T_fine.bin", h_Tf.data(), N);
    printf("tfc done: %ld steps, i_offset_history %d, i_left_end %d, l_offset_Vp %.17g\n", nsteps,
           h_para.i_offset_history, h_para.i_left_end, h_para.l_offset_Vp);
    return 0;
  }
#else
  if (mode == "step" || mode == "bench") {
    const bool bench = mode == "bench";
    std::string in_dir, out_dir;
    long nsteps;
    double dt, delta_initial = -1.0;
    int pull_first = 0, i_offset_arg = 0, auto_offset = 0;
    if (bench) {
      nsteps = atol(argv[2]);
      dt = atof(argv[3]);
      if (argc > 4) delta_initial = atof(argv[4]);
    } else {
      in_dir = argv[2];
      out_dir = argv[3];
      nsteps = atol(argv[4]);
      dt = atof(argv[5]);
      delta_initial = atof(argv[6]);
      pull_first = atoi(argv[7]);
      auto_offset = std::string(argv[8]) == "auto";
      i_offset_arg = auto_offset ? 0 : atoi(argv[8]);
    }
    std::vector<double> h_c(N), h_phi(N), h_psi(N);
    if (bench) {
      // reference initial condition kernel fills the fields
    } else {
      h_c = read_doubles(in_dir + "/c.bin", N);
      h_phi = read_doubles(in_dir + "/phi.bin", N);
      h_psi = read_doubles(in_dir + "/psi.bin", N);
    }
    constants h_para;
    fill_constants(&h_para, dt, delta_initial);
    real h_orientation[num_axes * num_orientation];
    set_orientation(h_orientation, alpha0, beta0, gamma0);

    real *d_c, *d_phi, *d_psi, *d_c_next, *d_phi_next, *d_psi_next, *d_orientation, *d_temp;
    constants *d_para;
    const size_t bytes = N * sizeof(real);
    CK(cudaMalloc(&d_c, bytes));
    CK(cudaMalloc(&d_phi, bytes));
    CK(cudaMalloc(&d_psi, bytes));
    CK(cudaMalloc(&d_c_next, bytes));
    CK(cudaMalloc(&d_phi_next, bytes));
    CK(cudaMalloc(&d_psi_next, bytes));
    CK(cudaMalloc(&d_orientation, sizeof(h_orientation)));
    CK(cudaMalloc(&d_para, sizeof(constants)));
    CK(cudaMemcpy(d_para, &h_para, sizeof(constants), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_orientation, h_orientation, sizeof(h_orientation), cudaMemcpyHostToDevice));
    CK(cudaMemset(d_c_next, 0, bytes));
    CK(cudaMemset(d_phi_next, 0, bytes));
    CK(cudaMemset(d_psi_next, 0, bytes));
    dim3 threadsPerBlock(BLOCK_SIZE_X, BLOCK_SIZE_Y);
    dim3 numBlocks(Nx_all / threadsPerBlock.x, Ny_all / threadsPerBlock.y);
    if (bench) {
      initial<<<numBlocks, threadsPerBlock>>>(d_c, d_phi, d_psi, d_orientation, d_para);
      CK(cudaGetLastError());
    } else {
      CK(cudaMemcpy(d_c, h_c.data(), bytes, cudaMemcpyHostToDevice));
      CK(cudaMemcpy(d_phi, h_phi.data(), bytes, cudaMemcpyHostToDevice));
      CK(cudaMemcpy(d_psi, h_psi.data(), bytes, cudaMemcpyHostToDevice));
    }
    if (pull_first) {
      int i_offset = i_offset_arg;
      if (auto_offset) i_offset = get_itip_all_grain(h_psi.data()) - i_tip_target;
      printf("pull_back i_offset %d\n", i_offset);
      pull_back<<<numBlocks, threadsPerBlock>>>(d_c, d_phi, d_psi, d_c_next, d_phi_next, d_psi_next, i_offset, 0);
      CK(cudaGetLastError());
      d_temp = d_c; d_c = d_c_next; d_c_next = d_temp;
      d_temp = d_phi; d_phi = d_phi_next; d_phi_next = d_temp;
      d_temp = d_psi; d_psi = d_psi_next; d_psi_next = d_temp;
    }
    const int i_offset_history = 0;
    double l_offset_Vp = 0.0;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    const long warm = bench ? 10 : 0;
    for (long step = -warm; step < nsteps; ++step) {
      if (step == 0) CK(cudaEventRecord(e0));
      const long s = step < 0 ? 0 : step;
      compute_phi<<<numBlocks, threadsPerBlock>>>(d_c, d_phi, d_psi, NULL, d_c_next, d_phi_next, d_psi_next,
                                                  d_orientation, NULL, d_para, s, i_offset_history, l_offset_Vp);
      compute_psi<<<numBlocks, threadsPerBlock>>>(d_c, d_phi, d_psi, d_c_next, d_phi_next, d_psi_next,
                                                  d_orientation, NULL, d_para, s);
      compute_c_CALPHAD<<<numBlocks, threadsPerBlock>>>(d_c, d_phi, d_psi, NULL, d_c_next, d_phi_next, d_psi_next,
                                                        d_orientation, NULL, d_para, s, i_offset_history, l_offset_Vp);
      d_temp = d_c; d_c = d_c_next; d_c_next = d_temp;
      d_temp = d_phi; d_phi = d_phi_next; d_phi_next = d_temp;
      d_temp = d_psi; d_psi = d_psi_next; d_psi_next = d_temp;
      // constants.hpp: if_Vp_ramp false -> constant Vp (main.cu:235-236)
      if (step >= 0) l_offset_Vp += Vp * h_para.dt * tau0 / (SS * W0);
    }
    CK(cudaEventRecord(e1));
    CK(cudaEventSynchronize(e1));
    CK(cudaGetLastError());
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    if (bench) {
      const double cells = (double)(Nx_all - 2) * (Ny_all - 2) * nsteps;
      printf("{\"grid\": [%d, %d], \"steps\": %ld, \"ms\": %.4f, \"gcell_steps_per_s\": %.4f}\n",
             Nx_all, Ny_all, nsteps, ms, cells / (ms * 1e-3) / 1e9);
    } else {
      CK(cudaMemcpy(h_c.data(), d_c, bytes, cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(h_phi.data(), d_phi, bytes, cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(h_psi.data(), d_psi, bytes, cudaMemcpyDeviceToHost));
      write_doubles(out_dir + "/c.bin", h_c.data(), N);
      write_doubles(out_dir + "/phi.bin", h_phi.data(), N);
      write_doubles(out_dir + "/psi.bin", h_psi.data(), N);
      printf("step done: %ld steps, %.3f ms\n", nsteps, ms);
    }
    return 0;
  }
#endif
  fprintf(stderr, "unknown mode %s\n", mode.c_str());
  return 1;
}

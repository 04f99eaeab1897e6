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
  fprintf(stderr, "unknown mode %s\n", mode.c_str());
  return 1;
}

// ref3_harness.cu — drives the reference's own 3D kernels (test infrastructure).
//
// Compiled by oracle/ref_build.sh together with a copy of the reference's
// multi/peritectic_multiGPU/TiAg.cu whose grid macros (Nx, Ny, devNz) are set
// to the harness size; the reference's main() is renamed.  The kernels
// computeMu, boundaryMuX/Y/Z, diffuse and boundaryX/Y/Z (TiAg.cu:461-605) run
// on one GPU in the order of the reference loop (TiAg.cu:269-340), on fields
// supplied by the caller, and their raw FP64 outputs are written.
//
//   ref3_harness step <in_dir> <out_dir> <nsteps>
//       in_dir/{phi1,phi2,c}.bin -> out_dir/{phi1,phi2,c}.bin after nsteps
//       steps, and out_dir/mu0.bin (mu of the input, ghost layers included)
//   ref3_harness bench <nsteps>
//       times the reference's per-step kernels (CUDA events) on its own
//       initial state; prints one JSON line
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include REF3_SOURCE
#undef main

#define CK(x)                                                                                            \
  do {                                                                                                   \
    cudaError_t e_ = (x);                                                                                \
    if (e_ != cudaSuccess) {                                                                             \
      fprintf(stderr, "CUDA %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, __LINE__);               \
      exit(3);                                                                                           \
    }                                                                                                    \
  } while (0)

static const size_t kCells = (size_t)Nx * Ny * devNz;

static std::vector<double> read_field(const std::string &path) {
  std::vector<double> v(kCells);
  FILE *f = fopen(path.c_str(), "rb");
  if (!f || fread(v.data(), sizeof(double), kCells, f) != kCells) {
    fprintf(stderr, "cannot read %s\n", path.c_str());
    exit(2);
  }
  fclose(f);
  return v;
}

static void write_field(const std::string &path, const double *d_src) {
  std::vector<double> v(kCells);
  CK(cudaMemcpy(v.data(), d_src, kCells * sizeof(double), cudaMemcpyDeviceToHost));
  FILE *f = fopen(path.c_str(), "wb");
  if (!f) {
    fprintf(stderr, "cannot write %s\n", path.c_str());
    exit(2);
  }
  fwrite(v.data(), sizeof(double), kCells, f);
  fclose(f);
}

struct Fields {
  double *phi1, *phi2, *c, *mu, *phi1_n, *phi2_n, *c_n;
};

// the launch shapes of the reference loop (TiAg.cu:157-164)
static const dim3 kTpb(BLOCK_SIZE_X, BLOCK_SIZE_Y, BLOCK_SIZE_Z);
static const dim3 kBlocks(Nx / BLOCK_SIZE_X, Ny / BLOCK_SIZE_Y, devNz / BLOCK_SIZE_Z);
static const dim3 kTpbX(BLOCK_SIZE_Y, BLOCK_SIZE_Z), kBlocksX(Ny / BLOCK_SIZE_Y, devNz / BLOCK_SIZE_Z);
static const dim3 kTpbY(BLOCK_SIZE_X, BLOCK_SIZE_Z), kBlocksY(Nx / BLOCK_SIZE_X, devNz / BLOCK_SIZE_Z);
static const dim3 kTpbZ(BLOCK_SIZE_X, BLOCK_SIZE_Y), kBlocksZ(Nx / BLOCK_SIZE_X, Ny / BLOCK_SIZE_Y);

static void compute_mu(Fields &F) {
  computeMu<<<kBlocks, kTpb>>>(F.phi1, F.phi2, F.c, F.mu);
  boundaryMuX<<<kBlocksX, kTpbX>>>(F.mu);
  boundaryMuY<<<kBlocksY, kTpbY>>>(F.mu);
  boundaryMuZ<<<kBlocksZ, kTpbZ>>>(F.mu);
}

static void one_step(Fields &F, int step) {
  compute_mu(F);
  diffuse<<<kBlocks, kTpb>>>(F.phi1, F.phi2, F.c, F.mu, F.phi1_n, F.phi2_n, F.c_n, 0, step);
  boundaryX<<<kBlocksX, kTpbX>>>(F.phi1_n, F.phi2_n, F.c_n);
  boundaryY<<<kBlocksY, kTpbY>>>(F.phi1_n, F.phi2_n, F.c_n);
  boundaryZ<<<kBlocksZ, kTpbZ>>>(F.phi1_n, F.phi2_n, F.c_n);
  std::swap(F.phi1, F.phi1_n);
  std::swap(F.phi2, F.phi2_n);
  std::swap(F.c, F.c_n);
}

static Fields alloc_fields() {
  Fields F;
  double **all[7] = {&F.phi1, &F.phi2, &F.c, &F.mu, &F.phi1_n, &F.phi2_n, &F.c_n};
  for (double **p : all) {
    CK(cudaMalloc((void **)p, kCells * sizeof(double)));
    CK(cudaMemset(*p, 0, kCells * sizeof(double)));
  }
  return F;
}

static void free_fields(Fields &F) {
  double *all[7] = {F.phi1, F.phi2, F.c, F.mu, F.phi1_n, F.phi2_n, F.c_n};
  for (double *p : all) cudaFree(p);
}

int main(int argc, char **argv) {
  if (argc >= 5 && std::string(argv[1]) == "step") {
    const std::string in = argv[2], out = argv[3];
    const int nsteps = atoi(argv[4]);
    Fields F = alloc_fields();
    const char *names[3] = {"phi1", "phi2", "c"};
    double *dst[3] = {F.phi1, F.phi2, F.c};
    for (int k = 0; k < 3; ++k) {
      std::vector<double> h = read_field(in + "/" + names[k] + ".bin");
      CK(cudaMemcpy(dst[k], h.data(), kCells * sizeof(double), cudaMemcpyHostToDevice));
    }
    compute_mu(F);
    CK(cudaDeviceSynchronize());
    write_field(out + "/mu0.bin", F.mu);
    for (int s = 0; s < nsteps; ++s) one_step(F, s);
    CK(cudaDeviceSynchronize());
    write_field(out + "/phi1.bin", F.phi1);
    write_field(out + "/phi2.bin", F.phi2);
    write_field(out + "/c.bin", F.c);
    free_fields(F);
    return 0;
  }
  if (argc >= 3 && std::string(argv[1]) == "bench") {
    const int nsteps = atoi(argv[2]);
    // the reference's own initial state (TiAg.cu initial, one slab of devNz planes)
    std::vector<double> h1((size_t)Nx * Ny * Nz), h2(h1.size()), hc(h1.size()), hm(h1.size());
    int other = 0;
    initial(h1.data(), h2.data(), hc.data(), hm.data(), &other);
    Fields F = alloc_fields();
    const size_t off = (size_t)Nx * Ny * (Nz - devNz);  // the top slab (holds the front and caps)
    CK(cudaMemcpy(F.phi1, h1.data() + off, kCells * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(F.phi2, h2.data() + off, kCells * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(F.c, hc.data() + off, kCells * sizeof(double), cudaMemcpyHostToDevice));
    for (int s = 0; s < 5; ++s) one_step(F, s);
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0));
    for (int s = 0; s < nsteps; ++s) one_step(F, 5 + s);
    CK(cudaEventRecord(e1));
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    const double cells = (double)(Nx - 2) * (Ny - 2) * (devNz - 2);
    printf("{\"ms_per_step\": %.6f, \"gcell_steps_s\": %.4f, \"grid\": [%d, %d, %d]}\n", ms / nsteps,
           cells * nsteps / (ms * 1e-3) / 1e9, Nx, Ny, devNz);
    free_fields(F);
    return 0;
  }
  fprintf(stderr, "usage: ref3_harness step <in_dir> <out_dir> <nsteps> | bench <nsteps>\n");
  return 1;
}

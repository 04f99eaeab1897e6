// rs_kernels.cuh — launcher declarations and block-reduction helpers.
#pragma once

#include <cuda.h>

#include "rs_common.cuh"

namespace rs {

// Per-block partial results of a grid pass: sum of interior c (FP64) and the
// largest column with psi > 0 (the coarse tip, get_itip_all_grain fun.cu:1745).
struct BlockPartial {
  double mass;
  int32_t itip;
  int32_t pad;
};

template <int NT>
__device__ __forceinline__ void block_partial(double mass, int itip, BlockPartial *out) {
  __shared__ double s_m[NT / 32];
  __shared__ int s_i[NT / 32];
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mass += __shfl_down_sync(0xffffffffu, mass, o);
  itip = __reduce_max_sync(0xffffffffu, itip);
  if ((tid & 31) == 0) {
    s_m[tid >> 5] = mass;
    s_i[tid >> 5] = itip;
  }
  __syncthreads();
  if (tid == 0) {
    double m = 0.0;
    int it = 0;
#pragma unroll
    for (int w = 0; w < NT / 32; ++w) {
      m += s_m[w];
      it = max(it, s_i[w]);
    }
    BlockPartial b;
    b.mass = m;
    b.itip = it;
    b.pad = 0;
    out[blockIdx.y * gridDim.x + blockIdx.x] = b;
  }
}

// Inputs of the TMA-staged FP32 kernel: descriptors of the current psi and c
// fields (built on the host) and the context's per-column table workspace.
struct SurrArgs;
// Final reduction of the per-tile partials fused into the tile kernel: the
// last CTA to finish (a counter in device memory, reset by that CTA) sums
// them in the order of reduce_partials_kernel.  counter == nullptr: none.
struct FinalRed {
  unsigned int *counter;
  const BlockPartial *partials;
  int nparts;
  double mass_offset;
  double *mass_out;
  int32_t *itip_out;
};
// The fused final reduction, run by the 128 threads of the CTA that finished
// last: the partials are summed in reduce_partials_kernel's order (slot v =
// 0..255 adds partials v, v + 256, ... in turn, then a tree over the slots).
// Each thread takes slots tid and tid + 128 and issues eight 16-byte loads
// per slot before adding any of them, so the pass costs a few L2 round trips
// rather than one per partial.  sm_m / sm_i: 256 doubles / ints of shared
// scratch; sync(): the barrier of the 128 threads.
template <typename Sync>
__device__ __forceinline__ void final_reduce(const FinalRed &FR, double *sm_m, int *sm_i, int tid, Sync sync) {
  constexpr int kB = 8;
  static_assert(sizeof(BlockPartial) == 16, "a partial is one 16-byte load");
  const int n = FR.nparts;
  const double2 *P = reinterpret_cast<const double2 *>(FR.partials);
  auto itip_of = [](double2 x) { return (int)(uint32_t)(unsigned long long)__double_as_longlong(x.y); };
  double m[2] = {0.0, 0.0};
  int it[2] = {0, 0};
  int j = 0;
  for (; (j + kB) * 256 <= n; j += kB) {
    double2 x[2][kB];
#pragma unroll
    for (int s = 0; s < 2; ++s)
#pragma unroll
      for (int u = 0; u < kB; ++u) x[s][u] = __ldcg(P + tid + 128 * s + (j + u) * 256);
#pragma unroll
    for (int s = 0; s < 2; ++s)
#pragma unroll
      for (int u = 0; u < kB; ++u) {
        m[s] += x[s][u].x;
        it[s] = max(it[s], itip_of(x[s][u]));
      }
  }
  for (; j * 256 < n; ++j)
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const int k = tid + 128 * s + j * 256;
      if (k < n) {
        const double2 x = __ldcg(P + k);
        m[s] += x.x;
        it[s] = max(it[s], itip_of(x));
      }
    }
#pragma unroll
  for (int s = 0; s < 2; ++s) {
    sm_m[tid + 128 * s] = m[s];
    sm_i[tid + 128 * s] = it[s];
  }
  sync();
  for (int sz = 128; sz > 0; sz >>= 1) {
    if (tid < sz) {
      sm_m[tid] += sm_m[tid + sz];
      sm_i[tid] = max(sm_i[tid], sm_i[tid + sz]);
    }
    sync();
  }
  if (tid == 0) {
    if (FR.mass_out) *FR.mass_out = sm_m[0] + FR.mass_offset;
    if (FR.itip_out) *FR.itip_out = max(1, sm_i[0]);  // get_itip_all_grain starts at 1
    if (FR.counter) *FR.counter = 0u;
  }
}

struct TmaMaps {
  CUtensorMap psi;
  CUtensorMap c;
  float *col_tab;   // kColTabFields arrays of col_tab_len floats (FP32 step)
  int col_tab_len;
  double *col_tab64;  // kColTabFields arrays of col_tab64_len doubles (FP64 step)
  int col_tab64_len;
  const SurrArgs *surr;  // learned CALPHAD surrogate, or nullptr (exact)
  FinalRed red;          // counter, offset and outputs (partials, nparts set by the launcher)
  int pipeline;          // the persistent warp-role kernel instead of one tile per CTA
};
constexpr int kTileOutW = 128;                  // output columns of an FP32 tile
constexpr int kTmaBoxW32 = kTileOutW + 8;        // input columns (4 each side keep x 16-byte aligned)
constexpr int kTileOutW64 = 64;                  // output columns of an FP64 tile
constexpr int kTmaBoxW64 = kTileOutW64 + 8;      // its input columns
constexpr int kTileRows = 16;    // output rows of a tile
constexpr int kTmaBoxH = kTileRows + 2;  // input rows of a tile
constexpr int kTfcTileRows32 = 8;        // output rows of an FP32 coarse-grid-temperature tile
constexpr int kColTabFields = 5;
// length of the per-column table (entry k is column k - 4) for nx_all columns
inline int col_tab_len(int nx_all) { return ((nx_all + kTileOutW - 1) / kTileOutW) * kTileOutW + kTmaBoxW32; }
inline int col_tab64_len(int nx_all) {
  return ((nx_all + kTileOutW64 - 1) / kTileOutW64) * kTileOutW64 + kTmaBoxW64;
}

// ---- launchers (return 0, or -1 when a size limit is exceeded)
int launch_step_f64(const StepCoef &K, const StepScalars &P, const double *psi, const double *c,
                    double *psi_n, double *c_n, double *phi_n, BlockPartial *partials,
                    int max_partials, int *nblocks_out, const TmaMaps *tm, int *err, cudaStream_t st);
int launch_step_f32(const StepCoef &K, const StepScalars &P, const float *psi, const float *c,
                    float *psi_n, float *c_n, float *phi_n, BlockPartial *partials, int max_partials,
                    int *nblocks_out, const TmaMaps *tm, int *err, cudaStream_t st);
template <typename R>
struct Coef;
// FP32 TMA-staged kernel (rs_step_f32.cu): frozen temperature, no pull-back.
// Launches the per-column table kernel and the tile kernel; nparts_out gets
// the number of partials written.
int launch_step_f32_tma(const StepCoef &K, const Coef<float> &F, const StepScalars &P, const TmaMaps &tm,
                        float *psi_n, float *c_n, float *phi_n, BlockPartial *partials, int max_partials,
                        int *nparts_out, int *err, cudaStream_t st);
// FP64 TMA-staged kernel (rs_step_f64t.cu): frozen temperature, no pull-back,
// even nx_all; column table + tile kernel, final reduction fused.
int launch_step_f64_tma(const StepCoef &K, const Coef<double> &F, const StepScalars &P, const TmaMaps &tm,
                        double *psi_n, double *c_n, double *phi_n, BlockPartial *partials, int max_partials,
                        int *nparts_out, int *err, cudaStream_t st);
// The final reduction of FR (counter unused) as a programmatic dependent of
// the kernel just launched on st, which wrote the partials: it is scheduled
// while that kernel runs and waits for its completion on the device
// (griddepcontrol.wait), so no host-side launch gap follows the step.  The
// step kernel must execute griddepcontrol.launch_dependents.  Same order of
// summation as launch_reduce_partials.
int launch_reduce_partials_dep(const FinalRed &FR, cudaStream_t st);
void launch_reduce_partials(const BlockPartial *partials, int n, double mass_offset,
                            double *mass_out, int32_t *itip_out, cudaStream_t st);

// frame / reductions / tip (rs_frame.cu); precision 0 = double, 1 = float
void launch_pull_back(int precision, const StepCoef &K, const void *c, const void *psi,
                      const void *phi, void *c_n, void *psi_n, void *phi_n, int i_offset,
                      cudaStream_t st);
int launch_grid_partials(int precision, const StepCoef &K, const void *c, const void *psi,
                         double c_offset, BlockPartial *partials, int max_partials,
                         int *nblocks_out, cudaStream_t st);
void launch_precise_tip(int precision, const StepCoef &K, const void *psi, int *row_last,
                        double *row_f, double *row_g, rs_tip *out, cudaStream_t st);

// initial conditions and coarse temperature (rs_init.cu)
void launch_initial_reference(int precision, const StepCoef &K, int i_tip_target, void *c,
                              void *psi, void *phi, cudaStream_t st);
void launch_initial_planar(int precision, const StepCoef &K, int i_tip_target, double c_liquid,
                           double c_solid, uint64_t seed, void *c, void *psi, void *phi,
                           cudaStream_t st);

struct TfcCoef {
  int32_t nx, ny, pitch, ratio;
  int32_t NxT, NyT, NxT_all, NyT_all;
  int32_t jTmin, jTmax;
  int32_t ratio_dt_dtT, Sint;
  double Tcold, Thot, dx, dxT, dtT, Lcp, W0, GG, S, DT, Gmuk;
};
void launch_temperature_init(const TfcCoef &T, double *d_T, cudaStream_t st);
// adv = Vp_ramp(step tau0 dt) tau0 / (S W0), per step (fun.cu:1563)
void launch_temperature_substep(const TfcCoef &T, const double *Tin, double *Tout,
                                const double *dphidt, double adv, cudaStream_t st);
void launch_interpolate_temperature(const TfcCoef &T, const StepCoef &K, const double *d_T,
                                    double *d_T_fine, int i_left_end, cudaStream_t st);
void launch_integrate_phi(int precision, const TfcCoef &T, const void *psi, const void *psi_n,
                          double *dphidt, int i_left_end, int i_offset, cudaStream_t st);

// records a message for rs_last_error() and returns code (rs_capi.cu)
int set_error(int code, const char *msg);

}  // namespace rs

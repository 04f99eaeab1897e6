// rs_mlp.cuh — layout and device evaluation of the CALPHAD surrogate network
// (3 -> 32 -> 32 -> 2, SiLU), shared by the training kernels (rs_mlp.cu) and
// the surrogate form of the FP32 tile kernel (rs_step_f32.cu).
#pragma once

#include "rs_kernels.cuh"

namespace rs {

constexpr int kMlpH = 32;
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kMlpH * 3;
constexpr int kOffW2 = kOffB1 + kMlpH;
constexpr int kOffB2 = kOffW2 + kMlpH * kMlpH;
constexpr int kOffW3 = kOffB2 + kMlpH;
constexpr int kOffB3 = kOffW3 + 2 * kMlpH;
constexpr int kMlpNParams = kOffB3 + 2;
static_assert(kMlpNParams == RS_MLP_NPARAMS, "parameter count of the C-ABI");

// training box and output scaling (mirrors rs_mlp_box)
struct MlpBox {
  double T_lo, T_hi, c_lo, c_hi;
  double y_mean[2], y_scale[2];
};

struct MlpView {
  const float *p;
  __host__ __device__ explicit MlpView(const float *q) : p(q) {}
  __host__ __device__ float w1(int h, int q) const { return p[kOffW1 + h * 3 + q]; }
  __host__ __device__ float b1(int h) const { return p[kOffB1 + h]; }
  __host__ __device__ float w2(int i, int j) const { return p[kOffW2 + i * kMlpH + j]; }
  __host__ __device__ float b2(int i) const { return p[kOffB2 + i]; }
  __host__ __device__ float w3(int q, int i) const { return p[kOffW3 + q * kMlpH + i]; }
  __host__ __device__ float b3(int q) const { return p[kOffB3 + q]; }
};

__device__ __forceinline__ float sigm(float z) { return 1.f / (1.f + expf(-z)); }
__device__ __forceinline__ float silu(float z) { return z * sigm(z); }
__device__ __forceinline__ float silu_grad(float z) {
  const float s = sigm(z);
  return s * (1.f + z * (1.f - s));
}

__device__ __forceinline__ void mlp_forward_full(const MlpView &W, const float x[3], float z1[kMlpH],
                                                 float a1[kMlpH], float z2[kMlpH], float a2[kMlpH], float o[2]) {
#pragma unroll
  for (int h = 0; h < kMlpH; ++h) {
    z1[h] = W.b1(h) + W.w1(h, 0) * x[0] + W.w1(h, 1) * x[1] + W.w1(h, 2) * x[2];
    a1[h] = silu(z1[h]);
  }
#pragma unroll
  for (int i = 0; i < kMlpH; ++i) {
    float s = W.b2(i);
#pragma unroll
    for (int j = 0; j < kMlpH; ++j) s += W.w2(i, j) * a1[j];
    z2[i] = s;
    a2[i] = silu(s);
  }
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    float s = W.b3(q);
#pragma unroll
    for (int i = 0; i < kMlpH; ++i) s += W.w3(q, i) * a2[i];
    o[q] = s;
  }
}

__device__ __forceinline__ void mlp_forward(const MlpView &W, const float x[3], float o[2]) {
  float z1[kMlpH], a1[kMlpH], z2[kMlpH], a2[kMlpH];
  mlp_forward_full(W, x, z1, a1, z2, a2, o);
}

int launch_mlp_sample(double cinf, double RR, const MlpBox &box, int64_t n, uint64_t seed, float *x, float *y,
                      cudaStream_t st, bool g_input = false);
int launch_mlp_grad(const MlpBox &box, const float *w, int64_t n, const float *x, const float *y, float *grad,
                    double *loss, cudaStream_t st);
int launch_mlp_adam(float *w, const float *grad, float *m, float *v, int64_t t, float lr, float scale,
                    cudaStream_t st);
int launch_mlp_forward(const MlpBox &box, const float *w, int64_t n, const float *x, float *out, cudaStream_t st);

}  // namespace rs

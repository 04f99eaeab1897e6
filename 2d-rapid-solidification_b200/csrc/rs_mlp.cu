// rs_mlp.cu — the learned stand-in for the per-cell CALPHAD evaluation:
// training data from the exact evaluator, forward/backward and Adam kernels.
//
// Network: (T, c, phi) -> (mu'', dG), 3 -> 32 -> 32 -> 2, SiLU, inputs scaled
// to [-1, 1] over the training box, outputs scaled by the box's
// mean/scale.  mu'' is the chemical potential relative to the melt's column
// value used by the FP32 tile kernel (rs_step_f32.cu),
//   mu'' = -(g+1) C0(T) - delta (L0_BCC + L0_Liq + g (L0_BCC - L0_Liq)) + RT lam(c),
// and dG = Gl - Gs = (1-c) A_Nb + c A_Ti + c (1-c) (L0_Liq - L0_BCC)
// (fun.cu:1671-1720 regrouped, rs_common.cuh).  Targets are evaluated in FP64
// with the same device functions as the exact kernels.
//
// Parameters are one flat FP32 vector (RS_MLP_NPARAMS):
//   W1[32][3], b1[32], W2[32][32], b2[32], W3[2][32], b3[2]   (row = output unit)
#include <cooperative_groups.h>

#include "rs_mlp.cuh"

namespace cg = cooperative_groups;

namespace rs {
namespace {

constexpr int kGradThreads = 128;
constexpr int kGradCtas = 8;  // CTAs of the one gradient cluster (portable size)

// g: the interpolation weight, gg(phi) for the 2D model, 2 gS - 1 for the 3D one
__device__ __forceinline__ double mu2_exact(double T, double c, double g, double cinf, double RR) {
  const TTerms tt = t_terms(T, RR);
  const double D = 0.5 * (tt.dGs - tt.dGl);
  const double C0 = -D - 0.5 * (kL0Bcc - kL0Liq) * (1.0 - 2.0 * cinf);
  const double lam = log(c / (1.0 - c)) - log(cinf / (1.0 - cinf));
  return -(g + 1.0) * C0 - (c - cinf) * ((kL0Bcc + kL0Liq) + g * (kL0Bcc - kL0Liq)) + tt.RT * lam;
}

__device__ __forceinline__ double dG_exact(double T, double c, double RR) {
  const TTerms tt = t_terms(T, RR);
  return (1.0 - c) * tt.A_nb + c * tt.A_ti + c * (1.0 - c) * (kL0Liq - kL0Bcc);
}

// G_INPUT: the third input is g itself (3D model) instead of phi (2D model)
template <bool G_INPUT>
__global__ void sample_kernel(const double cinf, const double RR, const MlpBox box, const int64_t n,
                              const uint32_t seed_lo, const uint32_t seed_hi, float *__restrict__ x,
                              float *__restrict__ y) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  uint32_t r[4] = {(uint32_t)k, (uint32_t)((uint64_t)k >> 32), 0x4D4C5053u, 0u};
  philox4x32(r, seed_lo, seed_hi);
  const double u0 = u53(r[0], r[1]), u1 = u53(r[2], r[3]);
  uint32_t r2[4] = {(uint32_t)k, (uint32_t)((uint64_t)k >> 32), 0x4D4C5054u, 0u};
  philox4x32(r2, seed_lo, seed_hi);
  const double u2 = u53(r2[0], r2[1]);
  const double T = box.T_lo + (box.T_hi - box.T_lo) * u0;
  const double c = box.c_lo + (box.c_hi - box.c_lo) * u1;
  const double phi = -1.0 + 2.0 * u2;
  x[3 * k + 0] = (float)(2.0 * u0 - 1.0);
  x[3 * k + 1] = (float)(2.0 * u1 - 1.0);
  x[3 * k + 2] = (float)phi;
  const double g = G_INPUT ? phi : phi * (1.875 + phi * phi * (-1.25 + 0.375 * phi * phi));
  y[2 * k + 0] = (float)mu2_exact(T, c, g, cinf, RR);
  y[2 * k + 1] = (float)dG_exact(T, c, RR);
}

// The gradient of one call is computed by ONE cluster of kGradCtas CTAs, so
// that its sums have a fixed order and two trainings with the same seed give
// the same weights: CTA r takes the sample chunks r, r + kGradCtas, ... of
// kGradThreads samples; per chunk, one thread per sample runs forward, loss
// and backward into shared memory, and each thread then adds the chunk's
// contribution to the weight gradients it owns (parameters t, t + 128, ...)
// in sample order.  At the end CTA 0 adds the CTAs' partial gradients and
// losses, read from their shared memory (distributed shared memory), in rank
// order, to grad and loss.
constexpr int kParamsPerThread = (kMlpNParams + kGradThreads - 1) / kGradThreads;

__global__ void __cluster_dims__(kGradCtas, 1, 1) __launch_bounds__(kGradThreads)
    grad_kernel(const MlpBox box, const float *__restrict__ w, const int64_t n, const float *__restrict__ x,
                const float *__restrict__ y, float *__restrict__ grad, double *__restrict__ loss) {
  extern __shared__ float sh[];
  float *sx = sh;                                   // [kGradThreads][3]
  float *h1 = sx + kGradThreads * 3;                // [kGradThreads][H]
  float *h2 = h1 + kGradThreads * kMlpH;            // [kGradThreads][H]
  float *d1 = h2 + kGradThreads * kMlpH;            // [kGradThreads][H]
  float *d2 = d1 + kGradThreads * kMlpH;            // [kGradThreads][H]
  float *d3 = d2 + kGradThreads * kMlpH;            // [kGradThreads][2]
  float *part = d3 + kGradThreads * 2;              // [kMlpNParams] this CTA's gradient
  __shared__ double sloss[kGradThreads / 32];
  __shared__ double cta_loss;
  cg::cluster_group cluster = cg::this_cluster();
  const unsigned rank = cluster.block_rank();
  const MlpView W(w);
  const int t = threadIdx.x;
  float acc[kParamsPerThread];
#pragma unroll
  for (int i = 0; i < kParamsPerThread; ++i) acc[i] = 0.f;
  double lsum = 0.0;  // thread 0: this CTA's loss
  for (int64_t base = (int64_t)rank * kGradThreads; base < n; base += (int64_t)kGradCtas * kGradThreads) {
    const int64_t k = base + t;
    const bool live = k < n;
    float xi[3] = {0.f, 0.f, 0.f};
    if (live)
      for (int q = 0; q < 3; ++q) xi[q] = x[3 * k + q];
    float z1[kMlpH], a1[kMlpH], z2[kMlpH], a2[kMlpH], o[2];
    mlp_forward_full(W, xi, z1, a1, z2, a2, o);
    float e[2] = {0.f, 0.f};
    double l = 0.0;
    if (live) {
      for (int q = 0; q < 2; ++q) {
        e[q] = o[q] - (float)((y[2 * k + q] - box.y_mean[q]) / box.y_scale[q]);
        l += (double)e[q] * e[q];
      }
    }
    // backward: dL/do = 2 e (dead samples carry 0 deltas)
    float g3[2] = {2.f * e[0], 2.f * e[1]};
    float g2[kMlpH], g1[kMlpH];
#pragma unroll
    for (int i = 0; i < kMlpH; ++i) {
      const float s = g3[0] * W.w3(0, i) + g3[1] * W.w3(1, i);
      g2[i] = s * silu_grad(z2[i]);
    }
#pragma unroll
    for (int j = 0; j < kMlpH; ++j) {
      float s = 0.f;
#pragma unroll
      for (int i = 0; i < kMlpH; ++i) s += g2[i] * W.w2(i, j);
      g1[j] = s * silu_grad(z1[j]);
    }
    for (int q = 0; q < 3; ++q) sx[t * 3 + q] = xi[q];
    for (int i = 0; i < kMlpH; ++i) {
      h1[t * kMlpH + i] = a1[i];
      h2[t * kMlpH + i] = a2[i];
      d1[t * kMlpH + i] = g1[i];
      d2[t * kMlpH + i] = g2[i];
    }
    d3[t * 2 + 0] = g3[0];
    d3[t * 2 + 1] = g3[1];
    for (int off = 16; off > 0; off >>= 1) l += __shfl_down_sync(0xffffffffu, l, off);
    if ((t & 31) == 0) sloss[t >> 5] = l;
    __syncthreads();
    if (t == 0)
      for (int q = 0; q < kGradThreads / 32; ++q) lsum += sloss[q];
    // this chunk's weight gradients, summed over its samples in order
#pragma unroll
    for (int i = 0; i < kParamsPerThread; ++i) {
      const int p = t + i * kGradThreads;
      if (p >= kMlpNParams) break;
      float s = 0.f;
      if (p < kOffB1) {  // W1[h][q]
        const int h = p / 3, q = p % 3;
        for (int m = 0; m < kGradThreads; ++m) s += d1[m * kMlpH + h] * sx[m * 3 + q];
      } else if (p < kOffW2) {
        const int h = p - kOffB1;
        for (int m = 0; m < kGradThreads; ++m) s += d1[m * kMlpH + h];
      } else if (p < kOffB2) {  // W2[i][j]
        const int i2 = (p - kOffW2) / kMlpH, j = (p - kOffW2) % kMlpH;
        for (int m = 0; m < kGradThreads; ++m) s += d2[m * kMlpH + i2] * h1[m * kMlpH + j];
      } else if (p < kOffW3) {
        const int i2 = p - kOffB2;
        for (int m = 0; m < kGradThreads; ++m) s += d2[m * kMlpH + i2];
      } else if (p < kOffB3) {  // W3[q][i]
        const int q = (p - kOffW3) / kMlpH, i2 = (p - kOffW3) % kMlpH;
        for (int m = 0; m < kGradThreads; ++m) s += d3[m * 2 + q] * h2[m * kMlpH + i2];
      } else {
        const int q = p - kOffB3;
        for (int m = 0; m < kGradThreads; ++m) s += d3[m * 2 + q];
      }
      acc[i] += s;
    }
    __syncthreads();  // the chunk's arrays are read before the next chunk writes them
  }
#pragma unroll
  for (int i = 0; i < kParamsPerThread; ++i) {
    const int p = t + i * kGradThreads;
    if (p < kMlpNParams) part[p] = acc[i];
  }
  if (t == 0) cta_loss = lsum;
  cluster.sync();  // every CTA's partial is in its shared memory
  if (rank == 0) {
    for (int p = t; p < kMlpNParams; p += kGradThreads) {
      float s = 0.f;
      for (unsigned r = 0; r < kGradCtas; ++r) s += cluster.map_shared_rank(part, r)[p];
      grad[p] += s;
    }
    if (t == 0) {
      double l = 0.0;
      for (unsigned r = 0; r < kGradCtas; ++r) l += *cluster.map_shared_rank(&cta_loss, r);
      *loss += l;
    }
  }
  cluster.sync();  // CTA 0 has read the others' shared memory before they exit
}

// Adam (Kingma & Ba 2015) on the gradient scaled by `scale` (1 / batch size)
__global__ void adam_kernel(float *__restrict__ w, const float *__restrict__ grad, float *__restrict__ m,
                            float *__restrict__ v, const int64_t t, const float lr, const float scale) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kMlpNParams) return;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float g = grad[p] * scale;
  const float mm = b1 * m[p] + (1.f - b1) * g;
  const float vv = b2 * v[p] + (1.f - b2) * g * g;
  m[p] = mm;
  v[p] = vv;
  const float mh = mm / (1.f - powf(b1, (float)t)), vh = vv / (1.f - powf(b2, (float)t));
  w[p] -= lr * mh / (sqrtf(vh) + eps);
}

__global__ void forward_kernel(const MlpBox box, const float *__restrict__ w, const int64_t n,
                               const float *__restrict__ x, float *__restrict__ out) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const MlpView W(w);
  const float xi[3] = {x[3 * k], x[3 * k + 1], x[3 * k + 2]};
  float o[2];
  mlp_forward(W, xi, o);
  out[2 * k] = (float)(o[0] * box.y_scale[0] + box.y_mean[0]);
  out[2 * k + 1] = (float)(o[1] * box.y_scale[1] + box.y_mean[1]);
}

}  // namespace

int launch_mlp_sample(double cinf, double RR, const MlpBox &box, int64_t n, uint64_t seed, float *x, float *y,
                      cudaStream_t st, bool g_input) {
  if (n <= 0) return 0;
  auto kfn = g_input ? sample_kernel<true> : sample_kernel<false>;
  kfn<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(cinf, RR, box, n, (uint32_t)seed, (uint32_t)(seed >> 32), x, y);
  return 0;
}

int launch_mlp_grad(const MlpBox &box, const float *w, int64_t n, const float *x, const float *y, float *grad,
                    double *loss, cudaStream_t st) {
  if (n <= 0) return 0;
  const size_t smem = sizeof(float) * (kGradThreads * (3 + 4 * kMlpH + 2) + kMlpNParams);
  static std::atomic<unsigned long long> attr{0};
  if (!smem_limit_once((const void *)grad_kernel, (int)smem, attr)) return -3;
  grad_kernel<<<kGradCtas, kGradThreads, smem, st>>>(box, w, n, x, y, grad, loss);  // one cluster
  return 0;
}

int launch_mlp_adam(float *w, const float *grad, float *m, float *v, int64_t t, float lr, float scale,
                    cudaStream_t st) {
  adam_kernel<<<(kMlpNParams + 255) / 256, 256, 0, st>>>(w, grad, m, v, t, lr, scale);
  return 0;
}

int launch_mlp_forward(const MlpBox &box, const float *w, int64_t n, const float *x, float *out, cudaStream_t st) {
  if (n <= 0) return 0;
  forward_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(box, w, n, x, out);
  return 0;
}

}  // namespace rs

// rs_surrogate.cuh — warp-level tensor-core evaluation of the CALPHAD
// surrogate (rs_mlp.cuh) inside the FP32 tile kernel.
//
// One call evaluates 16 cells (one m16 tile) for the whole warp:
//   layer 1 (3 -> 32) in FP32 on the CUDA cores, each lane producing exactly
//     the fp16 elements of the A fragment it holds (cells g and g+8, features
//     2t, 2t+1, 2t+8, 2t+9 of each 16-feature half; g = lane/4, t = lane%4);
//   layer 2 (32 -> 32) as 4 n8 tiles x 2 k16 steps of
//     mma.sync.m16n8k16.row.col.f32.f16.f16.f32 (FP16 weights and
//     activations, FP32 accumulation; activations are O(1) and weights O(1),
//     far inside the FP16 range, and FP16 resolves 2^-11 against BF16's 2^-8);
//   layer 3 (32 -> 2, padded to n8): the layer-2 accumulators, after SiLU,
//     are exactly the A fragments of the next k16 steps (two adjacent n8
//     tiles form one k16 tile), 2 more mma;
// lanes with t = 0 receive the two outputs of cells g and g+8.
// SiLU is x sigma(x) with sigma(x) = (1 + tanh(x/2)) / 2 (tanh.approx.f32).
#pragma once

#include <cuda_fp16.h>

#include "rs_mlp.cuh"

namespace rs {

constexpr int kSurrB16 = kMlpH * kMlpH + 8 * kMlpH;  // 16-bit W2, then W3 padded to 8 rows

struct SurrArgs {
  const float *w;                 // FP32 parameters (rs_mlp.cuh layout)
  const uint16_t *b16;            // FP16 W2[32][32], W3[8][32] (rows 2..7 zero)
  unsigned long long *audit;      // [0] max |mu'' error| (float bits), [1] max |dG error|, [2] fallbacks, [3] audits
  float T_mid, T_ihalf, c_mid, c_ihalf;  // input scaling: (v - mid) * ihalf
  float T_lo, T_hi, c_lo, c_hi;          // training box
  float y_mean[2], y_scale[2];           // output scaling
};

// per-lane constants of the surrogate (fragments of W2^T, W3^T; the layer-1
// weights of the lane's 8 features; layer-2 bias of its accumulator columns)
struct SurrConst {
  uint32_t w2[4][2][2];  // [n-tile][k-tile][reg]
  uint32_t w3[2][2];     // [k-tile][reg]
  float w1[8][3], b1[8];
  float b2[4][2];
  float b3[2];
};

__device__ __forceinline__ int surr_feature(int lane, int k) {  // k = 0..7: the lane's layer-1 features
  const int t = lane & 3, kt = k >> 2, e = k & 3;
  return 16 * kt + 2 * t + (e & 1) + ((e >> 1) << 3);
}

__device__ __forceinline__ SurrConst surr_load(const SurrArgs &A, int lane) {
  SurrConst C;
  const int g = lane >> 2, t = lane & 3;
  const MlpView W(A.w);
#pragma unroll
  for (int nt = 0; nt < 4; ++nt)
#pragma unroll
    for (int kt = 0; kt < 2; ++kt) {
      const int n = 8 * nt + g, k = 16 * kt + 2 * t;
      C.w2[nt][kt][0] = *reinterpret_cast<const uint32_t *>(A.b16 + n * kMlpH + k);
      C.w2[nt][kt][1] = *reinterpret_cast<const uint32_t *>(A.b16 + n * kMlpH + k + 8);
    }
#pragma unroll
  for (int kt = 0; kt < 2; ++kt) {
    const int k = 16 * kt + 2 * t;
    C.w3[kt][0] = *reinterpret_cast<const uint32_t *>(A.b16 + kMlpH * kMlpH + g * kMlpH + k);
    C.w3[kt][1] = *reinterpret_cast<const uint32_t *>(A.b16 + kMlpH * kMlpH + g * kMlpH + k + 8);
  }
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int h = surr_feature(lane, k);
    C.w1[k][0] = W.w1(h, 0);
    C.w1[k][1] = W.w1(h, 1);
    C.w1[k][2] = W.w1(h, 2);
    C.b1[k] = W.b1(h);
  }
#pragma unroll
  for (int nt = 0; nt < 4; ++nt) {
    C.b2[nt][0] = W.b2(8 * nt + 2 * t);
    C.b2[nt][1] = W.b2(8 * nt + 2 * t + 1);
  }
  C.b3[0] = t == 0 ? W.b3(0) : 0.f;
  C.b3[1] = t == 0 ? W.b3(1) : 0.f;
  return C;
}

__device__ __forceinline__ float silu_fast(float x) {
  float th;
  asm("tanh.approx.f32 %0, %1;" : "=f"(th) : "f"(0.5f * x));
  return x * fmaf(0.5f, th, 0.5f);
}

__device__ __forceinline__ uint32_t pack_h2(float lo, float hi) {
  const __half2 v = __floats2half2_rn(lo, hi);
  return *reinterpret_cast<const uint32_t *>(&v);
}

__device__ __forceinline__ void mma_f16(float d[4], const uint32_t a[4], const uint32_t b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// in0, in1: scaled inputs (T, c, phi) of cells g and g+8 of the tile.
// Lanes with t = 0 get out0 / out1 (scaled network outputs of those cells).
__device__ __forceinline__ void surr_tile16(const SurrConst &C, const float in0[3], const float in1[3], float out0[2],
                                            float out1[2]) {
  // layer 1 straight into A fragments
  uint32_t a[2][4];
#pragma unroll
  for (int kt = 0; kt < 2; ++kt) {
    float v0[4], v1[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int k = 4 * kt + e;
      v0[e] = silu_fast(fmaf(C.w1[k][2], in0[2], fmaf(C.w1[k][1], in0[1], fmaf(C.w1[k][0], in0[0], C.b1[k]))));
      v1[e] = silu_fast(fmaf(C.w1[k][2], in1[2], fmaf(C.w1[k][1], in1[1], fmaf(C.w1[k][0], in1[0], C.b1[k]))));
    }
    a[kt][0] = pack_h2(v0[0], v0[1]);  // row g,   cols 2t, 2t+1
    a[kt][1] = pack_h2(v1[0], v1[1]);  // row g+8, cols 2t, 2t+1
    a[kt][2] = pack_h2(v0[2], v0[3]);  // row g,   cols 2t+8, 2t+9
    a[kt][3] = pack_h2(v1[2], v1[3]);  // row g+8, cols 2t+8, 2t+9
  }
  // layer 2
  float d[4][4];
#pragma unroll
  for (int nt = 0; nt < 4; ++nt) {
    d[nt][0] = d[nt][2] = C.b2[nt][0];
    d[nt][1] = d[nt][3] = C.b2[nt][1];
    mma_f16(d[nt], a[0], C.w2[nt][0]);
    mma_f16(d[nt], a[1], C.w2[nt][1]);
  }
  // layer 3: accumulators of n-tiles 2kt, 2kt+1 are the A fragment of k-tile kt
  float o[4] = {C.b3[0], C.b3[1], C.b3[0], C.b3[1]};
#pragma unroll
  for (int kt = 0; kt < 2; ++kt) {
    uint32_t a3[4];
    a3[0] = pack_h2(silu_fast(d[2 * kt][0]), silu_fast(d[2 * kt][1]));
    a3[1] = pack_h2(silu_fast(d[2 * kt][2]), silu_fast(d[2 * kt][3]));
    a3[2] = pack_h2(silu_fast(d[2 * kt + 1][0]), silu_fast(d[2 * kt + 1][1]));
    a3[3] = pack_h2(silu_fast(d[2 * kt + 1][2]), silu_fast(d[2 * kt + 1][3]));
    mma_f16(o, a3, C.w3[kt]);
  }
  out0[0] = o[0];
  out0[1] = o[1];
  out1[0] = o[2];
  out1[1] = o[3];
}

// host side (rs_capi.cu): device copies of a trained network for a step
// kernel (allocated on first use) and its kernel arguments; reading and
// clearing an audit record (synchronizes the stream); the box check
cudaError_t surrogate_setup(const float *d_w, const rs_mlp_box *box, float **w, uint16_t **b16,
                            unsigned long long **audit, SurrArgs *s);
cudaError_t surrogate_audit_read(unsigned long long *audit, cudaStream_t st, double *max_err_mu, double *max_err_dG,
                                 int64_t *n_fallback, int64_t *n_audit);
bool surrogate_box_ok(const rs_mlp_box *b);

__device__ __forceinline__ bool surr_audit_cell(int64_t step, int64_t cell) {
  const uint64_t h = ((uint64_t)cell * 0x9E3779B97F4A7C15ull) ^ ((uint64_t)step * 0xC2B2AE3D27D4EB4Full);
  return ((h >> 40) & 1023u) == 0u;
}

}  // namespace rs

// rs_common.cuh — device/host helpers shared by the phase-field kernels.
//
// Physics follows the reference (fun.cu); every helper cites the lines it
// restates.  Kernel-side coefficients are precomputed on the host into
// StepCoef so that no kernel re-derives constants per cell.
#pragma once

#include <atomic>
#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/rs_b200.h"

namespace rs {
// Raises a kernel's dynamic shared-memory limit on the current device, once
// per device: the attribute belongs to each device's context, so a process
// that drives several GPUs must set it on every one.  `done` is the call
// site's bit set of devices already set (devices 0..63; others every call).
inline bool smem_limit_once(const void *kernel, int bytes, std::atomic<unsigned long long> &done) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return false;
  const unsigned long long bit = dev >= 0 && dev < 64 ? 1ull << dev : 0ull;
  if (bit && (done.load(std::memory_order_acquire) & bit)) return true;
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) != cudaSuccess) return false;
  done.fetch_or(bit, std::memory_order_acq_rel);
  return true;
}
}  // namespace rs

namespace rs {
// CTAs of a kernel resident at once on the current device (occupancy x SMs),
// computed once per device; -1 on a CUDA error
inline int resident_ctas(const void *kfn, int threads, size_t smem, std::atomic<int> (&cache)[64]) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return -1;
  int n = dev >= 0 && dev < 64 ? cache[dev].load(std::memory_order_relaxed) : 0;
  if (n == 0) {
    int per_sm = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, threads, smem) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      return -1;
    n = per_sm * sms;
    if (dev >= 0 && dev < 64) cache[dev].store(n, std::memory_order_relaxed);
  }
  return n;
}
}  // namespace rs

#define RS_HD __host__ __device__ __forceinline__

namespace rs {

// Redlich-Kister L0 terms (fun.cu:1668-1669, constant in T)
constexpr double kL0Bcc = 12315.25;
constexpr double kL0Liq = 5144.29;

// ---------------------------------------------------------------- CALPHAD
// SGTE-style pure-element Gibbs energies (fun.cu:1628-1666).  logT is passed
// in so that one log serves all four functions at a temperature.  With
// iT = 1/T > 0 the c/T terms are evaluated as c * iT (one division for all
// four functions, used where the result is rounded to FP32); with iT = 0 they
// divide as the reference does.
RS_HD double over_T(double c, double T, double iT) { return iT > 0.0 ? c * iT : c / T; }

RS_HD double g_ti_bcc(double T, double logT, double iT = 0.0) {
  if (T >= 1155.0 && T < 1941.0)
    return 6667.385 + 105.366379 * T - 22.3771 * T * logT + 1.21707e-3 * (T * T) -
           0.84534e-6 * ((T * T) * T) - over_T(2002750.0, T, iT);
  else if (T >= 1941.0)
    return 26483.26 - 182.426471 * T + 19.0900905 * T * logT - 22.00832e-3 * (T * T) +
           1.228863e-6 * ((T * T) * T) + over_T(1400501.0, T, iT);
  return NAN;
}
RS_HD double g_ti_liq(double T, double logT, double iT = 0.0) {
  if (T >= 1300.0 && T < 1941.0)
    return 369519.198 - 2554.0225 * T + 342.059267 * T * logT - 163.409355e-3 * (T * T) +
           12.457117e-6 * ((T * T) * T) - over_T(67034516.0, T, iT);
  else if (T >= 1941.0 && T < 4000.0)
    return -19887.066 + 298.7367 * T - 46.29 * T * logT;
  return NAN;
}
RS_HD double g_nb_bcc(double T, double logT, double iT = 0.0) {
  if (T >= 298.15 && T < 2750.0)
    return -8519.353 + 142.045475 * T - 26.4711 * T * logT + 0.203475e-3 * (T * T) -
           0.35012e-6 * ((T * T) * T) + over_T(93399.0, T, iT);
  else if (T >= 2750.0) {
    const double t3 = (T * T) * T;
    if (iT > 0.0) {
      const double i3 = (iT * iT) * iT;
      return -37669.3 + 271.720843 * T - 41.77 * T * logT + 1528.238e29 * ((i3 * i3) * i3);
    }
    return -37669.3 + 271.720843 * T - 41.77 * T * logT + 1528.238e29 / ((t3 * t3) * t3);
  }
  return NAN;
}
RS_HD double g_nb_liq(double T, double logT, double iT = 0.0) {
  if (T >= 298.15 && T < 2750.0) {
    const double t2 = T * T;
    return 21262.202 + 131.229057 * T - 26.4711 * T * logT + 0.203475e-3 * t2 -
           0.35012e-6 * (t2 * T) + over_T(93399.0, T, iT) - 306.098e-25 * (((t2 * t2) * t2) * T);
  } else if (T >= 2750.0)
    return -7499.398 + 260.756148 * T - 41.77 * T * logT;
  return NAN;
}

// Temperature-only CALPHAD groups.  With these, per cell
//   mu    = 0.5(1+g) Gsc + 0.5(1-g) Glc          (fun.cu:1443-1452)
//   Gsc   = dGs + L0_BCC (1-2c) + RT log(c/(1-c)) (fun.cu:1711-1720)
//   Glc   = dGl + L0_Liq (1-2c) + RT log(c/(1-c)) (fun.cu:1700-1709)
//   Gl-Gs = (1-c) A_Nb + c A_Ti + c(1-c)(L0_Liq - L0_BCC)
// (the ideal-mixing terms of Gl and Gs, fun.cu:1671-1698, cancel exactly).
struct TTerms {
  double dGs;   // G_Ti_BCC - G_Nb_BCC
  double dGl;   // G_Ti_Liq - G_Nb_Liq
  double A_nb;  // G_Nb_Liq - G_Nb_BCC
  double A_ti;  // G_Ti_Liq - G_Ti_BCC
  double RT;    // RR T
};

// recip: evaluate the c/T terms with one reciprocal (FP32 tables)
RS_HD TTerms t_terms(double T, double RR, bool recip = false) {
  const double lT = log(T);
  const double iT = recip ? 1.0 / T : 0.0;
  const double tb = g_ti_bcc(T, lT, iT), tl = g_ti_liq(T, lT, iT);
  const double nb = g_nb_bcc(T, lT, iT), nl = g_nb_liq(T, lT, iT);
  TTerms r;
  r.dGs = tb - nb;
  r.dGl = tl - nl;
  r.A_nb = nl - nb;
  r.A_ti = tl - tb;
  r.RT = RR * T;
  return r;
}

// interpolation functions (fun.cu:189-196)
RS_HD double gg(double p) {
  const double p2 = p * p;
  return 1.875 * p - 1.25 * (p2 * p) + 0.375 * ((p2 * p2) * p);
}
RS_HD double dgg_dp(double p) {
  const double a = 1.0 - p * p;
  return 1.875 * (a * a);
}
RS_HD double qq(double AA, double p) {
  const double a = 1.0 - p;
  return 0.5 * AA * a - 0.25 * (AA - 1) * (a * a);
}

// ---------------------------------------------------------------- Philox
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): counter-based RNG,
// so noise for (seed, step, cell) needs no stored state.
RS_HD void philox4x32(uint32_t x[4], uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    const uint64_t p0 = (uint64_t)0xD2511F53u * x[0];
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * x[2];
    const uint32_t y0 = (uint32_t)(p1 >> 32) ^ x[1] ^ k0;
    const uint32_t y2 = (uint32_t)(p0 >> 32) ^ x[3] ^ k1;
    x[0] = y0;
    x[1] = (uint32_t)p1;
    x[2] = y2;
    x[3] = (uint32_t)p0;
  }
}
RS_HD double u53(uint32_t a, uint32_t b) {
  return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6) + 0.5) * (1.0 / 9007199254740992.0);
}
// counter layout of the interface noise draw for (step, cell)
RS_HD void noise_counter(uint32_t x[4], int64_t step, int64_t cell) {
  x[0] = (uint32_t)cell;
  x[1] = (uint32_t)((uint64_t)cell >> 32);
  x[2] = (uint32_t)step;
  x[3] = (uint32_t)((uint64_t)step >> 32) ^ 0x4E4F4953u;
}

// Launch order of the column blocks of a 2D step: k-th block launched -> block
// index, for n blocks with the front in block f: f, then f-1 down to 0 (the
// solid and mushy zone behind it), then n-1 down to f+1 (melt).  The slow
// blocks at the front start first instead of being left for the last wave.
__host__ __device__ __forceinline__ int front_first_block(int k, int f, int n) {
  f = f < 0 ? 0 : (f > n - 1 ? n - 1 : f);
  const int b = f - k;  // 0 <= k < n
  return b < 0 ? b + n : b;
}

// ---------------------------------------------------------------- coefficients
// Everything the step kernel needs, derived once on the host.
struct StepCoef {
  int32_t nx, ny, pitch;
  int32_t jmin, jmax;   // rows copied into ghost rows 0 and ny-1
  int32_t one_eps;
  int32_t tfc;
  int32_t ratio;        // TFC coarse/fine ratio
  int32_t NxT_all;
  double dx;
  double inv_2dx, inv_dx2, inv_4dx2, inv_2dx2;
  double dt;
  double eps1, eps2, epk1;
  double ox1, ox2, oy1, oy2, oz1, oz2;   // orientation rows (fun.cu:1080-1085)
  double drive;       // 1 / (2 hh v0)        (fun.cu:1195)
  double inv_h0v0;    // 1 / (h0 v0)          (fun.cu:1454)
  double cfac;        // dt Dl / (Gamma muk0) / dx^2 (fun.cu:1461)
  double AA;
  double RR;
  double cinf;
  double Tmelt, deltaT0;
  double dxT;         // TFC: dx * ratio
  double noise_amp;   // amplitude * sqrt(dt); 0 = off
  uint32_t seed_lo, seed_hi;
  double W0, S;       // tip radius scale dx W0 S (fun.cu:2941)
  int32_t NyT_all;
  int32_t j_offset;   // band mode: global row of local row 0 (noise key); else 0
  // FP32 path: chemical potential relative to the melt composition
  double Lref;        // log(cinf / (1 - cinf))
};

// Per-step frozen-temperature line: T(i) = Tmelt + deltaT0 (d0 + d1 i)
// (get_delta, fun.cu:1610-1619, regrouped per step on the host).
struct StepScalars {
  int64_t step;
  double d0, d1;
  int32_t pull_back, i_offset;
  int32_t i_left_end_T;
  // column the moving frame keeps the front at (i_tip_target): the order the
  // 2D step kernels launch their column blocks in (front_first_block);
  // results do not depend on it
  int32_t i_front;
  // tries of a bounded device-side wait before it gives up (0: the kernel's
  // default); a test option makes it tiny so that the give-up path runs
  uint32_t wait_limit;
  const double *T_coarse;
  // the current fields (the tile kernels gather a pull-back step's shifted
  // tile through them instead of a TMA box)
  const void *src_psi, *src_c;
};

}  // namespace rs

// rs_peri3d_common.cuh — pieces shared by the 3D three-phase step kernels
// (rs_peri3d.cu: TiAg.cu's grand potentials; rs_peri3d_tinb.cu: the Ti-Nb
// CALPHAD energy): tiling constants, the Folch-Plapp interpolation, the
// kernel constants and the bounded plane wait.
#pragma once

#include <cuda.h>

#include "rs_peri3d.cuh"
#include "rs_step_common.cuh"

namespace rs {

constexpr int kP3Threads = 256;
constexpr int kP3BY = 16;            // output rows of a CTA
constexpr int kP3Slots = 4;          // input plane ring
constexpr int kP3MuSlots = 4;        // mu plane ring
constexpr uint32_t kP3WaitLimit = 1u << 22;

template <typename R>
struct P3Cfg {
  static constexpr int BX = 256 / (int)sizeof(R);    // output columns: 64 (FP32), 32 (FP64)
  static constexpr int BXin = BX + 16 / (int)sizeof(R);  // + halo rounded to 16 bytes
  static constexpr int BYin = kP3BY + 2;
  static constexpr int kPlane = BXin * BYin;          // elements of one field plane
  // a TMA destination starts on a 128-byte boundary: field planes padded
  static constexpr int kPlaneAl = ((kPlane * (int)sizeof(R) + 127) / 128) * 128 / (int)sizeof(R);
  static constexpr int kCellsPerThread = BX * kP3BY / kP3Threads;
};

// Folch-Plapp interpolation and derivatives (TiAg.cu:72-74 g, gp1, gp2)
template <typename R>
__device__ __forceinline__ R g3(R pi, R pj, R pk) {
  return pi * pi * R(0.25) * (R(15) * (R(1) - pi) * (R(1) + pi - (pk - pj) * (pk - pj)) + pi * (R(9) * (pi * pi) - R(5)));
}
template <typename R>
__device__ __forceinline__ R gp1(R pi, R pj, R pk) {
  return R(3.75) * pi *
         (R(-4) * (pi * pi) + R(3) * (pi * pi * pi) + R(2) - pi + (R(3) * pi - R(2)) * ((pj - pk) * (pj - pk)));
}
template <typename R>
__device__ __forceinline__ R gp2(R pi, R pj, R pk) {
  return R(7.5) * (pi - R(1)) * (pi * pi) * (pj - pk);
}

template <typename R>
struct K3 {  // kernel constants in the working precision
  int nx, ny, nz, z_chunk;
  R dt, dxi, dyi, dzi, dxi2, dyi2, dzi2;
  R a1, a2, a3, b, lam, Da2, Db2, cfx, cfy, cfz;
  R r1, r2, r3;
  double B11, B12, B21, B22, T_ref, G_T, V_T, z_T;
  // energy 1 (Ti-Nb CALPHAD): q(p) = p (AA - AA1 p) with AA1 = AA - 1; the
  // per-plane table of the step (tinb_table_kernel); the FP32 offset of c
  R AA, AA1;
  double RR, c_ref, c_off;
  const double *tab;
  // energy 1, FP32 pair kernel: far-melt form of the solute log term,
  // lam = log(c/(1-c)) - log(c_ref/(1-c_ref)) = sum_k melt_a[k-1] d^k for
  // |d| <= melt_tiny, d = c - c_ref (four terms, |d| <= 1e-2 min(c_ref,
  // 1-c_ref): the remainder is below 4e-9 of lam; see Coef::melt_a)
  R melt_a[4];
  R melt_tiny;
};

template <typename R>
K3<R> make_k3(const rs3_params &p) {
  K3<R> k;
  k.nx = p.nx;
  k.ny = p.ny;
  k.nz = p.nz;
  k.z_chunk = p.z_chunk > 0 ? p.z_chunk : 32;
  k.dt = (R)p.dt;
  k.dxi = (R)p.dx_inv;
  k.dyi = (R)p.dy_inv;
  k.dzi = (R)p.dz_inv;
  k.dxi2 = (R)(p.dx_inv * p.dx_inv);
  k.dyi2 = (R)(p.dy_inv * p.dy_inv);
  k.dzi2 = (R)(p.dz_inv * p.dz_inv);
  k.a1 = (R)p.a1;
  k.a2 = (R)p.a2;
  k.a3 = (R)p.a3;
  k.b = (R)p.b;
  k.lam = (R)p.lambda;
  // c' = c + dt alpha sum_d din^2 (H+ - H-) / 2 with H = M dmu, M = phi1 + phi1'
  // (+ Da (phi2 + phi2') + Db (phi3 + phi3')), TiAg.cu:543-552
  k.Da2 = (R)p.Da;
  k.Db2 = (R)p.Db;
  k.cfx = (R)(0.5 * p.dt * p.alpha * p.dx_inv * p.dx_inv);
  k.cfy = (R)(0.5 * p.dt * p.alpha * p.dy_inv * p.dy_inv);
  k.cfz = (R)(0.5 * p.dt * p.alpha * p.dz_inv * p.dz_inv);
  k.r1 = (R)p.A1;
  k.r2 = (R)(-p.A1 - p.A2);
  k.r3 = (R)(-p.A1 + p.A2);
  k.B11 = p.B11;
  k.B12 = p.B12;
  k.B21 = p.B21;
  k.B22 = p.B22;
  k.T_ref = p.T_ref;
  k.G_T = p.G_T;
  k.V_T = p.V_T;
  k.z_T = p.z_T;
  k.AA = (R)p.AA;
  k.AA1 = (R)(p.AA - 1.0);
  k.RR = p.RR;
  k.c_ref = p.c_ref;
  k.c_off = 0.0;
  k.tab = nullptr;
  for (int j = 0; j < 4; ++j) k.melt_a[j] = (R)0;
  k.melt_tiny = (R)-1;  // never (energy 0 has no log term)
  if (p.energy == 1 && p.c_ref > 0.0 && p.c_ref < 1.0) {
    double pc = 1.0, pm = 1.0;
    for (int j = 1; j <= 4; ++j) {
      pc /= p.c_ref;
      pm /= 1.0 - p.c_ref;
      k.melt_a[j - 1] = (R)(((j % 2 ? pc : -pc) + pm) / j);
    }
    k.melt_tiny = (R)(1e-2 * (p.c_ref < 0.5 ? p.c_ref : 1.0 - p.c_ref));
  }
  return k;
}

// A box element counts as pure melt for a plane's flag when it lies outside
// the array (no stencil of an output cell reaches it) or holds phi1 == 1 and
// phi2 == 0 exactly.  Where planes z-1 .. z+1 are pure melt in this sense,
// every phase term and Laplacian of an output cell of plane z is an exact
// zero: phi1 and phi2 stay 1 and 0, and every face mobility phi1 + phi1' is
// exactly 2 (the solid terms vanish).
template <typename R>
__device__ __forceinline__ bool p3_melt_cell(const K3<R> &k, R p1, R p2, int x, int y) {
  return x >= k.nx || y >= k.ny || (p1 == R(1) && p2 == R(0));
}

template <typename R>
__device__ __forceinline__ bool p3_wait(uint64_t *bar, uint32_t parity, int *err) {
  uint32_t tries = 0;
  while (!mbar_try_wait(bar, parity))
    if (++tries >= kP3WaitLimit) {
      atomicExch(err, 1);
      return false;
    }
  return true;
}

}  // namespace rs

// rs_step_f32.cu — fused FP32 bulk time step (16 B per cell-step).
//
// Same step as rs_step_f64.cu (fun.cu:1143-1467) with the bulk arithmetic in
// FP32 and the cancellation-prone parts kept exact:
//   * c is stored as delta = c - cinf.  Near the melt composition delta is
//     small, so an FP32 delta carries ~30x more absolute precision than an
//     FP32 c, and updates far below ulp(c) still land (solute conservation).
//   * The chemical potential mu (fun.cu:1443-1452, O(1e4) J/mol) only enters
//     the flux through neighbour differences of O(1e-1..1e2) J/mol.  It is
//     split as mu = K(T) + mu' with the composition-independent column part
//       K(T) = (dGs + dGl)/2 + (L0_BCC + L0_Liq)(1 - 2 cinf)/2 + RT L(cinf)
//     evaluated in FP64 once per tile column (its i-differences are passed
//     as FP32), and the small remainder
//       mu' = g D(T) - delta (L0_BCC + L0_Liq) + g (L0_BCC - L0_Liq)(1 - 2c)/2
//             + RT log1p(delta / (cinf (1 - c)))
//     with D = (dGs - dGl)/2, evaluated in FP32 per cell.
//   * The Gl - Gs driving force uses the per-column FP64 groups
//     A_Nb = G_Nb_Liq - G_Nb_BCC, A_Ti = G_Ti_Liq - G_Ti_BCC.
// Frozen temperature only (T depends on the column).
#include "rs_kernels.cuh"

namespace rs {

struct ColF {
  float A_nb, A_ti, D, RT;
};

__device__ __forceinline__ float ggf(float p) {
  const float p2 = p * p;
  return p * (1.875f + p2 * (-1.25f + 0.375f * p2));
}
__device__ __forceinline__ float dggf(float p) {
  const float a = 1.0f - p * p;
  return 1.875f * (a * a);
}

struct CoefF {
  float inv_2dx, inv_dx2, inv_4dx2, inv_2dx2, dt;
  float eps1, eps2, epk1, ox1, ox2, oy1, oy2, oz1, oz2;
  float drive, cflux, AA, cinf, Lref, noise_amp, floor_delta;
};

__device__ __forceinline__ float anisotropy_f32(const StepCoef &K, const CoefF &F, float phi00, float phi10,
                                                float phim0, float phi01, float phi0m, float phi11,
                                                float phim1, float phi1m, float phimm, float &as,
                                                float &ak) {
  const float px = (phi10 - phim0) * F.inv_2dx;
  const float py = (phi01 - phi0m) * F.inv_2dx;
  const float g2 = px * px + py * py;
  const float dxx = (phi10 - 2.0f * phi00 + phim0) * F.inv_dx2;
  const float dyy = (phi01 - 2.0f * phi00 + phi0m) * F.inv_dx2;
  const float dxy = ((phi11 - phim1) - (phi1m - phimm)) * F.inv_4dx2;
  const float lap = (2.0f / 3.0f) * (dxx + dyy) +
                    (1.0f / 3.0f) * ((phi11 + phim1) + (phi1m + phimm) - 4.0f * phi00) * F.inv_2dx2;
  float dtx = 0.f, dty = 0.f, cs = 0.f, sn = 0.f;
  if (g2 > 1.0e-30f) {  // |grad phi| > 1e-15 (fun.cu:1056)
    const float inv_a = rsqrtf(g2);
    const float inv_g2 = inv_a * inv_a;
    dtx = (px * dxy - py * dxx) * inv_g2;
    dty = (px * dyy - py * dxy) * inv_g2;
    cs = px * inv_a;
    sn = py * inv_a;
  }
  const float nx = F.ox1 * cs + F.ox2 * sn;
  const float ny = F.oy1 * cs + F.oy2 * sn;
  const float nz = F.oz1 * cs + F.oz2 * sn;
  const float nx1 = F.ox2 * cs - F.ox1 * sn;
  const float ny1 = F.oy2 * cs - F.oy1 * sn;
  const float nz1 = F.oz2 * cs - F.oz1 * sn;
  const float nx3 = nx * nx * nx, ny3 = ny * ny * ny, nz3 = nz * nz * nz;
  const float np4 = nx3 * nx + ny3 * ny + nz3 * nz;
  const float dnp4_1 = 4.0f * (nx3 * nx1 + ny3 * ny1 + nz3 * nz1);
  const float ax = nx * nx1, ay = ny * ny1, az = nz * nz1;
  const float dnp4_2 = 4.0f * (3.0f * (ax * ax + ay * ay + az * az) - np4);
  float da1, da2;
  if (K.one_eps) {
    ak = (1.0f - 3.0f * F.epk1) + 4.0f * F.epk1 * np4;
    as = (1.0f - 3.0f * F.eps1) + 4.0f * F.eps1 * np4;
    da1 = 4.0f * F.eps1 * dnp4_1;
    da2 = 4.0f * F.eps1 * dnp4_2;
  } else {
    const float xyz = nx * ny * nz;
    ak = 1.0f + F.epk1 * (np4 - 0.6f);
    as = 1.0f + F.eps1 * (np4 - 0.6f) + F.eps2 * (3.0f * np4 + 66.0f * (xyz * xyz) - 17.0f / 7.0f);
    const float t1 = nx1 * ny * nz + nx * ny1 * nz + nx * ny * nz1;
    const float dnp2_1 = 2.0f * xyz * t1;
    float dnp2_2 = (nx1 * ny * nz) * (nx1 * ny * nz) + (nx * ny1 * nz) * (nx * ny1 * nz) +
                   (nx * ny * nz1) * (nx * ny * nz1);
    dnp2_2 += -nx * nx * (ny * nz) * (ny * nz) - ny * ny * (nx * nz) * (nx * nz) -
              nz * nz * (nx * ny) * (nx * ny);
    dnp2_2 += 4.0f * xyz * (nx1 * ny1 * nz + nx * ny1 * nz1 + nx1 * ny * nz1);
    dnp2_2 *= 2.0f;
    da1 = (F.eps1 + 3.0f * F.eps2) * dnp4_1 + 66.0f * F.eps2 * dnp2_1;
    da2 = (F.eps1 + 3.0f * F.eps2) * dnp4_2 + 66.0f * F.eps2 * dnp2_2;
  }
  return (as * as) * lap + 2.0f * as * da1 * (dtx * px + dty * py) +
         (da2 * as + da1 * da1) * (dty * px - dtx * py);
}

template <int BX, int BY, int RY>
__global__ void __launch_bounds__(BX *BY)
    step_f32_kernel(const StepCoef K, const CoefF F, const StepScalars P, const float *__restrict__ psi,
                    const float *__restrict__ cd, float *__restrict__ psi_n, float *__restrict__ cd_n,
                    float *__restrict__ phi_n, BlockPartial *partials) {
  constexpr int TX = BX, TY = BY * RY, RW = TX + 2, RH = TY + 2, NT = BX * BY;
  __shared__ float s_phi[RH * RW];
  __shared__ float s_S[RH * RW];
  __shared__ float s_mu[RH * RW];
  __shared__ float s_d[RH * RW];
  __shared__ ColF s_col[RW];
  __shared__ float s_dK[RW];  // K(i+1) - K(i)
  __shared__ double s_K[RW];

  const int nx = K.nx, ny = K.ny, pitch = K.pitch;
  const int x0 = 1 + blockIdx.x * TX, y0 = 1 + blockIdx.y * TY;
  const int tid = threadIdx.y * BX + threadIdx.x;

  // per-column CALPHAD groups in FP64 (T depends on the column only)
  for (int rx = tid; rx < RW; rx += NT) {
    const int gi = x0 - 1 + rx;
    const double T = (P.d0 + P.d1 * gi) * K.deltaT0 + K.Tmelt;
    const TTerms t = t_terms(T, K.RR);
    ColF col;
    col.A_nb = (float)t.A_nb;
    col.A_ti = (float)t.A_ti;
    col.D = (float)(0.5 * (t.dGs - t.dGl));
    col.RT = (float)t.RT;
    s_col[rx] = col;
    s_K[rx] = 0.5 * (t.dGs + t.dGl) + 0.5 * (kL0Bcc + kL0Liq) * (1.0 - 2.0 * K.cinf) + t.RT * K.Lref;
  }
  __syncthreads();
  for (int rx = tid; rx < RW - 1; rx += NT) s_dK[rx] = (float)(s_K[rx + 1] - s_K[rx]);

  constexpr float kL0sum = (float)(kL0Bcc + kL0Liq);
  constexpr float kL0half = (float)(0.5 * (kL0Bcc - kL0Liq));
  for (int idx = tid; idx < RH * RW; idx += NT) {
    const int ry = idx / RW, rx = idx - ry * RW;
    const int gi = x0 - 1 + rx, gj = y0 - 1 + ry;
    if (gi >= nx || gj >= ny) continue;
    int si = gi;
    if (P.pull_back) si = min(max(gi + P.i_offset, 1), nx - 2);
    const int64_t src = (int64_t)gj * pitch + si;
    const float pv = psi[src];
    const float dv = (P.pull_back && si >= nx - 2) ? 0.0f : cd[src];
    const float cv = F.cinf + dv;
    const float omc = 1.0f - cv;
    s_phi[idx] = fminf(fmaxf(pv, -1.0f), 1.0f);
    s_d[idx] = dv;
    const float a = 1.0f - pv;
    s_S[idx] = (0.5f * F.AA * a - 0.25f * (F.AA - 1.0f) * (a * a)) * cv * omc;
    const bool corner = (rx == 0 || rx == RW - 1) && (ry == 0 || ry == RH - 1);
    if (!corner) {
      const ColF col = s_col[rx];
      const float g = ggf(pv);
      float lam = -F.Lref;  // L(c) = 0 outside (1e-8, 1 - 1e-8)
      if (cv > 1.e-8f && omc > 1.e-8f) lam = log1pf(dv / (F.cinf * omc));
      s_mu[idx] = g * col.D - dv * kL0sum + g * kL0half * (1.0f - 2.0f * cv) + col.RT * lam;
    }
  }
  __syncthreads();

  double mass = 0.0;
  int itip = 0;
  const int jmin = K.jmin, jmax = K.jmax;
#pragma unroll 1
  for (int k = 0; k < RY; ++k) {
    const int tx = threadIdx.x, ty = threadIdx.y + k * BY;
    const int gi = x0 + tx, gj = y0 + ty;
    if (gi > nx - 2 || gj > ny - 2) continue;
    const int r = (ty + 1) * RW + (tx + 1);
    const float phi00 = s_phi[r];
    float as, ak;
    const float aniso = anisotropy_f32(K, F, phi00, s_phi[r + 1], s_phi[r - 1], s_phi[r + RW], s_phi[r - RW],
                                       s_phi[r + RW + 1], s_phi[r + RW - 1], s_phi[r - RW + 1],
                                       s_phi[r - RW - 1], as, ak);
    const float d00 = s_d[r];
    const float c00 = F.cinf + d00;
    const ColF col = s_col[tx + 1];
    const float dG = (1.0f - c00) * col.A_nb + c00 * col.A_ti + c00 * (1.0f - c00) * (float)(kL0Liq - kL0Bcc);
    const float term = phi00 - phi00 * phi00 * phi00 + aniso + dG * dggf(phi00) * F.drive;
    float pn = phi00 + __fdividef(F.dt * ak, as * as) * term;
    if (F.noise_amp > 0.0f) {
      const float w = 1.0f - phi00 * phi00;
      if (w > 1.0e-3f) {
        uint32_t x[4];
        noise_counter(x, P.step, (int64_t)gj * nx + gi);
        philox4x32(x, K.seed_lo, K.seed_hi);
        const float u1 = ((x[0] >> 8) + 0.5f) * (1.0f / 16777216.0f);
        const float u2 = ((x[2] >> 8) + 0.5f) * (1.0f / 16777216.0f);
        pn += F.noise_amp * w * (sqrtf(-2.0f * __logf(u1)) * __cosf(6.2831853f * u2));
      }
    }
    const float psi_new = pn > 1.0f ? 1.0f : pn;

    const float S00 = s_S[r], S10 = s_S[r + 1], Sm0 = s_S[r - 1], S01 = s_S[r + RW], S0m = s_S[r - RW];
    const float S11 = s_S[r + RW + 1], Sm1 = s_S[r + RW - 1], S1m = s_S[r - RW + 1], Smm = s_S[r - RW - 1];
    const float Shh = 0.25f * (S11 + S10 + S01 + S00);
    const float Shn = 0.25f * (S10 + S00 + S1m + S0m);
    const float Snh = 0.25f * (Sm1 + S01 + Sm0 + S00);
    const float Snn = 0.25f * (Sm0 + Smm + S0m + S00);
    const float f00 = s_mu[r];
    const float F10 = (S10 + S00 + Shh + Shn) * (s_mu[r + 1] - f00 + s_dK[tx + 1]);
    const float Fm0 = (S00 + Sm0 + Snh + Snn) * (s_mu[r - 1] - f00 - s_dK[tx]);
    const float F01 = (S01 + S00 + Shh + Snh) * (s_mu[r + RW] - f00);
    const float F0m = (S00 + S0m + Shn + Snn) * (s_mu[r - RW] - f00);
    const float dd = F.cflux * (F10 + F01 + Fm0 + F0m);
    const float d_new = fmaxf(d00 + dd, F.floor_delta);

    const float phi_new = fminf(fmaxf(psi_new, -1.0f), 1.0f);
    const int gx2 = gi == 1 ? 0 : (gi == nx - 2 ? nx - 1 : -1);
    const int gy2 = gj == jmin ? 0 : (gj == jmax ? ny - 1 : -1);
    auto put = [&](int ii, int jj) {
      const int64_t o = (int64_t)jj * pitch + ii;
      psi_n[o] = psi_new;
      cd_n[o] = d_new;
      if (phi_n) phi_n[o] = phi_new;
    };
    put(gi, gj);
    if (gx2 >= 0) put(gx2, gj);
    if (gy2 >= 0) {
      put(gi, gy2);
      if (gx2 >= 0) put(gx2, gy2);
    }
    if (partials) {
      mass += (double)d_new;
      if (psi_new > 0.0f) itip = max(itip, gi == nx - 2 ? nx - 1 : gi);
    }
  }
  if (partials) block_partial<NT>(mass, itip, partials);
}

static CoefF make_coef_f(const StepCoef &K) {
  CoefF F;
  F.inv_2dx = (float)K.inv_2dx;
  F.inv_dx2 = (float)K.inv_dx2;
  F.inv_4dx2 = (float)K.inv_4dx2;
  F.inv_2dx2 = (float)K.inv_2dx2;
  F.dt = (float)K.dt;
  F.eps1 = (float)K.eps1;
  F.eps2 = (float)K.eps2;
  F.epk1 = (float)K.epk1;
  F.ox1 = (float)K.ox1; F.ox2 = (float)K.ox2;
  F.oy1 = (float)K.oy1; F.oy2 = (float)K.oy2;
  F.oz1 = (float)K.oz1; F.oz2 = (float)K.oz2;
  F.drive = (float)K.drive;
  F.cflux = (float)(0.25 * K.cfac * K.inv_h0v0);  // 0.25 of the face-mobility average folded in
  F.AA = (float)K.AA;
  F.cinf = (float)K.cinf;
  F.Lref = (float)K.Lref;
  F.noise_amp = (float)K.noise_amp;
  F.floor_delta = (float)(1.0e-6 - K.cinf);
  return F;
}

int launch_step_f32(const StepCoef &K, const StepScalars &P, const float *psi, const float *c, float *psi_n,
                    float *c_n, float *phi_n, BlockPartial *partials, int max_partials, int *nblocks_out,
                    cudaStream_t st) {
  const CoefF F = make_coef_f(K);
  const int ni = K.nx - 2, nj = K.ny - 2;
  const bool small = (int64_t)ni * nj < 148 * 4 * 1024;
  dim3 block(32, 8);
  dim3 grid((ni + 31) / 32, small ? (nj + 7) / 8 : (nj + 31) / 32);
  const int nb = grid.x * grid.y;
  if (partials && nb > max_partials) return -1;
  if (small)
    step_f32_kernel<32, 8, 1><<<grid, block, 0, st>>>(K, F, P, psi, c, psi_n, c_n, phi_n, partials);
  else
    step_f32_kernel<32, 8, 4><<<grid, block, 0, st>>>(K, F, P, psi, c, psi_n, c_n, phi_n, partials);
  if (nblocks_out) *nblocks_out = nb;
  return 0;
}

}  // namespace rs

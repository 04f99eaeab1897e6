// rs_step_f64.cu — fused FP64 time step (the drop-in exact path).
//
// One kernel replaces the reference's per-step launch sequence
//   [pull_back] -> compute_phi -> compute_psi -> compute_c_CALPHAD
// (fun.cu:451-478 / main.cu:179-213):
//   * the moving-frame shift of pull_back (fun.cu:1469-1492) is applied as a
//     read-side index remap while the tile is staged, so a pull-back step
//     costs no extra pass;
//   * phi = clamp(psi, -1, 1) for one orientation (compute_psi,
//     fun.cu:1232-1273), so only psi and c are read and written
//     (32 B per cell-step);
//   * per cell, S = q(psi) c (1-c) and the chemical potential mu
//     (fun.cu:1424-1452) are evaluated once into shared memory instead of
//     once per neighbour; the frozen-temperature CALPHAD groups are evaluated
//     once per column of the tile;
//   * ghost cells are written by the cell they copy (compute_boundary_individual,
//     fun.cu:1220-1230), corners included.
// Optional per-block partials (sum of c, max tip column) feed rs_mass/rs_itip
// style reductions without another pass over the grid.
#include "rs_kernels.cuh"

namespace rs {

// get_anisotropy (fun.cu:1030-1139) on nine clamped phi values.
__device__ __forceinline__ double anisotropy_f64(const StepCoef &K, double phi00, double phi10,
                                                 double phim0, double phi01, double phi0m,
                                                 double phi11, double phim1, double phi1m,
                                                 double phimm, double &as, double &ak) {
  const double dphi_dx = (phi10 - phim0) * K.inv_2dx;
  const double dphi_dy = (phi01 - phi0m) * K.inv_2dx;
  const double g2 = dphi_dx * dphi_dx + dphi_dy * dphi_dy;
  const double abs_g = sqrt(g2);
  const double dxx = (phi10 - 2.0 * phi00 + phim0) * K.inv_dx2;
  const double dyy = (phi01 - 2.0 * phi00 + phi0m) * K.inv_dx2;
  const double dxy = (phi11 - phim1 - phi1m + phimm) * K.inv_4dx2;
  double lap = (2.0 / 3.0) * (dxx + dyy);
  lap += (1.0 / 3.0) * (phi11 + phim1 + phi1m + phimm - 4.0 * phi00) * K.inv_2dx2;

  double dtx = 0.0, dty = 0.0, cs = 0.0, sn = 0.0;
  if (abs_g > 1.0e-15) {
    const double inv_a = 1.0 / abs_g;
    const double inv_g2 = inv_a * inv_a;
    dtx = (dphi_dx * dxy - dphi_dy * dxx) * inv_g2;
    dty = (dphi_dx * dyy - dphi_dy * dxy) * inv_g2;
    cs = dphi_dx * inv_a;
    sn = dphi_dy * inv_a;
  }
  const double nx = K.ox1 * cs + K.ox2 * sn;
  const double ny = K.oy1 * cs + K.oy2 * sn;
  const double nz = K.oz1 * cs + K.oz2 * sn;
  const double nx1 = -K.ox1 * sn + K.ox2 * cs;
  const double ny1 = -K.oy1 * sn + K.oy2 * cs;
  const double nz1 = -K.oz1 * sn + K.oz2 * cs;
  const double nx3 = nx * nx * nx, ny3 = ny * ny * ny, nz3 = nz * nz * nz;
  const double np4 = nx3 * nx + ny3 * ny + nz3 * nz;
  const double dnp4_1 = 4.0 * (nx3 * nx1 + ny3 * ny1 + nz3 * nz1);
  // second theta-derivative; d(n)/d(theta)^2 = -n (fun.cu:1094-1103)
  const double ax = nx * nx1, ay = ny * ny1, az = nz * nz1;
  const double dnp4_2 =
      4.0 * ((3.0 * (ax * ax) - nx3 * nx) + (3.0 * (ay * ay) - ny3 * ny) + (3.0 * (az * az) - nz3 * nz));
  double da1, da2;
  if (K.one_eps) {
    ak = 1.0 - 3.0 * K.epk1 + 4.0 * K.epk1 * np4;
    as = 1.0 - 3.0 * K.eps1 + 4.0 * K.eps1 * np4;
    da1 = 4.0 * K.eps1 * dnp4_1;
    da2 = 4.0 * K.eps1 * dnp4_2;
  } else {
    const double xyz = nx * ny * nz;
    ak = 1.0 + K.epk1 * (np4 - 0.6);
    as = 1.0 + K.eps1 * (np4 - 0.6) + K.eps2 * (3.0 * np4 + 66.0 * (xyz * xyz) - 17.0 / 7.0);
    const double t1 = nx1 * ny * nz + nx * ny1 * nz + nx * ny * nz1;
    const double dnp2_1 = 2.0 * xyz * t1;
    double dnp2_2 = (nx1 * ny * nz) * (nx1 * ny * nz) + (nx * ny1 * nz) * (nx * ny1 * nz) +
                    (nx * ny * nz1) * (nx * ny * nz1);
    dnp2_2 += -nx * nx * (ny * nz) * (ny * nz) - ny * ny * (nx * nz) * (nx * nz) -
              nz * nz * (nx * ny) * (nx * ny);
    dnp2_2 += 4.0 * xyz * (nx1 * ny1 * nz + nx * ny1 * nz1 + nx1 * ny * nz1);
    dnp2_2 *= 2.0;
    da1 = (K.eps1 + 3.0 * K.eps2) * dnp4_1 + 66.0 * K.eps2 * dnp2_1;
    da2 = (K.eps1 + 3.0 * K.eps2) * dnp4_2 + 66.0 * K.eps2 * dnp2_2;
  }
  return (as * as) * lap + 2.0 * as * da1 * (dtx * dphi_dx + dty * dphi_dy) +
         (da2 * as + da1 * da1) * (dty * dphi_dx - dtx * dphi_dy);
}

// bilinear coarse -> fine temperature (interpolate_temperature, fun.cu:1580-1608)
__device__ __forceinline__ double t_fine(const StepCoef &K, const double *__restrict__ T, int ile,
                                         int i, int j) {
  int iT = (i - 1 + ile) / K.ratio;
  int jT = (int)((j - 1 + K.dxT) / K.ratio);
  const double x = (i - 1.0 + ile) / K.ratio - iT;
  const double y = (j - 1.0 + K.dxT) / K.ratio - jT;
  // the reference reads past the coarse array when the window leaves it; clamp
  iT = min(max(iT, 0), K.NxT_all - 2);
  jT = min(max(jT, 0), K.NyT_all - 2);
  const double f00 = T[(int64_t)jT * K.NxT_all + iT];
  const double f10 = T[(int64_t)jT * K.NxT_all + iT + 1];
  const double f01 = T[(int64_t)(jT + 1) * K.NxT_all + iT];
  const double f11 = T[(int64_t)(jT + 1) * K.NxT_all + iT + 1];
  const double a10 = f10 - f00, a01 = f01 - f00, a11 = f11 - f10 - f01 + f00;
  return f00 + a10 * x + a01 * y + a11 * x * y;
}

template <int BX, int BY, int RY>
__global__ void __launch_bounds__(BX *BY)
    step_f64_kernel(const StepCoef K, const StepScalars P, const double *__restrict__ psi,
                    const double *__restrict__ c, double *__restrict__ psi_n,
                    double *__restrict__ c_n, double *__restrict__ phi_n, BlockPartial *partials) {
  constexpr int TX = BX, TY = BY * RY, RW = TX + 2, RH = TY + 2, NT = BX * BY;
  __shared__ double s_phi[RH * RW];
  __shared__ double s_S[RH * RW];
  __shared__ double s_mu[RH * RW];
  __shared__ double s_c[RH * RW];
  __shared__ TTerms s_col[RW];

  const int nx = K.nx, ny = K.ny, pitch = K.pitch;
  const int x0 = 1 + blockIdx.x * TX, y0 = 1 + blockIdx.y * TY;
  const int tid = threadIdx.y * BX + threadIdx.x;

  if (!K.tfc) {
    for (int rx = tid; rx < RW; rx += NT) {
      const int gi = x0 - 1 + rx;
      const double T = (P.d0 + P.d1 * gi) * K.deltaT0 + K.Tmelt;
      s_col[rx] = t_terms(T, K.RR);
    }
    __syncthreads();
  }

  // stage psi, c (+ pull-back remap) and per-cell phi, S, mu
  for (int idx = tid; idx < RH * RW; idx += NT) {
    const int ry = idx / RW, rx = idx - ry * RW;
    const int gi = x0 - 1 + rx, gj = y0 - 1 + ry;
    if (gi >= nx || gj >= ny) continue;
    int si = gi;
    if (P.pull_back) si = min(max(gi + P.i_offset, 1), nx - 2);
    const int64_t src = (int64_t)gj * pitch + si;
    const double pv = psi[src];
    const double cv = (P.pull_back && si >= nx - 2) ? K.cinf : c[src];
    s_phi[idx] = fmin(fmax(pv, -1.0), 1.0);
    s_c[idx] = cv;
    s_S[idx] = qq(K.AA, pv) * cv * (1.0 - cv);
    const bool corner = (rx == 0 || rx == RW - 1) && (ry == 0 || ry == RH - 1);
    if (!corner) {
      const TTerms t = K.tfc ? t_terms(t_fine(K, P.T_coarse, P.i_left_end_T, gi, gj), K.RR) : s_col[rx];
      const double g = gg(pv);
      const double onemc = 1.0 - cv;
      double L = 0.0;
      if (cv > 1.e-8 && onemc > 1.e-8) L = t.RT * log(cv / onemc);
      const double tl0 = 1.0 - 2.0 * cv;
      const double gsc = t.dGs + kL0Bcc * tl0 + L;
      const double glc = t.dGl + kL0Liq * tl0 + L;
      s_mu[idx] = 0.5 * (1.0 + g) * gsc + 0.5 * (1.0 - g) * glc;
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
    // ---- phi (compute_phi, fun.cu:1143-1218)
    const double phi00 = s_phi[r];
    double as, ak;
    const double aniso = anisotropy_f64(K, phi00, s_phi[r + 1], s_phi[r - 1], s_phi[r + RW], s_phi[r - RW],
                                        s_phi[r + RW + 1], s_phi[r + RW - 1], s_phi[r - RW + 1],
                                        s_phi[r - RW - 1], as, ak);
    const double c00 = s_c[r];
    TTerms t0;
    if (K.tfc)
      t0 = t_terms(t_fine(K, P.T_coarse, P.i_left_end_T, gi, gj), K.RR);
    else
      t0 = s_col[tx + 1];
    const double dG = (1.0 - c00) * t0.A_nb + c00 * t0.A_ti + c00 * (1.0 - c00) * (kL0Liq - kL0Bcc);
    const double term = phi00 - phi00 * phi00 * phi00 + aniso + dG * dgg_dp(phi00) * K.drive;
    double pn = phi00 + K.dt * ak / (as * as) * term;
    if (K.noise_amp > 0.0) {
      const double w = 1.0 - phi00 * phi00;
      if (w > 1.0e-3) {
        uint32_t x[4];
        noise_counter(x, P.step, (int64_t)gj * nx + gi);
        philox4x32(x, K.seed_lo, K.seed_hi);
        const double u1 = u53(x[0], x[1]), u2 = u53(x[2], x[3]);
        pn += K.noise_amp * w * (sqrt(-2.0 * log(u1)) * cospi(2.0 * u2));
      }
    }
    const double psi_new = pn > 1.0 ? 1.0 : pn;  // renormalisation (fun.cu:1252-1261)

    // ---- c (compute_c_CALPHAD, fun.cu:1365-1467)
    const double S00 = s_S[r], S10 = s_S[r + 1], Sm0 = s_S[r - 1], S01 = s_S[r + RW], S0m = s_S[r - RW];
    const double S11 = s_S[r + RW + 1], Sm1 = s_S[r + RW - 1], S1m = s_S[r - RW + 1], Smm = s_S[r - RW - 1];
    const double Shh = 0.25 * (S11 + S10 + S01 + S00);
    const double Shn = 0.25 * (S10 + S00 + S1m + S0m);
    const double Snh = 0.25 * (Sm1 + S01 + Sm0 + S00);
    const double Snn = 0.25 * (Sm0 + Smm + S0m + S00);
    const double f00 = s_mu[r];
    const double F10 = 0.25 * (S10 + S00 + Shh + Shn) * (s_mu[r + 1] - f00);
    const double F01 = 0.25 * (S01 + S00 + Shh + Snh) * (s_mu[r + RW] - f00);
    const double Fm0 = 0.25 * (S00 + Sm0 + Snh + Snn) * (s_mu[r - 1] - f00);
    const double F0m = 0.25 * (S00 + S0m + Shn + Snn) * (s_mu[r - RW] - f00);
    const double dc = K.cfac * ((F10 + F01 + Fm0 + F0m) * K.inv_h0v0);
    const double c_new = fmax(c00 + dc, 1.0e-6);

    // ---- stores, ghosts (compute_boundary_individual, fun.cu:1220-1230)
    const double phi_new = fmin(fmax(psi_new, -1.0), 1.0);
    const int gx2 = gi == 1 ? 0 : (gi == nx - 2 ? nx - 1 : -1);
    const int gy2 = gj == jmin ? 0 : (gj == jmax ? ny - 1 : -1);
    auto put = [&](int ii, int jj) {
      const int64_t o = (int64_t)jj * pitch + ii;
      psi_n[o] = psi_new;
      c_n[o] = c_new;
      if (phi_n) phi_n[o] = phi_new;
    };
    put(gi, gj);
    if (gx2 >= 0) put(gx2, gj);
    if (gy2 >= 0) {
      put(gi, gy2);
      if (gx2 >= 0) put(gx2, gy2);
    }
    if (partials) {
      mass += c_new;
      if (psi_new > 0.0) itip = max(itip, gi == nx - 2 ? nx - 1 : gi);
    }
  }
  if (partials) block_partial<NT>(mass, itip, partials);
}

int launch_step_f64(const StepCoef &K, const StepScalars &P, const double *psi, const double *c,
                    double *psi_n, double *c_n, double *phi_n, BlockPartial *partials,
                    int max_partials, int *nblocks_out, cudaStream_t st) {
  const int ni = K.nx - 2, nj = K.ny - 2;
  // small grids: shorter tiles so that every SM gets work
  const bool small = (int64_t)ni * nj < 148 * 4 * 1024;
  dim3 block(32, 8);
  dim3 grid((ni + 31) / 32, small ? (nj + 7) / 8 : (nj + 31) / 32);
  const int nb = grid.x * grid.y;
  if (partials && nb > max_partials) return -1;
  if (small)
    step_f64_kernel<32, 8, 1><<<grid, block, 0, st>>>(K, P, psi, c, psi_n, c_n, phi_n, partials);
  else
    step_f64_kernel<32, 8, 4><<<grid, block, 0, st>>>(K, P, psi, c, psi_n, c_n, phi_n, partials);
  if (nblocks_out) *nblocks_out = nb;
  return 0;
}

}  // namespace rs

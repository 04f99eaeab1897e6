// rs_step.cu — the fused phase-field time step, FP64 (exact drop-in) and FP32
// (bulk) from one kernel template.
//
// One launch replaces the reference's per-step sequence
//   [pull_back] -> compute_phi -> compute_psi -> compute_c_CALPHAD
// (fun.cu:451-478, main.cu:179-213):
//   * the pull_back column shift (fun.cu:1469-1492) is a read-side remap of
//     the source column, so a pull-back step costs no extra pass;
//   * one orientation: phi = clamp(psi, -1, 1) (compute_psi,
//     fun.cu:1232-1273), so only psi and c are read and written;
//   * ghost cells (compute_boundary_individual, fun.cu:1220-1230) are written
//     by the cell they copy, corners included.
//
// Layout of the work: a warp owns a strip of 30 output columns (32 input
// columns with a one-column halo on each side) and marches down H rows.  Each
// row of psi and c is loaded once per warp with a coalesced 32-lane load
// (issued P rows ahead), the per-cell quantities phi, S = q(psi)c(1-c)
// (fun.cu:1424-1432) and the chemical potential mu (fun.cu:1443-1452) are
// computed once per cell, vertical neighbours come from a three-row register
// window and horizontal neighbours from warp shuffles.  No shared memory, no
// block barriers.
//
// Arithmetic (identical mathematics to the reference, regrouped):
//   * anisotropy (get_anisotropy, fun.cu:1030-1139): with n = R (cos, sin, 0),
//     |n|^4 = k0 + k1 cos2t + k2 sin2t + k3 cos4t + k4 sin4t exactly, and
//     cos2t = (px^2 - py^2)/|grad phi|^2, sin2t = 2 px py/|grad phi|^2, so
//     a_s, a_k and both theta-derivatives need one reciprocal and no sqrt or
//     trigonometry.  k0..k4 come from the orientation on the host.
//   * mu = K(T) + mu', with the composition-independent column part
//     K(T) = (dGs+dGl)/2 + (L0_BCC+L0_Liq)(1-2cinf)/2 + RT log(cinf/(1-cinf))
//     in FP64 per column (only its i-differences enter the fluxes) and
//     mu' = g D - delta (L0_BCC+L0_Liq) + g (L0_BCC-L0_Liq)(1-2c)/2
//           + RT [log(c/(1-c)) - log(cinf/(1-cinf))],  D = (dGs-dGl)/2,
//     delta = c - cinf.  FP32 needs this split (mu ~ 1e4 J/mol while the
//     fluxes see neighbour differences of 1e-1..1e2 J/mol).
//   * Gl - Gs = (1-c) A_Nb + c A_Ti + c(1-c)(L0_Liq - L0_BCC): the ideal-mixing
//     terms of Gl and Gs (fun.cu:1671-1698) cancel exactly.
//   * exact shortcuts, warp-uniform: if all nine phi of every cell of the row
//     are the same +-1, phi_next = phi (phi - phi^3 = 0, g'(+-1) = 0, grad = 0);
//     if all nine S are 0 (solid, q(1) = 0) the solute update is dc = 0.
//     Both give bit-identical results to the general formulas.
// FP32 field sets store delta = c - cinf (see include/rs_b200.h).
#include <cuda.h>

#include <type_traits>

#include "rs_kernels.cuh"

namespace rs {

// FP32 chemical-potential remainder log(c/(1-c)) - log(cinf/(1-cinf)) =
// log((1+s)/(1-s)) = 2 atanh(s), s = delta / (2 cinf (1-c) + delta):
// odd series to s^9 for |s| < 1/9 (truncation < 1e-10 relative), hardware
// log beyond.
__device__ __forceinline__ float lam_fast(float d, float omc, float two_cinf) {
  const float s = __fdividef(d, fmaf(two_cinf, omc, d));
  const float s2 = s * s;
  float p = fmaf(s2, 1.0f / 9.0f, 1.0f / 7.0f);
  p = fmaf(s2, p, 1.0f / 5.0f);
  p = fmaf(s2, p, 1.0f / 3.0f);
  p = fmaf(s2, p, 1.0f);
  float r = (s + s) * p;
  if (fabsf(s) >= 1.0f / 9.0f) r = __logf(__fdividef(1.0f + s, 1.0f - s));
  return r;
}

template <typename R>
struct Tr;

template <>
struct Tr<double> {
  using S = double;  // storage
  static constexpr bool kDelta = false;
  __device__ static double rcp(double x) { return 1.0 / x; }
  __device__ static double div(double a, double b) { return a / b; }
  // RT (log(c/(1-c)) - Lref), with the L(c) = 0 guard of fun.cu:1704-1706
  __device__ static double lam(double c, double omc, double d, double cinf, double Lref) {
    if (c > 1.e-8 && omc > 1.e-8) return log(c / omc) - Lref;
    return -Lref;
  }
  __device__ static double normal(uint32_t x[4]) {
    const double u1 = u53(x[0], x[1]), u2 = u53(x[2], x[3]);
    return sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
  }
};

template <>
struct Tr<float> {
  using S = float;
  static constexpr bool kDelta = true;
  __device__ static float rcp(float x) { return __fdividef(1.0f, x); }
  __device__ static float div(float a, float b) { return __fdividef(a, b); }
  __device__ static float lam(float c, float omc, float d, float cinf, float Lref) {
    if (c > 1.e-8f && omc > 1.e-8f) return lam_fast(d, omc, cinf + cinf);
    return -Lref;
  }
  __device__ static float normal(uint32_t x[4]) {
    const float u1 = ((x[0] >> 8) + 0.5f) * (1.0f / 16777216.0f);
    const float u2 = ((x[2] >> 8) + 0.5f) * (1.0f / 16777216.0f);
    return sqrtf(-2.0f * __logf(u1)) * __cosf(6.2831853f * u2);
  }
};

// Kernel constants in the working precision.
template <typename R>
struct Coef {
  R inv_2dx, inv_dx2, inv_4dx2, inv_2dx2, dt;
  R eps1, eps2, epk1;
  R k0, k1, k2, k3, k4;                  // |n|^4 harmonics
  R ox1, ox2, oy1, oy2, oz1, oz2;        // two-eps fallback
  R as0, ak0;                            // a_s, a_k at |grad phi| = 0
  R drive, cflux, AA, cinf, Lref, noise_amp, c_floor;
  int one_eps;
};

template <typename R>
Coef<R> make_coef(const StepCoef &K) {
  Coef<R> F;
  F.inv_2dx = (R)K.inv_2dx;
  F.inv_dx2 = (R)K.inv_dx2;
  F.inv_4dx2 = (R)K.inv_4dx2;
  F.inv_2dx2 = (R)K.inv_2dx2;
  F.dt = (R)K.dt;
  F.eps1 = (R)K.eps1;
  F.eps2 = (R)K.eps2;
  F.epk1 = (R)K.epk1;
  // n_k = a_k cos + b_k sin for the three crystal axes (rows of the
  // orientation matrix, fun.cu:1080-1085); sum of n_k^4 in harmonics
  const double ab[3][2] = {{K.ox1, K.ox2}, {K.oy1, K.oy2}, {K.oz1, K.oz2}};
  double k0 = 0, k1 = 0, k2 = 0, k3 = 0, k4 = 0;
  for (int k = 0; k < 3; ++k) {
    const double a = ab[k][0], b = ab[k][1];
    const double a2 = a * a, b2 = b * b;
    k0 += (3 * a2 * a2 + 6 * a2 * b2 + 3 * b2 * b2) / 8;
    k1 += (a2 * a2 - b2 * b2) / 2;
    k2 += a2 * a * b + a * b2 * b;
    k3 += (a2 * a2 - 6 * a2 * b2 + b2 * b2) / 8;
    k4 += (a2 * a * b - a * b2 * b) / 2;
  }
  F.k0 = (R)k0;
  F.k1 = (R)k1;
  F.k2 = (R)k2;
  F.k3 = (R)k3;
  F.k4 = (R)k4;
  F.ox1 = (R)K.ox1;
  F.ox2 = (R)K.ox2;
  F.oy1 = (R)K.oy1;
  F.oy2 = (R)K.oy2;
  F.oz1 = (R)K.oz1;
  F.oz2 = (R)K.oz2;
  if (K.one_eps) {
    F.as0 = (R)(1.0 - 3.0 * K.eps1);
    F.ak0 = (R)(1.0 - 3.0 * K.epk1);
  } else {
    F.as0 = (R)(1.0 + K.eps1 * (0.0 - 0.6) + K.eps2 * (0.0 - 17.0 / 7.0));
    F.ak0 = (R)(1.0 + K.epk1 * (0.0 - 0.6));
  }
  F.drive = (R)K.drive;
  F.cflux = (R)(0.25 * K.cfac * K.inv_h0v0);  // face-mobility 1/4 folded in
  F.AA = (R)K.AA;
  F.cinf = (R)K.cinf;
  F.Lref = (R)K.Lref;
  F.noise_amp = (R)K.noise_amp;
  F.c_floor = (R)1.0e-6;
  F.one_eps = K.one_eps;
  return F;
}

// anisotropic operator of get_anisotropy (fun.cu:1030-1139)
template <typename R>
__device__ __forceinline__ R anisotropy(const Coef<R> &F, R phi00, R phi10, R phim0,
                                        R phi01, R phi0m, R phi11, R phim1, R phi1m, R phimm, R &as,
                                        R &ak) {
  const R px = (phi10 - phim0) * F.inv_2dx;
  const R py = (phi01 - phi0m) * F.inv_2dx;
  const R g2 = px * px + py * py;
  const R dxx = (phi10 - R(2) * phi00 + phim0) * F.inv_dx2;
  const R dyy = (phi01 - R(2) * phi00 + phi0m) * F.inv_dx2;
  const R dxy = (phi11 - phim1 - phi1m + phimm) * F.inv_4dx2;
  const R lap = (R(2) / R(3)) * (dxx + dyy) +
                (R(1) / R(3)) * (phi11 + phim1 + phi1m + phimm - R(4) * phi00) * F.inv_2dx2;
  // |grad phi| > 1e-15 (fun.cu:1056)
  if (!(g2 > R(1.0e-30))) {
    as = F.as0;
    ak = F.ak0;
    return (as * as) * lap;
  }
  const R ig2 = Tr<R>::rcp(g2);
  const R dtx = (px * dxy - py * dxx) * ig2;
  const R dty = (px * dyy - py * dxy) * ig2;
  R da1, da2;
  if (F.one_eps) {
    const R C2 = (px * px - py * py) * ig2;
    const R S2 = R(2) * px * py * ig2;
    const R C4 = C2 * C2 - S2 * S2;
    const R S4 = R(2) * S2 * C2;
    const R np4 = F.k0 + F.k1 * C2 + F.k2 * S2 + F.k3 * C4 + F.k4 * S4;
    const R d1 = R(2) * (F.k2 * C2 - F.k1 * S2) + R(4) * (F.k4 * C4 - F.k3 * S4);
    const R d2 = R(-4) * (F.k1 * C2 + F.k2 * S2) - R(16) * (F.k3 * C4 + F.k4 * S4);
    ak = R(1) - R(3) * F.epk1 + R(4) * F.epk1 * np4;
    as = R(1) - R(3) * F.eps1 + R(4) * F.eps1 * np4;
    da1 = R(4) * F.eps1 * d1;
    da2 = R(4) * F.eps1 * d2;
  } else {
    // (eps1, eps2) form needs the sextic (n_x n_y n_z)^2: explicit directions
    const R ia = sqrt(ig2);
    const R cs = px * ia, sn = py * ia;
    const R nx = F.ox1 * cs + F.ox2 * sn, ny = F.oy1 * cs + F.oy2 * sn, nz = F.oz1 * cs + F.oz2 * sn;
    const R nx1 = F.ox2 * cs - F.ox1 * sn, ny1 = F.oy2 * cs - F.oy1 * sn, nz1 = F.oz2 * cs - F.oz1 * sn;
    const R nx3 = nx * nx * nx, ny3 = ny * ny * ny, nz3 = nz * nz * nz;
    const R np4 = nx3 * nx + ny3 * ny + nz3 * nz;
    const R dnp4_1 = R(4) * (nx3 * nx1 + ny3 * ny1 + nz3 * nz1);
    const R ax = nx * nx1, ay = ny * ny1, az = nz * nz1;
    const R dnp4_2 = R(4) * (R(3) * (ax * ax + ay * ay + az * az) - np4);
    const R xyz = nx * ny * nz;
    ak = R(1) + F.epk1 * (np4 - R(0.6));
    as = R(1) + F.eps1 * (np4 - R(0.6)) + F.eps2 * (R(3) * np4 + R(66) * (xyz * xyz) - R(17) / R(7));
    const R t1 = nx1 * ny * nz + nx * ny1 * nz + nx * ny * nz1;
    const R dnp2_1 = R(2) * xyz * t1;
    R dnp2_2 = (nx1 * ny * nz) * (nx1 * ny * nz) + (nx * ny1 * nz) * (nx * ny1 * nz) +
               (nx * ny * nz1) * (nx * ny * nz1);
    dnp2_2 += -nx * nx * (ny * nz) * (ny * nz) - ny * ny * (nx * nz) * (nx * nz) - nz * nz * (nx * ny) * (nx * ny);
    dnp2_2 += R(4) * xyz * (nx1 * ny1 * nz + nx * ny1 * nz1 + nx1 * ny * nz1);
    dnp2_2 *= R(2);
    da1 = (F.eps1 + R(3) * F.eps2) * dnp4_1 + R(66) * F.eps2 * dnp2_1;
    da2 = (F.eps1 + R(3) * F.eps2) * dnp4_2 + R(66) * F.eps2 * dnp2_2;
  }
  return (as * as) * lap + R(2) * as * da1 * (dtx * px + dty * py) + (da2 * as + da1 * da1) * (dty * px - dtx * py);
}

__device__ __forceinline__ double t_fine_at(const StepCoef &K, const double *__restrict__ T, int ile, int i, int j) {
  // interpolate_temperature (fun.cu:1580-1608); indices clamped where the
  // reference would read outside the coarse array
  int iT = (i - 1 + ile) / K.ratio;
  int jT = (int)((j - 1 + K.dxT) / K.ratio);
  const double x = (i - 1.0 + ile) / K.ratio - iT;
  const double y = (j - 1.0 + K.dxT) / K.ratio - jT;
  iT = min(max(iT, 0), K.NxT_all - 2);
  jT = min(max(jT, 0), K.NyT_all - 2);
  const double f00 = T[(int64_t)jT * K.NxT_all + iT];
  const double f10 = T[(int64_t)jT * K.NxT_all + iT + 1];
  const double f01 = T[(int64_t)(jT + 1) * K.NxT_all + iT];
  const double f11 = T[(int64_t)(jT + 1) * K.NxT_all + iT + 1];
  const double a10 = f10 - f00, a01 = f01 - f00, a11 = f11 - f10 - f01 + f00;
  return f00 + a10 * x + a01 * y + a11 * x * y;
}

// column (or, with TFC, cell) CALPHAD groups in the working precision
template <typename R>
struct ColT {
  R A_nb, A_ti, D, RT;
  double Kc;  // K(T), FP64
};

template <typename R>
__device__ __forceinline__ ColT<R> col_terms(const StepCoef &K, double T) {
  const TTerms t = t_terms(T, K.RR);
  ColT<R> c;
  c.A_nb = (R)t.A_nb;
  c.A_ti = (R)t.A_ti;
  c.D = (R)(0.5 * (t.dGs - t.dGl));
  c.RT = (R)t.RT;
  c.Kc = 0.5 * (t.dGs + t.dGl) + 0.5 * (kL0Bcc + kL0Liq) * (1.0 - 2.0 * K.cinf) + t.RT * K.Lref;
  return c;
}

// Per-lane state of a warp marching down a strip of 30 output columns, and
// the work for one incoming row.  Shared by the register-prefetch kernel and
// the TMA-pipelined kernel so both execute identical arithmetic.
template <typename R, bool TFC>
struct Strip {
  using S = typename Tr<R>::S;
  static constexpr unsigned FULL = 0xffffffffu;
  int gi, gic, gx2, y_last;
  bool out_lane;
  ColT<R> col;
  R dKr;
  // three-row window: index 0 = row r-1, 1 = row r, 2 = row r+1
  R p0, p1, p2, pl0, pl1, pl2, pr0, pr1, pr2;
  R s0, s1, s2, sl1, sl2, sr0, sr1, sr2;
  R m1, m2;        // mu' of rows r, r+1
  R d1, d2;        // stored c value (FP32: c - cinf) of rows r, r+1
  R jv_lo, jv_hi;  // solute flux through the faces (r-1/2) and (r+1/2)
  bool sol0, sol1, sol2, liq0, liq1, liq2;
  R A1nb, A1ti, A2nb, A2ti;  // TFC: driving-force groups of rows r, r+1
  R kr1, kr2;                // TFC: K(i+1) - K(i) of rows r, r+1
  double Kc2;
  double mass;
  int itip;

  __device__ __forceinline__ void init(const StepCoef &K, const StepScalars &PS, int gi_, int y_last_, bool active) {
    gi = gi_;
    gic = min(gi, K.nx - 1);
    gx2 = gi == 1 ? 0 : (gi == K.nx - 2 ? K.nx - 1 : -1);
    y_last = y_last_;
    out_lane = active && (threadIdx.x & 31) >= 1 && (threadIdx.x & 31) <= 30 && gi <= K.nx - 2;
    p0 = p1 = p2 = pl0 = pl1 = pl2 = pr0 = pr1 = pr2 = R(0);
    s0 = s1 = s2 = sl1 = sl2 = sr0 = sr1 = sr2 = R(0);
    m1 = m2 = d1 = d2 = jv_lo = jv_hi = R(0);
    sol0 = sol1 = sol2 = liq0 = liq1 = liq2 = false;
    A1nb = A1ti = A2nb = A2ti = kr1 = kr2 = R(0);
    Kc2 = 0.0;
    mass = 0.0;
    itip = 0;
    dKr = R(0);
    if (!TFC) {
      // frozen temperature: CALPHAD groups of this column, once per strip
      const double T = (PS.d0 + PS.d1 * gi) * K.deltaT0 + K.Tmelt;
      col = col_terms<R>(K, T);
      const double Kn = __shfl_down_sync(FULL, col.Kc, 1);
      dKr = (R)(Kn - col.Kc);  // K(i+1) - K(i)
    }
  }

  // row `row` (k-th row of the strip, k = 0 is y0-1) arrives with psi = pv and
  // stored c value cv_s; once three rows are in the window, row-1 is output.
  __device__ __forceinline__ void step_row(const StepCoef &K, const Coef<R> &F, const StepScalars &PS, R pv, R cv_s,
                                           int k, int row, S *__restrict__ psi_n, S *__restrict__ c_n,
                                           S *__restrict__ phi_n, bool red) {
    const R cinf = F.cinf;
    // ---- per-cell quantities of the new row
    const R d = Tr<R>::kDelta ? cv_s : cv_s - cinf;
    const R c = Tr<R>::kDelta ? cinf + cv_s : cv_s;
    const R omc = R(1) - c;
    const R ph = fmin(fmax(pv, R(-1)), R(1));
    const R a = R(1) - pv;
    const R Sv = (R(0.5) * F.AA * a - R(0.25) * (F.AA - R(1)) * (a * a)) * c * omc;
    const R p2v = pv * pv;
    const R g = pv * (R(1.875) + p2v * (R(-1.25) + R(0.375) * p2v));
    ColT<R> ct = col;
    if (TFC) ct = col_terms<R>(K, t_fine_at(K, PS.T_coarse, PS.i_left_end_T, gic, min(row, K.ny - 1)));
    constexpr R L0sum = R(kL0Bcc + kL0Liq);
    constexpr R L0half = R(0.5 * (kL0Bcc - kL0Liq));
    const R mu = g * ct.D - d * L0sum + g * L0half * (R(1) - R(2) * c) + ct.RT * Tr<R>::lam(c, omc, d, cinf, F.Lref);
    const bool row_sol = __ballot_sync(FULL, ph == R(1)) == FULL;
    const bool row_liq = __ballot_sync(FULL, ph == R(-1)) == FULL;

    // ---- shift the window
    p0 = p1; p1 = p2; p2 = ph;
    pl0 = pl1; pl1 = pl2; pl2 = __shfl_up_sync(FULL, ph, 1);
    pr0 = pr1; pr1 = pr2; pr2 = __shfl_down_sync(FULL, ph, 1);
    s0 = s1; s1 = s2; s2 = Sv;
    sl1 = sl2; sl2 = __shfl_up_sync(FULL, Sv, 1);
    sr0 = sr1; sr1 = sr2; sr2 = __shfl_down_sync(FULL, Sv, 1);
    m1 = m2; m2 = mu;
    d1 = d2; d2 = cv_s;
    sol0 = sol1; sol1 = sol2; sol2 = row_sol;
    liq0 = liq1; liq1 = liq2; liq2 = row_liq;
    R ku = R(0);
    if (TFC) {
      ku = (R)(ct.Kc - Kc2);
      Kc2 = ct.Kc;
      A1nb = A2nb; A1ti = A2ti; A2nb = ct.A_nb; A2ti = ct.A_ti;
      kr1 = kr2;
      kr2 = (R)(__shfl_down_sync(FULL, ct.Kc, 1) - ct.Kc);
    }
    if (k < 1) return;
    // flux through the face between rows row-1 and row (compute_c_CALPHAD
    // F01/F0m, fun.cu:1455-1459): weight (S00 + S01 + Shh + Snh)/4
    jv_lo = jv_hi;
    jv_hi = (R(1.5) * (s1 + s2) + R(0.25) * ((sr1 + sr2) + (sl1 + sl2))) * (m2 - m1 + ku);
    if (k < 2) return;

    // ---- output row r = row - 1
    const int r = row - 1;
    R psi_new = p1;
    // phi: exact shortcut when the three rows are all +1 or all -1
    if (!((sol0 && sol1 && sol2) || (liq0 && liq1 && liq2))) {
      R as, ak;
      const R an = anisotropy<R>(F, p1, pr1, pl1, p2, p0, pr2, pl2, pr0, pl0, as, ak);
      const R c00 = Tr<R>::kDelta ? cinf + d1 : d1;
      const R Anb = TFC ? A1nb : col.A_nb, Ati = TFC ? A1ti : col.A_ti;
      const R dG = (R(1) - c00) * Anb + c00 * Ati + c00 * (R(1) - c00) * R(kL0Liq - kL0Bcc);
      const R q = R(1) - p1 * p1;
      const R term = p1 - p1 * p1 * p1 + an + dG * (R(1.875) * (q * q)) * F.drive;
      R pn = p1 + Tr<R>::div(F.dt * ak, as * as) * term;
      if (F.noise_amp > R(0) && q > R(1.0e-3)) {
        uint32_t x[4];
        noise_counter(x, PS.step, (int64_t)r * K.nx + gi);
        philox4x32(x, K.seed_lo, K.seed_hi);
        pn += F.noise_amp * q * Tr<R>::normal(x);
      }
      psi_new = pn > R(1) ? R(1) : pn;  // renormalisation (fun.cu:1252-1261)
    }
    // c: flux through the face (i+1/2, r) (F10/Fm0), weight (S00+S10+Shh+Shn)/4
    const R mr = __shfl_down_sync(FULL, m1, 1);
    const R jh = (R(1.5) * (s1 + sr1) + R(0.25) * ((s2 + sr2) + (s0 + sr0))) * (mr - m1 + (TFC ? kr1 : dKr));
    const R jh_left = __shfl_up_sync(FULL, jh, 1);
    const R dc = F.cflux * ((jh - jh_left) + (jv_hi - jv_lo));
    const R dn = fmax(d1 + dc, Tr<R>::kDelta ? F.c_floor - cinf : F.c_floor);  // floor, fun.cu:1464

    // ---- stores (+ ghost copies, fun.cu:1220-1230)
    if (out_lane && r <= y_last) {
      const S vpsi = (S)psi_new;
      const S vc = (S)dn;
      const int pitch = K.pitch;
      const int64_t o = (int64_t)r * pitch + gi;
      psi_n[o] = vpsi;
      c_n[o] = vc;
      if (phi_n) phi_n[o] = (S)fmin(fmax(psi_new, R(-1)), R(1));
      if (gx2 >= 0) {
        const int64_t o2 = (int64_t)r * pitch + gx2;
        psi_n[o2] = vpsi;
        c_n[o2] = vc;
        if (phi_n) phi_n[o2] = (S)fmin(fmax(psi_new, R(-1)), R(1));
      }
      if (r == K.jmin || r == K.jmax) {
        const int gy2 = r == K.jmin ? 0 : K.ny - 1;
        const int64_t o3 = (int64_t)gy2 * pitch + gi;
        psi_n[o3] = vpsi;
        c_n[o3] = vc;
        if (phi_n) phi_n[o3] = (S)fmin(fmax(psi_new, R(-1)), R(1));
        if (gx2 >= 0) {
          const int64_t o4 = (int64_t)gy2 * pitch + gx2;
          psi_n[o4] = vpsi;
          c_n[o4] = vc;
          if (phi_n) phi_n[o4] = (S)fmin(fmax(psi_new, R(-1)), R(1));
        }
      }
      if (red) {
        mass += (double)vc;
        if (psi_new > R(0)) itip = max(itip, gi == K.nx - 2 ? K.nx - 1 : gi);
      }
    }
  }

  __device__ __forceinline__ void write_partial(BlockPartial *partials, int64_t slot) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mass += __shfl_down_sync(FULL, mass, o);
    itip = __reduce_max_sync(FULL, itip);
    if ((threadIdx.x & 31) == 0) {
      BlockPartial b;
      b.mass = mass;
      b.itip = itip;
      b.pad = 0;
      partials[slot] = b;
    }
  }
};

// Register-prefetch kernel: every lane loads its own column P rows ahead.
// Handles the pull-back remap, the coarse-grid temperature and any pitch.
template <typename R, int H, int P, bool TFC>
__global__ void __launch_bounds__(128, sizeof(R) == 4 ? 4 : 3)
    step_kernel(const StepCoef K, const Coef<R> F, const StepScalars PS, const typename Tr<R>::S *__restrict__ psi,
                const typename Tr<R>::S *__restrict__ cst, typename Tr<R>::S *__restrict__ psi_n,
                typename Tr<R>::S *__restrict__ c_n, typename Tr<R>::S *__restrict__ phi_n, BlockPartial *partials) {
  using S = typename Tr<R>::S;
  const int nx = K.nx, ny = K.ny, pitch = K.pitch;
  const int wc = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);  // warp column
  const int X = 1 + 30 * wc;                                            // first output column
  const int gi = X - 1 + (int)(threadIdx.x & 31);                       // this lane's column
  const int y0 = 1 + blockIdx.y * H;
  const int y_last = min(y0 + H - 1, ny - 2);
  const bool active_warp = X <= nx - 2;

  // source column of this lane (pull_back remap, fun.cu:1476-1487)
  int si = min(gi, nx - 1);
  bool fill = false;
  if (PS.pull_back) {
    si = min(max(si + PS.i_offset, 1), nx - 2);
    fill = si >= nx - 2;
  }
  S qp[P], qc[P];
  auto load_row = [&](int row, S &pv, S &cv) {
    const int rr = min(row, ny - 1);
    const int64_t o = (int64_t)rr * pitch + si;
    pv = psi[o];
    cv = fill ? (Tr<R>::kDelta ? S(0) : S(K.cinf)) : cst[o];
  };
#pragma unroll
  for (int s = 0; s < P; ++s) load_row(y0 - 1 + s, qp[s], qc[s]);

  Strip<R, TFC> st;
  st.init(K, PS, gi, y_last, active_warp);
  const int nrows = y_last - y0 + 3;  // rows y0-1 .. y_last+1
  if (active_warp) {
    for (int base = 0; base < nrows; base += P) {
#pragma unroll
      for (int s = 0; s < P; ++s) {
        const int k = base + s;
        if (k >= nrows) break;
        const int row = y0 - 1 + k;
        const R pv = (R)qp[s], cv = (R)qc[s];
        load_row(row + P, qp[s], qc[s]);
        st.step_row(K, F, PS, pv, cv, k, row, psi_n, c_n, phi_n, partials != nullptr);
      }
    }
  }
  if (partials)
    st.write_partial(partials, ((int64_t)blockIdx.y * gridDim.x + blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5));
}

// ---------------------------------------------------------------- TMA kernel
// phi update of one interface cell (compute_phi, fun.cu:1143-1218, with the
// renormalisation of compute_psi); only warps that see an interface row run it.
template <typename R>
__device__ __forceinline__ R phi_cell(const Coef<R> *__restrict__ Fp, R p00, R p10, R pm0, R p01, R p0m, R p11,
                                   R pm1, R p1m, R pmm, R c00, R Anb, R Ati, int64_t step, int64_t cell,
                                   uint32_t seed_lo, uint32_t seed_hi) {
  const Coef<R> &F = *Fp;
  R as, ak;
  const R an = anisotropy<R>(F, p00, p10, pm0, p01, p0m, p11, pm1, p1m, pmm, as, ak);
  const R dG = (R(1) - c00) * Anb + c00 * Ati + c00 * (R(1) - c00) * R(kL0Liq - kL0Bcc);
  const R q = R(1) - p00 * p00;
  const R term = p00 - p00 * p00 * p00 + an + dG * (R(1.875) * (q * q)) * F.drive;
  R pn = p00 + Tr<R>::div(F.dt * ak, as * as) * term;
  if (F.noise_amp > R(0) && q > R(1.0e-3)) {
    uint32_t x[4];
    noise_counter(x, step, cell);
    philox4x32(x, seed_lo, seed_hi);
    pn += F.noise_amp * q * Tr<R>::normal(x);
  }
  return pn > R(1) ? R(1) : pn;  // renormalisation (fun.cu:1252-1261)
}

// Per-lane state for two adjacent columns A = 2l, B = 2l+1 of a 64-column
// warp strip (62 output columns).  Same per-cell arithmetic as Strip.
template <typename R>
struct Strip2 {
  using S = typename Tr<R>::S;
  static constexpr unsigned FULL = 0xffffffffu;
  int giA, y_last;
  bool outA, outB;
  bool inA, inB;      // column inside the array (cells outside never block the bulk vote)
  bool ghA, ghB;      // column with a ghost copy (1 -> 0, nx-2 -> nx-1)
  ColT<R> colA, colB;
  R dKA, dKB;  // K(i+1) - K(i) for A (A->B face) and B (B->R face)
  R pA0, pA1, pA2, pB0, pB1, pB2, pL0, pL1, pL2, pR0, pR1, pR2;
  R sA0, sA1, sA2, sB0, sB1, sB2, sL1, sL2, sR0, sR1, sR2;
  R mA1, mA2, mB1, mB2;
  R dA1, dA2, dB1, dB2;
  R jvA_lo, jvA_hi, jvB_lo, jvB_hi;
  bool sol0, sol1, sol2, liq0, liq1, liq2;
  double mass;
  int itip;

  __device__ __forceinline__ void init(const StepCoef &K, const StepScalars &PS, int giA_, int y_last_) {
    const int lane = threadIdx.x & 31;
    giA = giA_;
    y_last = y_last_;
    outA = lane >= 1 && giA <= K.nx - 2;
    outB = lane <= 30 && giA + 1 <= K.nx - 2;
    inA = giA <= K.nx - 1;
    inB = giA + 1 <= K.nx - 1;
    ghA = giA == 1 || giA == K.nx - 2;
    ghB = giA + 1 == 1 || giA + 1 == K.nx - 2;
    pA0 = pA1 = pA2 = pB0 = pB1 = pB2 = pL0 = pL1 = pL2 = pR0 = pR1 = pR2 = R(0);
    sA0 = sA1 = sA2 = sB0 = sB1 = sB2 = sL1 = sL2 = sR0 = sR1 = sR2 = R(0);
    mA1 = mA2 = mB1 = mB2 = dA1 = dA2 = dB1 = dB2 = R(0);
    jvA_lo = jvA_hi = jvB_lo = jvB_hi = R(0);
    sol0 = sol1 = sol2 = liq0 = liq1 = liq2 = false;
    mass = 0.0;
    itip = 0;
    colA = col_terms<R>(K, (PS.d0 + PS.d1 * giA) * K.deltaT0 + K.Tmelt);
    colB = col_terms<R>(K, (PS.d0 + PS.d1 * (giA + 1)) * K.deltaT0 + K.Tmelt);
    dKA = (R)(colB.Kc - colA.Kc);
    dKB = (R)(__shfl_down_sync(FULL, colA.Kc, 1) - colB.Kc);
  }

  __device__ __forceinline__ R mu_of(const Coef<R> &F, const ColT<R> &ct, R pv, R cv_s, R &ph, R &Sv) const {
    const R cinf = F.cinf;
    const R d = Tr<R>::kDelta ? cv_s : cv_s - cinf;
    const R c = Tr<R>::kDelta ? cinf + cv_s : cv_s;
    const R omc = R(1) - c;
    ph = fmin(fmax(pv, R(-1)), R(1));
    const R a = R(1) - pv;
    Sv = (R(0.5) * F.AA * a - R(0.25) * (F.AA - R(1)) * (a * a)) * c * omc;
    const R p2v = pv * pv;
    const R g = pv * (R(1.875) + p2v * (R(-1.25) + R(0.375) * p2v));
    constexpr R L0sum = R(kL0Bcc + kL0Liq);
    constexpr R L0half = R(0.5 * (kL0Bcc - kL0Liq));
    return g * ct.D - d * L0sum + g * L0half * (R(1) - R(2) * c) + ct.RT * Tr<R>::lam(c, omc, d, cinf, F.Lref);
  }

  // ghost copies of a stored cell (compute_boundary_individual, fun.cu:1220-1230)
  __device__ __forceinline__ void ghosts(const StepCoef &K, S *__restrict__ psi_n, S *__restrict__ c_n,
                                         S *__restrict__ phi_n, int r, int gi, bool gh, bool grow, R psi_new,
                                         R dn) {
    const S vpsi = (S)psi_new;
    const S vc = (S)dn;
    const int pitch = K.pitch;
    const S vphi = (S)fmin(fmax(psi_new, R(-1)), R(1));
    const int gx2 = gi == 1 ? 0 : K.nx - 1;
    if (gh) {
      const int64_t o2 = (int64_t)r * pitch + gx2;
      psi_n[o2] = vpsi;
      c_n[o2] = vc;
      if (phi_n) phi_n[o2] = vphi;
    }
    if (grow) {
      const int gy2 = r == K.jmin ? 0 : K.ny - 1;
      const int64_t o3 = (int64_t)gy2 * pitch + gi;
      psi_n[o3] = vpsi;
      c_n[o3] = vc;
      if (phi_n) phi_n[o3] = vphi;
      if (gh) {
        const int64_t o4 = (int64_t)gy2 * pitch + gx2;
        psi_n[o4] = vpsi;
        c_n[o4] = vc;
        if (phi_n) phi_n[o4] = vphi;
      }
    }
  }

  __device__ __forceinline__ void step_row(const StepCoef &K, const Coef<R> *Fp, const StepScalars &PS, R pvA, R pvB,
                                           R cvA, R cvB, int k, int row, S *__restrict__ psi_n, S *__restrict__ c_n,
                                           S *__restrict__ phi_n, bool red) {
    const Coef<R> &F = *Fp;
    R phA, phB, SA, SB;
    const R muA = mu_of(F, colA, pvA, cvA, phA, SA);
    const R muB = mu_of(F, colB, pvB, cvB, phB, SB);
    const bool row_sol = __ballot_sync(FULL, (phA == R(1) || !inA) && (phB == R(1) || !inB)) == FULL;
    const bool row_liq = __ballot_sync(FULL, (phA == R(-1) || !inA) && (phB == R(-1) || !inB)) == FULL;
    // shift the window; the left neighbour of A is the previous lane's B,
    // the right neighbour of B the next lane's A
    pA0 = pA1; pA1 = pA2; pA2 = phA;
    pB0 = pB1; pB1 = pB2; pB2 = phB;
    pL0 = pL1; pL1 = pL2; pL2 = __shfl_up_sync(FULL, phB, 1);
    pR0 = pR1; pR1 = pR2; pR2 = __shfl_down_sync(FULL, phA, 1);
    sA0 = sA1; sA1 = sA2; sA2 = SA;
    sB0 = sB1; sB1 = sB2; sB2 = SB;
    sL1 = sL2; sL2 = __shfl_up_sync(FULL, SB, 1);
    sR0 = sR1; sR1 = sR2; sR2 = __shfl_down_sync(FULL, SA, 1);
    mA1 = mA2; mA2 = muA;
    mB1 = mB2; mB2 = muB;
    dA1 = dA2; dA2 = cvA;
    dB1 = dB2; dB2 = cvB;
    sol0 = sol1; sol1 = sol2; sol2 = row_sol;
    liq0 = liq1; liq1 = liq2; liq2 = row_liq;
    if (k < 1) return;
    // fluxes through the faces between rows row-1 and row (weights as Strip)
    jvA_lo = jvA_hi;
    jvA_hi = (R(1.5) * (sA1 + sA2) + R(0.25) * ((sB1 + sB2) + (sL1 + sL2))) * (mA2 - mA1);
    jvB_lo = jvB_hi;
    jvB_hi = (R(1.5) * (sB1 + sB2) + R(0.25) * ((sR1 + sR2) + (sA1 + sA2))) * (mB2 - mB1);
    if (k < 2) return;

    const int r = row - 1;
    R psiA = pA1, psiB = pB1;
    if (!((sol0 && sol1 && sol2) || (liq0 && liq1 && liq2))) {
      const int64_t cell = (int64_t)r * K.nx + giA;
      psiA = phi_cell<R>(Fp, pA1, pB1, pL1, pA2, pA0, pB2, pL2, pB0, pL0, Tr<R>::kDelta ? F.cinf + dA1 : dA1,
                         colA.A_nb, colA.A_ti, PS.step, cell, K.seed_lo, K.seed_hi);
      psiB = phi_cell<R>(Fp, pB1, pR1, pA1, pB2, pB0, pR2, pA2, pR0, pA0, Tr<R>::kDelta ? F.cinf + dB1 : dB1,
                         colB.A_nb, colB.A_ti, PS.step, cell + 1, K.seed_lo, K.seed_hi);
    }
    const R mR = __shfl_down_sync(FULL, mA1, 1);
    const R jhAB = (R(1.5) * (sA1 + sB1) + R(0.25) * ((sA2 + sB2) + (sA0 + sB0))) * (mB1 - mA1 + dKA);
    const R jhBR = (R(1.5) * (sB1 + sR1) + R(0.25) * ((sB2 + sR2) + (sB0 + sR0))) * (mR - mB1 + dKB);
    const R jhLA = __shfl_up_sync(FULL, jhBR, 1);
    const R floorv = Tr<R>::kDelta ? F.c_floor - F.cinf : F.c_floor;
    const R dnA = fmax(dA1 + F.cflux * ((jhAB - jhLA) + (jvA_hi - jvA_lo)), floorv);
    const R dnB = fmax(dB1 + F.cflux * ((jhBR - jhAB) + (jvB_hi - jvB_lo)), floorv);
    if (r <= y_last) {
      const int64_t o = (int64_t)r * K.pitch + giA;
      if (outA && outB) {
        // the pair is 8- (FP32) or 16-byte (FP64) aligned: one vector store
        using V = typename std::conditional<sizeof(S) == 4, float2, double2>::type;
        *reinterpret_cast<V *>(psi_n + o) = V{(S)psiA, (S)psiB};
        *reinterpret_cast<V *>(c_n + o) = V{(S)dnA, (S)dnB};
        if (phi_n)
          *reinterpret_cast<V *>(phi_n + o) = V{(S)fmin(fmax(psiA, R(-1)), R(1)), (S)fmin(fmax(psiB, R(-1)), R(1))};
      } else {
        if (outA) {
          psi_n[o] = (S)psiA;
          c_n[o] = (S)dnA;
          if (phi_n) phi_n[o] = (S)fmin(fmax(psiA, R(-1)), R(1));
        }
        if (outB) {
          psi_n[o + 1] = (S)psiB;
          c_n[o + 1] = (S)dnB;
          if (phi_n) phi_n[o + 1] = (S)fmin(fmax(psiB, R(-1)), R(1));
        }
      }
      const bool grow = r == K.jmin || r == K.jmax;
      if (outA && (ghA || grow)) ghosts(K, psi_n, c_n, phi_n, r, giA, ghA, grow, psiA, dnA);
      if (outB && (ghB || grow)) ghosts(K, psi_n, c_n, phi_n, r, giA + 1, ghB, grow, psiB, dnB);
      if (red) {
        if (outA) {
          mass += (double)(S)dnA;
          if (psiA > R(0)) itip = max(itip, giA == K.nx - 2 ? K.nx - 1 : giA);
        }
        if (outB) {
          mass += (double)(S)dnB;
          if (psiB > R(0)) itip = max(itip, giA + 1 == K.nx - 2 ? K.nx - 1 : giA + 1);
        }
      }
    }
  }

  __device__ __forceinline__ void write_partial(BlockPartial *partials, int64_t slot) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mass += __shfl_down_sync(FULL, mass, o);
    itip = __reduce_max_sync(FULL, itip);
    if ((threadIdx.x & 31) == 0) {
      BlockPartial b;
      b.mass = mass;
      b.itip = itip;
      b.pad = 0;
      partials[slot] = b;
    }
  }
};

// A CTA of four warps covers 4 x 62 = 248 output columns; its 250-column
// input window (start 16-byte aligned) is brought into shared memory by TMA
// in tiles of kTmaRT rows through a ring of stages, so many row tiles are in
// flight per SM without holding them in registers.  One elected thread issues
// the copies; completion is tracked by an mbarrier per stage.  Waits are
// bounded: a wait that gives up sets *err and the kernel finishes without
// hanging (the host reports RS_E_STATE).  blockIdx.x runs along the strip
// (j) and blockIdx.y along the columns (i), so the CTAs holding the front and
// the solid behind it (low i, where the moving frame keeps the interface) are
// scheduled first.
constexpr int kTmaOut = 248;
constexpr int kTmaRT = kTmaBoxH;
constexpr uint32_t kWaitLimit = 1u << 20;
template <typename R>
struct TmaCfg {
  static constexpr int W = sizeof(R) == 4 ? kTmaBoxW32 : kTmaBoxW64;
  static constexpr int NS = sizeof(R) == 4 ? 4 : 3;
  static constexpr int TILE = ((kTmaRT * W * (int)sizeof(R) + 127) / 128) * 128 / (int)sizeof(R);
  static constexpr size_t smem = (size_t)NS * 2 * TILE * sizeof(R) + NS * sizeof(uint64_t);
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

template <typename R, int H>
__global__ void __launch_bounds__(128, sizeof(R) == 4 ? 4 : 3)
    step_tma_kernel(const __grid_constant__ StepCoef K, const __grid_constant__ Coef<R> F,
                    const __grid_constant__ StepScalars PS, const __grid_constant__ CUtensorMap tm_psi,
                    const __grid_constant__ CUtensorMap tm_c, typename Tr<R>::S *__restrict__ psi_n,
                    typename Tr<R>::S *__restrict__ c_n, typename Tr<R>::S *__restrict__ phi_n,
                    BlockPartial *partials, int *err) {
  using S = typename Tr<R>::S;
  using Cfg = TmaCfg<R>;
  constexpr int W = Cfg::W, NS = Cfg::NS, TILE = Cfg::TILE;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  S *tiles = reinterpret_cast<S *>(smem_raw);  // [stage][field][row][col]
  uint64_t *full = reinterpret_cast<uint64_t *>(smem_raw + (size_t)NS * 2 * TILE * sizeof(S));

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int xw = kTmaOut * blockIdx.y;      // first input column (16-byte aligned)
  const int col = 62 * warp + 2 * lane;      // smem column of this lane's A cell
  const int y0 = 1 + blockIdx.x * H;
  const int y_last = min(y0 + H - 1, K.ny - 2);
  const int nrows = y_last - y0 + 3;         // rows y0-1 .. y_last+1
  const int ntiles = (nrows + kTmaRT - 1) / kTmaRT;
  constexpr uint32_t kStageBytes = 2u * kTmaRT * W * sizeof(S);  // bytes the two boxes deliver

  // self-check: TMA destinations must be 128-byte aligned
  if (smem_u32(tiles) & 127u) {
    if (threadIdx.x == 0) atomicExch(err, 2);
    return;
  }
  if (threadIdx.x == 0) {
#pragma unroll
    for (int s = 0; s < NS; ++s) mbar_init(&full[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int t = 0; t < NS && t < ntiles; ++t) {
      mbar_expect_tx(&full[t], kStageBytes);
      tma_load_2d(tiles + (2 * t) * TILE, &tm_psi, &full[t], xw, y0 - 1 + t * kTmaRT);
      tma_load_2d(tiles + (2 * t + 1) * TILE, &tm_c, &full[t], xw, y0 - 1 + t * kTmaRT);
    }
  }

  Strip2<R> st;
  st.init(K, PS, xw + col, y_last);
  const bool red = partials != nullptr;
  using V = typename std::conditional<sizeof(S) == 4, float2, double2>::type;
  for (int t = 0; t < ntiles; ++t) {
    const int s = t % NS;
    const uint32_t parity = (uint32_t)(t / NS) & 1u;
    uint32_t tries = 0;
    while (!mbar_try_wait(&full[s], parity)) {
      if (++tries >= kWaitLimit) {
        atomicExch(err, 1);
        break;
      }
    }
    const S *tp = tiles + (2 * s) * TILE + col;
    const S *tc = tiles + (2 * s + 1) * TILE + col;
#pragma unroll 1
    for (int rr = 0; rr < kTmaRT; ++rr) {
      const int k = t * kTmaRT + rr;
      if (k >= nrows) break;
      const V pv = *reinterpret_cast<const V *>(tp + rr * W);
      const V cv = *reinterpret_cast<const V *>(tc + rr * W);
      st.step_row(K, &F, PS, (R)pv.x, (R)pv.y, (R)cv.x, (R)cv.y, k, y0 - 1 + k, psi_n, c_n, phi_n, red);
    }
    __syncthreads();  // stage s is free
    if (threadIdx.x == 0 && t + NS < ntiles) {
      mbar_expect_tx(&full[s], kStageBytes);
      tma_load_2d(tiles + (2 * s) * TILE, &tm_psi, &full[s], xw, y0 - 1 + (t + NS) * kTmaRT);
      tma_load_2d(tiles + (2 * s + 1) * TILE, &tm_c, &full[s], xw, y0 - 1 + (t + NS) * kTmaRT);
    }
  }
  if (partials) st.write_partial(partials, ((int64_t)blockIdx.y * gridDim.x + blockIdx.x) * 4 + warp);
}

template <typename R>
static int launch(const StepCoef &K, const StepScalars &P, const typename Tr<R>::S *psi, const typename Tr<R>::S *c,
                  typename Tr<R>::S *psi_n, typename Tr<R>::S *c_n, typename Tr<R>::S *phi_n, BlockPartial *partials,
                  int max_partials, int *nwarps_out, const TmaMaps *tm, int *err, cudaStream_t st) {
  const Coef<R> F = make_coef<R>(K);
  const int ni = K.nx - 2, nj = K.ny - 2;
  const bool tfc = K.tfc != 0;
  if (tm && !tfc && !P.pull_back && sizeof(R) == 4) {
    // TMA pipeline: CTAs of 248 output columns x H rows, column-major order
    const int cx = (ni + kTmaOut - 1) / kTmaOut;
    // short strips: a warp that crosses the interface does the anisotropic
    // update on every row of its strip, so strips are kept short
    int H = 16;
    dim3 grid((nj + H - 1) / H, cx), block(128);
    const int nw = grid.x * grid.y * 4;
    if (partials && nw > max_partials) return -1;
    const size_t smem = TmaCfg<R>::smem;
    static bool attr_done[4] = {false, false, false, false};
    const int hidx = H == 64 ? 0 : (H == 32 ? 1 : (H == 16 ? 2 : 3));
    auto kfn = H == 64 ? step_tma_kernel<R, 64>
                       : (H == 32 ? step_tma_kernel<R, 32> : (H == 16 ? step_tma_kernel<R, 16> : step_tma_kernel<R, 8>));
    if (!attr_done[hidx]) {
      if (cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return -3;
      attr_done[hidx] = true;
    }
    kfn<<<grid, block, smem, st>>>(K, F, P, tm->psi, tm->c, psi_n, c_n, phi_n, partials, err);
    if (nwarps_out) *nwarps_out = nw;
    return 0;
  }
  const int wcols = (ni + 29) / 30;
  constexpr int WPB = 4;  // warps per block (adjacent column strips)
  constexpr int PF = 3;   // rows in flight per lane (multiple of the 3-row window)
  int H = 64;
  while (H > 16 && (int64_t)wcols * ((nj + H - 1) / H) < 148 * 16) H /= 2;
  dim3 block(32 * WPB), grid((wcols + WPB - 1) / WPB, (nj + H - 1) / H);
  const int nw = grid.x * grid.y * WPB;
  if (partials && nw > max_partials) return -1;
#define RS_LAUNCH(HH)                                                                                   \
  if (tfc)                                                                                              \
    step_kernel<R, HH, PF, true><<<grid, block, 0, st>>>(K, F, P, psi, c, psi_n, c_n, phi_n, partials); \
  else                                                                                                  \
    step_kernel<R, HH, PF, false><<<grid, block, 0, st>>>(K, F, P, psi, c, psi_n, c_n, phi_n, partials);
  if (H == 64) {
    RS_LAUNCH(64)
  } else if (H == 32) {
    RS_LAUNCH(32)
  } else {
    RS_LAUNCH(16)
  }
#undef RS_LAUNCH
  if (nwarps_out) *nwarps_out = nw;
  return 0;
}

int launch_step_f64(const StepCoef &K, const StepScalars &P, const double *psi, const double *c, double *psi_n,
                    double *c_n, double *phi_n, BlockPartial *partials, int max_partials, int *nb, const TmaMaps *tm,
                    int *err, cudaStream_t st) {
  return launch<double>(K, P, psi, c, psi_n, c_n, phi_n, partials, max_partials, nb, tm, err, st);
}

int launch_step_f32(const StepCoef &K, const StepScalars &P, const float *psi, const float *c, float *psi_n,
                    float *c_n, float *phi_n, BlockPartial *partials, int max_partials, int *nb, const TmaMaps *tm,
                    int *err, cudaStream_t st) {
  if (K.tfc) return -2;
  return launch<float>(K, P, psi, c, psi_n, c_n, phi_n, partials, max_partials, nb, tm, err, st);
}

}  // namespace rs

// rs_step_common.cuh — per-cell arithmetic shared by the step kernels:
// working-precision traits, kernel constants, the anisotropic operator, the
// CALPHAD column groups, the interface phi update and the TMA/mbarrier
// primitives.  The mathematics is stated in rs_step.cu.
#pragma once

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
  // far-melt form of the solute log term lam = log(c/(1-c)) -
  // log(cinf/(1-cinf)): its Taylor polynomial in delta = c - cinf,
  //   lam = sum_k a_k delta^k,  a_k = ((-1)^(k-1) / cinf^k + 1 / (1-cinf)^k) / k,
  // melt_a[k-1] = a_k, used where |delta| <= melt_tiny.  With m = min(cinf,
  // 1-cinf), |a_k| <= 2 / (k m^k): FP64 takes 6 terms for |delta| <= 1e-3 m
  // (the rest below 3e-19 of lam), FP32 4 terms for |delta| <= 1e-2 m (below
  // 4e-9); the polynomial is the function to the working precision's
  // rounding, with no division.  Far from the front the melt sits within
  // these bounds of cinf: the solute boundary layer ahead of the front decays
  // exponentially.
  R melt_a[6];
  R melt_tiny;
  // delta range of the bulk-melt series form: s = delta / (A + B delta), A =
  // 2 cinf (1 - cinf), B = 1 - 2 cinf, so |s| < 1/9 for -A/(9+B) < delta <
  // A/(9-B) (taken 0.1 % inside), evaluated in the working precision
  R ser_lo, ser_hi;
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
  {
    const bool dbl = sizeof(R) == sizeof(double);
    const int nt = dbl ? 6 : 4;
    double pc = 1.0, pm = 1.0;
    for (int k = 1; k <= 6; ++k) {
      pc /= K.cinf;
      pm /= 1.0 - K.cinf;
      F.melt_a[k - 1] = k <= nt ? (R)(((k % 2 ? pc : -pc) + pm) / k) : (R)0;
    }
    F.melt_tiny = (R)((dbl ? 1e-3 : 1e-2) * (K.cinf < 0.5 ? K.cinf : 1.0 - K.cinf));
    const R ci = (R)K.cinf, sA = (R)2 * ci * ((R)1 - ci), sB = (R)1 - (R)2 * ci;
    F.ser_hi = (R)0.999 * sA / ((R)9 - sB);
    F.ser_lo = -(R)0.999 * sA / ((R)9 + sB);
  }
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

// TFC (the coarse-grid temperature, fun.cu:1580-1608): every cell has its own
// temperature, bilinear from the coarse grid, so the column table entries of
// the tile kernels become per-cell CALPHAD groups, and K + C0 varies along
// both axes: the FP64 tile kernel stores mu = mu'' + (K + C0) of the cell, the
// FP32 one keeps K + C0 in FP64 beside mu'' and adds its face differences.
struct CellGroups {
  double RT, C0, KC;  // RT, C0 and K + C0 at the cell's temperature
  double Anb, Ati;    // the driving-force groups
};
// the CALPHAD groups at temperature T (lT = log T).  K + C0 = G_Ti_Liq -
// G_Nb_Liq + L0_Liq (1 - 2 cinf) + RT Lref needs the liquid functions only,
// which is all the melt rows use; full adds C0 and the driving-force groups
// (the solid functions).  Every caller takes K + C0 from this one expression,
// so a cell's value does not depend on which row form or tile evaluates it.
__device__ __forceinline__ CellGroups groups_at(const StepCoef &K, double T, double lT, bool full) {
  const double tl = g_ti_liq(T, lT), nl = g_nb_liq(T, lT);
  CellGroups g;
  g.RT = K.RR * T;
  g.KC = (tl - nl) + kL0Liq * (1.0 - 2.0 * K.cinf) + g.RT * K.Lref;
  g.C0 = g.Anb = g.Ati = 0.0;
  if (full) {
    const double tb = g_ti_bcc(T, lT), nb = g_nb_bcc(T, lT);
    g.C0 = -0.5 * ((tb - nb) - (tl - nl)) - 0.5 * (kL0Bcc - kL0Liq) * (1.0 - 2.0 * K.cinf);
    g.Anb = nl - nb;
    g.Ati = tl - tb;
  }
  return g;
}
// log T near a reference T0: log T0 + log1p(u), u = (T - T0)/T0, by
// the Taylor series of log1p to u^8 where |u| <= 2^-6 (the remainder, below
// |u|^9/9 < 7e-18, is under 1 % of an ulp of log T), else log itself.  The
// tile kernels take T0 per lane: over its cells T changes by far less than
// 1.5 %.
struct LogRef {
  double T0, lT0, iT0;  // T0, log T0, 1 / T0
};
__device__ __forceinline__ LogRef log_ref(double T0) { return LogRef{T0, log(T0), 1.0 / T0}; }
__device__ __forceinline__ double log_near(const LogRef &L, double T) {
  const double u = (T - L.T0) * L.iT0;
  if (fabs(u) > 0.015625) return log(T);
  double p = -1.0 / 8.0;
  p = fma(p, u, 1.0 / 7.0);
  p = fma(p, u, -1.0 / 6.0);
  p = fma(p, u, 1.0 / 5.0);
  p = fma(p, u, -1.0 / 4.0);
  p = fma(p, u, 1.0 / 3.0);
  p = fma(p, u, -1.0 / 2.0);
  p = fma(p, u, 1.0);
  return fma(p, u, L.lT0);
}
// K + C0 near a tile's reference temperature T0 as its Taylor polynomial in
// T - T0 (degree 6).  For T in [1941, 2750) K, G_Ti_Liq - G_Nb_Liq is one SGTE
// expression a + bT + cT lnT + dT^2 + eT^3 + f/T + hT^7 (the coefficients of
// g_ti_liq's upper and g_nb_liq's lower piece, fun.cu:1628-1669), whose
// derivatives are closed forms; the remainder after degree 6 is below
// |KC^(7)| |T - T0|^7 / 7! < 2e-16 J/mol for |T - T0| <= 4 K.  The constant
// term is the cell form itself (groups_at) at T0.  Cells farther than 4 K from
// T0, or all cells when T0 is not in [1945, 2746) K (so that the cells within
// 4 K of it stay in [1941, 2750) K), take groups_at.
struct KcPoly {
  LogRef lr;     // T0, log T0, 1 / T0 (also log_near's reference)
  double c[7];   // KC^(k)(T0) / k!
  int ok;        // T0 in [1945, 2746)
};
__device__ __forceinline__ KcPoly kc_poly(const StepCoef &K, double T0) {
  KcPoly P;
  P.lr = log_ref(T0);
  P.ok = T0 >= 1945.0 && T0 < 2746.0;
  constexpr double c = -46.29 + 26.4711, d = -0.203475e-3, e = 0.35012e-6, f = -93399.0, h = 306.098e-25;
  const double b = (298.7367 - 131.229057) + K.RR * K.Lref;
  const double T = T0, lT = P.lr.lT0, i1 = P.lr.iT0;
  const double i2 = i1 * i1, i3 = i2 * i1, i4 = i2 * i2, i5 = i4 * i1, i6 = i3 * i3, i7 = i6 * i1;
  const double T2 = T * T, T3 = T2 * T, T4 = T2 * T2, T5 = T4 * T, T6 = T3 * T3;
  P.c[0] = groups_at(K, T, lT, false).KC;
  P.c[1] = b + c * (lT + 1.0) + 2.0 * d * T + 3.0 * e * T2 - f * i2 + 7.0 * h * T6;
  P.c[2] = (c * i1 + 2.0 * d + 6.0 * e * T + 2.0 * f * i3 + 42.0 * h * T5) / 2.0;
  P.c[3] = (-c * i2 + 6.0 * e - 6.0 * f * i4 + 210.0 * h * T4) / 6.0;
  P.c[4] = (2.0 * c * i3 + 24.0 * f * i5 + 840.0 * h * T3) / 24.0;
  P.c[5] = (-6.0 * c * i4 - 120.0 * f * i6 + 2520.0 * h * T2) / 120.0;
  P.c[6] = (24.0 * c * i5 + 720.0 * f * i7 + 5040.0 * h * T) / 720.0;
  return P;
}
// K + C0 at T from P, or false where the polynomial does not apply
__device__ __forceinline__ bool kc_eval(const KcPoly &P, double T, double &kc) {
  const double u = T - P.lr.T0;
  if (!(P.ok && fabs(u) <= 4.0)) return false;
  double r = P.c[6];
#pragma unroll
  for (int k = 5; k >= 0; --k) r = fma(r, u, P.c[k]);
  kc = r;
  return true;
}
// the cell form of the groups, out of line: the general rows and the cells
// the polynomial does not cover are few, and one copy of the code keeps the
// tile kernels' instruction footprint small
static __device__ __noinline__ CellGroups groups_cell(const StepCoef &K, const LogRef &L, double T, bool full) {
  return groups_at(K, T, log_near(L, T), full);
}
// every group of a cell, the logarithm exact (interface cells), out of line
static __device__ __noinline__ CellGroups groups_exact(const StepCoef &K, double T) {
  return groups_at(K, T, log(T), true);
}
// the groups a cell needs: RT and K + C0 always, C0 where full (the general
// row form; the melt forms multiply C0 by g + 1 = 0)
__device__ __forceinline__ void cell_tfc(const StepCoef &K, const KcPoly &P, double T, bool full, double &RT,
                                         double &C0, double &KC) {
  RT = K.RR * T;
  C0 = 0.0;
  const bool poly = kc_eval(P, T, KC);
  if (!poly || full) {
    const CellGroups g = groups_cell(K, P.lr, T, full);
    C0 = g.C0;
    if (!poly) KC = g.KC;
  }
}
// interpolate_temperature's coordinates (fun.cu:1588-1594), split into the
// column part (fixed per lane) and the row part (one per row): the same
// expressions as t_fine_at, so the same temperature
__device__ __forceinline__ void tfc_col(const StepCoef &K, int ile, int i, int &iT, double &x) {
  i = min(max(i, 0), K.nx - 1);
  iT = (i - 1 + ile) / K.ratio;
  x = (i - 1.0 + ile) / K.ratio - iT;
  iT = min(max(iT, 0), K.NxT_all - 2);
}
__device__ __forceinline__ void tfc_row(const StepCoef &K, int j, int &jT, double &y) {
  j = min(j, K.ny - 1);
  jT = (int)((j - 1 + K.dxT) / K.ratio);
  y = (j - 1.0 + K.dxT) / K.ratio - jT;
  jT = min(max(jT, 0), K.NyT_all - 2);
}
__device__ __forceinline__ double tfc_T(const StepCoef &K, const double *__restrict__ T, int iT, double x, int jT,
                                        double y) {
  const double *r0 = T + (int64_t)jT * K.NxT_all + iT, *r1 = r0 + K.NxT_all;
  const double f00 = r0[0], f10 = r0[1], f01 = r1[0], f11 = r1[1];
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

// phi update of one interface cell (compute_phi, fun.cu:1143-1218, with the
// renormalisation of compute_psi); only warps that see an interface row run it.
// with the driving force dG = Gl - Gs of the cell given
template <typename R>
__device__ __forceinline__ R phi_cell_dG(const Coef<R> *__restrict__ Fp, R p00, R p10, R pm0, R p01, R p0m, R p11,
                                      R pm1, R p1m, R pmm, R dG, int64_t step, int64_t cell, uint32_t seed_lo,
                                      uint32_t seed_hi) {
  const Coef<R> &F = *Fp;
  R as, ak;
  const R an = anisotropy<R>(F, p00, p10, pm0, p01, p0m, p11, pm1, p1m, pmm, as, ak);
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

template <typename R>
__device__ __forceinline__ R phi_cell(const Coef<R> *__restrict__ Fp, R p00, R p10, R pm0, R p01, R p0m, R p11,
                                   R pm1, R p1m, R pmm, R c00, R Anb, R Ati, int64_t step, int64_t cell,
                                   uint32_t seed_lo, uint32_t seed_hi) {
  const R dG = (R(1) - c00) * Anb + c00 * Ati + c00 * (R(1) - c00) * R(kL0Liq - kL0Bcc);
  return phi_cell_dG<R>(Fp, p00, p10, pm0, p01, p0m, p11, pm1, p1m, pmm, dG, step, cell, seed_lo, seed_hi);
}

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
// non-blocking: whether the phase has completed now (try_wait may suspend the
// thread for a while first; a wait bounded by a count of test_wait polls
// gives up after that many polls, which the tests use to reach the give-up
// path)
__device__ __forceinline__ bool mbar_test_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// one try of a bounded wait: the suspending try_wait, or (test limit set) a
// non-blocking poll
__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity, bool poll) {
  return poll ? mbar_test_wait(bar, parity) : mbar_try_wait(bar, parity);
}
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void mbar_inval(uint64_t *bar) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Grid-wide barrier of a cooperative launch (every CTA resident): each CTA
// adds 1 to *bar (cleared before the launch) and waits until it reaches
// target, the barrier's ordinal times gridDim.x.  Thread 0 releases the CTA's
// prior writes (including completed bulk async stores) before it arrives and,
// once through, orders them before the CTA's later TMA loads (proxy fence).
// The wait is bounded: after `limit` polls it sets *err = 3 and the CTA's
// threads all get false.
__device__ __forceinline__ bool grid_barrier(unsigned *bar, unsigned target, int *err, uint32_t limit) {
  __syncthreads();
  int ok = 1;
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(bar, 1u);
    uint32_t tries = 0;
    while (true) {
      unsigned v;
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(bar) : "memory");
      if (v >= target) break;
      if (++tries >= limit) {
        atomicExch(err, 3);
        ok = 0;
        break;
      }
      __nanosleep(64);
    }
    asm volatile("fence.proxy.async.global;" ::: "memory");
  }
  return __syncthreads_and(ok) != 0;
}

// L2 prefetch of the box a tma_load_2d at (x, y) would copy (no shared memory,
// no barrier; the same 16-byte alignment of x as the load)
__device__ __forceinline__ void tma_prefetch_2d(const CUtensorMap *map, int x, int y) {
  asm volatile("cp.async.bulk.prefetch.tensor.2d.L2.global.tile [%0, {%1, %2}];" ::"l"(map), "r"(x), "r"(y)
               : "memory");
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::
          "r"(smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}


}  // namespace rs

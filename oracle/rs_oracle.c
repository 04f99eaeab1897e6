/*
 * rs_oracle.c — CPU FP64 restatement of the reference's coupled phase-field
 * step (TEST INFRASTRUCTURE ONLY; see rs_oracle.h).
 *
 * Reference files: fun.cu (kernels, CALPHAD, tip tracker), src/constants.hpp
 * (parameter set), src/main.cu (loop shape).  Expressions keep the reference's
 * operation order so that the oracle and the reference's own kernels agree to
 * the last few ulps; build with -ffp-contract=off.
 */
#include "rs_oracle.h"

#include <math.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define POW2(x) ((x) * (x))
#define POW3(x) (POW2(x) * (x))
#define POW4(x) (POW2(POW2(x)))
#define POW5(x) (POW2(POW2(x)) * (x))
#define POW7(x) (POW2(POW2(x)) * POW2(x) * (x))
#define POW9(x) (POW3(POW3(x)))

/* PI as the reference writes it (fun.cu:59) */
#define REF_PI 3.1415927

static inline int64_t pos(const rs_params *p, int i, int j) {
  return (int64_t)j * p->nx_all + i;
}

/* ------------------------------------------------------------------ params */
/* src/constants.hpp:185-350 (Material, Simulation namespaces) */
void ro_default_params(rs_params *p) {
  memset(p, 0, sizeof(*p));
  p->nx_all = 768;  /* constants.hpp:254 */
  p->ny_all = 832;  /* constants.hpp:255 */
  p->i_tip_target = 768 - 268; /* constants.hpp:272 */
  p->periodic_j = 1;           /* boundaryCondition 0 */
  p->tfc = 1;                  /* main.cu:17 ifTFC 1 */
  p->one_eps = 1;              /* if_1_eps true */
  p->vp_ramp = 0;              /* if_Vp_ramp false */
  p->n_orientation = 1;
  p->cinf = 0.632514105;
  p->W0 = 0.25;
  p->S = 5.0;
  p->Gamma = 199.0;
  p->muk0 = 0.57;
  p->Tmelt = 2161.59;
  p->T_ref = 2118.35;
  p->Dl = 2.05;
  p->DT = 1.1e4;
  p->latent_heat = 22003.0;
  p->molar_weight = 64.418;
  p->num_moles = 93353.43470588748;
  p->cp = 40.0;
  p->RR = 8.3145;
  p->v0 = 1.17e-5;
  p->AA = 12.0; /* SS == 5 */
  p->ke = 0.8146631243899296;
  p->dx = 0.6;  /* SS == 5 */
  p->dt = 0.0;  /* set_parameters rule */
  p->GG = 10 * 0.001;
  p->Vp = 1.0;
  p->eps1 = 0.06;
  p->eps2 = 0.0;
  p->epk1 = 0.15;
  p->delta_initial = -1.0;
  p->l_offset_Vp_initial = 0.0;
  p->i_offset_history_initial = 0;
  p->ratio_dxT_dx = 10;
  /* set_orientation(alpha0=beta0=gamma0=0) -> identity */
  p->orientation[0] = 1.0; p->orientation[4] = 1.0; p->orientation[8] = 1.0;
  p->noise_amplitude = 0.0;
  p->seed = 0;
  p->Tcold = 2000.0;
  p->length_sample_um = 50.0;
  p->total_time_ns = 120.0 * 1000.0;
  p->num_fields_output = 120;
  p->num_tip_output = 120;
  p->num_check_point_output = 120;
  p->step_pull_back = 0;
}

/* set_parameters, fun.cu:1984-2058; dimensional groups from the macro block
 * fun.cu:57-112 */
void ro_derive(const rs_params *p, rs_derived *d) {
  memset(d, 0, sizeof(*d));
  const double SS = p->S;
  d->W = SS * p->W0;
  d->tau0 = POW2(SS * p->W0) / (p->Gamma * p->muk0);
  d->deltaT0 = p->Tmelt - p->T_ref;
  d->a1 = 2.0 * sqrt(2.0) / 3.0;
  const double latentHeat2 = p->latent_heat * p->num_moles;
  const double surface_tension = p->Gamma * 1e-9 * latentHeat2 / p->Tmelt;
  d->hh = surface_tension / (d->a1 * SS * p->W0 * 1.0e-9);
  d->h0 = p->RR * p->Tmelt / p->v0;

  const double DD = p->Dl * d->tau0 / POW2(SS * p->W0);
  double dt;
  if (p->dt > 0) {
    dt = p->dt;
  } else {
    dt = 0.6 * p->dx * p->dx / (4.0 * DD);
    if (dt > 0.6 * p->dx * p->dx / 4.0) dt = 0.6 * p->dx * p->dx / 4.0;
  }
  d->dt = dt;
  const double tau0 = d->tau0;
  d->total_step = (int64_t)(p->total_time_ns / (tau0 * dt));
  d->step_fields = (int32_t)(p->total_time_ns / p->num_fields_output / (tau0 * dt));
  d->step_tip = (int32_t)(p->total_time_ns / p->num_tip_output / (tau0 * dt));
  d->step_check_point = (int32_t)(p->total_time_ns / p->num_check_point_output / (tau0 * dt));
  if (p->step_pull_back > 0) {
    d->step_pull_back = p->step_pull_back;
  } else if (p->vp_ramp) {
    d->step_pull_back = (int32_t)(SS * p->W0 * p->dx / (1.0 * dt * tau0));
  } else {
    d->step_pull_back = (int32_t)(SS * p->W0 * p->dx / (p->Vp * dt * tau0));
  }

  /* TFC block, fun.cu:2025-2057 */
  const int r = p->ratio_dxT_dx;
  const double DDT = p->DT * tau0 / POW2(SS * p->W0 * r);
  const double dtT = 0.9 * p->dx * p->dx / (4.0 * DDT);
  int ratio = 1;
  if (dtT < dt) ratio = (int)ceil(dt / dtT);
  d->ratio_dt_dtT = ratio;
  d->dtT = dt / ratio;
  const double length = p->length_sample_um;
  d->length_sample = ceil(length * 1000 / (p->dx * SS * p->W0 * r)) * (p->dx * SS * p->W0 * r);
  d->NxT = (int32_t)(d->length_sample / (p->dx * SS * p->W0 * r) + 2);
  d->NxT_all = (int32_t)(ceil(1.0 * d->NxT / 64) * 64);
  d->NyT = ((p->ny_all - 2) / r) + 2;
  d->NyT_all = (int32_t)(ceil(1.0 * d->NyT / 4) * 4);
  d->Thot = p->Tcold + p->GG * d->length_sample;
  d->i_left_end_initial = (int32_t)((p->Tmelt - d->deltaT0 - p->Tcold) /
                                        (p->GG * p->dx * SS * p->W0) -
                                    p->i_tip_target);
}

/* ------------------------------------------------------------------ CALPHAD */
/* fun.cu:1628-1637 */
double ro_G_Ti_BCC(double T) {
  if (T >= 1155.0 && T < 1941.0)
    return 6667.385 + 105.366379 * T - 22.3771 * T * log(T) + 1.21707e-3 * POW2(T) -
           0.84534e-6 * POW3(T) - 2002750.0 / T;
  else if (T >= 1941.0)
    return 26483.26 - 182.426471 * T + 19.0900905 * T * log(T) - 22.00832e-3 * POW2(T) +
           1.228863e-6 * POW3(T) + 1400501.0 / T;
  return NAN;
}
/* fun.cu:1639-1647 */
double ro_G_Ti_Liq(double T) {
  if (T >= 1300.0 && T < 1941.0)
    return 369519.198 - 2554.0225 * T + 342.059267 * T * log(T) - 163.409355e-3 * POW2(T) +
           12.457117e-6 * POW3(T) - 67034516.0 / T;
  else if (T >= 1941.0 && T < 4000.0)
    return -19887.066 + 298.7367 * T - 46.29 * T * log(T);
  return NAN;
}
/* fun.cu:1649-1656 */
double ro_G_Nb_BCC(double T) {
  if (T >= 298.15 && T < 2750.0)
    return -8519.353 + 142.045475 * T - 26.4711 * T * log(T) + 0.203475e-3 * POW2(T) -
           0.35012e-6 * POW3(T) + 93399.0 / T;
  else if (T >= 2750.0)
    return -37669.3 + 271.720843 * T - 41.77 * T * log(T) + 1528.238e29 / POW9(T);
  return NAN;
}
/* fun.cu:1658-1666 */
double ro_G_Nb_Liq(double T) {
  if (T >= 298.15 && T < 2750.0)
    return 21262.202 + 131.229057 * T - 26.4711 * T * log(T) + 0.203475e-3 * POW2(T) -
           0.35012e-6 * POW3(T) + 93399.0 / T - 306.098e-25 * POW7(T);
  else if (T >= 2750.0)
    return -7499.398 + 260.756148 * T - 41.77 * T * log(T);
  return NAN;
}

#define L0_BCC 12315.25 /* fun.cu:1668 */
#define L0_LIQ 5144.29  /* fun.cu:1669 */

/* fun.cu:1671-1684 */
double ro_Gl(const rs_params *p, double T, double c) {
  const double RR = p->RR;
  double onemc = 1.0 - c;
  double log_part;
  if (c < 1.e-8)
    log_part = RR * T * (onemc * log(onemc));
  else if (onemc < 1.e-8)
    log_part = RR * T * (c * log(c));
  else
    log_part = RR * T * (onemc * log(onemc) + c * log(c));
  double mix_part = c * onemc * L0_LIQ;
  return log_part + onemc * ro_G_Nb_Liq(T) + c * ro_G_Ti_Liq(T) + mix_part;
}
/* fun.cu:1686-1698 */
double ro_Gs(const rs_params *p, double T, double c) {
  const double RR = p->RR;
  double onemc = 1.0 - c;
  double log_part;
  if (c < 1.e-8)
    log_part = RR * T * (onemc * log(onemc));
  else if (onemc < 1.e-8)
    log_part = RR * T * (c * log(c));
  else
    log_part = RR * T * (onemc * log(onemc) + c * log(c));
  double mix_part = c * onemc * L0_BCC;
  return log_part + onemc * ro_G_Nb_BCC(T) + c * ro_G_Ti_BCC(T) + mix_part;
}
/* fun.cu:1700-1709 */
double ro_Glc(const rs_params *p, double T, double c) {
  double termL0 = L0_LIQ * (1.0 - 2.0 * c);
  double onemc = 1.0 - c;
  double log_part = 0.;
  if (c > 1.e-8 && onemc > 1.e-8) log_part = p->RR * T * log(c / onemc);
  return ro_G_Ti_Liq(T) - ro_G_Nb_Liq(T) + termL0 + log_part;
}
/* fun.cu:1711-1720 */
double ro_Gsc(const rs_params *p, double T, double c) {
  double termL0 = L0_BCC * (1.0 - 2.0 * c);
  double onemc = 1.0 - c;
  double log_part = 0.;
  if (c > 1.e-8 && onemc > 1.e-8) log_part = p->RR * T * log(c / onemc);
  return ro_G_Ti_BCC(T) - ro_G_Nb_BCC(T) + termL0 + log_part;
}

void ro_calphad_table(const rs_params *p, int which, const double *T,
                      const double *c, double *out, int64_t n) {
  for (int64_t k = 0; k < n; ++k) {
    switch (which) {
      case 0: out[k] = ro_Gl(p, T[k], c[k]); break;
      case 1: out[k] = ro_Gs(p, T[k], c[k]); break;
      case 2: out[k] = ro_Glc(p, T[k], c[k]); break;
      default: out[k] = ro_Gsc(p, T[k], c[k]); break;
    }
  }
}

/* ------------------------------------------------------------------ FTA */
/* get_delta, fun.cu:1610-1619 */
double ro_get_delta(const rs_params *p, const rs_derived *d, int i,
                    int i_offset_history, double l_offset_Vp) {
  const double GG = p->GG, dx = p->dx, SS = p->S, W0 = p->W0;
  const double deltaT0 = d->deltaT0;
  return p->delta_initial +
         GG * (i - p->i_tip_target + i_offset_history - p->i_offset_history_initial) * dx *
             SS * W0 / deltaT0 -
         GG * (l_offset_Vp - p->l_offset_Vp_initial) * SS * W0 / deltaT0;
}

/* Vp_ramp, fun.cu:1974-1982 */
double ro_vp_ramp(const rs_params *p, double t) {
  if (p->vp_ramp) {
    t = t * 0.001;
    return p->Vp + 0.0107587 * t;
  }
  return p->Vp;
}

/* ------------------------------------------------------------------ Philox */
static inline void philox_round(uint32_t x[4], const uint32_t k[2]) {
  const uint64_t p0 = (uint64_t)0xD2511F53u * x[0];
  const uint64_t p1 = (uint64_t)0xCD9E8D57u * x[2];
  const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
  const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
  const uint32_t y0 = hi1 ^ x[1] ^ k[0];
  const uint32_t y2 = hi0 ^ x[3] ^ k[1];
  x[0] = y0; x[1] = lo1; x[2] = y2; x[3] = lo0;
}
void ro_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t x[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
  uint32_t k[2] = {key[0], key[1]};
  for (int r = 0; r < 10; ++r) {
    if (r) { k[0] += 0x9E3779B9u; k[1] += 0xBB67AE85u; }
    philox_round(x, k);
  }
  out[0] = x[0]; out[1] = x[1]; out[2] = x[2]; out[3] = x[3];
}
/* 53-bit uniform in (0, 1) from two words */
static inline double u53(uint32_t a, uint32_t b) {
  return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6) + 0.5) * (1.0 / 9007199254740992.0);
}
/* standard normal for (seed, step, cell): Box-Muller on one Philox draw */
static double noise_normal(uint64_t seed, int64_t step, int64_t cell) {
  const uint32_t ctr[4] = {(uint32_t)cell, (uint32_t)((uint64_t)cell >> 32), (uint32_t)step,
                           (uint32_t)((uint64_t)step >> 32) ^ 0x4E4F4953u};
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t o[4];
  ro_philox4x32(ctr, key, o);
  const double u1 = u53(o[0], o[1]);
  const double u2 = u53(o[2], o[3]);
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

/* ------------------------------------------------------------------ step */
static inline double gg(double p) { return 1.875 * (p) - 1.25 * POW3(p) + 0.375 * POW5(p); }
static inline double dgg_dp(double p) { return 1.875 * POW2(1.0 - POW2(p)); }
static inline double qq(double AA, double p) {
  return 0.5 * AA * (1.0 - (p)) - 0.25 * (AA - 1) * POW2(1.0 - (p));
}

/* get_anisotropy, fun.cu:1030-1139 */
static double get_anisotropy(const rs_params *p, const double *phi, double *as,
                             double *ak, int i, int j) {
  const double dx = p->dx;
  double phi00 = phi[pos(p, i, j)];
  double phi10 = phi[pos(p, i + 1, j)];
  double phi01 = phi[pos(p, i, j + 1)];
  double phim0 = phi[pos(p, i - 1, j)];
  double phi0m = phi[pos(p, i, j - 1)];
  double phi11 = phi[pos(p, i + 1, j + 1)];
  double phim1 = phi[pos(p, i - 1, j + 1)];
  double phi1m = phi[pos(p, i + 1, j - 1)];
  double phimm = phi[pos(p, i - 1, j - 1)];

  double dphi_dx = (phi10 - phim0) / (2.0 * dx);
  double dphi_dy = (phi01 - phi0m) / (2.0 * dx);
  double abs_gradient_phi = sqrt(POW2(dphi_dx) + POW2(dphi_dy));

  double dphi_dx_dx = (phi10 - 2.0 * phi00 + phim0) / (dx * dx);
  double dphi_dy_dy = (phi01 - 2.0 * phi00 + phi0m) / (dx * dx);
  double dphi_dx_dy = (phi11 - phim1 - phi1m + phimm) / (4. * dx * dx);

  double laplacian_phi = 2.0 / 3.0 * (dphi_dx_dx + dphi_dy_dy);
  laplacian_phi += 1.0 / 3.0 * (phi11 + phim1 + phi1m + phimm - 4.0 * phi00) / (2.0 * dx * dx);

  double dtheta_dx, dtheta_dy, cos_theta, sin_theta;
  if (abs_gradient_phi > 1.0e-15) {
    dtheta_dx = (dphi_dx * dphi_dx_dy - dphi_dy * dphi_dx_dx) / POW2(abs_gradient_phi);
    dtheta_dy = (dphi_dx * dphi_dy_dy - dphi_dy * dphi_dx_dy) / POW2(abs_gradient_phi);
    cos_theta = dphi_dx / abs_gradient_phi;
    sin_theta = dphi_dy / abs_gradient_phi;
  } else {
    dtheta_dx = 0.0;
    dtheta_dy = 0.0;
    cos_theta = 0.0;
    sin_theta = 0.0;
  }

  const double *o = p->orientation;
  double x1 = o[0], x2 = o[1], y1 = o[3], y2 = o[4], z1 = o[6], z2 = o[7];

  double nxp = x1 * cos_theta + x2 * sin_theta;
  double nyp = y1 * cos_theta + y2 * sin_theta;
  double nzp = z1 * cos_theta + z2 * sin_theta;
  double dnxp_dtheta_1 = -x1 * sin_theta + x2 * cos_theta;
  double dnyp_dtheta_1 = -y1 * sin_theta + y2 * cos_theta;
  double dnzp_dtheta_1 = -z1 * sin_theta + z2 * cos_theta;
  double dnxp_dtheta_2 = -nxp;
  double dnyp_dtheta_2 = -nyp;
  double dnzp_dtheta_2 = -nzp;

  double np4 = POW4(nxp) + POW4(nyp) + POW4(nzp);
  double dnp4_dtheta_1 = 4.0 * (POW3(nxp) * dnxp_dtheta_1 + POW3(nyp) * dnyp_dtheta_1 +
                                POW3(nzp) * dnzp_dtheta_1);
  double dnp4_dtheta_2 = 3.0 * POW2(nxp * dnxp_dtheta_1) + POW3(nxp) * dnxp_dtheta_2;
  dnp4_dtheta_2 += 3.0 * POW2(nyp * dnyp_dtheta_1) + POW3(nyp) * dnyp_dtheta_2;
  dnp4_dtheta_2 += 3.0 * POW2(nzp * dnzp_dtheta_1) + POW3(nzp) * dnzp_dtheta_2;
  dnp4_dtheta_2 *= 4;

  const double eps1 = p->eps1, eps2 = p->eps2, epk1 = p->epk1;
  double da_dtheta_1, da_dtheta_2;
  if (p->one_eps) {
    *ak = 1.0 - 3.0 * epk1 + 4.0 * epk1 * np4;
    *as = 1.0 - 3.0 * eps1 + 4.0 * eps1 * np4;
    da_dtheta_1 = 4.0 * eps1 * dnp4_dtheta_1;
    da_dtheta_2 = 4.0 * eps1 * dnp4_dtheta_2;
  } else {
    *ak = 1.0 + epk1 * (np4 - 0.6);
    *as = 1.0 + eps1 * (np4 - 0.6) + eps2 * (3.0 * np4 + 66.0 * POW2(nxp * nyp * nzp) - 17.0 / 7.0);
    double dnp2_dtheta_1 = 2.0 * nxp * nyp * nzp *
                           (dnxp_dtheta_1 * nyp * nzp + nxp * dnyp_dtheta_1 * nzp +
                            nxp * nyp * dnzp_dtheta_1);
    double dnp2_dtheta_2 = POW2(dnxp_dtheta_1 * nyp * nzp) + POW2(nxp * dnyp_dtheta_1 * nzp) +
                           POW2(nxp * nyp * dnzp_dtheta_1);
    dnp2_dtheta_2 += nxp * dnxp_dtheta_2 * POW2(nyp * nzp) + nyp * dnyp_dtheta_2 * POW2(nxp * nzp) +
                     nzp * dnzp_dtheta_2 * POW2(nxp * nyp);
    dnp2_dtheta_2 += 4.0 * nxp * nyp * nzp *
                     (dnxp_dtheta_1 * dnyp_dtheta_1 * nzp + nxp * dnyp_dtheta_1 * dnzp_dtheta_1 +
                      dnxp_dtheta_1 * nyp * dnzp_dtheta_1);
    dnp2_dtheta_2 *= 2.0;
    da_dtheta_1 = (eps1 + 3.0 * eps2) * dnp4_dtheta_1 + 66.0 * eps2 * dnp2_dtheta_1;
    da_dtheta_2 = (eps1 + 3.0 * eps2) * dnp4_dtheta_2 + 66.0 * eps2 * dnp2_dtheta_2;
  }

  double anisotropy = POW2(*as) * laplacian_phi +
                      2.0 * (*as) * da_dtheta_1 * (dtheta_dx * dphi_dx + dtheta_dy * dphi_dy) +
                      (da_dtheta_2 * (*as) + POW2(da_dtheta_1)) *
                          (dtheta_dy * dphi_dx - dtheta_dx * dphi_dy);
  return anisotropy;
}

/* ghost copy of one field after the interior update: compute_boundary_individual
 * (fun.cu:1220-1230) in its sequentially consistent reading. */
static void apply_ghosts(const rs_params *p, double *f) {
  const int Nx = p->nx_all, Ny = p->ny_all;
  const int jmin = p->periodic_j ? Ny - 2 : 1;
  const int jmax = p->periodic_j ? 1 : Ny - 2;
  for (int j = 1; j <= Ny - 2; ++j) {
    f[pos(p, 0, j)] = f[pos(p, 1, j)];
    f[pos(p, Nx - 1, j)] = f[pos(p, Nx - 2, j)];
  }
  if (p->band) return; /* row bands: the ghost rows are the neighbouring bands' rows */
  for (int i = 0; i < Nx; ++i) {
    f[pos(p, i, 0)] = f[pos(p, i, jmin)];
    f[pos(p, i, Ny - 1)] = f[pos(p, i, jmax)];
  }
}

void ro_step(const rs_params *p, const rs_derived *d, const double *c,
             const double *phi, const double *psi, const double *T_fine,
             double *c_next, double *phi_next, double *psi_next, int64_t step,
             int i_offset_history, double l_offset_Vp) {
  const int Nx = p->nx_all, Ny = p->ny_all;
  const double dx = p->dx, dt = d->dt;
  const double hh = d->hh, v0 = p->v0, h0 = d->h0;
  const double deltaT0 = d->deltaT0, Tmelt = p->Tmelt;

  /* compute_phi, fun.cu:1143-1218 (N_or = 1: sum_phi = 0, tau = 1) */
#pragma omp parallel for schedule(static)
  for (int j = 1; j < Ny - 1; ++j) {
    for (int i = 1; i < Nx - 1; ++i) {
      const int64_t ps = pos(p, i, j);
      double c00 = c[ps];
      double phi00 = phi[ps];
      double sum_phi = 0;
      double as, ak;
      double anisotropy = get_anisotropy(p, phi, &as, &ak, i, j);
      double term = phi00 - POW3(phi00) + anisotropy;
      double T00;
      if (T_fine) {
        T00 = T_fine[ps];
      } else {
        double delta = ro_get_delta(p, d, i, i_offset_history, l_offset_Vp);
        T00 = delta * deltaT0 + Tmelt;
      }
      term += (ro_Gl(p, T00, c00) - ro_Gs(p, T00, c00)) * dgg_dp(phi00) / (2.0 * hh * v0);
      double tau = 1.0 + 1.0e4 * POW2(0.5 * (1.0 + phi00)) * sum_phi;
      double pn = phi00 + dt * ak / (POW2(as) * tau) * term;
      /* interface noise (reference if_noise block, fun.cu:1200-1215, is dead
       * code; here an additive Gaussian term confined to the interface) */
      if (p->noise_amplitude > 0.0) {
        double w = 1.0 - phi00 * phi00;
        if (w > 1.0e-3)
          pn += p->noise_amplitude * sqrt(dt) * w *
                noise_normal(p->seed, step, ps + (p->band ? (int64_t)p->j_offset * p->nx_all : 0));
      }
      phi_next[ps] = pn;
    }
  }

  /* compute_psi, fun.cu:1232-1273 */
#pragma omp parallel for schedule(static)
  for (int j = 1; j < Ny - 1; ++j) {
    for (int i = 1; i < Nx - 1; ++i) {
      const int64_t ps = pos(p, i, j);
      psi_next[ps] = (p->n_orientation - 1) + phi_next[ps];
      double num_phi_higher_than_minus1 = 0;
      if (phi_next[ps] > -1) num_phi_higher_than_minus1++;
      double psi_temp = p->n_orientation - 1;
      if (psi_next[ps] > 1.0) {
        psi_temp = p->n_orientation - 1;
        phi_next[ps] -= (psi_next[ps] - 1.0) * (phi_next[ps] > -1) / num_phi_higher_than_minus1;
        psi_temp += phi_next[ps];
        psi_next[ps] = psi_temp;
      }
      phi_next[ps] = fmax(phi_next[ps], -1.0);
      phi_next[ps] = fmin(phi_next[ps], 1.0);
    }
  }
  apply_ghosts(p, psi_next);
  apply_ghosts(p, phi_next);

  /* compute_c_CALPHAD, fun.cu:1365-1467 */
  const double AA = p->AA;
#pragma omp parallel for schedule(static)
  for (int j = 1; j < Ny - 1; ++j) {
    for (int i = 1; i < Nx - 1; ++i) {
      int64_t ps00 = pos(p, i, j);
      int64_t ps10 = pos(p, i + 1, j);
      int64_t psm0 = pos(p, i - 1, j);
      int64_t ps01 = pos(p, i, j + 1);
      int64_t ps0m = pos(p, i, j - 1);
      int64_t ps11 = pos(p, i + 1, j + 1);
      int64_t psm1 = pos(p, i - 1, j + 1);
      int64_t ps1m = pos(p, i + 1, j - 1);
      int64_t psmm = pos(p, i - 1, j - 1);

      double c00 = c[ps00], c10 = c[ps10], cm0 = c[psm0], c01 = c[ps01], c0m = c[ps0m];
      double c11 = c[ps11], cm1 = c[psm1], c1m = c[ps1m], cmm = c[psmm];
      double psi00 = psi[ps00], psi10 = psi[ps10], psim0 = psi[psm0], psi01 = psi[ps01];
      double psi0m = psi[ps0m], psi11 = psi[ps11], psim1 = psi[psm1], psi1m = psi[ps1m];
      double psimm = psi[psmm];

      double T00, T10, Tm0, T01, T0m;
      if (T_fine) {
        T00 = T_fine[ps00];
        T10 = T_fine[ps10];
        Tm0 = T_fine[psm0];
        T01 = T_fine[ps01];
        T0m = T_fine[ps0m];
      } else {
        double delta00 = ro_get_delta(p, d, i, i_offset_history, l_offset_Vp);
        double delta10 = ro_get_delta(p, d, i + 1, i_offset_history, l_offset_Vp);
        double deltam0 = ro_get_delta(p, d, i - 1, i_offset_history, l_offset_Vp);
        T00 = delta00 * deltaT0 + Tmelt;
        T10 = delta10 * deltaT0 + Tmelt;
        Tm0 = deltam0 * deltaT0 + Tmelt;
        T01 = T00;
        T0m = T00;
      }

      double g00 = gg(psi00), g10 = gg(psi10), g01 = gg(psi01), gm0 = gg(psim0), g0m = gg(psi0m);

      double S00 = qq(AA, psi00) * c00 * (1.0 - c00);
      double S10 = qq(AA, psi10) * c10 * (1.0 - c10);
      double S01 = qq(AA, psi01) * c01 * (1.0 - c01);
      double Sm0 = qq(AA, psim0) * cm0 * (1.0 - cm0);
      double S0m = qq(AA, psi0m) * c0m * (1.0 - c0m);
      double S11 = qq(AA, psi11) * c11 * (1.0 - c11);
      double Sm1 = qq(AA, psim1) * cm1 * (1.0 - cm1);
      double S1m = qq(AA, psi1m) * c1m * (1.0 - c1m);
      double Smm = qq(AA, psimm) * cmm * (1.0 - cmm);

      double Shh = 0.25 * (S11 + S10 + S01 + S00);
      double Shn = 0.25 * (S10 + S00 + S1m + S0m);
      double Snh = 0.25 * (Sm1 + S01 + Sm0 + S00);
      double Snn = 0.25 * (Sm0 + Smm + S0m + S00);

      double f00 = 0.5 * (1.0 + g00) * ro_Gsc(p, T00, c00) + 0.5 * (1.0 - g00) * ro_Glc(p, T00, c00);
      double f10 = 0.5 * (1.0 + g10) * ro_Gsc(p, T10, c10) + 0.5 * (1.0 - g10) * ro_Glc(p, T10, c10);
      double f01 = 0.5 * (1.0 + g01) * ro_Gsc(p, T01, c01) + 0.5 * (1.0 - g01) * ro_Glc(p, T01, c01);
      double fm0 = 0.5 * (1.0 + gm0) * ro_Gsc(p, Tm0, cm0) + 0.5 * (1.0 - gm0) * ro_Glc(p, Tm0, cm0);
      double f0m = 0.5 * (1.0 + g0m) * ro_Gsc(p, T0m, c0m) + 0.5 * (1.0 - g0m) * ro_Glc(p, T0m, c0m);

      double denom = 1.0 / (h0 * v0);
      double F10 = 0.25 * (S10 + S00 + Shh + Shn) * (f10 - f00) * denom;
      double F01 = 0.25 * (S01 + S00 + Shh + Snh) * (f01 - f00) * denom;
      double Fm0 = 0.25 * (S00 + Sm0 + Snh + Snn) * (fm0 - f00) * denom;
      double F0m = 0.25 * (S00 + S0m + Shn + Snn) * (f0m - f00) * denom;

      double dc = dt * p->Dl / (p->Gamma * p->muk0) * (F10 + F01 + Fm0 + F0m) / (dx * dx);
      c_next[ps00] = fmax(c00 + dc, 1.0e-6);
    }
  }
  apply_ghosts(p, c_next);
}

/* ------------------------------------------------------------------ frame */
/* pull_back, fun.cu:1469-1492 */
void ro_pull_back(const rs_params *p, const double *c, const double *phi,
                  const double *psi, double *c_next, double *phi_next,
                  double *psi_next, int i_offset) {
  const int Nx = p->nx_all, Ny = p->ny_all;
#pragma omp parallel for schedule(static)
  for (int j = 0; j < Ny; ++j) {
    for (int i = 0; i < Nx; ++i) {
      int i_next = i + i_offset;
      if (i_next < 1) i_next = 1;
      if (i_next > Nx - 2) i_next = Nx - 2;
      if (i_next < Nx - 2)
        c_next[pos(p, i, j)] = c[pos(p, i_next, j)];
      else
        c_next[pos(p, i, j)] = p->cinf;
      if (phi && phi_next) phi_next[pos(p, i, j)] = phi[pos(p, i_next, j)];
      psi_next[pos(p, i, j)] = psi[pos(p, i_next, j)];
    }
  }
}

/* get_itip_all_grain, fun.cu:1745-1754 (phi_interface = 0) */
int ro_itip_all_grain(const rs_params *p, const double *psi) {
  int i_tip = 1;
  for (int j = 0; j < p->ny_all; j++)
    for (int i = i_tip; i < p->nx_all; i++)
      if (psi[pos(p, i, j)] > 0.0) i_tip = i;
  return i_tip;
}

double ro_mass(const rs_params *p, const double *c) {
  double m = 0.0;
  for (int j = 1; j < p->ny_all - 1; ++j) {
    double row = 0.0;
    for (int i = 1; i < p->nx_all - 1; ++i) row += c[pos(p, i, j)];
    m += row;
  }
  return m;
}

/* ------------------------------------------------------------------ tip */
/* deal_with_boundary, fun.cu:2624-2641 (periodic); no-flux reflects */
static int deal_with_boundary(const rs_params *p, int x, int N0, int Nn) {
  int Nmin = N0 < Nn ? N0 : Nn;
  int Nmax = N0 > Nn ? N0 : Nn;
  if (p->periodic_j) {
    if (x <= Nmin - 1) x += (Nmax - Nmin + 1);
    else if (x >= Nmax + 1) x -= (Nmax - Nmin + 1);
  } else {
    if (x < Nmin) x = 2 * Nmin - x;
    else if (x > Nmax) x = 2 * Nmax - x;
  }
  return x;
}

/* solve_5x5, fun.cu:2648-2691 */
static void solve_5x5(double A[5][5], double b[5], double c[5]) {
  int n = 5, pp[5];
  for (int i = 0; i < n; i++) pp[i] = i;
  for (int k = 0; k < n - 1; k++) {
    double max_val = fabs(A[pp[k]][k]);
    int max_idx = k;
    for (int i = k + 1; i < n; i++) {
      if (fabs(A[pp[i]][k]) > max_val) {
        max_val = fabs(A[pp[i]][k]);
        max_idx = i;
      }
    }
    int temp = pp[k];
    pp[k] = pp[max_idx];
    pp[max_idx] = temp;
    for (int i = k + 1; i < n; i++) {
      double factor = A[pp[i]][k] / A[pp[k]][k];
      for (int jj = k; jj < n; jj++) A[pp[i]][jj] -= factor * A[pp[k]][jj];
      b[pp[i]] -= factor * b[pp[k]];
    }
  }
  for (int i = n - 1; i >= 0; i--) {
    double sum = 0.0;
    for (int jj = i + 1; jj < n; jj++) sum += A[pp[i]][jj] * c[jj];
    c[i] = (b[pp[i]] - sum) / A[pp[i]][i];
  }
}

/* get_precise_x, fun.cu:2694-2738 */
static double get_precise_x(const double *x, const double *y, int n) {
  double A[5][5] = {{0}}, b[5] = {0}, c[5] = {0};
  for (int i = 0; i < n; i++) {
    double xi = x[i], yi = y[i];
    double yp[9];
    yp[0] = 1.0;
    for (int k = 1; k <= 8; k++) yp[k] = yp[k - 1] * yi;
    for (int jj = 0; jj < 5; jj++) {
      b[jj] += xi * yp[jj];
      for (int k = 0; k < 5; k++) A[jj][k] += yp[jj + k];
    }
  }
  solve_5x5(A, b, c);
  double phi = 0.0;
  return c[0] + c[1] * phi + c[2] * phi * phi + c[3] * phi * phi * phi + c[4] * phi * phi * phi * phi;
}

/* solve_3x3, fun.cu:2740-2786 */
static int solve_3x3(double A[3][3], double cc[3], double x[3]) {
  for (int k = 0; k < 3; ++k) {
    int pivot = k;
    double maxval = fabs(A[k][k]);
    for (int i = k + 1; i < 3; ++i)
      if (fabs(A[i][k]) > maxval) {
        maxval = fabs(A[i][k]);
        pivot = i;
      }
    if (maxval < 1e-14) return -1;
    if (pivot != k) {
      for (int jj = 0; jj < 3; ++jj) {
        double tmp = A[k][jj];
        A[k][jj] = A[pivot][jj];
        A[pivot][jj] = tmp;
      }
      double tmpb = cc[k];
      cc[k] = cc[pivot];
      cc[pivot] = tmpb;
    }
    double piv = A[k][k];
    for (int i = k + 1; i < 3; ++i) {
      double factor = A[i][k] / piv;
      A[i][k] = 0.0;
      for (int jj = k + 1; jj < 3; ++jj) A[i][jj] -= factor * A[k][jj];
      cc[i] -= factor * cc[k];
    }
  }
  for (int i = 2; i >= 0; --i) {
    double sum = cc[i];
    for (int jj = i + 1; jj < 3; ++jj) sum -= A[i][jj] * x[jj];
    x[i] = sum / A[i][i];
  }
  return 0;
}

/* fit_parabola, fun.cu:2809-2865 */
static int fit_parabola(const double *x, const double *y, int n, double *x0,
                        double *y0, double *R) {
  if (n < 3) return -1;
  double M[3][3] = {{0}}, cc[3] = {0}, aa[3];
  for (int i = 0; i < n; ++i) {
    double yi = y[i], xi = x[i];
    double f0 = 1.0, f1 = yi, f2 = yi * yi;
    M[0][0] += f0 * f0; M[0][1] += f0 * f1; M[0][2] += f0 * f2;
    M[1][0] += f1 * f0; M[1][1] += f1 * f1; M[1][2] += f1 * f2;
    M[2][0] += f2 * f0; M[2][1] += f2 * f1; M[2][2] += f2 * f2;
    cc[0] += f0 * xi; cc[1] += f1 * xi; cc[2] += f2 * xi;
  }
  if (solve_3x3(M, cc, aa) != 0) return -2;
  double aa0 = aa[0], aa1 = aa[1], aa2 = aa[2];
  if (fabs(aa2) < 1e-14) return -3;
  double R_loc = 1.0 / (2.0 * aa2);
  double y0_loc = -aa1 / (2.0 * aa2);
  double x0_loc = aa0 - (y0_loc * y0_loc) / (2.0 * R_loc);
  *x0 = x0_loc;
  *y0 = y0_loc;
  *R = R_loc;
  return 0;
}

/* get_tip_int_at_j, fun.cu:2867-2878 */
static int get_tip_int_at_j(const rs_params *p, const double *psi, int i_initial, int j) {
  int itip = 0;
  /* the reference starts at i_initial even when it is negative (reading the
   * previous row); the oracle starts at 0 */
  for (int i = i_initial < 0 ? 0 : i_initial; i < p->nx_all - 1; i++)
    if (psi[pos(p, i, j)] > 0.0) itip = i;
  return itip;
}

/* index guard: the reference reads psi[pos(i, j)] with i possibly outside
 * [0, Nx-1] when no interface exists in a row; here it is clamped. */
static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* get_precise_tip, fun.cu:2880-2954 */
void ro_precise_tip(const rs_params *p, const rs_derived *d, const double *psi, rs_tip *tip) {
  const int Nx = p->nx_all, Ny = p->ny_all;
  /* get_tip_int, fun.cu:2880-2893 */
  double itip = 0.0;
  int ti = 0, tj = 0;
  for (int j = 0; j < Ny; j++) {
    int i0 = get_tip_int_at_j(p, psi, (int)itip, j);
    double iphi0 = (psi[pos(p, clampi(i0 + 1, 0, Nx - 1), j)] - psi[pos(p, i0, j)]) *
                       (0.0 - psi[pos(p, i0, j)]) + i0;
    if (iphi0 > itip) {
      itip = iphi0;
      ti = (int)itip;
      tj = j;
    }
  }
  tip->i = ti;
  tip->j = tj;

  double i_data[5], psi_data[5], x_data[5], y_data[5];
  const int mi = 2, mj = 2;
  const int jmin = p->periodic_j ? Ny - 2 : 1;
  const int jmax = p->periodic_j ? 1 : Ny - 2;
  int ind = 0;
  for (int j = tj - mj; j <= tj - mj + 4; j++) {
    int j0 = deal_with_boundary(p, j, jmin, jmax);
    int i0 = get_tip_int_at_j(p, psi, ti - 5, j0);
    for (int i = i0 - mi; i <= i0 - mi + 4; i++) {
      i_data[i - (i0 - mi)] = i;
      psi_data[i - (i0 - mi)] = psi[pos(p, clampi(i, 0, Nx - 1), j0)];
    }
    x_data[ind] = get_precise_x(i_data, psi_data, 5);
    y_data[ind] = j0;
    ind++;
  }
  double x0 = 0, y0 = 0, R = 0;
  int status = fit_parabola(x_data, y_data, 5, &x0, &y0, &R);
  tip->status = status;
  tip->x = x0;
  tip->y = y0;
  tip->R = fabs(R) * p->dx * p->W0 * p->S;
  if (tip->R > 1e5) tip->R = 1e5;
  if (tip->R < 1.0) tip->R = 1.0;
  (void)d;
}

/* ------------------------------------------------------------------ IC */
/* set_orientation is applied by the caller; initial, fun.cu:983-1021 */
void ro_initial(const rs_params *p, double *c, double *phi, double *psi) {
  const int Nx = p->nx_all, Ny = p->ny_all;
  for (int j = 0; j < Ny; ++j) {
    for (int i = 0; i < Nx; ++i) {
      const int64_t ps = pos(p, i, j);
      double itip = p->i_tip_target + 0.5 * sin(2.0 * REF_PI * j / Ny);
      double ph = -tanh((i - itip) * p->dx / sqrt(2.0));
      double cc = 0.3184 * tanh(((i - itip) * p->dx - 0.08) / 0.67) + 0.6816;
      if (phi) phi[ps] = ph;
      c[ps] = cc * p->cinf;
      psi[ps] = (p->n_orientation - 1) + ph;
    }
  }
}

/* planar front with a seeded per-row offset; ghost rows take the offset of
 * their periodic (or mirrored) partner row */
void ro_initial_planar(const rs_params *p, double *c, double *phi, double *psi,
                       double c_liquid, double c_solid, uint64_t seed) {
  const int Nx = p->nx_all, Ny = p->ny_all;
  const int jmin = p->periodic_j ? Ny - 2 : 1;
  const int jmax = p->periodic_j ? 1 : Ny - 2;
  for (int j = 0; j < Ny; ++j) {
    int js = p->band ? j + p->j_offset : (j == 0 ? jmin : (j == Ny - 1 ? jmax : j));
    const uint32_t ctr[4] = {(uint32_t)js, 0u, 0u, 0x49434F46u};
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t o[4];
    ro_philox4x32(ctr, key, o);
    double i0 = p->i_tip_target + (u53(o[0], o[1]) - 0.5);
    for (int i = 0; i < Nx; ++i) {
      const int64_t ps = pos(p, i, j);
      double ph = -tanh((i - i0) * p->dx / sqrt(2.0));
      double h = 0.5 * (1.0 + ph);
      if (phi) phi[ps] = ph;
      psi[ps] = ph;
      c[ps] = c_liquid + (c_solid - c_liquid) * h;
    }
  }
}

/* ------------------------------------------------------------------ TFC */
static inline int64_t psT(const rs_derived *d, int iT, int jT) {
  return (int64_t)jT * d->NxT_all + iT;
}

/* initial_temperature, fun.cu:1023-1028 */
void ro_initial_temperature(const rs_params *p, const rs_derived *d, double *T) {
  for (int jT = 0; jT < d->NyT_all; ++jT)
    for (int iT = 0; iT < d->NxT_all; ++iT)
      T[psT(d, iT, jT)] =
          p->Tcold + (iT - 1) * (int)p->S * p->W0 * p->dx * p->ratio_dxT_dx * p->GG;
}

/* integrate_phi, fun.cu:1494-1535 */
void ro_integrate_phi(const rs_params *p, const rs_derived *d, double *dphidt,
                      const double *psi, const double *psi_next, int i_left_end) {
  const int Nx = p->nx_all, r = p->ratio_dxT_dx;
  const int iT1 = i_left_end / r;
  const int iTn = (i_left_end + Nx - 3) / r;
  for (int jT = 0; jT < d->NyT_all; ++jT) {
    for (int iT = 0; iT < d->NxT_all; ++iT) {
      double integral = 0;
      if (iT >= iT1 && iT <= iTn && jT >= 1 && jT <= d->NyT - 2) {
        int i0 = r * iT + 1 - i_left_end;
        int in = i0 + r - 1;
        if (i0 < 1) i0 = 1;
        if (in > Nx - 2) in = Nx - 2;
        for (int j = 1 + r * (jT - 1); j <= r * jT; j++)
          for (int i = i0; i <= in; i++) integral += psi_next[pos(p, i, j)] - psi[pos(p, i, j)];
        dphidt[psT(d, iT, jT)] = integral * 0.5;
      } else {
        dphidt[psT(d, iT, jT)] = 0;
      }
    }
  }
}

/* compute_temperature (one sub-step), fun.cu:1537-1578 */
void ro_compute_temperature(const rs_params *p, const rs_derived *d,
                            const double *T, double *T_next,
                            const double *dphidt, int64_t step) {
  const int NxT = d->NxT, NyT = d->NyT, r = p->ratio_dxT_dx;
  const double dxT = p->dx * r;
  const double tau0 = d->tau0, SS = p->S, W0 = p->W0;
  const double Lcp = p->latent_heat / p->cp;
  for (int jT = 1; jT <= NyT - 2; ++jT) {
    for (int iT = 1; iT <= NxT - 2; ++iT) {
      double T00 = T[psT(d, iT, jT)];
      double T10 = T[psT(d, iT + 1, jT)];
      double Tm0 = T[psT(d, iT - 1, jT)];
      double T01 = T[psT(d, iT, jT + 1)];
      double T0m = T[psT(d, iT, jT - 1)];
      double laplacian = (T10 + Tm0 + T01 + T0m - 4.0 * T00) / POW2(dxT);
      double dTdt = ro_vp_ramp(p, step * tau0 * d->dt) * tau0 / (SS * W0) * (T10 - Tm0) / (2.0 * dxT) +
                    laplacian * p->DT / (p->Gamma * p->muk0);
      T_next[psT(d, iT, jT)] = T[psT(d, iT, jT)] + d->dtT * dTdt +
                               Lcp * dphidt[psT(d, iT, jT)] / (d->ratio_dt_dtT * (r * r));
    }
  }
  const int jTmin = p->periodic_j ? NyT - 2 : 1;
  const int jTmax = p->periodic_j ? 1 : NyT - 2;
  for (int jT = 0; jT < d->NyT_all; ++jT) {
    T_next[psT(d, 0, jT)] = p->Tcold;
    T_next[psT(d, NxT - 1, jT)] = d->Thot;
  }
  for (int iT = 0; iT < d->NxT_all; ++iT) {
    T_next[psT(d, iT, 0)] = T_next[psT(d, iT, jTmin)];
    T_next[psT(d, iT, NyT - 1)] = T_next[psT(d, iT, jTmax)];
  }
}

/* interpolate_temperature, fun.cu:1580-1608 */
void ro_interpolate_temperature(const rs_params *p, const rs_derived *d,
                                const double *T, double *T_fine, int i_left_end) {
  const int Nx = p->nx_all, Ny = p->ny_all, r = p->ratio_dxT_dx;
  const double dxT = p->dx * r;
  for (int j = 0; j < Ny; ++j) {
    for (int i = 0; i < Nx; ++i) {
      int iT = (i - 1 + i_left_end) / r;
      int jT = (int)((j - 1 + dxT) / r);
      double x = (i - 1.0 + i_left_end) / r - iT;
      double y = (j - 1.0 + dxT) / r - jT;
      double f00 = T[psT(d, iT, jT)];
      double f10 = T[psT(d, iT + 1, jT)];
      double f01 = T[psT(d, iT, jT + 1)];
      double f11 = T[psT(d, iT + 1, jT + 1)];
      double a00 = f00;
      double a10 = f10 - f00;
      double a01 = f01 - f00;
      double a11 = f11 - f10 - f01 + f00;
      T_fine[pos(p, i, j)] = a00 + a10 * x + a01 * y + a11 * x * y;
    }
  }
}

/* ------------------------------------------------------------------ driver */
int ro_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

int ro_run_steps(const rs_params *p, const rs_derived *d, double *c, double *phi,
                 double *psi, double *c2, double *phi2, double *psi2,
                 int64_t step0, int64_t nsteps, int i_offset_history,
                 double l_offset_Vp0) {
  double l = l_offset_Vp0;
  double *a[3] = {c, phi, psi}, *b[3] = {c2, phi2, psi2};
  for (int64_t s = 0; s < nsteps; ++s) {
    const int64_t step = step0 + s;
    ro_step(p, d, a[0], a[1], a[2], NULL, b[0], b[1], b[2], step, i_offset_history, l);
    for (int k = 0; k < 3; ++k) {
      double *t = a[k];
      a[k] = b[k];
      b[k] = t;
    }
    l += ro_vp_ramp(p, step * d->tau0 * d->dt) * d->dt * d->tau0 / (p->S * p->W0);
  }
  if (a[0] != c) {
    const size_t n = (size_t)p->nx_all * p->ny_all * sizeof(double);
    memcpy(c, a[0], n);
    memcpy(phi, a[1], n);
    memcpy(psi, a[2], n);
  }
  return ro_num_threads();
}

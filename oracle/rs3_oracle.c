/*
 * rs3_oracle.c — CPU FP64 restatement of the reference's 3D three-phase
 * (peritectic) step, multi/peritectic_multiGPU/TiAg.cu.
 *
 * TEST INFRASTRUCTURE ONLY: the checker of the 3D CUDA path.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load it; the
 * product never links or calls it.
 *
 * Same operation order as the reference kernels (FP64, built with
 * -ffp-contract=off), one domain (the reference's z slabs of several GPUs
 * joined into one).  The frozen temperature T(z, step) is an extension; with
 * G_T = 0 every plane has the reference's constant T.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "rs_oracle.h"

#define P3(p, x, y, z) ((((int64_t)(z) * (p)->ny) + (y)) * (int64_t)(p)->nx + (x))

/* Folch-Plapp interpolation g_i and its derivatives, written as the
 * reference's macros g, gp1, gp2 (TiAg.cu:72-74) */
static inline double g3(double pi, double pj, double pk) {
  return pi * pi * 0.25 * (15.0 * (1 - pi) * (1 + pi - (pk - pj) * (pk - pj)) + pi * (9.0 * (pi * pi) - 5.0));
}
static inline double gp1(double pi, double pj, double pk) {
  return 3.75 * pi * (-4.0 * (pi * pi) + 3.0 * (pi * pi * pi) + 2.0 - pi + (3.0 * pi - 2.0) * ((pj - pk) * (pj - pk)));
}
static inline double gp2(double pi, double pj, double pk) { return 7.5 * (pi - 1.0) * (pi * pi) * (pj - pk); }

void ro3_default_params(rs3_params *p) {
  memset(p, 0, sizeof(*p));
  p->nx = 512; /* Nx, Ny, devNz (TiAg.cu:23-28) */
  p->ny = 512;
  p->nz = 128;
  p->dt = 0.015; /* DT, DXin.. (TiAg.cu:20-23) */
  p->dx_inv = p->dy_inv = p->dz_inv = 2.0;
  p->a1 = 0.0; /* TiAg.cu:37-40 */
  p->a2 = 4.43;
  p->a3 = 6.09;
  p->b = 12.0;
  p->lambda = 30.0; /* TiAg.cu:42-45 */
  p->alpha = 2.0;
  p->Da = 0.0;
  p->Db = 0.0;
  p->A1 = 0.391701; /* TiAg.cu:54-59 */
  p->A2 = 0.216598;
  p->B11 = 0.0685881;
  p->B21 = 0.037927;
  p->B12 = -0.466867;
  p->B22 = -0.0662661;
  p->T_ref = 60.0 * 0.000321787; /* TiAg.cu:52 */
  p->energy = 0;
  p->AA = 1.0;
  p->RR = 8.3145;
  p->c_ref = 0.0;
}

/* T of plane z at a step; B1, B2 (TiAg.cu:61-62) */
static void plane_B(const rs3_params *p, int z, int64_t step, double *B1, double *B2) {
  const double T = p->G_T == 0.0 ? p->T_ref : p->T_ref + p->G_T * ((double)z - p->z_T - p->V_T * (double)step);
  *B1 = p->B11 + p->B12 * T;
  *B2 = p->B21 + p->B22 * T;
}

/* ca, cb, cla, clb at T_ref (TiAg.cu:64-67) */
void ro3_equilibrium(const rs3_params *p, double out[4]) {
  const double B1 = p->B11 + p->B12 * p->T_ref, B2 = p->B21 + p->B22 * p->T_ref;
  out[0] = (B1 + 0.5 * B2) / (p->A1 + 0.5 * p->A2) - p->A1 - p->A2;
  out[1] = (B1 - 0.5 * B2) / (p->A1 - 0.5 * p->A2) - p->A1 + p->A2;
  out[2] = (B1 + 0.5 * B2) / (p->A1 + 0.5 * p->A2) + p->A1;
  out[3] = (B1 - 0.5 * B2) / (p->A1 - 0.5 * p->A2) + p->A1;
}

/* boundaryX, boundaryY, boundaryZ in that order (TiAg.cu:565-605) */
void ro3_boundary(const rs3_params *p, double *f) {
  const int nx = p->nx, ny = p->ny, nz = p->nz;
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y) {
      f[P3(p, 0, y, z)] = f[P3(p, nx - 2, y, z)];
      f[P3(p, nx - 1, y, z)] = f[P3(p, 1, y, z)];
    }
  for (int z = 0; z < nz; ++z)
    for (int x = 0; x < nx; ++x) {
      f[P3(p, x, 0, z)] = f[P3(p, x, ny - 2, z)];
      f[P3(p, x, ny - 1, z)] = f[P3(p, x, 1, z)];
    }
  for (int y = 0; y < ny; ++y)
    for (int x = 0; x < nx; ++x) {
      f[P3(p, x, y, 0)] = f[P3(p, x, y, 1)];
      f[P3(p, x, y, nz - 1)] = f[P3(p, x, y, nz - 2)];
    }
}

/* energy 1 (Ti-Nb CALPHAD): T of plane z at a step, in K */
static double plane_T(const rs3_params *p, int z, int64_t step) {
  return p->T_ref + p->G_T * ((double)z - p->z_T - p->V_T * (double)step);
}
/* the 2D parameter set whose CALPHAD functions serve energy 1 (only RR is read) */
static rs_params calphad_params(const rs3_params *p) {
  rs_params q;
  ro_default_params(&q);
  q.RR = p->RR;
  return q;
}

/* computeMu on every cell, then boundaryMu* (TiAg.cu:461-500).  Energy 1:
 * mu = g1 Glc + (1 - g1) Gsc at the plane's T (fun.cu:1443-1452 with
 * 0.5 (1 + g) = 1 - g1), the ghost planes then images as in boundaryMu. */
static void mu_at(const rs3_params *p, int64_t step, const double *phi1, const double *phi2, const double *c,
                  double *mu) {
  const double r1 = p->A1, r2 = -p->A1 - p->A2, r3 = -p->A1 + p->A2;
  const int64_t n = (int64_t)p->nx * p->ny * p->nz;
  if (p->energy == 1) {
    const rs_params q = calphad_params(p);
    const int64_t plane = (int64_t)p->nx * p->ny;
#pragma omp parallel for schedule(static)
    for (int64_t ps = 0; ps < n; ++ps) {
      const double T = plane_T(p, (int)(ps / plane), step);
      const double p1 = phi1[ps], p2 = phi2[ps], p3 = 1.0 - p1 - p2;
      const double g1 = g3(p1, p2, p3), gS = 1.0 - g1;
      mu[ps] = gS * ro_Gsc(&q, T, c[ps]) + g1 * ro_Glc(&q, T, c[ps]);
    }
  } else {
#pragma omp parallel for schedule(static)
    for (int64_t ps = 0; ps < n; ++ps) {
      const double p1 = phi1[ps], p2 = phi2[ps], p3 = 1.0 - p1 - p2;
      mu[ps] = c[ps] - r1 * g3(p1, p2, p3) - r2 * g3(p2, p3, p1) - r3 * g3(p3, p1, p2);
    }
  }
  ro3_boundary(p, mu);
}

void ro3_mu(const rs3_params *p, const double *phi1, const double *phi2, const double *c, double *mu) {
  mu_at(p, 0, phi1, phi2, c, mu);
}

/* diffuse on the interior (TiAg.cu:503-561) with the given mu */
static void diffuse(const rs3_params *p, int64_t step, const double *phi1, const double *phi2, const double *c,
                    const double *mu, double *phi1_n, double *phi2_n, double *c_n) {
  const int nx = p->nx, ny = p->ny, nz = p->nz;
  const double DXin = p->dx_inv, DYin = p->dy_inv, DZin = p->dz_inv;
  const double r1 = p->A1, r2 = -p->A1 - p->A2, r3 = -p->A1 + p->A2;
  const double a1 = p->a1, a2 = p->a2, a3 = p->a3, b = p->b, lam = p->lambda;
  const double Da = p->Da, Db = p->Db;
  const int tinb = p->energy == 1;
  const rs_params q = calphad_params(p);
#pragma omp parallel for schedule(static)
  for (int z = 1; z < nz - 1; ++z) {
    double B1, B2;
    plane_B(p, z, step, &B1, &B2);
    const double s1 = B1, s2 = -B1 - B2, s3 = -B1 + B2;
    const double Tz = tinb ? plane_T(p, z, step) : 0.0;
    for (int y = 1; y < ny - 1; ++y)
      for (int x = 1; x < nx - 1; ++x) {
        const int64_t ps = P3(p, x, y, z);
        const int64_t xp = P3(p, x + 1, y, z), xm = P3(p, x - 1, y, z);
        const int64_t yp = P3(p, x, y + 1, z), ym = P3(p, x, y - 1, z);
        const int64_t zp = P3(p, x, y, z + 1), zm = P3(p, x, y, z - 1);
        const double p1 = phi1[ps], p2 = phi2[ps], p3 = 1.0 - p1 - p2, muu = mu[ps];
        double fcphi1, fcphi2, fcphi3;
        if (tinb) {
          /* the liquid's grand potential against both grains: Gl - Gs at the
           * cell (fun.cu:1192-1193), for (s1 - r1 mu) - (s_j - r_j mu) */
          const double dG = ro_Gl(&q, Tz, c[ps]) - ro_Gs(&q, Tz, c[ps]);
          fcphi1 = lam * (gp1(p1, p2, p3) * dG);
          fcphi2 = lam * (gp2(p1, p2, p3) * dG);
          fcphi3 = lam * (gp2(p1, p3, p2) * dG);
        } else {
          fcphi1 = lam * (gp1(p1, p2, p3) * (s1 - r1 * muu) + gp2(p2, p1, p3) * (s2 - r2 * muu) +
                          gp2(p3, p1, p2) * (s3 - r3 * muu));
          fcphi2 = lam * (gp2(p1, p2, p3) * (s1 - r1 * muu) + gp1(p2, p3, p1) * (s2 - r2 * muu) +
                          gp2(p3, p2, p1) * (s3 - r3 * muu));
          fcphi3 = lam * (gp2(p1, p3, p2) * (s1 - r1 * muu) + gp2(p2, p3, p1) * (s2 - r2 * muu) +
                          gp1(p3, p1, p2) * (s3 - r3 * muu));
        }
        const double lap1 = (phi1[xp] + phi1[xm] - 2.0 * p1) * DXin * DXin +
                            (phi1[yp] + phi1[ym] - 2.0 * p1) * DYin * DYin +
                            (phi1[zp] + phi1[zm] - 2.0 * p1) * DZin * DZin;
        const double lap2 = (phi2[xp] + phi2[xm] - 2.0 * p2) * DXin * DXin +
                            (phi2[yp] + phi2[ym] - 2.0 * p2) * DYin * DYin +
                            (phi2[zp] + phi2[zm] - 2.0 * p2) * DZin * DZin;
        const double lap3 = -lap1 - lap2;
        const double fphi1 = 2.0 * p1 * (1.0 - p1) * (1.0 - 2.0 * p1) +
                             a1 * ((p2 * p3) * (p2 * p3)) * (3.0 + 2 * b * p1) +
                             2.0 * a2 * p1 * (p3 * p3) * (3 * p1 * p3 + 3.0 * p2 + b * (p2 * p2)) +
                             2.0 * a3 * p1 * (p2 * p2) * (3.0 * p1 * p2 + 3.0 * p3 + b * (p3 * p3)) + fcphi1;
        const double fphi2 = 2.0 * p2 * (1.0 - p2) * (1.0 - 2.0 * p2) +
                             2.0 * a1 * p2 * (p3 * p3) * (3 * p2 * p3 + 3.0 * p1 + b * (p1 * p1)) +
                             a2 * ((p1 * p3) * (p1 * p3)) * (3.0 + 2 * b * p2) +
                             2.0 * a3 * p2 * (p1 * p1) * (3.0 * p1 * p2 + 3.0 * p3 + b * (p3 * p3)) + fcphi2;
        const double fphi3 = 2.0 * p3 * (1.0 - p3) * (1.0 - 2.0 * p3) +
                             2.0 * a1 * p3 * (p2 * p2) * (3.0 * p2 * p3 + 3.0 * p1 + b * (p1 * p1)) +
                             2.0 * a2 * p3 * (p1 * p1) * (3 * p1 * p3 + 3.0 * p2 + b * (p2 * p2)) +
                             a3 * ((p1 * p2) * (p1 * p2)) * (3.0 + 2 * b * p3) + fcphi3;
        const double muphi1 = fphi1 - lap1, muphi2 = fphi2 - lap2, muphi3 = fphi3 - lap3;
        const double phi1t = -(2.0 * muphi1 - muphi2 - muphi3) * 0.333333333333333333333333333;
        const double phi2t = -(2.0 * muphi2 - muphi1 - muphi3) * 0.333333333333333333333333333;
        phi1_n[ps] = p1 + p->dt * phi1t;
        phi2_n[ps] = p2 + p->dt * phi2t;
        /* solute: face mobilities 0.5 (phi1 + phi1') (+ Da, Db terms); energy 1:
         * 0.5 (S + S'), S = [q(phi1) + Da phi2 + Db phi3] c (1 - c) with
         * q(p) = p (AA - (AA - 1) p) (fun.cu:189, 1424-1464 in the liquid fraction) */
#define SCELL(n) \
  ((phi1[n] * (p->AA - (p->AA - 1.0) * phi1[n]) + Da * phi2[n] + Db * (1.0 - phi1[n] - phi2[n])) * c[n] * (1.0 - c[n]))
#define HFACE(n, dmu, din)                                                                                    \
  ((tinb ? 0.5 * (SCELL(ps) + SCELL(n))                                                                       \
         : 0.5 * (p1 + phi1[n]) + Da * 0.5 * (p2 + phi2[n]) + Db * 0.5 * (p3 + 1.0 - phi1[n] - phi2[n])) * \
   (dmu) * (din))
        const double Hxp = HFACE(xp, mu[xp] - muu, DXin), Hxn = HFACE(xm, muu - mu[xm], DXin);
        const double Hyp = HFACE(yp, mu[yp] - muu, DYin), Hyn = HFACE(ym, muu - mu[ym], DYin);
        const double Hzp = HFACE(zp, mu[zp] - muu, DZin), Hzn = HFACE(zm, muu - mu[zm], DZin);
#undef HFACE
#undef SCELL
        c_n[ps] = c[ps] + p->dt * p->alpha * ((Hxp - Hxn) * DXin + (Hyp - Hyn) * DYin + (Hzp - Hzn) * DZin);
      }
  }
}

/* one step of the reference loop (TiAg.cu:269-340): computeMu, boundaryMu,
 * diffuse, boundary; mu_out (optional) receives the mu that was used */
void ro3_step(const rs3_params *p, int64_t step, const double *phi1, const double *phi2, const double *c,
              double *phi1_n, double *phi2_n, double *c_n, double *mu_out) {
  const int64_t n = (int64_t)p->nx * p->ny * p->nz;
  double *mu = mu_out ? mu_out : (double *)malloc(sizeof(double) * n);
  mu_at(p, step, phi1, phi2, c, mu);
  diffuse(p, step, phi1, phi2, c, mu, phi1_n, phi2_n, c_n);
  ro3_boundary(p, phi1_n);
  ro3_boundary(p, phi2_n);
  ro3_boundary(p, c_n);
  if (!mu_out) free(mu);
}

double ro3_mass(const rs3_params *p, const double *c) {
  double s = 0.0;
  for (int z = 1; z < p->nz - 1; ++z)
    for (int y = 1; y < p->ny - 1; ++y)
      for (int x = 1; x < p->nx - 1; ++x) s += c[P3(p, x, y, z)];
  return s;
}

static inline double u53(uint32_t a, uint32_t b) {
  return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6) + 0.5) * (1.0 / 9007199254740992.0);
}

/* alpha cap centres: seeded uniform (x, y) over the interior */
void ro3_cap_centres(const rs3_params *p, int n_alpha, uint64_t seed, double *cx, double *cy) {
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  for (int k = 0; k < n_alpha; ++k) {
    const uint32_t ctr[4] = {(uint32_t)k, 0u, 0u, 0x43415053u};
    uint32_t o[4];
    ro_philox4x32(ctr, key, o);
    cx[k] = 1.0 + (p->nx - 2) * u53(o[0], o[1]);
    cy[k] = 1.0 + (p->ny - 2) * u53(o[2], o[3]);
  }
}

/* the initial state of rs3_initial (cap shape of TiAg.cu:400-444) */
void ro3_initial(const rs3_params *p, double z_front, double amp, int n_alpha, double cap_radius, uint64_t seed,
                 double *phi1, double *phi2, double *c) {
  double eq[4];
  ro3_equilibrium(p, eq);
  const double ca = eq[0], cb = eq[1], clb = eq[3];
  const double theta = 1.33;
  const double radius = cap_radius / sin(theta), roff = cap_radius / tan(theta);
  double cx[64], cy[64];
  if (n_alpha > 64) n_alpha = 64;
  ro3_cap_centres(p, n_alpha, seed, cx, cy);
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  for (int y = 1; y < p->ny - 1; ++y)
    for (int x = 1; x < p->nx - 1; ++x) {
      const uint32_t ctr[4] = {(uint32_t)x, (uint32_t)y, 0u, 0x5A465254u};
      uint32_t o[4];
      ro_philox4x32(ctr, key, o);
      const double zc = z_front + amp * (2.0 * u53(o[0], o[1]) - 1.0);
      for (int z = 1; z < p->nz - 1; ++z) {
        const int64_t ps = P3(p, x, y, z);
        int cap = 0;
        if (z >= zc)
          for (int k = 0; k < n_alpha; ++k) {
            const double dx = x - cx[k], dy = y - cy[k], dz = z - (z_front - roff);
            if (dx * dx + dy * dy + dz * dz <= radius * radius) cap = 1;
          }
        if (cap) {
          phi1[ps] = 0.0;
          phi2[ps] = 1.0;
          c[ps] = ca;
        } else if (z < zc) {
          phi1[ps] = 0.0;
          phi2[ps] = 0.0;
          c[ps] = cb;
        } else {
          phi1[ps] = 1.0;
          phi2[ps] = 0.0;
          c[ps] = clb;
        }
      }
    }
  ro3_boundary(p, phi1);
  ro3_boundary(p, phi2);
  ro3_boundary(p, c);
}

/* the initial state of rs3_initial_grains: solid c_solid below the seeded
 * front (phase 2 for x <= (nx - 2) / 2, phase 3 beyond), melt c_liquid above */
void ro3_initial_grains(const rs3_params *p, double z_front, double amp, double c_liquid, double c_solid,
                        uint64_t seed, double *phi1, double *phi2, double *c) {
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  for (int y = 1; y < p->ny - 1; ++y)
    for (int x = 1; x < p->nx - 1; ++x) {
      const uint32_t ctr[4] = {(uint32_t)x, (uint32_t)y, 0u, 0x5A465254u};
      uint32_t o[4];
      ro_philox4x32(ctr, key, o);
      const double zc = z_front + amp * (2.0 * u53(o[0], o[1]) - 1.0);
      const int first = x <= (p->nx - 2) / 2;
      for (int z = 1; z < p->nz - 1; ++z) {
        const int64_t ps = P3(p, x, y, z);
        if (z < zc) {
          phi1[ps] = 0.0;
          phi2[ps] = first ? 1.0 : 0.0;
          c[ps] = c_solid;
        } else {
          phi1[ps] = 1.0;
          phi2[ps] = 0.0;
          c[ps] = c_liquid;
        }
      }
    }
  ro3_boundary(p, phi1);
  ro3_boundary(p, phi2);
  ro3_boundary(p, c);
}

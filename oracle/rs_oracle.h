/*
 * rs_oracle.h — CPU FP64 restatement of the reference's phase-field step.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * it.  The product (2d-rapid-solidification_b200) never links or calls it.
 *
 * Every function follows the reference source line by line (same operation
 * order, FP64, built with -ffp-contract=off); the file:line it restates is
 * given beside it.  Where the reference has a data race (ghost corners written
 * by two threads, fun.cu:1220-1230), the oracle takes the sequentially
 * consistent reading: interior cells first, then ghost columns, then ghost
 * rows (which then carry the corner values).
 */
#ifndef RS_ORACLE_H_
#define RS_ORACLE_H_

#include <stdint.h>
#include "../include/rs_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* parameters (constants.hpp values) and set_parameters (fun.cu:1984-2058) */
void ro_default_params(rs_params *p);
void ro_derive(const rs_params *p, rs_derived *d);

/* CALPHAD Ti-Nb (fun.cu:1628-1720) */
double ro_G_Ti_BCC(double T);
double ro_G_Ti_Liq(double T);
double ro_G_Nb_BCC(double T);
double ro_G_Nb_Liq(double T);
double ro_Gl(const rs_params *p, double T, double c);
double ro_Gs(const rs_params *p, double T, double c);
double ro_Glc(const rs_params *p, double T, double c);
double ro_Gsc(const rs_params *p, double T, double c);
void ro_calphad_table(const rs_params *p, int which, const double *T,
                      const double *c, double *out, int64_t n);

/* frozen temperature (fun.cu:1610-1619) */
double ro_get_delta(const rs_params *p, const rs_derived *d, int i,
                    int i_offset_history, double l_offset_Vp);
double ro_vp_ramp(const rs_params *p, double t_ns);

/* Philox4x32-10 counter RNG (Salmon et al., SC'11) */
void ro_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* one step: compute_phi + compute_psi + compute_c_CALPHAD
 * (fun.cu:1143-1218, 1232-1273, 1365-1467).  T_fine NULL -> frozen T. */
void ro_step(const rs_params *p, const rs_derived *d, const double *c,
             const double *phi, const double *psi, const double *T_fine,
             double *c_next, double *phi_next, double *psi_next, int64_t step,
             int i_offset_history, double l_offset_Vp);

/* pull_back (fun.cu:1469-1492), every cell including ghosts */
void ro_pull_back(const rs_params *p, const double *c, const double *phi,
                  const double *psi, double *c_next, double *phi_next,
                  double *psi_next, int i_offset);

/* get_itip_all_grain (fun.cu:1745-1754) */
int ro_itip_all_grain(const rs_params *p, const double *psi);
/* get_precise_tip (fun.cu:2895-2954) */
void ro_precise_tip(const rs_params *p, const rs_derived *d, const double *psi,
                    rs_tip *tip);
/* sum of c over interior cells */
double ro_mass(const rs_params *p, const double *c);

/* initial conditions */
void ro_initial(const rs_params *p, double *c, double *phi, double *psi);
void ro_initial_planar(const rs_params *p, double *c, double *phi, double *psi,
                       double c_liquid, double c_solid, uint64_t seed);

/* TFC (fun.cu:1023-1028, 1494-1608) */
void ro_initial_temperature(const rs_params *p, const rs_derived *d, double *T);
void ro_integrate_phi(const rs_params *p, const rs_derived *d, double *dphidt,
                      const double *psi, const double *psi_next, int i_left_end);
void ro_compute_temperature(const rs_params *p, const rs_derived *d,
                            const double *T, double *T_next,
                            const double *dphidt, int64_t step);
void ro_interpolate_temperature(const rs_params *p, const rs_derived *d,
                                const double *T, double *T_fine, int i_left_end);

/* K plain steps with pointer swaps (timed CPU baseline); returns number of
 * OpenMP threads used.  Result left in c/phi/psi. */
int ro_run_steps(const rs_params *p, const rs_derived *d, double *c, double *phi,
                 double *psi, double *c2, double *phi2, double *psi2,
                 int64_t step0, int64_t nsteps, int i_offset_history,
                 double l_offset_Vp0);
int ro_num_threads(void);

/* ---- 3D three-phase step (multi/peritectic_multiGPU/TiAg.cu), rs3_oracle.c ---- */
void ro3_default_params(rs3_params *p);
void ro3_equilibrium(const rs3_params *p, double out[4]); /* ca, cb, cla, clb */
void ro3_boundary(const rs3_params *p, double *f);
void ro3_mu(const rs3_params *p, const double *phi1, const double *phi2, const double *c, double *mu);
void ro3_step(const rs3_params *p, int64_t step, const double *phi1, const double *phi2, const double *c,
              double *phi1_n, double *phi2_n, double *c_n, double *mu_out);
double ro3_mass(const rs3_params *p, const double *c);
void ro3_cap_centres(const rs3_params *p, int n_alpha, uint64_t seed, double *cx, double *cy);
void ro3_initial(const rs3_params *p, double z_front, double amp, int n_alpha, double cap_radius, uint64_t seed,
                 double *phi1, double *phi2, double *c);
void ro3_initial_grains(const rs3_params *p, double z_front, double amp, double c_liquid, double c_solid,
                        uint64_t seed, double *phi1, double *phi2, double *c);

#ifdef __cplusplus
}
#endif
#endif

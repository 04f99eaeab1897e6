// rs_io.cpp — the reference's snapshot and restart file layouts (host code).
//
//  * parameters.txt: written with save_parameters' layout (fun.cu:2060-2202,
//    src/main.cu:1786-1920) and read back positionally as load_parameters does
//    (fun.cu:2204-2388), so restarts pass between this code and the reference
//    in both directions.  Like the reference, the file carries %g values
//    (6 significant digits); a restart reads dt from it.
//  * check_point_<field>.bin: raw FP64, i fastest, Ny_all rows of Nx_all
//    (save_check_point / load_check_point, fun.cu:1848-1872, 1894-1918).  A
//    missing or short file is an error here (the reference prints "not found!"
//    and continues with uninitialised memory).
//  * check_point_temperature.bin: the NyT x NxT physical part of the coarse T
//    (fun.cu:1874-1892, 1946-1971).
//  * <field>_<k>.txt snapshots: "%g\t" per cell, one line per row, every di-th
//    column and dj-th row (save_field, fun.cu:1768-1790).
#include <cmath>
#include <cstdio>
#include <cstring>

#include "../../include/rs_b200.h"

namespace rs {
int set_error(int code, const char *msg);
}

namespace {

int io_fail(const char *what, const char *path) {
  char msg[512];
  snprintf(msg, sizeof(msg), "%s: %s", what, path ? path : "(null)");
  return rs::set_error(RS_E_IO, msg);
}

}  // namespace

extern "C" {

int rs_write_parameters(const char *path, const rs_params *p, const rs_run_state *s) {
  if (!path || !p || !s) return rs::set_error(RS_E_INVALID, "rs_write_parameters: null argument");
  rs_derived d;
  int rc = rs_derive(p, &d);
  if (rc) return rc;
  FILE *fp = fopen(path, "w");
  if (!fp) return io_fail("rs_write_parameters: cannot open", path);
  const double SS = p->S, W0 = p->W0, dx = p->dx, tau0 = d.tau0;
  const double dt = s->dt > 0 ? s->dt : d.dt;
  const double deltaT0 = d.deltaT0;
  const double a1 = 2.0 * std::sqrt(2.0) / 3.0;
  const double d0 = p->Gamma / deltaT0;
  const double bb = 0.5 * std::log(p->ke);
  const double lambda = -bb * a1 * SS * W0 / d0 / (1.0 - p->ke);
  const double Lcp = p->latent_heat / p->cp;
  const double density = 1.0e-6 * p->num_moles * p->molar_weight;
  const double latentHeat2 = p->latent_heat * p->num_moles;
  const double surface_tension = p->Gamma * 1e-9 * latentHeat2 / p->Tmelt;
  const double hh = surface_tension / (a1 * SS * W0 * 1.0e-9);
  const double h0 = p->RR * p->Tmelt / p->v0;
  const int itt = p->i_tip_target;
  // the reference prints its long counters with %d
  const int step32 = (int)s->step, total32 = (int)d.total_step;

  fprintf(fp, "----------------------------------------- Dynamically changing variables\n");
  fprintf(fp, "%-13d step\n", step32);
  fprintf(fp, "%-13d i_offset_history, accumulated i offset\n", s->i_offset_history);
  fprintf(fp, "%-13g l_offset_Vp, unit: [W]; offset due to pulling velocity\n", s->l_offset_Vp);
  fprintf(fp, "%-13g delta_initial, initial dimensionless temperature\n", s->delta);
  fprintf(fp, "\n");

  fprintf(fp, "-----------------------------------------\n");
  fprintf(fp, "%-13d Nx_all\n", p->nx_all);
  fprintf(fp, "%-13d Ny_all\n", p->ny_all);
  fprintf(fp, "%-13g dx => %g nm\n", dx, dx * W0 * SS);
  fprintf(fp, "%-13g W0 [nm], physical interface thickness\n", W0 * 1.0);
  fprintf(fp, "%-13g S, scale factor\n", SS * 1.0);
  fprintf(fp, "%-13g W=S*W0, nm, effective interface thickness\n", SS * W0);
  fprintf(fp, "%-13d i_tip_target => %g um\n", itt, itt * dx * SS * W0 * 1e-3);
  fprintf(fp, "\n");

  fprintf(fp, "%-13g dt => %g ns\n", dt, dt * tau0);
  fprintf(fp, "%-13g tau0 [ns]; characteristic time\n", tau0);
  fprintf(fp, "%-13d total steps      => %g us\n", total32, p->total_time_ns * 1e-3);
  fprintf(fp, "%-13d step_fields      => %g us\n", d.step_fields, d.step_fields * tau0 * dt * 1e-3);
  fprintf(fp, "%-13d step_check_point => %g us\n", d.step_check_point, d.step_check_point * tau0 * dt * 1e-3);
  fprintf(fp, "%-13d step_tip         => %g ns\n", d.step_tip, d.step_tip * tau0 * dt);
  fprintf(fp, "%-13d step_pull_back   => %g ns\n", d.step_pull_back, d.step_pull_back * tau0 * dt);
  fprintf(fp, "\n");

  fprintf(fp, "%-13g Gamma [K*nm], Gibbs-Thomson coefficient\n", p->Gamma);
  fprintf(fp, "%-13g muk0 [nm/ns/K], interface kinetic coefficient\n", p->muk0);
  fprintf(fp, "%-13g nm^2/ns => %g m^2/s, Dl, diffusivity in the liquid\n", p->Dl, p->Dl * 1e-9);
  fprintf(fp, "%-13g K/nm => %g K/m, G, thermal gradient\n", p->GG, p->GG * 1e9);
  fprintf(fp, "%-13g Vp [m/s], pulling velocity \n", p->Vp);
  fprintf(fp, "\n");

  fprintf(fp, "%-13g Tmelt [K], melting temperature \n", p->Tmelt);
  fprintf(fp, "%-13g cinf, nominal composition \n", p->cinf);
  fprintf(fp, "%-13g deltaT0 [K], |me|*cinf for dilute alloys \n", deltaT0);
  fprintf(fp, "%-13g d0 [nm] = Gamma/deltaT0, capillary length, only for dilute alloys\n", d0);
  fprintf(fp, "%-13g ke, partition coefficient, only for dilute alloys\n", p->ke);
  fprintf(fp, "%-13g b=ln(ke)/2, only for dilute alloys\n", bb);
  fprintf(fp, "%-13g lambda, only for dilute alloys\n", lambda);
  fprintf(fp, "\n");

  fprintf(fp, "%-13g gamma0 [degrees], orientation angle\n", s->gamma0 * 1.0);
  fprintf(fp, "%-13g gamma1 [degrees], orientation angle\n", s->gamma1 * 1.0);
  fprintf(fp, "%-13g eps1, anisotropy parameter of the interfacial free energy \n", p->eps1);
  fprintf(fp, "%-13g eps2, anisotropy parameter of the interfacial free energy \n", p->eps2 * 1.0);
  fprintf(fp, "%-13g epk1, anisotropy parameter of the kinetic coefficient \n", p->epk1);
  fprintf(fp, "%-13ld random_seed\n", (long)p->seed);
  fprintf(fp, "%-13s path_input\n", s->path_input ? s->path_input : "./");
  fprintf(fp, "\n");

  fprintf(fp, "%-13g latentHeat [J/mol], latent heat\n", p->latent_heat);
  fprintf(fp, "%-13g cp [J/mol/K], specific heat\n", p->cp * 1.0);
  fprintf(fp, "%-13g Lcp = latentHeat/cp [K]\n", Lcp);
  fprintf(fp, "%-13g molar_weight [g/mol] \n", p->molar_weight);
  fprintf(fp, "%-13g density [g/cm^3]\n", density);
  fprintf(fp, "%-13g num_moles [mol/m^3], number of moles per m^3\n", p->num_moles);
  fprintf(fp, "%-13g latentHeat2 [J/m^3], latent heat\n", latentHeat2);
  fprintf(fp, "%-13g surface_tension [J/m^2]\n", surface_tension);
  fprintf(fp, "%-13g hh = surface_tension/(a1*S*W0*1e-9) [J/m^3]\n", hh);
  fprintf(fp, "%-13g h0 = RR*Tmelt/v0 [J/m^3]\n", h0);
  fprintf(fp, "\n");

  if (p->tfc) {
    const int r = p->ratio_dxT_dx;
    const double dxT = dx * r;
    fprintf(fp, "----------------------------------------- Variables for temperature field calculation (TFC)\n");
    fprintf(fp, "-------------------- Dynamically changing variables\n");
    fprintf(fp, "%-13d i_left_end_initial, The i index of the left border of PF in the T field.\n",
            s->i_left_end_initial);
    fprintf(fp, "%-13d i_left_end, The i index of the left border of PF in the T field.\n", s->i_left_end);
    fprintf(fp, "\n");
    fprintf(fp, "%-13g dxT => %g nm\n", dxT, dxT * SS * W0);
    fprintf(fp, "%-13d dxT/dx, larger dx for the temperature field\n", r);
    fprintf(fp, "%-13d NxT => %g um\n", d.NxT, d.NxT * dxT / 1000);
    fprintf(fp, "%-13d NyT => %g um\n", d.NyT, d.NyT * dxT / 1000);
    fprintf(fp, "%-13d NxT_all => %g um, some lattices not used\n", d.NxT_all, d.NxT_all * dxT / 1000);
    fprintf(fp, "%-13d NyT_all => %g um, some lattices not used\n", d.NyT_all, d.NyT_all * dxT / 1000);
    fprintf(fp, "%-13g sample length [nm] => %g um\n", d.length_sample, d.length_sample / 1000);
    fprintf(fp, "\n");
    fprintf(fp, "%-13g dtT => %g ns\n", d.dtT, d.dtT * tau0);
    fprintf(fp, "%-13d dt/dtT, smaller dt for the temperature field\n", d.ratio_dt_dtT);
    fprintf(fp, "\n");
    fprintf(fp, "%-13g D_T [nm^2/ns], thermal diffusivity\n", p->DT * 1.0);
    fprintf(fp, "%-13g Tcold [K]\n", p->Tcold);
    fprintf(fp, "%-13g Thot [K]\n", d.Thot);
  }
  const bool ok = ferror(fp) == 0;
  fclose(fp);
  return ok ? RS_OK : io_fail("rs_write_parameters: write failed", path);
}

// positional read of the same layout (load_parameters, fun.cu:2204-2388)
int rs_read_parameters(const char *path, int32_t tfc, rs_run_state *s) {
  if (!path || !s) return rs::set_error(RS_E_INVALID, "rs_read_parameters: null argument");
  FILE *fp = fopen(path, "r");
  if (!fp) return io_fail("rs_read_parameters: not found", path);
  memset(s, 0, sizeof(*s));
  char dummy[512], str[256];
  double tmp;
  long tl;
  int ti;
  int n = 0, want = 0;
#define RD(fmt, dst)                                   \
  do {                                                 \
    ++want;                                            \
    n += fscanf(fp, fmt, dst);                         \
    if (!fgets(dummy, sizeof(dummy), fp)) dummy[0] = 0; \
  } while (0)
  if (!fgets(dummy, sizeof(dummy), fp)) {
    fclose(fp);
    return io_fail("rs_read_parameters: empty file", path);
  }
  RD("%ld", &tl);
  s->step = tl;
  RD("%d", &s->i_offset_history);
  RD("%lf", &s->l_offset_Vp);
  RD("%lf", &s->delta);
  if (!fgets(dummy, sizeof(dummy), fp)) dummy[0] = 0;  // blank line
  if (!fgets(dummy, sizeof(dummy), fp)) dummy[0] = 0;  // separator
  for (int k = 0; k < 7; ++k) RD("%lf", &tmp);          // Nx_all .. i_tip_target
  RD("%lf", &s->dt);
  RD("%lf", &tmp);                                      // tau0
  RD("%ld", &tl);                                       // total steps
  for (int k = 0; k < 4; ++k) RD("%d", &ti);            // step_fields .. step_pull_back
  for (int k = 0; k < 5; ++k) RD("%lf", &tmp);          // Gamma .. Vp
  for (int k = 0; k < 7; ++k) RD("%lf", &tmp);          // Tmelt .. lambda
  RD("%lf", &s->gamma0);
  RD("%lf", &s->gamma1);
  for (int k = 0; k < 3; ++k) RD("%lf", &tmp);          // eps1, eps2, epk1
  RD("%ld", &tl);                                       // random_seed
  RD("%255s", str);                                     // path_input
  for (int k = 0; k < 10; ++k) RD("%lf", &tmp);         // latentHeat .. h0
  if (tfc) {
    for (int k = 0; k < 3; ++k)
      if (!fgets(dummy, sizeof(dummy), fp)) dummy[0] = 0;
    RD("%d", &s->i_left_end_initial);
    RD("%d", &s->i_left_end);
    RD("%lf", &tmp);  // dxT
    RD("%d", &ti);    // ratio_dxT_dx
    RD("%d", &s->NxT);
    RD("%d", &s->NyT);
    RD("%d", &s->NxT_all);
    RD("%d", &s->NyT_all);
    RD("%lf", &s->length_sample);
    RD("%lf", &s->dtT);
    RD("%d", &s->ratio_dt_dtT);
    RD("%lf", &tmp);  // D_T
    RD("%lf", &s->Tcold);
    RD("%lf", &s->Thot);
  }
#undef RD
  fclose(fp);
  if (n != want) return io_fail("rs_read_parameters: truncated or malformed", path);
  return RS_OK;
}

int rs_write_check_point(const char *path, const double *h, int32_t nx_all, int32_t ny_all) {
  if (!path || !h || nx_all <= 0 || ny_all <= 0) return rs::set_error(RS_E_INVALID, "rs_write_check_point: bad argument");
  FILE *fp = fopen(path, "wb");
  if (!fp) return io_fail("rs_write_check_point: cannot open", path);
  const size_t n = (size_t)nx_all * ny_all;
  const size_t w = fwrite(h, sizeof(double), n, fp);
  fclose(fp);
  return w == n ? RS_OK : io_fail("rs_write_check_point: short write", path);
}

int rs_read_check_point(const char *path, double *h, int32_t nx_all, int32_t ny_all) {
  if (!path || !h || nx_all <= 0 || ny_all <= 0) return rs::set_error(RS_E_INVALID, "rs_read_check_point: bad argument");
  FILE *fp = fopen(path, "rb");
  if (!fp) return io_fail("rs_read_check_point: not found", path);
  const size_t n = (size_t)nx_all * ny_all;
  const size_t r = fread(h, sizeof(double), n, fp);
  fclose(fp);
  return r == n ? RS_OK : io_fail("rs_read_check_point: file shorter than Nx_all*Ny_all doubles", path);
}

int rs_write_check_point_temperature(const char *path, const double *hT, int32_t NxT, int32_t NyT, int32_t NxT_all) {
  if (!path || !hT || NxT <= 0 || NyT <= 0 || NxT_all < NxT)
    return rs::set_error(RS_E_INVALID, "rs_write_check_point_temperature: bad argument");
  FILE *fp = fopen(path, "wb");
  if (!fp) return io_fail("rs_write_check_point_temperature: cannot open", path);
  size_t w = 0;
  for (int jT = 0; jT < NyT; ++jT) w += fwrite(hT + (size_t)jT * NxT_all, sizeof(double), NxT, fp);
  fclose(fp);
  return w == (size_t)NxT * NyT ? RS_OK : io_fail("rs_write_check_point_temperature: short write", path);
}

int rs_read_check_point_temperature(const char *path, double *hT, int32_t NxT, int32_t NyT, int32_t NxT_all) {
  if (!path || !hT || NxT <= 0 || NyT <= 0 || NxT_all < NxT)
    return rs::set_error(RS_E_INVALID, "rs_read_check_point_temperature: bad argument");
  FILE *fp = fopen(path, "rb");
  if (!fp) return io_fail("rs_read_check_point_temperature: not found", path);
  size_t r = 0;
  for (int jT = 0; jT < NyT; ++jT) r += fread(hT + (size_t)jT * NxT_all, sizeof(double), NxT, fp);
  fclose(fp);
  return r == (size_t)NxT * NyT ? RS_OK : io_fail("rs_read_check_point_temperature: short file", path);
}

int rs_write_field_text(const char *path, const double *h, int32_t nx_all, int32_t ny_all, int32_t di, int32_t dj) {
  if (!path || !h || nx_all <= 0 || ny_all <= 0 || di <= 0 || dj <= 0)
    return rs::set_error(RS_E_INVALID, "rs_write_field_text: bad argument");
  FILE *fp = fopen(path, "w");
  if (!fp) return io_fail("rs_write_field_text: cannot open", path);
  for (int j = 0; j < ny_all; j += dj) {
    for (int i = 0; i < nx_all; i += di) fprintf(fp, "%g\t", h[(size_t)j * nx_all + i]);
    fprintf(fp, "\n");
  }
  const bool ok = ferror(fp) == 0;
  fclose(fp);
  return ok ? RS_OK : io_fail("rs_write_field_text: write failed", path);
}

}  // extern "C"

// rs_peri3d.cuh — launchers of the 3D three-phase step (rs_peri3d.cu).
#pragma once

#include <cuda.h>

#include "rs_common.cuh"

namespace rs {

constexpr int kP3MaxCaps = 16;

// tensor maps of one field set (3D, dims nx, ny, nz; box of
// peri3d_box_width x peri3d_box_height x 1 elements)
struct P3Maps {
  CUtensorMap phi1, phi2, c;
};

// initial state: front, cap centres (host-drawn), compositions
struct P3Init {
  uint64_t seed;
  double z_front, amp, radius, roff;
  double ca, cb, clb;
  int n_alpha;
  double cx[kP3MaxCaps], cy[kP3MaxCaps];
};

double peri3d_c_offset(const rs3_params &p);  // FP32 sets hold c - this
int peri3d_box_width(int precision);
int peri3d_box_height(int precision);
int peri3d_x2_box_width();
int peri3d_x2_box_height();
int launch_peri3d_step_x2(const rs3_params &p, const P3Maps &m, float *o1, float *o2, float *oc, int64_t step,
                          int *err, cudaStream_t st);
int launch_peri3d_step(const rs3_params &p, const P3Maps &m, int precision, void *o1, void *o2, void *oc,
                       int64_t step, int *err, cudaStream_t st);
int launch_peri3d_mu(const rs3_params &p, int precision, const void *f1, const void *f2, const void *fc, void *mu,
                     cudaStream_t st);
int launch_peri3d_mass(const rs3_params &p, int precision, const void *fc, double *partial, int nparts, double *out,
                       cudaStream_t st);
int launch_peri3d_init(const rs3_params &p, int precision, const P3Init &ini, void *f1, void *f2, void *fc,
                       cudaStream_t st);
// ghost layers of a set as images (x, then y, then z)
int launch_peri3d_ghosts(const rs3_params &p, int precision, void *f1, void *f2, void *fc, cudaStream_t st);

// energy 1 (Ti-Nb CALPHAD, rs_peri3d_tinb.cu): TMA box of a field set, the
// per-plane table (doubles), the step (table kernel + step kernel; surr:
// the FP32 surrogate or null), mu of every cell at step 0's temperature,
// and the two-grain initial state
struct SurrArgs;
// (surr: the FP32 step runs the surrogate's scalar kernel; otherwise FP32 runs
// on packed pairs with the TiAg pair kernel's box)
int tinb_box_width(int precision, bool surr);
int tinb_box_height(int precision, bool surr);
int tinb_table_len(const rs3_params &p);
int launch_tinb_step(const rs3_params &p, const P3Maps &m, int precision, void *o1, void *o2, void *oc, int64_t step,
                     int *err, double *tab, const SurrArgs *surr, cudaStream_t st);
int launch_tinb_mu(const rs3_params &p, int precision, const void *f1, const void *f2, const void *fc, void *mu,
                   double *tab, cudaStream_t st);
int launch_grains_init(const rs3_params &p, int precision, uint64_t seed, double z_front, double amp,
                       double c_liquid, double c_solid, void *f1, void *f2, void *fc, cudaStream_t st);

}  // namespace rs

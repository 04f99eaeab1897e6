// rs_ensemble.cuh — per-run descriptor of the batched ensemble: everything the
// FP32 tile kernel takes as launch arguments for one field set, plus the
// run's step state, kept in device memory so that one launch serves every
// run and a CUDA graph of it can be replayed step after step.
#pragma once

#include "rs_step_common.cuh"
#include "rs_surrogate.cuh"

namespace rs {

// Tile shapes of the ensemble kernels: kW = 128 output columns by
// shape_rows(s) output rows (shape 0 is the single-run kernel's 16 x 128).
constexpr int kTileShapes = 3;
__host__ __device__ constexpr int shape_rows(int s) { return s == 1 ? 8 : s == 2 ? 32 : 16; }

struct alignas(64) EnsRun {
  // per tile shape: field sets A (0) and B (1), TMA boxes shape_rows + 2 rows
  // high; current = step & 1
  CUtensorMap map_psi[kTileShapes][2], map_c[kTileShapes][2];
  StepCoef K;
  Coef<float> F;
  float *psi[2], *c[2];
  float *tab;  // the run's column table (rs_step_f32.cu layout)
  int32_t tab_len;
  int32_t nrt[kTileShapes], ntiles[kTileShapes];  // per tile shape: row tiles, tiles
  int32_t active;       // 0: the run is stepped outside the batched launch this step
  int32_t hist;         // i_offset_history
  int32_t hist_init, i_tip_target;
  int32_t pad;
  int64_t step;
  double l, inc_l;      // l_offset_Vp and its per-step increment
  // frozen temperature line (get_delta, fun.cu:1610-1619), evaluated as rs_step does
  double delta_initial, d1, GG, S, W0, deltaT0, l_init;
  SurrArgs surr;  // the run's learned CALPHAD surrogate (surr.w == nullptr: exact)
};

// launches of rs_step_f32.cu for the ensemble: table blocks listed by
// (run, block of that run), tiles in `order` as run << 16 | tile of that run
// surr: every run evaluates its cells through its surrogate (all runs have one)
// shape: the tile shape (0 .. kTileShapes - 1) the order's tile indices refer to
int launch_ensemble(const EnsRun *runs, int nruns, const int32_t *tblk, int ntblk, const int32_t *order, int ntiles,
                    int shape, bool advance, bool surr, int *err, cudaStream_t st);
// the persistent walk: nsteps steps of every run in one cooperative launch;
// lv[s * nruns + r]: l_offset_Vp of run r at step s of the launch (s = 0 ..
// nsteps); bar: two device counters (grid barrier, tile tickets), cleared here
// before the launch; 0 on success
// barrier_limit: polls of a grid-barrier wait before it gives up (0: the default)
int launch_ensemble_walk(EnsRun *runs, int nruns, const int32_t *tblk, int ntblk, const int32_t *order, int ntiles,
                         int shape, int nsteps, const double *lv, bool advance, bool surr, unsigned *bar, int *err,
                         uint32_t barrier_limit, cudaStream_t st);

}  // namespace rs

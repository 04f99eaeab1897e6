/*
 * rs_b200.h — C-ABI of the B200 coupled phase-field time step
 * (Ti–Nb directional solidification, quantitative phase field + CALPHAD).
 *
 * The reference program has no library API: its hot path sits behind the kernel
 * launch sites of the host step loop (src/main.cu:191-233, identical to
 * fun.cu:466-506) with kernel signatures in src/main.hpp:54-83.  Every entry
 * point below replaces one of those launch sites (or one host routine that
 * copies a full field to the host), cited per function.
 *
 * Conventions
 *  - Grid: nx_all x ny_all cells including a one-cell ghost ring; cell (i, j)
 *    lives at  j * pitch + i  (reference pos(i,j) = j*Nx_all + i, fun.cu:176).
 *    i is the growth axis (contiguous), j is periodic (or no-flux).
 *  - The caller owns every field buffer (device memory) and passes a CUDA
 *    stream (a cudaStream_t cast to void*; NULL = legacy default stream).
 *    Launchers never allocate: per-context workspaces come from rs_create.
 *  - Every function returns 0 on success or a negative RS_E* code; the
 *    message of the last failure on the calling thread is rs_last_error().
 *  - One orientation (N_or = 1): the order parameter phi equals
 *    clamp(psi, -1, 1) after every reference step (compute_psi,
 *    fun.cu:1232-1273), so a field set stores psi and c; phi is optional and,
 *    when given, is written as the clamped copy for drop-in callers.
 */
#ifndef RS_B200_H_
#define RS_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RS_ABI_VERSION 9

/* status codes */
#define RS_OK 0
#define RS_E_INVALID (-1)   /* bad argument (sizes, pointers, alignment) */
#define RS_E_CUDA (-2)      /* a CUDA runtime call failed */
#define RS_E_UNSUPPORTED (-3)
#define RS_E_STATE (-4)     /* e.g. a device-side bounded wait gave up */
#define RS_E_IO (-5)        /* file missing, truncated or malformed */

/* field precision tags */
#define RS_F64 0
#define RS_F32 1

typedef void *rs_stream_t; /* cudaStream_t */

/*
 * Run parameters.  Defaults (rs_default_params) are the reference's
 * constants.hpp parameter set (src/constants.hpp:185-350); the macro names of
 * the reference are given beside each field.
 */
typedef struct rs_params {
  /* grid and switches */
  int32_t nx_all;          /* Nx_all (run.sh -DNx_all) */
  int32_t ny_all;          /* Ny_all */
  int32_t i_tip_target;    /* i_tip_target (Nx-268 in the reference) */
  int32_t periodic_j;      /* Periodic: 1 periodic j, 0 no-flux */
  int32_t tfc;             /* ifTFC: 1 coarse-grid temperature, 0 frozen */
  int32_t one_eps;         /* if_1_eps: 1 -> (eps1), 0 -> (eps1, eps2) */
  int32_t vp_ramp;         /* if_Vp_ramp */
  int32_t n_orientation;   /* num_orientation; only 1 is supported */
  /* material (constants.hpp Material namespace) */
  double cinf;             /* nominal Ti mole fraction of the melt */
  double W0;               /* nm */
  double S;                /* SS = W/W0 */
  double Gamma;            /* K nm */
  double muk0;             /* nm/ns/K */
  double Tmelt;            /* K */
  double T_ref;            /* K; deltaT0 = Tmelt - T_ref */
  double Dl;               /* nm^2/ns */
  double DT;               /* nm^2/ns, thermal diffusivity (TFC) */
  double latent_heat;      /* J/mol */
  double molar_weight;     /* g/mol */
  double num_moles;        /* mol/m^3 */
  double cp;               /* J/mol/K */
  double RR;               /* J/mol/K */
  double v0;               /* m^3/mol */
  double AA;               /* interface mobility enhancement (12 for SS=5) */
  double ke;               /* dilute-model partition coefficient (reported only) */
  /* run */
  double dx;               /* grid spacing in units of W */
  double dt;               /* time step in units of tau0; <= 0: set_parameters rule */
  double GG;               /* K/nm, temperature gradient */
  double Vp;               /* m/s, pulling velocity */
  double eps1, eps2, epk1; /* anisotropy strengths */
  double delta_initial;    /* initial dimensionless undercooling at i_tip_target */
  double l_offset_Vp_initial;
  int32_t i_offset_history_initial;
  int32_t ratio_dxT_dx;    /* coarse/fine spacing ratio (TFC), 10 */
  double orientation[9];   /* crystal axes projected on the lab frame */
  /* interface noise (off in the reference; Philox keyed by seed, step, cell) */
  double noise_amplitude;
  uint64_t seed;
  /* TFC */
  double Tcold;            /* K */
  double length_sample_um; /* um, coarse-domain length (50 in fun.cu) */
  /* host-loop cadence (reference set_parameters) */
  double total_time_ns;
  int32_t num_fields_output;
  int32_t num_tip_output;
  int32_t num_check_point_output;
  int32_t step_pull_back;  /* <= 0: derived as in set_parameters */
  /* Row bands of one domain over several devices (the reference's
   * fun_multi.cu splits j the same way).  band = 1: this context holds global
   * rows j_offset .. j_offset + ny_all - 1, its ghost rows 0 and ny_all - 1
   * are supplied by the caller (the neighbouring bands' edge rows), the step
   * does not write them, and the interface noise is keyed by the global row.
   * Frozen temperature only; rs_precise_tip needs the whole domain. */
  int32_t j_offset;
  int32_t band;
} rs_params;

/* Quantities derived from rs_params exactly as set_parameters does
 * (fun.cu:1984-2058) plus the dimensional groups of the macro set. */
typedef struct rs_derived {
  double tau0, deltaT0, a1, W, hh, h0, dt, dtT, length_sample, Thot;
  int64_t total_step;
  int32_t step_fields, step_tip, step_check_point, step_pull_back;
  int32_t ratio_dt_dtT, NxT, NyT, NxT_all, NyT_all, i_left_end_initial;
} rs_derived;

/* A field set on the device.  psi and c are required; phi is optional.
 * RS_F64 sets hold c itself (the reference's layout).  RS_F32 sets hold
 * c - cinf: the offset keeps FP32 updates far below ulp(c) (solute
 * conservation); rs_mass adds cinf back. */
typedef struct rs_fields {
  void *c;
  void *psi;
  void *phi;          /* may be NULL; written as clamp(psi,-1,1) when set */
  int32_t precision;  /* RS_F64 or RS_F32 */
  int32_t pitch;      /* elements per row; 0 means nx_all */
} rs_fields;

/* Per-step arguments: the scalars the reference passes to its kernels by
 * value (fun.cu:466-478) plus the fused moving-frame shift. */
typedef struct rs_step_args {
  int64_t step;
  int32_t i_offset_history; /* accumulated shift, enters the frozen T */
  int32_t pull_back;        /* 1: apply pull_back(i_offset) to cur first */
  int32_t i_offset;         /* shift of this pull-back */
  int32_t i_left_end;       /* TFC: left border of the phase-field window */
  int32_t i_left_end_T;     /* TFC: i_left_end the fine T was interpolated with */
  int32_t reserved;
  double l_offset_Vp;       /* pulled distance in W */
  const void *T_coarse;     /* TFC: coarse T (double, NxT_all x NyT_all) */
  double *mass_out;         /* device-writable (device memory, or the device
                               address of an rs_host_alloc buffer): if set,
                               receives sum of interior c_next */
  int32_t *itip_out;        /* device-writable: if set, receives max i with psi_next>0 */
} rs_step_args;

/* Precise tip (fun.cu:2612-2622 TIP). */
typedef struct rs_tip {
  int32_t i, j;
  int32_t status;   /* fit_parabola status: 0 ok, -2 singular, -3 flat */
  int32_t reserved;
  double x, y, R;
} rs_tip;

typedef struct rs_ctx rs_ctx;

/* ---- library ---- */
int rs_abi_version(void);
const char *rs_last_error(void);
size_t rs_sizeof_params(void);
size_t rs_sizeof_step_args(void);

/* Fill the constants.hpp parameter set (src/constants.hpp:185-350). */
int rs_default_params(rs_params *p);
/* Derived quantities, as set_parameters (fun.cu:1984-2058). */
int rs_derive(const rs_params *p, rs_derived *d);

/* Context: validates parameters, uploads orientation and per-context
 * workspaces (reduction partials, tip rows).  Replaces the cudaMalloc block of
 * main() for everything that is not a caller-owned field (fun.cu:374-409). */
int rs_create(const rs_params *p, rs_ctx **out);
int rs_destroy(rs_ctx *ctx);
int rs_get_derived(const rs_ctx *ctx, rs_derived *d);

/* Options: RS_OPT_TMA (default 1) stages the step's field tiles into shared
 * memory (TMA copies; a pull-back step's shifted tile by a gather), frozen and
 * coarse-grid temperature; 0 selects the register-prefetch kernel (always used
 * for fields whose rows are not 16-byte aligned).
 * RS_OPT_WAIT_LIMIT (default 0: the kernels' own limit of 2^20 suspending
 * tries) bounds the tile kernels' waits for their TMA loads; when set, a wait
 * polls without suspending and gives up after that many polls.  A tile whose
 * wait gives up is not computed or stored, and rs_device_status reports
 * RS_E_STATE.  Tests set it to 1 to run that path.  Set on run 0's context
 * of an ensemble, it also bounds the persistent walk's grid-barrier waits
 * (polls; default 2^22).
 * RS_OPT_PIPELINE (default 0) runs the frozen-temperature tile step (FP64,
 * and FP32 without a surrogate) as a persistent kernel of warp roles (a TMA producer warp, a
 * phase-1 group and a flux/update/store group working on three tiles at
 * once) instead of one tile per CTA; both give the same fields bit for
 * bit. */
#define RS_OPT_TMA 1
#define RS_OPT_WAIT_LIMIT 2
#define RS_OPT_PIPELINE 3
int rs_set_option(rs_ctx *ctx, int32_t option, int64_t value);

/* Device-side waits are bounded: if one gave up since the last call, returns
 * RS_E_STATE (and clears the flag).  Synchronizes the stream. */
int rs_device_status(rs_ctx *ctx, rs_stream_t stream);

/* ---- hot path ---- */
/* One fused time step: pull_back (optional, fun.cu:1469-1492) +
 * compute_phi (fun.cu:1143-1218) + compute_psi (fun.cu:1232-1273) +
 * compute_c_CALPHAD (fun.cu:1365-1467), frozen temperature (get_delta,
 * fun.cu:1610-1619) or on-the-fly interpolated coarse T (TFC,
 * interpolate_temperature fun.cu:1580-1608), ghost cells included.
 * cur and next must not alias.  Replaces the launches at main.cu:191-213. */
int rs_step(rs_ctx *ctx, const rs_fields *cur, const rs_fields *next,
            const rs_step_args *args, rs_stream_t stream);

/* Column shift of the moving frame, standalone form of the pull_back kernel
 * (fun.cu:1469-1492, launched at main.cu:179-181). */
int rs_pull_back(rs_ctx *ctx, const rs_fields *cur, const rs_fields *next,
                 int32_t i_offset, rs_stream_t stream);

/* Coarse tip column: max i (>= 1) with psi > 0 over every row
 * (get_itip_all_grain, fun.cu:1745-1754), reduced on the device into
 * *d_itip instead of copying psi to the host (set_pull_back, fun.cu:697). */
int rs_itip(rs_ctx *ctx, const rs_fields *f, int32_t *d_itip, rs_stream_t stream);

/* Precise tip on the device (get_precise_tip, fun.cu:2895-2954: row scan
 * get_tip_int 2880, quartic fits get_precise_x 2694, parabola fit_parabola
 * 2809).  *d_tip is device memory. */
int rs_precise_tip(rs_ctx *ctx, const rs_fields *f, rs_tip *d_tip, rs_stream_t stream);

/* Precise tip without any device allocation (no counterpart in the
 * reference): same result as rs_precise_tip, for callers that cannot
 * allocate device memory (their device memory belongs to a pool allocator
 * that forbids cudaMalloc once the run starts, or their loop must not take
 * the device-wide synchronisation of cudaMalloc/cudaFree).  Needs no rs_ctx;
 * per-row scratch is a static device array of RS_NOALLOC_TIP_MAX_ROWS rows
 * (320 KiB, held by every GPU that loads the library); larger ny_all is
 * rejected with RS_E_INVALID.  The first call on a device looks up the
 * array's device address and should come before any stream capture; the
 * address is kept for the life of the process, so a cudaDeviceReset of that
 * device leaves it stale (do not call this entry point on a device after
 * resetting it).  All calls share the scratch: calls whose kernels overlap
 * on the GPU race. */
#define RS_NOALLOC_TIP_MAX_ROWS 16384
int rs_precise_tip_noalloc(const rs_params *p, const rs_fields *f, rs_tip *d_tip, rs_stream_t stream);

/* Sum of c over the interior cells in double precision into *d_mass: the
 * numerator of get_average (fun.cu:1756-1766), reduced on the device. */
int rs_mass(rs_ctx *ctx, const rs_fields *f, double *d_mass, rs_stream_t stream);

/* Page-locked host memory mapped into the device's address space (no
 * counterpart in the reference, which copies get_average's inputs to the
 * host): *host and *device address the same zeroed bytes.  Passing
 * device-side addresses of it as rs_step_args.mass_out / itip_out lets the
 * step's reduction write its result straight into host memory, so a host loop
 * reads every step's mass after that step completes (an event or stream
 * synchronisation) without a copy call.  Free with rs_host_free. */
int rs_host_alloc(size_t bytes, void **host, void **device);
int rs_host_free(void *host);

/* ---- initial conditions ---- */
/* Reference initial condition (kernel initial, fun.cu:983-1021): tanh front
 * at i_tip_target + 0.5 sin(2 pi j / Ny), c = cinf (0.3184 tanh + 0.6816). */
int rs_initial(rs_ctx *ctx, const rs_fields *f, rs_stream_t stream);
/* Planar front at i_tip_target + U(-1/2, 1/2) per row j (Philox keyed by
 * seed and j), phi = -tanh((i - i0(j)) dx / sqrt 2), c blended from
 * c_solid (phi = 1) to c_liquid (phi = -1). */
int rs_initial_planar(rs_ctx *ctx, const rs_fields *f, double c_liquid,
                      double c_solid, uint64_t seed, rs_stream_t stream);

/* ---- coarse temperature (TFC) ---- */
/* initial_temperature (fun.cu:1023-1028). T is double, NxT_all x NyT_all. */
int rs_temperature_init(rs_ctx *ctx, double *d_T, rs_stream_t stream);
/* ratio_dt_dtT sub-steps of compute_temperature (fun.cu:1537-1578) on the
 * coarse grid with the latent-heat source dphidt.  T and T_next are swapped
 * internally; the final T is left in d_T. */
int rs_temperature_step(rs_ctx *ctx, double *d_T, double *d_T_next,
                        const double *d_dphidt, int64_t step, rs_stream_t stream);
/* integrate_phi (fun.cu:1494-1535): latent-heat source per coarse cell,
 * 0.5 * sum of (psi_next - psi) over its ratio x ratio fine cells.  When the
 * last rs_step on this context fused a pull-back into its read of cur, psi of
 * cur is read through the same shift, as the reference integrates after its
 * pull_back swap (fun.cu:451-486). */
int rs_integrate_phi(rs_ctx *ctx, const rs_fields *cur, const rs_fields *next,
                     double *d_dphidt, int32_t i_left_end, rs_stream_t stream);
/* interpolate_temperature (fun.cu:1580-1608): bilinear coarse -> fine. */
int rs_interpolate_temperature(rs_ctx *ctx, const double *d_T, double *d_T_fine,
                               int32_t i_left_end, rs_stream_t stream);

/* ---- restart and snapshot files (host only) ---- */
/* Dynamic state recorded in parameters.txt (fields of the reference's
 * constants struct, src/main.hpp:10-53). */
typedef struct rs_run_state {
  int64_t step;
  int32_t i_offset_history;
  int32_t i_left_end_initial;
  int32_t i_left_end;
  int32_t ratio_dt_dtT, NxT, NyT, NxT_all, NyT_all;
  double l_offset_Vp;
  double delta;            /* printed as "delta_initial" (save_parameters prints para->delta) */
  double dt;               /* written: <= 0 means the derived dt; read: the file's %g value */
  double dtT, length_sample, Tcold, Thot;
  double gamma0, gamma1;   /* orientation angles reported in the file (degrees) */
  const char *path_input;  /* reported input path; NULL writes "./" */
} rs_run_state;
/* save_parameters layout (fun.cu:2060-2202). */
int rs_write_parameters(const char *path, const rs_params *p, const rs_run_state *s);
/* load_parameters positional read (fun.cu:2204-2388); tfc: read the TFC block. */
int rs_read_parameters(const char *path, int32_t tfc, rs_run_state *s);
/* check_point_<field>.bin: raw FP64, i fastest (fun.cu:1848-1872, 1894-1918). */
int rs_write_check_point(const char *path, const double *h_field, int32_t nx_all, int32_t ny_all);
int rs_read_check_point(const char *path, double *h_field, int32_t nx_all, int32_t ny_all);
/* check_point_temperature.bin: NyT x NxT of the NxT_all-pitched coarse T
 * (fun.cu:1874-1892, 1946-1971). */
int rs_write_check_point_temperature(const char *path, const double *h_T, int32_t NxT, int32_t NyT, int32_t NxT_all);
int rs_read_check_point_temperature(const char *path, double *h_T, int32_t NxT, int32_t NyT, int32_t NxT_all);
/* <field>_<k>.txt snapshot, "%g\t" per cell (save_field, fun.cu:1768-1790). */
int rs_write_field_text(const char *path, const double *h_field, int32_t nx_all, int32_t ny_all, int32_t di,
                        int32_t dj);

/* ---- learned CALPHAD surrogate (no counterpart in the reference) ----
 * A 3 -> 32 -> 32 -> 2 SiLU network mapping (T, c, phi), scaled to [-1, 1]
 * over a training box, to the two per-cell CALPHAD terms of the FP32 step:
 * the chemical potential relative to the melt's column value (mu'') and the
 * driving force Gl - Gs (fun.cu:1671-1720).  Parameters are one FP32 vector
 * of RS_MLP_NPARAMS: W1[32][3], b1[32], W2[32][32], b2[32], W3[2][32], b3[2].
 * Outputs are scaled: raw = y_mean + y_scale * network output. */
#define RS_MLP_NPARAMS 1250
typedef struct rs_mlp_box {
  double T_lo, T_hi;       /* K */
  double c_lo, c_hi;       /* Ti mole fraction */
  double y_mean[2], y_scale[2];
} rs_mlp_box;
/* n training samples, uniform over the box (Philox keyed by seed and index):
 * d_x[n][3] scaled inputs, d_y[n][2] exact targets (FP64 evaluator, rounded). */
int rs_mlp_sample(const rs_params *p, const rs_mlp_box *box, int64_t n, uint64_t seed, float *d_x, float *d_y,
                  rs_stream_t stream);
/* The same with the third input the interpolation weight itself, g = 2 gS - 1
 * in [-1, 1] (gS the solid weight), for the 3D model's energy 1, where g comes
 * from the Folch-Plapp weights rather than from one phi: x[2] = g and the mu''
 * target uses g where rs_mlp_sample uses gg(phi). */
int rs_mlp_sample_g(const rs_params *p, const rs_mlp_box *box, int64_t n, uint64_t seed, float *d_x, float *d_y,
                    rs_stream_t stream);
/* Adds the gradient of sum over samples of |out - (y - y_mean)/y_scale|^2 to
 * d_grad (not cleared) and the loss to *d_loss (double, not cleared). */
int rs_mlp_grad(const rs_mlp_box *box, const float *d_w, int64_t n, const float *d_x, const float *d_y,
                float *d_grad, double *d_loss, rs_stream_t stream);
/* One Adam step (beta 0.9/0.999, eps 1e-8) on scale * d_grad; t counts from 1. */
int rs_mlp_adam(float *d_w, const float *d_grad, float *d_m, float *d_v, int64_t t, float lr, float scale,
                rs_stream_t stream);
/* FP32 forward pass: d_out[n][2] raw (unscaled) outputs. */
int rs_mlp_forward(const rs_mlp_box *box, const float *d_w, int64_t n, const float *d_x, float *d_out,
                   rs_stream_t stream);
/* Selects the surrogate for the FP32 step of this context (d_w = NULL: the
 * exact evaluation).  The context keeps a copy of the weights (FP16 for the
 * two tensor-core layers, FP32 for the first) and of the box.  The network
 * stands in for the cells outside the exact bulk-melt form; cells whose T or
 * c lie outside the box, and one cell in 1024 per step of those (audit), are
 * evaluated exactly.  Frozen temperature only: RS_E_UNSUPPORTED on a context
 * with the coarse-grid temperature. */
int rs_set_surrogate(rs_ctx *ctx, const float *d_w, const rs_mlp_box *box);
/* Largest |surrogate - exact| of mu'' and dG over the audited cells and the
 * counts of fallback and audited cells since the last call; clears them.
 * Synchronizes the stream. */
int rs_surrogate_audit(rs_ctx *ctx, double *max_err_mu, double *max_err_dG, int64_t *n_fallback,
                       int64_t *n_audit, rs_stream_t stream);

/* ---- batched ensemble (no counterpart in the reference) ----
 * Many independent FP32 runs of uneven size stepped by one launch of the tile
 * kernel over all their tiles (plus one launch for their column tables).
 * Each run has its own context (parameters, frozen temperature, moving frame)
 * and two caller-owned FP32 field sets A and B; A holds the fields at even
 * steps.  Step state lives on the device, so stretches of steps in which no
 * run pulls back are replayed from a CUDA graph; a run's pull-back step
 * (every step_pull_back of its own) is taken by rs_itip + rs_step on its
 * context, as main.cu does.  Runs must use the frozen temperature without
 * the Vp ramp.  Surrogate path: when every run's context has a network set
 * (rs_set_surrogate) before the first rs_ensemble_steps or
 * rs_ensemble_autotune, the batched launch evaluates the cells through each
 * run's network (fallback and audit as in rs_step); a mix of runs with and
 * without one is rejected with RS_E_UNSUPPORTED. */
typedef struct rs_ens rs_ens;
int rs_ensemble_create(const rs_params *params, int32_t nruns, rs_ens **out);
int rs_ensemble_destroy(rs_ens *e);
/* the context of a run (initial conditions, mass, tip, ... of its fields) */
int rs_ensemble_context(rs_ens *e, int32_t run, rs_ctx **ctx);
/* the run's two field sets (FP32, 16-byte aligned, pitch nx_all) */
int rs_ensemble_bind(rs_ens *e, int32_t run, const rs_fields *a, const rs_fields *b);
/* nsteps steps of every run; returns after queueing them on the stream
 * (pull-back steps read one int back) */
int rs_ensemble_steps(rs_ens *e, int64_t nsteps, rs_stream_t stream);
/* a run's step, i_offset_history, l_offset_Vp and current set (0 = A, 1 = B) */
int rs_ensemble_state(rs_ens *e, int32_t run, int64_t *step, int32_t *i_offset_history, double *l_offset_Vp,
                      int32_t *current);
/* Times the stepping paths over reps launches of one step without advancing
 * the runs and keeps the fastest.  Path k uses the tile shape k / 6: 128
 * columns by 16 (shape 0, the single-run kernel's), 8 (shape 1) or 32
 * (shape 2) rows.  Within a shape, k % 6 = 0-2 launch the column tables and
 * the tiles per step (replayed from a CUDA graph) with the tile order 0 run
 * by run, 1 largest runs first, 2 runs interleaved; k % 6 = 3-5 are the same
 * orders as the persistent walk, one cooperative launch per stretch of steps
 * without a pull-back (device-side grid barriers between the tables and the
 * tiles of a step and between steps, bounded: one that gives up sets the
 * status rs_device_status reports on run 0's context).  ms_out[RS_ENS_PATHS]
 * receives the mean times, *choice the path. */
#define RS_ENS_PATHS 18
int rs_ensemble_autotune(rs_ens *e, int32_t reps, double *ms_out, int32_t *choice, rs_stream_t stream);
/* selects a stepping path (0 .. RS_ENS_PATHS - 1, as rs_ensemble_autotune
 * numbers them) */
int rs_ensemble_set_path(rs_ens *e, int32_t path);

/* ---- 3D three-phase variant (one GPU) ----
 * The reference's 3D peritectic model, multi/peritectic_multiGPU/TiAg.cu:
 * two stored order parameters phi1 (liquid) and phi2 (solid alpha), the
 * third phase phi3 = 1 - phi1 - phi2 (solid beta), the diffusion potential
 * mu = c - sum_i r_i g_i(phi) (computeMu, TiAg.cu:461-470) and the explicit
 * update of phi1, phi2 and c (diffuse, TiAg.cu:503-561), with periodic x, y
 * and no-flux z ghost layers (the boundaryMu and boundary kernels,
 * TiAg.cu:472-500, 565-605).  Cell (x, y, z) lives at (z * ny + y) * nx + x (TiAg.cu pos).
 * One domain on one GPU: the reference's z-slab exchange between GPUs
 * (TiAg.cu:279-331) has no counterpart.
 * Extension beyond the reference: a frozen temperature
 *   T(z, step) = T_ref + G_T (z - z_T - V_T step)
 * enters through B1(T) = B11 + B12 T, B2(T) = B21 + B22 T (TiAg.cu:61-62);
 * G_T = 0 is the reference's isothermal model.
 *
 * energy = 1: the Ti-Nb CALPHAD free energy of the 2D model (fun.cu:1628-1720)
 * on the same three-phase structure (no counterpart in the reference, whose
 * 3D program has no CALPHAD).  The database has one solid phase, BCC, so
 * phases 2 and 3 are two BCC grains.  c is the Ti mole fraction, T (K) the
 * frozen line above with T_ref in K and G_T in K per cell, and per cell
 *   mu  = g1 Glc(T, c) + (1 - g1) Gsc(T, c)         (fun.cu:1443-1452, 1700-1720)
 *   dG  = Gl(T, c) - Gs(T, c)                       (fun.cu:1192-1193, 1671-1698)
 * with g1 the liquid's Folch-Plapp weight.  dG is the grand-potential
 * difference of the liquid against both grains: lambda dG takes the place of
 * TiAg's lambda (s_1 - r_1 mu) - lambda (s_j - r_j mu), so lambda is the
 * coupling per J/mol (1 / (2 hh v0) of the 2D model gives its phase equation
 * in the two-phase limit).  The solute update is
 *   c' = c + dt alpha sum_faces (S + S')/2 (mu' - mu) / dx^2,
 *   S  = [q(phi1) + Da phi2 + Db phi3] c (1 - c),  q(p) = p (AA - (AA - 1) p)
 * (fun.cu:1424-1464 with the liquid fraction phi1 for (1 - psi)/2), alpha the
 * solute coefficient per J/mol (Dl / (Gamma muk0 h0 v0) of the 2D model). */
typedef struct rs3_params {
  int32_t nx, ny, nz;               /* extents incl. ghost layers (TiAg Nx, Ny, devNz) */
  int32_t z_chunk;                  /* planes per CTA of the z march (0: 32) */
  double dt;                        /* DT */
  double dx_inv, dy_inv, dz_inv;    /* DXin, DYin, DZin */
  double a1, a2, a3, b;             /* three-phase well terms */
  double lambda, alpha, Da, Db;     /* coupling, diffusivity, solid diffusivities */
  double A1, A2, B11, B12, B21, B22;
  double T_ref;                     /* T of TiAg.cu (60 * 0.000321787) */
  double G_T;                       /* dT per cell along z */
  double V_T;                       /* isotherm speed, cells per step */
  double z_T;                       /* plane where T = T_ref at step 0 */
  int32_t energy;                   /* 0 TiAg.cu's grand potentials; 1 Ti-Nb CALPHAD (above) */
  int32_t reserved;
  double AA;                        /* energy 1: interface mobility enhancement of q */
  double RR;                        /* energy 1: gas constant, J/mol/K */
  double c_ref;                     /* energy 1: Ti fraction of the melt; FP32 sets hold c - c_ref */
} rs3_params;

/* A 3D field set on the device (nx * ny * nz elements each, 16-byte aligned).
 * RS_F64 sets hold c itself; RS_F32 sets hold c - rs3_c_offset() (the melt's
 * composition clb at T_ref), which keeps the melt's small solute updates
 * above FP32 rounding.  rs3_mu and rs3_mass return true mu and sum c. */
typedef struct rs3_fields {
  void *phi1;
  void *phi2;
  void *c;
  int32_t precision; /* RS_F64 or RS_F32 */
  int32_t reserved;
} rs3_fields;

typedef struct rs3_ctx rs3_ctx;

/* TiAg.cu's constants (TiAg.cu:19-62) on a 512 x 512 x 128 domain, isothermal */
int rs3_default_params(rs3_params *p);
size_t rs3_sizeof_params(void);
int rs3_create(const rs3_params *p, rs3_ctx **out);
int rs3_destroy(rs3_ctx *ctx);
/* One step (TiAg.cu:269-340): computeMu, boundaryMu, diffuse, boundary,
 * fused into one launch: next = step(cur), ghost layers included. */
int rs3_step(rs3_ctx *ctx, const rs3_fields *cur, const rs3_fields *next, int64_t step, rs_stream_t stream);
/* mu of every cell, ghost layers as images (computeMu + boundaryMu);
 * d_mu has the set's precision; energy 1: the CALPHAD mu (J/mol) at the
 * temperature of step 0 */
int rs3_mu(rs3_ctx *ctx, const rs3_fields *f, void *d_mu, rs_stream_t stream);
/* FP64 sum of c over the interior (the avg_c numerator, TiAg.cu:237-249) */
int rs3_mass(rs3_ctx *ctx, const rs3_fields *f, double *d_mass, rs_stream_t stream);
/* Initial state: solid beta below the plane z_front + U(-amp, amp) (one
 * seeded draw per (x, y) column), liquid above, and n_alpha spherical alpha
 * caps of base radius cap_radius and contact angle 1.33 rad on the front at
 * seeded (x, y) positions (the cap shape of TiAg.cu initial, 400-444).
 * Compositions are the model's own equilibrium values at T_ref (TiAg.cu ca,
 * cb, clb): beta cb, alpha ca, liquid clb.  Ghost layers are images. */
int rs3_initial(rs3_ctx *ctx, const rs3_fields *f, double z_front, double amp, int32_t n_alpha,
                double cap_radius, uint64_t seed, rs_stream_t stream);
/* Initial state of two grains: below the plane z_front + U(-amp, amp) (one
 * seeded draw per (x, y) column) solid of composition c_solid, phase 2 for
 * x <= (nx - 2) / 2 and phase 3 beyond; melt of composition c_liquid above.
 * Ghost layers are images. */
int rs3_initial_grains(rs3_ctx *ctx, const rs3_fields *f, double z_front, double amp, double c_liquid,
                       double c_solid, uint64_t seed, rs_stream_t stream);
/* the offset of c in RS_F32 sets: clb at T_ref (TiAg.cu:67); c_ref for energy 1 */
int rs3_c_offset(const rs3_params *p, double *out);
/* RS_E_STATE if a step kernel's bounded wait for a plane load gave up */
int rs3_device_status(rs3_ctx *ctx, rs_stream_t stream);
/* Energy 1, FP32 sets: the learned CALPHAD surrogate (trained on samples of
 * rs_mlp_sample_g with cinf = c_ref) in place of the per-cell evaluation of
 * mu'' and dG of every cell that is not bulk melt (phi1 = 1 exactly, which
 * keeps its exact series form); out-of-box cells and one in 1024 per step of
 * the others (audit) are evaluated exactly.  d_w = NULL: the exact path. */
int rs3_set_surrogate(rs3_ctx *ctx, const float *d_w, const rs_mlp_box *box);
/* as rs_surrogate_audit */
int rs3_surrogate_audit(rs3_ctx *ctx, double *max_err_mu, double *max_err_dG, int64_t *n_fallback,
                        int64_t *n_audit, rs_stream_t stream);

/* ---- host-side helpers (no device work) ---- */
/* CALPHAD Ti-Nb evaluator (fun.cu:1628-1720), host build of the same code
 * the kernels use.  which: 0 Gl, 1 Gs, 2 Glc, 3 Gsc. */
int rs_calphad_eval(int32_t which, const double *T, const double *c, double *out, size_t n);

#ifdef __cplusplus
}
#endif
#endif /* RS_B200_H_ */

// rs_capi.cu — the extern "C" boundary (include/rs_b200.h).
//
// Parameter defaults are the reference's constants.hpp set
// (src/constants.hpp:185-350); derived quantities follow set_parameters
// (fun.cu:1984-2058).  Contexts own only small workspaces (reduction partials,
// per-row tip data) allocated at creation; no launcher allocates.
#include <cudaTypedefs.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>
#include <algorithm>

#include "rs_ensemble.cuh"
#include "rs_mlp.cuh"
#include "rs_surrogate.cuh"

namespace {

thread_local char g_err[512] = "";

int fail(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

int cuda_check(const char *what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(RS_E_CUDA, "%s: %s", what, cudaGetErrorString(e));
  return RS_OK;
}

}  // namespace

namespace rs {
// lets other translation units of the library report through rs_last_error()
int set_error(int code, const char *msg) { return fail(code, "%s", msg); }
}  // namespace rs

struct TmaEntry {
  const void *ptr;
  int precision;
  int rows;  // box height
  CUtensorMap map;
};

struct rs_ctx {
  rs_params p;
  rs_derived d;
  rs::StepCoef K;
  rs::TfcCoef T;
  int device;
  rs::BlockPartial *partials;
  int max_partials;
  int *row_last;
  double *row_f, *row_g;
  int *d_err;          // set by a device-side bounded wait that gave up
  const void *pb_cur;  // psi of the cur set of the last rs_step that fused a pull-back
  int32_t pb_offset;   // and its shift (read by rs_integrate_phi)
  float *col_tab;      // per-column CALPHAD table of the FP32 TMA kernel
  int col_tab_len;
  double *col_tab64;   // and of the FP64 TMA kernel
  int col_tab64_len;
  rs::SurrArgs surr;   // learned CALPHAD surrogate of the FP32 step (surr.w == nullptr: exact)
  float *mlp_w;        // its FP32 parameters (device)
  uint16_t *mlp_b16;   // FP16 W2 (32 x 32) and W3 padded to 8 rows (device)
  unsigned long long *mlp_audit;  // max error bits of mu'' and dG, fallback and audit counts
  unsigned int *red_counter;  // fused final reduction of the FP32 tile kernel (device, 0 between launches)
  int use_tma;         // RS_OPT_TMA
  uint32_t wait_limit; // RS_OPT_WAIT_LIMIT (0: the kernels' default)
  int pipeline;        // RS_OPT_PIPELINE
  TmaEntry tma[8];     // tensor-map cache keyed by field pointer
  int tma_n, tma_next;
};

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  });
  return fn;
}

// 2D tiled descriptor of one field (row pitch = nx_all elements), box of
// kTmaBoxW32/64 x kTmaBoxH elements, zero fill outside the array.  Returns false
// when TMA cannot be used (alignment, driver entry point).
// box_rows: the box height (input rows of a tile)
bool encode_map(const rs_params &p, const void *ptr, int precision, int box_rows, CUtensorMap *out) {
  auto enc = encode_fn();
  const size_t es = precision == RS_F64 ? 8 : 4;
  const uint64_t row_bytes = (uint64_t)p.nx_all * es;
  if (!enc || ((uintptr_t)ptr % 16) || (row_bytes % 16)) return false;
  cuuint64_t dims[2] = {(cuuint64_t)p.nx_all, (cuuint64_t)p.ny_all};
  cuuint64_t strides[1] = {row_bytes};
  cuuint32_t box[2] = {(cuuint32_t)(precision == RS_F64 ? rs::kTmaBoxW64 : rs::kTmaBoxW32), (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  const CUresult r = enc(out, precision == RS_F64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                         2, const_cast<void *>(ptr), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// box_rows: kTmaBoxH, or kTfcTileRows32 + 2 for FP32 coarse-grid-temperature steps
bool field_map(rs_ctx *c, const void *ptr, int precision, int box_rows, CUtensorMap *out) {
  for (int k = 0; k < c->tma_n; ++k)
    if (c->tma[k].ptr == ptr && c->tma[k].precision == precision && c->tma[k].rows == box_rows) {
      *out = c->tma[k].map;
      return true;
    }
  CUtensorMap m;
  if (!encode_map(c->p, ptr, precision, box_rows, &m)) return false;
  TmaEntry &e = c->tma[c->tma_next];
  e.ptr = ptr;
  e.precision = precision;
  e.rows = box_rows;
  e.map = m;
  c->tma_next = (c->tma_next + 1) % 8;
  if (c->tma_n < 8) ++c->tma_n;
  *out = m;
  return true;
}

}  // namespace

extern "C" {

int rs_abi_version(void) { return RS_ABI_VERSION; }
const char *rs_last_error(void) { return g_err; }
size_t rs_sizeof_params(void) { return sizeof(rs_params); }
size_t rs_sizeof_step_args(void) { return sizeof(rs_step_args); }

int rs_default_params(rs_params *p) {
  if (!p) return fail(RS_E_INVALID, "rs_default_params: null");
  memset(p, 0, sizeof(*p));
  // Simulation namespace (constants.hpp:253-350)
  p->nx_all = 768;
  p->ny_all = 832;
  p->i_tip_target = 768 - 268;
  p->periodic_j = 1;        // boundaryCondition 0
  p->tfc = 1;               // ifTFC 1 (main.cu:17)
  p->one_eps = 1;           // if_1_eps
  p->vp_ramp = 0;           // if_Vp_ramp
  p->n_orientation = 1;
  // Material namespace (constants.hpp:185-237)
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
  p->AA = 12.0;             // SS == 5
  p->ke = 0.8146631243899296;
  p->dx = 0.6;              // SS == 5
  p->dt = 0.0;
  p->GG = 10 * 0.001;
  p->Vp = 1.0;
  p->eps1 = 0.06;
  p->eps2 = 0.0;
  p->epk1 = 0.15;
  p->delta_initial = -1.0;
  p->ratio_dxT_dx = 10;
  p->orientation[0] = p->orientation[4] = p->orientation[8] = 1.0;  // Euler angles 0
  p->Tcold = 2000.0;
  p->length_sample_um = 50.0;
  p->total_time_ns = 120.0 * 1000.0;
  p->num_fields_output = p->num_tip_output = p->num_check_point_output = 120;
  return RS_OK;
}

int rs_derive(const rs_params *p, rs_derived *d) {
  if (!p || !d) return fail(RS_E_INVALID, "rs_derive: null");
  memset(d, 0, sizeof(*d));
  const double SS = p->S, W0 = p->W0, dx = p->dx;
  d->W = SS * W0;
  d->tau0 = (SS * W0) * (SS * W0) / (p->Gamma * p->muk0);
  d->deltaT0 = p->Tmelt - p->T_ref;
  d->a1 = 2.0 * std::sqrt(2.0) / 3.0;
  const double latentHeat2 = p->latent_heat * p->num_moles;
  const double surface_tension = p->Gamma * 1e-9 * latentHeat2 / p->Tmelt;
  d->hh = surface_tension / (d->a1 * SS * W0 * 1.0e-9);
  d->h0 = p->RR * p->Tmelt / p->v0;
  const double DD = p->Dl * d->tau0 / ((SS * W0) * (SS * W0));
  double dt = p->dt;
  if (!(dt > 0)) {
    dt = 0.6 * dx * dx / (4.0 * DD);
    if (dt > 0.6 * dx * dx / 4.0) dt = 0.6 * dx * dx / 4.0;
  }
  d->dt = dt;
  const double tau0 = d->tau0;
  d->total_step = (int64_t)(p->total_time_ns / (tau0 * dt));
  if (p->num_fields_output > 0) d->step_fields = (int32_t)(p->total_time_ns / p->num_fields_output / (tau0 * dt));
  if (p->num_tip_output > 0) d->step_tip = (int32_t)(p->total_time_ns / p->num_tip_output / (tau0 * dt));
  if (p->num_check_point_output > 0)
    d->step_check_point = (int32_t)(p->total_time_ns / p->num_check_point_output / (tau0 * dt));
  if (p->step_pull_back > 0)
    d->step_pull_back = p->step_pull_back;
  else if (p->vp_ramp)
    d->step_pull_back = (int32_t)(SS * W0 * dx / (1.0 * dt * tau0));
  else
    d->step_pull_back = (int32_t)(SS * W0 * dx / (p->Vp * dt * tau0));
  const int r = p->ratio_dxT_dx > 0 ? p->ratio_dxT_dx : 10;
  const double DDT = p->DT * tau0 / ((SS * W0 * r) * (SS * W0 * r));
  const double dtT = 0.9 * dx * dx / (4.0 * DDT);
  int ratio = 1;
  if (dtT < dt) ratio = (int)std::ceil(dt / dtT);
  d->ratio_dt_dtT = ratio;
  d->dtT = dt / ratio;
  d->length_sample = std::ceil(p->length_sample_um * 1000 / (dx * SS * W0 * r)) * (dx * SS * W0 * r);
  d->NxT = (int32_t)(d->length_sample / (dx * SS * W0 * r) + 2);
  d->NxT_all = (int32_t)(std::ceil(1.0 * d->NxT / 64) * 64);
  d->NyT = ((p->ny_all - 2) / r) + 2;
  d->NyT_all = (int32_t)(std::ceil(1.0 * d->NyT / 4) * 4);
  d->Thot = p->Tcold + p->GG * d->length_sample;
  d->i_left_end_initial =
      (int32_t)((p->Tmelt - d->deltaT0 - p->Tcold) / (p->GG * dx * SS * W0) - p->i_tip_target);
  return RS_OK;
}

static int validate_params(const rs_params *p) {
  if (p->n_orientation != 1) return fail(RS_E_UNSUPPORTED, "n_orientation=%d: only one orientation is supported", p->n_orientation);
  if (p->nx_all < 8 || p->ny_all < 8) return fail(RS_E_INVALID, "grid %dx%d: need at least 8x8 cells", p->nx_all, p->ny_all);
  if ((int64_t)p->nx_all * p->ny_all > (int64_t)1 << 31)
    return fail(RS_E_INVALID, "grid %dx%d exceeds 2^31 cells", p->nx_all, p->ny_all);
  if (!(p->dx > 0) || !(p->W0 > 0) || !(p->S > 0) || !(p->Gamma > 0) || !(p->muk0 > 0) || !(p->v0 > 0))
    return fail(RS_E_INVALID, "non-positive material or grid constant");
  if (!(p->cinf > 0 && p->cinf < 1)) return fail(RS_E_INVALID, "cinf=%g outside (0,1)", p->cinf);
  if (p->tfc && p->ratio_dxT_dx < 1) return fail(RS_E_INVALID, "ratio_dxT_dx=%d", p->ratio_dxT_dx);
  if (p->band && p->tfc) return fail(RS_E_UNSUPPORTED, "band mode: frozen temperature only");
  if (p->band < 0 || p->band > 1 || p->j_offset < 0) return fail(RS_E_INVALID, "band=%d j_offset=%d", p->band, p->j_offset);
  for (int k = 0; k < 9; ++k)
    if (!std::isfinite(p->orientation[k])) return fail(RS_E_INVALID, "orientation[%d] not finite", k);
  return RS_OK;
}

static void make_coef(const rs_params *p, const rs_derived *d, rs::StepCoef *K, rs::TfcCoef *T) {
  memset(K, 0, sizeof(*K));
  K->nx = p->nx_all;
  K->ny = p->ny_all;
  K->pitch = p->nx_all;
  K->jmin = p->band ? -1 : (p->periodic_j ? p->ny_all - 2 : 1);  // band: ghost rows come from the caller
  K->jmax = p->band ? -1 : (p->periodic_j ? 1 : p->ny_all - 2);
  K->j_offset = p->band ? p->j_offset : 0;
  K->one_eps = p->one_eps;
  K->tfc = p->tfc;
  K->ratio = p->ratio_dxT_dx;
  K->NxT_all = d->NxT_all;
  K->NyT_all = d->NyT_all;
  const double dx = p->dx;
  K->dx = dx;
  K->inv_2dx = 1.0 / (2.0 * dx);
  K->inv_dx2 = 1.0 / (dx * dx);
  K->inv_4dx2 = 1.0 / (4. * dx * dx);
  K->inv_2dx2 = 1.0 / (2.0 * dx * dx);
  K->dt = d->dt;
  K->eps1 = p->eps1;
  K->eps2 = p->eps2;
  K->epk1 = p->epk1;
  K->ox1 = p->orientation[0];
  K->ox2 = p->orientation[1];
  K->oy1 = p->orientation[3];
  K->oy2 = p->orientation[4];
  K->oz1 = p->orientation[6];
  K->oz2 = p->orientation[7];
  K->drive = 1.0 / (2.0 * d->hh * p->v0);
  K->inv_h0v0 = 1.0 / (d->h0 * p->v0);
  K->cfac = d->dt * p->Dl / (p->Gamma * p->muk0) / (dx * dx);
  K->AA = p->AA;
  K->RR = p->RR;
  K->cinf = p->cinf;
  K->Tmelt = p->Tmelt;
  K->deltaT0 = d->deltaT0;
  K->dxT = dx * p->ratio_dxT_dx;
  K->noise_amp = p->noise_amplitude > 0 ? p->noise_amplitude * std::sqrt(d->dt) : 0.0;
  K->seed_lo = (uint32_t)p->seed;
  K->seed_hi = (uint32_t)(p->seed >> 32);
  K->W0 = p->W0;
  K->S = p->S;
  K->Lref = std::log(p->cinf / (1.0 - p->cinf));

  memset(T, 0, sizeof(*T));
  T->nx = p->nx_all;
  T->ny = p->ny_all;
  T->pitch = p->nx_all;
  T->ratio = p->ratio_dxT_dx;
  T->NxT = d->NxT;
  T->NyT = d->NyT;
  T->NxT_all = d->NxT_all;
  T->NyT_all = d->NyT_all;
  T->jTmin = p->periodic_j ? d->NyT - 2 : 1;
  T->jTmax = p->periodic_j ? 1 : d->NyT - 2;
  T->ratio_dt_dtT = d->ratio_dt_dtT;
  T->Sint = (int32_t)p->S;
  T->Tcold = p->Tcold;
  T->Thot = d->Thot;
  T->dx = dx;
  T->dxT = dx * p->ratio_dxT_dx;
  T->dtT = d->dtT;
  T->Lcp = p->latent_heat / p->cp;
  T->W0 = p->W0;
  T->GG = p->GG;
  T->S = p->S;
  T->DT = p->DT;
  T->Gmuk = p->Gamma * p->muk0;
}

int rs_create(const rs_params *p, rs_ctx **out) {
  if (!p || !out) return fail(RS_E_INVALID, "rs_create: null argument");
  *out = nullptr;
  int rc = validate_params(p);
  if (rc) return rc;
  rs_ctx *c = new (std::nothrow) rs_ctx;
  if (!c) return fail(RS_E_INVALID, "rs_create: out of host memory");
  memset(c, 0, sizeof(*c));
  c->p = *p;
  rs_derive(p, &c->d);
  make_coef(&c->p, &c->d, &c->K, &c->T);
  if (cudaGetDevice(&c->device) != cudaSuccess) {
    delete c;
    return fail(RS_E_CUDA, "rs_create: no CUDA device");
  }
  const int ni = p->nx_all - 2, nj = p->ny_all - 2;
  c->max_partials = ((ni + 31) / 32) * ((nj + 7) / 8) + (p->ny_all + 7) / 8 + 64;
  cudaError_t e = cudaMalloc(&c->partials, sizeof(rs::BlockPartial) * c->max_partials);
  if (e == cudaSuccess) e = cudaMalloc(&c->row_last, sizeof(int) * p->ny_all);
  if (e == cudaSuccess) e = cudaMalloc(&c->row_f, sizeof(double) * p->ny_all);
  if (e == cudaSuccess) e = cudaMalloc(&c->row_g, sizeof(double) * p->ny_all);
  if (e == cudaSuccess) e = cudaMalloc(&c->d_err, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(c->d_err, 0, sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&c->red_counter, sizeof(unsigned int));
  if (e == cudaSuccess) e = cudaMemset(c->red_counter, 0, sizeof(unsigned int));
  c->col_tab_len = rs::col_tab_len(p->nx_all);
  if (e == cudaSuccess) e = cudaMalloc(&c->col_tab, sizeof(float) * rs::kColTabFields * c->col_tab_len);
  c->col_tab64_len = rs::col_tab64_len(p->nx_all);
  if (e == cudaSuccess) e = cudaMalloc(&c->col_tab64, sizeof(double) * rs::kColTabFields * c->col_tab64_len);
  c->use_tma = 1;
  if (e != cudaSuccess) {
    rs_destroy(c);
    return fail(RS_E_CUDA, "rs_create: cudaMalloc: %s", cudaGetErrorString(e));
  }
  *out = c;
  return RS_OK;
}

int rs_destroy(rs_ctx *c) {
  if (!c) return RS_OK;
  cudaFree(c->partials);
  cudaFree(c->row_last);
  cudaFree(c->row_f);
  cudaFree(c->row_g);
  cudaFree(c->d_err);
  cudaFree(c->red_counter);
  cudaFree(c->col_tab);
  cudaFree(c->col_tab64);
  cudaFree(c->mlp_w);
  cudaFree(c->mlp_b16);
  cudaFree(c->mlp_audit);
  delete c;
  return RS_OK;
}

int rs_get_derived(const rs_ctx *c, rs_derived *d) {
  if (!c || !d) return fail(RS_E_INVALID, "rs_get_derived: null");
  *d = c->d;
  return RS_OK;
}

static int check_fields(const rs_ctx *c, const rs_fields *f, const char *what, bool need_c = true) {
  if (!f) return fail(RS_E_INVALID, "%s: null field set", what);
  if (f->precision != RS_F64 && f->precision != RS_F32)
    return fail(RS_E_INVALID, "%s: precision tag %d", what, f->precision);
  if (!f->psi || (need_c && !f->c)) return fail(RS_E_INVALID, "%s: psi and c are required", what);
  const int pitch = f->pitch ? f->pitch : c->p.nx_all;
  if (pitch != c->p.nx_all) return fail(RS_E_UNSUPPORTED, "%s: pitch %d != nx_all %d", what, pitch, c->p.nx_all);
  const size_t al = f->precision == RS_F64 ? 8 : 4;
  if (((uintptr_t)f->psi | (uintptr_t)f->c | (uintptr_t)f->phi) % al)
    return fail(RS_E_INVALID, "%s: misaligned field pointer", what);
  return RS_OK;
}

static rs::StepScalars step_scalars(const rs_ctx *c, const rs_step_args *a, const rs_fields *cur) {
  const rs_params &p = c->p;
  rs::StepScalars P;
  memset(&P, 0, sizeof(P));
  P.step = a->step;
  // get_delta (fun.cu:1610-1619): delta(i) = d0 + d1 i
  const double d1 = p.GG * p.dx * p.S * p.W0 / c->d.deltaT0;
  P.d1 = d1;
  P.d0 = p.delta_initial + d1 * (double)(-p.i_tip_target + a->i_offset_history - p.i_offset_history_initial) -
         p.GG * (a->l_offset_Vp - p.l_offset_Vp_initial) * p.S * p.W0 / c->d.deltaT0;
  P.pull_back = a->pull_back ? 1 : 0;
  P.i_offset = a->i_offset;
  P.i_left_end_T = a->i_left_end_T;
  P.i_front = p.i_tip_target;
  P.wait_limit = c->wait_limit;
  P.T_coarse = (const double *)a->T_coarse;
  P.src_psi = cur->psi;
  P.src_c = cur->c;
  return P;
}

int rs_step(rs_ctx *c, const rs_fields *cur, const rs_fields *next, const rs_step_args *a, rs_stream_t stream) {
  if (!c || !a) return fail(RS_E_INVALID, "rs_step: null argument");
  int rc = check_fields(c, cur, "rs_step cur");
  if (!rc) rc = check_fields(c, next, "rs_step next");
  if (rc) return rc;
  if (cur->precision != next->precision) return fail(RS_E_INVALID, "rs_step: cur/next precision differ");
  if (cur->psi == next->psi || cur->c == next->c || (next->phi && (next->phi == cur->psi || next->phi == cur->c)))
    return fail(RS_E_INVALID, "rs_step: cur and next alias");
  if (c->p.tfc && !a->T_coarse) return fail(RS_E_INVALID, "rs_step: TFC needs T_coarse");
  const rs::StepScalars P = step_scalars(c, a, cur);
  cudaStream_t st = (cudaStream_t)stream;
  c->pb_cur = a->pull_back ? cur->psi : nullptr;
  c->pb_offset = a->pull_back ? a->i_offset : 0;
  const bool red = a->mass_out || a->itip_out;
  int nb = 0;
  int lr;
  rs::TmaMaps tm;
  const rs::TmaMaps *tmp = nullptr;
  // the TMA kernels store whole rows by 16-byte bulk copies
  const uintptr_t vec = 16;
  const bool out_aligned =
      ((uintptr_t)next->psi % vec) == 0 && ((uintptr_t)next->c % vec) == 0 && ((uintptr_t)next->phi % vec) == 0;
  const int box_rows = c->p.tfc && cur->precision == RS_F32 ? rs::kTfcTileRows32 + 2 : rs::kTmaBoxH;
  if (c->use_tma && out_aligned && field_map(c, cur->psi, cur->precision, box_rows, &tm.psi) &&
      field_map(c, cur->c, cur->precision, box_rows, &tm.c)) {
    tm.col_tab = c->col_tab;
    tm.col_tab_len = c->col_tab_len;
    tm.col_tab64 = c->col_tab64;
    tm.col_tab64_len = c->col_tab64_len;
    tm.surr = c->surr.w && cur->precision == RS_F32 ? &c->surr : nullptr;
    tm.pipeline = c->pipeline;
    tm.red = {};
    if (red) {  // both tile kernels reduce their partials themselves
      tm.red.counter = c->red_counter;
      tm.red.mass_offset =
          cur->precision == RS_F32 ? (double)(c->p.nx_all - 2) * (c->p.ny_all - 2) * c->p.cinf : 0.0;
      tm.red.mass_out = a->mass_out;
      tm.red.itip_out = a->itip_out;
    }
    tmp = &tm;
  }
  if (cur->precision == RS_F64)
    lr = rs::launch_step_f64(c->K, P, (const double *)cur->psi, (const double *)cur->c, (double *)next->psi,
                             (double *)next->c, (double *)next->phi, red ? c->partials : nullptr,
                             c->max_partials, &nb, tmp, c->d_err, st);
  else
    lr = rs::launch_step_f32(c->K, P, (const float *)cur->psi, (const float *)cur->c, (float *)next->psi,
                             (float *)next->c, (float *)next->phi, red ? c->partials : nullptr,
                             c->max_partials, &nb, tmp, c->d_err, st);
  if (lr == -3) return fail(RS_E_CUDA, "rs_step: cannot configure shared memory of the TMA kernel");
  if (lr) return fail(RS_E_INVALID, "rs_step: grid too large for the reduction workspace");
  if ((rc = cuda_check("rs_step"))) return rc;
  // (the tile kernels reduce their partials themselves)
  if (red && !tmp) {
    const double off = cur->precision == RS_F32 ? (double)(c->p.nx_all - 2) * (c->p.ny_all - 2) * c->p.cinf : 0.0;
    rs::launch_reduce_partials(c->partials, nb, off, a->mass_out, a->itip_out, st);
    if ((rc = cuda_check("rs_step reduce"))) return rc;
  }
  return RS_OK;
}

int rs_set_option(rs_ctx *c, int32_t option, int64_t value) {
  if (!c) return fail(RS_E_INVALID, "rs_set_option: null ctx");
  switch (option) {
    case RS_OPT_TMA:
      c->use_tma = value ? 1 : 0;
      return RS_OK;
    case RS_OPT_PIPELINE:
      c->pipeline = value ? 1 : 0;
      return RS_OK;
    case RS_OPT_WAIT_LIMIT:
      if (value < 0 || value > (int64_t)1 << 30) return fail(RS_E_INVALID, "rs_set_option: wait limit %lld", (long long)value);
      c->wait_limit = (uint32_t)value;
      return RS_OK;
    default:
      return fail(RS_E_INVALID, "rs_set_option: unknown option %d", option);
  }
}

int rs_host_alloc(size_t bytes, void **host, void **device) {
  if (!host || !device || !bytes) return fail(RS_E_INVALID, "rs_host_alloc: bad argument");
  *host = *device = nullptr;
  void *h = nullptr, *d = nullptr;
  cudaError_t e = cudaHostAlloc(&h, bytes, cudaHostAllocMapped | cudaHostAllocPortable);
  if (e == cudaSuccess) {
    e = cudaHostGetDevicePointer(&d, h, 0);
    if (e != cudaSuccess) cudaFreeHost(h);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(RS_E_CUDA, "rs_host_alloc: %s", cudaGetErrorString(e));
  }
  memset(h, 0, bytes);
  *host = h;
  *device = d;
  return RS_OK;
}

int rs_host_free(void *host) {
  if (!host) return RS_OK;
  const cudaError_t e = cudaFreeHost(host);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(RS_E_CUDA, "rs_host_free: %s", cudaGetErrorString(e));
  }
  return RS_OK;
}

int rs_device_status(rs_ctx *c, rs_stream_t stream) {
  if (!c) return fail(RS_E_INVALID, "rs_device_status: null ctx");
  int h = 0;
  cudaStream_t st = (cudaStream_t)stream;
  if (cudaMemcpyAsync(&h, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return cuda_check("rs_device_status");
  if (h) {
    cudaMemsetAsync(c->d_err, 0, sizeof(int), st);
    cudaMemsetAsync(c->red_counter, 0, sizeof(unsigned int), st);  // an aborted launch may have left it counting
    return fail(RS_E_STATE, "a device-side wait gave up (pipeline stalled); results of the affected steps are invalid");
  }
  return RS_OK;
}

int rs_pull_back(rs_ctx *c, const rs_fields *cur, const rs_fields *next, int32_t i_offset, rs_stream_t stream) {
  if (!c) return fail(RS_E_INVALID, "rs_pull_back: null ctx");
  int rc = check_fields(c, cur, "rs_pull_back cur");
  if (!rc) rc = check_fields(c, next, "rs_pull_back next");
  if (rc) return rc;
  if (cur->precision != next->precision) return fail(RS_E_INVALID, "rs_pull_back: precision differs");
  if (cur->psi == next->psi || cur->c == next->c) return fail(RS_E_INVALID, "rs_pull_back: cur and next alias");
  rs::launch_pull_back(cur->precision, c->K, cur->c, cur->psi, cur->phi, next->c, next->psi, next->phi, i_offset,
                       (cudaStream_t)stream);
  return cuda_check("rs_pull_back");
}

int rs_itip(rs_ctx *c, const rs_fields *f, int32_t *d_itip, rs_stream_t stream) {
  if (!c || !d_itip) return fail(RS_E_INVALID, "rs_itip: null argument");
  int rc = check_fields(c, f, "rs_itip");
  if (rc) return rc;
  int nb = 0;
  if (rs::launch_grid_partials(f->precision, c->K, f->c, f->psi, c->p.cinf, c->partials, c->max_partials, &nb,
                               (cudaStream_t)stream))
    return fail(RS_E_INVALID, "rs_itip: workspace too small");
  rs::launch_reduce_partials(c->partials, nb, 0.0, nullptr, d_itip, (cudaStream_t)stream);
  return cuda_check("rs_itip");
}

int rs_mass(rs_ctx *c, const rs_fields *f, double *d_mass, rs_stream_t stream) {
  if (!c || !d_mass) return fail(RS_E_INVALID, "rs_mass: null argument");
  int rc = check_fields(c, f, "rs_mass");
  if (rc) return rc;
  int nb = 0;
  if (rs::launch_grid_partials(f->precision, c->K, f->c, f->psi, c->p.cinf, c->partials, c->max_partials, &nb,
                               (cudaStream_t)stream))
    return fail(RS_E_INVALID, "rs_mass: workspace too small");
  rs::launch_reduce_partials(c->partials, nb, 0.0, d_mass, nullptr, (cudaStream_t)stream);
  return cuda_check("rs_mass");
}

int rs_precise_tip(rs_ctx *c, const rs_fields *f, rs_tip *d_tip, rs_stream_t stream) {
  if (!c || !d_tip) return fail(RS_E_INVALID, "rs_precise_tip: null argument");
  if (c->p.band) return fail(RS_E_UNSUPPORTED, "rs_precise_tip: needs the whole domain, not a band");
  int rc = check_fields(c, f, "rs_precise_tip", false);
  if (rc) return rc;
  rs::launch_precise_tip(f->precision, c->K, f->psi, c->row_last, c->row_f, c->row_g, d_tip, (cudaStream_t)stream);
  return cuda_check("rs_precise_tip");
}

int rs_initial(rs_ctx *c, const rs_fields *f, rs_stream_t stream) {
  if (!c) return fail(RS_E_INVALID, "rs_initial: null ctx");
  int rc = check_fields(c, f, "rs_initial");
  if (rc) return rc;
  rs::launch_initial_reference(f->precision, c->K, c->p.i_tip_target, f->c, f->psi, f->phi, (cudaStream_t)stream);
  return cuda_check("rs_initial");
}

int rs_initial_planar(rs_ctx *c, const rs_fields *f, double c_liquid, double c_solid, uint64_t seed,
                      rs_stream_t stream) {
  if (!c) return fail(RS_E_INVALID, "rs_initial_planar: null ctx");
  int rc = check_fields(c, f, "rs_initial_planar");
  if (rc) return rc;
  if (!(c_liquid > 0 && c_liquid < 1 && c_solid > 0 && c_solid < 1))
    return fail(RS_E_INVALID, "rs_initial_planar: compositions must lie in (0,1)");
  rs::launch_initial_planar(f->precision, c->K, c->p.i_tip_target, c_liquid, c_solid, seed, f->c, f->psi, f->phi,
                            (cudaStream_t)stream);
  return cuda_check("rs_initial_planar");
}

int rs_temperature_init(rs_ctx *c, double *d_T, rs_stream_t stream) {
  if (!c || !d_T) return fail(RS_E_INVALID, "rs_temperature_init: null argument");
  rs::launch_temperature_init(c->T, d_T, (cudaStream_t)stream);
  return cuda_check("rs_temperature_init");
}

static double vp_ramp(const rs_params &p, double t) {
  if (p.vp_ramp) return p.Vp + 0.0107587 * (t * 0.001);  // Vp_ramp, fun.cu:1974-1982
  return p.Vp;
}

int rs_temperature_step(rs_ctx *c, double *d_T, double *d_T_next, const double *d_dphidt, int64_t step,
                        rs_stream_t stream) {
  if (!c || !d_T || !d_T_next || !d_dphidt) return fail(RS_E_INVALID, "rs_temperature_step: null argument");
  if (d_T == d_T_next) return fail(RS_E_INVALID, "rs_temperature_step: T and T_next alias");
  cudaStream_t st = (cudaStream_t)stream;
  const double adv = vp_ramp(c->p, step * c->d.tau0 * c->d.dt) * c->d.tau0 / (c->p.S * c->p.W0);
  double *a = d_T, *b = d_T_next;
  for (int s = 0; s < c->d.ratio_dt_dtT; ++s) {
    rs::launch_temperature_substep(c->T, a, b, d_dphidt, adv, st);
    double *t = a;
    a = b;
    b = t;
  }
  if (a != d_T) {
    const size_t bytes = sizeof(double) * (size_t)c->d.NxT_all * c->d.NyT_all;
    if (cudaMemcpyAsync(d_T, a, bytes, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
      return cuda_check("rs_temperature_step copy");
  }
  return cuda_check("rs_temperature_step");
}

int rs_interpolate_temperature(rs_ctx *c, const double *d_T, double *d_T_fine, int32_t i_left_end,
                               rs_stream_t stream) {
  if (!c || !d_T || !d_T_fine) return fail(RS_E_INVALID, "rs_interpolate_temperature: null argument");
  rs::launch_interpolate_temperature(c->T, c->K, d_T, d_T_fine, i_left_end, (cudaStream_t)stream);
  return cuda_check("rs_interpolate_temperature");
}

int rs_integrate_phi(rs_ctx *c, const rs_fields *cur, const rs_fields *next, double *d_dphidt, int32_t i_left_end,
                     rs_stream_t stream) {
  if (!c || !d_dphidt) return fail(RS_E_INVALID, "rs_integrate_phi: null argument");
  int rc = check_fields(c, cur, "rs_integrate_phi cur", false);
  if (!rc) rc = check_fields(c, next, "rs_integrate_phi next", false);
  if (rc) return rc;
  // a pull-back fused into the last rs_step on this cur shifted its read side only
  const int off = (c->pb_cur && cur->psi == c->pb_cur) ? c->pb_offset : 0;
  rs::launch_integrate_phi(cur->precision, c->T, cur->psi, next->psi, d_dphidt, i_left_end, off,
                           (cudaStream_t)stream);
  return cuda_check("rs_integrate_phi");
}

// ---------------------------------------------------------------- surrogate
static rs::MlpBox to_box(const rs_mlp_box *b) {
  rs::MlpBox m;
  m.T_lo = b->T_lo;
  m.T_hi = b->T_hi;
  m.c_lo = b->c_lo;
  m.c_hi = b->c_hi;
  for (int q = 0; q < 2; ++q) {
    m.y_mean[q] = b->y_mean[q];
    m.y_scale[q] = b->y_scale[q];
  }
  return m;
}

static bool box_ok(const rs_mlp_box *b) {
  return b && b->T_hi > b->T_lo && b->c_hi > b->c_lo && b->c_lo > 0.0 && b->c_hi < 1.0 && b->y_scale[0] > 0.0 &&
         b->y_scale[1] > 0.0;
}

int rs_mlp_sample(const rs_params *p, const rs_mlp_box *box, int64_t n, uint64_t seed, float *d_x, float *d_y,
                  rs_stream_t stream) {
  if (!p || !d_x || !d_y || n < 0) return fail(RS_E_INVALID, "rs_mlp_sample: bad argument");
  if (!box || !(box->T_hi > box->T_lo) || !(box->c_hi > box->c_lo) || box->c_lo <= 0.0 || box->c_hi >= 1.0)
    return fail(RS_E_INVALID, "rs_mlp_sample: box must have T_lo < T_hi and 0 < c_lo < c_hi < 1");
  rs::launch_mlp_sample(p->cinf, p->RR, to_box(box), n, seed, d_x, d_y, (cudaStream_t)stream);
  return cuda_check("rs_mlp_sample");
}

int rs_mlp_sample_g(const rs_params *p, const rs_mlp_box *box, int64_t n, uint64_t seed, float *d_x, float *d_y,
                    rs_stream_t stream) {
  if (!p || !d_x || !d_y || n < 0) return fail(RS_E_INVALID, "rs_mlp_sample_g: bad argument");
  if (!box || !(box->T_hi > box->T_lo) || !(box->c_hi > box->c_lo) || box->c_lo <= 0.0 || box->c_hi >= 1.0)
    return fail(RS_E_INVALID, "rs_mlp_sample_g: box must have T_lo < T_hi and 0 < c_lo < c_hi < 1");
  rs::launch_mlp_sample(p->cinf, p->RR, to_box(box), n, seed, d_x, d_y, (cudaStream_t)stream, true);
  return cuda_check("rs_mlp_sample_g");
}

int rs_mlp_grad(const rs_mlp_box *box, const float *d_w, int64_t n, const float *d_x, const float *d_y,
                float *d_grad, double *d_loss, rs_stream_t stream) {
  if (!box_ok(box) || !d_w || !d_x || !d_y || !d_grad || !d_loss || n < 0)
    return fail(RS_E_INVALID, "rs_mlp_grad: bad argument");
  if (rs::launch_mlp_grad(to_box(box), d_w, n, d_x, d_y, d_grad, d_loss, (cudaStream_t)stream))
    return fail(RS_E_CUDA, "rs_mlp_grad: cannot configure shared memory");
  return cuda_check("rs_mlp_grad");
}

int rs_mlp_adam(float *d_w, const float *d_grad, float *d_m, float *d_v, int64_t t, float lr, float scale,
                rs_stream_t stream) {
  if (!d_w || !d_grad || !d_m || !d_v || t < 1) return fail(RS_E_INVALID, "rs_mlp_adam: bad argument");
  rs::launch_mlp_adam(d_w, d_grad, d_m, d_v, t, lr, scale, (cudaStream_t)stream);
  return cuda_check("rs_mlp_adam");
}

int rs_mlp_forward(const rs_mlp_box *box, const float *d_w, int64_t n, const float *d_x, float *d_out,
                   rs_stream_t stream) {
  if (!box_ok(box) || !d_w || !d_x || !d_out || n < 0) return fail(RS_E_INVALID, "rs_mlp_forward: bad argument");
  rs::launch_mlp_forward(to_box(box), d_w, n, d_x, d_out, (cudaStream_t)stream);
  return cuda_check("rs_mlp_forward");
}

static uint16_t to_f16(float f) {  // round to nearest even
  return __half_as_ushort(__float2half_rn(f));
}

}  // extern "C"

namespace rs {

// Device copies of a trained network for a step kernel: FP32 parameters, FP16
// copies of the two tensor-core layers (W2[i][j], W3 padded to 8 rows) and a
// cleared audit record, allocated on first use; fills the kernel arguments.
cudaError_t surrogate_setup(const float *d_w, const rs_mlp_box *box, float **w, uint16_t **b16,
                            unsigned long long **audit, SurrArgs *s) {
  cudaError_t e = cudaSuccess;
  if (!*w) e = cudaMalloc(w, sizeof(float) * kMlpNParams);
  if (e == cudaSuccess && !*b16) e = cudaMalloc(b16, sizeof(uint16_t) * kSurrB16);
  if (e == cudaSuccess && !*audit) {
    e = cudaMalloc(audit, sizeof(unsigned long long) * 4);
    if (e == cudaSuccess) e = cudaMemset(*audit, 0, sizeof(unsigned long long) * 4);
  }
  float hw[kMlpNParams];
  if (e == cudaSuccess) e = cudaMemcpy(hw, d_w, sizeof(hw), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return e;
  uint16_t hb[kSurrB16];
  memset(hb, 0, sizeof(hb));
  for (int k = 0; k < kMlpH * kMlpH; ++k) hb[k] = to_f16(hw[kOffW2 + k]);
  for (int k = 0; k < 2 * kMlpH; ++k) hb[kMlpH * kMlpH + k] = to_f16(hw[kOffW3 + k]);
  e = cudaMemcpy(*w, hw, sizeof(hw), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(*b16, hb, sizeof(hb), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return e;
  s->w = *w;
  s->b16 = *b16;
  s->audit = *audit;
  s->T_mid = (float)(0.5 * (box->T_lo + box->T_hi));
  s->T_ihalf = (float)(2.0 / (box->T_hi - box->T_lo));
  s->c_mid = (float)(0.5 * (box->c_lo + box->c_hi));
  s->c_ihalf = (float)(2.0 / (box->c_hi - box->c_lo));
  s->T_lo = (float)box->T_lo;
  s->T_hi = (float)box->T_hi;
  s->c_lo = (float)box->c_lo;
  s->c_hi = (float)box->c_hi;
  for (int q = 0; q < 2; ++q) {
    s->y_mean[q] = (float)box->y_mean[q];
    s->y_scale[q] = (float)box->y_scale[q];
  }
  return cudaSuccess;
}

// Reads and clears an audit record (max error bits of mu'' and dG, fallback
// and audit counts); synchronizes the stream.
cudaError_t surrogate_audit_read(unsigned long long *audit, cudaStream_t st, double *max_err_mu, double *max_err_dG,
                                 int64_t *n_fallback, int64_t *n_audit) {
  unsigned long long h[4] = {0, 0, 0, 0};
  if (audit) {
    cudaError_t e = cudaMemcpyAsync(h, audit, sizeof(h), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(audit, 0, sizeof(h), st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
  }
  float f[2];
  for (int q = 0; q < 2; ++q) {
    const uint32_t u = (uint32_t)h[q];
    memcpy(&f[q], &u, 4);
  }
  if (max_err_mu) *max_err_mu = f[0];
  if (max_err_dG) *max_err_dG = f[1];
  if (n_fallback) *n_fallback = (int64_t)h[2];
  if (n_audit) *n_audit = (int64_t)h[3];
  return cudaSuccess;
}

bool surrogate_box_ok(const rs_mlp_box *b) { return box_ok(b); }

}  // namespace rs

extern "C" {

int rs_set_surrogate(rs_ctx *c, const float *d_w, const rs_mlp_box *box) {
  if (!c) return fail(RS_E_INVALID, "rs_set_surrogate: null context");
  if (!d_w) {
    c->surr.w = nullptr;
    return RS_OK;
  }
  if (!box_ok(box)) return fail(RS_E_INVALID, "rs_set_surrogate: bad box");
  if (c->p.tfc) return fail(RS_E_UNSUPPORTED, "rs_set_surrogate: frozen temperature only");
  const cudaError_t e = rs::surrogate_setup(d_w, box, &c->mlp_w, &c->mlp_b16, &c->mlp_audit, &c->surr);
  if (e != cudaSuccess) return fail(RS_E_CUDA, "rs_set_surrogate: %s", cudaGetErrorString(e));
  return RS_OK;
}

int rs_surrogate_audit(rs_ctx *c, double *max_err_mu, double *max_err_dG, int64_t *n_fallback, int64_t *n_audit,
                       rs_stream_t stream) {
  if (!c) return fail(RS_E_INVALID, "rs_surrogate_audit: null context");
  if (rs::surrogate_audit_read(c->mlp_audit, (cudaStream_t)stream, max_err_mu, max_err_dG, n_fallback, n_audit) !=
      cudaSuccess)
    return fail(RS_E_CUDA, "rs_surrogate_audit: copy failed");
  return RS_OK;
}

// ---------------------------------------------------------------- ensemble
struct rs_ens {
  int n = 0;
  std::vector<rs_ctx *> ctx;
  std::vector<rs_fields> A, B;
  std::vector<int> bound;
  rs::EnsRun *h_runs = nullptr;  // pinned host mirror of the descriptors
  rs::EnsRun *d_runs = nullptr;
  // per tile shape: the three tile orders and the number of tiles
  int32_t *d_tblk = nullptr, *d_order[rs::kTileShapes][3] = {};
  int ntblk = 0, ntiles[rs::kTileShapes] = {}, choice = 0, shape = 0;
  bool ready = false;
  bool surr = false;  // every run steps through its learned surrogate
  cudaGraphExec_t exec[rs::kTileShapes][3] = {};
  cudaStream_t cap = nullptr;
  int32_t *d_itip = nullptr, *h_itip = nullptr;
  bool walk = false;            // stretches without pull-back as one persistent launch (else graph replays)
  unsigned *d_bar = nullptr;    // grid-barrier counter and tile ticket counter of the persistent walk
  double *h_lv = nullptr, *d_lv = nullptr;  // l_offset_Vp of every run at each step of a walk launch
};

namespace {
constexpr int64_t kMaxWalk = 1024;  // steps per persistent launch

// l_offset_Vp of every run at steps 0 .. k of a walk from the mirror's state,
// by the additions ens_advance_kernel makes, on the device; the stream is
// synchronized first, so the pinned buffer is free
int ens_walk_l(rs_ens *e, int64_t k, cudaStream_t st) {
  if (cudaStreamSynchronize(st) != cudaSuccess) return -1;
  for (int r = 0; r < e->n; ++r) {
    double l = e->h_runs[r].l;
    for (int64_t s = 0; s <= k; ++s) {
      e->h_lv[s * e->n + r] = l;
      l += e->h_runs[r].inc_l;
    }
  }
  return cudaMemcpyAsync(e->d_lv, e->h_lv, sizeof(double) * (k + 1) * e->n, cudaMemcpyHostToDevice, st) ==
                 cudaSuccess
             ? 0
             : -1;
}
}  // namespace

namespace {

int ens_prepare(rs_ens *e) {
  if (e->ready) return RS_OK;
  for (int r = 0; r < e->n; ++r)
    if (!e->bound[r]) return fail(RS_E_STATE, "rs_ensemble: run %d has no field sets bound", r);
  // the surrogate path: every run has its network set (rs_set_surrogate on
  // its context), or none has
  int nsurr = 0;
  for (int r = 0; r < e->n; ++r) {
    e->h_runs[r].surr = e->ctx[r]->surr;
    nsurr += e->ctx[r]->surr.w != nullptr;
  }
  if (nsurr != 0 && nsurr != e->n)
    return fail(RS_E_UNSUPPORTED, "rs_ensemble: %d of %d runs have a surrogate: all or none", nsurr, e->n);
  e->surr = nsurr == e->n;
  std::vector<int32_t> tblk;
  for (int r = 0; r < e->n; ++r) {
    const int nb = (e->h_runs[r].tab_len + 126) / 127;
    for (int b = 0; b < nb; ++b) tblk.push_back((r << 16) | b);
  }
  e->ntblk = (int)tblk.size();
  cudaError_t c = cudaMalloc(&e->d_runs, sizeof(rs::EnsRun) * e->n);
  if (c == cudaSuccess) c = cudaMalloc(&e->d_tblk, sizeof(int32_t) * tblk.size());
  if (c == cudaSuccess) c = cudaMemcpy(e->d_tblk, tblk.data(), sizeof(int32_t) * tblk.size(), cudaMemcpyHostToDevice);
  // per tile shape, the tile orders: run by run, largest runs first, interleaved
  for (int sh = 0; sh < rs::kTileShapes && c == cudaSuccess; ++sh) {
    auto nt = [&](int r) { return e->h_runs[r].ntiles[sh]; };
    std::vector<int32_t> ord[3];
    for (int r = 0; r < e->n; ++r)
      for (int t = 0; t < nt(r); ++t) ord[0].push_back((r << 16) | t);
    std::vector<int> by(e->n);
    for (int r = 0; r < e->n; ++r) by[r] = r;
    std::stable_sort(by.begin(), by.end(), [&](int a, int b) { return nt(a) > nt(b); });
    for (int r : by)
      for (int t = 0; t < nt(r); ++t) ord[1].push_back((r << 16) | t);
    int tmax = 0;
    for (int r = 0; r < e->n; ++r) tmax = std::max(tmax, nt(r));
    for (int t = 0; t < tmax; ++t)
      for (int r = 0; r < e->n; ++r)
        if (t < nt(r)) ord[2].push_back((r << 16) | t);
    e->ntiles[sh] = (int)ord[0].size();
    for (int k = 0; k < 3 && c == cudaSuccess; ++k) {
      c = cudaMalloc(&e->d_order[sh][k], sizeof(int32_t) * e->ntiles[sh]);
      if (c == cudaSuccess)
        c = cudaMemcpy(e->d_order[sh][k], ord[k].data(), sizeof(int32_t) * e->ntiles[sh], cudaMemcpyHostToDevice);
    }
  }
  if (c == cudaSuccess) c = cudaMemcpy(e->d_runs, e->h_runs, sizeof(rs::EnsRun) * e->n, cudaMemcpyHostToDevice);
  if (c == cudaSuccess) c = cudaStreamCreateWithFlags(&e->cap, cudaStreamNonBlocking);
  if (c == cudaSuccess) c = cudaMalloc(&e->d_bar, 2 * sizeof(unsigned));
  if (c == cudaSuccess) c = cudaMalloc(&e->d_lv, sizeof(double) * (kMaxWalk + 1) * e->n);
  if (c == cudaSuccess) c = cudaMallocHost(&e->h_lv, sizeof(double) * (kMaxWalk + 1) * e->n);
  if (c != cudaSuccess) return fail(RS_E_CUDA, "rs_ensemble: %s", cudaGetErrorString(c));
  e->ready = true;
  return RS_OK;
}

int ens_graph(rs_ens *e, cudaGraphExec_t *out) {
  cudaGraphExec_t &ex = e->exec[e->shape][e->choice];
  if (ex) {
    *out = ex;
    return RS_OK;
  }
  cudaGraph_t g = nullptr;
  cudaError_t c = cudaStreamBeginCapture(e->cap, cudaStreamCaptureModeThreadLocal);
  if (c == cudaSuccess) {
    rs::launch_ensemble(e->d_runs, e->n, e->d_tblk, e->ntblk, e->d_order[e->shape][e->choice], e->ntiles[e->shape],
                        e->shape, true, e->surr, e->ctx[0]->d_err, e->cap);
    c = cudaStreamEndCapture(e->cap, &g);
  }
  if (c == cudaSuccess) c = cudaGraphInstantiate(&ex, g, 0);
  if (g) cudaGraphDestroy(g);
  if (c != cudaSuccess) return fail(RS_E_CUDA, "rs_ensemble: graph capture: %s", cudaGetErrorString(c));
  *out = ex;
  return RS_OK;
}

}  // namespace

int rs_ensemble_create(const rs_params *params, int32_t nruns, rs_ens **out) {
  if (!params || !out || nruns < 1 || nruns > 32767) return fail(RS_E_INVALID, "rs_ensemble_create: bad argument");
  *out = nullptr;
  for (int r = 0; r < nruns; ++r)
    if (params[r].tfc || params[r].vp_ramp || params[r].band)
      return fail(RS_E_UNSUPPORTED, "rs_ensemble_create: run %d: the ensemble steps frozen-temperature runs "
                                    "without the Vp ramp", r);
  rs_ens *e = new (std::nothrow) rs_ens;
  if (!e) return fail(RS_E_INVALID, "rs_ensemble_create: out of host memory");
  e->n = nruns;
  e->ctx.assign(nruns, nullptr);
  e->A.resize(nruns);
  e->B.resize(nruns);
  e->bound.assign(nruns, 0);
  int rc = RS_OK;
  for (int r = 0; r < nruns && rc == RS_OK; ++r) rc = rs_create(&params[r], &e->ctx[r]);
  cudaError_t c = cudaSuccess;
  if (rc == RS_OK) c = cudaMallocHost(&e->h_runs, sizeof(rs::EnsRun) * nruns);
  if (rc == RS_OK && c == cudaSuccess) c = cudaMalloc(&e->d_itip, sizeof(int32_t));
  if (rc == RS_OK && c == cudaSuccess) c = cudaMallocHost(&e->h_itip, sizeof(int32_t));
  if (rc == RS_OK && c != cudaSuccess) rc = fail(RS_E_CUDA, "rs_ensemble_create: %s", cudaGetErrorString(c));
  if (rc != RS_OK) {
    const std::string msg = rs_last_error();
    rs_ensemble_destroy(e);
    return fail(rc, "%s", msg.c_str());
  }
  memset(e->h_runs, 0, sizeof(rs::EnsRun) * nruns);
  *out = e;
  return RS_OK;
}

int rs_ensemble_destroy(rs_ens *e) {
  if (!e) return RS_OK;
  for (int sh = 0; sh < rs::kTileShapes; ++sh)
    for (int k = 0; k < 3; ++k) {
      if (e->exec[sh][k]) cudaGraphExecDestroy(e->exec[sh][k]);
      cudaFree(e->d_order[sh][k]);
    }
  if (e->cap) cudaStreamDestroy(e->cap);
  cudaFree(e->d_runs);
  cudaFree(e->d_tblk);
  cudaFree(e->d_itip);
  cudaFree(e->d_bar);
  cudaFree(e->d_lv);
  cudaFreeHost(e->h_lv);
  cudaFreeHost(e->h_itip);
  cudaFreeHost(e->h_runs);
  for (rs_ctx *c : e->ctx) rs_destroy(c);
  delete e;
  return RS_OK;
}

int rs_ensemble_context(rs_ens *e, int32_t run, rs_ctx **ctx) {
  if (!e || !ctx || run < 0 || run >= e->n) return fail(RS_E_INVALID, "rs_ensemble_context: bad argument");
  *ctx = e->ctx[run];
  return RS_OK;
}

int rs_ensemble_bind(rs_ens *e, int32_t run, const rs_fields *a, const rs_fields *b) {
  if (!e || !a || !b || run < 0 || run >= e->n) return fail(RS_E_INVALID, "rs_ensemble_bind: bad argument");
  if (e->ready) return fail(RS_E_STATE, "rs_ensemble_bind: the ensemble has started");
  rs_ctx *c = e->ctx[run];
  const rs_fields *fs[2] = {a, b};
  rs::EnsRun &R = e->h_runs[run];
  for (int k = 0; k < 2; ++k) {
    const rs_fields *f = fs[k];
    if (f->precision != RS_F32 || !f->c || !f->psi || (f->pitch && f->pitch != c->p.nx_all) ||
        ((uintptr_t)f->c % 16) || ((uintptr_t)f->psi % 16) || (c->p.nx_all % 4))
      return fail(RS_E_INVALID, "rs_ensemble_bind: run %d: FP32 field sets, 16-byte aligned, pitch nx_all, "
                                "nx_all a multiple of 4", run);
    for (int sh = 0; sh < rs::kTileShapes; ++sh)
      if (!encode_map(c->p, f->psi, RS_F32, rs::shape_rows(sh) + 2, &R.map_psi[sh][k]) ||
          !encode_map(c->p, f->c, RS_F32, rs::shape_rows(sh) + 2, &R.map_c[sh][k]))
        return fail(RS_E_CUDA, "rs_ensemble_bind: run %d: no tensor map", run);
    R.psi[k] = (float *)f->psi;
    R.c[k] = (float *)f->c;
  }
  const rs_params &p = c->p;
  R.K = c->K;
  R.F = rs::make_coef<float>(c->K);
  R.tab = c->col_tab;
  R.tab_len = c->col_tab_len;
  for (int sh = 0; sh < rs::kTileShapes; ++sh) {
    const int tr = rs::shape_rows(sh);
    R.nrt[sh] = (p.ny_all - 2 + tr - 1) / tr;
    R.ntiles[sh] = R.nrt[sh] * ((p.nx_all + rs::kTileOutW - 1) / rs::kTileOutW);
    if (R.ntiles[sh] > 65535)
      return fail(RS_E_INVALID, "rs_ensemble_bind: run %d is too large for the ensemble", run);
  }
  if ((R.tab_len + 126) / 127 > 65535)
    return fail(RS_E_INVALID, "rs_ensemble_bind: run %d is too large for the ensemble", run);
  R.active = 1;
  R.hist = R.hist_init = p.i_offset_history_initial;
  R.i_tip_target = p.i_tip_target;
  R.step = 0;
  R.l = R.l_init = p.l_offset_Vp_initial;
  R.inc_l = p.Vp * c->d.dt * c->d.tau0 / (p.S * p.W0);
  R.delta_initial = p.delta_initial;
  R.d1 = p.GG * p.dx * p.S * p.W0 / c->d.deltaT0;
  R.GG = p.GG;
  R.S = p.S;
  R.W0 = p.W0;
  R.deltaT0 = c->d.deltaT0;
  e->A[run] = *a;
  e->B[run] = *b;
  e->bound[run] = 1;
  return RS_OK;
}

int rs_ensemble_steps(rs_ens *e, int64_t nsteps, rs_stream_t stream) {
  if (!e || nsteps < 0) return fail(RS_E_INVALID, "rs_ensemble_steps: bad argument");
  int rc = ens_prepare(e);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  bool dirty = false;  // the host mirror differs from the device copy
  while (nsteps > 0) {
    int64_t m = INT64_MAX;  // steps until the next pull-back of any run
    for (int r = 0; r < e->n; ++r) {
      const int64_t spb = e->ctx[r]->d.step_pull_back;
      m = std::min(m, (spb - e->h_runs[r].step % spb) % spb);
    }
    if (m > 0) {  // no pull-back: replay the graph
      if (dirty) {
        if (cudaMemcpyAsync(e->d_runs, e->h_runs, sizeof(rs::EnsRun) * e->n, cudaMemcpyHostToDevice, st) !=
            cudaSuccess)
          return fail(RS_E_CUDA, "rs_ensemble_steps: state upload failed");
        dirty = false;
      }
      const int64_t k = std::min(m, nsteps);
      if (e->walk) {  // the stretch as persistent launches of up to kMaxWalk steps
        for (int64_t q = 0; q < k; q += kMaxWalk) {
          const int64_t kq = std::min(kMaxWalk, k - q);
          if (ens_walk_l(e, kq, st) ||
              rs::launch_ensemble_walk(e->d_runs, e->n, e->d_tblk, e->ntblk, e->d_order[e->shape][e->choice],
                                       e->ntiles[e->shape], e->shape, (int)kq, e->d_lv, true, e->surr, e->d_bar,
                                       e->ctx[0]->d_err, e->ctx[0]->wait_limit, st))
            return fail(RS_E_CUDA, "rs_ensemble_steps: persistent launch failed");
          for (int r = 0; r < e->n; ++r)  // the mirror follows (the next chunk starts from it)
            for (int64_t s2 = 0; s2 < kq; ++s2) {
              e->h_runs[r].step += 1;
              e->h_runs[r].l += e->h_runs[r].inc_l;
            }
        }
      } else {
        cudaGraphExec_t ex;
        if ((rc = ens_graph(e, &ex))) return rc;
        for (int64_t q = 0; q < k; ++q)
          if (cudaGraphLaunch(ex, st) != cudaSuccess) return fail(RS_E_CUDA, "rs_ensemble_steps: graph launch");
      }
      if (!e->walk)
        for (int r = 0; r < e->n; ++r)
          for (int64_t q = 0; q < k; ++q) {
            e->h_runs[r].step += 1;
            e->h_runs[r].l += e->h_runs[r].inc_l;
          }
      nsteps -= k;
      continue;
    }
    // a pull-back step (set_pull_back, fun.cu:693-742) for the runs due, the
    // batched launch for the others
    if (cudaStreamSynchronize(st) != cudaSuccess) return fail(RS_E_CUDA, "rs_ensemble_steps: sync failed");
    for (int r = 0; r < e->n; ++r) {
      rs::EnsRun &R = e->h_runs[r];
      R.active = 1;
      if (R.step % e->ctx[r]->d.step_pull_back) continue;
      const int par = (int)(R.step & 1);
      const rs_fields &cur = par ? e->B[r] : e->A[r], &nxt = par ? e->A[r] : e->B[r];
      if ((rc = rs_itip(e->ctx[r], &cur, e->d_itip, stream))) return rc;
      if (cudaMemcpyAsync(e->h_itip, e->d_itip, sizeof(int32_t), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
          cudaStreamSynchronize(st) != cudaSuccess)
        return fail(RS_E_CUDA, "rs_ensemble_steps: tip readback failed");
      rs_step_args a;
      memset(&a, 0, sizeof(a));
      a.step = R.step;
      a.pull_back = 1;
      a.i_offset = *e->h_itip - e->ctx[r]->p.i_tip_target;
      R.hist += a.i_offset;
      a.i_offset_history = R.hist;
      a.l_offset_Vp = R.l;
      if ((rc = rs_step(e->ctx[r], &cur, &nxt, &a, stream))) return rc;
      R.active = 0;
      R.step += 1;
      R.l += R.inc_l;
    }
    if (cudaMemcpyAsync(e->d_runs, e->h_runs, sizeof(rs::EnsRun) * e->n, cudaMemcpyHostToDevice, st) != cudaSuccess)
      return fail(RS_E_CUDA, "rs_ensemble_steps: state upload failed");
    rs::launch_ensemble(e->d_runs, e->n, e->d_tblk, e->ntblk, e->d_order[e->shape][e->choice], e->ntiles[e->shape],
                        e->shape, true, e->surr, e->ctx[0]->d_err, st);
    if ((rc = cuda_check("rs_ensemble_steps"))) return rc;
    // the upload above reads h_runs: finish it before the mirror changes
    if (cudaStreamSynchronize(st) != cudaSuccess) return fail(RS_E_CUDA, "rs_ensemble_steps: sync failed");
    for (int r = 0; r < e->n; ++r) {
      rs::EnsRun &R = e->h_runs[r];
      if (R.active) {
        R.step += 1;
        R.l += R.inc_l;
      }
      R.active = 1;
    }
    dirty = true;
    nsteps -= 1;
  }
  if (dirty) {
    if (cudaMemcpyAsync(e->d_runs, e->h_runs, sizeof(rs::EnsRun) * e->n, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      return fail(RS_E_CUDA, "rs_ensemble_steps: state upload failed");
  }
  return RS_OK;
}

int rs_ensemble_state(rs_ens *e, int32_t run, int64_t *step, int32_t *i_offset_history, double *l_offset_Vp,
                      int32_t *current) {
  if (!e || run < 0 || run >= e->n) return fail(RS_E_INVALID, "rs_ensemble_state: bad argument");
  const rs::EnsRun &R = e->h_runs[run];
  if (step) *step = R.step;
  if (i_offset_history) *i_offset_history = R.hist;
  if (l_offset_Vp) *l_offset_Vp = R.l;
  if (current) *current = (int32_t)(R.step & 1);
  return RS_OK;
}

int rs_ensemble_autotune(rs_ens *e, int32_t reps, double *ms_out, int32_t *choice, rs_stream_t stream) {
  if (!e || reps < 1) return fail(RS_E_INVALID, "rs_ensemble_autotune: bad argument");
  int rc = ens_prepare(e);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  if (cudaMemcpyAsync(e->d_runs, e->h_runs, sizeof(rs::EnsRun) * e->n, cudaMemcpyHostToDevice, st) != cudaSuccess)
    return fail(RS_E_CUDA, "rs_ensemble_autotune: state upload failed");
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  double best = 1e300;
  int pick = 0;
  // without advancing, a launch recomputes the same step: the runs do not move
  // (path k: tile shape k / 6; k % 6 < 3: the per-step launches with tile
  // order k % 6; k % 6 >= 3: one-step persistent walks with tile order
  // k % 6 - 3)
  auto launch = [&](int k) {
    const int sh = k / 6, o = k % 6;
    if (o < 3)
      return rs::launch_ensemble(e->d_runs, e->n, e->d_tblk, e->ntblk, e->d_order[sh][o], e->ntiles[sh], sh, false,
                                 e->surr, e->ctx[0]->d_err, st);
    return rs::launch_ensemble_walk(e->d_runs, e->n, e->d_tblk, e->ntblk, e->d_order[sh][o - 3], e->ntiles[sh], sh,
                                    1, e->d_lv, false, e->surr, e->d_bar, e->ctx[0]->d_err, 0, st);
  };
  if (ens_walk_l(e, 1, st)) return fail(RS_E_CUDA, "rs_ensemble_autotune: state upload failed");
  for (int k = 0; k < RS_ENS_PATHS; ++k) {
    bool bad = launch(k) != 0;
    cudaEventRecord(t0, st);
    for (int q = 0; q < reps && !bad; ++q) bad = launch(k) != 0;
    cudaEventRecord(t1, st);
    float ms = 0.f;
    if (bad || cudaEventSynchronize(t1) != cudaSuccess || cudaEventElapsedTime(&ms, t0, t1) != cudaSuccess) {
      cudaEventDestroy(t0);
      cudaEventDestroy(t1);
      return fail(RS_E_CUDA, "rs_ensemble_autotune: timing failed");
    }
    const double mean = ms / reps;
    if (ms_out) ms_out[k] = mean;
    if (mean < best) {
      best = mean;
      pick = k;
    }
  }
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  e->shape = pick / 6;
  e->choice = pick % 3;
  e->walk = pick % 6 >= 3;
  if (choice) *choice = pick;
  return cuda_check("rs_ensemble_autotune");
}

int rs_ensemble_set_path(rs_ens *e, int32_t path) {
  if (!e || path < 0 || path >= RS_ENS_PATHS)
    return fail(RS_E_INVALID, "rs_ensemble_set_path: path 0..%d", RS_ENS_PATHS - 1);
  e->shape = path / 6;
  e->choice = path % 3;
  e->walk = path % 6 >= 3;
  return RS_OK;
}

// Host build of the Ti-Nb evaluator (fun.cu:1671-1720) from the same
// pure-element functions the kernels use.
int rs_calphad_eval(int32_t which, const double *T, const double *cc, double *out, size_t n) {
  if (!T || !cc || !out) return fail(RS_E_INVALID, "rs_calphad_eval: null argument");
  const double RR = 8.3145;
  for (size_t k = 0; k < n; ++k) {
    const double t = T[k], c = cc[k], lT = std::log(t), onemc = 1.0 - c;
    double v;
    if (which == 0 || which == 1) {
      double log_part;
      if (c < 1.e-8)
        log_part = RR * t * (onemc * std::log(onemc));
      else if (onemc < 1.e-8)
        log_part = RR * t * (c * std::log(c));
      else
        log_part = RR * t * (onemc * std::log(onemc) + c * std::log(c));
      if (which == 0)
        v = log_part + onemc * rs::g_nb_liq(t, lT) + c * rs::g_ti_liq(t, lT) + c * onemc * rs::kL0Liq;
      else
        v = log_part + onemc * rs::g_nb_bcc(t, lT) + c * rs::g_ti_bcc(t, lT) + c * onemc * rs::kL0Bcc;
    } else if (which == 2 || which == 3) {
      double log_part = 0.;
      if (c > 1.e-8 && onemc > 1.e-8) log_part = RR * t * std::log(c / onemc);
      if (which == 2)
        v = rs::g_ti_liq(t, lT) - rs::g_nb_liq(t, lT) + rs::kL0Liq * (1.0 - 2.0 * c) + log_part;
      else
        v = rs::g_ti_bcc(t, lT) - rs::g_nb_bcc(t, lT) + rs::kL0Bcc * (1.0 - 2.0 * c) + log_part;
    } else {
      return fail(RS_E_INVALID, "rs_calphad_eval: which=%d", which);
    }
    out[k] = v;
  }
  return RS_OK;
}

}  // extern "C"

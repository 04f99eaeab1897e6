// rs_capi3.cu — extern "C" boundary of the 3D three-phase step
// (include/rs_b200.h, "3D three-phase variant"; model
// multi/peritectic_multiGPU/TiAg.cu).
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "rs_peri3d.cuh"
#include "rs_surrogate.cuh"

namespace rs {
int set_error(int code, const char *msg);
}

struct rs3_ctx {
  rs3_params p;
  int *err;            // device: bounded-wait failures of the step kernel
  double *partials;    // device: mass partial sums
  int nparts;
  struct Entry {
    const void *f1, *f2, *fc;
    int precision;
    bool surr;  // maps for the surrogate's scalar kernel (energy 1, FP32)
    rs::P3Maps maps;
  } cache[4];
  int ncache, next;
  double *tab;                    // energy 1: per-plane CALPHAD table of the step (device)
  rs::SurrArgs surr;              // energy 1, FP32: learned surrogate (surr.w == nullptr: exact)
  float *mlp_w;
  uint16_t *mlp_b16;
  unsigned long long *mlp_audit;
};

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode3() {
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

int bad(int code, const char *msg) { return rs::set_error(code, msg); }

bool params_ok(const rs3_params *p) {
  if (!(p && p->nx >= 4 && p->ny >= 4 && p->nz >= 4 && p->nx % 4 == 0 && p->dt > 0.0 && p->z_chunk >= 0 &&
        (int64_t)p->nx * p->ny * p->nz < ((int64_t)1 << 40)))
    return false;
  if (p->energy == 0) return true;
  return p->energy == 1 && p->c_ref > 0.0 && p->c_ref < 1.0 && p->RR > 0.0 && p->T_ref > 0.0 && p->AA >= 1.0;
}

bool fields_ok(const rs3_fields *f) {
  return f && f->phi1 && f->phi2 && f->c && (f->precision == RS_F64 || f->precision == RS_F32) &&
         ((uintptr_t)f->phi1 % 16 == 0) && ((uintptr_t)f->phi2 % 16 == 0) && ((uintptr_t)f->c % 16 == 0);
}

// surr: the step runs the energy-1 FP32 surrogate kernel (its own box)
bool encode_field(const rs3_params &p, const void *ptr, int precision, bool surr, CUtensorMap *out) {
  auto enc = encode3();
  if (!enc) return false;
  const size_t es = precision == RS_F64 ? 8 : 4;
  cuuint64_t dims[3] = {(cuuint64_t)p.nx, (cuuint64_t)p.ny, (cuuint64_t)p.nz};
  cuuint64_t strides[2] = {(cuuint64_t)p.nx * es, (cuuint64_t)p.nx * p.ny * es};
  const bool tinb = p.energy == 1;
  cuuint32_t box[3] = {(cuuint32_t)(tinb ? rs::tinb_box_width(precision, surr) : rs::peri3d_box_width(precision)),
                       (cuuint32_t)(tinb ? rs::tinb_box_height(precision, surr) : rs::peri3d_box_height(precision)),
                       1};
  cuuint32_t estr[3] = {1, 1, 1};
  return enc(out, precision == RS_F64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
             const_cast<void *>(ptr), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool maps_of(rs3_ctx *c, const rs3_fields *f, rs::P3Maps *m) {
  const bool surr = c->p.energy == 1 && f->precision == RS_F32 && c->surr.w != nullptr;
  for (int k = 0; k < c->ncache; ++k) {
    const rs3_ctx::Entry &e = c->cache[k];
    if (e.f1 == f->phi1 && e.f2 == f->phi2 && e.fc == f->c && e.precision == f->precision && e.surr == surr) {
      *m = e.maps;
      return true;
    }
  }
  rs::P3Maps n;
  if (!encode_field(c->p, f->phi1, f->precision, surr, &n.phi1) ||
      !encode_field(c->p, f->phi2, f->precision, surr, &n.phi2) || !encode_field(c->p, f->c, f->precision, surr, &n.c))
    return false;
  rs3_ctx::Entry &e = c->cache[c->next];
  e.f1 = f->phi1;
  e.f2 = f->phi2;
  e.fc = f->c;
  e.precision = f->precision;
  e.surr = surr;
  e.maps = n;
  c->next = (c->next + 1) % 4;
  if (c->ncache < 4) ++c->ncache;
  *m = n;
  return true;
}

int launched(const char *what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    char msg[256];
    snprintf(msg, sizeof(msg), "%s: %s", what, cudaGetErrorString(e));
    return bad(RS_E_CUDA, msg);
  }
  return RS_OK;
}

}  // namespace

extern "C" {

size_t rs3_sizeof_params(void) { return sizeof(rs3_params); }

int rs3_default_params(rs3_params *p) {
  if (!p) return bad(RS_E_INVALID, "rs3_default_params: null");
  memset(p, 0, sizeof(*p));
  p->nx = 512;  // Nx, Ny, devNz (TiAg.cu:23-28)
  p->ny = 512;
  p->nz = 128;
  p->dt = 0.015;  // DT, DXin, DYin, DZin (TiAg.cu:19-22)
  p->dx_inv = p->dy_inv = p->dz_inv = 2.0;
  p->a1 = 0.0;  // a1, a2, a3, b (TiAg.cu:37-40)
  p->a2 = 4.43;
  p->a3 = 6.09;
  p->b = 12.0;
  p->lambda = 30.0;  // lambda, alpha, Da, Db (TiAg.cu:42-45)
  p->alpha = 2.0;
  p->Da = 0.0;
  p->Db = 0.0;
  p->A1 = 0.391701;  // A1, A2, B11, B21, B12, B22 (TiAg.cu:54-59)
  p->A2 = 0.216598;
  p->B11 = 0.0685881;
  p->B21 = 0.037927;
  p->B12 = -0.466867;
  p->B22 = -0.0662661;
  p->T_ref = 60.0 * 0.000321787;  // T (TiAg.cu:52)
  p->energy = 0;
  p->AA = 1.0;  // energy 1 fields: q(phi1) = phi1 unless set
  p->RR = 8.3145;
  p->c_ref = 0.0;
  return RS_OK;
}

int rs3_create(const rs3_params *p, rs3_ctx **out) {
  if (!out || !params_ok(p)) return bad(RS_E_INVALID, "rs3_create: bad parameters (nx % 4, extents >= 4)");
  rs3_ctx *c = new rs3_ctx();
  c->p = *p;
  c->nparts = 148 * 8;
  cudaError_t e = cudaMalloc(&c->err, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(c->err, 0, sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&c->partials, sizeof(double) * c->nparts);
  if (e == cudaSuccess && p->energy == 1) e = cudaMalloc(&c->tab, sizeof(double) * rs::tinb_table_len(*p));
  if (e != cudaSuccess) {
    cudaFree(c->err);
    cudaFree(c->partials);
    delete c;
    return bad(RS_E_CUDA, "rs3_create: device allocation failed");
  }
  *out = c;
  return RS_OK;
}

int rs3_destroy(rs3_ctx *c) {
  if (!c) return RS_OK;
  cudaFree(c->err);
  cudaFree(c->partials);
  cudaFree(c->tab);
  cudaFree(c->mlp_w);
  cudaFree(c->mlp_b16);
  cudaFree(c->mlp_audit);
  delete c;
  return RS_OK;
}

int rs3_step(rs3_ctx *c, const rs3_fields *cur, const rs3_fields *next, int64_t step, rs_stream_t stream) {
  if (!c || !fields_ok(cur) || !fields_ok(next) || cur->precision != next->precision)
    return bad(RS_E_INVALID, "rs3_step: bad field sets (16-byte aligned, same precision)");
  if (cur->phi1 == next->phi1 || cur->phi2 == next->phi2 || cur->c == next->c)
    return bad(RS_E_INVALID, "rs3_step: next must not alias cur");
  rs::P3Maps m;
  if (!maps_of(c, cur, &m)) return bad(RS_E_UNSUPPORTED, "rs3_step: tensor maps unavailable");
  const int rc =
      c->p.energy == 1
          ? rs::launch_tinb_step(c->p, m, cur->precision, next->phi1, next->phi2, next->c, step, c->err, c->tab,
                                 c->surr.w && cur->precision == RS_F32 ? &c->surr : nullptr, (cudaStream_t)stream)
          : rs::launch_peri3d_step(c->p, m, cur->precision, next->phi1, next->phi2, next->c, step, c->err,
                                   (cudaStream_t)stream);
  if (rc) return bad(RS_E_CUDA, "rs3_step: shared memory configuration failed");
  return launched("rs3_step");
}

int rs3_mu(rs3_ctx *c, const rs3_fields *f, void *d_mu, rs_stream_t stream) {
  if (!c || !fields_ok(f) || !d_mu) return bad(RS_E_INVALID, "rs3_mu: bad argument");
  if (c->p.energy == 1)
    rs::launch_tinb_mu(c->p, f->precision, f->phi1, f->phi2, f->c, d_mu, c->tab, (cudaStream_t)stream);
  else
    rs::launch_peri3d_mu(c->p, f->precision, f->phi1, f->phi2, f->c, d_mu, (cudaStream_t)stream);
  return launched("rs3_mu");
}

int rs3_mass(rs3_ctx *c, const rs3_fields *f, double *d_mass, rs_stream_t stream) {
  if (!c || !fields_ok(f) || !d_mass) return bad(RS_E_INVALID, "rs3_mass: bad argument");
  rs::launch_peri3d_mass(c->p, f->precision, f->c, c->partials, c->nparts, d_mass, (cudaStream_t)stream);
  return launched("rs3_mass");
}

int rs3_initial(rs3_ctx *c, const rs3_fields *f, double z_front, double amp, int32_t n_alpha, double cap_radius,
                uint64_t seed, rs_stream_t stream) {
  if (!c || !fields_ok(f) || n_alpha < 0 || n_alpha > rs::kP3MaxCaps || cap_radius < 0.0)
    return bad(RS_E_INVALID, "rs3_initial: bad argument (n_alpha <= 16)");
  const rs3_params &p = c->p;
  rs::P3Init ini;
  memset(&ini, 0, sizeof(ini));
  ini.seed = seed;
  ini.z_front = z_front;
  ini.amp = amp;
  const double theta = 1.33;  // contact angle of the caps (TiAg.cu initial)
  ini.radius = cap_radius / std::sin(theta);
  ini.roff = cap_radius / std::tan(theta);
  // equilibrium compositions at T_ref (TiAg.cu:64-67 ca, cb, clb)
  const double B1 = p.B11 + p.B12 * p.T_ref, B2 = p.B21 + p.B22 * p.T_ref;
  ini.ca = (B1 + 0.5 * B2) / (p.A1 + 0.5 * p.A2) - p.A1 - p.A2;
  ini.cb = (B1 - 0.5 * B2) / (p.A1 - 0.5 * p.A2) - p.A1 + p.A2;
  ini.clb = (B1 - 0.5 * B2) / (p.A1 - 0.5 * p.A2) + p.A1;
  ini.n_alpha = n_alpha;
  for (int k = 0; k < n_alpha; ++k) {  // seeded cap centres over the interior
    uint32_t r[4] = {(uint32_t)k, 0u, 0u, 0x43415053u};
    rs::philox4x32(r, (uint32_t)seed, (uint32_t)(seed >> 32));
    ini.cx[k] = 1.0 + (p.nx - 2) * rs::u53(r[0], r[1]);
    ini.cy[k] = 1.0 + (p.ny - 2) * rs::u53(r[2], r[3]);
  }
  rs::launch_peri3d_init(p, f->precision, ini, f->phi1, f->phi2, f->c, (cudaStream_t)stream);
  return launched("rs3_initial");
}

int rs3_initial_grains(rs3_ctx *c, const rs3_fields *f, double z_front, double amp, double c_liquid,
                       double c_solid, uint64_t seed, rs_stream_t stream) {
  if (!c || !fields_ok(f) || !(c_liquid > 0.0 && c_liquid < 1.0) || !(c_solid > 0.0 && c_solid < 1.0) || amp < 0.0)
    return bad(RS_E_INVALID, "rs3_initial_grains: bad argument");
  rs::launch_grains_init(c->p, f->precision, seed, z_front, amp, c_liquid, c_solid, f->phi1, f->phi2, f->c,
                         (cudaStream_t)stream);
  return launched("rs3_initial_grains");
}

int rs3_set_surrogate(rs3_ctx *c, const float *d_w, const rs_mlp_box *box) {
  if (!c) return bad(RS_E_INVALID, "rs3_set_surrogate: null context");
  if (c->p.energy != 1) return bad(RS_E_UNSUPPORTED, "rs3_set_surrogate: the surrogate serves energy 1");
  if (!d_w) {
    c->surr.w = nullptr;
    return RS_OK;
  }
  if (!rs::surrogate_box_ok(box)) return bad(RS_E_INVALID, "rs3_set_surrogate: bad box");
  if (rs::surrogate_setup(d_w, box, &c->mlp_w, &c->mlp_b16, &c->mlp_audit, &c->surr) != cudaSuccess)
    return bad(RS_E_CUDA, "rs3_set_surrogate: device copy failed");
  return RS_OK;
}

int rs3_surrogate_audit(rs3_ctx *c, double *max_err_mu, double *max_err_dG, int64_t *n_fallback, int64_t *n_audit,
                        rs_stream_t stream) {
  if (!c) return bad(RS_E_INVALID, "rs3_surrogate_audit: null context");
  if (rs::surrogate_audit_read(c->mlp_audit, (cudaStream_t)stream, max_err_mu, max_err_dG, n_fallback, n_audit) !=
      cudaSuccess)
    return bad(RS_E_CUDA, "rs3_surrogate_audit: copy failed");
  return RS_OK;
}

int rs3_c_offset(const rs3_params *p, double *out) {
  if (!p || !out) return bad(RS_E_INVALID, "rs3_c_offset: null");
  *out = rs::peri3d_c_offset(*p);
  return RS_OK;
}

int rs3_device_status(rs3_ctx *c, rs_stream_t stream) {
  if (!c) return bad(RS_E_INVALID, "rs3_device_status: null");
  int h = 0;
  if (cudaMemcpyAsync(&h, c->err, sizeof(int), cudaMemcpyDeviceToHost, (cudaStream_t)stream) != cudaSuccess ||
      cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess)
    return bad(RS_E_CUDA, "rs3_device_status: copy failed");
  if (h == 1) return bad(RS_E_STATE, "rs3_step: a plane load did not arrive within the wait limit");
  if (h == 2) return bad(RS_E_STATE, "rs3_step: shared memory not 128-byte aligned");
  return RS_OK;
}

}  // extern "C"

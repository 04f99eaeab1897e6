// rs_frame.cu — moving frame, grid reductions and the device tip tracker.
//
//  * pull_back (fun.cu:1469-1492): standalone column shift of every cell.
//  * grid partials: per-block FP64 sum of interior c and max tip column;
//    replaces the full-grid D2H copy + host scan of set_pull_back
//    (fun.cu:693-699, get_itip_all_grain fun.cu:1745-1754).
//  * precise tip (get_precise_tip, fun.cu:2895-2954): one warp per row finds
//    the last psi > 0 column with a warp max-reduction; one thread replays the
//    reference's sequential row scan (get_tip_int, fun.cu:2880-2893) over the
//    per-row results and performs the quartic and parabola least-squares fits
//    (fun.cu:2648-2865) in FP64.  This file is compiled with -fmad=false so that
//    the fits round like the reference's host code.
#include <cstdio>
#include <cstring>
#include <mutex>

#include "rs_kernels.cuh"

namespace rs {

// ---------------------------------------------------------------- pull_back
template <typename R>
__global__ void pull_back_kernel(const StepCoef K, const R *__restrict__ c, const R *__restrict__ psi,
                                 const R *__restrict__ phi, R *__restrict__ c_n,
                                 R *__restrict__ psi_n, R *__restrict__ phi_n, int i_offset,
                                 R c_fill) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= K.nx || j >= K.ny) return;
  int i_next = i + i_offset;
  i_next = max(i_next, 1);
  i_next = min(i_next, K.nx - 2);
  const int64_t d = (int64_t)j * K.pitch + i, s = (int64_t)j * K.pitch + i_next;
  c_n[d] = i_next < K.nx - 2 ? c[s] : c_fill;
  psi_n[d] = psi[s];
  if (phi_n) phi_n[d] = phi ? phi[s] : fmin(fmax(psi[s], R(-1)), R(1));
}

void launch_pull_back(int precision, const StepCoef &K, const void *c, const void *psi,
                      const void *phi, void *c_n, void *psi_n, void *phi_n, int i_offset,
                      cudaStream_t st) {
  dim3 b(64, 4), g((K.nx + 63) / 64, (K.ny + 3) / 4);
  if (precision == RS_F64)
    pull_back_kernel<double><<<g, b, 0, st>>>(K, (const double *)c, (const double *)psi,
                                              (const double *)phi, (double *)c_n, (double *)psi_n,
                                              (double *)phi_n, i_offset, K.cinf);
  else  // FP32 field sets hold c - cinf: the inflowing melt is 0
    pull_back_kernel<float><<<g, b, 0, st>>>(K, (const float *)c, (const float *)psi,
                                             (const float *)phi, (float *)c_n, (float *)psi_n,
                                             (float *)phi_n, i_offset, 0.0f);
}

// ---------------------------------------------------------------- reductions
template <typename R>
__global__ void __launch_bounds__(256) grid_partials_kernel(const StepCoef K, const R *__restrict__ c,
                                                            const R *__restrict__ psi, double c_offset,
                                                            BlockPartial *out) {
  // one block per 8 rows; every cell (ghosts included) for the tip column,
  // interior cells for the mass
  const int j0 = blockIdx.x * 8;
  double m = 0.0;
  int it = 0;
  for (int jj = threadIdx.y; jj < 8; jj += blockDim.y) {
    const int j = j0 + jj;
    if (j >= K.ny) break;
    const bool interior_row = j >= 1 && j <= K.ny - 2;
    for (int i = threadIdx.x; i < K.nx; i += blockDim.x) {
      const int64_t o = (int64_t)j * K.pitch + i;
      if (psi[o] > R(0)) it = max(it, i);
      if (interior_row && i >= 1 && i <= K.nx - 2) m += (double)c[o] + c_offset;
    }
  }
  block_partial<256>(m, it, out);
}

int launch_grid_partials(int precision, const StepCoef &K, const void *c, const void *psi,
                         double c_offset, BlockPartial *partials, int max_partials,
                         int *nblocks_out, cudaStream_t st) {
  const int nb = (K.ny + 7) / 8;
  if (nb > max_partials) return -1;
  dim3 b(64, 4);
  if (precision == RS_F64)
    grid_partials_kernel<double><<<nb, b, 0, st>>>(K, (const double *)c, (const double *)psi, 0.0, partials);
  else
    grid_partials_kernel<float><<<nb, b, 0, st>>>(K, (const float *)c, (const float *)psi, c_offset, partials);
  *nblocks_out = nb;
  return 0;
}

__global__ void __launch_bounds__(256) reduce_partials_kernel(const BlockPartial *__restrict__ p, int n,
                                                              double mass_offset, double *mass_out,
                                                              int32_t *itip_out) {
  __shared__ double s_m[256];
  __shared__ int s_i[256];
  double m = 0.0;
  int it = 0;
  for (int k = threadIdx.x; k < n; k += 256) {
    m += p[k].mass;
    it = max(it, p[k].itip);
  }
  s_m[threadIdx.x] = m;
  s_i[threadIdx.x] = it;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      s_m[threadIdx.x] += s_m[threadIdx.x + s];
      s_i[threadIdx.x] = max(s_i[threadIdx.x], s_i[threadIdx.x + s]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    if (mass_out) *mass_out = s_m[0] + mass_offset;
    if (itip_out) *itip_out = max(1, s_i[0]);  // get_itip_all_grain starts at 1
  }
}

void launch_reduce_partials(const BlockPartial *partials, int n, double mass_offset,
                            double *mass_out, int32_t *itip_out, cudaStream_t st) {
  reduce_partials_kernel<<<1, 256, 0, st>>>(partials, n, mass_offset, mass_out, itip_out);
}

__global__ void __launch_bounds__(128) reduce_partials_dep_kernel(const FinalRed FR) {
  __shared__ double s_m[256];
  __shared__ int s_i[256];
  asm volatile("griddepcontrol.wait;" ::: "memory");  // the step grid has completed, its writes visible
  final_reduce(FR, s_m, s_i, (int)threadIdx.x, [] { __syncthreads(); });
}

int launch_reduce_partials_dep(const FinalRed &FR, cudaStream_t st) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(1);
  cfg.blockDim = dim3(128);
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, reduce_partials_dep_kernel, FR) == cudaSuccess ? 0 : -3;
}

// ---------------------------------------------------------------- precise tip
// per row j: last column i in [0, nx-2] with psi > 0 (or -1), and the two
// values get_tip_int can produce for the row: f_j at i0 = last, g_j at i0 = 0.
template <typename R>
__global__ void tip_rows_kernel(const StepCoef K, const R *__restrict__ psi, int *row_last,
                                double *row_f, double *row_g) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= K.ny) return;
  const int j = warp;
  const R *row = psi + (int64_t)j * K.pitch;
  int last = -1;
  for (int i = lane; i <= K.nx - 2; i += 32)
    if (row[i] > R(0)) last = i;
  last = __reduce_max_sync(0xffffffffu, last);
  if (lane == 0) {
    row_last[j] = last;
    if (last >= 0) {
      const double a = (double)row[last], b = (double)row[last + 1];
      row_f[j] = (b - a) * (0.0 - a) + last;
    } else {
      row_f[j] = 0.0;
    }
    const double a = (double)row[0], b = (double)row[1];
    row_g[j] = (b - a) * (0.0 - a) + 0;
  }
}

// solve_5x5 (fun.cu:2648-2691): Gaussian elimination with partial pivoting
__device__ void solve_5x5_d(double A[5][5], double b[5], double c[5]) {
  int p[5];
  for (int i = 0; i < 5; i++) p[i] = i;
  for (int k = 0; k < 4; k++) {
    double max_val = fabs(A[p[k]][k]);
    int max_idx = k;
    for (int i = k + 1; i < 5; i++)
      if (fabs(A[p[i]][k]) > max_val) {
        max_val = fabs(A[p[i]][k]);
        max_idx = i;
      }
    const int t = p[k];
    p[k] = p[max_idx];
    p[max_idx] = t;
    for (int i = k + 1; i < 5; i++) {
      const double factor = A[p[i]][k] / A[p[k]][k];
      for (int j = k; j < 5; j++) A[p[i]][j] -= factor * A[p[k]][j];
      b[p[i]] -= factor * b[p[k]];
    }
  }
  for (int i = 4; i >= 0; i--) {
    double sum = 0.0;
    for (int j = i + 1; j < 5; j++) sum += A[p[i]][j] * c[j];
    c[i] = (b[p[i]] - sum) / A[p[i]][i];
  }
}

// get_precise_x (fun.cu:2694-2738): quartic x(psi) through 5 points, x at psi = 0
__device__ double precise_x_d(const double *x, const double *y) {
  double A[5][5], b[5], c[5];
  for (int j = 0; j < 5; ++j) {
    b[j] = 0.0;
    c[j] = 0.0;
    for (int k = 0; k < 5; ++k) A[j][k] = 0.0;
  }
  for (int i = 0; i < 5; i++) {
    double yp[9];
    yp[0] = 1.0;
    for (int k = 1; k <= 8; k++) yp[k] = yp[k - 1] * y[i];
    for (int j = 0; j < 5; j++) {
      b[j] += x[i] * yp[j];
      for (int k = 0; k < 5; k++) A[j][k] += yp[j + k];
    }
  }
  solve_5x5_d(A, b, c);
  return c[0];  // c0 + c1 0 + ... evaluated at phi_interface = 0
}

// solve_3x3 (fun.cu:2740-2786)
__device__ int solve_3x3_d(double A[3][3], double cc[3], double x[3]) {
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
      for (int j = 0; j < 3; ++j) {
        const double t = A[k][j];
        A[k][j] = A[pivot][j];
        A[pivot][j] = t;
      }
      const double t = cc[k];
      cc[k] = cc[pivot];
      cc[pivot] = t;
    }
    const double piv = A[k][k];
    for (int i = k + 1; i < 3; ++i) {
      const double factor = A[i][k] / piv;
      A[i][k] = 0.0;
      for (int j = k + 1; j < 3; ++j) A[i][j] -= factor * A[k][j];
      cc[i] -= factor * cc[k];
    }
  }
  for (int i = 2; i >= 0; --i) {
    double sum = cc[i];
    for (int j = i + 1; j < 3; ++j) sum -= A[i][j] * x[j];
    x[i] = sum / A[i][i];
  }
  return 0;
}

// fit_parabola (fun.cu:2809-2865)
__device__ int fit_parabola_d(const double *x, const double *y, double *x0, double *y0, double *R) {
  double M[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, cc[3] = {0, 0, 0}, aa[3] = {0, 0, 0};
  for (int i = 0; i < 5; ++i) {
    const double f0 = 1.0, f1 = y[i], f2 = y[i] * y[i];
    M[0][0] += f0 * f0; M[0][1] += f0 * f1; M[0][2] += f0 * f2;
    M[1][0] += f1 * f0; M[1][1] += f1 * f1; M[1][2] += f1 * f2;
    M[2][0] += f2 * f0; M[2][1] += f2 * f1; M[2][2] += f2 * f2;
    cc[0] += f0 * x[i]; cc[1] += f1 * x[i]; cc[2] += f2 * x[i];
  }
  if (solve_3x3_d(M, cc, aa) != 0) return -2;
  if (fabs(aa[2]) < 1e-14) return -3;
  const double R_loc = 1.0 / (2.0 * aa[2]);
  const double y0_loc = -aa[1] / (2.0 * aa[2]);
  *x0 = aa[0] - (y0_loc * y0_loc) / (2.0 * R_loc);
  *y0 = y0_loc;
  *R = R_loc;
  return 0;
}

template <typename R>
__global__ void tip_fit_kernel(const StepCoef K, const R *__restrict__ psi, const int *__restrict__ row_last,
                               const double *__restrict__ row_f, const double *__restrict__ row_g,
                               rs_tip *out) {
  if (threadIdx.x != 0) return;
  // get_tip_int (fun.cu:2880-2893): sequential over rows, the scan start of
  // row j is the running tip int(itip)
  double itip = 0.0;
  int ti = 0, tj = 0;
  for (int j = 0; j < K.ny; ++j) {
    const int s = (int)itip;
    const int last = row_last[j];
    const double v = (last >= 0 && last >= s) ? row_f[j] : row_g[j];
    if (v > itip) {
      itip = v;
      ti = (int)itip;
      tj = j;
    }
  }
  double xd[5], yd[5];
  const int ny = K.ny;
  for (int k = 0; k < 5; ++k) {
    int j = tj - 2 + k;
    // deal_with_boundary (fun.cu:2624-2641) with (jmin, jmax)
    const int nmin = min(K.jmin, K.jmax), nmax = max(K.jmin, K.jmax);
    if (K.jmin > K.jmax) {  // periodic
      if (j <= nmin - 1) j += (nmax - nmin + 1);
      else if (j >= nmax + 1) j -= (nmax - nmin + 1);
    } else {                // no-flux: mirror
      if (j < nmin) j = 2 * nmin - j;
      else if (j > nmax) j = 2 * nmax - j;
    }
    j = min(max(j, 0), ny - 1);
    const int s = max(ti - 5, 0);
    const int last = row_last[j];
    const int i0 = (last >= 0 && last >= s) ? last : 0;
    double id[5], pd[5];
    for (int m = 0; m < 5; ++m) {
      const int i = i0 - 2 + m;
      id[m] = i;
      pd[m] = (double)psi[(int64_t)j * K.pitch + min(max(i, 0), K.nx - 1)];
    }
    xd[k] = precise_x_d(id, pd);
    yd[k] = j;
  }
  double x0 = 0.0, y0 = 0.0, Rr = 0.0;
  const int status = fit_parabola_d(xd, yd, &x0, &y0, &Rr);
  rs_tip t;
  t.i = ti;
  t.j = tj;
  t.status = status;
  t.reserved = 0;
  t.x = x0;
  t.y = y0;
  double Rn = fabs(Rr) * K.dx * K.W0 * K.S;
  if (Rn > 1e5) Rn = 1e5;
  if (Rn < 1.0) Rn = 1.0;
  t.R = Rn;
  *out = t;
}

void launch_precise_tip(int precision, const StepCoef &K, const void *psi, int *row_last,
                        double *row_f, double *row_g, rs_tip *out, cudaStream_t st) {
  const int threads = 256, rows_per_block = threads / 32;
  const int nb = (K.ny + rows_per_block - 1) / rows_per_block;
  if (precision == RS_F64) {
    tip_rows_kernel<double><<<nb, threads, 0, st>>>(K, (const double *)psi, row_last, row_f, row_g);
    tip_fit_kernel<double><<<1, 32, 0, st>>>(K, (const double *)psi, row_last, row_f, row_g, out);
  } else {
    tip_rows_kernel<float><<<nb, threads, 0, st>>>(K, (const float *)psi, row_last, row_f, row_g);
    tip_fit_kernel<float><<<1, 32, 0, st>>>(K, (const float *)psi, row_last, row_f, row_g, out);
  }
}

}  // namespace rs

// ---------------------------------------------------------------- no-allocation tip
// rs_precise_tip_noalloc: the precise tip for callers that cannot allocate
// device memory.  rs_precise_tip takes its per-row scratch (last psi > 0
// column and the two candidate tip values of every row) from a context that
// rs_create fills with cudaMalloc.  Some hosts cannot do that: a host that
// hands all device memory to its own pool allocator and forbids cudaMalloc
// once it runs, or a time-stepping loop that must not take the implicit
// device-wide synchronisation of cudaMalloc/cudaFree.  This entry point needs
// no context: its scratch is the file-scope array below, which every GPU that
// loads the library holds (RS_NOALLOC_TIP_MAX_ROWS rows, 20 bytes per row,
// 320 KiB) until the process exits.
//
// Host code cannot use the array's name as a device address (it names a host
// stand-in); the device address is looked up once per device with
// cudaGetSymbolAddress, with that device current, on the first call made on
// that device.  Make that first call before any stream capture.
//
// Every call shares the same scratch and it keeps the last call's contents.
// Nothing in it needs to start at zero: each call writes every row entry it
// later reads.  Calls whose kernels overlap on the GPU (different streams,
// different host threads) race on the scratch and must be ordered by the
// caller.
namespace rs {
namespace {

struct alignas(256) TipScratch {
  int last[RS_NOALLOC_TIP_MAX_ROWS];
  double f[RS_NOALLOC_TIP_MAX_ROWS];
  double g[RS_NOALLOC_TIP_MAX_ROWS];
};
static __device__ __align__(256) TipScratch g_tip_scratch;

constexpr int kMaxDevices = 64;
struct DeviceScratch {
  TipScratch *ptr;
  bool ready;
};
DeviceScratch g_dev_scratch[kMaxDevices];
std::mutex g_dev_scratch_mu;

int tip_scratch_for_current_device(TipScratch **out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return rs::set_error(RS_E_CUDA, "rs_precise_tip_noalloc: no CUDA device");
  if (dev < 0 || dev >= kMaxDevices) return rs::set_error(RS_E_UNSUPPORTED, "rs_precise_tip_noalloc: device index too large");
  std::lock_guard<std::mutex> lock(g_dev_scratch_mu);
  DeviceScratch &d = g_dev_scratch[dev];
  if (!d.ready) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_tip_scratch);
    if (e != cudaSuccess) {
      char msg[256];
      snprintf(msg, sizeof(msg), "rs_precise_tip_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
      return rs::set_error(RS_E_CUDA, msg);
    }
    d.ptr = static_cast<TipScratch *>(p);
    d.ready = true;
  }
  *out = d.ptr;
  return RS_OK;
}

}  // namespace
}  // namespace rs

extern "C" int rs_precise_tip_noalloc(const rs_params *p, const rs_fields *f, rs_tip *d_tip, rs_stream_t stream) {
  if (!p || !f || !d_tip || !f->psi) return rs::set_error(RS_E_INVALID, "rs_precise_tip_noalloc: null argument");
  if (f->precision != RS_F64 && f->precision != RS_F32)
    return rs::set_error(RS_E_INVALID, "rs_precise_tip_noalloc: precision tag");
  if (p->nx_all < 8 || p->ny_all < 8) return rs::set_error(RS_E_INVALID, "rs_precise_tip_noalloc: grid below 8x8");
  if (p->band) return rs::set_error(RS_E_UNSUPPORTED, "rs_precise_tip_noalloc: needs the whole domain, not a band");
  if (p->ny_all > RS_NOALLOC_TIP_MAX_ROWS)
    return rs::set_error(RS_E_INVALID, "rs_precise_tip_noalloc: ny_all exceeds RS_NOALLOC_TIP_MAX_ROWS");
  const int pitch = f->pitch ? f->pitch : p->nx_all;
  if (pitch != p->nx_all) return rs::set_error(RS_E_UNSUPPORTED, "rs_precise_tip_noalloc: pitch must equal nx_all");
  if ((uintptr_t)f->psi % (f->precision == RS_F64 ? 8 : 4))
    return rs::set_error(RS_E_INVALID, "rs_precise_tip_noalloc: misaligned psi");
  rs::TipScratch *sc = nullptr;
  int rc = rs::tip_scratch_for_current_device(&sc);
  if (rc) return rc;
  // the tip kernels read only these geometry fields of the step coefficients
  rs::StepCoef K;
  memset(&K, 0, sizeof(K));
  K.nx = p->nx_all;
  K.ny = p->ny_all;
  K.pitch = pitch;
  K.jmin = p->periodic_j ? p->ny_all - 2 : 1;
  K.jmax = p->periodic_j ? 1 : p->ny_all - 2;
  K.dx = p->dx;
  K.W0 = p->W0;
  K.S = p->S;
  rs::launch_precise_tip(f->precision, K, f->psi, sc->last, sc->f, sc->g, d_tip, (cudaStream_t)stream);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    char msg[256];
    snprintf(msg, sizeof(msg), "rs_precise_tip_noalloc: %s", cudaGetErrorString(e));
    return rs::set_error(RS_E_CUDA, msg);
  }
  return RS_OK;
}



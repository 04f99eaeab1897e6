// rs_init.cu — initial conditions and the coarse-grid temperature (TFC).
//
//  * initial (fun.cu:983-1021): tanh front at i_tip_target + 0.5 sin(2 pi j/Ny)
//  * planar seeded front: one Philox draw per row j gives the row's front
//    offset in [-1/2, 1/2) cell
//  * initial_temperature, compute_temperature, interpolate_temperature,
//    integrate_phi (fun.cu:1023-1028, 1494-1608) on the reference's coarse
//    layout psT(iT, jT) = jT NxT_all + iT.  Ghost rows of the coarse grid are
//    computed from the row they copy, so one launch per sub-step needs no
//    second boundary pass.
// FP32 field sets store c - cinf; the initial-condition kernels write that.
#include "rs_kernels.cuh"

namespace rs {

template <typename R>
__device__ __forceinline__ void store_cell(const StepCoef &K, R *c, R *psi, R *phi, int64_t o,
                                           double cv, double pv);
template <>
__device__ __forceinline__ void store_cell<double>(const StepCoef &K, double *c, double *psi,
                                                   double *phi, int64_t o, double cv, double pv) {
  c[o] = cv;
  psi[o] = pv;
  if (phi) phi[o] = pv;
}
template <>
__device__ __forceinline__ void store_cell<float>(const StepCoef &K, float *c, float *psi, float *phi,
                                                  int64_t o, double cv, double pv) {
  c[o] = (float)(cv - K.cinf);
  psi[o] = (float)pv;
  if (phi) phi[o] = (float)pv;
}

template <typename R>
__global__ void initial_reference_kernel(const StepCoef K, int itt, R *c, R *psi, R *phi) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= K.nx || j >= K.ny) return;
  const double PI_REF = 3.1415927;  // fun.cu:59
  const double itip = itt + 0.5 * sin(2.0 * PI_REF * j / K.ny);
  const double ph = -tanh((i - itip) * K.dx / sqrt(2.0));
  const double cc = 0.3184 * tanh(((i - itip) * K.dx - 0.08) / 0.67) + 0.6816;
  store_cell<R>(K, c, psi, phi, (int64_t)j * K.pitch + i, cc * K.cinf, ph);
}

template <typename R>
__global__ void initial_planar_kernel(const StepCoef K, int itt, double c_l, double c_s, uint32_t k0,
                                      uint32_t k1, R *c, R *psi, R *phi) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= K.nx || j >= K.ny) return;
  // the row's draw: ghost rows take their image row's; in band mode every
  // row, ghost rows included, takes its global row's
  const int js = K.jmin < 0 ? j + K.j_offset : (j == 0 ? K.jmin : (j == K.ny - 1 ? K.jmax : j));
  uint32_t x[4] = {(uint32_t)js, 0u, 0u, 0x49434F46u};
  philox4x32(x, k0, k1);
  const double i0 = itt + (u53(x[0], x[1]) - 0.5);
  const double ph = -tanh((i - i0) * K.dx / sqrt(2.0));
  const double h = 0.5 * (1.0 + ph);
  store_cell<R>(K, c, psi, phi, (int64_t)j * K.pitch + i, c_l + (c_s - c_l) * h, ph);
}

void launch_initial_reference(int precision, const StepCoef &K, int itt, void *c, void *psi,
                              void *phi, cudaStream_t st) {
  dim3 b(64, 4), g((K.nx + 63) / 64, (K.ny + 3) / 4);
  if (precision == RS_F64)
    initial_reference_kernel<double><<<g, b, 0, st>>>(K, itt, (double *)c, (double *)psi, (double *)phi);
  else
    initial_reference_kernel<float><<<g, b, 0, st>>>(K, itt, (float *)c, (float *)psi, (float *)phi);
}

void launch_initial_planar(int precision, const StepCoef &K, int itt, double c_l, double c_s,
                           uint64_t seed, void *c, void *psi, void *phi, cudaStream_t st) {
  dim3 b(64, 4), g((K.nx + 63) / 64, (K.ny + 3) / 4);
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  if (precision == RS_F64)
    initial_planar_kernel<double><<<g, b, 0, st>>>(K, itt, c_l, c_s, k0, k1, (double *)c, (double *)psi,
                                                   (double *)phi);
  else
    initial_planar_kernel<float><<<g, b, 0, st>>>(K, itt, c_l, c_s, k0, k1, (float *)c, (float *)psi,
                                                  (float *)phi);
}

// ---------------------------------------------------------------- TFC
__global__ void temperature_init_kernel(const TfcCoef T, double *d_T) {
  const int iT = blockIdx.x * blockDim.x + threadIdx.x;
  const int jT = blockIdx.y * blockDim.y + threadIdx.y;
  if (iT >= T.NxT_all || jT >= T.NyT_all) return;
  d_T[(int64_t)jT * T.NxT_all + iT] = T.Tcold + (iT - 1) * T.Sint * T.W0 * T.dx * T.ratio * T.GG;
}

void launch_temperature_init(const TfcCoef &T, double *d_T, cudaStream_t st) {
  dim3 b(64, 4), g((T.NxT_all + 63) / 64, (T.NyT_all + 3) / 4);
  temperature_init_kernel<<<g, b, 0, st>>>(T, d_T);
}

// compute_temperature (fun.cu:1537-1578) for the interior cell (iT, jT)
__device__ __forceinline__ double t_update(const TfcCoef &T, const double *__restrict__ Tin,
                                           const double *__restrict__ dphidt, double adv, int iT,
                                           int jT) {
  const int64_t o = (int64_t)jT * T.NxT_all + iT;
  const double T00 = Tin[o], T10 = Tin[o + 1], Tm0 = Tin[o - 1];
  const double T01 = Tin[o + T.NxT_all], T0m = Tin[o - T.NxT_all];
  const double laplacian = (T10 + Tm0 + T01 + T0m - 4.0 * T00) / (T.dxT * T.dxT);
  const double dTdt = adv * (T10 - Tm0) / (2.0 * T.dxT) + laplacian * T.DT / T.Gmuk;
  return T00 + T.dtT * dTdt + T.Lcp * dphidt[o] / (T.ratio_dt_dtT * (T.ratio * T.ratio));
}

__global__ void temperature_substep_kernel(const TfcCoef T, const double *__restrict__ Tin,
                                           double *__restrict__ Tout, const double *__restrict__ dphidt,
                                           double adv) {
  const int iT = blockIdx.x * blockDim.x + threadIdx.x;
  const int jT = blockIdx.y * blockDim.y + threadIdx.y;
  if (iT >= T.NxT_all || jT >= T.NyT_all) return;
  const int64_t o = (int64_t)jT * T.NxT_all + iT;
  if (iT == 0) {
    Tout[o] = T.Tcold;
  } else if (iT == T.NxT - 1) {
    Tout[o] = T.Thot;
  } else if (iT <= T.NxT - 2) {
    if (jT >= 1 && jT <= T.NyT - 2)
      Tout[o] = t_update(T, Tin, dphidt, adv, iT, jT);
    else if (jT == 0)
      Tout[o] = t_update(T, Tin, dphidt, adv, iT, T.jTmin);
    else if (jT == T.NyT - 1)
      Tout[o] = t_update(T, Tin, dphidt, adv, iT, T.jTmax);
  }
}

void launch_temperature_substep(const TfcCoef &T, const double *Tin, double *Tout, const double *dphidt,
                                double adv, cudaStream_t st) {
  dim3 b(64, 4), g((T.NxT_all + 63) / 64, (T.NyT_all + 3) / 4);
  temperature_substep_kernel<<<g, b, 0, st>>>(T, Tin, Tout, dphidt, adv);
}

__global__ void interpolate_temperature_kernel(const TfcCoef T, const double *__restrict__ d_T,
                                               double *__restrict__ d_T_fine, int ile) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= T.nx || j >= T.ny) return;
  int iT = (i - 1 + ile) / T.ratio;
  int jT = (int)((j - 1 + T.dxT) / T.ratio);
  const double x = (i - 1.0 + ile) / T.ratio - iT;
  const double y = (j - 1.0 + T.dxT) / T.ratio - jT;
  iT = min(max(iT, 0), T.NxT_all - 2);
  jT = min(max(jT, 0), T.NyT_all - 2);
  const double f00 = d_T[(int64_t)jT * T.NxT_all + iT];
  const double f10 = d_T[(int64_t)jT * T.NxT_all + iT + 1];
  const double f01 = d_T[(int64_t)(jT + 1) * T.NxT_all + iT];
  const double f11 = d_T[(int64_t)(jT + 1) * T.NxT_all + iT + 1];
  const double a10 = f10 - f00, a01 = f01 - f00, a11 = f11 - f10 - f01 + f00;
  d_T_fine[(int64_t)j * T.pitch + i] = f00 + a10 * x + a01 * y + a11 * x * y;
}

void launch_interpolate_temperature(const TfcCoef &T, const StepCoef &, const double *d_T,
                                    double *d_T_fine, int ile, cudaStream_t st) {
  dim3 b(64, 4), g((T.nx + 63) / 64, (T.ny + 3) / 4);
  interpolate_temperature_kernel<<<g, b, 0, st>>>(T, d_T, d_T_fine, ile);
}

// integrate_phi (fun.cu:1494-1535): latent-heat source per coarse cell, summed
// in the reference's order (rows outer, columns inner)
template <typename R>
// psi is read through the pull_back column remap of i_offset (0: none), so
// the source of a step whose shift was fused into rs_step sees the shifted
// field, as after the reference's pull_back swap (fun.cu:451-463).
__global__ void integrate_phi_kernel(const TfcCoef T, const R *__restrict__ psi, const R *__restrict__ psi_n,
                                     double *__restrict__ dphidt, int ile, int i_offset) {
  const int iT = blockIdx.x * blockDim.x + threadIdx.x;
  const int jT = blockIdx.y * blockDim.y + threadIdx.y;
  if (iT >= T.NxT_all || jT >= T.NyT_all) return;
  const int r = T.ratio;
  const int iT1 = ile / r, iTn = (ile + T.nx - 3) / r;
  double integral = 0;
  if (iT >= iT1 && iT <= iTn && jT >= 1 && jT <= T.NyT - 2) {
    int i0 = r * iT + 1 - ile;
    int in = i0 + r - 1;
    if (i0 < 1) i0 = 1;
    if (in > T.nx - 2) in = T.nx - 2;
    for (int j = 1 + r * (jT - 1); j <= r * jT; j++)
      for (int i = i0; i <= in; i++) {
        const int64_t o = (int64_t)j * T.pitch + i;
        const int is = i_offset ? min(max(i + i_offset, 1), T.nx - 2) : i;  // pull_back, fun.cu:1476-1487
        integral += (double)psi_n[o] - (double)psi[(int64_t)j * T.pitch + is];
      }
    dphidt[(int64_t)jT * T.NxT_all + iT] = integral * 0.5;
  } else {
    dphidt[(int64_t)jT * T.NxT_all + iT] = 0;
  }
}

void launch_integrate_phi(int precision, const TfcCoef &T, const void *psi, const void *psi_n,
                          double *dphidt, int ile, int i_offset, cudaStream_t st) {
  dim3 b(64, 4), g((T.NxT_all + 63) / 64, (T.NyT_all + 3) / 4);
  if (precision == RS_F64)
    integrate_phi_kernel<double><<<g, b, 0, st>>>(T, (const double *)psi, (const double *)psi_n, dphidt, ile, i_offset);
  else
    integrate_phi_kernel<float><<<g, b, 0, st>>>(T, (const float *)psi, (const float *)psi_n, dphidt, ile, i_offset);
}

}  // namespace rs

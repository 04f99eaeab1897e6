// rs_step.cu — the fused phase-field time step, FP64 (exact drop-in) and FP32
// (bulk) from one kernel template.
//
// One launch replaces the reference's per-step sequence
//   [pull_back] -> compute_phi -> compute_psi -> compute_c_CALPHAD
// (fun.cu:451-478, main.cu:179-213):
//   * the pull_back column shift (fun.cu:1469-1492) is a read-side remap of
//     the source column, so a pull-back step costs no extra pass;
//   * one orientation: phi = clamp(psi, -1, 1) (compute_psi,
//     fun.cu:1232-1273), so only psi and c are read and written;
//   * ghost cells (compute_boundary_individual, fun.cu:1220-1230) are written
//     by the cell they copy, corners included.
//
// Three kernels: this file's register-prefetch kernel (unaligned fields,
// RS_OPT_TMA = 0) and the TMA-staged tile kernels of rs_step_f32.cu (FP32) and
// rs_step_f64t.cu (FP64): frozen and coarse-grid temperature, pull-back steps
// included (those gather their shifted tile).
//
// Layout of the work here: a warp owns a strip of 30 output columns (32 input
// columns with a one-column halo on each side) and marches down H rows (H
// chosen per launch, below).
// Each row of psi and c is loaded once per warp with a coalesced 32-lane load
// (issued P rows ahead), the per-cell quantities phi, S = q(psi)c(1-c)
// (fun.cu:1424-1432) and the chemical potential mu (fun.cu:1443-1452) are
// computed once per cell, vertical neighbours come from a three-row register
// window and horizontal neighbours from warp shuffles.  No shared memory, no
// block barriers.  Column blocks launch from the one holding the front
// (front_first_block): its interface rows are the slowest.
//
// Arithmetic (identical mathematics to the reference, regrouped):
//   * anisotropy (get_anisotropy, fun.cu:1030-1139): with n = R (cos, sin, 0),
//     |n|^4 = k0 + k1 cos2t + k2 sin2t + k3 cos4t + k4 sin4t exactly, and
//     cos2t = (px^2 - py^2)/|grad phi|^2, sin2t = 2 px py/|grad phi|^2, so
//     a_s, a_k and both theta-derivatives need one reciprocal and no sqrt or
//     trigonometry.  k0..k4 come from the orientation on the host.
//   * mu = K(T) + mu', with the composition-independent column part
//     K(T) = (dGs+dGl)/2 + (L0_BCC+L0_Liq)(1-2cinf)/2 + RT log(cinf/(1-cinf))
//     in FP64 per column (only its i-differences enter the fluxes) and
//     mu' = g D - delta (L0_BCC+L0_Liq) + g (L0_BCC-L0_Liq)(1-2c)/2
//           + RT [log(c/(1-c)) - log(cinf/(1-cinf))],  D = (dGs-dGl)/2,
//     delta = c - cinf.  FP32 needs this split (mu ~ 1e4 J/mol while the
//     fluxes see neighbour differences of 1e-1..1e2 J/mol).
//   * Gl - Gs = (1-c) A_Nb + c A_Ti + c(1-c)(L0_Liq - L0_BCC): the ideal-mixing
//     terms of Gl and Gs (fun.cu:1671-1698) cancel exactly.
//   * FP64 rows whose cells all have |s| < 1/9 take
//     log(c/(1-c)) - log(cinf/(1-cinf)) = 2 atanh(s), s = delta/(2 cinf (1-c)
//     + delta), as a series to s^15 in place of the logarithm;
//   * exact shortcuts, warp-uniform: if all nine phi of every cell of the row
//     are the same +-1, phi_next = phi (phi - phi^3 = 0, g'(+-1) = 0, grad = 0);
//     if all nine S are 0 (solid, q(1) = 0) the solute update is dc = 0.
//     Both give bit-identical results to the general formulas.
// FP32 field sets store delta = c - cinf (see include/rs_b200.h).
#include "rs_step_common.cuh"

namespace rs {

__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }

// Per-lane state of a warp marching down a strip of 30 output columns, and
// the work for one incoming row.
template <typename R, bool TFC>
struct Strip {
  using S = typename Tr<R>::S;
  static constexpr unsigned FULL = 0xffffffffu;
  int gi, gic, gx2, y_last;
  bool out_lane;
  ColT<R> col;
  R dKr;
  // three-row window: index 0 = row r-1, 1 = row r, 2 = row r+1
  R p0, p1, p2, pl0, pl1, pl2, pr0, pr1, pr2;
  R s0, s1, s2, sl1, sl2, sr0, sr1, sr2;
  R m1, m2;        // mu' of rows r, r+1
  R d1, d2;        // stored c value (FP32: c - cinf) of rows r, r+1
  R jv_lo, jv_hi;  // solute flux through the faces (r-1/2) and (r+1/2)
  bool sol0, sol1, sol2, liq0, liq1, liq2;
  R A1nb, A1ti, A2nb, A2ti;  // TFC: driving-force groups of rows r, r+1
  R kr1, kr2;                // TFC: K(i+1) - K(i) of rows r, r+1
  double Kc2;
  double mass;
  int itip;

  __device__ __forceinline__ void init(const StepCoef &K, const StepScalars &PS, int gi_, int y_last_, bool active) {
    gi = gi_;
    gic = min(gi, K.nx - 1);
    gx2 = gi == 1 ? 0 : (gi == K.nx - 2 ? K.nx - 1 : -1);
    y_last = y_last_;
    out_lane = active && (threadIdx.x & 31) >= 1 && (threadIdx.x & 31) <= 30 && gi <= K.nx - 2;
    p0 = p1 = p2 = pl0 = pl1 = pl2 = pr0 = pr1 = pr2 = R(0);
    s0 = s1 = s2 = sl1 = sl2 = sr0 = sr1 = sr2 = R(0);
    m1 = m2 = d1 = d2 = jv_lo = jv_hi = R(0);
    sol0 = sol1 = sol2 = liq0 = liq1 = liq2 = false;
    A1nb = A1ti = A2nb = A2ti = kr1 = kr2 = R(0);
    Kc2 = 0.0;
    mass = 0.0;
    itip = 0;
    dKr = R(0);
    if (!TFC) {
      // frozen temperature: CALPHAD groups of this column, once per strip
      const double T = (PS.d0 + PS.d1 * gi) * K.deltaT0 + K.Tmelt;
      col = col_terms<R>(K, T);
      const double Kn = __shfl_down_sync(FULL, col.Kc, 1);
      dKr = (R)(Kn - col.Kc);  // K(i+1) - K(i)
    }
  }

  // row `row` (k-th row of the strip, k = 0 is y0-1) arrives with psi = pv and
  // stored c value cv_s; once three rows are in the window, row-1 is output.
  __device__ __forceinline__ void step_row(const StepCoef &K, const Coef<R> &F, const StepScalars &PS, R pv, R cv_s,
                                           int k, int row, S *__restrict__ psi_n, S *__restrict__ c_n,
                                           S *__restrict__ phi_n, bool red) {
    const R cinf = F.cinf;
    // ---- per-cell quantities of the new row
    const R d = Tr<R>::kDelta ? cv_s : cv_s - cinf;
    const R c = Tr<R>::kDelta ? cinf + cv_s : cv_s;
    const R omc = R(1) - c;
    const R ph = fmin(fmax(pv, R(-1)), R(1));
    const R a = R(1) - pv;
    const R Sv = (R(0.5) * F.AA * a - R(0.25) * (F.AA - R(1)) * (a * a)) * c * omc;
    const R p2v = pv * pv;
    const R g = pv * (R(1.875) + p2v * (R(-1.25) + R(0.375) * p2v));
    ColT<R> ct = col;
    if (TFC) ct = col_terms<R>(K, t_fine_at(K, PS.T_coarse, PS.i_left_end_T, gic, min(row, K.ny - 1)));
    constexpr R L0sum = R(kL0Bcc + kL0Liq);
    constexpr R L0half = R(0.5 * (kL0Bcc - kL0Liq));
    R lam;
    if constexpr (sizeof(R) == 8) {
      // rows whose cells all have |s| < 1/9 (the melt, and a solid near the
      // melt's composition): log(c/(1-c)) - Lref = 2 atanh(s),
      // s = delta / (2 cinf (1 - c) + delta), by its series to s^15
      // (truncation below 3.3e-17 relative) instead of a logarithm and a
      // second division; the difference is rounding-level, and free of the
      // cancellation of log(c/(1-c)) - Lref
      const R sv = d / (R(2) * cinf * omc + d);
      if (__all_sync(FULL, fabs(sv) < R(1.0 / 9.0))) {
        const R s2 = sv * sv;
        R p = R(1.0 / 15.0);
        p = fma(p, s2, R(1.0 / 13.0));
        p = fma(p, s2, R(1.0 / 11.0));
        p = fma(p, s2, R(1.0 / 9.0));
        p = fma(p, s2, R(1.0 / 7.0));
        p = fma(p, s2, R(1.0 / 5.0));
        p = fma(p, s2, R(1.0 / 3.0));
        lam = R(2) * fma(sv * s2, p, sv);
      } else {
        lam = Tr<R>::lam(c, omc, d, cinf, F.Lref);
      }
    } else {
      lam = Tr<R>::lam(c, omc, d, cinf, F.Lref);
    }
    const R mu = g * ct.D - d * L0sum + g * L0half * (R(1) - R(2) * c) + ct.RT * lam;
    const bool row_sol = __ballot_sync(FULL, ph == R(1)) == FULL;
    const bool row_liq = __ballot_sync(FULL, ph == R(-1)) == FULL;

    // ---- shift the window
    p0 = p1; p1 = p2; p2 = ph;
    pl0 = pl1; pl1 = pl2; pl2 = __shfl_up_sync(FULL, ph, 1);
    pr0 = pr1; pr1 = pr2; pr2 = __shfl_down_sync(FULL, ph, 1);
    s0 = s1; s1 = s2; s2 = Sv;
    sl1 = sl2; sl2 = __shfl_up_sync(FULL, Sv, 1);
    sr0 = sr1; sr1 = sr2; sr2 = __shfl_down_sync(FULL, Sv, 1);
    m1 = m2; m2 = mu;
    d1 = d2; d2 = cv_s;
    sol0 = sol1; sol1 = sol2; sol2 = row_sol;
    liq0 = liq1; liq1 = liq2; liq2 = row_liq;
    R ku = R(0);
    if (TFC) {
      ku = (R)(ct.Kc - Kc2);
      Kc2 = ct.Kc;
      A1nb = A2nb; A1ti = A2ti; A2nb = ct.A_nb; A2ti = ct.A_ti;
      kr1 = kr2;
      kr2 = (R)(__shfl_down_sync(FULL, ct.Kc, 1) - ct.Kc);
    }
    if (k < 1) return;
    // flux through the face between rows row-1 and row (compute_c_CALPHAD
    // F01/F0m, fun.cu:1455-1459): weight (S00 + S01 + Shh + Snh)/4
    jv_lo = jv_hi;
    // face fluxes are rounded products: a contracted product would round a
    // face differently at the end of a strip, and so depend on the tiling
    jv_hi = mul_rn((R(1.5) * (s1 + s2) + R(0.25) * ((sr1 + sr2) + (sl1 + sl2))), (m2 - m1 + ku));
    if (k < 2) return;

    // ---- output row r = row - 1
    const int r = row - 1;
    R psi_new = p1;
    // phi: exact shortcut when the three rows are all +1 or all -1
    if (!((sol0 && sol1 && sol2) || (liq0 && liq1 && liq2))) {
      R as, ak;
      const R an = anisotropy<R>(F, p1, pr1, pl1, p2, p0, pr2, pl2, pr0, pl0, as, ak);
      const R c00 = Tr<R>::kDelta ? cinf + d1 : d1;
      const R Anb = TFC ? A1nb : col.A_nb, Ati = TFC ? A1ti : col.A_ti;
      const R dG = (R(1) - c00) * Anb + c00 * Ati + c00 * (R(1) - c00) * R(kL0Liq - kL0Bcc);
      const R q = R(1) - p1 * p1;
      const R term = p1 - p1 * p1 * p1 + an + dG * (R(1.875) * (q * q)) * F.drive;
      R pn = p1 + Tr<R>::div(F.dt * ak, as * as) * term;
      if (F.noise_amp > R(0) && q > R(1.0e-3)) {
        uint32_t x[4];
        noise_counter(x, PS.step, (int64_t)(r + K.j_offset) * K.nx + gi);
        philox4x32(x, K.seed_lo, K.seed_hi);
        pn += F.noise_amp * q * Tr<R>::normal(x);
      }
      psi_new = pn > R(1) ? R(1) : pn;  // renormalisation (fun.cu:1252-1261)
    }
    // c: flux through the face (i+1/2, r) (F10/Fm0), weight (S00+S10+Shh+Shn)/4
    const R mr = __shfl_down_sync(FULL, m1, 1);
    const R jh = mul_rn((R(1.5) * (s1 + sr1) + R(0.25) * ((s2 + sr2) + (s0 + sr0))), (mr - m1 + (TFC ? kr1 : dKr)));
    const R jh_left = __shfl_up_sync(FULL, jh, 1);
    const R dc = F.cflux * ((jh - jh_left) + (jv_hi - jv_lo));
    const R dn = fmax(d1 + dc, Tr<R>::kDelta ? F.c_floor - cinf : F.c_floor);  // floor, fun.cu:1464

    // ---- stores (+ ghost copies, fun.cu:1220-1230)
    if (out_lane && r <= y_last) {
      const S vpsi = (S)psi_new;
      const S vc = (S)dn;
      const int pitch = K.pitch;
      const int64_t o = (int64_t)r * pitch + gi;
      psi_n[o] = vpsi;
      c_n[o] = vc;
      if (phi_n) phi_n[o] = (S)fmin(fmax(psi_new, R(-1)), R(1));
      if (gx2 >= 0) {
        const int64_t o2 = (int64_t)r * pitch + gx2;
        psi_n[o2] = vpsi;
        c_n[o2] = vc;
        if (phi_n) phi_n[o2] = (S)fmin(fmax(psi_new, R(-1)), R(1));
      }
      if (r == K.jmin || r == K.jmax) {
        const int gy2 = r == K.jmin ? 0 : K.ny - 1;
        const int64_t o3 = (int64_t)gy2 * pitch + gi;
        psi_n[o3] = vpsi;
        c_n[o3] = vc;
        if (phi_n) phi_n[o3] = (S)fmin(fmax(psi_new, R(-1)), R(1));
        if (gx2 >= 0) {
          const int64_t o4 = (int64_t)gy2 * pitch + gx2;
          psi_n[o4] = vpsi;
          c_n[o4] = vc;
          if (phi_n) phi_n[o4] = (S)fmin(fmax(psi_new, R(-1)), R(1));
        }
      }
      if (red) {
        mass += (double)vc;
        if (psi_new > R(0)) itip = max(itip, gi == K.nx - 2 ? K.nx - 1 : gi);
      }
    }
  }

  __device__ __forceinline__ void write_partial(BlockPartial *partials, int64_t slot) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mass += __shfl_down_sync(FULL, mass, o);
    itip = __reduce_max_sync(FULL, itip);
    if ((threadIdx.x & 31) == 0) {
      BlockPartial b;
      b.mass = mass;
      b.itip = itip;
      b.pad = 0;
      partials[slot] = b;
    }
  }
};

// Register-prefetch kernel: every lane loads its own column P rows ahead.
// Handles the pull-back remap, the coarse-grid temperature and any pitch.
// HC: rows per block fixed at compile time, or 0 for the launch argument H_rt
template <typename R, int HC, int P, bool TFC>
__global__ void __launch_bounds__(128, sizeof(R) == 4 ? 4 : 3)
    step_kernel(const StepCoef K, const Coef<R> F, const StepScalars PS, const typename Tr<R>::S *__restrict__ psi,
                const typename Tr<R>::S *__restrict__ cst, typename Tr<R>::S *__restrict__ psi_n,
                typename Tr<R>::S *__restrict__ c_n, typename Tr<R>::S *__restrict__ phi_n, BlockPartial *partials,
                const int H_rt) {
  const int H = HC > 0 ? HC : H_rt;
  using S = typename Tr<R>::S;
  const int nx = K.nx, ny = K.ny, pitch = K.pitch;
  const int wpb = blockDim.x >> 5;
  // blockIdx.x walks the row blocks of one column block, blockIdx.y the column
  // blocks, from the one holding column PS.i_front
  const int ncb = gridDim.y, rb = blockIdx.x;
  const int cb = front_first_block((int)blockIdx.y, max(PS.i_front - 1, 0) / (30 * wpb), ncb);
  const int wc = cb * wpb + (int)(threadIdx.x >> 5);     // warp column
  const int X = 1 + 30 * wc;                             // first output column
  const int gi = X - 1 + (int)(threadIdx.x & 31);        // this lane's column
  const int y0 = 1 + rb * H;
  const int y_last = min(y0 + H - 1, ny - 2);
  const bool active_warp = X <= nx - 2;

  // source column of this lane (pull_back remap, fun.cu:1476-1487)
  int si = min(gi, nx - 1);
  bool fill = false;
  if (PS.pull_back) {
    si = min(max(si + PS.i_offset, 1), nx - 2);
    fill = si >= nx - 2;
  }
  S qp[P], qc[P];
  auto load_row = [&](int row, S &pv, S &cv) {
    const int rr = min(row, ny - 1);
    const int64_t o = (int64_t)rr * pitch + si;
    pv = psi[o];
    cv = fill ? (Tr<R>::kDelta ? S(0) : S(K.cinf)) : cst[o];
  };
#pragma unroll
  for (int s = 0; s < P; ++s) load_row(y0 - 1 + s, qp[s], qc[s]);

  Strip<R, TFC> st;
  st.init(K, PS, gi, y_last, active_warp);
  const int nrows = y_last - y0 + 3;  // rows y0-1 .. y_last+1
  if (active_warp) {
    for (int base = 0; base < nrows; base += P) {
#pragma unroll
      for (int s = 0; s < P; ++s) {
        const int k = base + s;
        if (k >= nrows) break;
        const int row = y0 - 1 + k;
        const R pv = (R)qp[s], cv = (R)qc[s];
        load_row(row + P, qp[s], qc[s]);
        st.step_row(K, F, PS, pv, cv, k, row, psi_n, c_n, phi_n, partials != nullptr);
      }
    }
  }
  if (partials) st.write_partial(partials, ((int64_t)rb * ncb + cb) * wpb + (int)(threadIdx.x >> 5));
}

template <typename R>
static int launch(const StepCoef &K, const StepScalars &P, const typename Tr<R>::S *psi, const typename Tr<R>::S *c,
                  typename Tr<R>::S *psi_n, typename Tr<R>::S *c_n, typename Tr<R>::S *phi_n, BlockPartial *partials,
                  int max_partials, int *nwarps_out, const TmaMaps *tm, int *err, cudaStream_t st) {
  const Coef<R> F = make_coef<R>(K);
  const int ni = K.nx - 2, nj = K.ny - 2;
  const bool tfc = K.tfc != 0;
  if (tm) {
    if constexpr (sizeof(R) == 4)
      return launch_step_f32_tma(K, make_coef<float>(K), P, *tm, (float *)psi_n, (float *)c_n, (float *)phi_n,
                                 partials, max_partials, nwarps_out, err, st);
    else
      return launch_step_f64_tma(K, F, P, *tm, (double *)psi_n, (double *)c_n, (double *)phi_n, partials,
                                 max_partials, nwarps_out, err, st);
  }
  const int wcols = (ni + 29) / 30;
  constexpr int WPB = 4;  // warps per block (adjacent column strips)
  constexpr int PF = 3;   // rows in flight per lane (multiple of the 3-row window)
  // rows per block.  Frozen temperature, and FP32: 64, halved while the grid
  // has fewer than 16 warp strips per SM; the blocks at the front take far
  // longer than the others, and a part-filled last wave absorbs them (a grid
  // of exactly full waves measured slower with a front, faster without one).
  // FP64 with the coarse-grid temperature, where every cell evaluates its
  // CALPHAD groups in FP64 and the blocks cost about the same: the height in
  // [16, 64] whose grid fills its last wave of resident blocks best, by
  // (waves) x (H + 4) (H rows, 2 halo rows and about 2 rows' worth of
  // per-strip setup), among heights giving at least three waves where there
  // are such (FP32 measured no gain from it)
  constexpr bool kFillable = sizeof(R) == 8;
  const bool fill = kFillable && tfc;
  const int ncb = (wcols + WPB - 1) / WPB;
  int H = 64;
  while (!fill && H > 16 && (int64_t)wcols * ((nj + H - 1) / H) < 148 * 16) H /= 2;
  int64_t best = fill ? INT64_MAX : 0;
  int resident = 1;
  if constexpr (kFillable) {
    if (fill) {
      static std::atomic<int> resident_of[64];
      resident = resident_ctas((const void *)step_kernel<R, 0, PF, true>, 32 * WPB, 0, resident_of);
      if (resident <= 0) return -3;
    }
  }
  for (int pass = 0; pass < 2 && best == INT64_MAX; ++pass) {
    for (int h = 16; h <= 64; ++h) {
      const int64_t blocks = (int64_t)ncb * ((nj + h - 1) / h);
      const int64_t waves = (blocks + resident - 1) / resident;
      if (pass == 0 && waves < 3) continue;
      const int64_t cost = waves * (h + 4);
      if (cost < best) {
        best = cost;
        H = h;
      }
    }
  }
  dim3 block(32 * WPB), grid((nj + H - 1) / H, ncb);
  if (grid.y > 65535) return -1;
  const int nw = grid.x * grid.y * WPB;
  if (partials && nw > max_partials) return -1;
#define RS_LAUNCH(HC, TF) step_kernel<R, HC, PF, TF><<<grid, block, 0, st>>>(K, F, P, psi, c, psi_n, c_n, phi_n, partials, H)
  if constexpr (kFillable) {
    if (fill) RS_LAUNCH(0, true);
  }
  if (!fill) {
    if (H == 64) {
      if (tfc) RS_LAUNCH(64, true); else RS_LAUNCH(64, false);
    } else if (H == 32) {
      if (tfc) RS_LAUNCH(32, true); else RS_LAUNCH(32, false);
    } else {
      if (tfc) RS_LAUNCH(16, true); else RS_LAUNCH(16, false);
    }
  }
#undef RS_LAUNCH
  if (nwarps_out) *nwarps_out = nw;
  return 0;
}

int launch_step_f64(const StepCoef &K, const StepScalars &P, const double *psi, const double *c, double *psi_n,
                    double *c_n, double *phi_n, BlockPartial *partials, int max_partials, int *nb, const TmaMaps *tm,
                    int *err, cudaStream_t st) {
  return launch<double>(K, P, psi, c, psi_n, c_n, phi_n, partials, max_partials, nb, tm, err, st);
}

int launch_step_f32(const StepCoef &K, const StepScalars &P, const float *psi, const float *c, float *psi_n,
                    float *c_n, float *phi_n, BlockPartial *partials, int max_partials, int *nb, const TmaMaps *tm,
                    int *err, cudaStream_t st) {
  return launch<float>(K, P, psi, c, psi_n, c_n, phi_n, partials, max_partials, nb, tm, err, st);
}

}  // namespace rs

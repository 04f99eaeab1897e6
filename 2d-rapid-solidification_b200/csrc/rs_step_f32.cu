// rs_step_f32.cu — the FP32 fused phase-field step on TMA-staged tiles.
//
// Same equations as the register-prefetch kernel of rs_step.cu
// (compute_phi / compute_psi / compute_c_CALPHAD, fun.cu:1143-1467).  One
// step is two launches:
//   * column_table_kernel: the per-column CALPHAD groups of this step's frozen
//     temperature (t_terms in FP64, get_delta fun.cu:1610-1619), rounded to
//     FP32, plus the FP64 column differences of the composition-independent
//     part of mu;
//   * tile_kernel, launched as a programmatic dependent of the table kernel:
//     its CTAs start, issue their TMA loads, and wait for the table only
//     where they first read it.
//
// A CTA of 128 threads owns a tile of 16 output rows x 128 output columns
// (x0 .. x0+127, x0 a multiple of 128).  Its input, 18 rows x 136 columns
// (x0-4 .. x0+131, so the TMA x coordinate stays 16-byte aligned), arrives in
// shared memory by one TMA box per field.  Four adjacent columns per lane.
//   phase 1  per-cell S = q(psi) c (1-c) and mu'' (below) of the 18 input
//            rows into shared memory, with per-row flags "every psi == -1" /
//            "== +1" and per-lane phi masks; the halo columns x0-1 and
//            x0+128 are computed by 36 threads of warps 2 and 3 (one input
//            row fewer than warps 0 and 1);
//   phase 2  each warp computes 4 output rows: fluxes through the faces from
//            the shared S and mu'', the c update (kept in registers); cells
//            whose 3x3 phi neighbourhood is not uniformly +-1 are listed;
//   phase 3  the listed interface cells are updated one per thread
//            (phi_cell), so a tile's interface work is spread over the CTA;
//   phase 4  new psi and c are written into the shared tile, ghost columns
//            copied there, and each output row leaves by one bulk async copy
//            per field (ghost rows by one more, except in row-band mode);
//   partials when the caller wants the solute mass or the coarse tip, each
//            CTA writes its partial sums and the last CTA to finish reduces
//            them all (same order as the separate reduction kernel).
// Arithmetic:
//   * mu = K(T) + C0(T) + mu'' with C0 = -D - (L0_BCC - L0_Liq)(1 - 2 cinf)/2
//     (D, K(T) as in rs_step.cu), so
//       mu'' = -(g+1) C0 - delta (L0_BCC + L0_Liq + g (L0_BCC - L0_Liq)) + RT lam,
//     which is small in the melt; K + C0 enters only through its FP64 column
//     differences dK;
//   * rows whose cells are all bulk liquid (psi = -1 exactly, |s| < 1/9) take
//     the short form: g(-1) = -1 and q(-1) = 1, so
//     mu'' = -2 L0_Liq delta + RT lam(delta) and S = c (1 - c);
//   * rows whose cells have psi = +1 exactly over their 3x3 neighbourhoods
//     (deep solid) store S = mu'' = 0: q(1) = 0, so every face weight touching
//     the row is 0 and its mu'' enters no flux (no network pass either);
//   * face weights use pair sums: the face (i, r+1/2) has
//     6 P_i + P_{i-1} + P_{i+1} with P_i = S(i,r) + S(i,r+1), and the face
//     (i+1/2, r) has 6 Q_r + Q_{r-1} + Q_{r+1} with Q_r = S(i,r) + S(i+1,r):
//     four times the 1.5 / 0.25 weights of rs_step.cu, the 4 folded into the
//     flux constant; face fluxes are rounded products, so a cell's result
//     does not depend on where the tiling puts it;
//   * interface noise is keyed by the global cell (row + j_offset in
//     row-band mode).
// Launch order: the tile columns from the one holding the front
// (front_first_block), whose interface and network work is the slowest.
// After phase 1 each CTA prefetches into L2 the input tile of the block
// launched one resident wave later, so the tiles of the next wave arrive
// while this wave computes (the CTAs of a wave otherwise load, compute and
// store in step).
// The coarse-grid temperature (TFC, interpolate_temperature fun.cu:1580-1608)
// takes tile_kernel_tfc alone: every cell evaluates its CALPHAD groups from its
// own bilinear temperature (K + C0 by its Taylor polynomial about the tile's
// centre temperature, kc_poly), keeps K + C0 in FP64 in shared memory, and the
// faces add its differences, rounded to FP32, along both axes; tiles of 8
// output rows, so that the FP64 array fits with five CTAs per SM.
// Fields store psi and delta = c - cinf (include/rs_b200.h).
#include "rs_step_common.cuh"
#include "rs_surrogate.cuh"
#include "rs_ensemble.cuh"

namespace rs {
namespace {

constexpr int kW = kTileOutW;     // output columns of a tile
constexpr int kWin = kTmaBoxW32;  // input columns of a tile (kW + 8)
constexpr int kTR = kTileRows;    // output rows of a tile
constexpr int kTRin = kTmaBoxH;   // input rows of a tile
constexpr int kThreads = 128;
constexpr int kWarps = kThreads / 32;
constexpr int kRowsPerWarp = kTR / kWarps;
constexpr int kHaloL = 3, kHaloR = kW + 4;  // box columns of x0-1 and x0+kW
constexpr uint32_t kWaitLimit = 1u << 20;
constexpr unsigned FULL = 0xffffffffu;
static_assert(kW == 32 * 4, "four columns per lane");
static_assert(kTR % kWarps == 0 && kRowsPerWarp == 4, "four output rows per warp");
static_assert(kTRin <= 32, "row flags are 32-bit masks");
static_assert(64 + 2 * kTRin <= kThreads && 4 * kTR <= kThreads, "one thread per halo cell and per row copy");

// column table arrays (kColTabFields of them, col_tab_len floats each);
// entry k describes column k - 4
enum { kTabRT = 0, kTabC0 = 1, kTabDK = 2, kTabAnb = 3, kTabAti = 4 };

// Shared memory of one tile of TR output rows x kW output columns (input
// TR + 2 rows); the ensemble kernels take TR = 8, 16 or 32 (kTileShapes), the
// single-run kernel TR = kTR.
template <int TR, bool TFC = false>
struct alignas(128) TileSmemT {
  static constexpr int kRin = TR + 2;  // input rows
  using Mask = std::conditional_t<(kRin <= 32), uint32_t, unsigned long long>;  // one bit per input row
  // TMA destinations (128-byte aligned); rows 1..TR receive the new psi / c - cinf
  alignas(128) float psi[kRin][kWin];
  alignas(128) float d[kRin][kWin];
  alignas(16) float S[kRin][kWin];  // after phase 2: new psi of the listed cells
  alignas(16) float mu[kRin][kWin];
  // TFC: K + C0 of every cell in FP64 (the face terms are its differences)
  alignas(16) double kc[TFC ? kRin : 1][TFC ? kWin : 2];
  uint16_t list[TR * kW];   // interface cells: row << 8 | output column
  uint8_t pmask[kRin][32];  // per lane: bits 0-3 psi <= -1, bits 4-7 psi >= 1 of its four cells
  uint8_t hmask[kRin][2];   // halo cells: bit 0 psi <= -1, bit 1 psi >= 1
  Mask liq, sol;            // bit r: every cell of input row r has psi == -1 / +1
  double ty[kRin];          // TFC: the row part of each input row's temperature
  int tj[kRin];             // (tfc_row), once per tile
  std::conditional_t<TFC, KcPoly, char> kp;  // TFC: K + C0 near the tile's temperature
  double hx[2];             // TFC: column part of the halo columns' temperatures
  int hiT[2];
  int nlist;
  double part_mass[kWarps];
  int part_itip[kWarps];
  uint64_t full;
  int last;  // this CTA finished last (fused final reduction)
};
using TileSmem = TileSmemT<kTR>;

static_assert(offsetof(TileSmem, psi) % 128 == 0 && offsetof(TileSmem, d) % 128 == 0 &&
                  offsetof(TileSmemT<8>, d) % 128 == 0 && offsetof(TileSmemT<32>, d) % 128 == 0,
              "TMA destinations start on 128-byte boundaries");
static_assert(sizeof(TileSmemT<8>::S) >= 256 * sizeof(double) && sizeof(TileSmemT<8>::mu) >= 256 * sizeof(int),
              "the final reduction's scratch fits S and mu");
static_assert((kWin * sizeof(float)) % 16 == 0, "rows stay 16-byte aligned for float4 and bulk copies");

__device__ __forceinline__ float4 ld4(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ void st4(float *p, float a, float b, float c, float e) {
  *reinterpret_cast<float4 *>(p) = make_float4(a, b, c, e);
}
__device__ __forceinline__ float clamp1(float v) { return fminf(fmaxf(v, -1.f), 1.f); }

// general per-cell terms (fun.cu:1424-1452)
__device__ __forceinline__ void cell_terms(const Coef<float> &F, float pv, float dv, float RT, float C0, float &S,
                                           float &mu) {
  constexpr float L0sum = (float)(kL0Bcc + kL0Liq);
  constexpr float L0half = (float)(0.5 * (kL0Bcc - kL0Liq));
  const float c = F.cinf + dv, om = 1.f - c;
  const float a = 1.f - pv;
  S = (0.5f * F.AA * a - 0.25f * (F.AA - 1.f) * (a * a)) * c * om;
  const float p2 = pv * pv;
  const float g = pv * (1.875f + p2 * (-1.25f + 0.375f * p2));
  const float lam = Tr<float>::lam(c, om, dv, F.cinf, F.Lref);
  mu = -(g + 1.f) * C0 - dv * fmaf(2.f * L0half, g, L0sum) + RT * lam;
}

// shared -> global bulk copy (16-byte aligned addresses, size a multiple of 16)
__device__ __forceinline__ void bulk_store(void *gdst, const void *ssrc, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gdst), "r"(smem_u32(ssrc)),
               "r"(bytes)
               : "memory");
}

// One thread per column, one t_terms each (c/T terms by one reciprocal: the
// groups are rounded to FP32); K + C0 of the next column comes from the
// neighbouring thread, so blocks overlap by one column and write 127 entries.
constexpr int kTabBlock = 128;
// kc: kTabBlock doubles of shared scratch
__device__ __forceinline__ void table_block(const StepCoef &K, const double d0, const double d1, const int len,
                                            float *__restrict__ tab, const int blk, double *kc) {
  const int k = blk * (kTabBlock - 1) + threadIdx.x;  // table entry; column k - 4
  const int gi = min(max(k - 4, 0), K.nx - 1);
  const double T = (d0 + d1 * gi) * K.deltaT0 + K.Tmelt;  // get_delta, fun.cu:1610-1619
  const TTerms tt = t_terms(T, K.RR, true);
  const double D = 0.5 * (tt.dGs - tt.dGl);
  const double C0 = -D - 0.5 * (kL0Bcc - kL0Liq) * (1.0 - 2.0 * K.cinf);
  kc[threadIdx.x] = 0.5 * (tt.dGs + tt.dGl) + 0.5 * (kL0Bcc + kL0Liq) * (1.0 - 2.0 * K.cinf) + tt.RT * K.Lref + C0;
  __syncthreads();
  if (threadIdx.x == kTabBlock - 1 || k >= len) return;
  tab[kTabRT * len + k] = (float)tt.RT;
  tab[kTabC0 * len + k] = (float)C0;
  tab[kTabDK * len + k] = (float)(kc[threadIdx.x + 1] - kc[threadIdx.x]);  // (K + C0)(i+1) - (K + C0)(i)
  tab[kTabAnb * len + k] = (float)tt.A_nb;
  tab[kTabAti * len + k] = (float)tt.A_ti;
}

__global__ void __launch_bounds__(kTabBlock) column_table_kernel(const StepCoef K, const double d0, const double d1,
                                                                 const int len, float *__restrict__ tab) {
  // the tile kernel may start now; it waits for this grid before reading tab
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  __shared__ double kc[kTabBlock];
  table_block(K, d0, d1, len, tab, blockIdx.x, kc);
}

// SURR: mu'' and the driving force of in-box cells that are not bulk melt
// come from the learned surrogate (rs_surrogate.cuh) instead of the exact
// evaluation.  Bulk-melt cells (psi == -1 exactly, delta in the series range)
// keep the exact series form: it is exact and cheaper than the network.
// The work of one CTA on tile (row tile tr, column tile tc) of a field set;
// part: this tile's partial (mass, coarse tip), or nullptr.
// TR: output rows of the tile (8, 16 or 32; the tensor maps' box is TR + 2
// rows high).
template <bool SURR, int TR, typename Prefetch, bool TFC = false>
__device__ __forceinline__ void tile_body(const StepCoef &K, const Coef<float> &F, const StepScalars &PS,
                                          const CUtensorMap *tm_psi, const CUtensorMap *tm_c,
                                          const float *__restrict__ tab, const int tab_len, float *__restrict__ psi_n,
                                          float *__restrict__ c_n, float *__restrict__ phi_n, BlockPartial *part,
                                          int *err, const SurrArgs &SA, const int tr, const int tc,
                                          const FinalRed *FR, const Prefetch &prefetch) {
  // the tile's shape (these hide the single-run constants of the same names)
  constexpr int kTR = TR, kTRin = TR + 2, kRowsPerWarp = TR / kWarps;
  static_assert(TR % kWarps == 0 && kRowsPerWarp * 4 <= 32, "output rows split evenly over the warps");
  // halo-column threads: the last warps, which have one input row fewer
  constexpr int kHalo0 = (64 + 2 * kTRin <= kThreads) ? 64 : kThreads - 2 * kTRin;
  static_assert(kHalo0 >= 0 && 4 * kTR <= kThreads, "one thread per halo cell and per row copy");
  static_assert(!(SURR && TFC), "the surrogate takes the frozen temperature");
  using Smem = TileSmemT<TR, TFC>;
  using Mask = typename Smem::Mask;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  Smem &sm = *reinterpret_cast<Smem *>(smem_raw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int x0 = kW * tc;       // first output column of the tile
  const int y0 = 1 + kTR * tr;  // first output row; input rows y0-1 .. y0+kTR
  constexpr uint32_t kTileBytes = 2u * kTRin * kWin * sizeof(float);

  if (smem_u32(smem_raw) & 127u) {  // TMA destinations must be 128-byte aligned
    if (threadIdx.x == 0) atomicExch(err, 2);
    return;
  }
  // a pull-back step reads column clamp(i + i_offset, 1, nx - 2) for column i
  // (pull_back, fun.cu:1469-1492): no TMA box has that shape, so the CTA
  // gathers its tile instead (same box, zeros outside the array, delta = 0
  // where the source is column nx - 2: the melt entering at the right edge)
  const bool pb = PS.pull_back != 0;
  if (threadIdx.x == 0) {
    mbar_init(&sm.full, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    if (!pb) {
      mbar_expect_tx(&sm.full, kTileBytes);
      tma_load_2d(&sm.psi[0][0], tm_psi, &sm.full, x0 - 4, y0 - 1);
      tma_load_2d(&sm.d[0][0], tm_c, &sm.full, x0 - 4, y0 - 1);
    }
    sm.liq = 0;
    sm.sol = 0;
    sm.nlist = 0;
  }

  const int col = 4 * lane;  // tile column of this lane's first cell
  const int gi = x0 + col;   // its global column
  const int bc = col + 4;    // its box column
  uint32_t outm = 0;         // per cell: an interior (output) cell
#pragma unroll
  for (int q = 0; q < 4; ++q)
    if (gi + q >= 1 && gi + q <= K.nx - 2) outm |= 1u << q;
  // launch constants of the row loops in registers (one read of the
  // arguments, which may live in global memory for the ensemble)
  const int ny = K.ny, nx = K.nx;
  const float cinf = F.cinf, tiny = F.melt_tiny;
  const float ma0 = F.melt_a[0], ma1 = F.melt_a[1], ma2 = F.melt_a[2], ma3 = F.melt_a[3];
  const float two_cinf = F.cinf + F.cinf;
  const float cflux4 = 0.25f * F.cflux;
  const float floor_d = F.c_floor - F.cinf;
  constexpr float KL = (float)(-2.0 * kL0Liq);
  const float d_hi = F.ser_hi, d_lo = F.ser_lo;  // series range of delta (Coef)
  constexpr uint32_t kMinus1 = 0xBF800000u, kPlus1 = 0x3F800000u;

  // the column table of this step (programmatic dependency on its kernel)
  asm volatile("griddepcontrol.wait;" ::: "memory");
  // the step's final reduction (a programmatic dependent) may be scheduled now
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const float *tRT = tab + kTabRT * tab_len + 4, *tC0 = tab + kTabC0 * tab_len + 4;
  const float *tDK = tab + kTabDK * tab_len + 4;
  float4 RTv = make_float4(0.f, 0.f, 0.f, 0.f), C0v = RTv, dKv = RTv;
  float dKl = 0.f;
  if constexpr (!TFC) {
    RTv = ld4(tRT + gi);
    C0v = ld4(tC0 + gi);
  }
  if constexpr (!TFC && !SURR) {
    // dK of the lane's faces, loaded now so that the load hides under the
    // tile's (the surrogate path, short of registers, loads them after phase 1)
    dKv = ld4(tDK + gi);
    dKl = tDK[gi - 1];
  }
  // TFC: RT and C0 per row, from each cell's own temperature
  float RTa[4] = {RTv.x, RTv.y, RTv.z, RTv.w}, C0a[4] = {C0v.x, C0v.y, C0v.z, C0v.w};
  // TFC: the column part of each cell's temperature (interpolate_temperature,
  // fun.cu:1580-1608); the row part and K + C0 about the tile's centre once
  // per tile, in shared memory
  int tiT[4] = {0, 0, 0, 0};
  double tx[4] = {0.0, 0.0, 0.0, 0.0};
  if constexpr (TFC) {
#pragma unroll
    for (int q = 0; q < 4; ++q) tfc_col(K, PS.i_left_end_T, gi + q, tiT[q], tx[q]);
    if (threadIdx.x < kTRin) tfc_row(K, y0 - 1 + (int)threadIdx.x, sm.tj[threadIdx.x], sm.ty[threadIdx.x]);
    if (threadIdx.x >= kTRin + 1 && threadIdx.x < kTRin + 3) {  // the halo columns x0-1, x0+kW
      const int side = (int)threadIdx.x - (kTRin + 1);
      tfc_col(K, PS.i_left_end_T, side ? x0 + kW : x0 - 1, sm.hiT[side], sm.hx[side]);
    }
    if (threadIdx.x == kTRin) {
      int iT, jT;
      double x, y;
      tfc_col(K, PS.i_left_end_T, x0 + kW / 2, iT, x);
      tfc_row(K, y0 + kTR / 2, jT, y);
      sm.kp = kc_poly(K, tfc_T(K, PS.T_coarse, iT, x, jT, y));
    }
  }
  // TFC: all groups of one cell, the logarithm exact (halo and interface cells)
  auto tfc_cell = [&](int gx, int row) {
    int iT, jT;
    double x, y;
    tfc_col(K, PS.i_left_end_T, gx, iT, x);
    tfc_row(K, row, jT, y);
    return groups_exact(K, tfc_T(K, PS.T_coarse, iT, x, jT, y));
  };
  // surrogate: per-lane fragments, and the scaled inputs as T(x) = TnA + TnB x
  // (tile column x; frozen T is linear in the column) and c = cnA + delta c_ihalf
  float TnA = 0.f, TnB = 0.f, cnA = 0.f;
  const float *tAnb = tab + kTabAnb * tab_len + 4, *tAti = tab + kTabAti * tab_len + 4;
  if constexpr (SURR) {
    const double T0 = (PS.d0 + PS.d1 * x0) * K.deltaT0 + K.Tmelt;
    TnA = (float)((T0 - SA.T_mid) * SA.T_ihalf);
    TnB = (float)(PS.d1 * K.deltaT0 * SA.T_ihalf);
    cnA = (F.cinf - SA.c_mid) * SA.c_ihalf;
  }
  // a cell the series form covers (the network is not used there)
  auto melt_cell = [&](int rr, int b) {
    const float dv = sm.d[rr][b];
    return __float_as_uint(sm.psi[rr][b]) == kMinus1 && dv < d_hi && dv > d_lo;
  };
  // a halo cell's mu'' enters only the face to the tile's edge column, whose
  // weight is 0 when psi is exactly +1 on both columns over rows rr-1..rr+1;
  // column -1 (left-most tile) enters no face at all (column 0 is a ghost)
  auto halo_mu_used = [&](int rr, int b) {
    if (b == kHaloL && x0 == 0) return false;
    const int b2 = b == kHaloL ? b + 1 : b - 1;
    bool solid = true;
    for (int r2 = max(rr - 1, 0); r2 <= min(rr + 1, kTRin - 1); ++r2)
      solid = solid && __float_as_uint(sm.psi[r2][b]) == kPlus1 && __float_as_uint(sm.psi[r2][b2]) == kPlus1;
    return !solid;
  };
  // per lane, bit q: psi is exactly +1 over the 3x3 neighbourhood of cell
  // bc+q (rows of the box only: faces to rows outside it are not computed;
  // column -1 of the left-most tile enters no face, column 0 being a ghost).
  // S = q(1) c (1 - c) = 0 there, so every face weight touching the cell is 0
  // and its mu'' enters no flux (0 times a finite difference)
  auto solid3 = [&](int rr) -> uint32_t {
    const int xh = lane == 0 ? kHaloL : kHaloR;
    uint32_t v = 0xFu;
    bool hs = true;  // the halo column beside lanes 0 and 31
    for (int r2 = max(rr - 1, 0); r2 <= min(rr + 1, kTRin - 1); ++r2) {
      const float4 q4 = ld4(&sm.psi[r2][bc]);
      v &= (__float_as_uint(q4.x) == kPlus1 ? 1u : 0u) | (__float_as_uint(q4.y) == kPlus1 ? 2u : 0u) |
           (__float_as_uint(q4.z) == kPlus1 ? 4u : 0u) | (__float_as_uint(q4.w) == kPlus1 ? 8u : 0u);
      hs = hs && __float_as_uint(sm.psi[r2][xh]) == kPlus1;
    }
    uint32_t lf = __shfl_up_sync(FULL, v >> 3, 1) & 1u, rt = __shfl_down_sync(FULL, v, 1) & 1u;
    if (lane == 0) lf = (hs || x0 == 0) ? 1u : 0u;
    if (lane == 31) rt = hs ? 1u : 0u;
    const uint32_t e = lf | (v << 1) | (rt << 5);  // bit k: box column bc-1+k
    return e & (e >> 1) & (e >> 2) & 0xFu;
  };
  auto net_inputs = [&](int rr, int b, float in[3]) {  // b: box column
    in[0] = fmaf(TnB, (float)(b - 4), TnA);
    in[1] = fmaf(sm.d[rr][b], SA.c_ihalf, cnA);
    in[2] = clamp1(sm.psi[rr][b]);
  };
  // store the surrogate mu'' of one cell, or keep the exact value already in
  // place (out-of-box and audited cells); audited cells record the errors
  auto net_store = [&](int rr, int b, const float in[3], const float o[2]) {
    const int gx = x0 + b - 4;
    const float T = SA.T_mid + in[0] / SA.T_ihalf, c = F.cinf + sm.d[rr][b];
    const bool inbox = T >= SA.T_lo && T <= SA.T_hi && c >= SA.c_lo && c <= SA.c_hi;
    const bool real = gx >= 0 && gx <= K.nx - 1;
    const bool audit = real && surr_audit_cell(PS.step, (int64_t)(y0 - 1 + rr + K.j_offset) * K.nx + gx);
    const float mu_net = fmaf(o[0], SA.y_scale[0], SA.y_mean[0]);
    if (inbox && !audit) {
      sm.mu[rr][b] = mu_net;
    } else if (real) {
      if (!inbox) atomicAdd(&SA.audit[2], 1ull);
      if (audit) {
        const float dG_ex = (1.f - c) * tAnb[gx] + c * tAti[gx] + c * (1.f - c) * (float)(kL0Liq - kL0Bcc);
        const float dG_net = fmaf(o[1], SA.y_scale[1], SA.y_mean[1]);
        atomicMax(&SA.audit[0], (unsigned long long)__float_as_uint(fabsf(mu_net - sm.mu[rr][b])));
        atomicMax(&SA.audit[1], (unsigned long long)__float_as_uint(fabsf(dG_net - dG_ex)));
        atomicAdd(&SA.audit[3], 1ull);
      }
    }
  };
  // the partial sums of this tile and the fused final reduction (the last
  // CTA to finish sums every partial, in reduce_partials_kernel's order)
  auto finish = [&](double mass, int itip) {
    if (!part) return;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mass += __shfl_down_sync(FULL, mass, o);
    itip = __reduce_max_sync(FULL, itip);
    if (lane == 0) {
      sm.part_mass[warp] = mass;
      sm.part_itip[warp] = itip;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      BlockPartial b;
      b.mass = 0.0;
      b.itip = 0;
#pragma unroll
      for (int w = 0; w < kWarps; ++w) {
        b.mass += sm.part_mass[w];
        b.itip = max(b.itip, sm.part_itip[w]);
      }
      b.pad = 0;
      *part = b;
    }
    if (!FR) return;
    if (threadIdx.x == 0) {
      __threadfence();
      sm.last = atomicAdd(FR->counter, 1u) == (unsigned)(FR->nparts - 1);
    }
    __syncthreads();
    if (!sm.last) return;
    __threadfence();
    double *sm_m = reinterpret_cast<double *>(&sm.S[0][0]);  // S and mu are free now
    int *sm_i = reinterpret_cast<int *>(&sm.mu[0][0]);
    final_reduce(*FR, sm_m, sm_i, (int)threadIdx.x, [] { __syncthreads(); });
  };
  if (pb) {
    const float *__restrict__ gpsi = static_cast<const float *>(PS.src_psi);
    const float *__restrict__ gd = static_cast<const float *>(PS.src_c);
    for (int k = threadIdx.x; k < kTRin * kWin; k += kThreads) {
      const int rr = k / kWin, x = k % kWin;
      const int row = y0 - 1 + rr, g = x0 - 4 + x;
      float pv = 0.f, dv = 0.f;
      if (row <= ny - 1 && g >= 0 && g <= nx - 1) {
        const int si = min(max(g + PS.i_offset, 1), nx - 2);
        const int64_t o = (int64_t)row * K.pitch + si;
        pv = gpsi[o];
        dv = si >= nx - 2 ? 0.f : gd[o];
      }
      sm.psi[rr][x] = pv;
      sm.d[rr][x] = dv;
    }
  }
  __syncthreads();  // barrier initialised, flags cleared (a pull-back tile gathered)
  if (!pb) {
    // bounded wait for the tile; if any thread gives up, the whole CTA skips
    // the tile: no phase runs on a partly filled tile and nothing is stored.
    // Thread 0 first waits (bounded again) for the load still in flight into
    // this CTA's shared memory, and the CTA still reports a (zero) partial,
    // so the fused final reduction keeps its count
    const uint32_t limit = PS.wait_limit ? PS.wait_limit : kWaitLimit;
    uint32_t tries = 0;
    bool gave_up = false;
    while (!mbar_try(&sm.full, 0, PS.wait_limit != 0)) {
      if (++tries >= limit) {
        gave_up = true;
        break;
      }
    }
    if (__syncthreads_or(gave_up)) {
      if (threadIdx.x == 0) {
        atomicExch(err, 1);
        for (uint32_t t = 0; t < kWaitLimit && !mbar_try_wait(&sm.full, 0); ++t) {
        }
      }
      __syncthreads();
      finish(0.0, 0);
      return;
    }
  }
  // columns beyond the array (right-most tiles; zero-filled by TMA) become
  // bulk melt, so they never force the general path; no output reads them
  if (x0 + kW + 4 > K.nx) {
    for (int k = threadIdx.x; k < kTRin * kWin; k += kThreads) {
      const int rr = k / kWin, x = k % kWin;
      if (x0 - 4 + x >= K.nx) {
        sm.psi[rr][x] = -1.f;
        sm.d[rr][x] = 0.f;
      }
    }
    __syncthreads();
  }

  // ---- phase 1: per-cell terms; warp w takes input rows w, w+4, ...
  // The warp's row flags (warp-uniform) are OR-ed into sm.liq / sm.sol once;
  // rows flagged there store no phi masks (phase 2 takes 0x0F / 0xF0)
  Mask liq_rows = 0, sol_rows = 0;
#pragma unroll 1
  for (int rr = warp; rr < kTRin; rr += kWarps) {
    if (y0 - 1 + rr > ny - 1) {  // beyond the array (last tile): never read by an output
      st4(&sm.S[rr][bc], 0.f, 0.f, 0.f, 0.f);
      st4(&sm.mu[rr][bc], 0.f, 0.f, 0.f, 0.f);
      if constexpr (TFC) {
        *reinterpret_cast<double2 *>(&sm.kc[rr][bc]) = make_double2(0.0, 0.0);
        *reinterpret_cast<double2 *>(&sm.kc[rr][bc + 2]) = make_double2(0.0, 0.0);
      }
      liq_rows |= Mask(1) << rr;
      sol_rows |= Mask(1) << rr;
      continue;
    }
    const float4 pv4 = ld4(&sm.psi[rr][bc]), dv4 = ld4(&sm.d[rr][bc]);
    const float pv[4] = {pv4.x, pv4.y, pv4.z, pv4.w}, dv[4] = {dv4.x, dv4.y, dv4.z, dv4.w};
    float Sv[4], mv[4];
    // bulk melt: every psi exactly -1 (bit tests) and every delta in the
    // series range
    const uint32_t b0 = __float_as_uint(pv[0]), b1 = __float_as_uint(pv[1]), b2 = __float_as_uint(pv[2]),
                   b3 = __float_as_uint(pv[3]);
    const uint32_t band = b0 & b1 & b2 & b3, bor = b0 | b1 | b2 | b3;
    const float dmx = fmaxf(fmaxf(dv[0], dv[1]), fmaxf(dv[2], dv[3]));
    const float dmn = fminf(fminf(dv[0], dv[1]), fminf(dv[2], dv[3]));
    const bool liq4 = band == kMinus1 && bor == kMinus1;
    // the row's form (warp-uniform): far melt, bulk melt or general (voted
    // here with TFC, where it decides which groups to evaluate)
    bool far = false, bulk = false;
    if constexpr (TFC) {  // the melt forms need RT and K + C0 only
      far = __all_sync(FULL, liq4 && fmaxf(dmx, -dmn) <= tiny);
      bulk = !far && __all_sync(FULL, liq4 && dmx < d_hi && dmn > d_lo);
      const int jT = sm.tj[rr];
      const double y = sm.ty[rr];
      double kq[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        double RT, C0;
        cell_tfc(K, sm.kp, tfc_T(K, PS.T_coarse, tiT[q], tx[q], jT, y), !(far || bulk), RT, C0, kq[q]);
        RTa[q] = (float)RT;
        C0a[q] = (float)C0;
      }
      *reinterpret_cast<double2 *>(&sm.kc[rr][bc]) = make_double2(kq[0], kq[1]);
      *reinterpret_cast<double2 *>(&sm.kc[rr][bc + 2]) = make_double2(kq[2], kq[3]);
    }
    uint32_t code, s3 = 0u;
    if (TFC ? far : __all_sync(FULL, liq4 && fmaxf(dmx, -dmn) <= tiny)) {
      // far melt: lam by its Taylor polynomial in delta (Coef::melt_a);
      // mu'' = RT lam - 2 L0_Liq delta = delta (RT p + KL), lam = delta p
      code = 1u | 4u;  // 4: every cell in the exact melt form
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const float c = cinf + dv[q], om = 1.f - c;
        float p = fmaf(ma3, dv[q], ma2);
        p = fmaf(p, dv[q], ma1);
        p = fmaf(p, dv[q], ma0);
        Sv[q] = c * om;
        mv[q] = dv[q] * fmaf(RTa[q], p, KL);
      }
    } else if (TFC ? bulk : __all_sync(FULL, liq4 && dmx < d_hi && dmn > d_lo)) {
      code = 1u | 4u;  // 4: every cell in the series form
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const float c = cinf + dv[q], om = 1.f - c;
        const float sv = __fdividef(dv[q], fmaf(two_cinf, om, dv[q]));
        const float s2 = sv * sv;
        // atanh(s) to s^7: relative truncation below 2.6e-9 for |s| < 1/9
        float p = fmaf(s2, 1.f / 7.f, 1.f / 5.f);
        p = fmaf(s2, p, 1.f / 3.f);
        const float ath = fmaf(sv * s2, p, sv);  // atanh(s); lam = 2 atanh(s)
        Sv[q] = c * om;
        mv[q] = fmaf(RTa[q] + RTa[q], ath, dv[q] * KL);
      }
    } else {
      const bool sol4 = band == kPlus1 && bor == kPlus1;
      code = (__all_sync(FULL, liq4) ? 1u : 0u) | (__all_sync(FULL, sol4) ? 2u : 0u);
      // deep solid row: no cell's mu'' enters a flux (solid3), so S = mu'' = 0
      // gives the same fluxes.  The surrogate also skips solid3 cells, which
      // pays only where a whole 16-cell network pass (lanes 4m .. 4m+3) is
      // solid
      bool want = (code & 2u) != 0u;
      if constexpr (SURR) {
        const uint32_t fs = __ballot_sync(FULL, sol4);
        want = want || (fs & (fs >> 1) & (fs >> 2) & (fs >> 3) & 0x11111111u) != 0u;
      }
      if (want) s3 = solid3(rr);
      const bool deep = (code & 2u) && __all_sync(FULL, s3 == 0xFu);
      if (deep) {
        code |= 8u;  // 8: mu'' not needed (no network pass either)
#pragma unroll
        for (int q = 0; q < 4; ++q) Sv[q] = mv[q] = 0.f;
      } else {
        uint32_t L = 0u, Sm = 0u;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          if (pv[q] <= -1.f) L |= 1u << q;
          if (pv[q] >= 1.f) Sm |= 1u << q;
          cell_terms(F, pv[q], dv[q], RTa[q], C0a[q], Sv[q], mv[q]);
        }
        sm.pmask[rr][lane] = (uint8_t)(L | (Sm << 4));
      }
    }
    st4(&sm.S[rr][bc], Sv[0], Sv[1], Sv[2], Sv[3]);
    st4(&sm.mu[rr][bc], mv[0], mv[1], mv[2], mv[3]);
    liq_rows |= Mask(code & 1u) << rr;
    sol_rows |= Mask((code >> 1) & 1u) << rr;
    if constexpr (SURR) {  // the row's non-melt cells through the network, 16 at a time
      if (!(code & (4u | 8u))) {
        __syncwarp();
        const SurrConst SC = surr_load(SA, lane);
        const int g = lane >> 2;
        const bool any3 = __any_sync(FULL, s3 != 0u);
#pragma unroll 1
        for (int mt = 0; mt < kW / 16; ++mt) {
          const int ba = 4 + 16 * mt + g, bb = ba + 8;
          bool na = !melt_cell(rr, ba), nb = !melt_cell(rr, bb);
          if (any3) {  // warp-uniform
            const uint32_t sa = __shfl_sync(FULL, s3, (ba - 4) >> 2), sb = __shfl_sync(FULL, s3, (bb - 4) >> 2);
            na = na && !((sa >> ((ba - 4) & 3)) & 1u);
            nb = nb && !((sb >> ((bb - 4) & 3)) & 1u);
          }
          if (!__any_sync(FULL, na || nb)) continue;
          float in0[3], in1[3], o0[2], o1[2];
          net_inputs(rr, ba, in0);
          net_inputs(rr, bb, in1);
          surr_tile16(SC, in0, in1, o0, o1);
          if ((lane & 3) == 0) {
            if (na) net_store(rr, ba, in0, o0);
            if (nb) net_store(rr, bb, in1, o1);
          }
        }
      }
    }
  }
  if (lane == 0) {
    if (liq_rows) atomicOr(&sm.liq, liq_rows);
    if (sol_rows) atomicOr(&sm.sol, sol_rows);
  }
  // halo columns x0-1 and x0+kW, one thread per cell, on warps 2 and 3, which
  // have one input row fewer than warps 0 and 1 (surrogate: warp 3 alone,
  // then the same network pass as the rows)
  if (SURR ? warp == 3 : (threadIdx.x >= kHalo0 && threadIdx.x < kHalo0 + 2 * kTRin)) {
   for (int i = SURR ? lane : (int)threadIdx.x - kHalo0; i < 2 * kTRin; i += 32) {
    const int rr = i >> 1, side = i & 1;
    const int x = side ? kHaloR : kHaloL, g = x0 - 4 + x;
    float Sh = 0.f, mh = 0.f;
    double kh = 0.0;
    uint8_t hm = 3u;
    if (y0 - 1 + rr <= K.ny - 1) {
      const float pv = sm.psi[rr][x];
      if constexpr (TFC) {
        // C0 enters mu'' as (g + 1) C0, 0 at psi = -1 exactly: the liquid
        // groups suffice there
        double RT, C0;
        cell_tfc(K, sm.kp, tfc_T(K, PS.T_coarse, sm.hiT[side], sm.hx[side], sm.tj[rr], sm.ty[rr]),
                 __float_as_uint(pv) != kMinus1, RT, C0, kh);
        cell_terms(F, pv, sm.d[rr][x], (float)RT, (float)C0, Sh, mh);
      } else {
        cell_terms(F, pv, sm.d[rr][x], tRT[g], tC0[g], Sh, mh);
      }
      hm = (pv <= -1.f ? 1u : 0u) | (pv >= 1.f ? 2u : 0u);
    }
    sm.S[rr][x] = Sh;
    sm.mu[rr][x] = mh;
    if constexpr (TFC) sm.kc[rr][x] = kh;
    sm.hmask[rr][side] = hm;
    if (!SURR) break;
   }
   if constexpr (SURR) {
    __syncwarp();
    const int g = lane >> 2;
#pragma unroll 1
    for (int mt = 0; mt < (2 * kTRin + 15) / 16; ++mt) {
      const int ia = 16 * mt + g, ib = ia + 8;
      const int ra = ia < 2 * kTRin ? ia >> 1 : 0, rb = ib < 2 * kTRin ? ib >> 1 : 0;
      const int xa = (ia & 1) ? kHaloR : kHaloL, xb = (ib & 1) ? kHaloR : kHaloL;
      const bool na = ia < 2 * kTRin && y0 - 1 + ra <= K.ny - 1 && !melt_cell(ra, xa) && halo_mu_used(ra, xa);
      const bool nb = ib < 2 * kTRin && y0 - 1 + rb <= K.ny - 1 && !melt_cell(rb, xb) && halo_mu_used(rb, xb);
      if (!__any_sync(FULL, na || nb)) continue;
      const SurrConst SC = surr_load(SA, lane);
      float in0[3], in1[3], o0[2], o1[2];
      net_inputs(ra, xa, in0);
      net_inputs(rb, xb, in1);
      surr_tile16(SC, in0, in1, o0, o1);
      if ((lane & 3) == 0) {
        if (na) net_store(ra, xa, in0, o0);
        if (nb) net_store(rb, xb, in1, o1);
      }
    }
   }
  }
  if constexpr (SURR) {
    dKv = ld4(tDK + gi);
    dKl = tDK[gi - 1];
  }
  const float dKa[5] = {dKl, dKv.x, dKv.y, dKv.z, dKv.w};  // faces x-1|x for x = col .. col+4
  __syncthreads();
  // phase 1 done: pull the tile of the CTA that will start about one resident
  // wave later into L2, so its loads overlap the rest of this wave's
  // arithmetic (issued after the own load and phase 1, it measured fastest)
  if (threadIdx.x == 0 && !pb) prefetch();

  // ---- phase 2: warp w computes output rows 1 + 4w .. 4 + 4w of the tile
  const Mask liq = sm.liq, sol = sm.sol;
  const bool red = part != nullptr;
  double mass = 0.0;
  int itip = 0;
  struct Row {
    float s[4], m[4], sl, sr, ml, mr, q[5];  // q[f]: S pair sum of the face left of cell f (f = 0..4)
    double k[4], kl, kr;                     // TFC: K + C0 of the cells and of their neighbours
  };
  auto load_row = [&](int rr, Row &R) {
    const float4 s = ld4(&sm.S[rr][bc]), m = ld4(&sm.mu[rr][bc]);
    R.s[0] = s.x; R.s[1] = s.y; R.s[2] = s.z; R.s[3] = s.w;
    R.m[0] = m.x; R.m[1] = m.y; R.m[2] = m.z; R.m[3] = m.w;
    R.sl = __shfl_up_sync(FULL, s.w, 1);
    R.ml = __shfl_up_sync(FULL, m.w, 1);
    R.sr = __shfl_down_sync(FULL, s.x, 1);
    R.mr = __shfl_down_sync(FULL, m.x, 1);
    if (lane == 0) {
      R.sl = sm.S[rr][kHaloL];
      R.ml = sm.mu[rr][kHaloL];
    }
    if (lane == 31) {
      R.sr = sm.S[rr][kHaloR];
      R.mr = sm.mu[rr][kHaloR];
    }
    if constexpr (TFC) {
      const double2 k01 = *reinterpret_cast<const double2 *>(&sm.kc[rr][bc]);
      const double2 k23 = *reinterpret_cast<const double2 *>(&sm.kc[rr][bc + 2]);
      R.k[0] = k01.x; R.k[1] = k01.y; R.k[2] = k23.x; R.k[3] = k23.y;
      R.kl = __shfl_up_sync(FULL, R.k[3], 1);
      R.kr = __shfl_down_sync(FULL, R.k[0], 1);
      if (lane == 0) R.kl = sm.kc[rr][kHaloL];
      if (lane == 31) R.kr = sm.kc[rr][kHaloR];
    }
    R.q[0] = R.sl + R.s[0];
    R.q[1] = R.s[0] + R.s[1];
    R.q[2] = R.s[1] + R.s[2];
    R.q[3] = R.s[2] + R.s[3];
    R.q[4] = R.s[3] + R.sr;
  };
  // fluxes through the faces between rows A and B = A+1 (compute_c_CALPHAD
  // F01/F0m).  Face fluxes are rounded products (__fmul_rn): a contracted
  // product would round a face differently depending on where the face falls
  // in a warp's rows, and so on the tiling (row bands must equal the whole
  // domain bit for bit).
  auto vface = [&](const Row &A, const Row &B, float jv[4]) {
    float pp[6];
    pp[0] = A.sl + B.sl;
#pragma unroll
    for (int q = 0; q < 4; ++q) pp[q + 1] = A.s[q] + B.s[q];
    pp[5] = A.sr + B.sr;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      float dm = B.m[q] - A.m[q];
      if constexpr (TFC) dm = dm + (float)(B.k[q] - A.k[q]);  // K + C0 differs along y too
      jv[q] = __fmul_rn(fmaf(6.f, pp[q + 1], pp[q] + pp[q + 2]), dm);
    }
  };

  const int rbase = 1 + kRowsPerWarp * warp;
  Row ra, rb, rc;
  float jv_lo[4], jv_hi[4];
  float dn[kRowsPerWarp][4];
  uint32_t needs_all = 0u;  // 4 bits per output row
  load_row(rbase - 1, ra);
  load_row(rbase, rb);
  vface(ra, rb, jv_lo);
#pragma unroll
  for (int j = 0; j < kRowsPerWarp; ++j) {
    const int rr = rbase + j;  // tile input row of the output row
    load_row(rr + 1, rc);
    vface(rb, rc, jv_hi);
    // fluxes through the faces (x-1/2, r) for x = col .. col+4
    const float mm[6] = {rb.ml, rb.m[0], rb.m[1], rb.m[2], rb.m[3], rb.mr};
    float jh[5], dKf[5];
    if constexpr (TFC) {  // the cells' own K + C0 differences, rounded from FP64
      const double kk[6] = {rb.kl, rb.k[0], rb.k[1], rb.k[2], rb.k[3], rb.kr};
#pragma unroll
      for (int f = 0; f < 5; ++f) dKf[f] = (float)(kk[f + 1] - kk[f]);
    } else {
#pragma unroll
      for (int f = 0; f < 5; ++f) dKf[f] = dKa[f];
    }
#pragma unroll
    for (int f = 0; f < 5; ++f) jh[f] = __fmul_rn(fmaf(6.f, rb.q[f], ra.q[f] + rc.q[f]), mm[f + 1] - mm[f] + dKf[f]);
    const float4 dv4 = ld4(&sm.d[rr][bc]);
    const float dv[4] = {dv4.x, dv4.y, dv4.z, dv4.w};
#pragma unroll
    for (int q = 0; q < 4; ++q)
      dn[j][q] = fmaxf(fmaf(cflux4, (jh[q + 1] - jh[q]) + (jv_hi[q] - jv_lo[q]), dv[q]), floor_d);
    const bool live = y0 - 1 + rr <= ny - 2;
    if (red && live) {
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if ((outm >> q) & 1u) mass += (double)dn[j][q];
    }
    // phi: cells whose 3x3 neighbourhood is not uniformly +-1 are listed
    const Mask w3 = Mask(7) << (rr - 1);
    if (live && (liq & w3) != w3 && (sol & w3) != w3) {
      auto pm = [&](int k) -> uint32_t {  // rows flagged all -1 / all +1 store no masks
        return ((liq >> k) & 1u) ? 0x0Fu : ((sol >> k) & 1u) ? 0xF0u : (uint32_t)sm.pmask[k][lane];
      };
      const uint32_t pk = pm(rr - 1) | (pm(rr) << 8) | (pm(rr + 1) << 16);
      uint32_t lf = __shfl_up_sync(FULL, pk, 1), rt = __shfl_down_sync(FULL, pk, 1);
      if (lane == 0) {
        lf = 0u;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const uint32_t h = sm.hmask[rr - 1 + k][0];
          lf |= ((h & 1u) << (8 * k + 3)) | (((h >> 1) & 1u) << (8 * k + 7));
        }
      }
      if (lane == 31) {
        rt = 0u;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const uint32_t h = sm.hmask[rr - 1 + k][1];
          rt |= ((h & 1u) << (8 * k)) | (((h >> 1) & 1u) << (8 * k + 4));
        }
      }
      uint32_t Lv = 0x3Fu, Sv = 0x3Fu;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const uint32_t L = (pk >> (8 * k)) & 0xFu, S = (pk >> (8 * k + 4)) & 0xFu;
        Lv &= (L << 1) | ((lf >> (8 * k + 3)) & 1u) | (((rt >> (8 * k)) & 1u) << 5);
        Sv &= (S << 1) | ((lf >> (8 * k + 7)) & 1u) | (((rt >> (8 * k + 4)) & 1u) << 5);
      }
      const uint32_t needs = ~((Lv & (Lv >> 1) & (Lv >> 2)) | (Sv & (Sv >> 1) & (Sv >> 2))) & outm;
      const uint32_t cnt = __popc(needs);
      uint32_t incl = cnt;  // inclusive warp scan of the counts
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += v;
      }
      const uint32_t total = __shfl_sync(FULL, incl, 31);
      int base = 0;
      if (lane == 31 && total) base = atomicAdd(&sm.nlist, (int)total);
      base = __shfl_sync(FULL, base, 31);
      uint32_t off = (uint32_t)base + incl - cnt;
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if ((needs >> q) & 1u) sm.list[off++] = (uint16_t)((rr << 8) | (col + q));
      needs_all |= needs << (4 * j);
    }
    ra = rb;
    rb = rc;
#pragma unroll
    for (int q = 0; q < 4; ++q) jv_lo[q] = jv_hi[q];
  }
  __syncthreads();

  // ---- phase 3: interface cells, one per thread (compute_phi, fun.cu:1143-1218)
  const int nlist = sm.nlist;
  if constexpr (SURR) {
    // network driving force of the listed cells, 16 per warp pass, into the
    // mu'' slots of those cells (mu'' is not read after phase 2)
    if (nlist > 16 * warp) {
      const SurrConst SC = surr_load(SA, lane);
      const int g = lane >> 2;
#pragma unroll 1
      for (int base = 16 * warp; base < nlist; base += 16 * kWarps) {
        const int ia = base + g, ib = ia + 8;
        const uint32_t ea = sm.list[min(ia, nlist - 1)], eb = sm.list[min(ib, nlist - 1)];
        const int ra = (int)(ea >> 8), xa = (int)(ea & 0xFFu) + 4, rb = (int)(eb >> 8), xb = (int)(eb & 0xFFu) + 4;
        float in0[3], in1[3], o0[2], o1[2];
        net_inputs(ra, xa, in0);
        net_inputs(rb, xb, in1);
        surr_tile16(SC, in0, in1, o0, o1);
        __syncwarp();  // every lane has read its inputs before any slot is overwritten
        if ((lane & 3) == 0) {
          if (ia < nlist) sm.mu[ra][xa] = fmaf(o0[1], SA.y_scale[1], SA.y_mean[1]);
          if (ib < nlist) sm.mu[rb][xb] = fmaf(o1[1], SA.y_scale[1], SA.y_mean[1]);
        }
      }
    }
    __syncthreads();
  }
  for (int idx = threadIdx.x; idx < nlist; idx += kThreads) {
    const uint32_t e = sm.list[idx];
    const int rr = (int)(e >> 8), x = (int)(e & 0xFFu) + 4;  // box column
    const int r = y0 - 1 + rr, g = x0 + x - 4;
    const float c00 = F.cinf + sm.d[rr][x];
    float Anb, Ati;
    if constexpr (TFC) {
      const CellGroups cg = tfc_cell(g, r);
      Anb = (float)cg.Anb;
      Ati = (float)cg.Ati;
    } else {
      Anb = tAnb[g];
      Ati = tAti[g];
    }
    float dG = (1.f - c00) * Anb + c00 * Ati + c00 * (1.f - c00) * (float)(kL0Liq - kL0Bcc);
    if constexpr (SURR) {  // driving force from the surrogate for in-box, unaudited cells
      float in[3];
      net_inputs(rr, x, in);
      const float T = SA.T_mid + in[0] / SA.T_ihalf;
      if (T >= SA.T_lo && T <= SA.T_hi && c00 >= SA.c_lo && c00 <= SA.c_hi &&
          !surr_audit_cell(PS.step, (int64_t)(r + K.j_offset) * K.nx + g))
        dG = sm.mu[rr][x];
    }
    const float res = phi_cell_dG<float>(
        &F, clamp1(sm.psi[rr][x]), clamp1(sm.psi[rr][x + 1]), clamp1(sm.psi[rr][x - 1]), clamp1(sm.psi[rr + 1][x]),
        clamp1(sm.psi[rr - 1][x]), clamp1(sm.psi[rr + 1][x + 1]), clamp1(sm.psi[rr + 1][x - 1]),
        clamp1(sm.psi[rr - 1][x + 1]), clamp1(sm.psi[rr - 1][x - 1]), dG, PS.step, (int64_t)(r + K.j_offset) * K.nx + g, K.seed_lo,
        K.seed_hi);
    sm.S[rr][x] = res;
    if (red && res > 0.f) itip = max(itip, g == K.nx - 2 ? K.nx - 1 : g);
  }
  __syncthreads();

  // ---- phase 4: new psi and c into the tile rows
#pragma unroll
  for (int j = 0; j < kRowsPerWarp; ++j) {
    const int rr = rbase + j;
    const float4 pv4 = ld4(&sm.psi[rr][bc]);
    // phi_next = phi where uniformly +-1: an output cell is not listed only
    // where psi <= -1 or >= 1 over its 3x3 neighbourhood, so clamp(psi) is
    // its sign (cells outside the interior are not stored or are overwritten
    // by the ghost copies); listed cells take phase 3's result
    float po[4] = {pv4.x > 0.f ? 1.f : -1.f, pv4.y > 0.f ? 1.f : -1.f, pv4.z > 0.f ? 1.f : -1.f,
                   pv4.w > 0.f ? 1.f : -1.f};
    const uint32_t lb = (needs_all >> (4 * j)) & 0xFu;
    if (lb) {
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if ((lb >> q) & 1u) po[q] = sm.S[rr][bc + q];
    }
    st4(&sm.psi[rr][bc], po[0], po[1], po[2], po[3]);
    st4(&sm.d[rr][bc], dn[j][0], dn[j][1], dn[j][2], dn[j][3]);
  }
  if (red) {  // coarse tip: the last column with phi > 0 (listed cells counted again, harmlessly)
#pragma unroll
    for (int j = 0; j < kRowsPerWarp; ++j) {
      const int rr = rbase + j;
      const float4 po4 = ld4(&sm.psi[rr][bc]);
      const float po[4] = {po4.x, po4.y, po4.z, po4.w};
      if (y0 - 1 + rr > ny - 2) continue;
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (((outm >> q) & 1u) && po[q] > 0.f) itip = max(itip, gi + q == nx - 2 ? nx - 1 : gi + q);
    }
  }
  const int nrow = min(kTR, K.ny - 1 - y0);  // output rows of this tile inside the interior
  const int ncol = min(kW, K.nx - x0);       // columns of this tile inside the array (a multiple of 4)
  if (x0 == 0 || x0 + kW >= K.nx) {
    // ghost columns 0 and nx-1 (compute_boundary_individual, fun.cu:1220-1230)
    __syncthreads();
    if (threadIdx.x < nrow) {
      const int rr = 1 + threadIdx.x;
      if (x0 == 0) {
        sm.psi[rr][4] = sm.psi[rr][5];
        sm.d[rr][4] = sm.d[rr][5];
      }
      if (x0 + kW >= K.nx) {
        const int x = K.nx - 1 - x0 + 4;
        sm.psi[rr][x] = sm.psi[rr][x - 1];
        sm.d[rr][x] = sm.d[rr][x - 1];
      }
    }
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // tile writes -> bulk copies
  __syncthreads();

  // ---- bulk copies: thread (row j, field, kind): kind 0 the row itself,
  // kind 1 its ghost copies (row jmin -> 0, row jmax -> ny-1)
  if (threadIdx.x < 4 * kTR) {
    const int j = threadIdx.x >> 2, field = threadIdx.x & 1, kind = (threadIdx.x >> 1) & 1;
    const int r = y0 + j;
    if (j < nrow) {
      float *f = field ? c_n : psi_n;
      const float *src = field ? &sm.d[1 + j][4] : &sm.psi[1 + j][4];
      const uint32_t bytes = (uint32_t)ncol * 4u;
      bool any = false;
      if (kind == 0) {
        bulk_store(f + (int64_t)r * K.pitch + x0, src, bytes);
        any = true;
      } else {
        if (r == K.jmin) {
          bulk_store(f + x0, src, bytes);
          any = true;
        }
        if (r == K.jmax) {
          bulk_store(f + (int64_t)(K.ny - 1) * K.pitch + x0, src, bytes);
          any = true;
        }
      }
      if (any) asm volatile("cp.async.bulk.commit_group;" ::: "memory");
    }
  }
  if (phi_n) {  // phi = clamp(psi) of the same rows, plain stores
    for (int k = threadIdx.x; k < nrow * ncol; k += kThreads) {
      const int j = k / ncol, x = k % ncol, r = y0 + j;
      const float v = clamp1(sm.psi[1 + j][4 + x]);
      phi_n[(int64_t)r * K.pitch + x0 + x] = v;
      if (r == K.jmin) phi_n[x0 + x] = v;
      if (r == K.jmax) phi_n[(int64_t)(K.ny - 1) * K.pitch + x0 + x] = v;
    }
  }

  finish(mass, itip);
  // shared memory stays allocated until the copies have read it
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

template <bool SURR>
__global__ void __launch_bounds__(kThreads, SURR ? 4 : 5)
    tile_kernel(const __grid_constant__ StepCoef K, const __grid_constant__ Coef<float> F,
                const __grid_constant__ StepScalars PS, const __grid_constant__ CUtensorMap tm_psi,
                const __grid_constant__ CUtensorMap tm_c, const float *__restrict__ tab, const int tab_len,
                float *__restrict__ psi_n, float *__restrict__ c_n, float *__restrict__ phi_n, BlockPartial *partials,
                int *err, const __grid_constant__ SurrArgs SA, const __grid_constant__ FinalRed FR,
                const int wave) {
  // blockIdx.x walks the tile rows of one tile column (they share halo rows
  // in L2), blockIdx.y the tile columns, from the one holding column PS.i_front
  const int f = max(PS.i_front, 0) / kW;
  const int tr = blockIdx.x;
  const int tc = front_first_block((int)blockIdx.y, f, (int)gridDim.y);
  // the block launched `wave` (CTAs resident at once) positions later
  const unsigned nxt = blockIdx.y * gridDim.x + blockIdx.x + (unsigned)wave;
  int pf_tr = -1, pf_tc = -1;
  if (wave > 0 && nxt < gridDim.x * gridDim.y) {
    pf_tr = (int)(nxt % gridDim.x);
    pf_tc = front_first_block((int)(nxt / gridDim.x), f, (int)gridDim.y);
  }
  auto prefetch = [&]() {
    if (pf_tc >= 0) {
      tma_prefetch_2d(&tm_psi, kW * pf_tc - 4, kTR * pf_tr);
      tma_prefetch_2d(&tm_c, kW * pf_tc - 4, kTR * pf_tr);
    }
  };
  tile_body<SURR, kTR>(K, F, PS, &tm_psi, &tm_c, tab, tab_len, psi_n, c_n, phi_n,
                  partials ? partials + ((int64_t)tc * gridDim.x + tr) : nullptr, err, SA, tr, tc,
                  partials && FR.counter ? &FR : nullptr, prefetch);
}

// The coarse-grid temperature (TFC): tiles of kTfcTileRows32 output rows, whose
// per-cell K + C0 (FP64) fits beside the tile with six CTAs per SM; per-cell
// CALPHAD groups instead of the column table.
constexpr int kTfcTR = kTfcTileRows32;
__global__ void __launch_bounds__(kThreads, 5)
    tile_kernel_tfc(const __grid_constant__ StepCoef K, const __grid_constant__ Coef<float> F,
                    const __grid_constant__ StepScalars PS, const __grid_constant__ CUtensorMap tm_psi,
                    const __grid_constant__ CUtensorMap tm_c, const float *__restrict__ tab, const int tab_len,
                    float *__restrict__ psi_n, float *__restrict__ c_n, float *__restrict__ phi_n,
                    BlockPartial *partials, int *err, const __grid_constant__ FinalRed FR, const int wave) {
  const int f = max(PS.i_front, 0) / kW;
  const int tr = blockIdx.x;
  const int tc = front_first_block((int)blockIdx.y, f, (int)gridDim.y);
  const unsigned nxt = blockIdx.y * gridDim.x + blockIdx.x + (unsigned)wave;
  int pf_tr = -1, pf_tc = -1;
  if (wave > 0 && nxt < gridDim.x * gridDim.y) {
    pf_tr = (int)(nxt % gridDim.x);
    pf_tc = front_first_block((int)(nxt / gridDim.x), f, (int)gridDim.y);
  }
  auto prefetch = [&]() {
    if (pf_tc >= 0) {
      tma_prefetch_2d(&tm_psi, kW * pf_tc - 4, kTfcTR * pf_tr);
      tma_prefetch_2d(&tm_c, kW * pf_tc - 4, kTfcTR * pf_tr);
    }
  };
  const SurrArgs none = {};
  tile_body<false, kTfcTR, decltype(prefetch), true>(
      K, F, PS, &tm_psi, &tm_c, tab, tab_len, psi_n, c_n, phi_n,
      partials ? partials + ((int64_t)tc * gridDim.x + tr) : nullptr, err, none, tr, tc,
      partials && FR.counter ? &FR : nullptr, prefetch);
}

// ---------------------------------------------------------------- ensemble
// d0 of the frozen temperature line, evaluated in the order rs_step uses on
// the host (no contraction), so an ensemble run matches the same run stepped
// alone bit for bit
__device__ __forceinline__ double ens_d0(const EnsRun &R, const double l) {
  double t = __dmul_rn(R.GG, __dsub_rn(l, R.l_init));
  t = __dmul_rn(t, R.S);
  t = __dmul_rn(t, R.W0);
  t = __ddiv_rn(t, R.deltaT0);
  const double k = (double)(-R.i_tip_target + R.hist - R.hist_init);
  return __dsub_rn(__dadd_rn(R.delta_initial, __dmul_rn(R.d1, k)), t);
}

__global__ void __launch_bounds__(kTabBlock) ens_table_kernel(const EnsRun *__restrict__ runs,
                                                              const int32_t *__restrict__ tblk) {
  const int32_t e = tblk[blockIdx.x];
  const EnsRun &R = runs[e >> 16];
  if (!R.active) return;
  __shared__ double kc[kTabBlock];
  table_block(R.K, ens_d0(R, R.l), R.d1, R.tab_len, R.tab, e & 0xFFFF, kc);
}

// CTAs per SM the tile kernels are built for, by tile height (32-row tiles
// take 83 KB of shared memory: two per SM)
constexpr int min_ctas(bool surr, int TR) { return TR > 16 ? 2 : surr ? 4 : 5; }

template <bool SURR, int SHAPE>
__global__ void __launch_bounds__(kThreads, min_ctas(SURR, shape_rows(SHAPE)))
    ens_tile_kernel(const EnsRun *__restrict__ runs, const int32_t *__restrict__ order, int *err, const int wave) {
  constexpr int TR = shape_rows(SHAPE);
  const int32_t e = order[blockIdx.x];
  const EnsRun &R = runs[e >> 16];
  if (!R.active) return;
  const int t = e & 0xFFFF, par = (int)(R.step & 1);
  StepScalars PS;
  memset(&PS, 0, sizeof(PS));
  PS.step = R.step;
  PS.d0 = ens_d0(R, R.l);
  PS.d1 = R.d1;
  const SurrArgs none = {};
  // the tile of the block launched `wave` (CTAs resident at once) positions
  // later, looked up by the issuing thread only: it may belong to another run
  auto prefetch = [&]() {
    const int nb = (int)blockIdx.x + wave;
    if (wave <= 0 || nb >= (int)gridDim.x) return;
    const int32_t e2 = order[nb];
    const EnsRun &R2 = runs[e2 >> 16];
    if (!R2.active) return;
    const int t2 = e2 & 0xFFFF, p2 = (int)(R2.step & 1), n2 = R2.nrt[SHAPE];
    tma_prefetch_2d(&R2.map_psi[SHAPE][p2], kW * (t2 / n2) - 4, TR * (t2 % n2));
    tma_prefetch_2d(&R2.map_c[SHAPE][p2], kW * (t2 / n2) - 4, TR * (t2 % n2));
  };
  const int nrt = R.nrt[SHAPE];
  tile_body<SURR, TR>(R.K, R.F, PS, &R.map_psi[SHAPE][par], &R.map_c[SHAPE][par], R.tab, R.tab_len, R.psi[par ^ 1],
                      R.c[par ^ 1], nullptr, nullptr, err, SURR ? R.surr : none, t % nrt, t / nrt, nullptr,
                      prefetch);
}

__global__ void ens_advance_kernel(EnsRun *runs, const int nruns) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nruns || !runs[r].active) return;
  runs[r].step += 1;
  runs[r].l += runs[r].inc_l;
}

// The persistent walk: one cooperative launch for nsteps steps of every run.
// Per step the CTAs compute the runs' column tables (table blocks b, b + G,
// ...), meet at a grid barrier, step the tiles b, b + G, ... of the order
// with tile_body, wait for their bulk stores to complete, and meet again.  A
// run's state at step s of the launch is step + s and l = lv[s * nruns + r],
// which the host fills by the additions of inc_l that ens_advance_kernel
// makes, so every tile computes what the per-step launches compute, bit for
// bit.  The barriers are bounded: one that gives up sets *err; a CTA that
// sees *err set stops working but keeps arriving at the barriers, so the
// others do not wait out their limits.  advance: at the end (block 0, after
// the last barrier) the runs move on to step + nsteps and l = lv[nsteps *
// nruns + r].
constexpr uint32_t kWalkBarrierLimit = 1u << 22;

template <bool SURR, int SHAPE>
__global__ void __launch_bounds__(kThreads, min_ctas(SURR, shape_rows(SHAPE)))
    ens_walk_kernel(EnsRun *__restrict__ runs, const int nruns, const int32_t *__restrict__ tblk, const int ntblk,
                    const int32_t *__restrict__ order, const int ntiles, const int nsteps,
                    const double *__restrict__ lv, const int advance, unsigned *bar, int *err,
                    const uint32_t barrier_limit) {
  constexpr int TR = shape_rows(SHAPE);
  extern __shared__ __align__(128) unsigned char smem_raw[];
  TileSmemT<TR> &sm = *reinterpret_cast<TileSmemT<TR> *>(smem_raw);
  const unsigned G = gridDim.x;
  unsigned target = 0;
  bool dead = false;
  const SurrArgs none = {};
  auto l_at = [&](int r, int s) { return lv[(int64_t)s * nruns + r]; };
  for (int s = 0; s < nsteps; ++s) {
    if (!dead)
      for (int i = blockIdx.x; i < ntblk; i += G) {
        const int32_t e = tblk[i];
        const EnsRun &R = runs[e >> 16];
        if (R.active) table_block(R.K, ens_d0(R, l_at(e >> 16, s)), R.d1, R.tab_len, R.tab, e & 0xFFFF,
                                  reinterpret_cast<double *>(smem_raw));
        __syncthreads();  // the scratch is reused by the next block
      }
    target += G;
    if (!grid_barrier(bar, target, err, barrier_limit)) dead = true;
    // tiles are handed out by a ticket counter (bar[1]): a CTA takes the next
    // tile of the order when it finishes one, so the step ends when the
    // work does, whatever the tiles cost; each CTA takes one ticket past the
    // last tile per step, so step s's tickets start at s (ntiles + G)
    const unsigned t0 = (unsigned)s * ((unsigned)ntiles + G);
    while (!dead) {
      __shared__ int tk;
      if (threadIdx.x == 0) tk = (int)(atomicAdd(bar + 1, 1u) - t0);
      __syncthreads();
      const int i = tk;
      __syncthreads();  // every thread has read the ticket
      if (i < 0 || i >= ntiles) break;  // (i < 0 only after an error left tickets untaken)
      {
        const int32_t e = order[i];
        const EnsRun &R = runs[e >> 16];
        if (!R.active) continue;  // (every thread: the run is the same)
        const int t = e & 0xFFFF;
        const int64_t step = R.step + s;
        const int par = (int)(step & 1);
        StepScalars PS;
        memset(&PS, 0, sizeof(PS));
        PS.step = step;
        PS.d0 = ens_d0(R, l_at(e >> 16, s));
        PS.d1 = R.d1;
        // L2 prefetch of this CTA's next tile of the step (as the per-step
        // launch prefetches the tile one resident wave later)
        auto prefetch = [&]() {
          const int i2 = i + (int)G;
          if (i2 >= ntiles) return;
          const int32_t e2 = order[i2];
          const EnsRun &R2 = runs[e2 >> 16];
          if (!R2.active) return;
          const int t2 = e2 & 0xFFFF, p2 = (int)((R2.step + s) & 1), n2 = R2.nrt[SHAPE];
          tma_prefetch_2d(&R2.map_psi[SHAPE][p2], kW * (t2 / n2) - 4, TR * (t2 % n2));
          tma_prefetch_2d(&R2.map_c[SHAPE][p2], kW * (t2 / n2) - 4, TR * (t2 % n2));
        };
        const int nrt = R.nrt[SHAPE];
        tile_body<SURR, TR>(R.K, R.F, PS, &R.map_psi[SHAPE][par], &R.map_c[SHAPE][par], R.tab, R.tab_len,
                            R.psi[par ^ 1], R.c[par ^ 1], nullptr, nullptr, err, SURR ? R.surr : none, t % nrt,
                            t / nrt, nullptr, prefetch);
        __syncthreads();  // every thread is done with the tile's barrier and shared memory
        if (threadIdx.x == 0) mbar_inval(&sm.full);
        if (__syncthreads_or(*(volatile int *)err != 0)) dead = true;
      }
    }
    // the bulk stores of this step complete before the barrier releases them
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    target += G;
    if (!grid_barrier(bar, target, err, barrier_limit)) dead = true;
  }
  if (advance && blockIdx.x == 0 && !dead)
    for (int r = threadIdx.x; r < nruns; r += blockDim.x)
      if (runs[r].active) {
        runs[r].l = l_at(r, nsteps);
        runs[r].step += nsteps;
      }
}


// ---------------------------------------------------------------- persistent pipeline (exact FP32)
// The exact path of tile_body split into phase functions run by warp roles of
// persistent CTAs, as the FP64 pipeline of rs_step_f64t.cu: a producer warp
// issuing the TMA loads of tile k+2 into a three-slot input ring, four warps
// computing phase 1 of tile k+1 into a two-slot staging ring, four warps
// doing phases 2-4 of tile k and its bulk stores; mbarrier hand-offs, named
// barriers per group, every wait bounded.  Same arithmetic, expression for
// expression, as tile_body.
struct alignas(128) InSlot32 {  // both arrays are TMA destinations: 128-byte aligned
  alignas(128) float psi[kTRin][kWin];
  alignas(128) float d[kTRin][kWin];
};
struct alignas(16) StSlot32 {
  float S[kTRin][kWin];  // after phase 2: new psi of the listed cells
  float mu[kTRin][kWin];
  uint8_t pmask[kTRin][32];  // per lane: bits 0-3 psi <= -1, bits 4-7 psi >= 1 of its four cells
  uint8_t hmask[kTRin][2];   // halo cells: bit 0 psi <= -1, bit 1 psi >= 1
  uint32_t liq, sol;         // bit r: every cell of input row r has psi == -1 / +1
};
struct P2Smem32 {
  uint16_t list[kTR * kW];  // interface cells: row << 8 | output column
  int nlist;
  int last;
  double part_mass[kWarps];
  int part_itip[kWarps];
};
constexpr int kRing = 3, kStage = 2;
struct alignas(128) PipeSmem32 {
  InSlot32 in[kRing];
  StSlot32 st[kStage];
  P2Smem32 p2;
  uint64_t in_full[kRing], in_empty[kRing], st_full[kStage], st_empty[kStage];
  int abort;
};
static_assert(sizeof(InSlot32) % 128 == 0 && offsetof(InSlot32, psi) % 128 == 0 && offsetof(InSlot32, d) % 128 == 0,
              "ring slots and their TMA destinations stay 128-byte aligned");
static_assert(offsetof(PipeSmem32, in) % 128 == 0, "the ring starts on a 128-byte boundary");
constexpr uint32_t kTileBytes32 = 2u * kTRin * kWin * sizeof(float);
constexpr uint32_t kMinus1f = 0xBF800000u, kPlus1f = 0x3F800000u;
constexpr int kPipeThreads = 32 + 2 * kThreads;
enum { kBarP1 = 1, kBarP2 = 2 };

__device__ __forceinline__ void gsync(int id) { asm volatile("bar.sync %0, 128;" ::"r"(id) : "memory"); }
__device__ __forceinline__ bool group_and(bool v, int id) {
  uint32_t r;
  asm volatile(
      "{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n barrier.red.and.pred q, %2, 128, p;\n"
      " selp.u32 %0, 1, 0, q;\n}\n"
      : "=r"(r)
      : "r"((uint32_t)v), "r"(id)
      : "memory");
  return r != 0;
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// bounded wait on an mbarrier phase; gives up (error flag, abort flag) after
// the limit or when another role has given up
__device__ __forceinline__ bool pipe_wait(uint64_t *bar, uint32_t parity, volatile int *abort, uint32_t limit,
                                          int *err, bool poll) {
  uint32_t tries = 0;
  while (!mbar_try(bar, parity, poll)) {
    if (*abort) return false;
    if (++tries >= limit) {
      atomicExch(err, 1);
      *abort = 1;
      return false;
    }
  }
  return true;
}

// one phase group's view of a tile and of its own lane
struct View32 {
  const StepCoef &K;
  const Coef<float> &F;
  const StepScalars &PS;
  const float *tRT, *tC0, *tDK, *tAnb, *tAti;  // column tables, indexed by column
  int x0, y0, gw, lane, gtid, col, gi, bc;
  uint32_t outm;
  __device__ View32(const StepCoef &K_, const Coef<float> &F_, const StepScalars &PS_, const float *tab, int len,
                    int x0_, int y0_, int gtid_)
      : K(K_), F(F_), PS(PS_), tRT(tab + kTabRT * len + 4), tC0(tab + kTabC0 * len + 4),
        tDK(tab + kTabDK * len + 4), tAnb(tab + kTabAnb * len + 4), tAti(tab + kTabAti * len + 4), x0(x0_),
        y0(y0_), gw(gtid_ >> 5), lane(gtid_ & 31), gtid(gtid_) {
    col = 4 * lane;
    gi = x0 + col;
    bc = col + 4;
    outm = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q)
      if (gi + q >= 1 && gi + q <= K.nx - 2) outm |= 1u << q;
  }
};

__device__ __forceinline__ void fix_beyond32(const View32 &V, InSlot32 &in) {
  if (V.x0 + kW + 4 <= V.K.nx) return;
  for (int k = V.gtid; k < kTRin * kWin; k += kThreads) {
    const int rr = k / kWin, x = k % kWin;
    if (V.x0 - 4 + x >= V.K.nx) {
      in.psi[rr][x] = -1.f;
      in.d[rr][x] = 0.f;
    }
  }
}

// phase 1 of the group warp's input rows and of the halo columns (st.liq and
// st.sol 0 on entry)
__device__ __forceinline__ void phase1_32(const View32 &V, const InSlot32 &in, StSlot32 &st) {
  const Coef<float> &F = V.F;
  const int lane = V.lane, bc = V.bc;
  const float two_cinf = F.cinf + F.cinf;
  constexpr float KL = (float)(-2.0 * kL0Liq);
  const float d_hi = F.ser_hi, d_lo = F.ser_lo;  // series range of delta (Coef)
  const float4 RTv = ld4(V.tRT + V.gi), C0v = ld4(V.tC0 + V.gi);
  const float RTa[4] = {RTv.x, RTv.y, RTv.z, RTv.w}, C0a[4] = {C0v.x, C0v.y, C0v.z, C0v.w};
  auto solid3 = [&](int rr) -> uint32_t {
    const int xh = lane == 0 ? kHaloL : kHaloR;
    uint32_t v = 0xFu;
    bool hs = true;
    for (int r2 = max(rr - 1, 0); r2 <= min(rr + 1, kTRin - 1); ++r2) {
      const float4 q4 = ld4(&in.psi[r2][bc]);
      v &= (__float_as_uint(q4.x) == kPlus1f ? 1u : 0u) | (__float_as_uint(q4.y) == kPlus1f ? 2u : 0u) |
           (__float_as_uint(q4.z) == kPlus1f ? 4u : 0u) | (__float_as_uint(q4.w) == kPlus1f ? 8u : 0u);
      hs = hs && __float_as_uint(in.psi[r2][xh]) == kPlus1f;
    }
    uint32_t lf = __shfl_up_sync(FULL, v >> 3, 1) & 1u, rt = __shfl_down_sync(FULL, v, 1) & 1u;
    if (lane == 0) lf = (hs || V.x0 == 0) ? 1u : 0u;
    if (lane == 31) rt = hs ? 1u : 0u;
    const uint32_t e = lf | (v << 1) | (rt << 5);
    return e & (e >> 1) & (e >> 2) & 0xFu;
  };
#pragma unroll 1
  for (int rr = V.gw; rr < kTRin; rr += kWarps) {
    if (V.y0 - 1 + rr > V.K.ny - 1) {
      st4(&st.S[rr][bc], 0.f, 0.f, 0.f, 0.f);
      st4(&st.mu[rr][bc], 0.f, 0.f, 0.f, 0.f);
      st.pmask[rr][lane] = 0xFFu;
      if (lane == 0) {
        atomicOr(&st.liq, 1u << rr);
        atomicOr(&st.sol, 1u << rr);
      }
      continue;
    }
    const float4 pv4 = ld4(&in.psi[rr][bc]), dv4 = ld4(&in.d[rr][bc]);
    const float pv[4] = {pv4.x, pv4.y, pv4.z, pv4.w}, dv[4] = {dv4.x, dv4.y, dv4.z, dv4.w};
    float Sv[4], mv[4];
    const uint32_t b0 = __float_as_uint(pv[0]), b1 = __float_as_uint(pv[1]), b2 = __float_as_uint(pv[2]),
                   b3 = __float_as_uint(pv[3]);
    const uint32_t band = b0 & b1 & b2 & b3, bor = b0 | b1 | b2 | b3;
    const float dmx = fmaxf(fmaxf(dv[0], dv[1]), fmaxf(dv[2], dv[3]));
    const float dmn = fminf(fminf(dv[0], dv[1]), fminf(dv[2], dv[3]));
    const bool liq4 = band == kMinus1f && bor == kMinus1f;
    uint32_t code;
    if (__all_sync(FULL, liq4 && fmaxf(dmx, -dmn) <= F.melt_tiny)) {
      // far melt (as tile_body)
      code = 1u;
      st.pmask[rr][lane] = 0x0Fu;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const float c = F.cinf + dv[q], om = 1.f - c;
        float p = fmaf(F.melt_a[3], dv[q], F.melt_a[2]);
        p = fmaf(p, dv[q], F.melt_a[1]);
        p = fmaf(p, dv[q], F.melt_a[0]);
        Sv[q] = c * om;
        mv[q] = dv[q] * fmaf(RTa[q], p, KL);
      }
    } else if (__all_sync(FULL, liq4 && dmx < d_hi && dmn > d_lo)) {
      code = 1u;
      st.pmask[rr][lane] = 0x0Fu;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const float c = F.cinf + dv[q], om = 1.f - c;
        const float sv = __fdividef(dv[q], fmaf(two_cinf, om, dv[q]));
        const float s2 = sv * sv;
        float p = fmaf(s2, 1.f / 7.f, 1.f / 5.f);
        p = fmaf(s2, p, 1.f / 3.f);
        const float ath = fmaf(sv * s2, p, sv);
        Sv[q] = c * om;
        mv[q] = fmaf(RTa[q] + RTa[q], ath, dv[q] * KL);
      }
    } else {
      const bool sol4 = band == kPlus1f && bor == kPlus1f;
      code = (__all_sync(FULL, liq4) ? 1u : 0u) | (__all_sync(FULL, sol4) ? 2u : 0u);
      const uint32_t s3 = (code & 2u) ? solid3(rr) : 0u;
      if ((code & 2u) && __all_sync(FULL, s3 == 0xFu)) {
        st.pmask[rr][lane] = 0xF0u;
#pragma unroll
        for (int q = 0; q < 4; ++q) Sv[q] = mv[q] = 0.f;
      } else {
        uint32_t L = 0u, Sm = 0u;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          if (pv[q] <= -1.f) L |= 1u << q;
          if (pv[q] >= 1.f) Sm |= 1u << q;
          cell_terms(F, pv[q], dv[q], RTa[q], C0a[q], Sv[q], mv[q]);
        }
        st.pmask[rr][lane] = (uint8_t)(L | (Sm << 4));
      }
    }
    st4(&st.S[rr][bc], Sv[0], Sv[1], Sv[2], Sv[3]);
    st4(&st.mu[rr][bc], mv[0], mv[1], mv[2], mv[3]);
    if (lane == 0) {
      if (code & 1u) atomicOr(&st.liq, 1u << rr);
      if (code & 2u) atomicOr(&st.sol, 1u << rr);
    }
  }
  if (V.gtid >= 64 && V.gtid < 64 + 2 * kTRin) {
    const int i = V.gtid - 64;
    const int rr = i >> 1, side = i & 1;
    const int x = side ? kHaloR : kHaloL, g = V.x0 - 4 + x;
    float Sh = 0.f, mh = 0.f;
    uint8_t hm = 3u;
    if (V.y0 - 1 + rr <= V.K.ny - 1) {
      const float pv = in.psi[rr][x];
      cell_terms(F, pv, in.d[rr][x], V.tRT[g], V.tC0[g], Sh, mh);
      hm = (pv <= -1.f ? 1u : 0u) | (pv >= 1.f ? 2u : 0u);
    }
    st.S[rr][x] = Sh;
    st.mu[rr][x] = mh;
    st.hmask[rr][side] = hm;
  }
}

// phase 2 of the group warp's output rows (nlist 0 on entry); returns the
// listed cells, 4 bits per output row
__device__ __forceinline__ uint32_t phase2_32(const View32 &V, const InSlot32 &in, const StSlot32 &st, P2Smem32 &p2,
                                              float dn[kRowsPerWarp][4], double &mass, bool red) {
  const Coef<float> &F = V.F;
  const int lane = V.lane, bc = V.bc;
  const float cflux4 = 0.25f * F.cflux;
  const float floor_d = F.c_floor - F.cinf;
  const float4 dKv = ld4(V.tDK + V.gi);
  const float dKl = V.tDK[V.gi - 1];
  const float dKa[5] = {dKl, dKv.x, dKv.y, dKv.z, dKv.w};
  const uint32_t liq = st.liq, sol = st.sol;
  struct Row {
    float s[4], m[4], sl, sr, ml, mr, q[5];
  };
  auto load_row = [&](int rr, Row &R) {
    const float4 s = ld4(&st.S[rr][bc]), m = ld4(&st.mu[rr][bc]);
    R.s[0] = s.x; R.s[1] = s.y; R.s[2] = s.z; R.s[3] = s.w;
    R.m[0] = m.x; R.m[1] = m.y; R.m[2] = m.z; R.m[3] = m.w;
    R.sl = __shfl_up_sync(FULL, s.w, 1);
    R.ml = __shfl_up_sync(FULL, m.w, 1);
    R.sr = __shfl_down_sync(FULL, s.x, 1);
    R.mr = __shfl_down_sync(FULL, m.x, 1);
    if (lane == 0) {
      R.sl = st.S[rr][kHaloL];
      R.ml = st.mu[rr][kHaloL];
    }
    if (lane == 31) {
      R.sr = st.S[rr][kHaloR];
      R.mr = st.mu[rr][kHaloR];
    }
    R.q[0] = R.sl + R.s[0];
    R.q[1] = R.s[0] + R.s[1];
    R.q[2] = R.s[1] + R.s[2];
    R.q[3] = R.s[2] + R.s[3];
    R.q[4] = R.s[3] + R.sr;
  };
  auto vface = [&](const Row &A, const Row &B, float jv[4]) {
    float pp[6];
    pp[0] = A.sl + B.sl;
#pragma unroll
    for (int q = 0; q < 4; ++q) pp[q + 1] = A.s[q] + B.s[q];
    pp[5] = A.sr + B.sr;
#pragma unroll
    for (int q = 0; q < 4; ++q) jv[q] = __fmul_rn(fmaf(6.f, pp[q + 1], pp[q] + pp[q + 2]), B.m[q] - A.m[q]);
  };
  const int rbase = 1 + kRowsPerWarp * V.gw;
  Row ra, rb, rc;
  float jv_lo[4], jv_hi[4];
  uint32_t needs_all = 0u;
  load_row(rbase - 1, ra);
  load_row(rbase, rb);
  vface(ra, rb, jv_lo);
#pragma unroll
  for (int j = 0; j < kRowsPerWarp; ++j) {
    const int rr = rbase + j;
    load_row(rr + 1, rc);
    vface(rb, rc, jv_hi);
    const float mm[6] = {rb.ml, rb.m[0], rb.m[1], rb.m[2], rb.m[3], rb.mr};
    float jh[5];
#pragma unroll
    for (int f = 0; f < 5; ++f) jh[f] = __fmul_rn(fmaf(6.f, rb.q[f], ra.q[f] + rc.q[f]), mm[f + 1] - mm[f] + dKa[f]);
    const float4 dv4 = ld4(&in.d[rr][bc]);
    const float dv[4] = {dv4.x, dv4.y, dv4.z, dv4.w};
#pragma unroll
    for (int q = 0; q < 4; ++q)
      dn[j][q] = fmaxf(fmaf(cflux4, (jh[q + 1] - jh[q]) + (jv_hi[q] - jv_lo[q]), dv[q]), floor_d);
    const bool live = V.y0 - 1 + rr <= V.K.ny - 2;
    if (red && live) {
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if ((V.outm >> q) & 1u) mass += (double)dn[j][q];
    }
    const uint32_t w3 = 7u << (rr - 1);
    if (live && (liq & w3) != w3 && (sol & w3) != w3) {
      const uint32_t pk = (uint32_t)st.pmask[rr - 1][lane] | ((uint32_t)st.pmask[rr][lane] << 8) |
                          ((uint32_t)st.pmask[rr + 1][lane] << 16);
      uint32_t lf = __shfl_up_sync(FULL, pk, 1), rt = __shfl_down_sync(FULL, pk, 1);
      if (lane == 0) {
        lf = 0u;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const uint32_t h = st.hmask[rr - 1 + k][0];
          lf |= ((h & 1u) << (8 * k + 3)) | (((h >> 1) & 1u) << (8 * k + 7));
        }
      }
      if (lane == 31) {
        rt = 0u;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const uint32_t h = st.hmask[rr - 1 + k][1];
          rt |= ((h & 1u) << (8 * k)) | (((h >> 1) & 1u) << (8 * k + 4));
        }
      }
      uint32_t Lv = 0x3Fu, Sv = 0x3Fu;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const uint32_t L = (pk >> (8 * k)) & 0xFu, S = (pk >> (8 * k + 4)) & 0xFu;
        Lv &= (L << 1) | ((lf >> (8 * k + 3)) & 1u) | (((rt >> (8 * k)) & 1u) << 5);
        Sv &= (S << 1) | ((lf >> (8 * k + 7)) & 1u) | (((rt >> (8 * k + 4)) & 1u) << 5);
      }
      const uint32_t needs = ~((Lv & (Lv >> 1) & (Lv >> 2)) | (Sv & (Sv >> 1) & (Sv >> 2))) & V.outm;
      const uint32_t cnt = __popc(needs);
      uint32_t incl = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += v;
      }
      const uint32_t total = __shfl_sync(FULL, incl, 31);
      int base = 0;
      if (lane == 31 && total) base = atomicAdd(&p2.nlist, (int)total);
      base = __shfl_sync(FULL, base, 31);
      uint32_t off = (uint32_t)base + incl - cnt;
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if ((needs >> q) & 1u) p2.list[off++] = (uint16_t)((rr << 8) | (V.col + q));
      needs_all |= needs << (4 * j);
    }
    ra = rb;
    rb = rc;
#pragma unroll
    for (int q = 0; q < 4; ++q) jv_lo[q] = jv_hi[q];
  }
  return needs_all;
}

// phase 3: listed interface cells, one per group thread; new psi into np
__device__ __forceinline__ void phase3_32(const View32 &V, const InSlot32 &in, const P2Smem32 &p2,
                                          float (*np)[kWin], bool red, int &itip) {
  const int nlist = p2.nlist;
  for (int idx = V.gtid; idx < nlist; idx += kThreads) {
    const uint32_t e = p2.list[idx];
    const int rr = (int)(e >> 8), x = (int)(e & 0xFFu) + 4;
    const int r = V.y0 - 1 + rr, g = V.x0 + x - 4;
    const float c00 = V.F.cinf + in.d[rr][x];
    const float dG = (1.f - c00) * V.tAnb[g] + c00 * V.tAti[g] + c00 * (1.f - c00) * (float)(kL0Liq - kL0Bcc);
    const float res = phi_cell_dG<float>(
        &V.F, clamp1(in.psi[rr][x]), clamp1(in.psi[rr][x + 1]), clamp1(in.psi[rr][x - 1]),
        clamp1(in.psi[rr + 1][x]), clamp1(in.psi[rr - 1][x]), clamp1(in.psi[rr + 1][x + 1]),
        clamp1(in.psi[rr + 1][x - 1]), clamp1(in.psi[rr - 1][x + 1]), clamp1(in.psi[rr - 1][x - 1]), dG,
        V.PS.step, (int64_t)(r + V.K.j_offset) * V.K.nx + g, V.K.seed_lo, V.K.seed_hi);
    np[rr][x] = res;
    if (red && res > 0.f) itip = max(itip, g == V.K.nx - 2 ? V.K.nx - 1 : g);
  }
}

// phase 4: new psi and c of the group warp's rows into the input tile
__device__ __forceinline__ void phase4_32(const View32 &V, InSlot32 &in, const float (*np)[kWin], uint32_t needs_all,
                                          const float dn[kRowsPerWarp][4], bool red, int &itip) {
  const int rbase = 1 + kRowsPerWarp * V.gw, bc = V.bc;
#pragma unroll
  for (int j = 0; j < kRowsPerWarp; ++j) {
    const int rr = rbase + j;
    const float4 pv4 = ld4(&in.psi[rr][bc]);
    const float pv[4] = {pv4.x, pv4.y, pv4.z, pv4.w};
    const bool live = V.y0 - 1 + rr <= V.K.ny - 2;
    float po[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const bool listed = (needs_all >> (4 * j + q)) & 1u;
      po[q] = listed ? np[rr][bc + q] : clamp1(pv[q]);
      if (red && live && !listed && ((V.outm >> q) & 1u) && po[q] > 0.f)
        itip = max(itip, V.gi + q == V.K.nx - 2 ? V.K.nx - 1 : V.gi + q);
    }
    st4(&in.psi[rr][bc], po[0], po[1], po[2], po[3]);
    st4(&in.d[rr][bc], dn[j][0], dn[j][1], dn[j][2], dn[j][3]);
  }
}

// ghost columns, bulk copies of the rows (group threads < 64) and phi;
// returns whether this thread committed a bulk group
__device__ __forceinline__ bool store_tile32(const View32 &V, InSlot32 &in, float *__restrict__ psi_n,
                                             float *__restrict__ c_n, float *__restrict__ phi_n, int bar) {
  const StepCoef &K = V.K;
  const int x0 = V.x0, y0 = V.y0;
  const int nrow = min(kTR, K.ny - 1 - y0);
  const int ncol = min(kW, K.nx - x0);
  if (x0 == 0 || x0 + kW >= K.nx) {
    gsync(bar);
    if (V.gtid < nrow) {
      const int rr = 1 + V.gtid;
      if (x0 == 0) {
        in.psi[rr][4] = in.psi[rr][5];
        in.d[rr][4] = in.d[rr][5];
      }
      if (x0 + kW >= K.nx) {
        const int x = K.nx - 1 - x0 + 4;
        in.psi[rr][x] = in.psi[rr][x - 1];
        in.d[rr][x] = in.d[rr][x - 1];
      }
    }
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  gsync(bar);
  bool any = false;
  if (V.gtid < 4 * kTR) {
    const int j = V.gtid >> 2, field = V.gtid & 1, kind = (V.gtid >> 1) & 1;
    const int r = y0 + j;
    if (j < nrow) {
      float *fo = field ? c_n : psi_n;
      const float *src = field ? &in.d[1 + j][4] : &in.psi[1 + j][4];
      const uint32_t bytes = (uint32_t)ncol * 4u;
      if (kind == 0) {
        bulk_store(fo + (int64_t)r * K.pitch + x0, src, bytes);
        any = true;
      } else {
        if (r == K.jmin) {
          bulk_store(fo + x0, src, bytes);
          any = true;
        }
        if (r == K.jmax) {
          bulk_store(fo + (int64_t)(K.ny - 1) * K.pitch + x0, src, bytes);
          any = true;
        }
      }
      if (any) asm volatile("cp.async.bulk.commit_group;" ::: "memory");
    }
  }
  if (phi_n) {
    for (int k = V.gtid; k < nrow * ncol; k += kThreads) {
      const int j = k / ncol, x = k % ncol, r = y0 + j;
      const float v = clamp1(in.psi[1 + j][4 + x]);
      phi_n[(int64_t)r * K.pitch + x0 + x] = v;
      if (r == K.jmin) phi_n[x0 + x] = v;
      if (r == K.jmax) phi_n[(int64_t)(K.ny - 1) * K.pitch + x0 + x] = v;
    }
  }
  return any;
}

// the tile's partial sums and the fused final reduction (scratch of at least
// 256 doubles and 256 ints)
__device__ __forceinline__ void finish32(const View32 &V, P2Smem32 &p2, double mass, int itip, BlockPartial *part,
                                         const FinalRed *FR, double *sm_m, int *sm_i, int bar) {
  if (!part) return;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mass += __shfl_down_sync(FULL, mass, o);
  itip = __reduce_max_sync(FULL, itip);
  if (V.lane == 0) {
    p2.part_mass[V.gw] = mass;
    p2.part_itip[V.gw] = itip;
  }
  gsync(bar);
  if (V.gtid == 0) {
    BlockPartial b;
    b.mass = 0.0;
    b.itip = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
      b.mass += p2.part_mass[w];
      b.itip = max(b.itip, p2.part_itip[w]);
    }
    b.pad = 0;
    *part = b;
  }
  if (!FR) return;
  if (V.gtid == 0) {
    __threadfence();
    p2.last = atomicAdd(FR->counter, 1u) == (unsigned)(FR->nparts - 1);
  }
  gsync(bar);
  if (!p2.last) return;
  __threadfence();
  final_reduce(*FR, sm_m, sm_i, V.gtid, [&] { gsync(bar); });
}

__device__ __forceinline__ void tile_of32(int t, int nrt, int ncb, int f, int &tr, int &tc) {
  tr = t % nrt;
  tc = front_first_block(t / nrt, f, ncb);
}

__global__ void __launch_bounds__(kPipeThreads, 2)
    pipe_kernel_f32(const __grid_constant__ StepCoef K, const __grid_constant__ Coef<float> F,
                    const __grid_constant__ StepScalars PS, const __grid_constant__ CUtensorMap tm_psi,
                    const __grid_constant__ CUtensorMap tm_c, const float *__restrict__ tab, const int tab_len,
                    float *__restrict__ psi_n, float *__restrict__ c_n, float *__restrict__ phi_n,
                    BlockPartial *partials, int *err, const __grid_constant__ FinalRed FR, const int nrt,
                    const int ncb) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  PipeSmem32 &sm = *reinterpret_cast<PipeSmem32 *>(smem_raw);
  const int warp = threadIdx.x >> 5;
  const int ntiles = nrt * ncb;
  const int f = max(PS.i_front, 0) / kW;
  const FinalRed *FRp = partials && FR.counter ? &FR : nullptr;
  const uint32_t limit = PS.wait_limit ? PS.wait_limit : kWaitLimit;
  const bool poll = PS.wait_limit != 0;
  volatile int *abort = &sm.abort;
  if (smem_u32(smem_raw) & 127u) {
    if (threadIdx.x == 0) atomicExch(err, 2);
    return;
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < kRing; ++s) {
      mbar_init(&sm.in_full[s], 1);
      mbar_init(&sm.in_empty[s], 1);
    }
    for (int s = 0; s < kStage; ++s) {
      mbar_init(&sm.st_full[s], 1);
      mbar_init(&sm.st_empty[s], 1);
    }
    sm.abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("griddepcontrol.wait;" ::: "memory");
  // the step's final reduction (a programmatic dependent) may be scheduled now
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  __syncthreads();

  if (warp == 0) {  // producer
    if ((threadIdx.x & 31) == 0) {
      int k = 0;
      for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++k) {
        const int s = k % kRing;
        if (k >= kRing && !pipe_wait(&sm.in_empty[s], ((k / kRing) - 1) & 1, abort, limit, err, poll)) break;
        int tr, tc;
        tile_of32(t, nrt, ncb, f, tr, tc);
        mbar_expect_tx(&sm.in_full[s], kTileBytes32);
        tma_load_2d(&sm.in[s].psi[0][0], &tm_psi, &sm.in_full[s], kW * tc - 4, kTR * tr);
        tma_load_2d(&sm.in[s].d[0][0], &tm_c, &sm.in_full[s], kW * tc - 4, kTR * tr);
      }
      // only the last kRing loads can still be in flight: they land before the CTA exits
      for (int q = max(k - kRing, 0); q < k; ++q)
        for (uint32_t tt = 0; tt < kWaitLimit && !mbar_try_wait(&sm.in_full[q % kRing], (q / kRing) & 1); ++tt) {
        }
    }
    return;
  }
  if (warp <= kWarps) {  // phase 1
    const int gtid = (int)threadIdx.x - 32;
    int k = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++k) {
      const int s = k % kRing, q = k % kStage;
      bool ok = pipe_wait(&sm.in_full[s], (k / kRing) & 1, abort, limit, err, poll);
      if (ok && k >= kStage) ok = pipe_wait(&sm.st_empty[q], ((k / kStage) - 1) & 1, abort, limit, err, poll);
      if (!group_and(ok, kBarP1)) break;
      int tr, tc;
      tile_of32(t, nrt, ncb, f, tr, tc);
      const View32 V(K, F, PS, tab, tab_len, kW * tc, 1 + kTR * tr, gtid);
      if (gtid == 0) {
        sm.st[q].liq = 0u;
        sm.st[q].sol = 0u;
      }
      fix_beyond32(V, sm.in[s]);
      gsync(kBarP1);
      phase1_32(V, sm.in[s], sm.st[q]);
      gsync(kBarP1);
      if (gtid == 0) mbar_arrive(&sm.st_full[q]);
    }
    return;
  }
  // phases 2-4
  const int gtid = (int)threadIdx.x - 32 - kThreads;
  int k = 0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++k) {
    const int s = k % kRing, q = k % kStage;
    if (!group_and(pipe_wait(&sm.st_full[q], (k / kStage) & 1, abort, limit, err, poll), kBarP2)) break;
    int tr, tc;
    tile_of32(t, nrt, ncb, f, tr, tc);
    const View32 V(K, F, PS, tab, tab_len, kW * tc, 1 + kTR * tr, gtid);
    BlockPartial *part = partials ? partials + ((int64_t)tc * nrt + tr) : nullptr;
    const bool red = part != nullptr;
    if (gtid == 0) sm.p2.nlist = 0;
    gsync(kBarP2);
    double mass = 0.0;
    int itip = 0;
    float dn[kRowsPerWarp][4];
    const uint32_t needs_all = phase2_32(V, sm.in[s], sm.st[q], sm.p2, dn, mass, red);
    gsync(kBarP2);
    phase3_32(V, sm.in[s], sm.p2, sm.st[q].S, red, itip);
    gsync(kBarP2);
    phase4_32(V, sm.in[s], sm.st[q].S, needs_all, dn, red, itip);
    const bool issued = store_tile32(V, sm.in[s], psi_n, c_n, phi_n, kBarP2);
    finish32(V, sm.p2, mass, itip, part, FRp, reinterpret_cast<double *>(&sm.st[q].mu[0][0]),
             reinterpret_cast<int *>(&sm.st[q].mu[8][0]), kBarP2);
    if (issued) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
    gsync(kBarP2);
    if (gtid == 0) {
      mbar_arrive(&sm.st_empty[q]);
      mbar_arrive(&sm.in_empty[s]);
    }
  }
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

}  // namespace

namespace {
// the ensemble kernels of one tile shape, and their shared memory
using EnsTileFn = void (*)(const EnsRun *, const int32_t *, int *, int);
using EnsWalkFn = void (*)(EnsRun *, int, const int32_t *, int, const int32_t *, int, int, const double *, int,
                           unsigned *, int *, uint32_t);
template <int SHAPE>
void ens_kernels(bool surr, EnsTileFn &tile, EnsWalkFn &walk, size_t &smem) {
  tile = surr ? ens_tile_kernel<true, SHAPE> : ens_tile_kernel<false, SHAPE>;
  walk = surr ? ens_walk_kernel<true, SHAPE> : ens_walk_kernel<false, SHAPE>;
  smem = sizeof(TileSmemT<shape_rows(SHAPE)>);
}
bool ens_kernels(int shape, bool surr, EnsTileFn &tile, EnsWalkFn &walk, size_t &smem) {
  switch (shape) {
    case 0: ens_kernels<0>(surr, tile, walk, smem); return true;
    case 1: ens_kernels<1>(surr, tile, walk, smem); return true;
    case 2: ens_kernels<2>(surr, tile, walk, smem); return true;
    default: return false;
  }
}
static_assert(kTileShapes == 3, "ens_kernels covers every tile shape");
}  // namespace

int launch_ensemble(const EnsRun *runs, int nruns, const int32_t *tblk, int ntblk, const int32_t *order, int ntiles,
                    int shape, bool advance, bool surr, int *err, cudaStream_t st) {
  EnsTileFn kfn;
  EnsWalkFn wfn;
  size_t smem;
  if (!ens_kernels(shape, surr, kfn, wfn, smem)) return -1;
  static std::atomic<unsigned long long> attr_done[2][kTileShapes];
  if (!smem_limit_once((const void *)kfn, (int)smem, attr_done[surr][shape])) return -3;
  static std::atomic<int> wave_of[2][kTileShapes][64];
  const int wave = resident_ctas((const void *)kfn, kThreads, smem, wave_of[surr][shape]);
  if (wave < 0) return -3;
  ens_table_kernel<<<ntblk, kTabBlock, 0, st>>>(runs, tblk);
  kfn<<<ntiles, kThreads, smem, st>>>(runs, order, err, wave);
  if (advance) ens_advance_kernel<<<(nruns + 63) / 64, 64, 0, st>>>(const_cast<EnsRun *>(runs), nruns);
  return 0;
}

int launch_ensemble_walk(EnsRun *runs, int nruns, const int32_t *tblk, int ntblk, const int32_t *order, int ntiles,
                         int shape, int nsteps, const double *lv, bool advance, bool surr, unsigned *bar, int *err,
                         uint32_t barrier_limit, cudaStream_t st) {
  if (nsteps <= 0) return 0;
  EnsTileFn tfn;
  EnsWalkFn kfn;
  size_t smem;
  if (!ens_kernels(shape, surr, tfn, kfn, smem)) return -1;
  static_assert(sizeof(TileSmemT<8>) >= kTabBlock * sizeof(double), "table scratch fits the tile's shared memory");
  static std::atomic<unsigned long long> attr_done[2][kTileShapes];
  if (!smem_limit_once((const void *)kfn, (int)smem, attr_done[surr][shape])) return -3;
  static std::atomic<int> res_of[2][kTileShapes][64];
  const int res = resident_ctas((const void *)kfn, kThreads, smem, res_of[surr][shape]);
  if (res <= 0) return -3;
  const int grid = std::max(1, std::min(res, std::max(ntiles, ntblk)));
  if (cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned), st) != cudaSuccess) return -2;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  const int adv = advance ? 1 : 0;
  const uint32_t lim = barrier_limit ? barrier_limit : kWalkBarrierLimit;
  if (cudaLaunchKernelEx(&cfg, kfn, runs, nruns, tblk, ntblk, order, ntiles, nsteps, lv, adv, bar, err, lim) !=
      cudaSuccess)
    return -2;
  return 0;
}

int launch_step_f32_tma(const StepCoef &K, const Coef<float> &F, const StepScalars &P, const TmaMaps &tm,
                        float *psi_n, float *c_n, float *phi_n, BlockPartial *partials, int max_partials,
                        int *nparts_out, int *err, cudaStream_t st) {
  const int nj = K.ny - 2;
  if (K.nx % 4 || K.pitch != K.nx) return -1;  // rows are copied in 16-byte units
  // column-major: consecutive CTAs share a column strip and its halo rows in L2
  const dim3 grid((nj + kTR - 1) / kTR, (K.nx + kW - 1) / kW), block(kThreads);
  if (grid.y > 65535 || (int64_t)grid.x * grid.y > (1 << 30)) return -1;
  const int nparts = grid.x * grid.y;
  if (partials && nparts > max_partials) return -1;
  if (tm.col_tab_len < (int)grid.y * kW + kWin) return -1;
  const bool surr = tm.surr != nullptr;
  if (K.tfc) {
    // the coarse-grid temperature: no table kernel, so the tile kernel runs
    // in plain stream order (it issues its TMA loads before
    // griddepcontrol.wait, which is safe only after the table kernel); the
    // maps' boxes are kTfcTR + 2 rows high
    if (!P.T_coarse || surr) return -1;
    const dim3 tg((nj + kTfcTR - 1) / kTfcTR, grid.y);
    const int np = (int)(tg.x * tg.y);
    if (partials && np > max_partials) return -1;
    const size_t tsmem = sizeof(TileSmemT<kTfcTR, true>);
    static std::atomic<unsigned long long> tattr{0};
    if (!smem_limit_once((const void *)tile_kernel_tfc, (int)tsmem, tattr)) return -3;
    static std::atomic<int> twave[64];
    const int wave = resident_ctas((const void *)tile_kernel_tfc, kThreads, tsmem, twave);
    if (wave < 0) return -3;
    cudaLaunchConfig_t tc = {};
    tc.gridDim = tg;
    tc.blockDim = block;
    tc.dynamicSmemBytes = tsmem;
    tc.stream = st;
    FinalRed fr = tm.red;
    fr.partials = partials;
    fr.nparts = np;
    FinalRed none = fr;
    none.counter = nullptr;
    const float *tab = tm.col_tab;
    if (cudaLaunchKernelEx(&tc, tile_kernel_tfc, K, F, P, tm.psi, tm.c, tab, tm.col_tab_len, psi_n, c_n, phi_n,
                           partials, err, none, wave) != cudaSuccess)
      return -3;
    if (partials && (fr.mass_out || fr.itip_out) && launch_reduce_partials_dep(fr, st)) return -3;
    if (nparts_out) *nparts_out = np;
    return 0;
  }
  if (tm.pipeline && !surr && !P.pull_back) {  // the persistent warp-role kernel (exact path)
    const int nrt = (int)grid.x, ncb = (int)grid.y;
    const size_t psmem = sizeof(PipeSmem32);
    static std::atomic<unsigned long long> pattr{0};
    if (!smem_limit_once((const void *)pipe_kernel_f32, (int)psmem, pattr)) return -3;
    static std::atomic<int> president[64];
    const int res = resident_ctas((const void *)pipe_kernel_f32, kPipeThreads, psmem, president);
    if (res <= 0) return -3;
    column_table_kernel<<<(tm.col_tab_len + kTabBlock - 2) / (kTabBlock - 1), kTabBlock, 0, st>>>(
        K, P.d0, P.d1, tm.col_tab_len, tm.col_tab);
    cudaLaunchConfig_t pc = {};
    pc.gridDim = dim3((unsigned)std::min(res, nparts));
    pc.blockDim = dim3(kPipeThreads);
    pc.dynamicSmemBytes = psmem;
    pc.stream = st;
    cudaLaunchAttribute pa[1];
    pa[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    pa[0].val.programmaticStreamSerializationAllowed = 1;
    pc.attrs = pa;
    pc.numAttrs = 1;
    // the final reduction is a programmatic dependent launch after the step
    FinalRed pfr = tm.red;
    pfr.partials = partials;
    pfr.nparts = nparts;
    FinalRed none = pfr;
    none.counter = nullptr;
    const float *ptab = tm.col_tab;
    if (cudaLaunchKernelEx(&pc, pipe_kernel_f32, K, F, P, tm.psi, tm.c, ptab, tm.col_tab_len, psi_n, c_n, phi_n,
                           partials, err, none, nrt, ncb) != cudaSuccess)
      return -3;
    if (partials && (pfr.mass_out || pfr.itip_out) && launch_reduce_partials_dep(pfr, st)) return -3;
    if (nparts_out) *nparts_out = nparts;
    return 0;
  }
  const size_t smem = sizeof(TileSmem);
  auto kfn = surr ? tile_kernel<true> : tile_kernel<false>;
  static std::atomic<unsigned long long> attr_done[2];
  if (!smem_limit_once((const void *)kfn, (int)smem, attr_done[surr])) return -3;
  static std::atomic<int> wave_of[2][64];
  const int wave = resident_ctas((const void *)kfn, kThreads, smem, wave_of[surr]);
  if (wave < 0) return -3;
  SurrArgs sa = {};
  if (surr) sa = *tm.surr;
  column_table_kernel<<<(tm.col_tab_len + kTabBlock - 2) / (kTabBlock - 1), kTabBlock, 0, st>>>(K, P.d0, P.d1, tm.col_tab_len, tm.col_tab);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  const float *tab = tm.col_tab;
  // the final reduction is a programmatic dependent launch after the step
  FinalRed fr = tm.red;
  fr.partials = partials;
  fr.nparts = nparts;
  FinalRed none = fr;
  none.counter = nullptr;
  if (cudaLaunchKernelEx(&cfg, kfn, K, F, P, tm.psi, tm.c, tab, tm.col_tab_len, psi_n, c_n, phi_n, partials, err,
                         sa, none, wave) != cudaSuccess)
    return -3;
  if (partials && (fr.mass_out || fr.itip_out) && launch_reduce_partials_dep(fr, st)) return -3;
  if (nparts_out) *nparts_out = nparts;
  return 0;
}

}  // namespace rs

// rs_step_f64t.cu — the FP64 (exact, drop-in) fused phase-field step on
// TMA-staged tiles.
//
// Same equations as the register-prefetch kernel of rs_step.cu
// (compute_phi / compute_psi / compute_c_CALPHAD, fun.cu:1143-1467) and the
// same tile organisation as the FP32 kernel of rs_step_f32.cu, in FP64 on the
// reference's own field layout (psi and c as doubles).  One step is two
// launches:
//   * column_table_kernel_f64: the per-column CALPHAD groups of this step's
//     frozen temperature (col_terms, get_delta fun.cu:1610-1619) in FP64;
//   * tile_kernel_f64, launched as a programmatic dependent of the table
//     kernel: its CTAs start, issue their TMA loads, and wait for the table
//     only where they first read it.
//
// A CTA of 128 threads owns a tile of 16 output rows x 64 output columns
// (x0 .. x0+63, x0 a multiple of 64).  Its input, 18 rows x 72 columns
// (x0-4 .. x0+67, so the TMA x coordinate stays 16-byte aligned), arrives in
// shared memory by one TMA box per field.  Two adjacent columns per lane
// (16-byte double2 shared-memory accesses).
//   phase 1  per-cell S = q(psi) c (1-c) and mu'' of the 18 input rows into
//            shared memory, with per-row flags "every psi == -1" / "== +1"
//            and per-lane phi masks; the halo columns x0-1 and x0+64 are
//            computed by 36 threads of warps 2 and 3 (one input row fewer);
//   phase 2  each warp computes 4 output rows: face fluxes from the shared S
//            and mu'' (neighbours straight from shared memory), the c update
//            (kept in registers); cells whose 3x3 phi neighbourhood is not
//            uniformly +-1 are listed;
//   phase 3  the listed interface cells are updated one per thread;
//   phase 4  new psi and c are written into the shared tile, ghost columns
//            copied there, and each output row leaves by one bulk async copy
//            per field (ghost rows by one more, except in row-band mode);
//   partials the solute mass (FP64) and coarse tip of the tile; the last CTA
//            to finish reduces them all.
// Arithmetic (identical mathematics to the reference, regrouped as in the
// FP32 tile kernel):
//   * mu = K(T) + C0(T) + mu'', C0 = -D - (L0_BCC - L0_Liq)(1 - 2 cinf)/2, so
//       mu'' = -(g+1) C0 - delta (L0_BCC + L0_Liq + g (L0_BCC - L0_Liq)) + RT lam
//     and K + C0 enters only through its column differences dK;
//   * lam = log(c/(1-c)) - log(cinf/(1-cinf)) = 2 atanh(s),
//     s = delta / (2 cinf (1-c) + delta), by its series to s^15 where every
//     cell of the warp's row has |s| < 1/9 (truncation below 3.3e-17
//     relative), else by the logarithm;
//   * bulk melt rows (psi = -1 exactly, delta in the series range): g = -1,
//     q = 1, so mu'' = -2 L0_Liq delta + RT lam and S = c (1 - c); far-melt
//     rows (|delta| <= 1e-3 min(cinf, 1-cinf) as well) take lam as its
//     Taylor polynomial in delta (Coef::melt_a), without the division of s;
//   * deep solid rows (psi = +1 over the 3x3 neighbourhoods) store
//     S = mu'' = 0: every face weight touching them is 0;
//   * face weights by pair sums (6 P_i + P_{i-1} + P_{i+1}, four times the
//     1.5 / 0.25 weights, the 4 folded into the flux constant); face fluxes
//     are rounded products, so a cell's result does not depend on the tiling.
// Launch order: the tile columns from the one holding the front
// (front_first_block).  After phase 1 each CTA prefetches into L2 the input
// tile of the block launched one resident wave later.
// The coarse-grid temperature (TFC, interpolate_temperature
// fun.cu:1580-1608): no table kernel; every cell evaluates its CALPHAD groups
// from its own bilinear temperature (K + C0 by its Taylor polynomial about
// the tile's centre temperature, kc_poly; C0 in general rows and cells out of
// the polynomial's range by the Gibbs functions) and stores
// mu = mu'' + (K + C0), so the faces take plain differences of mu.  The tile kernel then runs in plain stream
// order: it issues its TMA loads before griddepcontrol.wait.
//
// Two kernels run these phases (same functions, same results bit for bit):
//   * tile_kernel_f64: one tile per CTA of 128 threads, the phases in series
//     separated by CTA barriers, five CTAs per SM;
//   * pipe_kernel_f64: persistent CTAs of three warp roles that work on
//     three tiles at once -- one producer warp issuing the TMA loads of tile
//     k+2 into a three-slot input ring, four warps computing phase 1 of tile
//     k+1 into a two-slot staging ring, four warps doing phases 2-4 of tile k
//     and its bulk stores.  Hand-offs are mbarriers (full / empty per slot),
//     each role synchronises its own warps by a named barrier, every wait is
//     bounded (a wait that gives up sets the error flag and the CTA stops
//     after draining its loads and stores).
#include "rs_step_common.cuh"

namespace rs {
namespace {

constexpr int kW = kTileOutW64;   // output columns of a tile
constexpr int kWin = kTmaBoxW64;  // input columns of a tile (kW + 8)
constexpr int kTR = kTileRows;    // output rows of a tile
constexpr int kTRin = kTmaBoxH;   // input rows of a tile
constexpr int kThreads = 128;     // threads of a phase group
constexpr int kWarps = kThreads / 32;
constexpr int kRowsPerWarp = kTR / kWarps;
constexpr int kHaloL = 3, kHaloR = kW + 4;  // box columns of x0-1 and x0+kW
constexpr uint32_t kWaitLimit = 1u << 20;
constexpr unsigned FULL = 0xffffffffu;
constexpr unsigned long long kMinus1 = 0xBFF0000000000000ull, kPlus1 = 0x3FF0000000000000ull;
constexpr uint32_t kTileBytes = 2u * kTRin * kWin * sizeof(double);
static_assert(kW == 32 * 2, "two columns per lane");
static_assert(kTR % kWarps == 0 && kRowsPerWarp == 4, "four output rows per warp");
static_assert(kTRin <= 32, "row flags are 32-bit masks");
static_assert(64 + 2 * kTRin <= kThreads && 4 * kTR <= kThreads, "one thread per halo cell and per row copy");

// column table arrays (kColTabFields of them, len doubles each); entry k
// describes column k - 4
enum { kTabRT = 0, kTabC0 = 1, kTabDK = 2, kTabAnb = 3, kTabAti = 4 };

// the input tile: TMA destinations (128-byte aligned); after phase 3 rows
// 1..16 receive the new psi / c for the bulk stores
struct alignas(128) InSlot {  // both arrays are TMA destinations: 128-byte aligned
  alignas(128) double psi[kTRin][kWin];
  alignas(128) double c[kTRin][kWin];
};
// phase 1 -> phases 2-4: per-cell terms and row flags
struct alignas(16) StSlot {
  double S[kTRin][kWin];  // after phase 2: new psi of the listed cells
  double mu[kTRin][kWin];
  uint8_t pmask[kTRin][32];  // per lane: bits 0-1 psi <= -1, bits 4-5 psi >= 1 of its two cells
                             // (rows flagged in liq / sol store none)
  uint8_t hmask[kTRin][2];   // halo cells: bit 0 psi <= -1, bit 1 psi >= 1
  uint32_t liq, sol;         // bit r: every cell of input row r has psi == -1 / +1
  double ty[kTRin];          // TFC: the row part of each input row's temperature
  int tj[kTRin];             // (tfc_row), once per tile
  KcPoly kp;                 // TFC: K + C0 near the tile's temperature
  double hx[2];              // TFC: column part of the halo columns' temperatures
  int hiT[2];
};
// phases 2-4: the interface list and the partial sums
struct P2Smem {
  uint16_t list[kTR * kW];  // interface cells: row << 8 | output column
  int nlist;
  int last;  // this CTA finished last (fused final reduction)
  double part_mass[kWarps];
  int part_itip[kWarps];
};
struct alignas(128) TileSmem64 {
  InSlot in;
  StSlot st;
  P2Smem p2;
  uint64_t full;
};
constexpr int kRing = 3, kStage = 2;
struct alignas(128) PipeSmem64 {
  InSlot in[kRing];
  StSlot st[kStage];
  P2Smem p2;
  uint64_t in_full[kRing], in_empty[kRing], st_full[kStage], st_empty[kStage];
  int abort;  // a wait gave up: every role stops
};
static_assert(sizeof(InSlot) % 128 == 0 && offsetof(InSlot, psi) % 128 == 0 && offsetof(InSlot, c) % 128 == 0,
              "ring slots and their TMA destinations stay 128-byte aligned");
static_assert(offsetof(PipeSmem64, in) % 128 == 0 && offsetof(TileSmem64, in) % 128 == 0,
              "the input slots start on 128-byte boundaries");
static_assert((kWin * sizeof(double)) % 16 == 0, "rows stay 16-byte aligned for double2 and bulk copies");

__device__ __forceinline__ double2 ld2(const double *p) { return *reinterpret_cast<const double2 *>(p); }
__device__ __forceinline__ void st2(double *p, double a, double b) {
  *reinterpret_cast<double2 *>(p) = make_double2(a, b);
}
__device__ __forceinline__ double clamp1(double v) { return fmin(fmax(v, -1.0), 1.0); }
__device__ __forceinline__ unsigned long long bits(double v) { return (unsigned long long)__double_as_longlong(v); }
// barrier of one phase group of 128 threads (id 0 with 128-thread CTAs: the CTA)
__device__ __forceinline__ void gsync(int id) { asm volatile("bar.sync %0, 128;" ::"r"(id) : "memory"); }
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// 2 atanh(s) by its odd series to s^15 (|s| < 1/9: truncation below
// 3.3e-17 relative)
__device__ __forceinline__ double lam_series(double s) {
  const double s2 = s * s;
  double p = 1.0 / 15.0;
  p = fma(p, s2, 1.0 / 13.0);
  p = fma(p, s2, 1.0 / 11.0);
  p = fma(p, s2, 1.0 / 9.0);
  p = fma(p, s2, 1.0 / 7.0);
  p = fma(p, s2, 1.0 / 5.0);
  p = fma(p, s2, 1.0 / 3.0);
  return 2.0 * fma(s * s2, p, s);
}

// general per-cell terms (fun.cu:1424-1452); series: use 2 atanh(s)
__device__ __forceinline__ void cell_terms(const Coef<double> &F, double pv, double c, double s, bool series,
                                           double RT, double C0, double &S, double &mu) {
  constexpr double L0sum = kL0Bcc + kL0Liq;
  constexpr double L0half = 0.5 * (kL0Bcc - kL0Liq);
  const double om = 1.0 - c, dv = c - F.cinf;
  const double a = 1.0 - pv;
  S = (0.5 * F.AA * a - 0.25 * (F.AA - 1.0) * (a * a)) * c * om;
  const double p2 = pv * pv;
  const double g = pv * (1.875 + p2 * (-1.25 + 0.375 * p2));
  const double lam = series ? lam_series(s) : Tr<double>::lam(c, om, dv, F.cinf, F.Lref);
  mu = -(g + 1.0) * C0 - dv * fma(2.0 * L0half, g, L0sum) + RT * lam;
}

// shared -> global bulk copy (16-byte aligned addresses, size a multiple of 16)
__device__ __forceinline__ void bulk_store(void *gdst, const void *ssrc, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gdst), "r"(smem_u32(ssrc)),
               "r"(bytes)
               : "memory");
}

// One thread per column, one exact FP64 col_terms each; K + C0 of the next
// column comes from the neighbouring thread, so blocks overlap by one column
// and write 127 entries.
constexpr int kTabBlock = 128;
__global__ void __launch_bounds__(kTabBlock) column_table_kernel_f64(const StepCoef K, const double d0,
                                                                     const double d1, const int len,
                                                                     double *__restrict__ tab) {
  // the tile kernel may start now; it waits for this grid before reading tab
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  __shared__ double kc[kTabBlock];
  const int k = blockIdx.x * (kTabBlock - 1) + threadIdx.x;  // table entry; column k - 4
  const int gi = min(max(k - 4, 0), K.nx - 1);
  const double T = (d0 + d1 * gi) * K.deltaT0 + K.Tmelt;  // get_delta, fun.cu:1610-1619
  const ColT<double> ct = col_terms<double>(K, T);
  const double C0 = -ct.D - 0.5 * (kL0Bcc - kL0Liq) * (1.0 - 2.0 * K.cinf);
  kc[threadIdx.x] = ct.Kc + C0;
  __syncthreads();
  if (threadIdx.x == kTabBlock - 1 || k >= len) return;
  tab[kTabRT * len + k] = ct.RT;
  tab[kTabC0 * len + k] = C0;
  tab[kTabDK * len + k] = kc[threadIdx.x + 1] - kc[threadIdx.x];  // (K + C0)(i+1) - (K + C0)(i)
  tab[kTabAnb * len + k] = ct.A_nb;
  tab[kTabAti * len + k] = ct.A_ti;
}

// the column table, indexed by column
struct Tab {
  const double *RT, *C0, *DK, *Anb, *Ati;
  __device__ Tab(const double *tab, int len)
      : RT(tab + kTabRT * len + 4), C0(tab + kTabC0 * len + 4), DK(tab + kTabDK * len + 4),
        Anb(tab + kTabAnb * len + 4), Ati(tab + kTabAti * len + 4) {}
};

// Everything one phase group needs about a tile and its own lane.
struct TileView {
  const StepCoef &K;
  const Coef<double> &F;
  const StepScalars &PS;
  Tab T;
  int x0, y0;  // first output column, first output row (input rows y0-1 .. y0+kTR)
  int gw, lane, gtid;  // warp and lane within the group, thread of the group
  int col, gi, bc;     // the lane's first cell: tile column, global column, box column
  uint32_t outm;       // per cell of the lane: an interior (output) cell
  __device__ TileView(const StepCoef &K_, const Coef<double> &F_, const StepScalars &PS_, const double *tab,
                      int tab_len, int x0_, int y0_, int gtid_)
      : K(K_), F(F_), PS(PS_), T(tab, tab_len), x0(x0_), y0(y0_), gw(gtid_ >> 5), lane(gtid_ & 31), gtid(gtid_) {
    col = 2 * lane;
    gi = x0 + col;
    bc = col + 4;
    outm = 0;
#pragma unroll
    for (int q = 0; q < 2; ++q)
      if (gi + q >= 1 && gi + q <= K.nx - 2) outm |= 1u << q;
  }
};

// The column table entries a lane uses: RT and C0 of its two columns, dK of
// the faces left of its columns and of the next one.  The tile kernel loads
// them before it waits for its tile, so their latency hides under the load.
struct LaneCols {
  double RT[2], C0[2], dK[3];
  int tiT[2];       // TFC: the coarse column left of each of the lane's two columns
  double tx[2];     // and the column's offset from it, in coarse cells
};
__device__ __forceinline__ CellGroups cell_groups(const TileView &V, int gx, int row) {
  int iT, jT;
  double x, y;
  tfc_col(V.K, V.PS.i_left_end_T, gx, iT, x);
  tfc_row(V.K, row, jT, y);
  return groups_exact(V.K, tfc_T(V.K, V.PS.T_coarse, iT, x, jT, y));
}

template <bool TFC>
__device__ __forceinline__ LaneCols lane_cols(const TileView &V) {
  LaneCols L;
  if constexpr (TFC) {  // per cell (cell_groups); no column differences
    L.RT[0] = L.RT[1] = L.C0[0] = L.C0[1] = 0.0;
    L.dK[0] = L.dK[1] = L.dK[2] = 0.0;
    tfc_col(V.K, V.PS.i_left_end_T, V.gi, L.tiT[0], L.tx[0]);
    tfc_col(V.K, V.PS.i_left_end_T, V.gi + 1, L.tiT[1], L.tx[1]);
    return L;
  }
  const double2 RTv = ld2(V.T.RT + V.gi), C0v = ld2(V.T.C0 + V.gi);
  L.RT[0] = RTv.x;
  L.RT[1] = RTv.y;
  L.C0[0] = C0v.x;
  L.C0[1] = C0v.y;
  L.dK[0] = V.T.DK[V.gi - 1];  // faces x-1|x for x = col .. col+2
  L.dK[1] = V.T.DK[V.gi];
  L.dK[2] = V.T.DK[V.gi + 1];
  L.tiT[0] = L.tiT[1] = 0;
  L.tx[0] = L.tx[1] = 0.0;
  return L;
}

// columns beyond the array (right-most tiles; zero-filled by TMA) become
// bulk melt, so they never force the general path; no output reads them.
// Returns whether it wrote (the group then synchronises).
__device__ __forceinline__ bool fix_beyond(const TileView &V, InSlot &in) {
  if (V.x0 + kW + 4 <= V.K.nx) return false;
  for (int k = V.gtid; k < kTRin * kWin; k += kThreads) {
    const int rr = k / kWin, x = k % kWin;
    if (V.x0 - 4 + x >= V.K.nx) {
      in.psi[rr][x] = -1.0;
      in.c[rr][x] = V.F.cinf;
    }
  }
  return true;
}

// ---- phase 1: per-cell terms of the input rows of group warp gw (rows gw,
// gw+4, ...) and of the halo columns (group threads 64..99); st.liq and
// st.sol must be 0 on entry
template <bool TFC>
__device__ __forceinline__ void phase1(const TileView &V, const LaneCols &LC, const InSlot &in, StSlot &st) {
  const Coef<double> &F = V.F;
  const int lane = V.lane, bc = V.bc;
  const double cinf = F.cinf;
  constexpr double KL = -2.0 * kL0Liq;
  const double d_hi = F.ser_hi, d_lo = F.ser_lo;  // series range of delta (Coef)
  double RTa[2] = {LC.RT[0], LC.RT[1]}, C0a[2] = {LC.C0[0], LC.C0[1]}, KCa[2] = {0.0, 0.0};
  // per lane, bit q: psi is exactly +1 over the 3x3 neighbourhood of cell
  // bc+q (rows of the box only; column -1 of the left-most tile enters no
  // face, column 0 being a ghost).  S = q(1) c (1 - c) = 0 there, so every
  // face weight touching the cell is 0 and its mu'' enters no flux
  auto solid3 = [&](int rr) -> uint32_t {
    const int xh = lane == 0 ? kHaloL : kHaloR;
    uint32_t v = 0x3u;
    bool hs = true;  // the halo column beside lanes 0 and 31
    for (int r2 = max(rr - 1, 0); r2 <= min(rr + 1, kTRin - 1); ++r2) {
      const double2 q2 = ld2(&in.psi[r2][bc]);
      v &= (bits(q2.x) == kPlus1 ? 1u : 0u) | (bits(q2.y) == kPlus1 ? 2u : 0u);
      hs = hs && bits(in.psi[r2][xh]) == kPlus1;
    }
    uint32_t lf = __shfl_up_sync(FULL, v >> 1, 1) & 1u, rt = __shfl_down_sync(FULL, v, 1) & 1u;
    if (lane == 0) lf = (hs || V.x0 == 0) ? 1u : 0u;
    if (lane == 31) rt = hs ? 1u : 0u;
    const uint32_t e = lf | (v << 1) | (rt << 3);  // bit k: box column bc-1+k
    return e & (e >> 1) & (e >> 2) & 0x3u;
  };
  // constants of the row loop in registers (one read of the launch
  // arguments, not one per row)
  double ma[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) ma[k] = F.melt_a[k];
  const double tiny = F.melt_tiny;
  const int rows_in = V.K.ny - V.y0;  // input rows inside the array: rr <= ny - y0
  // this warp's row flags (warp-uniform), OR-ed into st.liq / st.sol once
  uint32_t liq_rows = 0u, sol_rows = 0u;
  // TFC: along a column the bilinear temperature is P + Q y within one coarse
  // row band jT; the lane keeps P and Q of its two columns for the band of
  // its last row (rows of a warp are 4 apart, bands `ratio` rows high)
  int band_jT = -1;
  double Pb[2] = {0.0, 0.0}, Qb[2] = {0.0, 0.0};
#pragma unroll 1
  for (int rr = V.gw; rr < kTRin; rr += kWarps) {
    if (rr > rows_in) {  // beyond the array (last tile): never read by an output
      st2(&st.S[rr][bc], 0.0, 0.0);
      st2(&st.mu[rr][bc], 0.0, 0.0);
      liq_rows |= 1u << rr;
      sol_rows |= 1u << rr;
      continue;
    }
    const double2 pv2 = ld2(&in.psi[rr][bc]), cv2 = ld2(&in.c[rr][bc]);
    const double pv[2] = {pv2.x, pv2.y}, cv[2] = {cv2.x, cv2.y};
    const double dv[2] = {cv[0] - cinf, cv[1] - cinf};
    double Sv[2], mv[2];
    const unsigned long long b0 = bits(pv[0]), b1 = bits(pv[1]);
    const bool liq2 = b0 == kMinus1 && b1 == kMinus1;
    const bool sol2 = b0 == kPlus1 && b1 == kPlus1;
    // the row's form (warp-uniform): far melt, bulk melt or general
    const bool far = __all_sync(FULL, liq2 && fmax(fabs(dv[0]), fabs(dv[1])) <= tiny);
    const bool bulk = !far && __all_sync(FULL, liq2 && fmax(dv[0], dv[1]) < d_hi && fmin(dv[0], dv[1]) > d_lo);
    if constexpr (TFC) {  // the melt forms need RT and K + C0 only
      const int jT = st.tj[rr];
      const double y = st.ty[rr];
      if (jT != band_jT) {  // warp-uniform: jT depends on the row only
        band_jT = jT;
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const double *r0 = V.PS.T_coarse + (int64_t)jT * V.K.NxT_all + LC.tiT[q], *r1 = r0 + V.K.NxT_all;
          const double f00 = r0[0], f10 = r0[1], f01 = r1[0], f11 = r1[1];
          Pb[q] = fma(f10 - f00, LC.tx[q], f00);
          Qb[q] = fma(f11 - f10 - f01 + f00, LC.tx[q], f01 - f00);
        }
      }
#pragma unroll
      for (int q = 0; q < 2; ++q)
        cell_tfc(V.K, st.kp, fma(Qb[q], y, Pb[q]), !(far || bulk), RTa[q], C0a[q], KCa[q]);
    }
    uint32_t code;
    bool deep = false;
    if (far) {
      // far melt: g = -1, q = 1, lam by its Taylor polynomial in delta
      // (Coef::melt_a, six terms); mu'' = RT lam - 2 L0_Liq delta
      // = delta (RT p + KL), lam = delta p
      code = 1u;
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        double p = ma[5];
#pragma unroll
        for (int k = 4; k >= 0; --k) p = fma(p, dv[q], ma[k]);
        Sv[q] = cv[q] * (1.0 - cv[q]);
        mv[q] = dv[q] * fma(RTa[q], p, KL);
      }
    } else if (bulk) {
      // bulk melt: g = -1, q = 1
      code = 1u;
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const double c = cv[q], om = 1.0 - c;
        const double sv = dv[q] / fma(2.0 * cinf, om, dv[q]);
        Sv[q] = c * om;
        mv[q] = fma(RTa[q], lam_series(sv), dv[q] * KL);
      }
    } else {
      code = (__all_sync(FULL, liq2) ? 1u : 0u) | (__all_sync(FULL, sol2) ? 2u : 0u);
      // deep solid row: no cell's mu'' enters a flux, so S = mu'' = 0 gives
      // the same fluxes
      const uint32_t s3 = (code & 2u) ? solid3(rr) : 0u;
      if ((code & 2u) && __all_sync(FULL, s3 == 0x3u)) {
        Sv[0] = Sv[1] = mv[0] = mv[1] = 0.0;
        deep = true;
      } else {
        double sv[2];
        bool small = true;
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          sv[q] = dv[q] / fma(2.0 * cinf, 1.0 - cv[q], dv[q]);
          small = small && fabs(sv[q]) < 1.0 / 9.0;
        }
        const bool series = __all_sync(FULL, small);
        uint32_t L = 0u, Sm = 0u;
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          if (pv[q] <= -1.0) L |= 1u << q;
          if (pv[q] >= 1.0) Sm |= 1u << q;
          cell_terms(F, pv[q], cv[q], sv[q], series, RTa[q], C0a[q], Sv[q], mv[q]);
        }
        st.pmask[rr][lane] = (uint8_t)(L | (Sm << 4));
      }
    }
    if (TFC && !deep) {  // mu = mu'' + (K + C0) of the cell itself
      mv[0] += KCa[0];
      mv[1] += KCa[1];
    }
    st2(&st.S[rr][bc], Sv[0], Sv[1]);
    st2(&st.mu[rr][bc], mv[0], mv[1]);
    liq_rows |= (code & 1u) << rr;
    sol_rows |= ((code >> 1) & 1u) << rr;
  }
  if (lane == 0) {
    if (liq_rows) atomicOr(&st.liq, liq_rows);
    if (sol_rows) atomicOr(&st.sol, sol_rows);
  }
  // halo columns x0-1 and x0+kW, one thread per cell, on group warps 2 and
  // 3, which have one input row fewer than warps 0 and 1
  if (V.gtid >= 64 && V.gtid < 64 + 2 * kTRin) {
    const int i = V.gtid - 64;
    const int rr = i >> 1, side = i & 1;
    const int x = side ? kHaloR : kHaloL, g = V.x0 - 4 + x;
    double Sh = 0.0, mh = 0.0;
    uint8_t hm = 3u;
    if (V.y0 - 1 + rr <= V.K.ny - 1) {
      const double pv = in.psi[rr][x], cv = in.c[rr][x];
      const double dv = cv - cinf;
      const double sv = dv / fma(2.0 * cinf, 1.0 - cv, dv);
      if constexpr (TFC) {
        // C0 enters mu'' as (g + 1) C0, 0 at psi = -1 exactly: the liquid
        // groups suffice there
        double RT, C0, KC;
        cell_tfc(V.K, st.kp, tfc_T(V.K, V.PS.T_coarse, st.hiT[side], st.hx[side], st.tj[rr], st.ty[rr]),
                 bits(pv) != kMinus1, RT, C0, KC);
        cell_terms(F, pv, cv, sv, fabs(sv) < 1.0 / 9.0, RT, C0, Sh, mh);
        mh += KC;
      } else {
        cell_terms(F, pv, cv, sv, fabs(sv) < 1.0 / 9.0, V.T.RT[g], V.T.C0[g], Sh, mh);
      }
      hm = (pv <= -1.0 ? 1u : 0u) | (pv >= 1.0 ? 2u : 0u);
    }
    st.S[rr][x] = Sh;
    st.mu[rr][x] = mh;
    st.hmask[rr][side] = hm;
  }
}

// ---- phase 2: group warp gw computes output rows 1 + 4gw .. 4 + 4gw:
// fluxes, the c update into dn, the interface cells into the list (nlist
// must be 0 on entry).  Returns the listed cells, 2 bits per output row.
__device__ __forceinline__ uint32_t phase2(const TileView &V, const LaneCols &LC, const InSlot &in,
                                           const StSlot &st, P2Smem &p2,
                                           double dn[kRowsPerWarp][2], double &mass, bool red) {
  const Coef<double> &F = V.F;
  const int lane = V.lane, bc = V.bc;
  const double cflux4 = 0.25 * F.cflux, c_floor = F.c_floor;
  const int rows_live = V.K.ny - 1 - V.y0;  // output rows inside the interior: rr <= ny - 1 - y0
  const uint32_t liq = st.liq, sol = st.sol;
  const double dKa[3] = {LC.dK[0], LC.dK[1], LC.dK[2]};  // faces x-1|x for x = col .. col+2
  struct Row {
    double s[2], m[2], sl, sr, ml, mr;
  };
  // S pair sums of the faces left of cell f (f = 0..2) of a row
  struct Pairs {
    double q[3];
  };
  auto load_row = [&](int rr, Row &R) {
    const double2 s = ld2(&st.S[rr][bc]), m = ld2(&st.mu[rr][bc]);
    R.s[0] = s.x;
    R.s[1] = s.y;
    R.m[0] = m.x;
    R.m[1] = m.y;
    R.sl = st.S[rr][bc - 1];  // lane 0: the halo column x0-1
    R.ml = st.mu[rr][bc - 1];
    R.sr = st.S[rr][bc + 2];  // lane 31: the halo column x0+kW
    R.mr = st.mu[rr][bc + 2];
  };
  auto pairs = [](const Row &R) {
    Pairs P;
    P.q[0] = R.sl + R.s[0];
    P.q[1] = R.s[0] + R.s[1];
    P.q[2] = R.s[1] + R.sr;
    return P;
  };
  // fluxes through the faces between rows A and B = A+1 (compute_c_CALPHAD
  // F01/F0m), rounded products so that a face rounds the same wherever the
  // tiling puts it
  auto vface = [&](const Row &A, const Row &B, double jv[2]) {
    const double pp[4] = {A.sl + B.sl, A.s[0] + B.s[0], A.s[1] + B.s[1], A.sr + B.sr};
#pragma unroll
    for (int q = 0; q < 2; ++q) jv[q] = __dmul_rn(fma(6.0, pp[q + 1], pp[q] + pp[q + 2]), B.m[q] - A.m[q]);
  };

  const int rbase = 1 + kRowsPerWarp * V.gw;
  Row rb, rc;
  Pairs pa, pb, pc;
  double jv_lo[2], jv_hi[2];
  uint32_t needs_all = 0u;
  {
    Row ra;
    load_row(rbase - 1, ra);
    load_row(rbase, rb);
    vface(ra, rb, jv_lo);
    pa = pairs(ra);
    pb = pairs(rb);
  }
#pragma unroll
  for (int j = 0; j < kRowsPerWarp; ++j) {
    const int rr = rbase + j;  // tile input row of the output row
    load_row(rr + 1, rc);
    pc = pairs(rc);
    vface(rb, rc, jv_hi);
    // fluxes through the faces (x-1/2, r) for x = col .. col+2
    const double mm[4] = {rb.ml, rb.m[0], rb.m[1], rb.mr};
    double jh[3];
#pragma unroll
    for (int fc = 0; fc < 3; ++fc)
      jh[fc] = __dmul_rn(fma(6.0, pb.q[fc], pa.q[fc] + pc.q[fc]), mm[fc + 1] - mm[fc] + dKa[fc]);
    const double2 cv2 = ld2(&in.c[rr][bc]);
    const double cv[2] = {cv2.x, cv2.y};
#pragma unroll
    for (int q = 0; q < 2; ++q)
      dn[j][q] = fmax(fma(cflux4, (jh[q + 1] - jh[q]) + (jv_hi[q] - jv_lo[q]), cv[q]), c_floor);
    const bool live = rr <= rows_live;
    if (red && live) {
#pragma unroll
      for (int q = 0; q < 2; ++q)
        if ((V.outm >> q) & 1u) mass += dn[j][q];
    }
    // phi: cells whose 3x3 neighbourhood is not uniformly +-1 are listed
    const uint32_t w3 = 7u << (rr - 1);
    if (live && (liq & w3) != w3 && (sol & w3) != w3) {
      // per input row k: bits 0-1 psi <= -1, bits 4-5 psi >= 1 of the lane's cells
      // (rows flagged all -1 / all +1 store no masks: 0x03 / 0x30)
      auto pm = [&](int k) -> uint32_t {
        return ((liq >> k) & 1u) ? 0x03u : ((sol >> k) & 1u) ? 0x30u : (uint32_t)st.pmask[k][lane];
      };
      const uint32_t pk = pm(rr - 1) | (pm(rr) << 8) | (pm(rr + 1) << 16);
      const uint32_t lf = __shfl_up_sync(FULL, pk, 1), rt = __shfl_down_sync(FULL, pk, 1);
      // left neighbour's second cell: its bits 1 and 5; right neighbour's first: bits 0 and 4
      uint32_t lL = 0u, lS = 0u, rL = 0u, rS = 0u;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        lL |= ((lf >> (8 * k + 1)) & 1u) << k;
        lS |= ((lf >> (8 * k + 5)) & 1u) << k;
        rL |= ((rt >> (8 * k)) & 1u) << k;
        rS |= ((rt >> (8 * k + 4)) & 1u) << k;
      }
      if (lane == 0) {
        lL = lS = 0u;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const uint32_t h = st.hmask[rr - 1 + k][0];
          lL |= (h & 1u) << k;
          lS |= ((h >> 1) & 1u) << k;
        }
      }
      if (lane == 31) {
        rL = rS = 0u;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const uint32_t h = st.hmask[rr - 1 + k][1];
          rL |= (h & 1u) << k;
          rS |= ((h >> 1) & 1u) << k;
        }
      }
      // over the three rows, bit b: box column bc-1+b is liquid / solid
      uint32_t Lv = 0xFu, Sv = 0xFu;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const uint32_t L = (pk >> (8 * k)) & 0x3u, S = (pk >> (8 * k + 4)) & 0x3u;
        Lv &= ((lL >> k) & 1u) | (L << 1) | (((rL >> k) & 1u) << 3);
        Sv &= ((lS >> k) & 1u) | (S << 1) | (((rS >> k) & 1u) << 3);
      }
      const uint32_t needs = ~((Lv & (Lv >> 1) & (Lv >> 2)) | (Sv & (Sv >> 1) & (Sv >> 2))) & V.outm;
      const uint32_t cnt = __popc(needs);
      uint32_t incl = cnt;  // inclusive warp scan of the counts
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
      for (int q = 0; q < 2; ++q)
        if ((needs >> q) & 1u) p2.list[off++] = (uint16_t)((rr << 8) | (V.col + q));
      needs_all |= needs << (2 * j);
    }
    rb = rc;
    pa = pb;
    pb = pc;
#pragma unroll
    for (int q = 0; q < 2; ++q) jv_lo[q] = jv_hi[q];
  }
  return needs_all;
}

// ---- phase 3: the listed interface cells, one per group thread
// (compute_phi, fun.cu:1143-1218); new psi into np[rr][x]
template <bool TFC>
__device__ __forceinline__ void phase3(const TileView &V, const InSlot &in, const P2Smem &p2,
                                       double (*np)[kWin], bool red, int &itip) {
  const int nlist = p2.nlist;
  for (int idx = V.gtid; idx < nlist; idx += kThreads) {
    const uint32_t e = p2.list[idx];
    const int rr = (int)(e >> 8), x = (int)(e & 0xFFu) + 4;  // box column
    const int r = V.y0 - 1 + rr, g = V.x0 + x - 4;
    const double c00 = in.c[rr][x];
    double Anb, Ati;
    if constexpr (TFC) {
      const CellGroups cg = cell_groups(V, g, r);
      Anb = cg.Anb;
      Ati = cg.Ati;
    } else {
      Anb = V.T.Anb[g];
      Ati = V.T.Ati[g];
    }
    const double dG = (1.0 - c00) * Anb + c00 * Ati + c00 * (1.0 - c00) * (kL0Liq - kL0Bcc);
    const double res = phi_cell_dG<double>(
        &V.F, clamp1(in.psi[rr][x]), clamp1(in.psi[rr][x + 1]), clamp1(in.psi[rr][x - 1]),
        clamp1(in.psi[rr + 1][x]), clamp1(in.psi[rr - 1][x]), clamp1(in.psi[rr + 1][x + 1]),
        clamp1(in.psi[rr + 1][x - 1]), clamp1(in.psi[rr - 1][x + 1]), clamp1(in.psi[rr - 1][x - 1]), dG,
        V.PS.step, (int64_t)(r + V.K.j_offset) * V.K.nx + g, V.K.seed_lo, V.K.seed_hi);
    np[rr][x] = res;
    if (red && res > 0.0) itip = max(itip, g == V.K.nx - 2 ? V.K.nx - 1 : g);
  }
}

// ---- phase 4: new psi and c of group warp gw's rows into the input tile
// (after every group thread has finished phase 3)
__device__ __forceinline__ void phase4_rows(const TileView &V, InSlot &in, const double (*np)[kWin],
                                            uint32_t needs_all, const double dn[kRowsPerWarp][2], bool red,
                                            int &itip) {
  const int rbase = 1 + kRowsPerWarp * V.gw, bc = V.bc;
#pragma unroll
  for (int j = 0; j < kRowsPerWarp; ++j) {
    const int rr = rbase + j;
    const double2 pv2 = ld2(&in.psi[rr][bc]);
    // phi_next = phi where uniformly +-1: an output cell is not listed only
    // where psi <= -1 or >= 1 over its 3x3 neighbourhood, so clamp(psi) is
    // its sign (cells outside the interior are not stored or are overwritten
    // by the ghost copies); listed cells take phase 3's result
    double po[2] = {pv2.x > 0.0 ? 1.0 : -1.0, pv2.y > 0.0 ? 1.0 : -1.0};
    const uint32_t lb = (needs_all >> (2 * j)) & 3u;
    if (lb) {
#pragma unroll
      for (int q = 0; q < 2; ++q)
        if ((lb >> q) & 1u) po[q] = np[rr][bc + q];
    }
    st2(&in.psi[rr][bc], po[0], po[1]);
    st2(&in.c[rr][bc], dn[j][0], dn[j][1]);
  }
  if (red) {  // coarse tip: the last column with phi > 0 (listed cells counted again, harmlessly)
    const int rows_live = V.K.ny - 1 - V.y0, nx = V.K.nx;
#pragma unroll
    for (int j = 0; j < kRowsPerWarp; ++j) {
      const int rr = rbase + j;
      const double2 po2 = ld2(&in.psi[rr][bc]);
      const double po[2] = {po2.x, po2.y};
      if (rr > rows_live) continue;
#pragma unroll
      for (int q = 0; q < 2; ++q)
        if (((V.outm >> q) & 1u) && po[q] > 0.0) itip = max(itip, V.gi + q == nx - 2 ? nx - 1 : V.gi + q);
    }
  }
}

// ghost columns, then the tile's rows out by bulk copies (group threads
// < 64: row j, field, kind) and phi by plain stores; returns whether this
// thread committed a bulk group (it then waits for its reads before the
// tile's shared memory is reused)
__device__ __forceinline__ bool store_tile(const TileView &V, InSlot &in, double *__restrict__ psi_n,
                                           double *__restrict__ c_n, double *__restrict__ phi_n, int bar) {
  const StepCoef &K = V.K;
  const int x0 = V.x0, y0 = V.y0;
  const int nrow = min(kTR, K.ny - 1 - y0);  // output rows of this tile inside the interior
  const int ncol = min(kW, K.nx - x0);       // columns of this tile inside the array (even)
  if (x0 == 0 || x0 + kW >= K.nx) {
    // ghost columns 0 and nx-1 (compute_boundary_individual, fun.cu:1220-1230)
    gsync(bar);
    if (V.gtid < nrow) {
      const int rr = 1 + V.gtid;
      if (x0 == 0) {
        in.psi[rr][4] = in.psi[rr][5];
        in.c[rr][4] = in.c[rr][5];
      }
      if (x0 + kW >= K.nx) {
        const int x = K.nx - 1 - x0 + 4;
        in.psi[rr][x] = in.psi[rr][x - 1];
        in.c[rr][x] = in.c[rr][x - 1];
      }
    }
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // tile writes -> bulk copies
  gsync(bar);
  bool any = false;
  if (V.gtid < 4 * kTR) {
    const int j = V.gtid >> 2, field = V.gtid & 1, kind = (V.gtid >> 1) & 1;
    const int r = y0 + j;
    if (j < nrow) {
      double *fo = field ? c_n : psi_n;
      const double *src = field ? &in.c[1 + j][4] : &in.psi[1 + j][4];
      const uint32_t bytes = (uint32_t)ncol * 8u;
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
  if (phi_n) {  // phi = clamp(psi) of the same rows, plain stores
    for (int k = V.gtid; k < nrow * ncol; k += kThreads) {
      const int j = k / ncol, x = k % ncol, r = y0 + j;
      const double v = clamp1(in.psi[1 + j][4 + x]);
      phi_n[(int64_t)r * K.pitch + x0 + x] = v;
      if (r == K.jmin) phi_n[x0 + x] = v;
      if (r == K.jmax) phi_n[(int64_t)(K.ny - 1) * K.pitch + x0 + x] = v;
    }
  }
  return any;
}

// the tile's partial sums, and the fused final reduction (the last tile to
// finish sums every partial, in reduce_partials_kernel's order); scratch of
// at least 256 doubles and 256 ints
__device__ __forceinline__ void finish_tile(const TileView &V, P2Smem &p2, double mass, int itip,
                                            BlockPartial *part, const FinalRed *FR, double *sm_m, int *sm_i,
                                            int bar) {
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

// tile (row tr, column tc) of the launch order: tile columns from the one
// holding the front, tile rows of a column consecutive (they share halo rows
// in L2)
__device__ __forceinline__ void tile_of(int t, int nrt, int ncb, int f, int &tr, int &tc) {
  tr = t % nrt;
  tc = front_first_block(t / nrt, f, ncb);
}

// ---------------------------------------------------------------- one tile per CTA
// the input tile of a pull-back step: the same box as the TMA load (columns
// x0-4 .. x0+kW+3, rows y0-1 .. y0+kTR, zeros outside the array), each
// column i read from clamp(i + i_offset, 1, nx - 2), with c = cinf where that
// is nx - 2 (the melt entering at the right edge)
__device__ __forceinline__ void gather_pull_back(const StepCoef &K, const StepScalars &PS, int x0, int y0,
                                                 InSlot &in) {
  const double *__restrict__ psi = static_cast<const double *>(PS.src_psi);
  const double *__restrict__ c = static_cast<const double *>(PS.src_c);
  for (int k = threadIdx.x; k < kTRin * kWin; k += kThreads) {
    const int rr = k / kWin, x = k % kWin;
    const int row = y0 - 1 + rr, g = x0 - 4 + x;
    double pv = 0.0, cv = 0.0;
    if (row <= K.ny - 1 && g >= 0 && g <= K.nx - 1) {
      const int si = min(max(g + PS.i_offset, 1), K.nx - 2);
      const int64_t o = (int64_t)row * K.pitch + si;
      pv = psi[o];
      cv = si >= K.nx - 2 ? K.cinf : c[o];
    }
    in.psi[rr][x] = pv;
    in.c[rr][x] = cv;
  }
}

template <bool TFC>
__global__ void __launch_bounds__(kThreads, 5)
    tile_kernel_f64(const __grid_constant__ StepCoef K, const __grid_constant__ Coef<double> F,
                    const __grid_constant__ StepScalars PS, const __grid_constant__ CUtensorMap tm_psi,
                    const __grid_constant__ CUtensorMap tm_c, const double *__restrict__ tab, const int tab_len,
                    double *__restrict__ psi_n, double *__restrict__ c_n, double *__restrict__ phi_n,
                    BlockPartial *partials, int *err, const __grid_constant__ FinalRed FR, const int wave) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  TileSmem64 &sm = *reinterpret_cast<TileSmem64 *>(smem_raw);
  // blockIdx.x walks the tile rows of one tile column, blockIdx.y the tile
  // columns, from the one holding column PS.i_front
  const int f = max(PS.i_front, 0) / kW;
  // tile t = blockIdx.y * gridDim.x + blockIdx.x of tile_of's order
  const int tr = (int)blockIdx.x, tc = front_first_block((int)blockIdx.y, f, (int)gridDim.y);
  const int x0 = kW * tc, y0 = 1 + kTR * tr;
  BlockPartial *part = partials ? partials + ((int64_t)tc * gridDim.x + tr) : nullptr;
  const FinalRed *FRp = partials && FR.counter ? &FR : nullptr;

  if (smem_u32(smem_raw) & 127u) {  // TMA destinations must be 128-byte aligned
    if (threadIdx.x == 0) atomicExch(err, 2);
    return;
  }
  // a pull-back step reads column clamp(i + i_offset, 1, nx - 2) for column i
  // (pull_back, fun.cu:1469-1492): no TMA box has that shape, so the CTA
  // gathers its tile (gather_pull_back) instead
  const bool pb = PS.pull_back != 0;
  if (threadIdx.x == 0) {
    mbar_init(&sm.full, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    if (!pb) {
      mbar_expect_tx(&sm.full, kTileBytes);
      tma_load_2d(&sm.in.psi[0][0], &tm_psi, &sm.full, x0 - 4, y0 - 1);
      tma_load_2d(&sm.in.c[0][0], &tm_c, &sm.full, x0 - 4, y0 - 1);
    }
    sm.st.liq = 0u;
    sm.st.sol = 0u;
    sm.p2.nlist = 0;
  }
  // the column table of this step (programmatic dependency on its kernel)
  asm volatile("griddepcontrol.wait;" ::: "memory");
  // the step's final reduction (a programmatic dependent) may be scheduled now
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const TileView V(K, F, PS, tab, tab_len, x0, y0, (int)threadIdx.x);
  const LaneCols LC = lane_cols<TFC>(V);
  if constexpr (TFC) {  // the row part of the cells' temperatures, once per tile row
    if (threadIdx.x < kTRin) tfc_row(K, y0 - 1 + (int)threadIdx.x, sm.st.tj[threadIdx.x], sm.st.ty[threadIdx.x]);
    if (threadIdx.x >= kTRin + 1 && threadIdx.x < kTRin + 3) {  // the halo columns x0-1, x0+kW
      const int side = (int)threadIdx.x - (kTRin + 1);
      tfc_col(K, PS.i_left_end_T, side ? x0 + kW : x0 - 1, sm.st.hiT[side], sm.st.hx[side]);
    }
    if (threadIdx.x == kTRin) {  // K + C0 about the temperature of the tile's centre
      int iT, jT;
      double x, y;
      tfc_col(K, PS.i_left_end_T, x0 + kW / 2, iT, x);
      tfc_row(K, y0 + kTR / 2, jT, y);
      sm.st.kp = kc_poly(K, tfc_T(K, PS.T_coarse, iT, x, jT, y));
    }
  }
  if (pb) gather_pull_back(K, PS, x0, y0, sm.in);
  __syncthreads();  // barrier initialised, flags cleared (and the TFC row table written)
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
      finish_tile(V, sm.p2, 0.0, 0, part, FRp, &sm.st.S[0][0], reinterpret_cast<int *>(&sm.st.mu[0][0]), 0);
      return;
    }
  }
  if (fix_beyond(V, sm.in)) __syncthreads();
  phase1<TFC>(V, LC, sm.in, sm.st);
  __syncthreads();
  // phase 1 done: pull the tile of the CTA that will start about one resident
  // wave later into L2, so its loads overlap the rest of this wave's arithmetic
  if (threadIdx.x == 0 && wave > 0 && !pb) {
    const unsigned nxt = blockIdx.y * gridDim.x + blockIdx.x + (unsigned)wave;
    if (nxt < gridDim.x * gridDim.y) {
      int pr, pc;
      tile_of((int)nxt, (int)gridDim.x, (int)gridDim.y, f, pr, pc);
      tma_prefetch_2d(&tm_psi, kW * pc - 4, kTR * pr);
      tma_prefetch_2d(&tm_c, kW * pc - 4, kTR * pr);
    }
  }
  const bool red = part != nullptr;
  double mass = 0.0;
  int itip = 0;
  double dn[kRowsPerWarp][2];
  const uint32_t needs_all = phase2(V, LC, sm.in, sm.st, sm.p2, dn, mass, red);
  __syncthreads();
  phase3<TFC>(V, sm.in, sm.p2, sm.st.S, red, itip);  // S is free after phase 2
  __syncthreads();
  phase4_rows(V, sm.in, sm.st.S, needs_all, dn, red, itip);
  store_tile(V, sm.in, psi_n, c_n, phi_n, 0);
  finish_tile(V, sm.p2, mass, itip, part, FRp, &sm.st.mu[0][0], reinterpret_cast<int *>(&sm.st.mu[8][0]), 0);
  // shared memory stays allocated until the copies have read it
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

// ---------------------------------------------------------------- persistent, warp roles
constexpr int kPipeThreads = 32 + 2 * kThreads;  // producer warp, phase-1 group, phases 2-4 group
enum { kBarP1 = 1, kBarP2 = 2 };                 // named barriers of the two groups

// AND of a predicate over the 128 threads of a phase group (named barrier)
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

__global__ void __launch_bounds__(kPipeThreads, 2)
    pipe_kernel_f64(const __grid_constant__ StepCoef K, const __grid_constant__ Coef<double> F,
                    const __grid_constant__ StepScalars PS, const __grid_constant__ CUtensorMap tm_psi,
                    const __grid_constant__ CUtensorMap tm_c, const double *__restrict__ tab, const int tab_len,
                    double *__restrict__ psi_n, double *__restrict__ c_n, double *__restrict__ phi_n,
                    BlockPartial *partials, int *err, const __grid_constant__ FinalRed FR, const int nrt,
                    const int ncb) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  PipeSmem64 &sm = *reinterpret_cast<PipeSmem64 *>(smem_raw);
  const int warp = threadIdx.x >> 5;
  const int ntiles = nrt * ncb;
  const int f = max(PS.i_front, 0) / kW;
  const FinalRed *FRp = partials && FR.counter ? &FR : nullptr;
  const uint32_t limit = PS.wait_limit ? PS.wait_limit : kWaitLimit;
  const bool poll = PS.wait_limit != 0;
  volatile int *abort = &sm.abort;
  if (smem_u32(smem_raw) & 127u) {  // TMA destinations must be 128-byte aligned
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
  // the column table of this step (programmatic dependency on its kernel)
  asm volatile("griddepcontrol.wait;" ::: "memory");
  // the step's final reduction (a programmatic dependent) may be scheduled now
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  __syncthreads();

  if (warp == 0) {
    // ---- producer: the input boxes of this CTA's tiles, kRing - 1 ahead of
    // phases 2-4 (a slot is refilled once its tile's bulk stores have read it)
    if ((threadIdx.x & 31) == 0) {
      int k = 0;
      for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++k) {
        const int s = k % kRing;
        if (k >= kRing && !pipe_wait(&sm.in_empty[s], ((k / kRing) - 1) & 1, abort, limit, err, poll)) break;
        int tr, tc;
        tile_of(t, nrt, ncb, f, tr, tc);
        mbar_expect_tx(&sm.in_full[s], kTileBytes);
        tma_load_2d(&sm.in[s].psi[0][0], &tm_psi, &sm.in_full[s], kW * tc - 4, kTR * tr);
        tma_load_2d(&sm.in[s].c[0][0], &tm_c, &sm.in_full[s], kW * tc - 4, kTR * tr);
      }
      // loads still in flight into this CTA's shared memory complete before
      // it exits (bounded)
      // (a load's slot is only refilled after its tile is done, so only the
      // last kRing loads can still be in flight)
      for (int q = max(k - kRing, 0); q < k; ++q)
        for (uint32_t tt = 0; tt < kWaitLimit && !mbar_try_wait(&sm.in_full[q % kRing], (q / kRing) & 1); ++tt) {
        }
    }
    return;
  }
  if (warp <= kWarps) {
    // ---- phase 1 of tile k into staging slot k % kStage
    const int gtid = (int)threadIdx.x - 32;
    int k = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++k) {
      const int s = k % kRing, q = k % kStage;
      // every thread waits (bounded); the group goes on only if all of them saw the phases
      bool ok = pipe_wait(&sm.in_full[s], (k / kRing) & 1, abort, limit, err, poll);
      if (ok && k >= kStage) ok = pipe_wait(&sm.st_empty[q], ((k / kStage) - 1) & 1, abort, limit, err, poll);
      if (!group_and(ok, kBarP1)) break;
      int tr, tc;
      tile_of(t, nrt, ncb, f, tr, tc);
      const TileView V(K, F, PS, tab, tab_len, kW * tc, 1 + kTR * tr, gtid);
      if (gtid == 0) {
        sm.st[q].liq = 0u;
        sm.st[q].sol = 0u;
      }
      fix_beyond(V, sm.in[s]);
      gsync(kBarP1);
      phase1<false>(V, lane_cols<false>(V), sm.in[s], sm.st[q]);
      gsync(kBarP1);
      if (gtid == 0) mbar_arrive(&sm.st_full[q]);
    }
    return;
  }
  // ---- phases 2-4 of tile k: fluxes, interface cells, stores
  const int gtid = (int)threadIdx.x - 32 - kThreads;
  int k = 0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++k) {
    const int s = k % kRing, q = k % kStage;
    if (!group_and(pipe_wait(&sm.st_full[q], (k / kStage) & 1, abort, limit, err, poll), kBarP2)) break;
    int tr, tc;
    tile_of(t, nrt, ncb, f, tr, tc);
    const TileView V(K, F, PS, tab, tab_len, kW * tc, 1 + kTR * tr, gtid);
    BlockPartial *part = partials ? partials + ((int64_t)tc * nrt + tr) : nullptr;
    const bool red = part != nullptr;
    if (gtid == 0) sm.p2.nlist = 0;
    gsync(kBarP2);
    double mass = 0.0;
    int itip = 0;
    double dn[kRowsPerWarp][2];
    const uint32_t needs_all = phase2(V, lane_cols<false>(V), sm.in[s], sm.st[q], sm.p2, dn, mass, red);
    gsync(kBarP2);
    phase3<false>(V, sm.in[s], sm.p2, sm.st[q].S, red, itip);  // S of the slot is free after phase 2
    gsync(kBarP2);
    phase4_rows(V, sm.in[s], sm.st[q].S, needs_all, dn, red, itip);
    const bool issued = store_tile(V, sm.in[s], psi_n, c_n, phi_n, kBarP2);
    finish_tile(V, sm.p2, mass, itip, part, FRp, &sm.st[q].mu[0][0], reinterpret_cast<int *>(&sm.st[q].mu[8][0]),
                kBarP2);
    // the slots are free once the bulk copies have read the input tile
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

int launch_step_f64_tma(const StepCoef &K, const Coef<double> &F, const StepScalars &P, const TmaMaps &tm,
                        double *psi_n, double *c_n, double *phi_n, BlockPartial *partials, int max_partials,
                        int *nparts_out, int *err, cudaStream_t st) {
  const int nj = K.ny - 2;
  if (K.nx % 2 || K.pitch != K.nx) return -1;  // rows are copied in 16-byte units
  const int nrt = (nj + kTR - 1) / kTR, ncb = (K.nx + kW - 1) / kW;
  if (ncb > 65535 || (int64_t)nrt * ncb > (1 << 30)) return -1;
  const int nparts = nrt * ncb;
  if (partials && nparts > max_partials) return -1;
  if (!tm.col_tab64 || tm.col_tab64_len < ncb * kW + kWin) return -1;
  // the coarse-grid temperature: per-cell groups, no column table (the
  // persistent pipeline has no TFC form and is not taken then)
  const bool tfc = K.tfc != 0;
  if (tfc && !P.T_coarse) return -1;
  const bool pipe = tm.pipeline != 0 && !tfc && !P.pull_back;
  const int which = pipe ? 1 : tfc ? 2 : 0;
  const size_t smem = pipe ? sizeof(PipeSmem64) : sizeof(TileSmem64);
  const void *kfn = pipe ? (const void *)pipe_kernel_f64
                         : tfc ? (const void *)tile_kernel_f64<true> : (const void *)tile_kernel_f64<false>;
  static std::atomic<unsigned long long> attr_done[3];
  if (!smem_limit_once(kfn, (int)smem, attr_done[which])) return -3;
  static std::atomic<int> resident_of[3][64];
  const int resident = resident_ctas(kfn, pipe ? kPipeThreads : kThreads, smem, resident_of[which]);
  if (resident <= 0) return -3;
  if (!tfc)
    column_table_kernel_f64<<<(tm.col_tab64_len + kTabBlock - 2) / (kTabBlock - 1), kTabBlock, 0, st>>>(
        K, P.d0, P.d1, tm.col_tab64_len, tm.col_tab64);
  cudaLaunchConfig_t cfg = {};
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  // a programmatic dependent of the table kernel only: the tile kernel issues
  // its TMA loads before griddepcontrol.wait, which is safe after the table
  // kernel (it writes no field) but not after the previous step's kernels,
  // so a TFC step (no table kernel) launches in plain stream order
  cfg.numAttrs = tfc ? 0 : 1;
  const double *tab = tm.col_tab64;
  // the final reduction is a programmatic dependent launch after the step
  FinalRed fr = tm.red;
  fr.partials = partials;
  fr.nparts = nparts;
  FinalRed none = fr;
  none.counter = nullptr;
  cudaError_t e;
  if (pipe) {
    // persistent: every CTA resident at once, each walking tiles b, b + G, ...
    cfg.gridDim = dim3((unsigned)std::min(resident, nparts));
    cfg.blockDim = dim3(kPipeThreads);
    e = cudaLaunchKernelEx(&cfg, pipe_kernel_f64, K, F, P, tm.psi, tm.c, tab, tm.col_tab64_len, psi_n, c_n, phi_n,
                           partials, err, none, nrt, ncb);
  } else {
    // column-major: consecutive CTAs share a column strip and its halo rows in L2
    cfg.gridDim = dim3(nrt, ncb);
    cfg.blockDim = dim3(kThreads);
    e = cudaLaunchKernelEx(&cfg, tfc ? tile_kernel_f64<true> : tile_kernel_f64<false>, K, F, P, tm.psi, tm.c, tab,
                           tm.col_tab64_len, psi_n, c_n, phi_n, partials, err, none, resident);
  }
  if (e != cudaSuccess) return -3;
  if (partials && (fr.mass_out || fr.itip_out) && launch_reduce_partials_dep(fr, st)) return -3;
  if (nparts_out) *nparts_out = nparts;
  return 0;
}

}  // namespace rs

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
// A CTA of 128 threads owns a tile of kTileRows output rows x 124 output
// columns (input 18 x 128, one TMA box per field; tiles start every 124
// columns, so every TMA x coordinate is 16-byte aligned).  Four adjacent
// columns per lane.
//   phase 1  per-cell S = q(psi) c (1-c) and mu'' (below) of all 18 input
//            rows into shared memory, plus per-row flags "every cell has
//            psi == -1" / "== +1";
//   phase 2  each warp writes 4 output rows: fluxes through the faces from
//            the shared S and mu'', the c update, stores; psi is copied
//            where the 3x3 phi neighbourhood is uniformly +-1 (then
//            phi_next = phi exactly) and the other cells are listed;
//   phase 3  the listed interface cells are updated one per thread
//            (phi_cell), so a tile's interface work is spread over the CTA.
// Arithmetic:
//   * mu = K(T) + C0(T) + mu'' with C0 = -D - (L0_BCC - L0_Liq)(1 - 2 cinf)/2
//     (D, K(T) as in rs_step.cu), so
//       mu'' = -(g+1) C0 - delta (L0_BCC + L0_Liq + g (L0_BCC - L0_Liq)) + RT lam,
//     which is small in the melt; K + C0 enters only through its FP64 column
//     differences dK;
//   * rows whose cells are all bulk liquid (psi = -1 exactly, |s| < 1/9) take
//     the short form: g(-1) = -1 and q(-1) = 1, so
//     mu'' = -2 L0_Liq delta + RT lam(delta) and S = c (1 - c);
//   * face weights use pair sums: the face (i, r+1/2) has
//     6 P_i + P_{i-1} + P_{i+1} with P_i = S(i,r) + S(i,r+1), and the face
//     (i+1/2, r) has 6 Q_r + Q_{r-1} + Q_{r+1} with Q_r = S(i,r) + S(i+1,r):
//     four times the 1.5 / 0.25 weights of rs_step.cu, the 4 folded into the
//     flux constant.
// Fields store psi and delta = c - cinf (include/rs_b200.h).
#include "rs_step_common.cuh"

namespace rs {
namespace {

constexpr int kIn = kTmaBoxW32;     // input columns of a tile
constexpr int kOut = kIn - 4;       // output columns of a tile
constexpr int kTR = kTileRows;      // output rows of a tile
constexpr int kTRin = kTmaBoxH;     // input rows of a tile
constexpr int kThreads = 128;
constexpr int kWarps = kThreads / 32;
constexpr int kRowsPerWarp = kTR / kWarps;
constexpr uint32_t kWaitLimit = 1u << 20;
constexpr unsigned FULL = 0xffffffffu;
static_assert(kIn == 32 * 4, "four columns per lane");
static_assert(kTR % kWarps == 0, "output rows are split evenly over the warps");
static_assert(kTRin <= 32, "row flags are 32-bit masks");

// column table arrays (kColTabFields of them, col_tab_len floats each)
enum { kTabRT = 0, kTabC0 = 1, kTabDK = 2, kTabAnb = 3, kTabAti = 4 };

struct alignas(128) TileSmem {
  float psi[kTRin][kIn];  // TMA destinations
  float d[kTRin][kIn];
  float S[kTRin][kIn];
  float mu[kTRin][kIn];
  uint16_t list[kTR * kOut];  // interface cells: row << 8 | column
  uint8_t pmask[kTRin][32];   // per lane: bits 0-3 psi <= -1, bits 4-7 psi >= 1 of its four cells
  uint32_t liq, sol;          // bit r: every cell of input row r has psi == -1 / +1
  int nlist;
  double part_mass[kWarps];
  int part_itip[kWarps];
  uint64_t full;
};

__device__ __forceinline__ float4 ld4(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ void st4(float *p, float a, float b, float c, float e) {
  *reinterpret_cast<float4 *>(p) = make_float4(a, b, c, e);
}
__device__ __forceinline__ float clamp1(float v) { return fminf(fmaxf(v, -1.f), 1.f); }

__global__ void __launch_bounds__(128) column_table_kernel(const StepCoef K, const double d0, const double d1,
                                                           const int len, float *__restrict__ tab) {
  // the tile kernel may start now; it waits for this grid before reading tab
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= len) return;
  auto kc = [&](int col, TTerms &tt, double &C0) {
    const int gi = min(col, K.nx - 1);
    const double T = (d0 + d1 * gi) * K.deltaT0 + K.Tmelt;  // get_delta, fun.cu:1610-1619
    tt = t_terms(T, K.RR);
    const double D = 0.5 * (tt.dGs - tt.dGl);
    C0 = -D - 0.5 * (kL0Bcc - kL0Liq) * (1.0 - 2.0 * K.cinf);
    return 0.5 * (tt.dGs + tt.dGl) + 0.5 * (kL0Bcc + kL0Liq) * (1.0 - 2.0 * K.cinf) + tt.RT * K.Lref + C0;
  };
  TTerms t0, t1;
  double c0, c1;
  const double k0 = kc(i, t0, c0), k1 = kc(i + 1, t1, c1);
  tab[kTabRT * len + i] = (float)t0.RT;
  tab[kTabC0 * len + i] = (float)c0;
  tab[kTabDK * len + i] = (float)(k1 - k0);  // (K + C0)(i+1) - (K + C0)(i)
  tab[kTabAnb * len + i] = (float)t0.A_nb;
  tab[kTabAti * len + i] = (float)t0.A_ti;
}

__global__ void __launch_bounds__(kThreads, 5)
    tile_kernel(const __grid_constant__ StepCoef K, const __grid_constant__ Coef<float> F,
                const __grid_constant__ StepScalars PS, const __grid_constant__ CUtensorMap tm_psi,
                const __grid_constant__ CUtensorMap tm_c, const float *__restrict__ tab, const int tab_len,
                float *__restrict__ psi_n, float *__restrict__ c_n, float *__restrict__ phi_n, BlockPartial *partials,
                int *err) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  TileSmem &sm = *reinterpret_cast<TileSmem *>(smem_raw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int x0 = kOut * blockIdx.y;  // first input column of the tile
  const int y0 = 1 + kTR * blockIdx.x;  // first output row; input rows y0-1 .. y0+kTR
  constexpr uint32_t kTileBytes = 2u * kTRin * kIn * sizeof(float);

  if (smem_u32(smem_raw) & 127u) {  // TMA destinations must be 128-byte aligned
    if (threadIdx.x == 0) atomicExch(err, 2);
    return;
  }
  if (threadIdx.x == 0) {
    mbar_init(&sm.full, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    mbar_expect_tx(&sm.full, kTileBytes);
    tma_load_2d(&sm.psi[0][0], &tm_psi, &sm.full, x0, y0 - 1);
    tma_load_2d(&sm.d[0][0], &tm_c, &sm.full, x0, y0 - 1);
    sm.liq = 0u;
    sm.sol = 0u;
    sm.nlist = 0;
  }

  const int col = 4 * lane;  // tile column of this lane's first cell
  const int gi = x0 + col;   // its global column
  uint32_t outm = 0;  // per cell: an output cell
#pragma unroll
  for (int q = 0; q < 4; ++q)
    if (col + q >= 1 && col + q <= kOut && gi + q <= K.nx - 2) outm |= 1u << q;
  // interior tiles: no ghost column, every lane's cells are outputs except
  // cell 0 of lane 0 and cells 1..3 of lane 31
  const bool interior = x0 >= 4 && x0 + kOut <= K.nx - 3;
  const float two_cinf = F.cinf + F.cinf;
  const float cflux4 = 0.25f * F.cflux;
  const float floor_d = F.c_floor - F.cinf;
  constexpr float KL = (float)(-2.0 * kL0Liq);
  constexpr float L0sum = (float)(kL0Bcc + kL0Liq);
  constexpr float L0half = (float)(0.5 * (kL0Bcc - kL0Liq));
  // delta range of the series form: s = delta / (A + B delta) with
  // A = 2 cinf (1 - cinf), B = 1 - 2 cinf, so |s| < 1/9 for
  // -A/(9+B) < delta < A/(9-B) (taken 0.1 % inside)
  const float sA = 2.f * F.cinf * (1.f - F.cinf), sB = 1.f - 2.f * F.cinf;
  const float d_hi = 0.999f * sA / (9.f - sB), d_lo = -0.999f * sA / (9.f + sB);
  constexpr uint32_t kMinus1 = 0xBF800000u, kPlus1 = 0x3F800000u;

  // the column table of this step (programmatic dependency on its kernel)
  asm volatile("griddepcontrol.wait;" ::: "memory");
  const float4 RTv = ld4(tab + kTabRT * tab_len + gi), C0v = ld4(tab + kTabC0 * tab_len + gi);
  const float RTa[4] = {RTv.x, RTv.y, RTv.z, RTv.w}, C0a[4] = {C0v.x, C0v.y, C0v.z, C0v.w};
  __syncthreads();  // barrier initialised, flags cleared
  {
    uint32_t tries = 0;
    while (!mbar_try_wait(&sm.full, 0)) {
      if (++tries >= kWaitLimit) {
        atomicExch(err, 1);
        break;
      }
    }
  }

  // columns beyond the array (right-most tiles; zero-filled by TMA) become
  // bulk melt, so they never force the general path; no output reads them
  if (x0 + kIn > K.nx) {
    for (int k = threadIdx.x; k < kTRin * kIn; k += kThreads) {
      const int rr = k / kIn, x = k % kIn;
      if (x0 + x >= K.nx) {
        sm.psi[rr][x] = -1.f;
        sm.d[rr][x] = 0.f;
      }
    }
    __syncthreads();
  }

  // ---- phase 1: per-cell terms; warp w takes input rows w, w+4, ...
#pragma unroll 1
  for (int rr = warp; rr < kTRin; rr += kWarps) {
    const int y = y0 - 1 + rr;
    if (y > K.ny - 1) {  // beyond the array (last tile): never read by an output
      st4(&sm.S[rr][col], 0.f, 0.f, 0.f, 0.f);
      st4(&sm.mu[rr][col], 0.f, 0.f, 0.f, 0.f);
      sm.pmask[rr][lane] = 0xFFu;
      if (lane == 0) {
        atomicOr(&sm.liq, 1u << rr);
        atomicOr(&sm.sol, 1u << rr);
      }
      continue;
    }
    const float4 pv4 = ld4(&sm.psi[rr][col]), dv4 = ld4(&sm.d[rr][col]);
    const float pv[4] = {pv4.x, pv4.y, pv4.z, pv4.w}, dv[4] = {dv4.x, dv4.y, dv4.z, dv4.w};
    float cc[4], om[4], Sv[4], mv[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      cc[q] = F.cinf + dv[q];
      om[q] = 1.f - cc[q];
    }
    // the row is bulk melt when every psi is exactly -1 and every delta is in
    // the series range (bit tests on psi, min/max on delta)
    const uint32_t b0 = __float_as_uint(pv[0]), b1 = __float_as_uint(pv[1]), b2 = __float_as_uint(pv[2]),
                   b3 = __float_as_uint(pv[3]);
    const uint32_t band = b0 & b1 & b2 & b3, bor = b0 | b1 | b2 | b3;
    const float dmx = fmaxf(fmaxf(dv[0], dv[1]), fmaxf(dv[2], dv[3]));
    const float dmn = fminf(fminf(dv[0], dv[1]), fminf(dv[2], dv[3]));
    const bool liq4 = band == kMinus1 && bor == kMinus1;
    uint32_t code;
    if (__all_sync(FULL, liq4 && dmx < d_hi && dmn > d_lo)) {
      code = 5u;
      sm.pmask[rr][lane] = 0x0Fu;
      // lam = 2 atanh(s) by its odd series
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const float sv = __fdividef(dv[q], fmaf(two_cinf, om[q], dv[q]));
        const float s2 = sv * sv;
        float p = fmaf(s2, 1.f / 9.f, 1.f / 7.f);
        p = fmaf(s2, p, 1.f / 5.f);
        p = fmaf(s2, p, 1.f / 3.f);
        const float lh = fmaf(sv * s2, p, sv);  // atanh(s)
        Sv[q] = cc[q] * om[q];
        mv[q] = fmaf(RTa[q] + RTa[q], lh, dv[q] * KL);
      }
    } else {
      const bool sol4 = band == kPlus1 && bor == kPlus1;
      code = (__all_sync(FULL, liq4) ? 1u : 0u) | (__all_sync(FULL, sol4) ? 2u : 0u);
      uint32_t L = 0u, Sm = 0u;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (pv[q] <= -1.f) L |= 1u << q;
        if (pv[q] >= 1.f) Sm |= 1u << q;
      }
      sm.pmask[rr][lane] = (uint8_t)(L | (Sm << 4));
      // general form (fun.cu:1424-1452)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const float a = 1.f - pv[q];
        Sv[q] = (0.5f * F.AA * a - 0.25f * (F.AA - 1.f) * (a * a)) * cc[q] * om[q];
        const float p2 = pv[q] * pv[q];
        const float g = pv[q] * (1.875f + p2 * (-1.25f + 0.375f * p2));
        const float lam = Tr<float>::lam(cc[q], om[q], dv[q], F.cinf, F.Lref);
        mv[q] = -(g + 1.f) * C0a[q] - dv[q] * fmaf(2.f * L0half, g, L0sum) + RTa[q] * lam;
      }
    }
    st4(&sm.S[rr][col], Sv[0], Sv[1], Sv[2], Sv[3]);
    st4(&sm.mu[rr][col], mv[0], mv[1], mv[2], mv[3]);
    if (lane == 0) {
      if (code & 1u) atomicOr(&sm.liq, 1u << rr);
      if (code & 2u) atomicOr(&sm.sol, 1u << rr);
    }
  }
  const float4 dKv = ld4(tab + kTabDK * tab_len + gi);
  const float dKa[4] = {dKv.x, dKv.y, dKv.z, dKv.w};
  __syncthreads();

  // ---- phase 2: warp w writes output rows 1 + 4w .. 4 + 4w of the tile
  const uint32_t liq = sm.liq, sol = sm.sol;
  const bool red = partials != nullptr;
  double mass = 0.0;
  int itip = 0;
  struct Row {
    float s[4], m[4], s4, m4, q[4];
  };
  auto load_row = [&](int rr, Row &R) {
    const float4 s = ld4(&sm.S[rr][col]), m = ld4(&sm.mu[rr][col]);
    R.s[0] = s.x; R.s[1] = s.y; R.s[2] = s.z; R.s[3] = s.w;
    R.m[0] = m.x; R.m[1] = m.y; R.m[2] = m.z; R.m[3] = m.w;
    R.s4 = __shfl_down_sync(FULL, s.x, 1);  // column 4 (next lane's first cell)
    R.m4 = __shfl_down_sync(FULL, m.x, 1);
    R.q[0] = R.s[0] + R.s[1];
    R.q[1] = R.s[1] + R.s[2];
    R.q[2] = R.s[2] + R.s[3];
    R.q[3] = R.s[3] + R.s4;
  };
  // fluxes through the faces between rows A and B = A+1 (compute_c_CALPHAD F01/F0m)
  auto vface = [&](const Row &A, const Row &B, float jv[4]) {
    float pp[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) pp[q] = A.s[q] + B.s[q];
    const float pl = __shfl_up_sync(FULL, pp[3], 1), pr = __shfl_down_sync(FULL, pp[0], 1);
#pragma unroll
    for (int q = 0; q < 4; ++q)
      jv[q] = fmaf(6.f, pp[q], (q ? pp[q - 1] : pl) + (q < 3 ? pp[q + 1] : pr)) * (B.m[q] - A.m[q]);
  };
  auto put = [&](float *f, int64_t o, float a, float b, float c, float e) {
    *reinterpret_cast<float4 *>(f + o) = make_float4(a, b, c, e);
  };

  const int rbase = 1 + kRowsPerWarp * warp;
  Row ra, rb, rc;
  float jv_lo[4], jv_hi[4];
  load_row(rbase - 1, ra);
  load_row(rbase, rb);
  vface(ra, rb, jv_lo);
#pragma unroll
  for (int j = 0; j < kRowsPerWarp; ++j) {
    const int rr = rbase + j;  // tile input row of the output row
    load_row(rr + 1, rc);
    vface(rb, rc, jv_hi);
    const int r = y0 - 1 + rr;  // global row
    if (r <= K.ny - 2) {
      // fluxes through the faces (i+1/2, r)
      const float mnext[4] = {rb.m[1], rb.m[2], rb.m[3], rb.m4};
      float jh[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) jh[q] = fmaf(6.f, rb.q[q], ra.q[q] + rc.q[q]) * (mnext[q] - rb.m[q] + dKa[q]);
      const float jl = __shfl_up_sync(FULL, jh[3], 1);
      const float4 dv4 = ld4(&sm.d[rr][col]), pv4 = ld4(&sm.psi[rr][col]);
      const float dv[4] = {dv4.x, dv4.y, dv4.z, dv4.w};
      float dn[4], po[4] = {pv4.x, pv4.y, pv4.z, pv4.w};
#pragma unroll
      for (int q = 0; q < 4; ++q)
        dn[q] = fmaxf(fmaf(cflux4, (jh[q] - (q ? jh[q - 1] : jl)) + (jv_hi[q] - jv_lo[q]), dv[q]), floor_d);
      // phi: copied where the 3x3 neighbourhood is uniformly +-1, listed otherwise
      uint32_t needs = 0u;
      const uint32_t w3 = 7u << (rr - 1);
      const bool uni_liq = (liq & w3) == w3;
      if (!uni_liq && (sol & w3) != w3) {
        // phi masks of rows rr-1 .. rr+1, this lane's cells with one cell of
        // each neighbouring lane
        const uint32_t pk = (uint32_t)sm.pmask[rr - 1][lane] | ((uint32_t)sm.pmask[rr][lane] << 8) |
                            ((uint32_t)sm.pmask[rr + 1][lane] << 16);
        const uint32_t lf = __shfl_up_sync(FULL, pk, 1), rt = __shfl_down_sync(FULL, pk, 1);
        uint32_t Lv = 0x3Fu, Sv = 0x3Fu;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const uint32_t L = (pk >> (8 * k)) & 0xFu, S = (pk >> (8 * k + 4)) & 0xFu;
          Lv &= (L << 1) | ((lf >> (8 * k + 3)) & 1u) | (((rt >> (8 * k)) & 1u) << 5);
          Sv &= (S << 1) | ((lf >> (8 * k + 7)) & 1u) | (((rt >> (8 * k + 4)) & 1u) << 5);
        }
        needs = ~((Lv & (Lv >> 1) & (Lv >> 2)) | (Sv & (Sv >> 1) & (Sv >> 2))) & outm;
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
        for (int q = 0; q < 4; ++q) {
          if ((needs >> q) & 1u) sm.list[off++] = (uint16_t)((rr << 8) | (col + q));
          po[q] = clamp1(po[q]);  // placeholder; the listed cells are rewritten in phase 3
        }
      }
      // stores, ghost copies (compute_boundary_individual, fun.cu:1220-1230)
      auto store_row = [&](int rowi) {
        const int64_t o = (int64_t)rowi * K.pitch + gi;
        if (interior) {
          if (lane != 0 && lane != 31) {
            put(psi_n, o, po[0], po[1], po[2], po[3]);
            put(c_n, o, dn[0], dn[1], dn[2], dn[3]);
            if (phi_n) put(phi_n, o, clamp1(po[0]), clamp1(po[1]), clamp1(po[2]), clamp1(po[3]));
          } else {
            // lane 0: cell 1 alone, cells 2-3 as a pair; lane 31: cell 0
            const int64_t o1 = lane == 0 ? o + 1 : o;
            const float p1 = lane == 0 ? po[1] : po[0], c1 = lane == 0 ? dn[1] : dn[0];
            psi_n[o1] = p1;
            c_n[o1] = c1;
            if (phi_n) phi_n[o1] = clamp1(p1);
            if (lane == 0) {
              *reinterpret_cast<float2 *>(psi_n + o + 2) = make_float2(po[2], po[3]);
              *reinterpret_cast<float2 *>(c_n + o + 2) = make_float2(dn[2], dn[3]);
              if (phi_n) *reinterpret_cast<float2 *>(phi_n + o + 2) = make_float2(clamp1(po[2]), clamp1(po[3]));
            }
          }
        } else if ((outm & 0xEu) == 0xEu && ((outm & 1u) || gi == 0)) {
          // cells 1..3 are outputs; cell 0 is an output or the ghost column 0
          const float p0 = (outm & 1u) ? po[0] : po[1], c0 = (outm & 1u) ? dn[0] : dn[1];
          put(psi_n, o, p0, po[1], po[2], po[3]);
          put(c_n, o, c0, dn[1], dn[2], dn[3]);
          if (phi_n) put(phi_n, o, clamp1(p0), clamp1(po[1]), clamp1(po[2]), clamp1(po[3]));
          if (gi + 3 == K.nx - 2) {
            psi_n[o + 4] = po[3];
            c_n[o + 4] = dn[3];
            if (phi_n) phi_n[o + 4] = clamp1(po[3]);
          }
        } else {
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            if (!((outm >> q) & 1u)) continue;
            psi_n[o + q] = po[q];
            c_n[o + q] = dn[q];
            if (phi_n) phi_n[o + q] = clamp1(po[q]);
            if (gi + q == K.nx - 2) {
              psi_n[o + q + 1] = po[q];
              c_n[o + q + 1] = dn[q];
              if (phi_n) phi_n[o + q + 1] = clamp1(po[q]);
            }
          }
        }
      };
      store_row(r);
      if (r == K.jmin) store_row(0);
      if (r == K.jmax) store_row(K.ny - 1);
      if (red) {
#pragma unroll
        for (int q = 0; q < 4; ++q)
          if ((outm >> q) & 1u) mass += (double)dn[q];
        if (!uni_liq) {
#pragma unroll
          for (int q = 0; q < 4; ++q)
            if (((outm & ~needs) >> q) & 1u && po[q] > 0.f) itip = max(itip, gi + q == K.nx - 2 ? K.nx - 1 : gi + q);
        }
      }
    }
    ra = rb;
    rb = rc;
#pragma unroll
    for (int q = 0; q < 4; ++q) jv_lo[q] = jv_hi[q];
  }
  __syncthreads();

  // ---- phase 3: interface cells, one per thread (compute_phi, fun.cu:1143-1218)
  const int nlist = sm.nlist;
  for (int idx = threadIdx.x; idx < nlist; idx += kThreads) {
    const uint32_t e = sm.list[idx];
    const int rr = (int)(e >> 8), x = (int)(e & 0xFFu);
    const int r = y0 - 1 + rr, g = x0 + x;
    const float res = phi_cell<float>(
        &F, clamp1(sm.psi[rr][x]), clamp1(sm.psi[rr][x + 1]), clamp1(sm.psi[rr][x - 1]), clamp1(sm.psi[rr + 1][x]),
        clamp1(sm.psi[rr - 1][x]), clamp1(sm.psi[rr + 1][x + 1]), clamp1(sm.psi[rr + 1][x - 1]),
        clamp1(sm.psi[rr - 1][x + 1]), clamp1(sm.psi[rr - 1][x - 1]), F.cinf + sm.d[rr][x],
        tab[kTabAnb * tab_len + g], tab[kTabAti * tab_len + g], PS.step, (int64_t)r * K.nx + g, K.seed_lo,
        K.seed_hi);
    const float ph = clamp1(res);
    const int gx = g == 1 ? 0 : (g == K.nx - 2 ? K.nx - 1 : -1);
    auto put1 = [&](int row) {
      const int64_t o = (int64_t)row * K.pitch;
      psi_n[o + g] = res;
      if (phi_n) phi_n[o + g] = ph;
      if (gx >= 0) {
        psi_n[o + gx] = res;
        if (phi_n) phi_n[o + gx] = ph;
      }
    };
    put1(r);
    if (r == K.jmin) put1(0);
    if (r == K.jmax) put1(K.ny - 1);
    if (red && res > 0.f) itip = max(itip, g == K.nx - 2 ? K.nx - 1 : g);
  }

  if (partials) {
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
      partials[(int64_t)blockIdx.y * gridDim.x + blockIdx.x] = b;
    }
  }
}

}  // namespace

int launch_step_f32_tma(const StepCoef &K, const Coef<float> &F, const StepScalars &P, const TmaMaps &tm,
                        float *psi_n, float *c_n, float *phi_n, BlockPartial *partials, int max_partials,
                        int *nparts_out, int *err, cudaStream_t st) {
  const int ni = K.nx - 2, nj = K.ny - 2;
  // column-major: consecutive CTAs share a column strip and its halo rows in L2
  const dim3 grid((nj + kTR - 1) / kTR, (ni + kOut - 1) / kOut), block(kThreads);
  const int nparts = grid.x * grid.y;
  if (partials && nparts > max_partials) return -1;
  if (tm.col_tab_len < (int)grid.y * kOut + kIn) return -1;
  const size_t smem = sizeof(TileSmem);
  static bool attr_done = false;
  if (!attr_done) {
    if (cudaFuncSetAttribute(tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
      return -3;
    attr_done = true;
  }
  column_table_kernel<<<(tm.col_tab_len + 127) / 128, 128, 0, st>>>(K, P.d0, P.d1, tm.col_tab_len, tm.col_tab);
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
  if (cudaLaunchKernelEx(&cfg, tile_kernel, K, F, P, tm.psi, tm.c, tab, tm.col_tab_len, psi_n, c_n, phi_n, partials,
                         err) != cudaSuccess)
    return -3;
  if (nparts_out) *nparts_out = nparts;
  return 0;
}

}  // namespace rs

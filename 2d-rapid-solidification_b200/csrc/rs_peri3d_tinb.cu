// rs_peri3d_tinb.cu — the 3D three-phase step with the Ti-Nb CALPHAD free
// energy (rs3_params.energy = 1; include/rs_b200.h states the model).
//
// The step of rs_peri3d.cu (TiAg.cu's three-phase structure, one fused TMA
// z march per step) with TiAg's linear grand potentials replaced by the
// CALPHAD energy of the 2D model:
//   mu = g1 Glc(T, c) + (1 - g1) Gsc(T, c)                (fun.cu:1443-1452, 1700-1720)
//   dG = Gl - Gs = (1-c) A_Nb + c A_Ti + c (1-c) (L0_Liq - L0_BCC)
//        (fun.cu:1192-1193; the ideal-mixing terms of fun.cu:1671-1698 cancel)
// with dG driving phase 1 against both solids (two BCC grains), and the
// solute flux with the face mobility (S + S') / 2, S = q(phi1) c (1 - c)
// (fun.cu:1424-1464).  The per-plane CALPHAD groups of a step (the frozen T
// depends on z only) come from tinb_table_kernel, launched before the step:
// T, RT, dGl, dGs, A_Nb, A_Ti, C0 and dK, the plane-to-plane difference of
// the melt's mu.
//
// FP64 carries mu itself.  FP32 sets hold delta = c - c_ref and the kernel
// carries mu'' = mu - mu_ref(T), mu relative to the melt of composition c_ref
// at the plane's T, in the form of the 2D FP32 tile kernel (rs_step_f32.cu):
//   mu'' = -(g+1) C0 - delta (L0_BCC + L0_Liq + g (L0_BCC - L0_Liq)) + RT lam,
//   g = 1 - 2 g1,  C0 = -(dGs - dGl)/2 - (L0_BCC - L0_Liq)(1 - 2 c_ref)/2,
//   lam = log(c/(1-c)) - log(c_ref/(1-c_ref)),
// so that differences within a plane are those of mu and a z face adds dK.
// SURR (FP32): the learned surrogate (rs_surrogate.cuh) gives mu'' and dG of
// every cell that is not bulk melt (phi1 = 1, phi2 = 0 exactly); bulk melt
// keeps the exact form, out-of-box cells and one cell in 1024 per step of
// the others (audit) are evaluated exactly.
// Algorithmic bytes per cell-step: 3 fields read + 3 written.
#include <cuda.h>

#include "rs_f32x2.cuh"
#include "rs_peri3d_common.cuh"
#include "rs_surrogate.cuh"

namespace rs {
namespace {

constexpr int kTW = 8;  // doubles per plane in the table
enum { kTT = 0, kTRT, kTdGl, kTdGs, kTAnb, kTAti, kTC0, kTdK };

// the per-plane CALPHAD groups of one step: one thread per plane z of 0..nz-1
__global__ void tinb_table_kernel(const K3<double> k, const int64_t step, double *__restrict__ tab) {
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= k.nz) return;
  const double lref = log(k.c_ref / (1.0 - k.c_ref));
  auto terms = [&](int zz, double &T) {
    T = k.T_ref + k.G_T * ((double)zz - k.z_T - k.V_T * (double)step);
    return t_terms(T, k.RR);
  };
  double T0, T1;
  const TTerms t0 = terms(z, T0), t1 = terms(z + 1, T1);
  // mu of the melt c_ref at the plane's T (g1 = 1: Glc, fun.cu:1700-1709)
  const double m0 = t0.dGl + kL0Liq * (1.0 - 2.0 * k.c_ref) + t0.RT * lref;
  const double m1 = t1.dGl + kL0Liq * (1.0 - 2.0 * k.c_ref) + t1.RT * lref;
  double *e = tab + (int64_t)kTW * z;
  e[kTT] = T0;
  e[kTRT] = t0.RT;
  e[kTdGl] = t0.dGl;
  e[kTdGs] = t0.dGs;
  e[kTAnb] = t0.A_nb;
  e[kTAti] = t0.A_ti;
  e[kTC0] = -0.5 * (t0.dGs - t0.dGl) - 0.5 * (kL0Bcc - kL0Liq) * (1.0 - 2.0 * k.c_ref);
  e[kTdK] = m1 - m0;
}

template <typename R>
struct PlaneT {  // a plane's table entries in the working precision
  R RT, dGl, dGs, Anb, Ati, C0, dK;
  float T;
};

template <typename R>
__device__ __forceinline__ PlaneT<R> plane_terms(const double *tab, int z) {
  const double *e = tab + (int64_t)kTW * z;
  PlaneT<R> t;
  t.T = (float)e[kTT];
  t.RT = (R)e[kTRT];
  t.dGl = (R)e[kTdGl];
  t.dGs = (R)e[kTdGs];
  t.Anb = (R)e[kTAnb];
  t.Ati = (R)e[kTAti];
  t.C0 = (R)e[kTC0];
  t.dK = (R)e[kTdK];
  return t;
}

// mu of a cell, FP64 (the reference's operation order: Glc and Gsc, then the
// weighted sum of fun.cu:1443-1452 with 0.5 (1 + g) = 1 - g1)
__device__ __forceinline__ double mu_cell(const PlaneT<double> &t, double p1, double p2, double c) {
  const double p3 = 1.0 - p1 - p2;
  const double g1 = g3(p1, p2, p3), gS = 1.0 - g1;
  const double omc = 1.0 - c;
  const double lp = (c > 1.e-8 && omc > 1.e-8) ? t.RT * log(c / omc) : 0.0;
  const double Glc = t.dGl + kL0Liq * (1.0 - 2.0 * c) + lp;
  const double Gsc = t.dGs + kL0Bcc * (1.0 - 2.0 * c) + lp;
  return gS * Gsc + g1 * Glc;
}

// mu'' of a cell, FP32 (d = c - c_ref); lref = log(c_ref/(1-c_ref))
__device__ __forceinline__ float mu_cell(const PlaneT<float> &t, float p1, float p2, float d, float c_ref,
                                         float lref) {
  const float p3 = 1.f - p1 - p2;
  const float g = 1.f - 2.f * g3(p1, p2, p3);
  const float c = c_ref + d, omc = 1.f - c;
  const float lam = (c > 1.e-8f && omc > 1.e-8f) ? lam_fast(d, omc, c_ref + c_ref) : -lref;
  return -(g + 1.f) * t.C0 - d * fmaf((float)(kL0Bcc - kL0Liq), g, (float)(kL0Bcc + kL0Liq)) + t.RT * lam;
}

template <typename R>
__device__ __forceinline__ R dG_cell(const PlaneT<R> &t, R c) {
  return (R(1) - c) * t.Anb + c * t.Ati + c * (R(1) - c) * (R)(kL0Liq - kL0Bcc);
}

// one cell per lane through the network: two m16 passes (lanes 0-15, 16-31);
// x: this lane's scaled inputs, out: its scaled outputs
__device__ __forceinline__ void surr_cells32(const SurrConst &SC, const float x[3], float out[2]) {
  constexpr unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31, g = lane >> 2;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    float in0[3], in1[3], o0[2], o1[2];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      in0[i] = __shfl_sync(FULL, x[i], 16 * h + g);
      in1[i] = __shfl_sync(FULL, x[i], 16 * h + g + 8);
    }
    surr_tile16(SC, in0, in1, o0, o1);
    // cell j of this pass has its outputs in lane 4 (j mod 8), slot j / 8
    const int j = lane - 16 * h, src = 4 * (j & 7);
    const float a0 = __shfl_sync(FULL, o0[0], src), a1 = __shfl_sync(FULL, o0[1], src);
    const float b0 = __shfl_sync(FULL, o1[0], src), b1 = __shfl_sync(FULL, o1[1], src);
    if (j >= 0 && j < 16) {
      out[0] = j < 8 ? a0 : b0;
      out[1] = j < 8 ? a1 : b1;
    }
  }
}

template <typename R, bool SURR>
struct TSmem {
  alignas(128) R in[kP3Slots][3][P3Cfg<R>::kPlaneAl];  // [slot][field][row][col]
  alignas(16) R mu[kP3MuSlots][P3Cfg<R>::kPlane];      // mu (FP64) or mu'' (FP32)
  alignas(16) R S[kP3MuSlots][P3Cfg<R>::kPlane];       // face-mobility terms
  // surrogate dG of the output cells of three planes: plane z+1 is written
  // (before the plane barrier) while slower threads still read plane z-1
  alignas(16) float dG[3][SURR ? P3Cfg<R>::BX * kP3BY : 1];
  uint64_t full[kP3Slots];
  int melt[8];  // per plane (q mod 8): the box is pure melt inside the array (p3_melt_cell)
};

// SD: solid diffusivities Da or Db non-zero
template <typename R, bool SD, bool SURR>
__global__ void __launch_bounds__(kP3Threads, 2)
    tinb_kernel(const __grid_constant__ K3<R> k, const __grid_constant__ CUtensorMap m1,
                const __grid_constant__ CUtensorMap m2, const __grid_constant__ CUtensorMap mc,
                R *__restrict__ o1, R *__restrict__ o2, R *__restrict__ oc, const int64_t step, int *err,
                const __grid_constant__ SurrArgs SA) {
  static_assert(!SURR || sizeof(R) == 4, "the surrogate serves the FP32 step");
  using C = P3Cfg<R>;
  constexpr bool kF32 = sizeof(R) == 4;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  TSmem<R, SURR> &sm = *reinterpret_cast<TSmem<R, SURR> *>(smem_raw);
  const int tid = threadIdx.x;
  const int xb = C::BX * blockIdx.x;   // first box column (array x); outputs xb+1 .. xb+BX
  const int yb = kP3BY * blockIdx.y;   // first box row (array y); outputs yb+1 .. yb+BY
  const int zo0 = 1 + k.z_chunk * blockIdx.z;
  const int zo1 = min(zo0 + k.z_chunk, k.nz - 1);
  if (zo0 >= zo1) return;
  const int zin0 = zo0 - 1, zin1 = zo1;
  constexpr uint32_t kBytes = 3u * C::kPlane * sizeof(R);
  if (smem_u32(smem_raw) & 127u) {
    if (tid == 0) atomicExch(err, 2);
    return;
  }
  static_assert((C::kPlaneAl * sizeof(R)) % 128 == 0, "TMA destinations 128-byte aligned");
  auto issue = [&](int z) {
    const int q = z - zin0, s = q % kP3Slots;
    mbar_expect_tx(&sm.full[s], kBytes);
    tma_load_3d(&sm.in[s][0][0], &m1, &sm.full[s], xb, yb, z);
    tma_load_3d(&sm.in[s][1][0], &m2, &sm.full[s], xb, yb, z);
    tma_load_3d(&sm.in[s][2][0], &mc, &sm.full[s], xb, yb, z);
  };
  if (tid == 0) {
    for (int s = 0; s < kP3Slots; ++s) mbar_init(&sm.full[s], 1);
    for (int s = 0; s < 8; ++s) sm.melt[s] = 1;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    for (int z = zin0; z <= min(zin1, zin0 + kP3Slots - 1); ++z) issue(z);
  }
  __syncthreads();
  int issued = min(zin1, zin0 + kP3Slots - 1);
  const float c_ref = (float)k.c_ref;
  const float lref = (float)log(k.c_ref / (1.0 - k.c_ref));
  const int64_t plane = (int64_t)k.nx * k.ny;

  // mu (or mu'') and S of plane z into its slots; the surrogate's dG too
  auto mu_plane = [&](int z) {
    const int q = z - zin0, s = q % kP3Slots;
    const bool got = p3_wait<R>(&sm.full[s], (uint32_t)((q / kP3Slots) & 1), err);
    R *mu = sm.mu[q % kP3MuSlots], *Sv = sm.S[q % kP3MuSlots];
    const R *f1 = sm.in[s][0], *f2 = sm.in[s][1], *fc = sm.in[s][2];
    // a ghost plane images its neighbour, T included (mu of the ghost equals
    // the imaged cell's, as TiAg.cu's boundaryMu leaves it)
    const PlaneT<R> t = plane_terms<R>(k.tab, z == 0 ? 1 : (z == k.nz - 1 ? k.nz - 2 : z));
    if (!got) return false;
    bool all_melt = true;  // this thread's box elements (p3_melt_cell)
    if constexpr (!SURR) {
      for (int e = tid; e < C::kPlane; e += kP3Threads) {
        const R p1 = f1[e], p2 = f2[e], cv = fc[e];
        all_melt = all_melt && p3_melt_cell(k, p1, p2, xb + e % C::BXin, yb + e / C::BXin);
        R c, m;
        if constexpr (kF32) {
          c = c_ref + cv;
          m = mu_cell(t, p1, p2, cv, c_ref, lref);
        } else {
          c = cv;
          m = mu_cell(t, p1, p2, cv);
        }
        R q1 = p1 * (k.AA - k.AA1 * p1);
        if constexpr (SD) q1 += k.Da2 * p2 + k.Db2 * (R(1) - p1 - p2);
        mu[e] = m;
        Sv[e] = q1 * (c * (R(1) - c));
      }
    } else {
      constexpr unsigned FULL = 0xffffffffu;
      const int warp = tid >> 5, lane = tid & 31;
      float *dg = sm.dG[q % 3];
      const bool T_in = t.T >= SA.T_lo && t.T <= SA.T_hi;
      const float xT = (t.T - SA.T_mid) * SA.T_ihalf;
      for (int base = 32 * warp; base < C::kPlane; base += kP3Threads) {
        const int e = base + lane;
        const bool in = e < C::kPlane;
        const float p1 = in ? f1[e] : 1.f, p2 = in ? f2[e] : 0.f, d = in ? fc[e] : 0.f;
        const float c = c_ref + d;
        const bool melt = p1 == 1.f && p2 == 0.f;
        const bool inbox = T_in && c >= SA.c_lo && c <= SA.c_hi;
        // array cell of box element e (its audit key)
        const int64_t cell = (int64_t)z * plane + (int64_t)(yb + e / C::BXin) * k.nx + (xb + e % C::BXin);
        const bool net = in && !melt && inbox;
        const bool audit = net && surr_audit_cell(step, cell);
        float m = 0.f, dGv = 0.f;
        if (!net || audit) {
          m = mu_cell(t, p1, p2, d, c_ref, lref);
          dGv = dG_cell(t, c);
        }
        if (__any_sync(FULL, net)) {
          const SurrConst SC = surr_load(SA, lane);
          const float x[3] = {xT, (c - SA.c_mid) * SA.c_ihalf, 1.f - 2.f * g3(p1, p2, 1.f - p1 - p2)};
          float o[2] = {0.f, 0.f};
          surr_cells32(SC, x, o);
          const float m_net = fmaf(o[0], SA.y_scale[0], SA.y_mean[0]);
          const float dG_net = fmaf(o[1], SA.y_scale[1], SA.y_mean[1]);
          if (audit) {
            atomicMax(&SA.audit[0], (unsigned long long)__float_as_uint(fabsf(m_net - m)));
            atomicMax(&SA.audit[1], (unsigned long long)__float_as_uint(fabsf(dG_net - dGv)));
            atomicAdd(&SA.audit[3], 1ull);
          } else if (net) {
            m = m_net;
            dGv = dG_net;
          }
        }
        if (in && !melt && !inbox) atomicAdd(&SA.audit[2], 1ull);
        if (in) all_melt = all_melt && p3_melt_cell(k, p1, p2, xb + e % C::BXin, yb + e / C::BXin);
        if (in) {
          const float q1 = p1 * (k.AA - k.AA1 * p1) + (SD ? k.Da2 * p2 + k.Db2 * (1.f - p1 - p2) : 0.f);
          mu[e] = m;
          Sv[e] = q1 * (c * (1.f - c));
          const int r = e / C::BXin, col = e % C::BXin;
          if (r >= 1 && r <= kP3BY && col >= 1 && col <= C::BX) dg[(r - 1) * C::BX + col - 1] = dGv;
        }
      }
    }
    if (!all_melt) sm.melt[q & 7] = 0;
    return true;
  };
  // a load that did not arrive in time: wait (bounded) for every load still
  // in flight before the CTA leaves, so none lands in reused shared memory
  auto drain = [&](int from) {
    if (tid == 0)
      for (int z = from; z <= issued; ++z) {
        const int q = z - zin0;
        uint32_t tries = 0;
        while (!mbar_try_wait(&sm.full[q % kP3Slots], (uint32_t)((q / kP3Slots) & 1)) && ++tries < kP3WaitLimit) {
        }
      }
  };
  bool ok = mu_plane(zin0);
  ok = mu_plane(zin0 + 1) && ok;
  if (!__syncthreads_and(ok)) {
    drain(zin0);
    return;
  }

  constexpr int K = C::kCellsPerThread;
  const int ix = tid % C::BX, iy0 = (tid / C::BX) * K;
  const int gx = xb + 1 + ix;
  const bool xin = gx <= k.nx - 2;
  const int xg = gx == k.nx - 2 ? 0 : (gx == 1 ? k.nx - 1 : -1);
  const R third = R(1) / R(3);

  for (int z = zo0; z < zo1; ++z) {
    // one barrier per plane (see rs_peri3d.cu): afterwards the input slot of
    // plane z-2 takes the load of plane z+2
    if (!__syncthreads_and(mu_plane(z + 1))) {
      drain(z + 1);
      return;
    }
    if (z + 2 <= zin1 && z + 2 > issued) {
      if (tid == 0) issue(z + 2);
      issued = z + 2;
    }
    const int q = z - zin0;
    // planes z-1 .. z+1 pure melt wherever a stencil of an output cell reaches
    // (p3_melt_cell); the flag of plane z+3 is re-armed here (its computation,
    // mu_plane(z+3) before the barrier of iteration z+2, is separated from
    // this write by the barrier of z+1)
    const bool melt3 = sm.melt[(q - 1) & 7] && sm.melt[q & 7] && sm.melt[(q + 1) & 7];
    if (tid == 0) sm.melt[(q + 3) & 7] = 1;
    const R *c1 = sm.in[q % kP3Slots][0], *c2 = sm.in[q % kP3Slots][1], *cc = sm.in[q % kP3Slots][2];
    const R *d1 = sm.in[(q - 1) % kP3Slots][0], *d2 = sm.in[(q - 1) % kP3Slots][1];
    const R *u1 = sm.in[(q + 1) % kP3Slots][0], *u2 = sm.in[(q + 1) % kP3Slots][1];
    const R *mu = sm.mu[q % kP3MuSlots], *mud = sm.mu[(q - 1) % kP3MuSlots], *muu = sm.mu[(q + 1) % kP3MuSlots];
    const R *Sc = sm.S[q % kP3MuSlots], *Sd = sm.S[(q - 1) % kP3MuSlots], *Su = sm.S[(q + 1) % kP3MuSlots];
    const PlaneT<R> t = plane_terms<R>(k.tab, z);
    // z faces of mu'' add the melt's mu difference between the planes (FP32);
    // a face to a ghost plane has none (the ghost's mu'' is taken at this T)
    const R dKu = kF32 && z + 1 < k.nz - 1 ? t.dK : R(0);
    const R dKd = kF32 && z - 1 > 0 ? (R)k.tab[(int64_t)kTW * (z - 1) + kTdK] : R(0);
    const int zg = z == 1 ? 0 : (z == k.nz - 2 ? k.nz - 1 : -1);
    // the cell and every ghost cell that images it
    auto store_cell = [&](int gy, R n1, R n2, R nc) {
      const int yg = gy == k.ny - 2 ? 0 : (gy == 1 ? k.ny - 1 : -1);
      if ((xg & yg & zg) < 0) {
        const int64_t o = (int64_t)z * plane + (int64_t)gy * k.nx + gx;
        o1[o] = n1;
        o2[o] = n2;
        oc[o] = nc;
      } else {
        const int xs[2] = {gx, xg}, ys[2] = {gy, yg}, zs[2] = {z, zg};
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
          for (int bq = 0; bq < 2; ++bq)
#pragma unroll
            for (int cq = 0; cq < 2; ++cq) {
              if (xs[a] < 0 || ys[bq] < 0 || zs[cq] < 0) continue;
              const int64_t o = (int64_t)zs[cq] * plane + (int64_t)ys[bq] * k.nx + xs[a];
              o1[o] = n1;
              o2[o] = n2;
              oc[o] = nc;
            }
      }
    };
    if (xin && melt3) {
      // pure melt (p3_melt_cell): phi1, phi2 stay exactly 1 and 0 (every phase
      // term and Laplacian is a zero); the solute update is the general one
      const int e0 = (iy0 + 1) * C::BXin + ix + 1;
      R wm[K + 2], ws[K + 2];
#pragma unroll
      for (int r = 0; r < K + 2; ++r) {
        wm[r] = mu[e0 + (r - 1) * C::BXin];
        ws[r] = Sc[e0 + (r - 1) * C::BXin];
      }
#pragma unroll
      for (int r = 0; r < K; ++r) {
        const int gy = yb + 1 + iy0 + r;
        if (gy > k.ny - 2) break;
        const int e = e0 + r * C::BXin;
        const R m0 = wm[r + 1], S0 = ws[r + 1];
        const R jx = (S0 + Sc[e + 1]) * (mu[e + 1] - m0) - (S0 + Sc[e - 1]) * (m0 - mu[e - 1]);
        const R jy = (S0 + ws[r + 2]) * (wm[r + 2] - m0) - (S0 + ws[r]) * (m0 - wm[r]);
        const R jz = (S0 + Su[e]) * ((muu[e] - m0) + dKu) - (S0 + Sd[e]) * ((m0 - mud[e]) + dKd);
        store_cell(gy, R(1), R(0), cc[e] + (k.cfx * jx + k.cfy * jy + k.cfz * jz));
      }
    } else if (xin) {
      const int e0 = (iy0 + 1) * C::BXin + ix + 1;
      R w1[K + 2], w2[K + 2], wm[K + 2], ws[K + 2];
#pragma unroll
      for (int r = 0; r < K + 2; ++r) {
        const int e = e0 + (r - 1) * C::BXin;
        w1[r] = c1[e];
        w2[r] = c2[e];
        wm[r] = mu[e];
        ws[r] = Sc[e];
      }
#pragma unroll
      for (int r = 0; r < K; ++r) {
        const int gy = yb + 1 + iy0 + r;
        if (gy > k.ny - 2) break;
        const int e = e0 + r * C::BXin;
        const R p1 = w1[r + 1], p2 = w2[r + 1], m0 = wm[r + 1], S0 = ws[r + 1], p3 = R(1) - p1 - p2;
        const R cv = cc[e];
        R dGv;
        if constexpr (SURR)
          dGv = (R)sm.dG[q % 3][(iy0 + r) * C::BX + ix];
        else
          dGv = dG_cell(t, kF32 ? (R)(c_ref + cv) : cv);
        const R d12 = p1 - p2, d23 = p2 - p3, d31 = p3 - p1;
        // driving force of phase 1 against both grains (gp1 = G_1, gp2 = Q_1 (pj - pk))
        const R Q1 = R(7.5) * (p1 - R(1)) * (p1 * p1);
        const R G1 = R(3.75) * p1 * ((((R(3) * p1 - R(4)) * p1 - R(1)) * p1 + R(2)) + (R(3) * p1 - R(2)) * (d23 * d23));
        const R A = Q1 * d23 * dGv;
        // multi-well terms (fphi, TiAg.cu:522-527) with their shared factors
        const R s12 = p1 * p2, s13 = p1 * p3, s23 = p2 * p3;
        const R U1 = R(3) * s23 + R(3) * p1 + k.b * (p1 * p1), U2 = R(3) * s13 + R(3) * p2 + k.b * (p2 * p2),
                U3 = R(3) * s12 + R(3) * p3 + k.b * (p3 * p3);
        const R F1 = R(2) * p1 * (R(1) - p1) * (R(1) - R(2) * p1) + k.a1 * (s23 * s23) * (R(3) + R(2) * k.b * p1) +
                     R(2) * k.a2 * p1 * (p3 * p3) * U2 + R(2) * k.a3 * p1 * (p2 * p2) * U3 + k.lam * (G1 * dGv);
        const R F2 = R(2) * p2 * (R(1) - p2) * (R(1) - R(2) * p2) + R(2) * k.a1 * p2 * (p3 * p3) * U1 +
                     k.a2 * (s13 * s13) * (R(3) + R(2) * k.b * p2) + R(2) * k.a3 * p2 * (p1 * p1) * U3 + k.lam * A;
        const R F3 = R(2) * p3 * (R(1) - p3) * (R(1) - R(2) * p3) + R(2) * k.a1 * p3 * (p2 * p2) * U1 +
                     R(2) * k.a2 * p3 * (p1 * p1) * U2 + k.a3 * (s12 * s12) * (R(3) + R(2) * k.b * p3) - k.lam * A;
        (void)d12;
        (void)d31;
        const R x1p = c1[e + 1], x1m = c1[e - 1], x2p = c2[e + 1], x2m = c2[e - 1];
        const R z1p = u1[e], z1m = d1[e], z2p = u2[e], z2m = d2[e];
        const R lap1 = (x1p + x1m - R(2) * p1) * k.dxi2 + (w1[r + 2] + w1[r] - R(2) * p1) * k.dyi2 +
                       (z1p + z1m - R(2) * p1) * k.dzi2;
        const R lap2 = (x2p + x2m - R(2) * p2) * k.dxi2 + (w2[r + 2] + w2[r] - R(2) * p2) * k.dyi2 +
                       (z2p + z2m - R(2) * p2) * k.dzi2;
        const R n1 = p1 + k.dt * (lap1 - (R(2) * F1 - F2 - F3) * third);
        const R n2 = p2 + k.dt * (lap2 - (R(2) * F2 - F1 - F3) * third);
        // solute: face mobility (S + S') / 2 (the 1/2 is in cf)
        const R jx = (S0 + Sc[e + 1]) * (mu[e + 1] - m0) - (S0 + Sc[e - 1]) * (m0 - mu[e - 1]);
        const R jy = (S0 + ws[r + 2]) * (wm[r + 2] - m0) - (S0 + ws[r]) * (m0 - wm[r]);
        const R jz = (S0 + Su[e]) * ((muu[e] - m0) + dKu) - (S0 + Sd[e]) * ((m0 - mud[e]) + dKd);
        const R nc = cv + (k.cfx * jx + k.cfy * jy + k.cfz * jz);
        store_cell(gy, n1, n2, nc);
      }
    }
  }
}

// mu of every cell (rs3_mu), ghost layers as images; FP32 sets add c_off
template <typename R>
__global__ void __launch_bounds__(256) tinb_mu_kernel(const K3<R> k, const R *__restrict__ f1,
                                                      const R *__restrict__ f2, const R *__restrict__ fc,
                                                      R *__restrict__ mu) {
  const int64_t n = (int64_t)k.nx * k.ny * k.nz;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int x = (int)(i % k.nx), y = (int)((i / k.nx) % k.ny), z = (int)(i / ((int64_t)k.nx * k.ny));
    x = x == 0 ? k.nx - 2 : (x == k.nx - 1 ? 1 : x);
    y = y == 0 ? k.ny - 2 : (y == k.ny - 1 ? 1 : y);
    z = z == 0 ? 1 : (z == k.nz - 1 ? k.nz - 2 : z);
    const int64_t j = ((int64_t)z * k.ny + y) * k.nx + x;
    const PlaneT<double> t = plane_terms<double>(k.tab, z);
    mu[i] = (R)mu_cell(t, (double)f1[j], (double)f2[j], (double)fc[j] + k.c_off);
  }
}

// two grains under a seeded front, melt above (rs3_initial_grains)
template <typename R>
__global__ void grains_init_kernel(const K3<R> k, const uint64_t seed, const double z_front, const double amp,
                                   const double c_liquid, const double c_solid, R *__restrict__ f1,
                                   R *__restrict__ f2, R *__restrict__ fc) {
  const int x = 1 + blockIdx.x * blockDim.x + threadIdx.x, y = 1 + blockIdx.y;
  if (x > k.nx - 2 || y > k.ny - 2) return;
  uint32_t r[4] = {(uint32_t)x, (uint32_t)y, 0u, 0x5A465254u};
  philox4x32(r, (uint32_t)seed, (uint32_t)(seed >> 32));
  const double zc = z_front + amp * (2.0 * u53(r[0], r[1]) - 1.0);
  const bool first = x <= (k.nx - 2) / 2;
  for (int z = 1; z <= k.nz - 2; ++z) {
    const int64_t o = ((int64_t)z * k.ny + y) * k.nx + x;
    if (z < zc) {
      f1[o] = R(0);
      f2[o] = first ? R(1) : R(0);
      fc[o] = (R)(c_solid - k.c_off);
    } else {
      f1[o] = R(1);
      f2[o] = R(0);
      fc[o] = (R)(c_liquid - k.c_off);
    }
  }
}

// ---------------------------------------------------------------- FP32 exact step on packed pairs
// The exact FP32 step of tinb_kernel<float> with every thread computing two
// x-adjacent cells per instruction (add/sub/mul/fma.rn.f32x2, rs_f32x2.cuh;
// each lane rounds as the scalar FP32 operation), in the tiling of the TiAg
// pair kernel (rs_peri3d_x2.cu): output cells x0 .. x0+63 (x0 a multiple of
// 64, pairs start on even x), rows y0+1 .. y0+14; input box x0-4 .. x0+67 x
// y0 .. y0+15 per field and plane by 3D TMA into a four-slot ring; 224
// threads, warp w owns rows 2w, 2w+1, lane j the pair x0+2j, x0+2j+1.  mu''
// and S of each plane (tile and halo) are computed once into four-slot rings,
// so one barrier per plane suffices, as in tinb_kernel.  The surrogate path
// keeps the scalar kernel.
constexpr int kT2Threads = 224, kT2BX = 64, kT2BXin = 72, kT2BY = 14, kT2BYin = 16;
constexpr unsigned long long kOne2 = 0x3F8000003F800000ull, kAbs2 = 0x7FFFFFFF7FFFFFFFull;
__device__ __forceinline__ unsigned long long f2bits(f2 v) { return (unsigned long long)v; }
constexpr int kT2Plane = kT2BXin * kT2BYin;  // 1152 floats = 4608 bytes (36 x 128)
constexpr int kT2Slots = 4, kT2MuSlots = 4;
static_assert((kT2Plane * 4) % 128 == 0, "TMA destinations stay 128-byte aligned");
static_assert(kT2Threads == 32 * (kT2BY / 2) && kT2BX == 64, "a warp per row pair, a lane per column pair");

struct T2Smem {
  alignas(128) float in[kT2Slots][3][kT2Plane];
  alignas(16) float mu[kT2MuSlots][kT2Plane];  // mu'' (FP32 form, see mu_cell)
  alignas(16) float S[kT2MuSlots][kT2Plane];   // face-mobility terms q(phi1) c (1 - c)
  uint64_t full[kT2Slots];
  // per plane (q mod 8): every cell of the box inside the array is pure melt,
  // phi1 == 1 and phi2 == 0 exactly
  int melt[8];
};

// A1: the a1 well terms are non-zero; SD: solid diffusivities Da or Db non-zero
template <bool A1, bool SD>
__global__ void __launch_bounds__(kT2Threads, 2)
    tinb_x2_kernel(const __grid_constant__ K3<float> k, const __grid_constant__ CUtensorMap m1,
                   const __grid_constant__ CUtensorMap m2, const __grid_constant__ CUtensorMap mc,
                   float *__restrict__ o1, float *__restrict__ o2, float *__restrict__ oc, int *err) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T2Smem &sm = *reinterpret_cast<T2Smem *>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int x0 = kT2BX * blockIdx.x;  // first output column of the tile
  const int yb = kT2BY * blockIdx.y;  // box row 0 = array row yb; outputs yb+1 .. yb+14
  const int zo0 = 1 + k.z_chunk * blockIdx.z;
  const int zo1 = min(zo0 + k.z_chunk, k.nz - 1);
  if (zo0 >= zo1) return;
  const int zin0 = zo0 - 1, zin1 = zo1;
  constexpr uint32_t kBytes = 3u * kT2Plane * sizeof(float);
  if (smem_u32(smem_raw) & 127u) {
    if (tid == 0) atomicExch(err, 2);
    return;
  }
  auto issue = [&](int z) {
    const int q = z - zin0, s = q % kT2Slots;
    mbar_expect_tx(&sm.full[s], kBytes);
    tma_load_3d(&sm.in[s][0][0], &m1, &sm.full[s], x0 - 4, yb, z);
    tma_load_3d(&sm.in[s][1][0], &m2, &sm.full[s], x0 - 4, yb, z);
    tma_load_3d(&sm.in[s][2][0], &mc, &sm.full[s], x0 - 4, yb, z);
  };
  if (tid == 0) {
    for (int s = 0; s < kT2Slots; ++s) mbar_init(&sm.full[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    for (int z = zin0; z <= min(zin1, zin0 + kT2Slots - 1); ++z) issue(z);
    for (int s = 0; s < 8; ++s) sm.melt[s] = 1;
  }
  __syncthreads();
  int issued = min(zin1, zin0 + kT2Slots - 1);
  const float c_ref = (float)k.c_ref;
  const float lref = (float)log(k.c_ref / (1.0 - k.c_ref));
  const f2 one = bc(1.f);
  constexpr float L0d = (float)(kL0Bcc - kL0Liq), L0s = (float)(kL0Bcc + kL0Liq), L0x = (float)(kL0Liq - kL0Bcc);

  // mu'' and S of plane z (tile and halo) into their ring slots
  auto mu_plane = [&](int z) {
    const int q = z - zin0, s = q % kT2Slots;
    const bool got = p3_wait<float>(&sm.full[s], (uint32_t)((q / kT2Slots) & 1), err);
    // a ghost plane images its neighbour, T included
    const PlaneT<float> t = plane_terms<float>(k.tab, z == 0 ? 1 : (z == k.nz - 1 ? k.nz - 2 : z));
    if (!got) return false;
    float *mu = sm.mu[q % kT2MuSlots], *Sv = sm.S[q % kT2MuSlots];
    const float *f1 = sm.in[s][0], *f2p = sm.in[s][1], *fc = sm.in[s][2];
    bool all_melt = true;  // this thread's pairs inside the array
    for (int e = 2 * tid; e < kT2Plane; e += 2 * kT2Threads) {
      const f2 p1 = ld2(f1 + e), p2 = ld2(f2p + e), d = ld2(fc + e);
      // a pair lies wholly inside or outside the array (nx % 4 == 0, even x)
      const int ax = x0 - 4 + e % kT2BXin, ay = yb + e / kT2BXin;
      const bool inside = ax >= 0 && ax < k.nx && ay < k.ny;
      const bool melt = f2bits(p1) == kOne2 && (f2bits(p2) & kAbs2) == 0ull;
      all_melt = all_melt && (melt || !inside);
      if (melt && fmaxf(fabsf(lo_of(d)), fabsf(hi_of(d))) <= k.melt_tiny) {
        // far melt: g = -1, q(1) c (1 - c); lam by its Taylor polynomial
        // (K3::melt_a), mu'' = d (RT p - 2 L0_Liq), lam = d p
        f2 pp = fma2(bc(k.melt_a[3]), d, bc(k.melt_a[2]));
        pp = fma2(pp, d, bc(k.melt_a[1]));
        pp = fma2(pp, d, bc(k.melt_a[0]));
        const f2 c = add2(bc(c_ref), d);
        st2(mu + e, mul2(d, fma2(bc(t.RT), pp, bc((float)(-2.0 * kL0Liq)))));
        st2(Sv + e, mul2(mul2(p1, fma2(bc(-k.AA1), p1, bc(k.AA))), mul2(c, sub2(one, c))));
        continue;
      }
      const f2 p3 = sub2(sub2(one, p1), p2);
      // g3(p1, p2, p3) = p1^2 / 4 (15 (1 - p1)(1 + p1 - (p3 - p2)^2) + p1 (9 p1^2 - 5)); g = 1 - 2 g3
      const f2 dk = sub2(p3, p2);
      const f2 a = mul2(mul2(sub2(one, p1), bc(15.f)), fma2(dk, mul2(dk, bc(-1.f)), add2(one, p1)));
      const f2 gq = mul2(mul2(p1, p1), fma2(p1, fma2(mul2(p1, p1), bc(9.f), bc(-5.f)), a));
      const f2 g = fma2(gq, bc(-0.5f), one);
      const f2 c = add2(bc(c_ref), d), omc = sub2(one, c);
      // lam per lane (the logarithm's guard as in mu_cell)
      const float cl = lo_of(c), ch = hi_of(c), ol = lo_of(omc), oh = hi_of(omc);
      const f2 lam = pk(cl > 1.e-8f && ol > 1.e-8f ? lam_fast(lo_of(d), ol, c_ref + c_ref) : -lref,
                        ch > 1.e-8f && oh > 1.e-8f ? lam_fast(hi_of(d), oh, c_ref + c_ref) : -lref);
      // mu'' = -(g + 1) C0 - d (L0_BCC + L0_Liq + g (L0_BCC - L0_Liq)) + RT lam
      f2 m = mul2(add2(g, one), bc(-t.C0));
      m = fma2(d, mul2(fma2(bc(L0d), g, bc(L0s)), bc(-1.f)), m);
      m = fma2(bc(t.RT), lam, m);
      f2 q1 = mul2(p1, fma2(bc(-k.AA1), p1, bc(k.AA)));
      if constexpr (SD) q1 = fma2(bc(k.Db2), p3, fma2(bc(k.Da2), p2, q1));
      st2(mu + e, m);
      st2(Sv + e, mul2(q1, mul2(c, omc)));
    }
    if (!all_melt) sm.melt[q & 7] = 0;
    return true;
  };
  auto drain = [&](int from) {
    if (tid == 0)
      for (int z = from; z <= issued; ++z) {
        const int q = z - zin0;
        uint32_t tries = 0;
        while (!mbar_try_wait(&sm.full[q % kT2Slots], (uint32_t)((q / kT2Slots) & 1)) && ++tries < kP3WaitLimit) {
        }
      }
  };
  bool ok = mu_plane(zin0);
  ok = mu_plane(zin0 + 1) && ok;
  if (!__syncthreads_and(ok)) {
    drain(zin0);
    return;
  }

  const int gx = x0 + 2 * lane;                                        // array x of the pair's first cell
  const bool v0 = gx >= 1 && gx <= k.nx - 2, v1 = gx + 1 <= k.nx - 2;  // outputs
  const bool any = v0 || v1;
  const int ry = 2 * warp;                           // first output row of the thread (tile row)
  const int ec = (ry + 1) * kT2BXin + 2 * lane + 4;  // box element of its first cell (even)
  const int64_t plane = (int64_t)k.nx * k.ny;
  const bool xedge = !(v0 && v1) || gx == 1 || gx + 1 == k.nx - 2;  // a ghost column is involved
  const f2 dt = bc(k.dt), dt3 = bc(k.dt * (1.f / 3.f));

  for (int z = zo0; z < zo1; ++z) {
    // one barrier per plane: afterwards the input slot of plane z-2 takes the
    // load of plane z+2 (mu'' and S have four slots: plane z+1 overwrites z-3)
    if (!__syncthreads_and(mu_plane(z + 1))) {
      drain(z + 1);
      return;
    }
    if (z + 2 <= zin1 && z + 2 > issued) {
      if (tid == 0) issue(z + 2);
      issued = z + 2;
    }
    const int q = z - zin0;
    // planes z-1 .. z+1 pure melt wherever a stencil of an output cell reaches:
    // phi1 and phi2 stay exactly 1 and 0 (every phase term and Laplacian is
    // an exact zero there), only c is updated.  The flag of plane z+3 is
    // re-armed here: its computation (mu_plane(z+3), before the barrier of
    // iteration z+2) is separated from this write by the barrier of z+1.
    const bool melt3 = sm.melt[(q - 1) & 7] && sm.melt[q & 7] && sm.melt[(q + 1) & 7];
    if (tid == 0) sm.melt[(q + 3) & 7] = 1;
    if (!any) continue;
    const float *c1 = sm.in[q % kT2Slots][0], *c2 = sm.in[q % kT2Slots][1], *cc = sm.in[q % kT2Slots][2];
    const float *d1 = sm.in[(q - 1) % kT2Slots][0], *d2 = sm.in[(q - 1) % kT2Slots][1];
    const float *u1 = sm.in[(q + 1) % kT2Slots][0], *u2 = sm.in[(q + 1) % kT2Slots][1];
    const float *mu = sm.mu[q % kT2MuSlots], *mud = sm.mu[(q - 1) % kT2MuSlots], *muu = sm.mu[(q + 1) % kT2MuSlots];
    const float *Sc = sm.S[q % kT2MuSlots], *Sd = sm.S[(q - 1) % kT2MuSlots], *Su = sm.S[(q + 1) % kT2MuSlots];
    const PlaneT<float> t = plane_terms<float>(k.tab, z);
    // z faces of mu'' add the melt's mu difference between the planes; a face
    // to a ghost plane has none (the ghost's mu'' is taken at this T)
    const f2 dKu = bc(z + 1 < k.nz - 1 ? t.dK : 0.f);
    const f2 dKd = bc(z - 1 > 0 ? (float)k.tab[(int64_t)kTW * (z - 1) + kTdK] : 0.f);
    const int zg = z == 1 ? 0 : (z == k.nz - 2 ? k.nz - 1 : -1);
    // column window rows ry-1 .. ry+2 of phi1, phi2, mu'', S (pairs)
    f2 w1[4], w2[4], wm[4], ws[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int e = ec + (r - 1) * kT2BXin;
      w1[r] = ld2(c1 + e);
      w2[r] = ld2(c2 + e);
      wm[r] = ld2(mu + e);
      ws[r] = ld2(Sc + e);
    }
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int gy = yb + 1 + ry + r;
      if (gy > k.ny - 2) break;
      const int e = ec + r * kT2BXin;
      const f2 p1 = w1[r + 1], p2 = w2[r + 1], m0 = wm[r + 1], S0 = ws[r + 1];
      const f2 cv = ld2(cc + e);
      // x neighbours: (left, right) pairs from the pairs beside this one
      const f2 Lm = ld2(mu + e - 2), Rm = ld2(mu + e + 2), Ls = ld2(Sc + e - 2), Rs = ld2(Sc + e + 2);
      const f2 mxm = pk(hi_of(Lm), lo_of(m0)), mxp = pk(hi_of(m0), lo_of(Rm));
      const f2 sxm = pk(hi_of(Ls), lo_of(S0)), sxp = pk(hi_of(S0), lo_of(Rs));

      f2 n1 = bc(1.f), n2 = bc(0.f);
      if (!melt3) {
      const f2 L1 = ld2(c1 + e - 2), R1 = ld2(c1 + e + 2), L2 = ld2(c2 + e - 2), R2 = ld2(c2 + e + 2);
      const f2 x1m = pk(hi_of(L1), lo_of(p1)), x1p = pk(hi_of(p1), lo_of(R1));
      const f2 x2m = pk(hi_of(L2), lo_of(p2)), x2p = pk(hi_of(p2), lo_of(R2));
      const f2 p3 = sub2(sub2(one, p1), p2);
      // driving force of phase 1 against both grains (fun.cu:1192-1193)
      const f2 c = add2(bc(c_ref), cv), omc = sub2(one, c);
      const f2 dGv = fma2(mul2(c, omc), bc(L0x), fma2(c, bc(t.Ati), mul2(omc, bc(t.Anb))));
      const f2 d23 = sub2(p2, p3);
      // gp2 = Q_1 (pj - pk), Q_1 = 7.5 (p1 - 1) p1^2; gp1 = G_1
      const f2 Q1 = mul2(fma2(p1, bc(7.5f), bc(-7.5f)), mul2(p1, p1));
      f2 Ga = fma2(p1, bc(3.f), bc(-4.f));
      Ga = fma2(Ga, p1, bc(-1.f));
      Ga = fma2(Ga, p1, bc(2.f));
      const f2 G1 = mul2(mul2(p1, bc(3.75f)), fma2(fma2(p1, bc(3.f), bc(-2.f)), mul2(d23, d23), Ga));
      const f2 A = mul2(mul2(Q1, d23), dGv);
      // multi-well terms (fphi, TiAg.cu:522-527) with their shared factors
      const f2 s12 = mul2(p1, p2), s13 = mul2(p1, p3), s23 = mul2(p2, p3);
      const f2 p1s = mul2(p1, p1), p2s = mul2(p2, p2), p3s = mul2(p3, p3);
      const f2 U2 = fma2(s13, bc(3.f), mul2(p2, fma2(p2, bc(k.b), bc(3.f))));
      const f2 U3 = fma2(s12, bc(3.f), mul2(p3, fma2(p3, bc(k.b), bc(3.f))));
      const f2 k2 = mul2(U2, bc(2.f * k.a2)), k3 = mul2(U3, bc(2.f * k.a3));
      auto dw = [&](f2 p) { return mul2(fma2(fma2(p, bc(4.f), bc(-6.f)), p, bc(2.f)), p); };  // 2p(1-p)(1-2p)
      f2 F1 = fma2(mul2(p1, p3s), k2, dw(p1));
      F1 = fma2(mul2(p1, p2s), k3, F1);
      F1 = fma2(mul2(G1, dGv), bc(k.lam), F1);
      f2 F2 = fma2(mul2(s13, s13), mul2(fma2(p2, bc(2.f * k.b), bc(3.f)), bc(k.a2)), dw(p2));
      F2 = fma2(mul2(p2, p1s), k3, F2);
      F2 = fma2(A, bc(k.lam), F2);
      f2 F3 = fma2(mul2(p3, p1s), k2, dw(p3));
      F3 = fma2(mul2(s12, s12), mul2(fma2(p3, bc(2.f * k.b), bc(3.f)), bc(k.a3)), F3);
      F3 = fma2(A, bc(-k.lam), F3);
      if constexpr (A1) {
        const f2 U1 = fma2(s23, bc(3.f), mul2(p1, fma2(p1, bc(k.b), bc(3.f))));
        const f2 k1 = mul2(U1, bc(2.f * k.a1));
        F1 = fma2(mul2(s23, s23), mul2(fma2(p1, bc(2.f * k.b), bc(3.f)), bc(k.a1)), F1);
        F2 = fma2(mul2(p2, p3s), k1, F2);
        F3 = fma2(mul2(p3, p2s), k1, F3);
      }
      // Laplacians
      auto lap = [&](f2 p, f2 xp, f2 xm, f2 yp, f2 ym, f2 zp, f2 zm) {
        f2 l = mul2(fma2(p, bc(-2.f), add2(xp, xm)), bc(k.dxi2));
        l = fma2(fma2(p, bc(-2.f), add2(yp, ym)), bc(k.dyi2), l);
        return fma2(fma2(p, bc(-2.f), add2(zp, zm)), bc(k.dzi2), l);
      };
      const f2 lap1 = lap(p1, x1p, x1m, w1[r + 2], w1[r], ld2(u1 + e), ld2(d1 + e));
      const f2 lap2 = lap(p2, x2p, x2m, w2[r + 2], w2[r], ld2(u2 + e), ld2(d2 + e));
      // phi_i' = phi_i + dt lap_i - dt (2F_i - F_j - F_k) / 3
      const f2 T3 = mul2(add2(add2(F1, F2), F3), dt3);
      n1 = fma2(F1, bc(-k.dt), add2(T3, fma2(lap1, dt, p1)));
      n2 = fma2(F2, bc(-k.dt), add2(T3, fma2(lap2, dt, p2)));
      }
      // solute: face mobility (S + S') / 2 (the 1/2 is in cf)
      const f2 jx = fma2(add2(S0, sxp), sub2(mxp, m0), mul2(add2(S0, sxm), sub2(mxm, m0)));
      const f2 jy = fma2(add2(S0, ws[r + 2]), sub2(wm[r + 2], m0), mul2(add2(S0, ws[r]), sub2(wm[r], m0)));
      const f2 jz = fma2(add2(S0, ld2(Su + e)), add2(sub2(ld2(muu + e), m0), dKu),
                         mul2(add2(S0, ld2(Sd + e)), sub2(sub2(ld2(mud + e), m0), dKd)));
      const f2 nc = add2(cv, fma2(bc(k.cfz), jz, fma2(bc(k.cfy), jy, mul2(bc(k.cfx), jx))));
      // stores: the pair, and every ghost cell that images one of its cells
      const int yg = gy == k.ny - 2 ? 0 : (gy == 1 ? k.ny - 1 : -1);
      const int64_t o = (int64_t)z * plane + (int64_t)gy * k.nx + gx;
      if (!xedge && (yg & zg) < 0) {
        st2(o1 + o, n1);
        st2(o2 + o, n2);
        st2(oc + o, nc);
      } else {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int x = gx + h;
          if (!(h ? v1 : v0)) continue;
          const float a = h ? hi_of(n1) : lo_of(n1), bb = h ? hi_of(n2) : lo_of(n2), cvv = h ? hi_of(nc) : lo_of(nc);
          const int xg = x == k.nx - 2 ? 0 : (x == 1 ? k.nx - 1 : -1);
          const int xs[2] = {x, xg}, ys[2] = {gy, yg}, zs[2] = {z, zg};
#pragma unroll
          for (int ia = 0; ia < 2; ++ia)
#pragma unroll
            for (int ib = 0; ib < 2; ++ib)
#pragma unroll
              for (int ic = 0; ic < 2; ++ic) {
                if (xs[ia] < 0 || ys[ib] < 0 || zs[ic] < 0) continue;
                const int64_t oo = (int64_t)zs[ic] * plane + (int64_t)ys[ib] * k.nx + xs[ia];
                o1[oo] = a;
                o2[oo] = bb;
                oc[oo] = cvv;
              }
        }
      }
    }
  }
}

template <bool A1, bool SD>
int launch_tinb_x2(const K3<float> &k, const P3Maps &m, float *o1, float *o2, float *oc, int *err, cudaStream_t st) {
  const size_t smem = sizeof(T2Smem) + 128;
  auto kfn = tinb_x2_kernel<A1, SD>;
  static std::atomic<unsigned long long> attr;
  if (!smem_limit_once((const void *)kfn, (int)smem, attr)) return -3;
  const dim3 grid((k.nx + kT2BX - 1) / kT2BX, (k.ny - 2 + kT2BY - 1) / kT2BY, (k.nz - 2 + k.z_chunk - 1) / k.z_chunk);
  kfn<<<grid, kT2Threads, smem, st>>>(k, m.phi1, m.phi2, m.c, o1, o2, oc, err);
  return 0;
}

template <typename R, bool SD, bool SURR>
int launch_tinb(const K3<R> &k, const P3Maps &m, R *o1, R *o2, R *oc, int64_t step, int *err, const SurrArgs &sa,
                cudaStream_t st) {
  using C = P3Cfg<R>;
  const size_t smem = sizeof(TSmem<R, SURR>) + 128;
  auto kfn = tinb_kernel<R, SD, SURR>;
  static std::atomic<unsigned long long> attr;
  if (!smem_limit_once((const void *)kfn, (int)smem, attr)) return -3;
  const dim3 grid((k.nx - 2 + C::BX - 1) / C::BX, (k.ny - 2 + kP3BY - 1) / kP3BY,
                  (k.nz - 2 + k.z_chunk - 1) / k.z_chunk);
  kfn<<<grid, kP3Threads, smem, st>>>(k, m.phi1, m.phi2, m.c, o1, o2, oc, step, err, sa);
  return 0;
}

}  // namespace

int tinb_box_width(int precision, bool surr) {
  return precision == RS_F64 ? P3Cfg<double>::BXin : surr ? P3Cfg<float>::BXin : kT2BXin;
}
int tinb_box_height(int precision, bool surr) { return precision == RS_F32 && !surr ? kT2BYin : kP3BY + 2; }
int tinb_table_len(const rs3_params &p) { return kTW * p.nz; }

int launch_tinb_step(const rs3_params &p, const P3Maps &m, int precision, void *o1, void *o2, void *oc, int64_t step,
                     int *err, double *tab, const SurrArgs *surr, cudaStream_t st) {
  {
    K3<double> kt = make_k3<double>(p);
    tinb_table_kernel<<<(p.nz + 127) / 128, 128, 0, st>>>(kt, step, tab);
  }
  const bool sd = p.Da != 0.0 || p.Db != 0.0;
  SurrArgs none;
  memset(&none, 0, sizeof(none));
  if (precision == RS_F64) {
    if (surr) return -4;
    K3<double> k = make_k3<double>(p);
    k.tab = tab;
    return sd ? launch_tinb<double, true, false>(k, m, (double *)o1, (double *)o2, (double *)oc, step, err, none, st)
              : launch_tinb<double, false, false>(k, m, (double *)o1, (double *)o2, (double *)oc, step, err, none,
                                                  st);
  }
  K3<float> k = make_k3<float>(p);
  k.tab = tab;
  k.c_off = p.c_ref;
  float *f1 = (float *)o1, *f2 = (float *)o2, *fc = (float *)oc;
  if (surr)
    return sd ? launch_tinb<float, true, true>(k, m, f1, f2, fc, step, err, *surr, st)
              : launch_tinb<float, false, true>(k, m, f1, f2, fc, step, err, *surr, st);
  // the exact FP32 step on packed pairs
  const bool a1 = p.a1 != 0.0;
  return a1 ? (sd ? launch_tinb_x2<true, true>(k, m, f1, f2, fc, err, st)
                  : launch_tinb_x2<true, false>(k, m, f1, f2, fc, err, st))
            : (sd ? launch_tinb_x2<false, true>(k, m, f1, f2, fc, err, st)
                  : launch_tinb_x2<false, false>(k, m, f1, f2, fc, err, st));
}

int launch_tinb_mu(const rs3_params &p, int precision, const void *f1, const void *f2, const void *fc, void *mu,
                   double *tab, cudaStream_t st) {
  K3<double> kt = make_k3<double>(p);
  tinb_table_kernel<<<(p.nz + 127) / 128, 128, 0, st>>>(kt, 0, tab);
  const int64_t n = (int64_t)p.nx * p.ny * p.nz;
  const unsigned blocks = (unsigned)std::min<int64_t>((n + 255) / 256, 148 * 16);
  if (precision == RS_F64) {
    K3<double> k = make_k3<double>(p);
    k.tab = tab;
    tinb_mu_kernel<double><<<blocks, 256, 0, st>>>(k, (const double *)f1, (const double *)f2, (const double *)fc,
                                                   (double *)mu);
  } else {
    K3<float> k = make_k3<float>(p);
    k.tab = tab;
    k.c_off = p.c_ref;
    tinb_mu_kernel<float><<<blocks, 256, 0, st>>>(k, (const float *)f1, (const float *)f2, (const float *)fc,
                                                  (float *)mu);
  }
  return 0;
}

int launch_grains_init(const rs3_params &p, int precision, uint64_t seed, double z_front, double amp,
                       double c_liquid, double c_solid, void *f1, void *f2, void *fc, cudaStream_t st) {
  const dim3 g((p.nx - 2 + 127) / 128, p.ny - 2);
  const double c_off = peri3d_c_offset(p);
  if (precision == RS_F64) {
    grains_init_kernel<double><<<g, 128, 0, st>>>(make_k3<double>(p), seed, z_front, amp, c_liquid, c_solid,
                                                  (double *)f1, (double *)f2, (double *)fc);
  } else {
    K3<float> k = make_k3<float>(p);
    k.c_off = c_off;
    grains_init_kernel<float><<<g, 128, 0, st>>>(k, seed, z_front, amp, c_liquid, c_solid, (float *)f1,
                                                 (float *)f2, (float *)fc);
  }
  return launch_peri3d_ghosts(p, precision, f1, f2, fc, st);
}

}  // namespace rs

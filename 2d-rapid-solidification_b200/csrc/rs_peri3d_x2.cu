// rs_peri3d_x2.cu — the FP32 3D three-phase step on packed FP32 pairs.
//
// Same model and pipeline as the FP64 kernel of rs_peri3d.cu (TiAg.cu
// computeMu + diffuse + boundary, one TMA z march per CTA), but every thread
// computes two x-adjacent cells at once with the sm_100 packed FP32
// instructions (add/sub/mul/fma.rn.f32x2): half the arithmetic and shared
// memory instructions of the scalar form, each lane rounded exactly as the
// scalar FP32 operation.
//
// Field storage: an FP32 set holds c - c_off (c_off = clb, the melt's
// composition at T_ref, rs3_c_offset), so that the small solute updates of
// the melt are not lost below ulp(c); mu is carried as mu - c_off (only its
// differences and s_i - r_i mu enter), with c_off folded into the s_i.
//
// Tile: output cells x0 .. x0+63 (x0 a multiple of 64, pairs start on even
// x), rows y0+1 .. y0+14.  Input box per field and plane: x0-4 .. x0+67
// (72 columns, TMA x 16-byte aligned) x y0 .. y0+15 (16 rows).  224 threads:
// warp w owns rows 2w, 2w+1, lane j the pair x0+2j, x0+2j+1.  The x = 0 and
// x = nx-1 members of a pair are ghost cells and are not outputs.
#include <cuda.h>

#include "rs_f32x2.cuh"
#include "rs_peri3d.cuh"
#include "rs_step_common.cuh"

namespace rs {
namespace {

constexpr int kX2Threads = 224;
constexpr int kX2BX = 64, kX2BXin = 72, kX2BY = 14, kX2BYin = 16;
constexpr int kX2Plane = kX2BXin * kX2BYin;  // 1152 floats = 4608 bytes (36 x 128)
constexpr int kX2Slots = 4, kX2MuSlots = 4;
constexpr uint32_t kX2WaitLimit = 1u << 22;
static_assert((kX2Plane * 4) % 128 == 0, "TMA destinations stay 128-byte aligned");
static_assert(kX2Threads == 32 * (kX2BY / 2) && kX2BX == 64, "a warp per row pair, a lane per column pair");

struct X2Smem {
  alignas(128) float in[kX2Slots][3][kX2Plane];
  alignas(128) float mu[kX2MuSlots][kX2Plane];
  uint64_t full[kX2Slots];
  // per plane (q mod 8): every cell of the box inside the array is pure melt,
  // phi1 == 1 and phi2 == 0 exactly
  int melt[8];
};
constexpr unsigned long long kOne2 = 0x3F8000003F800000ull, kAbs2 = 0x7FFFFFFF7FFFFFFFull;

// kernel constants, FP32
struct X2K {
  int nx, ny, nz, z_chunk;
  float a1, a2, a3, b, lam, Da, Db;
  float r1, r2, r3;
  float dt, dt3, dxi2, dyi2, dzi2, cfx, cfy, cfz;
  double B11, B12, B21, B22, T_ref, G_T, V_T, z_T;
  double r1d, r2d, r3d, c_off;  // r_i in FP64 and the storage offset of c
};

// mu = c - sum r_i g_i (TiAg.cu:461-470), with
// g_i = p_i^2 / 4 (15 - 15 p_i^2 + 9 p_i^3 - 5 p_i - 15 (1 - p_i) (p_k - p_j)^2)
__device__ __forceinline__ f2 mu2(const X2K &k, f2 p1, f2 p2, f2 c) {
  const f2 p3 = sub2(sub2(bc(1.f), p1), p2);
  const f2 d12 = sub2(p1, p2), d23 = sub2(p2, p3), d31 = sub2(p3, p1);
  auto g = [&](f2 p, f2 d) {
    f2 poly = fma2(p, bc(9.f), bc(-15.f));
    poly = fma2(poly, p, bc(-5.f));
    poly = fma2(poly, p, bc(15.f));
    poly = fma2(fma2(p, bc(15.f), bc(-15.f)), mul2(d, d), poly);
    return mul2(mul2(p, p), poly);
  };
  f2 m = fma2(g(p3, d12), bc(-0.25f * k.r3), c);
  m = fma2(g(p2, d31), bc(-0.25f * k.r2), m);
  return fma2(g(p1, d23), bc(-0.25f * k.r1), m);
}

template <bool A1, bool SD>
__global__ void __launch_bounds__(kX2Threads, 3)
    peri3d_x2_kernel(const __grid_constant__ X2K k, const __grid_constant__ CUtensorMap m1,
                     const __grid_constant__ CUtensorMap m2, const __grid_constant__ CUtensorMap mc,
                     float *__restrict__ o1, float *__restrict__ o2, float *__restrict__ oc, const int64_t step,
                     int *err) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  X2Smem &sm = *reinterpret_cast<X2Smem *>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int x0 = kX2BX * blockIdx.x;         // first output column of the tile
  const int yb = kX2BY * blockIdx.y;         // box row 0 = array row yb; outputs yb+1 .. yb+14
  const int zo0 = 1 + k.z_chunk * blockIdx.z;
  const int zo1 = min(zo0 + k.z_chunk, k.nz - 1);
  if (zo0 >= zo1) return;
  const int zin0 = zo0 - 1, zin1 = zo1;
  constexpr uint32_t kBytes = 3u * kX2Plane * sizeof(float);
  if (smem_u32(smem_raw) & 127u) {
    if (tid == 0) atomicExch(err, 2);
    return;
  }
  auto issue = [&](int z) {
    const int q = z - zin0, s = q % kX2Slots;
    mbar_expect_tx(&sm.full[s], kBytes);
    tma_load_3d(&sm.in[s][0][0], &m1, &sm.full[s], x0 - 4, yb, z);
    tma_load_3d(&sm.in[s][1][0], &m2, &sm.full[s], x0 - 4, yb, z);
    tma_load_3d(&sm.in[s][2][0], &mc, &sm.full[s], x0 - 4, yb, z);
  };
  if (tid == 0) {
    for (int s = 0; s < kX2Slots; ++s) mbar_init(&sm.full[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    for (int z = zin0; z <= min(zin1, zin0 + kX2Slots - 1); ++z) issue(z);
    for (int s = 0; s < 8; ++s) sm.melt[s] = 1;
  }
  __syncthreads();
  int issued = min(zin1, zin0 + kX2Slots - 1);
  auto wait_plane = [&](int z) {
    const int q = z - zin0;
    uint32_t tries = 0;
    while (!mbar_try_wait(&sm.full[q % kX2Slots], (uint32_t)((q / kX2Slots) & 1)))
      if (++tries >= kX2WaitLimit) {
        atomicExch(err, 1);
        return false;
      }
    return true;
  };
  auto mu_plane = [&](int z) {
    const bool got = wait_plane(z);
    const int q = z - zin0, s = q % kX2Slots;
    float *mu = sm.mu[q % kX2MuSlots];
    const float *f1 = sm.in[s][0], *f2p = sm.in[s][1], *fc = sm.in[s][2];
    if (got) {
      bool all_melt = true;  // this thread's pairs inside the array
      for (int e = 2 * tid; e < kX2Plane; e += 2 * kX2Threads) {
        const f2 p1 = ld2(f1 + e), p2 = ld2(f2p + e);
        st2(mu + e, mu2(k, p1, p2, ld2(fc + e)));
        // a pair lies wholly inside or outside the array (nx % 4 == 0, even x)
        const int ax = x0 - 4 + e % kX2BXin, ay = yb + e / kX2BXin;
        const bool inside = ax >= 0 && ax < k.nx && ay < k.ny;
        all_melt = all_melt && (!inside || ((unsigned long long)p1 == kOne2 && ((unsigned long long)p2 & kAbs2) == 0ull));
      }
      if (!all_melt) sm.melt[q & 7] = 0;
    }
    return got;
  };
  auto drain = [&](int from) {
    if (tid == 0)
      for (int z = from; z <= issued; ++z) {
        const int q = z - zin0;
        uint32_t tries = 0;
        while (!mbar_try_wait(&sm.full[q % kX2Slots], (uint32_t)((q / kX2Slots) & 1)) && ++tries < kX2WaitLimit) {
        }
      }
  };
  bool ok = mu_plane(zin0);
  ok = mu_plane(zin0 + 1) && ok;
  if (!__syncthreads_and(ok)) {
    drain(zin0);
    return;
  }

  const int gx = x0 + 2 * lane;                        // array x of the pair's first cell
  const bool v0 = gx >= 1 && gx <= k.nx - 2, v1 = gx + 1 <= k.nx - 2;  // outputs
  const bool any = v0 || v1;
  const int ry = 2 * warp;                             // first output row of the thread (tile row)
  const int ec = (ry + 1) * kX2BXin + 2 * lane + 4;    // box element of its first cell (even)
  const int64_t plane = (int64_t)k.nx * k.ny;
  const bool xedge = !(v0 && v1) || gx == 1 || gx + 1 == k.nx - 2;  // a ghost column is involved

  for (int z = zo0; z < zo1; ++z) {
    // one barrier per plane: after it every thread has finished plane z-1,
    // so the input slot of plane z-2 takes the load of plane z+2 (mu has
    // four slots: mu(z+1) overwrites mu(z-3))
    if (!__syncthreads_and(mu_plane(z + 1))) {
      drain(z + 1);
      return;
    }
    if (z + 2 <= zin1 && z + 2 > issued) {
      if (tid == 0) issue(z + 2);
      issued = z + 2;
    }
    const int q = z - zin0;
    // planes z-1 .. z+1 pure melt wherever a stencil of an output cell
    // reaches (the flag of plane z+3 is re-armed here: its computation,
    // mu_plane(z+3) before the barrier of iteration z+2, is separated from
    // this write by the barrier of z+1)
    const bool melt3 = sm.melt[(q - 1) & 7] && sm.melt[q & 7] && sm.melt[(q + 1) & 7];
    if (tid == 0) sm.melt[(q + 3) & 7] = 1;
    const float *c1 = sm.in[q % kX2Slots][0], *c2 = sm.in[q % kX2Slots][1], *cc = sm.in[q % kX2Slots][2];
    const float *d1 = sm.in[(q - 1) % kX2Slots][0], *d2 = sm.in[(q - 1) % kX2Slots][1];
    const float *u1 = sm.in[(q + 1) % kX2Slots][0], *u2 = sm.in[(q + 1) % kX2Slots][1];
    const float *mu = sm.mu[q % kX2MuSlots], *mud = sm.mu[(q - 1) % kX2MuSlots], *muu = sm.mu[(q + 1) % kX2MuSlots];
    const double Tz = k.G_T == 0.0 ? k.T_ref : k.T_ref + k.G_T * ((double)z - k.z_T - k.V_T * (double)step);
    const double B1 = k.B11 + k.B12 * Tz, B2 = k.B21 + k.B22 * Tz;
    // s_i - r_i c_off: the fields hold c - c_off, so mu - c_off is what mu2 returns
    const f2 s1 = bc((float)(B1 - k.r1d * k.c_off)), s2 = bc((float)(-B1 - B2 - k.r2d * k.c_off)),
             s3 = bc((float)(-B1 + B2 - k.r3d * k.c_off));
    const int zg = z == 1 ? 0 : (z == k.nz - 2 ? k.nz - 1 : -1);
    // stores: the pair, and every ghost cell that images one of its cells
    auto store_pair = [&](int gy, f2 n1, f2 n2, f2 nc) {
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
          const float a = h ? hi_of(n1) : lo_of(n1), bb = h ? hi_of(n2) : lo_of(n2), cv = h ? hi_of(nc) : lo_of(nc);
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
                oc[oo] = cv;
              }
        }
      }
    };
    if (any && melt3) {
      // pure-melt neighbourhood: phi1 and phi2 stay exactly 1 and 0 (every
      // phase term and Laplacian is a zero there) and every face mobility is
      // phi1 + phi1' = 2 exactly (the solid terms vanish), so the solute
      // update is c + sum_d cf_d 2 ((mu+ - mu) + (mu- - mu)), the general
      // form's value bit for bit
#pragma unroll
      for (int r = 0; r < 2; ++r) {
        const int gy = yb + 1 + ry + r;
        if (gy > k.ny - 2) break;
        const int e = ec + r * kX2BXin;
        const f2 m0 = ld2(mu + e);
        const f2 Lm = ld2(mu + e - 2), Rm = ld2(mu + e + 2);
        auto face_m = [&](f2 mp, f2 mm) { return mul2(bc(2.f), add2(sub2(mp, m0), sub2(mm, m0))); };
        f2 nc = fma2(face_m(pk(hi_of(m0), lo_of(Rm)), pk(hi_of(Lm), lo_of(m0))), bc(k.cfx), ld2(cc + e));
        nc = fma2(face_m(ld2(mu + e + kX2BXin), ld2(mu + e - kX2BXin)), bc(k.cfy), nc);
        nc = fma2(face_m(ld2(muu + e), ld2(mud + e)), bc(k.cfz), nc);
        store_pair(gy, bc(1.f), bc(0.f), nc);
      }
    } else if (any) {
      // column window rows ry-1 .. ry+2 of phi1, phi2, mu (pairs)
      f2 w1[4], w2[4], wm[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int e = ec + (r - 1) * kX2BXin;
        w1[r] = ld2(c1 + e);
        w2[r] = ld2(c2 + e);
        wm[r] = ld2(mu + e);
      }
#pragma unroll
      for (int r = 0; r < 2; ++r) {
        const int gy = yb + 1 + ry + r;
        if (gy > k.ny - 2) break;
        const int e = ec + r * kX2BXin;
        const f2 p1 = w1[r + 1], p2 = w2[r + 1], m0 = wm[r + 1];
        // x neighbours: (left, right) pairs from the pairs beside this one
        const f2 L1 = ld2(c1 + e - 2), R1 = ld2(c1 + e + 2), L2 = ld2(c2 + e - 2), R2 = ld2(c2 + e + 2);
        const f2 Lm = ld2(mu + e - 2), Rm = ld2(mu + e + 2);
        const f2 x1m = pk(hi_of(L1), lo_of(p1)), x1p = pk(hi_of(p1), lo_of(R1));
        const f2 x2m = pk(hi_of(L2), lo_of(p2)), x2p = pk(hi_of(p2), lo_of(R2));
        const f2 mxm = pk(hi_of(Lm), lo_of(m0)), mxp = pk(hi_of(m0), lo_of(Rm));
        const f2 z1p = ld2(u1 + e), z1m = ld2(d1 + e), z2p = ld2(u2 + e), z2m = ld2(d2 + e);
        const f2 mzp = ld2(muu + e), mzm = ld2(mud + e);
        const f2 y1p = w1[r + 2], y1m = w1[r], y2p = w2[r + 2], y2m = w2[r], myp = wm[r + 2], mym = wm[r];

        const f2 p3 = sub2(sub2(bc(1.f), p1), p2);
        const f2 d12 = sub2(p1, p2), d23 = sub2(p2, p3), d31 = sub2(p3, p1);
        // gp2(pi, pj, pk) = Q_i (pj - pk), Q_i = 7.5 (p_i - 1) p_i^2
        const f2 Q1 = mul2(fma2(p1, bc(7.5f), bc(-7.5f)), mul2(p1, p1));
        const f2 Q2 = mul2(fma2(p2, bc(7.5f), bc(-7.5f)), mul2(p2, p2));
        const f2 Q3 = mul2(fma2(p3, bc(7.5f), bc(-7.5f)), mul2(p3, p3));
        // gp1(pi, pj, pk) = 3.75 p_i (3p_i^3 - 4p_i^2 - p_i + 2 + (3p_i - 2)(pj - pk)^2)
        auto G = [&](f2 p, f2 d) {
          f2 a = fma2(p, bc(11.25f), bc(-15.f));
          a = fma2(a, p, bc(-3.75f));
          a = fma2(a, p, bc(7.5f));
          a = fma2(fma2(p, bc(11.25f), bc(-7.5f)), mul2(d, d), a);
          return mul2(p, a);
        };
        const f2 G1 = G(p1, d23), G2 = G(p2, d31), G3 = G(p3, d12);
        // grand-potential differences s_i - r_i mu (fcphi, TiAg.cu:514-516)
        const f2 o1w = fma2(m0, bc(-k.r1), s1), o2w = fma2(m0, bc(-k.r2), s2), o3w = fma2(m0, bc(-k.r3), s3);
        const f2 A = mul2(mul2(Q1, d23), o1w), Bq = mul2(mul2(Q2, d31), o2w), Cq = mul2(mul2(Q3, d12), o3w);
        // multi-well terms (fphi, TiAg.cu:522-527): U_i and the shared products
        const f2 s12 = mul2(p1, p2), s13 = mul2(p1, p3), s23 = mul2(p2, p3);
        const f2 p1s = mul2(p1, p1), p2s = mul2(p2, p2), p3s = mul2(p3, p3);
        const f2 U2 = fma2(s13, bc(3.f), mul2(p2, fma2(p2, bc(k.b), bc(3.f))));
        const f2 U3 = fma2(s12, bc(3.f), mul2(p3, fma2(p3, bc(k.b), bc(3.f))));
        const f2 k2 = mul2(U2, bc(2.f * k.a2)), k3 = mul2(U3, bc(2.f * k.a3));
        auto dw = [&](f2 p) { return mul2(fma2(fma2(p, bc(4.f), bc(-6.f)), p, bc(2.f)), p); };  // 2p(1-p)(1-2p)
        f2 F1 = fma2(mul2(p1, p3s), k2, dw(p1));
        F1 = fma2(mul2(p1, p2s), k3, F1);
        F1 = fma2(fma2(G1, o1w, sub2(Cq, Bq)), bc(k.lam), F1);
        f2 F2 = fma2(mul2(s13, s13), mul2(fma2(p2, bc(2.f * k.b), bc(3.f)), bc(k.a2)), dw(p2));
        F2 = fma2(mul2(p2, p1s), k3, F2);
        F2 = fma2(fma2(G2, o2w, sub2(A, Cq)), bc(k.lam), F2);
        f2 F3 = fma2(mul2(p3, p1s), k2, dw(p3));
        F3 = fma2(mul2(s12, s12), mul2(fma2(p3, bc(2.f * k.b), bc(3.f)), bc(k.a3)), F3);
        F3 = fma2(fma2(G3, o3w, sub2(Bq, A)), bc(k.lam), F3);
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
        const f2 lap1 = lap(p1, x1p, x1m, y1p, y1m, z1p, z1m), lap2 = lap(p2, x2p, x2m, y2p, y2m, z2p, z2m);
        // phi_i' = phi_i + dt lap_i - dt (2F_i - F_j - F_k) / 3  (TiAg.cu:529-537)
        const f2 T3 = mul2(add2(add2(F1, F2), F3), bc(k.dt3));
        const f2 n1 = fma2(F1, bc(-k.dt), add2(T3, fma2(lap1, bc(k.dt), p1)));
        const f2 n2 = fma2(F2, bc(-k.dt), add2(T3, fma2(lap2, bc(k.dt), p2)));
        // solute: c' = c + sum_d cf_d (M+ (mu+ - mu) + M- (mu- - mu)), M = phi1 + phi1'
        // (+ solid terms), TiAg.cu:543-552
        auto mob = [&](f2 q1, f2 q2) {
          f2 m = add2(p1, q1);
          if constexpr (SD) {
            m = fma2(add2(p2, q2), bc(k.Da), m);
            m = fma2(sub2(sub2(add2(p3, bc(1.f)), q1), q2), bc(k.Db), m);
          }
          return m;
        };
        auto face2 = [&](f2 qp1, f2 qp2, f2 mp, f2 qm1, f2 qm2, f2 mm) {
          return fma2(mob(qp1, qp2), sub2(mp, m0), mul2(mob(qm1, qm2), sub2(mm, m0)));
        };
        f2 nc = fma2(face2(x1p, x2p, mxp, x1m, x2m, mxm), bc(k.cfx), ld2(cc + e));
        nc = fma2(face2(y1p, y2p, myp, y1m, y2m, mym), bc(k.cfy), nc);
        nc = fma2(face2(z1p, z2p, mzp, z1m, z2m, mzm), bc(k.cfz), nc);
        store_pair(gy, n1, n2, nc);
      }
    }
  }
}

}  // namespace

int peri3d_x2_box_width() { return kX2BXin; }
int peri3d_x2_box_height() { return kX2BYin; }

int launch_peri3d_step_x2(const rs3_params &p, const P3Maps &m, float *o1, float *o2, float *oc, int64_t step,
                          int *err, cudaStream_t st) {
  X2K k;
  k.nx = p.nx;
  k.ny = p.ny;
  k.nz = p.nz;
  k.z_chunk = p.z_chunk > 0 ? p.z_chunk : 32;
  k.a1 = (float)p.a1;
  k.a2 = (float)p.a2;
  k.a3 = (float)p.a3;
  k.b = (float)p.b;
  k.lam = (float)p.lambda;
  k.Da = (float)p.Da;
  k.Db = (float)p.Db;
  k.r1 = (float)p.A1;
  k.r2 = (float)(-p.A1 - p.A2);
  k.r3 = (float)(-p.A1 + p.A2);
  k.dt = (float)p.dt;
  k.dt3 = (float)(p.dt / 3.0);
  k.dxi2 = (float)(p.dx_inv * p.dx_inv);
  k.dyi2 = (float)(p.dy_inv * p.dy_inv);
  k.dzi2 = (float)(p.dz_inv * p.dz_inv);
  k.cfx = (float)(0.5 * p.dt * p.alpha * p.dx_inv * p.dx_inv);
  k.cfy = (float)(0.5 * p.dt * p.alpha * p.dy_inv * p.dy_inv);
  k.cfz = (float)(0.5 * p.dt * p.alpha * p.dz_inv * p.dz_inv);
  k.B11 = p.B11;
  k.B12 = p.B12;
  k.B21 = p.B21;
  k.B22 = p.B22;
  k.T_ref = p.T_ref;
  k.G_T = p.G_T;
  k.V_T = p.V_T;
  k.z_T = p.z_T;
  k.r1d = p.A1;
  k.r2d = -p.A1 - p.A2;
  k.r3d = -p.A1 + p.A2;
  k.c_off = peri3d_c_offset(p);
  const bool a1 = p.a1 != 0.0, sd = p.Da != 0.0 || p.Db != 0.0;
  auto kfn = a1 ? (sd ? peri3d_x2_kernel<true, true> : peri3d_x2_kernel<true, false>)
                : (sd ? peri3d_x2_kernel<false, true> : peri3d_x2_kernel<false, false>);
  const size_t smem = sizeof(X2Smem) + 128;
  static std::atomic<unsigned long long> attr[4];
  const int which = (a1 ? 2 : 0) + (sd ? 1 : 0);
  if (!smem_limit_once((const void *)kfn, (int)smem, attr[which])) return -3;
  const dim3 grid((p.nx + kX2BX - 1) / kX2BX, (p.ny - 2 + kX2BY - 1) / kX2BY, (p.nz - 2 + k.z_chunk - 1) / k.z_chunk);
  kfn<<<grid, kX2Threads, smem, st>>>(k, m.phi1, m.phi2, m.c, o1, o2, oc, step, err);
  return 0;
}

}  // namespace rs

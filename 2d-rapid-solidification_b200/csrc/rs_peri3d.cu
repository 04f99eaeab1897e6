// rs_peri3d.cu — the 3D three-phase (peritectic) step on one GPU.
//
// Model: multi/peritectic_multiGPU/TiAg.cu — stored phi1 (liquid), phi2
// (solid alpha), phi3 = 1 - phi1 - phi2 (solid beta); mu = c - sum r_i g_i
// (computeMu, TiAg.cu:461-470); the update of phi1, phi2, c (diffuse,
// TiAg.cu:503-561); periodic x, y and no-flux z ghost layers (TiAg.cu:472-500,
// 565-605).  The reference runs five kernels per step (computeMu, three
// boundaryMu, diffuse) plus three boundary kernels and keeps mu as a field;
// here one kernel does the step and mu never leaves shared memory.
//
// The FP32 step runs on packed FP32 pairs (rs_peri3d_x2.cu); this file's
// step kernel is the FP64 one.
// Kernel: a CTA owns a column of BX x BY output cells (x, y) and marches
// through a chunk of z planes.  Every input plane (BX+4 (FP32) or BX+2 (FP64)
// columns x BY+2 rows of phi1, phi2 and c) arrives by one 3D TMA box per
// field into a four-slot ring; the load of plane z+2 is in flight while plane
// z is computed.  mu of each plane (tile plus x/y halo) is computed once into
// a four-slot ring.  Outputs go straight to global memory (32 consecutive x
// per warp), and each output that a ghost cell images (x = 1, nx-2; y = 1,
// ny-2; z = 1, nz-2) is written to its ghost cells too, which is what the
// reference's boundary kernels leave there.
// Algorithmic bytes per cell-step: 3 fields read + 3 written.
#include <cuda.h>

#include "rs_peri3d_common.cuh"

namespace rs {
namespace {

template <typename R>
struct P3Smem {
  alignas(128) R in[kP3Slots][3][P3Cfg<R>::kPlaneAl];  // [slot][field][row][col]
  alignas(16) R mu[kP3MuSlots][P3Cfg<R>::kPlane];
  uint64_t full[kP3Slots];
  int melt[8];  // per plane (q mod 8): the box is pure melt inside the array (p3_melt)
};

// mu = c - sum_i r_i g_i (computeMu, TiAg.cu:461-470)
template <typename R>
__device__ __forceinline__ R mu_of(const K3<R> &k, R p1, R p2, R c) {
  const R p3 = R(1) - p1 - p2;
  return c - k.r1 * g3(p1, p2, p3) - k.r2 * g3(p2, p3, p1) - k.r3 * g3(p3, p1, p2);
}

// SD: solid diffusivities Da or Db non-zero (the reference sets both to 0)
template <typename R, bool SD>
__global__ void __launch_bounds__(kP3Threads, sizeof(R) == 4 ? 3 : 2)
    peri3d_kernel(const __grid_constant__ K3<R> k, const __grid_constant__ CUtensorMap m1,
                  const __grid_constant__ CUtensorMap m2, const __grid_constant__ CUtensorMap mc,
                  R *__restrict__ o1, R *__restrict__ o2, R *__restrict__ oc, const int64_t step, int *err) {
  using C = P3Cfg<R>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  P3Smem<R> &sm = *reinterpret_cast<P3Smem<R> *>(smem_raw);
  const int tid = threadIdx.x;
  const int xb = C::BX * blockIdx.x;   // first box column (array x); outputs xb+1 .. xb+BX
  const int yb = kP3BY * blockIdx.y;   // first box row (array y); outputs yb+1 .. yb+BY
  const int zo0 = 1 + k.z_chunk * blockIdx.z;                 // first output plane
  const int zo1 = min(zo0 + k.z_chunk, k.nz - 1);            // one past the last
  if (zo0 >= zo1) return;
  const int zin0 = zo0 - 1, zin1 = zo1;  // input planes zin0 .. zin1
  constexpr uint32_t kBytes = 3u * C::kPlane * sizeof(R);
  if (smem_u32(smem_raw) & 127u) {
    if (tid == 0) atomicExch(err, 2);
    return;
  }
  static_assert((P3Cfg<R>::kPlaneAl * sizeof(R)) % 128 == 0, "TMA destinations 128-byte aligned");
  auto issue = [&](int z) {  // plane z into its ring slot
    const int q = z - zin0, s = q % kP3Slots;
    mbar_expect_tx(&sm.full[s], kBytes);
    tma_load_3d(&sm.in[s][0][0], &m1, &sm.full[s], xb, yb, z);
    tma_load_3d(&sm.in[s][1][0], &m2, &sm.full[s], xb, yb, z);
    tma_load_3d(&sm.in[s][2][0], &mc, &sm.full[s], xb, yb, z);
  };
  if (tid == 0) {
    for (int s = 0; s < kP3Slots; ++s) mbar_init(&sm.full[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    for (int z = zin0; z <= min(zin1, zin0 + kP3Slots - 1); ++z) issue(z);
    for (int s = 0; s < 8; ++s) sm.melt[s] = 1;
  }
  __syncthreads();
  int issued = min(zin1, zin0 + kP3Slots - 1);  // last plane whose load was issued
  // mu of plane z into its slot (tile and halo); false if its load never came
  auto mu_plane = [&](int z) {
    const int q = z - zin0, s = q % kP3Slots;
    const bool got = p3_wait<R>(&sm.full[s], (uint32_t)((q / kP3Slots) & 1), err);
    R *mu = sm.mu[q % kP3MuSlots];
    const R *f1 = sm.in[s][0], *f2 = sm.in[s][1], *fc = sm.in[s][2];
    if (got) {
      bool all_melt = true;
      for (int e = tid; e < C::kPlane; e += kP3Threads) {
        mu[e] = mu_of(k, f1[e], f2[e], fc[e]);
        all_melt = all_melt && p3_melt_cell(k, f1[e], f2[e], xb + e % C::BXin, yb + e / C::BXin);
      }
      if (!all_melt) sm.melt[q & 7] = 0;
    }
    return got;
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

  // this thread's cells: column ix, a strip of K consecutive rows (the y
  // neighbours of the strip come from a register window)
  constexpr int K = C::kCellsPerThread;
  const int ix = tid % C::BX, iy0 = (tid / C::BX) * K;
  const int gx = xb + 1 + ix;  // array x of the output
  const bool xin = gx <= k.nx - 2;
  const int xg = gx == k.nx - 2 ? 0 : (gx == 1 ? k.nx - 1 : -1);  // ghost column it images
  const int64_t plane = (int64_t)k.nx * k.ny;
  const R third = R(1) / R(3);

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
    // the plane's B1, B2 (TiAg.cu:61-62) with the frozen T of this step
    const double Tz = k.G_T == 0.0 ? k.T_ref : k.T_ref + k.G_T * ((double)z - k.z_T - k.V_T * (double)step);
    const double B1 = k.B11 + k.B12 * Tz, B2 = k.B21 + k.B22 * Tz;
    const R s1 = (R)B1, s2 = (R)(-B1 - B2), s3 = (R)(-B1 + B2);
    const int zg = z == 1 ? 0 : (z == k.nz - 2 ? k.nz - 1 : -1);
    // the cell and every ghost cell that images it
    auto store_cell = [&](int gy, R n1, R n2, R nc) {
      const int yg = gy == k.ny - 2 ? 0 : (gy == 1 ? k.ny - 1 : -1);
      if ((xg & yg & zg) < 0) {  // no ghost cell images this one
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
      // pure melt (p3_melt_cell): phi1, phi2 stay 1 and 0 and the face
      // mobilities are 2, the values the general form gives bit for bit
      const int e0 = (iy0 + 1) * C::BXin + ix + 1;
      R wm[K + 2];
  #pragma unroll
      for (int r = 0; r < K + 2; ++r) wm[r] = mu[e0 + (r - 1) * C::BXin];
  #pragma unroll
      for (int r = 0; r < K; ++r) {
        const int gy = yb + 1 + iy0 + r;
        if (gy > k.ny - 2) break;
        const int e = e0 + r * C::BXin;
        const R m0 = wm[r + 1];
        const R jx = R(2) * (mu[e + 1] - m0) - R(2) * (m0 - mu[e - 1]);
        const R jy = R(2) * (wm[r + 2] - m0) - R(2) * (m0 - wm[r]);
        const R jz = R(2) * (muu[e] - m0) - R(2) * (m0 - mud[e]);
        store_cell(gy, R(1), R(0), cc[e] + (k.cfx * jx + k.cfy * jy + k.cfz * jz));
      }
    } else if (xin) {
      const int e0 = (iy0 + 1) * C::BXin + ix + 1;  // box element of the strip's first cell
      R w1[K + 2], w2[K + 2], wm[K + 2];            // the strip's column, rows iy0-1 .. iy0+K
  #pragma unroll
      for (int r = 0; r < K + 2; ++r) {
        const int e = e0 + (r - 1) * C::BXin;
        w1[r] = c1[e];
        w2[r] = c2[e];
        wm[r] = mu[e];
      }
  #pragma unroll
      for (int r = 0; r < K; ++r) {
        const int gy = yb + 1 + iy0 + r;
        if (gy > k.ny - 2) break;
        const int e = e0 + r * C::BXin;
        const R p1 = w1[r + 1], p2 = w2[r + 1], m0 = wm[r + 1], p3 = R(1) - p1 - p2;
        const R d12 = p1 - p2, d23 = p2 - p3, d31 = p3 - p1;
        // chemical driving forces (fcphi, TiAg.cu:514-516), with
        // gp1(pi, pj, pk) = G_i and gp2(pi, pj, pk) = Q_i (pj - pk)
        const R Q1 = R(7.5) * (p1 - R(1)) * (p1 * p1), Q2 = R(7.5) * (p2 - R(1)) * (p2 * p2),
                Q3 = R(7.5) * (p3 - R(1)) * (p3 * p3);
        const R G1 = R(3.75) * p1 * ((((R(3) * p1 - R(4)) * p1 - R(1)) * p1 + R(2)) + (R(3) * p1 - R(2)) * (d23 * d23));
        const R G2 = R(3.75) * p2 * ((((R(3) * p2 - R(4)) * p2 - R(1)) * p2 + R(2)) + (R(3) * p2 - R(2)) * (d31 * d31));
        const R G3 = R(3.75) * p3 * ((((R(3) * p3 - R(4)) * p3 - R(1)) * p3 + R(2)) + (R(3) * p3 - R(2)) * (d12 * d12));
        const R o1w = s1 - k.r1 * m0, o2w = s2 - k.r2 * m0, o3w = s3 - k.r3 * m0;
        const R A = Q1 * d23 * o1w, Bq = Q2 * d31 * o2w, Cq = Q3 * d12 * o3w;
        // multi-well terms (fphi, TiAg.cu:522-527) with their shared factors
        const R s12 = p1 * p2, s13 = p1 * p3, s23 = p2 * p3;
        const R U1 = R(3) * s23 + R(3) * p1 + k.b * (p1 * p1), U2 = R(3) * s13 + R(3) * p2 + k.b * (p2 * p2),
                U3 = R(3) * s12 + R(3) * p3 + k.b * (p3 * p3);
        const R F1 = R(2) * p1 * (R(1) - p1) * (R(1) - R(2) * p1) + k.a1 * (s23 * s23) * (R(3) + R(2) * k.b * p1) +
                     R(2) * k.a2 * p1 * (p3 * p3) * U2 + R(2) * k.a3 * p1 * (p2 * p2) * U3 +
                     k.lam * (G1 * o1w - Bq + Cq);
        const R F2 = R(2) * p2 * (R(1) - p2) * (R(1) - R(2) * p2) + R(2) * k.a1 * p2 * (p3 * p3) * U1 +
                     k.a2 * (s13 * s13) * (R(3) + R(2) * k.b * p2) + R(2) * k.a3 * p2 * (p1 * p1) * U3 +
                     k.lam * (A + G2 * o2w - Cq);
        const R F3 = R(2) * p3 * (R(1) - p3) * (R(1) - R(2) * p3) + R(2) * k.a1 * p3 * (p2 * p2) * U1 +
                     R(2) * k.a2 * p3 * (p1 * p1) * U2 + k.a3 * (s12 * s12) * (R(3) + R(2) * k.b * p3) +
                     k.lam * (-A + Bq + G3 * o3w);
        // neighbours
        const R x1p = c1[e + 1], x1m = c1[e - 1], x2p = c2[e + 1], x2m = c2[e - 1];
        const R z1p = u1[e], z1m = d1[e], z2p = u2[e], z2m = d2[e];
        const R lap1 = (x1p + x1m - R(2) * p1) * k.dxi2 + (w1[r + 2] + w1[r] - R(2) * p1) * k.dyi2 +
                       (z1p + z1m - R(2) * p1) * k.dzi2;
        const R lap2 = (x2p + x2m - R(2) * p2) * k.dxi2 + (w2[r + 2] + w2[r] - R(2) * p2) * k.dyi2 +
                       (z2p + z2m - R(2) * p2) * k.dzi2;
        // phi_i' = phi_i - dt (2 mu_i - mu_j - mu_k) / 3 with mu_i = F_i - lap_i and
        // lap_3 = -lap_1 - lap_2 (TiAg.cu:529-537)
        const R n1 = p1 + k.dt * (lap1 - (R(2) * F1 - F2 - F3) * third);
        const R n2 = p2 + k.dt * (lap2 - (R(2) * F2 - F1 - F3) * third);
        // solute: face mobility (phi1 + phi1') / 2 (+ solid terms), TiAg.cu:543-552
        auto mob = [&](R q1, R q2) {
          R m = p1 + q1;
          if constexpr (SD) m += k.Da2 * (p2 + q2) + k.Db2 * (p3 + R(1) - q1 - q2);
          return m;
        };
        const R jx = mob(x1p, x2p) * (mu[e + 1] - m0) - mob(x1m, x2m) * (m0 - mu[e - 1]);
        const R jy = mob(w1[r + 2], w2[r + 2]) * (wm[r + 2] - m0) - mob(w1[r], w2[r]) * (m0 - wm[r]);
        const R jz = mob(z1p, z2p) * (muu[e] - m0) - mob(z1m, z2m) * (m0 - mud[e]);
        const R nc = cc[e] + (k.cfx * jx + k.cfy * jy + k.cfz * jz);
        store_cell(gy, n1, n2, nc);
      }
    }
  }
}

// mu of every cell with image ghost layers (rs3_mu)
// (FP32 sets hold c - c_off: c_off is added back here and in the mass)
template <typename R>
__global__ void __launch_bounds__(256) peri3d_mu_kernel(const K3<R> k, const R *__restrict__ f1,
                                                        const R *__restrict__ f2, const R *__restrict__ fc,
                                                        R *__restrict__ mu, const double c_off) {
  const int64_t n = (int64_t)k.nx * k.ny * k.nz;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int x = (int)(i % k.nx), y = (int)((i / k.nx) % k.ny), z = (int)(i / ((int64_t)k.nx * k.ny));
    // image of a ghost cell: periodic x, y; no-flux z
    x = x == 0 ? k.nx - 2 : (x == k.nx - 1 ? 1 : x);
    y = y == 0 ? k.ny - 2 : (y == k.ny - 1 ? 1 : y);
    z = z == 0 ? 1 : (z == k.nz - 1 ? k.nz - 2 : z);
    const int64_t j = ((int64_t)z * k.ny + y) * k.nx + x;
    mu[i] = (R)((double)mu_of(k, f1[j], f2[j], fc[j]) + c_off);
  }
}

template <typename R>
__global__ void __launch_bounds__(256) peri3d_mass_kernel(const K3<R> k, const R *__restrict__ fc,
                                                          double *__restrict__ partial, const double c_off) {
  double s = 0.0;
  const int64_t nxi = k.nx - 2, nyi = k.ny - 2, n = nxi * nyi * (k.nz - 2);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t x = 1 + i % nxi, y = 1 + (i / nxi) % nyi, z = 1 + i / (nxi * nyi);
    s += (double)fc[(z * k.ny + y) * k.nx + x] + c_off;
  }
  __shared__ double sh[8];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t += sh[w];
    partial[blockIdx.x] = t;
  }
}

__global__ void peri3d_sum_kernel(const double *__restrict__ partial, int n, double *__restrict__ out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < n; ++i) t += partial[i];
    *out = t;
  }
}

// initial state (rs3_initial); one thread per (x, y) column of the interior
template <typename R>
__global__ void peri3d_init_kernel(const K3<R> k, const P3Init ini, R *__restrict__ f1, R *__restrict__ f2,
                                   R *__restrict__ fc, const double c_off) {
  const int x = 1 + blockIdx.x * blockDim.x + threadIdx.x, y = 1 + blockIdx.y;
  if (x > k.nx - 2 || y > k.ny - 2) return;
  uint32_t r[4] = {(uint32_t)x, (uint32_t)y, 0u, 0x5A465254u};
  philox4x32(r, (uint32_t)ini.seed, (uint32_t)(ini.seed >> 32));
  const double zc = ini.z_front + ini.amp * (2.0 * u53(r[0], r[1]) - 1.0);
  const int64_t plane = (int64_t)k.nx * k.ny;
  for (int z = 1; z <= k.nz - 2; ++z) {
    bool cap = false;
    if (z >= zc)
      for (int c = 0; c < ini.n_alpha; ++c) {
        const double dx = x - ini.cx[c], dy = y - ini.cy[c], dz = z - (ini.z_front - ini.roff);
        if (dx * dx + dy * dy + dz * dz <= ini.radius * ini.radius) cap = true;
      }
    const int64_t o = (int64_t)z * plane + (int64_t)y * k.nx + x;
    if (cap) {
      f1[o] = R(0);
      f2[o] = R(1);
      fc[o] = (R)(ini.ca - c_off);
    } else if (z < zc) {
      f1[o] = R(0);
      f2[o] = R(0);
      fc[o] = (R)(ini.cb - c_off);
    } else {
      f1[o] = R(1);
      f2[o] = R(0);
      fc[o] = (R)(ini.clb - c_off);
    }
  }
}

// ghost layers as images, in the reference's order (x, then y, then z)
template <typename R>
__global__ void peri3d_ghost_kernel(const K3<R> k, int axis, R *__restrict__ f1, R *__restrict__ f2,
                                    R *__restrict__ fc) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x, bidx = blockIdx.y;
  const int64_t plane = (int64_t)k.nx * k.ny;
  int64_t d0, s0, d1, s1;
  if (axis == 0) {  // (y, z) = (a, bidx)
    if (a >= k.ny || bidx >= k.nz) return;
    const int64_t base = (int64_t)bidx * plane + (int64_t)a * k.nx;
    d0 = base;
    s0 = base + k.nx - 2;
    d1 = base + k.nx - 1;
    s1 = base + 1;
  } else if (axis == 1) {  // (x, z)
    if (a >= k.nx || bidx >= k.nz) return;
    const int64_t base = (int64_t)bidx * plane + a;
    d0 = base;
    s0 = base + (int64_t)(k.ny - 2) * k.nx;
    d1 = base + (int64_t)(k.ny - 1) * k.nx;
    s1 = base + k.nx;
  } else {  // (x, y)
    if (a >= k.nx || bidx >= k.ny) return;
    const int64_t base = (int64_t)bidx * k.nx + a;
    d0 = base;
    s0 = base + plane;
    d1 = base + (int64_t)(k.nz - 1) * plane;
    s1 = base + (int64_t)(k.nz - 2) * plane;
  }
  f1[d0] = f1[s0];
  f2[d0] = f2[s0];
  fc[d0] = fc[s0];
  f1[d1] = f1[s1];
  f2[d1] = f2[s1];
  fc[d1] = fc[s1];
}

template <typename R>
int launch_step(const rs3_params &p, const P3Maps &m, R *o1, R *o2, R *oc, int64_t step, int *err, cudaStream_t st) {
  using C = P3Cfg<R>;
  const K3<R> k = make_k3<R>(p);
  const size_t smem = sizeof(P3Smem<R>) + 128;
  const bool sd = p.Da != 0.0 || p.Db != 0.0;
  auto kfn = sd ? peri3d_kernel<R, true> : peri3d_kernel<R, false>;
  static std::atomic<unsigned long long> attr[2];
  if (!smem_limit_once((const void *)kfn, (int)smem, attr[sd])) return -3;
  const dim3 grid((p.nx - 2 + C::BX - 1) / C::BX, (p.ny - 2 + kP3BY - 1) / kP3BY,
                  (p.nz - 2 + k.z_chunk - 1) / k.z_chunk);
  kfn<<<grid, kP3Threads, smem, st>>>(k, m.phi1, m.phi2, m.c, o1, o2, oc, step, err);
  return 0;
}

}  // namespace

double peri3d_c_offset(const rs3_params &p) {  // clb at T_ref (TiAg.cu:67); c_ref for energy 1
  if (p.energy == 1) return p.c_ref;
  const double B1 = p.B11 + p.B12 * p.T_ref, B2 = p.B21 + p.B22 * p.T_ref;
  return (B1 - 0.5 * B2) / (p.A1 - 0.5 * p.A2) + p.A1;
}

int peri3d_box_width(int precision) { return precision == RS_F64 ? P3Cfg<double>::BXin : peri3d_x2_box_width(); }
int peri3d_box_height(int precision) { return precision == RS_F64 ? kP3BY + 2 : peri3d_x2_box_height(); }

int launch_peri3d_step(const rs3_params &p, const P3Maps &m, int precision, void *o1, void *o2, void *oc,
                       int64_t step, int *err, cudaStream_t st) {
  if (precision == RS_F64)
    return launch_step<double>(p, m, (double *)o1, (double *)o2, (double *)oc, step, err, st);
  return launch_peri3d_step_x2(p, m, (float *)o1, (float *)o2, (float *)oc, step, err, st);
}

int launch_peri3d_mu(const rs3_params &p, int precision, const void *f1, const void *f2, const void *fc, void *mu,
                     cudaStream_t st) {
  const int64_t n = (int64_t)p.nx * p.ny * p.nz;
  const unsigned blocks = (unsigned)std::min<int64_t>((n + 255) / 256, 148 * 16);
  if (precision == RS_F64)
    peri3d_mu_kernel<double><<<blocks, 256, 0, st>>>(make_k3<double>(p), (const double *)f1, (const double *)f2,
                                                     (const double *)fc, (double *)mu, 0.0);
  else
    peri3d_mu_kernel<float><<<blocks, 256, 0, st>>>(make_k3<float>(p), (const float *)f1, (const float *)f2,
                                                    (const float *)fc, (float *)mu, peri3d_c_offset(p));
  return 0;
}

int launch_peri3d_mass(const rs3_params &p, int precision, const void *fc, double *partial, int nparts, double *out,
                       cudaStream_t st) {
  if (precision == RS_F64)
    peri3d_mass_kernel<double><<<nparts, 256, 0, st>>>(make_k3<double>(p), (const double *)fc, partial, 0.0);
  else
    peri3d_mass_kernel<float><<<nparts, 256, 0, st>>>(make_k3<float>(p), (const float *)fc, partial,
                                                      peri3d_c_offset(p));
  peri3d_sum_kernel<<<1, 32, 0, st>>>(partial, nparts, out);
  return 0;
}

int launch_peri3d_init(const rs3_params &p, int precision, const P3Init &ini, void *f1, void *f2, void *fc,
                       cudaStream_t st) {
  const dim3 g((p.nx - 2 + 127) / 128, p.ny - 2);
  if (precision == RS_F64)
    peri3d_init_kernel<double><<<g, 128, 0, st>>>(make_k3<double>(p), ini, (double *)f1, (double *)f2, (double *)fc,
                                                  0.0);
  else
    peri3d_init_kernel<float><<<g, 128, 0, st>>>(make_k3<float>(p), ini, (float *)f1, (float *)f2, (float *)fc,
                                                 peri3d_c_offset(p));
  return launch_peri3d_ghosts(p, precision, f1, f2, fc, st);
}

int launch_peri3d_ghosts(const rs3_params &p, int precision, void *f1, void *f2, void *fc, cudaStream_t st) {
  const int ext[3][2] = {{p.ny, p.nz}, {p.nx, p.nz}, {p.nx, p.ny}};
  for (int axis = 0; axis < 3; ++axis) {
    const dim3 gg((ext[axis][0] + 127) / 128, ext[axis][1]);
    if (precision == RS_F64)
      peri3d_ghost_kernel<double><<<gg, 128, 0, st>>>(make_k3<double>(p), axis, (double *)f1, (double *)f2,
                                                      (double *)fc);
    else
      peri3d_ghost_kernel<float><<<gg, 128, 0, st>>>(make_k3<float>(p), axis, (float *)f1, (float *)f2, (float *)fc);
  }
  return 0;
}

}  // namespace rs

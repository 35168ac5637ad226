// les_learned.cuh -- kernels of the learned sub-grid closure inside the RK3
// stage (imodel = LES_SGS_LEARNED).
//
// The network is evaluated at the cell centres of the physical (unpadded)
// grid.  Per stage:
//   1. k_lgrad_y: y-inverse transforms of the nine velocity-gradient spectra
//      at every level (x-spectral, y-physical), with the level combinations
//      of the staggered grid applied in spectral space:
//        ux, vx = i kx u^, i kx v^;  uy, vy = i ky u^, i ky v^
//        wx, wy = i k (w^(k) + w^(k-1)) / 2        (w-levels k-1, k; w(0) = w(nnz) = 0)
//        wz     = (w^(k) - w^(k-1)) / dz
//        uz, vz = (u^(k+1) - u^(k-1)) / (2 dz), one-sided at k = 1 and nnz
//                 (the centred average of the w-level differences with
//                  UZ(0) = UZ(1) and UZ(nnz) = UZ(nnz-1), as derivs1.f90 /
//                  derivs2.f90 set the wall rows)
//   2. k_learned_row: inverse x transforms, normalised bf16 features, the
//      network on the tensor cores, tau_ij and the per-CTA sums of the
//      dissipation -tau_ij S_ij, forward x transforms of tau (one kernel,
//      nothing in between goes to HBM);
//   3. k_learned_flag: plane-and-level mean of the dissipation (FP64, fixed
//      order); flag = 1 when it is >= 0, else 0 (Deardorff fallback);
//   ... the padded-grid kernels (their interior momentum stresses are
//      multiplied by 1 - flag) ...
//   4. k_col_small: y transforms of tau at every level;
//   5. k_ldiv: the stress divergence added to the new tendencies (when flag):
//        ru += -i kx tau11^ - i ky tau12^ - (tau13w^(k) - tau13w^(k-1)) / dz
//        rv += -i kx tau12^ - i ky tau22^ - (tau23w^(k) - tau23w^(k-1)) / dz
//        rw += -i kx tau13w^ - i ky tau23w^ - (tau33^(k+1) - tau33^(k)) / dz   (w-levels)
//      with tau13w(k) = (tau13(k) + tau13(k+1)) / 2 on the w-levels 2..nnz-2
//      and 0 on the walls and the wall-adjacent w-levels 1 and nnz-1: there
//      the padded kernels keep the wall model's and the Deardorff shear
//      stresses (the network, trained on cell-centre stresses, under-predicts
//      the flux through the first face, and coarse runs lose their near-wall
//      velocity without this).
// The kinetic-energy equation keeps the Deardorff eddy diffusivity.
#pragma once
#include "les_kernels.cuh"
#include "les_mlp.cuh"

namespace les {

// Feature order: (ux, vx, wx, uy, vy, wy, uz, vz, wz) = plane j of the
// gradient planes, then z+, then Delta.
template <class T, int N>
__global__ void __launch_bounds__(ColCfg<N, T>::THREADS)
k_lgrad_y(const cx<T>* __restrict__ uh, const cx<T>* __restrict__ vh, const cx<T>* __restrict__ wh,
          cx<T>* __restrict__ gy, int KX, int NZ, T kx0, T ky0, T dzm, const cx<T>* __restrict__ tw) {
  using C = ColCfg<N, T>;
  extern __shared__ __align__(16) unsigned char smraw[];
  cx<T>* sm = reinterpret_cast<cx<T>*>(smraw);
  const int z = blockIdx.y + 1;  // cell centre 1..NZ
  const int f = blockIdx.z;      // feature plane 0..8
  const int c0 = blockIdx.x * C::TC;
  const size_t nm = (size_t)N * KX;
  auto at = [&](const cx<T>* a, int k, size_t o) -> cx<T> { return a[(size_t)(k - 1) * nm + o]; };
  auto wl = [&](int k, size_t o) -> cx<T> {  // w-level k, zero on the walls
    return (k >= 1 && k <= NZ - 1) ? at(wh, k, o) : zero_cx<T>();
  };
  fft_core<N, +1, true, false, false>(C::TC, sm, tw, [&](int t, int n) -> cx<T> {
    const int kx = c0 + t;
    if (kx >= KX || n == N / 2) return zero_cx<T>();
    const size_t o = (size_t)n * KX + kx;
    const T xk = kx0 * (T)kx, yk = ky0 * (T)signed_k(n, N);
    switch (f) {
      case 0: return mul_i(at(uh, z, o)) * xk;
      case 1: return mul_i(at(vh, z, o)) * xk;
      case 2: return mul_i(wl(z, o) + wl(z - 1, o)) * ((T)0.5 * xk);
      case 3: return mul_i(at(uh, z, o)) * yk;
      case 4: return mul_i(at(vh, z, o)) * yk;
      case 5: return mul_i(wl(z, o) + wl(z - 1, o)) * ((T)0.5 * yk);
      case 6:
      case 7: {
        const cx<T>* a = (f == 6) ? uh : vh;
        if (z == 1) return (at(a, 2, o) - at(a, 1, o)) * dzm;
        if (z == NZ) return (at(a, NZ, o) - at(a, NZ - 1, o)) * dzm;
        return (at(a, z + 1, o) - at(a, z - 1, o)) * ((T)0.5 * dzm);
      }
      default: return (wl(z, o) - wl(z - 1, o)) * dzm;
    }
  }, [&](int t, int k, cx<T> v) {
    const int kx = c0 + t;
    if (kx < KX) gy[((size_t)f * NZ + (z - 1)) * nm + (size_t)k * KX + kx] = v;
  });
}

__device__ __forceinline__ float bf_lo(uint32_t u) { return __uint_as_float(u << 16); }
__device__ __forceinline__ float bf_hi(uint32_t u) { return __uint_as_float(u & 0xffff0000u); }

// ---------------------------------------------------------------------------
// The learned stage's x-direction work in one persistent kernel per SM: for
// a block of RB rows (one level z, consecutive y) of the gradient spectra
// from k_lgrad_y it does
//   1. the inverse x transforms of the nine gradient rows (five complex
//      transforms per row, two real rows each, as k_row_c2r),
//   2. the normalised bf16 features, one sample per thread (thread i =
//      point i of the block = row i%128 of group i/128's tile),
//   3. the network on the tensor cores (mlp_tile, four groups),
//   4. tau_ij and the dissipation -tau_ij S_ij (as MlpOutTau),
//   5. the forward x transforms of the six tau rows with the real-pair
//      separation of k_row_r2c, written as x-spectral rows th[6][NZ][NY][KX]
//      (kx < nx/2, unscaled) for the y transforms of k_col_small.
// Nothing between steps 1 and 5 goes to HBM.
// ---------------------------------------------------------------------------
template <int NX> struct LearnedRow {
  static constexpr int N1 = Split<NX>::N1, N2 = Split<NX>::N2, M12 = N1 > N2 ? N1 : N2;
  static constexpr int RB0 = 512 / NX, RB1 = 512 / (5 * M12);
  static constexpr int RB = (RB0 < RB1 ? RB0 : RB1) > 0 ? (RB0 < RB1 ? RB0 : RB1) : 1;  // rows per block
  template <class T> static constexpr size_t fft_bytes() {
    return (size_t)smem_fft_elems<NX, false>(5 * RB) * sizeof(cx<T>);
  }
  template <class T> static constexpr size_t smem() {
    return sizeof(MlpDev) + (size_t)4 * 16384 + fft_bytes<T>() + 256;
  }
};

template <class T, int NX>
__global__ void __launch_bounds__(512, 1)
k_learned_row(const MlpDev* __restrict__ prm, const cx<T>* __restrict__ gy, cx<T>* __restrict__ th, int NY,
              int NZ, T delta, T dz, T zl, T zplus_per_len, const cx<T>* __restrict__ tw,
              double* __restrict__ dissip_part, int* __restrict__ err) {
  using L = LearnedRow<NX>;
  constexpr int KX = NX / 2, RB = L::RB, NTI = 5 * RB, NTF = 3 * RB;
  extern __shared__ __align__(1024) unsigned char smraw_tc[];
  MlpDev* P = reinterpret_cast<MlpDev*>(smraw_tc);
  unsigned char* act_all = smraw_tc + sizeof(MlpDev);
  cx<T>* fb = reinterpret_cast<cx<T>*>(act_all + 4 * 16384);
  uint64_t* bars = reinterpret_cast<uint64_t*>(act_all + 4 * 16384 + L::template fft_bytes<T>());
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 4);
  double* red = reinterpret_cast<double*>(bars + 5);

  const int tid = threadIdx.x, g = tid >> 7, r = tid & 127, warp = tid >> 5, q = warp & 3;
  for (int i = tid; i < (int)(sizeof(MlpDev) / 16); i += blockDim.x)
    reinterpret_cast<uint4*>(P)[i] = reinterpret_cast<const uint4*>(prm)[i];
  if (tid < 4) tc::mbar_init(&bars[tid], 1);
  if (warp == 0) {
    tc::tmem_alloc(tslot, 256);
    tc::tmem_relinquish();
  }
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = *tslot;
  MlpGroup grp = mlp_group(P, act_all + (size_t)g * 16384, tbase, g, q, &bars[g]);

  const size_t R = (size_t)NZ * NY;
  const size_t plane = R * KX;
  double dsum = 0.0;
  bool failed = false;
  for (size_t r0 = (size_t)blockIdx.x * RB; r0 < R; r0 += (size_t)gridDim.x * RB) {
    // 1. inverse x transforms: transform t = 5*rr + j packs gradient rows 2j, 2j+1 of row r0+rr
    fft_core<NX, +1, false, false, true>(NTI, fb, tw, [&](int t, int n) -> cx<T> {
      const int rr = t / 5, j = t - 5 * rr;
      const size_t row = r0 + rr;
      if (row >= R) return zero_cx<T>();
      int k = n;
      bool mir = false;
      if (k >= KX) {
        if (NX - k < KX) { k = NX - k; mir = true; }
        else k = -1;
      }
      if (k < 0) return zero_cx<T>();
      cx<T> a = gy[(size_t)(2 * j) * plane + row * KX + k];
      cx<T> b = (j < 4) ? gy[(size_t)(2 * j + 1) * plane + row * KX + k] : zero_cx<T>();
      if (k == 0) { a.y = 0; b.y = 0; }
      if (mir) { a = conj(a); b = conj(b); }
      return mk(a.x - b.y, a.y + b.x);
    }, NoStore{});
    // 2. features of this thread's point
    const int rr = tid / NX, x = tid - (tid / NX) * NX;
    const size_t row = r0 + rr;
    const bool valid = (tid < RB * NX) && (row < R);
    uint4 f0 = make_uint4(0, 0, 0, 0), f1 = f0;
    if (valid) {
      T gv[9];
#pragma unroll
      for (int j = 0; j < 5; j++) {
        const cx<T> v = fb[(size_t)(5 * rr + j) * NX + x];
        gv[2 * j] = v.x;
        if (j < 4) gv[2 * j + 1] = v.y;
      }
      const int z = (int)(row / NY);
      const T zc = ((T)z + (T)0.5) * dz;
      const T zw = zc < zl - zc ? zc : zl - zc;
      float f[11];
#pragma unroll
      for (int j = 0; j < 9; j++) f[j] = (float)((gv[j] * delta - (T)P->in_shift[j]) * (T)P->in_scale[j]);
      f[9] = (float)((zw * zplus_per_len - (T)P->in_shift[9]) * (T)P->in_scale[9]);
      f[10] = (float)((delta - (T)P->in_shift[10]) * (T)P->in_scale[10]);
      f0 = make_uint4(pack_bf2(f[0], f[1]), pack_bf2(f[2], f[3]), pack_bf2(f[4], f[5]), pack_bf2(f[6], f[7]));
      f1 = make_uint4(pack_bf2(f[8], f[9]), pack_bf2(f[10], 0.f), 0u, 0u);
    }
    __syncthreads();  // every gradient read from fb before tau is written there
    // 3. the network
    float y[16];
    const bool ok = mlp_tile(grp, P, r, f0, f1, y);
    if (!ok) mlp_tile_failed(grp, r, err);
    // 4. tau into the forward transform rows: (tau11, tau12), (tau22, tau33), (tau13, tau23)
    if (valid && ok) {
      float t[6];
#pragma unroll
      for (int i = 0; i < 6; i++) t[i] = y[i] * P->out_scale[i] + P->out_shift[i];
      fb[(size_t)(3 * rr + 0) * NX + x] = mk((T)t[0], (T)t[3]);
      fb[(size_t)(3 * rr + 1) * NX + x] = mk((T)t[1], (T)t[2]);
      fb[(size_t)(3 * rr + 2) * NX + x] = mk((T)t[4], (T)t[5]);
      const float qv[9] = {bf_lo(f0.x), bf_hi(f0.x), bf_lo(f0.y), bf_hi(f0.y), bf_lo(f0.z),
                           bf_hi(f0.z), bf_lo(f0.w), bf_hi(f0.w), bf_lo(f1.x)};
      float gg[9];
#pragma unroll
      for (int j = 0; j < 9; j++) gg[j] = qv[j] / P->in_scale[j] + P->in_shift[j];
      const float s11 = gg[0], s22 = gg[4], s33 = gg[8];
      const float s12 = 0.5f * (gg[3] + gg[1]), s13 = 0.5f * (gg[6] + gg[2]), s23 = 0.5f * (gg[7] + gg[5]);
      dsum -= (double)t[0] * s11 + (double)t[1] * s22 + (double)t[2] * s33 +
              2.0 * ((double)t[3] * s12 + (double)t[4] * s13 + (double)t[5] * s23);
    }
    if (__syncthreads_or(!ok)) { failed = true; break; }
    // 5. forward x transforms and the real-pair separation
    fft_core<NX, -1, false, true, true>(NTF, fb, tw, NoLoad{}, NoStore{});
    for (int i = tid; i < NTF * KX; i += blockDim.x) {
      const int t = i / KX, k = i - t * KX;
      const int rr2 = t / 3, j = t - 3 * rr2;
      const size_t row2 = r0 + rr2;
      if (row2 >= R) continue;
      const cx<T> zk = fb[(size_t)t * NX + k], zm = conj(fb[(size_t)t * NX + (NX - k) % NX]);
      const cx<T> a = (zk + zm) * (T)0.5;
      const cx<T> d = zk - zm;
      const int fa = (j == 0) ? 0 : (j == 1 ? 1 : 4);  // tau11 | tau22 | tau13
      const int fbi = (j == 0) ? 3 : (j == 1 ? 2 : 5); // tau12 | tau33 | tau23
      th[(size_t)fa * plane + row2 * KX + k] = a;
      th[(size_t)fbi * plane + row2 * KX + k] = mk(d.y * (T)0.5, -d.x * (T)0.5);
    }
    __syncthreads();
  }
  (void)failed;
  for (int o = 16; o > 0; o >>= 1) dsum += __shfl_xor_sync(0xffffffffu, dsum, o);
  if ((tid & 31) == 0) red[warp] = dsum;
  tc::fence_before_sync();
  __syncthreads();
  if (tid == 0) {
    double sacc = 0.0;
    for (int w = 0; w < 16; w++) sacc += red[w];
    dissip_part[blockIdx.x] = sacc;
  }
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tbase, 256);
  }
}

// Mean dissipation (per-CTA sums in CTA order) -> flag and status.
static __global__ void k_learned_flag(const double* __restrict__ part, int nparts, double inv_n_delta,
                                      int* __restrict__ flag, double* __restrict__ status) {
  if (threadIdx.x != 0) return;
  double s = 0.0;
  for (int i = 0; i < nparts; i++) s += part[i];
  const double mean = s * inv_n_delta;
  const int use = (mean >= 0.0) ? 1 : 0;  // NaN -> fallback
  flag[0] = use;
  status[0] = mean;
  status[1] = (double)use;
}

// Stress divergence of the network's tau (spectral, all levels) into the
// new tendencies, when the stage uses the network.
template <class T>
__global__ void k_ldiv(const cx<T>* __restrict__ th, cx<T>* __restrict__ run, cx<T>* __restrict__ rvn,
                       cx<T>* __restrict__ rwn, const int* __restrict__ flag, StageArgs a) {
  if (!flag[0]) return;
  const int KX = a.KX, NY = a.NY, NZ = a.NZ;
  const int nm = KX * NY;
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  const int z = blockIdx.y + 1;
  if (m >= nm) return;
  const int ky = m / KX, kx = m - ky * KX;
  if (ky == NY / 2) return;
  const T xk = (T)(a.kx0 * kx), yk = (T)(a.ky0 * signed_k(ky, NY)), dzm = (T)a.dzm;
  auto tf = [&](int f, int k) -> cx<T> { return th[((size_t)f * NZ + (k - 1)) * nm + m]; };
  auto t13w = [&](int k) -> cx<T> { return (k >= 2 && k <= NZ - 2) ? (tf(4, k) + tf(4, k + 1)) * (T)0.5 : zero_cx<T>(); };
  auto t23w = [&](int k) -> cx<T> { return (k >= 2 && k <= NZ - 2) ? (tf(5, k) + tf(5, k + 1)) * (T)0.5 : zero_cx<T>(); };
  const size_t o = (size_t)(z - 1) * nm + m;
  const cx<T> du = mul_i(tf(0, z)) * (-xk) - mul_i(tf(3, z)) * yk - (t13w(z) - t13w(z - 1)) * dzm;
  const cx<T> dv = mul_i(tf(3, z)) * (-xk) - mul_i(tf(1, z)) * yk - (t23w(z) - t23w(z - 1)) * dzm;
  run[o] = run[o] + du;
  rvn[o] = rvn[o] + dv;
  if (z <= NZ - 1) {
    const cx<T> dw = mul_i(t13w(z)) * (-xk) - mul_i(t23w(z)) * yk - (tf(2, z + 1) - tf(2, z)) * dzm;
    rwn[o] = rwn[o] + dw;
  }
}

}  // namespace les

namespace les {

// ---------------------------------------------------------------------------
// Training data of the learned closure: explicit filtering of a fine run.
// z: box average over the fz fine cells of each coarse cell (fz = 1 or 2);
// x, y: the box filter of width Delta_c (the coarse cell) as the spectral
// transfer sin(k Delta_c / 2) / (k Delta_c / 2), then truncation to the
// coarse modes (|kx| < nxc/2, |ky| < nyc/2; the truncation of redim.f90:
// 277-318 without its Nyquist rows).  Filtered quantities at the coarse
// cell centres: u, v, wc, uu, vv, wc wc, u v, u wc, v wc (wc = w averaged to
// the fine centres), and w at the coarse w-levels (fz = 2: weights 1/4,
// 1/2, 1/4 of the fine w-levels 2K-1, 2K, 2K+1).
// ---------------------------------------------------------------------------
// With G (the fine run's nine gradient planes at the cell centres, [9][NZ][ps])
// and E (its TKE at the w-levels, plane k = level k), the fine run's own
// Deardorff stress -2 nu_t S_ij, nu_t = 0.1 dsl sqrt(max(e_c, emin)) with e_c
// the average of the two faces of the cell (faces 0 and nnz take the values
// of faces 1 and nnz-1), is added to the products before filtering, so the
// stresses come out as the filtered total sub-filter stress.
template <class T>
__global__ void k_filt_z(const T* __restrict__ U, const T* __restrict__ V, const T* __restrict__ W,
                         const T* __restrict__ G, const T* __restrict__ E, T dsl, T emin, T* __restrict__ S,
                         long long ps, int NZ, int NZc, int fz) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int K = blockIdx.y + 1;
  if (p >= ps) return;
  auto w = [&](int k) -> T { return (k >= 1 && k <= NZ - 1) ? W[(size_t)(k - 1) * ps + p] : (T)0; };
  auto ef = [&](int k) -> T {
    k = k < 1 ? 1 : (k > NZ - 1 ? NZ - 1 : k);
    return E[(size_t)k * ps + p];
  };
  const size_t N = (size_t)NZ * ps;
  T q[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int j = 0; j < fz; j++) {
    const int k = fz * (K - 1) + 1 + j;
    const T u = U[(size_t)(k - 1) * ps + p], v = V[(size_t)(k - 1) * ps + p];
    const T wc = (T)0.5 * (w(k) + w(k - 1));
    q[0] += u; q[1] += v; q[2] += wc;
    q[3] += u * u; q[4] += v * v; q[5] += wc * wc;
    q[6] += u * v; q[7] += u * wc; q[8] += v * wc;
    if (G) {
      const size_t o = (size_t)(k - 1) * ps + p;
      T g[9];
#pragma unroll
      for (int i = 0; i < 9; i++) g[i] = G[i * N + o];  // ux, vx, wx, uy, vy, wy, uz, vz, wz
      T ec = (T)0.5 * (ef(k) + ef(k - 1));
      ec = ec > emin ? ec : emin;
      const T nu2 = (T)0.2 * dsl * sqrt(ec);
      q[3] -= nu2 * g[0];
      q[4] -= nu2 * g[4];
      q[5] -= nu2 * g[8];
      q[6] -= nu2 * (T)0.5 * (g[3] + g[1]);
      q[7] -= nu2 * (T)0.5 * (g[6] + g[2]);
      q[8] -= nu2 * (T)0.5 * (g[7] + g[5]);
    }
  }
  const T inv = (T)1 / (T)fz;
  const size_t plane = (size_t)NZc * ps;
#pragma unroll
  for (int i = 0; i < 9; i++) S[i * plane + (size_t)(K - 1) * ps + p] = q[i] * inv;
  const T wst = (fz == 2) ? (T)0.25 * w(2 * K - 1) + (T)0.5 * w(2 * K) + (T)0.25 * w(2 * K + 1) : w(K);
  S[9 * plane + (size_t)(K - 1) * ps + p] = wst;
}

__host__ __device__ inline double box_transfer(double k, double width) {
  const double a = 0.5 * k * width;
  return a == 0.0 ? 1.0 : sin(a) / a;
}

// fine spectra [plane][NY][KX] -> coarse spectra [plane][NYc][KXc]
template <class T>
__global__ void k_filt_trunc(const cx<T>* __restrict__ F, cx<T>* __restrict__ C, int NY, int KX, int NYc, int KXc,
                             double kx0, double ky0, double wx, double wy) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  const int pl = blockIdx.y;
  if (m >= NYc * KXc) return;
  const int kyc = m / KXc, kxc = m - kyc * KXc;
  cx<T> v = zero_cx<T>();
  if (kyc != NYc / 2) {
    const int sk = signed_k(kyc, NYc);
    const int kyf = sk >= 0 ? sk : NY + sk;
    const double g = box_transfer(kx0 * kxc, wx) * box_transfer(ky0 * sk, wy);
    v = F[(size_t)pl * NY * KX + (size_t)kyf * KX + kxc] * (T)g;
  }
  C[(size_t)pl * NYc * KXc + m] = v;
}

// coarse filtered planes [10][N] -> out [9][N] (double):
// u, v, w (w-levels), tau11, tau22, tau33, tau12, tau13, tau23
template <class T>
__global__ void k_filt_tau(const T* __restrict__ Q, double* __restrict__ out, long long N) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  const double u = Q[p], v = Q[N + p], wc = Q[2 * N + p];
  out[p] = u;
  out[N + p] = v;
  out[2 * N + p] = Q[9 * N + p];
  out[3 * N + p] = Q[3 * N + p] - u * u;
  out[4 * N + p] = Q[4 * N + p] - v * v;
  out[5 * N + p] = Q[5 * N + p] - wc * wc;
  out[6 * N + p] = Q[6 * N + p] - u * v;
  out[7 * N + p] = Q[7 * N + p] - u * wc;
  out[8 * N + p] = Q[8 * N + p] - v * wc;
}

// raw features f32 [N][16]: 9 gradients * Delta, z+, Delta, zeros
template <class T>
__global__ void k_lfeat_raw(const T* __restrict__ g, float4* __restrict__ feat, long long N, long long plane, T delta,
                            T dz, T zl, T zplus_per_len) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  const int z = (int)(p / plane);
  const T zc = ((T)z + (T)0.5) * dz;
  const T zw = zc < zl - zc ? zc : zl - zc;
  float f[16];
#pragma unroll
  for (int j = 0; j < 9; j++) f[j] = (float)(g[(size_t)j * N + p] * delta);
  f[9] = (float)(zw * zplus_per_len);
  f[10] = (float)delta;
#pragma unroll
  for (int j = 11; j < 16; j++) f[j] = 0.f;
#pragma unroll
  for (int j = 0; j < 4; j++) feat[4 * p + j] = make_float4(f[4 * j], f[4 * j + 1], f[4 * j + 2], f[4 * j + 3]);
}

}  // namespace les

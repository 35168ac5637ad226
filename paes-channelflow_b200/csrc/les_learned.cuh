// les_learned.cuh -- kernels of the learned sub-grid closure inside the RK3
// stage (imodel = LES_SGS_LEARNED).
//
// The network is evaluated at the cell centres of the physical (unpadded)
// grid.  Per stage:
//   1. k_lgrad_y: y-inverse transforms (x-spectral, y-physical rows) of
//      u^, i ky u^, v^, i ky v^, w^, i ky w^ at every level;
//   2. k_lgrad_x: the nine velocity gradients at the cell centres from
//      those rows (the level combinations of the staggered grid and i kx
//      applied while loading the inverse x transforms):
//        ux, vx = i kx U, i kx V;  uy, vy = UY, VY
//        wx, wy = (i kx, 1) (W(k) + W(k-1)) / 2   (w-levels, w(0) = w(nnz) = 0)
//        wz     = (W(k) - W(k-1)) / dz
//        uz, vz = (U(k+1) - U(k-1)) / (2 dz), one-sided at k = 1 and nnz
//                 (the centred average of the w-level differences with
//                  UZ(0) = UZ(1) and UZ(nnz) = UZ(nnz-1), as derivs1.f90 /
//                  derivs2.f90 set the wall rows)
//      and from them the normalised bf16 features (or raw f32 features):
//      the closure is dimensionless, so that one network serves every grid
//      and filter width:
//        inputs  x_j = g_j / |G| (j = 0..8, g the nine gradients, |G| their
//                Frobenius norm), min(z_w / Delta, kZwCap), z_w / h
//                (z_w the distance to the nearest wall, h = zl / 2)
//        outputs c_ij, tau_ij = (Delta |G|)^2 c_ij
//      (an eddy viscosity is the special case c = -2 C^2 (|S|/|G|) S/|G|);
//      Delta |G| rides along in bf16 columns 11 (high part) and 12 (the
//      rounding remainder), which the network's padded first layer ignores;
//   3. k_mlp_infer<MlpOutTau>: tau_ij on the tensor cores with its local
//      backscatter removed (the component along S where tau:S > 0), and
//      per CTA the sums of the raw network's dissipation -tau_ij S_ij, of
//      the applied one and of the reference (C_s Delta)^2 |S|^3 (the
//      Smagorinsky estimate with Lilly's constant C_s = 0.17);
//   4. k_learned_flag: the means (FP64, fixed order); flag = 1 when the
//      raw network's is >= 0 and (guard > 0) the applied one lies within a
//      factor guard of the reference, else 0 (Deardorff fallback);
//   ... the padded-grid kernels (their interior momentum stresses are
//      multiplied by 1 - flag) ...
//   5. k_row_r2c + k_col_small: tau^ at every level;
//   6. k_ldiv: the stress divergence added to the new tendencies (when flag):
//        ru += -i kx tau11^ - i ky tau12^ - (tau13w^(k) - tau13w^(k-1)) / dz
//        rv += -i kx tau12^ - i ky tau22^ - (tau23w^(k) - tau23w^(k-1)) / dz
//        rw += -i kx tau13w^ - i ky tau23w^ - (tau33^(k+1) - tau33^(k)) / dz   (w-levels)
//      with tau13w(k) = (tau13(k) + tau13(k+1)) / 2 on the interior w-levels
//      and 0 on the walls (the wall model's stresses stay in the padded
//      kernels), plus a compact-stencil correction of the shear stresses
//      that damps the odd-even modes the averaged centre stresses cannot see
//      (k_ldiv).
// The kinetic-energy equation keeps the Deardorff eddy diffusivity.
#pragma once
#include "les_kernels.cuh"
#include "les_mlp.cuh"

namespace les {

// Blocks of k_lgrad_y: H = ColCfg's column count (64-byte row segments of
// the spectra), H transforms: the field or its y derivative.
template <int N, class T> struct LgyCfg {
  static constexpr int H = ColCfg<N, T>::TC;
  static constexpr int THREADS = H * Split<N>::N2;
  static constexpr size_t smem() { return (size_t)H * N * sizeof(cx<T>); }
};

// y-inverse rows gy[f][z][y][kx], f = 0..5: U, UY, V, VY, W, WY.  A block
// takes H columns of one component (blockIdx.z: u, v, w) at one level and
// transforms the field (d = blockIdx.x & 1 = 0) or its y derivative (d = 1);
// the two blocks of a column group are adjacent in launch order, so the
// second reads the spectral values from L2.
template <class T, int N>
__global__ void __launch_bounds__(LgyCfg<N, T>::THREADS)
k_lgrad_y(const cx<T>* __restrict__ uh, const cx<T>* __restrict__ vh, const cx<T>* __restrict__ wh,
          cx<T>* __restrict__ gy, int KX, int NZ, T ky0, const cx<T>* __restrict__ tw) {
  constexpr int H = LgyCfg<N, T>::H;
  extern __shared__ __align__(16) unsigned char smraw[];
  cx<T>* sm = reinterpret_cast<cx<T>*>(smraw);
  const int z = blockIdx.y + 1;
  const int c = blockIdx.z, d = blockIdx.x & 1;
  const int c0 = (blockIdx.x >> 1) * H;
  const size_t nm = (size_t)N * KX;
  const cx<T>* src = (c == 0 ? uh : (c == 1 ? vh : wh)) + (size_t)(z - 1) * nm;
  const bool zero = (c == 2 && z == NZ);  // w(nnz) = 0
  cx<T>* out = gy + ((size_t)(2 * c + d) * NZ + (z - 1)) * nm;
  fft_core<N, +1, true, false, false>(H, sm, tw, [&](int t, int n) -> cx<T> {
    const int kx = c0 + t;
    if (kx >= KX || n == N / 2 || zero) return zero_cx<T>();
    const cx<T> v = src[(size_t)n * KX + kx];
    return d ? mul_i(v) * (ky0 * (T)signed_k(n, N)) : v;
  }, [&](int t, int k, cx<T> v) {
    const int kx = c0 + t;
    if (kx < KX) out[(size_t)k * KX + kx] = v;
  });
}

// Rows per block of k_lgrad_x: five transforms per row, about 256 threads.
template <int NX> struct LgxCfg {
  static constexpr int N1 = Split<NX>::N1, N2 = Split<NX>::N2, M12 = N1 > N2 ? N1 : N2;
  static constexpr int RB = (256 / (5 * M12)) > 0 ? (256 / (5 * M12)) : 1;
  static constexpr int THREADS = 5 * RB * M12;
  static constexpr int BUF = smem_fft_elems<NX, false>(5 * RB);
  // transform buffer + the staged spectra (direct and mirrored combination
  // of each of the 5*RB transforms at kx < NX/2)
  template <class T> static constexpr size_t smem() { return (size_t)(BUF + 10 * RB * (NX / 2)) * sizeof(cx<T>); }
};

// Cap of the wall-distance input z_w / Delta: farther from the wall than
// kZwCap filter widths the closure sees one value.
constexpr float kZwCap = 16.0f;

// Gradients and features at the cell centres of RB rows (one level, RB
// consecutive y) per block.  RAW: f32 [N][16] unnormalised features
// x_0..x_10, Delta |G| in column 11, zeros in 12..15; otherwise bf16
// [N][16]: x_0..x_10 normalised with P's in_shift / in_scale, Delta |G| as
// bf16 high part (column 11) and remainder (column 12), zeros in 13..15.
// x order: (ux, vx, wx, uy, vy, wy, uz, vz, wz) / |G|, min(z_w/Delta,
// kZwCap), z_w / h.
template <class T, int NX, bool RAW>
__global__ void __launch_bounds__(LgxCfg<NX>::THREADS)
k_lgrad_x(const cx<T>* __restrict__ gy, void* __restrict__ feat, const MlpDev* __restrict__ P, int NY, int NZ,
          T kx0, T dzm, T delta, T dz, T zl, T inv_h, const cx<T>* __restrict__ tw) {
  using L = LgxCfg<NX>;
  constexpr int KX = NX / 2, RB = L::RB;
  extern __shared__ __align__(16) unsigned char smraw[];
  cx<T>* sm = reinterpret_cast<cx<T>*>(smraw);
  const int R = NZ * NY;
  const size_t plane = (size_t)R * KX;
  const int r0 = blockIdx.x * RB;
  // level (0-based) and y of the block's first row; row r0 + rr is at
  // y0 + rr, carried into the next level past NY - 1 (RB <= NY)
  const int zb = r0 / NY, y0 = r0 - zb * NY;
  auto row_zy = [&](int rr, int& z, int& y) {
    y = y0 + rr;
    z = zb;
    if (y >= NY) { y -= NY; z++; }
  };
  // row of field f at level k (1..NZ) and y
  auto rowp = [&](int f, int k, int y) -> const cx<T>* { return gy + (size_t)f * plane + ((size_t)(k - 1) * NY + y) * KX; };
  // Stage 1: the spectral combinations a + i b of the five transforms of
  // each row at kx = 0..KX-1, loaded once (coalesced along kx), kept as the
  // direct value (position kx) and the conjugate-symmetric one (NX - kx).
  cx<T>* zd = sm + L::BUF;             // [5*RB][KX]
  cx<T>* zm = zd + (size_t)5 * RB * KX;  // [5*RB][KX]
  for (int i = threadIdx.x; i < 5 * RB * KX; i += blockDim.x) {
    const int t = i / KX, k = i - t * KX;
    const int rr = t / 5, j = t - 5 * rr;
    cx<T> d = zero_cx<T>(), m = zero_cx<T>();
    if (r0 + rr < R) {
      int z, y;
      row_zy(rr, z, y);
      z += 1;
      const T xk = kx0 * (T)k;
      auto wl = [&](int f, int kk) -> cx<T> { return (kk >= 1 && kk <= NZ - 1) ? rowp(f, kk, y)[k] : zero_cx<T>(); };
      auto vz = [&](int f) -> cx<T> {
        if (z == 1) return (rowp(f, 2, y)[k] - rowp(f, 1, y)[k]) * dzm;
        if (z == NZ) return (rowp(f, NZ, y)[k] - rowp(f, NZ - 1, y)[k]) * dzm;
        return (rowp(f, z + 1, y)[k] - rowp(f, z - 1, y)[k]) * ((T)0.5 * dzm);
      };
      cx<T> a, b;
      switch (j) {
        case 0: a = mul_i(rowp(0, z, y)[k]) * xk; b = mul_i(rowp(2, z, y)[k]) * xk; break;      // ux, vx
        case 1: a = mul_i(wl(4, z) + wl(4, z - 1)) * ((T)0.5 * xk); b = rowp(1, z, y)[k]; break; // wx, uy
        case 2: a = rowp(3, z, y)[k]; b = (wl(5, z) + wl(5, z - 1)) * (T)0.5; break;            // vy, wy
        case 3: a = vz(0); b = vz(2); break;                                                    // uz, vz
        default: a = (wl(4, z) - wl(4, z - 1)) * dzm; b = zero_cx<T>(); break;                  // wz
      }
      if (k == 0) { a.y = 0; b.y = 0; }
      d = mk(a.x - b.y, a.y + b.x);  // a + i b
      m = mk(a.x + b.y, b.x - a.y);  // conj(a) + i conj(b)
    }
    zd[i] = d;
    zm[i] = m;
  }
  __syncthreads();
  // Stage 2: the inverse transforms from the staged spectra
  fft_core<NX, +1, false, false, true>(5 * RB, sm, tw, [&](int t, int n) -> cx<T> {
    if (n < KX) return zd[(size_t)t * KX + n];
    if (NX - n < KX) return zm[(size_t)t * KX + (NX - n)];
    return zero_cx<T>();
  }, NoStore{});
  // the feature normalisation, read once per thread
  float nsh[11], nsc[11];
#pragma unroll
  for (int jj = 0; jj < 11; jj++) {
    nsh[jj] = RAW ? 0.f : P->in_shift[jj];
    nsc[jj] = RAW ? 1.f : P->in_scale[jj];
  }
  for (int i = threadIdx.x; i < RB * NX; i += blockDim.x) {
    const int rr = i / NX, x = i - rr * NX;
    if (r0 + rr >= R) continue;
    T g[9];
#pragma unroll
    for (int j = 0; j < 5; j++) {
      const cx<T> v = sm[(size_t)(5 * rr + j) * NX + x];
      g[2 * j] = v.x;
      if (j < 4) g[2 * j + 1] = v.y;
    }
    int z, y;
    row_zy(rr, z, y);
    const T zc = ((T)z + (T)0.5) * dz;
    const T zw = zc < zl - zc ? zc : zl - zc;
    const size_t p = (size_t)(r0 + rr) * NX + x;
    T g2 = (T)0;
#pragma unroll
    for (int j = 0; j < 9; j++) g2 += g[j] * g[j];
    const T gm = sqrt(g2);
    const T rg = gm > (T)0 ? (T)1 / gm : (T)0;
    T xin[11];
#pragma unroll
    for (int j = 0; j < 9; j++) xin[j] = g[j] * rg;
    const T zd = zw / delta;
    xin[9] = zd < (T)kZwCap ? zd : (T)kZwCap;
    xin[10] = zw * inv_h;
    const float sc = (float)(gm * delta);  // Delta |G|
    if constexpr (RAW) {
      float4* o = reinterpret_cast<float4*>(feat) + 4 * p;
      o[0] = make_float4((float)xin[0], (float)xin[1], (float)xin[2], (float)xin[3]);
      o[1] = make_float4((float)xin[4], (float)xin[5], (float)xin[6], (float)xin[7]);
      o[2] = make_float4((float)xin[8], (float)xin[9], (float)xin[10], sc);
      o[3] = make_float4(0.f, 0.f, 0.f, 0.f);
    } else {
      float f[11];
#pragma unroll
      for (int jj = 0; jj < 11; jj++) f[jj] = (float)((xin[jj] - (T)nsh[jj]) * (T)nsc[jj]);
      const __nv_bfloat16 shi = __float2bfloat16_rn(sc);
      const float slo = sc - __bfloat162float(shi);
      uint4* o = reinterpret_cast<uint4*>(feat) + 2 * p;
      o[0] = make_uint4(pack_bf2(f[0], f[1]), pack_bf2(f[2], f[3]), pack_bf2(f[4], f[5]), pack_bf2(f[6], f[7]));
      o[1] = make_uint4(pack_bf2(f[8], f[9]), pack_bf2(f[10], sc), pack_bf2(slo, 0.f), 0u);
    }
  }
}

__device__ __forceinline__ float bf_lo(uint32_t u) { return __uint_as_float(u << 16); }
__device__ __forceinline__ float bf_hi(uint32_t u) { return __uint_as_float(u & 0xffff0000u); }

// Delta |G| from the bf16 columns 11 (high part) and 12 (remainder).
__device__ __forceinline__ float feat_scale(uint4 f1) { return bf_hi(f1.y) + bf_lo(f1.z); }

// Squared constant of the reference dissipation (C_s Delta)^2 |S|^3 of the
// fallback test: Lilly's inertial-range Smagorinsky constant C_s = 0.17.
constexpr double kRefCs2 = 0.17 * 0.17;

// Network outputs -> tau planes [6][N] (tau11, tau22, tau33, tau12, tau13,
// tau23).  The network's stress is tau = (Delta |G|)^2 (y * out_scale +
// out_shift); where it would transfer energy from the sub-filter scales to
// the resolved ones (tau_ij S_ij > 0, local backscatter) its component
// along S is removed, tau' = tau - (tau:S / S:S) S, so that the applied
// stress never injects energy at a point (-tau':S = max(-tau:S, 0)).
// Planes 6, 7: tau13' g_uz + tau23' g_vz and g_uz^2 + g_vz^2 (g = the
// gradients times Delta, for the network's effective viscosity).  Returns,
// each times Delta (k_learned_flag divides the sums by N Delta): the raw
// network's dissipation -tau:S, the applied -tau':S, and the reference
// (C_s Delta)^2 |S|^3.
template <class T> struct MlpOutTau {
  T* tau;  // [8][N]
  long long N;
  __device__ double3 operator()(long long p, bool valid, const float (&y)[16], uint4 f0, uint4 f1,
                                const MlpDev* P) const {
    if (!valid) return make_double3(0.0, 0.0, 0.0);
    const float s = feat_scale(f1);
    const float s2 = s * s;
    float t[6];
#pragma unroll
    for (int i = 0; i < 6; i++) t[i] = s2 * (y[i] * P->out_scale[i] + P->out_shift[i]);
    const float q[9] = {bf_lo(f0.x), bf_hi(f0.x), bf_lo(f0.y), bf_hi(f0.y), bf_lo(f0.z),
                        bf_hi(f0.z), bf_lo(f0.w), bf_hi(f0.w), bf_lo(f1.x)};
    float g[9];
#pragma unroll
    for (int j = 0; j < 9; j++) g[j] = (q[j] * P->in_rscale[j] + P->in_shift[j]) * s;  // d_i u_j * Delta
    // per-point arithmetic in f32 (the network's own precision is bf16); the
    // sums over the points are accumulated in f64 by the caller
    const float sv[6] = {g[0], g[4], g[8], 0.5f * (g[3] + g[1]), 0.5f * (g[6] + g[2]), 0.5f * (g[7] + g[5])};
    const float ss = sv[0] * sv[0] + sv[1] * sv[1] + sv[2] * sv[2] +
                     2.0f * (sv[3] * sv[3] + sv[4] * sv[4] + sv[5] * sv[5]);  // S:S
    const float ts = t[0] * sv[0] + t[1] * sv[1] + t[2] * sv[2] +
                     2.0f * (t[3] * sv[3] + t[4] * sv[4] + t[5] * sv[5]);  // tau:S
    float applied = -ts;
    if (ts > 0.0f && ss > 0.0f) {
      const float a = -ts / ss;
#pragma unroll
      for (int i = 0; i < 6; i++) t[i] += a * sv[i];
      applied = 0.0f;
    }
#pragma unroll
    for (int i = 0; i < 6; i++) tau[(size_t)i * N + p] = (T)t[i];
    tau[(size_t)6 * N + p] = (T)(t[4] * g[6] + t[5] * g[7]);
    tau[(size_t)7 * N + p] = (T)(g[6] * g[6] + g[7] * g[7]);
    const float sm2 = 2.0f * ss;  // (|S| Delta)^2
    return make_double3((double)-ts, (double)applied, kRefCs2 * (double)(sm2 * sqrtf(sm2)));
  }
};

// Mean dissipations (per-CTA triples of sums in CTA order: the raw
// network's, the applied, the reference) -> flag, status [applied mean,
// flag, reference mean, raw mean] and the stage counters [stages, stages
// that used the network].  The network is used when its raw mean
// dissipation is >= 0 (NaN falls back) and, with guard > 0, the applied
// mean lies within a factor guard of the reference.
static __global__ void k_learned_flag(const double* __restrict__ part, int nparts, double inv_n_delta, double guard,
                                      int* __restrict__ flag, double* __restrict__ status,
                                      unsigned long long* __restrict__ counts) {
  if (threadIdx.x != 0) return;
  double sr = 0.0, sa = 0.0, sf = 0.0;
  for (int i = 0; i < nparts; i++) { sr += part[3 * i]; sa += part[3 * i + 1]; sf += part[3 * i + 2]; }
  const double raw = sr * inv_n_delta, applied = sa * inv_n_delta, ref = sf * inv_n_delta;
  int use = (raw >= 0.0) ? 1 : 0;  // NaN -> fallback
  if (guard > 0.0 && !(ref > 0.0 && applied <= guard * ref && guard * applied >= ref)) use = 0;
  flag[0] = use;
  status[0] = applied;
  status[1] = (double)use;
  status[2] = ref;
  status[3] = raw;
  counts[0] += 1ull;
  counts[1] += (unsigned long long)use;
}

// Per-level partial sums of tau planes 6 and 7 (MlpOutTau): grid (NZ,
// kNuChunks), partial [z][chunk][2], summed in chunk order by k_ldiv.
constexpr int kNuChunks = 16;
template <class T>
__global__ void k_learned_nu(const T* __restrict__ tau, double* __restrict__ part, size_t ps, long long N) {
  const int z = blockIdx.x;
  const size_t chunk = (ps + kNuChunks - 1) / kNuChunks;
  const size_t q0 = (size_t)blockIdx.y * chunk, q1 = q0 + chunk < ps ? q0 + chunk : ps;
  const T* A = tau + (size_t)6 * N + (size_t)z * ps;
  const T* B = tau + (size_t)7 * N + (size_t)z * ps;
  double sa = 0.0, sb = 0.0;
  for (size_t q = q0 + threadIdx.x; q < q1; q += blockDim.x) { sa += (double)A[q]; sb += (double)B[q]; }
  __shared__ double red[2][32];
  for (int o = 16; o > 0; o >>= 1) {
    sa += __shfl_xor_sync(0xffffffffu, sa, o);
    sb += __shfl_xor_sync(0xffffffffu, sb, o);
  }
  if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = sa; red[1][threadIdx.x >> 5] = sb; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double ta = 0.0, tb = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) { ta += red[0][w]; tb += red[1][w]; }
    part[((size_t)z * kNuChunks + blockIdx.y) * 2] = ta;
    part[((size_t)z * kNuChunks + blockIdx.y) * 2 + 1] = tb;
  }
}

// Face viscosity nu[j], j = 0..NZ, from the partial sums (chunk order):
// cell values -sum A / sum B * Delta clipped to [0, xkmax], face j = mean of
// cells j and j+1 (0 outside 2..NZ-2, where no correction is applied).
static __global__ void k_learned_nu_face(const double* __restrict__ part, double* __restrict__ nuf, int NZ,
                                         double dsl, double xkmax) {
  for (int j = threadIdx.x; j <= NZ; j += blockDim.x) {
    double v = 0.0;
    if (j >= 2 && j <= NZ - 2) {
      double c[2];
      for (int i = 0; i < 2; i++) {
        const int k = j + i;  // cells j, j+1 (1-based)
        double sa = 0.0, sb = 0.0;
        for (int q = 0; q < kNuChunks; q++) {
          sa += part[((size_t)(k - 1) * kNuChunks + q) * 2];
          sb += part[((size_t)(k - 1) * kNuChunks + q) * 2 + 1];
        }
        double nu = sb > 0.0 ? -sa / sb * dsl : 0.0;
        c[i] = nu < 0.0 ? 0.0 : (nu > xkmax ? xkmax : nu);
      }
      v = 0.5 * (c[0] + c[1]);
    }
    nuf[j] = v;
  }
}

// Stress divergence of the network's tau (spectral, all levels) into the
// new tendencies, when the stage uses the network.  On the faces 2..nnz-2
// (where the stencil fits) the shear stresses get the compact-stencil correction
//   -nu(j) (3 (u(j+1) - u(j)) - (u(j+2) - u(j-1))) / (4 dz)   (and for v):
// O(dz^2 u''') for smooth profiles, the diffusive flux -nu du/dz for the
// odd-even mode that the centre-to-face averaged network stress cannot see.
// nu is the network's own effective viscosity: per level
// -sum(tau13 uz + tau23 vz) / sum(uz^2 + vz^2), clipped to [0, xkmax],
// averaged to the face.
template <class T>
__global__ void k_ldiv(const cx<T>* __restrict__ th, cx<T>* __restrict__ run, cx<T>* __restrict__ rvn,
                       cx<T>* __restrict__ rwn, const cx<T>* __restrict__ uh, const cx<T>* __restrict__ vh,
                       const double* __restrict__ nuf, const int* __restrict__ flag, StageArgs a) {
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
  auto t13w = [&](int k) -> cx<T> { return (k >= 1 && k <= NZ - 1) ? (tf(4, k) + tf(4, k + 1)) * (T)0.5 : zero_cx<T>(); };
  auto t23w = [&](int k) -> cx<T> { return (k >= 1 && k <= NZ - 1) ? (tf(5, k) + tf(5, k + 1)) * (T)0.5 : zero_cx<T>(); };
  const size_t o = (size_t)(z - 1) * nm + m;
  auto lv = [&](const cx<T>* f, int k) -> cx<T> { return f[(size_t)(k - 1) * nm + m]; };
  auto tc = [&](const cx<T>* f, int j) -> cx<T> {
    if (j < 2 || j > NZ - 2) return zero_cx<T>();
    const cx<T> d3 = ((lv(f, j + 1) - lv(f, j)) * (T)3 - (lv(f, j + 2) - lv(f, j - 1))) * ((T)0.25 * dzm);
    return d3 * (T)(-nuf[j]);
  };
  const cx<T> du = mul_i(tf(0, z)) * (-xk) - mul_i(tf(3, z)) * yk - (t13w(z) - t13w(z - 1)) * dzm -
                   (tc(uh, z) - tc(uh, z - 1)) * dzm;
  const cx<T> dv = mul_i(tf(3, z)) * (-xk) - mul_i(tf(1, z)) * yk - (t23w(z) - t23w(z - 1)) * dzm -
                   (tc(vh, z) - tc(vh, z - 1)) * dzm;
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
// z: box average over the fz fine cells of each coarse cell (fz = 1 or even);
// x, y: the box filter of width Delta_c (the coarse cell) as the spectral
// transfer sin(k Delta_c / 2) / (k Delta_c / 2), then truncation to the
// coarse modes (|kx| < nxc/2, |ky| < nyc/2; the truncation of redim.f90:
// 277-318 without its Nyquist rows).  Filtered quantities at the coarse
// cell centres: u, v, wc, uu, vv, wc wc, u v, u wc, v wc (wc = w averaged to
// the fine centres), and w at the coarse w-levels: the box of width fz fine
// cells centred on the coarse face K (fine face fz K) by the trapezoid rule,
// weights 1/(2 fz) on the fine faces fz K -/+ fz/2 and 1/fz between (fz = 2:
// 1/4, 1/2, 1/4 of the fine w-levels 2K-1, 2K, 2K+1).
// ---------------------------------------------------------------------------
// With F (the fine run's raw features at the cell centres, f32 [NZ*ps][16]:
// columns 0..8 the gradients over |G|, column 11 dsl |G|)
// and E (its TKE at the w-levels, plane k = level k), the fine run's own
// Deardorff stress -2 nu_t S_ij, nu_t = 0.1 dsl sqrt(max(e_c, emin)) with e_c
// the average of the two faces of the cell (faces 0 and nnz take the values
// of faces 1 and nnz-1), is added to the products before filtering, so the
// stresses come out as the filtered total sub-filter stress.
template <class T>
__global__ void k_filt_z(const T* __restrict__ U, const T* __restrict__ V, const T* __restrict__ W,
                         const float* __restrict__ F, const T* __restrict__ E, T dsl, T emin, T* __restrict__ S,
                         long long ps, int NZ, int NZc, int fz) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int K = blockIdx.y + 1;
  if (p >= ps) return;
  auto w = [&](int k) -> T { return (k >= 1 && k <= NZ - 1) ? W[(size_t)(k - 1) * ps + p] : (T)0; };
  auto ef = [&](int k) -> T {
    k = k < 1 ? 1 : (k > NZ - 1 ? NZ - 1 : k);
    return E[(size_t)k * ps + p];
  };
  T q[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int j = 0; j < fz; j++) {
    const int k = fz * (K - 1) + 1 + j;
    const T u = U[(size_t)(k - 1) * ps + p], v = V[(size_t)(k - 1) * ps + p];
    const T wc = (T)0.5 * (w(k) + w(k - 1));
    q[0] += u; q[1] += v; q[2] += wc;
    q[3] += u * u; q[4] += v * v; q[5] += wc * wc;
    q[6] += u * v; q[7] += u * wc; q[8] += v * wc;
    if (F) {
      const size_t o = (size_t)(k - 1) * ps + p;
      T g[9];
      const T gs = (T)F[o * 16 + 11] / dsl;  // |G|
#pragma unroll
      for (int i = 0; i < 9; i++) g[i] = (T)F[o * 16 + i] * gs;  // ux, vx, wx, uy, vy, wy, uz, vz, wz
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
  T wst = w(K);
  if (fz > 1) {
    const int c = fz * K, hf = fz / 2;
    wst = (T)0.5 * (w(c - hf) + w(c + hf));
    for (int j = c - hf + 1; j < c + hf; j++) wst += w(j);
    wst *= inv;
  }
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

}  // namespace les

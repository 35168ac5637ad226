// les_kernels.cuh -- device kernels of one RK3 stage on a device-resident
// channel domain.
//
// State (spectral on the small grid, which represents exactly the
// Nyquist-free fields the reference carries after deal()):
//   uh, vh, wh        small spectra u^ = FFT2(u)/(nx*ny), [z][ky][kx], kx < nx/2
//   ruo, rvo, rwo     tendencies of the previous stage (spectral)
//   mu, mv, mru, mrv  FP64 shadows of the kx=ky=0 modes (mean profiles)
//   e, re             SGS TKE and its tendency in physical space (the e
//                     update clips at emin, comp2.f90:38)
// Work arrays on the 3/2-padded grid (nxb = 3nx/2, nyb = 3ny/2):
//   "mixed" arrays    x-spectral, y-physical  [z][y][kx]  (kx < nx/2)
//   "padded" arrays   physical                [z][y][x]
//
// One stage (les.F90:254-285) is:
//   k_e_prep, k_col_fwd_small   e ghosts + zeta update + spectrum of e
//   k_y_inverse, k_x_inverse    expand() of u, v, w, e fused with the
//                               spectral derivatives ux..ey (derivs1/2)
//   k_clip_y, k_clip_x          derivatives of max(E, emin) - E
//   k_wall_sums/final           plane means for sufsim / sufsim_upper
//   k_flux                      compadv1, complen, compsgs1, compsgs3
//                               pointwise, written as flux fields
//   k_x_forward, k_y_forward    compress() fused with -d/dx, -d/dy of the
//                               fluxes; the e part also inverts re
//   k_e_update                  e = max(e + dtab1*re, emin)
//   k_press                     comprhs + press (tridv) per (kx, ky), FP64
//   k_update                    comp2 in spectral space, FP64
#pragma once
#include <cooperative_groups.h>

#include "fft_core.cuh"
#include "les_tma.cuh"

namespace les {

// ---------------------------------------------------------------------------
// launch shapes
// ---------------------------------------------------------------------------
template <int N> struct RowCfg {
  static constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2;
  static constexpr int NT = (128 / N2) > 0 ? (128 / N2) : 1;  // row transforms per CTA
  static constexpr int THREADS = NT * N2;
  template <class T> static constexpr size_t smem() { return (size_t)smem_fft_elems<N, false>(NT) * sizeof(cx<T>); }
};
template <int N, class T> struct ColCfg {
  static constexpr int N2 = Split<N>::N2;
  static constexpr int TCB = (sizeof(T) == 8) ? 4 : 8;  // 64-byte row segments
  static constexpr int TC = (TCB * N2 >= 64) ? TCB : (64 / N2);
  static constexpr int THREADS = TC * N2;
  static constexpr size_t buf() { return (size_t)TC * N * sizeof(cx<T>); }
};

// Scalars of one stage (double; kernels cast).
struct StageArgs {
  int NX, NY, NZ, MX, MY, KX;
  int imodel, isurface, tke_production, zeta;
  int mnout_sgs;  // record the SGS means (mnout and istage == 1)
  double dz, dzm, dzm2, todzm, kx0, ky0;
  double emin, ceps, dsl, forcing, nu, xkmax;
  double dtab1, dtab2, dtabm;
  double zl, ugal, vgal;
};

// Wall-model scalars for one wall (lowerbc.f90:56-124 / upperbc.f90:63-122).
struct WallSide {
  double u1xy, v1xy, vsfc, utau, windm, ufluc2mroot, vfluc2mroot, suflucm, svflucm;
  double moengu2mroot, moengv2mroot, auuwm, auvwm, denom;
};
struct WallParams {
  WallSide w[2];  // 0 = lower (level 1), 1 = upper (level nnz)
  double dudt, dvdt, utau_s;
};

// Device error word bits.
constexpr int ERR_NAN = 1, ERR_UTAU = 2;

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------
template <class T> __device__ __forceinline__ T tmax(T a, T b) { return a > b ? a : b; }
template <class T> __device__ __forceinline__ T tmin(T a, T b) { return a < b ? a : b; }

// ---------------------------------------------------------------------------
// Generic small-grid transforms (upload, download, deal, expand, compress)
// ---------------------------------------------------------------------------

// Rows of real planes -> first KOUT complex modes of each row (unscaled).
// in: nrows rows of length N (row r at in + r*N); out: row r at out + r*KOUT.
template <class T, int N>
__global__ void __launch_bounds__(RowCfg<N>::THREADS)
k_row_r2c(const T* __restrict__ in, cx<T>* __restrict__ out, int nrows, int KOUT, const cx<T>* __restrict__ tw) {
  using C = RowCfg<N>;
  extern __shared__ __align__(16) unsigned char smraw[];
  cx<T>* sm = reinterpret_cast<cx<T>*>(smraw);
  const int p0 = blockIdx.x * C::NT;
  const int npair = (nrows + 1) / 2;
  fft_core<N, -1, false, false, true>(C::NT, sm, tw, [&](int t, int n) {
    int p = p0 + t;
    cx<T> v = zero_cx<T>();
    if (p < npair) v = mk(in[(size_t)(2 * p) * N + n], (2 * p + 1 < nrows) ? in[(size_t)(2 * p + 1) * N + n] : (T)0);
    return v;
  }, NoStore{});
  for (int i = threadIdx.x; i < C::NT * KOUT; i += blockDim.x) {
    int t = i / KOUT, k = i - t * KOUT, p = p0 + t;
    if (p >= npair) continue;
    cx<T> zk = sm[t * N + k], zm = conj(sm[t * N + (N - k) % N]);
    cx<T> a = (zk + zm) * (T)0.5;
    cx<T> d = zk - zm;
    out[(size_t)(2 * p) * KOUT + k] = a;
    if (2 * p + 1 < nrows) out[(size_t)(2 * p + 1) * KOUT + k] = mk(d.y * (T)0.5, -d.x * (T)0.5);
  }
}

// First KIN complex modes of each row (higher modes zero, imaginary parts of
// mode 0 ignored as in a c2r transform) -> real rows of length N.
template <class T, int N>
__global__ void __launch_bounds__(RowCfg<N>::THREADS)
k_row_c2r(const cx<T>* __restrict__ in, T* __restrict__ out, int nrows, int KIN, const cx<T>* __restrict__ tw) {
  using C = RowCfg<N>;
  extern __shared__ __align__(16) unsigned char smraw[];
  cx<T>* sm = reinterpret_cast<cx<T>*>(smraw);
  const int p0 = blockIdx.x * C::NT;
  const int npair = (nrows + 1) / 2;
  fft_core<N, +1, false, false, false>(C::NT, sm, tw, [&](int t, int n) {
    int p = p0 + t;
    cx<T> v = zero_cx<T>();
    if (p < npair) {
      int k = n;
      bool mir = false;
      if (k >= KIN) {
        if (N - k < KIN && N - k > 0 && N - k != N / 2) { k = N - k; mir = true; }
        else k = -1;
      }
      if (k >= 0) {
        cx<T> a = in[(size_t)(2 * p) * KIN + k];
        cx<T> b = (2 * p + 1 < nrows) ? in[(size_t)(2 * p + 1) * KIN + k] : zero_cx<T>();
        if (k == 0 || (2 * k == N)) { a.y = 0; b.y = 0; }
        if (mir) { a = conj(a); b = conj(b); }
        v = mk(a.x - b.y, a.y + b.x);
      }
    }
    return v;
  }, [&](int t, int n, cx<T> v) {
    int p = p0 + t;
    if (p >= npair) return;
    out[(size_t)(2 * p) * N + n] = v.x;
    if (2 * p + 1 < nrows) out[(size_t)(2 * p + 1) * N + n] = v.y;
  });
}

// Columns of x-spectral planes [plane][N][KX] (KX columns) -> forward DFT
// along y, times `scale`, Nyquist row N/2 dropped (deal semantics).
// With INV = true: inverse DFT, no scaling.
template <class T, int N, bool INV, bool DROP = !INV>
__global__ void __launch_bounds__(ColCfg<N, T>::THREADS)
k_col_small(const cx<T>* __restrict__ in, cx<T>* __restrict__ out, int KX, T scale, const cx<T>* __restrict__ tw) {
  using C = ColCfg<N, T>;
  extern __shared__ __align__(16) unsigned char smraw[];
  cx<T>* sm = reinterpret_cast<cx<T>*>(smraw);
  const size_t plane = (size_t)blockIdx.y * N * KX;
  const int kx0 = blockIdx.x * C::TC;
  // in-place use (in == out) is safe: every load of the tile precedes the
  // __syncthreads() inside fft_core that precedes every store
  fft_core<N, INV ? +1 : -1, true, false, false>(C::TC, sm, tw, [&](int t, int n) {
    int kx = kx0 + t;
    return (kx < KX) ? in[plane + (size_t)n * KX + kx] : zero_cx<T>();
  }, [&](int t, int k, cx<T> v) {
    int kx = kx0 + t;
    if (kx >= KX) return;
    if (!INV) v = (DROP && k == N / 2) ? zero_cx<T>() : v * scale;
    out[plane + (size_t)k * KX + kx] = v;
  });
}

// Padding / truncation between the small (N) and padded (M = 3N/2) y-grid,
// on x-spectral columns.
//   PAD:   small spectrum column (N) -> inverse DFT of the zero-padded
//          column (M) [expand]
//   TRUNC: padded column (M) -> forward DFT, keep |ky| < N/2, times scale,
//          inverse DFT of the small column (N) [compress]
template <class T, int NS>
__global__ void __launch_bounds__(ColCfg<3 * NS / 2, T>::THREADS)
k_col_pad(const cx<T>* __restrict__ in, cx<T>* __restrict__ out, int KX, const cx<T>* __restrict__ tw) {
  constexpr int M = 3 * NS / 2;
  using C = ColCfg<M, T>;
  extern __shared__ __align__(16) unsigned char smraw[];
  cx<T>* sm = reinterpret_cast<cx<T>*>(smraw);
  const int kx0 = blockIdx.x * C::TC;
  const cx<T>* src = in + (size_t)blockIdx.y * NS * KX;
  cx<T>* dst = out + (size_t)blockIdx.y * M * KX;
  fft_core<M, +1, true, false, false>(C::TC, sm, tw, [&](int t, int n) {
    int kx = kx0 + t;
    int ky = (n < NS / 2) ? n : ((n > NS) ? n - NS / 2 : -1);
    return (kx < KX && ky >= 0) ? src[(size_t)ky * KX + kx] : zero_cx<T>();
  }, [&](int t, int n, cx<T> v) {
    int kx = kx0 + t;
    if (kx < KX) dst[(size_t)n * KX + kx] = v;
  });
}

template <class T, int NS>
__global__ void __launch_bounds__(ColCfg<3 * NS / 2, T>::THREADS)
k_col_trunc(const cx<T>* __restrict__ in, cx<T>* __restrict__ out, int KX, T scale, const cx<T>* __restrict__ tw) {
  constexpr int M = 3 * NS / 2;
  using C = ColCfg<M, T>;
  extern __shared__ __align__(16) unsigned char smraw[];
  cx<T>* sm = reinterpret_cast<cx<T>*>(smraw);
  cx<T>* sm2 = sm + C::TC * M;
  const int kx0 = blockIdx.x * C::TC;
  const cx<T>* src = in + (size_t)blockIdx.y * M * KX;
  cx<T>* dst = out + (size_t)blockIdx.y * NS * KX;
  fft_core<M, -1, true, false, true>(C::TC, sm, tw, [&](int t, int n) {
    int kx = kx0 + t;
    return (kx < KX) ? src[(size_t)n * KX + kx] : zero_cx<T>();
  }, NoStore{});
  for (int i = threadIdx.x; i < C::TC * NS; i += blockDim.x) {
    int t = i % C::TC, ky = i / C::TC;
    int n = (ky < NS / 2) ? ky : ky + NS / 2;
    sm2[ky * C::TC + t] = (ky == NS / 2) ? zero_cx<T>() : sm[n * C::TC + t] * scale;
  }
  __syncthreads();
  fft_core<NS, +1, true, true, false>(C::TC, sm2, tw, NoLoad{}, [&](int t, int n, cx<T> v) {
    int kx = kx0 + t;
    if (kx < KX) dst[(size_t)n * KX + kx] = v;
  });
}

// ---------------------------------------------------------------------------
// Stage kernels
// ---------------------------------------------------------------------------
// lower/upper ghosts of e (lowerbc.f90:13-17, upperbc.f90:20-24), the
// zeta part of the stage for e (comp1.f90:131), and the x-transform of e
// (first half of expand, filter_fftw.f90:262-263).  e has levels 0..NZ+1.
template <class T, int NX>
__global__ void __launch_bounds__(RowCfg<NX>::THREADS)
k_e_prep(T* __restrict__ e, const T* __restrict__ re, cx<T>* __restrict__ Xe, int NY, int NZ, T dtab2, int zeta,
         const cx<T>* __restrict__ tw) {
  using C = RowCfg<NX>;
  constexpr int KX = NX / 2;
  extern __shared__ __align__(16) unsigned char smraw[];
  cx<T>* sm = reinterpret_cast<cx<T>*>(smraw);
  const int z = blockIdx.y + 1;  // 1..NZ-1
  const int p0 = blockIdx.x * C::NT;
  const size_t plane = (size_t)NY * NX;
  T* ez = e + (size_t)z * plane;
  fft_core<NX, -1, false, false, true>(C::NT, sm, tw, [&](int t, int n) {
    int p = p0 + t;
    return (p < NY / 2) ? mk(ez[(size_t)(2 * p) * NX + n], ez[(size_t)(2 * p + 1) * NX + n]) : zero_cx<T>();
  }, NoStore{});
  cx<T>* out = Xe + (size_t)(z - 1) * NY * KX;
  for (int i = threadIdx.x; i < C::NT * KX; i += blockDim.x) {
    int t = i / KX, k = i - t * KX, p = p0 + t;
    if (p >= NY / 2) continue;
    cx<T> zk = sm[t * NX + k], zm = conj(sm[t * NX + (NX - k) % NX]);
    cx<T> d = zk - zm;
    out[(size_t)(2 * p) * KX + k] = (zk + zm) * (T)0.5;
    out[(size_t)(2 * p + 1) * KX + k] = mk(d.y * (T)0.5, -d.x * (T)0.5);
  }
  for (int i = threadIdx.x; i < C::NT * NX; i += blockDim.x) {
    int t = i / NX, n = i - t * NX, p = p0 + t;
    if (p >= NY / 2) continue;
#pragma unroll
    for (int r = 0; r < 2; r++) {
      size_t off = (size_t)(2 * p + r) * NX + n;
      T val = ez[off];
      if (z == 1) e[off] = val;
      if (z == NZ - 1) {
        e[(size_t)NZ * plane + off] = val;
        e[(size_t)(NZ + 1) * plane + off] = val;
      }
      if (zeta) ez[off] = val - dtab2 * re[(size_t)(z - 1) * plane + off];
    }
  }
}

struct Ptr8 { void* p[8]; };
struct Ptr12 { void* p[12]; };

// expand() of u, v, w, e in y fused with d/dy: for field f = blockIdx.z
// (u, v, w, e), out[2f] = IFFT_M(pad(s)) and out[2f+1] = IFFT_M(i*ky*pad(s)),
// TC columns per block.  The field and its derivative go to separate blocks
// (h = blockIdx.x & 1), adjacent in launch order so that the second reads
// the columns from L2: half the block of a paired form, so that two blocks
// share an SM and one's loads overlap the other's transform and stores
// (measured 22% faster in FP32 than TC paired transforms per block).
// Thread 0 of a field block first has the TMA prefetch into L2 the columns
// of the field block `pdist` blocks ahead (les_tma.cuh; maps: tensor maps of
// src[0..3] as [NZ*NS][KX] rows; pdist 0 prefetches nothing).
template <class T, int NS>
__global__ void __launch_bounds__(ColCfg<3 * NS / 2, T>::THREADS)
k_y_inverse(Ptr8 src, Ptr8 dst, int KX, int NZ, T ky0, const cx<T>* __restrict__ tw,
            const __grid_constant__ ColMaps maps, unsigned pdist) {
  constexpr int M = 3 * NS / 2;
  using C = ColCfg<M, T>;
  if ((blockIdx.x & 1) == 0)
    prefetch_tile_ahead<T, NS, C::TC>(maps, pdist, [&](unsigned bx, unsigned by, unsigned bz, int& q, int& cg,
                                                       int& row0) {
      q = (int)bz; cg = (int)(bx >> 1); row0 = (int)by * NS;
      return !(bz >= 2 && (int)by + 1 == NZ);
    });
  extern __shared__ __align__(16) unsigned char smraw[];
  cx<T>* sm = reinterpret_cast<cx<T>*>(smraw);
  const int f = blockIdx.z, h = blockIdx.x & 1, z = blockIdx.y + 1;
  if (f >= 2 && z == NZ) return;
  const int kx0 = (blockIdx.x >> 1) * C::TC;
  const cx<T>* in = reinterpret_cast<const cx<T>*>(src.p[f]) + (size_t)(z - 1) * NS * KX;
  cx<T>* out = reinterpret_cast<cx<T>*>(dst.p[2 * f + h]) + (size_t)(z - 1) * M * KX;
  fft_core<M, +1, true, false, false>(C::TC, sm, tw, [&](int t, int n) {
    const int kx = kx0 + t;
    const int ky = (n < NS / 2) ? n : ((n > NS) ? n - NS / 2 : -1);
    cx<T> v = (kx < KX && ky >= 0) ? in[(size_t)ky * KX + kx] : zero_cx<T>();
    if (h) v = mul_i(v) * (ky0 * (T)signed_k(n, M));
    return v;
  }, [&](int t, int n, cx<T> v) {
    const int kx = kx0 + t;
    if (kx < KX) out[(size_t)n * KX + kx] = v;
  });
}

// expand() in x fused with d/dx: six paired inverse row transforms give
// U,UX | V,VX | W,WX | UY,VY | WY,E | EX,EY on the padded grid.
// src: Um, UYm, Vm, VYm, Wm, WYm, Em, EYm; dst: U, UX, UY, V, VX, VY, W, WX,
// WY, E, EX, EY.  blockIdx.z = group.
template <class T, int NSX>
__global__ void __launch_bounds__(RowCfg<3 * NSX / 2>::THREADS)
k_x_inverse(Ptr8 src, Ptr12 dst, int MY, int NZ, T kx0, const cx<T>* __restrict__ tw) {
  constexpr int MX = 3 * NSX / 2;
  constexpr int KX = NSX / 2;
  using C = RowCfg<MX>;
  extern __shared__ __align__(16) unsigned char smraw[];
  cx<T>* sm = reinterpret_cast<cx<T>*>(smraw);
  const int g = blockIdx.z, z = blockIdx.y + 1;
  if (z == NZ && (g == 2 || g == 4 || g == 5)) return;
  // (source A, ikx on A, source B, ikx on B, output A, output B)
  const int sA[6] = {0, 2, 4, 1, 5, 6}, mA[6] = {0, 0, 0, 0, 0, 1};
  const int sB[6] = {0, 2, 4, 3, 6, 7}, mB[6] = {1, 1, 1, 0, 0, 0};
  const int oA[6] = {0, 3, 6, 2, 8, 10}, oB[6] = {1, 4, 7, 5, 9, 11};
  const size_t zoff = (size_t)(z - 1) * MY;
  const cx<T>* A = reinterpret_cast<const cx<T>*>(src.p[sA[g]]) + zoff * KX;
  const cx<T>* B = reinterpret_cast<const cx<T>*>(src.p[sB[g]]) + zoff * KX;
  const bool ma = mA[g], mb = mB[g];
  const int y0 = blockIdx.x * C::NT;
  T* outA = reinterpret_cast<T*>(dst.p[oA[g]]) + zoff * MX;
  T* outB = reinterpret_cast<T*>(dst.p[oB[g]]) + zoff * MX;
  fft_core<MX, +1, false, false, false>(C::NT, sm, tw, [&](int t, int n) {
    int y = y0 + t;
    cx<T> v = zero_cx<T>();
    if (y < MY) {
      int k = -1;
      bool mir = false;
      if (n < KX) k = n;
      else if (n > MX - KX) { k = MX - n; mir = true; }
      if (k >= 0) {
        cx<T> a = A[(size_t)y * KX + k], b = B[(size_t)y * KX + k];
        T kk = kx0 * (T)k;
        if (ma) a = mul_i(a) * kk;
        if (mb) b = mul_i(b) * kk;
        if (k == 0) { a.y = 0; b.y = 0; }
        if (mir) { a = conj(a); b = conj(b); }
        v = mk(a.x - b.y, a.y + b.x);
      }
    }
    return v;
  }, [&](int t, int n, cx<T> v) {
    int y = y0 + t;
    if (y >= MY) return;
    outA[(size_t)y * MX + n] = v.x;
    outB[(size_t)y * MX + n] = v.y;
  });
}

// yderiv of delta = max(emin - E, 0) on padded planes (column pairs),
// added to EY.  This and k_clip_x make EX, EY the derivatives of the
// clipped ebuf = max(expand(e), emin) (comp1.f90:109,121; derivs2.f90:20-21).
template <class T, int NSY>
__global__ void __launch_bounds__(ColCfg<3 * NSY / 2, T>::THREADS)
k_clip_y(const T* __restrict__ E, T* __restrict__ EY, int MX, T emin, T ky0, const cx<T>* __restrict__ tw) {
  constexpr int M = 3 * NSY / 2;
  using C = ColCfg<M, T>;
  extern __shared__ __align__(16) unsigned char smraw[];
  cx<T>* sm = reinterpret_cast<cx<T>*>(smraw);
  const size_t zoff = (size_t)blockIdx.y * M * MX;
  const int c0 = blockIdx.x * C::TC, ncp = MX / 2;
  const cx<T>* Ez = reinterpret_cast<const cx<T>*>(E + zoff);
  fft_core<M, -1, true, false, true>(C::TC, sm, tw, [&](int t, int n) {
    int c = c0 + t;
    cx<T> v = zero_cx<T>();
    if (c < ncp) {
      cx<T> ev = Ez[(size_t)n * ncp + c];
      v = mk(tmax(emin - ev.x, (T)0), tmax(emin - ev.y, (T)0));
    }
    return v;
  }, NoStore{});
  for (int i = threadIdx.x; i < C::TC * M; i += blockDim.x) {
    int t = i % C::TC, k = i / C::TC;
    T kk = (k == 0 || 2 * k == M) ? (T)0 : ky0 * (T)signed_k(k, M) / (T)M;
    sm[k * C::TC + t] = mul_i(sm[k * C::TC + t]) * kk;
  }
  __syncthreads();
  cx<T>* EYz = reinterpret_cast<cx<T>*>(EY + zoff);
  fft_core<M, +1, true, true, false>(C::TC, sm, tw, NoLoad{}, [&](int t, int n, cx<T> d) {
    int c = c0 + t;
    if (c >= ncp) return;
    cx<T> o = EYz[(size_t)n * ncp + c];
    EYz[(size_t)n * ncp + c] = mk(o.x + d.x, o.y + d.y);
  });
}

// xderiv of delta (row pairs), added to EX; E <- max(E, emin).
template <class T, int NSX>
__global__ void __launch_bounds__(RowCfg<3 * NSX / 2>::THREADS)
k_clip_x(T* __restrict__ E, T* __restrict__ EX, int MY, T emin, T kx0, const cx<T>* __restrict__ tw) {
  constexpr int MX = 3 * NSX / 2;
  using C = RowCfg<MX>;
  extern __shared__ __align__(16) unsigned char smraw[];
  cx<T>* sm = reinterpret_cast<cx<T>*>(smraw);
  const size_t zoff = (size_t)blockIdx.y * MY * MX;
  const int p0 = blockIdx.x * C::NT, np = MY / 2;
  T* Ez = E + zoff;
  T* EXz = EX + zoff;
  fft_core<MX, -1, false, false, true>(C::NT, sm, tw, [&](int t, int n) {
    int p = p0 + t;
    cx<T> v = zero_cx<T>();
    if (p < np) {
      T a = Ez[(size_t)(2 * p) * MX + n], b = Ez[(size_t)(2 * p + 1) * MX + n];
      v = mk(tmax(emin - a, (T)0), tmax(emin - b, (T)0));
    }
    return v;
  }, NoStore{});
  for (int i = threadIdx.x; i < C::NT * MX; i += blockDim.x) {
    int t = i / MX, k = i - t * MX;
    T kk = (k == 0 || 2 * k == MX) ? (T)0 : kx0 * (T)signed_k(k, MX) / (T)MX;
    sm[t * MX + k] = mul_i(sm[t * MX + k]) * kk;
  }
  __syncthreads();
  fft_core<MX, +1, false, true, false>(C::NT, sm, tw, NoLoad{}, [&](int t, int n, cx<T> d) {
    int p = p0 + t;
    if (p >= np) return;
#pragma unroll
    for (int r = 0; r < 2; r++) {
      size_t off = (size_t)(2 * p + r) * MX + n;
      EXz[off] += r ? d.y : d.x;
      Ez[off] = tmax(Ez[off], emin);
    }
  });
}

// Block-wide sum of NV doubles per thread, written (not accumulated) to
// out[q] by thread 0: a fixed reduction order, so results are reproducible.
template <int NV>
__device__ __forceinline__ void block_sum_store(double (&v)[NV], double* out) {
  __shared__ double red[32][NV];
#pragma unroll
  for (int q = 0; q < NV; q++)
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < NV; q++) red[warp][q] = v[q];
  __syncthreads();
  if (warp == 0) {
    const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int q = 0; q < NV; q++) {
      double s = (lane < nw) ? red[lane][q] : 0.0;
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (lane == 0) out[q] = s;
    }
  }
}

// Per-level totals of per-block partial sums: one block per level z,
// out[z*ostride + q] = sum over p < nparts of part[(z*nparts + p)*nq + q],
// q < nq <= 8, summed in a fixed order.
static __global__ void __launch_bounds__(256) k_sum_parts(const double* __restrict__ part, int nparts, int nq,
                                                          double* __restrict__ out, int ostride) {
  const size_t z = blockIdx.x;
  double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int p = threadIdx.x; p < nparts; p += blockDim.x)
#pragma unroll
    for (int q = 0; q < 8; q++)
      if (q < nq) s[q] += part[(z * nparts + p) * nq + q];
  double t[8];
  block_sum_store<8>(s, t);
  if (threadIdx.x == 0)
    for (int q = 0; q < nq; q++) out[z * ostride + q] = t[q];
}

// Raw sums over the padded planes U, V at level 1 (blockIdx.y = 0) and nnz
// (blockIdx.y = 1): sum U, V, wind, U^2, V^2, wind^2, wind*U, wind*V, one
// partial per block in part[side][block][8] (summed in order by k_wall_final).
template <class T>
__global__ void k_wall_sums(const T* __restrict__ U, const T* __restrict__ V, int NZ, size_t P, double* part) {
  const int side = blockIdx.y;
  const size_t off = side == 0 ? 0 : (size_t)(NZ - 1) * P;
  double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < P; i += (size_t)gridDim.x * blockDim.x) {
    double u = (double)U[off + i], v = (double)V[off + i];
    double wd = (double)sqrt((T)(U[off + i] * U[off + i] + V[off + i] * V[off + i]));
    s[0] += u; s[1] += v; s[2] += wd; s[3] += u * u; s[4] += v * v; s[5] += wd * wd; s[6] += wd * u; s[7] += wd * v;
  }
  block_sum_store<8>(s, part + ((size_t)side * gridDim.x + blockIdx.x) * 8);
}

// Wall-model scalars for both walls (lowerbc.f90:56-124, upperbc.f90:63-122)
// and the global dudt, dvdt (lowerbc.f90:70-72) from the FP64 mean shadows.
static __global__ void k_wall_final(const double* __restrict__ part, int nblk, const double* __restrict__ mru,
                             const double* __restrict__ mrv, StageArgs a, double P, double vk, double zody,
                             double ufree, WallParams* wp, int* err) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double acc[16];
  for (int q = 0; q < 16; q++) acc[q] = 0.0;
  for (int side = 0; side < 2; side++)
    for (int b = 0; b < nblk; b++)
      for (int q = 0; q < 8; q++) acc[side * 8 + q] += part[((size_t)side * nblk + b) * 8 + q];
  double su = 0, sv = 0;
  for (int z = 0; z < a.NZ; z++) { su += mru[z]; sv += mrv[z]; }
  wp->dudt = su / a.NZ;
  wp->dvdt = sv / a.NZ;
  wp->utau_s = sqrt(a.zl / 2 * sqrt(wp->dvdt * wp->dvdt + (a.forcing - wp->dudt) * (a.forcing - wp->dudt)));
  for (int side = 0; side < 2; side++) {
    const double* s = acc + side * 8;
    WallSide& w = wp->w[side];
    double mU = s[0] / P, mV = s[1] / P;
    w.u1xy = mU + (side ? a.ugal : 0.0);
    w.v1xy = mV + (side ? a.vgal : 0.0);
    double windm = s[2] / P;
    w.vsfc = sqrt(w.u1xy * w.u1xy + w.v1xy * w.v1xy);
    windm = fmax(windm, ufree);
    windm = fmax(windm, 0.01);
    w.windm = windm;
    w.vsfc = fmax(w.vsfc, 0.01);
    w.utau = w.vsfc * vk / zody;
    if (w.utau > 10.0) atomicOr(err, ERR_UTAU);
    double tep = fmin(fmax(w.u1xy / w.vsfc, -1.0), 1.0);
    double thta = acos(tep);
    double ut2 = w.utau * w.utau;
    double sg = copysign(1.0, w.v1xy);
    double sgn_wall = side ? 1.0 : -1.0;
    w.auuwm = sgn_wall * ut2 * cos(thta);
    w.auvwm = sgn_wall * ut2 * sin(thta) * sg;
    // fluctuation moments: ufluc = U + ugal - u1xy = U - cu
    double cu = w.u1xy - a.ugal, cv = w.v1xy - a.vgal;
    double Suu = s[3] - 2 * cu * s[0] + P * cu * cu;
    double Svv = s[4] - 2 * cv * s[1] + P * cv * cv;
    double Sss = s[5] - 2 * windm * s[2] + P * windm * windm;
    double Sus = s[6] - windm * s[0] - cu * s[2] + P * cu * windm;
    double Svs = s[7] - windm * s[1] - cv * s[2] + P * cv * windm;
    w.ufluc2mroot = sqrt(Suu / P);
    w.vfluc2mroot = sqrt(Svv / P);
    w.suflucm = Sus / P;
    w.svflucm = Svs / P;
    double Smu = w.u1xy * w.u1xy * Sss + 2 * w.u1xy * windm * Sus + windm * windm * Suu;
    w.moengu2mroot = sqrt(Smu / P);
    w.moengv2mroot = w.moengu2mroot;  // moengv2m = sum(moengu2) in the reference (lowerbc.f90:121)
    w.denom = sqrt((windm * w.u1xy + w.suflucm) * (windm * w.u1xy + w.suflucm) +
                   (windm * w.v1xy + w.svflucm) * (windm * w.v1xy + w.svflucm));
  }
}

// Wall stress tau13, tau23 at one point (lowerbc.f90:126-161, upperbc.f90:124-158).
template <class T>
__device__ __forceinline__ void wall_stress(const WallSide& w, const WallParams& wp, const StageArgs& a, int side,
                                            T U, T V, T& tu, T& tv) {
  const double sg = side ? 1.0 : -1.0;
  const double ut2 = w.utau * w.utau;
  double Ud = (double)U + a.ugal, Vd = (double)V + a.vgal;
  double uf = Ud - w.u1xy, vf = Vd - w.v1xy;
  double wind = (double)sqrt(U * U + V * V);
  double ru, rv;
  switch (a.isurface) {
    case 1: ru = sg * ut2 / w.vsfc * Ud; rv = sg * ut2 / w.vsfc * Vd; break;
    case 2:
      ru = sg * ut2 / (w.windm * w.vsfc) * (w.windm * uf + wind * w.u1xy);
      rv = sg * ut2 / (w.windm * w.vsfc) * (w.windm * vf + wind * w.v1xy);
      break;
    case 3:
      ru = w.auuwm - sg * 0.35 * uf * ut2 / w.ufluc2mroot;
      rv = w.auvwm - sg * 0.35 * vf * ut2 / w.vfluc2mroot;
      break;
    case 4: ru = sg * ut2 * (wind * Ud) / w.denom; rv = sg * ut2 * (wind * Vd) / w.denom; break;
    case 5: {
      double sf = wind - w.windm;
      double mu = sf * w.u1xy + w.windm * uf, mv = sf * w.v1xy + w.windm * vf;
      ru = w.auuwm - sg * 0.35 * ut2 * mu / w.moengu2mroot;
      rv = w.auvwm - sg * 0.35 * ut2 * mv / w.moengv2mroot;
      break;
    }
    default: {  // 6
      double au = -a.zl / 2 * (a.forcing - wp.dudt), av = -a.zl / 2 * (-wp.dvdt);
      ru = -sg * au + sg * w.utau * wp.utau_s * uf / w.vsfc;
      rv = -sg * av + sg * w.utau * wp.utau_s * vf / w.vsfc;
      break;
    }
  }
  tu = (T)ru;
  tv = (T)rv;
}

// Padded-grid pointwise part of comp1 for level z (blockIdx.y + 1):
// compadv1 + complen + compsgs1 + compsgs3 written as the fields whose x/y
// derivatives and values the compress step needs:
//   u: A=UU+tuu (-d/dx), B=UV+tuv (-d/dy), Pu (value)
//   v: B (-d/dx), C=VV+tvv (-d/dy), Pv
//   w: D=0.5(U0+U1)W0+tuw (-d/dx), G=0.5(V0+V1)W0+tvw (-d/dy), Pw
//   e: F=0.5E0(U0+U1)-2xkk EX (-d/dx), H=0.5E0(V0+V1)-2xkk EY (-d/dy), Pe
// in: U,UX,UY,V,VX,VY,W,WX,WY,E,EX,EY   out: A,B,C,D,G,F,H,Pu,Pv,Pw,Pe
// stats: divz[z] (comp1.f90:145) and the SGS means (compsgs3.f90:71-78).
struct Ptr11 { void* p[11]; };
template <class T>
__global__ void __launch_bounds__(256)
k_flux(Ptr12 in, Ptr11 out, StageArgs a, const WallParams* __restrict__ wpp, double* __restrict__ divpart,
       double* __restrict__ sgspart) {
  const int z = blockIdx.y + 1;
  const int NZ = a.NZ;
  const size_t P = (size_t)a.MX * a.MY;
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = idx < P;
  const size_t q = valid ? idx : 0;
  const T* pU = (const T*)in.p[0]; const T* pUX = (const T*)in.p[1]; const T* pUY = (const T*)in.p[2];
  const T* pV = (const T*)in.p[3]; const T* pVX = (const T*)in.p[4]; const T* pVY = (const T*)in.p[5];
  const T* pW = (const T*)in.p[6]; const T* pWX = (const T*)in.p[7]; const T* pWY = (const T*)in.p[8];
  const T* pE = (const T*)in.p[9]; const T* pEX = (const T*)in.p[10]; const T* pEY = (const T*)in.p[11];
  auto at = [&](const T* f, int L, int lo, int hi) -> T { return (L >= lo && L <= hi) ? f[(size_t)(L - 1) * P + q] : (T)0; };
  auto Uat = [&](int L) { return at(pU, L, 1, NZ); };
  auto Vat = [&](int L) { return at(pV, L, 1, NZ); };
  auto Wat = [&](int L) { return at(pW, L, 1, NZ - 1); };
  auto Eat = [&](int L) { int Lc = L < 1 ? 1 : (L > NZ - 1 ? NZ - 1 : L); return pE[(size_t)(Lc - 1) * P + q]; };
  auto UXat = [&](int L) { return at(pUX, L, 1, NZ); };
  auto UYat = [&](int L) { return at(pUY, L, 1, NZ); };
  auto VXat = [&](int L) { return at(pVX, L, 1, NZ); };
  auto VYat = [&](int L) { return at(pVY, L, 1, NZ); };
  auto WXat = [&](int L) { return at(pWX, L, 1, NZ - 1); };
  auto WYat = [&](int L) { return at(pWY, L, 1, NZ - 1); };
  const T dzm = (T)a.dzm;
  auto WZat = [&](int L) -> T { return (L >= 1 && L <= NZ) ? (Wat(L) - Wat(L - 1)) * dzm : (T)0; };
  auto UZat = [&](int L) -> T { int Lc = L < 1 ? 1 : (L > NZ - 1 ? NZ - 1 : L); return (Uat(Lc + 1) - Uat(Lc)) * dzm; };
  auto VZat = [&](int L) -> T { int Lc = L < 1 ? 1 : (L > NZ - 1 ? NZ - 1 : L); return (Vat(Lc + 1) - Vat(Lc)) * dzm; };
  auto shear = [&](int L) -> T {
    T ux0 = UXat(L), ux1 = UXat(L + 1), vy0 = VYat(L), vy1 = VYat(L + 1), wz0 = WZat(L), wz1 = WZat(L + 1);
    T s0 = UYat(L) + VXat(L), s1 = UYat(L + 1) + VXat(L + 1);
    T c = UZat(L) + WXat(L), d = VZat(L) + WYat(L);
    return ux0 * ux0 + ux1 * ux1 + vy0 * vy0 + vy1 * vy1 + wz0 * wz0 + wz1 * wz1 + (T)0.5 * s0 * s0 +
           (T)0.5 * s1 * s1 + c * c + d * d;
  };
  const T xkmax = (T)a.xkmax, nu = (T)a.nu, dsl = (T)a.dsl;
  auto XKK = [&](int L) -> T {
    T v;
    if (a.imodel == 4) v = tmin(((T)0.1 * dsl) * ((T)0.1 * dsl) * sqrt(shear(L)), xkmax);
    else v = tmin((T)0.1 * dsl * sqrt(Eat(L)), xkmax);
    return v + nu;
  };
  const WallParams& wp = *wpp;
  T twl_u = 0, twl_v = 0;
  auto TUWat = [&](int L, T xk, T& tu, T& tv) {
    if (L == 0) wall_stress<T>(wp.w[0], wp, a, 0, Uat(1), Vat(1), tu, tv);
    else if (L == NZ) wall_stress<T>(wp.w[1], wp, a, 1, Uat(NZ), Vat(NZ), tu, tv);
    else { tu = -xk * (UZat(L) + WXat(L)); tv = -xk * (VZat(L) + WYat(L)); }
  };
  (void)twl_u; (void)twl_v;
  const T xkm = XKK(z - 1), xk0 = XKK(z);
  const T xkp = (z < NZ) ? XKK(z + 1) : (T)0;
  const T U0 = Uat(z), U1 = Uat(z + 1), Um = Uat(z - 1);
  const T V0 = Vat(z), V1 = Vat(z + 1), Vm = Vat(z - 1);
  const T W0 = Wat(z), W1 = Wat(z + 1), Wm = Wat(z - 1);
  const T ux = UXat(z), uy = UYat(z), vx = VXat(z), vy = VYat(z);
  const T s = xkm + xk0;
  const T tuu = -s * ux, tvv = -s * vy, tuv = -s * (uy + vx) * (T)0.5;
  T tuw0, tvw0, tuwm, tvwm;
  TUWat(z, xk0, tuw0, tvw0);
  TUWat(z - 1, xkm, tuwm, tvwm);
  const T todzm = (T)a.todzm;
  T* o[11];
#pragma unroll
  for (int i = 0; i < 11; i++) o[i] = (T*)out.p[i] + (size_t)(z - 1) * P + q;
  const T wz0 = WZat(z);
  const T tww0 = -(xkm + xk0) * wz0;
  if (valid) {
    *o[0] = U0 * U0 + tuu;
    *o[1] = U0 * V0 + tuv;
    *o[2] = V0 * V0 + tvv;
    *o[7] = -((U1 + U0) * W0 - (Um + U0) * Wm) * todzm + (T)a.forcing - (tuw0 - tuwm) * dzm;
    *o[8] = -((V1 + V0) * W0 - (Vm + V0) * Wm) * todzm - (tvw0 - tvwm) * dzm;
    if (z < NZ) {
      const T wz1 = WZat(z + 1);
      const T tww1 = -(xk0 + xkp) * wz1;
      *o[3] = (T)0.5 * (U0 + U1) * W0 + tuw0;
      *o[4] = (T)0.5 * (V0 + V1) * W0 + tvw0;
      T hp = (T)0.5 * (W1 + W0), hm = (T)0.5 * (W0 + Wm);
      *o[9] = -(hp * hp - hm * hm) * dzm - (tww1 - tww0) * dzm;
      const int le = z < NZ - 2 ? z : NZ - 2;
      const T ex = pEX[(size_t)(le - 1) * P + q], ey = pEY[(size_t)(le - 1) * P + q];
      const T E0 = Eat(z), E1 = Eat(z + 1), Em = Eat(z - 1);
      *o[5] = (T)0.5 * E0 * (U0 + U1) - (T)2 * xk0 * ex;
      *o[6] = (T)0.5 * E0 * (V0 + V1) - (T)2 * xk0 * ey;
      T pe = -(W1 * E1 - Wm * Em) * todzm +
             ((xkp + xk0) * (E1 - E0) - (xk0 + xkm) * (E0 - Em)) * (T)a.dzm2 - (T)a.ceps * E0 * sqrt(E0);
      if (a.tke_production) pe += xk0 * shear(z);
      *o[10] = pe;
    } else {
      *o[4] = (T)0;  // G at the top level (pairs with C in the forward transform)
    }
  }
  // statistics: divz (every stage) and the SGS means (stage 1 with mnout),
  // one partial sum per (level, block)
  const size_t slot = (size_t)(z - 1) * gridDim.x + blockIdx.x;
  {
    T d = ux + vy + wz0;
    double s1[1] = {valid ? (double)(d * d) : 0.0};
    block_sum_store<1>(s1, divpart + slot);
  }
  if (a.mnout_sgs) {
    __syncthreads();
    double st[6];
    st[0] = valid ? (double)tuu : 0.0;
    st[1] = valid ? (double)tvv : 0.0;
    st[2] = valid ? (double)tuv : 0.0;
    st[3] = valid ? (double)tww0 : 0.0;
    st[4] = valid ? (double)tuw0 : 0.0;
    st[5] = valid ? (double)tvw0 : 0.0;
    block_sum_store<6>(st, sgspart + slot * 6);
  }
}

// compress() in x fused with -d/dx: six paired forward row transforms of the
// flux fields, keep kx < nx/2, combine:
//   g0 (A, Pu) -> Xu1 = -ikx A^ + Pu^      g1 (B, Pv) -> Xv1 = -ikx B^ + Pv^, Xu2 = B^
//   g2 (C, G)  -> Xv2 = C^, Xw2 = G^       g3 (D, Pw) -> Xw1 = -ikx D^ + Pw^
//   g4 (F, Pe) -> Xe1 = -ikx F^ + Pe^      g5 (H, -)  -> Xe2 = H^
// in: A,B,C,D,G,F,H,Pu,Pv,Pw,Pe; out: Xu1,Xu2,Xv1,Xv2,Xw1,Xw2,Xe1,Xe2
template <class T, int NSX>
__global__ void __launch_bounds__(RowCfg<3 * NSX / 2>::THREADS)
k_x_forward(Ptr11 in, Ptr8 out, int MY, int NZ, T kx0, const cx<T>* __restrict__ tw) {
  constexpr int MX = 3 * NSX / 2;
  constexpr int KX = NSX / 2;
  using C = RowCfg<MX>;
  extern __shared__ __align__(16) unsigned char smraw[];
  cx<T>* sm = reinterpret_cast<cx<T>*>(smraw);
  const int g = blockIdx.z, z = blockIdx.y + 1;
  if (z == NZ && g >= 3) return;
  const int sA[6] = {0, 1, 2, 3, 5, 6}, sB[6] = {7, 8, 4, 9, 10, -1};
  const size_t zoff = (size_t)(z - 1) * MY;
  const T* A = (const T*)in.p[sA[g]] + zoff * MX;
  const T* B = sB[g] >= 0 ? (const T*)in.p[sB[g]] + zoff * MX : nullptr;
  const int y0 = blockIdx.x * C::NT;
  fft_core<MX, -1, false, false, true>(C::NT, sm, tw, [&](int t, int n) {
    int y = y0 + t;
    return (y < MY) ? mk(A[(size_t)y * MX + n], B ? B[(size_t)y * MX + n] : (T)0) : zero_cx<T>();
  }, NoStore{});
  auto O = [&](int j) { return (cx<T>*)out.p[j] + zoff * KX; };
  for (int i = threadIdx.x; i < C::NT * KX; i += blockDim.x) {
    int t = i / KX, k = i - t * KX, y = y0 + t;
    if (y >= MY) continue;
    cx<T> zk = sm[t * MX + k], zm = conj(sm[t * MX + (MX - k) % MX]);
    cx<T> ah = (zk + zm) * (T)0.5;
    cx<T> d = zk - zm;
    cx<T> bh = mk(d.y * (T)0.5, -d.x * (T)0.5);
    T kk = kx0 * (T)k;
    cx<T> dxa = mk(kk * ah.y, -kk * ah.x);  // -i kx a^
    size_t o = (size_t)y * KX + k;
    switch (g) {
      case 0: O(0)[o] = dxa + bh; break;
      case 1: O(2)[o] = dxa + bh; O(1)[o] = ah; break;
      case 2: O(3)[o] = ah; if (z < NZ) O(5)[o] = bh; break;
      case 3: O(4)[o] = dxa + bh; break;
      case 4: O(6)[o] = dxa + bh; break;
      default: O(7)[o] = ah; break;
    }
  }
}

// compress() in y fused with -d/dy: for field f (u, v, w, e)
//   R^(ky) = (FFT_M(X1) - i ky FFT_M(X2)) / (MX*MY) at the kept ky,
// rw's plane mean removed (comp1.f90:172).  R^ of u, v, w is written to
// rnew[f]; for e, re = IFFT_N(R^) (x-spectral) is written to rnew[3].
// A cluster of two CTAs per column group (blockIdx.x = 2 group + rank):
// rank 0 transforms X1, rank 1 X2, each into its own shared memory; after a
// cluster barrier each rank combines half of the kept ky rows, reading the
// other rank's transform through distributed shared memory (for e, rank 0
// combines all rows in place and runs the inverse N-point transform after a
// second cluster barrier).  Half the shared memory and threads of a CTA that
// held both transforms: FP64 2.6% faster, FP32 unchanged.  Thread 0 first
// has the TMA prefetch into L2 the columns of the block `pdist` blocks
// ahead (les_tma.cuh; maps: tensor maps of X[0..7] as [NZ*M][KX] rows;
// pdist 0 prefetches nothing).
template <class T, int NS>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(ColCfg<3 * NS / 2, T>::THREADS)
k_y_forward(Ptr8 X, Ptr8 rnew, int KX, int NZ, T ky0, T scale, const cx<T>* __restrict__ tw,
            const __grid_constant__ ColMaps maps, unsigned pdist) {
  constexpr int M = 3 * NS / 2;
  using C = ColCfg<M, T>;
  constexpr int TC = C::TC;
  prefetch_tile_ahead<T, M, TC>(maps, pdist, [&](unsigned bx, unsigned by, unsigned bz, int& q, int& cg, int& row0) {
    q = 2 * (int)bz + (int)(bx & 1); cg = (int)(bx >> 1); row0 = (int)by * M;
    return !(bz >= 2 && (int)by + 1 == NZ);
  });
  extern __shared__ __align__(16) unsigned char smraw[];
  cx<T>* sm = reinterpret_cast<cx<T>*>(smraw);
  cooperative_groups::cluster_group cluster = cooperative_groups::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int f = blockIdx.z, z = blockIdx.y + 1;
  if (f >= 2 && z == NZ) return;
  const int kx0 = (blockIdx.x >> 1) * TC;
  const cx<T>* Xs = (const cx<T>*)X.p[2 * f + rank] + (size_t)(z - 1) * M * KX;
  // the twiddles of the M-point transform staged in shared memory (measured
  // faster here than reading them through L1)
  const cx<T>* tws = stage_twiddles<M>(sm + (size_t)TC * M, tw);
  fft_core_tab<M, -1, true, false, true>(TC, sm, tws, [&](int t, int n) {
    int kx = kx0 + t;
    return (kx < KX) ? Xs[(size_t)n * KX + kx] : zero_cx<T>();
  }, NoStore{});
  cluster.sync();
  const cx<T>* s1 = cluster.map_shared_rank(sm, 0);
  const cx<T>* s2 = cluster.map_shared_rank(sm, 1);
  cx<T>* dst = (cx<T>*)rnew.p[f] + (size_t)(z - 1) * NS * KX;
  constexpr int ITEMS = TC * NS;
  const int lo = (f == 3) ? 0 : rank * (ITEMS / 2);
  const int hi = (f == 3) ? (rank == 0 ? ITEMS : 0) : lo + ITEMS / 2;
  for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    int t = i % TC, ky = i / TC, kx = kx0 + t;
    int n = (ky < NS / 2) ? ky : ky + NS / 2;
    cx<T> v = zero_cx<T>();
    if (ky != NS / 2) {
      cx<T> y1 = s1[n * TC + t], y2 = s2[n * TC + t];
      T kk = ky0 * (T)signed_k(ky, NS);
      v = mk(y1.x + kk * y2.y, y1.y - kk * y2.x) * scale;
      if (f == 2 && kx == 0 && ky == 0) v = zero_cx<T>();
    }
    if (f < 3) { if (kx < KX) dst[(size_t)ky * KX + kx] = v; }
    else sm[ky * TC + t] = v;
  }
  cluster.sync();
  if (f == 3 && rank == 0) {
    fft_core<NS, +1, true, true, false>(TC, sm, tw, NoLoad{}, [&](int t, int n, cx<T> v) {
      int kx = kx0 + t;
      if (kx < KX) dst[(size_t)n * KX + kx] = v;
    });
  }
}

// comp2's e update (comp2.f90:38) with re from its x-spectral rows:
// re = c2r(rem), e = max(e + dtab1*re, emin), levels 1..nnz-1.
template <class T, int NX>
__global__ void __launch_bounds__(RowCfg<NX>::THREADS)
k_e_update(const cx<T>* __restrict__ rem, T* __restrict__ re, T* __restrict__ e, int NY, T dtab1, T emin,
           const cx<T>* __restrict__ tw) {
  using C = RowCfg<NX>;
  constexpr int KX = NX / 2;
  extern __shared__ __align__(16) unsigned char smraw[];
  cx<T>* sm = reinterpret_cast<cx<T>*>(smraw);
  const int z = blockIdx.y + 1;
  const int p0 = blockIdx.x * C::NT;
  const size_t plane = (size_t)NY * NX;
  const cx<T>* in = rem + (size_t)(z - 1) * NY * KX;
  T* rez = re + (size_t)(z - 1) * plane;
  T* ez = e + (size_t)z * plane;
  fft_core<NX, +1, false, false, false>(C::NT, sm, tw, [&](int t, int n) {
    int p = p0 + t;
    cx<T> v = zero_cx<T>();
    if (p < NY / 2) {
      int k = -1;
      bool mir = false;
      if (n < KX) k = n;
      else if (n > KX) { k = NX - n; mir = true; }
      if (k >= 0) {
        cx<T> a = in[(size_t)(2 * p) * KX + k], b = in[(size_t)(2 * p + 1) * KX + k];
        if (k == 0) { a.y = 0; b.y = 0; }
        if (mir) { a = conj(a); b = conj(b); }
        v = mk(a.x - b.y, a.y + b.x);
      }
    }
    return v;
  }, [&](int t, int n, cx<T> v) {
    int p = p0 + t;
    if (p >= NY / 2) return;
#pragma unroll
    for (int r = 0; r < 2; r++) {
      size_t off = (size_t)(2 * p + r) * NX + n;
      T rv = r ? v.y : v.x;
      rez[off] = rv;
      ez[off] = tmax(ez[off] + dtab1 * rv, emin);
    }
  });
}

// comprhs + press + tridv for every (kx, ky) column in z, in FP64
// (comprhs.f90:17-35, press.F90:37-101, tridv.f90:29-53).
//   rhs = ikx (Ru + u*/dtab1) + iky (Rv + v*/dtab1) + (Q(z) - Q(z-1))/dz,
//   Q = w*/dtab1 + Rw, u* = u - dtab2*Ru_old (comp1.f90:127).
// Thomas sweeps use scratch d[z][mode], r[z][mode].
template <class T, bool RHS_IN_PH>
__global__ void k_press(const cx<T>* __restrict__ uh, const cx<T>* __restrict__ vh, const cx<T>* __restrict__ wh,
                        const cx<T>* __restrict__ ruo, const cx<T>* __restrict__ rvo, const cx<T>* __restrict__ rwo,
                        const cx<T>* __restrict__ run, const cx<T>* __restrict__ rvn, const cx<T>* __restrict__ rwn,
                        cx<double>* __restrict__ ph, double* __restrict__ dscr, cx<double>* __restrict__ rscr,
                        StageArgs a) {
  const int KX = a.KX, NY = a.NY, NZ = a.NZ;
  const int nm = KX * NY;
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= nm) return;
  const int ky = m / KX, kx = m - ky * KX;
  if (ky == NY / 2 || (kx == 0 && ky == 0)) {
    for (int z = 0; z < NZ; z++) ph[(size_t)z * nm + m] = mk(0.0, 0.0);
    return;
  }
  const double xk = a.kx0 * kx, yk = a.ky0 * signed_k(ky, NY);
  const double k2 = xk * xk + yk * yk, dzdz = a.dz * a.dz;
  const double dtabm = a.dtabm, dtab2 = a.zeta ? a.dtab2 : 0.0;
  auto ld = [&](const cx<T>* f, int z) -> cx<double> {
    cx<T> v = f[(size_t)(z - 1) * nm + m];
    return mk((double)v.x, (double)v.y);
  };
  cx<double> qprev = mk(0.0, 0.0), rprev = mk(0.0, 0.0);
  double dprev = 0.0;
  for (int z = 1; z <= NZ; z++) {
    cx<double> us = ld(uh, z) - ld(ruo, z) * dtab2;
    cx<double> vs = ld(vh, z) - ld(rvo, z) * dtab2;
    cx<double> q = mk(0.0, 0.0);
    if (z < NZ) q = (ld(wh, z) - ld(rwo, z) * dtab2) * dtabm + ld(rwn, z);
    cx<double> gu = ld(run, z) + us * dtabm, gv = ld(rvn, z) + vs * dtabm;
    cx<double> rhs = mul_i(gu) * xk + mul_i(gv) * yk + (q - qprev) * a.dzm;
    if (RHS_IN_PH) rhs = ph[(size_t)(z - 1) * nm + m];
    cx<double> r = rhs * dzdz;
    double b = -dzdz * k2 - ((z == 1 || z == NZ) ? 1.0 : 2.0);
    double d;
    if (z == 1) d = 1.0 / b;
    else {
      double fac = dprev;
      d = 1.0 / (b - fac);
      r = r - rprev * fac;
    }
    dscr[(size_t)(z - 1) * nm + m] = d;
    rscr[(size_t)(z - 1) * nm + m] = r;
    dprev = d; rprev = r; qprev = q;
  }
  cx<double> p = rprev * dprev;
  ph[(size_t)(NZ - 1) * nm + m] = p;
  for (int z = NZ - 1; z >= 1; z--) {
    double d = dscr[(size_t)(z - 1) * nm + m];
    cx<double> r = rscr[(size_t)(z - 1) * nm + m];
    p = (r - p) * d;
    ph[(size_t)(z - 1) * nm + m] = p;
  }
}

// comp2 (comp2.f90:15-43) in spectral space, FP64 arithmetic:
//   Ru' = Ru - ikx p, Rv' = Rv - iky p, Rw' = Rw - (p(z+1)-p(z))/dz (mean 0),
//   u = u* + dtab1 Ru', ..., w plane mean removed.  The kx=ky=0 modes of u, v
//   and their tendencies live in the FP64 shadows mu, mv, mru, mrv.
template <class T>
__global__ void k_update(cx<T>* uh, cx<T>* vh, cx<T>* wh, const cx<T>* ruo, const cx<T>* rvo, const cx<T>* rwo,
                         const cx<T>* run, const cx<T>* rvn, const cx<T>* rwn, cx<T>* ruout, cx<T>* rvout,
                         cx<T>* rwout, const cx<double>* __restrict__ ph, double* __restrict__ mu,
                         double* __restrict__ mv, double* __restrict__ mru, double* __restrict__ mrv, StageArgs a,
                         int* err) {
  const int KX = a.KX, NY = a.NY, NZ = a.NZ;
  const int nm = KX * NY;
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  const int z = blockIdx.y + 1;
  if (m >= nm) return;
  const int ky = m / KX, kx = m - ky * KX;
  if (ky == NY / 2) return;
  const double xk = a.kx0 * kx, yk = a.ky0 * signed_k(ky, NY);
  const double dtab1 = a.dtab1, dtab2 = a.zeta ? a.dtab2 : 0.0;
  const size_t o = (size_t)(z - 1) * nm + m;
  auto d2 = [](cx<T> v) { return mk((double)v.x, (double)v.y); };
  auto t2 = [](cx<double> v) { return mk((T)v.x, (T)v.y); };
  const cx<double> p = ph[o];
  bool bad = false;
  if (m == 0) {
    double us = mu[z - 1] - dtab2 * mru[z - 1];
    double vs = mv[z - 1] - dtab2 * mrv[z - 1];
    double rpu = (double)run[o].x, rpv = (double)rvn[o].x;
    double un = us + dtab1 * rpu, vn = vs + dtab1 * rpv;
    mu[z - 1] = un; mv[z - 1] = vn; mru[z - 1] = rpu; mrv[z - 1] = rpv;
    uh[o] = t2(mk(un, 0.0)); vh[o] = t2(mk(vn, 0.0));
    ruout[o] = t2(mk(rpu, 0.0)); rvout[o] = t2(mk(rpv, 0.0));
    if (z < NZ) { wh[o] = t2(mk(0.0, 0.0)); rwout[o] = t2(mk(0.0, 0.0)); }
    bad = !isfinite(un) || !isfinite(vn);
  } else {
    cx<double> rpu = d2(run[o]) - mul_i(p) * xk;
    cx<double> rpv = d2(rvn[o]) - mul_i(p) * yk;
    cx<double> un = d2(uh[o]) - d2(ruo[o]) * dtab2 + rpu * dtab1;
    cx<double> vn = d2(vh[o]) - d2(rvo[o]) * dtab2 + rpv * dtab1;
    uh[o] = t2(un); vh[o] = t2(vn); ruout[o] = t2(rpu); rvout[o] = t2(rpv);
    bad = !isfinite(un.x + un.y + vn.x + vn.y);
    if (z < NZ) {
      cx<double> p1 = ph[o + nm];
      cx<double> rpw = d2(rwn[o]) - (p1 - p) * a.dzm;
      cx<double> wn = d2(wh[o]) - d2(rwo[o]) * dtab2 + rpw * dtab1;
      wh[o] = t2(wn); rwout[o] = t2(rpw);
      bad = bad || !isfinite(wn.x + wn.y);
    }
  }
  if (bad) atomicOr(err, ERR_NAN);
}

// comprhs (comprhs.f90:17-35) alone: ph = rhs in the small-spectrum
// convention (used by the split entry points; k_press recomputes it inline).
template <class T>
__global__ void k_rhs(const cx<T>* __restrict__ uh, const cx<T>* __restrict__ vh, const cx<T>* __restrict__ wh,
                      const cx<T>* __restrict__ ru, const cx<T>* __restrict__ rv, const cx<T>* __restrict__ rw,
                      cx<double>* __restrict__ ph, StageArgs a) {
  const int KX = a.KX, NY = a.NY, NZ = a.NZ;
  const int nm = KX * NY;
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  const int z = blockIdx.y + 1;
  if (m >= nm) return;
  const int ky = m / KX, kx = m - ky * KX;
  const size_t o = (size_t)(z - 1) * nm + m;
  if (ky == NY / 2) { ph[o] = mk(0.0, 0.0); return; }
  const double xk = a.kx0 * kx, yk = a.ky0 * signed_k(ky, NY);
  auto d2 = [](cx<T> v) { return mk((double)v.x, (double)v.y); };
  cx<double> q = mk(0.0, 0.0), qm = mk(0.0, 0.0);
  if (z < NZ) q = d2(wh[o]) * a.dtabm + d2(rw[o]);
  if (z > 1) qm = d2(wh[o - nm]) * a.dtabm + d2(rw[o - nm]);
  cx<double> gu = d2(ru[o]) + d2(uh[o]) * a.dtabm, gv = d2(rv[o]) + d2(vh[o]) * a.dtabm;
  ph[o] = mul_i(gu) * xk + mul_i(gv) * yk + (q - qm) * a.dzm;
}

// The zeta part of the stage on u, v, w (comp1.f90:126-133) as a separate
// pass, for the split entry points: u -= dtab2*ru (spectral + FP64 shadows).
template <class T>
__global__ void k_zeta(cx<T>* uh, cx<T>* vh, cx<T>* wh, const cx<T>* ruo, const cx<T>* rvo, const cx<T>* rwo,
                       double* mu, double* mv, const double* mru, const double* mrv, StageArgs a) {
  const int nm = a.KX * a.NY;
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  const int z = blockIdx.y + 1;
  if (m >= nm) return;
  const size_t o = (size_t)(z - 1) * nm + m;
  const T d = (T)a.dtab2;
  if (m == 0) {
    mu[z - 1] -= a.dtab2 * mru[z - 1];
    mv[z - 1] -= a.dtab2 * mrv[z - 1];
    uh[o] = mk((T)mu[z - 1], (T)0);
    vh[o] = mk((T)mv[z - 1], (T)0);
  } else {
    uh[o] = uh[o] - ruo[o] * d;
    vh[o] = vh[o] - rvo[o] * d;
  }
  if (z < a.NZ) wh[o] = wh[o] - rwo[o] * d;
}

// SplitMix64 (Steele, Lea & Flood 2014) as a counter-based stream: output n
// of the stream seeded with s is mix(s + (n+1)*0x9e3779b97f4a7c15).
static __device__ __forceinline__ uint64_t splitmix64_at(uint64_t s, uint64_t n) {
  uint64_t z = s + (n + 1) * 0x9e3779b97f4a7c15ULL;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

// Seeded initial condition on the small grid (levels 1..nnz): parabolic mean
// plus uniform(-amp, amp)*utau perturbations for field f (0 u, 1 v, 2 w).
template <class T>
__global__ void k_ic_fill(T* __restrict__ out, int f, unsigned long long seed, int NX, int NY, int NZ, double dz,
                          double hh, double ub, double amp, double utau) {
  const size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t tot = (size_t)NX * NY * NZ;
  if (n >= tot) return;
  const int iz = (int)(n / ((size_t)NX * NY)) + 1;
  double mean = 0.0;
  if (f == 0) {
    double zm = ((double)iz - 0.5) * dz;
    double eta = (zm - hh) / hh;
    mean = 1.5 * ub * (1.0 - eta * eta);
  }
  uint64_t r = splitmix64_at((uint64_t)seed + (uint64_t)f, (uint64_t)n);
  double u01 = (double)(r >> 11) * (1.0 / 9007199254740992.0);
  double val = mean + (2.0 * u01 - 1.0) * amp * utau;
  if (f == 2 && iz == NZ) val = 0.0;
  out[n] = (T)val;
}

// Per-level plane sums (FP64) of up to 4 small-grid fields: acc[z*8 + q].
// One block per level (blockIdx.y), so the sums are reproducible.
template <class T>
__global__ void __launch_bounds__(1024) k_plane_sums(const T* __restrict__ f0, const T* __restrict__ f1, const T* __restrict__ f2,
                             const T* __restrict__ f3, size_t P, double* acc) {
  const size_t off = (size_t)blockIdx.y * P;
  double s[4] = {0, 0, 0, 0};
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < P; i += (size_t)gridDim.x * blockDim.x) {
    if (f0) s[0] += (double)f0[off + i];
    if (f1) s[1] += (double)f1[off + i];
    if (f2) s[2] += (double)f2[off + i];
    if (f3) s[3] += (double)f3[off + i];
  }
  block_sum_store<4>(s, acc + (size_t)blockIdx.y * 8);
}

// Moments of compmn (compmn.F90:29-62) at level iz = blockIdx.y + 1:
// u, v, w are small-grid physical fields on levels 1..nnz (u, v at nnz+1 are
// zero); means[z*8 + 0/1] hold the plane means of u and v.  One block per
// level, as k_plane_sums.
template <class T>
__global__ void __launch_bounds__(1024) k_moments(const T* __restrict__ u, const T* __restrict__ v, const T* __restrict__ w, size_t P, int NZ,
                          const double* __restrict__ means, double* acc) {
  const int iz = blockIdx.y + 1;
  const size_t off = (size_t)(iz - 1) * P;
  const T um = (T)means[(size_t)(iz - 1) * 8 + 0], vm = (T)means[(size_t)(iz - 1) * 8 + 1];
  const T um1 = iz < NZ ? (T)means[(size_t)iz * 8 + 0] : (T)0;
  const T vm1 = iz < NZ ? (T)means[(size_t)iz * 8 + 1] : (T)0;
  double s[6] = {0, 0, 0, 0, 0, 0};
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < P; i += (size_t)gridDim.x * blockDim.x) {
    T u1 = iz < NZ ? u[off + P + i] : (T)0;
    T v1 = iz < NZ ? v[off + P + i] : (T)0;
    T ul = (T)0.5 * ((u[off + i] - um) + u1 - um1);
    T vl = (T)0.5 * ((v[off + i] - vm) + v1 - vm1);
    T w0 = w[off + i];
    s[0] += (double)(ul * ul); s[1] += (double)(vl * vl); s[2] += (double)(w0 * w0);
    s[3] += (double)(ul * w0); s[4] += (double)(vl * w0); s[5] += (double)(ul * vl);
  }
  block_sum_store<6>(s, acc + (size_t)(iz - 1) * 8);
}

// Max |u|, |v|, |w| for the CFL time step (les.F90:205-207).
template <class T>
__global__ void k_absmax3(const T* __restrict__ u, const T* __restrict__ v, const T* __restrict__ w, size_t n,
                          unsigned long long* out) {
  T m[3] = {0, 0, 0};
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    m[0] = tmax(m[0], (T)fabs(u[i])); m[1] = tmax(m[1], (T)fabs(v[i])); m[2] = tmax(m[2], (T)fabs(w[i]));
  }
#pragma unroll
  for (int q = 0; q < 3; q++) {
    double d = (double)m[q];
    for (int o = 16; o > 0; o >>= 1) d = fmax(d, __shfl_xor_sync(0xffffffffu, d, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out + q, (unsigned long long)__double_as_longlong(d));
  }
}

// comp2's e update in physical space (split entry points).
template <class T>
__global__ void k_e_update_phys(T* __restrict__ e, const T* __restrict__ re, size_t n, T dtab1, T emin) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) e[i] = tmax(e[i] + dtab1 * re[i], emin);
}

// Elementwise helpers.
template <class T>
__global__ void k_fill(T* p, size_t n, T v) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}
template <class S, class D>
__global__ void k_convert(const S* __restrict__ in, D* __restrict__ out, size_t n) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (D)in[i];
}
// Set the kx=ky=0 mode of every level of a spectral array from FP64 values.
template <class T>
__global__ void k_set_mean(cx<T>* __restrict__ sp, const double* __restrict__ mean, size_t nm, int NZ) {
  int z = blockIdx.x * blockDim.x + threadIdx.x;
  if (z < NZ) sp[(size_t)z * nm] = mk((T)mean[z], (T)0);
}

// Batched 1D spectral derivative (xderiv/yderiv of filter_fftw.f90:138-248)
// along rows or columns of real planes, pairing rows/columns.
template <class T, int N>
__global__ void __launch_bounds__(RowCfg<N>::THREADS)
k_op_xderiv(const T* __restrict__ in, T* __restrict__ out, int nrows, T k0, const cx<T>* __restrict__ tw) {
  using C = RowCfg<N>;
  extern __shared__ __align__(16) unsigned char smraw[];
  cx<T>* sm = reinterpret_cast<cx<T>*>(smraw);
  const int p0 = blockIdx.x * C::NT;
  const int npair = (nrows + 1) / 2;
  fft_core<N, -1, false, false, true>(C::NT, sm, tw, [&](int t, int n) {
    int p = p0 + t;
    return (p < npair) ? mk(in[(size_t)(2 * p) * N + n], (2 * p + 1 < nrows) ? in[(size_t)(2 * p + 1) * N + n] : (T)0)
                       : zero_cx<T>();
  }, NoStore{});
  for (int i = threadIdx.x; i < C::NT * N; i += blockDim.x) {
    int t = i / N, k = i - t * N;
    T kk = (k == 0 || 2 * k == N) ? (T)0 : k0 * (T)signed_k(k, N) / (T)N;
    sm[t * N + k] = mul_i(sm[t * N + k]) * kk;
  }
  __syncthreads();
  fft_core<N, +1, false, true, false>(C::NT, sm, tw, NoLoad{}, [&](int t, int n, cx<T> v) {
    int p = p0 + t;
    if (p >= npair) return;
    out[(size_t)(2 * p) * N + n] = v.x;
    if (2 * p + 1 < nrows) out[(size_t)(2 * p + 1) * N + n] = v.y;
  });
}
template <class T, int N>
__global__ void __launch_bounds__(ColCfg<N, T>::THREADS)
k_op_yderiv(const T* __restrict__ in, T* __restrict__ out, int n1, T k0, const cx<T>* __restrict__ tw) {
  using C = ColCfg<N, T>;
  extern __shared__ __align__(16) unsigned char smraw[];
  cx<T>* sm = reinterpret_cast<cx<T>*>(smraw);
  const size_t plane = (size_t)blockIdx.y * N * n1;
  const int ncp = (n1 + 1) / 2, c0 = blockIdx.x * C::TC;
  fft_core<N, -1, true, false, true>(C::TC, sm, tw, [&](int t, int n) {
    int c = c0 + t;
    return (c < ncp) ? mk(in[plane + (size_t)n * n1 + 2 * c], (2 * c + 1 < n1) ? in[plane + (size_t)n * n1 + 2 * c + 1] : (T)0)
                     : zero_cx<T>();
  }, NoStore{});
  for (int i = threadIdx.x; i < C::TC * N; i += blockDim.x) {
    int t = i % C::TC, k = i / C::TC;
    T kk = (k == 0 || 2 * k == N) ? (T)0 : k0 * (T)signed_k(k, N) / (T)N;
    sm[k * C::TC + t] = mul_i(sm[k * C::TC + t]) * kk;
  }
  __syncthreads();
  fft_core<N, +1, true, true, false>(C::TC, sm, tw, NoLoad{}, [&](int t, int n, cx<T> v) {
    int c = c0 + t;
    if (c >= ncp) return;
    out[plane + (size_t)n * n1 + 2 * c] = v.x;
    if (2 * c + 1 < n1) out[plane + (size_t)n * n1 + 2 * c + 1] = v.y;
  });
}

// tridv (tridv.f90:1-55) for one right-hand side per thread; bdar is
// (ny, n, 4) column-major.
static __global__ void k_op_tridv(double* bdar, int ny, int n) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ny) return;
  double* b = bdar;
  double* d = bdar + (size_t)ny * n;
  double* a = bdar + (size_t)2 * ny * n;
  double* r = bdar + (size_t)3 * ny * n;
  auto I = [ny, j](int i) { return (size_t)(i - 1) * ny + j; };
  if (n <= 1) { r[I(1)] = r[I(1)] / d[I(1)]; return; }
  d[I(1)] = 1.0 / d[I(1)];
  for (int i = 2; i <= n; i++) {
    double fac = b[I(i)] * d[I(i - 1)];
    d[I(i)] = 1.0 / (d[I(i)] - fac * a[I(i - 1)]);
    r[I(i)] = r[I(i)] - fac * r[I(i - 1)];
  }
  r[I(n)] = r[I(n)] * d[I(n)];
  for (int i = n - 1; i >= 1; i--) r[I(i)] = d[I(i)] * (r[I(i)] - a[I(i)] * r[I(i + 1)]);
}

}  // namespace les

// fft_core.cuh -- shared-memory / register FFT building blocks for sm_100a.
//
// All transforms in this project have lengths 2^a 3^b up to 1152 (the
// small grid nx, ny and the 3/2-padded grid 3nx/2, 3ny/2).  A length
// N = N1*N2 transform runs as the four-step algorithm inside one CTA:
//   pass A: each work item loads N1 strided inputs, does an N1-point DFT in
//           registers and multiplies by the outer twiddles W_N^(n2*k1);
//   one shared-memory transpose;
//   pass B: each work item does an N2-point DFT in registers and stores N2
//           outputs.
// Row transforms (contiguous data) map consecutive threads to consecutive
// elements; column transforms map consecutive threads to consecutive
// columns so that global loads and stores stay coalesced in both cases.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <cmath>

namespace les {

template <class T> struct alignas(2 * sizeof(T)) cx { T x, y; };

template <class T> __host__ __device__ __forceinline__ cx<T> mk(T a, T b) { cx<T> r; r.x = a; r.y = b; return r; }
template <class T> __device__ __forceinline__ cx<T> operator+(cx<T> a, cx<T> b) { return mk(a.x + b.x, a.y + b.y); }
template <class T> __device__ __forceinline__ cx<T> operator-(cx<T> a, cx<T> b) { return mk(a.x - b.x, a.y - b.y); }
template <class T> __device__ __forceinline__ cx<T> operator*(cx<T> a, T s) { return mk(a.x * s, a.y * s); }
// FP32 complex sums, differences and real scalings as one packed f32x2
// instruction each (sm_100a; each component rounded to nearest as the
// scalar form): the butterflies of every FP32 transform issue half the
// additions.
template <> __device__ __forceinline__ cx<float> operator+<float>(cx<float> a, cx<float> b) {
  cx<float> r;
  asm("{\n\t.reg .b64 a, b, r;\n\tmov.b64 a, {%2, %3};\n\tmov.b64 b, {%4, %5};\n\t"
      "add.rn.f32x2 r, a, b;\n\tmov.b64 {%0, %1}, r;\n\t}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
template <> __device__ __forceinline__ cx<float> operator*<float>(cx<float> a, float sc) {
  cx<float> r;
  asm("{\n\t.reg .b64 a, b, r;\n\tmov.b64 a, {%2, %3};\n\tmov.b64 b, {%4, %4};\n\t"
      "mul.rn.f32x2 r, a, b;\n\tmov.b64 {%0, %1}, r;\n\t}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(sc));
  return r;
}
template <> __device__ __forceinline__ cx<float> operator-<float>(cx<float> a, cx<float> b) {
  cx<float> r;
  asm("{\n\t.reg .b64 a, b, r;\n\tmov.b64 a, {%2, %3};\n\tmov.b64 b, {%4, %5};\n\t"
      "sub.rn.f32x2 r, a, b;\n\tmov.b64 {%0, %1}, r;\n\t}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
template <class T> __device__ __forceinline__ cx<T> cmul(cx<T> a, cx<T> b) {
  return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <class T> __device__ __forceinline__ cx<T> conj(cx<T> a) { return mk(a.x, -a.y); }
// i*a
template <class T> __device__ __forceinline__ cx<T> mul_i(cx<T> a) { return mk(-a.y, a.x); }
template <class T> __device__ __forceinline__ cx<T> zero_cx() { return mk((T)0, (T)0); }

// W_384^j = exp(-2 pi i j / 384) in constant memory.  One copy per
// translation unit (no relocatable device code); every unit exports an
// upload function built on upload_tu_twiddles() that the host calls once per
// device before the first launch.
constexpr int TWN = 384;
static __constant__ double2 c_tw64[TWN];
static __constant__ float2 c_tw32[TWN];
static inline cudaError_t upload_tu_twiddles() {
  double2 a[TWN];
  float2 b[TWN];
  const long double pi = 3.141592653589793238462643383279502884L;
  for (int j = 0; j < TWN; j++) {
    long double t = -2.0L * pi * j / TWN;
    a[j] = make_double2((double)cosl(t), (double)sinl(t));
    b[j] = make_float2((float)cosl(t), (float)sinl(t));
  }
  cudaError_t e = cudaMemcpyToSymbol(c_tw64, a, sizeof(a));
  if (e != cudaSuccess) return e;
  return cudaMemcpyToSymbol(c_tw32, b, sizeof(b));
}

template <class T> __device__ __forceinline__ cx<T> ctw(int j);
template <> __device__ __forceinline__ cx<double> ctw<double>(int j) { double2 v = c_tw64[j]; return mk(v.x, v.y); }
template <> __device__ __forceinline__ cx<float> ctw<float>(int j) { float2 v = c_tw32[j]; return mk(v.x, v.y); }

// v * W_384^(S*j) for a compile-time j (after unrolling); S = -1 forward.
template <int S, class T> __device__ __forceinline__ cx<T> twmul(cx<T> v, int j) {
  j = j % TWN;
  if (j == 0) return v;
  if (j == TWN / 2) return mk(-v.x, -v.y);
  if (j == TWN / 4) return (S < 0) ? mk(v.y, -v.x) : mk(-v.y, v.x);      // -i / +i
  if (j == 3 * TWN / 4) return (S < 0) ? mk(-v.y, v.x) : mk(v.y, -v.x);  // +i / -i
  cx<T> w = ctw<T>(j);
  if (S > 0) w.y = -w.y;
  return cmul(v, w);
}

// In-register DFT of length N (N divides 384), natural order in and out.
template <int N, int S, class T> struct Dft;

template <int S, class T> struct Dft<1, S, T> {
  static __device__ __forceinline__ void run(cx<T>*) {}
};
template <int S, class T> struct Dft<2, S, T> {
  static __device__ __forceinline__ void run(cx<T>* v) {
    cx<T> a = v[0] + v[1], b = v[0] - v[1];
    v[0] = a; v[1] = b;
  }
};
template <int S, class T> struct Dft<3, S, T> {
  static __device__ __forceinline__ void run(cx<T>* v) {
    const T s3 = (T)0.86602540378443864676372317075293618;  // sin(2 pi / 3)
    cx<T> t1 = v[1] + v[2];
    cx<T> t2 = v[0] - t1 * (T)0.5;
    cx<T> d = v[1] - v[2];
    T sg = (S < 0) ? -s3 : s3;
    cx<T> t3 = mk(-sg * d.y, sg * d.x);
    v[0] = v[0] + t1; v[1] = t2 + t3; v[2] = t2 - t3;
  }
};
template <int S, class T> struct Dft<4, S, T> {
  static __device__ __forceinline__ void run(cx<T>* v) {
    cx<T> a0 = v[0] + v[2], a1 = v[0] - v[2];
    cx<T> b0 = v[1] + v[3], b1 = v[1] - v[3];
    cx<T> ib1 = (S < 0) ? mk(b1.y, -b1.x) : mk(-b1.y, b1.x);
    v[0] = a0 + b0; v[2] = a0 - b0; v[1] = a1 + ib1; v[3] = a1 - ib1;
  }
};
template <int N, int S, class T> struct Dft {
  static constexpr int R = (N % 4 == 0) ? 4 : ((N % 2 == 0) ? 2 : 3);
  static constexpr int M = N / R;
  static_assert(TWN % N == 0, "register DFT length must divide 384");
  static __device__ __forceinline__ void run(cx<T>* v) {
    cx<T> a[R][M];
#pragma unroll
    for (int r = 0; r < R; r++)
#pragma unroll
      for (int m = 0; m < M; m++) a[r][m] = v[r + R * m];
#pragma unroll
    for (int r = 0; r < R; r++) Dft<M, S, T>::run(a[r]);
#pragma unroll
    for (int r = 1; r < R; r++)
#pragma unroll
      for (int k = 1; k < M; k++) a[r][k] = twmul<S>(a[r][k], r * k * (TWN / N));
#pragma unroll
    for (int k = 0; k < M; k++) {
      cx<T> b[R];
#pragma unroll
      for (int r = 0; r < R; r++) b[r] = a[r][k];
      Dft<R, S, T>::run(b);
#pragma unroll
      for (int q = 0; q < R; q++) v[k + M * q] = b[q];
    }
  }
};

// Factorisation N = N1 * N2 used by the block transform.
template <int N> struct Split;
template <> struct Split<16> { static constexpr int N1 = 4, N2 = 4; };
template <> struct Split<24> { static constexpr int N1 = 4, N2 = 6; };
template <> struct Split<32> { static constexpr int N1 = 4, N2 = 8; };
template <> struct Split<48> { static constexpr int N1 = 6, N2 = 8; };
template <> struct Split<64> { static constexpr int N1 = 8, N2 = 8; };
template <> struct Split<96> { static constexpr int N1 = 8, N2 = 12; };
template <> struct Split<128> { static constexpr int N1 = 8, N2 = 16; };
template <> struct Split<144> { static constexpr int N1 = 12, N2 = 12; };
template <> struct Split<192> { static constexpr int N1 = 12, N2 = 16; };
template <> struct Split<256> { static constexpr int N1 = 16, N2 = 16; };
template <> struct Split<288> { static constexpr int N1 = 12, N2 = 24; };
template <> struct Split<384> { static constexpr int N1 = 16, N2 = 24; };
template <> struct Split<512> { static constexpr int N1 = 16, N2 = 32; };
template <> struct Split<576> { static constexpr int N1 = 24, N2 = 24; };
template <> struct Split<768> { static constexpr int N1 = 24, N2 = 32; };

// Outer twiddles exp(-2 pi i j / N) for every supported N, concatenated.
// tw_off(N) is the offset of the table for N.
struct TwTable {
  const void* base;  // cx<T>*
};
constexpr int kSizes[] = {16, 24, 32, 48, 64, 96, 128, 144, 192, 256, 288, 384, 512, 576, 768};
constexpr int kNumSizes = sizeof(kSizes) / sizeof(int);
__host__ __device__ constexpr int tw_off(int n) {
  return n == 16 ? 0 :
         n == 24 ? 16 :
         n == 32 ? 40 :
         n == 48 ? 72 :
         n == 64 ? 120 :
         n == 96 ? 184 :
         n == 128 ? 280 :
         n == 144 ? 408 :
         n == 192 ? 552 :
         n == 256 ? 744 :
         n == 288 ? 1000 :
         n == 384 ? 1288 :
         n == 512 ? 1672 :
         n == 576 ? 2184 :
         n == 768 ? 2760 : -1;
}
constexpr int kTwTotal = tw_off(768) + 768;

template <int N> struct BlockFft {
  static constexpr int N1 = Split<N>::N1;
  static constexpr int N2 = Split<N>::N2;
  // shared-memory elements needed for `ntrans` transforms
  static constexpr int smem_elems(int ntrans) { return ntrans * N1 * (N2 + 1); }
};

// One batch of `ntrans` complex transforms of length N in a CTA.
//   load(t, n)      -> input element n of transform t
//   store(t, k, v)  <- output element k of transform t
// TFAST = true maps consecutive threads to consecutive transforms (column
// transforms); false maps them to consecutive elements (row transforms).
// tw: the concatenated outer-twiddle table (global memory).
// The caller must __syncthreads() before reusing `sm`.
template <int N, int S, bool TFAST, class T, class LoadF, class StoreF>
__device__ __forceinline__ void block_fft(int ntrans, cx<T>* sm, const cx<T>* __restrict__ tw, LoadF load,
                                          StoreF store) {
  constexpr int N1 = Split<N>::N1;
  constexpr int N2 = Split<N>::N2;
  constexpr int LD = N2 + 1;
  const cx<T>* twn = tw + tw_off(N);
  const int nA = ntrans * N2;
  for (int it = threadIdx.x; it < nA; it += blockDim.x) {
    int t, n2;
    if (TFAST) { t = it % ntrans; n2 = it / ntrans; }
    else { t = it / N2; n2 = it - t * N2; }
    cx<T> v[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; n1++) v[n1] = load(t, n2 + N2 * n1);
    Dft<N1, S, T>::run(v);
#pragma unroll
    for (int k1 = 0; k1 < N1; k1++) {
      cx<T> w = twn[n2 * k1];
      if (S > 0) w.y = -w.y;
      cx<T> r = (k1 == 0) ? v[k1] : cmul(v[k1], w);
      if (TFAST) sm[(k1 * N2 + n2) * ntrans + t] = r;
      else sm[(t * N1 + k1) * LD + n2] = r;
    }
  }
  __syncthreads();
  const int nB = ntrans * N1;
  for (int it = threadIdx.x; it < nB; it += blockDim.x) {
    int t, k1;
    if (TFAST) { t = it % ntrans; k1 = it / ntrans; }
    else { t = it / N1; k1 = it - t * N1; }
    cx<T> v[N2];
#pragma unroll
    for (int n2 = 0; n2 < N2; n2++) v[n2] = TFAST ? sm[(k1 * N2 + n2) * ntrans + t] : sm[(t * N1 + k1) * LD + n2];
    Dft<N2, S, T>::run(v);
#pragma unroll
    for (int k2 = 0; k2 < N2; k2++) store(t, k1 + N1 * k2, v[k2]);
  }
}

// Row variant with the result left in shared memory in natural order:
// sm[t*N + k] = X_t[k].  Requires blockDim.x >= ntrans*N2 (>= ntrans*N1) and
// BlockFft<N>::smem_elems(ntrans) elements of `sm` (>= ntrans*N).  Ends with
// a __syncthreads().
template <int N, int S, class T, class LoadF>
__device__ __forceinline__ void row_fft_to_smem(int ntrans, cx<T>* sm, const cx<T>* __restrict__ tw,
                                                LoadF load) {
  constexpr int N1 = Split<N>::N1;
  constexpr int N2 = Split<N>::N2;
  constexpr int LD = N2 + 1;
  const cx<T>* twn = tw + tw_off(N);
  const int it = threadIdx.x;
  if (it < ntrans * N2) {
    int t = it / N2, n2 = it - t * N2;
    cx<T> v[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; n1++) v[n1] = load(t, n2 + N2 * n1);
    Dft<N1, S, T>::run(v);
#pragma unroll
    for (int k1 = 0; k1 < N1; k1++) {
      cx<T> w = twn[n2 * k1];
      if (S > 0) w.y = -w.y;
      sm[(t * N1 + k1) * LD + n2] = (k1 == 0) ? v[k1] : cmul(v[k1], w);
    }
  }
  __syncthreads();
  cx<T> v[N2];
  const bool active = it < ntrans * N1;
  int t = 0, k1 = 0;
  if (active) {
    t = it / N1; k1 = it - t * N1;
#pragma unroll
    for (int n2 = 0; n2 < N2; n2++) v[n2] = sm[(t * N1 + k1) * LD + n2];
  }
  __syncthreads();
  if (active) {
    Dft<N2, S, T>::run(v);
#pragma unroll
    for (int k2 = 0; k2 < N2; k2++) sm[t * N + k1 + N1 * k2] = v[k2];
  }
  __syncthreads();
}

// In-place transform of `ntrans` sequences held in shared memory in natural
// order, result in natural order.
//   ROWS layout: element n of transform t at sm[t*N + n]
//   COLS layout: element n of transform t at sm[n*ntrans + t]
// Requires blockDim.x >= ntrans*N2 and smem_fft_elems<N, COLS>(ntrans)
// elements.  Starts and ends with a __syncthreads().
template <int N, bool COLS>
__host__ __device__ constexpr int smem_fft_elems(int ntrans) {
  return COLS ? ntrans * N : ((ntrans * Split<N>::N1 * (Split<N>::N2 + 1) > ntrans * N)
                                  ? ntrans * Split<N>::N1 * (Split<N>::N2 + 1)
                                  : ntrans * N);
}
template <int N, int S, bool COLS, class T>
__device__ __forceinline__ void smem_fft(int ntrans, cx<T>* sm, const cx<T>* __restrict__ tw) {
  constexpr int N1 = Split<N>::N1;
  constexpr int N2 = Split<N>::N2;
  constexpr int LD = N2 + 1;
  const cx<T>* twn = tw + tw_off(N);
  const int it = threadIdx.x;
  __syncthreads();
  // pass A
  {
    const bool active = it < ntrans * N2;
    int t = 0, n2 = 0;
    cx<T> v[N1];
    if (active) {
      if (COLS) { t = it % ntrans; n2 = it / ntrans; }
      else { t = it / N2; n2 = it - t * N2; }
#pragma unroll
      for (int n1 = 0; n1 < N1; n1++)
        v[n1] = COLS ? sm[(n2 + N2 * n1) * ntrans + t] : sm[t * N + n2 + N2 * n1];
    }
    __syncthreads();
    if (active) {
      Dft<N1, S, T>::run(v);
#pragma unroll
      for (int k1 = 0; k1 < N1; k1++) {
        cx<T> w = twn[n2 * k1];
        if (S > 0) w.y = -w.y;
        cx<T> r = (k1 == 0) ? v[k1] : cmul(v[k1], w);
        if (COLS) sm[(k1 * N2 + n2) * ntrans + t] = r;
        else sm[(t * N1 + k1) * LD + n2] = r;
      }
    }
    __syncthreads();
  }
  // pass B
  {
    const bool active = it < ntrans * N1;
    int t = 0, k1 = 0;
    cx<T> v[N2];
    if (active) {
      if (COLS) { t = it % ntrans; k1 = it / ntrans; }
      else { t = it / N1; k1 = it - t * N1; }
#pragma unroll
      for (int n2 = 0; n2 < N2; n2++)
        v[n2] = COLS ? sm[(k1 * N2 + n2) * ntrans + t] : sm[(t * N1 + k1) * LD + n2];
    }
    __syncthreads();
    if (active) {
      Dft<N2, S, T>::run(v);
#pragma unroll
      for (int k2 = 0; k2 < N2; k2++) {
        int k = k1 + N1 * k2;
        if (COLS) sm[k * ntrans + t] = v[k2];
        else sm[t * N + k] = v[k2];
      }
    }
    __syncthreads();
  }
}

// General four-step transform of `ntrans` sequences with one shared-memory
// transpose.  Input comes from global memory through load(t, n) (pass A
// issues N1 independent loads per thread before any arithmetic) or, with
// IN_SMEM, from `sm` in natural layout; output goes to store(t, k, v) or,
// with OUT_SMEM, back to `sm` in natural layout.
//   natural layout: rows  sm[t*N + n];  cols (COLS) sm[n*ntrans + t]
// Requires blockDim.x >= ntrans*N2 and smem_fft_elems<N, COLS>(ntrans)
// elements; every thread of the block must call it.  Ends with a
// __syncthreads() when OUT_SMEM.  fft_core_tab takes the length-N twiddle
// table itself (e.g. staged in shared memory by stage_twiddles); fft_core
// reads it from the global table.
template <int N, int S, bool COLS, bool IN_SMEM, bool OUT_SMEM, class T, class LoadF, class StoreF>
__device__ __forceinline__ void fft_core_tab(int ntrans, cx<T>* sm, const cx<T>* twn, LoadF load, StoreF store) {
  constexpr int N1 = Split<N>::N1;
  constexpr int N2 = Split<N>::N2;
  constexpr int LD = N2 + 1;
  const int it = threadIdx.x;
  {
    const bool active = it < ntrans * N2;
    int t = 0, n2 = 0;
    if (COLS) { t = it % ntrans; n2 = it / ntrans; }
    else { t = it / N2; n2 = it - t * N2; }
    cx<T> v[N1];
    if (active) {
#pragma unroll
      for (int n1 = 0; n1 < N1; n1++) {
        const int n = n2 + N2 * n1;
        if constexpr (IN_SMEM) v[n1] = COLS ? sm[n * ntrans + t] : sm[t * N + n];
        else v[n1] = load(t, n);
      }
    }
    if (IN_SMEM) __syncthreads();
    if (active) {
      Dft<N1, S, T>::run(v);
#pragma unroll
      for (int k1 = 0; k1 < N1; k1++) {
        cx<T> w = twn[n2 * k1];
        if (S > 0) w.y = -w.y;
        cx<T> r = (k1 == 0) ? v[k1] : cmul(v[k1], w);
        if (COLS) sm[(k1 * N2 + n2) * ntrans + t] = r;
        else sm[(t * N1 + k1) * LD + n2] = r;
      }
    }
  }
  __syncthreads();
  {
    const bool active = it < ntrans * N1;
    int t = 0, k1 = 0;
    if (COLS) { t = it % ntrans; k1 = it / ntrans; }
    else { t = it / N1; k1 = it - t * N1; }
    cx<T> v[N2];
    if (active) {
#pragma unroll
      for (int n2 = 0; n2 < N2; n2++)
        v[n2] = COLS ? sm[(k1 * N2 + n2) * ntrans + t] : sm[(t * N1 + k1) * LD + n2];
    }
    if (OUT_SMEM) __syncthreads();
    if (active) {
      Dft<N2, S, T>::run(v);
#pragma unroll
      for (int k2 = 0; k2 < N2; k2++) {
        const int k = k1 + N1 * k2;
        if constexpr (OUT_SMEM) {
          if (COLS) sm[k * ntrans + t] = v[k2];
          else sm[t * N + k] = v[k2];
        } else {
          store(t, k, v[k2]);
        }
      }
    }
    if (OUT_SMEM) __syncthreads();
  }
}
template <int N, int S, bool COLS, bool IN_SMEM, bool OUT_SMEM, class T, class LoadF, class StoreF>
__device__ __forceinline__ void fft_core(int ntrans, cx<T>* sm, const cx<T>* __restrict__ tw, LoadF load,
                                         StoreF store) {
  fft_core_tab<N, S, COLS, IN_SMEM, OUT_SMEM, T>(ntrans, sm, tw + tw_off(N), load, store);
}
// Copy of the length-N twiddle table into shared memory `dst` (N entries),
// by the whole block; ends with a barrier.
template <int N, class T>
__device__ __forceinline__ const cx<T>* stage_twiddles(cx<T>* dst, const cx<T>* __restrict__ tw) {
  const cx<T>* g = tw + tw_off(N);
  for (int i = threadIdx.x; i < N; i += blockDim.x) dst[i] = g[i];
  __syncthreads();
  return dst;
}
struct NoLoad {
  __device__ int operator()(int, int) const { return 0; }
};
struct NoStore {
  template <class V> __device__ void operator()(int, int, V) const {}
};

// Signed wavenumber index of FFT bin k for length n (k > n/2 -> k - n).
__host__ __device__ __forceinline__ int signed_k(int k, int n) { return (k > n / 2) ? k - n : k; }

}  // namespace les

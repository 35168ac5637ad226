// les_ops.cu -- operator-level transforms on caller-owned device buffers:
// xderiv, yderiv, expand, compress, deal (filter_fftw.f90:138-329).
#include "les_engine.cuh"

namespace les {
cudaError_t upload_twiddles_ops() { return upload_tu_twiddles(); }

template <class T>
void op_xderiv(const T* in, T* out, int n1, int n2, int howmany, double len, cudaStream_t s) {
  const cx<T>* tw = (const cx<T>*)twiddles(-1, sizeof(T) == 8);
  const double pi = 4.0 * std::atan(1.0);
  int nrows = n2 * howmany;
  bool ok = with_any(n1, [&](auto cn) {
    constexpr int N = decltype(cn)::value;
    using C = RowCfg<N>;
    launch(k_op_xderiv<T, N>, dim3(cdiv((nrows + 1) / 2, C::NT)), dim3(C::THREADS), C::template smem<T>(), s, in,
           out, nrows, (T)(2.0 * pi / len), tw);
  });
  if (!ok) throw CudaError("xderiv: unsupported length", LES_EINVAL);
}

template <class T>
void op_yderiv(const T* in, T* out, int n1, int n2, int howmany, double len, cudaStream_t s) {
  const cx<T>* tw = (const cx<T>*)twiddles(-1, sizeof(T) == 8);
  const double pi = 4.0 * std::atan(1.0);
  bool ok = with_any(n2, [&](auto cn) {
    constexpr int N = decltype(cn)::value;
    using C = ColCfg<N, T>;
    launch(k_op_yderiv<T, N>, dim3(cdiv((n1 + 1) / 2, C::TC), howmany), dim3(C::THREADS), C::buf(), s, in, out, n1,
           (T)(2.0 * pi / len), tw);
  });
  if (!ok) throw CudaError("yderiv: unsupported length", LES_EINVAL);
}

// expand: r2c rows (nx) -> forward y (ny, scaled, Nyquist dropped) -> pad and
// inverse y (3ny/2) -> c2r rows (3nx/2).  t1: howmany*ny*nx/2, t2: howmany*(3ny/2)*nx/2.
template <class T>
void op_expand(const T* in, T* out, int nx, int ny, int howmany, cudaStream_t s, cx<T>* t1, cx<T>* t2) {
  const cx<T>* tw = (const cx<T>*)twiddles(-1, sizeof(T) == 8);
  const int KX = nx / 2, MX = 3 * nx / 2, MY = 3 * ny / 2;
  if (!supported_small(nx) || !supported_small(ny)) throw CudaError("expand: unsupported size", LES_EINVAL);
  with_small(nx, [&](auto cn) {
    constexpr int N = decltype(cn)::value;
    using C = RowCfg<N>;
    launch(k_row_r2c<T, N>, dim3(cdiv(howmany * ny / 2 + 1, C::NT)), dim3(C::THREADS), C::template smem<T>(), s, in,
           t1, howmany * ny, KX, tw);
  });
  with_small(ny, [&](auto cn) {
    constexpr int N = decltype(cn)::value;
    using C = ColCfg<N, T>;
    launch(k_col_small<T, N, false>, dim3(cdiv(KX, C::TC), howmany), dim3(C::THREADS), C::buf(), s,
           (const cx<T>*)t1, t1, KX, (T)(1.0 / ((double)nx * ny)), tw);
    using CM = ColCfg<3 * N / 2, T>;
    launch(k_col_pad<T, N>, dim3(cdiv(KX, CM::TC), howmany), dim3(CM::THREADS), CM::buf(), s, (const cx<T>*)t1, t2,
           KX, tw);
  });
  with_small(nx, [&](auto cn) {
    constexpr int N = decltype(cn)::value;
    using C = RowCfg<3 * N / 2>;
    launch(k_row_c2r<T, 3 * N / 2>, dim3(cdiv(howmany * MY / 2 + 1, C::NT)), dim3(C::THREADS),
           C::template smem<T>(), s, (const cx<T>*)t2, out, howmany * MY, KX, tw);
  });
  (void)MX;
}

// compress: r2c rows (3nx/2, keep nx/2) -> forward y (3ny/2), truncate,
// scale, inverse y (ny) -> c2r rows (nx).
template <class T>
void op_compress(const T* in, T* out, int nx, int ny, int howmany, cudaStream_t s, cx<T>* t1, cx<T>* t2) {
  const cx<T>* tw = (const cx<T>*)twiddles(-1, sizeof(T) == 8);
  const int KX = nx / 2, MX = 3 * nx / 2, MY = 3 * ny / 2;
  if (!supported_small(nx) || !supported_small(ny)) throw CudaError("compress: unsupported size", LES_EINVAL);
  with_small(nx, [&](auto cn) {
    constexpr int N = decltype(cn)::value;
    using C = RowCfg<3 * N / 2>;
    launch(k_row_r2c<T, 3 * N / 2>, dim3(cdiv(howmany * MY / 2 + 1, C::NT)), dim3(C::THREADS),
           C::template smem<T>(), s, in, t2, howmany * MY, KX, tw);
  });
  with_small(ny, [&](auto cn) {
    constexpr int N = decltype(cn)::value;
    using CM = ColCfg<3 * N / 2, T>;
    launch(k_col_trunc<T, N>, dim3(cdiv(KX, CM::TC), howmany), dim3(CM::THREADS), 2 * CM::buf(), s,
           (const cx<T>*)t2, t1, KX, (T)(1.0 / ((double)MX * MY)), tw);
  });
  with_small(nx, [&](auto cn) {
    constexpr int N = decltype(cn)::value;
    using C = RowCfg<N>;
    launch(k_row_c2r<T, N>, dim3(cdiv(howmany * ny / 2 + 1, C::NT)), dim3(C::THREADS), C::template smem<T>(), s,
           (const cx<T>*)t1, out, howmany * ny, KX, tw);
  });
}

template <class T>
void op_deal(T* x, int nx, int ny, int howmany, cudaStream_t s, cx<T>* t1) {
  const cx<T>* tw = (const cx<T>*)twiddles(-1, sizeof(T) == 8);
  const int KX = nx / 2;
  if (!supported_small(nx) || !supported_small(ny)) throw CudaError("deal: unsupported size", LES_EINVAL);
  with_small(nx, [&](auto cn) {
    constexpr int N = decltype(cn)::value;
    using C = RowCfg<N>;
    launch(k_row_r2c<T, N>, dim3(cdiv(howmany * ny / 2 + 1, C::NT)), dim3(C::THREADS), C::template smem<T>(), s,
           (const T*)x, t1, howmany * ny, KX, tw);
  });
  with_small(ny, [&](auto cn) {
    constexpr int N = decltype(cn)::value;
    using C = ColCfg<N, T>;
    launch(k_col_small<T, N, false>, dim3(cdiv(KX, C::TC), howmany), dim3(C::THREADS), C::buf(), s,
           (const cx<T>*)t1, t1, KX, (T)(1.0 / ((double)nx * ny)), tw);
    launch(k_col_small<T, N, true>, dim3(cdiv(KX, C::TC), howmany), dim3(C::THREADS), C::buf(), s,
           (const cx<T>*)t1, t1, KX, (T)1, tw);
  });
  with_small(nx, [&](auto cn) {
    constexpr int N = decltype(cn)::value;
    using C = RowCfg<N>;
    launch(k_row_c2r<T, N>, dim3(cdiv(howmany * ny / 2 + 1, C::NT)), dim3(C::THREADS), C::template smem<T>(), s,
           (const cx<T>*)t1, x, howmany * ny, KX, tw);
  });
}

template void op_xderiv<double>(const double*, double*, int, int, int, double, cudaStream_t);
template void op_xderiv<float>(const float*, float*, int, int, int, double, cudaStream_t);
template void op_yderiv<double>(const double*, double*, int, int, int, double, cudaStream_t);
template void op_yderiv<float>(const float*, float*, int, int, int, double, cudaStream_t);
template void op_expand<double>(const double*, double*, int, int, int, cudaStream_t, cx<double>*, cx<double>*);
template void op_expand<float>(const float*, float*, int, int, int, cudaStream_t, cx<float>*, cx<float>*);
template void op_compress<double>(const double*, double*, int, int, int, cudaStream_t, cx<double>*, cx<double>*);
template void op_compress<float>(const float*, float*, int, int, int, cudaStream_t, cx<float>*, cx<float>*);
template void op_deal<double>(double*, int, int, int, cudaStream_t, cx<double>*);
template void op_deal<float>(float*, int, int, int, cudaStream_t, cx<float>*);

}  // namespace les

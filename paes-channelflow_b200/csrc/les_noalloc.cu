// les_noalloc.cu -- les_op_expand_noalloc: the expand() transform with its
// scratch in a fixed device array instead of memory allocated per call.
//
// Who needs this: callers that must not allocate device memory while they
// run, e.g. a host that has reserved all free device memory up front, a
// driver that calls from inside a region where allocation is forbidden or
// would serialise other streams, or an embedding whose allocator policy
// bans hidden allocations.  les_op_expand obtains two scratch buffers with
// cudaMallocAsync; this variant uses a static array that, once placed on a
// device, stays there until the process exits.
//
// Limits and caveats:
//  - capacity: kNoAllocBytes (16 MiB) per device; the scratch a call needs
//    is howmany * (nx/2) * (ny + 3*ny/2) complex values (16 bytes each for
//    real_bytes = 8, 8 bytes for real_bytes = 4).  Larger calls are rejected
//    with LES_EINVAL before anything is launched.
//  - every GPU that loads the library holds the 16 MiB array until exit.
//  - all calls share the one array: calls that overlap on the GPU (different
//    streams, or threads, without ordering between them) race and corrupt
//    each other's results.  Order them on one stream or with events.
//  - the first call on each device does a one-time set-up (it looks up the
//    array's device address and copies the twiddle tables); make that first
//    call before any stream capture on that device.
//  - when the array is placed: under CUDA's lazy module loading (the default
//    since CUDA 12.2) this file's device code, the 16 MiB array and the
//    twiddle tables are loaded onto a device by that first call's
//    cudaGetSymbolAddress, not when the library is loaded.  That load takes
//    device memory, so a host that reserves all free device memory up front
//    must make its first call on each device before reserving (or run with
//    CUDA_MODULE_LOADING=EAGER, which loads them with the CUDA context).
//  - nothing in the array needs clearing: every scratch element a call
//    reads is written earlier by the same call.
#include <mutex>
#include <set>
#include <string>

#include "les_engine.cuh"

namespace les {

void set_op_error(const char* msg);

namespace {

constexpr size_t kNoAllocBytes = size_t(16) << 20;

// The scratch of les_op_expand_noalloc (see the limits above).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];
// Outer-twiddle tables of this translation unit (no allocation needed).
static __device__ __align__(256) double2 g_noalloc_tw64[kTwTotal];
static __device__ __align__(256) float2 g_noalloc_tw32[kTwTotal];

struct NoAllocDevice {
  unsigned char* scratch = nullptr;
  const void* tw64 = nullptr;
  const void* tw32 = nullptr;
};
std::mutex g_noalloc_mu;
std::map<int, NoAllocDevice> g_noalloc_dev;

// One-time set-up on the current device: the host-side names of the static
// arrays are only stand-ins, so their device addresses are looked up here.
const NoAllocDevice& noalloc_setup(int dev) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  auto it = g_noalloc_dev.find(dev);
  if (it != g_noalloc_dev.end()) return it->second;
  NoAllocDevice d;
  void* p = nullptr;
  LES_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
  d.scratch = (unsigned char*)p;
  LES_CUDA(upload_tu_twiddles());
  std::vector<double2> t64(kTwTotal);
  std::vector<float2> t32(kTwTotal);
  const long double pi = 3.141592653589793238462643383279502884L;
  for (int si = 0; si < kNumSizes; si++) {
    int n = kSizes[si], off = tw_off(n);
    for (int j = 0; j < n; j++) {
      long double a = -2.0L * pi * j / n;
      t64[off + j] = make_double2((double)cosl(a), (double)sinl(a));
      t32[off + j] = make_float2((float)cosl(a), (float)sinl(a));
    }
  }
  LES_CUDA(cudaMemcpyToSymbol(g_noalloc_tw64, t64.data(), sizeof(double2) * kTwTotal));
  LES_CUDA(cudaMemcpyToSymbol(g_noalloc_tw32, t32.data(), sizeof(float2) * kTwTotal));
  LES_CUDA(cudaGetSymbolAddress(&p, g_noalloc_tw64));
  d.tw64 = p;
  LES_CUDA(cudaGetSymbolAddress(&p, g_noalloc_tw32));
  d.tw32 = p;
  return g_noalloc_dev.emplace(dev, d).first->second;
}

// Same four launches as op_expand, on the static scratch.
template <class T>
void expand_static(const T* in, T* out, int nx, int ny, int howmany, cudaStream_t s, const cx<T>* tw, cx<T>* t1,
                   cx<T>* t2) {
  const int KX = nx / 2, MY = 3 * ny / 2;
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
}

}  // namespace
}  // namespace les

using namespace les;

extern "C" int les_op_expand_noalloc(const void* xs, void* xl, int nx, int ny, int howmany, int real_bytes,
                                     void* stream) {
  if (!xs || !xl || howmany <= 0 || (real_bytes != 4 && real_bytes != 8) || !supported_small(nx) ||
      !supported_small(ny)) {
    set_op_error("les_op_expand_noalloc: bad arguments");
    return LES_EINVAL;
  }
  const size_t cbytes = (size_t)2 * real_bytes;
  const size_t n1 = (size_t)howmany * ny * (nx / 2);
  const size_t n2 = (size_t)howmany * (3 * ny / 2) * (nx / 2);
  const size_t off2 = (n1 * cbytes + 255) / 256 * 256;
  if (off2 + n2 * cbytes > kNoAllocBytes) {
    set_op_error("les_op_expand_noalloc: howmany*(nx/2)*(ny+3ny/2) complex values exceed the 16 MiB static scratch");
    return LES_EINVAL;
  }
  try {
    int dev;
    LES_CUDA(cudaGetDevice(&dev));
    const NoAllocDevice& d = noalloc_setup(dev);
    cudaStream_t s = (cudaStream_t)stream;
    if (real_bytes == 8)
      expand_static<double>((const double*)xs, (double*)xl, nx, ny, howmany, s, (const cx<double>*)d.tw64,
                            (cx<double>*)d.scratch, (cx<double>*)(d.scratch + off2));
    else
      expand_static<float>((const float*)xs, (float*)xl, nx, ny, howmany, s, (const cx<float>*)d.tw32,
                           (cx<float>*)d.scratch, (cx<float>*)(d.scratch + off2));
  } catch (CudaError& e) {
    set_op_error(e.what());
    return e.code;
  } catch (std::exception& e) {
    set_op_error(e.what());
    return LES_EINVAL;
  }
  return LES_OK;
}

// les_probe.cu -- vector FMA throughput of the device, measured by this
// library's own kernel: the compute roof the transform kernels are read
// against (their FP32 / FP64 work is FMA-pipe work, not tensor-core work).
//
// Each thread runs 8 independent fused multiply-add chains; with 16 CTAs of
// 256 threads per SM the pipes see enough independent instructions to
// stay busy.  Timed with CUDA events on a private stream after a warm-up
// launch; flop/s = 2 * 8 * iterations * threads / seconds.
#include <cuda_runtime.h>

#include "../../include/les_gpu.h"

namespace {

template <class T>
__global__ void __launch_bounds__(256) k_fma_probe(T* __restrict__ out, int iters, T b, T c) {
  T a[8];
#pragma unroll
  for (int i = 0; i < 8; i++) a[i] = (T)(threadIdx.x + i) * (T)1e-3;
  for (int k = 0; k < iters; k++) {
#pragma unroll
    for (int i = 0; i < 8; i++) a[i] = fma(a[i], b, c);
  }
  T s = (T)0;
#pragma unroll
  for (int i = 0; i < 8; i++) s += a[i];
  if (s == (T)-1234.5) out[0] = s;  // keeps every chain live; never true for these inputs
}

template <class T>
int probe(int device, double* flops_per_s) {
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) return LES_ECUDA;
  if (cudaSetDevice(device) != cudaSuccess) return LES_EINVAL;
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  const int blocks = 16 * nsm, threads = 256, iters = 4096;
  T* out = nullptr;
  cudaStream_t s = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = LES_OK;
  float ms = 0.f;
  if (cudaMalloc((void**)&out, sizeof(T)) != cudaSuccess || cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) ||
      cudaEventCreate(&e0) || cudaEventCreate(&e1)) {
    rc = LES_ECUDA;
  } else {
    k_fma_probe<T><<<blocks, threads, 0, s>>>(out, iters, (T)0.999, (T)1e-4);  // warm-up
    cudaEventRecord(e0, s);
    k_fma_probe<T><<<blocks, threads, 0, s>>>(out, iters, (T)0.999, (T)1e-4);
    cudaEventRecord(e1, s);
    if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess || ms <= 0.f)
      rc = LES_ECUDA;
  }
  if (rc == LES_OK) *flops_per_s = 2.0 * 8.0 * iters * (double)blocks * threads / (ms * 1e-3);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (s) cudaStreamDestroy(s);
  if (out) cudaFree(out);
  cudaSetDevice(prev);
  return rc;
}

}  // namespace

extern "C" int les_probe_fma_rate(int real_bytes, int device, double* flops_per_s) {
  if (!flops_per_s || (real_bytes != 4 && real_bytes != 8)) return LES_EINVAL;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return LES_ENOTBUILT;
  if (device < 0 || device >= n) return LES_EINVAL;
  return real_bytes == 8 ? probe<double>(device, flops_per_s) : probe<float>(device, flops_per_s);
}

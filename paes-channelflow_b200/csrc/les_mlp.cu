// les_mlp.cu -- host side of the learned closure's perceptron (les_mlp.h):
// parameter packing, the inference / training launches and the Adam state.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/les_mlp.h"
#include "les_engine.cuh"
#include "les_mlp.cuh"

using namespace les;

struct les_mlp {
  int device = 0;
  MlpDev* dev = nullptr;  // device parameters used by the kernels
  DevBuf<float> master, m1, m2, grad, part;
  DevBuf<double> lpart;
  DevBuf<int> err;
  std::vector<float> norm = std::vector<float>(kMlpNNorm, 0.f);
  int adam_step = 0;
  unsigned long long wait_ns = kMmaWaitNs;  // MlpDev::wait_ns
  int nsm = 148;
  std::string msg;
};

namespace les {
const MlpDev* mlp_dev_params(const les_mlp* m) { return m ? m->dev : nullptr; }
int mlp_device(const les_mlp* m) { return m ? m->device : -1; }
}  // namespace les

namespace {

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int d) {
    cudaGetDevice(&prev);
    if (prev != d) LES_CUDA(cudaSetDevice(d));
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

template <class F> int mlp_guard(les_mlp* m, F&& fn) {
  if (!m) return LES_EINVAL;
  try {
    DeviceGuard g(m->device);
    fn();
    return LES_OK;
  } catch (CudaError& e) {
    m->msg = e.what();
    return e.code;
  } catch (std::exception& e) {
    m->msg = e.what();
    return LES_EINVAL;
  }
}

// Host image of MlpDev from flat f32 parameters and normalisation.
void pack_params(const float* p, const float* norm, MlpDev& d) {
  std::memset(&d, 0, sizeof(d));
  const __nv_bfloat16 zero = __float2bfloat16_rn(0.f);
  for (auto& v : d.w1) v = zero;
  for (auto& v : d.w2) v = zero;
  for (auto& v : d.w3) v = zero;
  for (auto& v : d.w4) v = zero;
  for (int o = 0; o < 64; o++)
    for (int k = 0; k < kMlpIn; k++) d.w1[tc::tile_elem(o, k, 16)] = __float2bfloat16_rn(p[kPW1 + o * kMlpIn + k]);
  for (int o = 0; o < 64; o++)
    for (int k = 0; k < 64; k++) {
      d.w2[tc::tile_elem(o, k, 64)] = __float2bfloat16_rn(p[kPW2 + o * 64 + k]);
      d.w3[tc::tile_elem(o, k, 64)] = __float2bfloat16_rn(p[kPW3 + o * 64 + k]);
    }
  for (int o = 0; o < kMlpOut; o++)
    for (int k = 0; k < 64; k++) d.w4[tc::tile_elem(o, k, 64)] = __float2bfloat16_rn(p[kPW4 + o * 64 + k]);
  for (int i = 0; i < 64; i++) { d.b1[i] = p[kPB1 + i]; d.b2[i] = p[kPB2 + i]; d.b3[i] = p[kPB3 + i]; }
  for (int i = 0; i < kMlpOut; i++) d.b4[i] = p[kPB4 + i];
  for (int i = 0; i < kMlpIn; i++) {
    d.in_shift[i] = norm[i];
    d.in_scale[i] = norm[kMlpIn + i];
    d.in_rscale[i] = norm[kMlpIn + i] != 0.f ? 1.f / norm[kMlpIn + i] : 0.f;
  }
  for (int i = 0; i < kMlpOut; i++) {
    d.out_scale[i] = norm[2 * kMlpIn + i];
    d.out_shift[i] = norm[2 * kMlpIn + kMlpOut + i];
  }
}

void check_samples(const void* feat, const void* y, long long n) {
  if (!feat || !y || n <= 0) throw std::invalid_argument("null sample buffer or n <= 0");
  if (((uintptr_t)feat % 16) || ((uintptr_t)y % 16)) throw std::invalid_argument("sample buffers must be 16-byte aligned");
}

void read_err(les_mlp* m, cudaStream_t s) {
  int e = 0;
  LES_CUDA(cudaMemcpyAsync(&e, m->err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  LES_CUDA(cudaStreamSynchronize(s));
  if (e) {
    LES_CUDA(cudaMemsetAsync(m->err.p, 0, sizeof(int), s));
    throw CudaError("tensor-core MMA did not complete within its wait limit", LES_ETIMEOUT);
  }
}

// loss and gradient partials of a batch; returns the number of partials
int train_partials(les_mlp* m, const void* feat, const float* target, long long n, cudaStream_t s) {
  const long long ntiles = (n + 127) / 128;
  const int grid = (int)std::min<long long>(ntiles, m->nsm);
  launch(k_mlp_train, dim3(grid), dim3(128), kTrainSmemLaunch, s, (const MlpDev*)m->dev, (const uint4*)feat,
         (const float4*)target, n, m->part.p, m->lpart.p, m->err.p);
  return grid;
}

double host_loss(les_mlp* m, int nparts, long long n, cudaStream_t s) {
  std::vector<double> lp(nparts);
  LES_CUDA(cudaMemcpyAsync(lp.data(), m->lpart.p, nparts * sizeof(double), cudaMemcpyDeviceToHost, s));
  read_err(m, s);
  double l = 0.0;
  for (double v : lp) l += v;
  return l / ((double)n * kMlpOut);
}

}  // namespace

extern "C" {

int les_mlp_create(int device, les_mlp** out) {
  if (!out) return LES_EINVAL;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return LES_ENOTBUILT;
  if (device < 0 || device >= ndev) return LES_EINVAL;
  les_mlp* m = new les_mlp();
  m->device = device;
  int rc = mlp_guard(m, [&] {
    int cc = 0;
    LES_CUDA(cudaDeviceGetAttribute(&cc, cudaDevAttrComputeCapabilityMajor, device));
    if (cc != 10) throw CudaError("the learned closure's kernels are built for sm_100a only", LES_ENOTBUILT);
    LES_CUDA(cudaDeviceGetAttribute(&m->nsm, cudaDevAttrMultiProcessorCount, device));
    LES_CUDA(cudaMalloc((void**)&m->dev, sizeof(MlpDev)));
    LES_CUDA(cudaMemset(m->dev, 0, sizeof(MlpDev)));
    LES_CUDA(cudaMemcpy(&m->dev->wait_ns, &m->wait_ns, sizeof(m->wait_ns), cudaMemcpyHostToDevice));
    for (auto* b : {&m->master, &m->m1, &m->m2, &m->grad}) b->alloc(kMlpNParam);
    m->part.alloc((size_t)m->nsm * kMlpNParam);
    m->lpart.alloc(m->nsm);
    m->err.alloc(1);
  });
  if (rc) {
    les_mlp_destroy(m);
    return rc;
  }
  *out = m;
  return LES_OK;
}

void les_mlp_destroy(les_mlp* m) {
  if (!m) return;
  {
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(m->device);
    cudaDeviceSynchronize();
    if (m->dev) cudaFree(m->dev);
    for (auto* b : {&m->master, &m->m1, &m->m2, &m->grad, &m->part}) b->release();
    m->lpart.release();
    m->err.release();
    if (prev >= 0) cudaSetDevice(prev);
  }
  delete m;
}

const char* les_mlp_last_error(const les_mlp* m) { return m ? m->msg.c_str() : "null les_mlp"; }

int les_mlp_set_params(les_mlp* m, const float* params, const float* norm) {
  if (!m || !params || !norm) return LES_EINVAL;
  return mlp_guard(m, [&] {
    for (int i = 0; i < kMlpNParam; i++)
      if (!std::isfinite(params[i])) throw std::invalid_argument("non-finite parameter");
    for (int i = 0; i < kMlpNNorm; i++)
      if (!std::isfinite(norm[i])) throw std::invalid_argument("non-finite normalisation");
    MlpDev h;
    pack_params(params, norm, h);
    h.wait_ns = m->wait_ns;
    LES_CUDA(cudaMemcpy(m->dev, &h, sizeof(MlpDev), cudaMemcpyHostToDevice));
    LES_CUDA(cudaMemcpy(m->master.p, params, kMlpNParam * sizeof(float), cudaMemcpyHostToDevice));
    LES_CUDA(cudaMemset(m->m1.p, 0, kMlpNParam * sizeof(float)));
    LES_CUDA(cudaMemset(m->m2.p, 0, kMlpNParam * sizeof(float)));
    m->norm.assign(norm, norm + kMlpNNorm);
    m->adam_step = 0;
  });
}

int les_mlp_set_wait_limit(les_mlp* m, double seconds) {
  if (!m || !(seconds >= 0.0 && seconds <= 60.0)) return LES_EINVAL;
  return mlp_guard(m, [&] {
    m->wait_ns = (unsigned long long)(seconds * 1e9);
    LES_CUDA(cudaDeviceSynchronize());  // no kernel reads the old value any more
    LES_CUDA(cudaMemcpy(&m->dev->wait_ns, &m->wait_ns, sizeof(m->wait_ns), cudaMemcpyHostToDevice));
  });
}

int les_mlp_get_params(les_mlp* m, float* params, float* norm) {
  if (!m) return LES_EINVAL;
  return mlp_guard(m, [&] {
    LES_CUDA(cudaDeviceSynchronize());
    if (params) LES_CUDA(cudaMemcpy(params, m->master.p, kMlpNParam * sizeof(float), cudaMemcpyDeviceToHost));
    if (norm) std::memcpy(norm, m->norm.data(), kMlpNNorm * sizeof(float));
  });
}

int les_mlp_forward(les_mlp* m, const void* feat, long long n, float* y, void* stream) {
  if (!m) return LES_EINVAL;
  return mlp_guard(m, [&] {
    check_samples(feat, y, n);
    cudaStream_t s = (cudaStream_t)stream;
    const long long ntiles = (n + 127) / 128;
    const int grid = (int)std::min<long long>((ntiles + kInferGroups - 1) / kInferGroups, (long long)m->nsm * kInferCtasPerSm);
    launch(k_mlp_infer<MlpOutRaw>, dim3(grid), dim3(128 * kInferGroups), kInferSmem, s, (const MlpDev*)m->dev,
           (const uint4*)feat, n, MlpOutRaw{y}, (double*)nullptr, m->err.p);
  });
}

int les_mlp_loss_grad(les_mlp* m, const void* feat, const float* target, long long n, float* grad, double* loss,
                      void* stream) {
  if (!m || !grad) return LES_EINVAL;
  return mlp_guard(m, [&] {
    check_samples(feat, target, n);
    cudaStream_t s = (cudaStream_t)stream;
    const int np = train_partials(m, feat, target, n, s);
    launch(k_mlp_reduce_adam, dim3(cdiv(kMlpNParam, 256)), dim3(256), 0, s, (const float*)m->part.p, np, grad,
           m->master.p, m->m1.p, m->m2.p, m->dev, 0, 0.f, 0.f, 0.f, 0.f, 1.f, 1.f);
    const double l = host_loss(m, np, n, s);
    if (loss) *loss = l;
  });
}

int les_mlp_adam_step(les_mlp* m, const void* feat, const float* target, long long n, float lr, double* loss,
                      void* stream) {
  if (!m || !(lr > 0.f)) return LES_EINVAL;
  return mlp_guard(m, [&] {
    check_samples(feat, target, n);
    cudaStream_t s = (cudaStream_t)stream;
    const int np = train_partials(m, feat, target, n, s);
    m->adam_step++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = (float)(1.0 - std::pow(0.9, m->adam_step)), c2 = (float)(1.0 - std::pow(0.999, m->adam_step));
    launch(k_mlp_reduce_adam, dim3(cdiv(kMlpNParam, 256)), dim3(256), 0, s, (const float*)m->part.p, np, m->grad.p,
           m->master.p, m->m1.p, m->m2.p, m->dev, 1, lr, b1, b2, 1e-8f, c1, c2);
    if (loss) *loss = host_loss(m, np, n, s);
  });
}

}  // extern "C"

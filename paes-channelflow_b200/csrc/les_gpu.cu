// les_gpu.cu -- the C ABI (include/les_gpu.h): handles, status codes, twiddle
// tables, operator-level entry points.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <initializer_list>
#include <vector>
#include <functional>
#include <memory>
#include <mutex>
#include <set>
#include <string>
#include <thread>

#include "../../include/les_mlp.h"
#include "les_engine.cuh"

namespace les {
const MlpDev* mlp_dev_params(const les_mlp* m);
int mlp_device(const les_mlp* m);
}  // namespace les

namespace les {

EngineBase* make_engine_fp64(const les_config& c);
EngineBase* make_engine_fp32(const les_config& c);
cudaError_t upload_twiddles_engine_fp64();
cudaError_t upload_twiddles_engine_fp32();
cudaError_t upload_twiddles_ops();

thread_local long long* g_launch_counter = nullptr;
thread_local KernelTrace* g_trace = nullptr;

namespace {
std::mutex g_mu;
struct DeviceTables {
  void* tw64 = nullptr;
  void* tw32 = nullptr;
};
std::map<int, DeviceTables> g_tables;
std::set<std::pair<const void*, int>> g_smem_set;
}  // namespace

// Twiddle tables of the current (or given) device, built on first use:
// W_384^j in constant memory for the register DFTs and exp(-2 pi i j/N) for
// every supported N for the four-step outer twiddles.  Computed in long
// double on the host and rounded once.
const void* twiddles(int device, bool fp64) {
  if (device < 0) LES_CUDA(cudaGetDevice(&device));
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_tables.find(device);
  if (it == g_tables.end()) {
    int cur;
    LES_CUDA(cudaGetDevice(&cur));
    if (cur != device) LES_CUDA(cudaSetDevice(device));
    const long double pi = 3.141592653589793238462643383279502884L;
    LES_CUDA(upload_tu_twiddles());
    LES_CUDA(upload_twiddles_engine_fp64());
    LES_CUDA(upload_twiddles_engine_fp32());
    LES_CUDA(upload_twiddles_ops());
    std::vector<double2> t64(kTwTotal);
    std::vector<float2> t32(kTwTotal);
    for (int si = 0; si < kNumSizes; si++) {
      int n = kSizes[si], off = tw_off(n);
      for (int j = 0; j < n; j++) {
        long double a = -2.0L * pi * j / n;
        t64[off + j] = make_double2((double)cosl(a), (double)sinl(a));
        t32[off + j] = make_float2((float)cosl(a), (float)sinl(a));
      }
    }
    DeviceTables dt;
    LES_CUDA(cudaMalloc(&dt.tw64, sizeof(double2) * kTwTotal));
    LES_CUDA(cudaMalloc(&dt.tw32, sizeof(float2) * kTwTotal));
    LES_CUDA(cudaMemcpy(dt.tw64, t64.data(), sizeof(double2) * kTwTotal, cudaMemcpyHostToDevice));
    LES_CUDA(cudaMemcpy(dt.tw32, t32.data(), sizeof(float2) * kTwTotal, cudaMemcpyHostToDevice));
    it = g_tables.emplace(device, dt).first;
    if (cur != device) LES_CUDA(cudaSetDevice(cur));
  }
  return fp64 ? it->second.tw64 : it->second.tw32;
}

void set_smem_limit(const void* func, size_t bytes) {
  int dev;
  LES_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_mu);
  if (g_smem_set.count({func, dev})) return;
  LES_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  g_smem_set.insert({func, dev});
}

}  // namespace les

using namespace les;

// A restart file written by a host thread while the handle keeps running.
struct FieldJob {
  std::thread th;
  int rc = LES_OK;
  std::string err;
};

struct les_handle {
  les_config cfg;
  int device = 0;
  std::unique_ptr<EngineBase> eng;
  std::string err;
  long long launches = 0;
  std::unique_ptr<FieldJob> fjob;
};

namespace {
std::string g_static_err;

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int d) {
    cudaGetDevice(&prev);
    if (prev != d) cudaSetDevice(d);
  }
  ~DeviceGuard() {
    int cur;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

template <class F>
int guarded(les_handle* h, F&& fn) {
  if (!h) return LES_EINVAL;
  DeviceGuard g(h->device);
  g_launch_counter = &h->launches;
  int rc = LES_OK;
  try {
    fn();
  } catch (CudaError& e) {
    h->err = e.what();
    rc = e.code;
  } catch (std::invalid_argument& e) {
    h->err = e.what();
    rc = LES_EINVAL;
  } catch (std::logic_error& e) {
    h->err = e.what();
    rc = LES_ESTATE;
  } catch (std::exception& e) {
    h->err = e.what();
    rc = LES_EINVAL;
  }
  g_launch_counter = nullptr;
  return rc;
}

int check_config(const les_config* c, std::string& why) {
  if (!c) { why = "null config"; return LES_EINVAL; }
  if (!supported_small(c->nnx) || !supported_small(c->nny)) {
    why = "nnx, nny must be one of 16, 32, 64, 96, 128, 192, 256, 384, 512";
    return LES_EINVAL;
  }
  if (c->nnz < 4) { why = "nnz must be >= 4"; return LES_EINVAL; }
  if (c->imodel != LES_SGS_DEARDORFF && c->imodel != LES_SGS_SMAG && c->imodel != LES_SGS_LEARNED) {
    why = "imodel must be 3, 4 or 5";
    return LES_EINVAL;
  }
  if (c->isurface < 1 || c->isurface > 6) { why = "isurface must be 1..6"; return LES_EINVAL; }
  if (c->imodel == LES_SGS_LEARNED && c->tke_production) {
    why = "the learned closure keeps the shipped TKE equation (tke_production = 0)";
    return LES_EINVAL;
  }
  if (c->precision != LES_PREC_FP64 && c->precision != LES_PREC_MIXED) {
    why = "precision must be 8 (FP64) or 4 (mixed)";
    return LES_EINVAL;
  }
  if (!(c->xl > 0 && c->yl > 0 && c->zl > 0 && c->z0 > 0 && c->z0 < c->zl / c->nnz / 2)) {
    why = "domain lengths must be positive and z0 < dz/2";
    return LES_EINVAL;
  }
  return LES_OK;
}
}  // namespace

// ---- operator level ----
static thread_local std::string g_op_err;
namespace les {
// Message for les_op_last_error() from the other translation units.
void set_op_error(const char* msg) { g_op_err = msg ? msg : ""; }
}  // namespace les

template <class F>
static int op_guard(F&& fn) {
  try {
    fn();
    return LES_OK;
  } catch (CudaError& e) {
    g_op_err = e.what();
    return e.code;
  } catch (std::exception& e) {
    g_op_err = e.what();
    return LES_EINVAL;
  }
}


// Scratch of the expand / compress / deal entry points: stream-ordered
// allocations released on the same stream.
template <class T>
static void with_scratch(size_t n1, size_t n2, cudaStream_t s, const std::function<void(cx<T>*, cx<T>*)>& fn) {
  void* a = nullptr;
  void* b = nullptr;
  LES_CUDA(cudaMallocAsync(&a, std::max<size_t>(n1, 1) * sizeof(cx<T>), s));
  cudaError_t e2 = cudaMallocAsync(&b, std::max<size_t>(n2, 1) * sizeof(cx<T>), s);
  if (e2 != cudaSuccess) {
    cudaFreeAsync(a, s);
    throw CudaError("cudaMallocAsync", LES_ENOMEM);
  }
  try {
    fn((cx<T>*)a, (cx<T>*)b);
  } catch (...) {
    cudaFreeAsync(a, s);
    cudaFreeAsync(b, s);
    throw;
  }
  LES_CUDA(cudaFreeAsync(a, s));
  LES_CUDA(cudaFreeAsync(b, s));
}


extern "C" {

const char* les_op_last_error(void) { return g_op_err.c_str(); }

void les_gpu_default_config(les_config* c) {
  if (!c) return;
  std::memset(c, 0, sizeof(*c));
  // default.f90:1-32 and les.F90:92-121; the channel configs override these
  c->nnx = 32; c->nny = 32; c->nnz = 32;
  c->imodel = LES_SGS_DEARDORFF; c->isurface = 6; c->tke_production = 0; c->precision = LES_PREC_FP64;
  c->device = 0;
  c->xl = 5000.0; c->yl = 5000.0; c->zl = 2000.0; c->z0 = 0.16;
  c->dt = 1.0; c->cb = 0.0; c->skc = 1.0; c->nu = 0.0;
  c->ugal = 0.0; c->vgal = 0.0; c->ufree = 0.0;
  c->emin = 1.0e-6; c->forcing = 0.016;
}

size_t les_gpu_config_size(void) { return sizeof(les_config); }

int les_gpu_init(const les_config* cfg, les_handle** out) {
  if (!out) return LES_EINVAL;
  *out = nullptr;
  std::string why;
  int rc = check_config(cfg, why);
  if (rc) { g_static_err = why; return rc; }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    g_static_err = "no CUDA device";
    return LES_ENOTBUILT;
  }
  if (cfg->device < 0 || cfg->device >= ndev) { g_static_err = "bad device ordinal"; return LES_EINVAL; }
  les_handle* h = new les_handle();
  h->cfg = *cfg;
  h->device = cfg->device;
  rc = guarded(h, [&] {
    if (cfg->precision == LES_PREC_FP64) h->eng.reset(make_engine_fp64(*cfg));
    else h->eng.reset(make_engine_fp32(*cfg));
  });
  if (rc) {
    g_static_err = h->err;
    delete h;
    return rc;
  }
  *out = h;
  return LES_OK;
}

void les_gpu_finalize(les_handle* h) {
  if (!h) return;
  if (h->fjob && h->fjob->th.joinable()) h->fjob->th.join();
  {
    DeviceGuard g(h->device);
    h->eng.reset();
  }
  delete h;
}

const char* les_gpu_last_error(les_handle* h) { return h ? h->err.c_str() : g_static_err.c_str(); }

static int check_rb(int rb) { return (rb == 4 || rb == 8) ? LES_OK : LES_EINVAL; }

int les_gpu_upload(les_handle* h, const void* u, const void* v, const void* w, const void* e, const void* p,
                   int real_bytes) {
  if (check_rb(real_bytes)) return LES_EINVAL;
  return guarded(h, [&] { h->eng->upload(u, v, w, e, p, real_bytes); });
}
int les_gpu_download(les_handle* h, void* u, void* v, void* w, void* e, void* p, int real_bytes) {
  if (check_rb(real_bytes)) return LES_EINVAL;
  return guarded(h, [&] { h->eng->download(u, v, w, e, p, real_bytes); });
}
int les_gpu_regrid(les_handle* dst, les_handle* src) {
  if (!dst || !src) return LES_EINVAL;
  if (dst == src) {
    dst->err = "les_gpu_regrid: source and destination are the same handle";
    return LES_EINVAL;
  }
  return guarded(dst, [&] { dst->eng->regrid_from(*src->eng); });
}
int les_gpu_upload_tendencies(les_handle* h, const void* ru, const void* rv, const void* rw, const void* re,
                              int real_bytes) {
  if (check_rb(real_bytes)) return LES_EINVAL;
  return guarded(h, [&] { h->eng->upload_tend(ru, rv, rw, re, real_bytes); });
}
int les_gpu_download_tendencies(les_handle* h, void* ru, void* rv, void* rw, void* re, int real_bytes) {
  if (check_rb(real_bytes)) return LES_EINVAL;
  return guarded(h, [&] { h->eng->download_tend(ru, rv, rw, re, real_bytes); });
}

// Ghost planes are rebuilt inside comp1 from exactly the values lower/upper
// copy (lowerbc.f90:9-18, upperbc.f90:12-28), so these only validate.
int les_gpu_lower(les_handle* h) { return h ? LES_OK : LES_EINVAL; }
int les_gpu_upper(les_handle* h) { return h ? LES_OK : LES_EINVAL; }

int les_gpu_comp1(les_handle* h, int it, int mnout, int istage, double dtab1, double dtab2, double xkmax) {
  (void)it;
  if (istage < 1 || istage > 3 || !(dtab1 > 0)) return LES_EINVAL;
  return guarded(h, [&] { h->eng->comp1(mnout != 0, istage, dtab1, dtab2, xkmax); });
}
int les_gpu_comprhs(les_handle* h, double dtabm) {
  if (!(dtabm > 0)) return LES_EINVAL;
  return guarded(h, [&] { h->eng->comprhs(dtabm); });
}
int les_gpu_press(les_handle* h) { return guarded(h, [&] { h->eng->press(); }); }
int les_gpu_comp2(les_handle* h, double dtab1) {
  if (!(dtab1 > 0)) return LES_EINVAL;
  return guarded(h, [&] { h->eng->comp2(dtab1); });
}
int les_gpu_stage(les_handle* h, int it, int mnout, int istage, double dtab1, double dtab2, double xkmax) {
  (void)it;
  if (istage < 1 || istage > 3 || !(dtab1 > 0)) return LES_EINVAL;
  return guarded(h, [&] { h->eng->stage(mnout != 0, istage, dtab1, dtab2, xkmax); });
}
int les_gpu_step(les_handle* h, int it, int mnout, double dt) {
  if (!(dt > 0)) return LES_EINVAL;
  return guarded(h, [&] { h->eng->step(mnout != 0 || it == 0, dt); });
}

int les_gpu_stats(les_handle* h, double* meanbuf, double* scalars) {
  return guarded(h, [&] { h->eng->stats(meanbuf, scalars); });
}
int les_gpu_spectra(les_handle* h, int field, int iz, double* zspecx, double* zspec2d) {
  if (!h || field < 0 || field > 3 || iz < 1 || iz > h->cfg.nnz || !zspecx || !zspec2d) return LES_EINVAL;
  return guarded(h, [&] { h->eng->spectra(field, iz, zspecx, zspec2d); });
}

int les_gpu_sync(les_handle* h, double timeout_s) {
  if (!h) return LES_EINVAL;
  int rc = guarded(h, [&] {
    cudaStream_t s = h->eng->stream();
    auto t0 = std::chrono::steady_clock::now();
    for (;;) {
      cudaError_t q = cudaStreamQuery(s);
      if (q == cudaSuccess) break;
      if (q != cudaErrorNotReady) throw CudaError(std::string("stream: ") + cudaGetErrorString(q), LES_ECUDA);
      double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      if (timeout_s >= 0 && el > timeout_s) throw CudaError("les_gpu_sync: timed out", LES_ETIMEOUT);
      std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
  });
  if (rc) return rc;
  int flags = 0;
  rc = guarded(h, [&] { flags = h->eng->read_error(); });
  if (rc) return rc;
  // a tensor-core wait that ran out leaves the network's stresses unset, so
  // it is reported before the NaN or wall-model states it may cause
  if (flags & ERR_MMA_TIMEOUT) { h->err = "a tensor-core MMA did not complete within its wait limit"; return LES_ETIMEOUT; }
  if (flags & ERR_UTAU) { h->err = "stop because utau > 10 (wall model blow-up guard)"; return LES_EUTAU; }
  if (flags & ERR_NAN) { h->err = "NaN/Inf in the state"; return LES_ENAN; }
  return LES_OK;
}

int les_gpu_make_ic(les_handle* h, unsigned long long seed, double ub, double amp, double utau, double e0) {
  return guarded(h, [&] { h->eng->make_ic(seed, ub, amp, utau, e0); });
}
int les_gpu_cfl_dt(les_handle* h, double cfl, double* dt) {
  if (!dt) return LES_EINVAL;
  return guarded(h, [&] { *dt = h->eng->cfl_dt(cfl); });
}
long long les_gpu_kernel_launches(les_handle* h) { return h ? h->launches : 0; }
void* les_gpu_stream(les_handle* h) { return (h && h->eng) ? (void*)h->eng->stream() : nullptr; }

int les_gpu_profile_stage(les_handle* h, int istage, double dt, double* ms, const void** kernels, int cap,
                          int* nkernels) {
  if (!h || istage < 1 || istage > 3 || !(dt > 0) || !nkernels) return LES_EINVAL;
  KernelTrace tr;
  cudaEvent_t start = nullptr;
  int rc = guarded(h, [&] {
    cudaStream_t s = h->eng->stream();
    LES_CUDA(cudaEventCreate(&start));
    LES_CUDA(cudaEventRecord(start, s));
    g_trace = &tr;
    try {
      h->eng->stage_eager(false, istage, dt);
    } catch (...) {
      g_trace = nullptr;
      throw;
    }
    g_trace = nullptr;
    LES_CUDA(cudaStreamSynchronize(s));
    int n = (int)tr.ev.size();
    *nkernels = n;
    for (int i = 0; i < n && i < cap; i++) {
      float t = 0.f;
      LES_CUDA(cudaEventElapsedTime(&t, i == 0 ? start : tr.ev[i - 1], tr.ev[i]));
      if (ms) ms[i] = t;
      if (kernels) kernels[i] = tr.fn[i];
    }
  });
  for (auto e : tr.ev) cudaEventDestroy(e);
  if (start) cudaEventDestroy(start);
  return rc;
}

int les_gpu_kernel_name(const void* kernel, char* buf, int cap) {
  if (!kernel || !buf || cap < 1) return LES_EINVAL;
  const char* name = nullptr;
  if (cudaFuncGetName(&name, kernel) != cudaSuccess || !name) {
    cudaGetLastError();
    buf[0] = 0;
    return LES_EINVAL;
  }
  snprintf(buf, (size_t)cap, "%s", name);
  return LES_OK;
}

int les_op_xderiv(const void* ain, void* ax, int n1, int n2, int howmany, double xl, int real_bytes, void* stream) {
  if (!ain || !ax || n1 <= 0 || n2 <= 0 || howmany <= 0 || !(xl > 0) || check_rb(real_bytes)) return LES_EINVAL;
  return op_guard([&] {
    if (real_bytes == 8) op_xderiv<double>((const double*)ain, (double*)ax, n1, n2, howmany, xl, (cudaStream_t)stream);
    else op_xderiv<float>((const float*)ain, (float*)ax, n1, n2, howmany, xl, (cudaStream_t)stream);
  });
}
int les_op_yderiv(const void* ain, void* ay, int n1, int n2, int howmany, double yl, int real_bytes, void* stream) {
  if (!ain || !ay || n1 <= 0 || n2 <= 0 || howmany <= 0 || !(yl > 0) || check_rb(real_bytes)) return LES_EINVAL;
  return op_guard([&] {
    if (real_bytes == 8) op_yderiv<double>((const double*)ain, (double*)ay, n1, n2, howmany, yl, (cudaStream_t)stream);
    else op_yderiv<float>((const float*)ain, (float*)ay, n1, n2, howmany, yl, (cudaStream_t)stream);
  });
}

int les_op_expand(const void* xs, void* xl, int nx, int ny, int howmany, int real_bytes, void* stream) {
  if (!xs || !xl || howmany <= 0 || check_rb(real_bytes) || !supported_small(nx) || !supported_small(ny))
    return LES_EINVAL;
  cudaStream_t s = (cudaStream_t)stream;
  size_t n1 = (size_t)howmany * ny * (nx / 2), n2 = (size_t)howmany * (3 * ny / 2) * (nx / 2);
  return op_guard([&] {
    if (real_bytes == 8)
      with_scratch<double>(n1, n2, s, [&](cx<double>* a, cx<double>* b) {
        op_expand<double>((const double*)xs, (double*)xl, nx, ny, howmany, s, a, b);
      });
    else
      with_scratch<float>(n1, n2, s, [&](cx<float>* a, cx<float>* b) {
        op_expand<float>((const float*)xs, (float*)xl, nx, ny, howmany, s, a, b);
      });
  });
}
int les_op_compress(const void* xl, void* xs, int nx, int ny, int howmany, int real_bytes, void* stream) {
  if (!xs || !xl || howmany <= 0 || check_rb(real_bytes) || !supported_small(nx) || !supported_small(ny))
    return LES_EINVAL;
  cudaStream_t s = (cudaStream_t)stream;
  size_t n1 = (size_t)howmany * ny * (nx / 2), n2 = (size_t)howmany * (3 * ny / 2) * (nx / 2);
  return op_guard([&] {
    if (real_bytes == 8)
      with_scratch<double>(n1, n2, s, [&](cx<double>* a, cx<double>* b) {
        op_compress<double>((const double*)xl, (double*)xs, nx, ny, howmany, s, a, b);
      });
    else
      with_scratch<float>(n1, n2, s, [&](cx<float>* a, cx<float>* b) {
        op_compress<float>((const float*)xl, (float*)xs, nx, ny, howmany, s, a, b);
      });
  });
}
int les_op_deal(void* x, int nx, int ny, int howmany, int real_bytes, void* stream) {
  if (!x || howmany <= 0 || check_rb(real_bytes) || !supported_small(nx) || !supported_small(ny)) return LES_EINVAL;
  cudaStream_t s = (cudaStream_t)stream;
  size_t n1 = (size_t)howmany * ny * (nx / 2);
  return op_guard([&] {
    if (real_bytes == 8)
      with_scratch<double>(n1, 1, s, [&](cx<double>* a, cx<double>*) { op_deal<double>((double*)x, nx, ny, howmany, s, a); });
    else
      with_scratch<float>(n1, 1, s, [&](cx<float>* a, cx<float>*) { op_deal<float>((float*)x, nx, ny, howmany, s, a); });
  });
}
int les_op_tridv(void* bdar, int ny, int n, int real_bytes, void* stream) {
  if (!bdar || ny <= 0 || n <= 0 || real_bytes != 8) return LES_EINVAL;
  return op_guard([&] {
    launch(k_op_tridv, dim3(cdiv(ny, 128)), dim3(128), 0, (cudaStream_t)stream, (double*)bdar, ny, n);
  });
}

}  // extern "C"

// ---- learned closure (les_mlp.h) ----
extern "C" int les_gpu_set_mlp(les_handle* h, les_mlp* m, double re_tau) {
  if (!h) return LES_EINVAL;
  if (m) {
    if (h->cfg.imodel != LES_SGS_LEARNED) { h->err = "les_gpu_set_mlp: imodel is not LES_SGS_LEARNED"; return LES_EINVAL; }
    if (les::mlp_device(m) != h->device) { h->err = "les_gpu_set_mlp: network and handle on different devices"; return LES_EINVAL; }
    if (!(re_tau > 0)) { h->err = "les_gpu_set_mlp: re_tau must be positive"; return LES_EINVAL; }
  }
  return guarded(h, [&] { h->eng->set_mlp(m ? les::mlp_dev_params(m) : nullptr, re_tau); });
}

extern "C" int les_gpu_learned_status(les_handle* h, int* used, double* dissipation) {
  if (!h) return LES_EINVAL;
  return guarded(h, [&] { h->eng->learned_status(used, dissipation); });
}

extern "C" int les_gpu_set_learned_guard(les_handle* h, double ratio) {
  if (!h || !(ratio == ratio)) return LES_EINVAL;
  return guarded(h, [&] { h->eng->set_learned_guard(ratio); });
}

extern "C" int les_gpu_learned_reference(les_handle* h, double* dissipation) {
  if (!h || !dissipation) return LES_EINVAL;
  return guarded(h, [&] { *dissipation = h->eng->learned_reference(); });
}

extern "C" int les_gpu_learned_counts(les_handle* h, long long* stages, long long* used) {
  if (!h) return LES_EINVAL;
  return guarded(h, [&] { h->eng->learned_counts(stages, used); });
}

extern "C" int les_gpu_learn_filter(les_handle* h, int fxy, int fz, int with_model, double* out) {
  if (!h || !out) return LES_EINVAL;
  return guarded(h, [&] {
    h->eng->learn_filter(fxy, fz, with_model, out);
    LES_CUDA(cudaStreamSynchronize(h->eng->stream()));
  });
}

extern "C" int les_gpu_learned_features(les_handle* h, float* feat) {
  if (!h || !feat) return LES_EINVAL;
  if ((uintptr_t)feat % 16) { h->err = "les_gpu_learned_features: feat must be 16-byte aligned"; return LES_EINVAL; }
  return guarded(h, [&] {
    h->eng->learned_features(0.0, feat);
    LES_CUDA(cudaStreamSynchronize(h->eng->stream()));
  });
}

// ---- restart files (read_write.f90, les.F90:69-82, 331-351) ----
// Fortran unformatted sequential records, each framed by its byte length
// as a 4-byte integer before and after it:
//   1: time, nnx, nny, nnz, xl, yl, zl      (reals, integers as 4 bytes)
//   2: dt, z0, utau                         (write_params)
//   3: divgls, fcor, ugtop, ugbot, vgtop, vgbot
//   3+iz, iz = 1..nnz: u, v, w, e, p(1:nnx,1:nny) of level iz (sav_field)
// Reals are real_bytes wide: 4 for the shipped build, 8 for -fdefault-real-8.
namespace {

struct Part { const void* p; size_t n; };

bool write_record(FILE* f, std::initializer_list<Part> parts) {
  size_t total = 0;
  for (const Part& q : parts) total += q.n;
  if (total > 0x7fffffffu) return false;
  const int32_t m = (int32_t)total;
  if (fwrite(&m, 4, 1, f) != 1) return false;
  for (const Part& q : parts)
    if (q.n && fwrite(q.p, 1, q.n, f) != q.n) return false;
  return fwrite(&m, 4, 1, f) == 1;
}

// reads one record of exactly `n` bytes into dst
bool read_record(FILE* f, void* dst, size_t n) {
  int32_t m0 = 0, m1 = 0;
  if (fread(&m0, 4, 1, f) != 1 || (size_t)m0 != n) return false;
  if (n && fread(dst, 1, n, f) != n) return false;
  return fread(&m1, 4, 1, f) == 1 && m1 == m0;
}

void put_real(std::vector<unsigned char>& b, double v, int rb) {
  const size_t o = b.size();
  b.resize(o + rb);
  if (rb == 8) std::memcpy(b.data() + o, &v, 8);
  else { const float x = (float)v; std::memcpy(b.data() + o, &x, 4); }
}
double get_real(const unsigned char* b, int rb) {
  if (rb == 8) { double v; std::memcpy(&v, b, 8); return v; }
  float x; std::memcpy(&x, b, 4); return (double)x;
}

// header records 1-3 -> dims, hdr[13] = time, xl, yl, zl, dt, z0, utau, divgls, fcor, ugtop, ugbot, vgtop, vgbot
int read_header(FILE* f, int rb, int* dims, double* hdr, std::string& why) {
  std::vector<unsigned char> r1(4 * rb + 12), r2(3 * rb), r3(6 * rb);
  if (!read_record(f, r1.data(), r1.size()) || !read_record(f, r2.data(), r2.size()) ||
      !read_record(f, r3.data(), r3.size())) {
    why = "not a .field file with real_bytes = " + std::to_string(rb);
    return LES_EINVAL;
  }
  hdr[0] = get_real(r1.data(), rb);
  std::memcpy(dims, r1.data() + rb, 12);
  for (int i = 0; i < 3; i++) hdr[1 + i] = get_real(r1.data() + rb + 12 + i * rb, rb);
  for (int i = 0; i < 3; i++) hdr[4 + i] = get_real(r2.data() + i * rb, rb);
  for (int i = 0; i < 6; i++) hdr[7 + i] = get_real(r3.data() + i * rb, rb);
  return LES_OK;
}

}  // namespace

extern "C" int les_gpu_field_header(const char* path, int real_bytes, int* dims, double* hdr) {
  if (!path || !dims || !hdr || (real_bytes != 4 && real_bytes != 8)) return LES_EINVAL;
  FILE* f = fopen(path, "rb");
  if (!f) { g_static_err = std::string("cannot open ") + path; return LES_EINVAL; }
  std::string why;
  const int rc = read_header(f, real_bytes, dims, hdr, why);
  fclose(f);
  if (rc) g_static_err = why;
  return rc;
}

extern "C" int les_gpu_field_wait(les_handle* h) {
  if (!h) return LES_EINVAL;
  if (!h->fjob) return LES_OK;
  if (h->fjob->th.joinable()) h->fjob->th.join();
  const int rc = h->fjob->rc;
  if (rc) h->err = h->fjob->err;
  h->fjob.reset();
  return rc;
}

extern "C" int les_gpu_write_field(les_handle* h, const char* path, double time, int real_bytes, int async) {
  if (!h || !path || (real_bytes != 4 && real_bytes != 8)) return LES_EINVAL;
  int rc = les_gpu_field_wait(h);  // one file at a time
  if (rc) return rc;
  const les_config c = h->cfg;
  const size_t ps = (size_t)c.nnx * c.nny, n = ps * c.nnz, bytes = n * real_bytes;
  unsigned char* buf[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  double utau = 0.0;
  rc = guarded(h, [&] {
    std::vector<double> mb((size_t)19 * c.nnz), sc(5);
    h->eng->stats(mb.data(), sc.data());
    utau = sc[0];
    for (auto& b : buf) LES_CUDA(cudaMallocHost((void**)&b, bytes));
    h->eng->download(buf[0], buf[1], buf[2], buf[3], buf[4], real_bytes);
  });
  if (rc) {
    for (auto& b : buf) if (b) cudaFreeHost(b);
    return rc;
  }
  std::unique_ptr<FieldJob> job(new FieldJob());
  FieldJob* jp = job.get();
  const std::string fname(path);
  auto work = [=]() {
    FILE* f = fopen(fname.c_str(), "wb");
    bool ok = f != nullptr;
    if (ok) {
      const int rb = real_bytes;
      std::vector<unsigned char> r1, r2, r3;
      put_real(r1, time, rb);
      const int32_t d[3] = {c.nnx, c.nny, c.nnz};
      const size_t o = r1.size();
      r1.resize(o + 12);
      std::memcpy(r1.data() + o, d, 12);
      put_real(r1, c.xl, rb); put_real(r1, c.yl, rb); put_real(r1, c.zl, rb);
      put_real(r2, c.dt, rb); put_real(r2, c.z0, rb); put_real(r2, utau, rb);
      // divgls, fcor, ugtop, ugbot, vgtop, vgbot.  The post-processing
      // programs take the run's Galilean shift from this record as
      // ugal = (max(0, max(ugtop, ugbot)) + min(0, min(ugtop, ugbot))) / 2
      // (calc_pdf.f90:99-100, calc_spectra.f90:130-131,
      // calc_integral_ls.f90:87-88); ugtop = ugbot = 2 ugal gives back ugal
      // for either sign (likewise v).  fcor is default.f90:23's value.
      put_real(r3, 0.0, rb);
      put_real(r3, 1e-4, rb);
      put_real(r3, 2.0 * c.ugal, rb); put_real(r3, 2.0 * c.ugal, rb);
      put_real(r3, 2.0 * c.vgal, rb); put_real(r3, 2.0 * c.vgal, rb);
      ok = write_record(f, {{r1.data(), r1.size()}}) && write_record(f, {{r2.data(), r2.size()}}) &&
           write_record(f, {{r3.data(), r3.size()}});
      const size_t pl = ps * rb;
      for (int iz = 0; ok && iz < c.nnz; iz++) {
        const size_t off = (size_t)iz * pl;
        ok = write_record(f, {{buf[0] + off, pl}, {buf[1] + off, pl}, {buf[2] + off, pl}, {buf[3] + off, pl},
                              {buf[4] + off, pl}});
      }
      ok = (fclose(f) == 0) && ok;
    }
    for (auto b : buf) cudaFreeHost(b);
    if (!ok) {
      jp->rc = LES_EINVAL;
      jp->err = "writing " + fname + " failed";
    }
  };
  if (async) {
    job->th = std::thread(work);
    h->fjob = std::move(job);
    return LES_OK;
  }
  work();
  rc = job->rc;
  if (rc) h->err = job->err;
  return rc;
}

extern "C" int les_gpu_read_field(les_handle* h, const char* path, int real_bytes, double* time) {
  if (!h || !path || (real_bytes != 4 && real_bytes != 8)) return LES_EINVAL;
  int rc = les_gpu_field_wait(h);
  if (rc) return rc;
  FILE* f = fopen(path, "rb");
  if (!f) { h->err = std::string("cannot open ") + path; return LES_EINVAL; }
  int dims[3];
  double hdr[13];
  rc = read_header(f, real_bytes, dims, hdr, h->err);
  if (!rc && (dims[0] != h->cfg.nnx || dims[1] != h->cfg.nny || dims[2] != h->cfg.nnz)) {
    h->err = "restart file grid differs from the handle's";
    rc = LES_EINVAL;
  }
  if (rc) { fclose(f); return rc; }
  const size_t ps = (size_t)dims[0] * dims[1], n = ps * dims[2], pl = ps * real_bytes;
  std::vector<unsigned char> a[5], rec(5 * pl);
  for (auto& v : a) v.resize(n * real_bytes);
  for (int iz = 0; iz < dims[2]; iz++) {
    if (!read_record(f, rec.data(), rec.size())) {
      fclose(f);
      h->err = "restart file is truncated or has another layout";
      return LES_EINVAL;
    }
    for (int q = 0; q < 5; q++) std::memcpy(a[q].data() + (size_t)iz * pl, rec.data() + q * pl, pl);
  }
  fclose(f);
  if (time) *time = hdr[0];
  return guarded(h, [&] {
    h->eng->upload(a[0].data(), a[1].data(), a[2].data(), a[3].data(), a[4].data(), real_bytes);
  });
}

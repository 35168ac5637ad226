// les_engine.cuh -- host-side orchestration of the device-resident domain.
// Engine<T> owns every device array of one handle and enqueues the kernels
// of les_kernels.cuh on the handle's stream.  T is the arithmetic type of the
// padded-grid transforms, advection and SGS (double for the plain FP64 form,
// float for the mixed form); the pressure solve, the kx=ky=0 modes and all
// reductions are FP64 in both forms.
#pragma once
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <cstdint>
#include <map>
#include <mutex>
#include <set>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "../../include/les_gpu.h"
#include "les_fused.cuh"
#include "les_learned.cuh"
#include "les_regrid.cuh"

namespace les {

struct CudaError : std::runtime_error {
  int code;
  CudaError(const std::string& m, int c) : std::runtime_error(m), code(c) {}
};

#define LES_CUDA(call)                                                                               \
  do {                                                                                               \
    cudaError_t _e = (call);                                                                         \
    if (_e != cudaSuccess)                                                                           \
      throw ::les::CudaError(std::string(#call) + ": " + cudaGetErrorString(_e),                     \
                             _e == cudaErrorMemoryAllocation ? LES_ENOMEM : LES_ECUDA);              \
  } while (0)

// Twiddle tables and shared-memory limits (defined in les_gpu.cu).
const void* twiddles(int device, bool fp64);
void set_smem_limit(const void* func, size_t bytes);
extern thread_local long long* g_launch_counter;

// Optional per-kernel timing: when set, an event is recorded after every
// launch on the launching stream (les_gpu_profile_stage).
struct KernelTrace {
  std::vector<cudaEvent_t> ev;
  std::vector<const void*> fn;
};
extern thread_local KernelTrace* g_trace;

template <class... KArgs, class... Args>
inline void launch(void (*k)(KArgs...), dim3 g, dim3 b, size_t smem, cudaStream_t s, Args... args) {
  if (g.x == 0 || g.y == 0 || g.z == 0) return;
  if (smem > 48 * 1024) set_smem_limit((const void*)k, smem);
  k<<<g, b, smem, s>>>(args...);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) throw CudaError(std::string("kernel launch: ") + cudaGetErrorString(e), LES_ECUDA);
  if (g_launch_counter) ++*g_launch_counter;
  if (g_trace) {
    cudaEvent_t ev;
    LES_CUDA(cudaEventCreate(&ev));
    LES_CUDA(cudaEventRecord(ev, s));
    g_trace->ev.push_back(ev);
    g_trace->fn.push_back((const void*)k);
  }
}

inline unsigned cdiv(size_t a, size_t b) { return (unsigned)((a + b - 1) / b); }
constexpr unsigned kWallBlocks = 148;  // one partial sum per SM-sized block group

// Compile-time dispatch of the small-grid transform length.
template <class F> bool with_small(int n, F&& f) {
  switch (n) {
    case 16: f(std::integral_constant<int, 16>{}); return true;
    case 32: f(std::integral_constant<int, 32>{}); return true;
    case 64: f(std::integral_constant<int, 64>{}); return true;
    case 96: f(std::integral_constant<int, 96>{}); return true;
    case 128: f(std::integral_constant<int, 128>{}); return true;
    case 192: f(std::integral_constant<int, 192>{}); return true;
    case 256: f(std::integral_constant<int, 256>{}); return true;
    case 384: f(std::integral_constant<int, 384>{}); return true;
    case 512: f(std::integral_constant<int, 512>{}); return true;
    default: return false;
  }
}
template <class F> bool with_any(int n, F&& f) {
  if (with_small(n, f)) return true;
  switch (n) {
    case 24: f(std::integral_constant<int, 24>{}); return true;
    case 48: f(std::integral_constant<int, 48>{}); return true;
    case 144: f(std::integral_constant<int, 144>{}); return true;
    case 288: f(std::integral_constant<int, 288>{}); return true;
    case 576: f(std::integral_constant<int, 576>{}); return true;
    case 768: f(std::integral_constant<int, 768>{}); return true;
    default: return false;
  }
}
inline bool supported_small(int n) { return with_small(n, [](auto) {}); }
inline bool supported_any(int n) { return with_any(n, [](auto) {}); }

template <class T> struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  void alloc(size_t count) {
    n = count;
    if (count) LES_CUDA(cudaMalloc((void**)&p, count * sizeof(T)));
    if (count) LES_CUDA(cudaMemset(p, 0, count * sizeof(T)));
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
};

// Device scratch of one call, freed when the call returns (also on errors).
struct TmpDev {
  std::vector<void*> p;
  TmpDev() = default;
  TmpDev(const TmpDev&) = delete;
  TmpDev& operator=(const TmpDev&) = delete;
  ~TmpDev() {
    for (void* q : p) cudaFree(q);
  }
  template <class U> U* get(size_t n) {
    void* q = nullptr;
    LES_CUDA(cudaMalloc(&q, (n ? n : 1) * sizeof(U)));
    p.push_back(q);
    return (U*)q;
  }
};

// Operator-level helpers on caller buffers (les_op_* entry points).
template <class T>
void op_expand(const T* in, T* out, int nx, int ny, int howmany, cudaStream_t s, cx<T>* t1, cx<T>* t2);
template <class T>
void op_compress(const T* in, T* out, int nx, int ny, int howmany, cudaStream_t s, cx<T>* t1, cx<T>* t2);
template <class T> void op_deal(T* x, int nx, int ny, int howmany, cudaStream_t s, cx<T>* t1);
template <class T> void op_xderiv(const T* in, T* out, int n1, int n2, int howmany, double len, cudaStream_t s);
template <class T> void op_yderiv(const T* in, T* out, int n1, int n2, int howmany, double len, cudaStream_t s);

// ---------------------------------------------------------------------------
struct EngineBase {
  virtual ~EngineBase() {}
  virtual void upload(const void* u, const void* v, const void* w, const void* e, const void* p, int rb) = 0;
  virtual void download(void* u, void* v, void* w, void* e, void* p, int rb) = 0;
  virtual void upload_tend(const void* ru, const void* rv, const void* rw, const void* re, int rb) = 0;
  virtual void download_tend(void* ru, void* rv, void* rw, void* re, int rb) = 0;
  virtual void comp1(bool mnout, int istage, double dtab1, double dtab2, double xkmax) = 0;
  virtual void comprhs(double dtabm) = 0;
  virtual void press() = 0;
  virtual void comp2(double dtab1) = 0;
  virtual void stage(bool mnout, int istage, double dtab1, double dtab2, double xkmax) = 0;
  virtual void step(bool mnout, double dt) = 0;
  virtual void stats(double* meanbuf, double* scalars) = 0;
  virtual void spectra(int field, int iz, double* zx, double* z2) = 0;
  virtual void make_ic(unsigned long long seed, double ub, double amp, double utau, double e0) = 0;
  virtual double cfl_dt(double cfl) = 0;
  virtual int read_error() = 0;
  virtual cudaStream_t stream() = 0;
  virtual void stage_eager(bool mnout, int istage, double dt) = 0;
  // learned closure: attach (or with p == nullptr detach) device parameters
  virtual void set_mlp(const MlpDev* p, double re_tau) = 0;
  virtual void learned_status(int* used, double* dissipation) = 0;
  // factor of the fallback test against the Deardorff dissipation (<= 0:
  // the sign test only) and the Deardorff mean dissipation of the last stage
  virtual void set_learned_guard(double ratio) = 0;
  virtual double learned_reference() = 0;
  // stages evaluated since the network was attached, and those that used it
  virtual void learned_counts(long long* stages, long long* used) = 0;
  virtual void learned_features(double re_tau, float* feat) = 0;
  virtual void learn_filter(int fxy, int fz, int with_model, double* out) = 0;
  // this state := the state of `src` regridded onto this grid (redim.f90)
  virtual void regrid_from(EngineBase& src) = 0;
};

template <class T>
struct Engine : EngineBase {
  les_config cfg;
  int dev;
  int NX, NY, NZ, MX, MY, KX;
  size_t ps, pb, nm, nmix;  // small plane, padded plane, modes/level, mixed plane
  cudaStream_t st = nullptr;
  const cx<T>* tw = nullptr;
  // spectral state
  DevBuf<cx<T>> uh, vh, wh, ruo, rvo, rwo, run, rvn, rwn;
  DevBuf<double> mu, mv, mru, mrv;
  DevBuf<cx<double>> ph, rscr;
  DevBuf<double> dscr;
  DevBuf<T> e, re;
  // work
  DevBuf<cx<T>> Xe, rem;
  DevBuf<cx<T>> mixed[8];
  DevBuf<T> pad[12];   // unfused path: padded physical fields
  DevBuf<T> flux[11];  // unfused path: flux fields
  // fused path (k_row_fused): clip corrections and wall-model planes
  bool fused = false;
  DevBuf<int> clipflag;
  DevBuf<T> ephys, dEX, dEY, wallpl;
  DevBuf<cx<T>> xout[8];  // Xu1..Xe2 written by k_row_fused (its inputs stay readable)
  DevBuf<double> divacc, sgsacc, wacc, acc;
  // per-(level, block) partial sums of divz and the SGS means, reduced into
  // divacc / sgsacc in a fixed order when the statistics are read
  DevBuf<double> divpart, sgspart;
  int nstat_parts = 0;
  DevBuf<WallParams> wp;
  DevBuf<int> err;
  DevBuf<unsigned long long> amax;
  // staging for transfers (small-grid physical)
  DevBuf<T> phys[4];
  DevBuf<unsigned char> stage_buf;
  // L2 prefetch of the y-column tiles by the TMA (les_tma.cuh): tensor maps
  // of k_y_inverse's spectral inputs and k_y_forward's mixed inputs, and the
  // prefetch distance in blocks (one resident wave; 0 = no prefetch)
  ColMaps yinv_maps{}, yfwd_maps{};
  unsigned yinv_pdist = 0, yfwd_pdist = 0;
  // learned closure (imodel = LES_SGS_LEARNED with a network attached)
  const MlpDev* mlp = nullptr;
  double re_tau = 0.0;
  int nsm = 148;
  DevBuf<cx<T>> lgy;   // [6][NZ][NY][KX] rows U, UY, V, VY, W, WY; then the tau rows th
  DevBuf<T> ltau;      // [8][NZ][NY][NX] tau at the cell centres + viscosity products
  DevBuf<uint4> lfeat; // [N][16] bf16 features
  DevBuf<float> fraw;  // [N][16] raw f32 features (training data)
  DevBuf<double> lpart, lstat, lnut;
  DevBuf<unsigned long long> lcount;  // [stages, stages that used the network]
  double lguard = 4.0;
  DevBuf<int> lflag;
  DevBuf<T> fscr, fcp;      // filter scratch: z-averaged fine planes, coarse planes
  DevBuf<cx<T>> fsh, fch;   // filter scratch: fine and coarse spectra
  // derived scalars
  double dz, dzm, dzm2, todzm, kx0, ky0, dsl, ceps, zody;
  // phase of the split entry points: 0 idle, 1 after comp1, 2 after comprhs, 3 after press
  int phase = 0;
  // CUDA graphs of whole steps, keyed by (dt bits, mnout)
  std::map<std::pair<uint64_t, int>, cudaGraphExec_t> graphs;

  explicit Engine(const les_config& c) : cfg(c) {
    LES_CUDA(cudaGetDevice(&dev));
    NX = c.nnx; NY = c.nny; NZ = c.nnz;
    MX = 3 * NX / 2; MY = 3 * NY / 2; KX = NX / 2;
    ps = (size_t)NX * NY; pb = (size_t)MX * MY; nm = (size_t)KX * NY; nmix = (size_t)MY * KX;
    dz = c.zl / NZ; dzm = 1.0 / dz; dzm2 = dzm * dzm; todzm = 0.5 / dz;
    const double pi = 4.0 * std::atan(1.0);
    kx0 = 2.0 * pi / c.xl; ky0 = 2.0 * pi / c.yl;
    double dx = c.xl / NX, dy = c.yl / NY;
    dsl = std::pow(dx * dy * dz, 1.0 / 3.0);
    ceps = 0.93 / dsl;
    zody = std::log(dz / 2.0 / c.z0);
    tw = (const cx<T>*)twiddles(dev, sizeof(T) == 8);
    LES_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    size_t ns = nm * NZ;
    for (auto* b : {&uh, &vh, &wh, &ruo, &rvo, &rwo, &run, &rvn, &rwn}) b->alloc(ns);
    for (auto* b : {&mu, &mv, &mru, &mrv}) b->alloc(NZ);
    ph.alloc(ns); rscr.alloc(ns); dscr.alloc(ns);
    e.alloc(ps * (NZ + 2)); re.alloc(ps * NZ);
    Xe.alloc(ns); rem.alloc(ns);
    for (auto& b : mixed) b.alloc(nmix * NZ);
    // the fused row kernel covers the Deardorff model without the optional
    // production term; Smagorinsky and tke_production use the unfused kernels
    fused = ((c.imodel == LES_SGS_DEARDORFF || c.imodel == LES_SGS_LEARNED) && c.tke_production == 0);
    LES_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    if (fused) {
      clipflag.alloc(NZ);
      ephys.alloc(pb * NZ); dEX.alloc(pb * NZ); dEY.alloc(pb * NZ);
      wallpl.alloc(pb * 4);
      for (auto& b : xout) b.alloc(nmix * NZ);
    } else {
      for (auto& b : pad) b.alloc(pb * NZ);
      for (auto& b : flux) b.alloc(pb * NZ);
    }
    divacc.alloc(NZ); sgsacc.alloc((size_t)NZ * 8); wacc.alloc((size_t)2 * kWallBlocks * 8); acc.alloc((size_t)NZ * 16);
    // one partial per padded row (k_row_fused) or per 256-point block (k_flux)
    nstat_parts = fused ? MY : (int)cdiv(pb, 256);
    divpart.alloc((size_t)NZ * nstat_parts); sgspart.alloc((size_t)NZ * nstat_parts * 6);
    wp.alloc(1); err.alloc(1); amax.alloc(4);
    for (auto& b : phys) b.alloc(ps * (NZ + 2));
    stage_buf.alloc(ps * NZ * 8);
    with_small(NY, [&](auto cn) { y_prefetch_setup<decltype(cn)::value>(); });
  }
  // Tensor maps and distances of the y-column prefetches.  The distance is
  // one resident wave of the kernel (resident blocks per SM x SMs, even so
  // that a k_y_forward block prefetches for a block of its own cluster rank
  // and a k_y_inverse field block for a field block); one wave ahead measured
  // faster than two or more.  Without the driver's tensor-map encoder or
  // with a geometry the TMA cannot box, the distance stays 0.
  template <int N> void y_prefetch_setup() {
    using CM = ColCfg<3 * N / 2, T>;
    auto wave = [&](const void* k, size_t smem) -> unsigned {
      if (smem > 48 * 1024) set_smem_limit(k, smem);
      int nb = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, CM::THREADS, smem) != cudaSuccess) {
        (void)cudaGetLastError();
        return 0;
      }
      return (unsigned)(nb * nsm) & ~1u;
    };
    void* src[4] = {uh.p, vh.p, wh.p, Xe.p};
    if (make_col_maps<T, N, CM::TC>(yinv_maps, src, 4, KX, NZ))
      yinv_pdist = wave((const void*)k_y_inverse<T, N>, CM::buf());
    void* X[8];
    for (int i = 0; i < 8; i++) X[i] = fused ? xout[i].p : mixed[i].p;
    if (make_col_maps<T, 3 * N / 2, CM::TC>(yfwd_maps, X, 8, KX, NZ))
      yfwd_pdist = wave((const void*)k_y_forward<T, N>, CM::buf() + (size_t)(3 * N / 2) * sizeof(cx<T>));
  }
  ~Engine() override {
    for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
    if (st) { cudaStreamSynchronize(st); cudaStreamDestroy(st); }
    for (auto* b : {&uh, &vh, &wh, &ruo, &rvo, &rwo, &run, &rvn, &rwn, &Xe, &rem}) b->release();
    for (auto* b : {&mu, &mv, &mru, &mrv, &dscr, &divacc, &sgsacc, &wacc, &acc, &divpart, &sgspart}) b->release();
    ph.release(); rscr.release(); e.release(); re.release(); wp.release(); err.release(); amax.release();
    stage_buf.release();
    for (auto& b : mixed) b.release();
    for (auto& b : pad) b.release();
    for (auto& b : flux) b.release();
    clipflag.release(); ephys.release(); dEX.release(); dEY.release(); wallpl.release();
    for (auto& b : xout) b.release();
    for (auto& b : phys) b.release();
    lgy.release(); ltau.release(); lfeat.release(); fraw.release(); lpart.release(); lnut.release(); lstat.release(); lflag.release(); lcount.release();
    fscr.release(); fcp.release(); fsh.release(); fch.release();
  }
  cudaStream_t stream() override { return st; }

  StageArgs args(double dtab1, double dtab2, double xkmax, int zeta, int mnout_sgs) const {
    StageArgs a;
    a.NX = NX; a.NY = NY; a.NZ = NZ; a.MX = MX; a.MY = MY; a.KX = KX;
    a.imodel = cfg.imodel == LES_SGS_SMAG ? 4 : 3;
    a.isurface = cfg.isurface; a.tke_production = cfg.tke_production; a.zeta = zeta; a.mnout_sgs = mnout_sgs;
    a.dz = dz; a.dzm = dzm; a.dzm2 = dzm2; a.todzm = todzm; a.kx0 = kx0; a.ky0 = ky0;
    a.emin = cfg.emin; a.ceps = ceps; a.dsl = dsl; a.forcing = cfg.forcing; a.nu = cfg.nu; a.xkmax = xkmax;
    a.dtab1 = dtab1; a.dtab2 = dtab2; a.dtabm = 1.0 / dtab1;
    a.zl = cfg.zl; a.ugal = cfg.ugal; a.vgal = cfg.vgal;
    return a;
  }

  // ---- transforms between the small physical grid and the spectral state ----
  // phys (NZ planes, x fastest) -> spectral [z][ky][kx] (deal semantics)
  void to_spectral(const T* src, cx<T>* dst, int nplanes) {
    with_small(NX, [&](auto cn) {
      constexpr int N = decltype(cn)::value;
      using C = RowCfg<N>;
      launch(k_row_r2c<T, N>, dim3(cdiv((size_t)nplanes * NY / 2 + 1, C::NT)), dim3(C::THREADS),
             C::template smem<T>(), st, src, Xe.p, nplanes * NY, KX, tw);
    });
    with_small(NY, [&](auto cn) {
      constexpr int N = decltype(cn)::value;
      using C = ColCfg<N, T>;
      launch(k_col_small<T, N, false>, dim3(cdiv(KX, C::TC), nplanes), dim3(C::THREADS), C::buf(), st,
             (const cx<T>*)Xe.p, dst, KX, (T)(1.0 / ((double)NX * NY)), tw);
    });
  }
  // spectral -> phys
  void to_physical(const cx<T>* src, T* dst, int nplanes) {
    with_small(NY, [&](auto cn) {
      constexpr int N = decltype(cn)::value;
      using C = ColCfg<N, T>;
      launch(k_col_small<T, N, true>, dim3(cdiv(KX, C::TC), nplanes), dim3(C::THREADS), C::buf(), st, src, Xe.p,
             KX, (T)1, tw);
    });
    with_small(NX, [&](auto cn) {
      constexpr int N = decltype(cn)::value;
      using C = RowCfg<N>;
      launch(k_row_c2r<T, N>, dim3(cdiv((size_t)nplanes * NY / 2 + 1, C::NT)), dim3(C::THREADS),
             C::template smem<T>(), st, (const cx<T>*)Xe.p, dst, nplanes * NY, KX, tw);
    });
  }
  // host array (rb bytes per real, NZ planes) -> device T array
  void h2d(const void* h, T* d, size_t n, int rb) {
    if (rb == (int)sizeof(T)) {
      LES_CUDA(cudaMemcpyAsync(d, h, n * sizeof(T), cudaMemcpyHostToDevice, st));
    } else {
      LES_CUDA(cudaMemcpyAsync(stage_buf.p, h, n * rb, cudaMemcpyHostToDevice, st));
      if (rb == 8) launch(k_convert<double, T>, dim3(cdiv(n, 256)), dim3(256), 0, st, (const double*)stage_buf.p, d, n);
      else launch(k_convert<float, T>, dim3(cdiv(n, 256)), dim3(256), 0, st, (const float*)stage_buf.p, d, n);
    }
  }
  void d2h(const T* d, void* h, size_t n, int rb) {
    if (rb == (int)sizeof(T)) {
      LES_CUDA(cudaMemcpyAsync(h, d, n * sizeof(T), cudaMemcpyDeviceToHost, st));
    } else {
      if (rb == 8) launch(k_convert<T, double>, dim3(cdiv(n, 256)), dim3(256), 0, st, d, (double*)stage_buf.p, n);
      else launch(k_convert<T, float>, dim3(cdiv(n, 256)), dim3(256), 0, st, d, (float*)stage_buf.p, n);
      LES_CUDA(cudaMemcpyAsync(h, stage_buf.p, n * rb, cudaMemcpyDeviceToHost, st));
    }
    LES_CUDA(cudaStreamSynchronize(st));
  }
  // FP64 plane means of the uploaded field, summed on the device in a fixed
  // order (k_plane_sums, one block per level) over the device copy of the
  // host values in their own width: phys[0] when the host reals are T, the
  // staging buffer h2d copied them to otherwise.
  void uploaded_plane_means(int rb, std::vector<double>& out) {
    LES_CUDA(cudaMemsetAsync(acc.p, 0, (size_t)NZ * 16 * sizeof(double), st));
    if (rb == (int)sizeof(T))
      launch(k_plane_sums<T>, dim3(1, NZ), dim3(1024), 0, st, (const T*)phys[0].p, (const T*)nullptr,
             (const T*)nullptr, (const T*)nullptr, ps, acc.p);
    else if (rb == 8)
      launch(k_plane_sums<double>, dim3(1, NZ), dim3(1024), 0, st, (const double*)stage_buf.p,
             (const double*)nullptr, (const double*)nullptr, (const double*)nullptr, ps, acc.p);
    else
      launch(k_plane_sums<float>, dim3(1, NZ), dim3(1024), 0, st, (const float*)stage_buf.p, (const float*)nullptr,
             (const float*)nullptr, (const float*)nullptr, ps, acc.p);
    std::vector<double> s((size_t)NZ * 8);
    LES_CUDA(cudaMemcpyAsync(s.data(), acc.p, s.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    LES_CUDA(cudaStreamSynchronize(st));
    out.resize(NZ);
    for (int z = 0; z < NZ; z++) out[z] = s[(size_t)z * 8] / (double)ps;
  }
  void upload_spectral(const void* h, int rb, cx<T>* dst, double* shadow, bool zero_top) {
    h2d(h, phys[0].p, ps * NZ, rb);
    std::vector<double> m;
    if (shadow) uploaded_plane_means(rb, m);  // before to_spectral: the staging buffer is still the host data
    to_spectral(phys[0].p, dst, NZ);
    if (shadow) {
      LES_CUDA(cudaMemcpyAsync(shadow, m.data(), NZ * sizeof(double), cudaMemcpyHostToDevice, st));
      launch(k_set_mean<T>, dim3(cdiv(NZ, 128)), dim3(128), 0, st, dst, (const double*)shadow, nm, NZ);
      LES_CUDA(cudaStreamSynchronize(st));
    }
    if (zero_top) LES_CUDA(cudaMemsetAsync(dst + nm * (NZ - 1), 0, nm * sizeof(cx<T>), st));
  }
  void upload(const void* u, const void* v, const void* w, const void* ee, const void* p, int rb) override {
    if (u) upload_spectral(u, rb, uh.p, mu.p, false);
    if (v) upload_spectral(v, rb, vh.p, mv.p, false);
    if (w) upload_spectral(w, rb, wh.p, nullptr, true);
    if (ee) {
      h2d(ee, phys[1].p, ps * NZ, rb);
      to_spectral(phys[1].p, run.p, NZ);  // run is scratch between stages
      to_physical(run.p, e.p + ps, NZ);
      LES_CUDA(cudaMemsetAsync(run.p, 0, nm * NZ * sizeof(cx<T>), st));
    }
    if (p) {
      h2d(p, phys[2].p, ps * NZ, rb);
      to_spectral(phys[2].p, rvn.p, NZ);
      launch(k_convert<T, double>, dim3(cdiv(nm * NZ * 2, 256)), dim3(256), 0, st, (const T*)rvn.p, (double*)ph.p,
             nm * NZ * 2);
      LES_CUDA(cudaMemsetAsync(rvn.p, 0, nm * NZ * sizeof(cx<T>), st));
    }
    LES_CUDA(cudaStreamSynchronize(st));
    phase = 0;
  }
  void upload_tend(const void* ru, const void* rv, const void* rw, const void* ree, int rb) override {
    if (ru) upload_spectral(ru, rb, ruo.p, mru.p, false);
    if (rv) upload_spectral(rv, rb, rvo.p, mrv.p, false);
    if (rw) upload_spectral(rw, rb, rwo.p, nullptr, true);
    if (ree) {
      h2d(ree, re.p, ps * NZ, rb);
      LES_CUDA(cudaMemsetAsync(re.p + ps * (NZ - 1), 0, ps * sizeof(T), st));
    }
    LES_CUDA(cudaStreamSynchronize(st));
  }
  void download_spectral(const cx<T>* src, void* h, int rb) {
    to_physical(src, phys[3].p, NZ);
    d2h(phys[3].p, h, ps * NZ, rb);
  }
  void download(void* u, void* v, void* w, void* ee, void* p, int rb) override {
    if (u) download_spectral(uh.p, u, rb);
    if (v) download_spectral(vh.p, v, rb);
    if (w) download_spectral(wh.p, w, rb);
    if (ee) d2h(e.p + ps, ee, ps * NZ, rb);
    if (p) download_pressure(p, rb);
    LES_CUDA(cudaStreamSynchronize(st));
  }
  // the pressure is FP64 in both forms
  DevBuf<double> pscr;
  void download_pressure(void* h, int rb) {
    if (!pscr.p) pscr.alloc(2 * ps * NZ);
    cx<double>* mixp = (cx<double>*)pscr.p;
    double* physp = pscr.p + ps * NZ;
    const cx<double>* tw64 = (const cx<double>*)twiddles(dev, true);
    with_small(NY, [&](auto cn) {
      constexpr int N = decltype(cn)::value;
      using C = ColCfg<N, double>;
      launch(k_col_small<double, N, true>, dim3(cdiv(KX, C::TC), NZ), dim3(C::THREADS), C::buf(), st,
             (const cx<double>*)ph.p, mixp, KX, 1.0, tw64);
    });
    with_small(NX, [&](auto cn) {
      constexpr int N = decltype(cn)::value;
      using C = RowCfg<N>;
      launch(k_row_c2r<double, N>, dim3(cdiv((size_t)NZ * NY / 2 + 1, C::NT)), dim3(C::THREADS),
             C::template smem<double>(), st, (const cx<double>*)mixp, physp, NZ * NY, KX, tw64);
    });
    if (rb == 8) {
      LES_CUDA(cudaMemcpyAsync(h, physp, ps * NZ * sizeof(double), cudaMemcpyDeviceToHost, st));
    } else {
      launch(k_convert<double, float>, dim3(cdiv(ps * NZ, 256)), dim3(256), 0, st, (const double*)physp,
             (float*)stage_buf.p, ps * NZ);
      LES_CUDA(cudaMemcpyAsync(h, stage_buf.p, ps * NZ * sizeof(float), cudaMemcpyDeviceToHost, st));
    }
    LES_CUDA(cudaStreamSynchronize(st));
  }
  void download_tend(void* ru, void* rv, void* rw, void* ree, int rb) override {
    if (ru) download_spectral(ruo.p, ru, rb);
    if (rv) download_spectral(rvo.p, rv, rb);
    if (rw) download_spectral(rwo.p, rw, rb);
    if (ree) d2h(re.p, ree, ps * NZ, rb);
  }

  // ---- the stage ----
  void comp1_kernels(const StageArgs& a) {
    const T dtab2 = (T)a.dtab2;
    // the learned closure reads the stage's start state (u, v, w and, for
    // its fallback test, e before k_e_prep's zeta update)
    if (learned_on()) learned_pre(a);
    with_small(NX, [&](auto cn) {
      constexpr int N = decltype(cn)::value;
      using C = RowCfg<N>;
      launch(k_e_prep<T, N>, dim3(cdiv(NY / 2, C::NT), NZ - 1), dim3(C::THREADS), C::template smem<T>(), st, e.p,
             (const T*)re.p, Xe.p, NY, NZ, dtab2, a.zeta, tw);
    });
    with_small(NY, [&](auto cn) {
      constexpr int N = decltype(cn)::value;
      using C = ColCfg<N, T>;
      launch(k_col_small<T, N, false>, dim3(cdiv(KX, C::TC), NZ - 1), dim3(C::THREADS), C::buf(), st,
             (const cx<T>*)Xe.p, Xe.p, KX, (T)(1.0 / ((double)NX * NY)), tw);
      using CM = ColCfg<3 * N / 2, T>;
      Ptr8 src{}, dst{};
      src.p[0] = uh.p; src.p[1] = vh.p; src.p[2] = wh.p; src.p[3] = Xe.p;
      for (int i = 0; i < 8; i++) dst.p[i] = mixed[i].p;
      launch(k_y_inverse<T, N>, dim3(2 * cdiv(KX, CM::TC), NZ, 4), dim3(CM::THREADS), CM::buf(), st, src, dst,
             KX, NZ, (T)ky0, tw, yinv_maps, yinv_pdist);
    });
    if (fused) {
      fused_middle(a);
    } else {
      unfused_middle(a);
    }
    with_small(NY, [&](auto cn) {
      constexpr int N = decltype(cn)::value;
      using C = ColCfg<3 * N / 2, T>;
      Ptr8 X{};
      for (int i = 0; i < 8; i++) X.p[i] = fused ? xout[i].p : mixed[i].p;  // Xu1..Xe2
      Ptr8 rn{};
      rn.p[0] = run.p; rn.p[1] = rvn.p; rn.p[2] = rwn.p; rn.p[3] = rem.p;
      // clusters of two CTAs (X1, X2) per column group
      size_t smem = C::buf() + (size_t)(3 * N / 2) * sizeof(cx<T>);
      launch(k_y_forward<T, N>, dim3(2 * cdiv(KX, C::TC), NZ, 4), dim3(C::THREADS), smem, st, X, rn, KX, NZ, (T)ky0,
             (T)(1.0 / ((double)MX * MY)), tw, yfwd_maps, yfwd_pdist);
    });
    if (learned_on()) learned_post(a);
  }

  // ---- learned closure ----
  bool learned_on() const { return mlp != nullptr && cfg.imodel == LES_SGS_LEARNED; }
  void learned_alloc() {
    if (lgy.p) return;
    lgy.alloc(6 * nm * NZ);
    ltau.alloc(8 * ps * NZ);
    lfeat.alloc(2 * ps * NZ);
    lpart.alloc((size_t)3 * nsm * kInferCtasPerSm);  // per-CTA triples: raw, applied, reference
    lnut.alloc((size_t)NZ * kNuChunks * 2 + NZ + 1);  // partial sums, then the face values
    lstat.alloc(4);
    lcount.alloc(2);
    lflag.alloc(1);
  }
  void set_mlp(const MlpDev* p, double rt) override {
    if (p && cfg.imodel != LES_SGS_LEARNED) throw std::invalid_argument("the handle's imodel is not LES_SGS_LEARNED");
    if (p) {
      learned_alloc();
      LES_CUDA(cudaMemsetAsync(lcount.p, 0, 2 * sizeof(unsigned long long), st));
    }
    mlp = p;
    re_tau = rt;
    for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);  // captured with the previous closure
    graphs.clear();
    graph_kernels.clear();
  }
  void set_learned_guard(double ratio) override {
    lguard = ratio;
    for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);  // captured with the previous factor
    graphs.clear();
  }
  double learned_reference() override {
    double v[3] = {0.0, 0.0, 0.0};
    if (learned_on()) {
      LES_CUDA(cudaMemcpyAsync(v, lstat.p, sizeof(v), cudaMemcpyDeviceToHost, st));
      LES_CUDA(cudaStreamSynchronize(st));
    }
    return v[2];
  }
  void learned_counts(long long* stages, long long* used) override {
    unsigned long long v[2] = {0ull, 0ull};
    if (learned_on()) {
      LES_CUDA(cudaMemcpyAsync(v, lcount.p, sizeof(v), cudaMemcpyDeviceToHost, st));
      LES_CUDA(cudaStreamSynchronize(st));
    }
    if (stages) *stages = (long long)v[0];
    if (used) *used = (long long)v[1];
  }
  void learned_status(int* used, double* dissipation) override {
    double v[2] = {0.0, 0.0};
    if (learned_on()) {
      LES_CUDA(cudaMemcpyAsync(v, lstat.p, sizeof(v), cudaMemcpyDeviceToHost, st));
      LES_CUDA(cudaStreamSynchronize(st));
    }
    if (used) *used = (int)v[1];
    if (dissipation) *dissipation = v[0];
  }
  // y-inverse rows of the velocity spectra, then gradients and features
  // at the cell centres (bf16 normalised by the attached network, or raw f32)
  void learned_features_into(void* feat, bool raw) {
    with_small(NY, [&](auto cn) {
      constexpr int NN = decltype(cn)::value;
      using C = LgyCfg<NN, T>;
      launch(k_lgrad_y<T, NN>, dim3(2 * cdiv(KX, C::H), NZ, 3), dim3(C::THREADS), C::smem(), st, (const cx<T>*)uh.p,
             (const cx<T>*)vh.p, (const cx<T>*)wh.p, lgy.p, KX, NZ, (T)ky0, tw);
    });
    const T inv_h = (T)(2.0 / cfg.zl);
    with_small(NX, [&](auto cn) {
      constexpr int NN = decltype(cn)::value;
      using L = LgxCfg<NN>;
      const unsigned grid = cdiv((size_t)NZ * NY, L::RB);
      if (raw)
        launch(k_lgrad_x<T, NN, true>, dim3(grid), dim3(L::THREADS), L::template smem<T>(), st, (const cx<T>*)lgy.p,
               feat, mlp, NY, NZ, (T)kx0, (T)dzm, (T)dsl, (T)dz, (T)cfg.zl, inv_h, tw);
      else
        launch(k_lgrad_x<T, NN, false>, dim3(grid), dim3(L::THREADS), L::template smem<T>(), st, (const cx<T>*)lgy.p,
               feat, mlp, NY, NZ, (T)kx0, (T)dzm, (T)dsl, (T)dz, (T)cfg.zl, inv_h, tw);
    });
  }
  // raw (unnormalised) features of the current state, f32 [N][16]
  // ---- regridding (redim.f90 on the device, then the restart's deal) ----
  void regrid_from(EngineBase& other) override {
    auto* sp = dynamic_cast<Engine<T>*>(&other);
    if (!sp) throw std::invalid_argument("regrid: both handles must use the same precision");
    if (sp == this) throw std::invalid_argument("regrid: source and destination are the same handle");
    Engine<T>& s = *sp;
    if (s.dev != dev) throw std::invalid_argument("regrid: both handles must be on the same device");
    if (s.cfg.xl != cfg.xl || s.cfg.yl != cfg.yl || s.cfg.zl != cfg.zl)
      throw std::invalid_argument("regrid: both grids must cover the same domain (xl, yl, zl)");
    TmpDev tmp;
    const std::vector<RegridLevel> h = regrid_table(s.NZ, NZ, cfg.zl);
    RegridLevel* tab = tmp.get<RegridLevel>(NZ);
    LES_CUDA(cudaMemcpyAsync(tab, h.data(), NZ * sizeof(RegridLevel), cudaMemcpyHostToDevice, st));
    LES_CUDA(cudaStreamSynchronize(s.st));  // the source state is complete
    const dim3 gs(cdiv(nm, 256), NZ);
    auto spec = [&](const cx<T>* a, cx<T>* b, int mode) {
      launch(k_regrid_spec<cx<T>, T>, gs, dim3(256), 0, st, a, b, (const RegridLevel*)tab, mode, s.KX, s.NY, KX, NY);
    };
    spec(s.uh.p, uh.p, kRegridCentre);
    spec(s.vh.p, vh.p, kRegridCentre);
    spec(s.wh.p, wh.p, kRegridFace);
    launch(k_regrid_spec<cx<double>, double>, gs, dim3(256), 0, st, (const cx<double>*)s.ph.p, ph.p,
           (const RegridLevel*)tab, (int)kRegridCentre, s.KX, s.NY, KX, NY);
    LES_CUDA(cudaMemsetAsync(wh.p + nm * (NZ - 1), 0, nm * sizeof(cx<T>), st));  // w(nnz) = 0
    for (auto pr : {std::make_pair(s.mu.p, mu.p), std::make_pair(s.mv.p, mv.p)})
      launch(k_regrid_mean, dim3(cdiv(NZ, 128)), dim3(128), 0, st, (const double*)pr.first, pr.second,
             (const RegridLevel*)tab, NZ);
    launch(k_set_mean<T>, dim3(cdiv(NZ, 128)), dim3(128), 0, st, uh.p, (const double*)mu.p, nm, NZ);
    launch(k_set_mean<T>, dim3(cdiv(NZ, 128)), dim3(128), 0, st, vh.p, (const double*)mv.p, nm, NZ);
    // e: chunks of at most min(NZ_old, NZ_new) levels (the old grid's
    // transform scratch holds NZ_old planes)
    const int chunk = std::min(s.NZ, NZ);
    T* ez = tmp.get<T>((size_t)chunk * s.ps);
    cx<T>* es = tmp.get<cx<T>>((size_t)chunk * s.nm);
    cx<T>* ed = tmp.get<cx<T>>((size_t)chunk * nm);
    double* emax = tmp.get<double>(NZ);
    for (int n0 = 0; n0 < NZ; n0 += chunk) {
      const int cnt = std::min(chunk, NZ - n0);
      launch(k_regrid_ez<T>, dim3(cdiv(s.ps, 256), cnt), dim3(256), 0, st, (const T*)(s.e.p + s.ps), ez,
             (const RegridLevel*)tab, n0, s.ps);
      launch(k_plane_max<T>, dim3(cnt), dim3(256), 0, st, (const T*)ez, s.ps, emax + n0);
      LES_CUDA(cudaStreamSynchronize(st));
      s.to_spectral(ez, es, cnt);  // on the source's stream, old grid
      LES_CUDA(cudaStreamSynchronize(s.st));
      launch(k_regrid_spec<cx<T>, T>, dim3(cdiv(nm, 256), cnt), dim3(256), 0, st, (const cx<T>*)es, ed,
             (const RegridLevel*)nullptr, (int)kRegridCopy, s.KX, s.NY, KX, NY);
      T* en = e.p + ps * (size_t)(n0 + 1);
      to_physical(ed, en, cnt);
      launch(k_regrid_eclamp<T>, dim3(cdiv(ps, 256), cnt), dim3(256), 0, st, en, (const double*)(emax + n0), ps);
    }
    // the restart's deal of e
    to_spectral(e.p + ps, run.p, NZ);
    to_physical(run.p, e.p + ps, NZ);
    LES_CUDA(cudaMemsetAsync(run.p, 0, nm * NZ * sizeof(cx<T>), st));
    LES_CUDA(cudaStreamSynchronize(st));
    phase = 0;
  }

  void learned_features(double rt, float* feat) override {
    if (phase != 0) throw std::logic_error("learned_features inside a split comp1..comp2 sequence");
    learned_alloc();
    (void)rt;  // the features do not depend on Re_tau
    learned_features_into(feat, true);
  }
  // explicit filter of the current state onto the grid (NX/fxy, NY/fxy, NZ/fz)
  void learn_filter(int fxy, int fz, int with_model, double* out) override {
    if (phase != 0) throw std::logic_error("learn_filter inside a split comp1..comp2 sequence");
    if (fxy < 1 || fz < 1 || (fz > 1 && fz % 2) || NX % fxy || NY % fxy || NZ % fz)
      throw std::invalid_argument("learn_filter: unsupported filter factors for this grid");
    const int NXc = NX / fxy, NYc = NY / fxy, NZc = NZ / fz, KXc = NXc / 2;
    if (!supported_small(NXc) || !supported_small(NYc) || NZc < 4)
      throw std::invalid_argument("learn_filter: unsupported coarse grid");
    const size_t npl = (size_t)10 * NZc, psc = (size_t)NXc * NYc, nmc = (size_t)KXc * NYc;
    if (fscr.n < npl * ps) { fscr.release(); fscr.alloc(npl * ps); }
    if (fsh.n < npl * nm) { fsh.release(); fsh.alloc(npl * nm); }
    if (fch.n < npl * nmc) { fch.release(); fch.alloc(npl * nmc); }
    if (fcp.n < npl * psc) { fcp.release(); fcp.alloc(npl * psc); }
    if (with_model) {
      learned_alloc();
      if (fraw.n < 16 * ps * NZ) { fraw.release(); fraw.alloc(16 * ps * NZ); }
      learned_features_into(fraw.p, true);
    }
    to_physical(uh.p, phys[0].p, NZ);
    to_physical(vh.p, phys[1].p, NZ);
    to_physical(wh.p, phys[2].p, NZ);
    launch(k_filt_z<T>, dim3(cdiv(ps, 256), NZc), dim3(256), 0, st, (const T*)phys[0].p, (const T*)phys[1].p,
           (const T*)phys[2].p, with_model ? (const float*)fraw.p : (const float*)nullptr, (const T*)e.p, (T)dsl,
           (T)cfg.emin, fscr.p, (long long)ps, NZ, NZc, fz);
    with_small(NX, [&](auto cn) {
      constexpr int NN = decltype(cn)::value;
      using C = RowCfg<NN>;
      launch(k_row_r2c<T, NN>, dim3(cdiv((npl * NY + 1) / 2, C::NT)), dim3(C::THREADS), C::template smem<T>(), st,
             (const T*)fscr.p, fsh.p, (int)(npl * NY), KX, tw);
    });
    with_small(NY, [&](auto cn) {
      constexpr int NN = decltype(cn)::value;
      using C = ColCfg<NN, T>;
      launch(k_col_small<T, NN, false>, dim3(cdiv(KX, C::TC), (unsigned)npl), dim3(C::THREADS), C::buf(), st,
             (const cx<T>*)fsh.p, fsh.p, KX, (T)(1.0 / ((double)NX * NY)), tw);
    });
    launch(k_filt_trunc<T>, dim3(cdiv(nmc, 256), (unsigned)npl), dim3(256), 0, st, (const cx<T>*)fsh.p, fch.p, NY,
           KX, NYc, KXc, kx0, ky0, cfg.xl / NXc, cfg.yl / NYc);
    with_small(NYc, [&](auto cn) {
      constexpr int NN = decltype(cn)::value;
      using C = ColCfg<NN, T>;
      launch(k_col_small<T, NN, true>, dim3(cdiv(KXc, C::TC), (unsigned)npl), dim3(C::THREADS), C::buf(), st,
             (const cx<T>*)fch.p, fch.p, KXc, (T)1, tw);
    });
    with_small(NXc, [&](auto cn) {
      constexpr int NN = decltype(cn)::value;
      using C = RowCfg<NN>;
      launch(k_row_c2r<T, NN>, dim3(cdiv((npl * NYc + 1) / 2, C::NT)), dim3(C::THREADS), C::template smem<T>(), st,
             (const cx<T>*)fch.p, fcp.p, (int)(npl * NYc), KXc, tw);
    });
    launch(k_filt_tau<T>, dim3(cdiv(psc * NZc, 256)), dim3(256), 0, st, (const T*)fcp.p, out, (long long)(psc * NZc));
  }
  // gradients -> features -> network -> tau and the fallback flag
  void learned_pre(const StageArgs& a) {
    const size_t N = ps * NZ;
    learned_features_into(lfeat.p, false);
    const long long ntiles = ((long long)N + 127) / 128;
    const int grid = (int)std::min<long long>((ntiles + kInferGroups - 1) / kInferGroups, (long long)nsm * kInferCtasPerSm);
    MlpOutTau<T> out{ltau.p, (long long)N};
    launch(k_mlp_infer<MlpOutTau<T>>, dim3(grid), dim3(128 * kInferGroups), kInferSmem, st, mlp,
           (const uint4*)lfeat.p, (long long)N, out, lpart.p, err.p);
    launch(k_learned_flag, dim3(1), dim3(32), 0, st, (const double*)lpart.p, grid, 1.0 / ((double)N * dsl), lguard,
           lflag.p, lstat.p, lcount.p);
  }
  // tau^ and its divergence into the new tendencies (th reuses lgy)
  void learned_post(const StageArgs& a) {
    with_small(NX, [&](auto cn) {
      constexpr int NN = decltype(cn)::value;
      using C = RowCfg<NN>;
      const size_t nrows = 6 * (size_t)NZ * NY;
      launch(k_row_r2c<T, NN>, dim3(cdiv((nrows + 1) / 2, C::NT)), dim3(C::THREADS), C::template smem<T>(), st,
             (const T*)ltau.p, lgy.p, (int)nrows, KX, tw);
    });
    with_small(NY, [&](auto cn) {
      constexpr int NN = decltype(cn)::value;
      using C = ColCfg<NN, T>;
      launch(k_col_small<T, NN, false>, dim3(cdiv(KX, C::TC), 6 * NZ), dim3(C::THREADS), C::buf(), st,
             (const cx<T>*)lgy.p, lgy.p, KX, (T)(1.0 / ((double)NX * NY)), tw);
    });
    launch(k_learned_nu<T>, dim3(NZ, kNuChunks), dim3(256), 0, st, (const T*)ltau.p, lnut.p, ps, (long long)(ps * NZ));
    double* nuf = lnut.p + (size_t)NZ * kNuChunks * 2;
    launch(k_learned_nu_face, dim3(1), dim3(256), 0, st, (const double*)lnut.p, nuf, NZ, dsl, a.xkmax);
    launch(k_ldiv<T>, dim3(cdiv(nm, 128), NZ), dim3(128), 0, st, (const cx<T>*)lgy.p, run.p, rvn.p, rwn.p,
           (const cx<T>*)uh.p, (const cx<T>*)vh.p, (const double*)nuf, (const int*)lflag.p, a);
  }
  // Wall-model plane sums from the physical U, V rows of levels 1 and nnz.
  void wall_params_from(const T* U, const T* V, size_t upper_off, const StageArgs& a) {
    (void)upper_off;
    launch(k_wall_sums<T>, dim3(kWallBlocks, 2), dim3(256), 0, st, U, V, 2, pb, wacc.p);
    launch(k_wall_final, dim3(1), dim3(32), 0, st, (const double*)wacc.p, (int)kWallBlocks, (const double*)mru.p,
           (const double*)mrv.p, a, (double)pb, 0.4, zody, cfg.ufree, wp.p, err.p);
  }
  void fused_middle(const StageArgs& a) {
    // clip flags and corrections of max(expand(e), emin)
    LES_CUDA(cudaMemsetAsync(clipflag.p, 0, NZ * sizeof(int), st));
    with_small(NX, [&](auto cn) {
      constexpr int N = decltype(cn)::value;
      using C = RowCfg<3 * N / 2>;
      launch(k_clip_flag<T, N>, dim3(cdiv(MY / 2, C::NT), NZ - 1), dim3(C::THREADS), C::template smem<T>(), st,
             (const cx<T>*)mixed[6].p, clipflag.p, MY, (T)cfg.emin, tw);
      launch(k_clip_phys<T, N>, dim3(cdiv(MY / 2, C::NT), NZ - 1), dim3(C::THREADS), C::template smem<T>(), st,
             (const cx<T>*)mixed[6].p, ephys.p, (const int*)clipflag.p, MY, tw);
    });
    with_small(NY, [&](auto cn) {
      constexpr int N = decltype(cn)::value;
      using C = ColCfg<3 * N / 2, T>;
      launch(k_clipd_y<T, N>, dim3(cdiv(MX / 2, C::TC), NZ - 1), dim3(C::THREADS), C::buf(), st,
             (const T*)ephys.p, dEY.p, (const int*)clipflag.p, MX, (T)cfg.emin, (T)ky0, tw);
    });
    with_small(NX, [&](auto cn) {
      constexpr int N = decltype(cn)::value;
      using C = RowCfg<3 * N / 2>;
      launch(k_clipd_x<T, N>, dim3(cdiv(MY / 2, C::NT), NZ - 1), dim3(C::THREADS), C::template smem<T>(), st,
             (const T*)ephys.p, dEX.p, (const int*)clipflag.p, MY, (T)cfg.emin, (T)kx0, tw);
      // physical U, V at levels 1 and nnz for the wall model: wallpl = [U1, Unz, V1, Vnz]
      using CR = RowCfg<3 * N / 2>;
      const int lv[2] = {1, NZ};
      for (int side = 0; side < 2; side++)
        for (int fld = 0; fld < 2; fld++)
          launch(k_row_c2r<T, 3 * N / 2>, dim3(cdiv(MY / 2 + 1, CR::NT)), dim3(CR::THREADS), CR::template smem<T>(),
                 st, (const cx<T>*)(mixed[fld == 0 ? 0 : 2].p + (size_t)(lv[side] - 1) * nmix),
                 wallpl.p + (size_t)(2 * fld + side) * pb, MY, KX, tw);
    });
    wall_params_from(wallpl.p, wallpl.p + 2 * pb, pb, a);
    // the fused row kernel
    FusedArgs fa{};
    for (int i = 0; i < 8; i++) { fa.in.p[i] = mixed[i].p; fa.out.p[i] = xout[i].p; }
    fa.dEX = dEX.p; fa.dEY = dEY.p; fa.clipflag = clipflag.p; fa.wp = wp.p;
    fa.divpart = divpart.p; fa.sgspart = sgspart.p;
    fa.lflag = learned_on() ? lflag.p : nullptr;
    with_small(NX, [&](auto cn) {
      constexpr int N = decltype(cn)::value;
      const int threads = FusedCfg<N>::template threads<T>();
      const size_t smem = FusedCfg<N>::template smem<T>();
      if (fused_chunks == 0) fused_chunks = fused_chunk_count((const void*)k_row_fused<T, N>, threads, smem);
      fa.zchunk = (int)cdiv(NZ, fused_chunks);
      launch(k_row_fused<T, N>, dim3(MY, (unsigned)cdiv(NZ, fa.zchunk)), dim3(threads), smem, st, fa, a, tw);
    });
  }
  // z chunks per padded row of the fused kernel: a CTA walks its chunk with
  // a sliding window, so chunks only add prologues (about half a level of
  // work each), while the last wave of CTAs leaves SMs idle.  Minimise
  // waves x (levels per chunk + 1/2) over 1..NZ/8 chunks, the waves counted
  // with the kernel's resident CTAs per SM.
  int fused_chunks = 0;
  int fused_chunk_count(const void* kernel, int threads, size_t smem) {
    if (smem > 48 * 1024) set_smem_limit(kernel, smem);
    int per_sm = 0;
    LES_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem));
    const double resident = (double)std::max(1, per_sm) * nsm;
    int best = 1;
    double best_cost = 0.0;
    for (int c = 1; c <= std::max(1, NZ / 8); c++) {
      const int zc = (int)cdiv(NZ, c), n = (int)cdiv(NZ, zc);
      const double cost = std::ceil((double)MY * n / resident) * (zc + 0.5);
      if (c == 1 || cost < best_cost) { best = c; best_cost = cost; }
    }
    return best;
  }
  void unfused_middle(const StageArgs& a) {
    Ptr8 msrc{};
    for (int i = 0; i < 8; i++) msrc.p[i] = mixed[i].p;
    Ptr12 pd{};
    for (int i = 0; i < 12; i++) pd.p[i] = pad[i].p;
    with_small(NX, [&](auto cn) {
      constexpr int N = decltype(cn)::value;
      using C = RowCfg<3 * N / 2>;
      launch(k_x_inverse<T, N>, dim3(cdiv(MY, C::NT), NZ, 6), dim3(C::THREADS), C::template smem<T>(), st, msrc, pd,
             MY, NZ, (T)kx0, tw);
    });
    // derivatives of the clipped TKE: E = pad[9], EX = pad[10], EY = pad[11]
    with_small(NY, [&](auto cn) {
      constexpr int N = decltype(cn)::value;
      using C = ColCfg<3 * N / 2, T>;
      launch(k_clip_y<T, N>, dim3(cdiv(MX / 2, C::TC), NZ - 1), dim3(C::THREADS), C::buf(), st,
             (const T*)pad[9].p, pad[11].p, MX, (T)cfg.emin, (T)ky0, tw);
    });
    with_small(NX, [&](auto cn) {
      constexpr int N = decltype(cn)::value;
      using C = RowCfg<3 * N / 2>;
      launch(k_clip_x<T, N>, dim3(cdiv(MY / 2, C::NT), NZ - 1), dim3(C::THREADS), C::template smem<T>(), st,
             pad[9].p, pad[10].p, MY, (T)cfg.emin, (T)kx0, tw);
    });
    // wall model scalars
    {
      launch(k_wall_sums<T>, dim3(kWallBlocks, 2), dim3(256), 0, st, (const T*)pad[0].p, (const T*)pad[3].p, NZ, pb,
             wacc.p);
      launch(k_wall_final, dim3(1), dim3(32), 0, st, (const double*)wacc.p, (int)kWallBlocks, (const double*)mru.p,
             (const double*)mrv.p, a, (double)pb, 0.4, zody, cfg.ufree, wp.p, err.p);
    }
    Ptr11 fl{};
    for (int i = 0; i < 11; i++) fl.p[i] = flux[i].p;
    launch(k_flux<T>, dim3(cdiv(pb, 256), NZ), dim3(256), 0, st, pd, fl, a, (const WallParams*)wp.p, divpart.p,
           sgspart.p);
    Ptr8 X{};
    for (int i = 0; i < 8; i++) X.p[i] = mixed[i].p;  // reuse the mixed buffers
    with_small(NX, [&](auto cn) {
      constexpr int N = decltype(cn)::value;
      using C = RowCfg<3 * N / 2>;
      launch(k_x_forward<T, N>, dim3(cdiv(MY, C::NT), NZ, 6), dim3(C::THREADS), C::template smem<T>(), st, fl, X, MY,
             NZ, (T)kx0, tw);
    });
  }
  // comp2's e update: re = c2r(rem) with plain stores, then the clipped
  // elementwise update (a read-modify-write inside the transform's store
  // phase would serialise on the load latency)
  void e_update(double dtab1) {
    with_small(NX, [&](auto cn) {
      constexpr int N = decltype(cn)::value;
      using C = RowCfg<N>;
      launch(k_row_c2r<T, N>, dim3(cdiv((size_t)(NZ - 1) * NY / 2 + 1, C::NT)), dim3(C::THREADS),
             C::template smem<T>(), st, (const cx<T>*)rem.p, re.p, (NZ - 1) * NY, KX, tw);
    });
    launch(k_e_update_phys<T>, dim3(cdiv(ps * (NZ - 1), 256)), dim3(256), 0, st, e.p + ps, (const T*)re.p,
           ps * (NZ - 1), (T)dtab1, (T)cfg.emin);
  }
  void press_kernel(const StageArgs& a, bool rhs_in_ph) {
    if (rhs_in_ph)
      launch(k_press<T, true>, dim3(cdiv(nm, 128)), dim3(128), 0, st, (const cx<T>*)uh.p, (const cx<T>*)vh.p,
             (const cx<T>*)wh.p, (const cx<T>*)ruo.p, (const cx<T>*)rvo.p, (const cx<T>*)rwo.p, (const cx<T>*)run.p,
             (const cx<T>*)rvn.p, (const cx<T>*)rwn.p, ph.p, dscr.p, rscr.p, a);
    else
      launch(k_press<T, false>, dim3(cdiv(nm, 128)), dim3(128), 0, st, (const cx<T>*)uh.p, (const cx<T>*)vh.p,
             (const cx<T>*)wh.p, (const cx<T>*)ruo.p, (const cx<T>*)rvo.p, (const cx<T>*)rwo.p, (const cx<T>*)run.p,
             (const cx<T>*)rvn.p, (const cx<T>*)rwn.p, ph.p, dscr.p, rscr.p, a);
  }
  void update_kernel(const StageArgs& a, const cx<T>* rnu, const cx<T>* rnv, const cx<T>* rnw) {
    launch(k_update<T>, dim3(cdiv(nm, 128), NZ), dim3(128), 0, st, uh.p, vh.p, wh.p, (const cx<T>*)ruo.p,
           (const cx<T>*)rvo.p, (const cx<T>*)rwo.p, rnu, rnv, rnw, ruo.p, rvo.p, rwo.p, (const cx<double>*)ph.p,
           mu.p, mv.p, mru.p, mrv.p, a, err.p);
  }

  double last_dtab1 = 0, last_xkmax = 0;
  void comp1(bool mnout, int istage, double dtab1, double dtab2, double xkmax) override {
    StageArgs a = args(dtab1, dtab2, xkmax, istage != 1, mnout && istage == 1);
    comp1_kernels(a);
    if (istage != 1)
      launch(k_zeta<T>, dim3(cdiv(nm, 128), NZ), dim3(128), 0, st, uh.p, vh.p, wh.p, (const cx<T>*)ruo.p,
             (const cx<T>*)rvo.p, (const cx<T>*)rwo.p, mu.p, mv.p, (const double*)mru.p, (const double*)mrv.p, a);
    // ru, rv, rw now hold the new tendencies (comp1.f90:164-172)
    std::swap(ruo.p, run.p); std::swap(rvo.p, rvn.p); std::swap(rwo.p, rwn.p);
    // re = compress(rebuf) in physical space (comp1.f90:168)
    with_small(NX, [&](auto cn) {
      constexpr int N = decltype(cn)::value;
      using C = RowCfg<N>;
      launch(k_row_c2r<T, N>, dim3(cdiv((size_t)(NZ - 1) * NY / 2 + 1, C::NT)), dim3(C::THREADS),
             C::template smem<T>(), st, (const cx<T>*)rem.p, re.p, (NZ - 1) * NY, KX, tw);
    });
    last_dtab1 = dtab1;
    phase = 1;
  }
  void comprhs(double dtabm) override {
    if (phase != 1) throw std::logic_error("comprhs called before comp1");
    StageArgs a = args(1.0 / dtabm, 0.0, 0.0, 0, 0);
    launch(k_rhs<T>, dim3(cdiv(nm, 128), NZ), dim3(128), 0, st, (const cx<T>*)uh.p, (const cx<T>*)vh.p,
           (const cx<T>*)wh.p, (const cx<T>*)ruo.p, (const cx<T>*)rvo.p, (const cx<T>*)rwo.p, ph.p, a);
    phase = 2;
  }
  void press() override {
    if (phase != 2) throw std::logic_error("press called before comprhs");
    StageArgs a = args(last_dtab1, 0.0, 0.0, 0, 0);
    press_kernel(a, true);
    phase = 3;
  }
  void comp2(double dtab1) override {
    if (phase != 3) throw std::logic_error("comp2 called before press");
    StageArgs a = args(dtab1, 0.0, 0.0, 0, 0);
    // zeta already applied by comp1; the new tendencies are in ruo, rvo, rwo
    update_kernel(a, ruo.p, rvo.p, rwo.p);
    // e = max(e + dtab1*re, emin) with re in physical space
    launch(k_e_update_phys<T>, dim3(cdiv(ps * (NZ - 1), 256)), dim3(256), 0, st, e.p + ps, (const T*)re.p,
           ps * (NZ - 1), (T)dtab1, (T)cfg.emin);
    phase = 0;
  }
  void stage_kernels(bool mnout, int istage, double dtab1, double dtab2, double xkmax) {
    StageArgs a = args(dtab1, dtab2, xkmax, istage != 1, mnout && istage == 1);
    comp1_kernels(a);
    e_update(dtab1);
    press_kernel(a, false);
    update_kernel(a, run.p, rvn.p, rwn.p);
  }
  void stage(bool mnout, int istage, double dtab1, double dtab2, double xkmax) override {
    if (phase != 0) throw std::logic_error("stage called inside a split comp1..comp2 sequence");
    stage_kernels(mnout, istage, dtab1, dtab2, xkmax);
  }
  void stage_eager(bool mnout, int istage, double dt) override {
    const double gama[3] = {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};
    const double zetas[3] = {0.0, 17.0 / 60.0, 5.0 / 12.0};
    stage_kernels(mnout, istage, dt * gama[istage - 1], dt * zetas[istage - 1], dz * dz / dt / 5.0);
  }
  void step_kernels(bool mnout, double dt) {
    const double gama[3] = {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};
    const double zetas[3] = {0.0, 17.0 / 60.0, 5.0 / 12.0};
    double xkmax = dz * dz / dt / 5.0;
    for (int s = 0; s < 3; s++) stage_kernels(mnout, s + 1, dt * gama[s], dt * zetas[s], xkmax);
  }
  void step(bool mnout, double dt) override {
    if (phase != 0) throw std::logic_error("step called inside a split comp1..comp2 sequence");
    uint64_t bits;
    std::memcpy(&bits, &dt, sizeof(bits));
    auto key = std::make_pair(bits, (int)mnout);
    auto it = graphs.find(key);
    if (it == graphs.end()) {
      if (graphs.size() > 8) {
        for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
        graphs.clear();
      }
      cudaGraph_t g;
      long long* saved = g_launch_counter;
      long long nk = 0;
      g_launch_counter = &nk;
      LES_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      try {
        step_kernels(mnout, dt);
      } catch (...) {
        g_launch_counter = saved;
        cudaStreamEndCapture(st, &g);
        if (g) cudaGraphDestroy(g);
        throw;
      }
      g_launch_counter = saved;
      graph_kernels[key] = nk;
      LES_CUDA(cudaStreamEndCapture(st, &g));
      cudaGraphExec_t ge;
      LES_CUDA(cudaGraphInstantiate(&ge, g, 0));
      cudaGraphDestroy(g);
      it = graphs.emplace(key, ge).first;
    }
    LES_CUDA(cudaGraphLaunch(it->second, st));
    if (g_launch_counter) *g_launch_counter += graph_kernels[key];
  }
  std::map<std::pair<uint64_t, int>, long long> graph_kernels;

  // ---- statistics (compmn.F90:1-64) ----
  void stats(double* meanbuf, double* scalars) override {
    to_physical(uh.p, phys[0].p, NZ);
    to_physical(vh.p, phys[1].p, NZ);
    to_physical(wh.p, phys[2].p, NZ);
    LES_CUDA(cudaMemsetAsync(acc.p, 0, (size_t)NZ * 16 * sizeof(double), st));
    launch(k_plane_sums<T>, dim3(1, NZ), dim3(1024), 0, st, (const T*)phys[0].p, (const T*)phys[1].p,
           (const T*)phys[2].p, (const T*)(e.p + ps), ps, acc.p);
    launch(k_sum_parts, dim3(NZ), dim3(256), 0, st, (const double*)divpart.p, nstat_parts, 1, divacc.p, 1);
    launch(k_sum_parts, dim3(NZ), dim3(256), 0, st, (const double*)sgspart.p, nstat_parts, 6, sgsacc.p, 8);
    std::vector<double> sums((size_t)NZ * 16), mshadow(NZ), vshadow(NZ);
    LES_CUDA(cudaMemcpyAsync(sums.data(), acc.p, sums.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    LES_CUDA(cudaMemcpyAsync(mshadow.data(), mu.p, NZ * sizeof(double), cudaMemcpyDeviceToHost, st));
    LES_CUDA(cudaMemcpyAsync(vshadow.data(), mv.p, NZ * sizeof(double), cudaMemcpyDeviceToHost, st));
    LES_CUDA(cudaStreamSynchronize(st));
    std::vector<double> means((size_t)NZ * 8, 0.0);
    for (int z = 0; z < NZ; z++) {
      means[(size_t)z * 8 + 0] = mshadow[z];
      means[(size_t)z * 8 + 1] = vshadow[z];
    }
    LES_CUDA(cudaMemcpyAsync(acc.p + (size_t)NZ * 8, means.data(), means.size() * sizeof(double),
                             cudaMemcpyHostToDevice, st));
    LES_CUDA(cudaMemsetAsync(acc.p, 0, (size_t)NZ * 8 * sizeof(double), st));
    launch(k_moments<T>, dim3(1, NZ), dim3(1024), 0, st, (const T*)phys[0].p, (const T*)phys[1].p,
           (const T*)phys[2].p, ps, NZ, (const double*)(acc.p + (size_t)NZ * 8), acc.p);
    std::vector<double> mom((size_t)NZ * 8), dv(NZ), sg((size_t)NZ * 8);
    WallParams w;
    LES_CUDA(cudaMemcpyAsync(mom.data(), acc.p, mom.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    LES_CUDA(cudaMemcpyAsync(dv.data(), divacc.p, NZ * sizeof(double), cudaMemcpyDeviceToHost, st));
    LES_CUDA(cudaMemcpyAsync(sg.data(), sgsacc.p, sg.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    LES_CUDA(cudaMemcpyAsync(&w, wp.p, sizeof(w), cudaMemcpyDeviceToHost, st));
    LES_CUDA(cudaStreamSynchronize(st));
    const double P = (double)ps, Pb = (double)pb;
    if (meanbuf) {
      for (int z = 0; z < NZ; z++) {
        double* M = meanbuf + (size_t)z * 19;
        double uu = mom[(size_t)z * 8 + 0] / P, vv = mom[(size_t)z * 8 + 1] / P, ww = mom[(size_t)z * 8 + 2] / P;
        M[0] = (uu + vv + ww) * 0.5;                       // englez
        M[1] = sums[(size_t)z * 8 + 3] / P;                // engsbz
        M[2] = dv[z] / Pb;                                 // divz
        M[3] = mshadow[z];                                 // uxym
        M[4] = vshadow[z];                                 // vxym
        M[5] = sums[(size_t)z * 8 + 2] / P;                // wxym
        M[6] = uu; M[7] = vv; M[8] = ww;                   // uule, vvle, wwle
        M[9] = mom[(size_t)z * 8 + 3] / P;                 // uwle
        M[10] = mom[(size_t)z * 8 + 4] / P;                // vwle
        M[11] = mom[(size_t)z * 8 + 5] / P;                // uvle
        M[12] = 0.0;                                       // pple (never assigned by compmn)
        M[13] = sg[(size_t)z * 8 + 0] / Pb;                // uusb
        M[14] = sg[(size_t)z * 8 + 1] / Pb;                // vvsb
        M[15] = sg[(size_t)z * 8 + 2] / Pb;                // uvsb
        M[16] = sg[(size_t)z * 8 + 3] / Pb;                // wwsb
        M[17] = sg[(size_t)z * 8 + 4] / Pb;                // uwsb
        M[18] = sg[(size_t)z * 8 + 5] / Pb;                // vwsb
      }
    }
    if (scalars) {
      scalars[0] = w.w[1].utau;
      scalars[1] = w.utau_s;
      scalars[2] = w.dudt;
      scalars[3] = w.dvdt;
      scalars[4] = w.w[0].utau;
    }
  }
  // spectra (spectra2.f90:1-70) of one level: the full half spectrum of
  // the physical plane on the device, the binning on the host.
  void spectra(int field, int iz, double* zx, double* z2) override {
    const int H = NX / 2 + 1;
    const T* plane;
    if (field == 3) {
      plane = e.p + (size_t)iz * ps;
    } else {
      const cx<T>* src = field == 0 ? uh.p : field == 1 ? vh.p : wh.p;
      to_physical(src + nm * (iz - 1), phys[3].p, 1);
      plane = phys[3].p;
    }
    cx<T>* half = (cx<T>*)phys[2].p;  // (NY, H) complex fits in NZ+2 small planes
    with_small(NX, [&](auto cn) {
      constexpr int N = decltype(cn)::value;
      using C = RowCfg<N>;
      launch(k_row_r2c<T, N>, dim3(cdiv(NY / 2 + 1, C::NT)), dim3(C::THREADS), C::template smem<T>(), st, plane,
             Xe.p, NY, H, tw);
    });
    with_small(NY, [&](auto cn) {
      constexpr int N = decltype(cn)::value;
      using C = ColCfg<N, T>;
      launch(k_col_small<T, N, false, false>, dim3(cdiv(H, C::TC), 1), dim3(C::THREADS), C::buf(), st,
             (const cx<T>*)Xe.p, half, H, (T)(1.0 / ((double)NX * NY)), tw);
    });
    std::vector<cx<T>> w((size_t)NY * H);
    LES_CUDA(cudaMemcpyAsync(w.data(), half, w.size() * sizeof(cx<T>), cudaMemcpyDeviceToHost, st));
    LES_CUDA(cudaStreamSynchronize(st));
    const double pi = 4.0 * std::atan(1.0);
    auto kxw = [&](int i) { int k = i - 1; return (k > NX / 2 ? k - NX : k) * 2.0 * pi / cfg.xl; };
    auto kyw = [&](int j) { int k = j - 1; return (k > NY / 2 ? k - NY : k) * 2.0 * pi / cfg.yl; };
    std::vector<double> sx(H, 0.0), s2(H, 0.0);
    std::vector<int> mcount(H, 0);
    for (int i = 1; i <= H; i++)
      for (int j = 1; j <= NY; j++) {
        cx<T> c = w[(size_t)(j - 1) * H + (i - 1)];
        sx[i - 1] += (double)c.x * c.x + (double)c.y * c.y;
      }
    for (int i = 2; i <= H - 1; i++) sx[i - 1] *= 2.0;
    for (int j = 1; j <= NY; j++)
      for (int i = 1; i <= H; i++) {
        double xk = kxw(i), yk = kyw(j);
        double dist = std::sqrt(xk * xk + yk * yk);
        double px = pi * NX / cfg.xl, py = pi * NY / cfg.yl;
        if (i == NX / 2 + 1 && j == NY / 2 + 1) dist = std::sqrt(px * px + py * py);
        else {
          if (i == NX / 2 + 1) dist = std::sqrt(px * px + yk * yk);
          if (j == NY / 2 + 1) dist = std::sqrt(xk * xk + py * py);
        }
        int iin = (int)std::lround(dist / (2.0 * pi / cfg.xl)) + 1;
        if (iin > NX / 2 + 1 || (i == 1 && j > NY / 2 + 1)) continue;
        cx<T> c = w[(size_t)(j - 1) * H + (i - 1)];
        s2[iin - 1] += (double)c.x * c.x + (double)c.y * c.y;
        mcount[iin - 1]++;
      }
    for (int i = 1; i <= H; i++) {
      int jj = i - 1;
      double denom = (i == 1) ? 1.0
                              : 2.0 * mcount[i - 1] / (pi * (jj + 0.5) * (jj + 0.5) - pi * (jj - 0.5) * (jj - 0.5));
      s2[i - 1] = 2.0 * s2[i - 1] / denom;
      zx[i - 1] = sx[i - 1];
      z2[i - 1] = s2[i - 1];
    }
  }

  void make_ic(unsigned long long seed, double ub, double amp, double utau, double e0) override {
    size_t n = ps * NZ;
    for (int f = 0; f < 3; f++)
      launch(k_ic_fill<T>, dim3(cdiv(n, 256)), dim3(256), 0, st, phys[f].p, f, seed, NX, NY, NZ, dz, cfg.zl / 2, ub,
             amp, utau);
    to_spectral(phys[0].p, uh.p, NZ);
    to_spectral(phys[1].p, vh.p, NZ);
    to_spectral(phys[2].p, wh.p, NZ);
    // FP64 plane means of the mean profile
    LES_CUDA(cudaMemsetAsync(acc.p, 0, (size_t)NZ * 16 * sizeof(double), st));
    launch(k_plane_sums<T>, dim3(1, NZ), dim3(1024), 0, st, (const T*)phys[0].p, (const T*)phys[1].p,
           (const T*)nullptr, (const T*)nullptr, ps, acc.p);
    std::vector<double> s((size_t)NZ * 16);
    LES_CUDA(cudaMemcpyAsync(s.data(), acc.p, s.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    LES_CUDA(cudaStreamSynchronize(st));
    std::vector<double> m1(NZ), m2(NZ);
    for (int z = 0; z < NZ; z++) { m1[z] = s[(size_t)z * 8] / ps; m2[z] = s[(size_t)z * 8 + 1] / ps; }
    LES_CUDA(cudaMemcpyAsync(mu.p, m1.data(), NZ * sizeof(double), cudaMemcpyHostToDevice, st));
    LES_CUDA(cudaMemcpyAsync(mv.p, m2.data(), NZ * sizeof(double), cudaMemcpyHostToDevice, st));
    launch(k_set_mean<T>, dim3(cdiv(NZ, 128)), dim3(128), 0, st, uh.p, (const double*)mu.p, nm, NZ);
    launch(k_set_mean<T>, dim3(cdiv(NZ, 128)), dim3(128), 0, st, vh.p, (const double*)mv.p, nm, NZ);
    LES_CUDA(cudaMemsetAsync(wh.p + nm * (NZ - 1), 0, nm * sizeof(cx<T>), st));
    launch(k_fill<T>, dim3(cdiv(ps * (NZ + 2), 256)), dim3(256), 0, st, e.p, ps * (NZ + 2), (T)e0);
    for (auto* b : {&ruo, &rvo, &rwo, &run, &rvn, &rwn})
      LES_CUDA(cudaMemsetAsync(b->p, 0, b->n * sizeof(cx<T>), st));
    for (auto* b : {&mru, &mrv}) LES_CUDA(cudaMemsetAsync(b->p, 0, NZ * sizeof(double), st));
    LES_CUDA(cudaMemsetAsync(re.p, 0, re.n * sizeof(T), st));
    // one projection: comprhs + press + comp2 with dtab1 = 1, zero tendencies
    StageArgs a = args(1.0, 0.0, 0.0, 0, 0);
    press_kernel(a, false);
    update_kernel(a, run.p, rvn.p, rwn.p);
    for (auto* b : {&ruo, &rvo, &rwo}) LES_CUDA(cudaMemsetAsync(b->p, 0, b->n * sizeof(cx<T>), st));
    for (auto* b : {&mru, &mrv}) LES_CUDA(cudaMemsetAsync(b->p, 0, NZ * sizeof(double), st));
    LES_CUDA(cudaMemsetAsync(ph.p, 0, ph.n * sizeof(cx<double>), st));
    LES_CUDA(cudaStreamSynchronize(st));
    phase = 0;
  }
  double cfl_dt(double cfl) override {
    to_physical(uh.p, phys[0].p, NZ);
    to_physical(vh.p, phys[1].p, NZ);
    to_physical(wh.p, phys[2].p, NZ);
    LES_CUDA(cudaMemsetAsync(amax.p, 0, 4 * sizeof(unsigned long long), st));
    size_t n = ps * NZ;
    launch(k_absmax3<T>, dim3(std::min<unsigned>(cdiv(n, 256), 1024)), dim3(256), 0, st, (const T*)phys[0].p,
           (const T*)phys[1].p, (const T*)phys[2].p, n, amax.p);
    unsigned long long h[4];
    LES_CUDA(cudaMemcpyAsync(h, amax.p, sizeof(h), cudaMemcpyDeviceToHost, st));
    LES_CUDA(cudaStreamSynchronize(st));
    double m[3];
    for (int q = 0; q < 3; q++) std::memcpy(&m[q], &h[q], sizeof(double));
    double ucfl = m[0] * MX / cfg.xl, vcfl = m[1] * MY / cfg.yl, wcfl = m[2] / dz;
    return cfl / std::max(std::max(ucfl, vcfl), std::max(wcfl, 0.5 / dz));
  }
  int read_error() override {
    int h = 0;
    LES_CUDA(cudaMemcpyAsync(&h, err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    LES_CUDA(cudaStreamSynchronize(st));
    return h;
  }
};

}  // namespace les

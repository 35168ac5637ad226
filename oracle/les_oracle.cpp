// les_oracle.cpp -- CPU ORACLE (test infrastructure only).
//
// A C++ restatement of the paes-channelflow per-timestep path, used by the
// tests and by bench.py's cpu_baseline leg as the checker.  It is never part
// of the product path.  It follows the Fortran routines statement by
// statement, including the sliding window of planes and the ring-buffer
// indices of comp1.f90, so that the product's level-parallel reformulation
// is checked against the reference's own control flow.
//
// Parity unpinned: the reference ships no tests, golden vectors or fixtures,
// and it cannot be built here (no Fortran compiler, no FFTW 2.x).  The
// restatement is pinned instead against (a) analytic known answers and
// (b) an independent numpy restatement (oracle/mini.py).
//
// FFTW 2.x (not vendored, version not pinned by configure.user:8-10) is
// replaced by a mixed-radix Stockham DFT with the same conventions:
// forward sign -1, rfftwnd forward scaled by 1/(n1*n2) in ffthrz, inverse
// unscaled, 1-D derivative pair scaled by 1/n after the inverse.
//
// Templated on the real type: double reproduces the -fdefault-real-8 build,
// float the shipped single-precision build (sums promoted with dble()).

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/les_gpu.h"
#include "mlp_oracle.h"

namespace orc {

template <class T> using cplx = std::complex<T>;

// ---------------------------------------------------------------------------
// Complex DFT of length n = 2^a 3^b (Stockham autosort, radix 4/2/3).
// Stands in for FFTW 2.x's rfftw / rfftwnd (filter_fftw.f90:49-74).
// ---------------------------------------------------------------------------
template <class T>
struct Dft {
  int n;
  std::vector<cplx<T>> w;  // w[k] = exp(-2 pi i k / n)
  explicit Dft(int n_) : n(n_), w(n_) {
    int m = n;
    while (m % 2 == 0) m /= 2;
    while (m % 3 == 0) m /= 3;
    if (m != 1) throw std::runtime_error("oracle DFT length must be 2^a 3^b");
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int k = 0; k < n; k++) {
      long double a = -2.0L * pi * (long double)k / (long double)n;
      w[k] = cplx<T>((T)cosl(a), (T)sinl(a));
    }
  }
  // Unnormalised transform, sign -1 forward / +1 backward.  x in/out,
  // y scratch of length n.
  void run(cplx<T>* x, cplx<T>* y, int sign) const {
    cplx<T>* a = x;
    cplx<T>* b = y;
    int ns = 1;
    const T s3 = (T)0.86602540378443864676372317075293618L;  // sin(2 pi/3)
    while (ns < n) {
      int rem = n / ns;
      int R = (rem % 4 == 0) ? 4 : ((rem % 2 == 0) ? 2 : 3);
      int m = n / R;
      int step = n / (ns * R);
      for (int j = 0; j < m; j++) {
        int k = j % ns;
        cplx<T> v[4];
        for (int r = 0; r < R; r++) {
          cplx<T> t = a[j + r * m];
          cplx<T> tw = w[(k * r * step) % n];
          if (sign > 0) tw = std::conj(tw);
          v[r] = (r == 0) ? t : t * tw;
        }
        if (R == 2) {
          cplx<T> t0 = v[0] + v[1], t1 = v[0] - v[1];
          v[0] = t0; v[1] = t1;
        } else if (R == 4) {
          cplx<T> a0 = v[0] + v[2], a1 = v[0] - v[2];
          cplx<T> b0 = v[1] + v[3], b1 = v[1] - v[3];
          // multiply b1 by sign*i
          cplx<T> ib1 = (sign < 0) ? cplx<T>(b1.imag(), -b1.real()) : cplx<T>(-b1.imag(), b1.real());
          v[0] = a0 + b0; v[2] = a0 - b0; v[1] = a1 + ib1; v[3] = a1 - ib1;
        } else {
          cplx<T> t1 = v[1] + v[2];
          cplx<T> t2 = v[0] - t1 * (T)0.5;
          cplx<T> d = v[1] - v[2];
          T sg = (sign < 0) ? -s3 : s3;
          cplx<T> t3(-sg * d.imag(), sg * d.real());  // sg*i*d
          v[0] = v[0] + t1; v[1] = t2 + t3; v[2] = t2 - t3;
        }
        int base = (j / ns) * ns * R + k;
        for (int r = 0; r < R; r++) b[base + r * ns] = v[r];
      }
      std::swap(a, b);
      ns *= R;
    }
    if (a != x) std::memcpy(x, a, sizeof(cplx<T>) * n);
  }
};

template <class T>
struct DftCache {
  std::vector<std::unique_ptr<Dft<T>>> d;
  const Dft<T>& get(int n) {
    for (auto& p : d)
      if (p->n == n) return *p;
    d.emplace_back(new Dft<T>(n));
    return *d.back();
  }
};

// Sum promoted to double: sum(dble(x)) (e.g. comp1.f90:145).
template <class T>
static double dsum(const T* x, size_t n) {
  double s = 0.0;
  for (size_t i = 0; i < n; i++) s += (double)x[i];
  return s;
}

// ---------------------------------------------------------------------------
// Spectral core: filter_fftw.f90.  Spectral planes are stored as complex
// [ky][kx], kx = 0..n1/2, the interleaved (n1+2, n2) layout of rfftwnd.
// ---------------------------------------------------------------------------
template <class T>
struct Spectral {
  DftCache<T> cache;

  // ffthrz(fa, n1, n2, -1) (filter_fftw.f90:107-130): 2-D real-to-complex,
  // scaled by 1/(n1*n2).
  void r2c(const T* in, cplx<T>* out, int n1, int n2) {
    const Dft<T>& dx = cache.get(n1);
    const Dft<T>& dy = cache.get(n2);
    int h = n1 / 2 + 1;
    std::vector<cplx<T>> tmp((size_t)h * n2);
#pragma omp parallel
    {
      std::vector<cplx<T>> a(std::max(n1, n2)), s(std::max(n1, n2));
#pragma omp for
      for (int y = 0; y < n2; y++) {
        for (int x = 0; x < n1; x++) a[x] = cplx<T>(in[(size_t)y * n1 + x], 0);
        dx.run(a.data(), s.data(), -1);
        for (int k = 0; k < h; k++) tmp[(size_t)y * h + k] = a[k];
      }
#pragma omp for
      for (int k = 0; k < h; k++) {
        for (int y = 0; y < n2; y++) a[y] = tmp[(size_t)y * h + k];
        dy.run(a.data(), s.data(), -1);
        T sc = (T)1 / (T)n1 / (T)n2;
        for (int y = 0; y < n2; y++) out[(size_t)y * h + k] = a[y] * sc;
      }
    }
  }
  // ffthrz(fa, n1, n2, +1): 2-D complex-to-real, unscaled.  Only the real
  // parts of the kx=0 and kx=n1/2 entries enter (rfftw c2r convention).
  void c2r(const cplx<T>* in, T* out, int n1, int n2) {
    const Dft<T>& dx = cache.get(n1);
    const Dft<T>& dy = cache.get(n2);
    int h = n1 / 2 + 1;
    std::vector<cplx<T>> tmp((size_t)h * n2);
#pragma omp parallel
    {
      std::vector<cplx<T>> a(std::max(n1, n2)), s(std::max(n1, n2));
#pragma omp for
      for (int k = 0; k < h; k++) {
        for (int y = 0; y < n2; y++) a[y] = in[(size_t)y * h + k];
        dy.run(a.data(), s.data(), +1);
        for (int y = 0; y < n2; y++) tmp[(size_t)y * h + k] = a[y];
      }
#pragma omp for
      for (int y = 0; y < n2; y++) {
        const cplx<T>* g = &tmp[(size_t)y * h];
        a[0] = cplx<T>(g[0].real(), 0);
        a[n1 / 2] = cplx<T>(g[n1 / 2].real(), 0);
        for (int k = 1; k < n1 / 2; k++) {
          a[k] = g[k];
          a[n1 - k] = std::conj(g[k]);
        }
        dx.run(a.data(), s.data(), +1);
        for (int x = 0; x < n1; x++) out[(size_t)y * n1 + x] = a[x].real();
      }
    }
  }
  // xderiv (filter_fftw.f90:138-187): batched 1-D transform along x,
  // multiply by i*xk, DC and Nyquist zeroed, inverse, times 1/n1.
  void xderiv(const T* ain, T* ax, const T* xk, int n1, int n2) {
    const Dft<T>& d = cache.get(n1);
    T nm1 = (T)1 / (T)n1;
#pragma omp parallel
    {
      std::vector<cplx<T>> a(n1), s(n1);
#pragma omp for
      for (int y = 0; y < n2; y++) {
        for (int x = 0; x < n1; x++) a[x] = cplx<T>(ain[(size_t)y * n1 + x], 0);
        d.run(a.data(), s.data(), -1);
        for (int k = 1; k < n1 / 2; k++) {
          // ax(k) = xk(n1-k) * Im ; ax(n1-k) = xk(k) * Re  (half-complex swap)
          T re = a[k].real(), im = a[k].imag();
          a[k] = cplx<T>(xk[n1 - k] * im, xk[k] * re);
          a[n1 - k] = std::conj(a[k]);
        }
        a[0] = 0;
        a[n1 / 2] = 0;
        d.run(a.data(), s.data(), +1);
        for (int x = 0; x < n1; x++) ax[(size_t)y * n1 + x] = a[x].real() * nm1;
      }
    }
  }
  // yderiv (filter_fftw.f90:194-248).
  void yderiv(const T* ain, T* ay, const T* yk, int n1, int n2) {
    const Dft<T>& d = cache.get(n2);
    T nm1 = (T)1 / (T)n2;
#pragma omp parallel
    {
      std::vector<cplx<T>> a(n2), s(n2);
#pragma omp for
      for (int x = 0; x < n1; x++) {
        for (int y = 0; y < n2; y++) a[y] = cplx<T>(ain[(size_t)y * n1 + x], 0);
        d.run(a.data(), s.data(), -1);
        for (int k = 1; k < n2 / 2; k++) {
          T re = a[k].real(), im = a[k].imag();
          a[k] = cplx<T>(yk[n2 - k] * im, yk[k] * re);
          a[n2 - k] = std::conj(a[k]);
        }
        a[0] = 0;
        a[n2 / 2] = 0;
        d.run(a.data(), s.data(), +1);
        for (int y = 0; y < n2; y++) ay[(size_t)y * n1 + x] = a[y].real() * nm1;
      }
    }
  }
  // expand (filter_fftw.f90:254-278): small spectrum, keep kx < nx/2 and
  // ky != ny/2, zero-pad, inverse on the 3/2 grid.
  void expand(const T* xs, T* xl, int nx, int ny) {
    int nxb = 3 * nx / 2, nyb = 3 * ny / 2;
    int hs = nx / 2 + 1, hb = nxb / 2 + 1;
    std::vector<cplx<T>> zs((size_t)hs * ny), zl((size_t)hb * nyb, cplx<T>(0, 0));
    r2c(xs, zs.data(), nx, ny);
    for (int ky = 0; ky < ny; ky++) {
      if (ky == ny / 2) continue;
      int kyb = (ky < ny / 2) ? ky : ky + (nyb - ny);
      for (int kx = 0; kx < nx / 2; kx++) zl[(size_t)kyb * hb + kx] = zs[(size_t)ky * hs + kx];
    }
    c2r(zl.data(), xl, nxb, nyb);
  }
  // compress (filter_fftw.f90:285-308).
  void compress(const T* xl, T* xs, int nx, int ny) {
    int nxb = 3 * nx / 2, nyb = 3 * ny / 2;
    int hs = nx / 2 + 1, hb = nxb / 2 + 1;
    std::vector<cplx<T>> zs((size_t)hs * ny, cplx<T>(0, 0)), zl((size_t)hb * nyb);
    r2c(xl, zl.data(), nxb, nyb);
    for (int ky = 0; ky < ny; ky++) {
      if (ky == ny / 2) continue;
      int kyb = (ky < ny / 2) ? ky : ky + (nyb - ny);
      for (int kx = 0; kx < nx / 2; kx++) zs[(size_t)ky * hs + kx] = zl[(size_t)kyb * hb + kx];
    }
    c2r(zs.data(), xs, nx, ny);
  }
  // deal (filter_fftw.f90:316-329).
  void deal(T* x, int nx, int ny) {
    int hs = nx / 2 + 1;
    std::vector<cplx<T>> z((size_t)hs * ny);
    r2c(x, z.data(), nx, ny);
    for (int ky = 0; ky < ny; ky++) z[(size_t)ky * hs + nx / 2] = 0;
    for (int kx = 0; kx < nx / 2; kx++) z[(size_t)(ny / 2) * hs + kx] = 0;
    c2r(z.data(), x, nx, ny);
  }
};

// tridv (tridv.f90:1-55): Thomas algorithm batched over ny right-hand sides;
// bdar(ny, n, 4) column-major = b (sub), d (diag), a (super), r (rhs).
template <class T>
void tridv(T* bdar, int ny, int n) {
  T* b = bdar;
  T* d = bdar + (size_t)ny * n;
  T* a = bdar + (size_t)2 * ny * n;
  T* r = bdar + (size_t)3 * ny * n;
  auto I = [ny](int j, int i) { return (size_t)(i - 1) * ny + (j - 1); };
  if (n <= 1) {
    for (int j = 1; j <= ny; j++) r[I(j, 1)] = r[I(j, 1)] / d[I(j, 1)];
    return;
  }
  for (int j = 1; j <= ny; j++) d[I(j, 1)] = (T)1 / d[I(j, 1)];
  for (int i = 2; i <= n; i++)
    for (int j = 1; j <= ny; j++) {
      T fac = b[I(j, i)] * d[I(j, i - 1)];
      d[I(j, i)] = (T)1 / (d[I(j, i)] - fac * a[I(j, i - 1)]);
      r[I(j, i)] = r[I(j, i)] - fac * r[I(j, i - 1)];
    }
  for (int j = 1; j <= ny; j++) r[I(j, n)] = r[I(j, n)] * d[I(j, n)];
  for (int ii = 1; ii <= n - 1; ii++) {
    int i = n - ii;
    for (int j = 1; j <= ny; j++) r[I(j, i)] = d[I(j, i)] * (r[I(j, i)] - a[I(j, i)] * r[I(j, i + 1)]);
  }
}

// A stack of planes with Fortran level bounds lo..hi (allocate.f90:14-36).
template <class T>
struct Levels {
  int lo = 0, hi = -1;
  size_t plane = 0;
  std::vector<T> data;
  void alloc(int lo_, int hi_, size_t plane_) {
    lo = lo_; hi = hi_; plane = plane_;
    data.assign((size_t)(hi - lo + 1) * plane, (T)0);
  }
  T* at(int iz) {
    if (iz < lo || iz > hi) throw std::runtime_error("level out of range");
    return data.data() + (size_t)(iz - lo) * plane;
  }
};

// ---------------------------------------------------------------------------
// The model state and routines (storage/compbuf modules).
// ---------------------------------------------------------------------------
template <class T>
struct Les {
  les_config cfg;
  int nnx, nny, nnz, nnxb, nnyb, ncx, ncy;
  size_t ps, pb;  // small and padded plane sizes
  T pi, xl, yl, zl, z0, dx, dy, dz, z1, zody, dzm, dzm2, todzm, dsl, ceps, almin;
  T xym, xymb, emin, vk, dt, dtab1 = 0, dtab2 = 0, dtabm = 0, xkmax = 0;
  T utau = 0, utau_s = 0, dudt = 0, dvdt = 0, ugal, vgal, ufree, forcing;
  T utau_lower = 0;
  std::vector<T> xk, yk, xkb, ykb;
  Levels<T> u, v, w, e, p, ru, rv, rw, re;
  // compbuf
  std::vector<std::vector<T>> ubuf, vbuf, wbuf, ebuf;  // indexed kb+offset
  std::vector<T> rubuf, rvbuf, rwbuf, rebuf;
  std::vector<std::vector<T>> UX, UY, UZ, VX, VY, VZ, WX, WY, WZ, XKK, ALK, SHEAR;
  std::vector<T> EX, EY, tauuu, tauuv, tauvv;
  std::vector<std::vector<T>> tauww, tauuw, tauvw;
  std::vector<double> meanbuf;  // (19, nnz) column-major
  Spectral<T> sp;
  // learned closure (imodel = LES_SGS_LEARNED with a network attached)
  bool learned = false, mlp_bf16 = true;
  std::vector<double> mlpP, mlpN;
  double re_tau = 0.0;
  int learned_used = 0;
  double learned_dissip = 0.0;
  // second fallback test: the network's mean dissipation must lie within a
  // factor `learned_guard` of the reference (Smagorinsky) dissipation on the
  // same state (learned_guard <= 0: only the sign test)
  double learned_guard = 4.0;
  double learned_dissip_r = 0.0, learned_dissip_raw = 0.0;
  long long learned_stages = 0, learned_stages_used = 0;
  T sgs_mom = (T)1;  // weight of the interior momentum stresses of compsgs1
  Levels<T> lru, lrv, lrw;

  // buffer window offsets: ubuf(-1:2), vbuf(-1:2), wbuf(-2:2), ebuf(-1:1)
  T* UB(int k) { return ubuf[k + 1].data(); }
  T* VB(int k) { return vbuf[k + 1].data(); }
  T* WB(int k) { return wbuf[k + 2].data(); }
  T* EB(int k) { return ebuf[k + 1].data(); }

  explicit Les(const les_config& c) : cfg(c) {
    nnx = c.nnx; nny = c.nny; nnz = c.nnz;
    if (nnx < 4 || nny < 4 || nnz < 4 || nnx % 2 || nny % 2) throw std::runtime_error("bad grid");
    // derived constants, les.F90:92-121
    pi = (T)4 * std::atan((T)1);
    nnxb = 3 * nnx / 2; nnyb = 3 * nny / 2;
    xymb = (T)1 / (T)nnxb / (T)nnyb;
    emin = (T)c.emin;
    ncx = nnx / 2 + 1; ncy = nny / 2 + 1;
    xym = (T)1 / (T)(nnx * nny);
    xl = (T)c.xl; yl = (T)c.yl; zl = (T)c.zl; z0 = (T)c.z0;
    dx = xl / (T)nnx; dy = yl / (T)nny; dz = zl / (T)nnz;
    z1 = dz / (T)2;
    zody = std::log(z1 / z0);
    dzm = (T)1 / dz; dzm2 = dzm * dzm; todzm = (T)0.5 / dz;
    dsl = std::pow(dx * dy * dz, (T)1 / (T)3);
    ceps = (T)0.93 / dsl;
    almin = (T)0.0075 * dsl;
    vk = (T)0.4;
    dt = (T)c.dt;
    ugal = (T)c.ugal; vgal = (T)c.vgal; ufree = (T)c.ufree; forcing = (T)c.forcing;
    ps = (size_t)nnx * nny;
    pb = (size_t)nnxb * nnyb;
    // allocate_arrays with np=(2,2,2,1), nm=(1,1,2,1) (buffers.f90, isbgr)
    u.alloc(0, nnz + 2, ps); v.alloc(0, nnz + 2, ps); w.alloc(-1, nnz + 2, ps);
    e.alloc(0, nnz + 1, ps);
    ru.alloc(1, nnz, ps); rv.alloc(1, nnz, ps); rw.alloc(0, nnz, ps); re.alloc(1, nnz, ps);
    p.alloc(1, nnz + 1, (size_t)(nnx + 2) * nny);
    auto planes = [&](std::vector<std::vector<T>>& v_, int n) { v_.assign(n, std::vector<T>(pb, (T)0)); };
    planes(ubuf, 4); planes(vbuf, 4); planes(wbuf, 5); planes(ebuf, 3);
    rubuf.assign(pb, 0); rvbuf.assign(pb, 0); rwbuf.assign(pb, 0); rebuf.assign(pb, 0);
    planes(UX, 4); planes(UY, 4); planes(UZ, 3); planes(VX, 4); planes(VY, 4); planes(VZ, 3);
    planes(WX, 3); planes(WY, 3); planes(WZ, 4); planes(XKK, 3); planes(ALK, 3); planes(SHEAR, 3);
    EX.assign(pb, 0); EY.assign(pb, 0); tauuu.assign(pb, 0); tauuv.assign(pb, 0); tauvv.assign(pb, 0);
    planes(tauww, 2); planes(tauuw, 2); planes(tauvw, 2);
    // alk is allocated but never assigned in the reference (complen.f90:21);
    // Deardorff's neutral length scale l = dsl is used (consistent with
    // ceps = 0.93/dsl, les.F90:120).
    for (auto& a : ALK) std::fill(a.begin(), a.end(), dsl);
    meanbuf.assign((size_t)19 * nnz, 0.0);
    initwave();
  }

  // initwave (init.f90:4-44)
  void initwave() {
    xkb.resize(nnxb); ykb.resize(nnyb); xk.resize(nnx); yk.resize(nny);
    for (int ix = 1; ix <= nnxb; ix++) {
      xkb[ix - 1] = (T)(ix - 1) * (T)2 * pi / xl;
      if (ix > nnxb / 2 + 1) xkb[ix - 1] = -(T)(nnxb - ix + 1) * (T)2 * pi / xl;
    }
    for (int iy = 1; iy <= nnyb; iy++) {
      ykb[iy - 1] = (T)(iy - 1) * (T)2 * pi / yl;
      if (iy > nnyb / 2 + 1) ykb[iy - 1] = -(T)(nnyb - iy + 1) * (T)2 * pi / yl;
    }
    for (int ix = 1; ix <= nnx; ix++) {
      xk[ix - 1] = (T)(ix - 1) * (T)2 * pi / xl;
      if (ix > ncx) xk[ix - 1] = -(T)(nnx - ix + 1) * (T)2 * pi / xl;
    }
    for (int iy = 1; iy <= nny; iy++) {
      yk[iy - 1] = (T)(iy - 1) * (T)2 * pi / yl;
      if (iy > ncy) yk[iy - 1] = -(T)(nny - iy + 1) * (T)2 * pi / yl;
    }
  }

  void xd(const T* a, T* o) { sp.xderiv(a, o, xkb.data(), nnxb, nnyb); }
  void yd(const T* a, T* o) { sp.yderiv(a, o, ykb.data(), nnxb, nnyb); }
  void expand_to(T* small, T* big) { sp.expand(small, big, nnx, nny); }
  void compress_to(const T* big, T* small) { sp.compress(big, small, nnx, nny); }

  // lower (lowerbc.f90:1-20)
  void lower() {
    std::fill_n(u.at(0), ps, (T)0);
    std::fill_n(v.at(0), ps, (T)0);
    std::fill_n(w.at(-1), ps, (T)0);
    std::fill_n(w.at(0), ps, (T)0);
    std::copy_n(e.at(1), ps, e.at(0));
  }
  // upper (upperbc.f90:1-30)
  void upper() {
    for (int iz = nnz + 1; iz <= nnz + 2; iz++) std::fill_n(u.at(iz), ps, (T)0);
    for (int iz = nnz + 1; iz <= nnz + 2; iz++) std::fill_n(v.at(iz), ps, (T)0);
    for (int iz = nnz; iz <= nnz + 1; iz++) std::copy_n(e.at(nnz - 1), ps, e.at(iz));
    for (int iz = nnz; iz <= nnz + 2; iz++) std::fill_n(w.at(iz), ps, (T)0);
    std::fill_n(rw.at(nnz), ps, (T)0);
  }

  // derivsbot (derivs1.f90:1-66) for iz = istart = 1, kb = 0.
  void derivsbot(int iz, int lm1, int l, int nm1, int n, int np1) {
    xd(UB(0), UX[n].data()); xd(UB(1), UX[np1].data());
    yd(UB(0), UY[n].data()); yd(UB(1), UY[np1].data());
    xd(VB(0), VX[n].data()); xd(VB(1), VX[np1].data());
    yd(VB(0), VY[n].data()); yd(VB(1), VY[np1].data());
    for (size_t i = 0; i < pb; i++) {
      WZ[n][i] = (WB(0)[i] - WB(-1)[i]) * dzm;
      WZ[np1][i] = (WB(1)[i] - WB(0)[i]) * dzm;
      UZ[l][i] = (UB(1)[i] - UB(0)[i]) * dzm;
      VZ[l][i] = (VB(1)[i] - VB(0)[i]) * dzm;
    }
    xd(WB(0), WX[l].data()); yd(WB(0), WY[l].data());
    if (iz != 1) throw std::runtime_error("oracle supports istart = 1 only");
    std::fill(UX[nm1].begin(), UX[nm1].end(), (T)0);
    std::fill(UY[nm1].begin(), UY[nm1].end(), (T)0);
    std::fill(VX[nm1].begin(), VX[nm1].end(), (T)0);
    std::fill(VY[nm1].begin(), VY[nm1].end(), (T)0);
    std::fill(WZ[nm1].begin(), WZ[nm1].end(), (T)0);
    std::fill(WX[lm1].begin(), WX[lm1].end(), (T)0);
    std::fill(WY[lm1].begin(), WY[lm1].end(), (T)0);
    UZ[lm1] = UZ[l];
    VZ[lm1] = VZ[l];
  }
  // derivs (derivs2.f90:1-42), kb = 0.
  void derivs(int iz, int l, int lp1, int np2) {
    if (iz < nnz - 1) {
      xd(UB(2), UX[np2].data()); yd(UB(2), UY[np2].data());
      xd(VB(2), VX[np2].data()); yd(VB(2), VY[np2].data());
      for (size_t i = 0; i < pb; i++) {
        WZ[np2][i] = (WB(2)[i] - WB(1)[i]) * dzm;
        UZ[lp1][i] = (UB(2)[i] - UB(1)[i]) * dzm;
        VZ[lp1][i] = (VB(2)[i] - VB(1)[i]) * dzm;
      }
      xd(WB(1), WX[lp1].data()); yd(WB(1), WY[lp1].data());
      xd(EB(0), EX.data()); yd(EB(0), EY.data());
    } else {
      std::fill(UX[np2].begin(), UX[np2].end(), (T)0);
      std::fill(UY[np2].begin(), UY[np2].end(), (T)0);
      std::fill(VX[np2].begin(), VX[np2].end(), (T)0);
      std::fill(VY[np2].begin(), VY[np2].end(), (T)0);
      UZ[lp1] = UZ[l];
      VZ[lp1] = VZ[l];
      std::fill(WZ[np2].begin(), WZ[np2].end(), (T)0);
      std::fill(WX[lp1].begin(), WX[lp1].end(), (T)0);
      std::fill(WY[lp1].begin(), WY[lp1].end(), (T)0);
    }
  }

  // compadv1 (compadv1.f90:3-66), kb = 0.
  void compadv1(int iz) {
    std::vector<T> f1(pb), f2(pb), tmp(pb);
    for (size_t i = 0; i < pb; i++) tmp[i] = UB(0)[i] * UB(0)[i];
    xd(tmp.data(), f1.data());
    for (size_t i = 0; i < pb; i++) tmp[i] = UB(0)[i] * VB(0)[i];
    yd(tmp.data(), f2.data());
    for (size_t i = 0; i < pb; i++)
      rubuf[i] = -f1[i] - f2[i] -
                 ((UB(1)[i] + UB(0)[i]) * WB(0)[i] - (UB(-1)[i] + UB(0)[i]) * WB(-1)[i]) * todzm;
    for (size_t i = 0; i < pb; i++) tmp[i] = UB(0)[i] * VB(0)[i];
    xd(tmp.data(), f1.data());
    for (size_t i = 0; i < pb; i++) tmp[i] = VB(0)[i] * VB(0)[i];
    yd(tmp.data(), f2.data());
    for (size_t i = 0; i < pb; i++)
      rvbuf[i] = -f1[i] - f2[i] -
                 ((VB(1)[i] + VB(0)[i]) * WB(0)[i] - (VB(-1)[i] + VB(0)[i]) * WB(-1)[i]) * todzm;
    if (iz == nnz) {
      std::fill(rwbuf.begin(), rwbuf.end(), (T)0);
    } else {
      for (size_t i = 0; i < pb; i++) tmp[i] = (UB(0)[i] + UB(1)[i]) * WB(0)[i];
      xd(tmp.data(), f1.data());
      for (size_t i = 0; i < pb; i++) tmp[i] = (VB(0)[i] + VB(1)[i]) * WB(0)[i];
      yd(tmp.data(), f2.data());
      for (size_t i = 0; i < pb; i++) {
        T a = (T)0.5 * (WB(1)[i] + WB(0)[i]);
        T b = (T)0.5 * (WB(0)[i] + WB(-1)[i]);
        rwbuf[i] = -(T)0.5 * f1[i] - (T)0.5 * f2[i] - (a * a - b * b) * dzm;
      }
    }
    if (iz != nnz) {
      for (size_t i = 0; i < pb; i++) tmp[i] = EB(0)[i] * (UB(0)[i] + UB(1)[i]);
      xd(tmp.data(), f1.data());
      for (size_t i = 0; i < pb; i++) tmp[i] = EB(0)[i] * (VB(0)[i] + VB(1)[i]);
      yd(tmp.data(), f2.data());
      for (size_t i = 0; i < pb; i++)
        rebuf[i] = -(T)0.5 * (f1[i] + f2[i]) - (WB(1)[i] * EB(1)[i] - WB(-1)[i] * EB(-1)[i]) * todzm;
    }
  }

  // complen (complen.f90:1-28) for ring slot l, ebuf offset kb.
  void complen(int l, int kb, int n, int np1) {
    T* sh = SHEAR[l].data();
    T* xk_ = XKK[l].data();
    const T* eb = EB(kb);
    T xkmx = xkmax;
    T nu = (T)cfg.nu;
    for (size_t i = 0; i < pb; i++) {
      T a = UY[n][i] + VX[n][i], b = UY[np1][i] + VX[np1][i];
      T c = UZ[l][i] + WX[l][i], d = VZ[l][i] + WY[l][i];
      sh[i] = UX[n][i] * UX[n][i] + UX[np1][i] * UX[np1][i] + VY[n][i] * VY[n][i] +
              VY[np1][i] * VY[np1][i] + WZ[n][i] * WZ[n][i] + WZ[np1][i] * WZ[np1][i] +
              (T)0.5 * a * a + (T)0.5 * b * b + c * c + d * d;
      T val;
      if (cfg.imodel == 4)
        val = std::min(((T)0.1 * dsl) * ((T)0.1 * dsl) * std::sqrt(sh[i]), xkmx);
      else
        val = std::min((T)0.1 * ALK[l][i] * std::sqrt(eb[i]), xkmx);
      xk_[i] = val + nu;
    }
  }

  // sufsim (lowerbc.f90:25-165) on ubuf(0), vbuf(0) = level 1.
  void sufsim(int km1) { wall(true, km1); }
  // sufsim_upper (upperbc.f90:33-160) on level nnz.
  void sufsim_upper(int k) { wall(false, k); }

  void wall(bool lowerwall, int slot) {
    const T* U0 = UB(0);
    const T* V0 = VB(0);
    T u1xy = (T)(dsum(U0, pb) * (double)xymb);
    T v1xy = (T)(dsum(V0, pb) * (double)xymb);
    if (!lowerwall) { u1xy += ugal; v1xy += vgal; }
    std::vector<T> wind(pb);
    for (size_t i = 0; i < pb; i++) wind[i] = std::sqrt(U0[i] * U0[i] + V0[i] * V0[i]);
    T windm = (T)(dsum(wind.data(), pb) * (double)xymb);
    T vsfc = std::sqrt(u1xy * u1xy + v1xy * v1xy);
    windm = std::max(windm, ufree);
    windm = std::max(windm, (T)0.01);
    vsfc = std::max(vsfc, (T)0.01);
    T ut = vsfc * vk / zody;
    utau = ut;
    if (lowerwall) {
      utau_lower = ut;
      // new modelling approach (lowerbc.f90:70-72): global means of ru, rv
      double s = 0.0, sv = 0.0;
      for (int iz = 1; iz <= nnz; iz++) { s += dsum(ru.at(iz), ps); sv += dsum(rv.at(iz), ps); }
      dudt = (T)(s / (double)((long long)nnx * nny * nnz));
      dvdt = (T)(sv / (double)((long long)nnx * nny * nnz));
      utau_s = std::sqrt(zl / (T)2 * std::sqrt((-dvdt) * (-dvdt) + (forcing - dudt) * (forcing - dudt)));
    }
    if (ut > (T)10) throw std::runtime_error("utau > 10");
    T tep = u1xy / vsfc;
    tep = std::min(tep, (T)1);
    tep = std::max(tep, (T)-1);
    T thta = std::acos(tep);
    T utau2 = ut * ut;
    T sgn = std::copysign((T)1, v1xy);
    T auuwm = lowerwall ? -utau2 * std::cos(thta) : utau2 * std::cos(thta);
    T auvwm = lowerwall ? -utau2 * std::sin(thta) * sgn : utau2 * std::sin(thta) * sgn;
    int isf = cfg.isurface;
    std::vector<T> ufluc(pb), vfluc(pb), sfluc(pb), moengu(pb), moengv(pb);
    T ufluc2mroot = 0, vfluc2mroot = 0, suflucm = 0, svflucm = 0, moengu2mroot = 0, moengv2mroot = 0;
    if (isf > 2) {
      double a1 = 0, a2 = 0, a3 = 0, a4 = 0, a5 = 0, a6 = 0;
      for (size_t i = 0; i < pb; i++) {
        sfluc[i] = wind[i] - windm;
        ufluc[i] = U0[i] + ugal - u1xy;
        vfluc[i] = V0[i] + vgal - v1xy;
        moengu[i] = sfluc[i] * u1xy + windm * ufluc[i];
        moengv[i] = sfluc[i] * v1xy + windm * vfluc[i];
        a1 += (double)(ufluc[i] * ufluc[i]);
        a2 += (double)(vfluc[i] * vfluc[i]);
        a3 += (double)(ufluc[i] * sfluc[i]);
        a4 += (double)(vfluc[i] * sfluc[i]);
        a5 += (double)(moengu[i] * moengu[i]);
        a6 += (double)(moengv[i] * moengv[i]);
      }
      (void)a6;
      ufluc2mroot = std::sqrt((T)(a1 * (double)xymb));
      vfluc2mroot = std::sqrt((T)(a2 * (double)xymb));
      suflucm = (T)(a3 * (double)xymb);
      svflucm = (T)(a4 * (double)xymb);
      moengu2mroot = std::sqrt((T)(a5 * (double)xymb));
      // moengv2m is built from moengu2 in the reference (lowerbc.f90:121)
      moengv2mroot = std::sqrt((T)(a5 * (double)xymb));
    }
    T* tu = tauuw[slot].data();
    T* tv = tauvw[slot].data();
    T sg = lowerwall ? (T)-1 : (T)1;
    switch (isf) {
      case 1:
        for (size_t i = 0; i < pb; i++) {
          tu[i] = sg * utau2 / vsfc * (U0[i] + ugal);
          tv[i] = sg * utau2 / vsfc * (V0[i] + vgal);
        }
        break;
      case 2:
        for (size_t i = 0; i < pb; i++) {
          T uf = U0[i] + ugal - u1xy, vf = V0[i] + vgal - v1xy;
          tu[i] = sg * utau2 / (windm * vsfc) * (windm * uf + wind[i] * u1xy);
          tv[i] = sg * utau2 / (windm * vsfc) * (windm * vf + wind[i] * v1xy);
        }
        break;
      case 3:
        for (size_t i = 0; i < pb; i++) {
          tu[i] = auuwm + sg * (T)-1 * (T)0.35 * ufluc[i] * utau2 / ufluc2mroot;
          tv[i] = auvwm + sg * (T)-1 * (T)0.35 * vfluc[i] * utau2 / vfluc2mroot;
        }
        break;
      case 4: {
        T denom = std::sqrt((windm * u1xy + suflucm) * (windm * u1xy + suflucm) +
                            (windm * v1xy + svflucm) * (windm * v1xy + svflucm));
        for (size_t i = 0; i < pb; i++) {
          tu[i] = sg * utau2 * (wind[i] * (U0[i] + ugal)) / denom;
          tv[i] = sg * utau2 * (wind[i] * (V0[i] + vgal)) / denom;
        }
        break;
      }
      case 5:
        for (size_t i = 0; i < pb; i++) {
          tu[i] = auuwm + sg * (T)-1 * (T)0.35 * utau2 * moengu[i] / moengu2mroot;
          tv[i] = auvwm + sg * (T)-1 * (T)0.35 * utau2 * moengv[i] / moengv2mroot;
        }
        break;
      case 6: {
        T au = -zl / (T)2 * (forcing - dudt);
        T av = -zl / (T)2 * (-dvdt);
        for (size_t i = 0; i < pb; i++) {
          if (lowerwall) {
            tu[i] = au - ut * utau_s * ufluc[i] / vsfc;
            tv[i] = av - ut * utau_s * vfluc[i] / vsfc;
          } else {
            tu[i] = -au + ut * utau_s * ufluc[i] / vsfc;
            tv[i] = -av + ut * utau_s * vfluc[i] / vsfc;
          }
        }
        break;
      }
      default:
        throw std::runtime_error("isurface must be 1..6");
    }
  }

  // compsgs1 (compsgs1.f90:1-53), kb = 0.
  void compsgs1(int iz, int j, int jp1, int k, int km1, int l, int lm1, int lp1, int nm1, int n, int np1,
                int np2) {
    const T mom = sgs_mom;
    const T momw = mom;
    if (iz == 1) {
      complen(lm1, -1, nm1, n);
      complen(l, 0, n, np1);
      for (size_t i = 0; i < pb; i++) tauww[j][i] = -mom * (XKK[lm1][i] + XKK[l][i]) * WZ[n][i];
      sufsim(km1);
    }
    if (iz != nnz) complen(lp1, 1, np1, np2);
    for (size_t i = 0; i < pb; i++) {
      T s = mom * (XKK[lm1][i] + XKK[l][i]);
      tauuu[i] = -s * UX[n][i];
      tauvv[i] = -s * VY[n][i];
      tauuv[i] = -s * (UY[n][i] + VX[n][i]) * (T)0.5;
    }
    if (iz == nnz) {
      std::fill(tauww[jp1].begin(), tauww[jp1].end(), (T)0);
      sufsim_upper(k);
    } else {
      for (size_t i = 0; i < pb; i++) {
        tauww[jp1][i] = -mom * (XKK[l][i] + XKK[lp1][i]) * WZ[np1][i];
        tauuw[k][i] = -momw * XKK[l][i] * (UZ[l][i] + WX[l][i]);
        tauvw[k][i] = -momw * XKK[l][i] * (VZ[l][i] + WY[l][i]);
      }
    }
  }

  // compsgs3 (compsgs3.f90:1-80), kb = 0.
  void compsgs3(int iz, int j, int jp1, int k, int km1, int l, int lm1, int lp1, bool mnout, int istage) {
    std::vector<T> f1(pb), f2(pb), tmp(pb);
    int i = iz;  // istart = 1
    if (iz != nnz) {
      for (size_t q = 0; q < pb; q++) { f1[q] = ((T)2 * XKK[l][q]) * EX[q]; f2[q] = ((T)2 * XKK[l][q]) * EY[q]; }
      std::vector<T> g1(pb), g2(pb);
      xd(f1.data(), g1.data());
      yd(f2.data(), g2.data());
      for (size_t q = 0; q < pb; q++) {
        T t = g1[q] + g2[q] +
              ((XKK[lp1][q] + XKK[l][q]) * (EB(1)[q] - EB(0)[q]) -
               (XKK[l][q] + XKK[lm1][q]) * (EB(0)[q] - EB(-1)[q])) * dzm2;
        rebuf[q] = rebuf[q] + t;
        t = -ceps * EB(0)[q] * std::sqrt(EB(0)[q]);
        rebuf[q] = rebuf[q] + t;
        if (cfg.tke_production) rebuf[q] = rebuf[q] + XKK[l][q] * SHEAR[l][q];
      }
    }
    xd(tauuu.data(), f1.data());
    yd(tauuv.data(), f2.data());
    for (size_t q = 0; q < pb; q++) rubuf[q] = rubuf[q] - f1[q] - f2[q] - (tauuw[k][q] - tauuw[km1][q]) * dzm;
    xd(tauuv.data(), f1.data());
    yd(tauvv.data(), f2.data());
    for (size_t q = 0; q < pb; q++) rvbuf[q] = rvbuf[q] - f1[q] - f2[q] - (tauvw[k][q] - tauvw[km1][q]) * dzm;
    if (iz != nnz) {
      xd(tauuw[k].data(), f1.data());
      yd(tauvw[k].data(), f2.data());
      for (size_t q = 0; q < pb; q++) rwbuf[q] = rwbuf[q] - f1[q] - f2[q] - (tauww[jp1][q] - tauww[j][q]) * dzm;
    } else {
      std::fill(rwbuf.begin(), rwbuf.end(), (T)0);
    }
    if (mnout && istage == 1) {
      double xb = (double)xymb;
      M(16, i) = dsum(tauuv.data(), pb) * xb;  // uvsb
      M(14, i) = dsum(tauuu.data(), pb) * xb;  // uusb
      M(15, i) = dsum(tauvv.data(), pb) * xb;  // vvsb
      M(17, i) = dsum(tauww[j].data(), pb) * xb;  // wwsb
      M(18, i) = dsum(tauuw[k].data(), pb) * xb;  // uwsb
      M(19, i) = dsum(tauvw[k].data(), pb) * xb;  // vwsb
      if (sizeof(T) == 4)
        for (int r : {14, 15, 16, 17, 18, 19}) M(r, i) = (double)(T)M(r, i);
    }
  }

  double& M(int row, int iz) { return meanbuf[(size_t)(iz - 1) * 19 + (row - 1)]; }

  // Learned closure (no reference counterpart; replaces complen/compsgs1's
  // interior stresses).  Velocity gradients at the cell centres of the small
  // grid from the stage's start state:
  //   ux.. = spectral x/y derivatives; wx, wy of (w(k) + w(k-1))/2;
  //   wz = (w(k) - w(k-1))/dz; uz, vz = centred (u(k+1) - u(k-1))/(2dz),
  //   one-sided at k = 1 and nnz (derivs1.f90 / derivs2.f90 wall rows);
  // dimensionless features (g / |G|, min(z_w / dsl, 16), z_w / h),
  // normalised, through the FP64 network; tau = (dsl |G|)^2 c with c the
  // de-normalised outputs, and where tau:S > 0 (local backscatter) the
  // component along S removed: tau' = tau - (tau:S / S:S) S.  The stage
  // uses the network when the raw mean of -tau_ij S_ij is >= 0 and, with
  // learned_guard > 0, the applied mean -tau':S lies within a factor
  // learned_guard of the reference mean dissipation (C_s dsl)^2 |S|^3
  // (|S|^2 = 2 S_ij S_ij; Lilly's constant C_s = 0.17), and then adds the
  // dealiased stress divergence of tau' to ru, rv, rw:
  //   ru += -d/dx tau11 - d/dy tau12 - (tau13w(k) - tau13w(k-1))/dz, ...
  // with tau13w(k) = (tau13(k) + tau13(k+1))/2 on the interior w-levels and 0
  // on the walls (the wall model's stresses stay in compsgs1), plus the
  // compact-stencil correction of the shear stresses on the faces 2..nnz-2.
  void learned_prepare() {
    const int NZ = nnz;
    std::vector<std::vector<T>> tau((size_t)6 * (NZ + 2), std::vector<T>(ps, (T)0));
    auto TA = [&](int f, int k) -> std::vector<T>& { return tau[(size_t)f * (NZ + 2) + k]; };
    std::vector<std::vector<T>> g(9, std::vector<T>(ps));
    std::vector<T> wc(ps);
    const double h = (double)zl / 2.0;
    double dsum_ = 0.0, dsumr_ = 0.0, dsumraw_ = 0.0;
    std::vector<double> nuA((size_t)NZ + 2, 0.0), nuB((size_t)NZ + 2, 0.0);
    for (int iz = 1; iz <= NZ; iz++) {
      sp.xderiv(u.at(iz), g[0].data(), xk.data(), nnx, nny);
      sp.xderiv(v.at(iz), g[1].data(), xk.data(), nnx, nny);
      for (size_t q = 0; q < ps; q++) wc[q] = (T)0.5 * (w.at(iz)[q] + w.at(iz - 1)[q]);
      sp.xderiv(wc.data(), g[2].data(), xk.data(), nnx, nny);
      sp.yderiv(u.at(iz), g[3].data(), yk.data(), nnx, nny);
      sp.yderiv(v.at(iz), g[4].data(), yk.data(), nnx, nny);
      sp.yderiv(wc.data(), g[5].data(), yk.data(), nnx, nny);
      for (size_t q = 0; q < ps; q++) {
        for (int c = 0; c < 2; c++) {
          Levels<T>& a = c == 0 ? u : v;
          T d;
          if (iz == 1) d = (a.at(2)[q] - a.at(1)[q]) * dzm;
          else if (iz == NZ) d = (a.at(NZ)[q] - a.at(NZ - 1)[q]) * dzm;
          else d = (a.at(iz + 1)[q] - a.at(iz - 1)[q]) * ((T)0.5 * dzm);
          g[6 + c][q] = d;
        }
        g[8][q] = (w.at(iz)[q] - w.at(iz - 1)[q]) * dzm;
      }
      const double zc = ((double)iz - 0.5) * (double)dz;
      const double zw = std::min(zc, (double)zl - zc);
      MlpTrace tr;
      const double zd = std::min(zw / (double)dsl, 16.0);
      for (size_t q = 0; q < ps; q++) {
        double f[kIn], x[kIn];
        double g2 = 0.0;
        for (int jj = 0; jj < 9; jj++) g2 += (double)g[jj][q] * (double)g[jj][q];
        const double gm = std::sqrt(g2), rg = gm > 0.0 ? 1.0 / gm : 0.0;
        for (int jj = 0; jj < 9; jj++) f[jj] = (double)g[jj][q] * rg;
        f[9] = zd;
        f[10] = zw / h;
        for (int jj = 0; jj < kIn; jj++) x[jj] = (f[jj] - mlpN[jj]) * mlpN[kIn + jj];
        mlp_forward(mlpP.data(), x, tr, mlp_bf16);
        const double sc = gm * (double)dsl, sc2 = sc * sc;
        double t[kOut];
        for (int o = 0; o < kOut; o++) t[o] = sc2 * (tr.y[o] * mlpN[2 * kIn + o] + mlpN[2 * kIn + kOut + o]);
        const double sv[6] = {(double)g[0][q], (double)g[4][q], (double)g[8][q], 0.5 * ((double)g[3][q] + g[1][q]),
                              0.5 * ((double)g[6][q] + g[2][q]), 0.5 * ((double)g[7][q] + g[5][q])};
        const double sS = sv[0] * sv[0] + sv[1] * sv[1] + sv[2] * sv[2] + 2.0 * (sv[3] * sv[3] + sv[4] * sv[4] + sv[5] * sv[5]);
        const double tS = t[0] * sv[0] + t[1] * sv[1] + t[2] * sv[2] + 2.0 * (t[3] * sv[3] + t[4] * sv[4] + t[5] * sv[5]);
        dsumraw_ += -tS;
        if (tS > 0.0 && sS > 0.0) {
          for (int o = 0; o < kOut; o++) t[o] -= tS / sS * sv[o];
        } else {
          dsum_ += -tS;
        }
        for (int o = 0; o < kOut; o++) TA(o, iz)[q] = (T)t[o];
        const double ss = 2.0 * sS;  // |S|^2
        dsumr_ += 0.17 * 0.17 * (double)dsl * (double)dsl * ss * std::sqrt(ss);
        nuA[iz] += t[4] * (double)g[6][q] + t[5] * (double)g[7][q];
        nuB[iz] += (double)g[6][q] * g[6][q] + (double)g[7][q] * g[7][q];
      }
    }
    learned_dissip = dsum_ / ((double)ps * NZ);
    learned_dissip_r = dsumr_ / ((double)ps * NZ);
    learned_dissip_raw = dsumraw_ / ((double)ps * NZ);
    learned_used = learned_dissip_raw >= 0.0 ? 1 : 0;  // NaN -> fallback
    if (learned_guard > 0.0 && !(learned_dissip_r > 0.0 && learned_dissip <= learned_guard * learned_dissip_r &&
                                 learned_guard * learned_dissip >= learned_dissip_r))
      learned_used = 0;
    learned_stages++;
    learned_stages_used += learned_used;
    if (!learned_used) return;
    // stress divergence
    std::vector<T> t13w_m(ps), t13w_p(ps), t23w_m(ps), t23w_p(ps), f1(ps), f2(ps);
    auto tw = [&](int f, int k, std::vector<T>& o) {
      if (k < 1 || k > NZ - 1) { std::fill(o.begin(), o.end(), (T)0); return; }
      for (size_t q = 0; q < ps; q++) o[q] = (T)0.5 * (TA(f, k)[q] + TA(f, k + 1)[q]);
    };
    for (int iz = 1; iz <= NZ; iz++) {
      tw(4, iz - 1, t13w_m); tw(4, iz, t13w_p); tw(5, iz - 1, t23w_m); tw(5, iz, t23w_p);
      T* a = lru.at(iz);
      sp.xderiv(TA(0, iz).data(), f1.data(), xk.data(), nnx, nny);
      sp.yderiv(TA(3, iz).data(), f2.data(), yk.data(), nnx, nny);
      for (size_t q = 0; q < ps; q++) a[q] = -f1[q] - f2[q] - (t13w_p[q] - t13w_m[q]) * dzm;
      sp.deal(a, nnx, nny);
      a = lrv.at(iz);
      sp.xderiv(TA(3, iz).data(), f1.data(), xk.data(), nnx, nny);
      sp.yderiv(TA(1, iz).data(), f2.data(), yk.data(), nnx, nny);
      for (size_t q = 0; q < ps; q++) a[q] = -f1[q] - f2[q] - (t23w_p[q] - t23w_m[q]) * dzm;
      sp.deal(a, nnx, nny);
      a = lrw.at(iz);
      if (iz <= NZ - 1) {
        sp.xderiv(t13w_p.data(), f1.data(), xk.data(), nnx, nny);
        sp.yderiv(t23w_p.data(), f2.data(), yk.data(), nnx, nny);
        for (size_t q = 0; q < ps; q++) a[q] = -f1[q] - f2[q] - (TA(2, iz + 1)[q] - TA(2, iz)[q]) * dzm;
        sp.deal(a, nnx, nny);
      } else {
        std::fill_n(a, ps, (T)0);
      }
    }
    // Compact-stencil correction on the learned faces 2..nnz-2 (odd-even
    // damping): tau13c(j) = -nu(j) D3[u](j), D3[u](j) = (3 (u(j+1) - u(j)) -
    // (u(j+2) - u(j-1))) / (4 dz); nu(j) the mean of the network's effective
    // viscosity -sum(tau13 uz + tau23 vz) / sum(uz^2 + vz^2) of the cells j
    // and j+1, each clipped to [0, xkmax]; the same for v.
    auto nuc = [&](int k) -> double {
      double nu = nuB[k] > 0.0 ? -nuA[k] / nuB[k] : 0.0;
      return std::min(std::max(nu, 0.0), (double)xkmax);
    };
    std::vector<T> nut((size_t)NZ + 1, (T)0);
    for (int j = 2; j <= NZ - 2; j++) nut[j] = (T)(0.5 * (nuc(j) + nuc(j + 1)));
    auto tc = [&](Levels<T>& f, int j, size_t q) -> T {
      if (j < 2 || j > NZ - 2) return (T)0;
      const T d3 = ((T)3 * (f.at(j + 1)[q] - f.at(j)[q]) - (f.at(j + 2)[q] - f.at(j - 1)[q])) * ((T)0.25 * dzm);
      return -nut[j] * d3;
    };
    for (int iz = 1; iz <= NZ; iz++) {
      T* a = lru.at(iz);
      T* b = lrv.at(iz);
      for (size_t q = 0; q < ps; q++) {
        a[q] -= (tc(u, iz, q) - tc(u, iz - 1, q)) * dzm;
        b[q] -= (tc(v, iz, q) - tc(v, iz - 1, q)) * dzm;
      }
    }
  }
  void set_mlp(const double* P, const double* N, double rt, bool bf16) {
    if (!P) { learned = false; return; }
    mlpP.assign(P, P + kNParam);
    mlpN.assign(N, N + kNNorm);
    re_tau = rt;
    mlp_bf16 = bf16;
    learned = true;
    if (lru.data.empty()) { lru.alloc(1, nnz, ps); lrv.alloc(1, nnz, ps); lrw.alloc(1, nnz, ps); }
  }

  // comp1 (comp1.f90:1-188) with istart = 1, iend = nnz, kb = 0.
  void comp1(int it, bool mnout, int istage) {
    (void)it;
    sgs_mom = (T)1;
    if (learned) {
      learned_prepare();
      if (learned_used) sgs_mom = (T)0;
    }
    for (int iz = 1; iz <= nnz; iz++) {
      int j = iz % 2 + 1 - 1, jp1 = (iz + 1) % 2 + 1 - 1;
      int k = iz % 2 + 1 - 1, km1 = (iz + 1) % 2 + 1 - 1;
      int lm1 = (iz + 2) % 3 + 1 - 1, l = iz % 3 + 1 - 1, lp1 = (iz + 1) % 3 + 1 - 1;
      int nm1 = (iz + 3) % 4 + 1 - 1, n = iz % 4 + 1 - 1, np1 = (iz + 1) % 4 + 1 - 1, np2 = (iz + 2) % 4 + 1 - 1;
      if (iz == 1) {
        for (int i = -1; i <= 1; i++) expand_to(u.at(i + 1), UB(i));
        for (int i = -1; i <= 1; i++) expand_to(v.at(i + 1), VB(i));
        for (int i = -2; i <= 1; i++) expand_to(w.at(i + 1), WB(i));
        for (int i = -1; i <= 0; i++) {
          expand_to(e.at(i + 1), EB(i));
          for (size_t q = 0; q < pb; q++) EB(i)[q] = std::max(EB(i)[q], emin);
        }
      }
      expand_to(u.at(iz + 2), UB(2));
      expand_to(v.at(iz + 2), VB(2));
      expand_to(w.at(iz + 2), WB(2));
      expand_to(e.at(iz + 1), EB(1));
      for (size_t q = 0; q < pb; q++) EB(1)[q] = std::max(EB(1)[q], emin);
      // modify by the zeta part of the RK3 stage (comp1.f90:126-133)
      if (istage != 1) {
        T* uu = u.at(iz); T* vv = v.at(iz);
        const T* r1 = ru.at(iz); const T* r2 = rv.at(iz);
        for (size_t q = 0; q < ps; q++) { uu[q] = uu[q] - dtab2 * r1[q]; vv[q] = vv[q] - dtab2 * r2[q]; }
        if (iz != nnz) {
          T* ww = w.at(iz); T* ee = e.at(iz);
          const T* r3 = rw.at(iz); const T* r4 = re.at(iz);
          for (size_t q = 0; q < ps; q++) { ww[q] = ww[q] - dtab2 * r3[q]; ee[q] = ee[q] - dtab2 * r4[q]; }
        }
      }
      if (iz == 1) derivsbot(iz, lm1, l, nm1, n, np1);
      if (iz != nnz) derivs(iz, l, lp1, np2);
      {
        double s = 0;
        for (size_t q = 0; q < pb; q++) {
          T d = UX[n][q] + VY[n][q] + WZ[n][q];
          s += (double)(d * d);
        }
        M(3, iz) = (double)(T)(s * (double)xymb);
      }
      compadv1(iz);
      for (size_t q = 0; q < pb; q++) rubuf[q] = rubuf[q] + forcing;
      compsgs1(iz, j, jp1, k, km1, l, lm1, lp1, nm1, n, np1, np2);
      compsgs3(iz, j, jp1, k, km1, l, lm1, lp1, mnout, istage);
      compress_to(rvbuf.data(), rv.at(iz));
      compress_to(rubuf.data(), ru.at(iz));
      if (iz != nnz) compress_to(rwbuf.data(), rw.at(iz));
      if (iz != nnz) compress_to(rebuf.data(), re.at(iz));
      if (learned && learned_used) {
        for (size_t q = 0; q < ps; q++) { ru.at(iz)[q] += lru.at(iz)[q]; rv.at(iz)[q] += lrv.at(iz)[q]; }
        if (iz != nnz)
          for (size_t q = 0; q < ps; q++) rw.at(iz)[q] += lrw.at(iz)[q];
      }
      if (iz != nnz) {
        T* r = rw.at(iz);
        T mean = (T)(dsum(r, ps) * (double)xym);
        for (size_t q = 0; q < ps; q++) r[q] = r[q] - mean;
      }
      if (iz == nnz) {
        std::fill_n(rw.at(iz), ps, (T)0);
        std::fill_n(re.at(iz), ps, (T)0);
      }
      if (iz != nnz) {
        // shift the window (comp1.f90:179-184)
        std::rotate(ubuf.begin(), ubuf.begin() + 1, ubuf.end());
        std::rotate(vbuf.begin(), vbuf.begin() + 1, vbuf.end());
        std::rotate(wbuf.begin(), wbuf.begin() + 1, wbuf.end());
        std::rotate(ebuf.begin(), ebuf.begin() + 1, ebuf.end());
      }
    }
  }

  // comprhs (comprhs.f90:1-37)
  void comprhs() {
    std::vector<T> a(ps), f1(ps), f2(ps);
    for (int iz = 1; iz <= nnz; iz++) {
      const T* r1 = ru.at(iz); const T* uu = u.at(iz);
      for (size_t q = 0; q < ps; q++) a[q] = r1[q] + uu[q] * dtabm;
      sp.xderiv(a.data(), f1.data(), xk.data(), nnx, nny);
      const T* r2 = rv.at(iz); const T* vv = v.at(iz);
      for (size_t q = 0; q < ps; q++) a[q] = r2[q] + vv[q] * dtabm;
      sp.yderiv(a.data(), f2.data(), yk.data(), nnx, nny);
      T* pp = p.at(iz);
      for (int y = 0; y < nny; y++)
        for (int x = 0; x < nnx; x++) {
          size_t q = (size_t)y * nnx + x;
          T val;
          if (iz == 1)
            val = f1[q] + f2[q] + dzm * (w.at(iz)[q] * dtabm + rw.at(iz)[q]);
          else if (iz == nnz)
            val = f1[q] + f2[q] - dzm * (w.at(iz - 1)[q] * dtabm + rw.at(iz - 1)[q]);
          else
            val = f1[q] + f2[q] +
                  ((w.at(iz)[q] - w.at(iz - 1)[q]) * dtabm + rw.at(iz)[q] - rw.at(iz - 1)[q]) * dzm;
          pp[(size_t)y * (nnx + 2) + x] = val;
        }
    }
  }

  // press (press.F90:1-115), single process.
  void press() {
    T dzdz = dz * dz;
    int hs = nnx / 2 + 1;
    std::vector<std::vector<cplx<T>>> ph(nnz, std::vector<cplx<T>>((size_t)hs * nny));
    std::vector<T> tmp(ps);
    for (int iz = 1; iz <= nnz; iz++) {
      T* pp = p.at(iz);
      for (int y = 0; y < nny; y++)
        for (int x = 0; x < nnx; x++) tmp[(size_t)y * nnx + x] = pp[(size_t)y * (nnx + 2) + x];
      sp.r2c(tmp.data(), ph[iz - 1].data(), nnx, nny);
    }
    // kp = 1..nnx is kx = 0..nnx/2-1 (Re and Im share xk2); lp = 1..nny
#pragma omp parallel
    {
      std::vector<T> bd((size_t)nny * nnz * 4);
#pragma omp for
      for (int kx = 0; kx < nnx / 2; kx++) {
        for (int part = 0; part < 2; part++) {
          T* b = bd.data();
          T* d = b + (size_t)nny * nnz;
          T* a = d + (size_t)nny * nnz;
          T* r = a + (size_t)nny * nnz;
          T xkk2 = xk[kx] * xk[kx];
          for (int iz = 1; iz <= nnz; iz++)
            for (int lp = 0; lp < nny; lp++) {
              size_t q = (size_t)(iz - 1) * nny + lp;
              T k2 = xkk2 + yk[lp] * yk[lp];
              b[q] = 1;
              d[q] = -dzdz * k2 - ((iz == 1 || iz == nnz) ? (T)1 : (T)2);
              a[q] = 1;
              cplx<T> c = ph[iz - 1][(size_t)lp * hs + kx];
              r[q] = dzdz * (part == 0 ? c.real() : c.imag());
            }
          if (kx == 0)
            for (int iz = 1; iz <= nnz; iz++) {
              size_t q = (size_t)(iz - 1) * nny;
              b[q] = 0; d[q] = 1; a[q] = 0; r[q] = 0;
            }
          tridv(bd.data(), nny, nnz);
          for (int iz = 1; iz <= nnz; iz++)
            for (int lp = 0; lp < nny; lp++) {
              cplx<T>& c = ph[iz - 1][(size_t)lp * hs + kx];
              T val = r[(size_t)(iz - 1) * nny + lp];
              c = (part == 0) ? cplx<T>(val, c.imag()) : cplx<T>(c.real(), val);
            }
        }
      }
    }
    for (int iz = 1; iz <= nnz; iz++) {
      auto& z = ph[iz - 1];
      z[0] = 0;
      for (int lp = 0; lp < nny; lp++) z[(size_t)lp * hs + nnx / 2] = 0;
      for (int kx = 0; kx < hs; kx++) z[(size_t)(nny / 2) * hs + kx] = 0;
      sp.c2r(z.data(), tmp.data(), nnx, nny);
      T* pp = p.at(iz);
      for (int y = 0; y < nny; y++) {
        for (int x = 0; x < nnx; x++) pp[(size_t)y * (nnx + 2) + x] = tmp[(size_t)y * nnx + x];
        pp[(size_t)y * (nnx + 2) + nnx] = 0;
        pp[(size_t)y * (nnx + 2) + nnx + 1] = 0;
      }
    }
  }

  // comp2 (comp2.f90:1-45)
  void comp2() {
    std::vector<T> pl(ps), f(ps);
    for (int iz = 1; iz <= nnz; iz++) {
      const T* pp = p.at(iz);
      for (int y = 0; y < nny; y++)
        for (int x = 0; x < nnx; x++) pl[(size_t)y * nnx + x] = pp[(size_t)y * (nnx + 2) + x];
      sp.xderiv(pl.data(), f.data(), xk.data(), nnx, nny);
      T* r1 = ru.at(iz);
      for (size_t q = 0; q < ps; q++) r1[q] = r1[q] - f[q];
      sp.yderiv(pl.data(), f.data(), yk.data(), nnx, nny);
      T* r2 = rv.at(iz);
      for (size_t q = 0; q < ps; q++) r2[q] = r2[q] - f[q];
      if (iz != nnz) {
        T* r3 = rw.at(iz);
        const T* pu = p.at(iz + 1);
        for (int y = 0; y < nny; y++)
          for (int x = 0; x < nnx; x++) {
            size_t q = (size_t)y * nnx + x;
            r3[q] = r3[q] - (pu[(size_t)y * (nnx + 2) + x] - pp[(size_t)y * (nnx + 2) + x]) * dzm;
          }
        T mean = (T)(dsum(r3, ps) * (double)xym);
        for (size_t q = 0; q < ps; q++) r3[q] = r3[q] - mean;
      }
      T* uu = u.at(iz); T* vv = v.at(iz);
      for (size_t q = 0; q < ps; q++) { uu[q] = uu[q] + dtab1 * r1[q]; vv[q] = vv[q] + dtab1 * r2[q]; }
      if (iz != nnz) {
        T* ww = w.at(iz); T* ee = e.at(iz);
        const T* r3 = rw.at(iz); const T* r4 = re.at(iz);
        for (size_t q = 0; q < ps; q++) {
          ww[q] = ww[q] + dtab1 * r3[q];
          ee[q] = std::max(ee[q] + dtab1 * r4[q], emin);
        }
        T mean = (T)(dsum(ww, ps) * (double)xym);
        for (size_t q = 0; q < ps; q++) ww[q] = ww[q] - mean;
      }
    }
  }

  // One RK3 stage in the order of les.F90:254-285.
  void stage(int it, bool mnout, int istage) {
    static const T gama[3] = {(T)8 / (T)15, (T)5 / (T)12, (T)3 / (T)4};
    static const T zetas[3] = {(T)0, (T)17 / (T)60, (T)5 / (T)12};
    dtab1 = dt * gama[istage - 1];
    dtab2 = dt * zetas[istage - 1];
    dtabm = (T)1 / dtab1;
    lower();
    upper();
    comp1(it, mnout, istage);
    comprhs();
    press();
    comp2();
  }
  // One time step (les.F90:216, 254-285); stats afterwards when mnout.
  void step(int it, bool mnout) {
    xkmax = dz * dz / dt / (T)5;
    for (int s = 1; s <= 3; s++) stage(it, mnout, s);
    if (mnout || it == 0) compmn();
  }

  double avg(const T* x) { return dsum(x, ps) * (double)xym; }
  // compmn (compmn.F90:1-64) (outputs that the reference stores).
  void compmn() {
    auto R = [](double x) { return (double)(T)x; };
    for (int iz = 1; iz <= nnz; iz++) {
      M(4, iz) = R(avg(u.at(iz)));
      M(5, iz) = R(avg(v.at(iz)));
      M(6, iz) = R(avg(w.at(iz)));
      M(2, iz) = R(avg(e.at(iz)));
    }
    std::vector<T> ul(ps), vl(ps), t(ps);
    for (int iz = 1; iz <= nnz; iz++) {
      T um = (T)M(4, iz), vm = (T)M(5, iz);
      T um1 = (iz != nnz) ? (T)M(4, iz + 1) : (T)avg(u.at(iz + 1));
      T vm1 = (iz != nnz) ? (T)M(5, iz + 1) : (T)avg(v.at(iz + 1));
      const T* u0 = u.at(iz); const T* u1 = u.at(iz + 1);
      const T* v0 = v.at(iz); const T* v1 = v.at(iz + 1);
      const T* w0 = w.at(iz);
      for (size_t q = 0; q < ps; q++) {
        ul[q] = (T)0.5 * ((u0[q] - um) + (u1[q]) - um1);
        vl[q] = (T)0.5 * ((v0[q] - vm) + (v1[q]) - vm1);
      }
      for (size_t q = 0; q < ps; q++) t[q] = ul[q] * ul[q];
      M(7, iz) = R(avg(t.data()));
      for (size_t q = 0; q < ps; q++) t[q] = vl[q] * vl[q];
      M(8, iz) = R(avg(t.data()));
      for (size_t q = 0; q < ps; q++) t[q] = w0[q] * w0[q];
      M(9, iz) = R(avg(t.data()));
      for (size_t q = 0; q < ps; q++) t[q] = ul[q] * w0[q];
      M(10, iz) = R(avg(t.data()));
      for (size_t q = 0; q < ps; q++) t[q] = vl[q] * w0[q];
      M(11, iz) = R(avg(t.data()));
      for (size_t q = 0; q < ps; q++) t[q] = ul[q] * vl[q];
      M(12, iz) = R(avg(t.data()));
      M(1, iz) = R(((T)M(7, iz) + (T)M(8, iz) + (T)M(9, iz)) * (T)0.5);
    }
  }

  // spectra (spectra2.f90:1-70) of one small plane.
  void spectra(const T* f, double* zspecx, double* zspec2d) {
    int hs = nnx / 2 + 1;
    std::vector<cplx<T>> wv((size_t)hs * nny);
    sp.r2c(f, wv.data(), nnx, nny);
    std::vector<T> sx(hs, 0), s2(hs, 0);
    std::vector<int> m(hs, 0);
    for (int i = 1; i <= ncx; i++)
      for (int j = 1; j <= nny; j++) {
        cplx<T> c = wv[(size_t)(j - 1) * hs + (i - 1)];
        sx[i - 1] += (c * std::conj(c)).real();
      }
    for (int i = 2; i <= ncx - 1; i++) sx[i - 1] *= (T)2;
    for (int j = 1; j <= nny; j++)
      for (int i = 1; i <= ncx; i++) {
        T dist = std::sqrt(xk[i - 1] * xk[i - 1] + yk[j - 1] * yk[j - 1]);
        if (i == nnx / 2 + 1 && j == nny / 2 + 1) {
          dist = std::sqrt((pi * nnx / xl) * (pi * nnx / xl) + (pi * nny / yl) * (pi * nny / yl));
        } else {
          if (i == nnx / 2 + 1) dist = std::sqrt((pi * nnx / xl) * (pi * nnx / xl) + yk[j - 1] * yk[j - 1]);
          if (j == nny / 2 + 1) dist = std::sqrt(xk[i - 1] * xk[i - 1] + (pi * nny / yl) * (pi * nny / yl));
        }
        int iin = (int)std::lround(dist / ((T)2 * pi / xl)) + 1;
        if (iin > nnx / 2 + 1 || (i == 1 && j > nny / 2 + 1)) continue;
        cplx<T> c = wv[(size_t)(j - 1) * hs + (i - 1)];
        s2[iin - 1] += (c * std::conj(c)).real();
        m[iin - 1] += 1;
      }
    for (int i = 1; i <= ncx; i++) {
      int jj = i - 1;
      T denom;
      if (i == 1) denom = 1;
      else denom = (T)2 * (T)m[i - 1] / (pi * ((T)jj + (T)0.5) * ((T)jj + (T)0.5) - pi * ((T)jj - (T)0.5) * ((T)jj - (T)0.5));
      s2[i - 1] = (T)2 * s2[i - 1] / denom;
    }
    for (int i = 0; i < hs; i++) { zspecx[i] = sx[i]; zspec2d[i] = s2[i]; }
  }
};

// SplitMix64 (Steele, Lea & Flood, OOPSLA 2014): the n-th output of a stream
// seeded with s is mix(s + (n+1)*gamma).
static inline uint64_t splitmix64(uint64_t& s) {
  uint64_t z = (s += 0x9e3779b97f4a7c15ULL);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

}  // namespace orc

// ---------------------------------------------------------------------------
// extern "C" API used through ctypes by the tests (oracle/oracle.py).
// ---------------------------------------------------------------------------
using namespace orc;

struct OrcHandle {
  int real_bytes;
  std::unique_ptr<Les<double>> d;
  std::unique_ptr<Les<float>> f;
  std::string err;
};

template <class F>
static int guarded(OrcHandle* h, F&& fn) {
  try {
    fn();
    return 0;
  } catch (std::exception& ex) {
    if (h) h->err = ex.what();
    return 1;
  }
}

#define DISPATCH(h, ...)                  \
  do {                                    \
    if ((h)->real_bytes == 8) {           \
      auto& L = *(h)->d;                  \
      __VA_ARGS__;                        \
    } else {                              \
      auto& L = *(h)->f;                  \
      __VA_ARGS__;                        \
    }                                     \
  } while (0)

template <class T, class S>
static void copy_levels(Levels<T>& f, const S* src, int nnx, int nny, int nnz, int stride_x) {
  for (int iz = 1; iz <= nnz; iz++) {
    T* dst = f.at(iz);
    for (int y = 0; y < nny; y++)
      for (int x = 0; x < nnx; x++)
        dst[(size_t)y * stride_x + x] = (T)src[((size_t)(iz - 1) * nny + y) * nnx + x];
  }
}
template <class T, class S>
static void read_levels(Levels<T>& f, S* dst, int nnx, int nny, int nnz, int stride_x) {
  for (int iz = 1; iz <= nnz; iz++) {
    const T* src = f.at(iz);
    for (int y = 0; y < nny; y++)
      for (int x = 0; x < nnx; x++)
        dst[((size_t)(iz - 1) * nny + y) * nnx + x] = (S)src[(size_t)y * stride_x + x];
  }
}

extern "C" {

void* orc_create(const les_config* cfg, int real_bytes) {
  OrcHandle* h = new OrcHandle();
  h->real_bytes = real_bytes;
  try {
    if (real_bytes == 8) h->d.reset(new Les<double>(*cfg));
    else h->f.reset(new Les<float>(*cfg));
  } catch (std::exception& ex) {
    delete h;
    return nullptr;
  }
  return h;
}
void orc_free(void* hp) { delete (OrcHandle*)hp; }

// Learned closure: attach the FP64 network (NULL params detach).
int orc_set_mlp(void* hp, const double* params, const double* norm, double re_tau, int bf16) {
  OrcHandle* h = (OrcHandle*)hp;
  return guarded(h, [&] { DISPATCH(h, L.set_mlp(params, norm, re_tau, bf16 != 0)); });
}
// Stress divergence of the last learned stage, (nnx, nny, nnz) FP64 each.
int orc_get_learned(void* hp, double* lru, double* lrv, double* lrw) {
  OrcHandle* h = (OrcHandle*)hp;
  return guarded(h, [&] {
    DISPATCH(h, {
      if (!L.learned) throw std::runtime_error("no network attached");
      read_levels(L.lru, lru, L.nnx, L.nny, L.nnz, L.nnx);
      read_levels(L.lrv, lrv, L.nnx, L.nny, L.nnz, L.nnx);
      read_levels(L.lrw, lrw, L.nnx, L.nny, L.nnz, L.nnx);
    });
  });
}
void orc_learned_status(void* hp, int* used, double* dissipation) {
  OrcHandle* h = (OrcHandle*)hp;
  DISPATCH(h, { if (used) *used = L.learned_used; if (dissipation) *dissipation = L.learned_dissip; });
}
// Raw network mean dissipation (before the backscatter projection) of the
// last learned stage.
double orc_learned_raw(void* hp) {
  OrcHandle* h = (OrcHandle*)hp;
  double d = 0.0;
  DISPATCH(h, { d = L.learned_dissip_raw; });
  return d;
}
// Reference (Smagorinsky) mean dissipation of the last learned stage.
double orc_learned_reference(void* hp) {
  OrcHandle* h = (OrcHandle*)hp;
  double d = 0.0;
  DISPATCH(h, { d = L.learned_dissip_r; });
  return d;
}
// Factor of the dissipation test (<= 0: sign test only).
void orc_set_learned_guard(void* hp, double ratio) {
  OrcHandle* h = (OrcHandle*)hp;
  DISPATCH(h, { L.learned_guard = ratio; });
}
const char* orc_error(void* hp) { return ((OrcHandle*)hp)->err.c_str(); }

// Fields as FP64 arrays of (nnx, nny, nnz), levels 1..nnz.
int orc_set_fields(void* hp, const double* u, const double* v, const double* w, const double* e,
                   const double* p) {
  OrcHandle* h = (OrcHandle*)hp;
  return guarded(h, [&] {
    DISPATCH(h, {
      if (u) copy_levels(L.u, u, L.nnx, L.nny, L.nnz, L.nnx);
      if (v) copy_levels(L.v, v, L.nnx, L.nny, L.nnz, L.nnx);
      if (w) copy_levels(L.w, w, L.nnx, L.nny, L.nnz, L.nnx);
      if (e) copy_levels(L.e, e, L.nnx, L.nny, L.nnz, L.nnx);
      if (p) copy_levels(L.p, p, L.nnx, L.nny, L.nnz, L.nnx + 2);
    });
  });
}
int orc_get_fields(void* hp, double* u, double* v, double* w, double* e, double* p) {
  OrcHandle* h = (OrcHandle*)hp;
  return guarded(h, [&] {
    DISPATCH(h, {
      if (u) read_levels(L.u, u, L.nnx, L.nny, L.nnz, L.nnx);
      if (v) read_levels(L.v, v, L.nnx, L.nny, L.nnz, L.nnx);
      if (w) read_levels(L.w, w, L.nnx, L.nny, L.nnz, L.nnx);
      if (e) read_levels(L.e, e, L.nnx, L.nny, L.nnz, L.nnx);
      if (p) read_levels(L.p, p, L.nnx, L.nny, L.nnz, L.nnx + 2);
    });
  });
}
int orc_set_tendencies(void* hp, const double* ru, const double* rv, const double* rw, const double* re) {
  OrcHandle* h = (OrcHandle*)hp;
  return guarded(h, [&] {
    DISPATCH(h, {
      if (ru) copy_levels(L.ru, ru, L.nnx, L.nny, L.nnz, L.nnx);
      if (rv) copy_levels(L.rv, rv, L.nnx, L.nny, L.nnz, L.nnx);
      if (rw) copy_levels(L.rw, rw, L.nnx, L.nny, L.nnz, L.nnx);
      if (re) copy_levels(L.re, re, L.nnx, L.nny, L.nnz, L.nnx);
    });
  });
}
int orc_get_tendencies(void* hp, double* ru, double* rv, double* rw, double* re) {
  OrcHandle* h = (OrcHandle*)hp;
  return guarded(h, [&] {
    DISPATCH(h, {
      if (ru) read_levels(L.ru, ru, L.nnx, L.nny, L.nnz, L.nnx);
      if (rv) read_levels(L.rv, rv, L.nnx, L.nny, L.nnz, L.nnx);
      if (rw) read_levels(L.rw, rw, L.nnx, L.nny, L.nnz, L.nnx);
      if (re) read_levels(L.re, re, L.nnx, L.nny, L.nnz, L.nnx);
    });
  });
}
// les.F90:185-190: deal() every level of u, v, w, e.
int orc_deal_fields(void* hp) {
  OrcHandle* h = (OrcHandle*)hp;
  return guarded(h, [&] {
    DISPATCH(h, {
      for (int iz = 1; iz <= L.nnz; iz++) {
        L.sp.deal(L.u.at(iz), L.nnx, L.nny);
        L.sp.deal(L.v.at(iz), L.nnx, L.nny);
        L.sp.deal(L.w.at(iz), L.nnx, L.nny);
        L.sp.deal(L.e.at(iz), L.nnx, L.nny);
      }
    });
  });
}
int orc_stage(void* hp, int it, int mnout, int istage) {
  OrcHandle* h = (OrcHandle*)hp;
  return guarded(h, [&] {
    DISPATCH(h, {
      L.xkmax = L.dz * L.dz / L.dt / (decltype(L.dt))5;
      L.stage(it, mnout != 0, istage);
    });
  });
}
int orc_step(void* hp, int it0, int nsteps, int mnout_every) {
  OrcHandle* h = (OrcHandle*)hp;
  return guarded(h, [&] {
    DISPATCH(h, {
      for (int s = 0; s < nsteps; s++) {
        int it = it0 + s;
        bool mn = (it == 0) || (mnout_every > 0 && (it % mnout_every) == 0);
        L.step(it, mn);
      }
    });
  });
}
// meanbuf (19 x nnz) and scalars (utau, utau_s, dudt, dvdt, utau_lower).
int orc_stats(void* hp, double* meanbuf, double* scalars) {
  OrcHandle* h = (OrcHandle*)hp;
  return guarded(h, [&] {
    DISPATCH(h, {
      if (meanbuf) std::copy(L.meanbuf.begin(), L.meanbuf.end(), meanbuf);
      if (scalars) {
        scalars[0] = L.utau; scalars[1] = L.utau_s; scalars[2] = L.dudt; scalars[3] = L.dvdt;
        scalars[4] = L.utau_lower;
      }
    });
  });
}
int orc_compmn(void* hp) {
  OrcHandle* h = (OrcHandle*)hp;
  return guarded(h, [&] { DISPATCH(h, { L.compmn(); }); });
}
int orc_spectra(void* hp, int field, int iz, double* zspecx, double* zspec2d) {
  OrcHandle* h = (OrcHandle*)hp;
  return guarded(h, [&] {
    DISPATCH(h, {
      auto* f = field == 0 ? &L.u : field == 1 ? &L.v : field == 2 ? &L.w : &L.e;
      L.spectra(f->at(iz), zspecx, zspec2d);
    });
  });
}

// The synthetic initial condition (documented recipe; replaces initvel):
// parabolic mean, SplitMix64 uniform perturbations (seed+0,1,2 for u,v,w,
// column-major order), e = e0, deal, then one projection with dtab1 = 1.
int orc_make_ic(void* hp, unsigned long long seed, double ub, double amp, double utau, double e0) {
  OrcHandle* h = (OrcHandle*)hp;
  return guarded(h, [&] {
    DISPATCH(h, {
      using T = std::remove_reference_t<decltype(L.dt)>;
      int nx = L.nnx, ny = L.nny, nz = L.nnz;
      T hh = L.zl / (T)2;
      Levels<T>* fl[3] = {&L.u, &L.v, &L.w};
      for (int f = 0; f < 3; f++) {
        uint64_t s = (uint64_t)seed + (uint64_t)f;
        for (int iz = 1; iz <= nz; iz++) {
          double zm = ((double)iz - 0.5) * (double)L.dz;
          double mean = 0.0;
          if (f == 0) {
            double eta = (zm - (double)hh) / (double)hh;
            mean = 1.5 * ub * (1.0 - eta * eta);
          }
          T* pl = fl[f]->at(iz);
          for (int y = 0; y < ny; y++)
            for (int x = 0; x < nx; x++) {
              uint64_t r = splitmix64(s);
              double u01 = (double)(r >> 11) * (1.0 / 9007199254740992.0);
              pl[(size_t)y * nx + x] = (T)(mean + (2.0 * u01 - 1.0) * amp * utau);
            }
        }
      }
      std::fill_n(L.w.at(nz), L.ps, (T)0);
      for (int iz = 1; iz <= nz; iz++) std::fill_n(L.e.at(iz), L.ps, (T)e0);
      std::fill(L.p.data.begin(), L.p.data.end(), (T)0);
      for (int iz = 1; iz <= nz; iz++) {
        L.sp.deal(L.u.at(iz), nx, ny);
        L.sp.deal(L.v.at(iz), nx, ny);
        L.sp.deal(L.w.at(iz), nx, ny);
        L.sp.deal(L.e.at(iz), nx, ny);
      }
      std::fill(L.ru.data.begin(), L.ru.data.end(), (T)0);
      std::fill(L.rv.data.begin(), L.rv.data.end(), (T)0);
      std::fill(L.rw.data.begin(), L.rw.data.end(), (T)0);
      std::fill(L.re.data.begin(), L.re.data.end(), (T)0);
      L.lower();
      L.upper();
      L.dtab1 = 1; L.dtabm = 1;
      L.comprhs();
      L.press();
      L.comp2();
      std::fill(L.ru.data.begin(), L.ru.data.end(), (T)0);
      std::fill(L.rv.data.begin(), L.rv.data.end(), (T)0);
      std::fill(L.rw.data.begin(), L.rw.data.end(), (T)0);
      std::fill(L.re.data.begin(), L.re.data.end(), (T)0);
      std::fill(L.p.data.begin(), L.p.data.end(), (T)0);
    });
  });
}

// Advective CFL time step (les.F90:205-208).
double orc_cfl_dt(void* hp, double cfl) {
  OrcHandle* h = (OrcHandle*)hp;
  double out = 0;
  DISPATCH(h, {
    double um = 0, vm = 0, wm = 0;
    for (int iz = 1; iz <= L.nnz; iz++)
      for (size_t q = 0; q < L.ps; q++) {
        um = std::max(um, std::fabs((double)L.u.at(iz)[q]));
        vm = std::max(vm, std::fabs((double)L.v.at(iz)[q]));
        wm = std::max(wm, std::fabs((double)L.w.at(iz)[q]));
      }
    double ucfl = um * L.nnxb / (double)L.xl, vcfl = vm * L.nnyb / (double)L.yl, wcfl = wm / (double)L.dz;
    out = cfl / std::max(std::max(ucfl, vcfl), std::max(wcfl, 0.5 / (double)L.dz));
  });
  return out;
}

void orc_set_dt(void* hp, double dt) {
  OrcHandle* h = (OrcHandle*)hp;
  DISPATCH(h, { L.dt = (decltype(L.dt))dt; });
}

// --- operator-level restatements for unit tests (FP64) ---
static Spectral<double>& spec64() {
  static Spectral<double> s;
  return s;
}
static void wavenumbers(int n, double len, std::vector<double>& k) {
  double pi = 4.0 * std::atan(1.0);
  k.resize(n);
  for (int i = 1; i <= n; i++) {
    k[i - 1] = (double)(i - 1) * 2.0 * pi / len;
    if (i > n / 2 + 1) k[i - 1] = -(double)(n - i + 1) * 2.0 * pi / len;
  }
}
void orc_xderiv(const double* a, double* o, int n1, int n2, double len) {
  std::vector<double> k;
  wavenumbers(n1, len, k);
  spec64().xderiv(a, o, k.data(), n1, n2);
}
void orc_yderiv(const double* a, double* o, int n1, int n2, double len) {
  std::vector<double> k;
  wavenumbers(n2, len, k);
  spec64().yderiv(a, o, k.data(), n1, n2);
}
void orc_expand(const double* s, double* b, int nx, int ny) { spec64().expand(s, b, nx, ny); }
void orc_compress(const double* b, double* s, int nx, int ny) { spec64().compress(b, s, nx, ny); }
void orc_deal(double* x, int nx, int ny) { spec64().deal(x, nx, ny); }
// ffthrz forward: out is complex [ny][nx/2+1] interleaved (re, im).
void orc_r2c(const double* in, double* out, int n1, int n2) {
  spec64().r2c(in, (std::complex<double>*)out, n1, n2);
}
void orc_c2r(const double* in, double* out, int n1, int n2) {
  spec64().c2r((const std::complex<double>*)in, out, n1, n2);
}
void orc_dft(double* x, int n, int sign) {
  Dft<double> d(n);
  std::vector<std::complex<double>> s(n);
  d.run((std::complex<double>*)x, s.data(), sign);
}
void orc_tridv(double* bdar, int ny, int n) { tridv(bdar, ny, n); }
int orc_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"

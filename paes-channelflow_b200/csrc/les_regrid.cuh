// les_regrid.cuh -- spectral regridding of the state onto another grid, the
// device form of the reference's redim.f90 (interpol redim.f90:202-269 and
// subroutine redim redim.f90:277-318) followed by the dealiasing a restarted
// run applies (les.F90:185-190).
//
// The state is spectral in x-y (u^ = FFT2(u) / (nx ny), kx < nx/2), so the
// x-y part of redim is a copy of the modes both grids hold,
//   kx < min(nx_old, nx_new) / 2,  |ky| < min(ny_old, ny_new) / 2,
// and zero elsewhere: redim zeroes the old Nyquist modes and the restart's
// deal zeroes the new ones.  The z interpolation is linear, so it is applied
// to the modes level by level with the weights of the host table (RegridLevel),
// which replays redim's walk over the old levels.  e is physical: its planes
// are interpolated in z, transformed on the old grid, copied, transformed
// back on the new grid, clamped to [1e-10, plane max of the interpolated e]
// (redim.f90:262-263) and dealt.
#pragma once
#include "les_kernels.cuh"

namespace les {

// One new level of redim's z interpolation: centre fields B + (B - A) * c
// from old levels a, b; face fields F1 + (F1 - F0) * d from old levels f0,
// f1 (1-based; 0 = the wall: w = 0, e = e(1)).
struct RegridLevel {
  int a, b, f0, f1;
  double c, d;
};

// Host replay of interpol's walk (redim.f90:202-269) for nznew new levels.
inline std::vector<RegridLevel> regrid_table(int nzold, int nznew, double zl) {
  std::vector<RegridLevel> t(nznew);
  const double dzold = zl / nzold, dznew = zl / nznew;
  int izo = 2;
  double zhold = izo * dzold - 0.5 * dzold;
  double zfold = (izo - 1) * dzold;
  for (int izn = 1; izn <= nznew; izn++) {
    const double zh = izn * dznew - 0.5 * dznew;
    const double zf = izn * dznew;
    while (zhold < zh && izo < nzold) {
      izo++;
      zhold = izo * dzold - 0.5 * dzold;
      zfold = (izo - 1) * dzold;
    }
    RegridLevel& r = t[izn - 1];
    r.a = izo - 1;
    r.b = izo;
    r.c = (zh - zhold) / dzold;
    if (zf <= zfold) { r.f0 = izo - 2; r.f1 = izo - 1; r.d = (zf - zfold) / dzold; }
    else { r.f0 = izo - 1; r.f1 = izo; r.d = (zf - (zfold + dzold)) / dzold; }
  }
  return t;
}

enum RegridMode { kRegridCentre = 0, kRegridFace = 1, kRegridCopy = 2 };

// New spectral levels [z][ky][kx] from old ones: mode copy between the grids
// with the z interpolation of `mode` (kRegridCopy: new level n = old level n).
// Grid (cdiv(KXd * NYd, 256), NZd).
template <class E, class R>
__global__ void k_regrid_spec(const E* __restrict__ src, E* __restrict__ dst, const RegridLevel* __restrict__ tab,
                              int mode, int KXs, int NYs, int KXd, int NYd) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = blockIdx.y;
  if (m >= KXd * NYd) return;
  const int kyd = m / KXd, kx = m - kyd * KXd;
  const int ky = kyd <= NYd / 2 ? kyd : kyd - NYd;
  const int kxm = KXs < KXd ? KXs : KXd;
  const int kym = (NYs < NYd ? NYs : NYd) / 2;
  E v;
  v.x = 0;
  v.y = 0;
  if (kx < kxm && ky < kym && ky > -kym) {
    const size_t nms = (size_t)KXs * NYs;
    const size_t ms = (size_t)(ky >= 0 ? ky : ky + NYs) * KXs + kx;
    auto L = [&](int k) -> E {  // old level k (1-based); 0 = the wall (w = 0)
      if (k < 1) { E z; z.x = 0; z.y = 0; return z; }
      return src[(size_t)(k - 1) * nms + ms];
    };
    if (mode == kRegridCopy) {
      v = L(n + 1);
    } else {
      const RegridLevel t = tab[n];
      const E A = L(mode == kRegridCentre ? t.a : t.f0), B = L(mode == kRegridCentre ? t.b : t.f1);
      const R w = (R)(mode == kRegridCentre ? t.c : t.d);
      v.x = B.x + (B.x - A.x) * w;
      v.y = B.y + (B.y - A.y) * w;
    }
  }
  dst[(size_t)n * KXd * NYd + m] = v;
}

// FP64 mean profiles (the kx = ky = 0 shadows) of centre fields.
static __global__ void k_regrid_mean(const double* __restrict__ src, double* __restrict__ dst,
                                     const RegridLevel* __restrict__ tab, int NZd) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= NZd) return;
  const RegridLevel t = tab[n];
  const double A = src[t.a - 1], B = src[t.b - 1];
  dst[n] = B + (B - A) * t.c;
}

// Interpolated e planes on the old grid for new levels n0 .. n0+cnt-1:
// e levels k = 1..NZs at e1 + (k-1)*P; level 0 reads e(1).  Grid
// (cdiv(P, 256), cnt).
template <class T>
__global__ void k_regrid_ez(const T* __restrict__ e1, T* __restrict__ out, const RegridLevel* __restrict__ tab,
                            int n0, size_t P) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P) return;
  const RegridLevel t = tab[n0 + blockIdx.y];
  const T F0 = e1[(size_t)((t.f0 < 1 ? 1 : t.f0) - 1) * P + i];
  const T F1 = e1[(size_t)(t.f1 - 1) * P + i];
  out[(size_t)blockIdx.y * P + i] = F1 + (F1 - F0) * (T)t.d;
}

// Maximum of each of `cnt` planes of P values (one block per plane).
template <class T>
__global__ void __launch_bounds__(256) k_plane_max(const T* __restrict__ a, size_t P, double* __restrict__ out) {
  __shared__ double red[256];
  const T* p = a + (size_t)blockIdx.x * P;
  double m = -1.0e300;
  for (size_t i = threadIdx.x; i < P; i += 256) m = fmax(m, (double)p[i]);
  red[threadIdx.x] = m;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = red[0];
}

// e = min(emax(level), max(e, 1e-10)) on cnt planes (redim.f90:262-263).
// Grid (cdiv(P, 256), cnt).
template <class T>
__global__ void k_regrid_eclamp(T* __restrict__ e, const double* __restrict__ emax, size_t P) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P) return;
  T& v = e[(size_t)blockIdx.y * P + i];
  const T lo = (T)1e-10, hi = (T)emax[blockIdx.y];
  const T c = v > lo ? v : lo;
  v = hi < c ? hi : c;
}

}  // namespace les

// les_fused.cuh -- the padded-grid part of comp1 as one kernel per (padded
// y row, z chunk): inverse x transforms of the mixed arrays, the pointwise
// advection / SGS fluxes, and the forward x transforms with -d/dx folded in,
// without ever writing the padded physical fields to HBM.
//
// The CTA walks up its z chunk keeping a window of physical rows in shared
// memory (levels z-1, z, z+1 of U, V, W, E, packed as complex rows U+iV and
// W+iE), exactly the sliding window of comp1.f90:91-121 / 179-184 but along
// one row of the padded plane.  Six teams (one warp each) each own one
// transform per phase:
//   phase I   (inverse)  w0: U+iV (z+1)   w1: W+iE (z+1)   w2: UX+iVX (z)
//                        w3: UY+iVY (z)   w4: WX+iWY (z)   w5: EX+iEY (le)
//             (when the learned closure supplies the interior momentum
//             stresses only ux and vy are needed, for the divergence
//             diagnostic: w2 transforms UX+iVY, w3 and w4 idle)
//   phase II  (pointwise, all threads) the eleven flux rows of k_flux
//   phase III (forward)  w0: A+iPu  w1: B+iPv  w2: C+iG  w3: D+iPw
//                        w4: F+iPe  w5: H
// Transforms are warp-synchronous four-step FFTs (lanes = N2 in pass A,
// N1 in pass B, __syncwarp between passes) or, for rows whose second
// factor exceeds 24 (768), three Stockham passes synchronised by the team's
// named barrier; block barriers only separate the three phases.
#pragma once
#include "les_kernels.cuh"

namespace les {

// XOR swizzle of natural-layout indices in the fused kernel's buffers:
// within each 128-byte block the low bits are XORed with the block index, so
// strided butterfly writes (stride R elements) land in distinct banks.  A
// bijection on [0, N) when N is a multiple of the block length.
template <class T, int N> struct Swz {
  static constexpr int SHIFT = (sizeof(cx<T>) == 16) ? 3 : 4;
  static constexpr int MASK = (N % (1 << SHIFT) == 0) ? ((1 << SHIFT) - 1) : 0;
  static __device__ __forceinline__ int f(int a) { return a ^ ((a >> SHIFT) & MASK); }
};

// Warp-level four-step transform of one length-N sequence in `buf`
// (smem_fft_elems<N,false>(1) elements).  IN: load(n) from global memory or,
// with IN_SMEM, buf in natural layout.  OUT: buf in natural layout.
template <int N, int S, bool IN_SMEM, class T, class LoadF>
__device__ __forceinline__ void warp_fft(cx<T>* buf, const cx<T>* twn, LoadF load) {
  constexpr int N1 = Split<N>::N1;
  constexpr int N2 = Split<N>::N2;
  constexpr int LD = N2 + 1;
  static_assert(N1 <= 32 && N2 <= 32, "warp transform needs N1, N2 <= 32");
  const int lane = threadIdx.x & 31;
  {
    cx<T> v[N1];
    if (lane < N2) {
#pragma unroll
      for (int n1 = 0; n1 < N1; n1++) {
        if constexpr (IN_SMEM) v[n1] = buf[Swz<T, N>::f(lane + N2 * n1)];
        else v[n1] = load(lane + N2 * n1);
      }
    }
    if (IN_SMEM) __syncwarp();
    if (lane < N2) {
      Dft<N1, S, T>::run(v);
#pragma unroll
      for (int k1 = 0; k1 < N1; k1++) {
        cx<T> w = twn[k1 * N2 + lane];  // [k1][n2] layout: consecutive lanes, no bank conflicts
        if (S > 0) w.y = -w.y;
        buf[k1 * LD + lane] = (k1 == 0) ? v[k1] : cmul(v[k1], w);
      }
    }
  }
  __syncwarp();
  {
    cx<T> v[N2];
    if (lane < N1) {
#pragma unroll
      for (int n2 = 0; n2 < N2; n2++) v[n2] = buf[lane * LD + n2];
    }
    __syncwarp();
    if (lane < N1) {
      Dft<N2, S, T>::run(v);
#pragma unroll
      for (int k2 = 0; k2 < N2; k2++) buf[Swz<T, N>::f(lane + N1 * k2)] = v[k2];
    }
  }
  __syncwarp();
}

// Team Stockham transform: TEAM threads (a multiple of 32) share one
// transform and synchronise with a named barrier `bar` (1..15), so several
// teams run independent transforms inside one CTA.  In place in buf
// (natural layout, N elements); each pass holds ceil(N/R/TEAM)*R values
// per thread.
template <int TEAM>
__device__ __forceinline__ void team_sync(int bar) {
  if (TEAM == 32) __syncwarp();
  else asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(TEAM) : "memory");
}
template <int N, int R, int NS, int S, bool FIRST, int TEAM, class T, class LoadF>
__device__ __forceinline__ void team_stockham_pass(cx<T>* buf, const cx<T>* twn, LoadF load, int tl, int bar) {
  constexpr int M = N / R;
  constexpr int J = (M + TEAM - 1) / TEAM;
  cx<T> v[J][R];
#pragma unroll
  for (int jj = 0; jj < J; jj++) {
    const int j = tl + TEAM * jj;
    if (j < M) {
      const int k = j % NS;
#pragma unroll
      for (int r = 0; r < R; r++) {
        cx<T> x;
        if constexpr (FIRST) x = load(j + r * M);
        else x = buf[Swz<T, N>::f(j + r * M)];
        if (NS > 1 && r > 0) {
          cx<T> w = twn[r * NS + k];  // this pass's table, [r][k] layout
          if (S > 0) w.y = -w.y;
          x = cmul(x, w);
        }
        v[jj][r] = x;
      }
    }
  }
  team_sync<TEAM>(bar);
#pragma unroll
  for (int jj = 0; jj < J; jj++) {
    const int j = tl + TEAM * jj;
    if (j < M) {
      const int k = j % NS;
      Dft<R, S, T>::run(v[jj]);
      const int base = (j / NS) * NS * R + k;
#pragma unroll
      for (int r = 0; r < R; r++) buf[Swz<T, N>::f(base + r * NS)] = v[jj][r];
    }
  }
  team_sync<TEAM>(bar);
}
template <int N> struct Radix3;
template <> struct Radix3<24> { static constexpr int R1 = 2, R2 = 2, R3 = 6; };
template <> struct Radix3<48> { static constexpr int R1 = 4, R2 = 2, R3 = 6; };
template <> struct Radix3<96> { static constexpr int R1 = 4, R2 = 4, R3 = 6; };
template <> struct Radix3<144> { static constexpr int R1 = 4, R2 = 6, R3 = 6; };
template <> struct Radix3<192> { static constexpr int R1 = 8, R2 = 4, R3 = 6; };
template <> struct Radix3<288> { static constexpr int R1 = 8, R2 = 6, R3 = 6; };
template <> struct Radix3<384> { static constexpr int R1 = 8, R2 = 8, R3 = 6; };
template <> struct Radix3<576> { static constexpr int R1 = 8, R2 = 6, R3 = 12; };
template <> struct Radix3<768> { static constexpr int R1 = 8, R2 = 8, R3 = 12; };
template <int N, int S, bool IN_SMEM, int TEAM, class T, class LoadF>
__device__ __forceinline__ void team_fft(cx<T>* buf, const cx<T>* twn, LoadF load, int tl, int bar) {
  constexpr int R1 = Radix3<N>::R1, R2 = Radix3<N>::R2, R3 = Radix3<N>::R3;
  static_assert(R1 * R2 * R3 == N, "radices must multiply to N");
  // twn: the per-pass tables of stockham_twiddles (pass 2 at 0, pass 3 at R1*R2)
  team_stockham_pass<N, R1, 1, S, !IN_SMEM, TEAM, T>(buf, twn, load, tl, bar);
  team_stockham_pass<N, R2, R1, S, false, TEAM, T>(buf, twn, load, tl, bar);
  team_stockham_pass<N, R3, R1 * R2, S, false, TEAM, T>(buf, twn + R1 * R2, load, tl, bar);
}
// Entries of the per-pass twiddle tables used by team_fft: pass 2 (NS = R1,
// radix R2) then pass 3 (NS = R1*R2, radix R3), each as [r][k] with entry
// W_N^(k*r*N/(NS*R)).  Returns the length of the table (R1*R2 + R1*R2*R3).
template <int N> __host__ __device__ constexpr int stockham_twiddle_len() {
  return Radix3<N>::R1 * Radix3<N>::R2 + N;
}
// exponent (in units of 2 pi / N) of entry i of the table
template <int N> __device__ __forceinline__ int stockham_twiddle_exp(int i) {
  constexpr int R1 = Radix3<N>::R1, R2 = Radix3<N>::R2, R3 = Radix3<N>::R3;
  if (i < R1 * R2) {
    const int r = i / R1, k = i % R1;  // NS = R1, R = R2
    return k * r * (N / (R1 * R2));
  }
  i -= R1 * R2;
  const int r = i / (R1 * R2), k = i % (R1 * R2);  // NS = R1*R2, R = R3
  return k * r * (N / (R1 * R2 * R3));
}

// Transform used by the fused kernel for a length: the two-pass warp form
// unless its N2-point register DFT has 24 points or more (288, 384, 576,
// 768), then the three-pass Stockham form (radices <= 12): the 24- and
// 32-point register DFTs spill, and on B200 the three passes ran 6-31%
// faster at 288-576.
template <int N, class T> struct FusedPlan {
  static constexpr bool three = (Split<N>::N2 >= 24);
  static constexpr int BUF = three ? N : smem_fft_elems<N, false>(1);
};
// One transform by a team of TEAM threads (tl = index in the team, bar = the
// team's named barrier; the two-pass warp form needs TEAM = 32).
template <int N, int S, bool IN_SMEM, int TEAM, class T, class LoadF>
__device__ __forceinline__ void fused_fft(cx<T>* buf, const cx<T>* twn, LoadF load, int tl, int bar) {
  if constexpr (FusedPlan<N, T>::three) {
    team_fft<N, S, IN_SMEM, TEAM, T>(buf, twn, load, tl, bar);
  } else {
    static_assert(TEAM == 32, "the two-pass transform is warp-synchronous");
    warp_fft<N, S, IN_SMEM, T>(buf, twn, load);
  }
}

struct FusedArgs {
  // mixed inputs (x-spectral, y physical on the padded grid): Um, UYm, Vm,
  // VYm, Wm, WYm, Em, EYm; outputs Xu1, Xu2, Xv1, Xv2, Xw1, Xw2, Xe1, Xe2
  Ptr8 in, out;
  const void* dEX;       // clip corrections (padded physical, levels 1..nnz-1)
  const void* dEY;
  const int* clipflag;   // per level 1..nnz-1 (index z-1)
  const WallParams* wp;
  double* divpart;  // [level][y] partial sums of divz, one writer each
  double* sgspart;  // [level][y][6] partial SGS means (stage 1 with mnout)
  // learned closure: when lflag is set and *lflag != 0 the interior momentum
  // stresses are left to the network (the wall-model rows stay)
  const int* lflag;
  int zchunk;
};

template <int NSX> struct FusedCfg {
  static constexpr int MX = 3 * NSX / 2;
  static constexpr int NBUF = 11;  // 6 level slots (3 levels x 2), 4 work buffers, 1 carried tuw/tvw
  // threads per transform: one warp.  (Two warps for the FP64 768-point
  // plan double the resident warps but cap the 384-thread block at 168
  // registers, which spills; on B200 that ran 9% slower.)
  template <class T> static constexpr int team() { return 32; }
  template <class T> static constexpr int threads() { return 6 * team<T>(); }
  template <class T> static constexpr int buf() { return FusedPlan<MX, T>::BUF; }
  // buffers + the twiddle table of length MX staged in shared memory
  template <class T> static constexpr size_t smem() {
    return ((size_t)NBUF * buf<T>() + MX + 64) * sizeof(cx<T>);
  }
};

// Square root of the TKE in the FP32 form: the hardware approximation
// (sqrt.approx.f32) instead of the correctly rounded sequence, 3% of the
// fused kernel (the mixed-form tolerances against the oracle bound its
// effect); FP64 keeps sqrt().
template <class T> __device__ __forceinline__ T tke_sqrt(T e) { return sqrt(e); }
template <> __device__ __forceinline__ float tke_sqrt<float>(float e) {
  float r;
  asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(e));
  return r;
}

template <class T, int NSX>
__global__ void __launch_bounds__(FusedCfg<NSX>::template threads<T>(), (sizeof(T) == 4) ? 2 : 1)
k_row_fused(FusedArgs f, StageArgs a, const cx<T>* __restrict__ tw) {
  constexpr int MX = 3 * NSX / 2;
  constexpr int KX = NSX / 2;
  constexpr int BUF = FusedCfg<NSX>::template buf<T>();
  constexpr int TEAM = FusedCfg<NSX>::template team<T>();
  extern __shared__ __align__(16) unsigned char smraw[];
  cx<T>* sm = reinterpret_cast<cx<T>*>(smraw);
  // twiddles staged once per CTA in the layout each transform reads with
  // consecutive lanes: [k1][n2] (two-pass) or the per-pass [r][k] tables
  // (three-pass Stockham)
  cx<T>* tws = sm + (size_t)11 * BUF;
  {
    const cx<T>* twg = tw + tw_off(MX);
    if constexpr (FusedPlan<MX, T>::three) {
      for (int i = threadIdx.x; i < stockham_twiddle_len<MX>(); i += blockDim.x)
        tws[i] = twg[stockham_twiddle_exp<MX>(i) % MX];
    } else {
      constexpr int N1 = Split<MX>::N1, N2 = Split<MX>::N2;
      for (int i = threadIdx.x; i < N1 * N2; i += blockDim.x) tws[i] = twg[(i / N2) * (i % N2)];
    }
  }
  __syncthreads();
  cx<T>* work[6];
#pragma unroll
  for (int i = 0; i < 4; i++) work[i] = sm + (size_t)(6 + i) * BUF;
  cx<T>* carry = sm + (size_t)10 * BUF;  // (TUW, TVW) of level z-1
  // level slots: slot s holds (U+iV) at sm + (2s)*BUF and (W+iE) at sm + (2s+1)*BUF
  auto UVs = [&](int s) { return sm + (size_t)(2 * s) * BUF; };
  auto WEs = [&](int s) { return sm + (size_t)(2 * s + 1) * BUF; };

  const int NZ = a.NZ, MY = a.MY;
  const int y = blockIdx.x;
  const int z0 = blockIdx.y * f.zchunk + 1;
  const int z1 = min(z0 + f.zchunk - 1, NZ);
  if (z0 > NZ) return;
  // team w (threads [TEAM w, TEAM (w+1))) owns transform w of every phase
  const int warp = threadIdx.x / TEAM, lane = threadIdx.x % TEAM;
  const int bar = 1 + warp;
  auto S = [](int q) { return Swz<T, MX>::f(q); };  // swizzled position of element q
  const T kx0 = (T)a.kx0, dzm = (T)a.dzm, todzm = (T)a.todzm, emin = (T)a.emin;
  const T xkmax = (T)a.xkmax, nu = (T)a.nu, c01 = (T)0.1 * (T)a.dsl;
  const WallParams& wp = *f.wp;
  // weight of the interior momentum stresses: 0 when the learned closure
  // supplies them (the wall rows stay)
  const bool learned = (f.lflag && f.lflag[0]);
  const T mom = learned ? (T)0 : (T)1;

  auto mixrow = [&](int j, int z) -> const cx<T>* {
    return reinterpret_cast<const cx<T>*>(f.in.p[j]) + ((size_t)(z - 1) * MY + y) * KX;
  };
  // complex row Z = A + iB of two real c2r outputs from x-spectral rows A, B
  // (optional i*kx on each; NULL = zero row)
  auto c2r_load = [&](const cx<T>* A, bool ma, const cx<T>* B, bool mb, int n) -> cx<T> {
    int k = -1;
    bool mir = false;
    if (n < KX) k = n;
    else if (n > MX - KX) { k = MX - n; mir = true; }
    if (k < 0) return zero_cx<T>();
    cx<T> av = A ? A[k] : zero_cx<T>(), bv = B ? B[k] : zero_cx<T>();
    T kk = kx0 * (T)k;
    if (ma) av = mul_i(av) * kk;
    if (mb) bv = mul_i(bv) * kk;
    if (k == 0) { av.y = 0; bv.y = 0; }
    if (mir) { av = conj(av); bv = conj(bv); }
    return mk(av.x - bv.y, av.y + bv.x);
  };
  // inverse transform of one (A, B) pair into buf (by the calling team)
  auto inv = [&](cx<T>* buf, const cx<T>* A, bool ma, const cx<T>* B, bool mb) {
    fused_fft<MX, +1, false, TEAM, T>(buf, tws, [&](int n) { return c2r_load(A, ma, B, mb, n); }, lane, bar);
  };
  auto clipE = [&](cx<T>* we) {
    for (int x = lane; x < MX; x += TEAM) we[S(x)].y = tmax(we[S(x)].y, emin);
    team_sync<TEAM>(bar);
  };
  auto xkk = [&](T e) { return tmin(c01 * tke_sqrt(e), xkmax) + nu; };

  // ---- prologue: slots for levels z0-1 and z0, carried tuw/tvw of z0-1 ----
  int sm1 = 0, s0 = 1, sp1 = 2;  // slots of z-1, z, z+1
  {
    // one transform per warp, described by (destination, A, ikx on A, B, ikx on B, clip E)
    cx<T>* dst = nullptr;
    const cx<T>* A = nullptr;
    const cx<T>* B = nullptr;
    bool ma = false, mb = false, ce = false;
    const int zm = z0 - 1;
    if (z0 == 1) {
      if (warp == 0) { dst = UVs(s0); A = mixrow(0, 1); B = mixrow(2, 1); }
      if (warp == 1) { dst = WEs(s0); A = mixrow(4, 1); B = mixrow(6, 1); ce = true; }
    } else {
      if (warp == 0) { dst = UVs(sm1); A = mixrow(0, zm); B = mixrow(2, zm); }
      if (warp == 1) { dst = WEs(sm1); A = mixrow(4, zm); B = mixrow(6, min(zm, NZ - 1)); ce = true; }
      if (warp == 2) { dst = UVs(s0); A = mixrow(0, z0); B = mixrow(2, z0); }
      if (warp == 3) { dst = WEs(s0); A = z0 < NZ ? mixrow(4, z0) : nullptr; B = mixrow(6, min(z0, NZ - 1)); ce = true; }
      if (warp == 4 && !learned) { dst = work[0]; A = mixrow(4, zm); ma = true; B = mixrow(5, zm); }  // WX + iWY at z0-1
    }
    if (dst) {
      inv(dst, A, ma, B, mb);
      if (ce) clipE(dst);
    }
  }
  __syncthreads();
  if (z0 == 1) {
    for (int x = threadIdx.x; x < MX; x += blockDim.x) {
      cx<T> uv = UVs(s0)[S(x)];
      UVs(sm1)[S(x)] = zero_cx<T>();
      WEs(sm1)[S(x)] = mk((T)0, WEs(s0)[S(x)].y);  // w(0) = 0, e(0) = e(1)
      T tu, tv;
      wall_stress<T>(wp.w[0], wp, a, 0, uv.x, uv.y, tu, tv);
      carry[x] = mk(tu, tv);
    }
  } else if (learned) {
    for (int x = threadIdx.x; x < MX; x += blockDim.x) carry[x] = zero_cx<T>();
  } else {
    for (int x = threadIdx.x; x < MX; x += blockDim.x) {
      cx<T> uvm = UVs(sm1)[S(x)], uv0 = UVs(s0)[S(x)], wxy = work[0][S(x)];
      T xk = xkk(WEs(sm1)[S(x)].y);
      T uz = (uv0.x - uvm.x) * dzm, vz = (uv0.y - uvm.y) * dzm;
      carry[x] = mk(-xk * (uz + wxy.x), -xk * (vz + wxy.y));
    }
  }
  __syncthreads();

  double divz_part = 0.0;
  double sgs_part[6] = {0, 0, 0, 0, 0, 0};
  for (int z = z0; z <= z1; z++) {
    const int le = z < NZ - 2 ? z : NZ - 2;
    // ---- phase I: inverse transforms (one per warp) ----
    {
      cx<T>* dst = nullptr;
      const cx<T>* A = nullptr;
      const cx<T>* B = nullptr;
      bool ma = false, mb = false, ce = false, zero = false;
      switch (warp) {
        case 0:  // U + iV at z+1
          dst = UVs(sp1);
          if (z + 1 <= NZ) { A = mixrow(0, z + 1); B = mixrow(2, z + 1); } else zero = true;
          break;
        case 1:  // W + iE at z+1 (w = 0 above nnz-1, e clamped to level nnz-1)
          dst = WEs(sp1);
          A = (z + 1 <= NZ - 1) ? mixrow(4, z + 1) : nullptr;
          B = mixrow(6, min(z + 1, NZ - 1));
          ce = true;
          break;
        case 2:
          if (learned) { dst = work[0]; A = mixrow(0, z); ma = true; B = mixrow(3, z); }  // UX + iVY
          else { dst = work[0]; A = mixrow(0, z); B = mixrow(2, z); ma = mb = true; }     // UX + iVX
          break;
        case 3: if (!learned) { dst = work[1]; A = mixrow(1, z); B = mixrow(3, z); } break;  // UY + iVY
        case 4:                                                                              // WX + iWY
          if (learned) break;
          dst = work[2];
          if (z <= NZ - 1) { A = mixrow(4, z); ma = true; B = mixrow(5, z); } else zero = true;
          break;
        default:  // EX + iEY at le
          if (z <= NZ - 1) { dst = work[3]; A = mixrow(6, le); ma = true; B = mixrow(7, le); }
          break;
      }
      if (zero) {
        for (int x = lane; x < MX; x += TEAM) dst[x] = zero_cx<T>();
        team_sync<TEAM>(bar);
      } else if (dst) {
        inv(dst, A, ma, B, mb);
        if (ce) clipE(dst);
      }
    }
    __syncthreads();
    // L2 prefetch (one thread, nothing waits on it) of the rows the next
    // level's phase I reads from DRAM: U, V, W, E at z+2 and VY, UY, WY, EY at
    // z+1 (U, V, W, E at z+1 were this level's window rows and are in L2)
    if (threadIdx.x == 0 && z + 1 <= z1) {
      constexpr unsigned RB = KX * sizeof(cx<T>);
      if (z + 2 <= NZ) { tma::prefetch_l2(mixrow(0, z + 2), RB); tma::prefetch_l2(mixrow(2, z + 2), RB); }
      if (z + 2 <= NZ - 1) { tma::prefetch_l2(mixrow(4, z + 2), RB); tma::prefetch_l2(mixrow(6, z + 2), RB); }
      tma::prefetch_l2(mixrow(3, z + 1), RB);
      if (!learned) tma::prefetch_l2(mixrow(1, z + 1), RB);
      if (z + 1 <= NZ - 1) {
        if (!learned) tma::prefetch_l2(mixrow(5, z + 1), RB);
        tma::prefetch_l2(mixrow(7, min(z + 1, NZ - 2)), RB);
      }
    }
    // ---- phase II: fluxes (k_flux) ----
    // the forward transforms of F+iPe and H reuse the z-1 window slots,
    // whose rows are dead once each point has read them
    work[4] = UVs(sm1);
    work[5] = WEs(sm1);
    const bool top = (z == NZ);
    const bool clip = (!top) && f.clipflag[le - 1];
    const T* dEX = reinterpret_cast<const T*>(f.dEX) + ((size_t)(le - 1) * MY + y) * MX;
    const T* dEY = reinterpret_cast<const T*>(f.dEY) + ((size_t)(le - 1) * MY + y) * MX;
    for (int x = threadIdx.x; x < MX; x += blockDim.x) {
      const cx<T> uvm = UVs(sm1)[S(x)], uv0 = UVs(s0)[S(x)], uv1 = UVs(sp1)[S(x)];
      const cx<T> wem = WEs(sm1)[S(x)], we0 = WEs(s0)[S(x)], we1 = WEs(sp1)[S(x)];
      // learned: work[0] holds (ux, vy); the other gradients are not needed
      const cx<T> w0 = work[0][S(x)];
      const cx<T> dxv = learned ? mk(w0.x, (T)0) : w0;
      const cx<T> dyv = learned ? mk((T)0, w0.y) : work[1][S(x)];
      const cx<T> wxy = learned ? zero_cx<T>() : work[2][S(x)];
      cx<T> exy = top ? zero_cx<T>() : work[3][S(x)];
      if (clip) { exy.x += dEX[x]; exy.y += dEY[x]; }
      const cx<T> tprev = carry[x];
      const T U0 = uv0.x, V0 = uv0.y, Um = uvm.x, Vm = uvm.y, U1 = uv1.x, V1 = uv1.y;
      const T W0 = we0.x, Wm = wem.x, W1 = we1.x, E0 = we0.y, Em = wem.y, E1 = we1.y;
      const T ux = dxv.x, vx = dxv.y, uy = dyv.x, vy = dyv.y;
      const T xkm = xkk(Em), xk0 = xkk(E0);
      const T s = mom * (xkm + xk0);
      const T tuu = -s * ux, tvv = -s * vy, tuv = -s * (uy + vx) * (T)0.5;
      T tuw0, tvw0;
      if (top) {
        wall_stress<T>(wp.w[1], wp, a, 1, U0, V0, tuw0, tvw0);
      } else {
        const T uz = (U1 - U0) * dzm, vz = (V1 - V0) * dzm;
        tuw0 = -mom * xk0 * (uz + wxy.x);
        tvw0 = -mom * xk0 * (vz + wxy.y);
      }
      const T wz0 = (W0 - Wm) * dzm;
      const T tww0 = -s * wz0;
      const T A = U0 * U0 + tuu, B = U0 * V0 + tuv, C = V0 * V0 + tvv;
      const T Pu = -((U1 + U0) * W0 - (Um + U0) * Wm) * todzm + (T)a.forcing - (tuw0 - tprev.x) * dzm;
      const T Pv = -((V1 + V0) * W0 - (Vm + V0) * Wm) * todzm - (tvw0 - tprev.y) * dzm;
      work[0][S(x)] = mk(A, Pu);
      work[1][S(x)] = mk(B, Pv);
      if (!top) {
        const T xkp = xkk(E1);
        const T wz1 = (W1 - W0) * dzm;
        const T tww1 = -mom * (xk0 + xkp) * wz1;
        const T D = (T)0.5 * (U0 + U1) * W0 + tuw0;
        const T G = (T)0.5 * (V0 + V1) * W0 + tvw0;
        const T hp = (T)0.5 * (W1 + W0), hm = (T)0.5 * (W0 + Wm);
        const T Pw = -(hp * hp - hm * hm) * dzm - (tww1 - tww0) * dzm;
        const T F = (T)0.5 * E0 * (U0 + U1) - (T)2 * xk0 * exy.x;
        const T H = (T)0.5 * E0 * (V0 + V1) - (T)2 * xk0 * exy.y;
        const T Pe = -(W1 * E1 - Wm * Em) * todzm +
                     ((xkp + xk0) * (E1 - E0) - (xk0 + xkm) * (E0 - Em)) * (T)a.dzm2 - (T)a.ceps * E0 * tke_sqrt(E0);
        work[2][S(x)] = mk(C, G);
        work[3][S(x)] = mk(D, Pw);
        work[4][S(x)] = mk(F, Pe);
        work[5][S(x)] = mk(H, (T)0);
      } else {
        work[2][S(x)] = mk(C, (T)0);
      }
      carry[x] = mk(tuw0, tvw0);
      const T d = ux + vy + wz0;
      divz_part += (double)(d * d);
      if (a.mnout_sgs) {
        sgs_part[0] += (double)tuu; sgs_part[1] += (double)tvv; sgs_part[2] += (double)tuv;
        sgs_part[3] += (double)tww0; sgs_part[4] += (double)tuw0; sgs_part[5] += (double)tvw0;
      }
    }
    __syncthreads();
    // per-level statistics of this row
    {
      const size_t slot = (size_t)(z - 1) * MY + y;
      double v1[1] = {divz_part};
      block_sum_store<1>(v1, f.divpart + slot);
      divz_part = 0.0;
      if (a.mnout_sgs) {
        __syncthreads();
        block_sum_store<6>(sgs_part, f.sgspart + slot * 6);
#pragma unroll
        for (int q = 0; q < 6; q++) sgs_part[q] = 0.0;
      }
    }
    // ---- phase III: forward transforms, -d/dx, truncation to kx < nx/2 ----
    if (!(top && warp >= 3)) {
      cx<T>* buf = work[warp];
      fused_fft<MX, -1, true, TEAM, T>(buf, tws, NoLoad{}, lane, bar);
      const size_t orow = ((size_t)(z - 1) * MY + y) * KX;
      auto O = [&](int j) { return reinterpret_cast<cx<T>*>(f.out.p[j]) + orow; };
      for (int k = lane; k < KX; k += TEAM) {
        cx<T> zk = buf[S(k)], zmr = conj(buf[S((MX - k) % MX)]);
        cx<T> ah = (zk + zmr) * (T)0.5;
        cx<T> dd = zk - zmr;
        cx<T> bh = mk(dd.y * (T)0.5, -dd.x * (T)0.5);
        T kk = kx0 * (T)k;
        cx<T> dxa = mk(kk * ah.y, -kk * ah.x);  // -i kx a^
        switch (warp) {
          case 0: O(0)[k] = dxa + bh; break;                          // Xu1
          case 1: O(2)[k] = dxa + bh; O(1)[k] = ah; break;            // Xv1, Xu2
          case 2: O(3)[k] = ah; if (!top) O(5)[k] = bh; break;        // Xv2, Xw2
          case 3: O(4)[k] = dxa + bh; break;                          // Xw1
          case 4: O(6)[k] = dxa + bh; break;                          // Xe1
          default: O(7)[k] = ah; break;                               // Xe2
        }
      }
    }
    __syncthreads();
    // rotate the window: z -> z-1, z+1 -> z
    const int t = sm1;
    sm1 = s0; s0 = sp1; sp1 = t;
  }
}

// Per-level flag: does max(expand(e), emin) clip anywhere on the padded
// plane?  Rows of Em (pairs) are inverted and compared with emin.
template <class T, int NSX>
__global__ void __launch_bounds__(RowCfg<3 * NSX / 2>::THREADS)
k_clip_flag(const cx<T>* __restrict__ Em, int* __restrict__ flags, int MY, T emin, const cx<T>* __restrict__ tw) {
  constexpr int MX = 3 * NSX / 2;
  constexpr int KX = NSX / 2;
  using C = RowCfg<MX>;
  extern __shared__ __align__(16) unsigned char smraw[];
  cx<T>* sm = reinterpret_cast<cx<T>*>(smraw);
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  const int z = blockIdx.y + 1;
  const int p0 = blockIdx.x * C::NT, np = MY / 2;
  const cx<T>* in = Em + (size_t)(z - 1) * MY * KX;
  fft_core<MX, +1, false, false, false>(C::NT, sm, tw, [&](int t, int n) {
    int p = p0 + t;
    cx<T> v = zero_cx<T>();
    if (p < np) {
      int k = -1;
      bool mir = false;
      if (n < KX) k = n;
      else if (n > MX - KX) { k = MX - n; mir = true; }
      if (k >= 0) {
        cx<T> av = in[(size_t)(2 * p) * KX + k], bv = in[(size_t)(2 * p + 1) * KX + k];
        if (k == 0) { av.y = 0; bv.y = 0; }
        if (mir) { av = conj(av); bv = conj(bv); }
        v = mk(av.x - bv.y, av.y + bv.x);
      }
    }
    return v;
  }, [&](int t, int n, cx<T> v) {
    int p = p0 + t;
    if (p < np && (v.x < emin || v.y < emin)) any = 1;
  });
  __syncthreads();
  if (threadIdx.x == 0 && any) atomicOr(flags + (z - 1), 1);
}

// Physical E (unclipped) of flagged levels, for the clip corrections.
template <class T, int NSX>
__global__ void __launch_bounds__(RowCfg<3 * NSX / 2>::THREADS)
k_clip_phys(const cx<T>* __restrict__ Em, T* __restrict__ E, const int* __restrict__ flags, int MY,
            const cx<T>* __restrict__ tw) {
  constexpr int MX = 3 * NSX / 2;
  constexpr int KX = NSX / 2;
  using C = RowCfg<MX>;
  const int z = blockIdx.y + 1;
  if (!flags[z - 1]) return;
  extern __shared__ __align__(16) unsigned char smraw[];
  cx<T>* sm = reinterpret_cast<cx<T>*>(smraw);
  const int p0 = blockIdx.x * C::NT, np = MY / 2;
  const cx<T>* in = Em + (size_t)(z - 1) * MY * KX;
  T* out = E + (size_t)(z - 1) * MY * MX;
  fft_core<MX, +1, false, false, false>(C::NT, sm, tw, [&](int t, int n) {
    int p = p0 + t;
    cx<T> v = zero_cx<T>();
    if (p < np) {
      int k = -1;
      bool mir = false;
      if (n < KX) k = n;
      else if (n > MX - KX) { k = MX - n; mir = true; }
      if (k >= 0) {
        cx<T> av = in[(size_t)(2 * p) * KX + k], bv = in[(size_t)(2 * p + 1) * KX + k];
        if (k == 0) { av.y = 0; bv.y = 0; }
        if (mir) { av = conj(av); bv = conj(bv); }
        v = mk(av.x - bv.y, av.y + bv.x);
      }
    }
    return v;
  }, [&](int t, int n, cx<T> v) {
    int p = p0 + t;
    if (p >= np) return;
    out[(size_t)(2 * p) * MX + n] = v.x;
    out[(size_t)(2 * p + 1) * MX + n] = v.y;
  });
}

// dEY = yderiv(delta), delta = max(emin - E, 0), flagged levels only.
template <class T, int NSY>
__global__ void __launch_bounds__(ColCfg<3 * NSY / 2, T>::THREADS)
k_clipd_y(const T* __restrict__ E, T* __restrict__ dEY, const int* __restrict__ flags, int MX, T emin, T ky0,
          const cx<T>* __restrict__ tw) {
  constexpr int M = 3 * NSY / 2;
  using C = ColCfg<M, T>;
  if (!flags[blockIdx.y]) return;
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
  cx<T>* out = reinterpret_cast<cx<T>*>(dEY + zoff);
  fft_core<M, +1, true, true, false>(C::TC, sm, tw, NoLoad{}, [&](int t, int n, cx<T> d) {
    int c = c0 + t;
    if (c < ncp) out[(size_t)n * ncp + c] = d;
  });
}

// dEX = xderiv(delta), flagged levels only.
template <class T, int NSX>
__global__ void __launch_bounds__(RowCfg<3 * NSX / 2>::THREADS)
k_clipd_x(const T* __restrict__ E, T* __restrict__ dEX, const int* __restrict__ flags, int MY, T emin, T kx0,
          const cx<T>* __restrict__ tw) {
  constexpr int MX = 3 * NSX / 2;
  using C = RowCfg<MX>;
  if (!flags[blockIdx.y]) return;
  extern __shared__ __align__(16) unsigned char smraw[];
  cx<T>* sm = reinterpret_cast<cx<T>*>(smraw);
  const size_t zoff = (size_t)blockIdx.y * MY * MX;
  const int p0 = blockIdx.x * C::NT, np = MY / 2;
  const T* Ez = E + zoff;
  T* out = dEX + zoff;
  fft_core<MX, -1, false, false, true>(C::NT, sm, tw, [&](int t, int n) {
    int p = p0 + t;
    cx<T> v = zero_cx<T>();
    if (p < np) {
      T av = Ez[(size_t)(2 * p) * MX + n], bv = Ez[(size_t)(2 * p + 1) * MX + n];
      v = mk(tmax(emin - av, (T)0), tmax(emin - bv, (T)0));
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
    out[(size_t)(2 * p) * MX + n] = d.x;
    out[(size_t)(2 * p + 1) * MX + n] = d.y;
  });
}

}  // namespace les

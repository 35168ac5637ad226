// les_mlp.cuh -- the learned SGS closure's perceptron on the sm_100a tensor
// cores: inference, and the forward/backward/Adam steps of its training.
//
// Network 11 -> 64 -> 64 -> 64 -> 6 (GELU, tanh form, after the hidden
// layers), bf16 weights and activations, f32 accumulation in tensor memory.
// A tile is 128 samples: sample r of the tile is row r of the A operand and
// lane r of the accumulator, so one thread owns one sample in every
// epilogue.  Layer l is D[128 x N] = A[128 x K] * W_l^T with K-major A (the
// activations) and K-major B (W_l stored [out][in]).
//
// Training adds, per tile:
//   dA_{l-1} = dZ_l * W_l       (M = 128 samples, B = W_l read MN-major)
//   dW_l    += dZ_l^T * A_{l-1} (M = 64 outputs, A = dZ_l and B = A_{l-1}
//                                 read MN-major: the reduction runs over the
//                                 tile's samples)
//   db_l    += dZ_l^T * 1       (same shape, B = a tile of ones)
// with dW, db accumulated in tensor memory over all tiles of a CTA, then
// written as per-CTA partial sums and reduced in a fixed order.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include "tc_sm100.cuh"

namespace les {

constexpr int kMlpIn = 11, kMlpHid = 64, kMlpOut = 6;
constexpr int kMlpNParam = 9478;
constexpr int kMlpNNorm = 34;
// offsets in the flat parameter vector: W1[64][11], b1, W2[64][64], b2, W3, b3, W4[6][64], b4
constexpr int kPW1 = 0, kPB1 = 704, kPW2 = 768, kPB2 = 4864, kPW3 = 4928, kPB3 = 9024, kPW4 = 9088, kPB4 = 9472;
constexpr int ERR_MMA_TIMEOUT = 4;
// Default limit of a wait for a tensor-core MMA (MlpDev::wait_ns, settable
// per network from the host), and the fixed limit of the wait that drains an
// outstanding MMA after a failure, before its tensor memory is released.
constexpr uint64_t kMmaWaitNs = 1000000000ull;  // 1 s

// Device-side parameters: bf16 weight tiles in the core-matrix layout
// (W1 padded to 16 inputs, W4 to 16 outputs), f32 biases and the feature /
// output normalisation.
struct MlpDev {
  __nv_bfloat16 w1[64 * 16];
  __nv_bfloat16 w2[64 * 64];
  __nv_bfloat16 w3[64 * 64];
  __nv_bfloat16 w4[16 * 64];
  float b1[64], b2[64], b3[64], b4[16];
  float in_shift[16], in_scale[16], out_scale[8], out_shift[8];
  float in_rscale[16];  // 1 / in_scale (0 where in_scale is 0)
  unsigned long long wait_ns;  // limit of each wait for an MMA (kMmaWaitNs by default)
  unsigned long long pad_;
};
static_assert(sizeof(MlpDev) % 16 == 0, "MlpDev is copied in 16-byte words");

constexpr float kGeluC = 0.7978845608028654f;  // sqrt(2/pi)
constexpr float kGeluA = 0.044715f;

// GELU of two pre-activations in bf16x2 arithmetic, packed bf16x2 result
__device__ __forceinline__ uint32_t gelu_pack(float a, float b) {
  const __nv_bfloat162 x = __floats2bfloat162_rn(a, b);
  const __nv_bfloat162 c = __floats2bfloat162_rn(kGeluC, kGeluC);
  const __nv_bfloat162 ca = __floats2bfloat162_rn(kGeluC * kGeluA, kGeluC * kGeluA);
  const __nv_bfloat162 h = __floats2bfloat162_rn(0.5f, 0.5f);
  const __nv_bfloat162 u = __hmul2(x, __hfma2(__hmul2(x, x), ca, c));
  const __nv_bfloat162 t = tc::tanh_bf2(u);
  const __nv_bfloat162 hx = __hmul2(x, h);
  return tc::bf2_bits(__hfma2(hx, t, hx));
}
// d GELU / dz in f32
__device__ __forceinline__ float gelu_grad(float z) {
  const float t = tc::tanh_f32(kGeluC * (z + kGeluA * z * z * z));
  return 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * kGeluC * (1.0f + 3.0f * kGeluA * z * z);
}
__device__ __forceinline__ uint32_t pack_bf2(float a, float b) { return tc::bf2_bits(__floats2bfloat162_rn(a, b)); }

// bar.red.or over a named barrier: true in every thread if `pred` was true
// in any of them.
__device__ __forceinline__ bool bar_any(int id, int count, bool pred) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 q, %3, 0;\n\tbar.red.or.pred p, %1, %2, q;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(r)
      : "r"(id), "r"(count), "r"((uint32_t)pred)
      : "memory");
  return r != 0;
}

// Bias + GELU of the 64 accumulator columns of this thread's lane, written
// as row r of a K = 64 activation tile.
__device__ __forceinline__ void hidden_epilogue(uint32_t taddr, const float* __restrict__ b, unsigned char* act,
                                                int r) {
#pragma unroll
  for (int c = 0; c < 4; c++) {
    float v[16];
    tc::tmem_ld16(taddr + 16 * c, v);
    uint32_t pk[8];
#pragma unroll
    for (int j = 0; j < 8; j++) pk[j] = gelu_pack(v[2 * j] + b[16 * c + 2 * j], v[2 * j + 1] + b[16 * c + 2 * j + 1]);
    *reinterpret_cast<uint4*>(act + 2 * tc::tile_elem(r, 16 * c, 64)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
    *reinterpret_cast<uint4*>(act + 2 * tc::tile_elem(r, 16 * c + 8, 64)) = make_uint4(pk[4], pk[5], pk[6], pk[7]);
  }
}

// Inference epilogue: 2 GELU(z) = z + z tanh(u) of the 64 accumulator
// columns (the biases are already in the accumulators), written as row r of
// a K = 64 activation tile.  The factor 2 is taken back by the halved
// weights of the next layer (infer_prologue); both scalings are exact in
// bf16, so the next layer's products equal those of GELU(z) and W.
__device__ __forceinline__ uint32_t gelu2_pack(float a, float b) {
  const __nv_bfloat162 x = __floats2bfloat162_rn(a, b);
  const __nv_bfloat162 c = __floats2bfloat162_rn(kGeluC, kGeluC);
  const __nv_bfloat162 ca = __floats2bfloat162_rn(kGeluC * kGeluA, kGeluC * kGeluA);
  const __nv_bfloat162 u = __hmul2(x, __hfma2(__hmul2(x, x), ca, c));
  return tc::bf2_bits(__hfma2(x, tc::tanh_bf2(u), x));
}
__device__ __forceinline__ void hidden_epilogue_infer(uint32_t taddr, unsigned char* act, int r) {
#pragma unroll
  for (int c = 0; c < 4; c++) {
    float v[16];
    tc::tmem_ld16(taddr + 16 * c, v);
    uint32_t pk[8];
#pragma unroll
    for (int j = 0; j < 8; j++) pk[j] = gelu2_pack(v[2 * j], v[2 * j + 1]);
    *reinterpret_cast<uint4*>(act + 2 * tc::tile_elem(r, 16 * c, 64)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
    *reinterpret_cast<uint4*>(act + 2 * tc::tile_elem(r, 16 * c + 8, 64)) = make_uint4(pk[4], pk[5], pk[6], pk[7]);
  }
}

// MMA issue of one layer (one elected thread): D = A * W^T over K.
template <int N, int K>
__device__ __forceinline__ void issue_layer(uint32_t d, uint32_t a_s, uint32_t w_s) {
  constexpr uint32_t sbo = (K / 8) * 128;
  constexpr uint32_t id = tc::idesc_bf16(128, N, false, false);
#pragma unroll
  for (int s = 0; s < K / 16; s++)
    tc::mma_bf16(d, tc::sdesc(a_s + 256 * s, 128, sbo), tc::sdesc(w_s + 256 * s, 128, sbo), id, s > 0 ? 1u : 0u);
}

// As issue_layer, then one more K = 16 slice that adds the bias: A = the
// tile of ones (columns 0..2), B = the layer's bias tile (three bf16 pieces
// per output in columns 0..2).
template <int N, int K>
__device__ __forceinline__ void issue_layer_bias(uint32_t d, uint32_t a_s, uint32_t w_s, uint32_t ones_s,
                                                 uint32_t bias_s) {
  issue_layer<N, K>(d, a_s, w_s);
  tc::mma_bf16(d, tc::sdesc(ones_s, 128, 256), tc::sdesc(bias_s, 128, 256), tc::idesc_bf16(128, N, false, false), 1u);
}

// Per-CTA folds of the inference copy of the parameters (the training
// kernels keep MlpDev as the host wrote it):
//  * the biases enter the accumulators through the tensor cores.  Each f32
//    bias b is split into bf16 pieces hi + mid + lo (24 bits: b itself);
//    layer 1 reads them from W1 columns 13..15 against feature columns
//    13..15 set to one in the A tile, layers 2..4 from a bias tile [N][16]
//    against a shared tile of ones [128][16] (kInferBiasBytes);
//  * W2, W3, W4 are halved for the doubled GELU of hidden_epilogue_infer.
// Ends with the proxy fence that makes these shared-memory writes, and the
// parameter copy before them, visible to the tensor cores.
constexpr int kInferBiasBytes = 4096 + 2048 + 2048 + 512;  // ones, bias tiles of layers 2, 3, 4
constexpr uint32_t kBf16One = 0x3F80u;

__device__ __forceinline__ void bias_pieces(float b, __nv_bfloat16 (&pc)[3]) {
  pc[0] = __float2bfloat16_rn(b);
  const float r1 = b - __bfloat162float(pc[0]);
  pc[1] = __float2bfloat16_rn(r1);
  pc[2] = __float2bfloat16_rn(r1 - __bfloat162float(pc[1]));
}

__device__ __forceinline__ void infer_prologue(MlpDev* P, unsigned char* tiles) {
  const __nv_bfloat162 h2 = __floats2bfloat162_rn(0.5f, 0.5f);
  __nv_bfloat162* w2 = reinterpret_cast<__nv_bfloat162*>(P->w2);
  __nv_bfloat162* w3 = reinterpret_cast<__nv_bfloat162*>(P->w3);
  __nv_bfloat162* w4 = reinterpret_cast<__nv_bfloat162*>(P->w4);
  for (int i = threadIdx.x; i < 64 * 64 / 2; i += blockDim.x) { w2[i] = __hmul2(w2[i], h2); w3[i] = __hmul2(w3[i], h2); }
  for (int i = threadIdx.x; i < 16 * 64 / 2; i += blockDim.x) w4[i] = __hmul2(w4[i], h2);
  __nv_bfloat16* ones = reinterpret_cast<__nv_bfloat16*>(tiles);
  __nv_bfloat16* bt[3] = {ones + 128 * 16, ones + 128 * 16 + 64 * 16, ones + 128 * 16 + 2 * 64 * 16};
  const float* bsrc[3] = {P->b2, P->b3, P->b4};
  const int nrow[3] = {64, 64, 16};
  for (int i = threadIdx.x; i < 128 * 16; i += blockDim.x) {
    const int row = i >> 4, k = i & 15;
    ones[tc::tile_elem(row, k, 16)] = __float2bfloat16_rn(k < 3 ? 1.0f : 0.0f);
  }
#pragma unroll
  for (int l = 0; l < 3; l++)
    for (int i = threadIdx.x; i < nrow[l] * 16; i += blockDim.x) {
      const int row = i >> 4, k = i & 15;
      __nv_bfloat16 pc[3];
      bias_pieces(bsrc[l][row], pc);
      bt[l][tc::tile_elem(row, k, 16)] = k < 3 ? pc[k] : __float2bfloat16_rn(0.0f);
    }
  for (int o = threadIdx.x; o < 64; o += blockDim.x) {
    __nv_bfloat16 pc[3];
    bias_pieces(P->b1[o], pc);
#pragma unroll
    for (int k = 0; k < 3; k++) P->w1[tc::tile_elem(o, 13 + k, 16)] = pc[k];
  }
  tc::fence_async_smem();
}

// ------------------------------------------------------------------------
// Inference.  G groups of 4 warps per CTA, each group owns one tile at a
// time, 64 tensor-memory columns and one 16 KB activation tile; the groups'
// epilogues overlap each other's MMAs.  Features: bf16 [n][16] (columns
// 0..10 normalised inputs; 11 and 12 meet zero columns of W1, so they may
// carry data for the epilogue; 13..15 are read as ones by the tensor cores,
// against the bias pieces of infer_prologue).  out(p, valid, y, f0, f1,
// P) consumes the 16 output columns (y[0..5] normalised outputs + biases)
// and returns three terms summed per CTA into dissip_part[3 blockIdx.x + j],
// j = 0, 1, 2 (when non-null).
// ------------------------------------------------------------------------
constexpr int kInferGroups = 4;
constexpr int kInferCtasPerSm = 2;  // 2 x 256 tensor-memory columns, 2 x 87 KB shared memory
// after the activation tiles: the tile of ones and the bias tiles
// (kInferBiasBytes), then G mbarriers, the tensor-memory slot and three
// doubles per warp for the per-CTA sums (40 + 384 bytes at 16 warps)
constexpr size_t kInferSmem = sizeof(MlpDev) + (size_t)kInferGroups * 16384 + kInferBiasBytes + 512;

// One group's view of its tile: shared-memory addresses of its activation
// tile and of the weight tiles, its 64 tensor-memory columns, its named
// barrier and mbarrier, and the mbarrier phase.
struct MlpGroup {
  unsigned char* act;
  uint32_t act_s, w1s, w2s, w3s, w4s, dcol, my_t;
  uint32_t ones_s, b2s, b3s, b4s;  // inference: tile of ones and bias tiles
  int bar;
  uint64_t* mbar;
  uint32_t parity;
};

__device__ __forceinline__ MlpGroup mlp_group(MlpDev* P, unsigned char* act, unsigned char* tiles, uint32_t tbase,
                                              int g, int q, uint64_t* mbar) {
  MlpGroup G;
  G.act = act;
  G.act_s = tc::smem_addr(act);
  G.w1s = tc::smem_addr(P->w1);
  G.w2s = tc::smem_addr(P->w2);
  G.w3s = tc::smem_addr(P->w3);
  G.w4s = tc::smem_addr(P->w4);
  G.ones_s = tc::smem_addr(tiles);
  G.b2s = G.ones_s + 4096;
  G.b3s = G.ones_s + 6144;
  G.b4s = G.ones_s + 8192;
  G.dcol = tbase + 64 * g;
  G.my_t = G.dcol + ((uint32_t)(q * 32) << 16);
  G.bar = 1 + g;
  G.mbar = mbar;
  G.parity = 0;
  return G;
}

// The network on one 128-sample tile by one group of 4 warps (thread r owns
// sample r): features f0, f1 (bf16 x 16) in, the 16 output columns of this
// sample's lane (outputs + b4) out, with the parameters as infer_prologue
// folded them.  Returns false in every thread of the group when an MMA did
// not complete within its wait limit.
__device__ __forceinline__ bool mlp_tile(MlpGroup& G, const MlpDev* P, int r, uint4 f0, uint4 f1,
                                         float (&y)[16]) {
  auto wait_mma = [&]() -> bool {
    const bool ok = tc::mbar_wait(G.mbar, G.parity, P->wait_ns);
    G.parity ^= 1;
    tc::fence_after_sync();
    return ok;
  };
  // feature columns 13..15 read as ones (they meet the bias pieces in W1)
  const uint4 f1a = make_uint4(f1.x, f1.y, (f1.z & 0xFFFFu) | (kBf16One << 16), kBf16One | (kBf16One << 16));
  *reinterpret_cast<uint4*>(G.act + 2 * tc::tile_elem(r, 0, 16)) = f0;
  *reinterpret_cast<uint4*>(G.act + 2 * tc::tile_elem(r, 8, 16)) = f1a;
  tc::fence_async_smem();
  tc::fence_before_sync();
  tc::bar_sync(G.bar, 128);
  if (r == 0) {
    tc::fence_after_sync();
    issue_layer<64, 16>(G.dcol, G.act_s, G.w1s);
    tc::mma_commit(G.mbar);
  }
  bool bad = !wait_mma();
  hidden_epilogue_infer(G.my_t, G.act, r);
  tc::fence_async_smem();
  tc::fence_before_sync();
  if (bar_any(G.bar, 128, bad)) return false;
  if (r == 0) {
    tc::fence_after_sync();
    issue_layer_bias<64, 64>(G.dcol, G.act_s, G.w2s, G.ones_s, G.b2s);
    tc::mma_commit(G.mbar);
  }
  bad = !wait_mma();
  hidden_epilogue_infer(G.my_t, G.act, r);
  tc::fence_async_smem();
  tc::fence_before_sync();
  if (bar_any(G.bar, 128, bad)) return false;
  if (r == 0) {
    tc::fence_after_sync();
    issue_layer_bias<64, 64>(G.dcol, G.act_s, G.w3s, G.ones_s, G.b3s);
    tc::mma_commit(G.mbar);
  }
  bad = !wait_mma();
  hidden_epilogue_infer(G.my_t, G.act, r);
  tc::fence_async_smem();
  tc::fence_before_sync();
  if (bar_any(G.bar, 128, bad)) return false;
  if (r == 0) {
    tc::fence_after_sync();
    issue_layer_bias<16, 64>(G.dcol, G.act_s, G.w4s, G.ones_s, G.b4s);
    tc::mma_commit(G.mbar);
  }
  bad = !wait_mma();
  tc::tmem_ld16(G.my_t, y);
  tc::fence_before_sync();
  return !bar_any(G.bar, 128, bad);
}

// After a failed tile: flag the error and give the outstanding commit a
// bounded wait before the tensor memory is released.
__device__ __forceinline__ void mlp_tile_failed(MlpGroup& G, int r, int* err) {
  if (r == 0) {
    atomicOr(err, ERR_MMA_TIMEOUT);
    tc::mbar_wait(G.mbar, G.parity ^ 1, kMmaWaitNs);
  }
}

template <class Out>
__global__ void __launch_bounds__(128 * kInferGroups, kInferCtasPerSm)
k_mlp_infer(const MlpDev* __restrict__ prm, const uint4* __restrict__ feat, long long n, Out out,
            double* __restrict__ dissip_part, int* __restrict__ err) {
  constexpr int G = kInferGroups;
  extern __shared__ __align__(1024) unsigned char smraw_tc[];
  MlpDev* P = reinterpret_cast<MlpDev*>(smraw_tc);
  unsigned char* act_all = smraw_tc + sizeof(MlpDev);
  unsigned char* tiles = act_all + (size_t)G * 16384;
  uint64_t* bars = reinterpret_cast<uint64_t*>(tiles + kInferBiasBytes);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + G);
  double* red = reinterpret_cast<double*>(bars + G + 1);

  const int tid = threadIdx.x, g = tid >> 7, r = tid & 127, warp = tid >> 5, q = warp & 3;
  for (int i = tid; i < (int)(sizeof(MlpDev) / 16); i += blockDim.x)
    reinterpret_cast<uint4*>(P)[i] = reinterpret_cast<const uint4*>(prm)[i];
  __syncthreads();
  infer_prologue(P, tiles);
  if (tid < G) tc::mbar_init(&bars[tid], 1);
  if (warp == 0) {
    tc::tmem_alloc(tslot, 64 * G);
    tc::tmem_relinquish();
  }
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = *tslot;
  MlpGroup grp = mlp_group(P, act_all + (size_t)g * 16384, tiles, tbase, g, q, &bars[g]);
  double dsum = 0.0, dsum2 = 0.0, dsum3 = 0.0;
  const long long ntiles = (n + 127) / 128;
  for (long long tile = (long long)blockIdx.x * G + g; tile < ntiles; tile += (long long)gridDim.x * G) {
    const long long p = tile * 128 + r;
    const bool valid = p < n;
    uint4 f0 = make_uint4(0, 0, 0, 0), f1 = f0;
    if (valid) { f0 = __ldg(feat + 2 * p); f1 = __ldg(feat + 2 * p + 1); }
    float y[16];
    if (!mlp_tile(grp, P, r, f0, f1, y)) {
      mlp_tile_failed(grp, r, err);
      break;
    }
    const double3 d = out(p, valid, y, f0, f1, P);
    dsum += d.x;
    dsum2 += d.y;
    dsum3 += d.z;
  }
  // per-CTA sums, fixed order
  for (int o = 16; o > 0; o >>= 1) {
    dsum += __shfl_xor_sync(0xffffffffu, dsum, o);
    dsum2 += __shfl_xor_sync(0xffffffffu, dsum2, o);
    dsum3 += __shfl_xor_sync(0xffffffffu, dsum3, o);
  }
  if ((tid & 31) == 0) { red[3 * warp] = dsum; red[3 * warp + 1] = dsum2; red[3 * warp + 2] = dsum3; }
  tc::fence_before_sync();
  __syncthreads();
  if (tid == 0 && dissip_part) {
    double s = 0.0, s2 = 0.0, s3 = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) { s += red[3 * w]; s2 += red[3 * w + 1]; s3 += red[3 * w + 2]; }
    dissip_part[3 * blockIdx.x] = s;
    dissip_part[3 * blockIdx.x + 1] = s2;
    dissip_part[3 * blockIdx.x + 2] = s3;
  }
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tbase, 64 * G);
  }
}

// Output functor of the operator entry point: normalised outputs y[0..5]
// as f32 [n][8] (columns 6, 7 zero).
struct MlpOutRaw {
  float* y;
  __device__ double3 operator()(long long p, bool valid, const float (&v)[16], uint4, uint4, const MlpDev*) const {
    if (valid) {
      float4* o = reinterpret_cast<float4*>(y + 8 * p);
      o[0] = make_float4(v[0], v[1], v[2], v[3]);
      o[1] = make_float4(v[4], v[5], 0.f, 0.f);
    }
    return make_double3(0.0, 0.0, 0.0);
  }
};

// ------------------------------------------------------------------------
// Training: loss and gradient of a batch.  One group (4 warps) per CTA and
// the whole tensor memory (512 columns):
//   Z1 [0,64) Z2 [64,128) Z3 [128,192) Z4 [192,208) dA3 [208,272)
//   dW1 [272,288) dW2 [288,352) dW3 [352,416) dW4^T [416,432)
//   db1 [432,448) db2 [448,464) db3 [464,480)
// dA2 reuses Z3's columns and dA1 Z2's once those pre-activations are read.
// Accumulators of M = 64 occupy lanes 0-15 of each 32-lane quarter: row m
// is lane 32*(m/16) + m%16.
// Shared memory: parameters, activation tiles A0 (K=16), A1..A3 (K=64),
// dZ tiles D (K=64) and D4 (K=16), a tile of ones (K=16).
// Per-CTA outputs: part[blockIdx.x][9478] gradient partial sums (flat
// parameter order) and lpart[blockIdx.x] the loss partial sum.
// ------------------------------------------------------------------------
constexpr size_t kTrainSmem = sizeof(MlpDev) + 4096 + 3 * 16384 + 16384 + 4096 + 4096 + 512;
// keep one CTA per SM: it owns all 512 tensor-memory columns
constexpr size_t kTrainSmemLaunch = kTrainSmem > 120 * 1024 ? kTrainSmem : 120 * 1024;

static __global__ void __launch_bounds__(128, 1)
k_mlp_train(const MlpDev* __restrict__ prm, const uint4* __restrict__ feat, const float4* __restrict__ target,
            long long n, float* __restrict__ part, double* __restrict__ lpart, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smraw_tc[];
  MlpDev* P = reinterpret_cast<MlpDev*>(smraw_tc);
  unsigned char* A0 = smraw_tc + sizeof(MlpDev);
  unsigned char* A1 = A0 + 4096;
  unsigned char* A2 = A1 + 16384;
  unsigned char* A3 = A2 + 16384;
  unsigned char* Dt = A3 + 16384;
  unsigned char* D4 = Dt + 16384;
  unsigned char* ONES = D4 + 4096;
  uint64_t* barp = reinterpret_cast<uint64_t*>(ONES + 4096);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(barp + 1);
  float* redf = reinterpret_cast<float*>(barp + 2);  // 4 warps x 8 floats
  double* redd = reinterpret_cast<double*>(barp + 2 + 16);

  const int r = threadIdx.x, warp = r >> 5, lane = r & 31;
  for (int i = r; i < (int)(sizeof(MlpDev) / 16); i += 128)
    reinterpret_cast<uint4*>(P)[i] = reinterpret_cast<const uint4*>(prm)[i];
  {
    const uint32_t one2 = pack_bf2(1.0f, 1.0f);
    for (int i = r; i < 4096 / 16; i += 128) reinterpret_cast<uint4*>(ONES)[i] = make_uint4(one2, one2, one2, one2);
  }
  if (r == 0) tc::mbar_init(barp, 1);
  if (warp == 0) {
    tc::tmem_alloc(tslot, 512);
    tc::tmem_relinquish();
  }
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  tc::fence_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tb = *tslot;
  const uint32_t lane_off = (uint32_t)(warp * 32) << 16;
  const uint32_t cZ1 = 0, cZ2 = 64, cZ3 = 128, cZ4 = 192, cdA3 = 208, cW1 = 272, cW2 = 288, cW3 = 352, cW4 = 416,
                 cB1 = 432, cB2 = 448, cB3 = 464;
  const uint32_t a0s = tc::smem_addr(A0), a1s = tc::smem_addr(A1), a2s = tc::smem_addr(A2), a3s = tc::smem_addr(A3),
                 dts = tc::smem_addr(Dt), d4s = tc::smem_addr(D4), ones = tc::smem_addr(ONES);
  const uint32_t w1s = tc::smem_addr(P->w1), w2s = tc::smem_addr(P->w2), w3s = tc::smem_addr(P->w3),
                 w4s = tc::smem_addr(P->w4);
  constexpr uint32_t idB64 = tc::idesc_bf16(128, 64, false, true);   // dA = dZ * W (W read MN-major)
  constexpr uint32_t idW64 = tc::idesc_bf16(64, 64, true, true);     // dW = dZ^T * A (both MN-major)
  constexpr uint32_t idW16 = tc::idesc_bf16(64, 16, true, true);
  uint32_t parity = 0;
  bool failed = false;
  uint32_t accw = 0;  // 0 until this CTA's first weight-gradient MMA
  const float inv_count = 1.0f / ((float)n * (float)kMlpOut);
  float db4[kMlpOut] = {0, 0, 0, 0, 0, 0};
  double lsum = 0.0;
  auto wait_mma = [&]() -> bool {
    const bool ok = tc::mbar_wait(barp, parity, P->wait_ns);
    parity ^= 1;
    tc::fence_after_sync();
    return ok;
  };
  auto sync_check = [&](bool bad) -> bool {
    tc::fence_async_smem();
    tc::fence_before_sync();
    return bar_any(1, 128, bad);
  };
  // dZ = dA * GELU'(Z + b) for the 64 columns of this lane, into tile Dt
  auto back_epilogue = [&](uint32_t c_dA, uint32_t c_Z, const float* b) {
#pragma unroll
    for (int c = 0; c < 4; c++) {
      float da[16], z[16];
      tc::tmem_ld16(tb + lane_off + c_dA + 16 * c, da);
      tc::tmem_ld16(tb + lane_off + c_Z + 16 * c, z);
      uint32_t pk[8];
#pragma unroll
      for (int j = 0; j < 8; j++)
        pk[j] = pack_bf2(da[2 * j] * gelu_grad(z[2 * j] + b[16 * c + 2 * j]),
                         da[2 * j + 1] * gelu_grad(z[2 * j + 1] + b[16 * c + 2 * j + 1]));
      *reinterpret_cast<uint4*>(Dt + 2 * tc::tile_elem(r, 16 * c, 64)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
      *reinterpret_cast<uint4*>(Dt + 2 * tc::tile_elem(r, 16 * c + 8, 64)) = make_uint4(pk[4], pk[5], pk[6], pk[7]);
    }
  };
  // weight / bias gradient MMAs of a hidden layer: dW (M=64 outputs) over the
  // tile's 128 samples, A = Dt (MN-major), B = the layer's input tile
  auto issue_dw = [&](uint32_t c_W, uint32_t c_B, uint32_t in_s, int kin) {
    const uint32_t lbo_in = (uint32_t)(kin / 8) * 128;
    const uint32_t id = kin == 64 ? idW64 : idW16;
#pragma unroll 1
    for (int s = 0; s < 8; s++) {
      const uint64_t a = tc::sdesc(dts + 2 * 1024 * s, 1024, 128);
      tc::mma_bf16(tb + c_W, a, tc::sdesc(in_s + 2 * lbo_in * s, lbo_in, 128), id, (accw | s) ? 1u : 0u);
      tc::mma_bf16(tb + c_B, a, tc::sdesc(ones + 2 * 256 * s, 256, 128), idW16, (accw | s) ? 1u : 0u);
    }
  };
  // dA = Dt * W (M = 128 samples, N = 64 inputs, K = 64 outputs)
  auto issue_da = [&](uint32_t c_dA, uint32_t w_s) {
#pragma unroll
    for (int s = 0; s < 4; s++)
      tc::mma_bf16(tb + c_dA, tc::sdesc(dts + 256 * s, 128, 1024), tc::sdesc(w_s + 2 * 1024 * s, 1024, 128), idB64,
                   s > 0 ? 1u : 0u);
  };

  const long long ntiles = (n + 127) / 128;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long p = tile * 128 + r;
    const bool valid = p < n;
    uint4 f0 = make_uint4(0, 0, 0, 0), f1 = f0;
    float4 t0 = make_float4(0.f, 0.f, 0.f, 0.f), t1 = t0;
    if (valid) {
      f0 = __ldg(feat + 2 * p); f1 = __ldg(feat + 2 * p + 1);
      t0 = __ldg(target + 2 * p); t1 = __ldg(target + 2 * p + 1);
    }
    *reinterpret_cast<uint4*>(A0 + 2 * tc::tile_elem(r, 0, 16)) = f0;
    *reinterpret_cast<uint4*>(A0 + 2 * tc::tile_elem(r, 8, 16)) = f1;
    if (sync_check(false)) { failed = true; break; }
    // ---- forward ----
    if (r == 0) { tc::fence_after_sync(); issue_layer<64, 16>(tb + cZ1, a0s, w1s); tc::mma_commit(barp); }
    bool bad = !wait_mma();
    hidden_epilogue(tb + lane_off + cZ1, P->b1, A1, r);
    if (sync_check(bad)) { failed = true; break; }
    if (r == 0) { tc::fence_after_sync(); issue_layer<64, 64>(tb + cZ2, a1s, w2s); tc::mma_commit(barp); }
    bad = !wait_mma();
    hidden_epilogue(tb + lane_off + cZ2, P->b2, A2, r);
    if (sync_check(bad)) { failed = true; break; }
    if (r == 0) { tc::fence_after_sync(); issue_layer<64, 64>(tb + cZ3, a2s, w3s); tc::mma_commit(barp); }
    bad = !wait_mma();
    hidden_epilogue(tb + lane_off + cZ3, P->b3, A3, r);
    if (sync_check(bad)) { failed = true; break; }
    if (r == 0) { tc::fence_after_sync(); issue_layer<16, 64>(tb + cZ4, a3s, w4s); tc::mma_commit(barp); }
    bad = !wait_mma();
    {
      float y[16];
      tc::tmem_ld16(tb + lane_off + cZ4, y);
      const float tg[6] = {t0.x, t0.y, t0.z, t0.w, t1.x, t1.y};
      float dy[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      if (valid) {
#pragma unroll
        for (int j = 0; j < kMlpOut; j++) {
          const float res = y[j] + P->b4[j] - tg[j];
          lsum += (double)res * (double)res;
          dy[j] = 2.0f * res * inv_count;
          db4[j] += dy[j];
        }
      }
      *reinterpret_cast<uint4*>(D4 + 2 * tc::tile_elem(r, 0, 16)) =
          make_uint4(pack_bf2(dy[0], dy[1]), pack_bf2(dy[2], dy[3]), pack_bf2(dy[4], dy[5]), 0u);
      *reinterpret_cast<uint4*>(D4 + 2 * tc::tile_elem(r, 8, 16)) = make_uint4(0u, 0u, 0u, 0u);
    }
    if (sync_check(bad)) { failed = true; break; }
    // ---- backward, layer 4: dW4^T (M = 64 inputs, N = 16 outputs) and dA3 ----
    if (r == 0) {
      tc::fence_after_sync();
#pragma unroll 1
      for (int s = 0; s < 8; s++)
        tc::mma_bf16(tb + cW4, tc::sdesc(a3s + 2 * 1024 * s, 1024, 128), tc::sdesc(d4s + 2 * 256 * s, 256, 128), idW16,
                     (accw | s) ? 1u : 0u);
      // dA3 = dZ4 * W4: K = 16 outputs, W4 tile read MN-major (rows = outputs)
      tc::mma_bf16(tb + cdA3, tc::sdesc(d4s, 128, 256), tc::sdesc(w4s, 1024, 128), idB64, 0u);
      tc::mma_commit(barp);
    }
    bad = !wait_mma();
    back_epilogue(cdA3, cZ3, P->b3);  // dZ3
    if (sync_check(bad)) { failed = true; break; }
    if (r == 0) {
      tc::fence_after_sync();
      issue_dw(cW3, cB3, a2s, 64);
      issue_da(cZ3, w3s);  // dA2 into Z3's columns
      tc::mma_commit(barp);
    }
    bad = !wait_mma();
    back_epilogue(cZ3, cZ2, P->b2);  // dZ2
    if (sync_check(bad)) { failed = true; break; }
    if (r == 0) {
      tc::fence_after_sync();
      issue_dw(cW2, cB2, a1s, 64);
      issue_da(cZ2, w2s);  // dA1 into Z2's columns
      tc::mma_commit(barp);
    }
    bad = !wait_mma();
    back_epilogue(cZ2, cZ1, P->b1);  // dZ1
    if (sync_check(bad)) { failed = true; break; }
    if (r == 0) {
      tc::fence_after_sync();
      issue_dw(cW1, cB1, a0s, 16);
      tc::mma_commit(barp);
    }
    bad = !wait_mma();
    accw = 1;
    if (sync_check(bad)) { failed = true; break; }
  }
  if (failed && r == 0) {
    atomicOr(err, ERR_MMA_TIMEOUT);
    tc::mbar_wait(barp, parity ^ 1, kMmaWaitNs);
  }
  // ---- per-CTA partial sums ----
  float* out = part + (size_t)blockIdx.x * kMlpNParam;
  if (accw) {
    // M = 64 accumulators: thread (warp q, lane l < 16) holds row 16q + l
    const int m = warp * 16 + lane;
    float v[16];
    // dW1 [64][11]
    tc::tmem_ld16(tb + lane_off + cW1, v);
    if (lane < 16)
      for (int i = 0; i < kMlpIn; i++) out[kPW1 + m * kMlpIn + i] = v[i];
    tc::tmem_ld16(tb + lane_off + cB1, v);
    if (lane < 16) out[kPB1 + m] = v[0];
    tc::tmem_ld16(tb + lane_off + cB2, v);
    if (lane < 16) out[kPB2 + m] = v[0];
    tc::tmem_ld16(tb + lane_off + cB3, v);
    if (lane < 16) out[kPB3 + m] = v[0];
#pragma unroll 1
    for (int c = 0; c < 4; c++) {
      tc::tmem_ld16(tb + lane_off + cW2 + 16 * c, v);
      if (lane < 16)
        for (int i = 0; i < 16; i++) out[kPW2 + m * 64 + 16 * c + i] = v[i];
      tc::tmem_ld16(tb + lane_off + cW3 + 16 * c, v);
      if (lane < 16)
        for (int i = 0; i < 16; i++) out[kPW3 + m * 64 + 16 * c + i] = v[i];
    }
    // dW4^T: row m = input, columns = outputs
    tc::tmem_ld16(tb + lane_off + cW4, v);
    if (lane < 16)
      for (int o = 0; o < kMlpOut; o++) out[kPW4 + o * 64 + m] = v[o];
  } else {
    for (int i = r; i < kPB4; i += 128) out[i] = 0.f;
  }
  // db4 and the loss: block sums in a fixed order
#pragma unroll
  for (int j = 0; j < kMlpOut; j++) {
    float s = db4[j];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) redf[warp * 8 + j] = s;
  }
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
  if (lane == 0) redd[warp] = lsum;
  tc::fence_before_sync();
  __syncthreads();
  if (r < kMlpOut) out[kPB4 + r] = redf[r] + redf[8 + r] + redf[16 + r] + redf[24 + r];
  if (r == 0) lpart[blockIdx.x] = redd[0] + redd[1] + redd[2] + redd[3];
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tb, 512);
  }
}

// Gradient = sum of the per-CTA partials in CTA order (times 1; the
// 1/(n*6) factor is inside), then optionally one Adam step on the f32
// master parameters, refreshing the bf16 tiles and f32 biases of `dev`.
static __global__ void k_mlp_reduce_adam(const float* __restrict__ part, int nparts, float* __restrict__ grad,
                                  float* __restrict__ master, float* __restrict__ m1, float* __restrict__ m2,
                                  MlpDev* __restrict__ dev, int adam, float lr, float b1, float b2, float eps,
                                  float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kMlpNParam) return;
  float g = 0.f;
  for (int c = 0; c < nparts; c++) g += part[(size_t)c * kMlpNParam + i];
  grad[i] = g;
  if (!adam) return;
  const float mm = b1 * m1[i] + (1.f - b1) * g;
  const float vv = b2 * m2[i] + (1.f - b2) * g * g;
  m1[i] = mm;
  m2[i] = vv;
  const float w = master[i] - lr * (mm / c1) / (sqrtf(vv / c2) + eps);
  master[i] = w;
  const __nv_bfloat16 wb = __float2bfloat16_rn(w);
  if (i < kPB1) { const int o = i / 11, k = i % 11; dev->w1[tc::tile_elem(o, k, 16)] = wb; }
  else if (i < kPW2) dev->b1[i - kPB1] = w;
  else if (i < kPB2) { const int j = i - kPW2; dev->w2[tc::tile_elem(j / 64, j % 64, 64)] = wb; }
  else if (i < kPW3) dev->b2[i - kPB2] = w;
  else if (i < kPB3) { const int j = i - kPW3; dev->w3[tc::tile_elem(j / 64, j % 64, 64)] = wb; }
  else if (i < kPW4) dev->b3[i - kPB3] = w;
  else if (i < kPB4) { const int j = i - kPW4; dev->w4[tc::tile_elem(j / 64, j % 64, 64)] = wb; }
  else dev->b4[i - kPB4] = w;
}

}  // namespace les

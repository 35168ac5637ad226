// les_tma.cuh -- L2 prefetch of y-column tiles by the tensor memory
// accelerator (TMA).
//
// The y-column transforms (k_y_inverse, k_y_forward) read one column tile
// per CTA: TC complex columns of an x-spectral array, every row of one level
// (NS spectral rows, or M = 3NS/2 padded rows), 64-byte row segments with a
// row stride of KX complex values.  A CTA loads its tile, transforms it and
// stores the result, so DRAM idles while the resident CTAs compute.  Here
// thread 0 of each CTA first asks the TMA to bring the tile of the CTA
// `pdist` blocks later in launch order (about one resident wave ahead) into
// L2 (cp.async.bulk.prefetch.tensor): that tile's DRAM reads overlap this
// wave's transforms, and its CTA later finds its columns in L2.  A prefetch
// has no destination in shared memory and nothing waits on it; the results
// are those of the kernels without it (checked bit for bit on B200 at
// 512x512x256: FP64 k_y_forward 3.65 -> 3.44 ms, k_y_inverse 2.11 -> 2.00 ms
// per stage; FP32 about 1%; two or more waves ahead was slower than one).
//
// The arrays are described to the TMA as 2-D tensors of real elements:
// dim 0 the 2KX reals of one row, dim 1 all rows of all levels.  A tile is
// NB boxes of 2TC x BR elements, BR = rows / NB <= 256.
//
// tma::prefetch_l2 is the untiled form (one contiguous range), used by
// k_row_fused for the rows its next sliding-window level reads.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cstring>
#include <mutex>
#include "fft_core.cuh"

namespace les {

namespace tma {
// Prefetch into L2 the box at element coordinates (x, y) of `map`.
__device__ __forceinline__ void prefetch_2d(const CUtensorMap* map, int x, int y) {
  asm volatile("cp.async.bulk.prefetch.tensor.2d.L2.global.tile [%0, {%1, %2}];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(x), "r"(y)
               : "memory");
}
// Prefetch into L2 `bytes` contiguous bytes at `p` (16-byte aligned, a
// multiple of 16 bytes).
__device__ __forceinline__ void prefetch_l2(const void* p, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(reinterpret_cast<uint64_t>(p)), "r"(bytes)
               : "memory");
}
}  // namespace tma

// Tensor maps of up to eight column-tile arrays.
struct ColMaps {
  CUtensorMap m[8];
};

// Box geometry of a tile of ROWS rows and TC complex columns.
template <class T, int ROWS, int TC> struct ColBox {
  static constexpr int NB = (ROWS + 255) / 256;  // boxes per tile
  static constexpr int BR = ROWS / NB;           // rows per box
  // the boxes tile the column exactly and a tile's column offset is a
  // multiple of 16 bytes (the TMA's rule for the innermost coordinate)
  static constexpr bool ok = (BR * NB == ROWS) && ((TC * sizeof(cx<T>)) % 16 == 0) && (2 * TC <= 256);
};

// Launch-order coordinates of the block `ahead` blocks after this one, or
// false past the end of the grid.
__device__ __forceinline__ bool block_ahead(unsigned ahead, unsigned& bx, unsigned& by, unsigned& bz) {
  const unsigned L = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z) + ahead;
  bx = L % gridDim.x;
  const unsigned r = L / gridDim.x;
  by = r % gridDim.y;
  bz = r / gridDim.y;
  return bz < gridDim.z;
}

// Thread 0's prefetch of the tile (column group cg of array q, rows
// [row0, row0 + ROWS)) of the block `pdist` blocks ahead; `tile` maps that
// block's launch coordinates to (q, cg, row0) and returns false for a block
// that reads nothing.
template <class T, int ROWS, int TC, class TileF>
__device__ __forceinline__ void prefetch_tile_ahead(const ColMaps& maps, unsigned pdist, TileF tile) {
  using B = ColBox<T, ROWS, TC>;
  if constexpr (B::ok) {
    if (threadIdx.x != 0 || pdist == 0) return;
    unsigned bx, by, bz;
    int q, cg, row0;
    if (!block_ahead(pdist, bx, by, bz) || !tile(bx, by, bz, q, cg, row0)) return;
#pragma unroll
    for (int r = 0; r < B::NB; r++) tma::prefetch_2d(&maps.m[q], 2 * cg * TC, row0 + r * B::BR);
  }
}

// Host side: cuTensorMapEncodeTiled through the runtime's driver entry
// point (no link-time dependency on libcuda).
inline PFN_cuTensorMapEncodeTiled_v12000 tma_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// Tensor maps of n <= 8 arrays of `levels` x ROWS rows of KX complex values,
// boxes of TC columns x BR rows.  Returns false when the geometry, an
// address or the driver does not allow them (the caller then launches with
// pdist = 0, which prefetches nothing).
template <class T, int ROWS, int TC>
inline bool make_col_maps(ColMaps& out, void* const* X, int n, int KX, int levels) {
  using B = ColBox<T, ROWS, TC>;
  std::memset(&out, 0, sizeof(out));
  if (!B::ok || n > 8) return false;
  PFN_cuTensorMapEncodeTiled_v12000 enc = tma_encoder();
  if (!enc) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)2 * KX, (cuuint64_t)levels * ROWS};
  const cuuint64_t strides[1] = {(cuuint64_t)2 * KX * sizeof(T)};
  const cuuint32_t box[2] = {(cuuint32_t)(2 * TC), (cuuint32_t)B::BR};
  const cuuint32_t estr[2] = {1, 1};
  if (strides[0] % 16 != 0) return false;
  for (int q = 0; q < n; q++) {
    if (reinterpret_cast<uintptr_t>(X[q]) % 16 != 0) return false;
    CUresult r = enc(&out.m[q], sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                     X[q], dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return false;
  }
  return true;
}

}  // namespace les

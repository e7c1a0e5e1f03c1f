// Host side of the tile kernels' TMA staging: tensor maps of float64 state
// arrays [nf][nx][ny] with the padded-tile box of k_flux2d.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#ifndef JB_TILE_TMA
#define JB_TILE_TMA 1  // 0: the tile kernels load their padded tiles with plain loads
#endif

namespace jb {

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against libcuda); null when the driver does not provide it.
inline EncodeTiledFn encode_tiled_fn() {
  static EncodeTiledFn fn = nullptr;
  static bool looked = false;
  if (!looked) {
    looked = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// Tensor map of base[nf][nx][ny] (float64, C order) with a box of
// box_y x box_x x nf elements (innermost first).  TMA needs a 16-byte aligned
// base and row pitch (ny even), and a box row of a multiple of 16 bytes;
// false (map zeroed) when any of these fails, and the kernel then loads its
// tile with plain loads.
inline bool tile_map(CUtensorMap* map, const double* base, int nf, int nx, int ny, int box_y, int box_x) {
  std::memset(map, 0, sizeof(*map));
  if (!JB_TILE_TMA || !base || (reinterpret_cast<uintptr_t>(base) & 15) || (ny & 1) || ((box_y * 8) & 15) ||
      nf > 256 || box_x > 256 || box_y > 256)
    return false;
  EncodeTiledFn enc = encode_tiled_fn();
  if (!enc) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)ny, (cuuint64_t)nx, (cuuint64_t)nf};
  const cuuint64_t strides[2] = {(cuuint64_t)ny * 8, (cuuint64_t)nx * ny * 8};
  const cuuint32_t box[3] = {(cuuint32_t)box_y, (cuuint32_t)box_x, (cuuint32_t)nf};
  const cuuint32_t estride[3] = {1, 1, 1};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double*>(base), dims, strides, box, estride,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace jb

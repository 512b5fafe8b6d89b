// Host side of the TMA column tiles: tensor maps over the intermediate buffers,
// encoded with the driver's cuTensorMapEncodeTiled (reached through the runtime's
// driver entry point, so the library does not link libcuda) and cached.
#include <cudaTypedefs.h>

#include <cstring>
#include <map>
#include <mutex>
#include <tuple>

#include "tma.cuh"

namespace fwix {

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

}  // namespace

cudaError_t tile_map(CUtensorMap* out, const void* base, int nx, int ny, long long nz, int box_rows, int box_cols) {
  using Key = std::tuple<const void*, int, int, long long, int, int>;
  static std::mutex mu;
  static std::map<Key, CUtensorMap> cache;
  const Key key{base, nx, ny, nz, box_rows, box_cols};
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(key);
    if (it != cache.end()) {
      *out = it->second;
      return cudaSuccess;
    }
  }
  auto fn = encode_fn();
  if (!fn || nz < 1 || nx < 1 || ny < 1 || box_rows < 1 || box_rows > 256 || (nx % 2) != 0 ||
      (box_cols != 16 && box_cols != 8) || ((uintptr_t)base & 15) != 0)
    return cudaErrorInvalidValue;
  CUtensorMap m;
  std::memset(&m, 0, sizeof(m));
  const cuuint64_t dims[3] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz};
  const cuuint64_t strides[2] = {(cuuint64_t)nx * 8, (cuuint64_t)nx * (cuuint64_t)ny * 8};
  const cuuint32_t box[3] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows, 1};
  const cuuint32_t elem[3] = {1, 1, 1};
  const CUresult r = fn(&m, CU_TENSOR_MAP_DATA_TYPE_INT64, 3, const_cast<void*>(base), dims, strides, box, elem,
                        CU_TENSOR_MAP_INTERLEAVE_NONE,
                        box_cols == 16 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
  std::lock_guard<std::mutex> lock(mu);
  cache[key] = m;
  *out = m;
  return cudaSuccess;
}

cudaError_t qtab_map(CUtensorMap* out, const void* base, int pny, int pnx, long long nslices, int box_cols) {
  using Key = std::tuple<const void*, int, int, long long, int>;
  static std::mutex mu;
  static std::map<Key, CUtensorMap> cache;
  const Key key{base, pny, pnx, nslices, box_cols};
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(key);
    if (it != cache.end()) {
      *out = it->second;
      return cudaSuccess;
    }
  }
  auto fn = encode_fn();
  if (!fn || nslices < 1 || pnx < box_cols || pny < 2 || pny > 256 || (pny % 2) != 0 || box_cols < 1 ||
      box_cols > 256 || ((uintptr_t)base & 15) != 0)
    return cudaErrorInvalidValue;
  CUtensorMap m;
  std::memset(&m, 0, sizeof(m));
  const cuuint64_t dims[3] = {(cuuint64_t)pny, (cuuint64_t)pnx, (cuuint64_t)nslices};
  const cuuint64_t strides[2] = {(cuuint64_t)pny * 8, (cuuint64_t)pny * (cuuint64_t)pnx * 8};
  const cuuint32_t box[3] = {(cuuint32_t)pny, (cuuint32_t)box_cols, 1};
  const cuuint32_t elem[3] = {1, 1, 1};
  const CUresult r = fn(&m, CU_TENSOR_MAP_DATA_TYPE_INT64, 3, const_cast<void*>(base), dims, strides, box, elem,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
  std::lock_guard<std::mutex> lock(mu);
  cache[key] = m;
  *out = m;
  return cudaSuccess;
}

}  // namespace fwix

// cimx_tma.cu — host side of the TMA tile loads: tensor-map encoding through
// the driver entry point, and the per-device status word that bounded
// device-side waits report into.
#include <cudaTypedefs.h>

#include <mutex>

#include "cimx_common.cuh"
#include "cimx_internal.h"
#include "cimx_tma.cuh"

namespace cimx {
namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

std::mutex g_status_mu;
int* g_status[64] = {nullptr};

}  // namespace

bool make_tensor_map_3d(CUtensorMap* map, const void* base, int dtype, long long X, long long Y,
                        long long Z, int box_x, int box_y, bool swizzle128) {
  auto fn = encode_fn();
  if (!fn) return false;
  CUtensorMapDataType t;
  switch (dtype) {
    case DT_F32: t = CU_TENSOR_MAP_DATA_TYPE_FLOAT32; break;
    case DT_U16: t = CU_TENSOR_MAP_DATA_TYPE_UINT16; break;
    case DT_U8: t = CU_TENSOR_MAP_DATA_TYPE_UINT8; break;
    default: return false;
  }
  const long long es = dtype_size(dtype);
  if ((reinterpret_cast<uintptr_t>(base) & 15) != 0) return false;
  if ((X * es) % 16 != 0 || box_x * es % 16 != 0) return false;
  if (swizzle128 && box_x * es > 128) return false;
  if (box_x > 256 || box_y > 256 || X >= (1ll << 32) || Y >= (1ll << 32) || Z >= (1ll << 32))
    return false;
  const cuuint64_t dims[3] = {(cuuint64_t)X, (cuuint64_t)Y, (cuuint64_t)Z};
  const cuuint64_t strides[2] = {(cuuint64_t)(X * es), (cuuint64_t)(X * Y * es)};
  if (strides[1] >= (1ull << 40)) return false;
  const cuuint32_t box[3] = {(cuuint32_t)box_x, (cuuint32_t)box_y, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(map, t, 3, const_cast<void*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE,
                  swizzle128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

int* device_status_word() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> g(g_status_mu);
  if (!g_status[dev]) {
    int* p = nullptr;
    if (cudaMalloc(&p, sizeof(int)) != cudaSuccess) return nullptr;
    cudaMemset(p, 0, sizeof(int));
    g_status[dev] = p;
  }
  return g_status[dev];
}

}  // namespace cimx

using namespace cimx;

extern "C" int cimx_device_status(int clear) {
  int* p = device_status_word();
  if (!p) return fail(CIMX_E_CUDA, "no device status word");
  int v = 0;
  cudaError_t e = cudaMemcpy(&v, p, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "status read");
  if (clear && v != 0) cudaMemset(p, 0, sizeof(int));
  return v;
}

// Host side of the TMA tile loads: tensor maps encoded through the driver's
// cuTensorMapEncodeTiled (found with cudaGetDriverEntryPoint, so the library needs no link
// against the driver library), cached by what they encode.
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>

#include "lsb_tma.cuh"

namespace lsb {

namespace {

using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                              const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeFn encoder() {
    static EncodeFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return (EncodeFn) nullptr;
        }
        return reinterpret_cast<EncodeFn>(p);
    }();
    return fn;
}

using Key = std::tuple<const void*, uint64_t, uint64_t, uint64_t, uint32_t, uint32_t>;
std::mutex g_mu;
std::map<Key, CUtensorMap> g_maps;

}  // namespace

bool tmap_f64_3d(CUtensorMap* out, const void* base, uint64_t nx, uint64_t rows, uint64_t nz, uint32_t box_x,
                 uint32_t box_rows) {
    const Key key{base, nx, rows, nz, box_x, box_rows};
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_maps.find(key);
    if (it != g_maps.end()) {
        *out = it->second;
        return true;
    }
    EncodeFn enc = encoder();
    if (!enc || box_x * 8 != 128 || box_rows == 0 || box_rows > 256 || (reinterpret_cast<uintptr_t>(base) & 15) ||
        (nx * 8) % 16)
        return false;
    const cuuint64_t dims[3] = {nx, rows, nz};
    const cuuint64_t strides[2] = {nx * 8, rows * nx * 8};  // bytes, of dims 1 and 2
    const cuuint32_t box[3] = {box_x, box_rows, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUtensorMap m;
    std::memset(&m, 0, sizeof(m));
    const CUresult r = enc(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<void*>(base), dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return false;
    g_maps.emplace(key, m);
    *out = m;
    return true;
}

// row maps: [rows][nx] of 4- or 8-byte elements, box of box_x x 1, no swizzle
using RowKey = std::tuple<const void*, uint64_t, uint64_t, uint32_t, uint32_t>;
std::map<RowKey, CUtensorMap> g_rowmaps;

bool tmap_rows(CUtensorMap* out, const void* base, uint32_t elem_bytes, uint64_t nx, uint64_t rows, uint32_t box_x) {
    const RowKey key{base, nx, rows, box_x, elem_bytes};
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_rowmaps.find(key);
    if (it != g_rowmaps.end()) {
        *out = it->second;
        return true;
    }
    EncodeFn enc = encoder();
    if (!enc || (elem_bytes != 4 && elem_bytes != 8) || box_x == 0 || box_x > 256 || (box_x * elem_bytes) % 16 ||
        nx % box_x || (reinterpret_cast<uintptr_t>(base) & 15) || (nx * elem_bytes) % 16)
        return false;
    const cuuint64_t dims[2] = {nx, rows};
    const cuuint64_t strides[1] = {nx * elem_bytes};
    const cuuint32_t box[2] = {box_x, 1};
    const cuuint32_t estr[2] = {1, 1};
    CUtensorMap m;
    std::memset(&m, 0, sizeof(m));
    const CUresult r = enc(&m, elem_bytes == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                           const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return false;
    g_rowmaps.emplace(key, m);
    *out = m;
    return true;
}

}  // namespace lsb

// Host side of the TMA copies: tensor maps encoded through the driver's
// cuTensorMapEncodeTiled, reached via cudaGetDriverEntryPoint so that the
// library does not link libcuda directly.
#include <cudaTypedefs.h>

#include <mutex>

#include "mr_internal.h"
#include "tma.cuh"

namespace {
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::once_flag g_once;
}  // namespace

int mr_tma_encode_3d(CUtensorMap *map, const void *base, const uint64_t dim[3],
                     const uint64_t stride_bytes[2], const uint32_t box[3]) {
    std::call_once(g_once, [] {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
        cudaGetLastError();
    });
    if (!g_encode) MR_FAIL(MR_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    const cuuint64_t gdim[3] = {dim[0], dim[1], dim[2]};
    const cuuint64_t gstr[2] = {stride_bytes[0], stride_bytes[1]};
    const cuuint32_t bdim[3] = {box[0], box[1], box[2]};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = g_encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<void *>(base),
                                gdim, gstr, bdim, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        MR_FAIL(MR_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d): extents %llu x %llu x %llu, box "
                "%u x %u x %u", (int)r, (unsigned long long)dim[0], (unsigned long long)dim[1],
                (unsigned long long)dim[2], box[0], box[1], box[2]);
    return MR_SUCCESS;
}

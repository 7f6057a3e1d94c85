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

int mr_tma_encode(CUtensorMap *map, const void *base, int rank, const uint64_t *dim,
                  const uint64_t *stride_bytes, const uint32_t *box) {
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
    MR_REQUIRE(rank >= 1 && rank <= 5, "tensor map rank %d outside [1, 5]", rank);
    cuuint64_t gdim[5], gstr[4];
    cuuint32_t bdim[5], estr[5];
    for (int d = 0; d < rank; ++d) {
        gdim[d] = dim[d];
        bdim[d] = box[d];
        estr[d] = 1;
        if (d + 1 < rank) gstr[d] = stride_bytes[d];
    }
    const CUresult r = g_encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, (cuuint32_t)rank,
                                const_cast<void *>(base), gdim, gstr, bdim, estr,
                                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        MR_FAIL(MR_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d): rank %d, extents %llu x %llu "
                "x ..., box %u x %u x ...", (int)r, rank, (unsigned long long)dim[0],
                (unsigned long long)(rank > 1 ? dim[1] : 1), box[0], rank > 1 ? box[1] : 1u);
    return MR_SUCCESS;
}

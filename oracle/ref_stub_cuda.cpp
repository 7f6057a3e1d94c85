// Link stub for building the reference's CUDA apply path without its
// mr_calc_toep.cu (which needs cufinufft, absent here). TEST INFRASTRUCTURE
// ONLY. The reference's mr_calc_mask.cu calls mr_toep_push_device (defined
// in src/cuda/mr_calc_toep.cu:76-91 of the reference): make the configured
// device current and report the previous one, or -1 when nothing changed.
#include <cuda_runtime.h>

#include "mr_aha/mr_aha.h"

int mr_toep_push_device(const mr_config *cfg, int *prev) {
    *prev = -1;
    if (cfg->gpu_device_id < 0) return MR_SUCCESS;
    int cur = 0;
    if (cudaGetDevice(&cur) != cudaSuccess) return MR_ERR_CUDA;
    if (cur != cfg->gpu_device_id) {
        if (cudaSetDevice(cfg->gpu_device_id) != cudaSuccess) return MR_ERR_CUDA;
        *prev = cur;
    }
    return MR_SUCCESS;
}

// Allocation-free variant of the one-shot apply, mr_b200_aha_toeplitz_noalloc.
//
// Who needs it: callers that cannot call cudaMalloc. A reconstruction that
// runs inside a host application whose GPU memory is owned by its own pool
// (MATLAB's gpuArray allocator, a framework's caching allocator that has
// reserved the free memory, a serving process with a fixed budget) may see
// an allocation fail or fragment that pool; a real-time loop on a scanner
// cannot afford the device-wide synchronisation that cudaMalloc and cudaFree
// imply, nor an out-of-memory error half way through a scan. mr_aha_toeplitz
// and mr_aha_plan_create allocate their work buffers and FFT tables; this
// entry point takes them from one fixed array that the library reserves on
// each GPU it is loaded on, so the caller only provides inputs and outputs.
//
// The array: MR_B200_NOALLOC_SCRATCH_BYTES (32 MiB) of device memory, held on
// every GPU that loads the library until the process exits. Operators whose
// work space (FFT tables, masked grid map and the per-coil-group
// intermediates) does not fit even one coil at a time are rejected with
// MR_ERR_UNSUPPORTED and a message giving the bytes needed.
//
// Sharing: every call uses the same array and it keeps the previous call's
// contents. Each call rewrites every part it reads before reading it (FFT
// tables, grid map, intermediates), so nothing has to start at zero, but two
// calls that overlap on the GPU (different streams or host threads without
// ordering between them) race on the array and give wrong results.
//
// Set-up: the device address of the array is looked up once per device with
// cudaGetSymbolAddress, on that device, by the first call made there; make
// that first call before capturing any stream.
#include <cstring>
#include <mutex>

#include "engine.h"
#include "mr_aha/mr_aha_b200.h"

static __device__ __align__(256) unsigned char g_noalloc_scratch[MR_B200_NOALLOC_SCRATCH_BYTES];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_mu;
char *g_addr[kMaxDevices] = {nullptr};

// Device address of the scratch array on the current device.
int scratch_address(char **out) {
    int dev = 0;
    MR_CUDA_TRY(cudaGetDevice(&dev));
    MR_REQUIRE(dev >= 0 && dev < kMaxDevices, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) {
            cudaGetLastError();
            MR_FAIL(MR_ERR_CUDA, "cudaGetSymbolAddress of the scratch array failed on device %d: %s",
                    dev, cudaGetErrorString(e));
        }
        g_addr[dev] = (char *)p;
    }
    *out = g_addr[dev];
    return MR_SUCCESS;
}
}  // namespace

extern "C" int mr_b200_aha_toeplitz_noalloc(const mr_config *cfg, const mr_complex *d_x,
                                            const mr_complex *d_SEs,
                                            const mr_complex *d_phi2_toep,
                                            const int64_t *d_mask, mr_complex *d_AhAx) {
    mr_clear_error();
    MR_REQUIRE(cfg != nullptr, "mr_b200_aha_toeplitz_noalloc: cfg is NULL");
    MR_REQUIRE(d_x != nullptr, "mr_b200_aha_toeplitz_noalloc: d_x is NULL");
    MR_REQUIRE(d_SEs != nullptr, "mr_b200_aha_toeplitz_noalloc: d_SEs is NULL");
    MR_REQUIRE(d_phi2_toep != nullptr, "mr_b200_aha_toeplitz_noalloc: d_phi2_toep is NULL");
    MR_REQUIRE(d_AhAx != nullptr, "mr_b200_aha_toeplitz_noalloc: d_AhAx is NULL");
    MR_REQUIRE((const void *)d_AhAx != (const void *)d_x,
               "mr_b200_aha_toeplitz_noalloc: d_AhAx must not alias d_x");
    if (cfg->is_masked)
        MR_REQUIRE(d_mask != nullptr,
                   "mr_b200_aha_toeplitz_noalloc: d_mask is required when is_masked is set");
    int prev = -1;
    int rc = mr_push_device(cfg, &prev);
    if (rc != MR_SUCCESS) return rc;
    char *scratch = nullptr;
    rc = scratch_address(&scratch);
    alignas(64) unsigned char storage[8192];
    if (rc == MR_SUCCESS && mr_plan_struct_size() > sizeof(storage)) {
        rc = MR_ERR_INTERNAL;
        mr_set_error("plan struct larger than its host storage");
    }
    size_t needed = 0;
    if (rc == MR_SUCCESS)
        rc = mr_plan_setup_in_scratch(cfg, scratch, MR_B200_NOALLOC_SCRATCH_BYTES, storage,
                                      &needed);
    if (rc == MR_SUCCESS) {
        mr_kernel_ref K;
        memset(&K, 0, sizeof(K));
        K.data = d_phi2_toep;
        K.kf = MR_KF_F32;
        rc = mr_plan_execute_k((mr_aha_plan)storage, reinterpret_cast<const float2 *>(d_x),
                               reinterpret_cast<const float2 *>(d_SEs), K, d_mask,
                               reinterpret_cast<float2 *>(d_AhAx), (cudaStream_t)cfg->stream);
    }
    mr_pop_device(prev);
    return rc;
}

// Configuration defaults and validation, derived sizes, status strings and
// the thread-local error buffer. Semantics follow the reference's
// src/common/mr_config.cpp:29-238 (the validation rules and default values
// are part of the ABI contract); the code is this library's own.
#include <cuda_runtime.h>

#include <cstring>
#include <string>

#include "mr_internal.h"
#include "mr_aha/mr_aha_b200.h"

namespace {
constexpr int kErrLen = 512;
thread_local char g_err[kErrLen] = {0};
thread_local std::string g_trace;
}  // namespace

thread_local int mr_trace_on = 0;

void mr_trace_note(const char *fmt, ...) {
    char line[160];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(line, sizeof(line), fmt, ap);
    va_end(ap);
    g_trace += line;
    g_trace += '\n';
}

extern "C" int mr_b200_trace_launches(int enable) {
    mr_clear_error();
    if (enable) g_trace.clear();
    mr_trace_on = enable ? 1 : 0;
    return MR_SUCCESS;
}

extern "C" int64_t mr_b200_trace_read(char *buf, size_t cap) {
    if (buf && cap > 0) {
        const size_t n = g_trace.size() < cap - 1 ? g_trace.size() : cap - 1;
        std::memcpy(buf, g_trace.data(), n);
        buf[n] = '\0';
    }
    return (int64_t)g_trace.size();
}

void mr_set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, kErrLen, fmt, ap);
    va_end(ap);
}

void mr_clear_error() {
    g_err[0] = '\0';
    (void)cudaGetLastError();
}

extern "C" const char *mr_last_error(void) { return g_err; }

extern "C" const char *mr_backend(void) { return "cuda"; }

extern "C" int mr_version(void) { return 1 * 10000 + 0 * 100 + 0; }

extern "C" const char *mr_status_string(int status) {
    switch (status) {
        case MR_SUCCESS: return "success";
        case MR_ERR_INVALID_ARG: return "invalid argument";
        case MR_ERR_INVALID_CONFIG: return "invalid configuration";
        case MR_ERR_ALLOC: return "GPU memory allocation failed";
        case MR_ERR_CUDA: return "CUDA runtime error";
        case MR_ERR_CUFFT: return "cuFFT error";
        case MR_ERR_CUFINUFFT: return "cufinufft error";
        case MR_ERR_UNSUPPORTED: return "unsupported configuration";
        case MR_ERR_INTERNAL: return "internal error";
        case MR_ERR_METAL: return "Metal error";
        case MR_ERR_VKFFT: return "VkFFT error";
        default: return "unknown status";
    }
}

extern "C" int mr_config_defaults(mr_config *cfg, mr_traj_type traj_type) {
    mr_clear_error();
    MR_REQUIRE(cfg != nullptr, "mr_config_defaults: cfg is NULL");
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->traj_type = traj_type;
    cfg->n_spatial = traj_type == MR_TRAJ_2D ? 2 : 3;
    for (int d = 0; d < 3; ++d) {
        cfg->n_dim[d] = 1;
        cfg->phi2_dim[d] = 1;
    }
    cfg->L = 1;
    cfg->triangulation = MR_TRI_LOWER;
    cfg->n_coils = 1;
    cfg->eps = 1e-6;
    cfg->gpu_device_id = 0;
    cfg->stream = nullptr;
    cfg->mem_fraction = 0.5;
    cfg->mask_radius = MR_DEFAULT_MASK_RADIUS;
    return MR_SUCCESS;
}

extern "C" int mr_config_validate(const mr_config *cfg) {
    mr_clear_error();
    MR_REQUIRE(cfg != nullptr, "mr_config_validate: cfg is NULL");
    const int tt = (int)cfg->traj_type;
    MR_REQUIRE_CFG(tt == MR_TRAJ_2D || tt == MR_TRAJ_3D || tt == MR_TRAJ_STACK,
                   "traj_type must be one of MR_TRAJ_2D, MR_TRAJ_3D, MR_TRAJ_STACK");
    const int want = tt == MR_TRAJ_2D ? 2 : 3;
    MR_REQUIRE_CFG(cfg->n_spatial == want,
                   "n_spatial is %d but trajectory type requires %d",
                   cfg->n_spatial, want);
    for (int d = 0; d < 3; ++d) {
        MR_REQUIRE_CFG(cfg->n_dim[d] >= 1, "n_dim[%d] = %d must be >= 1", d,
                       cfg->n_dim[d]);
        MR_REQUIRE_CFG(cfg->phi2_dim[d] >= 1, "phi2_dim[%d] = %d must be >= 1", d,
                       cfg->phi2_dim[d]);
        if (d >= cfg->n_spatial)
            MR_REQUIRE_CFG(cfg->n_dim[d] == 1 && cfg->phi2_dim[d] == 1,
                           "n_dim[%d] and phi2_dim[%d] must be 1 for a %dD "
                           "trajectory",
                           d, d, cfg->n_spatial);
        MR_REQUIRE_CFG(cfg->phi2_dim[d] >= cfg->n_dim[d],
                       "phi2_dim[%d] = %d must not be smaller than n_dim[%d] = %d",
                       d, cfg->phi2_dim[d], d, cfg->n_dim[d]);
    }
    if (tt == MR_TRAJ_STACK)
        MR_REQUIRE_CFG(cfg->phi2_dim[2] == cfg->n_dim[2],
                       "for MR_TRAJ_STACK, phi2_dim[2] (Mz = %d) must equal "
                       "n_dim[2] (Nz = %d)",
                       cfg->phi2_dim[2], cfg->n_dim[2]);
    MR_REQUIRE_CFG(cfg->L >= 1, "L = %d must be >= 1", cfg->L);
    MR_REQUIRE_CFG(cfg->n_coils >= 1, "n_coils = %d must be >= 1", cfg->n_coils);
    MR_REQUIRE_CFG(cfg->triangulation == MR_TRI_LOWER ||
                       cfg->triangulation == MR_TRI_UPPER,
                   "triangulation must be MR_TRI_LOWER or MR_TRI_UPPER");
    MR_REQUIRE_CFG(cfg->eps > 0.0 && cfg->eps < 1.0, "eps = %g must lie in (0, 1)",
                   cfg->eps);
    MR_REQUIRE_CFG(cfg->mask_radius >= 0, "mask_radius = %d must be >= 0",
                   cfg->mask_radius);
    if (cfg->is_masked) {
        const int64_t pad = mr_pad_size(cfg);
        MR_REQUIRE_CFG(cfg->num_masked > 0,
                       "num_masked = %lld must be > 0 when is_masked is set",
                       (long long)cfg->num_masked);
        MR_REQUIRE_CFG(cfg->num_masked <= pad,
                       "num_masked = %lld exceeds the upsampled grid size %lld",
                       (long long)cfg->num_masked, (long long)pad);
    }
    return MR_SUCCESS;
}

extern "C" int64_t mr_num_tri(int L) {
    return L <= 0 ? 0 : (int64_t)L * (L + 1) / 2;
}

extern "C" int64_t mr_image_size(const mr_config *cfg) {
    if (!cfg) return 0;
    return (int64_t)cfg->n_dim[0] * cfg->n_dim[1] * cfg->n_dim[2];
}

extern "C" int64_t mr_pad_size(const mr_config *cfg) {
    if (!cfg) return 0;
    return (int64_t)cfg->phi2_dim[0] * cfg->phi2_dim[1] * cfg->phi2_dim[2];
}

extern "C" int64_t mr_phi2_toep_size(const mr_config *cfg) {
    if (!cfg) return 0;
    return (cfg->is_masked ? cfg->num_masked : mr_pad_size(cfg)) * mr_num_tri(cfg->L);
}

extern "C" int64_t mr_x_size(const mr_config *cfg) {
    if (!cfg) return 0;
    return mr_image_size(cfg) * cfg->L;
}

extern "C" int64_t mr_se_size(const mr_config *cfg) {
    if (!cfg) return 0;
    return mr_image_size(cfg) * cfg->n_coils;
}

void mr_geom_from_config(const mr_config *cfg, mr_geom *g) {
    std::memset(g, 0, sizeof(*g));
    for (int d = 0; d < 3; ++d) {
        g->n[d] = cfg->n_dim[d];
        g->m[d] = cfg->phi2_dim[d];
        g->cn[d] = cfg->n_dim[d] / 2;
        g->cm[d] = cfg->phi2_dim[d] / 2;
    }
    g->L = cfg->L;
    g->upper = cfg->triangulation == MR_TRI_UPPER ? 1 : 0;
    g->vimg = mr_image_size(cfg);
    g->vpad = mr_pad_size(cfg);
}

int mr_env_int(const char *name, int dflt) {
    const char *e = std::getenv(name);
    if (!e || !e[0]) return dflt;
    char *end = nullptr;
    long v = std::strtol(e, &end, 10);
    if (end == e) return dflt;
    return (int)v;
}

int mr_push_device(const mr_config *cfg, int *prev) {
    *prev = -1;
    if (cfg->gpu_device_id < 0) return MR_SUCCESS;
    int cur = 0;
    MR_CUDA_TRY(cudaGetDevice(&cur));
    if (cur != cfg->gpu_device_id) {
        MR_CUDA_TRY(cudaSetDevice(cfg->gpu_device_id));
        *prev = cur;
    }
    return MR_SUCCESS;
}

void mr_pop_device(int prev) {
    if (prev >= 0) cudaSetDevice(prev);
}

int mr_memory_budget(const mr_config *cfg, size_t *budget) {
    size_t free_b = 0, total_b = 0;
    MR_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
    double f = cfg->mem_fraction;
    if (!(f > 0.0)) f = 0.5;
    if (f > 0.95) f = 0.95;
    *budget = (size_t)(f * (double)free_b);
    return MR_SUCCESS;
}

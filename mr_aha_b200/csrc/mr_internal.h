// Internal host-side helpers shared by every translation unit of
// libmr_aha_c.so: error recording, argument-check macros, the geometry
// descriptor handed to kernels by value, and small utilities.
#pragma once

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>

#include "mr_aha/mr_aha.h"

// Record a printf-style message in the calling thread's error buffer.
void mr_set_error(const char *fmt, ...);
// Clear the thread's error buffer and the CUDA runtime's sticky-free last error.
void mr_clear_error();

#define MR_FAIL(status, ...)        \
    do {                            \
        mr_set_error(__VA_ARGS__);  \
        return (status);            \
    } while (0)

#define MR_REQUIRE(cond, ...)                                   \
    do {                                                        \
        if (!(cond)) MR_FAIL(MR_ERR_INVALID_ARG, __VA_ARGS__);  \
    } while (0)

#define MR_REQUIRE_CFG(cond, ...)                                  \
    do {                                                           \
        if (!(cond)) MR_FAIL(MR_ERR_INVALID_CONFIG, __VA_ARGS__);  \
    } while (0)

#define MR_CUDA_TRY(call)                                                       \
    do {                                                                        \
        cudaError_t mr_e_ = (call);                                             \
        if (mr_e_ != cudaSuccess) {                                             \
            cudaGetLastError();                                                 \
            MR_FAIL(MR_ERR_CUDA, "%s failed at %s:%d: %s", #call, __FILE__,     \
                    __LINE__, cudaGetErrorString(mr_e_));                       \
        }                                                                       \
    } while (0)

// Launch trace of the calling thread (mr_b200_trace_launches): while it is
// on, every launch appends one line naming the kernel (the specialised
// launchers name their template arguments).
extern thread_local int mr_trace_on;
void mr_trace_note(const char *fmt, ...);

#define MR_LAUNCH_ERR(name)                                                     \
    do {                                                                        \
        cudaError_t mr_e_ = cudaGetLastError();                                 \
        if (mr_e_ != cudaSuccess)                                               \
            MR_FAIL(MR_ERR_CUDA, "kernel %s failed to launch: %s", name,        \
                    cudaGetErrorString(mr_e_));                                 \
    } while (0)

#define MR_LAUNCH_CHECK(name)                                                   \
    do {                                                                        \
        if (mr_trace_on) mr_trace_note("%s", name);                             \
        MR_LAUNCH_ERR(name);                                                    \
    } while (0)

// As MR_LAUNCH_CHECK, tracing a printf-style description of the launch.
#define MR_LAUNCH_CHECK_T(name, ...)                                            \
    do {                                                                        \
        if (mr_trace_on) mr_trace_note(__VA_ARGS__);                            \
        MR_LAUNCH_ERR(name);                                                    \
    } while (0)

// Geometry of one operator, passed by value to the kernels.
struct mr_geom {
    int n[3];        // image extents (x, y, z), unused axes 1
    int m[3];        // upsampled extents
    int cn[3];       // floor(n/2)
    int cm[3];       // floor(m/2)
    int L;
    int upper;       // 1 if the upper triangle is stored
    int64_t vimg;    // n0*n1*n2
    int64_t vpad;    // m0*m1*m2
};

void mr_geom_from_config(const mr_config *cfg, mr_geom *g);

inline int64_t mr_cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Integer environment override, or `dflt` when unset / unparsable.
int mr_env_int(const char *name, int dflt);

// Make cfg's device current (unless gpu_device_id < 0); *prev receives the
// device to restore, or -1.
int mr_push_device(const mr_config *cfg, int *prev);
void mr_pop_device(int prev);

// Free-memory budget: mem_fraction (NaN / <= 0 -> 0.5, capped at 0.95) of
// the free device memory right now.
int mr_memory_budget(const mr_config *cfg, size_t *budget);

/*
 * mr_aha.h -- C ABI of the B200 implementation of the Toeplitz-embedded
 * low-rank normal operator A^H A for non-Cartesian MRI.
 *
 * This header is the drop-in boundary: every function, struct, enum and
 * macro below has the name, C type, argument meaning and error behaviour of
 * the reference library's public header (include/mr_aha/mr_aha.h of the
 * reference project), so that its Python ctypes binding, its MATLAB MEX
 * gateways and its C callers link against libmr_aha_c.so unchanged. Each
 * declaration cites the reference declaration it replaces.
 *
 * Conventions (reference mr_aha.h:19-92):
 *   - arrays are column-major ([Nx, Ny, Nz, L] is row-major (L, Nz, Ny, Nx));
 *   - image and k-space arrays are centered: the origin is at index floor(n/2);
 *   - the L x L Gram / Toeplitz blocks are Hermitian, stored as one packed
 *     triangle, and multiply the rank ROW vector from the right, v <- v B;
 *   - single precision complex (8 bytes, {re, im}) for all array data;
 *   - every array argument is a DEVICE pointer owned by the caller;
 *   - every status-returning call returns 0 or a negative mr_status and
 *     leaves a message in mr_last_error() on failure.
 *
 * Hardware: NVIDIA B200 (sm_100a) only; one GPU per operator.
 */
#ifndef MR_AHA_MR_AHA_H
#define MR_AHA_MR_AHA_H

#include <stddef.h>
#include <stdint.h>

#define MR_EXPORT __attribute__((visibility("default")))

#ifdef __cplusplus
extern "C" {
#endif

#define MR_ALIGN8 __attribute__((aligned(8)))

/* Complex scalar: CUDA's cuFloatComplex in nvcc translation units, an
 * identical 8-byte {float x, y} elsewhere (reference mr_aha.h:163-183). */
#if defined(MR_AHA_CUDA_COMPLEX) || defined(__CUDACC__)
#include <cuComplex.h>
typedef cuFloatComplex mr_complex;
#else
typedef struct MR_ALIGN8 mr_complex_s {
    float x;
    float y;
} mr_complex;
#endif

/* Default neighbourhood radius of mr_calc_mask (reference mr_aha.h:205). */
#define MR_DEFAULT_MASK_RADIUS 2

/* Status codes (reference mr_aha.h:225-237). */
typedef enum mr_status {
    MR_SUCCESS = 0,
    MR_ERR_INVALID_ARG = -1,
    MR_ERR_INVALID_CONFIG = -2,
    MR_ERR_ALLOC = -3,
    MR_ERR_CUDA = -4,
    MR_ERR_CUFFT = -5,
    MR_ERR_CUFINUFFT = -6,
    MR_ERR_UNSUPPORTED = -7,
    MR_ERR_INTERNAL = -8,
    MR_ERR_METAL = -9,
    MR_ERR_VKFFT = -10
} mr_status;

/* Replaces reference mr_aha.h:246. Static text for a status value. */
MR_EXPORT const char *mr_status_string(int status);
/* Replaces reference mr_aha.h:265. Thread-local message of the last failure;
 * cleared at the start of every status-returning call. */
MR_EXPORT const char *mr_last_error(void);
/* Replaces reference mr_aha.h:276. Always "cuda". */
MR_EXPORT const char *mr_backend(void);

/* Trajectory family (reference mr_aha.h:291-297). */
typedef enum mr_traj_type {
    MR_TRAJ_2D = 0,
    MR_TRAJ_3D = 1,
    MR_TRAJ_STACK = 2
} mr_traj_type;

/* Stored triangle, column-major packed (reference mr_aha.h:314-317):
 * lower (i >= j) at t = j*L - j*(j-1)/2 + (i - j); upper (i <= j) at
 * t = j*(j+1)/2 + i. */
typedef enum mr_triangulation {
    MR_TRI_LOWER = 0,
    MR_TRI_UPPER = 1
} mr_triangulation;

/* Operator description; byte-identical to reference mr_aha.h:332-414. */
typedef struct mr_config {
    mr_traj_type traj_type;
    int n_spatial;        /* 2 for MR_TRAJ_2D, 3 otherwise                    */
    int n_dim[3];         /* image size [Nx, Ny, Nz], unused entries 1        */
    int phi2_dim[3];      /* upsampled grid [Mx, My, Mz], M >= N; Mz = Nz for a stack */
    int L;                /* rank                                             */
    mr_triangulation triangulation;
    int is_masked;        /* kernel stored only at num_masked grid points     */
    int64_t num_masked;
    int n_coils;
    double eps;           /* requested kernel accuracy, 0 < eps < 1           */
    int gpu_device_id;    /* CUDA ordinal, -1 = caller's current device       */
    void *stream;         /* cudaStream_t, NULL = legacy default stream       */
    double mem_fraction;  /* share of free device memory for work buffers     */
    int verbose;
    int mask_radius;
} mr_config;

/* Replaces reference mr_aha.h:433. Zero, then set the documented defaults. */
MR_EXPORT int mr_config_defaults(mr_config *cfg, mr_traj_type traj_type);
/* Replaces reference mr_aha.h:457. Host-only consistency checks. */
MR_EXPORT int mr_config_validate(const mr_config *cfg);

/* Element counts (reference mr_aha.h:474-518). */
MR_EXPORT int64_t mr_num_tri(int L);
MR_EXPORT int64_t mr_image_size(const mr_config *cfg);
MR_EXPORT int64_t mr_pad_size(const mr_config *cfg);
MR_EXPORT int64_t mr_phi2_toep_size(const mr_config *cfg);
MR_EXPORT int64_t mr_x_size(const mr_config *cfg);
MR_EXPORT int64_t mr_se_size(const mr_config *cfg);

/* Reusable stateless apply plan (reference mr_aha.h:535). */
typedef struct mr_aha_plan_s *mr_aha_plan;

/* Replaces reference mr_aha.h:578. Allocates the work buffers and FFT
 * tables for cfg on cfg->gpu_device_id; issues no work. */
MR_EXPORT int mr_aha_plan_create(const mr_config *cfg, mr_aha_plan *plan_out);

/* Replaces reference mr_aha.h:635. d_AhAx = A^H A d_x, asynchronous on
 * cfg->stream. d_phi2_toep is [Mx,My,Mz,(L^2+L)/2] (or [num_masked, ...]
 * with d_mask); d_AhAx must not alias d_x. */
MR_EXPORT int mr_aha_plan_execute(mr_aha_plan plan, const mr_complex *d_x,
                                  const mr_complex *d_SEs,
                                  const mr_complex *d_phi2_toep,
                                  const int64_t *d_mask, mr_complex *d_AhAx);

/* Replaces reference mr_aha.h:653. NULL is a no-op. */
MR_EXPORT int mr_aha_plan_destroy(mr_aha_plan plan);

/* Replaces reference mr_aha.h:670. create + execute + destroy. */
MR_EXPORT int mr_aha_toeplitz(const mr_config *cfg, const mr_complex *d_x,
                              const mr_complex *d_SEs,
                              const mr_complex *d_phi2_toep,
                              const int64_t *d_mask, mr_complex *d_AhAx);

/* Operator object (reference mr_aha.h:681-1086). */
#define MR_OP_MAX_DEVICES 16
#define MR_OP_ALL_DEVICES (-1)
#define MR_OP_SHARE_PRIMARY 1

typedef enum mr_op_method {
    MR_OP_TOEPLITZ = 0,
    MR_OP_NUFFT = 1
} mr_op_method;

typedef enum mr_toep_dist {
    MR_TOEP_DIST_AUTO = 0,
    MR_TOEP_DIST_SPLIT = 1,
    MR_TOEP_DIST_REPLICATE = 2,
    MR_TOEP_DIST_BROADCAST = 3
} mr_toep_dist;

/* Byte-identical to reference mr_aha.h:814-842. */
typedef struct mr_op_inputs {
    const mr_complex *d_SEs;
    const mr_complex *d_phi2;
    const float *d_traj;
    int64_t Ntrajs;
    int64_t Nkx;
    const int64_t *d_mask;
    const mr_complex *d_phi2_toep;
} mr_op_inputs;

/* Byte-identical to reference mr_aha.h:849-874. */
typedef struct mr_op_options {
    mr_op_method method;
    const int *devices;
    int n_devices;
    mr_toep_dist toep_dist;
    int flags;
    double nufft_upsampfac;
    int nufft_gpu_method;
} mr_op_options;

typedef struct mr_op_s *mr_op;

#define MR_OP_TOEP_SUPPLIED 0
#define MR_OP_TOEP_BROADCAST 1
#define MR_OP_TOEP_SPLIT 2
#define MR_OP_TOEP_REPLICATE 3
#define MR_OP_TOEP_NONE 4

/* Byte-identical to reference mr_aha.h:905-952. */
typedef struct mr_op_info_t {
    int method;
    int n_devices;
    int devices[MR_OP_MAX_DEVICES];
    int coil_begin[MR_OP_MAX_DEVICES];
    int coil_count[MR_OP_MAX_DEVICES];
    int group[MR_OP_MAX_DEVICES];
    int n_split_coils;
    int peer_access;
    double peer_bandwidth_gbs;
    int toep_source;
    int toep_devices;
    double toep_ms;
    double toep_component_ms;
    double toep_gather_gbs;
    double create_ms;
} mr_op_info_t;

/* Replaces reference mr_aha.h:967. */
MR_EXPORT int mr_op_options_defaults(mr_op_options *opt);
/* Replaces reference mr_aha.h:1004. Synchronous; builds (or takes) the
 * kernel and the apply plan on the primary device. One device only: a
 * request for further devices is accepted and served by the primary. */
MR_EXPORT int mr_op_create(const mr_config *cfg, const mr_op_inputs *in,
                           const mr_op_options *opt, mr_op *op_out);
/* Replaces reference mr_aha.h:1026. Asynchronous on cfg->stream. */
MR_EXPORT int mr_op_execute(mr_op op, const mr_complex *d_x, mr_complex *d_AhAx);
/* Replaces reference mr_aha.h:1038. */
MR_EXPORT int mr_op_info(mr_op op, mr_op_info_t *info);
/* Replaces reference mr_aha.h:1059. Borrowed pointer, reference layout. */
MR_EXPORT int mr_op_kernel(mr_op op, int k, const mr_complex **d_phi2_toep);
/* Replaces reference mr_aha.h:1070. */
MR_EXPORT int mr_op_destroy(mr_op op);
/* Replaces reference mr_aha.h:1086. */
MR_EXPORT int mr_op_abandon(mr_op op);

/* Replaces reference mr_aha.h:1150. Builds phi2_toep from the Gram blocks
 * [Ntrajs, (Nkz,) L, L] and trajectory [Ntrajs, Nkx, ndim]; synchronous. */
MR_EXPORT int mr_calc_toep(const mr_config *cfg, const mr_complex *d_phi2,
                           const float *d_traj, int64_t Ntrajs, int64_t Nkx,
                           const int64_t *d_mask, mr_complex *d_phi2_toep);

/* Replaces reference mr_aha.h:1199. Centered inverse FFT / prod(M) (+ mask
 * gather) of n_comp point-spread functions into components [t0, t0+n_comp). */
MR_EXPORT int mr_calc_toep_from_psf(const mr_config *cfg, const mr_complex *d_psf,
                                    int64_t t0, int64_t n_comp,
                                    const int64_t *d_mask, mr_complex *d_phi2_toep);

/* Replaces reference mr_aha.h:1254. Neighbourhood mask from the trajectory;
 * d_mask NULL only counts. */
MR_EXPORT int mr_calc_mask(const mr_config *cfg, const float *d_traj,
                           int64_t Ntrajs, int64_t Nkx, int64_t *d_mask,
                           int64_t *num_masked_out);

/* Replaces reference src/common/mr_shared_stub.cpp:23 (not in the reference
 * header): major*10000 + minor*100 + patch. */
MR_EXPORT int mr_version(void);

#ifdef __cplusplus
}
#endif

#endif /* MR_AHA_MR_AHA_H */

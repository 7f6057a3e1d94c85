/*
 * mr_aha_b200.h -- entry points of the B200 implementation that have no
 * counterpart in the reference library (its public header has no precision,
 * solver or accounting API). They extend an mr_op created through the
 * reference-compatible mr_aha.h.
 */
#ifndef MR_AHA_MR_AHA_B200_H
#define MR_AHA_MR_AHA_B200_H

#include "mr_aha/mr_aha.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Kernel storage formats of an operator. */
#define MR_B200_KF_COMPLEX64 0 /* 8 bytes per packed element (reference layout)   */
#define MR_B200_KF_BF16 1      /* bfloat16 (re, im) + one float scale per location */
#define MR_B200_KF_INT16 2     /* int16 (re, im) block floating point + one float
                                  scale per location: value = scale * code,
                                  |code| <= 32767, scale = max |re|,|im| / 32767 */

/* No reference counterpart. Store the operator's kernel in `format` for all
 * later applies (FFTs and arithmetic stay FP32). keep_complex64 = 0 frees the
 * complex64 copy (then mr_op_kernel fails with MR_ERR_UNSUPPORTED and the
 * format cannot be changed again). Synchronous. */
MR_EXPORT int mr_b200_op_set_kernel_format(mr_op op, int format, int keep_complex64);

/* No reference counterpart. Current kernel format of the operator. */
MR_EXPORT int mr_b200_op_kernel_format(mr_op op, int *format);

/* No reference counterpart. One mr_op_execute with a CUDA event recorded on
 * the operator's stream around every kernel: ms[k] is the time of launch k,
 * names + 32*k its NUL-terminated pass name (names may be NULL). Synchronous.
 * (Per-stage timing like the reference's MR_AHA_CUDA_PROFILE printout,
 * src/cuda/mr_aha.cu:520-623, returned to the caller instead.) */
MR_EXPORT int mr_b200_op_profile(mr_op op, const mr_complex *d_x, mr_complex *d_AhAx,
                                 float *ms, char *names, int max_passes, int *n_passes);

/* No reference counterpart. Number of kernels one mr_op_execute launches. */
MR_EXPORT int mr_b200_op_launches(mr_op op, int *n);

/* Size of the library's static device scratch array used by
 * mr_b200_aha_toeplitz_noalloc (reserved on every GPU that loads the
 * library, until the process exits). */
#define MR_B200_NOALLOC_SCRATCH_BYTES (32u * 1024u * 1024u)

/* No counterpart in the reference. The same result as mr_aha_toeplitz
 * (same arguments), for callers that cannot allocate device memory: its work
 * buffers and FFT tables come from the library's static scratch array
 * (MR_B200_NOALLOC_SCRATCH_BYTES per GPU) instead of cudaMalloc, and it
 * calls no allocation routine. Problems whose work space does not fit even
 * one coil at a time return MR_ERR_UNSUPPORTED. Asynchronous on cfg->stream.
 * All calls share the array: calls that overlap on the GPU race. The first
 * call on a device looks up the array's device address there; make it
 * before any stream capture. */
MR_EXPORT int mr_b200_aha_toeplitz_noalloc(const mr_config *cfg, const mr_complex *d_x,
                                           const mr_complex *d_SEs,
                                           const mr_complex *d_phi2_toep,
                                           const int64_t *d_mask, mr_complex *d_AhAx);

#ifdef __cplusplus
}
#endif

#endif /* MR_AHA_MR_AHA_B200_H */

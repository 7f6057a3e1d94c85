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
 * operator's complex64 copy, or, for a kernel borrowed from the caller
 * (MR_OP_SHARE_PRIMARY), stops referencing it so that the caller may free it;
 * then mr_op_kernel fails with MR_ERR_UNSUPPORTED and the format cannot be
 * changed again. Synchronous. */
MR_EXPORT int mr_b200_op_set_kernel_format(mr_op op, int format, int keep_complex64);

/* No reference counterpart. Current kernel format of the operator. */
MR_EXPORT int mr_b200_op_kernel_format(mr_op op, int *format);

/* Checkpoint of a 16-bit kernel (the reference saves only the complex64 one,
 * through mr_op_kernel, include/mr_aha/mr_aha.h:1040-1059). Save: copies the
 * operator's codes -- nloc x ntri (re, im) pairs of 16-bit codes, 4 bytes
 * each, layout [ntri][nloc]; nloc = num_masked for a masked operator, else
 * the grid size -- and its nloc float scales into the caller's device
 * buffers, and reports the format; MR_ERR_UNSUPPORTED when the kernel is
 * complex64. Load: copies such codes and scales into the operator, which
 * from then on applies in that 16-bit format only (its complex64 kernel and
 * blocked copy are released; mr_op_kernel then fails). Synchronous. */
MR_EXPORT int mr_b200_op_save_kernel16(mr_op op, int *format, void *d_codes, float *d_scale);
MR_EXPORT int mr_b200_op_load_kernel16(mr_op op, int format, const void *d_codes,
                                       const float *d_scale);

/* No reference counterpart. One mr_op_execute with a CUDA event recorded on
 * the operator's stream around every kernel: ms[k] is the time of launch k,
 * names + 32*k its NUL-terminated pass name (names may be NULL). Synchronous.
 * (Per-stage timing like the reference's MR_AHA_CUDA_PROFILE printout,
 * src/cuda/mr_aha.cu:520-623, returned to the caller instead.) */
MR_EXPORT int mr_b200_op_profile(mr_op op, const mr_complex *d_x, mr_complex *d_AhAx,
                                 float *ms, char *names, int max_passes, int *n_passes);

/* No reference counterpart. An operator that owns its complex64 kernel
 * also keeps, when the device has room at creation, a blocked copy of it
 * (the 32 frequencies of a warp contiguous per packed component) that the
 * half-length pass 3 reads with constant offsets; it doubles the complex64
 * kernel's footprint (a masked operator's copy covers the whole grid, zero
 * outside the mask). A 16-bit format (rank <= 16, unmasked) gets its own
 * blocked copy of the codes and scales when it is set, likewise. enable = 0 frees the copy (callers that budget device
 * memory themselves), enable = 1 builds it if the plan can use it and the
 * device has room. *built (may be NULL) tells whether a copy exists. */
MR_EXPORT int mr_b200_op_blocked_copy(mr_op op, int enable, int *built);

/* No reference counterpart. Device memory the operator holds (its owned
 * kernel copies, 16-bit kernel and scales, owned maps / mask, plan work
 * buffers); borrowed arrays are not counted. */
MR_EXPORT int mr_b200_op_device_bytes(mr_op op, uint64_t *bytes);

/* No reference counterpart. Device status of the operator's kernels since the
 * last call: 0, or MR_B200_DEV_ERR_TMA_TIMEOUT when a kernel gave up a
 * bounded wait for a TMA copy (its results are then not valid). Reads and
 * clears the status word; synchronises the operator's stream. */
#define MR_B200_DEV_ERR_TMA_TIMEOUT 1
MR_EXPORT int mr_b200_op_device_status(mr_op op, int *status);

/* mr_op_execute (reference include/mr_aha/mr_aha.h:1026) with HOST buffers:
 * h_x and h_AhAx hold mr_x_size(cfg) complex values in host memory. The call
 * is asynchronous and pipelined: it queues a copy of h_x into one of two
 * device slots (own copy stream), the apply on the operator's stream, and the
 * copy of the result to h_AhAx (second copy stream), and returns; the copies
 * of consecutive calls overlap the applies around them. Both buffers must
 * stay valid and h_x unmodified until mr_b200_op_host_sync returns. Overlap
 * needs page-locked host memory (cudaHostAlloc / cudaHostRegister); pageable
 * buffers give the same results with the copies serialised. The slots (4 x
 * the image size on the device) are allocated by the first call and freed by
 * mr_b200_op_host_release or mr_op_destroy. Not for concurrent calls on one
 * operator. */
MR_EXPORT int mr_b200_op_execute_host(mr_op op, const mr_complex *h_x, mr_complex *h_AhAx);
/* Waits for every queued host-buffer apply of the operator (their results
 * are then in the host buffers); returns the first CUDA error. */
MR_EXPORT int mr_b200_op_host_sync(mr_op op);
/* Waits, then frees the device slots of the host-buffer applies. */
MR_EXPORT int mr_b200_op_host_release(mr_op op);

/* No reference counterpart. Number of kernels one mr_op_execute launches. */
MR_EXPORT int mr_b200_op_launches(mr_op op, int *n);

/* No reference counterpart (the reference fixes its cuFFT plans and kernel
 * families at plan time). Autotune the operator: time full applies (`reps`
 * each, on a constant trial input) for every candidate kernel of each pass
 * -- strided-pass tile widths and kernel generation, pass-3 kernel (half
 * length / specialised / in-place / ping-pong) and coils per tile -- one pass
 * at a time, and keep the fastest. Later operators and plans of the same
 * geometry in this process start from the tuned choice. Every candidate
 * meets the same accuracy bar; results of different kernel generations differ
 * only by FP32 rounding. *ms (may be NULL) receives the tuned apply time.
 * Synchronous. */
MR_EXPORT int mr_b200_op_autotune(mr_op op, int reps, float *ms);

/* No reference counterpart. Launch trace of the calling host thread:
 * enable = 1 clears the trace and records, for every kernel the library
 * launches from this thread afterwards, one line naming it (the specialised
 * kernels with their template arguments, e.g.
 * "k_xbdh<N=320,L=16,NC=1,F32,256,blocked>"); enable = 0 stops recording.
 * For tests and tuning: it shows which instantiation ran each pass. */
MR_EXPORT int mr_b200_trace_launches(int enable);

/* No reference counterpart. Copies the calling thread's trace into buf
 * (NUL-terminated, truncated to cap - 1 bytes; buf may be NULL) and returns
 * its full length in bytes. */
MR_EXPORT int64_t mr_b200_trace_read(char *buf, size_t cap);

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

/* ---- Batched apply of independent operators (no reference counterpart:
 * the reference applies one operator per call). The operators may differ in
 * size, rank, coil count and trajectory type; all must live on one device and
 * appear once. Their passes run on n_streams worker streams (largest
 * operators first, each onto the least-loaded stream), so small operators
 * overlap on the GPU with large ones. */
typedef struct mr_b200_batch_s *mr_b200_batch;

#define MR_B200_BATCH_GRAPH 1 /* capture the batch as one CUDA graph; replay it
                                 (captured again when the array pointers change) */
#define MR_B200_BATCH_TUNE 2  /* mr_b200_op_autotune each distinct geometry at
                                 creation (synchronous) */

MR_EXPORT int mr_b200_batch_create(const mr_op *ops, int n_ops, int n_streams, int flags,
                                   mr_b200_batch *batch);

/* out[i] = A_i^H A_i x[i] for every operator i, ordered after earlier work on
 * `stream` (a cudaStream_t; NULL = legacy default) and before later work
 * there. Returns without waiting. Operators must not be executed elsewhere
 * while a batch execution is in flight (their work buffers are in use). */
MR_EXPORT int mr_b200_batch_execute(mr_b200_batch batch, const mr_complex *const *d_x,
                                    mr_complex *const *d_out, void *stream);

MR_EXPORT int mr_b200_batch_destroy(mr_b200_batch batch);

/* ---- Conjugate gradients on the device (no reference counterpart: the
 * reference's API stops at the operator and leaves the solver to the caller).
 * Solves (A^H A + lambda I) x = b for an operator `op`, with b and x device
 * arrays shaped like the operator's input ([Nx,Ny,Nz,L] complex64). Vectors
 * are FP32; inner products are accumulated in FP64 in a fixed order, so
 * results are deterministic; the step scalars stay in device memory, so no
 * iteration waits for the host. Work: three more vectors of x's size. */
typedef struct mr_b200_cg_s *mr_b200_cg;

#define MR_B200_CG_ZERO_X 1 /* start from x = 0 (x's contents are ignored)      */
#define MR_B200_CG_GRAPH 2  /* replay iterations from a captured CUDA graph     */

/* Set up a solve: r = b - (A^H A + lambda) x, p = r. Keeps b and x borrowed
 * (x is updated in place by every step). max_iters bounds the residual
 * history. Asynchronous on the operator's stream. */
MR_EXPORT int mr_b200_cg_create(mr_op op, const mr_complex *d_b, mr_complex *d_x, double lambda,
                                int flags, int max_iters, mr_b200_cg *cg);

/* Issue n_iter iterations (one apply and three vector kernels each) on the
 * solver's own stream, ordered after earlier work on the operator's stream and
 * before later work there. Returns without waiting for the GPU. */
MR_EXPORT int mr_b200_cg_step(mr_b200_cg cg, int n_iter);

/* *busy = 1 while iterations issued on the solver's stream are still
 * running on the GPU, else 0. Does not wait. */
MR_EXPORT int mr_b200_cg_busy(mr_b200_cg cg, int *busy);

/* Iterations issued so far (host-side count, including the ones in flight). */
MR_EXPORT int mr_b200_cg_iterations(mr_b200_cg cg, int *n);

/* Wait for the solver and copy |r_k|^2 for k = 0 .. min(iterations, max_iters)
 * (at most `max` values) to host `rr`; *n receives how many exist. */
MR_EXPORT int mr_b200_cg_residuals(mr_b200_cg cg, double *rr, int max, int *n);

/* Wait for the solver and free it (b and x stay the caller's). */
MR_EXPORT int mr_b200_cg_destroy(mr_b200_cg cg);

/* create + n_iter steps + residuals (rr: n_iter + 1 values, may be NULL) +
 * destroy. Synchronous. */
MR_EXPORT int mr_b200_cg_solve(mr_op op, const mr_complex *d_b, mr_complex *d_x, int n_iter,
                               double lambda, int flags, double *rr);

#ifdef __cplusplus
}
#endif

#endif /* MR_AHA_MR_AHA_B200_H */

// Internal interface of the apply engine (plans, passes, FFT tables) shared
// by the apply entry points, the operator object, the kernel builder and the
// precision / CG extensions.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "bd_device.cuh"
#include "fft_device.cuh"
#include "mr_internal.h"

// Factor M into supported radices; returns MR_SUCCESS or MR_ERR_UNSUPPORTED.
int mr_fft_factor(int M, mr_fft_axis *ax);
// Fill the twiddle table W_M^e (e < M) into host memory `h` (float2[M]).
void mr_fft_twiddles(int M, float2 *h);

// Pass descriptions -------------------------------------------------------

// Lines along a strided axis; a CTA transforms `xt` consecutive positions of
// the contiguous (x) dimension for one (outer, plane).
#define MR_LM_BUF 0
#define MR_LM_XS 1
#define MR_SM_BUF 0
#define MR_SM_COILSUM 1

struct mr_strided_args {
    mr_fft_axis ax;
    int nfast, xt, nxt, nouter, nplane;
    // source: BUF mode reads src; XS mode reads x (plane l) times S (coil)
    const float2 *src;
    int64_t s_plane, s_outer, s_axis;
    int n_in, shift_in;
    const float2 *xs_x;
    const float2 *xs_s;
    int64_t img_plane;   // elements of one image volume (x plane / S plane)
    int L, coil0;
    // destination: BUF mode writes dst; COILSUM writes out (plane l) summing
    // conj(S_c) * result over ncoil coils
    float2 *dst;
    int64_t d_plane, d_outer, d_axis;
    int n_out, shift_out;
    int ncoil, accumulate;
    float scale;
    int *status;         // device status word of the plan (MR_DEV_ERR_*), or NULL
    // TMA tensor maps of the pipelined z passes' tiles (encoded by the
    // launcher): map0 the image / input planes, map1 the coil maps
    CUtensorMap map0, map1;
};

// Lines along the contiguous axis (rows). Plain mode: rows r of src (stride
// s_row) to rows of dst (stride d_row). Block-diagonal mode: the CTA holds
// the L lines of nc coils at one (jy, jz) location and multiplies each
// frequency by the kernel block between the forward and inverse transform.
struct mr_x_args {
    mr_fft_axis ax;
    const float2 *src;
    float2 *dst;
    int64_t s_row, d_row;
    int64_t nrows;
    int rows_cta;
    int n_in, shift_in, n_out, shift_out;
    float scale;
    // block-diagonal mode
    int64_t plane_rows;  // rows per plane (My * Mz)
    int nloc;            // locations (My * Mz)
    int nchunk;          // coil chunks
    int nc;              // coils per CTA (last chunk may have fewer)
    int ncoil;           // coils in the group
    int L, upper;
    int My, Mz, cmx, cmy, cmz;
    mr_kernel_ref K;
    int *status;         // device status word of the plan (MR_DEV_ERR_*), or NULL
    // TMA tensor map of the source rows (pass 3 loads its tile with it),
    // encoded by the launcher
    CUtensorMap in_map;
};

int mr_launch_strided(int dir, int lmode, int smode, const mr_strided_args &a,
                      cudaStream_t s);
// In-place register-staged variants (passes2.cu) for lengths whose radices
// are all in {2, 3, 4, 5, 7, 8}: tile width 2^xts (from mr_strided2_xts, -1
// if none fits) and nc coils per block-diagonal tile (mr_xbd2_coils, 0 if
// none fits or L > 16).
int mr_launch_strided2(int dir, int lmode, int smode, const mr_strided_args &a, int xts,
                       cudaStream_t s);
int mr_launch_xbd2(const mr_x_args &a, cudaStream_t s);
int mr_strided2_xts(int M, int n_out, int smode, int nfast, size_t limit);
// Compile-time-specialised variants (passes3.cu): tile width for a length and
// store mode (`want` if instantiated, else the widest that fits; 0 if none),
// coils per tile of the instantiated block-diagonal pass for (M, L) (0 if none).
int mr_fixed_strided_xt(int M, int smode, int want = 0);
int mr_launch_strided3(int dir, int lmode, int smode, const mr_strided_args &a, cudaStream_t s);
int mr_fixed_xbd_coils(int M, int L);
int mr_launch_xbd3(const mr_x_args &a, cudaStream_t s);
// Half-length pass 3 (passes3.cu) for M = 2 n_in with the crop window equal
// to the pad window: coils per tile (0 if M != 2 n_in or not instantiated),
// and its launcher (a.nc set to that).
int mr_fixed_xbdh_coils(int M, int n_in, int L);
// Half-length strided passes (p3_yhalf.cu) for lines of M = 2N points over N
// image rows: tile width (`want` if instantiated, else the widest that fits;
// 0 if none or disabled), instantiated widths, and the launcher (dir -1:
// rows -> ramp-free spectrum; +1: spectrum -> rows). Forward and inverse are
// only valid together.
int mr_half_strided_xt(int N, int want);
int mr_half_strided_list(int N, int *xt, int max);
int mr_launch_strided_half(int dir, const mr_strided_args &a, cudaStream_t s);
// Autotuner candidates: every instantiated strided tile width of length M
// for the store mode, every instantiated coils-per-tile of pass 3 for (M, L),
// that fit shared memory; return how many were written (at most max).
int mr_fixed_strided_list(int M, int smode, int *xt, int max);
int mr_fixed_xbd_list(int M, int L, int *nc, int max);
// Time candidate kernel choices for every pass with full applies on the
// given arguments and keep the fastest (also for later plans of the same
// geometry in this process). *best_ms: the tuned apply's time.
int mr_plan_autotune(mr_aha_plan p, const float2 *x, const float2 *S, const mr_kernel_ref &K,
                     const int64_t *mask, float2 *out, int reps, float *best_ms);
int mr_launch_xbdh(const mr_x_args &a, cudaStream_t s);
int mr_xbd2_coils(int M, int L, int ncoil, size_t limit);
int mr_xbd2_stride(int M);
int mr_launch_xplain(int dir, const mr_x_args &a, cudaStream_t s);
int mr_launch_xbd(const mr_x_args &a, cudaStream_t s);

// Shared-memory bytes of a strided pass with tile width xt.
size_t mr_strided_smem(int M, int xt, int n_out, int smode);
// Largest power-of-two tile width (<= cap) that fits `limit` bytes.
int mr_pick_xt(int M, int n_out, int smode, int nfast, size_t limit);
size_t mr_xbd_smem(int M, int L, int nc);
size_t mr_xplain_smem(int M, int rows);

// Current device ordinal (0..63) and its opt-in shared memory per block.
int mr_current_device();
int mr_smem_limit();

// Plan helpers for internal callers --------------------------------------

// Optional per-pass timing of one execute: an event is recorded on the
// stream before the first and after every pass; pass names are static.
#define MR_PROF_MAX 64
struct mr_prof {
    int n;                         // events recorded
    cudaEvent_t ev[MR_PROF_MAX + 1];
    const char *name[MR_PROF_MAX]; // pass ending at event k + 1
};

int mr_plan_execute_k(mr_aha_plan plan, const float2 *x, const float2 *S,
                      const mr_kernel_ref &K, const int64_t *d_mask, float2 *out,
                      cudaStream_t s, mr_prof *prof = nullptr);
int mr_plan_kf_supported(mr_aha_plan plan);
int mr_plan_group(mr_aha_plan plan);
cudaStream_t mr_plan_stream(mr_aha_plan plan);
// Number of kernels one execute launches (for accounting).
int mr_plan_launch_count(mr_aha_plan plan);
// Reads and clears the plan's device status word (0, or an MR_DEV_ERR_* code
// a kernel recorded, e.g. a bounded wait that ran out); synchronises the
// plan's stream.
int mr_plan_device_status(mr_aha_plan plan, int *status);

// Plan over caller-provided device scratch: fills `storage` (at least
// mr_plan_struct_size() bytes, host memory) with a plan whose work buffers
// and FFT tables live in [scratch, scratch + bytes); launches the twiddle
// table kernel on cfg->stream; allocates nothing. *needed receives the
// bytes the chosen coil group uses.
size_t mr_plan_struct_size();
int mr_plan_setup_in_scratch(const mr_config *cfg, char *scratch, size_t bytes, void *storage,
                             size_t *needed);

// Device bytes a plan holds (work buffers, FFT tables).
size_t mr_plan_device_bytes(mr_aha_plan p);
// Whether the plan's pass 3 is the half-length kernel on an unmasked grid
// with Mx % 32 == 0 (it can then read a blocked kernel copy).
int mr_plan_half_pass3(mr_aha_plan p);

// Operator internals shared with the solver (op.cu).
int mr_op_execute_on(mr_op op, const float2 *x, float2 *out, cudaStream_t s);
const mr_config *mr_op_config(mr_op op);
int mr_op_device(mr_op op);
cudaStream_t mr_op_stream(mr_op op);

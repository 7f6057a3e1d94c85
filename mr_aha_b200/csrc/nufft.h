// Non-uniform FFTs of this library (nufft.cu): type 1 (samples -> centred
// modes) and type 2 (centred modes -> samples) in two or three dimensions,
// batched over planes that share the sample positions. Used by the kernel
// build when spreading is cheaper than the closed form (toep.cu) and by the
// NUFFT-method operator (op.cu). No reference counterpart in this form: the
// reference calls cufinufft (src/cuda/mr_calc_toep.cu:386-464,
// src/cuda/mr_nufft_op.cu:495-547), which is not part of this library.
#pragma once

#include "engine.h"

struct mr_nufft;

// dims: 2 or 3. modes: mode counts (x, y[, z]); mode k of an axis of M modes
// is stored at the centred index k + floor(M / 2), k in [-floor(M/2),
// ceil(M/2)). traj: device float32 coordinates (radians, periodic 2 pi),
// coordinate d of sample m at traj[d * npts + m]; the plan keeps the pointer.
// eps: requested tolerance; sigma: oversampling factor (<= 1: 2.0).
// max_planes: most planes per call. fp64: type-1 spreading accumulates in
// double precision (the FFTs stay FP32).
int mr_nufft_create(int dims, const int *modes, const float *traj, int64_t npts, double eps,
                    double sigma, int max_planes, int fp64, mr_nufft **out);
void mr_nufft_destroy(mr_nufft *p);

// Device bytes a plan with these parameters allocates.
size_t mr_nufft_plan_bytes(int dims, const int *modes, double eps, double sigma, int max_planes,
                           int fp64);

// Spreading width (grid points per axis) and oversampled grid extents the
// plan uses.
int mr_nufft_width(const mr_nufft *p);
void mr_nufft_grid(const mr_nufft *p, int *nf);

// Type 1, planes p < n: f[p][(z,) y, x] = sum_m c(p, m) exp(iflag i k . x_m),
// c(p, m) = c[p * cstride + (bcast > 0 ? m % bcast : m)], complex64 (double2
// for an fp64 plan). f: n planes of prod(modes) complex64, contiguous.
int mr_nufft_type1(mr_nufft *p, int iflag, const void *c, int64_t cstride, int64_t bcast, int n,
                   float2 *f, cudaStream_t s);

// Type 2, planes p < n: c[p * cstride + m] = sum_k f[p][k] exp(iflag i k . x_m).
int mr_nufft_type2(mr_nufft *p, int iflag, const float2 *f, int n, float2 *c, int64_t cstride,
                   cudaStream_t s);

// ---- NUFFT-method operator (MR_OP_NUFFT; reference src/cuda/mr_nufft_op.cu,
// python/mr_aha/nufft.py:473-552): per coil, x S_c (times the z modulation
// of a stack and its FFT along z), a type-2 NUFFT (sign -1, image modes) of
// every rank (and kz plane), the readout's Gram block applied to the rank
// vector of every sample (v <- v B), a type-1 NUFFT (sign +1) back, the
// inverse z FFT, and conj(S_c) accumulated over the coils. No kernel.
struct mr_nufft_op;

// Copies traj ([Ntrajs, Nkx, ndim] column-major) and phi2 into the engine;
// upsampfac <= 1 means 2.0. Synchronous.
int mr_nufft_op_create(const mr_config *cfg, const float2 *phi2, const float *traj,
                       int64_t Ntrajs, int64_t Nkx, double upsampfac, cudaStream_t s,
                       mr_nufft_op **out);
// out = A^H A x on stream s (asynchronous).
int mr_nufft_op_apply(mr_nufft_op *e, const float2 *x, const float2 *S, float2 *out,
                      cudaStream_t s);
size_t mr_nufft_op_bytes(const mr_nufft_op *e);
void mr_nufft_op_destroy(mr_nufft_op *e);
